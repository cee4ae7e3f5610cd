"""QVL screening (pa_set_screening(PA_SCREEN_QVL)): the triplet estimate
qvl_estimate of common/screening.f90:267-299, the commented-out alternative at
diabatization/intor.f90:137, against the oracle's restatement of the same
estimate (screener data of t_df_screener%init, :101-163, with thresh_ws = 1d-4).

The GPU path keeps its Schwarz-sorted staircase: the auxiliary shells are
sorted by a bound of estimate / Q_ab, and every triplet is tested with the
estimate itself, so the computed triplet set must be the oracle's."""

import numpy as np
import pytest

import oracle
from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.synthetic import config_workload
from pysisyphus_addons.diabatization import intor as dia

pytestmark = pytest.mark.gpu


def assert_tensor_close(x, ref, atol, rel_of_max):
    tol = atol + rel_of_max * np.abs(ref).max()
    err = np.abs(x - ref).max()
    assert err <= tol, f"max abs err {err:.3e} > {tol:.3e}"


@pytest.fixture(autouse=True, params=["reference", "exact"])
def boys(request):
    nat.set_boys_mode(request.param)
    oracle.set_boys_mode(request.param)
    yield request.param
    nat.set_boys_mode("reference")
    nat.set_screening("schwarz")
    oracle.set_screening("schwarz")
    nat.set_skip_metric(0)
    oracle.set_skip_metric(0)


def raw_pair(w, screening):
    nat.set_screening(screening)
    oracle.set_screening(screening)
    nat.set_skip_metric(1)
    oracle.set_skip_metric(1)
    got = dia.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    ref = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    return got, ref, oracle.last_stats()


def test_default_is_the_schwarz_estimate():
    assert nat.get_screening() == "schwarz"


@pytest.mark.parametrize("key", ["cfg1", "cfg2"])
def test_qvl_raw_contraction_vs_oracle(key):
    """The screened contraction sum_(a>=b) (ab|P) Dsym with the QVL estimate;
    the QVL set differs from the Schwarz set, so the two contractions differ by
    several times the tolerance (3.2e-11 against 6.4e-12 at 8 atoms)."""
    w = config_workload(key)
    got, ref, _ = raw_pair(w, "qvl")
    assert_tensor_close(got, ref, atol=1e-12, rel_of_max=1e-13)
    schwarz, _, _ = raw_pair(w, "schwarz")
    assert np.abs(got - schwarz).max() > 2 * (1e-12 + 1e-13 * np.abs(ref).max())


@pytest.mark.parametrize("key", ["cfg1", "cfg2"])
def test_qvl_triplet_counts_match_oracle(key):
    w = config_workload(key)
    _, _, st = raw_pair(w, "qvl")
    nat.set_screening("qvl")
    orb, aux = nat.Basis(w.shells, "orbital"), nat.Basis(w.shells_aux, "aux")
    t_all, t_comp, n_ints = nat.count_triplets(orb, aux)
    assert t_all == st["ntriplets"]
    assert t_comp == st["ntriplets"] - st["nskipped"]
    assert n_ints == st["nints"]
    # QVL cuts distant triplets that the Schwarz bound keeps
    nat.set_screening("schwarz")
    _, t_comp_s, _ = nat.count_triplets(orb, aux)
    assert t_comp < t_comp_s


def test_qvl_coulomb_tensor_vs_oracle():
    """Full path (metric solve and Coulomb-tensor assembly) at 8 atoms, at the
    tolerance of the Schwarz-screened 4d test (test_gpu_parity.py)."""
    w = config_workload("cfg1")
    nat.set_screening("qvl")
    oracle.set_screening("qvl")
    R = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    Rref = oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    assert_tensor_close(R, Rref, atol=1e-12, rel_of_max=1e-13)
