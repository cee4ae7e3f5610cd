"""Orbital g shells (lmax 4, auxiliary lmax 5): the bra classes L_ab 5-8 and
the three-center classes up to (L_ab, L_c) = (8, 5), which the 8- and 40-atom
workloads do not reach. Three atoms, seed 1: 24 orbital shells (90 functions),
51 auxiliary shells (201 functions); the metric has condition number ~3.6e9.

Schwarz values: the oracle's horizontal recurrence loses up to 7.4e-4
relative on pairs of a tight g shell with a shell on another atom (it loses
~1e-8 with d shells at 8 atoms, see test_gpu_parity.py); 40-digit values of
such pairs (tests/md_ref.py) agree with the device to 2.4e-15, so the device
is checked against those, and against the oracle on same-center pairs.

Tolerances of the contractions are about 5-10x the differences measured on a
B200: raw contraction 1.5e-12 of a maximum of 68, df (after the metric solve,
conditioning-bound) 1.4e-8, Coulomb tensor 7.9e-11 of a maximum of 70."""

import numpy as np
import pytest

import oracle
from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.synthetic import make_workload
from pysisyphus_addons.diabatization import intor as dia
from pysisyphus_addons.intor import intor as sch

pytestmark = pytest.mark.gpu


def assert_close(x, ref, atol, rel_of_max=0.0):
    tol = atol + rel_of_max * np.abs(ref).max()
    err = np.abs(x - ref).max()
    assert err <= tol, f"max abs err {err:.3e} > {tol:.3e}"


@pytest.fixture(scope="module")
def w():
    return make_workload(natoms=3, lmax=4, lauxmax=5, nstates=3, seed=1)


@pytest.fixture(params=["reference", "exact"])
def mode(request):
    nat.set_boys_mode(request.param)
    oracle.set_boys_mode(request.param)
    yield request.param
    nat.set_boys_mode("reference")
    oracle.set_boys_mode("reference")


def test_lmax4_workload_shape(w):
    assert w.shells.l_max == 4 and w.shells_aux.l_max == 5
    L = [s.L for s in w.shells]
    assert max(a + b for a in L for b in L) == 8


def test_lmax4_schwarz_high_precision(w):
    """Distant pairs with the tight g shell 7 (and the g shell 15) against
    40-digit McMurchie-Davidson values."""
    from md_ref import schwarz_pair_mp

    nat.set_boys_mode("exact")
    try:
        qg = sch.int_schwarz_bra(w.shells)
    finally:
        nat.set_boys_mode("reference")
    ia, ib = np.tril_indices(len(w.shells))
    index = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(ia, ib))}
    for a, b in ((12, 7), (20, 7), (20, 15)):
        assert w.shells[a].nprims == 1 and w.shells[b].nprims == 1
        ref = float(schwarz_pair_mp(w.shells[a], w.shells[b], dps=40))
        k = index[(a, b)]
        assert abs(qg[k] - ref) <= 1e-13 * ref, ((a, b), qg[k], ref)


def test_lmax4_schwarz_vs_oracle(w, mode):
    qg, qo = sch.int_schwarz_bra(w.shells), oracle.int_schwarz_bra(w.shells)
    ia, ib = np.tril_indices(len(w.shells))
    same = np.array([w.shells[a].center_ind == w.shells[b].center_ind for a, b in zip(ia, ib)])
    np.testing.assert_allclose(qg[same], qo[same], rtol=1e-12)
    np.testing.assert_allclose(qg, qo, rtol=1e-3, atol=1e-300)
    ag, ao = sch.int_schwarz_aux(w.shells_aux), oracle.int_schwarz_aux(w.shells_aux)
    np.testing.assert_allclose(ag, ao, rtol=1e-12)


def test_lmax4_triplet_counts(w, mode):
    oracle.set_skip_metric(1)
    try:
        oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    finally:
        oracle.set_skip_metric(0)
    st = oracle.last_stats()
    ntrip, ncomp, nints = nat.count_triplets(nat.Basis(w.shells, "orbital"), nat.Basis(w.shells_aux, "aux"))
    assert ntrip == st["ntriplets"]
    assert ntrip - ncomp == st["nskipped"]
    assert nints == st["nints"]


def test_lmax4_raw_contraction(w, mode):
    nat.set_skip_metric(1)
    oracle.set_skip_metric(1)
    try:
        df = dia.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
        ref = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    finally:
        nat.set_skip_metric(0)
        oracle.set_skip_metric(0)
    assert_close(df, ref, atol=1e-12, rel_of_max=1e-13)


def test_lmax4_df_and_coulomb_tensor(w, mode):
    df = dia.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    ref = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    assert_close(df, ref, atol=1e-7)
    R = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    Ro = oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    assert R.shape == (3, 3, 3, 3)
    assert_close(R, Ro, atol=1e-12, rel_of_max=1e-11)
