"""Every tile-shape variant of the three-center class kernels against the
oracle: the raw contraction (no metric solve) of the 8-atom workload, the
lmax 4 / lauxmax 5 three-atom workload (classes up to (8, 5)) and the
40-atom workload, with every class set to the variant. Variants change only
tile sizes, team sizes and occupancy, hence the summation order of the
product: the tolerance is the one of the default shapes' tests."""

import numpy as np
import pytest

import oracle
from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.synthetic import config_workload, make_workload
from pysisyphus_addons.diabatization import intor as dia

pytestmark = pytest.mark.gpu


def set_all(v):
    for lab in range(2 * nat.LMAX + 1):
        for lc in range(nat.LAUXMAX + 1):
            nat.set_tile_variant(lab, lc, v)


@pytest.fixture(autouse=True)
def restore():
    saved = {(a, b): nat.get_tile_variant(a, b) for a in range(2 * nat.LMAX + 1) for b in range(nat.LAUXMAX + 1)}
    yield
    for (a, b), v in saved.items():
        nat.set_tile_variant(a, b, v)
    nat.set_skip_metric(0)
    oracle.set_skip_metric(0)


def raw(shells, shells_aux, dens, impl, options):
    options.set_skip_metric(1)
    try:
        return impl.contract_coulomb_densities_2d(shells, shells_aux, dens)
    finally:
        options.set_skip_metric(0)


@pytest.fixture(scope="module")
def cases():
    out = {}
    for key, w in [("cfg1", config_workload("cfg1")),
                   ("lmax4", make_workload(natoms=3, lmax=4, lauxmax=5, nstates=3, seed=1)),
                   ("cfg2", config_workload("cfg2"))]:
        out[key] = (w, raw(w.shells, w.shells_aux, w.densities, oracle, oracle))
    return out


@pytest.mark.parametrize("variant", range(nat.TILE_VARIANTS))
@pytest.mark.parametrize("key,rel", [("cfg1", 2e-14), ("lmax4", 1e-13), ("cfg2", 1e-13)])
def test_variant_raw_contraction_vs_oracle(cases, variant, key, rel):
    w, ref = cases[key]
    set_all(variant)
    got = raw(w.shells, w.shells_aux, w.densities, dia, nat)
    err = np.abs(got - ref).max()
    assert err <= 1e-12 + rel * np.abs(ref).max(), f"variant {variant}: max abs err {err:.3e}"
