"""Basis caching of the reference-facing calls: the Python front end
(pysisyphus_addons._native.cached_basis) and the f_* entry points keep the
device copy of a basis, with its shell-pair lists, for later calls with
byte-identical basis arrays. A repeated call must give the same tensor bit
for bit, a changed basis must not hit the cache, and clearing the caches must
not change results."""

import numpy as np
import pytest

from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.shells import Shell, Shells
from pysisyphus_addons.common.synthetic import config_workload
from pysisyphus_addons.diabatization import intor as dia
from test_gpu_parity import _reference_call

pytestmark = pytest.mark.gpu


def _scaled(shells, factor):
    """The same shells with every exponent scaled (a different basis)."""
    out = []
    for s in shells:
        out.append(Shell(s.L, s.center, s.coeffs, np.asarray(s.exps) * factor, s.center_ind, s.atomic_num))
    return Shells(out)


def test_repeated_calls_hit_the_cache_and_agree():
    w = config_workload("cfg1")
    nat.set_boys_mode("reference")
    nat.clear_basis_cache()
    R1 = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    orb = nat.cached_basis(w.shells, "orbital")
    assert nat.cached_basis(w.shells, "orbital") is orb
    R2 = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    np.testing.assert_array_equal(R1, R2)
    # a different orbital basis is a different entry with a different result
    other = _scaled(w.shells, 1.1)
    assert nat.cached_basis(other, "orbital") is not orb
    R3 = dia.contract_coulomb_densities_4d(other, w.shells_aux, w.densities)
    assert np.abs(R3 - R1).max() > 1e-6
    # the same arrays as an auxiliary basis are another entry (other limits)
    assert nat.cached_basis(w.shells, "aux") is not orb
    nat.clear_basis_cache()
    np.testing.assert_array_equal(dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities), R1)


def test_reference_abi_calls_with_the_cache():
    w = config_workload("cfg1")
    nat.set_boys_mode("reference")
    nat.clear_basis_cache()
    ns = w.nstates
    a = _reference_call("f_contract_coulomb_densities_4d", w.shells, w.shells_aux, w.densities, (ns,) * 4, ns)
    b = _reference_call("f_contract_coulomb_densities_4d", w.shells, w.shells_aux, w.densities, (ns,) * 4, ns)
    np.testing.assert_array_equal(a, b)
    c = _reference_call("f_contract_coulomb_densities_4d", _scaled(w.shells, 0.9), w.shells_aux, w.densities,
                        (ns,) * 4, ns)
    assert np.abs(c - a).max() > 1e-6
    nat.clear_basis_cache()
    d = _reference_call("f_contract_coulomb_densities_4d", w.shells, w.shells_aux, w.densities, (ns,) * 4, ns)
    np.testing.assert_array_equal(a, d)
    assert nat.current_device() >= 0
