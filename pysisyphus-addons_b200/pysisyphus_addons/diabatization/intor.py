"""Density-fitted Coulomb tensors for Edmiston-Ruedenberg diabatization
(reference: pysisyphus_addons/diabatization/intor.py:4-36 and _intor.pyx)."""

import math

import numpy as np

from pysisyphus_addons import _native as nat


def _densities(densities):
    D = np.asarray(densities, dtype=np.float64)
    if D.ndim != 3 or D.shape[1] != D.shape[2]:
        raise ValueError("densities must have shape (ndens, nbf, nbf)")
    if D.flags.c_contiguous:
        return D, nat.PA_LAYOUT_C
    if D.flags.f_contiguous:
        return D, nat.PA_LAYOUT_FORTRAN
    return np.ascontiguousarray(D), nat.PA_LAYOUT_C


def contract_coulomb_densities_2d(shells, shells_aux, densities):
    """df(naux, ndens) = L^-1 sum_(a>=b) (ab|P) [D + (a!=b) D^T], F-ordered
    (diabatization/intor.f90:28-200)."""
    D, layout = _densities(densities)
    ndens, nbf, _ = D.shape
    orb = nat.cached_basis(shells, "orbital")
    aux = nat.cached_basis(shells_aux, "aux")
    out = np.zeros((aux.nsph, ndens), dtype=np.float64, order="F")
    nat.check(nat.load().pa_contract_coulomb_densities_2d(orb.handle, aux.handle, ndens, nbf,
                                                          nat.ptr(D), layout, nat.ptr(out)))
    return out


def contract_coulomb_densities_4d(shells, shells_aux, densities):
    """Coulomb tensor R[J,K,L,M] over nstates states, ndens = nstates(nstates+1)/2
    (diabatization/intor.f90:204-270)."""
    D, layout = _densities(densities)
    ndens, nbf, _ = D.shape
    nstates = int(math.isqrt(8 * ndens + 1) / 2.0 - 0.5)
    assert nstates * (nstates + 1) // 2 == ndens
    orb = nat.cached_basis(shells, "orbital")
    aux = nat.cached_basis(shells_aux, "aux")
    out = np.zeros((nstates,) * 4, dtype=np.float64, order="F")
    nat.check(nat.load().pa_contract_coulomb_densities_4d(orb.handle, aux.handle, ndens, nbf,
                                                          nat.ptr(D), layout, nstates,
                                                          nat.ptr(out)))
    return out
