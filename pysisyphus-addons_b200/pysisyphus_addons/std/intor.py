"""sTDDFT density-fitting tensors (reference: pysisyphus_addons/std/intor.py:8-63
and std/_intor.pyx:65-228; Fortran drivers std/intor.f90:15-292).

The functions call the reference-compatible C-ABI entry points f_intor_* of
libpa_b200.so with host arrays, as the reference's Cython module does, and
return F-ordered numpy arrays. The computation runs on the current CUDA device.
"""

import functools

import numpy as np

from pysisyphus_addons import _native as nat


@functools.singledispatch
def int_eri2c(shells, shells_aux):
    """(mu mu|nu nu) ~ T T^T with T = (mu mu|P) L^-T, shape (nbf, nbf)
    (std/intor.f90:120-139). The reference's Wavefunction overload loads the
    def2-universal-jfit auxiliary basis through pysisyphus, which is not a
    dependency here: pass both Shells objects."""
    k1, b1 = nat.basis_args(shells)
    k2, b2 = nat.basis_args(shells_aux)
    nbf = nat.nsph(shells)
    out = np.zeros((nbf, nbf), dtype=np.float64, order="F")
    nat.check(nat.load().f_intor_eri2c(*b1, *b2, nbf, nat.ptr(out)))
    return out


def int_df1c(shells, shells_aux):
    """(mu mu|P) L^-T, shape (nbf, naux) (std/intor.f90:15-118)."""
    k1, b1 = nat.basis_args(shells)
    k2, b2 = nat.basis_args(shells_aux)
    nbf, naux = nat.nsph(shells), nat.nsph(shells_aux)
    out = np.zeros((nbf, naux), dtype=np.float64, order="F")
    nat.check(nat.load().f_intor_df1c(*b1, *b2, nbf, naux, nat.ptr(out)))
    return out


def int_df2c_mo(shells, shells_aux, mo_tensor):
    """MO-pair-packed (pq|P) L^-T for the MO coefficients mo_tensor (nbf, nmos):
    row p(p+1)/2 + q (0-based, q <= p), shape (nmos(nmos+1)/2, naux)
    (std/intor.f90:141-292)."""
    C = np.asfortranarray(mo_tensor, dtype=np.float64)
    if C.ndim != 2:
        raise ValueError("mo_tensor must have shape (nbf, nmos)")
    nbf, nmos = C.shape
    k1, b1 = nat.basis_args(shells)
    k2, b2 = nat.basis_args(shells_aux)
    naux = nat.nsph(shells_aux)
    out = np.zeros((nmos * (nmos + 1) // 2, naux), dtype=np.float64, order="F")
    nat.check(nat.load().f_intor_df2c_mo(*b1, *b2, nbf, nmos, nat.ptr(C), naux, nat.ptr(out)))
    return out
