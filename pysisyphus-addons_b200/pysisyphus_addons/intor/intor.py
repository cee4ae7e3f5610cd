"""Schwarz vectors (reference: pysisyphus_addons/intor/intor.py:4-11)."""

import numpy as np

from pysisyphus_addons import _native as nat


def int_schwarz_aux(shells):
    """sqrt(||(c|c)||_F) for every shell c (common/integrals/intor.f90:97-129)."""
    lib = nat.load()
    keep, args = nat.basis_args(shells)
    out = np.zeros(args[0], dtype=np.float64)
    nat.check(lib.f_int_schwarz_aux(*args, nat.ptr(out)))
    return out


def int_schwarz_bra(shells):
    """sqrt(||(ab|ab)||_F) for shell pairs a >= b, packed a(a+1)/2 + b
    (common/integrals/intor.f90:131-160)."""
    lib = nat.load()
    keep, args = nat.basis_args(shells)
    n = args[0]
    out = np.zeros(n * (n + 1) // 2, dtype=np.float64)
    nat.check(lib.f_int_schwarz_bra(*args, nat.ptr(out)))
    return out
