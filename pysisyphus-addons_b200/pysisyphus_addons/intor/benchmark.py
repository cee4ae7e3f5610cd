"""The screening-estimator study (reference: pysisyphus_addons/intor/benchmark.py
and intor/benchmark.f90:15-132).

benchmark_int3c2e(shells, shells_aux) calls the reference-compatible entry
point f_benchmark_int3c2e: it prints the basis sizes, the time and the number
of shell triplets the QVL estimate would skip, and writes int_estimates.bin (4
doubles per record) to the working directory, as the reference does.
int3c2e_estimates returns the records as an array instead.
"""

import ctypes

import numpy as np

from pysisyphus_addons import _native as nat


def benchmark_int3c2e(shells, shells_aux):
    k1, b1 = nat.basis_args(shells)
    k2, b2 = nat.basis_args(shells_aux)
    nat.check(nat.load().f_benchmark_int3c2e(*b1, *b2))


def int3c2e_estimates(shells, shells_aux):
    """(records (n, 4), nskipped): per record schwarz_estimate, qvl_estimate,
    ||(ab|c)||_2 and the distance of the pair's contracted center to the
    auxiliary center, for every non-concentric shell pair with Schwarz value
    above 1e-10 and every auxiliary shell (intor/benchmark.f90:82-118);
    nskipped counts the records with qvl_estimate < 1e-10."""
    orb, aux = nat.Basis(shells, "orbital"), nat.Basis(shells_aux, "aux")
    lib = nat.load()
    n, sk = ctypes.c_longlong(), ctypes.c_longlong()
    nat.check(lib.pa_int3c2e_estimates(orb.handle, aux.handle, 0, None, ctypes.byref(n), ctypes.byref(sk)))
    rec = np.zeros((max(n.value, 1), 4))
    nat.check(lib.pa_int3c2e_estimates(orb.handle, aux.handle, n.value, nat.ptr(rec), ctypes.byref(n),
                                       ctypes.byref(sk)))
    return rec[: n.value], sk.value
