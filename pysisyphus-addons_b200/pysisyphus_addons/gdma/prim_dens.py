"""Density of diffuse primitive pairs on grid points, for GDMA (reference:
pysisyphus_addons/gdma/prim_dens.pyx:26-50; Fortran gdma/prim_dens.f90:100-259).

eval_prim_density calls the reference-compatible C-ABI entry point
f_eval_prim_density of libpa_b200.so on the current CUDA device and writes the
result into rho_pseudo, as the reference's Cython function does.
"""

import ctypes

import numpy as np

from pysisyphus_addons import _native as nat


def eval_prim_density(Ls_inds, prim_data, coords3d, P_tot_cart, switch, rho_pseudo):
    """rho_pseudo[i] = sum over primitive pairs a <= b with exponent sum below
    `switch` of (2 - delta_ab) c_a c_b exp(-mu |A-B|^2) exp(-p |r_i - P|^2)
    sum_(nu, mu) P[a_nu, b_mu] x_a^nu x_b^mu.

    Ls_inds (nprims, 2): angular momentum and 0-based Cartesian start index of
    each primitive's shell; prim_data (nprims, 5): contraction coefficient,
    exponent, x, y, z; coords3d (npoints, 3); P_tot_cart (nbfs, nbfs) Cartesian
    density matrix (symmetric); rho_pseudo (npoints,) is overwritten."""
    Li = np.asfortranarray(np.asarray(Ls_inds, dtype=np.int32).T)
    Pd = np.asfortranarray(np.asarray(prim_data, dtype=np.float64).T)
    C = np.asfortranarray(np.asarray(coords3d, dtype=np.float64).T)
    P = np.asfortranarray(P_tot_cart, dtype=np.float64)
    if Li.shape[0] != 2 or Pd.shape[0] != 5 or Li.shape[1] != Pd.shape[1]:
        raise ValueError("Ls_inds must be (nprims, 2) and prim_data (nprims, 5)")
    if C.shape[0] != 3 or P.ndim != 2 or P.shape[0] != P.shape[1]:
        raise ValueError("coords3d must be (npoints, 3) and P_tot_cart square")
    npoints = C.shape[1]
    rho = np.zeros(npoints, dtype=np.float64)
    nat.check(nat.load().f_eval_prim_density(Li.shape[1], npoints, P.shape[0], nat.ptr(Li, ctypes.c_int),
                                             nat.ptr(Pd), nat.ptr(C), nat.ptr(P), float(switch), nat.ptr(rho)))
    rho_pseudo[:] = rho
    return rho_pseudo
