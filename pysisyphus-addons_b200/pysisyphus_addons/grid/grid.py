"""Densities on grid points (reference: pysisyphus_addons/grid/grid.py:1-22 and
grid/_grid.pyx:35-75; Fortran driver grid/grid.f90:110-286).

The functions call the reference-compatible C-ABI entry point f_eval_densities
of libpa_b200.so with host arrays, as the reference's Cython module does, and
return F-ordered numpy arrays. The computation runs on the current CUDA device.
"""

import numpy as np

from pysisyphus_addons import _native as nat


def eval_density(shells, grid3d, density, **kwargs):
    """One density matrix: returns the (npoints,) density on the grid."""
    assert density.ndim == 2
    return eval_densities(shells, grid3d, density[None, ...], **kwargs)[0]


def eval_densities(shells, grid3d, densities, blk_size=100, thresh=1e-8):
    """Densities on grid points, shape (ndens, npoints), F-ordered.

    grid3d: (npoints, 3) coordinates; densities: Cartesian AO density matrices
    (ndens, nbfs, nbfs) in pysisyphus order. Points are taken in consecutive
    blocks of blk_size; a basis-function pair contributes to a block when its
    density element times the block means of both functions reaches thresh
    (grid/grid.f90:236-258)."""
    keep, b = nat.basis_args(shells)
    G = np.asfortranarray(np.asarray(grid3d, dtype=np.float64).T)  # (3, npoints)
    if G.ndim != 2 or G.shape[0] != 3:
        raise ValueError("grid3d must have shape (npoints, 3)")
    D = np.asfortranarray(densities, dtype=np.float64)
    if D.ndim != 3 or D.shape[1] != D.shape[2]:
        raise ValueError("densities must have shape (ndens, nbfs, nbfs)")
    ndens, nbfs = D.shape[0], D.shape[1]
    npoints = G.shape[1]
    out = np.zeros((ndens, npoints), dtype=np.float64, order="F")
    nat.check(nat.load().f_eval_densities(*b, npoints, nat.ptr(G), ndens, nbfs, nat.ptr(D), nat.ptr(out),
                                          int(blk_size), float(thresh)))
    return out
