"""Shared inputs of the grid-density and GDMA tests: Cartesian sizes, random
symmetric Cartesian density matrices, grids, and the primitive-data packing
that pysisyphus' get_prim_data produces for prim_dens (one row per primitive
of every shell: (L, 0-based Cartesian start) and (normalized coefficient,
exponent, x, y, z))."""

import numpy as np

from pysisyphus_addons.common.shells import Shell, Shells


def ncart(L):
    return (L + 1) * (L + 2) // 2


def cart_size(shells):
    return sum(ncart(s.L) for s in shells)


def random_density(rng, n, ndens=1):
    D = rng.normal(size=(ndens, n, n))
    return D + D.transpose(0, 2, 1)


def box_grid(shells, n=2000, margin=3.0, seed=1):
    C = np.array([s.center for s in shells])
    lo, hi = C.min(0) - margin, C.max(0) + margin
    return np.random.default_rng(seed).uniform(lo, hi, size=(n, 3))


def normalized_coeffs(sh):
    """Contraction coefficients renormalized as common/normalization.f90:10-38."""
    c, e, L = np.asarray(sh.coeffs, float), np.asarray(sh.exps, float), sh.L
    lp = L + 1.5
    N = sum(c[i] * c[j] / (e[i] + e[j]) ** lp * np.sqrt(e[i] * e[j]) ** lp
            for i in range(len(e)) for j in range(len(e)))
    return c * np.sqrt(e**lp / (np.pi**1.5 / 2**L * N))


def prim_data(shells):
    Ls_inds, data = [], []
    off = 0
    for s in shells:
        for c, e in zip(normalized_coeffs(s), s.exps):
            Ls_inds.append((s.L, off))
            data.append((c, e, *s.center))
        off += ncart(s.L)
    return np.array(Ls_inds, dtype=np.int32), np.array(data, dtype=np.float64)


def one_atom_basis(lmax=4):
    """Shells s..g on one center, one with three primitives."""
    shells = [Shell(0, [0.1, -0.2, 0.3], [0.3, 0.5, 0.4], [5.0, 1.2, 0.3])]
    for L in range(1, lmax + 1):
        shells.append(Shell(L, [0.1, -0.2, 0.3], [1.0], [0.8 + 0.1 * L]))
    return Shells(shells)
