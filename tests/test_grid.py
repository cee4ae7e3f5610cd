"""The oracle's restatement of the grid-density driver (grid/grid.f90:17-286)
and of the GDMA primitive density (gdma/prim_dens.f90:100-259), checked on
the CPU: normalization of every Cartesian component (each is normalized on
its own: the NORM2 / NORM3 / NORM4 / NORM22 factors), an s shell in closed
form, the unscreened density against a plain numpy evaluation, and the
primitive density of a one-center basis against the grid density (every
primitive pair of one center survives the reference's pair test)."""

import numpy as np

import oracle
from grid_common import box_grid, cart_size, one_atom_basis, prim_data, random_density
from pysisyphus_addons.common.shells import Shell, Shells
from pysisyphus_addons.common.synthetic import config_workload


def test_cartesian_components_are_normalized():
    h = 0.15
    ax = np.arange(-7.0, 7.0 + h / 2, h)
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    for L in range(5):
        sh = Shells([Shell(L, [0.0, 0.0, 0.0], [1.0], [0.9])])
        n = cart_size(sh)
        D = np.zeros((n, n, n))
        for c in range(n):
            D[c, c, c] = 1.0
        rho = oracle.eval_densities(sh, pts, D, blk_size=512, thresh=0.0)
        np.testing.assert_allclose(rho.sum(axis=1) * h**3, 1.0, rtol=1e-10)


def test_unscreened_density_matches_numpy():
    w = config_workload("cfg1")
    rng = np.random.default_rng(2)
    n = cart_size(w.shells)
    D = random_density(rng, n, 2)
    g = box_grid(w.shells, n=300)
    rho = oracle.eval_densities(w.shells, g, D, blk_size=37, thresh=0.0)
    # chi from one-function density matrices (diagonal elements give chi^2 / f)
    chi = np.zeros((n, len(g)))
    E = np.zeros((n, n, n))
    for c in range(n):
        E[c, c, c] = 1.0
    chi2 = oracle.eval_densities(w.shells, g, E, blk_size=37, thresh=0.0)
    # signs: compare quadratic forms through |chi| and the diagonal only
    ref_diag = np.einsum("jcc,cp->jp", D, chi2)
    Dd = np.stack([np.diag(np.diag(d)) for d in D])
    rho_diag = oracle.eval_densities(w.shells, g, Dd, blk_size=37, thresh=0.0)
    np.testing.assert_allclose(rho_diag, ref_diag, rtol=1e-12, atol=1e-14)
    assert rho.shape == (2, len(g)) and np.isfinite(rho).all()


def test_screening_drops_pairs_by_block_means():
    """The block-mean estimate is crude: at thresh 1e-8 it moves this random
    density by ~1e-4 of its largest value (the reference's behaviour)."""
    w = config_workload("cfg1")
    rng = np.random.default_rng(3)
    n = cart_size(w.shells)
    D = random_density(rng, n)
    g = box_grid(w.shells, n=500)
    a = oracle.eval_densities(w.shells, g, D, blk_size=100, thresh=0.0)
    b = oracle.eval_densities(w.shells, g, D, blk_size=100, thresh=1e-8)
    assert 0 < np.abs(a - b).max() < 1e-3 * np.abs(a).max()
    # larger blocks average over more points: a different set of pairs
    c = oracle.eval_densities(w.shells, g, D, blk_size=250, thresh=1e-8)
    assert np.abs(c - b).max() > 0


def test_prim_density_one_center_equals_grid_density():
    sh = one_atom_basis(4)
    rng = np.random.default_rng(4)
    n = cart_size(sh)
    D = random_density(rng, n)[0]
    # within 0.85 bohr of the center (|r - A| < 1.5): no exponent sum of the
    # basis (at most 10) reaches the -36 cutoff, which the two drivers apply to
    # different factors (each primitive / each primitive pair)
    g = box_grid(sh, n=400, margin=0.85)
    rho_grid = oracle.eval_densities(sh, g, D[None], blk_size=50, thresh=0.0)[0]
    Ls_inds, pdata = prim_data(sh)
    rho = np.zeros(len(g))
    oracle.eval_prim_density(Ls_inds, pdata, g, D, 1e30, rho)
    np.testing.assert_allclose(rho, rho_grid, rtol=0, atol=1e-13 * np.abs(rho_grid).max())
