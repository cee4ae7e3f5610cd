"""Grid densities (f_eval_densities) and the GDMA primitive density
(f_eval_prim_density) on the GPU, through the reference-compatible C-ABI,
against the oracle's restatements of grid/grid.f90:110-286 and
gdma/prim_dens.f90:100-259 on the same inputs.

Tolerance: 1e-13 of the largest value. The screening decisions use the same
block means (summed over the block's points in the reference's order) and the
same product order, so they agree unless a pair sits within rounding of the
threshold; the sums over pairs run in a different order. Block sizes 1, 37,
100 (the reference's default) and 300 (more points than threads per block)
and thresholds 0 and 1e-8 are covered; ragged last blocks throughout."""

import numpy as np
import pytest

import oracle
from grid_common import box_grid, cart_size, one_atom_basis, prim_data, random_density
from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.shells import Shell, Shells
from pysisyphus_addons.common.synthetic import config_workload, make_workload
from pysisyphus_addons.gdma import prim_dens
from pysisyphus_addons.grid import grid

pytestmark = pytest.mark.gpu


def close(x, ref, rel_of_max):
    tol = rel_of_max * np.abs(ref).max()
    err = np.abs(x - ref).max()
    assert err <= tol, f"max abs err {err:.3e} > {tol:.3e}"


@pytest.mark.parametrize("blk,thresh", [(100, 1e-8), (37, 1e-8), (1, 1e-8), (300, 1e-8), (100, 0.0)])
def test_grid_densities_vs_oracle(blk, thresh):
    w = config_workload("cfg1")
    rng = np.random.default_rng(blk)
    n = cart_size(w.shells)
    D = random_density(rng, n, 2)
    g = box_grid(w.shells, n=3001, seed=blk)
    got = grid.eval_densities(w.shells, g, D, blk_size=blk, thresh=thresh)
    ref = oracle.eval_densities(w.shells, g, D, blk_size=blk, thresh=thresh)
    assert got.shape == (2, len(g)) and got.flags.f_contiguous
    close(got, ref, 1e-13)


def test_grid_density_g_shells_and_single_density():
    w = make_workload(4, lmax=4, lauxmax=0, nstates=1, seed=3)
    rng = np.random.default_rng(9)
    D = random_density(rng, cart_size(w.shells))[0]
    g = box_grid(w.shells, n=1500)
    got = grid.eval_density(w.shells, g, D)
    ref = oracle.eval_densities(w.shells, g, D[None])[0]
    assert got.shape == (len(g),)
    close(got, ref, 1e-13)


def test_grid_components_normalized_on_device():
    h = 0.15
    ax = np.arange(-7.0, 7.0 + h / 2, h)
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    sh = Shells([Shell(4, [0.0, 0.0, 0.0], [1.0], [0.9])])
    n = cart_size(sh)
    D = np.zeros((n, n, n))
    for c in range(n):
        D[c, c, c] = 1.0
    rho = grid.eval_densities(sh, pts, D, thresh=0.0)
    np.testing.assert_allclose(rho.sum(axis=1) * h**3, 1.0, rtol=1e-10)


def test_grid_errors_and_empty_inputs():
    w = config_workload("cfg1")
    n = cart_size(w.shells)
    g = box_grid(w.shells, n=10)
    with pytest.raises(nat.PaError) as e:
        grid.eval_densities(w.shells, g, np.zeros((1, n - 1, n - 1)))
    assert e.value.code == nat.PA_ERR_ARG
    with pytest.raises(nat.PaError) as e:
        grid.eval_densities(Shells([Shell(5, [0, 0, 0], [1.0], [1.0])]), g, np.zeros((1, 21, 21)))
    assert e.value.code == nat.PA_ERR_LMAX
    assert grid.eval_densities(w.shells, np.zeros((0, 3)), np.zeros((1, n, n))).shape == (1, 0)


@pytest.mark.parametrize("key,switch", [("cfg1", 1e30), ("cfg1", 2.0), ("lmax4", 3.0)])
def test_prim_density_vs_oracle(key, switch):
    if key == "cfg1":
        shells = config_workload("cfg1").shells
    else:
        shells = make_workload(4, lmax=4, lauxmax=0, nstates=1, seed=3).shells
    Ls_inds, pdata = prim_data(shells)
    rng = np.random.default_rng(5)
    P = random_density(rng, cart_size(shells))[0]
    g = box_grid(shells, n=2049)
    got = np.full(len(g), np.nan)
    prim_dens.eval_prim_density(Ls_inds, pdata, g, P, switch, got)
    ref = np.zeros(len(g))
    oracle.eval_prim_density(Ls_inds, pdata, g, P, switch, ref)
    close(got, ref, 1e-13)


def test_prim_density_one_center_equals_grid_density():
    sh = one_atom_basis(4)
    rng = np.random.default_rng(4)
    D = random_density(rng, cart_size(sh))[0]
    g = box_grid(sh, n=400, margin=0.85)
    rho = np.zeros(len(g))
    Ls_inds, pdata = prim_data(sh)
    prim_dens.eval_prim_density(Ls_inds, pdata, g, D, 1e30, rho)
    close(rho, grid.eval_density(sh, g, D, thresh=0.0), 1e-13)


def test_prim_density_no_pairs_and_errors():
    shells = config_workload("cfg1").shells
    Ls_inds, pdata = prim_data(shells)
    P = np.eye(cart_size(shells))
    g = box_grid(shells, n=50)
    rho = np.full(len(g), 7.0)
    prim_dens.eval_prim_density(Ls_inds, pdata, g, P, 0.0, rho)  # no pair below the switch
    assert (rho == 0.0).all()
    bad = Ls_inds.copy()
    bad[0, 0] = 5
    with pytest.raises(nat.PaError) as e:
        prim_dens.eval_prim_density(bad, pdata, g, P, 1e30, rho)
    assert e.value.code == nat.PA_ERR_LMAX
    bad = Ls_inds.copy()
    bad[-1, 1] = P.shape[0]
    with pytest.raises(nat.PaError) as e:
        prim_dens.eval_prim_density(bad, pdata, g, P, 1e30, rho)
    assert e.value.code == nat.PA_ERR_ARG
