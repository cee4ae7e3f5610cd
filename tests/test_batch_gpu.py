"""Batched form (pa_df_4d_batch): many molecules per call, one persistent
launch per shell-triplet class over all of them, recorded as a CUDA graph and
replayed. Each molecule's tensor must equal the single-molecule path's exactly:
the same work items, partial sums and ordered reductions run in both."""

import numpy as np
import pytest

from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.synthetic import batch_workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch():
    import torch

    torch.cuda.set_device(0)
    ws = batch_workloads(nmol=6, lmax=2, lauxmax=2, atoms=(3, 10), states=(1, 4), seed=7)
    orbs = [nat.Basis(w.shells, "orbital") for w in ws]
    auxs = [nat.Basis(w.shells_aux, "aux") for w in ws]
    dens = [torch.from_numpy(np.ascontiguousarray(w.densities)).cuda() for w in ws]
    return ws, orbs, auxs, dens


def single(torch, orb, aux, d, ns):
    out = torch.empty(ns**4, dtype=torch.float64, device="cuda")
    nat.check(nat.load().pa_df_4d(orb.handle, aux.handle, d.shape[0], d.shape[1], d.data_ptr(),
                                  nat.PA_LAYOUT_C, ns, out.data_ptr(), None))
    return out.cpu().numpy()


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_single_molecule_path(small_batch, use_graph):
    import torch

    ws, orbs, auxs, dens = small_batch
    ns = [w.nstates for w in ws]
    outs = [torch.full((k**4,), np.nan, dtype=torch.float64, device="cuda") for k in ns]
    nat.df_4d_batch(orbs, auxs, dens, ns, outs, use_graph=use_graph)
    for w, o, b, a, d in zip(ws, outs, orbs, auxs, dens):
        np.testing.assert_array_equal(o.cpu().numpy(), single(torch, b, a, d, w.nstates))
    if use_graph:
        # a replay of the recorded graph sees new density values at the same addresses
        first = [o.cpu().numpy().copy() for o in outs]
        for o in outs:
            o.fill_(np.nan)
        dens[0].mul_(2.0)
        nat.df_4d_batch(orbs, auxs, dens, ns, outs, use_graph=True)
        dens[0].mul_(0.5)
        np.testing.assert_allclose(outs[0].cpu().numpy(), 4.0 * first[0], rtol=1e-14, atol=1e-14)
        for o, f in zip(outs[1:], first[1:]):
            np.testing.assert_array_equal(o.cpu().numpy(), f)


def test_batch_matches_single_molecule_path_lmax4():
    """Orbital g and auxiliary h shells (lmax 4 / 5): the batched class kernels
    up to (L_ab, L_c) = (8, 5) equal the single-molecule path bit for bit. The
    three metrics are positive definite (smallest eigenvalues 2.5e-3, 9.3e-5
    and 1.8e-8)."""
    import torch

    torch.cuda.set_device(0)
    ws = batch_workloads(nmol=3, lmax=4, lauxmax=5, atoms=(2, 4), states=(1, 3), seed=11)
    assert all(w.shells.l_max == 4 and w.shells_aux.l_max == 5 for w in ws)
    orbs = [nat.Basis(w.shells, "orbital") for w in ws]
    auxs = [nat.Basis(w.shells_aux, "aux") for w in ws]
    dens = [torch.from_numpy(np.ascontiguousarray(w.densities)).cuda() for w in ws]
    ns = [w.nstates for w in ws]
    outs = [torch.full((k**4,), np.nan, dtype=torch.float64, device="cuda") for k in ns]
    nat.df_4d_batch(orbs, auxs, dens, ns, outs, use_graph=True)
    for w, o, b, a, d in zip(ws, outs, orbs, auxs, dens):
        np.testing.assert_array_equal(o.cpu().numpy(), single(torch, b, a, d, w.nstates))


def test_batch_graph_follows_the_screening_mode(small_batch):
    """The recorded graph is keyed on the options: after a switch to QVL
    screening the next batch call records anew and equals the single-molecule
    QVL path. QVL changes the triplet set of every molecule of this batch, so a
    stale replay of the Schwarz graph would be caught."""
    import torch

    ws, orbs, auxs, dens = small_batch
    ns = [w.nstates for w in ws]
    outs = [torch.full((k**4,), np.nan, dtype=torch.float64, device="cuda") for k in ns]
    nat.df_4d_batch(orbs, auxs, dens, ns, outs, use_graph=True)
    schwarz = [o.cpu().numpy().copy() for o in outs]
    nat.set_screening("qvl")
    try:
        nat.df_4d_batch(orbs, auxs, dens, ns, outs, use_graph=True)
        for w, o, b, a, d, s0 in zip(ws, outs, orbs, auxs, dens, schwarz):
            ref = single(torch, b, a, d, w.nstates)
            np.testing.assert_array_equal(o.cpu().numpy(), ref)
            assert not np.array_equal(ref, s0)
    finally:
        nat.set_screening("schwarz")


def test_batch_errors(small_batch):
    import torch

    ws, orbs, auxs, dens = small_batch
    outs = [torch.empty(w.nstates**4, dtype=torch.float64, device="cuda") for w in ws]
    with pytest.raises(nat.PaError):
        nat.df_4d_batch(orbs, auxs, dens, [w.nstates + 1 for w in ws], outs)
    nat.df_4d_batch([], [], [], [], [])  # an empty batch is a no-op
