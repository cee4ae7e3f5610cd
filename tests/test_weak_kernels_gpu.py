"""Weak-triplet kernels of the precision form (PA_PRECISION_MIXED with
pa_set_mixed_kernels(1)): shell triplets with Schwarz bound
Q_ab Q_c below the FP32 threshold run on their own kernels -- FP32 Boys
values, Hermite recurrence and solid harmonics, and the density product as a
split-BF16 tensor-core product (three BF16 slices per operand, six slice
products accumulated in FP32 in tensor memory over one step, FP64 across
steps) -- while the FP64 class kernels take the other triplets.

Every integral of a triplet is bounded by its Schwarz value, so FP32-level
errors (~1e-6 relative after the recurrences) on triplets below 1e-6 move the
raw contraction by ~1e-12 of its maximum at most. With the threshold at 1e30
every triplet takes the weak kernels, which exercises every class kernel
(L_ab, L_c) up to (8, 5) at FP32 accuracy."""

import numpy as np
import pytest

import oracle
from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.synthetic import batch_workloads, config_workload, make_workload
from pysisyphus_addons.diabatization import intor as dia

pytestmark = pytest.mark.gpu


def raw_df(w):
    nat.set_skip_metric(1)
    try:
        return dia.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    finally:
        nat.set_skip_metric(0)


@pytest.fixture(autouse=True)
def reset():
    nat.set_mixed_kernels(1)
    yield
    nat.set_precision("fp64")
    nat.set_mixed_kernels(0)
    nat.set_boys_mode("reference")
    nat.set_screening("schwarz")


def oracle_raw(w, mode="reference"):
    oracle.set_boys_mode(mode)
    oracle.set_skip_metric(1)
    try:
        return oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    finally:
        oracle.set_skip_metric(0)
        oracle.set_boys_mode("reference")


@pytest.mark.parametrize("mode", ["reference", "exact"])
def test_weak_kernels_default_threshold_cfg1(mode):
    w = config_workload("cfg1")
    nat.set_boys_mode(mode)
    ref = oracle_raw(w, mode)
    nat.set_precision("mixed", 1e-6)
    assert nat.get_mixed_kernels() == 1
    got = raw_df(w)
    err = np.abs(got - ref).max()
    assert err <= 1e-11 * np.abs(ref).max(), err


def test_every_triplet_on_the_weak_kernels_cfg1():
    w = config_workload("cfg1")
    ref = oracle_raw(w)
    nat.set_precision("mixed", 1e30)
    got = raw_df(w)
    err = np.abs(got - ref).max()
    # FP32 recurrences and a 24-bit split product: FP32-level error, and the
    # weak path is really taken (the FP64 path agrees to ~1e-14 of max)
    assert 1e-12 * np.abs(ref).max() < err <= 2e-6 * np.abs(ref).max(), err


def test_every_class_on_the_weak_kernels_lmax4():
    """Orbital g and auxiliary h shells: the weak kernels of every class up to
    (8, 5), per-thread (L <= 5) and team (L > 5) X builds, against the FP64
    path of the same device."""
    w = make_workload(natoms=3, lmax=4, lauxmax=5, nstates=3, seed=1)
    nat.set_boys_mode("exact")
    ref = raw_df(w)
    nat.set_precision("mixed", 1e30)
    got = raw_df(w)
    err = np.abs(got - ref).max()
    assert 1e-12 * np.abs(ref).max() < err <= 2e-6 * np.abs(ref).max(), err


def test_weak_kernels_against_fp32_recurrences_cfg2(golden_dir):
    """40 atoms at the 1e-6 threshold: the weak kernels and the FP32
    recurrences inside the FP64 kernels both stay within 1e-11 of the maximum
    of the FP64 oracle fixture, and within 2e-12 of each other."""
    w = config_workload("cfg2")
    fx = np.load(golden_dir / "oracle_cfg2_reference.npz")
    nat.set_precision("mixed", 1e-6)
    split = raw_df(w)
    nat.set_mixed_kernels(0)
    inner = raw_df(w)
    nat.set_mixed_kernels(1)
    m = np.abs(fx["raw"]).max()
    assert np.abs(split - fx["raw"]).max() <= 1e-11 * m
    assert np.abs(inner - fx["raw"]).max() <= 1e-11 * m
    assert np.abs(split - inner).max() <= 2e-12 * m


def test_weak_kernels_with_qvl_screening():
    w = config_workload("cfg1")
    nat.set_screening("qvl")
    ref = raw_df(w)
    nat.set_precision("mixed", 1e-6)
    got = raw_df(w)
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


def test_weak_kernels_batched_equal_single_molecule_path():
    """The batched weak kernels (several molecules per launch) and the
    single-molecule ones give the same tensors bit for bit."""
    import torch

    torch.cuda.set_device(0)
    ws = batch_workloads(nmol=4, lmax=2, lauxmax=2, atoms=(3, 10), states=(1, 4), seed=7)
    orbs = [nat.Basis(w.shells, "orbital") for w in ws]
    auxs = [nat.Basis(w.shells_aux, "aux") for w in ws]
    dens = [torch.from_numpy(np.ascontiguousarray(w.densities)).cuda() for w in ws]
    ns = [w.nstates for w in ws]
    nat.set_precision("mixed", 1e-6)
    outs = [torch.full((k**4,), np.nan, dtype=torch.float64, device="cuda") for k in ns]
    nat.df_4d_batch(orbs, auxs, dens, ns, outs, use_graph=True)
    for w, o, b, a, d in zip(ws, outs, orbs, auxs, dens):
        ref = torch.empty(w.nstates**4, dtype=torch.float64, device="cuda")
        nat.check(nat.load().pa_df_4d(b.handle, a.handle, d.shape[0], d.shape[1], d.data_ptr(),
                                      nat.PA_LAYOUT_C, w.nstates, ref.data_ptr(), None))
        np.testing.assert_array_equal(o.cpu().numpy(), ref.cpu().numpy())
