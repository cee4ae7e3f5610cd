"""Parity at the sizes of the measured workloads: the 40-atom tensor (lmax 3 /
lauxmax 4, 8 states), the 200-atom cluster (lmax 4 / lauxmax 5) on sampled
auxiliary shells, and molecules of the 64-molecule batch.

The metric solve at 40 atoms. (P|Q) has condition number ~7e13 there, so no
two FP64 solvers of the same raw tensor agree on the Coulomb tensor to 1e-12:
LAPACK's dpotrf + dtrsm and the reference's own dpotrf + dtrtri + dtrmm
(common/linalg.f90:60-82, diabatization/intor.f90:198) are 1.2e-8 and 3.0e-8
away from the exact solution of the same problem (measured against the
long-double solve below). The tests therefore pin the GPU's linear algebra
against an extended-precision solve of the GPU's own (P|Q) and raw
contraction:
  - backward error ||L L^T - (P|Q)||_F / ||(P|Q)||_F of the GPU factor below
    n eps (a backward-stable Cholesky);
  - forward error of df = L^-1 raw and of the tensor against the long-double
    solve no larger than twice LAPACK's on the same input, and below the
    first-order bound cond(P|Q) eps for the tensor;
  - the pipeline's df equal, bit for bit, to the standalone factor + solve of
    the same (P|Q) and raw contraction.
The inputs of that solve, (P|Q) and the raw contraction, are compared with the
oracle at 1e-13 of their largest element.

The 200-atom cluster is sampled: every surviving (ab|c) of the full orbital
basis (4950 functions, all pairs up to (gg|) screened against the sample)
with eight auxiliary shells of every angular momentum s..h on atoms spread
over the cluster, in the plain FP64 form and in the precision form.
"""

import numpy as np
import pytest
import scipy.linalg as sl

import oracle
from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.shells import Shells
from pysisyphus_addons.common.synthetic import batch_workloads, config_workload
from pysisyphus_addons.diabatization import intor as dia
from pysisyphus_addons.std import intor as std

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


def close(x, ref, rel_of_max, atol=0.0):
    tol = atol + rel_of_max * np.abs(ref).max()
    err = np.abs(x - ref).max()
    assert err <= tol, f"max abs err {err:.3e} > {tol:.3e}"
    return err


def raw_df(shells, shells_aux, dens):
    nat.set_skip_metric(1)
    try:
        return dia.contract_coulomb_densities_2d(shells, shells_aux, dens)
    finally:
        nat.set_skip_metric(0)


@pytest.fixture(autouse=True)
def reset_options():
    yield
    nat.set_skip_metric(0)
    nat.set_precision("fp64")
    nat.set_boys_mode("reference")
    nat.set_metric_shift(0.0)
    oracle.set_skip_metric(0)
    oracle.set_boys_mode("reference")
    oracle.set_metric_shift(0.0)


@pytest.fixture(scope="module")
def cfg2_gpu():
    """The 40-atom workload's GPU results in reference Boys mode."""
    nat.set_boys_mode("reference")
    w = config_workload("cfg2")
    aux = nat.Basis(w.shells_aux, "aux")
    M = nat.metric(aux)
    raw = raw_df(w.shells, w.shells_aux, w.densities)
    df = dia.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    R = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    return w, M, raw, df, R


def test_cfg2_metric_and_raw_vs_oracle(cfg2_gpu, golden_dir):
    w, M, raw, _, _ = cfg2_gpu
    oracle.set_boys_mode("reference")
    close(M, oracle.int2c2e(w.shells_aux), 1e-13, atol=1e-13)
    fx = np.load(golden_dir / "oracle_cfg2_reference.npz")
    close(raw, fx["raw"], 1e-13)


def test_cfg2_factor_backward_error(cfg2_gpu):
    w, M, raw, df, _ = cfg2_gpu
    n = M.shape[0]
    L, Y = nat.cholesky_solve(M, raw)
    # the pipeline solves with the same factor: its df is this solve, bit for bit
    np.testing.assert_array_equal(Y, df)
    be = oracle.chol_backward_error_ld(M, L)
    be_lapack = oracle.chol_backward_error_ld(M, np.linalg.cholesky(M))
    assert be <= n * EPS, (be, n * EPS)
    assert be <= 4.0 * be_lapack, (be, be_lapack)


def test_cfg2_forward_error_vs_extended_precision(cfg2_gpu):
    w, M, raw, df, R = cfg2_gpu
    ns = w.nstates
    Y_ld = oracle.chol_solve_ld(M, raw)
    R_ld = oracle.coulomb_from_df(Y_ld, ns)
    Lf = sl.cholesky(M, lower=True)
    Y_lp = sl.solve_triangular(Lf, raw, lower=True)
    R_lp = oracle.coulomb_from_df(Y_lp, ns)
    err_df, err_df_lp = np.abs(df - Y_ld).max(), np.abs(Y_lp - Y_ld).max()
    err_R, err_R_lp = np.abs(R - R_ld).max(), np.abs(R_lp - R_ld).max()
    assert err_df <= 2.0 * err_df_lp, (err_df, err_df_lp)
    assert err_R <= 2.0 * err_R_lp, (err_R, err_R_lp)
    ev = np.linalg.eigvalsh(M)
    kappa = ev[-1] / ev[0]
    assert err_R <= kappa * EPS * np.abs(R_ld).max(), (err_R, kappa)


@pytest.mark.parametrize("mode", ["reference", "exact"])
def test_cfg1_forward_error_vs_extended_precision(mode):
    nat.set_boys_mode(mode)
    w = config_workload("cfg1")
    M = nat.metric(nat.Basis(w.shells_aux, "aux"))
    raw = raw_df(w.shells, w.shells_aux, w.densities)
    R = dia.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    R_ld = oracle.coulomb_from_df(oracle.chol_solve_ld(M, raw), w.nstates)
    R_lp = oracle.coulomb_from_df(sl.solve_triangular(sl.cholesky(M, lower=True), raw, lower=True), w.nstates)
    err, err_lp = np.abs(R - R_ld).max(), np.abs(R_lp - R_ld).max()
    # condition number 3.4e6: both errors sit near the rounding floor (LAPACK's
    # ~2e-15 of the largest element, the GPU's ~1e-14), where backward-stable
    # solvers differ by small factors
    assert err <= 8.0 * err_lp + 16 * EPS * np.abs(R_ld).max(), (err, err_lp)


# ---------------------------------------------------------------------------
# 200 atoms, sampled auxiliary shells

AUX_PER_ATOM = 17  # 6 s, 4 p, 3 d, 2 f, 1 g, 1 h (auxiliary basis generator)
# (atom, shell within the atom): s(0.1), h, p(0.25), d(0.625), f(0.1), g, h, s(1.5625)
CFG5_SAMPLE = ((0, 0), (0, 16), (50, 7), (100, 12), (150, 13), (199, 15), (120, 16), (77, 3))


@pytest.fixture(scope="module")
def cfg5():
    w = config_workload("cfg5")
    sub = Shells([w.shells_aux.shells[a * AUX_PER_ATOM + k] for a, k in CFG5_SAMPLE])
    assert sorted({s.L for s in sub.shells}) == [0, 1, 2, 3, 4, 5]
    return w, sub


@pytest.fixture(scope="module")
def cfg5_oracle_raw(cfg5):
    w, sub = cfg5
    oracle.set_boys_mode("exact")
    oracle.set_skip_metric(1)
    try:
        ref = oracle.contract_coulomb_densities_2d(w.shells, sub, w.densities)
        st = oracle.last_stats()
    finally:
        oracle.set_skip_metric(0)
        oracle.set_boys_mode("reference")
    return ref, st


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cfg5_sampled_raw_contraction_vs_oracle(cfg5, cfg5_oracle_raw, precision):
    """All surviving (ab|c) of the 200-atom orbital basis with the sampled
    auxiliary shells, contracted with the 36 densities, in the plain form and
    in the precision form (FP32 recurrences for triplets with Schwarz bound
    below 1e-6): 5e-13 of the largest element. Both forms measure 1.5e-13 of
    it -- the same value, so the FP32 triplets add nothing visible; the floor
    is the oracle's horizontal recurrence, which loses digits for g shells
    paired with shells on distant atoms (tests/test_lmax4_gpu.py pins the
    device against 40-digit values there)."""
    w, sub = cfg5
    ref, st = cfg5_oracle_raw
    nat.set_boys_mode("exact")
    nat.set_precision(precision, 1e-6)
    got = raw_df(w.shells, sub, w.densities)
    close(got, ref, 5e-13)


def test_cfg5_sampled_screening_counts(cfg5, cfg5_oracle_raw):
    """Each side's triplet count is the count of its own Schwarz products at
    or above float32(1e-10). The two sets differ on 637 of 7.7e6 triplets:
    pairs with g shells on distant atoms, whose Schwarz values the oracle's
    horizontal recurrence overestimates (up to ~10x for these tiny values), so
    the oracle keeps triplets the device skips. In every flipped triplet the
    oracle's product is the larger, and for the flipped pair with the largest
    disagreement a 40-digit evaluation sides with the device."""
    from pysisyphus_addons.intor import intor as sch

    w, sub = cfg5
    _, st = cfg5_oracle_raw
    nat.set_boys_mode("exact")
    oracle.set_boys_mode("exact")
    thr = float(np.float32(1e-10))
    ntrip, ncomp, nints = nat.count_triplets(nat.Basis(w.shells, "orbital"), nat.Basis(sub, "aux"))
    pg = sch.int_schwarz_bra(w.shells)[:, None] * sch.int_schwarz_aux(sub)[None, :]
    po = oracle.int_schwarz_bra(w.shells)[:, None] * oracle.int_schwarz_aux(sub)[None, :]
    assert ntrip == st["ntriplets"] == pg.size
    assert ncomp == int((pg >= thr).sum())
    assert ntrip - st["nskipped"] == int((po >= thr).sum())
    flip = (pg >= thr) != (po >= thr)
    assert flip.sum() < 1e-3 * ncomp
    assert np.all(po[flip] > pg[flip])
    from md_ref import schwarz_pair_mp

    qg, qo = sch.int_schwarz_bra(w.shells), oracle.int_schwarz_bra(w.shells)
    rows = np.nonzero(flip.any(axis=1))[0]
    ia, ib = np.tril_indices(len(w.shells))
    single = [r for r in rows if w.shells[ia[r]].nprims == 1 and w.shells[ib[r]].nprims == 1]
    k = max(single, key=lambda r: qo[r] / qg[r])
    ref = float(schwarz_pair_mp(w.shells[ia[k]], w.shells[ib[k]], dps=40))
    assert abs(qg[k] - ref) <= 1e-10 * ref < abs(qo[k] - ref), (qg[k], qo[k], ref)


def test_cfg5_sampled_metric_solve_vs_oracle(cfg5, cfg5_oracle_raw):
    """df of the sampled auxiliary basis (49 functions, a well conditioned
    metric): the GPU metric against the oracle's, and the GPU df against the
    long-double solve of the oracle's metric and raw contraction."""
    w, sub = cfg5
    ref_raw, _ = cfg5_oracle_raw
    nat.set_boys_mode("exact")
    oracle.set_boys_mode("exact")
    M = nat.metric(nat.Basis(sub, "aux"))
    Mo = oracle.int2c2e(sub)
    close(M, Mo, 1e-13, atol=1e-14)
    df = dia.contract_coulomb_densities_2d(w.shells, sub, w.densities)
    Y_ld = oracle.chol_solve_ld(Mo, ref_raw)
    ev = np.linalg.eigvalsh(Mo)
    assert ev[-1] / ev[0] < 1e6
    close(df, Y_ld, 1e-12)


@pytest.fixture(scope="module")
def cfg5_std(cfg5):
    w, _ = cfg5
    sub = Shells([w.shells_aux.shells[a * AUX_PER_ATOM + k] for a, k in ((0, 16), (100, 12), (77, 3))])
    C = np.asfortranarray(w.mo_coeffs[:, :60])  # 20 occupied + 40 virtual orbitals
    return w, sub, C


def test_cfg5_sampled_std_df2c_mo_vs_oracle(cfg5_std):
    """sTDDFT MO-pair tensor over 20 occupied + 40 virtual orbitals (1830
    packed pairs) of the 200-atom orbital basis, sampled auxiliary shells h, d
    and s; raw (before L^-T), both value skips of std/intor.f90:247,269
    applied. The skips drop integrals and half-transformed values at or below
    1e-10; values that close to the threshold are skipped on one side and kept
    on the other when the two evaluations differ in the last digits, and each
    such flip moves an element by up to ~1e-10 times an MO coefficient. The
    bound is 2e-11 absolute (measured 5.9e-12, against 1.7e-13 for the
    well-separated contributions at 1e-12 of the largest element)."""
    w, sub, C = cfg5_std
    nat.set_boys_mode("exact")
    oracle.set_boys_mode("exact")
    nat.set_skip_metric(1)
    oracle.set_skip_metric(1)
    got = std.int_df2c_mo(w.shells, sub, C)
    ref = oracle.int_df2c_mo(w.shells, sub, C)
    assert got.shape == (1830, sub.sph_size)
    close(got, ref, 0.0, atol=2e-11)


def test_cfg5_sampled_std_df1c_vs_oracle(cfg5_std):
    w, sub, _ = cfg5_std
    nat.set_boys_mode("exact")
    oracle.set_boys_mode("exact")
    nat.set_skip_metric(1)
    oracle.set_skip_metric(1)
    close(std.int_df1c(w.shells, sub), oracle.int_df1c(w.shells, sub), 1e-13)


# ---------------------------------------------------------------------------
# molecules of the 64-molecule batch against the oracle

BATCH_CHECK = (1, 14, 10, 39)  # 5, 5, 7 and 21 atoms; 13, 4, 12 and 9 states


@pytest.fixture(scope="module")
def batch():
    import torch

    ws = batch_workloads(nmol=64)
    orbs = [nat.Basis(w.shells, "orbital") for w in ws]
    auxs = [nat.Basis(w.shells_aux, "aux") for w in ws]
    dens = [torch.from_numpy(np.ascontiguousarray(w.densities)).cuda() for w in ws]
    return ws, orbs, auxs, dens


def run_batch(batch, skip_metric):
    import torch

    ws, orbs, auxs, dens = batch
    outs = [torch.zeros(w.nstates**4, dtype=torch.float64, device="cuda") for w in ws]
    nat.set_boys_mode("exact")
    nat.set_metric_shift(1e-7)
    nat.set_skip_metric(skip_metric)
    try:
        nat.df_4d_batch(orbs, auxs, dens, [w.nstates for w in ws], outs, use_graph=True,
                        stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
    finally:
        nat.set_skip_metric(0)
    return [o.cpu().numpy().reshape((w.nstates,) * 4, order="F") for o, w in zip(outs, ws)]


def test_batch_molecules_raw_vs_oracle(batch):
    """The whole 64-molecule batch in one graph (exact Boys, metric shift
    1e-7, as measured); without the metric the tensor is a product of raw
    contractions: 1e-13 of its largest element against the oracle."""
    ws = batch[0]
    Rs = run_batch(batch, skip_metric=1)
    oracle.set_boys_mode("exact")
    oracle.set_skip_metric(1)
    for i in BATCH_CHECK:
        w = ws[i]
        ref = oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
        close(Rs[i], ref, 1e-13)


def test_batch_molecules_tensor_vs_extended_precision(batch):
    """With the shifted metric (condition number up to ~5e10): the batch's
    tensor against the long-double solve of the GPU's own shifted metric and
    raw contraction, within twice LAPACK's distance from it plus 1e-12 of the
    largest element. The metric itself is compared with the oracle's at 1e-13
    of its largest element (the raw contraction in the test above)."""
    ws, orbs, auxs, _ = batch
    Rs = run_batch(batch, skip_metric=0)
    nat.set_boys_mode("exact")
    oracle.set_boys_mode("exact")
    for i in BATCH_CHECK:
        w = ws[i]
        M0 = nat.metric(auxs[i])
        close(M0, oracle.int2c2e(w.shells_aux), 1e-13, atol=1e-14)
        raw = raw_df(w.shells, w.shells_aux, w.densities)
        M = M0 + 1e-7 * np.eye(w.shells_aux.sph_size)
        R_ld = oracle.coulomb_from_df(oracle.chol_solve_ld(M, raw), w.nstates)
        R_lp = oracle.coulomb_from_df(sl.solve_triangular(sl.cholesky(M, lower=True), raw, lower=True),
                                      w.nstates)
        err, err_lp = np.abs(Rs[i] - R_ld).max(), np.abs(R_lp - R_ld).max()
        assert err <= 2.0 * err_lp + 1e-12 * np.abs(R_ld).max(), (i, err, err_lp)
