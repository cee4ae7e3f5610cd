"""The oracle (CPU restatement of the reference) against the reference's own
golden vectors and known answers. No GPU needed."""

import json

import mpmath
import numpy as np
import pytest

import oracle
from pysisyphus_addons.common.shells import Shell, Shells


def load_bena2(golden_dir):
    basis = json.loads((golden_dir / "bena2_basis.json").read_text())
    shells = Shells([Shell(b["L"], b["center"], b["coeffs"], b["exps"], b["center_ind"], b["atomic_num"])
                     for b in basis])
    D = np.load(golden_dir / "bena2_densities.npy")
    ref = json.loads((golden_dir / "bena2_coulomb_ref.json").read_text())
    return shells, D, ref


@pytest.mark.parametrize("mode", ["reference", "exact"])
def test_golden_coulomb_tensor(golden_dir, mode):
    """tests/test_coulomb_tensor/test_coulomb_tensor.py:7-32 (aux = orbital basis)."""
    shells, D, ref = load_bena2(golden_dir)
    oracle.set_boys_mode(mode)
    R = oracle.contract_coulomb_densities_4d(shells, shells, D)
    assert R.shape == (2, 2, 2, 2)
    np.testing.assert_allclose(R, np.array(ref["tensor"]), atol=ref["atol"], rtol=ref["rtol"])
    # the diagonal agrees far tighter than the reference's rtol (about 7e-14 relative)
    np.testing.assert_allclose(R, np.array(ref["tensor"]), atol=1e-12, rtol=2e-13)


def test_overlap_pins_basis_convention(golden_dir):
    """Normalization, shell ordering and m = -l..l phases reproduce ORCA's S."""
    from md_ref import overlap_matrix

    shells, D, _ = load_bena2(golden_dir)
    S_orca = np.load(golden_dir / "bena2_overlap.npy")
    S = overlap_matrix(shells)
    np.testing.assert_allclose(S, S_orca, atol=1e-9)
    # 24 electrons in the state densities
    assert abs(np.trace(D[0] @ S) - 24.0) < 1e-8
    assert abs(np.trace(D[2] @ S) - 24.0) < 1e-8


def test_erfinv_known_answers():
    """tests_fortran/test_erfinv.f90:25-29."""
    assert oracle.erfinv(0.0) == 0.0
    assert oracle.erfinv(0.9) == 1.1630871536766727
    assert oracle.erfinv(-0.9) == -1.1630871536766727
    assert abs(oracle.erfinv(0.5) - 0.4769362762044698) < 1e-15
    assert abs(oracle.erfinv(-0.5) + 0.4769362762044698) < 1e-15


def test_contracted_center_known_answers():
    """tests_fortran/test_screening.f90:28-64."""
    A, B = np.zeros(3), np.ones(3)
    R = oracle.contracted_center([1.0], [1.0], A, [1.0], [1.0], A)
    assert np.linalg.norm(R - A) <= 1e-14
    axs = [1.0, 0.5]
    R = oracle.contracted_center(axs, axs, A, axs, axs, B)
    assert np.linalg.norm(R - (A + B) / 2) <= 1e-14
    R = oracle.contracted_center([1.0, 0.5, 0.25], [1.0, 0.5, 0.25], A, [1.0, 0.5], [1.0, 0.5], B)
    assert np.linalg.norm(R - 0.53650793650794) <= 1e-13


def _boys_mp(n, x):
    mpmath.mp.dps = 40
    if x == 0:
        return 1.0 / (2 * n + 1)
    return float(mpmath.quad(lambda t: t ** (2 * n) * mpmath.exp(-x * t * t), [0, 1]))


@pytest.mark.parametrize("x", [0.0, 1e-9, 0.37, 5.0, 12.345, 26.99, 27.0, 33.3, 45.0, 120.0])
def test_boys_exact_vs_mpmath(x):
    oracle.set_boys_mode("exact")
    F = oracle.boys(16, x)
    for n in range(17):
        ref = _boys_mp(n, x)
        assert abs(F[n] - ref) <= 2e-15 * abs(ref), (n, x, F[n], ref)


@pytest.mark.parametrize("x", [0.0, 0.37, 5.0, 12.345, 26.99])
def test_boys_reference_mode_interpolation(x):
    """5-point interpolation on the 0.01 grid: ~1e-12 relative (boys.f90:53-85)."""
    oracle.set_boys_mode("reference")
    F = oracle.boys(14, x)
    for n in range(15):
        ref = _boys_mp(n, x)
        assert abs(F[n] - ref) <= 5e-12 * abs(ref), (n, x)


def test_boys_reference_mode_asymptotic():
    """x >= 27 uses (2n-1)!!/2^(n+1) sqrt(pi/x^(2n+1)) (boys.f90:44-49,92)."""
    oracle.set_boys_mode("reference")
    x = 30.0
    F = oracle.boys(8, x)
    for n in range(9):
        df = np.prod(np.arange(2 * n - 1, 0, -2)) if n > 0 else 1.0
        assert F[n] == pytest.approx(df / 2 ** (n + 1) * np.sqrt(np.pi / x ** (2 * n + 1)), rel=1e-14)


def test_schwarz_is_frobenius_of_block(golden_dir):
    """int_schwarz_bra / int_schwarz_aux follow test_schwarz_integrals.py:17-54:
    sqrt of the Frobenius norm of the (ab|ab) / (c|c) blocks."""
    shells, _, _ = load_bena2(golden_dir)
    oracle.set_boys_mode("exact")
    bra = oracle.int_schwarz_bra(shells)
    aux = oracle.int_schwarz_aux(shells)
    for a in (0, 5, 7):
        for b in range(a + 1):
            blk = oracle.eri_block(shells[a], shells[b], shells[a], shells[b])
            assert bra[a * (a + 1) // 2 + b] == pytest.approx(np.sqrt(np.linalg.norm(blk)), rel=1e-14)
        blk = oracle.eri_block(shells[a], None, shells[a], None)
        assert aux[a] == pytest.approx(np.sqrt(np.linalg.norm(blk)), rel=1e-14)


def test_oracle_matches_committed_fixture_cfg1(golden_dir):
    from pysisyphus_addons.common.synthetic import config_workload

    w = config_workload("cfg1")
    for mode in ("reference", "exact"):
        oracle.set_boys_mode(mode)
        R = oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
        fx = np.load(golden_dir / f"oracle_cfg1_{mode}.npz")
        np.testing.assert_allclose(R, fx["R"], atol=1e-13, rtol=0)


def test_eri_symmetries():
    """Permutational symmetry and translation invariance of contracted blocks."""
    rng = np.random.default_rng(3)
    sh = [Shell(L, rng.uniform(-1, 1, 3), rng.uniform(0.3, 1, 2), rng.uniform(0.2, 3, 2)) for L in (2, 1, 3)]
    oracle.set_boys_mode("exact")
    abc = oracle.eri_block(sh[0], sh[1], sh[2], None)[..., 0]
    bac = oracle.eri_block(sh[1], sh[0], sh[2], None)[..., 0]
    np.testing.assert_allclose(abc, bac.transpose(1, 0, 2), atol=1e-14)
    shift = np.array([0.3, -1.2, 2.0])
    moved = [Shell(s.L, s.center + shift, s.coeffs, s.exps) for s in sh]
    abc2 = oracle.eri_block(moved[0], moved[1], moved[2], None)[..., 0]
    np.testing.assert_allclose(abc, abc2, atol=1e-13)
    pq = oracle.eri_block(sh[2], None, sh[0], None)[:, 0, :, 0]
    qp = oracle.eri_block(sh[0], None, sh[2], None)[:, 0, :, 0]
    np.testing.assert_allclose(pq, qp.T, atol=1e-14)


def _qvl_count_numpy(shells, shells_aux, qb, qa, thresh):
    """Independent numpy restatement of t_df_screener%init
    (common/screening.f90:101-163) and qvl_estimate (:267-299): the number of
    triplets a >= b, c whose estimate reaches the threshold."""
    erfi = oracle.erfinv(1.0 - 1e-4)

    def norm_coeffs(s):
        e, c, lp = np.asarray(s.exps, float), np.asarray(s.coeffs, float), s.L + 1.5
        N = (c[:, None] * c[None, :] * (e[:, None] * e[None, :]) ** (lp / 2) / (e[:, None] + e[None, :]) ** lp).sum()
        return c * np.sqrt(e**lp / (np.pi**1.5 / 2**s.L * N))

    orb = list(shells)
    coefs = [norm_coeffs(s) for s in orb]
    cen = np.array([s.center for s in orb], float)
    count = 0
    for a in range(len(orb)):
        for b in range(a + 1):
            ea, eb = np.asarray(orb[a].exps, float), np.asarray(orb[b].exps, float)
            px = ea[:, None] + eb[None, :]
            P = (ea[:, None, None] * cen[a] + eb[None, :, None] * cen[b]) / px[:, :, None]
            w = np.abs(coefs[a][:, None] * coefs[b][None, :])
            R = (w[:, :, None] * P).sum(axis=(0, 1)) / w.sum()
            ext = (np.sqrt(2.0 / px) * erfi + np.linalg.norm(R - P, axis=2)).max()
            den = (ea.min() + eb.min()) ** 0.25
            q = qb[a * (a + 1) // 2 + b]
            for c, sc in enumerate(shells_aux):
                ec = np.asarray(sc.exps, float)
                arg = (-np.log(1e-8) + 0.5 * np.log(ec)) / ec
                ext_c = np.where(arg < 0, 0.01, np.sqrt(np.maximum(arg, 0))).max()
                beta = ec.min() ** (-(2 * sc.L + 3) / 4) * np.sqrt(float(np.prod(np.arange(2 * sc.L - 1, 0, -2))))
                dist = np.linalg.norm(R - np.asarray(sc.center, float))
                est = q * qa[c] if dist <= ext + ext_c else q * np.pi * np.sqrt(2.0) * beta / (den * dist ** (sc.L + 1))
                count += est >= thresh
    return count


def test_oracle_qvl_screening_cfg1():
    """qvl_estimate in the oracle's Coulomb contraction (the commented-out line
    diabatization/intor.f90:137): the computed triplet set matches an
    independent numpy restatement of the screener, differs from the Schwarz
    set, and moves the raw contraction by little (the skipped triplets are
    distant ones)."""
    from pysisyphus_addons.common.synthetic import config_workload

    w = config_workload("cfg1")
    oracle.set_skip_metric(1)
    try:
        ref = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
        st_s = oracle.last_stats()
        oracle.set_screening("qvl")
        got = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
        st_q = oracle.last_stats()
    finally:
        oracle.set_screening("schwarz")
        oracle.set_skip_metric(0)
    qb = oracle.int_schwarz_bra(w.shells)
    qa = oracle.int_schwarz_aux(w.shells_aux)
    n_np = _qvl_count_numpy(w.shells, w.shells_aux, qb, qa, float(np.float32(1e-10)))
    assert st_q["ntriplets"] - st_q["nskipped"] == n_np
    assert st_q["nskipped"] != st_s["nskipped"]
    diff = np.abs(got - ref).max()
    assert 0.0 < diff < 1e-9 * np.abs(ref).max()


def test_oracle_schwarz_f_g_shells_high_precision():
    """Oracle Schwarz values of same-center pairs with f and g shells (f-d and
    g-p, L_ab 5) against 30-digit McMurchie-Davidson values (tests/md_ref.py):
    the reference's golden vectors stop at d functions. On pairs of a tight g
    shell with a shell on another atom the oracle's horizontal recurrence loses
    up to 7.4e-4 relative; the device is pinned there by test_lmax4_gpu.py."""
    from md_ref import schwarz_pair_mp
    from pysisyphus_addons.common.synthetic import make_workload

    w = make_workload(natoms=3, lmax=4, lauxmax=5, nstates=3, seed=1)
    oracle.set_boys_mode("exact")
    try:
        q = oracle.int_schwarz_bra(w.shells)
    finally:
        oracle.set_boys_mode("reference")
    ia, ib = np.tril_indices(len(w.shells))
    index = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(ia, ib))}
    for a, b, L in ((6, 5, (3, 2)), (7, 3, (4, 1)), (14, 13, (3, 2))):
        sa, sb = w.shells[a], w.shells[b]
        assert (sa.L, sb.L) == L and sa.center_ind == sb.center_ind
        ref = float(schwarz_pair_mp(sa, sb, dps=30))
        assert abs(q[index[(a, b)]] - ref) <= 1e-13 * ref, ((a, b), q[index[(a, b)]], ref)


def test_long_double_solve_against_mpmath():
    """The extended-precision factor + solve used to check FP64 solves of
    ill-conditioned metrics: a Hilbert matrix (condition number ~1e13 at n 10)
    against 50-digit arithmetic. The long-double solve's error is ~1e4x below
    the FP64 LAPACK solve's (the ratio of the unit roundoffs is 4.9e-4)."""
    import mpmath
    import scipy.linalg as sl

    n = 10
    H = np.array([[1.0 / (i + j + 1) for j in range(n)] for i in range(n)])
    b = np.arange(1.0, n + 1.0)
    Y, L = oracle.chol_solve_ld(H, b[:, None], want_L=True)
    mpmath.mp.dps = 50
    Lm = mpmath.cholesky(mpmath.matrix(H.tolist()))
    ym = mpmath.lu_solve(Lm, mpmath.matrix(b.tolist()))
    y_ref = np.array([float(v) for v in ym])
    err_ld = np.abs(Y[:, 0] - y_ref).max()
    err_lp = np.abs(sl.solve_triangular(np.linalg.cholesky(H), b, lower=True) - y_ref).max()
    assert err_ld <= 2e-3 * err_lp, (err_ld, err_lp)
    assert oracle.chol_backward_error_ld(H, L) < 1e-16
    assert oracle.chol_backward_error_ld(H, np.linalg.cholesky(H)) < 1e-15
    with pytest.raises(np.linalg.LinAlgError):
        oracle.chol_solve_ld(np.diag([1.0, -1.0]), np.ones((2, 1)))


def test_coulomb_from_df_matches_driver():
    from pysisyphus_addons.common.synthetic import config_workload

    w = config_workload("cfg1")
    oracle.set_boys_mode("reference")
    df = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    R = oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
    np.testing.assert_allclose(oracle.coulomb_from_df(df, w.nstates), R, rtol=0, atol=1e-12 * np.abs(R).max())


def test_reused_screening_gives_the_same_result():
    from pysisyphus_addons.common.shells import Shells
    from pysisyphus_addons.common.synthetic import config_workload

    w = config_workload("cfg1")
    oracle.set_boys_mode("reference")
    a = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    oracle.set_reuse_screening(1)
    try:
        b = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
        c = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)  # from the cache
        sub = Shells(w.shells[:-1])  # another basis: recomputed, not taken from the cache
        d = oracle.contract_coulomb_densities_2d(sub, w.shells_aux, w.densities[:, :sub.sph_size, :sub.sph_size])
    finally:
        oracle.set_reuse_screening(0)
    e = oracle.contract_coulomb_densities_2d(sub, w.shells_aux, w.densities[:, :sub.sph_size, :sub.sph_size])
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)
    np.testing.assert_array_equal(d, e)
