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
