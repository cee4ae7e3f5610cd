"""The allocation-free Cholesky solve (pa_cholesky_solve_noalloc) through the C-ABI.

This entry point serves callers that cannot allocate device memory when they
call the library: applications whose GPU memory belongs entirely to another
allocator, and code that must not call cudaMalloc / cudaFree because those
calls can synchronize the device. Its scratch is one fixed device array shared
by all calls, so the checks below run two calls in a row on different sizes
(the second call must not see anything the first one left behind) and compare
each with the allocating entry point pa_cholesky_solve on the same input, at
the tolerance of the other Cholesky tests (1e-12 of the largest element).

The file name sorts last so that a run stopping at its first failure has run
every other test before this one.
"""

import ctypes

import numpy as np
import pytest

from pysisyphus_addons import _native as nat

pytestmark = pytest.mark.gpu


def _spd(rng, n):
    X = rng.normal(size=(n, n))
    return X @ X.T + n * np.eye(n)


def _noalloc(torch, A, B):
    """(L, L^-1 B) from the allocation-free entry point; buffers are owned here."""
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).cuda()
    dB = torch.from_numpy(np.asfortranarray(B).ravel(order="F").copy()).cuda()
    dX = torch.full_like(dB, np.nan)
    n, nrhs = B.shape
    stream = torch.cuda.current_stream()
    rc = nat.load().pa_cholesky_solve_noalloc(n, dA.data_ptr(), nrhs, dB.data_ptr(), dX.data_ptr(),
                                              stream.cuda_stream)
    nat.check(rc)
    L = dA.cpu().numpy().reshape(n, n, order="F")
    Y = dX.cpu().numpy().reshape(n, nrhs, order="F")
    # B is an input only
    np.testing.assert_array_equal(dB.cpu().numpy().reshape(n, nrhs, order="F"), B)
    return L, Y


def test_noalloc_cholesky_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    rng = np.random.default_rng(11)
    # two calls in a row: a larger problem first, then a smaller one that reuses
    # only the front of the shared scratch array
    for n, nrhs in ((700, 130), (65, 7)):
        A = _spd(rng, n)
        B = rng.normal(size=(n, nrhs))
        L, Y = _noalloc(torch, A, B)
        Lref, Yref = nat.cholesky_solve(A, B)
        np.testing.assert_allclose(np.tril(L), np.tril(Lref), atol=1e-12 * np.abs(Lref).max(), rtol=0)
        np.testing.assert_array_equal(np.triu(L, 1), np.triu(A, 1))
        np.testing.assert_allclose(Y, Yref, atol=1e-12 * np.abs(Yref).max(), rtol=0)
        # and directly against LAPACK (numpy's factor, scipy's triangular solve)
        from scipy.linalg import solve_triangular

        Lnp = np.linalg.cholesky(A)
        np.testing.assert_allclose(np.tril(L), Lnp, atol=1e-12 * np.abs(Lnp).max(), rtol=0)
        Ynp = solve_triangular(Lnp, B, lower=True)
        np.testing.assert_allclose(Y, Ynp, atol=1e-12 * np.abs(Ynp).max(), rtol=0)


def test_noalloc_cholesky_rejects_oversized_requests():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    n, nrhs = 2240, 405  # 35 * 4096 + 2240 * 405 + 32 > 2^20 doubles
    assert 35 * 4096 + n * nrhs + 32 > nat.PA_NOALLOC_SCRATCH_DOUBLES
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    rc = nat.load().pa_cholesky_solve_noalloc(n, p, nrhs, p, p, ctypes.c_void_p(0))
    assert rc == nat.PA_ERR_SCRATCH
    assert "scratch" in nat.load().pa_last_error().decode()
    # a request within the limit is accepted
    A = _spd(np.random.default_rng(5), 64)
    B = np.ones((64, 1))
    L, Y = _noalloc(torch, A, B)
    np.testing.assert_allclose(np.tril(L) @ Y, B, atol=1e-12)


def test_noalloc_cholesky_reports_non_spd():
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    A = np.diag([4.0, 1.0, -2.0, 3.0])
    with pytest.raises(nat.PaError) as e:
        _noalloc(torch, A, np.ones((4, 1)))
    assert e.value.code == nat.PA_ERR_NOT_SPD
    # a later good call starts from a cleared status word
    L, Y = _noalloc(torch, np.diag([4.0, 1.0, 2.0, 3.0]), np.ones((4, 1)))
    np.testing.assert_allclose(Y[:, 0], 1.0 / np.sqrt([4.0, 1.0, 2.0, 3.0]), rtol=1e-15)


def test_lookahead_factor_is_bitwise_the_plain_order():
    """pa_cholesky_solve runs the factorization with one step of lookahead: the
    trailing update of each step is split into the next block column (main
    stream) and the rest (second stream). pa_cholesky_solve_noalloc keeps one
    update per step on one stream. Both tile the update into the same 64 x 64
    blocks with the same k order, so the factors and solutions agree bit for
    bit."""
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    rng = np.random.default_rng(5)
    n, nrhs = 900, 9  # 15 block columns: lookahead active for 13 steps
    A = _spd(rng, n)
    B = rng.normal(size=(n, nrhs))
    L, Y = _noalloc(torch, A, B)
    Lref, Yref = nat.cholesky_solve(A, B)
    np.testing.assert_array_equal(np.tril(L), np.tril(Lref))
    np.testing.assert_array_equal(Y, Yref)


def test_noalloc_cholesky_rejects_output_overlapping_the_matrix():
    """L is read while X is written: an output inside A is refused before any
    device work; X == B is allowed (B is copied to the scratch array first)."""
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    n, nrhs = 64, 2
    A = _spd(np.random.default_rng(3), n)
    dA = torch.from_numpy(np.asfortranarray(A).ravel(order="F").copy()).cuda()
    dB = torch.ones(n * nrhs, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    lib = nat.load()
    rc = lib.pa_cholesky_solve_noalloc(n, dA.data_ptr(), nrhs, dB.data_ptr(), dA.data_ptr() + 8 * 100, s)
    assert rc == nat.PA_ERR_ARG and "overlaps" in lib.pa_last_error().decode()
    np.testing.assert_array_equal(dA.cpu().numpy().reshape(n, n, order="F"), A)  # untouched
    Lref, Yref = nat.cholesky_solve(A, np.ones((n, nrhs)))
    nat.check(lib.pa_cholesky_solve_noalloc(n, dA.data_ptr(), nrhs, dB.data_ptr(), dB.data_ptr(), s))
    np.testing.assert_allclose(dB.cpu().numpy().reshape(n, nrhs, order="F"), Yref,
                               atol=1e-12 * np.abs(Yref).max(), rtol=0)


def test_noalloc_cholesky_on_a_second_device():
    """The scratch address is looked up in the current context: a call on
    device 1 after one on device 0 uses device 1's copy of the array."""
    torch = pytest.importorskip("torch")
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    rng = np.random.default_rng(13)
    A = _spd(rng, 200)
    B = rng.normal(size=(200, 5))
    Lref, Yref = nat.cholesky_solve(A, B)
    for dev in (0, 1, 0):
        torch.cuda.set_device(dev)
        L, Y = _noalloc(torch, A, B)
        np.testing.assert_allclose(Y, Yref, atol=1e-12 * np.abs(Yref).max(), rtol=0)
    torch.cuda.set_device(0)
