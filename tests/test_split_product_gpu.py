"""The split-BF16 tcgen05 product of the precision form (three BF16 slices per
operand, six slice products accumulated in FP32 in tensor memory) against an
FP64 product: the layout, descriptors and drain used by the weak-triplet
three-center kernels, on plain matrices."""

import numpy as np
import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def run(A, B):
    from pysisyphus_addons import _native

    m, k = A.shape
    n = B.shape[0]
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    C = np.zeros((m, n))
    _native.check(_native.load().pa_split_product_check(m, n, k, _native.ptr(A), _native.ptr(B), _native.ptr(C)))
    return C


@pytest.mark.parametrize("m,n,k", [(128, 48, 128), (128, 40, 96), (56, 24, 40), (7, 8, 16), (121, 40, 1),
                                   (64, 16, 65)])
def test_split_product_matches_fp64(m, n, k):
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    # entries over several decades, both signs (the weak-triplet X rows span
    # many orders of magnitude)
    A = rng.standard_normal((m, k)) * 10.0 ** rng.uniform(-6, 2, (m, k))
    B = rng.standard_normal((n, k)) * 10.0 ** rng.uniform(-3, 1, (n, k))
    C = run(A, B)
    ref = A @ B.T
    # 24-bit slices of each operand, six slice products per term, FP32
    # accumulation: the error is below 6 k 2^-23 + 2^-20 times sum |a_i b_i|
    bound = (6 * k * 2.0**-23 + 2.0**-20) * (np.abs(A) @ np.abs(B).T) + 1e-300
    assert np.all(np.abs(C - ref) <= bound), float(np.max(np.abs(C - ref) / bound))


def test_split_product_exact_on_small_integers():
    rng = np.random.default_rng(3)
    A = rng.integers(-8, 9, (128, 64)).astype(np.float64)
    B = rng.integers(-8, 9, (48, 64)).astype(np.float64)
    assert np.array_equal(run(A, B), A @ B.T)


def test_split_product_rejects_bad_shapes():
    from pysisyphus_addons import _native

    A = np.zeros((129, 4))
    B = np.zeros((8, 4))
    C = np.zeros((129, 8))
    rc = _native.load().pa_split_product_check(129, 8, 4, _native.ptr(A), _native.ptr(B), _native.ptr(C))
    assert rc == _native.PA_ERR_ARG
