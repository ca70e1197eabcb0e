"""The sliced int8 tensor-core GEMM (gli_b200_dgemm_sliced_dev).

C = A B^T with FP64 inputs and output, evaluated on the tcgen05 tensor cores by
splitting every row into 7-bit int8 slices.  The public entry point keeps 7
slices and 8 product classes, so it must agree with an FP64 product to FP64
level: exactly for integer-valued operands (every slice product is an exact
int32 sum) and to within 2^-46 of K max|a| max|b| for random operands.  The
cases run smallest first, so that a layout error shows on a single tile.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dgemm(a, b, ldc=None):
    import torch

    import gausslectronitegrate_b200 as gli

    lib = gli.lib()
    if lib.gli_b200_device_count() == 0:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    M, K = a.shape
    N = b.shape[0]
    ldc = ldc or N
    da = torch.tensor(a, dtype=torch.float64, device="cuda")
    db = torch.tensor(b, dtype=torch.float64, device="cuda")
    dc = torch.full((M, ldc), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = lib.gli_b200_dgemm_sliced_dev(C.c_void_p(da.data_ptr()), K, C.c_void_p(db.data_ptr()), K,
                                       C.c_void_p(dc.data_ptr()), ldc, M, N, K, C.c_void_p(stream.cuda_stream))
    assert rc == 0, lib.gli_b200_last_error_message().decode()
    stream.synchronize()
    return dc.cpu().numpy()[:, :N]


@pytest.mark.parametrize("M,N,K", [(128, 64, 32), (128, 64, 96), (200, 70, 130), (300, 129, 1000)])
def test_integer_operands_exact(M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    a = rng.integers(-1000, 1001, size=(M, K)).astype(np.float64)
    b = rng.integers(-1000, 1001, size=(N, K)).astype(np.float64)
    c = _dgemm(a, b)
    expected = a.astype(np.int64) @ b.astype(np.int64).T
    np.testing.assert_array_equal(c, expected.astype(np.float64))


@pytest.mark.parametrize("M,N,K", [(128, 64, 32), (257, 65, 77), (640, 384, 2048)])
def test_random_operands_fp64_level(M, N, K):
    rng = np.random.default_rng(M + N + K)
    a = rng.standard_normal((M, K)) * np.exp(rng.uniform(-20, 20, size=(M, 1)))  # rows of very different scale
    b = rng.standard_normal((N, K))
    c = _dgemm(a, b)
    expected = a @ b.T
    bound = 2.0**-46 * K * np.abs(a).max(axis=1)[:, None] * np.abs(b).max(axis=1)[None, :]
    err = np.abs(c - expected)
    assert np.all(err <= bound), f"max err/bound {np.max(err / bound):.3g}"


def test_zero_rows_and_leading_dimension():
    rng = np.random.default_rng(5)
    a = rng.standard_normal((130, 40))
    a[3] = 0.0
    b = rng.standard_normal((66, 40))
    b[65] = 0.0
    c = _dgemm(a, b, ldc=80)
    assert np.all(c[3] == 0.0) and np.all(c[:, 65] == 0.0)
    np.testing.assert_allclose(c, a @ b.T, rtol=0, atol=1e-12)


def test_rejects_bad_arguments():
    import gausslectronitegrate_b200 as gli

    lib = gli.lib()
    rc = lib.gli_b200_dgemm_sliced_dev(None, 4, None, 4, None, 4, 4, 4, 4, None)
    assert rc == 2
    rc = lib.gli_b200_dgemm_sliced_dev(C.c_void_p(16), 4, C.c_void_p(16), 4, C.c_void_p(16), 4, 4, 4, 9000, None)
    assert rc == 2  # leading dimensions below K are rejected before anything runs
