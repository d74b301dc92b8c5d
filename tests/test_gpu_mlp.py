"""Warm-start network kernels on the tcgen05 tensor cores: the BF16 GEMM
against a float64 product of the same BF16 values (FP32 accumulation: 2e-5 of
the row scale)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> BF16 bit patterns."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_value(bits: np.ndarray) -> np.ndarray:
    return (bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


@pytest.fixture(scope="module")
def lib():
    from aerocfd_b200 import _lib, build
    build.build()
    return _lib.load()


@pytest.mark.parametrize("M,N,K,splits", [(128, 128, 64, 1), (256, 384, 192, 1), (128, 256, 1024, 4), (384, 128, 640, 3)])
def test_tensor_core_gemm(lib, M, N, K, splits):
    rng = np.random.default_rng(M + N + K)
    a = bf16_bits(rng.standard_normal((M, K)))
    b = bf16_bits(rng.standard_normal((N, K)))
    c = np.zeros((M, N), dtype=np.float32)
    p = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    rc = lib.aero_mlp_gemm(p(a), p(b), p(c), M, N, K, splits)
    assert rc == 0, lib.aero_last_error()
    ref = bf16_value(a) @ bf16_value(b).T
    scale = np.sqrt(K) * 4.0
    err = np.max(np.abs(c - ref)) / scale
    print("max abs err / scale", err)
    assert err < 2e-5
