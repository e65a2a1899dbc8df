"""Learned refinement predictor on the GPU: the tcgen05 GEMM behind its
layers against numpy with the same BF16 rounding."""
import ctypes as C

import numpy as np
import pytest

from agal_b200 import _lib

pytestmark = pytest.mark.gpu


def bf16_bits(x):
    """Round-to-nearest-even FP32 -> BF16 bit patterns, and the rounded values."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r, (r.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("M,N,K", [(128, 32, 16), (300, 32, 288), (1000, 17, 864), (64, 8, 80)])
def test_tcgen05_gemm_matches_numpy(M, N, K):
    rng = np.random.default_rng(M + N + K)
    a_bits, a = bf16_bits(rng.standard_normal((M, K)))
    b_bits, b = bf16_bits(rng.standard_normal((N, K)))
    d = np.zeros((M, N), np.float32)
    rc = _lib.lib().agal_learn_gemm_bf16(a_bits.ctypes.data_as(C.c_void_p), b_bits.ctypes.data_as(C.c_void_p),
                                        d.ctypes.data_as(C.c_void_p), M, N, K)
    assert rc == 0
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    # products of BF16 values are exact in FP32; only the FP32 accumulation rounds
    assert np.abs(d - ref).max() <= 1e-5 * np.abs(ref).max() + 1e-5
