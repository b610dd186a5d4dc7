"""tcgen05.mma operand conventions (umma.cuh) against a CPU product.

Every learned-potential kernel reads its operands through the same two
descriptor forms -- K-major and the MN-major view of the interleaved layout --
so one 128 x N x K GEMM per form pins them before the MLP kernels use them.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> bf16 bit patterns."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def bf16_value(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32)


def test_bf16_rounding_helper():
    x = np.array([1.0, 1.00390625, 1.01171875, -3.5, 1e-3], np.float32)
    v = bf16_value(bf16_bits(x))
    assert v[0] == 1.0 and v[1] == 1.0 and v[2] == 1.015625 and v[3] == -3.5
    assert abs(v[4] - 1e-3) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("K,N", [(32, 128), (128, 128), (128, 32), (64, 256)])
def test_umma_tile(mode, K, N):
    from fuller_md_en_b200 import _lib
    lib = _lib.load()
    ctx = ctypes.c_void_p()
    assert lib.fmd_ctx_create(ctypes.byref(ctx), 0) == 0
    try:
        rng = np.random.default_rng(K * 1000 + N * 10 + mode)
        A = bf16_bits(rng.normal(size=(128, K)).astype(np.float32))
        Bt = bf16_bits(rng.normal(size=(N, K)).astype(np.float32))
        D = np.zeros((128, N), np.float32)
        rc = lib.fmd_umma_selftest(ctx, A.ctypes.data, Bt.ctypes.data, K, N, mode,
                                   D.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        assert rc == 0, lib.fmd_ctx_last_error(ctx)
        ref = bf16_value(A).astype(np.float64) @ bf16_value(Bt).astype(np.float64).T
        np.testing.assert_allclose(D, ref, rtol=1e-5, atol=1e-4 * np.sqrt(K))
    finally:
        lib.fmd_ctx_destroy(ctx)
