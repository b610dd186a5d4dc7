"""tcgen05.mma operand conventions (umma.cuh) against a CPU product.

Every learned-potential kernel reads its operands through the same two
descriptor forms -- K-major and the MN-major view of the interleaved layout --
so one 128 x N x K GEMM per form pins them before the MLP kernels use them.
The GEMM kernel is test code (tests/cuda/umma_selftest.cu, built into
tests/_build/), not part of the product library.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import pytest

# test-only library built from tests/cuda/umma_selftest.cu by the package's build
SELFTEST = Path(__file__).resolve().parent / "_build" / "libfmd_umma_selftest.so"


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
    lib = ctypes.CDLL(str(SELFTEST))
    lib.fmd_umma_selftest.restype = ctypes.c_int
    lib.fmd_umma_selftest.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_float)]
    rng = np.random.default_rng(K * 1000 + N * 10 + mode)
    A = bf16_bits(rng.normal(size=(128, K)).astype(np.float32))
    Bt = bf16_bits(rng.normal(size=(N, K)).astype(np.float32))
    D = np.zeros((128, N), np.float32)
    rc = lib.fmd_umma_selftest(A.ctypes.data, Bt.ctypes.data, K, N, mode,
                               D.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert rc == 0, rc
    ref = bf16_value(A).astype(np.float64) @ bf16_value(Bt).astype(np.float64).T
    np.testing.assert_allclose(D, ref, rtol=1e-5, atol=1e-4 * np.sqrt(K))
