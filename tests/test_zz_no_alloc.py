"""fmd_rebo_forces_noalloc: the REBO force for callers that cannot allocate
device memory (a framework's graph capture, a caller-owned memory pool, an
allocator-free driver).  Device buffers here come from PyTorch, as they would
come from such a caller; the entry point itself gets no context and
allocates nothing.  Its output must equal the regular fmd_rebo_forces on the
same inputs, call after call, although the two calls share the library's
static scratch.

Collected last on purpose (file name), and self-contained, so it runs the
same alone in a fresh process or after the rest of the suite."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import csr_rows, rel

pytestmark = pytest.mark.gpu

TOL = 1e-10   # the FP64 force tolerance used by the other parity tests


def _rebo_list(g, na):
    cr = np.ascontiguousarray(g["cnt_rebo"], np.int32)
    lr = np.zeros(na * 12, np.int32)
    for k, r in enumerate(csr_rows(cr, g["csr_rebo"])):
        lr[k * 12:k * 12 + len(r)] = r
    return cr, lr


def test_rebo_noalloc_matches_rebo_forces(golden):
    import torch
    from fuller_md_en_b200 import Context, _lib

    lib = _lib.load()
    g = golden("airebo_nc2")
    na = g["pos"].size // 3
    cr, lr = _rebo_list(g, na)
    h = np.ascontiguousarray(g["h"], np.float64)
    hi = np.ascontiguousarray(g["hi"], np.float64)
    dp = ctypes.POINTER(ctypes.c_double)

    dev = torch.device("cuda:0")
    d_pos = torch.tensor(g["pos"], dtype=torch.float64, device=dev)
    d_nlc = torch.tensor(cr, dtype=torch.int32, device=dev)
    d_nll = torch.tensor(lr, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    results = []
    for _ in range(2):   # two calls in a row through the same static scratch
        d_F = torch.zeros(3 * na, dtype=torch.float64, device=dev)
        d_W = torch.zeros(9, dtype=torch.float64, device=dev)
        d_E = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        rc = lib.fmd_rebo_forces_noalloc(ctypes.c_void_p(d_pos.data_ptr()), h.ctypes.data_as(dp),
                                         hi.ctypes.data_as(dp), ctypes.c_void_p(d_nlc.data_ptr()),
                                         ctypes.c_void_p(d_nll.data_ptr()), 12, na,
                                         ctypes.c_void_p(d_F.data_ptr()), ctypes.c_void_p(d_W.data_ptr()),
                                         ctypes.c_void_p(d_E.data_ptr()), ctypes.c_void_p(stream))
        assert rc == _lib.FMD_OK
        torch.cuda.synchronize(dev)
        results.append((d_F.cpu().numpy(), d_W.cpu().numpy(), float(d_E.cpu()[0])))

    # the regular (allocating, host-pointer) entry point on the same inputs
    ctx = Context(0)
    F_ref, W_ref = np.zeros(3 * na), np.zeros(9)
    E_ref = ctx.compute_rebo(F_ref, W_ref, g["pos"], h, hi, cr, lr, na)
    ctx.close()

    for F, W, E in results:
        assert abs(E - E_ref) <= TOL * abs(E_ref)
        assert rel(F, F_ref) < TOL
        assert rel(W, W_ref) < TOL
    assert abs(E_ref - float(g["E_rebo"])) <= TOL * abs(float(g["E_rebo"]))

    # sizes beyond the scratch capacity are refused before anything runs
    rc = lib.fmd_rebo_forces_noalloc(ctypes.c_void_p(d_pos.data_ptr()), h.ctypes.data_as(dp), hi.ctypes.data_as(dp),
                                     ctypes.c_void_p(d_nlc.data_ptr()), ctypes.c_void_p(d_nll.data_ptr()), 12,
                                     131072 + 1, ctypes.c_void_p(d_F.data_ptr()), ctypes.c_void_p(d_W.data_ptr()),
                                     ctypes.c_void_p(d_E.data_ptr()), ctypes.c_void_p(stream))
    assert rc == _lib.FMD_ERR_CAPACITY
