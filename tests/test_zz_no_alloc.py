"""fmd_rebo_forces_noalloc: the REBO force for callers that cannot allocate
device memory (a memory pool that owns all device memory and forbids side
allocations, a driver that must not touch the allocator after start-up).
Device buffers here come from PyTorch, as they would come from such a
caller's pool; the entry point itself gets no context and allocates nothing.
Its output must equal the regular fmd_rebo_forces on the same inputs, call
after call, although the calls share the library's static scratch; the
caller's current device must be unchanged afterwards.

Collected last on purpose (file name), and self-contained, so it runs the
same alone in a fresh process or after the rest of the suite."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import csr_rows, rel

pytestmark = pytest.mark.gpu

TOL = 1e-10   # the FP64 force tolerance used by the other parity tests
MAX_ATOMS = 131072


def _rebo_list(g, na):
    cr = np.ascontiguousarray(g["cnt_rebo"], np.int32)
    lr = np.zeros(na * 12, np.int32)
    for k, r in enumerate(csr_rows(cr, g["csr_rebo"])):
        lr[k * 12:k * 12 + len(r)] = r
    return cr, lr


def _noalloc_calls(lib, pos, h, hi, cr, lr, na, ncalls=2):
    """ncalls back-to-back calls on the current stream; after each call the
    host h/hi arrays are overwritten before the GPU has run anything, since
    the call takes them by value."""
    import torch
    dp = ctypes.POINTER(ctypes.c_double)
    dev = torch.device("cuda:0")
    d_pos = torch.tensor(pos, dtype=torch.float64, device=dev)
    d_nlc = torch.tensor(cr, dtype=torch.int32, device=dev)
    d_nll = torch.tensor(lr, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    before = torch.cuda.current_device()
    out = []
    for _ in range(ncalls):
        hh = np.array(h, np.float64)
        hhi = np.array(hi, np.float64)
        d_F = torch.zeros(3 * na, dtype=torch.float64, device=dev)
        d_W = torch.zeros(9, dtype=torch.float64, device=dev)
        d_E = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        rc = lib.fmd_rebo_forces_noalloc(ctypes.c_void_p(d_pos.data_ptr()), hh.ctypes.data_as(dp),
                                         hhi.ctypes.data_as(dp), ctypes.c_void_p(d_nlc.data_ptr()),
                                         ctypes.c_void_p(d_nll.data_ptr()), 12, na,
                                         ctypes.c_void_p(d_F.data_ptr()), ctypes.c_void_p(d_W.data_ptr()),
                                         ctypes.c_void_p(d_E.data_ptr()), ctypes.c_void_p(stream))
        hh[:] = np.nan
        hhi[:] = np.nan
        assert rc == 0
        assert torch.cuda.current_device() == before
        torch.cuda.synchronize(dev)
        out.append((d_F.cpu().numpy(), d_W.cpu().numpy(), float(d_E.cpu()[0])))
    return out, (d_pos, d_nlc, d_nll, stream)


def test_rebo_noalloc_matches_rebo_forces(golden):
    from fuller_md_en_b200 import Context, _lib

    lib = _lib.load()
    g = golden("airebo_nc2")
    na = g["pos"].size // 3
    cr, lr = _rebo_list(g, na)
    h = np.ascontiguousarray(g["h"], np.float64)
    hi = np.ascontiguousarray(g["hi"], np.float64)
    results, (d_pos, d_nlc, d_nll, stream) = _noalloc_calls(lib, g["pos"], h, hi, cr, lr, na)

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
    import torch
    dp = ctypes.POINTER(ctypes.c_double)
    d_F = torch.zeros(3, dtype=torch.float64, device="cuda:0")
    rc = lib.fmd_rebo_forces_noalloc(ctypes.c_void_p(d_pos.data_ptr()), h.ctypes.data_as(dp), hi.ctypes.data_as(dp),
                                     ctypes.c_void_p(d_nlc.data_ptr()), ctypes.c_void_p(d_nll.data_ptr()), 12,
                                     MAX_ATOMS + 1, ctypes.c_void_p(d_F.data_ptr()), ctypes.c_void_p(d_F.data_ptr()),
                                     ctypes.c_void_p(d_F.data_ptr()), ctypes.c_void_p(stream))
    assert rc == _lib.FMD_ERR_CAPACITY


def test_rebo_noalloc_capped_grid_nc8():
    """122,880 atoms: more than the 1,024 blocks of the static partials hold
    at four threads per atom, so the grid is capped and the kernel's
    grid-stride loop covers the rest."""
    from fuller_md_en_b200 import Context, crystal, _lib

    lib = _lib.load()
    s = crystal.atomistic(8, jitter=0.01, seed=5)
    pos, h, hi, mol = s["pos"], s["h"], s["hi"], s["mol_id"]
    na = pos.size // 3
    assert 4 * na > 1024 * 128 and na <= MAX_ATOMS
    ctx = Context(0)
    cr, lr, _ = ctx.build_nlist_rebo(pos, h, hi, na, mol)
    F_ref, W_ref = np.zeros(3 * na), np.zeros(9)
    E_ref = ctx.compute_rebo(F_ref, W_ref, pos, h, hi, cr, lr, na)
    ctx.close()
    results, _ = _noalloc_calls(lib, pos, h, hi, cr, lr, na)
    for F, W, E in results:
        assert abs(E - E_ref) <= TOL * abs(E_ref)
        assert rel(F, F_ref) < TOL
        assert rel(W, W_ref) < TOL
