"""Learned bond-order potential: parameter handling and the fmd_sg_* calls.

The network stands in for b_ij of the reference's compute_rebo
(fuller_airebo_npt_md_serial_omp_acc.cpp, AI:275-421); everything else of
that routine is kept.  See include/fullermd.h for the model definition.
Parameters are a dict of numpy arrays
    W1 (32,128), W2 (128,128), W3 (128,128), w4 (128,), m (32,), s (32,), b0, bs
flattened in that order for the C-ABI.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import _lib

D, H = 32, 128
_SHAPES = (("W1", (D, H)), ("W2", (H, H)), ("W3", (H, H)), ("w4", (H,)), ("m", (D,)), ("s", (D,)))
NPARAM = D * H + 2 * H * H + H + 2 * D + 2


def flatten(P: dict) -> np.ndarray:
    parts = [np.asarray(P[k], np.float64).reshape(-1) for k, _ in _SHAPES]
    v = np.concatenate(parts + [np.array([P["b0"], P["bs"]], np.float64)])
    assert v.size == NPARAM
    return np.ascontiguousarray(v)


def unflatten(v: np.ndarray) -> dict:
    v = np.asarray(v, np.float64)
    out, o = {}, 0
    for k, shp in _SHAPES:
        n = int(np.prod(shp))
        out[k] = v[o:o + n].reshape(shp).copy()
        o += n
    out["b0"], out["bs"] = float(v[o]), float(v[o + 1])
    return out


def init_params(seed: int = 0) -> dict:
    """Random weights (N(0, 1/fan_in)), zero bias rows, identity scaling."""
    rng = np.random.default_rng(seed)
    P = dict(W1=rng.normal(0, 1 / np.sqrt(D), (D, H)), W2=rng.normal(0, 1 / np.sqrt(H), (H, H)),
             W3=rng.normal(0, 1 / np.sqrt(H), (H, H)), w4=rng.normal(0, 1 / np.sqrt(H), H),
             m=np.zeros(D), s=np.ones(D), b0=0.0, bs=1.0)
    P["W1"][D - 1] = 0.0
    P["W2"][H - 1] = 0.0
    P["W3"][H - 1] = 0.0
    P["w4"][H - 1] = 0.0
    return P


def save(P: dict, path: str | Path) -> None:
    np.savez(path, **{k: np.asarray(v) for k, v in P.items()})


def load_params(path: str | Path) -> dict:
    with np.load(path) as z:
        P = {k: z[k] for k in z.files}
    P["b0"], P["bs"] = float(P["b0"]), float(P["bs"])
    return P


class Surrogate:
    """A model on one context's device (fmd_sg)."""

    def __init__(self, ctx, P: dict):
        self.lib = _lib.load()
        self.ctx = ctx
        self.h = ctypes.c_void_p()
        v = flatten(P)
        rc = self.lib.fmd_sg_create(ctx.h, v.ctypes.data_as(_lib._dp), ctypes.byref(self.h))
        ctx.check(rc, "fmd_sg_create")
        ctx.adopt(self)

    def close(self):
        if self.h:
            self.lib.fmd_sg_destroy(self.h)
            self.h = ctypes.c_void_p()
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, P: dict):
        v = flatten(P)
        self.ctx.check(self.lib.fmd_sg_set_params(self.h, v.ctypes.data_as(_lib._dp)), "fmd_sg_set_params")

    def params(self) -> dict:
        v = np.zeros(NPARAM)
        self.ctx.check(self.lib.fmd_sg_get_params(self.h, v.ctypes.data_as(_lib._dp)), "fmd_sg_get_params")
        return unflatten(v)

    def rebo_forces(self, pos, h, hi, cnt, lst, cap: int = 12):
        """(E, F[3na], W[9]) of the REBO term with the learned bond order."""
        pos = np.ascontiguousarray(pos, np.float64)
        na = pos.size // 3
        F = np.zeros(3 * na); W = np.zeros(9); E = ctypes.c_double()
        d = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(_lib._dp)
        ip = lambda a: np.ascontiguousarray(a, np.int32).ctypes.data_as(_lib._ip)
        cnt = np.ascontiguousarray(cnt, np.int32); lst = np.ascontiguousarray(lst, np.int32)
        h = np.ascontiguousarray(h, np.float64); hi = np.ascontiguousarray(hi, np.float64)
        rc = self.lib.fmd_sg_rebo_forces(self.h, d(pos), d(h), d(hi), ip(cnt), ip(lst), cap, na,
                                         F.ctypes.data_as(_lib._dp), W.ctypes.data_as(_lib._dp), ctypes.byref(E))
        self.ctx.check(rc, "fmd_sg_rebo_forces")
        return E.value, F, W

    def last_rows(self) -> dict:
        n = ctypes.c_int()
        self.ctx.check(self.lib.fmd_sg_last_rows(self.h, 0, ctypes.byref(n), None, None, None, None, None),
                       "fmd_sg_last_rows")
        R = n.value
        ri = np.zeros(R, np.int32); rj = np.zeros(R, np.int32)
        xn = np.zeros((R, D), np.float32); b = np.zeros(R, np.float32); gx = np.zeros((R, D), np.float32)
        fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        rc = self.lib.fmd_sg_last_rows(self.h, R, ctypes.byref(n), ri.ctypes.data_as(_lib._ip),
                                       rj.ctypes.data_as(_lib._ip), fp(xn), fp(b), fp(gx))
        self.ctx.check(rc, "fmd_sg_last_rows")
        return dict(i=ri, j=rj, xn=xn, b=b, gx=gx)

    # ---- training ---------------------------------------------------------
    def loss_grad(self, pos, h, hi, cnt, lst, F_ref, E_ref, W_ref, wE=1.0, wF=1.0, wW=1.0, cap: int = 12):
        """(loss, gradient dict) of one snapshot against given reference values."""
        pos = np.ascontiguousarray(pos, np.float64)
        na = pos.size // 3
        d = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(_lib._dp)
        ip = lambda a: np.ascontiguousarray(a, np.int32).ctypes.data_as(_lib._ip)
        keep = [np.ascontiguousarray(a, t) for a, t in ((pos, np.float64), (h, np.float64), (hi, np.float64),
                                                      (cnt, np.int32), (lst, np.int32), (F_ref, np.float64),
                                                      (W_ref, np.float64))]
        g = np.zeros(NPARAM)
        L = ctypes.c_double()
        rc = self.lib.fmd_sg_loss_grad(self.h, d(keep[0]), d(keep[1]), d(keep[2]), ip(keep[3]), ip(keep[4]), cap,
                                       na, d(keep[5]), float(E_ref), d(keep[6]), wE, wF, wW, ctypes.byref(L),
                                       g.ctypes.data_as(_lib._dp))
        self.ctx.check(rc, "fmd_sg_loss_grad")
        return L.value, unflatten(g)

    def train(self, data: "Dataset", steps: int, batch: int = 4, lr: float = 3e-3, lr_final: float = 3e-5,
              wE: float = 1.0, wF: float = 1.0, wW: float = 1.0, clip: float = 0.0, seed: int = 0,
              n_train: int = 0) -> np.ndarray:
        """Adam on the GPU; returns (steps, 2): loss and batch force RMSE (eV/A) per step."""
        a = _lib.SgTrainArgs(steps, batch, n_train, seed, lr, lr_final, wE, wF, wW, clip)
        hist = np.zeros(2 * steps)
        rc = self.lib.fmd_sg_train(self.h, data.h, ctypes.byref(a), hist.ctypes.data_as(_lib._dp))
        self.ctx.check(rc, "fmd_sg_train")
        return hist.reshape(steps, 2)

    def eval(self, data: "Dataset", first: int = 0, n: int | None = None) -> np.ndarray:
        """Force RMSE (eV/A) against the reference REBO forces, per snapshot."""
        n = len(data) - first if n is None else n
        out = np.zeros(n)
        rc = self.lib.fmd_sg_eval(self.h, data.h, first, n, out.ctypes.data_as(_lib._dp))
        self.ctx.check(rc, "fmd_sg_eval")
        return out

    def feature_stats(self, data: "Dataset", first: int = 0, n: int | None = None):
        n = len(data) - first if n is None else n
        m = np.zeros(D); s = np.zeros(D)
        rc = self.lib.fmd_sg_feature_stats(self.h, data.h, first, n, m.ctypes.data_as(_lib._dp),
                                           s.ctypes.data_as(_lib._dp))
        self.ctx.check(rc, "fmd_sg_feature_stats")
        return m, s


class Dataset:
    """Training snapshots on the device (fmd_sg_data); reference REBO energy,
    forces and virial come from the plain REBO kernel."""

    def __init__(self, ctx):
        self.lib = _lib.load()
        self.ctx = ctx
        self.h = ctypes.c_void_p()
        ctx.check(self.lib.fmd_sg_data_create(ctx.h, ctypes.byref(self.h)), "fmd_sg_data_create")
        ctx.adopt(self)

    def __len__(self) -> int:
        return int(self.lib.fmd_sg_data_count(self.h))

    def add(self, pos, h, hi, cnt, lst, cap: int = 12) -> None:
        pos = np.ascontiguousarray(pos, np.float64)
        d = lambda a: np.ascontiguousarray(a, np.float64)
        ia = lambda a: np.ascontiguousarray(a, np.int32)
        arrs = [pos, d(h), d(hi), ia(cnt), ia(lst)]
        rc = self.lib.fmd_sg_data_add(self.h, arrs[0].ctypes.data_as(_lib._dp), arrs[1].ctypes.data_as(_lib._dp),
                                      arrs[2].ctypes.data_as(_lib._dp), arrs[3].ctypes.data_as(_lib._ip),
                                      arrs[4].ctypes.data_as(_lib._ip), cap, pos.size // 3)
        self.ctx.check(rc, "fmd_sg_data_add")

    def add_system(self, system) -> None:
        self.ctx.check(self.lib.fmd_sg_data_add_system(self.h, system.h), "fmd_sg_data_add_system")

    def reference(self, k: int):
        """(E, W9, F) of snapshot k from the plain REBO kernel."""
        na = ctypes.c_int()
        self.ctx.check(self.lib.fmd_sg_data_get(self.h, k, ctypes.byref(na), None, None, None), "fmd_sg_data_get")
        E = ctypes.c_double(); W = np.zeros(9); F = np.zeros(3 * na.value)
        self.ctx.check(self.lib.fmd_sg_data_get(self.h, k, ctypes.byref(na), ctypes.byref(E),
                                                W.ctypes.data_as(_lib._dp), F.ctypes.data_as(_lib._dp)),
                       "fmd_sg_data_get")
        return E.value, W, F

    def close(self):
        if self.h:
            self.lib.fmd_sg_data_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_dataset(ctx, nc: int = 5, runs: int = 40, steps: int = 50, every: int = 1,
                     T_range=(300.0, 1500.0), P_range=(0.0, 5.0), jitter: float = 0.01, dt: float = 0.5,
                     nlup: int = 20, seed: int = 0) -> "Dataset":
    """Training snapshots from the plain AIREBO kernel's own trajectories.

    `runs` short NPT runs of C60 FCC nc x nc x nc, each at a temperature and
    pressure drawn uniformly from T_range (K) and P_range (GPa) with its own
    seed, advance `steps` steps on the device; every `every` steps the state
    is added (device to device) with its REBO energy, forces and virial from
    the plain kernel.  The reference force field heats its crystal within
    about a hundred steps (by then REBO rows fill their 12 slots, truncation
    makes the list asymmetric and the states are no longer a C60 crystal), so
    runs are kept to the first 50 steps."""
    from . import crystal
    from .api import RunConfig, System
    rng = np.random.default_rng(seed)
    data = Dataset(ctx)
    for r in range(runs):
        T = float(rng.uniform(*T_range))
        P = float(rng.uniform(*P_range))
        s = crystal.atomistic(nc, jitter=jitter, seed=int(rng.integers(1 << 30)), T=T)
        na = s["pos"].size // 3
        cfg = RunConfig(dt=dt, T=T, Pe=P, nsteps=steps, nlup=nlup, gavg_from=1, gavg_to=steps, nc=nc,
                        nmol=s["nmol"])
        sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"],
                             crystal.npt_atom(T, P, na))
        sysd.init()
        for g in range(1, steps + 1):
            sysd.enqueue(g, g)
            if g % every == 0:
                data.add_system(sysd)
        ctx.synchronize()
        sysd.close()
    return data


def fit(ctx, data: "Dataset", steps: int = 2000, batch: int = 4, lr: float = 3e-3, lr_final: float = 3e-5,
        wE: float = 0.1, wF: float = 1.0, wW: float = 0.1, n_train: int = 0, seed: int = 0,
        b0: float = 0.9, bs: float = 0.05) -> tuple["Surrogate", np.ndarray]:
    """A new model trained on the GPU: descriptor normalisation from the
    training snapshots, then Adam with the tensor-core forward/backward
    kernels.  Returns (model, history[steps, 2] = loss, batch force RMSE)."""
    P = init_params(seed)
    P["b0"], P["bs"] = b0, bs
    S = Surrogate(ctx, P)
    n = n_train if n_train > 0 else len(data)
    m, sd = S.feature_stats(data, 0, n)
    P["m"], P["s"] = m, sd + 1e-3
    S.set_params(P)
    hist = S.train(data, steps=steps, batch=batch, lr=lr, lr_final=lr_final, wE=wE, wF=wF, wW=wW, seed=seed,
                   n_train=n)
    return S, hist
