"""Python mirror of the reference's hot-path routines, backed by the B200
library.  Names, argument meaning and layouts follow the reference
(flat FP64 row-major arrays, int32 lists); each function cites the routine it
replaces.  Every call runs CUDA kernels; nothing here computes on the CPU.

Citations: LJ = src/fuller_LJ_npt_md_serial_omp_acc.cpp,
AI = src/fuller_airebo_npt_md_serial_omp_acc.cpp,
MM = src/fuller_LJ_npt_mmmd_serial_omp_acc.cpp.
"""
from __future__ import annotations

import ctypes
import weakref
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from ._lib import FmdError, NPT, MMTopology, RunParams, Obs, Avg

MAX_NEIGH_RIGID = 80      # LJ:108
MAX_LJ_NEIGH = 400        # AI:127, MM:119
MAX_REBO_NEIGH = 12       # AI:126
LJ_LIST_RC_AIREBO = 3.0 * 3.40 + 2.0    # AI:265 (LJ_RCUT + 2)
LJ_LIST_RC_MM = 3.0 * 3.431 + 2.0       # MM:339 (RCUT + 2)
REBO_LIST_RC = 2.0 + 0.3                # AI:116, AI:253


def _d(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def npt_from_array(a) -> NPT:
    """{xi, Q, Vg[9], W, Pe, Tt, Nf} -> fmd_npt."""
    s = NPT()
    s.xi, s.Q = float(a[0]), float(a[1])
    for k in range(9):
        s.Vg[k] = float(a[2 + k])
    s.W, s.Pe, s.Tt, s.Nf = float(a[11]), float(a[12]), float(a[13]), int(a[14])
    return s


def npt_to_array(s: NPT) -> np.ndarray:
    return np.array([s.xi, s.Q, *list(s.Vg), s.W, s.Pe, s.Tt, float(s.Nf)], dtype=np.float64)


class Context:
    """One device, one stream (fmd_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self.lib.fmd_ctx_create(ctypes.byref(h), device)
        if rc != 0:
            raise FmdError(rc, f"fmd_ctx_create(device={device}) failed: "
                           f"{self.lib.fmd_status_string(rc).decode()}")
        self.h = h
        self._owned = []          # weak references to handles made on this context

    def adopt(self, obj) -> None:
        """Registers a handle (system, batch, model, dataset) that must be
        released before the context itself."""
        self._owned.append(weakref.ref(obj))

    def check(self, rc: int, what: str) -> None:
        if rc != 0:
            msg = self.lib.fmd_ctx_last_error(self.h).decode()
            raise FmdError(rc, f"{what}: {msg}")

    def set_stream(self, stream_ptr: int) -> None:
        self.check(self.lib.fmd_ctx_set_stream(self.h, ctypes.c_void_p(stream_ptr)), "set_stream")

    def stream(self) -> int:
        return int(self.lib.fmd_ctx_get_stream(self.h) or 0)

    def set_precision(self, precision: int) -> None:
        """Pair arithmetic of the atomistic LJ term in host-pointer calls
        (_lib.FMD_PREC_FP64 or _lib.FMD_PREC_FP32_PAIR)."""
        self.check(self.lib.fmd_ctx_set_precision(self.h, int(precision)), "fmd_ctx_set_precision")

    def synchronize(self) -> None:
        self.check(self.lib.fmd_ctx_synchronize(self.h), "synchronize")

    def close(self) -> None:
        if self.h:
            # handles made on this context go first, newest first (a batch
            # before its systems); they hold the context's stream
            for r in reversed(self._owned):
                o = r()
                if o is not None:
                    o.close()
            self._owned.clear()
            self.lib.fmd_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- geometry (LJ:113-151) -------------------------------------------
    def mat_inv9(self, h) -> np.ndarray:
        h = _f64(h)
        hi = np.zeros(9)
        self.check(self.lib.fmd_mat_inv9(self.h, _d(h), _d(hi)), "mat_inv9")
        return hi

    def apply_pbc(self, pos, h, hi) -> np.ndarray:
        pos = _f64(pos).copy()
        n = pos.size // 3
        self.check(self.lib.fmd_apply_pbc(self.h, _d(pos), _d(_f64(h)), _d(_f64(hi)), n), "apply_pbc")
        return pos

    # ---- neighbour lists (a1-a3) -------------------------------------------
    def nlist_build_sym(self, pos, h, hi, n: int, rmcut: float, max_neigh: int = MAX_NEIGH_RIGID):
        """nlist_build_sym (LJ:257-268) -> (nl_count, nl_list, dropped)."""
        cnt = np.zeros(n, np.int32)
        lst = np.zeros(n * max_neigh, np.int32)
        drop = ctypes.c_int(0)
        self.check(self.lib.fmd_nlist_rigid(self.h, _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)), n, float(rmcut),
                                            max_neigh, _i(cnt), _i(lst), ctypes.byref(drop)), "nlist_build_sym")
        return cnt, lst, drop.value

    def build_nlist_lj(self, pos, h, hi, na: int, mol_id, rc_list: float = LJ_LIST_RC_AIREBO,
                       max_neigh: int = MAX_LJ_NEIGH):
        """build_nlist_lj (AI:263-272, MM:337-346) -> (nlc, nll, dropped)."""
        cnt = np.zeros(na, np.int32)
        lst = np.zeros(na * max_neigh, np.int32)
        drop = ctypes.c_int(0)
        self.check(self.lib.fmd_nlist_lj_half(self.h, _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)), na,
                                              _i(_i32(mol_id)), float(rc_list), max_neigh, _i(cnt), _i(lst),
                                              ctypes.byref(drop)), "build_nlist_lj")
        return cnt, lst, drop.value

    def build_nlist_rebo(self, pos, h, hi, na: int, mol_id, rc: float = REBO_LIST_RC,
                         max_neigh: int = MAX_REBO_NEIGH):
        """build_nlist_rebo (AI:251-261) -> (nlc, nll, dropped)."""
        cnt = np.zeros(na, np.int32)
        lst = np.zeros(na * max_neigh, np.int32)
        drop = ctypes.c_int(0)
        self.check(self.lib.fmd_nlist_rebo(self.h, _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)), na,
                                           _i(_i32(mol_id)), float(rc), max_neigh, _i(cnt), _i(lst),
                                           ctypes.byref(drop)), "build_nlist_rebo")
        return cnt, lst, drop.value

    # ---- forces ---------------------------------------------------------------
    def forces(self, pos, qv, body, h, hi, nl_count, nl_list, n: int, natom: int, rmcut2: float,
               max_neigh: int = MAX_NEIGH_RIGID, precision: int = _lib.FMD_PREC_FP64):
        """forces (LJ:271-400) -> (Ep, Fv, Tv, Wm9)."""
        F = np.zeros(3 * n)
        T = np.zeros(3 * n)
        W = np.zeros(9)
        Ep = ctypes.c_double(0)
        self.check(self.lib.fmd_lj_rigid_forces(self.h, _d(_f64(pos)), _d(_f64(qv)), _d(_f64(body)),
                                                _d(_f64(h)), _d(_f64(hi)), _i(_i32(nl_count)), _i(_i32(nl_list)),
                                                max_neigh, n, natom, float(rmcut2), precision, _d(F), _d(T),
                                                _d(W), ctypes.byref(Ep)), "forces")
        return Ep.value, F, T, W

    def compute_rebo(self, F: np.ndarray, vir9: np.ndarray, pos, h, hi, nlc, nll, na: int,
                     max_neigh: int = MAX_REBO_NEIGH) -> float:
        """compute_rebo (AI:275-421): adds into F and vir9 in place; returns Ep."""
        E = ctypes.c_double(0)
        self.check(self.lib.fmd_rebo_forces(self.h, _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)), _i(_i32(nlc)),
                                            _i(_i32(nll)), max_neigh, na, _d(F), _d(vir9), ctypes.byref(E)),
                   "compute_rebo")
        return E.value

    def compute_lj(self, F: np.ndarray, vir9: np.ndarray, pos, h, hi, nlc, nll, na: int,
                   ff: int = _lib.FMD_FF_AIREBO, max_neigh: int = MAX_LJ_NEIGH) -> float:
        """compute_lj (AI:424-473) / MM LJ block (MM:711-764): adds in place; returns Ep."""
        E = ctypes.c_double(0)
        self.check(self.lib.fmd_lj_half_forces(self.h, ff, _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)),
                                               _i(_i32(nlc)), _i(_i32(nll)), max_neigh, na, _d(F), _d(vir9),
                                               ctypes.byref(E)), "compute_lj")
        return E.value

    def rebo2_forces(self, F: np.ndarray, vir9: np.ndarray, pos, h, hi, nlc, nll, na: int, knots: "Rebo2Knots",
                     max_neigh: int = MAX_REBO_NEIGH) -> float:
        """REBO-II energy (fmd_rebo2_forces; no reference counterpart): adds
        -grad E into F and the full virial into vir9; returns E."""
        E = ctypes.c_double(0)
        self.check(self.lib.fmd_rebo2_forces(self.h, _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)), _i(_i32(nlc)),
                                             _i(_i32(nll)), max_neigh, na, ctypes.byref(knots.raw()), _d(F),
                                             _d(vir9), ctypes.byref(E)), "fmd_rebo2_forces")
        return E.value

    def lj_switch_forces(self, F: np.ndarray, vir9: np.ndarray, pos, h, hi, nlc_r, nll_r, nlc_l, nll_l, na: int,
                         knots: "Rebo2Knots", max_neigh_r: int = MAX_REBO_NEIGH,
                         max_neigh_l: int = MAX_LJ_NEIGH) -> float:
        """The switched-LJ correction (fmd_lj_switch_forces): adds into F and
        vir9; returns its energy (the switched LJ is compute_lj plus this)."""
        E = ctypes.c_double(0)
        self.check(self.lib.fmd_lj_switch_forces(self.h, _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)), _i(_i32(nlc_r)),
                                                 _i(_i32(nll_r)), max_neigh_r, _i(_i32(nlc_l)), _i(_i32(nll_l)),
                                                 max_neigh_l, na, ctypes.byref(knots.raw()), _d(F), _d(vir9),
                                                 ctypes.byref(E)), "fmd_lj_switch_forces")
        return E.value

    def compute_forces_airebo(self, pos, h, hi, nlc_r, nll_r, nlc_l, nll_l, na: int):
        """compute_forces (AI:477-495) -> (E3, F, vir9), E3 = (Ep, Ep_rebo, Ep_lj)."""
        F = np.zeros(3 * na)
        W = np.zeros(9)
        E = np.zeros(3)
        self.check(self.lib.fmd_airebo_forces(self.h, _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)), _i(_i32(nlc_r)),
                                              _i(_i32(nll_r)), _i(_i32(nlc_l)), _i(_i32(nll_l)), na, _d(F),
                                              _d(W), _d(E)), "compute_forces")
        return E, F, W

    def compute_forces_mm(self, topo: "Topology", pos, h, hi, nlc, nll, na: int, charge=None, mol_id=None):
        """compute_forces (MM:351-788) -> (E7, F, vir9)."""
        F = np.zeros(3 * na)
        W = np.zeros(9)
        E = np.zeros(7)
        has_q = 0
        q = np.zeros(1)
        m = np.zeros(1, np.int32)
        if charge is not None:
            q = _f64(charge)
            m = _i32(mol_id)
            has_q = int(np.any(np.abs(q) > 1e-10))
        self.check(self.lib.fmd_mm_forces(self.h, ctypes.byref(topo.c), _d(_f64(pos)), _d(_f64(h)), _d(_f64(hi)),
                                          _i(_i32(nlc)), _i(_i32(nll)), _d(q), _i(m), has_q, na, _d(F), _d(W),
                                          _d(E)), "compute_forces")
        return E, F, W

    # ---- one NPT step on host state -----------------------------------------
    def step_npt_rigid(self, st: dict, body, I0: float, Mmol: float, natom: int, rmcut2: float, dt: float,
                       nl_count, nl_list, max_neigh: int = MAX_NEIGH_RIGID, precision: int = _lib.FMD_PREC_FP64):
        """step_npt (LJ:434-538) on a state dict with pos, vel, qv, omg, F, T, W9, h, hi, npt
        (arrays updated in place); returns (Ep, KE)."""
        npt = npt_from_array(st["npt"])
        out = np.zeros(2)
        n = st["pos"].size // 3
        self.check(self.lib.fmd_rigid_step(self.h, _d(st["pos"]), _d(st["vel"]), _d(st["qv"]), _d(st["omg"]),
                                           _d(st["F"]), _d(st["T"]), _d(st["W9"]), _d(st["h"]), _d(st["hi"]),
                                           _d(_f64(body)), float(I0), float(Mmol), n, natom, float(rmcut2),
                                           float(dt), ctypes.byref(npt), _i(_i32(nl_count)), _i(_i32(nl_list)),
                                           max_neigh, precision, _d(out)), "step_npt")
        st["npt"][:] = npt_to_array(npt)
        return out[0], out[1]

    def step_npt_airebo(self, st: dict, dt: float, nlc_r, nll_r, nlc_l, nll_l):
        """step_npt (AI:518-590) on a state dict with pos, vel, F, vir9, h, hi, mass, npt;
        returns (Ep, Ep_rebo, Ep_lj, KE)."""
        npt = npt_from_array(st["npt"])
        out = np.zeros(4)
        na = st["pos"].size // 3
        self.check(self.lib.fmd_airebo_step(self.h, _d(st["pos"]), _d(st["vel"]), _d(st["F"]), _d(st["vir9"]),
                                            _d(st["h"]), _d(st["hi"]), _d(_f64(st["mass"])), na, float(dt),
                                            ctypes.byref(npt), _i(_i32(nlc_r)), _i(_i32(nll_r)), _i(_i32(nlc_l)),
                                            _i(_i32(nll_l)), _d(out)), "step_npt")
        st["npt"][:] = npt_to_array(npt)
        return tuple(out)

    def step_npt_mm(self, st: dict, dt: float, topo: "Topology", nlc, nll, charge=None, mol_id=None):
        """step_npt (MM:811-890); returns (Eb, Ea, Ed, Ei, Elj, Ecoul, Etot, KE)."""
        npt = npt_from_array(st["npt"])
        out = np.zeros(8)
        na = st["pos"].size // 3
        has_q = 0
        q = np.zeros(1)
        m = np.zeros(1, np.int32)
        if charge is not None:
            q = _f64(charge)
            m = _i32(mol_id)
            has_q = int(np.any(np.abs(q) > 1e-10))
        self.check(self.lib.fmd_mm_step(self.h, _d(st["pos"]), _d(st["vel"]), _d(st["F"]), _d(st["vir9"]),
                                        _d(st["h"]), _d(st["hi"]), na, float(dt), ctypes.byref(npt),
                                        ctypes.byref(topo.c), _i(_i32(nlc)), _i(_i32(nll)), _d(q), _i(m), has_q,
                                        _d(out)), "step_npt")
        st["npt"][:] = npt_to_array(npt)
        return tuple(out)


class Topology:
    """Owns the arrays behind an fmd_mm_topology (FlatTopology, MM:226-237).
    Index arrays are given as (n, k) int arrays, k = 2/3/4 atoms per term."""

    def __init__(self, bonds, kb, r0, angles, kth, th0, dihedrals, vn, mult, gamma, impropers, ki, igamma):
        self._keep = []

        def col(a, k):
            c = np.ascontiguousarray(a[:, k], dtype=np.int32)
            if c.size == 0:
                c = np.zeros(1, np.int32)
            self._keep.append(c)
            return _i(c)

        def dv(a):
            c = _f64(a)
            self._keep.append(c)
            return _d(c)

        def iv(a):
            c = _i32(a)
            self._keep.append(c)
            return _i(c)

        bonds = np.asarray(bonds, np.int32).reshape(-1, 2)
        angles = np.asarray(angles, np.int32).reshape(-1, 3)
        dihedrals = np.asarray(dihedrals, np.int32).reshape(-1, 4)
        impropers = np.asarray(impropers, np.int32).reshape(-1, 4)
        t = MMTopology()
        t.nb = len(bonds)
        t.b_i0, t.b_i1, t.b_kb, t.b_r0 = col(bonds, 0), col(bonds, 1), dv(kb), dv(r0)
        t.nang = len(angles)
        t.ang_i0, t.ang_i1, t.ang_i2 = col(angles, 0), col(angles, 1), col(angles, 2)
        t.ang_kth, t.ang_th0 = dv(kth), dv(th0)
        t.ndih = len(dihedrals)
        t.dih_i0, t.dih_i1, t.dih_i2, t.dih_i3 = (col(dihedrals, k) for k in range(4))
        t.dih_vn, t.dih_mult, t.dih_gamma = dv(vn), iv(mult), dv(gamma)
        t.nimp = len(impropers)
        t.imp_i0, t.imp_i1, t.imp_i2, t.imp_i3 = (col(impropers, k) for k in range(4))
        t.imp_ki, t.imp_gamma = dv(ki), dv(igamma)
        self.c = t


@dataclass
class RunConfig:
    dt: float
    T: float
    Pe: float
    T_cold: float = 4.0
    coldstart: int = 0
    warmup: int = 0
    nsteps: int = 0
    nlup: int = 20
    gavg_from: int = 1
    gavg_to: int = 0
    nc: int = 1
    nmol: int = 1
    precision: int = _lib.FMD_PREC_FP64
    use_graphs: int = 1

    def c(self) -> RunParams:
        p = RunParams()
        for k in RunParams._fields_:
            setattr(p, k[0], getattr(self, k[0]))
        return p


class System:
    """A device-resident system (fmd_system): state stays in HBM across steps."""

    def __init__(self, ctx: Context, handle: ctypes.c_void_p, n: int, kind: int):
        self.ctx, self.h, self.n, self.kind = ctx, handle, n, kind
        ctx.adopt(self)

    @classmethod
    def airebo(cls, ctx: Context, cfg: RunConfig, pos, vel, mass, mol_id, h, npt) -> "System":
        na = np.asarray(pos).size // 3
        out = ctypes.c_void_p()
        n = npt_from_array(npt)
        ctx.check(ctx.lib.fmd_system_create_airebo(ctx.h, ctypes.byref(cfg.c()), na, _d(_f64(pos)), _d(_f64(vel)),
                                                   _d(_f64(mass)), _i(_i32(mol_id)), _d(_f64(h)), ctypes.byref(n),
                                                   ctypes.byref(out)), "fmd_system_create_airebo")
        return cls(ctx, out, na, _lib.FMD_SYS_AIREBO)

    @classmethod
    def rigid(cls, ctx: Context, cfg: RunConfig, natom: int, body, I0: float, Mmol: float, rmcut: float,
              pos, vel, qv, omg, h, npt, max_neigh: int = MAX_NEIGH_RIGID) -> "System":
        n = np.asarray(pos).size // 3
        out = ctypes.c_void_p()
        s = npt_from_array(npt)
        ctx.check(ctx.lib.fmd_system_create_rigid(ctx.h, ctypes.byref(cfg.c()), n, natom, _d(_f64(body)), float(I0),
                                                  float(Mmol), float(rmcut), max_neigh, _d(_f64(pos)), _d(_f64(vel)),
                                                  _d(_f64(qv)), _d(_f64(omg)), _d(_f64(h)), ctypes.byref(s),
                                                  ctypes.byref(out)), "fmd_system_create_rigid")
        return cls(ctx, out, n, _lib.FMD_SYS_RIGID)

    @classmethod
    def mm(cls, ctx: Context, cfg: RunConfig, pos, vel, mol_id, topo: Topology, h, npt, charge=None) -> "System":
        na = np.asarray(pos).size // 3
        out = ctypes.c_void_p()
        s = npt_from_array(npt)
        q = _f64(charge) if charge is not None else None
        ctx.check(ctx.lib.fmd_system_create_mm(ctx.h, ctypes.byref(cfg.c()), na, _d(_f64(pos)), _d(_f64(vel)),
                                               _i(_i32(mol_id)), ctypes.byref(topo.c),
                                               _d(q) if q is not None else None, _d(_f64(h)), ctypes.byref(s),
                                               ctypes.byref(out)), "fmd_system_create_mm")
        sysm = cls(ctx, out, na, _lib.FMD_SYS_MM)
        sysm._topo = topo
        return sysm

    @classmethod
    def mm_replicated(cls, ctx: Context, cfg: RunConfig, nmol: int, natom_mol: int, pos, vel, mol_topo: Topology,
                      h, npt) -> "System":
        """An MM system of nmol contiguous molecules of natom_mol atoms (no
        charges) from ONE molecule's topology, replicated on the device
        (fmd_system_create_mm_replicated): the same system as System.mm with
        the full flat topology of the copies."""
        out = ctypes.c_void_p()
        s = npt_from_array(npt)
        ctx.check(ctx.lib.fmd_system_create_mm_replicated(ctx.h, ctypes.byref(cfg.c()), nmol, natom_mol,
                                                          _d(_f64(pos)), _d(_f64(vel)), ctypes.byref(mol_topo.c),
                                                          _d(_f64(h)), ctypes.byref(s), ctypes.byref(out)),
                  "fmd_system_create_mm_replicated")
        sysm = cls(ctx, out, nmol * natom_mol, _lib.FMD_SYS_MM)
        sysm._topo = mol_topo
        return sysm

    def init(self) -> None:
        self.ctx.check(self.ctx.lib.fmd_system_init(self.h), "fmd_system_init")

    def run(self, first: int, last: int) -> Obs:
        o = Obs()
        self.ctx.check(self.ctx.lib.fmd_system_run(self.h, first, last, ctypes.byref(o)), "fmd_system_run")
        return o

    def enqueue(self, first: int, last: int) -> None:
        """Enqueues steps first..last without synchronising."""
        self.ctx.check(self.ctx.lib.fmd_system_enqueue(self.h, first, last), "fmd_system_enqueue")

    def enqueue_obs(self, first: int, last: int, addr: int) -> None:
        """Enqueues steps first..last and an asynchronous copy of step `last`'s
        observables (an Obs) to host address `addr` (page-locked memory lets
        the copy overlap the next steps); wait_obs(last) completes it."""
        self.ctx.check(self.ctx.lib.fmd_system_enqueue_obs(self.h, first, last, ctypes.c_void_p(addr)),
                       "fmd_system_enqueue_obs")

    def wait_obs(self, step: int) -> None:
        self.ctx.check(self.ctx.lib.fmd_system_wait_obs(self.h, step), "fmd_system_wait_obs")

    def averages(self) -> Avg:
        a = Avg()
        self.ctx.check(self.ctx.lib.fmd_system_averages(self.h, ctypes.byref(a)), "fmd_system_averages")
        return a

    def download(self, out: dict | None = None):
        """State of the system: pos, vel (and qv, omg for rigid systems), h and
        the NPT state.  `out` may hold caller-owned float64 arrays of the
        right sizes (e.g. in pinned memory) for pos, vel, qv, omg and h, which
        are filled in place instead of fresh arrays."""
        n = self.n
        out = out or {}
        pos = out.get("pos") if out.get("pos") is not None else np.zeros(3 * n)
        vel = out.get("vel") if out.get("vel") is not None else np.zeros(3 * n)
        rigid = self.kind == _lib.FMD_SYS_RIGID
        qv = (out.get("qv") if out.get("qv") is not None else np.zeros(4 * n)) if rigid else None
        omg = (out.get("omg") if out.get("omg") is not None else np.zeros(3 * n)) if rigid else None
        h = out.get("h") if out.get("h") is not None else np.zeros(9)
        for a, m in ((pos, 3 * n), (vel, 3 * n), (qv, 4 * n), (omg, 3 * n), (h, 9)):
            if a is not None and (a.dtype != np.float64 or a.size != m or not a.flags.c_contiguous):
                raise ValueError("download: out arrays must be contiguous float64 of the state's sizes")
        npt = NPT()
        self.ctx.check(self.ctx.lib.fmd_system_download(self.h, _d(pos), _d(vel), _d(qv) if qv is not None else None,
                                                        _d(omg) if omg is not None else None, _d(h),
                                                        ctypes.byref(npt)), "fmd_system_download")
        return {"pos": pos, "vel": vel, "qv": qv, "omg": omg, "h": h, "npt": npt_to_array(npt)}

    def forces(self):
        """(F of the last force evaluation, torques or None, energies E[8])."""
        n = self.n
        F, E = np.zeros(3 * n), np.zeros(8)
        T = np.zeros(3 * n) if self.kind == _lib.FMD_SYS_RIGID else None
        self.ctx.check(self.ctx.lib.fmd_system_forces(self.h, _d(F), _d(T) if T is not None else None, _d(E)),
                       "fmd_system_forces")
        return F, T, E

    def lj_rows(self):
        """(full LJ gather row lengths of the last build, pruned row lengths of the last prune)."""
        full, pruned = np.zeros(self.n, np.int32), np.zeros(self.n, np.int32)
        self.ctx.check(self.ctx.lib.fmd_system_lj_rows(self.h, _i(full), _i(pruned)), "fmd_system_lj_rows")
        return full, pruned

    def lj_full_rows(self):
        """(row lengths, rows as an (n, stride) array) of the LJ gather's full rows of the last build."""
        stride = ctypes.c_int(0)
        self.ctx.check(self.ctx.lib.fmd_system_lj_full_rows(self.h, None, None, ctypes.byref(stride)),
                       "fmd_system_lj_full_rows")
        cnt = np.zeros(self.n, np.int32)
        lst = np.zeros(self.n * max(stride.value, 1), np.int32)
        self.ctx.check(self.ctx.lib.fmd_system_lj_full_rows(self.h, _i(cnt), _i(lst), ctypes.byref(stride)),
                       "fmd_system_lj_full_rows")
        return cnt, lst.reshape(self.n, -1)

    def lists(self, cap_a: int, cap_b: int = 0):
        n = self.n
        ca, la = np.zeros(n, np.int32), np.zeros(n * cap_a, np.int32)
        cb = np.zeros(n, np.int32) if cap_b else None
        lb = np.zeros(n * cap_b, np.int32) if cap_b else None
        self.ctx.check(self.ctx.lib.fmd_system_lists(self.h, _i(ca), _i(la), _i(cb) if cb is not None else None,
                                                     _i(lb) if lb is not None else None), "fmd_system_lists")
        return ca, la, cb, lb

    def virial(self):
        """(W9 of the last force evaluation, current kinetic energy)."""
        W = np.zeros(9)
        ke = ctypes.c_double(0)
        self.ctx.check(self.ctx.lib.fmd_system_virial(self.h, _d(W), ctypes.byref(ke)), "fmd_system_virial")
        return W, ke.value

    def kernel_ms(self, stage: int, reps: int = 20) -> float:
        """Mean duration (ms) of one launch of a stage, CUDA events on the context stream."""
        ms = ctypes.c_double(0)
        self.ctx.check(self.ctx.lib.fmd_system_kernel_ms(self.h, stage, reps, ctypes.byref(ms)), "kernel_ms")
        return ms.value

    def site_pairs(self) -> int:
        """Rigid systems: site pairs within the LJ cutoff in the current state
        (each molecule pair once), the site-pair kernel's work count."""
        k = ctypes.c_longlong(0)
        self.ctx.check(self.ctx.lib.fmd_system_site_pairs(self.h, ctypes.byref(k)), "fmd_system_site_pairs")
        return k.value

    def step_kernels(self, rebuild: bool, phase: bool = False, judge: bool = False) -> int:
        k = ctypes.c_int(0)
        self.ctx.check(self.ctx.lib.fmd_system_step_kernels(self.h, int(rebuild), int(phase) | (2 * int(judge)),
                                                            ctypes.byref(k)), "step_kernels")
        return k.value

    def lj_shape(self) -> dict:
        """Launch shape of the LJ gather chosen by the autotuner at init."""
        v = [ctypes.c_int(0) for _ in range(4)]
        self.ctx.check(self.ctx.lib.fmd_system_lj_shape(self.h, *[ctypes.byref(x) for x in v]), "fmd_system_lj_shape")
        return dict(zip(("threads", "unroll", "pipelined", "blocks"), (x.value for x in v)))

    def lj_shape_pruned(self) -> dict:
        """Launch shape of the LJ gather over the pruned rows (tuned on them at init)."""
        v = [ctypes.c_int(0) for _ in range(3)]
        self.ctx.check(self.ctx.lib.fmd_system_lj_shape_pruned(self.h, *[ctypes.byref(x) for x in v]),
                       "fmd_system_lj_shape_pruned")
        return dict(zip(("threads", "unroll", "feed"), (x.value for x in v)))

    def set_lj_shape(self, threads: int, unroll: int, feed: int) -> None:
        """Pins the LJ gather's launch shape (feed 0 plain, 1 pipelined, 2 staged rows)."""
        self.ctx.check(self.ctx.lib.fmd_system_set_lj_shape(self.h, threads, unroll, feed), "fmd_system_set_lj_shape")

    def set_physics(self, flags: int) -> None:
        """Opt-in physics corrections (fmd_physics bits, e.g.
        _lib.FMD_PHYS_MM_BONDED); before init().  Default 0: the reference's
        forces."""
        self.ctx.check(self.ctx.lib.fmd_system_set_physics(self.h, int(flags)), "fmd_system_set_physics")

    def set_rebo2(self, knots: "Rebo2Knots", flags: int) -> None:
        """REBO-II extension (fmd_system_set_rebo2): _lib.FMD_REBO2_BOND_ORDER
        and/or _lib.FMD_REBO2_LJ_SWITCH with the spline knots; before init()."""
        self.ctx.check(self.ctx.lib.fmd_system_set_rebo2(self.h, ctypes.byref(knots.raw()), int(flags)),
                       "fmd_system_set_rebo2")

    def set_lj_prune(self, delta: float) -> None:
        """Buffer (A) of the pruned LJ gather rows beyond the cutoff; 0 turns
        pruning off (the full rows every step).  Default 0.5."""
        self.ctx.check(self.ctx.lib.fmd_system_set_lj_prune(self.h, float(delta)), "fmd_system_set_lj_prune")

    def lj_prune(self) -> dict:
        """{'delta', 'evaluations': force evaluations since set-up, 'prunes':
        those that walked the full rows and pruned them}."""
        d = ctypes.c_double(0)
        n = [ctypes.c_longlong(0), ctypes.c_longlong(0)]
        self.ctx.check(self.ctx.lib.fmd_system_lj_prune(self.h, ctypes.byref(d), ctypes.byref(n[0]),
                                                        ctypes.byref(n[1])), "fmd_system_lj_prune")
        return {"delta": d.value, "evaluations": n[0].value, "prunes": n[1].value}

    def use_surrogate(self, model, judge_every: int = 100, rmse_max: float = 0.025) -> None:
        """Learned REBO term from `model` (a surrogate.Surrogate, or None for
        the plain kernel), judged by the plain REBO kernel every `judge_every`
        global steps; above `rmse_max` eV/A force RMSE the plain kernel takes
        over for the rest of the run."""
        self._sg_model = model              # the model must outlive its use here
        hm = model.h if model is not None else None
        self.ctx.check(self.ctx.lib.fmd_system_use_surrogate(self.h, hm, int(judge_every), float(rmse_max)),
                       "fmd_system_use_surrogate")

    def surrogate_status(self) -> dict:
        st = _lib.SgStatus()
        self.ctx.check(self.ctx.lib.fmd_system_surrogate_status(self.h, ctypes.byref(st)),
                       "fmd_system_surrogate_status")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def close(self) -> None:
        if self.h:
            self.ctx.lib.fmd_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Replicas advanced together (fmd_batch): MM systems of one context,
    each phase of a step one launch over all of them.  The systems stay
    usable for download/averages/lists and must outlive the batch."""

    def __init__(self, ctx: Context, systems: list, autotune: bool = True):
        self.ctx = ctx
        self.systems = list(systems)
        arr = (ctypes.c_void_p * len(self.systems))(*[s.h.value if isinstance(s.h, ctypes.c_void_p) else s.h
                                                       for s in self.systems])
        out = ctypes.c_void_p()
        ctx.check(ctx.lib.fmd_batch_create(ctx.h, len(self.systems), arr, int(autotune), ctypes.byref(out)),
                  "fmd_batch_create")
        self.h = out
        ctx.adopt(self)

    def enqueue(self, first: int, last: int) -> None:
        self.ctx.check(self.ctx.lib.fmd_batch_enqueue(self.h, first, last), "fmd_batch_enqueue")

    def run(self, first: int, last: int) -> list:
        self.ctx.check(self.ctx.lib.fmd_batch_run(self.h, first, last), "fmd_batch_run")
        return self.observables()

    def observables(self) -> list:
        obs = (Obs * len(self.systems))()
        self.ctx.check(self.ctx.lib.fmd_batch_observables(self.h, obs), "fmd_batch_observables")
        return list(obs)

    def tuning(self) -> dict:
        t = _lib.BatchTuning()
        self.ctx.check(self.ctx.lib.fmd_batch_get_tuning(self.h, ctypes.byref(t)), "fmd_batch_get_tuning")
        return {k: getattr(t, k) for k, _ in t._fields_}

    def step_kernels(self, rebuild: bool, phase: bool = False, conditional: bool = False) -> int:
        """Kernels launched on every replay of a step's graph; with
        conditional=True, those of its conditional fallback body instead."""
        k = ctypes.c_int(0)
        f = self.ctx.lib.fmd_batch_step_kernels_conditional if conditional else self.ctx.lib.fmd_batch_step_kernels
        self.ctx.check(f(self.h, int(rebuild), int(phase), ctypes.byref(k)), "fmd_batch_step_kernels")
        return k.value

    def close(self) -> None:
        if self.h:
            self.ctx.lib.fmd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mm_replica(ctx: Context, nc: int, T: float, P: float, dt: float = 0.1, seed: int = 42, nlup: int = 20,
               nsteps: int = 10 ** 6, jitter: float = 0.0, precision: int = _lib.FMD_PREC_FP64) -> System:
    """An MM system of C60 FCC nc x nc x nc (Ih C60 geometry, reference force
    constants) at temperature T (K) and pressure P (GPa), not yet initialised."""
    from . import crystal
    coords, topo = _c60_molecule_topology()
    s = crystal.atomistic(nc, coords=coords, jitter=jitter, seed=seed, T=T, mol_base=0)
    na, nmol = s["pos"].size // 3, s["nmol"]
    cfg = RunConfig(dt=dt, T=T, Pe=P, nsteps=nsteps, nlup=nlup, gavg_from=1, gavg_to=nsteps, nc=nc, nmol=nmol,
                    precision=precision)
    # one molecule's topology, replicated over the crystal on the device
    return System.mm_replicated(ctx, cfg, nmol, na // nmol, s["pos"], s["vel"], topo, s["h"],
                                crystal.npt_atom(T, P, na))


_MOL_TOPO = {}


def _c60_molecule_topology():
    """The Ih C60 geometry and its one-molecule MM topology (reference force
    constants), built once per process."""
    if "c60" not in _MOL_TOPO:
        from . import crystal
        coords = crystal.c60_ih()
        t = crystal.mm_topology(coords, crystal.bonds_from_geometry(coords), 1)
        topo = Topology(t["bonds"], t["kb"], t["r0"], t["angles"], t["kth"], t["th0"], t["dihedrals"], t["vn"],
                        t["mult"], t["gamma"], t["impropers"], t["ki"], t["igamma"])
        _MOL_TOPO["c60"] = (coords, topo)
    return _MOL_TOPO["c60"]
