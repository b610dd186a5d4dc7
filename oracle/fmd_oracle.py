"""ctypes access to the test-only checkers built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, never by the product package.

* ``Oracle``: the CPU restatement (fmd_oracle.c and the REBO-II extension's
  rebo2_oracle.c, _build/libfmd_oracle.so).
* ``Ref``: the unmodified reference translation units behind extern "C"
  shims (_ref/libref_*.so), when they have been built.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libfmd_oracle.so"
REF_DIR = HERE / "_ref"

_dp = POINTER(c_double)
_ip = POINTER(c_int)


def d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def i(a):
    return None if a is None else a.ctypes.data_as(_ip)


class FmoNpt(ctypes.Structure):
    _fields_ = [("xi", c_double), ("Q", c_double), ("Vg", c_double * 9), ("W", c_double), ("Pe", c_double),
                ("Tt", c_double), ("Nf", c_int)]

    @classmethod
    def of(cls, a):
        s = cls()
        s.xi, s.Q = a[0], a[1]
        for k in range(9):
            s.Vg[k] = a[2 + k]
        s.W, s.Pe, s.Tt, s.Nf = a[11], a[12], a[13], int(a[14])
        return s

    def arr(self):
        return np.array([self.xi, self.Q, *self.Vg, self.W, self.Pe, self.Tt, float(self.Nf)])


class LJParams(ctypes.Structure):
    _fields_ = [("sig2", c_double), ("eps", c_double), ("rc2", c_double), ("vshift", c_double),
                ("full_virial", c_int)]


class MMTopo(ctypes.Structure):
    _fields_ = [("nb", c_int), ("b_i0", _ip), ("b_i1", _ip), ("b_kb", _dp), ("b_r0", _dp),
                ("nang", c_int), ("a_i0", _ip), ("a_i1", _ip), ("a_i2", _ip), ("a_kth", _dp), ("a_th0", _dp),
                ("ndih", c_int), ("d_i0", _ip), ("d_i1", _ip), ("d_i2", _ip), ("d_i3", _ip), ("d_vn", _dp),
                ("d_mult", _ip), ("d_gamma", _dp),
                ("nimp", c_int), ("m_i0", _ip), ("m_i1", _ip), ("m_i2", _ip), ("m_i3", _ip), ("m_ki", _dp),
                ("m_gamma", _dp)]


class Rebo2Knots(ctypes.Structure):
    """fmo_rebo2_knots (the layout of fmd_rebo2_knots): P_CC(N, 0) knots
    [5][2], pi^rc_CC and T_CC knots [5][5][10][8]."""
    _fields_ = [("pcc", c_double * 10), ("pirc", c_double * 2000), ("tcc", c_double * 2000)]

    @classmethod
    def of(cls, pcc, pirc, tcc):
        s = cls()
        for name, a, n in (("pcc", pcc, 10), ("pirc", pirc, 2000), ("tcc", tcc, 2000)):
            a = np.ascontiguousarray(a, np.float64).reshape(-1)
            assert a.size == n, (name, a.size)
            ctypes.memmove(getattr(s, name), a.ctypes.data, 8 * n)
        return s


def make_topo(t: dict):
    """fmo_mm_topo over a dict of numpy arrays (keeps them alive in the dict)."""
    keep = {}

    def ic(name, k=None):
        a = t[name] if k is None else t[name][:, k]
        a = np.ascontiguousarray(a, dtype=np.int32)
        if a.size == 0:
            a = np.zeros(1, np.int32)
        keep[(name, k)] = a
        return i(a)

    def dc(name):
        a = np.ascontiguousarray(t[name], dtype=np.float64)
        if a.size == 0:
            a = np.zeros(1)
        keep[name] = a
        return d(a)

    c = MMTopo()
    c.nb = len(t["bonds"]); c.b_i0 = ic("bonds", 0); c.b_i1 = ic("bonds", 1); c.b_kb = dc("kb"); c.b_r0 = dc("r0")
    c.nang = len(t["angles"]); c.a_i0 = ic("angles", 0); c.a_i1 = ic("angles", 1); c.a_i2 = ic("angles", 2)
    c.a_kth = dc("kth"); c.a_th0 = dc("th0")
    c.ndih = len(t["dihedrals"])
    c.d_i0, c.d_i1, c.d_i2, c.d_i3 = (ic("dihedrals", k) for k in range(4))
    c.d_vn = dc("vn"); c.d_mult = ic("mult"); c.d_gamma = dc("gamma")
    c.nimp = len(t["impropers"])
    c.m_i0, c.m_i1, c.m_i2, c.m_i3 = (ic("impropers", k) for k in range(4))
    c.m_ki = dc("ki"); c.m_gamma = dc("igamma")
    return c, keep


class Oracle:
    """The CPU restatement (plain C, one thread)."""

    def __init__(self, path: Path = ORACLE_SO):
        if not path.exists():
            raise RuntimeError(f"{path} missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(str(path))
        self.L = L
        L.fmo_nlist_sym.restype = c_int
        L.fmo_nlist_half.restype = c_int
        L.fmo_nlist_intra.restype = c_int
        L.fmo_rigid_forces.restype = c_double
        L.fmo_rebo.restype = c_double
        L.fmo_lj_half.restype = c_double
        L.fmo_lj_params_airebo.restype = LJParams
        L.fmo_lj_params_mm.restype = LJParams
        L.fmo_dihedral_angle.restype = c_double
        L.fmo_mat_det9.restype = c_double
        for f in ("fmo_nlist_sym",):
            getattr(L, f).argtypes = [_dp, _dp, _dp, c_int, c_double, c_int, _ip, _ip]
        L.fmo_nlist_half.argtypes = [_dp, _dp, _dp, c_int, _ip, c_double, c_int, _ip, _ip]
        L.fmo_nlist_intra.argtypes = [_dp, _dp, _dp, c_int, _ip, c_double, c_int, _ip, _ip]
        L.fmo_nlist_half_rows.restype = c_int
        L.fmo_nlist_half_rows.argtypes = [_dp, _dp, _dp, c_int, _ip, c_double, c_int, c_int, c_int, _ip, _ip]
        L.fmo_rigid_forces.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip, c_int, c_int, c_int,
                                       c_double, _dp]
        L.fmo_rebo.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _ip, c_int, c_int]
        L.fmo_rebo_grad.argtypes = [_dp, _dp, _dp, _dp, _ip, _ip, c_int, c_int]
        L.fmo_rebo_grad.restype = c_double
        L.fmo_lj_half.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _ip, c_int, c_int, POINTER(LJParams)]
        L.fmo_airebo_forces.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip, c_int, _dp]
        L.fmo_mm_forces.argtypes = [_dp, _dp, _dp, _dp, _dp, POINTER(MMTopo), _ip, _ip, _dp, _ip, c_int, c_int, _dp]
        L.fmo_mm_topology_mol.argtypes = [_dp, c_int, _ip, c_int, _ip, _ip, _dp, _ip, _dp, _ip, _dp, _ip, _dp]
        L.fmo_rigid_step.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, c_double, c_double, c_int,
                                     c_int, c_double, c_double, POINTER(FmoNpt), _ip, _ip, c_int, _dp, _dp]
        L.fmo_airebo_step.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, c_int, c_double, POINTER(FmoNpt), _ip, _ip,
                                      _ip, _ip, _dp]
        L.fmo_mm_step.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, c_int, c_double, POINTER(FmoNpt), POINTER(MMTopo),
                                  _ip, _ip, _dp, _ip, c_int, _dp]
        K = POINTER(Rebo2Knots)
        L.fmo_rebo2_energy.restype = c_double
        L.fmo_rebo2_energy.argtypes = [_dp, _dp, _dp, _ip, _ip, c_int, c_int, K]
        L.fmo_lj_switch_energy.restype = c_double
        L.fmo_lj_switch_energy.argtypes = [_dp, _dp, _dp, _ip, _ip, c_int, _ip, _ip, c_int, c_int, K]
        L.fmo_rebo2_coordination.argtypes = [_dp, _dp, _dp, _ip, _ip, c_int, c_int, _dp]
        L.fmo_rebo2_bond_order.restype = c_double
        L.fmo_rebo2_bond_order.argtypes = [_dp, _dp, _dp, _ip, _ip, c_int, K, _dp, c_int, c_int, _dp]
        L.fmo_rebo2_spline3.restype = c_double
        L.fmo_rebo2_spline3.argtypes = [K, c_int, c_double, c_double, c_double]
        L.fmo_rebo2_spline_p.restype = c_double
        L.fmo_rebo2_spline_p.argtypes = [K, c_double]
        L.fmo_mat_inv9.argtypes = [_dp, _dp]
        L.fmo_apply_pbc.argtypes = [_dp, _dp, _dp, c_int]

    def mat_inv9(self, h):
        hi = np.zeros(9)
        self.L.fmo_mat_inv9(d(np.ascontiguousarray(h, np.float64)), d(hi))
        return hi

    def apply_pbc(self, pos, h, hi):
        p = np.array(pos, dtype=np.float64)
        self.L.fmo_apply_pbc(d(p), d(h), d(hi), p.size // 3)
        return p

    def nlist_sym(self, pos, h, hi, n, rmcut, cap=80):
        c = np.zeros(n, np.int32); l = np.zeros(n * cap, np.int32)
        dr = self.L.fmo_nlist_sym(d(pos), d(h), d(hi), n, rmcut, cap, i(c), i(l))
        return c, l, dr

    def nlist_half(self, pos, h, hi, na, mol_id, rc, cap=400):
        c = np.zeros(na, np.int32); l = np.zeros(na * cap, np.int32)
        dr = self.L.fmo_nlist_half(d(pos), d(h), d(hi), na, i(np.ascontiguousarray(mol_id, np.int32)), rc, cap,
                                   i(c), i(l))
        return c, l, dr

    def nlist_half_threaded(self, pos, h, hi, na, mol_id, rc, cap=400, threads=None, chunk=2048):
        """nlist_half with its rows split over host threads (the ctypes
        calls release the GIL); identical output, for systems where the
        O(na^2) serial build would take minutes."""
        import os
        from concurrent.futures import ThreadPoolExecutor
        pos = np.ascontiguousarray(pos, np.float64)
        mol = np.ascontiguousarray(mol_id, np.int32)
        c = np.zeros(na, np.int32); l = np.zeros(na * cap, np.int32)
        # rows near the start scan the most partners: interleave chunk sizes
        spans = [(a, min(a + chunk, na)) for a in range(0, na, chunk)]
        with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as ex:
            drops = list(ex.map(lambda s: self.L.fmo_nlist_half_rows(d(pos), d(h), d(hi), na, i(mol), rc, cap,
                                                                     s[0], s[1], i(c), i(l)), spans))
        return c, l, sum(drops)

    def nlist_intra(self, pos, h, hi, na, mol_id, rc=2.0 + 0.3, cap=12):
        c = np.zeros(na, np.int32); l = np.zeros(na * cap, np.int32)
        dr = self.L.fmo_nlist_intra(d(pos), d(h), d(hi), na, i(np.ascontiguousarray(mol_id, np.int32)), rc, cap,
                                    i(c), i(l))
        return c, l, dr

    def rigid_forces(self, pos, qv, body, h, hi, cnt, lst, n, natom, rmcut2, cap=80):
        F = np.zeros(3 * n); T = np.zeros(3 * n); W = np.zeros(9)
        e = self.L.fmo_rigid_forces(d(F), d(T), d(W), d(pos), d(qv), d(body), d(h), d(hi), i(cnt), i(lst), cap, n,
                                    natom, rmcut2, None)
        return e, F, T, W

    def rebo(self, pos, h, hi, cnt, lst, na, cap=12):
        F = np.zeros(3 * na); W = np.zeros(9)
        e = self.L.fmo_rebo(d(F), d(W), d(pos), d(h), d(hi), i(cnt), i(lst), cap, na)
        return e, F, W

    def lj(self, pos, h, hi, cnt, lst, na, mm=False, cap=400):
        F = np.zeros(3 * na); W = np.zeros(9)
        p = self.L.fmo_lj_params_mm() if mm else self.L.fmo_lj_params_airebo()
        e = self.L.fmo_lj_half(d(F), d(W), d(pos), d(h), d(hi), i(cnt), i(lst), cap, na, ctypes.byref(p))
        return e, F, W

    def airebo_forces(self, pos, h, hi, cr, lr, cl, ll, na):
        F = np.zeros(3 * na); W = np.zeros(9); E = np.zeros(3)
        self.L.fmo_airebo_forces(d(F), d(W), d(pos), d(h), d(hi), i(cr), i(lr), i(cl), i(ll), na, d(E))
        return E, F, W

    def rebo_grad(self, pos, h, hi, cr, lr, na, max_neigh=12):
        """Not the reference: the REBO energy with forces -grad E (the
        FMD_PHYS_REBO option's forces).  Returns (E, F)."""
        F = np.zeros(3 * na)
        E = self.L.fmo_rebo_grad(d(F), d(pos), d(h), d(hi), i(cr), i(lr), max_neigh, na)
        return E, F

    # REBO-II extension (no reference counterpart; rebo2_oracle.c)
    def rebo2_energy(self, pos, h, hi, cr, lr, na, knots: Rebo2Knots, max_neigh=12):
        return self.L.fmo_rebo2_energy(d(pos), d(h), d(hi), i(cr), i(lr), max_neigh, na, ctypes.byref(knots))

    def lj_switch_energy(self, pos, h, hi, cr, lr, cl, ll, na, knots: Rebo2Knots, max_neigh_r=12, max_neigh_l=400):
        return self.L.fmo_lj_switch_energy(d(pos), d(h), d(hi), i(cr), i(lr), max_neigh_r, i(cl), i(ll),
                                           max_neigh_l, na, ctypes.byref(knots))

    def rebo2_coordination(self, pos, h, hi, cr, lr, na, max_neigh=12):
        nc = np.zeros(na)
        self.L.fmo_rebo2_coordination(d(pos), d(h), d(hi), i(cr), i(lr), max_neigh, na, d(nc))
        return nc

    def rebo2_bond_order(self, pos, h, hi, cr, lr, knots: Rebo2Knots, ncoord, a, b, dab, max_neigh=12):
        dv = np.ascontiguousarray(dab, np.float64)
        return self.L.fmo_rebo2_bond_order(d(pos), d(h), d(hi), i(cr), i(lr), max_neigh, ctypes.byref(knots),
                                           d(ncoord), int(a), int(b), d(dv))

    def rebo2_spline3(self, knots: Rebo2Knots, which, x, y, z):
        return self.L.fmo_rebo2_spline3(ctypes.byref(knots), int(which), float(x), float(y), float(z))

    def rebo2_spline_p(self, knots: Rebo2Knots, x):
        return self.L.fmo_rebo2_spline_p(ctypes.byref(knots), float(x))

    def mm_topology_mol(self, coords, bonds):
        coords = np.ascontiguousarray(coords, np.float64).reshape(-1)
        bonds = np.ascontiguousarray(bonds, np.int32).reshape(-1)
        natom, nb = coords.size // 3, bonds.size // 2
        counts = np.zeros(4, np.int32)
        bi = np.zeros(max(1, 4 * nb) * 2, np.int32); br = np.zeros(max(1, 4 * nb))
        ai = np.zeros(max(1, 12 * nb) * 3, np.int32); at = np.zeros(max(1, 12 * nb))
        di = np.zeros(max(1, 36 * nb) * 4, np.int32); dg = np.zeros(max(1, 36 * nb))
        mi = np.zeros(max(1, natom) * 4, np.int32); mg = np.zeros(max(1, natom))
        self.L.fmo_mm_topology_mol(d(coords), natom, i(bonds), nb, i(counts), i(bi), d(br), i(ai), d(at), i(di),
                                   d(dg), i(mi), d(mg))
        nb_, na_, nd_, ni_ = counts
        return {"bonds": bi[:2 * nb_].reshape(-1, 2), "r0": br[:nb_], "angles": ai[:3 * na_].reshape(-1, 3),
                "th0": at[:na_], "dihedrals": di[:4 * nd_].reshape(-1, 4), "gamma": dg[:nd_],
                "impropers": mi[:4 * ni_].reshape(-1, 4), "igamma": mg[:ni_]}

    def mm_forces(self, topo: dict, pos, h, hi, cnt, lst, na, charge=None, mol_id=None):
        c, keep = make_topo(topo)
        F = np.zeros(3 * na); W = np.zeros(9); E = np.zeros(7)
        hq = int(charge is not None and np.any(np.abs(charge) > 1e-10))
        q = np.ascontiguousarray(charge if charge is not None else np.zeros(1), np.float64)
        m = np.ascontiguousarray(mol_id if mol_id is not None else np.zeros(1), np.int32)
        self.L.fmo_mm_forces(d(F), d(W), d(pos), d(h), d(hi), ctypes.byref(c), i(cnt), i(lst), d(q), i(m), hq, na,
                             d(E))
        return E, F, W

    def rigid_step(self, st, body, i0, mmol, natom, rmcut2, dt, cnt, lst, cap=80):
        npt = FmoNpt.of(st["npt"])
        out = np.zeros(2)
        n = st["pos"].size // 3
        self.L.fmo_rigid_step(d(st["pos"]), d(st["vel"]), d(st["qv"]), d(st["omg"]), d(st["F"]), d(st["T"]),
                              d(st["W9"]), d(st["h"]), d(st["hi"]), d(body), i0, mmol, n, natom, rmcut2, dt,
                              ctypes.byref(npt), i(cnt), i(lst), cap, None, d(out))
        st["npt"][:] = npt.arr()
        return out

    def airebo_step(self, st, dt, cr, lr, cl, ll):
        npt = FmoNpt.of(st["npt"])
        out = np.zeros(4)
        na = st["pos"].size // 3
        self.L.fmo_airebo_step(d(st["pos"]), d(st["vel"]), d(st["F"]), d(st["vir9"]), d(st["h"]), d(st["hi"]),
                               d(st["mass"]), na, dt, ctypes.byref(npt), i(cr), i(lr), i(cl), i(ll), d(out))
        st["npt"][:] = npt.arr()
        return out

    def mm_step(self, st, dt, topo, cnt, lst, charge=None, mol_id=None):
        c, keep = make_topo(topo)
        npt = FmoNpt.of(st["npt"])
        out = np.zeros(8)
        na = st["pos"].size // 3
        hq = int(charge is not None and np.any(np.abs(charge) > 1e-10))
        q = np.ascontiguousarray(charge if charge is not None else np.zeros(1), np.float64)
        m = np.ascontiguousarray(mol_id if mol_id is not None else np.zeros(1), np.int32)
        self.L.fmo_mm_step(d(st["pos"]), d(st["vel"]), d(st["F"]), d(st["vir9"]), d(st["h"]), d(st["hi"]), na, dt,
                           ctypes.byref(npt), ctypes.byref(c), i(cnt), i(lst), d(q), i(m), hq, d(out))
        st["npt"][:] = npt.arr()
        return out


def ref_available() -> bool:
    return all((REF_DIR / f).exists() for f in ("libref_ai.so", "libref_lj.so", "libref_mm.so", "libref_core.so"))


class Ref:
    """The reference's own routines (unmodified sources, extern "C" shims)."""

    def __init__(self, omp: bool = False):
        sfx = "_omp" if omp else ""
        self.ai = ctypes.CDLL(str(REF_DIR / f"libref_ai{sfx}.so"))
        self.lj = ctypes.CDLL(str(REF_DIR / f"libref_lj{sfx}.so"))
        self.mm = ctypes.CDLL(str(REF_DIR / f"libref_mm{sfx}.so"))
        self.core = ctypes.CDLL(str(REF_DIR / "libref_core.so"))
        for L, names in ((self.ai, ["ref_ai_compute_rebo", "ref_ai_compute_lj", "ref_ai_ke_total"]),
                         (self.lj, ["ref_lj_forces", "ref_lj_ke_trans", "ref_lj_ke_rot", "ref_lj_default_a0"]),
                         (self.core, ["ref_core_forces", "ref_core_rmcut"])):
            for nme in names:
                getattr(L, nme).restype = c_double
        self.lj.ref_lj_default_a0.argtypes = [c_double, ctypes.c_char_p, c_double]
        self.lj.ref_lj_nlist_build_sym.argtypes = [_dp, _dp, _dp, c_int, c_double, _ip, _ip]
        self.lj.ref_lj_forces.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip, c_int, c_int, c_double, _dp]
        self.lj.ref_lj_step_npt.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, c_double, c_double,
                                            c_int, c_int, c_double, c_double, _dp, _ip, _ip, _dp, _dp]
        self.ai.ref_ai_step_npt.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, c_int, c_double, _dp, _ip, _ip, _ip,
                                            _ip, _dp]
        self.ai.ref_ai_compute_rebo.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _ip, c_int]
        self.ai.ref_ai_compute_lj.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _ip, c_int]
        self.ai.ref_ai_compute_forces.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip, c_int, _dp]
        self.core.ref_core_rmcut.argtypes = []

    # AIREBO
    def ai_lists(self, pos, h, hi, na, mol_id):
        cr = np.zeros(na, np.int32); lr = np.zeros(na * 12, np.int32)
        cl = np.zeros(na, np.int32); ll = np.zeros(na * 400, np.int32)
        m = np.ascontiguousarray(mol_id, np.int32)
        self.ai.ref_ai_build_nlist_rebo(d(pos), d(h), d(hi), na, i(m), i(cr), i(lr))
        self.ai.ref_ai_build_nlist_lj(d(pos), d(h), d(hi), na, i(m), i(cl), i(ll))
        return cr, lr, cl, ll

    def ai_forces(self, pos, h, hi, cr, lr, cl, ll, na):
        F = np.zeros(3 * na); W = np.zeros(9); E = np.zeros(3)
        self.ai.ref_ai_compute_forces(d(F), d(W), d(pos), d(h), d(hi), i(cr), i(lr), i(cl), i(ll), na, d(E))
        return E, F, W

    def ai_rebo(self, pos, h, hi, cr, lr, na):
        F = np.zeros(3 * na); W = np.zeros(9)
        e = self.ai.ref_ai_compute_rebo(d(F), d(W), d(pos), d(h), d(hi), i(cr), i(lr), na)
        return e, F, W

    def ai_lj(self, pos, h, hi, cl, ll, na):
        F = np.zeros(3 * na); W = np.zeros(9)
        e = self.ai.ref_ai_compute_lj(d(F), d(W), d(pos), d(h), d(hi), i(cl), i(ll), na)
        return e, F, W

    def ai_step(self, st, dt, cr, lr, cl, ll):
        out = np.zeros(4)
        na = st["pos"].size // 3
        self.ai.ref_ai_step_npt(d(st["pos"]), d(st["vel"]), d(st["F"]), d(st["vir9"]), d(st["h"]), d(st["hi"]),
                                d(st["mass"]), na, dt, d(st["npt"]), i(cr), i(lr), i(cl), i(ll), d(out))
        return out

    # rigid LJ
    def lj_nlist(self, pos, h, hi, n, rmcut):
        c = np.zeros(n, np.int32); l = np.zeros(n * 80, np.int32)
        self.lj.ref_lj_nlist_build_sym(d(pos), d(h), d(hi), n, rmcut, i(c), i(l))
        return c, l

    def lj_forces(self, pos, qv, body, h, hi, cnt, lst, n, natom, rmcut2):
        F = np.zeros(3 * n); T = np.zeros(3 * n); W = np.zeros(9); lab = np.zeros(n * natom * 3)
        e = self.lj.ref_lj_forces(d(F), d(T), d(W), d(pos), d(qv), d(body), d(h), d(hi), i(cnt), i(lst), n, natom,
                                  rmcut2, d(lab))
        return e, F, T, W

    def lj_step(self, st, body, i0, mmol, natom, rmcut2, dt, cnt, lst):
        out = np.zeros(2)
        n = st["pos"].size // 3
        lab = np.zeros(n * natom * 3)
        self.lj.ref_lj_step_npt(d(st["pos"]), d(st["vel"]), d(st["qv"]), d(st["omg"]), d(st["F"]), d(st["T"]),
                                d(st["W9"]), d(st["h"]), d(st["hi"]), d(body), i0, mmol, n, natom, rmcut2, dt,
                                d(st["npt"]), i(cnt), i(lst), d(lab), d(out))
        return out
