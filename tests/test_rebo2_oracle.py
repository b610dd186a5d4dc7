"""The REBO-II extension's CPU restatement (oracle/rebo2_oracle.c) and the
product's spline expansion, on the CPU.

The reference has no REBO-II terms, so the pin is the zero-table limit: with
every knot zero the bond order is compute_rebo's (AI:301-323) and the energy
is the reference's own recorded E_rebo.  The spline terms themselves are
checked against their definition (interpolation of the knots), and the
product's per-cell coefficients (fmd_rebo2_coeffs) against the oracle's
direct Hermite evaluation."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from rebo2_cases import cluster, crystal_case, lists, oracle_knots, random_knots

from fuller_md_en_b200 import Rebo2Knots, crystal


def _golden_rows(g):
    na = g["pos"].size // 3
    cnt = g["cnt_rebo"]
    lst = np.zeros(na * 12, np.int32)
    off = 0
    for a in range(na):
        lst[a * 12:a * 12 + cnt[a]] = g["csr_rebo"][off:off + cnt[a]]
        off += cnt[a]
    return na, cnt, lst


@pytest.mark.parametrize("name", ["airebo_nc1", "airebo_nc2"])
def test_zero_knots_give_the_reference_rebo_energy(oracle, golden, name):
    g = golden(name)
    na, cnt, lst = _golden_rows(g)
    E = oracle.rebo2_energy(g["pos"], g["h"], g["hi"], cnt, lst, na, oracle_knots(Rebo2Knots()))
    assert abs(E - float(g["E_rebo"])) <= 1e-12 * abs(float(g["E_rebo"])), (E, float(g["E_rebo"]))


def test_oracle_splines_interpolate_their_knots(oracle):
    k = random_knots(3)
    K = oracle_knots(k)
    rng = np.random.default_rng(0)
    e = 1e-6
    for _ in range(40):
        x, y, z = int(rng.integers(0, 5)), int(rng.integers(0, 5)), int(rng.integers(0, 10))
        for which, tab in ((0, k.pirc), (1, k.tcc)):
            f = lambda a, b, c: oracle.rebo2_spline3(K, which, a, b, c)  # noqa: E731
            assert abs(f(x, y, z) - tab[x, y, z, 0]) < 1e-14
            # one-sided differences into the table at its edges
            for ax, (dx, dy, dz) in enumerate(((e, 0, 0), (0, e, 0), (0, 0, e))):
                lo = (x, y, z)[ax] == 0
                hi = (x, y, z)[ax] == (4, 4, 9)[ax]
                if lo:
                    d = (f(x + dx, y + dy, z + dz) - f(x, y, z)) / e
                elif hi:
                    d = (f(x, y, z) - f(x - dx, y - dy, z - dz)) / e
                else:
                    d = (f(x + dx, y + dy, z + dz) - f(x - dx, y - dy, z - dz)) / (2 * e)
                assert abs(d - tab[x, y, z, 1 + ax]) < 1e-6, (which, x, y, z, ax)
    for n in range(5):
        assert abs(oracle.rebo2_spline_p(K, n) - k.pcc[n, 0]) < 1e-14


def _eval_coeffs(c, x, y, z):
    """Evaluates the product's per-cell coefficients (fmd_rebo2_coeffs layout)."""
    def cell(v, n):
        v = min(max(v, 0.0), float(n))
        i = min(int(np.floor(v)), n - 1)
        return i, v - i
    (ix, u), (iy, v), (iz, w) = cell(x, 4), cell(y, 4), cell(z, 9)
    q = c[((ix * 4 + iy) * 9 + iz) * 64:((ix * 4 + iy) * 9 + iz + 1) * 64].reshape(4, 4, 4)  # [c][b][a]
    return float(np.einsum("cba,a,b,c->", q, u ** np.arange(4), v ** np.arange(4), w ** np.arange(4)))


def test_product_coefficients_are_the_oracle_splines(oracle):
    from fuller_md_en_b200 import _lib
    lib = _lib.load()
    k = random_knots(5)
    K = oracle_knots(k)
    out = np.zeros(16 + 2 * 9216)
    raw = k.raw()
    assert lib.fmd_rebo2_coeffs(ctypes.byref(raw), out.ctypes.data_as(_lib._dp)) == 0
    rng = np.random.default_rng(1)
    pts = np.column_stack([rng.uniform(-0.5, 4.5, 300), rng.uniform(-0.5, 4.5, 300), rng.uniform(-0.5, 9.5, 300)])
    for which in (0, 1):
        tab = out[16 + which * 9216:16 + (which + 1) * 9216]
        for x, y, z in pts:
            assert abs(_eval_coeffs(tab, x, y, z) - oracle.rebo2_spline3(K, which, x, y, z)) < 1e-13
    for x in rng.uniform(-0.5, 4.5, 100):
        xc = min(max(x, 0.0), 4.0)
        n = min(int(np.floor(xc)), 3)
        u = xc - n
        p = float(np.dot(out[4 * n:4 * n + 4], u ** np.arange(4)))
        assert abs(p - oracle.rebo2_spline_p(K, x)) < 1e-13


@pytest.mark.parametrize("case", ["cluster", "crystal"])
def test_energy_is_invariant_under_rigid_motion(oracle, case):
    s = cluster() if case == "cluster" else crystal_case()
    cr, lr, cl, ll = lists(oracle, s)
    K = oracle_knots(random_knots(9))
    na = s["na"]
    E0 = oracle.rebo2_energy(s["pos"], s["h"], s["hi"], cr, lr, na, K)
    S0 = oracle.lj_switch_energy(s["pos"], s["h"], s["hi"], cr, lr, cl, ll, na, K)
    # translation, then a rotation of atoms and cell together
    t = np.array([0.37, -1.21, 2.05])
    pos_t = (s["pos"].reshape(-1, 3) + t).reshape(-1)
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]]) @ \
        np.array([[1, 0, 0], [0, np.cos(0.4), -np.sin(0.4)], [0, np.sin(0.4), np.cos(0.4)]])
    h_r = (R @ s["h"].reshape(3, 3)).reshape(-1)
    pos_r = (s["pos"].reshape(-1, 3) @ R.T).reshape(-1)
    for pos, h in ((pos_t, s["h"]), (pos_r, h_r)):
        hi = crystal.inv9(h)
        E = oracle.rebo2_energy(pos, h, hi, cr, lr, na, K)
        S = oracle.lj_switch_energy(pos, h, hi, cr, lr, cl, ll, na, K)
        assert abs(E - E0) <= 1e-10 * abs(E0)
        assert abs(S - S0) <= 1e-10 * max(abs(S0), 1e-3)


def test_cases_exercise_every_branch(oracle):
    """The configurations reach the parts of the bond order the force tests
    must cover: non-integer coordination, the conjugation switch, pairs in
    the LJ switch range with b* inside the window."""
    s = cluster()
    cr, lr, _, _ = lists(oracle, s)
    nc = oracle.rebo2_coordination(s["pos"], s["h"], s["hi"], cr, lr, s["na"])
    assert np.any((nc > 2.05) & (nc < 2.95)) and np.any(nc > 3.05) and np.any(nc > 4.0)
    c = crystal_case()
    cr, lr, cl, ll = lists(oracle, c)
    K = oracle_knots(random_knots(9))
    nc = oracle.rebo2_coordination(c["pos"], c["h"], c["hi"], cr, lr, c["na"])
    P = c["pos"].reshape(-1, 3)
    H, Hi = c["h"].reshape(3, 3), c["hi"].reshape(3, 3)
    inwin = close = 0
    for i in range(c["na"]):
        for jn in range(cl[i]):
            j = ll[i * 400 + jn]
            d = P[j] - P[i]
            sfr = Hi @ d
            d = H @ (sfr - np.round(sfr))
            if np.linalg.norm(d) < 2 ** (1 / 6) * 3.4:
                close += 1
                b = oracle.rebo2_bond_order(c["pos"], c["h"], c["hi"], cr, lr, K, nc, i, j, d)
                inwin += 0.77 < b < 0.81
    assert close > 100 and inwin > 10, (close, inwin)


def test_switch_vanishes_beyond_its_range(oracle):
    s = crystal_case(jitter=0.0, scale=1.3)
    cr, lr, cl, ll = lists(oracle, s)
    K = oracle_knots(random_knots(2))
    assert oracle.lj_switch_energy(s["pos"], s["h"], s["hi"], cr, lr, cl, ll, s["na"], K) == 0.0


def test_coefficient_builder_rejects_null_arguments():
    from fuller_md_en_b200 import _lib
    lib = _lib.load()
    out = np.zeros(16 + 2 * 9216)
    raw = Rebo2Knots().raw()
    assert lib.fmd_rebo2_coeffs(None, out.ctypes.data_as(_lib._dp)) == _lib.FMD_ERR_ARG
    assert lib.fmd_rebo2_coeffs(ctypes.byref(raw), None) == _lib.FMD_ERR_ARG
    assert lib.fmd_rebo2_coeffs(ctypes.byref(raw), out.ctypes.data_as(_lib._dp)) == _lib.FMD_OK
    assert not np.any(out), "zero knots give zero coefficients"
