"""The REBO-II extension on the GPU (csrc/rebo2.cu) against its CPU
restatement (oracle/rebo2_oracle.c).

No reference counterpart exists, so parity of the spline terms is unpinned:
the kernels are checked against the mathematics of the oracle's energy.
* energies: the oracle's, to 1e-10 relative;
* forces: -grad E, by central differences of the oracle's energy;
* virial: the full virial, by central differences of the oracle's energy
  under homogeneous strain (dE/d eps_ab = -W_ba);
* zero knots: the reference's REBO energy (recorded E_rebo) and the
  gradient of it (fmo_rebo_grad, the FMD_PHYS_REBO forces).
Inside a system the extension's energies and forces are those of the
standalone entry points, and stay the oracle's along a run."""
from __future__ import annotations

import numpy as np
import pytest

from rebo2_cases import cluster, crystal_case, lists, oracle_knots, random_knots, strained

from fuller_md_en_b200 import Rebo2Knots, RunConfig, System, crystal
from fuller_md_en_b200._lib import FMD_PHYS_REBO, FMD_REBO2_BOND_ORDER, FMD_REBO2_LJ_SWITCH, FmdError

pytestmark = pytest.mark.gpu

H = 1e-5       # A, position step of the central differences
EPS = 1e-6     # strain step


def _fd_forces(energy, pos, comps):
    g = []
    for k in comps:
        p, m = pos.copy(), pos.copy()
        p[k] += H
        m[k] -= H
        g.append((energy(p) - energy(m)) / (2 * H))
    return np.array(g)


def _fd_virial(energy_at, s):
    """-dE/d eps_ab, arranged as W_ba."""
    W = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            ep = energy_at(*strained(s, a, b, EPS))
            em = energy_at(*strained(s, a, b, -EPS))
            W[b, a] = -(ep - em) / (2 * EPS)
    return W.reshape(-1)


def _golden_rows(g):
    na = g["pos"].size // 3
    cnt = g["cnt_rebo"]
    lst = np.zeros(na * 12, np.int32)
    off = 0
    for a in range(na):
        lst[a * 12:a * 12 + cnt[a]] = g["csr_rebo"][off:off + cnt[a]]
        off += cnt[a]
    return na, cnt, lst


def test_zero_knots_give_the_reference_energy_and_its_gradient(ctx, oracle, golden):
    g = golden("airebo_nc2")
    na, cnt, lst = _golden_rows(g)
    F, W = np.zeros(3 * na), np.zeros(9)
    E = ctx.rebo2_forces(F, W, g["pos"], g["h"], g["hi"], cnt, lst, na, Rebo2Knots())
    assert abs(E - float(g["E_rebo"])) <= 1e-10 * abs(float(g["E_rebo"]))
    _, Fg = oracle.rebo_grad(g["pos"], g["h"], g["hi"], cnt, lst, na)
    assert np.max(np.abs(F - Fg)) <= 1e-9 * np.max(np.abs(Fg)), np.max(np.abs(F - Fg))


@pytest.mark.parametrize("case", ["cluster", "crystal"])
def test_rebo2_energy_forces_virial(ctx, oracle, case):
    s = cluster() if case == "cluster" else crystal_case()
    cr, lr, _, _ = lists(oracle, s)
    k = random_knots(21)
    K = oracle_knots(k)
    na = s["na"]
    F, W = np.zeros(3 * na), np.zeros(9)
    E = ctx.rebo2_forces(F, W, s["pos"], s["h"], s["hi"], cr, lr, na, k)
    E0 = oracle.rebo2_energy(s["pos"], s["h"], s["hi"], cr, lr, na, K)
    assert abs(E - E0) <= 1e-10 * abs(E0), (E, E0)
    comps = np.random.default_rng(4).choice(3 * na, 30, replace=False)
    g = _fd_forces(lambda p: oracle.rebo2_energy(p, s["h"], s["hi"], cr, lr, na, K), s["pos"], comps)
    fmax = np.max(np.abs(F))
    assert np.max(np.abs(F[comps] + g)) <= 1e-6 * fmax + 1e-8, np.max(np.abs(F[comps] + g))
    Wfd = _fd_virial(lambda p, h, hi: oracle.rebo2_energy(p, h, hi, cr, lr, na, K), s)
    assert np.max(np.abs(W - Wfd)) <= 1e-6 * np.max(np.abs(Wfd)) + 1e-8, (W, Wfd)


def test_lj_switch_energy_forces_virial(ctx, oracle):
    s = crystal_case()
    cr, lr, cl, ll = lists(oracle, s)
    k = random_knots(22)
    K = oracle_knots(k)
    na = s["na"]
    F, W = np.zeros(3 * na), np.zeros(9)
    E = ctx.lj_switch_forces(F, W, s["pos"], s["h"], s["hi"], cr, lr, cl, ll, na, k)
    E0 = oracle.lj_switch_energy(s["pos"], s["h"], s["hi"], cr, lr, cl, ll, na, K)
    assert E0 != 0.0 and abs(E - E0) <= 1e-10 * abs(E0), (E, E0)
    comps = np.random.default_rng(6).choice(3 * na, 30, replace=False)
    g = _fd_forces(lambda p: oracle.lj_switch_energy(p, s["h"], s["hi"], cr, lr, cl, ll, na, K), s["pos"], comps)
    fmax = np.max(np.abs(F))
    assert np.max(np.abs(F[comps] + g)) <= 1e-6 * fmax + 1e-9, np.max(np.abs(F[comps] + g))
    Wfd = _fd_virial(lambda p, h, hi: oracle.lj_switch_energy(p, h, hi, cr, lr, cl, ll, na, K), s)
    assert np.max(np.abs(W - Wfd)) <= 1e-6 * np.max(np.abs(Wfd)) + 1e-9, (W, Wfd)


def _system(ctx, s, knots=None, flags=0, physics=0, nsteps=10):
    na = s["na"]
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=nsteps, nlup=5, nc=1, nmol=s["nmol"])
    y = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], crystal.npt_atom(300.0, 0.0, na))
    if physics:
        y.set_physics(physics)
    if flags:
        y.set_rebo2(knots, flags)
    y.init()
    return y


def test_system_with_rebo2_matches_the_oracle_along_a_run(ctx, oracle):
    s = crystal_case()
    k = random_knots(23)
    K = oracle_knots(k)
    na = s["na"]
    y = _system(ctx, s, k, FMD_REBO2_BOND_ORDER | FMD_REBO2_LJ_SWITCH)
    try:
        for last in (0, 7):
            if last:
                y.run(1, last)
            st = y.download()
            pos, h = st["pos"], st["h"]
            hi = crystal.inv9(h)
            u = dict(s, pos=pos, h=h, hi=hi)
            cr, lr, cl, ll = lists(oracle, u)
            F, _, E = y.forces()
            Er = oracle.rebo2_energy(pos, h, hi, cr, lr, na, K)
            El = oracle.lj(pos, h, hi, cl, ll, na)[0] + oracle.lj_switch_energy(pos, h, hi, cr, lr, cl, ll, na, K)
            assert abs(E[1] - Er) <= 1e-9 * abs(Er), (last, E[1], Er)
            assert abs(E[2] - El) <= 1e-9 * abs(El), (last, E[2], El)
            # the system's forces are the standalone terms' sum
            Fs, Ws = np.zeros(3 * na), np.zeros(9)
            ctx.rebo2_forces(Fs, Ws, pos, h, hi, cr, lr, na, k)
            ctx.compute_lj(Fs, Ws, pos, h, hi, cl, ll, na)
            ctx.lj_switch_forces(Fs, Ws, pos, h, hi, cr, lr, cl, ll, na, k)
            assert np.max(np.abs(F - Fs)) <= 1e-9 * np.max(np.abs(Fs)), (last, np.max(np.abs(F - Fs)))
    finally:
        y.close()


def test_system_zero_knots_is_the_physical_rebo(ctx):
    """With zero knots the REBO-II bond order is the reference's, so the
    system's forces are those of FMD_PHYS_REBO (the gradient of the
    reference's REBO energy)."""
    s = crystal_case(jitter=0.05, scale=1.0)
    a = _system(ctx, s, Rebo2Knots(), FMD_REBO2_BOND_ORDER)
    b = _system(ctx, s, physics=FMD_PHYS_REBO)
    try:
        Fa, _, Ea = a.forces()
        Fb, _, Eb = b.forces()
        assert abs(Ea[1] - Eb[1]) <= 1e-11 * abs(Eb[1])
        assert np.max(np.abs(Fa - Fb)) <= 1e-9 * np.max(np.abs(Fb))
    finally:
        a.close()
        b.close()


def test_set_rebo2_arguments(ctx):
    s = crystal_case()
    y = _system(ctx, s)
    try:
        with pytest.raises(FmdError):
            y.set_rebo2(Rebo2Knots(), FMD_REBO2_BOND_ORDER)       # after init
    finally:
        y.close()
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=10, nlup=5, nc=1, nmol=s["nmol"])
    z = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"],
                      crystal.npt_atom(300.0, 0.0, s["na"]))
    try:
        with pytest.raises(FmdError):
            z.set_rebo2(Rebo2Knots(), 8)                           # unknown flag
    finally:
        z.close()
