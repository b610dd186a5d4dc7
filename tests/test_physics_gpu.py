"""Opt-in physics corrections (fmd_system_set_physics).  They have no
reference counterpart, so they are checked against the mathematics: with
FMD_PHYS_MM_BONDED every MM force is -grad E of the MM energy, measured by
central differences of the system's own energy.  Without the flag the system
keeps the reference's bond and angle forces (+grad E, MM:389-398,
MM:468-491), which the same check rejects."""
from __future__ import annotations

import numpy as np
import pytest

from fuller_md_en_b200 import RunConfig, System, Topology, crystal
from fuller_md_en_b200._lib import FMD_PHYS_MM_BONDED, FmdError

pytestmark = pytest.mark.gpu

DELTA = 1e-5      # A


def _mm(ctx, s, t, pos, physics):
    na = pos.size // 3
    topo = Topology(t["bonds"], t["kb"], t["r0"], t["angles"], t["kth"], t["th0"], t["dihedrals"], t["vn"],
                    t["mult"], t["gamma"], t["impropers"], t["ki"], t["igamma"])
    cfg = RunConfig(dt=0.1, T=300.0, Pe=0.0, nsteps=10, nlup=20, nc=1, nmol=s["nmol"])
    y = System.mm(ctx, cfg, pos, s["vel"], s["mol_id"], topo, s["h"], crystal.npt_atom(300.0, 0.0, na))
    if physics:
        y.set_physics(physics)
    y.init()
    F, _, E = y.forces()
    y.close()
    return F, E[6]


def _fd_error(ctx, s, t, physics, comps):
    F, _ = _mm(ctx, s, t, s["pos"], physics)
    err = []
    for k in comps:
        p, m = s["pos"].copy(), s["pos"].copy()
        p[k] += DELTA
        m[k] -= DELTA
        g = (_mm(ctx, s, t, p, physics)[1] - _mm(ctx, s, t, m, physics)[1]) / (2 * DELTA)
        err.append(abs(F[k] + g))
    return max(err), float(np.max(np.abs(F)))


def _system():
    coords = crystal.c60_ih()
    s = crystal.atomistic(1, coords=coords, jitter=0.04, seed=17, T=300.0, mol_base=0)
    t = crystal.mm_topology(coords, crystal.bonds_from_geometry(coords), s["nmol"])
    return s, t


def test_mm_physical_forces_are_minus_grad_energy(ctx):
    s, t = _system()
    rng = np.random.default_rng(5)
    comps = rng.choice(s["pos"].size, 12, replace=False)
    err, fmax = _fd_error(ctx, s, t, FMD_PHYS_MM_BONDED, comps)
    assert err <= 1e-6 * fmax + 1e-8, (err, fmax)


def test_reference_mm_forces_are_not(ctx):
    s, t = _system()
    rng = np.random.default_rng(5)
    comps = rng.choice(s["pos"].size, 12, replace=False)
    err, fmax = _fd_error(ctx, s, t, 0, comps)
    assert err > 1e-2 * fmax, (err, fmax)


def test_physics_flag_checks(ctx):
    s, t = _system()
    na = s["pos"].size // 3
    topo = Topology(t["bonds"], t["kb"], t["r0"], t["angles"], t["kth"], t["th0"], t["dihedrals"], t["vn"],
                    t["mult"], t["gamma"], t["impropers"], t["ki"], t["igamma"])
    cfg = RunConfig(dt=0.1, T=300.0, Pe=0.0, nsteps=10, nlup=20, nc=1, nmol=s["nmol"])
    y = System.mm(ctx, cfg, s["pos"], s["vel"], s["mol_id"], topo, s["h"], crystal.npt_atom(300.0, 0.0, na))
    with pytest.raises(FmdError):
        y.set_physics(64)                      # unknown bit
    y.init()
    with pytest.raises(FmdError):
        y.set_physics(FMD_PHYS_MM_BONDED)      # after init
    y.close()
    a = crystal.atomistic(1, jitter=0.01, seed=2)
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=4, nlup=20, nc=1, nmol=a["nmol"])
    z = System.airebo(ctx, cfg, a["pos"], a["vel"], a["mass"], a["mol_id"], a["h"],
                      crystal.npt_atom(300.0, 0.0, a["pos"].size // 3))
    with pytest.raises(FmdError):
        z.set_physics(FMD_PHYS_MM_BONDED)      # not an MM system
    z.close()
