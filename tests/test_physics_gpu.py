"""Opt-in physics corrections (fmd_system_set_physics).  They have no
reference counterpart, so they are checked against the mathematics: with
FMD_PHYS_MM_BONDED every MM force, with FMD_PHYS_REBO every AIREBO force, is
-grad E of the system's own energy, measured by central differences.  Without
the flags the systems keep the reference's forces (MM bond and angle forces
+grad E, MM:389-398, MM:468-491; torsion and REBO three-body forces that are
not gradients), which the same check rejects."""
from __future__ import annotations

import numpy as np
import pytest

from fuller_md_en_b200 import RunConfig, System, Topology, crystal
from fuller_md_en_b200._lib import FMD_PHYS_MM_BONDED, FMD_PHYS_REBO, FmdError

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


def _airebo(ctx, s, pos, physics):
    na = pos.size // 3
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=4, nlup=20, nc=1, nmol=s["nmol"])
    y = System.airebo(ctx, cfg, pos, s["vel"], s["mass"], s["mol_id"], s["h"], crystal.npt_atom(300.0, 0.0, na))
    if physics:
        y.set_physics(physics)
    y.init()
    F, _, E = y.forces()
    y.close()
    return F, E[0]


def _airebo_fd(ctx, s, physics, comps):
    F, E = _airebo(ctx, s, s["pos"], physics)
    err = 0.0
    for k in comps:
        p, m = s["pos"].copy(), s["pos"].copy()
        p[k] += DELTA
        m[k] -= DELTA
        g = (_airebo(ctx, s, p, physics)[1] - _airebo(ctx, s, m, physics)[1]) / (2 * DELTA)
        err = max(err, abs(F[k] + g))
    return err, float(np.max(np.abs(F))), E


@pytest.mark.parametrize("scale,seed", [(1.0, 11), (0.65, 77), (0.7, 5)])
def test_rebo_physical_forces_are_minus_grad_energy(ctx, scale, seed):
    """AIREBO (REBO + LJ) with FMD_PHYS_REBO; scales 0.65 and 0.7 crowd the
    REBO rows past their 12 entries (asymmetric rows: bond orders from a row
    that lacks the bond's other atom)."""
    s = crystal.atomistic(1, coords=crystal.c60_ih() * scale, jitter=0.05, seed=seed)
    comps = np.random.default_rng(seed).choice(s["pos"].size, 12, replace=False)
    err, fmax, E = _airebo_fd(ctx, s, FMD_PHYS_REBO, comps)
    assert err <= 1e-6 * fmax + 1e-7, (err, fmax)
    _, E0 = _airebo(ctx, s, s["pos"], 0)
    assert abs(E - E0) <= 1e-12 * abs(E0)             # the energy is the reference's
    if scale == 1.0:
        err0, fmax0, _ = _airebo_fd(ctx, s, 0, comps)
        assert err0 > 1e-2 * fmax0, (err0, fmax0)      # the reference's three-body forces are not


def _qmul(a, b):
    return np.array([a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
                     a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
                     a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
                     a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]])


def _free_tops(ctx, physics, steps=100):
    """Rigid C60s 42 A apart (beyond the site cutoff): no forces or torques,
    so each is a free spherical top whose lab-frame angular velocity keeps
    its direction (the thermostat only scales it).  Returns, per molecule,
    the sine of the angle between the lab-frame rotation axis of
    q(t) q(0)^-1 and w."""
    from fuller_md_en_b200._lib import FMD_PHYS_QUAT  # noqa: F401
    s = crystal.rigid(1, seed=21, a0=60.0)
    n = s["n"]
    rmcut = 3.0 * 3.431 + 2 * s["Rmol"] + 1.0
    cfg = RunConfig(dt=1.0, T=300.0, Pe=0.0, nsteps=steps, nlup=25, nc=1, nmol=n)
    y = System.rigid(ctx, cfg, 60, s["body"], s["I0"], s["Mmol"], rmcut, s["pos"], s["vel"], s["qv"], s["omg"],
                     s["h"], crystal.npt_rigid(300.0, 0.0, n))
    if physics:
        y.set_physics(physics)
    y.init()
    y.run(1, steps)
    out = y.download()
    y.close()
    q0 = s["qv"].reshape(n, 4)
    q1, w = out["qv"].reshape(n, 4), out["omg"].reshape(n, 3)
    sines = []
    for a in range(n):
        d = _qmul(q1[a], q0[a] * np.array([1.0, -1.0, -1.0, -1.0]))
        v = d[1:] * np.sign(d[0])
        assert np.linalg.norm(v) > 1e-3                     # it did rotate
        sines.append(np.linalg.norm(np.cross(v / np.linalg.norm(v), w[a] / np.linalg.norm(w[a]))))
    return np.array(sines)


def test_quaternion_left_update_rotates_about_the_lab_axis(ctx):
    from fuller_md_en_b200._lib import FMD_PHYS_QUAT
    assert np.max(_free_tops(ctx, FMD_PHYS_QUAT)) < 1e-9
    assert np.min(_free_tops(ctx, 0)) > 1e-2                # the reference's right update does not
