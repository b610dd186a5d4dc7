"""Device-resident systems (lists rebuilt on the device, steps replayed as
CUDA graphs, schedule/rescale/averages on the device) against the reference
driver loop restated over the CPU oracle (tests/driver_loop.py).

Trajectories are chaotic, so runs are short (tens of steps, two list
rebuilds); energies must agree to 1e-8 relative, temperatures to 1e-8,
pressures to 1e-6 GPa absolute (pressure is a small difference of large
terms near 0 GPa), and the neighbour lists at the last rebuild bit for bit."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import driver_loop as DL
from conftest import rows, same_rows
from fuller_md_en_b200 import RunConfig, System, Topology, crystal

pytestmark = pytest.mark.gpu


def _airebo_case(nc=2, jitter=0.01, seed=21):
    s = crystal.atomistic(nc, jitter=jitter, seed=seed)
    na = s["pos"].size // 3
    npt = crystal.npt_atom(300.0, 0.0, na)
    return s, na, npt


def _oracle_init_airebo(O, s, na, npt):
    st = dict(pos=s["pos"].copy(), vel=s["vel"].copy(), h=s["h"].copy(), hi=crystal.inv9(s["h"]), mass=s["mass"],
              npt=npt.copy(), mol_id=s["mol_id"])
    cr, lr, _ = O.nlist_intra(st["pos"], st["h"], st["hi"], na, st["mol_id"])
    cl, ll, _ = O.nlist_half(st["pos"], st["h"], st["hi"], na, st["mol_id"], 3.0 * 3.40 + 2.0)
    st["pos"] = O.apply_pbc(st["pos"], st["h"], st["hi"])
    E, F, W = O.airebo_forces(st["pos"], st["h"], st["hi"], cr, lr, cl, ll, na)
    st["F"], st["vir9"] = F, W
    return st, (cr, lr, cl, ll)


@pytest.mark.parametrize("graphs", [0, 1])
def test_airebo_system_matches_driver(ctx, oracle, graphs):
    s, na, npt = _airebo_case()
    cold, warm, nsteps = 3, 4, 38
    total = cold + warm + nsteps
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, T_cold=4.0, coldstart=cold, warmup=warm, nsteps=nsteps, nlup=20,
                    gavg_from=cold + warm + 30, gavg_to=total, nc=2, nmol=s["nmol"], use_graphs=graphs)
    npt4 = npt.copy()
    npt4[13] = 4.0
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt4)
    sysd.init()
    st, lists = _oracle_init_airebo(oracle, s, na, npt4)
    ref, lists = DL.run_airebo(oracle, st, 1, total, 0.5, 300.0, 4.0, cold, warm, nlup=20, nc=2, lists=lists)
    for g in range(1, total + 1):
        o = sysd.run(g, g)
        r = ref[g - 1]
        assert o.step == g
        assert abs(o.T - r[1]) <= 1e-8 * max(1.0, abs(r[1])), (g, o.T, r[1])
        assert abs(o.P - r[2]) <= 1e-6, (g, o.P, r[2])
        assert abs(o.a - r[3]) <= 1e-12 * r[3]
        for k in range(3):
            assert abs(o.E[k] - r[4 + k]) <= 1e-8 * abs(r[4 + k]), (g, k, o.E[k], r[4 + k])
    avg = sysd.averages()
    win = [r for r in ref if cfg.gavg_from <= r[0] <= cfg.gavg_to]
    assert avg.n == len(win)
    assert abs(avg.sT / avg.n - np.mean([r[1] for r in win])) < 1e-8 * 300
    assert abs(avg.sE[2] / avg.n - np.mean([r[4] for r in win]) / s["nmol"]) < 1e-8 * 100
    # lists of the last rebuild (g = 40) bit-exact with the oracle's
    ca, la, cb, lb = sysd.lists(400, 12)
    assert same_rows(rows(ca, la, 400), rows(lists[2], lists[3], 400))
    assert same_rows(rows(cb, lb, 12), rows(lists[0], lists[1], 12))
    out = sysd.download()
    assert np.allclose(out["h"], st["h"], rtol=1e-12, atol=0)
    sysd.close()


def test_rigid_system_matches_driver(ctx, oracle):
    s = crystal.rigid(3, seed=8)
    n = s["n"]
    rmcut = 3.0 * 3.431 + 2 * s["Rmol"] + 1.0
    cold, warm, nsteps = 2, 3, 27
    total = cold + warm + nsteps
    npt = crystal.npt_rigid(300.0, 1.0, n)
    npt[13] = 4.0
    cfg = RunConfig(dt=1.0, T=300.0, Pe=1.0, T_cold=4.0, coldstart=cold, warmup=warm, nsteps=nsteps, nlup=25,
                    gavg_from=cold + warm + 20, gavg_to=total, nc=3, nmol=n)
    sysd = System.rigid(ctx, cfg, 60, s["body"], s["I0"], s["Mmol"], rmcut, s["pos"], s["vel"], s["qv"], s["omg"],
                        s["h"], npt)
    sysd.init()
    st = dict(pos=s["pos"].copy(), vel=s["vel"].copy(), qv=s["qv"].copy(), omg=s["omg"].copy(), h=s["h"].copy(),
              hi=crystal.inv9(s["h"]), npt=npt.copy())
    c, l, _ = oracle.nlist_sym(st["pos"], st["h"], st["hi"], n, rmcut)
    st["pos"] = oracle.apply_pbc(st["pos"], st["h"], st["hi"])
    e, F, T, W = oracle.rigid_forces(st["pos"], st["qv"], s["body"], st["h"], st["hi"], c, l, n, 60, rmcut * rmcut)
    st.update(F=F, T=T, W9=W)
    ref, lists = DL.run_rigid(oracle, st, 1, total, 1.0, 300.0, 4.0, cold, warm, s["body"], s["I0"], s["Mmol"], 60,
                              rmcut, nlup=25, nc=3, lists=(c, l))
    for g in range(1, total + 1):
        o = sysd.run(g, g)
        r = ref[g - 1]
        assert abs(o.T - r[1]) <= 1e-8 * max(1.0, abs(r[1])), (g, o.T, r[1])
        assert abs(o.P - r[2]) <= 1e-6, (g, o.P, r[2])
        assert abs(o.E[0] - r[4]) <= 1e-8 * abs(r[4]), (g, o.E[0], r[4])
    ca, la, _, _ = sysd.lists(80)
    assert same_rows(rows(ca, la, 80), rows(lists[0], lists[1], 80))
    out = sysd.download()
    q = out["qv"].reshape(-1, 4)
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-14)
    sysd.close()


def test_mm_system_matches_driver(ctx, oracle):
    coords = crystal.c60_ih()
    bonds = crystal.bonds_from_geometry(coords)
    s = crystal.atomistic(1, coords=coords, jitter=0.02, seed=31, mol_base=0)
    na, nmol = s["pos"].size // 3, s["nmol"]
    mol = oracle.mm_topology_mol(coords, bonds)
    kc = 1.0 / 23.06054783
    rep = lambda a, k: np.concatenate([a + m * 60 for m in range(nmol)]) if k else np.concatenate([a] * nmol)
    t = {"bonds": rep(mol["bonds"], 1), "kb": np.full(90 * nmol, 469.0 * kc), "r0": rep(mol["r0"], 0),
         "angles": rep(mol["angles"], 1), "kth": np.full(180 * nmol, 63.0 * kc), "th0": rep(mol["th0"], 0),
         "dihedrals": rep(mol["dihedrals"], 1), "vn": np.full(360 * nmol, 14.5 * kc),
         "mult": np.full(360 * nmol, 2, np.int32), "gamma": rep(mol["gamma"], 0),
         "impropers": rep(mol["impropers"], 1), "ki": np.full(60 * nmol, 15.0 * kc), "igamma": rep(mol["igamma"], 0),
         "mol_id": s["mol_id"]}
    topo = Topology(t["bonds"], t["kb"], t["r0"], t["angles"], t["kth"], t["th0"], t["dihedrals"], t["vn"],
                    t["mult"], t["gamma"], t["impropers"], t["ki"], t["igamma"])
    total = 24
    npt = crystal.npt_atom(300.0, 0.0, na)
    cfg = RunConfig(dt=0.1, T=300.0, Pe=0.0, nsteps=total, nlup=20, gavg_from=19, gavg_to=total, nc=1, nmol=nmol)
    sysd = System.mm(ctx, cfg, s["pos"], s["vel"], s["mol_id"], topo, s["h"], npt)
    sysd.init()
    st = dict(pos=s["pos"].copy(), vel=s["vel"].copy(), h=s["h"].copy(), hi=crystal.inv9(s["h"]), npt=npt.copy())
    c, l, _ = oracle.nlist_half(st["pos"], st["h"], st["hi"], na, t["mol_id"], 3.0 * 3.431 + 2.0)
    st["pos"] = oracle.apply_pbc(st["pos"], st["h"], st["hi"])
    E, F, W = oracle.mm_forces(t, st["pos"], st["h"], st["hi"], c, l, na)
    st.update(F=F, vir9=W)
    ref, _ = DL.run_mm(oracle, st, 1, total, 0.1, 300.0, 4.0, 0, 0, t, nlup=20, nc=1, lists=(c, l))
    for g in range(1, total + 1):
        o = sysd.run(g, g)
        r = ref[g - 1]
        assert abs(o.T - r[1]) <= 1e-8 * max(1.0, abs(r[1])), (g, o.T, r[1])
        for k in range(7):
            assert abs(o.E[k] - r[4 + k]) <= 1e-8 * max(1e-6, abs(r[4 + k])), (g, k, o.E[k], r[4 + k])
    sysd.close()


def test_run_before_init_is_an_error(ctx):
    from fuller_md_en_b200 import FmdError
    s, na, npt = _airebo_case(nc=1)
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=5, nlup=20, nc=1, nmol=s["nmol"])
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
    with pytest.raises(FmdError):
        sysd.run(1, 1)
    sysd.close()


@pytest.mark.parametrize("nc", [1, 3])
def test_mm_replicated_topology_is_the_full_topology(ctx, nc):
    """An MM system built from one molecule's topology replicated on the
    device (fmd_system_create_mm_replicated) is the system built from the
    full flat topology (build_flat_topology, MM:254-334): the same forces
    and energies at set-up and the same observables over steps that include
    a list rebuild (to 1e-9: the bonded forces are scattered with FP64
    atomics, whose order varies from run to run at the 1e-16 level)."""
    from fuller_md_en_b200 import RunConfig, System, Topology, crystal
    coords = crystal.c60_ih()
    bonds = crystal.bonds_from_geometry(coords)
    s = crystal.atomistic(nc, coords=coords, jitter=0.02, seed=17, T=400.0, mol_base=0)
    na, nmol = s["pos"].size // 3, s["nmol"]

    def topo(t):
        return Topology(t["bonds"], t["kb"], t["r0"], t["angles"], t["kth"], t["th0"], t["dihedrals"], t["vn"],
                        t["mult"], t["gamma"], t["impropers"], t["ki"], t["igamma"])

    cfg = RunConfig(dt=0.1, T=400.0, Pe=0.5, nsteps=100, nlup=20, nc=nc, nmol=nmol)
    npt = crystal.npt_atom(400.0, 0.5, na)
    full = System.mm(ctx, cfg, s["pos"], s["vel"], s["mol_id"], topo(crystal.mm_topology(coords, bonds, nmol)),
                     s["h"], npt)
    rep = System.mm_replicated(ctx, cfg, nmol, na // nmol, s["pos"], s["vel"],
                               topo(crystal.mm_topology(coords, bonds, 1)), s["h"], npt)
    full.init()
    rep.init()
    Fa, _, Ea = full.forces()
    Fb, _, Eb = rep.forces()
    assert np.max(np.abs(Fa - Fb)) <= 1e-12 * np.max(np.abs(Fa))
    assert np.max(np.abs(Ea - Eb)) <= 1e-12 * np.max(np.abs(Ea))
    for g in range(1, 23):
        a, b = full.run(g, g), rep.run(g, g)
        assert abs(a.T - b.T) <= 1e-9 * abs(a.T) and abs(a.P - b.P) <= 1e-9 * max(1.0, abs(a.P)), g
        for k in range(7):
            assert abs(a.E[k] - b.E[k]) <= 1e-9 * max(1e-6, abs(a.E[k])), (g, k)
    da, db = full.download(), rep.download()
    assert np.max(np.abs(da["pos"] - db["pos"])) < 1e-9
    full.close()
    rep.close()


def test_rigid_site_pair_count(ctx):
    """fmd_system_site_pairs: the site pairs within the cutoff (each molecule
    pair once) of a rigid system, against a count from the state on the host."""
    s = crystal.rigid(2, seed=3)
    n = s["n"]
    rmcut = 3.0 * 3.431 + 2 * s["Rmol"] + 1.0
    cfg = RunConfig(dt=1.0, T=300.0, Pe=0.0, nsteps=100, nlup=25, nc=2, nmol=n)
    sysd = System.rigid(ctx, cfg, 60, s["body"], s["I0"], s["Mmol"], rmcut, s["pos"], s["vel"], s["qv"], s["omg"],
                        s["h"], crystal.npt_rigid(300.0, 0.0, n))
    sysd.init()
    got = sysd.site_pairs()
    st = sysd.download()
    c, l, _, _ = sysd.lists(80)
    pos, qv, h = st["pos"].reshape(-1, 3), st["qv"].reshape(-1, 4), st["h"].reshape(3, 3)
    L = np.diag(h)
    body = np.asarray(s["body"]).reshape(-1, 3)

    def rot(q):
        w, x, y, z = q
        return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                         [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                         [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])

    lab = np.stack([body @ rot(q).T for q in qv])
    rc2 = (3.0 * 3.431) ** 2
    want = 0
    for i in range(n):
        for j in l[i * 80:i * 80 + c[i]]:
            if j <= i:
                continue
            m = pos[j] - pos[i]
            m -= L * np.round(m / L)
            if m @ m > rmcut * rmcut:
                continue
            d = m[None, None, :] + lab[j][None, :, :] - lab[i][:, None, :]
            want += int(np.count_nonzero((d * d).sum(axis=2) < rc2))
    assert got == want and got > 0
    sysd.close()


def test_pipelined_observables_match_synchronous_runs(ctx):
    """fmd_system_enqueue_obs / _wait_obs: each step's observables copied
    behind its step and read while the next step runs are those that
    fmd_system_run returns step by step."""
    from fuller_md_en_b200._lib import Obs
    s = crystal.atomistic(2, jitter=0.02, seed=5, T=300.0)
    na = s["pos"].size // 3

    def make():
        cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=100, nlup=5, nc=2, nmol=s["nmol"], use_graphs=1)
        y = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"],
                          crystal.npt_atom(300.0, 0.0, na))
        y.init()
        return y

    a, b = make(), make()
    try:
        ref = [a.run(g, g) for g in range(1, 13)]
        bufs = [Obs(), Obs()]
        got, prev = [], None
        for g in range(1, 13):
            b.enqueue_obs(g, g, ctypes.addressof(bufs[g & 1]))
            if prev is not None:
                b.wait_obs(prev)
                o = bufs[prev & 1]
                got.append((o.step, o.T, o.P, o.KE))
            prev = g
        b.wait_obs(prev)
        o = bufs[prev & 1]
        got.append((o.step, o.T, o.P, o.KE))
        for r, (st, T, P, KE) in zip(ref, got):
            assert st == r.step
            for x, y in ((T, r.T), (P, r.P), (KE, r.KE)):
                assert abs(x - y) <= 1e-9 * max(1.0, abs(y)), (st, x, y)
    finally:
        a.close()
        b.close()
