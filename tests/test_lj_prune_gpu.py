"""Pruned LJ gather rows (ljprune.cu) against the full rows and the reference.

A pruning gather walks the full rows and keeps the entries within rc + delta;
later steps walk those rows until the motion since the prune could bring a
dropped entry inside the cutoff.  The pairs and pair terms are then those of
the full rows, summed in another lane order: energies, forces and virials
agree with an unpruned system to summation order, and trajectories with the
reference driver loop to the tolerances of test_gpu_system.py."""
from __future__ import annotations

import numpy as np
import pytest

import driver_loop as DL
from conftest import rel, rows, same_rows
from fuller_md_en_b200 import RunConfig, System, crystal, mm_replica

pytestmark = pytest.mark.gpu

RC_AI = 3.0 * 3.40 + 2.0


def _system(ctx, s, nc, delta, T=300.0, nlup=20, nsteps=10):
    na = s["pos"].size // 3
    cfg = RunConfig(dt=0.5, T=T, Pe=0.0, nsteps=nsteps, nlup=nlup, nc=nc, nmol=s["nmol"])
    y = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], crystal.npt_atom(T, 0.0, na))
    y.set_lj_prune(delta)
    y.init()
    return y


def _agree(a, b, what, tol=1e-9):
    for q in range(3):
        assert abs(a.E[q] - b.E[q]) <= tol * abs(b.E[q]), (what, q, a.E[q], b.E[q])
    assert abs(a.P - b.P) <= 1e-6, (what, a.P, b.P)
    assert abs(a.T - b.T) <= tol * max(1.0, abs(b.T)), (what, a.T, b.T)


@pytest.mark.parametrize("nc,jitter,seed,delta", [(3, 0.01, 1, 0.5), (5, 0.01, 4, 0.3), (4, 0.05, 5, 1.0)])
def test_pruned_run_matches_full_rows(ctx, nc, jitter, seed, delta):
    s = crystal.atomistic(nc, jitter=jitter, seed=seed)
    p = _system(ctx, s, nc, delta, nsteps=60)
    f = _system(ctx, s, nc, 0.0, nsteps=60)
    assert p.lj_prune() == {"delta": delta, "evaluations": 1, "prunes": 1}   # set-up prunes
    assert f.lj_prune()["delta"] == 0.0
    Fp, _, Ep = p.forces()
    Ff, _, Ef = f.forces()
    assert rel(Fp, Ff) < 1e-13 and abs(Ep[2] - Ef[2]) <= 1e-13 * abs(Ef[2])
    for g in range(1, 61):
        _agree(p.run(g, g), f.run(g, g), g)
    Fp, _, Ep = p.forces()
    Ff, _, Ef = f.forces()
    assert rel(Fp, Ff) < 1e-9
    Wp, _ = p.virial()
    Wf, _ = f.virial()
    assert rel(Wp, Wf) < 1e-9
    st = p.lj_prune()
    assert st["evaluations"] == 61
    assert 4 <= st["prunes"] < 61, st          # every build (g = 20, 40, 60) prunes; most steps do not
    p.close()
    f.close()


def test_pruned_system_matches_driver(ctx, oracle):
    """Schedule, rescales and two list rebuilds, pruned rows on most steps."""
    s = crystal.atomistic(3, jitter=0.01, seed=23)
    na = s["pos"].size // 3
    npt = crystal.npt_atom(300.0, 0.0, na)
    npt[13] = 4.0
    cold, warm, nsteps = 3, 4, 38
    total = cold + warm + nsteps
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, T_cold=4.0, coldstart=cold, warmup=warm, nsteps=nsteps, nlup=20,
                    gavg_from=cold + warm + 30, gavg_to=total, nc=3, nmol=s["nmol"])
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
    sysd.init()
    assert sysd.lj_prune()["delta"] > 0.0                  # on by default
    st = dict(pos=s["pos"].copy(), vel=s["vel"].copy(), h=s["h"].copy(), hi=crystal.inv9(s["h"]), mass=s["mass"],
              npt=npt.copy(), mol_id=s["mol_id"])
    cr, lr, _ = oracle.nlist_intra(st["pos"], st["h"], st["hi"], na, st["mol_id"])
    cl, ll, _ = oracle.nlist_half(st["pos"], st["h"], st["hi"], na, st["mol_id"], RC_AI)
    st["pos"] = oracle.apply_pbc(st["pos"], st["h"], st["hi"])
    E, F, W = oracle.airebo_forces(st["pos"], st["h"], st["hi"], cr, lr, cl, ll, na)
    st["F"], st["vir9"] = F, W
    ref, lists = DL.run_airebo(oracle, st, 1, total, 0.5, 300.0, 4.0, cold, warm, nlup=20, nc=3,
                               lists=(cr, lr, cl, ll))
    for g in range(1, total + 1):
        o = sysd.run(g, g)
        r = ref[g - 1]
        assert abs(o.T - r[1]) <= 1e-8 * max(1.0, abs(r[1])), (g, o.T, r[1])
        assert abs(o.P - r[2]) <= 1e-6, (g, o.P, r[2])
        for k in range(3):
            assert abs(o.E[k] - r[4 + k]) <= 1e-8 * abs(r[4 + k]), (g, k, o.E[k], r[4 + k])
    stp = sysd.lj_prune()
    assert stp["prunes"] < stp["evaluations"] // 2, stp
    ca, la, _, _ = sysd.lists(400, 12)
    assert same_rows(rows(ca, la, 400), rows(lists[2], lists[3], 400))
    sysd.close()


def test_motion_triggers_reprune(ctx):
    """No list rebuilds and hot atoms: the displacement bound, not the build,
    triggers the prunes, and the run still matches the full rows (which the
    reference walks every step, stale or not)."""
    s = crystal.atomistic(3, jitter=0.01, seed=41, T=3000.0)
    p = _system(ctx, s, 3, 0.3, T=3000.0, nlup=100000, nsteps=200)
    f = _system(ctx, s, 3, 0.0, T=3000.0, nlup=100000, nsteps=200)
    for g in range(1, 201):
        _agree(p.run(g, g), f.run(g, g), g, tol=1e-8)
    st = p.lj_prune()
    assert st["evaluations"] == 201 and 3 <= st["prunes"] < 200, st
    p.close()
    f.close()


def test_buffers_agree(ctx):
    """Small, default and large buffers prune at different steps and agree."""
    s = crystal.atomistic(4, jitter=0.02, seed=12)
    outs = []
    counts = []
    for delta in (0.1, 0.5, 2.0):
        y = _system(ctx, s, 4, delta, nsteps=40)
        y.run(1, 40)
        outs.append((y.download()["pos"], y.forces()[2]))
        counts.append(y.lj_prune()["prunes"])
        y.close()
    assert counts[0] > counts[1] >= counts[2] >= 3, counts
    for pos, E in outs[1:]:
        assert np.max(np.abs(pos - outs[0][0])) < 1e-9
        assert abs(E[2] - outs[0][1][2]) <= 1e-10 * abs(E[2])


def test_mm_pruned_matches_full_rows(ctx):
    p = mm_replica(ctx, 3, 600.0, 1.0, seed=9, jitter=0.02, nsteps=50)
    f = mm_replica(ctx, 3, 600.0, 1.0, seed=9, jitter=0.02, nsteps=50)
    f.set_lj_prune(0.0)
    p.init()
    f.init()
    for g in range(1, 51):
        o, q = p.run(g, g), f.run(g, g)
        for k in range(7):
            assert abs(o.E[k] - q.E[k]) <= 1e-9 * max(1e-3, abs(q.E[k])), (g, k, o.E[k], q.E[k])
    st = p.lj_prune()
    assert st["evaluations"] == 51 and 3 <= st["prunes"] < 51, st
    p.close()
    f.close()


def test_fp32_pair_pruned_matches_full_rows(ctx):
    """FP32 pair algebra over pruned rows: the same pairs and FP32 pair terms
    as over the full rows (the cutoff test and the image stay FP64)."""
    from fuller_md_en_b200._lib import FMD_PREC_FP32_PAIR
    s = crystal.atomistic(3, jitter=0.02, seed=19)
    na = s["pos"].size // 3
    ys = []
    for delta in (0.5, 0.0):
        cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=40, nlup=20, nc=3, nmol=s["nmol"],
                        precision=FMD_PREC_FP32_PAIR)
        y = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"],
                          crystal.npt_atom(300.0, 0.0, na))
        y.set_lj_prune(delta)
        y.init()
        ys.append(y)
    for g in range(1, 41):
        _agree(ys[0].run(g, g), ys[1].run(g, g), g)
    st = ys[0].lj_prune()
    assert st["evaluations"] == 41 and 3 <= st["prunes"] < 41, st
    for y in ys:
        y.close()


def test_prune_off_and_bad_delta(ctx):
    from fuller_md_en_b200._lib import FmdError
    s = crystal.atomistic(2, jitter=0.01, seed=3)
    y = _system(ctx, s, 2, 0.0)
    assert y.lj_prune() == {"delta": 0.0, "evaluations": 0, "prunes": 0}
    with pytest.raises(FmdError):
        y.set_lj_prune(-1.0)
    y.set_lj_prune(0.7)                       # switching on after init recaptures and prunes next
    y.run(1, 5)
    st = y.lj_prune()
    assert st["delta"] == 0.7 and st["prunes"] >= 1 and st["evaluations"] == 5
    y.close()
