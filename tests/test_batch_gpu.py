"""Replica batches: uneven MM systems advanced together (one launch per step
phase, one CUDA graph per step) give each replica the trajectory it has when
run alone, across a list rebuild and the autotuner's launch shapes."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(1, 300.0, 0.0, 1), (2, 600.0, 1.0, 2), (1, 900.0, 3.0, 3), (2, 150.0, 0.5, 4)]


def _replicas(ctx):
    from fuller_md_en_b200 import mm_replica
    return [mm_replica(ctx, nc, T, P, seed=seed, jitter=0.01) for nc, T, P, seed in CASES]


@pytest.mark.parametrize("autotune", [True, False])
def test_batch_matches_single_systems(ctx, autotune):
    from fuller_md_en_b200 import Batch
    singles = _replicas(ctx)
    for s in singles:
        s.init()
    steps = 25                                   # crosses the rebuild at step 20
    ref = [[s.run(g, g) for g in range(1, steps + 1)] for s in singles]
    reps = _replicas(ctx)
    b = Batch(ctx, reps, autotune=autotune)
    t = b.tuning()
    assert t["blocks_lj"] >= len(reps) and t["blocks_atom"] >= len(reps)
    if autotune:
        assert t["lj_ms"] > 0 and t["bonded_ms"] > 0
    for g in range(1, steps + 1):
        obs = b.run(g, g)
        for r, o in enumerate(obs):
            q = ref[r][g - 1]
            assert o.step == q.step == g
            assert abs(o.T - q.T) <= 1e-9 * abs(q.T), (r, g, o.T, q.T)
            assert abs(o.P - q.P) <= 1e-9 * max(1.0, abs(q.P)), (r, g, o.P, q.P)
            for k in range(7):
                assert abs(o.E[k] - q.E[k]) <= 1e-9 * max(1e-6, abs(q.E[k])), (r, g, k, o.E[k], q.E[k])
    for s1, s2 in zip(singles, reps):
        d1, d2 = s1.download(), s2.download()
        assert np.max(np.abs(d1["pos"] - d2["pos"])) < 1e-9
        a1, a2 = s1.averages(), s2.averages()
        assert a1.n == a2.n and abs(a1.sT - a2.sT) <= 1e-9 * abs(a1.sT)
    assert b.step_kernels(True) > b.step_kernels(False)
    b.close()
    for s in singles + reps:
        s.close()


def test_batch_rejects_mixed_kinds(ctx):
    from fuller_md_en_b200 import Batch, FmdError, RunConfig, System, crystal
    reps = _replicas(ctx)[:1]
    s = crystal.atomistic(1, jitter=0.01, seed=5)
    na = s["pos"].size // 3
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=10, nlup=20, nc=1, nmol=s["nmol"])
    ai = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], crystal.npt_atom(300.0, 0.0, na))
    with pytest.raises(FmdError):
        Batch(ctx, reps + [ai])
    with pytest.raises(FmdError):
        Batch(ctx, reps + reps)
    ai.close()
    reps[0].close()


def _mm_system(ctx, nc, T, P, seed, shear=0.0):
    """An MM replica as mm_replica builds it, optionally with an off-diagonal
    cell entry (the molecule-wise list builder then rejects the cell and the
    cell-grid builder makes the lists)."""
    from fuller_md_en_b200 import RunConfig, System, Topology, crystal
    coords = crystal.c60_ih()
    bonds = crystal.bonds_from_geometry(coords)
    s = crystal.atomistic(nc, coords=coords, jitter=0.01, seed=seed, T=T, mol_base=0)
    na, nmol = s["pos"].size // 3, s["nmol"]
    t = crystal.mm_topology(coords, bonds, nmol)
    topo = Topology(t["bonds"], t["kb"], t["r0"], t["angles"], t["kth"], t["th0"], t["dihedrals"], t["vn"],
                    t["mult"], t["gamma"], t["impropers"], t["ki"], t["igamma"])
    h = s["h"].copy()
    h[1] += shear
    cfg = RunConfig(dt=0.1, T=T, Pe=P, nsteps=10 ** 6, nlup=20, gavg_from=1, gavg_to=10 ** 6, nc=nc, nmol=nmol)
    return System.mm(ctx, cfg, s["pos"], s["vel"], s["mol_id"], topo, h, crystal.npt_atom(T, P, na))


def test_batched_rebuild_with_fallback_replica(ctx):
    """The batch builds every replica's lists in one launch per phase; a
    replica whose molecule path is rejected (here a sheared cell) gets the
    cell-grid fallback from the conditional node of the rebuild graph.  Every
    replica's observables over a rebuild, and its lists after it, equal the
    same system's run alone."""
    from fuller_md_en_b200 import Batch
    cases = [(2, 300.0, 0.5, 11, 0.0), (2, 500.0, 2.0, 12, 0.8), (3, 700.0, 1.0, 13, 0.0)]
    singles = [_mm_system(ctx, *c) for c in cases]
    for s in singles:
        s.init()
    steps = 22
    ref = [[s.run(g, g) for g in range(1, steps + 1)] for s in singles]
    reps = [_mm_system(ctx, *c) for c in cases]
    b = Batch(ctx, reps, autotune=False)
    for g in range(1, steps + 1):
        obs = b.run(g, g)
        for r, o in enumerate(obs):
            q = ref[r][g - 1]
            assert abs(o.T - q.T) <= 1e-9 * abs(q.T), (r, g, o.T, q.T)
            for k in range(7):
                assert abs(o.E[k] - q.E[k]) <= 1e-9 * max(1e-6, abs(q.E[k])), (r, g, k, o.E[k], q.E[k])
    for s1, s2 in zip(singles, reps):
        c1, l1, _, _ = s1.lists(400)
        c2, l2, _, _ = s2.lists(400)
        assert np.array_equal(c1, c2)
        assert all(np.array_equal(l1[k * 400:k * 400 + c1[k]], l2[k * 400:k * 400 + c2[k]]) for k in range(len(c1)))
        f1, r1 = s1.lj_full_rows()
        f2, r2 = s2.lj_full_rows()
        assert np.array_equal(f1, f2)
        assert all(np.array_equal(r1[j, :f1[j]], r2[j, :f2[j]]) for j in range(len(f1)))
    b.close()
    for s in singles + reps:
        s.close()


def test_batched_rebuild_kernel_count(ctx):
    """With every replica on the molecule path, a rebuild step adds a fixed
    handful of launches however many replicas the batch holds."""
    from fuller_md_en_b200 import Batch
    for R in (4, 12):
        reps = [_mm_system(ctx, 1 + r % 2, 300.0 + 50 * r, 0.5, 100 + r) for r in range(R)]
        b = Batch(ctx, reps, autotune=False)
        plain, rebuild = b.step_kernels(False), b.step_kernels(True)
        assert rebuild - plain <= 12, (R, plain, rebuild)
        assert b.step_kernels(True, conditional=True) >= R     # the fallback body: per-replica kernels
        b.close()
        for s in reps:
            s.close()
