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
