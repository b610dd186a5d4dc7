"""One force stage of the benchmark workload, launched for a profiler.

    FMD_LJ_SHAPE=256,4,2 python -m fuller_md_en_b200.probe --stage lj_pruned

builds the benchmark system (C60 FCC nc=5, 30,000 atoms, jitter 0.01 A,
300 K, 0 GPa, dt 0.5 fs, lists every 20 steps), runs --steps steps and times
--reps launches of the stage with CUDA events (System.kernel_ms: one
untimed launch first, then the timed ones, then the current forces are
recomputed).  FMD_LJ_SHAPE pins the LJ gather's launch shape (threads,
entries per lane, row feed) so the launch sequence does not depend on the
autotuner: with --steps 0 and --reps 1, the LJ gather launches are set-up's
(one, pruning the full rows), the untimed and the timed launch of the stage,
then the recomputation's; a profiler capturing the gather's launch 3 sees
the timed, warm launch on the benchmark state.  For --stage rebo the REBO
kernels launch twice per force evaluation (geometry + bond order, forces):
set-up, one per step, then the untimed and the timed evaluation.
Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json

STAGES = {"lj_full": 0, "rebo": 1, "rebuild": 2, "forces": 3, "lj_pruned": 4}


def main() -> None:
    from . import Context, RunConfig, System, crystal
    ap = argparse.ArgumentParser()
    ap.add_argument("--stage", choices=sorted(STAGES), default="lj_pruned")
    ap.add_argument("--nc", type=int, default=5)
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--delta", type=float, default=0.5, help="pruned-row buffer (A)")
    args = ap.parse_args()
    ctx = Context(0)
    s = crystal.atomistic(args.nc, jitter=0.01, seed=42, T=300.0)
    na = s["pos"].size // 3
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=10 ** 6, nlup=20, nc=args.nc, nmol=s["nmol"])
    y = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], crystal.npt_atom(300.0, 0.0, na))
    y.set_lj_prune(args.delta)
    y.init()
    if args.steps > 0:
        y.run(1, args.steps)
    ms = y.kernel_ms(STAGES[args.stage], args.reps)
    full, pruned = y.lj_rows()
    print(json.dumps({"stage": args.stage, "ms_per_launch": ms, "atoms": na, "steps": args.steps,
                      "shape": y.lj_shape(), "full_row_entries": int(full.sum()),
                      "pruned_row_entries": int(pruned.sum()), "prune": y.lj_prune()}))
    y.close()
    ctx.close()


if __name__ == "__main__":
    main()
