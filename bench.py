"""Headline benchmark: plain AIREBO NPT MD on B200, atom-steps/s.

Workload (one GPU): C60 FCC nc=5 -> 500 molecules / 30,000 flexible carbon
atoms (Ih C60 with 1.39/1.45 A bonds), seeded Gaussian jitter 0.01 A,
300 K, 0 GPa, dt 0.5 fs, REBO + intermolecular LJ, Nose-Hoover +
Parrinello-Rahman, neighbour lists rebuilt on the device every 20 steps.
A step is one full MD step (forces + integrator, plus the list rebuild on
every 20th step), replayed as a CUDA graph on the device-resident system.

`value`: atom-steps/s from CUDA events around each step on the launching
stream; the working set (~75 MB) fits in L2, so L2 is flushed (a 512 MB
write) between timed steps, outside the timed windows.
`e2e`: the same metric through the public C-ABI with host buffers: state
uploaded, system initialised, steps run in monitor-sized chunks with the
observables read back at each chunk end, final state downloaded -- all inside
the wall-clock window.
`--impl reference`: the reference's own CPU code (oracle/_ref, compiled from
the reference sources, OpenMP build with all host threads) on the same
workload, a bounded sample of its steps.

Multi-GPU (`--gpus N` under torchrun): independent replicas, one per GPU
(the path has no exchange step); max of per-rank times, value = total work.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NC = 5
JITTER = 0.01
DT = 0.5
T_K = 300.0
P_GPA = 0.0
NLUP = 20
SEED = 42
WORKLOAD = ("AIREBO (REBO + LJ) NPT, C60 FCC nc=5: 500 molecules / 30,000 flexible C atoms, "
            "jitter 0.01 A, 300 K, 0 GPa, dt 0.5 fs, lists rebuilt every 20 steps")
METRIC = "atom-steps/s on 1 B200: plain AIREBO (REBO + LJ) NPT step"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        j = json.loads(p.read_text())
        return float(j["hbm_gbs"]), "of measured"
    return 6650.0, "of fallback"


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("FMD_CLOCKS_LOG", f"/tmp/fmd_clocks_{os.getpid()}.csv"))

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_system(ctx, rank: int):
    from fuller_md_en_b200 import RunConfig, System, crystal
    s = crystal.atomistic(NC, jitter=JITTER, seed=SEED + rank, T=T_K)
    na = s["pos"].size // 3
    cfg = RunConfig(dt=DT, T=T_K, Pe=P_GPA, nsteps=10 ** 6, nlup=NLUP, gavg_from=1, gavg_to=10 ** 6, nc=NC,
                    nmol=s["nmol"], use_graphs=1)
    npt = crystal.npt_atom(T_K, P_GPA, na)
    return s, na, cfg, npt


def list_bytes(sysd, na):
    """Algorithmic bytes of one LJ gather launch: list entries read (outgoing
    + incoming, int32), the two count arrays, positions of the atoms and their
    partners (FP64 x3, each atom read once), F written, accumulator read and
    cleared."""
    ca, la, cb, lb = sysd.lists(400, 12)
    n_out = int(ca.sum())
    return 2 * (n_out * 4) + 2 * na * 4 + na * 24 + 3 * na * 24, n_out


def run_ours(args, ws, rank, local):
    import torch
    from fuller_md_en_b200 import Context, System
    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream())
    s, na, cfg, npt = make_system(ctx, rank)

    # ---------------- device-resident run (value) ----------------
    # The reference force field heats the crystal within ~100 steps and the
    # per-step cost grows with it, so the timed steps are global steps 1..K of
    # a fresh system (the same trajectory the reference arm times); the W
    # warm-up steps run on a throwaway copy.
    W, K = args.warmup, args.steps
    warm = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
    warm.init()
    warm.run(1, W)
    warm.close()
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
    sysd.init()                                # lists, first forces, graph capture
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ctx.synchronize()
    clocks = Clocks(local)
    clocks.start()
    t_wall0 = time.perf_counter()
    for k in range(K):
        with torch.cuda.stream(stream):
            flush.zero_()                      # L2 flush, outside the timed window
        ev[k][0].record(stream)
        sysd.enqueue(1 + k, 1 + k)
        ev[k][1].record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms_total = float(sum(step_ms))
    obs = sysd.run(K + 1, K + 1)               # one more step: observables sanity
    if not math.isfinite(obs.E[0]):
        raise RuntimeError("non-finite energy in the benchmark run")
    if ws > 1:
        t = torch.tensor([ms_total], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_total = float(t.item())
    value = ws * na * K / (ms_total / 1e3)

    # ---------------- roofline of the dominant kernel ----------------
    stages = {"lj_gather": sysd.kernel_ms(0, 20), "rebo": sysd.kernel_ms(1, 20),
              "list_rebuild": sysd.kernel_ms(2, 5)}
    per_step = {"lj_gather": stages["lj_gather"], "rebo": stages["rebo"],
                "list_rebuild": stages["list_rebuild"] / NLUP}
    lj_bytes, n_pairs_listed = list_bytes(sysd, na)
    peak, peak_src = peaks()
    achieved = lj_bytes / (stages["lj_gather"] / 1e3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("k_lj_gather_nc5")
    n_prod = sysd.step_kernels(False, False)
    n_reb = sysd.step_kernels(True, False)
    launches = sum(n_reb if (1 + k) % NLUP == 0 else n_prod for k in range(K))
    sysd.close()

    # ---------------- end to end through the public API ----------------
    e2e = None
    if rank == 0 or ws > 1:
        from fuller_md_en_b200 import System as Sys
        ctx.synchronize()
        prn = max(1, K // 50)                  # the reference's default monitor cadence (LJ:830)
        t0 = time.perf_counter()
        sys2 = Sys.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
        sys2.init()
        g = 1
        nread = 0
        while g <= K:
            last = min(K, g + prn - 1)
            sys2.run(g, last)
            nread += 1
            g = last + 1
        out = sys2.download()
        e2e_s = time.perf_counter() - t0
        sys2.close()
        h2d = s["pos"].nbytes + s["vel"].nbytes + s["mass"].nbytes + s["mol_id"].nbytes + 9 * 8 + 15 * 8
        d2h = nread * 104 + out["pos"].nbytes + out["vel"].nbytes + 9 * 8 + 15 * 8
        e2e = {"value": ws * na * K / e2e_s, "unit": "atom-steps/s",
               "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
               "note": "wall clock: state upload, init (lists + first forces), K steps in chunks of "
                       f"{prn} with observables read back per chunk, state download"}
    ctx.close()
    del flush
    res = {
        "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": ms_total / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "atoms_per_gpu": na, "global_atoms": na * ws,
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                   "l2": "flushed between timed steps (512 MB write outside the timed windows); "
                         "working set ~75 MB < 126 MB L2",
                   "step_graph": "one CUDA graph per step variant", "wall_s_timed_loop": t_wall},
        "roofline": {"bound": "hbm", "kernel": "k_lj_gather (atomistic LJ gather)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": lj_bytes, "listed_pairs": n_pairs_listed,
                     "launch_ms": stages["lj_gather"]},
        "stage_ms_per_step": per_step,
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
    }
    return res


def ref_sample(K: int, omp: bool = True):
    """Times the reference's own step_npt + list builders (oracle/_ref) on the
    same workload: K steps with the list rebuild at its natural cadence."""
    from fuller_md_en_b200 import crystal
    from oracle.fmd_oracle import Ref
    R = Ref(omp=omp)
    s = crystal.atomistic(NC, jitter=JITTER, seed=SEED, T=T_K)
    na = s["pos"].size // 3
    st = dict(pos=s["pos"].copy(), vel=s["vel"].copy(), h=s["h"].copy(), hi=crystal.inv9(s["h"]),
              mass=s["mass"], npt=crystal.npt_atom(T_K, P_GPA, na), F=np.zeros(3 * na), vir9=np.zeros(9))
    lists = R.ai_lists(st["pos"], st["h"], st["hi"], na, s["mol_id"])
    E, F, W = R.ai_forces(st["pos"], st["h"], st["hi"], *lists, na)
    st["F"], st["vir9"] = F, W
    t_rebuild = 0.0
    t_steps = 0.0
    for g in range(1, K + 1):
        if g % NLUP == 0:
            t0 = time.perf_counter()
            st["hi"] = crystal.inv9(st["h"])
            lists = R.ai_lists(st["pos"], st["h"], st["hi"], na, s["mol_id"])
            t_rebuild += time.perf_counter() - t0
        t0 = time.perf_counter()
        R.ai_step(st, DT, *lists)
        t_steps += time.perf_counter() - t0
    return na, t_steps, t_rebuild


def run_reference(args, ws, rank):
    """--impl reference: rank 0 times the reference's CPU path."""
    if rank != 0:
        return None
    from oracle.fmd_oracle import ref_available
    if not ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference sources)"}
    cores = os.cpu_count() or 1
    # bounded sample: warm-up capped at 2 steps; timed: global steps 1..min(K, 60)
    # of the same fresh trajectory the GPU arm times (lists rebuilt at 20, 40, 60)
    Kw = min(args.warmup, 2)
    if Kw:
        ref_sample(Kw)
    K = min(args.steps, 60)
    na, ts, tr = ref_sample(K)
    per_step = (ts + tr) / K
    val = na / per_step
    return {"impl": "reference", "metric": METRIC, "value": val, "unit": "atom-steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "atoms": na},
            "cpu_baseline": {"value": val, "unit": "atom-steps/s", "cores": cores, "kind": "reference",
                             "sample": f"global steps 1..{K} of {args.steps} from the same initial state (lists "
                                       f"rebuilt at steps divisible by 20), reference OpenMP build, {cores} threads;"
                                       f" step_npt {ts / K * 1e3:.1f} ms/step, list build {tr:.2f} s total"},
            "e2e": {"value": val, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def cpu_baseline():
    from oracle.fmd_oracle import ref_available
    if not ref_available():
        return None
    cores = os.cpu_count() or 1
    K = 20
    na, ts, tr = ref_sample(K, omp=True)
    val = na / ((ts + tr) / K)
    na, ts1, tr1 = ref_sample(4, omp=False)
    return {"value": val, "unit": "atom-steps/s", "cores": cores, "kind": "reference",
            "sample": f"{K} steps incl. one list rebuild, reference OpenMP build, {cores} threads "
                      f"(serial build: step_npt {ts1 / 4 * 1e3:.0f} ms/step)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_init()
    if args.impl == "reference":
        res = run_reference(args, ws, rank)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if ws > 1:
        import torch
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = run_ours(args, ws, rank, local)
    if rank == 0:
        if not args.no_cpu_baseline and ws == 1:
            res["cpu_baseline"] = cpu_baseline()
        print(json.dumps(res), flush=True)
    if ws > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
