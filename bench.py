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
uploaded, system initialised, steps run in monitor-sized chunks with each
chunk's observables copied back (asynchronously, behind the chunk's steps)
and read on the host while the next chunk runs, final state downloaded -- all
inside the wall-clock window.
`surrogate`: the same workload with the learned REBO term in the step
(fuller_md_en_b200.surrogate): a model is trained here, on the GPU, on 2,000
snapshots of the plain kernel's own nc=5 trajectories (40 runs x 50 steps at
300-1500 K, 0-5 GPa), then the timed steps run with it, judged by the plain
REBO kernel every 100 steps (takeover above 25 meV/A force RMSE).  Force
RMSE is against the plain FP64 REBO kernel, which matches the reference's
compute_rebo to 1e-10 (GPU parity tests).
`--impl reference`: the reference's own CPU code (oracle/_ref, compiled from
the reference sources) on the same workload, a bounded sample of its steps,
serial and OpenMP builds (all host threads); the faster of the two is the
value.

Multi-GPU (`--gpus N` under torchrun): independent replicas, one per GPU
(the path has no exchange step); max of per-rank times, value = total work.
"""
from __future__ import annotations

import argparse
import ctypes
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
METRIC = "atom-steps/s on 1 B200: plain AIREBO vs learned surrogate, force RMSE vs FP64"


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


def make_system(ctx, rank: int, precision=None):
    """The workload; the reference's FP64 pair arithmetic unless `precision`
    says otherwise."""
    from fuller_md_en_b200 import RunConfig, System, crystal
    from fuller_md_en_b200._lib import FMD_PREC_FP64
    from fuller_md_en_b200.replicas import replica_seed
    s = crystal.atomistic(NC, jitter=JITTER, seed=replica_seed(SEED, rank), T=T_K)
    na = s["pos"].size // 3
    cfg = RunConfig(dt=DT, T=T_K, Pe=P_GPA, nsteps=10 ** 6, nlup=NLUP, gavg_from=1, gavg_to=10 ** 6, nc=NC,
                    nmol=s["nmol"], use_graphs=1,
                    precision=FMD_PREC_FP64 if precision is None else precision)
    npt = crystal.npt_atom(T_K, P_GPA, na)
    return s, na, cfg, npt


def list_bytes(sysd, na):
    """Algorithmic bytes of one LJ gather launch over the full rows and over
    the pruned rows of the last prune: row entries read (int32), the row
    lengths, positions of the atoms and their partners (FP64 x3, each atom
    read once), F written, accumulator read and cleared."""
    full, pruned = sysd.lj_rows()
    fixed = na * 4 + na * 24 + 3 * na * 24
    return (int(full.sum()) * 4 + fixed, int(pruned.sum()) * 4 + fixed, int(full.sum()), int(pruned.sum()))


def timed_steps(ctx, stream, sysd, K, flush):
    """CUDA-event time (ms) of global steps 1..K of an initialised system,
    L2 flushed before each step outside its window."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    torch.cuda.synchronize()
    ctx.synchronize()
    for k in range(K):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev[k][0].record(stream)
        sysd.enqueue(1 + k, 1 + k)
        ev[k][1].record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


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
    from fuller_md_en_b200.replicas import job_throughput, max_over_ranks
    ms_total = max_over_ranks(ms_total, device=f"cuda:{local}")
    value = job_throughput(na, K, ms_total, ws)

    # ---------------- roofline of the dominant kernel ----------------
    # The LJ gather over the pruned rows runs on most steps (the full-row
    # gather only when the rows are pruned again), so it is the kernel whose
    # roofline is reported.
    stages = {"lj_gather_pruned": sysd.kernel_ms(4, 20), "lj_gather_full": sysd.kernel_ms(0, 20),
              "rebo": sysd.kernel_ms(1, 20), "list_rebuild": sysd.kernel_ms(2, 5)}
    prune = sysd.lj_prune()
    per_step = {"lj_gather_pruned": stages["lj_gather_pruned"], "lj_gather_full": stages["lj_gather_full"],
                "lj_prune_fraction": prune["prunes"] / max(1, prune["evaluations"]), "rebo": stages["rebo"],
                "list_rebuild": stages["list_rebuild"] / NLUP}
    full_bytes, lj_bytes, n_full, n_pruned = list_bytes(sysd, na)
    lj_shape = {"full_rows": sysd.lj_shape(), "pruned_rows": sysd.lj_shape_pruned()}
    peak, peak_src = peaks()
    achieved = lj_bytes / (stages["lj_gather_pruned"] / 1e3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("k_lj_gather_pruned_nc5")
    composite = composite_roofline(sysd, na, ms_total / K, stages, per_step, peak, peak_src, clk)
    n_prod = sysd.step_kernels(False, False)
    n_reb = sysd.step_kernels(True, False)
    launches = sum(n_reb if (1 + k) % NLUP == 0 else n_prod for k in range(K))
    sysd.close()

    # ---------------- end to end through the public API ----------------
    # Measured before the legs that run the reference's OpenMP build on the
    # host: its worker threads keep spinning on every core for a while after
    # each parallel region and would slow this wall-clock window's host side.
    e2e = None
    if rank == 0 or ws > 1:
        from fuller_md_en_b200 import System as Sys
        ctx.synchronize()
        prn = max(1, K // 50)                  # the reference's default monitor cadence (LJ:830)

        def pinned(a):
            t = torch.empty(a.size, dtype=torch.float64 if a.dtype == np.float64 else torch.int32, pin_memory=True)
            v = t.numpy()
            v[:] = a.ravel()
            return t, v

        # inputs and the state's destination in pinned host memory, allocated
        # before the window (the arrays a caller keeps between runs)
        keep = [pinned(s[k]) for k in ("pos", "vel", "mass", "mol_id", "h")]
        hp = {k: v for k, (_, v) in zip(("pos", "vel", "mass", "mol_id", "h"), keep)}
        dst = {k: pinned(np.zeros(n))[1] for k, n in (("pos", 3 * na), ("vel", 3 * na), ("h", 9))}
        # two page-locked observable records: each chunk's copy is enqueued
        # behind its steps and read on the host while the next chunk runs
        from fuller_md_en_b200._lib import Obs
        obs_buf = torch.empty(2 * ctypes.sizeof(Obs), dtype=torch.uint8, pin_memory=True)
        obs_addr = [obs_buf.data_ptr(), obs_buf.data_ptr() + ctypes.sizeof(Obs)]
        seen = []
        t0 = time.perf_counter()
        sys2 = Sys.airebo(ctx, cfg, hp["pos"], hp["vel"], hp["mass"], hp["mol_id"], hp["h"], npt)
        t1 = time.perf_counter()
        sys2.init()
        t2 = time.perf_counter()
        g = 1
        nread = 0
        prev = None
        while g <= K:
            last = min(K, g + prn - 1)
            sys2.enqueue_obs(g, last, obs_addr[last & 1])
            if prev is not None:
                sys2.wait_obs(prev)
                seen.append(Obs.from_address(obs_addr[prev & 1]).T)
                nread += 1
            prev = last
            g = last + 1
        sys2.wait_obs(prev)
        seen.append(Obs.from_address(obs_addr[prev & 1]).T)
        nread += 1
        t3 = time.perf_counter()
        out = sys2.download(out=dst)
        e2e_s = time.perf_counter() - t0
        e2e_parts = {"create_ms": 1e3 * (t1 - t0), "init_ms": 1e3 * (t2 - t1), "steps_ms": 1e3 * (t3 - t2),
                     "download_ms": 1e3 * (t0 + e2e_s - t3)}
        # outside the window: the same download into fresh pageable arrays
        # (first-touch page faults of the destination) and into them again
        t4 = time.perf_counter()
        fresh = sys2.download()
        t5 = time.perf_counter()
        sys2.download(out={k: fresh[k] for k in ("pos", "vel", "h")})
        t6 = time.perf_counter()
        e2e_parts["download_fresh_pageable_ms"] = 1e3 * (t5 - t4)
        e2e_parts["download_touched_pageable_ms"] = 1e3 * (t6 - t5)
        sys2.close()
        h2d = s["pos"].nbytes + s["vel"].nbytes + s["mass"].nbytes + s["mol_id"].nbytes + 9 * 8 + 15 * 8
        d2h = nread * 104 + out["pos"].nbytes + out["vel"].nbytes + 9 * 8 + 15 * 8
        e2e = {"value": ws * na * K / e2e_s, "unit": "atom-steps/s",
               "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K, "wall_parts": e2e_parts,
               "last_T": seen[-1],
               "note": "wall clock: state upload from pinned host arrays, init (lists + first forces), K steps "
                       f"in chunks of {prn} with each chunk's observables copied back asynchronously and read "
                       "on the host while the next chunk runs, state download into pinned host arrays"}
    # ---------------- the same steps with FP32 pair arithmetic ----------------
    from fuller_md_en_b200._lib import FMD_PREC_FP32_PAIR
    _, _, cfg32, _ = make_system(ctx, rank, precision=FMD_PREC_FP32_PAIR)
    sys32 = System.airebo(ctx, cfg32, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
    sys32.init()
    ms32 = float(sum(timed_steps(ctx, stream, sys32, K, flush)))
    lj32_ms = sys32.kernel_ms(0, 20)
    sys32.close()
    value32 = ws * na * K / (ms32 / 1e3)

    # ---------------- learned surrogate on the same workload ----------------
    sg_res = None
    if not args.no_surrogate:
        sg_res = run_surrogate(args, ctx, stream, s, na, cfg, npt, flush, ws, local)

    # ---------------- batched MM replicas (uneven sizes, one launch per phase) ----------------
    batch_res = None
    if not args.no_batch:
        batch_res = run_batch(args, ctx, stream, flush, ws, rank)

    # ---------------- rigid-body LJ, C60 FCC nc=10 (240,000 sites) ----------------
    rigid_res = None
    if not args.no_rigid:
        rigid_res = run_rigid(args, ctx, stream, flush, ws, rank, local)

    ctx.close()
    del flush
    res = {
        "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": ms_total / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "fp32_pair": {"value": value32, "ms_per_step": ms32 / K, "lj_gather_ms": lj32_ms,
                      "note": "same steps with FP32 LJ pair algebra (FP64 minimum image, cutoff test and sums; "
                              "energy/virial within 1e-6 of the FP64 oracle)"},
        "config": {"workload": WORKLOAD, "atoms_per_gpu": na, "global_atoms": na * ws,
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                   "l2": "flushed between timed steps (512 MB write outside the timed windows); "
                         "working set ~75 MB < 126 MB L2",
                   "step_graph": "one CUDA graph per step variant", "wall_s_timed_loop": t_wall},
        "roofline": {"bound": "hbm", "kernel": "k_lj_gather_staged over the pruned rows (atomistic LJ gather)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": lj_bytes, "pruned_row_entries": n_pruned,
                     "full_row_entries": n_full, "full_rows_bytes_per_launch": full_bytes,
                     "launch_shape": lj_shape, "prune": prune,
                     "launch_ms": stages["lj_gather_pruned"], "composite": composite},
        "stage_ms_per_step": per_step,
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
        "surrogate": sg_res,
        "batch": batch_res,
        "rigid": rigid_res,
    }
    return res


def composite_roofline(sysd, na, step_ms, stages, per_step, hbm_peak, hbm_src, clk):
    """Composite roofline of the step: sum over its kernels of algorithmic
    work / peak, over the measured step time.  Work (per step, on the state at
    the end of the timed window): LJ 48 FLOP per listed pair within the
    cutoff (each pair once, after the reference's row truncation); REBO 400
    FLOP per bond (i < j, r <= 2.0 A); integrator 144 B per atom; list
    rebuild (every 20th step) the positions read and the rows written.  FP64
    peak: nominal, 64 FP64 FMA per clock per SM x 148 SMs x the SM clock
    (no measured FP64 figure exists); HBM: the measured copy bandwidth."""
    st = sysd.download()
    ca, la, cb, lb = sysd.lists(400, 12)
    pos = st["pos"].reshape(-1, 3)
    h = st["h"].reshape(3, 3)
    L = np.array([h[0, 0], h[1, 1], h[2, 2]])
    rc2 = (3.0 * 3.40) ** 2

    def pairs_within(cnt, lst, cap, r2max, upper_only):
        i = np.repeat(np.arange(na), cnt)
        j = np.concatenate([lst[k * cap:k * cap + cnt[k]] for k in range(na)]) if cnt.sum() else np.zeros(0, int)
        if upper_only:
            keep = j > i
            i, j = i[keep], j[keep]
        d = pos[j] - pos[i]
        d -= L * np.round(d / L)
        return int(np.count_nonzero((d * d).sum(axis=1) <= r2max))

    n_lj = pairs_within(ca, la, 400, rc2, False)
    n_bond = pairs_within(cb, lb, 12, 2.0 ** 2, True)
    sm_mhz = clk.get("sm_max_mhz") or 1965.0
    fp64_peak = 148 * 64 * 2 * sm_mhz * 1e6 / 1e12            # TFLOP/s
    list_b = na * 24 + na * 4 + 4 * int(ca.sum()) + 4 * int(cb.sum())
    work = {"lj": {"flop": 48 * n_lj, "pairs": n_lj, "peak": fp64_peak, "unit": "TFLOP/s"},
            "rebo": {"flop": 400 * n_bond, "bonds": n_bond, "peak": fp64_peak, "unit": "TFLOP/s"},
            "integrator": {"bytes": 144 * na, "peak": hbm_peak, "unit": "GB/s"},
            "list_rebuild": {"bytes_per_step": list_b / NLUP, "peak": hbm_peak, "unit": "GB/s"}}
    t_us = {"lj": work["lj"]["flop"] / (fp64_peak * 1e12) * 1e6,
            "rebo": work["rebo"]["flop"] / (fp64_peak * 1e12) * 1e6,
            "integrator": work["integrator"]["bytes"] / (hbm_peak * 1e9) * 1e6,
            "list_rebuild": work["list_rebuild"]["bytes_per_step"] / (hbm_peak * 1e9) * 1e6}
    for k in t_us:
        work[k]["roofline_us"] = t_us[k]
    total = sum(t_us.values())
    return {"frac": total / (step_ms * 1e3), "roofline_us_per_step": total, "step_us": step_ms * 1e3,
            "kernels": work, "fp64_peak_source": f"nominal (148 SMs x 64 FP64 FMA/clk x {sm_mhz:.0f} MHz)",
            "hbm_peak_source": hbm_src,
            "lj_kernel_frac_fp64": (work["lj"]["flop"] / (stages["lj_gather_pruned"] * 1e-3)) / (fp64_peak * 1e12)}


def surrogate_nc8(ctx, stream, flush, model, K, judge, rmse_max):
    """The learned-surrogate configuration's inference workload: C60 FCC nc=8
    (2,048 molecules / 122,880 atoms), 300 K, 0 GPa, dt 0.5 fs, with the model
    trained on nc=5 snapshots; steps 1..K timed for the plain kernel and for
    the learned term (judged every `judge` steps)."""
    from fuller_md_en_b200 import RunConfig, System, crystal
    s = crystal.atomistic(8, jitter=JITTER, seed=SEED, T=T_K)
    na = s["pos"].size // 3
    cfg = RunConfig(dt=DT, T=T_K, Pe=P_GPA, nsteps=10 ** 6, nlup=NLUP, gavg_from=1, gavg_to=10 ** 6, nc=8,
                    nmol=s["nmol"], use_graphs=1)
    npt = crystal.npt_atom(T_K, P_GPA, na)
    out = {"atoms": na, "steps": K}
    for mode in ("plain", "learned"):
        sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
        sysd.init()
        if mode == "learned":
            sysd.use_surrogate(model, judge_every=judge, rmse_max=rmse_max)
        ms = float(sum(timed_steps(ctx, stream, sysd, K, flush)))
        out[mode] = na * K / (ms / 1e3)
        out[f"rebo_term_ms_{mode}"] = sysd.kernel_ms(1, 10)
        if mode == "learned":
            out["judge"] = sysd.surrogate_status()
        sysd.close()
    out["unit"] = "atom-steps/s"
    return out


def run_rigid(args, ctx, stream, flush, ws, rank, local):
    """C60 FCC nc=10 as rigid bodies: 4,000 molecules x 60 sites = 240,000
    sites, 300 K, 1 GPa, dt 1 fs, molecule lists every 25 steps, FP32 site-pair
    arithmetic with FP64 per-molecule sums and FP64 integrator."""
    from fuller_md_en_b200 import RunConfig, System, crystal
    from fuller_md_en_b200._lib import FMD_PREC_FP32_PAIR
    from fuller_md_en_b200.replicas import job_throughput, max_over_ranks, replica_seed
    s = crystal.rigid(10, seed=replica_seed(SEED, rank))
    n = s["n"]
    rmcut = 3.0 * 3.431 + 2 * s["Rmol"] + 1.0
    cfg = RunConfig(dt=1.0, T=300.0, Pe=1.0, nsteps=10 ** 6, nlup=25, gavg_from=1, gavg_to=10 ** 6, nc=10, nmol=n,
                    precision=FMD_PREC_FP32_PAIR)
    sysd = System.rigid(ctx, cfg, 60, s["body"], s["I0"], s["Mmol"], rmcut, s["pos"], s["vel"], s["qv"], s["omg"],
                        s["h"], crystal.npt_rigid(300.0, 1.0, n))
    sysd.init()
    K = args.steps
    step_ms = timed_steps(ctx, stream, sysd, K, flush)
    obs = sysd.run(K + 1, K + 1)
    if not math.isfinite(obs.E[0]):
        raise RuntimeError("non-finite energy in the rigid benchmark run")
    pair_ms = sysd.kernel_ms(0, 10)
    pairs = sysd.site_pairs()
    sysd.close()
    ms = max_over_ranks(float(sum(step_ms)), device=f"cuda:{local}")
    sites = n * 60
    fp32_peak = 148 * 128 * 2 * 1965.0e6 / 1e12          # TFLOP/s, nominal
    achieved = 72.0 * pairs / (pair_ms * 1e-3) / 1e12
    out = {"value": job_throughput(sites, K, ms, ws), "unit": "site-steps/s", "ms_per_step": ms / K,
           "workload": "rigid-body LJ, C60 FCC nc=10: 4,000 molecules / 240,000 sites, 300 K, 1 GPa, dt 1 fs, "
                       "molecule lists every 25 steps, FP32 site pairs with FP64 sums and integrator",
           "site_pair_kernel_ms": pair_ms,
           "roofline": {"bound": "fp32 simt", "kernel": "k_rigid_w (site pairs)", "achieved": achieved,
                        "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                        "peak_source": "nominal (148 SMs x 128 FP32 lanes x 2 x 1965 MHz)",
                        "site_pairs_in_cutoff": pairs, "flop_per_pair": 72}}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = rigid_reference_sample(s, n, rmcut)
    return out


def rigid_reference_sample(s, n, rmcut, K=3):
    """The reference's own rigid step (oracle/_ref, OpenMP build, all host
    threads) on global steps 1..K of the same crystal, molecule list built once."""
    from fuller_md_en_b200 import crystal
    from oracle.fmd_oracle import Ref, ref_available
    if not ref_available():
        return None
    R = Ref(omp=True)
    st = dict(pos=s["pos"].copy(), vel=s["vel"].copy(), qv=s["qv"].copy(), omg=s["omg"].copy(), h=s["h"].copy(),
              hi=crystal.inv9(s["h"]), npt=crystal.npt_rigid(300.0, 1.0, n))
    c, l = R.lj_nlist(st["pos"], st["h"], st["hi"], n, rmcut)
    e, F, T, W = R.lj_forces(st["pos"], st["qv"], s["body"], st["h"], st["hi"], c, l, n, 60, rmcut * rmcut)
    st.update(F=F, T=T, W9=W)
    t0 = time.perf_counter()
    for _ in range(K):
        R.lj_step(st, s["body"], s["I0"], s["Mmol"], 60, rmcut * rmcut, 1.0, c, l)
    dt = (time.perf_counter() - t0) / K
    cores = os.cpu_count() or 1
    return {"value": n * 60 / dt, "unit": "site-steps/s", "cores": cores, "kind": "reference",
            "sample": f"{K} steps of the reference's step_npt (OpenMP build, {cores} threads), {dt * 1e3:.0f} ms/step"}


def run_batch(args, ctx, stream, flush, ws, rank):
    """64 MM replicas of C60 FCC, nc in {2,3,4,5} round-robin (16 each of
    1,920 / 6,480 / 15,360 / 30,000 atoms), T ~ U(100,1000) K, P ~ U(0,5) GPa,
    dt 0.1 fs: each step phase one launch over all replicas, launch shapes
    from the autotuner; steps 1..K timed with CUDA events."""
    from fuller_md_en_b200 import Batch, mm_replica
    rng = np.random.default_rng(SEED + 7 * rank)
    R = 64
    t0 = time.perf_counter()
    reps = [mm_replica(ctx, 2 + r % 4, float(rng.uniform(100.0, 1000.0)), float(rng.uniform(0.0, 5.0)),
                       seed=SEED + 1000 * rank + r, jitter=0.01) for r in range(R)]
    t1 = time.perf_counter()
    b = Batch(ctx, reps, autotune=True)
    t2 = time.perf_counter()
    atoms = sum(s.n for s in reps)
    K = args.steps
    step_ms = timed_steps(ctx, stream, b, K, flush)
    obs = b.observables()
    if not all(math.isfinite(o.E[6]) for o in obs):
        raise RuntimeError("non-finite energy in the batched replicas")
    ms = float(sum(step_ms))
    tune = b.tuning()
    nk = [b.step_kernels(False), b.step_kernels(True), b.step_kernels(True, conditional=True)]
    b.close()
    for s_ in reps:
        s_.close()
    return {"value": ws * atoms * K / (ms / 1e3), "unit": "atom-steps/s", "ms_per_step": ms / K,
            "replicas": R, "atoms": atoms, "sizes": "16 x {1920, 6480, 15360, 30000}",
            "workload": "MM (bond+angle+dihedral+improper+LJ; reference charges are zero, so no Coulomb), "
                        "C60 FCC nc in {2,3,4,5} round-robin, T ~ U(100,1000) K, P ~ U(0,5) GPa, dt 0.1 fs, "
                        "lists every 20 steps",
            "kernels_per_step": {"plain": nk[0], "rebuild": nk[1],
                                 "rebuild_fallback_body_not_launched": nk[2]},
            "tuning": tune, "setup_s": {"systems": t1 - t0, "batch_and_autotune": t2 - t1}}


def run_surrogate(args, ctx, stream, s, na, cfg, npt, flush, ws, local):
    """Trains the learned bond-order model on the GPU and times steps
    1..max(K, 201) with it in the step (judged every 100 steps by the plain
    kernel), beside the plain path on the same steps."""
    import torch
    from fuller_md_en_b200 import System
    from fuller_md_en_b200 import surrogate as sgm
    t0 = time.perf_counter()
    data = sgm.generate_dataset(ctx, nc=NC, runs=40, steps=50, every=1, seed=1000 + SEED)
    ctx.synchronize()
    t1 = time.perf_counter()
    n_train = int(0.9 * len(data))
    model, hist = sgm.fit(ctx, data, steps=args.sg_train_steps, batch=8, lr=3e-3, lr_final=3e-5, wE=0.1, wF=1.0,
                          wW=0.1, n_train=n_train, seed=0)
    ctx.synchronize()
    t2 = time.perf_counter()
    rm = model.eval(data)
    data.close()
    K = args.steps
    JUDGE, RMSE_MAX = 100, 0.025
    # REBO term alone on the fresh state: plain kernel vs learned term
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
    sysd.init()
    rebo_plain_ms = sysd.kernel_ms(1, 20)
    sysd.use_surrogate(model, judge_every=JUDGE, rmse_max=RMSE_MAX)
    rebo_sg_ms = sysd.kernel_ms(1, 20)
    sysd.close()
    # Timed steps 1..Ks of the fresh trajectory, Ks covering at least two
    # judge intervals whatever --steps is, so the plain kernel judges the
    # learned term inside the window; the plain path is timed on the same
    # steps of the same trajectory for the ratio.
    Ks = max(K, 2 * JUDGE + 1)
    plain = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
    plain.init()
    plain_ms = float(sum(timed_steps(ctx, stream, plain, Ks, flush)))
    plain.close()
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], npt)
    sysd.init()
    sysd.use_surrogate(model, judge_every=JUDGE, rmse_max=RMSE_MAX)
    step_ms = timed_steps(ctx, stream, sysd, Ks, flush)
    st = sysd.surrogate_status()
    sysd.close()
    take = st["takeover_step"]
    n_learned = Ks if take == 0 else take - 1
    ms_learned = float(sum(step_ms[:n_learned])) if n_learned > 0 else 0.0
    val = ws * na * Ks / (sum(step_ms) / 1e3)
    plain_window = ws * na * Ks / (plain_ms / 1e3)
    nc8 = surrogate_nc8(ctx, stream, flush, model, min(K, 100), JUDGE, RMSE_MAX)
    model.close()
    return {"value": val, "unit": "atom-steps/s", "window_steps": Ks, "plain_same_window": plain_window,
            "vs_plain": val / plain_window, "inference_nc8": nc8,
            "value_learned_steps_only": (na * n_learned / (ms_learned / 1e3)) if n_learned > 0 else None,
            "steps_on_learned_term": n_learned,
            "force_rmse_eV_per_A": {"held_out_mean": float(np.mean(rm[n_train:])),
                                    "held_out_max": float(np.max(rm[n_train:])),
                                    "train_mean": float(np.mean(rm[:n_train])),
                                    "judge_last": st["rmse_last"], "judge_max": st["rmse_max"],
                                    "vs": "plain FP64 REBO kernel (== reference compute_rebo to 1e-10)"},
            "judge": {"every": JUDGE, "rmse_max_eV_per_A": RMSE_MAX, "judged": st["judged"],
                      "takeover_step": take},
            "rebo_term_ms": {"plain": rebo_plain_ms, "learned": rebo_sg_ms},
            "training": {"snapshots": n_train, "held_out": len(rm) - n_train, "adam_steps": args.sg_train_steps,
                         "batch": 8, "dataset_s": t1 - t0, "train_s": t2 - t1,
                         "dataset": "plain AIREBO kernel trajectories, C60 FCC nc=5, 40 runs x 50 steps, "
                                    "T ~ U(300,1500) K, P ~ U(0,5) GPa"},
            "model": "32 descriptors -> 3 x 128 SiLU -> b_ij, BF16 tcgen05 MMA, FP32 accumulate"}


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
    # bounded sample: warm-up capped at 2 steps; timed: global steps 1..K' of
    # the same fresh trajectory the GPU arm times (lists rebuilt every 20),
    # K' = min(K, 40) for the serial build and min(K, 20) for the OpenMP one
    # (slower here: its force loops contend on atomics).
    Kw = min(args.warmup, 2)
    if Kw:
        ref_sample(Kw, omp=False)
    Ks, Ko = min(args.steps, 40), min(args.steps, 20)
    na, ts_s, tr_s = ref_sample(Ks, omp=False)
    _, ts_o, tr_o = ref_sample(Ko, omp=True)
    v_ser = na / ((ts_s + tr_s) / Ks)
    v_omp = na / ((ts_o + tr_o) / Ko)
    if v_ser >= v_omp:
        K, ts, tr, val, build, thr = Ks, ts_s, tr_s, v_ser, "serial", 1
    else:
        K, ts, tr, val, build, thr = Ko, ts_o, tr_o, v_omp, "OpenMP", cores
    per_step = (ts + tr) / K
    return {"impl": "reference", "metric": METRIC, "value": val, "unit": "atom-steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "atoms": na},
            "cpu_baseline": {"value": val, "unit": "atom-steps/s", "cores": thr, "kind": "reference",
                             "sample": f"global steps 1..K' of the same initial state the GPU arm times (lists "
                                       f"rebuilt at steps divisible by 20); value = faster build ({build}). "
                                       f"serial: K'={Ks}, {v_ser:.4g} atom-steps/s (step_npt {ts_s / Ks * 1e3:.1f} "
                                       f"ms/step, list builds {tr_s:.2f} s); OpenMP {cores} threads: K'={Ko}, "
                                       f"{v_omp:.4g} atom-steps/s (step_npt {ts_o / Ko * 1e3:.1f} ms/step, list "
                                       f"builds {tr_o:.2f} s)"},
            "e2e": {"value": val, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def cpu_baseline():
    """The reference's serial build (faster than its OpenMP build for this
    path on these hosts) on global steps 1..20, one list rebuild included."""
    from oracle.fmd_oracle import ref_available
    if not ref_available():
        return None
    K = 20
    na, ts, tr = ref_sample(K, omp=False)
    val = na / ((ts + tr) / K)
    return {"value": val, "unit": "atom-steps/s", "cores": 1, "kind": "reference",
            "sample": f"global steps 1..{K} of the bench trajectory incl. one list rebuild, reference serial build "
                      f"(step_npt {ts / K * 1e3:.0f} ms/step, list build {tr:.2f} s)"}


STAGES = {"lj_full": 0, "rebo": 1, "rebuild": 2, "forces": 3, "lj_pruned": 4, "rigid": 0, "sg": 1, "rebo2": 1,
          "lj_switch": 5}


def synthetic_rebo2_knots(seed: int = 0):
    """Spline knots of the tables' scale for timing the REBO-II kernels (the
    published tables are not in this repository; the kernels' cost does not
    depend on the knot values)."""
    from fuller_md_en_b200 import Rebo2Knots
    rng = np.random.default_rng(seed)
    pcc = np.column_stack([rng.uniform(-0.05, 0.05, 5), rng.uniform(-0.03, 0.03, 5)])

    def tri(shift, amp):
        t = rng.uniform(-0.3 * amp, 0.3 * amp, (5, 5, 10, 8))
        t[..., 0] = rng.uniform(-amp, amp, (5, 5, 10)) + shift
        return t

    return Rebo2Knots(pcc, tri(-0.05, 0.03), tri(0.0, 0.01))


def run_stage(args):
    """--stage: one force stage of a bench workload, launched for a profiler
    (no bench line).  Builds the system, runs --stage-steps steps, then times
    --reps launches of the stage with CUDA events (System.kernel_ms: one
    untimed launch first, then the timed ones, then the current forces are
    recomputed).  Stages of the AIREBO workload (C60 FCC --nc, default 5):
    lj_full / lj_pruned (the LJ gather over the full / pruned rows), rebo,
    rebuild, forces; "sg": the learned REBO term (a randomly initialised
    model: its kernels' cost does not depend on the weights); "rigid": the
    rigid site-pair kernel of C60 FCC --nc (default 10; 240,000 sites, 1 GPa,
    FP32 site pairs).  FMD_LJ_SHAPE pins the LJ gather's launch shape
    (threads, entries per lane, row feed) so the launch sequence does not
    depend on the autotuner: with --stage-steps 0 and --reps 1 the LJ gather
    launches are set-up's (one, pruning the full rows), the untimed and the
    timed launch of the stage, then the recomputation's, so a profiler
    capturing the gather's launch 3 sees the timed, warm launch on the bench
    state.  The REBO kernels launch twice per force evaluation (geometry +
    bond order, forces).  "rebo2" / "lj_switch": the REBO-II term (coordination
    and bond kernels) / the switched-LJ correction of the same workload with
    both extensions on and synthetic spline knots.  Prints one JSON line."""
    from fuller_md_en_b200 import Context, RunConfig, System, crystal
    from fuller_md_en_b200._lib import FMD_PREC_FP32_PAIR
    ctx = Context(0)
    if args.stage == "rigid":
        nc = args.nc or 10
        s = crystal.rigid(nc, seed=SEED)
        n = s["n"]
        rmcut = 3.0 * 3.431 + 2 * s["Rmol"] + 1.0
        cfg = RunConfig(dt=1.0, T=300.0, Pe=1.0, nsteps=10 ** 6, nlup=25, nc=nc, nmol=n, precision=FMD_PREC_FP32_PAIR)
        y = System.rigid(ctx, cfg, 60, s["body"], s["I0"], s["Mmol"], rmcut, s["pos"], s["vel"], s["qv"], s["omg"],
                         s["h"], crystal.npt_rigid(300.0, 1.0, n))
        y.init()
        if args.stage_steps > 0:
            y.run(1, args.stage_steps)
        ms = y.kernel_ms(STAGES[args.stage], args.reps)
        c, _, _, _ = y.lists(80)
        out = {"stage": args.stage, "ms_per_launch": ms, "molecules": n, "sites": 60 * n, "steps": args.stage_steps,
               "molecule_list_entries": int(c.sum())}
    else:
        nc = args.nc or NC
        s = crystal.atomistic(nc, jitter=JITTER, seed=SEED, T=T_K)
        na = s["pos"].size // 3
        cfg = RunConfig(dt=DT, T=T_K, Pe=P_GPA, nsteps=10 ** 6, nlup=NLUP, nc=nc, nmol=s["nmol"])
        y = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"],
                          crystal.npt_atom(T_K, P_GPA, na))
        y.set_lj_prune(args.delta)
        if args.stage in ("rebo2", "lj_switch"):
            from fuller_md_en_b200._lib import FMD_REBO2_BOND_ORDER, FMD_REBO2_LJ_SWITCH
            y.set_rebo2(synthetic_rebo2_knots(), FMD_REBO2_BOND_ORDER | FMD_REBO2_LJ_SWITCH)
        y.init()
        model = None
        if args.stage == "sg":
            from fuller_md_en_b200 import surrogate as sgm
            model = sgm.Surrogate(ctx, sgm.init_params(0))
            y.use_surrogate(model, judge_every=10 ** 6, rmse_max=1e9)
        if args.stage_steps > 0:
            y.run(1, args.stage_steps)
        ms = y.kernel_ms(STAGES[args.stage], args.reps)
        full, pruned = y.lj_rows()
        out = {"stage": args.stage, "ms_per_launch": ms, "atoms": na, "steps": args.stage_steps,
               "shape": y.lj_shape(), "full_row_entries": int(full.sum()), "pruned_row_entries": int(pruned.sum()),
               "prune": y.lj_prune()}
        if model is not None:
            y.close()
            model.close()
            y = None
    if y is not None:
        y.close()
    ctx.close()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-rigid", action="store_true")
    ap.add_argument("--sg-train-steps", type=int, default=6000)
    ap.add_argument("--stage", choices=sorted(STAGES), default=None,
                    help="profile one force stage instead of the bench (see run_stage)")
    ap.add_argument("--nc", type=int, default=0, help="--stage: crystal size (default 5, rigid 10)")
    ap.add_argument("--stage-steps", type=int, default=0, help="--stage: steps run before the timed launches")
    ap.add_argument("--reps", type=int, default=1, help="--stage: timed launches")
    ap.add_argument("--delta", type=float, default=0.5, help="--stage: pruned-row buffer (A)")
    args = ap.parse_args()
    if args.stage:
        run_stage(args)
        return
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
