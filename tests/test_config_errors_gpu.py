"""Per-step energy, virial and pressure error of each configuration against
the reference's FP64 arithmetic (the oracle), teacher-forced: after every
device step the oracle evaluates the forces at the GPU's own positions, cell
and lists, so the comparison measures the step's arithmetic, not the
divergence of two chaotic trajectories.  At every list rebuild inside the
window the device's lists are compared, bit for bit, with the reference
builder run on the state the device built them from (the state after the
previous step).

Errors are normalised as: energy |dE|/|E|; virial max|dW_ab| / ||W||_F
(off-diagonal entries are near zero, so per-entry relative error is
ill-posed); pressure |dP| / (|2 KE| + |tr W|) / (3V) scale.  Bounds: 1e-10
for the FP64 kernels, 1e-6 for FP32 pair arithmetic.  Run with -s to see the
per-step table; each test ends with one "max" line per configuration.

The oracle evaluations of a window run on host threads after the device
steps (the oracle's ctypes calls release the GIL), so the 240,000-site and
122,880-atom configurations finish in seconds to minutes."""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import rows, same_rows
from fuller_md_en_b200 import RunConfig, System, crystal, mm_replica
from fuller_md_en_b200._lib import FMD_PREC_FP32_PAIR, FMD_PREC_FP64

pytestmark = pytest.mark.gpu

EV2GPA = 160.21766208
RC_AI = 3.0 * 3.40 + 2.0
RC_MM = 3.0 * 3.431 + 2.0


def _pmap(fn, items):
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        return list(ex.map(fn, items))


def _errs(tag, g, E, Eref, W, Wref, KE, V, quiet=False):
    dE = abs(E - Eref) / abs(Eref)
    dW = np.max(np.abs(W - Wref)) / np.linalg.norm(Wref)
    P, Pref = (2 * KE + np.trace(W.reshape(3, 3))) / (3 * V), (2 * KE + np.trace(Wref.reshape(3, 3))) / (3 * V)
    dP = abs(P - Pref) / ((abs(2 * KE) + abs(np.trace(Wref.reshape(3, 3)))) / (3 * V))
    if not quiet:
        print(f"{tag} step {g:3d}: dE {dE:.2e}  dW {dW:.2e}  dP {dP:.2e}  (P {P * EV2GPA:+.4f} GPa)")
    return dE, dW, dP


def _report(tag, steps, errs, tol):
    e = np.array(errs)
    mx = e.max(axis=0)
    print(f"max {tag} steps {steps}: dE {mx[0]:.2e}  dW {mx[1]:.2e}  dP {mx[2]:.2e}  (bound {tol:g})")
    assert (mx < tol).all(), (tag, mx)


def _vol(h):
    return abs(np.linalg.det(np.asarray(h).reshape(3, 3)))


# ----------------------------------------------------------- rigid (C1, C2) --

def _rigid_window(ctx, oracle, tag, nc, prec, tol, steps, Pe, seed=31):
    s = crystal.rigid(nc, seed=seed)
    n = s["n"]
    rmcut = 3.0 * 3.431 + 2 * s["Rmol"] + 1.0
    cfg = RunConfig(dt=1.0, T=300.0, Pe=Pe, nsteps=max(steps, 100), nlup=25, nc=nc, nmol=n, precision=prec)
    sysd = System.rigid(ctx, cfg, 60, s["body"], s["I0"], s["Mmol"], rmcut, s["pos"], s["vel"], s["qv"], s["omg"],
                        s["h"], crystal.npt_rigid(300.0, Pe, n))
    sysd.init()
    recs, prev, rebuilds = [], None, 0
    for g in range(1, steps + 1):
        o = sysd.run(g, g)
        st = sysd.download()
        W, KE = sysd.virial()
        if g == 1 or g % 25 == 0:             # lists change only at a rebuild
            c, l, _, _ = sysd.lists(80)
        if g % 25 == 0:                       # rebuilt before step g from the state after g-1 (LJ:859-862)
            oc, ol, _ = oracle.nlist_sym(prev["pos"], prev["h"], crystal.inv9(prev["h"]), n, rmcut)
            assert np.array_equal(c, oc) and same_rows(rows(c, l, 80), rows(oc, ol, 80)), (tag, g)
            rebuilds += 1
        recs.append((g, o.E[0], W, KE, st, c, l))
        prev = st
    sysd.close()

    def ev(r):
        g, E, W, KE, st, c, l = r
        e, _, _, Wr = oracle.rigid_forces(st["pos"], st["qv"], s["body"], st["h"], crystal.inv9(st["h"]), c, l, n,
                                          60, rmcut * rmcut)
        return _errs(tag, g, E, e, W, Wr, KE, _vol(st["h"]), quiet=steps > 10)

    _report(tag, f"1-{steps} ({rebuilds} list rebuilds checked)", _pmap(ev, recs), tol)


@pytest.mark.parametrize("cfg_name,prec,tol", [("C1 rigid core nc=3", FMD_PREC_FP64, 1e-10),
                                               ("C1 rigid core nc=3 fp32", FMD_PREC_FP32_PAIR, 1e-6)])
def test_rigid_c1_config_errors(ctx, oracle, cfg_name, prec, tol):
    _rigid_window(ctx, oracle, cfg_name, 3, prec, tol, 50, 0.0)


def test_rigid_c2_first_100_steps(ctx, oracle):
    """C2: 4,000 C60 (240,000 sites) at 1 GPa with FP32 site pairs, every one
    of the first 100 steps, and the molecule lists of the rebuilds at steps
    25, 50 and 75."""
    _rigid_window(ctx, oracle, "C2 rigid nc=10 fp32", 10, FMD_PREC_FP32_PAIR, 1e-6, 100, 1.0)


# ------------------------------------------------------- AIREBO (C3, C5) --

def _airebo_window(ctx, oracle, tag, nc, prec, tol, check_steps, seed=42, init_lists=False):
    s = crystal.atomistic(nc, jitter=0.01, seed=seed, T=300.0)
    na = s["pos"].size // 3
    last = max(check_steps)
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=max(last, 100), nlup=20, nc=nc, nmol=s["nmol"], precision=prec)
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], crystal.npt_atom(300.0, 0.0, na))
    sysd.init()

    def check_lists(pos, h, g):
        ca, la, cb, lb = cur if g else sysd.lists(400, 12)
        hi = crystal.inv9(h)
        oc, ol, _ = oracle.nlist_half_threaded(pos, h, hi, na, s["mol_id"], RC_AI)
        orc, orl, _ = oracle.nlist_intra(pos, h, hi, na, s["mol_id"])
        assert np.array_equal(ca, oc) and same_rows(rows(ca, la, 400), rows(oc, ol, 400)), (tag, g)
        assert np.array_equal(cb, orc) and same_rows(rows(cb, lb, 12), rows(orc, orl, 12)), (tag, g)
        return int((oc == 400).sum())

    if init_lists:                             # lists from the unwrapped start positions (AI:830-836)
        sat = check_lists(s["pos"], s["h"], 0)
        print(f"{tag}: lists at init bit-exact ({na} atoms, {sat} rows truncated at 400)")
    recs, prev, rebuilds, cur = [], None, 0, None
    g = 0
    while g < last:
        g += 1
        o = sysd.run(g, g)
        if g == 1 or g % 20 == 0:              # lists change only at a rebuild
            cur = sysd.lists(400, 12)
        if g % 20 == 0:
            check_lists(prev["pos"], prev["h"], g)
            rebuilds += 1
        need_prev = (g + 1) % 20 == 0 and g + 1 <= last
        if g in check_steps or need_prev:
            st = sysd.download()
            if g in check_steps:
                W, KE = sysd.virial()
                recs.append((g, o.E[0], W, KE, st, *cur))
            prev = st
    sysd.close()

    def ev(r):
        g, E, W, KE, st, ca, la, cb, lb = r
        Er, _, Wr = oracle.airebo_forces(st["pos"], st["h"], crystal.inv9(st["h"]), cb, lb, ca, la, na)
        return _errs(tag, g, E, Er[0], W, Wr, KE, _vol(st["h"]), quiet=len(check_steps) > 10)

    _report(tag, f"{min(check_steps)}-{last} ({len(check_steps)} checked, {rebuilds} list rebuilds checked)",
            _pmap(ev, recs), tol)


@pytest.mark.parametrize("cfg_name,prec,tol", [("C3 AIREBO nc=5", FMD_PREC_FP64, 1e-10),
                                               ("C3 AIREBO nc=5 fp32 LJ", FMD_PREC_FP32_PAIR, 1e-6)])
def test_airebo_c3_config_errors(ctx, oracle, cfg_name, prec, tol):
    _airebo_window(ctx, oracle, cfg_name, 5, prec, tol, set(range(1, 42)))


def test_airebo_c5_nc8_lists_and_errors(ctx, oracle):
    """C5's plain path at its inference size: C60 FCC nc=8, 2,048 molecules /
    122,880 atoms.  Lists at init and at the rebuild of step 20 bit for bit;
    energy, virial and pressure at steps 1, 2, 10, 20 and 21."""
    _airebo_window(ctx, oracle, "C5 AIREBO nc=8", 8, FMD_PREC_FP64, 1e-10, {1, 2, 10, 20, 21}, seed=7,
                   init_lists=True)


# ------------------------------------------------------------- MM batch (C4) --

def test_mm_batch_c4_all_sizes(ctx, oracle):
    """C4: one replica of every size of the configuration (nc = 2, 3, 4, 5:
    1,920 / 6,480 / 15,360 / 30,000 atoms) at its own temperature and
    pressure, advanced as one batch.  Each replica's energy, virial and
    pressure at every step 1..22, and its list at the rebuild of step 20."""
    from fuller_md_en_b200 import Batch
    coords = crystal.c60_ih()
    bonds = crystal.bonds_from_geometry(coords)
    cases = [(2, 150.0, 0.5, 3), (3, 700.0, 2.0, 4), (4, 420.0, 4.6, 5), (5, 960.0, 1.3, 6)]
    reps = [mm_replica(ctx, nc, T, P, dt=0.1, seed=seed, jitter=0.01) for nc, T, P, seed in cases]
    b = Batch(ctx, reps)
    last = 22
    recs = {k: [] for k in range(len(reps))}
    prev = [None] * len(reps)
    mol = [None] * len(reps)
    cur = [None] * len(reps)
    for g in range(1, last + 1):
        obs = b.run(g, g)
        for k, (sysd, o) in enumerate(zip(reps, obs)):
            st = sysd.download()
            na = st["pos"].size // 3
            if g == 1 or g % 20 == 0:          # lists change only at a rebuild
                cur[k] = sysd.lists(400)[:2]
            c, l = cur[k]
            if g == 20:
                if mol[k] is None:
                    mol[k] = np.repeat(np.arange(na // 60, dtype=np.int32), 60)
                hp = crystal.inv9(prev[k]["h"])
                oc, ol, _ = oracle.nlist_half_threaded(prev[k]["pos"], prev[k]["h"], hp, na, mol[k], RC_MM)
                assert np.array_equal(c, oc) and same_rows(rows(c, l, 400), rows(oc, ol, 400)), (cases[k], g)
            W, KE = sysd.virial()
            recs[k].append((g, o.E[6], W, KE, st, c, l))
            prev[k] = st
    b.close()
    for r in reps:
        r.close()

    for k, (nc, T, P, seed) in enumerate(cases):
        na = recs[k][0][4]["pos"].size // 3
        t = crystal.mm_topology(coords, bonds, na // 60)
        tag = f"C4 MM replica nc={nc} ({na} atoms, {T:g} K, {P:g} GPa)"

        def ev(r, t=t, na=na, tag=tag):
            g, E, W, KE, st, c, l = r
            Er, _, Wr = oracle.mm_forces(t, st["pos"], st["h"], crystal.inv9(st["h"]), c, l, na)
            return _errs(tag, g, E, Er[6], W, Wr, KE, _vol(st["h"]), quiet=True)

        _report(tag, f"1-{last} (list rebuild at 20 checked)", _pmap(ev, recs[k]), 1e-10)
