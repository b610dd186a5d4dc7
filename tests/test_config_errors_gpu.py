"""Per-step energy, virial and pressure error of each configuration against
the reference's FP64 arithmetic (the oracle), teacher-forced: after every
device step the oracle evaluates the forces at the GPU's own positions, cell
and lists, so the comparison measures the step's arithmetic, not the
divergence of two chaotic trajectories.

Errors are normalised as: energy |dE|/|E|; virial max|dW_ab| / ||W||_F
(off-diagonal entries are near zero, so per-entry relative error is
ill-posed); pressure |dP| / (|2 KE| + |tr W|) / (3V) scale.  Bounds: 1e-10
for the FP64 kernels, 1e-6 for FP32 pair arithmetic.  Run with -s to see the
per-step table."""
from __future__ import annotations

import numpy as np
import pytest

from fuller_md_en_b200 import RunConfig, System, crystal, mm_replica
from fuller_md_en_b200._lib import FMD_PREC_FP32_PAIR, FMD_PREC_FP64

pytestmark = pytest.mark.gpu

EV2GPA = 160.21766208


def _errs(tag, g, E, Eref, W, Wref, KE, V):
    dE = abs(E - Eref) / abs(Eref)
    dW = np.max(np.abs(W - Wref)) / np.linalg.norm(Wref)
    P, Pref = (2 * KE + np.trace(W.reshape(3, 3))) / (3 * V), (2 * KE + np.trace(Wref.reshape(3, 3))) / (3 * V)
    dP = abs(P - Pref) / ((abs(2 * KE) + abs(np.trace(Wref.reshape(3, 3)))) / (3 * V))
    print(f"{tag} step {g:3d}: dE {dE:.2e}  dW {dW:.2e}  dP {dP:.2e}  (P {P * EV2GPA:+.4f} GPa)")
    return dE, dW, dP


@pytest.mark.parametrize("cfg_name,nc,prec,tol,steps", [
    ("C1 rigid core nc=3", 3, FMD_PREC_FP64, 1e-10, 5),
    ("C1 rigid core nc=3 fp32", 3, FMD_PREC_FP32_PAIR, 1e-6, 5),
    ("C2 rigid nc=10 fp32", 10, FMD_PREC_FP32_PAIR, 1e-6, 2),
])
def test_rigid_config_errors(ctx, oracle, cfg_name, nc, prec, tol, steps):
    s = crystal.rigid(nc, seed=31)
    n = s["n"]
    rmcut = 3.0 * 3.431 + 2 * s["Rmol"] + 1.0
    Pe = 1.0 if nc == 10 else 0.0
    cfg = RunConfig(dt=1.0, T=300.0, Pe=Pe, nsteps=100, nlup=25, nc=nc, nmol=n, precision=prec)
    sysd = System.rigid(ctx, cfg, 60, s["body"], s["I0"], s["Mmol"], rmcut, s["pos"], s["vel"], s["qv"], s["omg"],
                        s["h"], crystal.npt_rigid(300.0, Pe, n))
    sysd.init()
    for g in range(1, steps + 1):
        o = sysd.run(g, g)
        st = sysd.download()
        W, KE = sysd.virial()
        c, l, _, _ = sysd.lists(80)
        hi = crystal.inv9(st["h"])
        e, _, _, Wr = oracle.rigid_forces(st["pos"], st["qv"], s["body"], st["h"], hi, c, l, n, 60, rmcut * rmcut)
        V = abs(np.linalg.det(st["h"].reshape(3, 3)))
        dE, dW, dP = _errs(cfg_name, g, o.E[0], e, W, Wr, KE, V)
        assert dE < tol and dW < tol and dP < tol
    sysd.close()


@pytest.mark.parametrize("cfg_name,prec,tol", [("C3 AIREBO nc=5", FMD_PREC_FP64, 1e-10),
                                               ("C3 AIREBO nc=5 fp32 LJ", FMD_PREC_FP32_PAIR, 1e-6)])
def test_airebo_config_errors(ctx, oracle, cfg_name, prec, tol):
    s = crystal.atomistic(5, jitter=0.01, seed=42, T=300.0)
    na = s["pos"].size // 3
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=100, nlup=20, nc=5, nmol=s["nmol"], precision=prec)
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"], crystal.npt_atom(300.0, 0.0, na))
    sysd.init()
    prev = 0
    for g in (1, 2, 10, 21):                      # step 21 follows the rebuild at 20
        o = sysd.run(prev + 1, g)
        prev = g
        st = sysd.download()
        W, KE = sysd.virial()
        ca, la, cb, lb = sysd.lists(400, 12)
        hi = crystal.inv9(st["h"])
        Er, _, Wr = oracle.airebo_forces(st["pos"], st["h"], hi, cb, lb, ca, la, na)
        V = abs(np.linalg.det(st["h"].reshape(3, 3)))
        dE, dW, dP = _errs(cfg_name, g, o.E[0], Er[0], W, Wr, KE, V)
        assert dE < tol and dW < tol and dP < tol
    sysd.close()


def test_mm_batch_config_errors(ctx, oracle):
    """C4 (reduced): replicas of uneven size advanced as one batch; each
    replica's energy, virial and pressure against the oracle."""
    from fuller_md_en_b200 import Batch
    coords = crystal.c60_ih()
    bonds = crystal.bonds_from_geometry(coords)
    cases = [(2, 150.0, 0.5, 3), (3, 700.0, 2.0, 4)]
    reps = [mm_replica(ctx, nc, T, P, dt=0.1, seed=seed, jitter=0.01) for nc, T, P, seed in cases]
    b = Batch(ctx, reps)
    obs = b.run(1, 3)
    for (nc, T, P, seed), sysd, o in zip(cases, reps, obs):
        st = sysd.download()
        W, KE = sysd.virial()
        c, l, _, _ = sysd.lists(400)
        na = st["pos"].size // 3
        t = crystal.mm_topology(coords, bonds, na // 60)
        hi = crystal.inv9(st["h"])
        Er, _, Wr = oracle.mm_forces(t, st["pos"], st["h"], hi, c, l, na)
        V = abs(np.linalg.det(st["h"].reshape(3, 3)))
        dE, dW, dP = _errs(f"C4 MM replica nc={nc}", 3, o.E[6], Er[6], W, Wr, KE, V)
        assert dE < 1e-10 and dW < 1e-10 and dP < 1e-10
    b.close()
    for r in reps:
        r.close()
