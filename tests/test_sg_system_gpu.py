"""The learned REBO term inside a device-resident AIREBO system: the step
uses it, the plain REBO kernel judges it on schedule and takes over above
the threshold, and a trained network is compared with the same pipeline
without one (a constant bond order).

Models are trained here, on the GPU, from the plain kernel's own short
trajectories (surrogate.generate_dataset / fit)."""
from __future__ import annotations

import numpy as np
import pytest

from fuller_md_en_b200 import crystal

NC = 2


@pytest.fixture(scope="module")
def trained():
    from fuller_md_en_b200 import surrogate as sgm
    from fuller_md_en_b200.api import Context
    ctx = Context()
    data = sgm.generate_dataset(ctx, nc=NC, runs=12, steps=40, every=1, seed=5)
    n_train = int(0.75 * len(data))
    S, hist = sgm.fit(ctx, data, steps=2500, batch=8, lr=3e-3, lr_final=3e-5, n_train=n_train, seed=0)
    yield ctx, data, n_train, S, hist
    S.close()
    data.close()
    ctx.close()


def _system(ctx, seed=7):
    from fuller_md_en_b200 import RunConfig, System
    s = crystal.atomistic(NC, jitter=0.01, seed=seed, T=300.0)
    na = s["pos"].size // 3
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=1000, nlup=20, gavg_from=1, gavg_to=1000, nc=NC,
                    nmol=s["nmol"])
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"],
                         crystal.npt_atom(300.0, 0.0, na))
    sysd.init()
    return sysd, na


@pytest.mark.gpu
def test_trained_network_gains_over_constant_bond_order(trained):
    """The same rows, assembly and forces with the network removed (output
    weights zero, so b = b0 everywhere) against the trained network, on
    held-out snapshots of the plain kernel's trajectories."""
    from fuller_md_en_b200 import surrogate as sgm
    ctx, data, n_train, S, hist = trained
    assert np.isfinite(hist).all()
    rm = S.eval(data, n_train)
    P0 = S.params()
    P0["w4"] = np.zeros_like(P0["w4"])
    S0 = sgm.Surrogate(ctx, P0)
    rm0 = S0.eval(data, n_train)
    S0.close()
    assert rm.mean() < 0.025, rm.mean()                 # eV/A, held-out snapshots
    assert rm.mean() < 0.05 * rm0.mean(), (rm.mean(), rm0.mean())


@pytest.mark.gpu
def test_system_step_uses_learned_term_and_judge(trained):
    ctx, data, n_train, S, _ = trained
    sysd, na = _system(ctx)
    sysd.use_surrogate(S, judge_every=10, rmse_max=0.2)
    obs = sysd.run(1, 30)
    st = sysd.surrogate_status()
    assert st["attached"] == 1 and st["active"] == 1 and st["judged"] == 3 and st["takeover_step"] == 0
    assert 0.0 < st["rmse_last"] <= st["rmse_max"] < 0.2
    # the step's REBO energy is the learned term's energy of the final state
    out = sysd.download()
    _, _, cb, lb = sysd.lists(400, 12)
    hi = ctx.mat_inv9(out["h"])
    E_sg, _, _ = S.rebo_forces(out["pos"], out["h"], hi, cb, lb)
    assert abs(obs.E[1] - E_sg) <= 1e-9 * abs(E_sg), (obs.E[1], E_sg)
    F = np.zeros(3 * na); W = np.zeros(9)
    E_plain = ctx.compute_rebo(F, W, out["pos"], out["h"], hi, cb, lb, na)
    assert obs.E[1] != E_plain
    sysd.close()


@pytest.mark.gpu
def test_plain_kernel_takes_over_above_threshold(trained):
    ctx, data, n_train, S, _ = trained
    sysd, na = _system(ctx, seed=8)
    sysd.use_surrogate(S, judge_every=5, rmse_max=1e-9)
    sysd.run(1, 4)
    assert sysd.surrogate_status()["active"] == 1
    obs = sysd.run(5, 12)
    st = sysd.surrogate_status()
    assert st["active"] == 0 and st["takeover_step"] == 5 and st["judged"] == 1
    assert st["rmse_last"] > 1e-9
    # after the takeover the step's REBO term is the plain kernel's
    out = sysd.download()
    _, _, cb, lb = sysd.lists(400, 12)
    hi = ctx.mat_inv9(out["h"])
    F = np.zeros(3 * na); W = np.zeros(9)
    E_plain = ctx.compute_rebo(F, W, out["pos"], out["h"], hi, cb, lb, na)
    assert abs(obs.E[1] - E_plain) <= 1e-9 * abs(E_plain), (obs.E[1], E_plain)
    # detaching returns to the plain kernel, attaching again resets the record
    sysd.use_surrogate(None)
    assert sysd.surrogate_status()["attached"] == 0
    sysd.use_surrogate(S, judge_every=5, rmse_max=1.0)
    st = sysd.surrogate_status()
    assert st["active"] == 1 and st["judged"] == 0
    sysd.run(13, 15)
    assert sysd.surrogate_status()["judged"] == 1
    sysd.close()


@pytest.mark.gpu
def test_surrogate_bad_arguments_are_errors(trained):
    from fuller_md_en_b200 import FmdError
    ctx, data, n_train, S, _ = trained
    sysd, na = _system(ctx)
    with pytest.raises(FmdError):
        sysd.use_surrogate(S, judge_every=-1)
    with pytest.raises(FmdError):
        sysd.use_surrogate(S, judge_every=10, rmse_max=0.0)
    sysd.close()
