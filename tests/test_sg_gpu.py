"""The learned bond-order potential on the GPU against its FP64 CPU
restatement (oracle/sg_oracle.py).

Each stage is compared on the same inputs: rows, BF16 descriptors, the
tensor-core network (b and db/dx, with the restatement rounding the same
operands to BF16), and the FP64 force assembly.
"""
from __future__ import annotations

import numpy as np
import pytest

from fuller_md_en_b200 import crystal
from oracle import sg_oracle as sg


def _case(oracle, nc, seed, jitter=0.03):
    s = crystal.atomistic(nc, T=300.0, seed=seed, jitter=jitter)
    na = s["pos"].size // 3
    pos = s["pos"].copy()
    oracle.apply_pbc(pos, s["h"], s["hi"])
    cnt, lst, _ = oracle.nlist_intra(pos, s["h"], s["hi"], na, s["mol_id"])
    g = sg.rows(pos, s["h"], s["hi"], cnt, lst)
    X, J = sg.descriptors(g)
    P = sg.init_params(seed)
    P["m"] = X.mean(0); P["s"] = X.std(0) + 1e-3
    bex = sg.exact_bond_order(g)
    P["b0"], P["bs"] = float(bex.mean()), float(bex.std())
    return dict(pos=pos, h=s["h"], hi=s["hi"], cnt=cnt, lst=lst, g=g, X=X, J=J, P=P, na=na)


@pytest.mark.gpu
@pytest.mark.parametrize("nc,seed", [(1, 11), (3, 12)])
def test_surrogate_stages_match_restatement(oracle, nc, seed):
    from fuller_md_en_b200.api import Context
    from fuller_md_en_b200.surrogate import Surrogate
    c = _case(oracle, nc, seed)
    g, P = c["g"], c["P"]
    ctx = Context()
    S = Surrogate(ctx, P)
    E, F, W = S.rebo_forces(c["pos"], c["h"], c["hi"], c["cnt"], c["lst"])
    rows = S.last_rows()
    # rows: same directed bonds in the same order (atom, then list slot)
    np.testing.assert_array_equal(rows["i"], g["i"])
    np.testing.assert_array_equal(rows["j"], g["j"])
    # descriptors: FP32 on the GPU, FP64 here, both rounded to BF16
    Xn = sg.normalise(c["X"], P["m"], P["s"])
    ref = sg.bf16(Xn)
    tol = 2.0 ** -7 * np.abs(ref) + 1e-5
    assert np.all(np.abs(rows["xn"] - ref) <= tol)
    # network on the GPU's own BF16 descriptors
    b, cache = sg.mlp(P, rows["xn"].astype(np.float64), rnd=True)
    gx = sg.mlp_grad(P, cache, rnd=True)
    # BF16 rounding of a hidden activation can flip by one unit between the
    # two evaluations; bound the worst row loosely and the typical row tightly
    db = rows["b"] - b
    assert np.abs(db).max() <= 5e-3 * P["bs"]
    assert np.sqrt(np.mean(db ** 2)) <= 1e-4 * P["bs"]
    scale = np.abs(gx).max()
    np.testing.assert_allclose(rows["gx"][:, :-1], gx[:, :-1], rtol=0, atol=2e-2 * scale)
    # FP64 assembly with the GPU's b and gx
    Ea, Fa, Wa = sg.assemble(g, rows["b"].astype(np.float64),
                             sg.dbdk_from_gx(g, c["J"], rows["gx"].astype(np.float64), P["s"]))
    assert abs(E - Ea) <= 1e-9 * abs(Ea)
    np.testing.assert_allclose(F, Fa, rtol=0, atol=1e-5 * np.abs(Fa).max())
    np.testing.assert_allclose(W, Wa, rtol=0, atol=1e-9 * np.abs(Wa).max())
    S.close()
    ctx.close()


@pytest.mark.gpu
def test_surrogate_with_fitted_bond_order_is_close_to_rebo(oracle):
    """A network whose output layer is fitted (least squares on h3) to the
    reference bond order gives energies within a few percent of REBO: the
    assembly and the network agree on what b means."""
    from fuller_md_en_b200.api import Context
    from fuller_md_en_b200.surrogate import Surrogate
    c = _case(oracle, 1, 21)
    g, P = c["g"], c["P"]
    bex = sg.exact_bond_order(g)
    Xn = sg.normalise(c["X"], P["m"], P["s"])
    _, cache = sg.mlp(P, Xn)
    A = cache["h3"]
    y = (bex - P["b0"]) / P["bs"]
    P["w4"] = np.linalg.lstsq(A, y, rcond=None)[0]
    ctx = Context()
    S = Surrogate(ctx, P)
    E, F, W = S.rebo_forces(c["pos"], c["h"], c["hi"], c["cnt"], c["lst"])
    Er, Fr, Wr = oracle.rebo(c["pos"], c["h"], c["hi"], c["cnt"], c["lst"], c["na"])
    assert abs(E - Er) < 0.01 * abs(Er)
    S.close()
    ctx.close()


@pytest.mark.gpu
def test_loss_gradient_matches_restatement(oracle):
    """Double backpropagation on the tensor cores (k_sg_chain, k_sg_wgrad)
    against the FP64 restatement with the same BF16 rounding points; the
    restatement itself is checked against finite differences on the CPU."""
    from fuller_md_en_b200.api import Context
    from fuller_md_en_b200.surrogate import Surrogate
    c = _case(oracle, 1, 31, jitter=0.05)
    g, P = c["g"], c["P"]
    Er, Fr, Wr = oracle.rebo(c["pos"], c["h"], c["hi"], c["cnt"], c["lst"], c["na"])
    w = dict(wE=0.3, wF=1.0, wW=0.2)
    L, grads, _, _, _ = sg.loss_and_grad(P, g, Er, Fr, Wr, rnd=True, **w)
    ctx = Context()
    S = Surrogate(ctx, P)
    Lg, gg = S.loss_grad(c["pos"], c["h"], c["hi"], c["cnt"], c["lst"], Fr, Er, Wr, **w)
    assert abs(Lg - L) <= 2e-3 * L
    for k in ("W1", "W2", "W3", "w4"):
        a, b = gg[k].ravel(), grads[k].ravel()
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        assert rel < 3e-2 and cos > 0.999, (k, rel, cos)
    assert np.all(gg["m"] == 0) and np.all(gg["s"] == 0)
    S.close()
    ctx.close()


@pytest.mark.gpu
def test_training_reduces_force_error(oracle):
    from fuller_md_en_b200 import surrogate as sgm
    from fuller_md_en_b200.api import Context
    ctx = Context()
    ds = sgm.Dataset(ctx)
    for seed in range(6):
        s = crystal.atomistic(1, T=300.0, seed=100 + seed, jitter=0.05)
        na = s["pos"].size // 3
        pos = s["pos"].copy()
        oracle.apply_pbc(pos, s["h"], s["hi"])
        cnt, lst, _ = oracle.nlist_intra(pos, s["h"], s["hi"], na, s["mol_id"])
        ds.add(pos, s["h"], s["hi"], cnt, lst)
        E, W, F = ds.reference(len(ds) - 1)
        Er, Fr, Wr = oracle.rebo(pos, s["h"], s["hi"], cnt, lst, na)
        assert abs(E - Er) <= 1e-9 * abs(Er)         # references come from the plain REBO kernel
        np.testing.assert_allclose(F, Fr, rtol=0, atol=1e-9)
    P = sgm.init_params(1)
    S = sgm.Surrogate(ctx, P)
    m, sd = S.feature_stats(ds)
    P["m"], P["s"] = m, sd + 1e-3
    P["b0"], P["bs"] = 0.9, 0.05
    S.set_params(P)
    before = S.eval(ds)
    hist = S.train(ds, steps=400, batch=2, lr=3e-3, lr_final=1e-4, seed=3)
    after = S.eval(ds)
    assert np.isfinite(hist).all()
    assert hist[-50:, 0].mean() < 0.1 * hist[:50, 0].mean()
    assert after.mean() < 0.3 * before.mean(), (before, after)
    S.close()
    ds.close()
    ctx.close()
