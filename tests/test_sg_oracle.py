"""The CPU restatement of the learned bond-order potential (oracle/sg_oracle.py).

1. With the reference's own bond order and its derivative, the assembly
   reproduces compute_rebo of the C oracle (pinned to the reference).
2. The gradient network (db/dx) and the double-backpropagation weight
   gradients agree with central finite differences in FP64.
"""
from __future__ import annotations

import numpy as np
import pytest

from fuller_md_en_b200 import crystal
from oracle import sg_oracle as sg


@pytest.fixture(scope="module")
def snap(oracle):
    s = crystal.atomistic(1, T=300.0, seed=5, jitter=0.03)
    na = s["pos"].size // 3
    pos = s["pos"].copy()
    oracle.apply_pbc(pos, s["h"], s["hi"])
    cnt, lst, _ = oracle.nlist_intra(pos, s["h"], s["hi"], na, s["mol_id"])
    E, F, W = oracle.rebo(pos, s["h"], s["hi"], cnt, lst, na)
    g = sg.rows(pos, s["h"], s["hi"], cnt, lst)
    return dict(pos=pos, h=s["h"], hi=s["hi"], cnt=cnt, lst=lst, E=E, F=F, W=W, g=g, na=na)


def test_rows_cover_every_bond(snap):
    g = snap["g"]
    assert len(g["i"]) == 3 * snap["na"]          # C60: three bonds per atom
    assert np.all(g["i"][g["partner"]] == g["j"]) and np.all(g["j"][g["partner"]] == g["i"])
    assert len(g["srow"]) == 2 * len(g["i"])      # two other neighbours per row


def test_assembly_with_reference_bond_order_matches_rebo(snap):
    g = snap["g"]
    E, F, W = sg.assemble(g, sg.exact_bond_order(g), sg.exact_dbdk(g))
    assert abs(E - snap["E"]) <= 1e-10 * abs(snap["E"])
    np.testing.assert_allclose(F, snap["F"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(W, snap["W"], rtol=0, atol=1e-9)


def test_descriptor_jacobian_finite_difference(snap):
    g = snap["g"]
    X, J = sg.descriptors(g)
    rng = np.random.default_rng(1)
    for s in rng.choice(len(g["srow"]), 6, replace=False):
        for a in range(3):
            gp = dict(g); gm = dict(g)
            gp["dk"] = g["dk"].copy(); gm["dk"] = g["dk"].copy()
            gp["dk"][s, a] += 1e-6; gm["dk"][s, a] -= 1e-6
            gp["rk"] = np.sqrt((gp["dk"] ** 2).sum(1)); gm["rk"] = np.sqrt((gm["dk"] ** 2).sum(1))
            fd = (sg.descriptors(gp)[0] - sg.descriptors(gm)[0])[g["srow"][s]] / 2e-6
            np.testing.assert_allclose(J[s, :, a], fd, rtol=1e-5, atol=1e-7)


def _params(snap):
    P = sg.init_params(3)
    X, _ = sg.descriptors(snap["g"])
    P["m"] = X.mean(0); P["s"] = X.std(0) + 1e-3
    P["b0"], P["bs"] = 0.88, 0.08
    return P


def test_gradient_network_finite_difference(snap):
    P = _params(snap)
    X, _ = sg.descriptors(snap["g"])
    Xn = sg.normalise(X, P["m"], P["s"])[:40]
    b, c = sg.mlp(P, Xn)
    gx = sg.mlp_grad(P, c)
    for f in range(sg.D - 1):
        e = np.zeros(sg.D); e[f] = 1e-6
        fd = (sg.mlp(P, Xn + e)[0] - sg.mlp(P, Xn - e)[0]) / 2e-6
        np.testing.assert_allclose(gx[:, f], fd, rtol=1e-6, atol=1e-9)


def test_weight_gradients_finite_difference(snap):
    P = _params(snap)
    g = snap["g"]
    Et, Ft, Wt = snap["E"], snap["F"], snap["W"]
    L, grads, _, _, _ = sg.loss_and_grad(P, g, Et, Ft, Wt, wE=0.3, wF=1.0, wW=0.2)
    rng = np.random.default_rng(7)
    checked = 0
    for key, shape in (("W1", (sg.D, sg.H)), ("W2", (sg.H, sg.H)), ("W3", (sg.H, sg.H)), ("w4", (sg.H,))):
        for _ in range(5):
            idx = tuple(int(rng.integers(0, n)) for n in shape)
            if key == "w4" and checked == 0:
                idx = (sg.H - 1,)                 # the output bias
            Pp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in P.items()}
            Pm = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in P.items()}
            h = 1e-5
            Pp[key][idx] += h; Pm[key][idx] -= h
            Lp = sg.loss_and_grad(Pp, g, Et, Ft, Wt, wE=0.3, wF=1.0, wW=0.2)[0]
            Lm = sg.loss_and_grad(Pm, g, Et, Ft, Wt, wE=0.3, wF=1.0, wW=0.2)[0]
            fd = (Lp - Lm) / (2 * h)
            an = grads[key][idx]
            assert abs(an - fd) <= 1e-5 * max(1.0, abs(fd)) + 1e-7, (key, idx, an, fd)
            checked += 1
    assert checked == 20
