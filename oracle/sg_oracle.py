"""CPU FP64 restatement of the learned bond-order potential (test
infrastructure: only tests and the benchmark's checker import this).

The surrogate has no counterpart in the reference.  It stands in for the
bond order b_ij of compute_rebo (fuller_airebo_npt_md_serial_omp_acc.cpp,
AI:275-421) and keeps the rest of that routine: the pair functions fc, VR,
VA (AI:164-181), b_bar = (b_ij + b_ji)/2, the pair force and pair virial,
and the reference's construction of the three-body force, in which
F_k += -1/2 fc(r_ij) VA(r_ij) db_ij/dr_k and F_i -= the same (AI:368-390;
the reference writes db/dr_k as dbp * dG_ij/dr_k).  Only b_ij and
db_ij/dr_k come from the network.

Row = directed bond (i -> j): j in i's REBO list with r_ij <= 2.0.
Descriptor of a row (D = 32): x[a*8+b] = sum over the other list
neighbours k of i with r_ik <= 2.0 and fc(r_ik) >= 1e-15 of
fc(r_ik) T_a(rho(r_ik)) T_b(cos theta_jik), a < 4, b < 8, rho(r) =
(r - 1.55)/0.45, T_n Chebyshev polynomials; feature 31 (a=3, b=7) is
replaced by the constant 1 after normalisation (the first layer's bias).
Network: x_n = (x - m)/s; h_l = SiLU(h_{l-1} W_l) for l = 1..3, each with
128 columns of which column 127 is held at 1 (the next layer's bias);
y = h_3 . w_4; b = b0 + bs * y.  The GPU evaluates the same network with
BF16 operands and FP32 accumulation; ``rnd=True`` rounds the same
operands to BF16 here.

The weight gradient of a loss on energies, forces and virials needs the
derivative of db/dx with respect to the weights (double backpropagation);
``mlp_backward`` restates it step by step, as the GPU kernels do.
"""
from __future__ import annotations

import math

import numpy as np

D, H, NR, NA = 32, 128, 4, 8
DMIN, DMAX = 1.7, 2.0
Q_CC, A_CC, ALPHA = 0.3134602960833, 10953.544162170, 4.7465390606595
B1, BETA1 = 12388.79197798, 4.7204523127
B2, BETA2 = 17.56740646509, 1.4332132499
B3, BETA3 = 30.71493208065, 1.3826912506


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64).reshape(np.shape(x))


def fc(r):
    return np.where(r <= DMIN, 1.0, np.where(r >= DMAX, 0.0, 0.5 * (1.0 + np.cos(np.pi * (r - DMIN) / (DMAX - DMIN)))))


def dfc(r):
    inside = (r > DMIN) & (r < DMAX)
    return np.where(inside, -0.5 * np.pi / (DMAX - DMIN) * np.sin(np.pi * (r - DMIN) / (DMAX - DMIN)), 0.0)


def vr(r):
    return (1.0 + Q_CC / r) * A_CC * np.exp(-ALPHA * r)


def dvr(r):
    ex = A_CC * np.exp(-ALPHA * r)
    return (-Q_CC / (r * r)) * ex + (1.0 + Q_CC / r) * (-ALPHA) * ex


def va(r):
    return B1 * np.exp(-BETA1 * r) + B2 * np.exp(-BETA2 * r) + B3 * np.exp(-BETA3 * r)


def dva(r):
    return -BETA1 * B1 * np.exp(-BETA1 * r) - BETA2 * B2 * np.exp(-BETA2 * r) - BETA3 * B3 * np.exp(-BETA3 * r)


def cheb(x, n):
    """T_0..T_{n-1}(x) and their derivatives, shape (..., n)."""
    T = [np.ones_like(x), x]
    dT = [np.zeros_like(x), np.ones_like(x)]
    for _ in range(2, n):
        T.append(2 * x * T[-1] - T[-2])
        dT.append(2 * T[-2] + 2 * x * dT[-1] - dT[-2])
    return np.stack(T[:n], -1), np.stack(dT[:n], -1)


def mimg(d, h, hi):
    """mimg9 (AI:144-147) for an array of vectors."""
    h = np.asarray(h).reshape(3, 3); hi = np.asarray(hi).reshape(3, 3)
    s = d @ hi.T
    s = s - np.round(s)
    return s @ h.T


def rows(pos, h, hi, cnt, lst, cap=12):
    """Directed bonds and their three-body slots (the loops of AI:289-322)."""
    pos = np.asarray(pos).reshape(-1, 3)
    lst = np.asarray(lst).reshape(len(cnt), cap)
    ri, rj, rs = [], [], []
    for i in range(len(cnt)):
        for jn in range(cnt[i]):
            ri.append(i); rj.append(lst[i, jn]); rs.append(jn)
    ri = np.array(ri, np.int64); rj = np.array(rj, np.int64); rs = np.array(rs, np.int64)
    d = mimg(pos[rj] - pos[ri], h, hi)
    r = np.sqrt((d * d).sum(1))
    keep = r <= DMAX
    ri, rj, rs, d, r = ri[keep], rj[keep], rs[keep], d[keep], r[keep]
    index = {(int(a), int(b)): q for q, (a, b) in enumerate(zip(ri, rj))}
    partner = np.array([index[(int(b), int(a))] for a, b in zip(ri, rj)], np.int64)
    srow, sk = [], []
    for q in range(len(ri)):
        i = ri[q]
        for kn in range(cnt[i]):
            k = lst[i, kn]
            if k != rj[q]:
                srow.append(q); sk.append(k)
    srow = np.array(srow, np.int64); sk = np.array(sk, np.int64)
    dk = mimg(pos[sk] - pos[ri[srow]], h, hi) if len(sk) else np.zeros((0, 3))
    rk = np.sqrt((dk * dk).sum(1))
    ok = (rk <= DMAX) & (fc(rk) >= 1e-15)
    return dict(i=ri, j=rj, d=d, r=r, partner=partner, srow=srow[ok], k=sk[ok], dk=dk[ok], rk=rk[ok], na=len(cnt))


def descriptors(g):
    """Raw features (R x D, column 31 zero) and their Jacobian with respect to
    r_k for every slot (S x D x 3)."""
    R = len(g["i"])
    d = g["d"][g["srow"]]; r = g["r"][g["srow"]]
    dk, rk = g["dk"], g["rk"]
    c = np.clip((d * dk).sum(1) / (r * rk), -1.0, 1.0)
    rho = (rk - 1.55) / 0.45
    Tr, dTr = cheb(rho, NR)
    Ta, dTa = cheb(c, NA)
    f, df = fc(rk), dfc(rk)
    phi = f[:, None] * Tr                                  # S x NR
    dphi = df[:, None] * Tr + f[:, None] * dTr / 0.45      # d phi / d r_k
    feat = (phi[:, :, None] * Ta[:, None, :]).reshape(-1, D)
    feat[:, D - 1] = 0.0
    X = np.zeros((R, D))
    np.add.at(X, g["srow"], feat)
    rhat_k = dk / rk[:, None]
    rhat_j = d / r[:, None]
    dc = (rhat_j - c[:, None] * rhat_k) / rk[:, None]      # d cos / d r_k (AI:385)
    J = (dphi[:, :, None, None] * Ta[:, None, :, None] * rhat_k[:, None, None, :]
         + phi[:, :, None, None] * dTa[:, None, :, None] * dc[:, None, None, :]).reshape(-1, D, 3)
    J[:, D - 1, :] = 0.0
    return X, J


def normalise(X, m, s):
    Xn = (X - m) / s
    Xn[:, D - 1] = 1.0
    return Xn


def silu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s)), s * (1.0 - s) * (2.0 + z * (1.0 - 2.0 * s))


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    P = dict(W1=rng.normal(0, 1 / math.sqrt(D), (D, H)), W2=rng.normal(0, 1 / math.sqrt(H), (H, H)),
             W3=rng.normal(0, 1 / math.sqrt(H), (H, H)), w4=rng.normal(0, 1 / math.sqrt(H), H),
             m=np.zeros(D), s=np.ones(D), b0=0.0, bs=1.0)
    for k in ("W1",):
        P[k][D - 1, :] = 0.0
    for k in ("W2", "W3"):
        P[k][H - 1, :] = 0.0
    P["w4"][H - 1] = 0.0
    return P


def mlp(P, Xn, rnd=False):
    R = (lambda a: bf16(a)) if rnd else (lambda a: a)
    c = {}
    x = R(Xn)
    c["x"] = x
    a = x
    for l, W in ((1, P["W1"]), (2, P["W2"]), (3, P["W3"])):
        z = a @ R(W)
        hval, s1, s2 = silu(z)
        hval[:, H - 1] = 1.0
        c[f"z{l}"], c[f"s{l}"], c[f"q{l}"] = z, s1, s2
        c[f"h{l}"] = R(hval) if l < 3 else hval
        a = c[f"h{l}"]
    y = c["h3"] @ P["w4"]
    return P["b0"] + P["bs"] * y, c


def mlp_grad(P, c, rnd=False):
    """gx = db/dx_n (R x D) through the gradient network."""
    R = (lambda a: bf16(a)) if rnd else (lambda a: a)
    g3 = P["bs"] * P["w4"][None, :] * c["s3"]
    g3[:, H - 1] = 0.0
    c["g3"] = R(g3)
    t2 = c["g3"] @ R(P["W3"]).T
    g2 = t2 * c["s2"]; g2[:, H - 1] = 0.0
    c["t2"], c["g2"] = t2, R(g2)
    t1 = c["g2"] @ R(P["W2"]).T
    g1 = t1 * c["s1"]; g1[:, H - 1] = 0.0
    c["t1"], c["g1"] = t1, R(g1)
    gx = c["g1"] @ R(P["W1"]).T
    gx[:, D - 1] = 0.0
    return gx


def dbdk_from_gx(g, J, gx, s):
    """db_row/dr_k for every slot from the network gradient gx = db/dx_n."""
    gxr = gx / s[None, :]
    gxr[:, D - 1] = 0.0
    return np.einsum("sf,sfa->sa", gxr[g["srow"]], J)


def exact_dbdk(g):
    """db_ij/dr_k of the reference bond order: dbp * dG_ij/dr_k with
    dbp = -1/2 (1+G_ij)^(-3/2) (AI:371, AI:377-385)."""
    c2, d2 = 330.0 ** 2, 3.5 ** 2
    d = g["d"][g["srow"]]; r = g["r"][g["srow"]]
    rk = g["rk"]
    cos = np.clip((d * g["dk"]).sum(1) / (r * rk), -1.0, 1.0)
    hh = 1.0 + cos
    G = 0.00020813 * (1.0 + c2 / d2 - c2 / (d2 + hh ** 2))
    dG = 0.00020813 * 2.0 * c2 * hh / (d2 + hh ** 2) ** 2
    Gs = np.zeros(len(g["i"]))
    np.add.at(Gs, g["srow"], fc(rk) * G)
    dbp = -0.5 * (1.0 + Gs) ** -1.5
    rk_hat = g["dk"] / rk[:, None]
    rj_hat = d / r[:, None]
    dG_dk = (dfc(rk) * G)[:, None] * rk_hat + (fc(rk) * dG)[:, None] * (rj_hat - cos[:, None] * rk_hat) / rk[:, None]
    return dbp[g["srow"]][:, None] * dG_dk


def assemble(g, b, dbdk):
    """Energy, forces and virial of the REBO term with a given bond order:
    compute_rebo's pair block (AI:325-365) with b_bar = (b_ij + b_ji)/2 and
    its three-body blocks (AI:368-418) with db_ij/dr_k."""
    na = g["na"]
    r, d = g["r"], g["d"]
    f, df_ = fc(r), dfc(r)
    v_r, dv_r, v_a, dv_a = vr(r), dvr(r), va(r), dva(r)
    bbar = 0.5 * (b + b[g["partner"]])
    half = g["i"] < g["j"]
    E = float((f * (v_r - bbar * v_a))[half].sum())
    fpair = (df_ * (v_r - bbar * v_a) + f * (dv_r - bbar * dv_a)) / r
    F = np.zeros((na, 3))
    fp = (fpair[:, None] * d)[half]
    np.add.at(F, g["i"][half], fp)
    np.add.at(F, g["j"][half], -fp)
    W = -(d[half][:, :, None] * d[half][:, None, :] * fpair[half][:, None, None]).sum(0).reshape(9)
    f3 = -(0.5 * f * v_a)[g["srow"]][:, None] * dbdk
    np.add.at(F, g["k"], f3)
    np.add.at(F, g["i"][g["srow"]], -f3)
    return E, F.reshape(-1), W


def loss_terms(E, F, W, Et, Ft, Wt, na, wE=1.0, wF=1.0, wW=1.0):
    """L = wF mean(dF^2) + wE (dE/na)^2 + wW mean((dW/na)^2) and its
    adjoints dL/dE, dL/dF (3na), dL/dW (9)."""
    dE, dF, dW = E - Et, F - Ft, W - Wt
    L = wF * np.mean(dF ** 2) + wE * (dE / na) ** 2 + wW * np.mean((dW / na) ** 2)
    return L, 2 * wE * dE / na ** 2, 2 * wF * dF / dF.size, 2 * wW * dW / (9 * na ** 2)


def row_adjoints(g, J, s, lamE, lamF, lamW):
    """beta = dL/db (R) and u = dL/dgx (R x D) for the assembly above."""
    r, d = g["r"], g["d"]
    f, df_ = fc(r), dfc(r)
    v_a, dv_a = va(r), dva(r)
    lam = lamF.reshape(-1, 3)
    Lm = lamW.reshape(3, 3)
    dfp = ((lam[g["i"]] - lam[g["j"]]) * d).sum(1) - np.einsum("ra,ab,rb->r", d, Lm, d)
    # both rows of a bond carry the same bond quantities; the bond's terms are
    # accumulated once (i<j row) and split evenly by b_bar
    half = g["i"] < g["j"]
    phi = -(df_ * v_a + f * dv_a) / r
    bond = np.where(half, -0.5 * f * v_a * lamE + 0.5 * phi * dfp, 0.0)
    beta = bond + bond[g["partner"]]
    w = -(0.5 * f * v_a)[g["srow"]]
    dl = lam[g["k"]] - lam[g["i"][g["srow"]]]
    us = w[:, None] * np.einsum("sfa,sa->sf", J, dl)
    u = np.zeros((len(r), D))
    np.add.at(u, g["srow"], us)
    u = u / s[None, :]
    u[:, D - 1] = 0.0
    return beta, u


def mlp_backward(P, c, beta, u, rnd=False):
    """Weight gradients of L(b(x), gx(x)) given beta = dL/db and u = dL/dgx."""
    R = (lambda a: bf16(a)) if rnd else (lambda a: a)
    W1, W2, W3, w4, bs = R(P["W1"]), R(P["W2"]), R(P["W3"]), P["w4"], P["bs"]
    last = H - 1
    ybar = beta * bs
    u = R(u)
    gb1 = u @ W1
    tb1 = gb1 * c["s1"]; tb1[:, last] = 0.0
    zd1 = gb1 * c["t1"] * c["q1"]; zd1[:, last] = 0.0
    tb1 = R(tb1)
    gb2 = tb1 @ W2
    tb2 = gb2 * c["s2"]; tb2[:, last] = 0.0
    zd2 = gb2 * c["t2"] * c["q2"]; zd2[:, last] = 0.0
    tb2 = R(tb2)
    gb3 = tb2 @ W3
    via_g3 = (bs * gb3 * c["s3"]).sum(0)
    via_g3[last] = 0.0                       # g3 of the constant unit is held at 0
    dw4 = via_g3 + (ybar[:, None] * c["h3"]).sum(0)
    z3 = gb3 * bs * w4[None, :] * c["q3"] + ybar[:, None] * w4[None, :] * c["s3"]
    z3[:, last] = 0.0
    z3 = R(z3)
    hb2 = z3 @ W3.T
    z2 = zd2 + hb2 * c["s2"]; z2[:, last] = 0.0
    z2 = R(z2)
    hb1 = z2 @ W2.T
    z1 = zd1 + hb1 * c["s1"]; z1[:, last] = 0.0
    z1 = R(z1)
    dW1 = c["x"].T @ z1 + u.T @ c["g1"]
    dW2 = c["h1"].T @ z2 + tb1.T @ c["g2"]
    dW3 = c["h2"].T @ z3 + tb2.T @ c["g3"]
    return dict(W1=dW1, W2=dW2, W3=dW3, w4=dw4)


def evaluate(P, g, rnd=False):
    X, J = descriptors(g)
    Xn = normalise(X, P["m"], P["s"])
    b, c = mlp(P, Xn, rnd)
    gx = mlp_grad(P, c, rnd)
    E, F, W = assemble(g, b, dbdk_from_gx(g, J, gx, P["s"]))
    return dict(X=X, J=J, Xn=Xn, b=b, c=c, gx=gx, E=E, F=F, W=W)


def loss_and_grad(P, g, Et, Ft, Wt, rnd=False, wE=1.0, wF=1.0, wW=1.0):
    ev = evaluate(P, g, rnd)
    L, lE, lF, lW = loss_terms(ev["E"], ev["F"], ev["W"], Et, Ft, Wt, g["na"], wE, wF, wW)
    beta, u = row_adjoints(g, ev["J"], P["s"], lE, lF, lW)
    grads = mlp_backward(P, ev["c"], beta, u, rnd)
    return L, grads, ev, beta, u


def exact_bond_order(g):
    """The reference's b_ij = (1 + sum_k fc(r_ik) G(cos))^(-1/2) (AI:302-312)
    for each row, for checks of the assembly."""
    c2, d2 = 330.0 ** 2, 3.5 ** 2
    d = g["d"][g["srow"]]; r = g["r"][g["srow"]]
    cos = np.clip((d * g["dk"]).sum(1) / (r * g["rk"]), -1.0, 1.0)
    G = 0.00020813 * (1.0 + c2 / d2 - c2 / (d2 + (1.0 + cos) ** 2))
    Gs = np.zeros(len(g["i"]))
    np.add.at(Gs, g["srow"], fc(g["rk"]) * G)
    return (1.0 + Gs) ** -0.5
