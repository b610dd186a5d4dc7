"""The reference drivers' step loop (LJ:847-897, AI:871-912, MM:1192-1236)
restated over the CPU oracle, to check the device-resident systems, which run
the same loop on the GPU.  Test infrastructure."""
from __future__ import annotations

import math

import numpy as np

KB = 8.617333262e-5
EV2GPA = 160.21766208
CONV = 9.64853321e-3
MC = 12.011


def inst_T(ke, nf):
    return 2 * ke / (nf * KB)


def inst_P(W, ke, V):
    return (2 * ke + W[0] + W[4] + W[8]) / (3 * V) * EV2GPA


def det9(h):
    return h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) + h[2] * (h[3] * h[7] - h[4] * h[6])


def schedule(npt, g, T, T_cold, coldstart, warmup):
    if g <= coldstart:
        npt[13] = T_cold
    elif g <= coldstart + warmup:
        npt[13] = T_cold + (T - T_cold) * float(g - coldstart) / float(warmup)
    else:
        npt[13] = T
    if coldstart > 0 and g == coldstart + 1:
        npt[0] = 0.0
        npt[2:11] = 0.0
    if g <= coldstart:
        npt[2:11] = 0.0


def run_airebo(O, st, first, last, dt, T, T_cold, coldstart, warmup, nlup=20, nc=1, nmol=1, lists=None):
    """Runs steps first..last on state dict st (pos, vel, F, vir9, h, hi, mass,
    npt, mol_id); returns per-step observables [(g, Tn, Pn, an, Ep, Er, El)]."""
    na = st["pos"].size // 3
    obs = []
    for g in range(first, last + 1):
        schedule(st["npt"], g, T, T_cold, coldstart, warmup)
        if g % nlup == 0 or lists is None:
            st["hi"][:] = O.mat_inv9(st["h"])
            cr, lr, _ = O.nlist_intra(st["pos"], st["h"], st["hi"], na, st["mol_id"])
            cl, ll, _ = O.nlist_half(st["pos"], st["h"], st["hi"], na, st["mol_id"], 3.0 * 3.40 + 2.0)
            lists = (cr, lr, cl, ll)
        out = O.airebo_step(st, dt, *lists)
        nf = int(st["npt"][14])
        KE = out[3]
        V = abs(det9(st["h"]))
        Tn, Pn = inst_T(KE, nf), inst_P(st["vir9"], KE, V)
        if (g <= coldstart or g <= coldstart + warmup) and Tn > 0.1:
            tgt = T_cold if g <= coldstart else st["npt"][13]
            scale = math.sqrt(max(tgt, 0.1) / Tn)
            st["vel"] *= scale
            v = st["vel"].reshape(-1, 3)
            KE = 0.5 * float(np.sum(st["mass"] * np.sum(v * v, axis=1))) / CONV
            Tn = inst_T(KE, nf)
            st["npt"][0] = 0.0
            if g <= coldstart:
                st["npt"][2:11] = 0.0
        obs.append((g, Tn, Pn, st["h"][0] / nc, out[0], out[1], out[2]))
    return obs, lists


def run_rigid(O, st, first, last, dt, T, T_cold, coldstart, warmup, body, I0, Mmol, natom, rmcut, nlup=25, nc=1,
              lists=None):
    n = st["pos"].size // 3
    obs = []
    for g in range(first, last + 1):
        schedule(st["npt"], g, T, T_cold, coldstart, warmup)
        if g % nlup == 0 or lists is None:
            st["hi"][:] = O.mat_inv9(st["h"])
            c, l, _ = O.nlist_sym(st["pos"], st["h"], st["hi"], n, rmcut)
            lists = (c, l)
        Ep, KE = O.rigid_step(st, body, I0, Mmol, natom, rmcut * rmcut, dt, *lists)
        v = st["vel"].reshape(-1, 3)
        kt = 0.5 * Mmol * float(np.sum(v * v)) / CONV
        nf = int(st["npt"][14])
        V = abs(det9(st["h"]))
        Tn, Pn = inst_T(KE, nf), inst_P(st["W9"], kt, V)
        if (g <= coldstart or g <= coldstart + warmup) and Tn > 0.1:
            tgt = T_cold if g <= coldstart else st["npt"][13]
            scale = math.sqrt(max(tgt, 0.1) / Tn)
            st["vel"] *= scale
            st["omg"] *= scale
            v = st["vel"].reshape(-1, 3)
            w = st["omg"].reshape(-1, 3)
            kt = 0.5 * Mmol * float(np.sum(v * v)) / CONV
            KE = kt + 0.5 * I0 * float(np.sum(w * w)) / CONV
            Tn = inst_T(KE, nf)
            st["npt"][0] = 0.0
            if g <= coldstart:
                st["npt"][2:11] = 0.0
        obs.append((g, Tn, Pn, st["h"][0] / nc, Ep))
    return obs, lists


def run_mm(O, st, first, last, dt, T, T_cold, coldstart, warmup, topo, nlup=20, nc=1, lists=None):
    na = st["pos"].size // 3
    obs = []
    for g in range(first, last + 1):
        schedule(st["npt"], g, T, T_cold, coldstart, warmup)
        if g % nlup == 0 or lists is None:
            st["hi"][:] = O.mat_inv9(st["h"])
            c, l, _ = O.nlist_half(st["pos"], st["h"], st["hi"], na, topo["mol_id"], 3.0 * 3.431 + 2.0)
            lists = (c, l)
        out = O.mm_step(st, dt, topo, *lists)
        KE = out[7]
        nf = int(st["npt"][14])
        V = abs(det9(st["h"]))
        Tn, Pn = inst_T(KE, nf), inst_P(st["vir9"], KE, V)
        if (g <= coldstart or g <= coldstart + warmup) and Tn > 0.1:
            tgt = T_cold if g <= coldstart else st["npt"][13]
            scale = math.sqrt(max(tgt, 0.1) / Tn)
            st["vel"] *= scale
            v = st["vel"].reshape(-1, 3)
            KE = 0.5 * float(np.sum(MC * np.sum(v * v, axis=1))) / CONV
            Tn = inst_T(KE, nf)
            st["npt"][0] = 0.0
            if g <= coldstart:
                st["npt"][2:11] = 0.0
        obs.append((g, Tn, Pn, st["h"][0] / nc, *out[:7]))
    return obs, lists
