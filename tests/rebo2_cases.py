"""Inputs of the REBO-II extension tests: synthetic spline knots and two
carbon configurations.  The published REBO-II tables are not in this
repository, so the knots are seeded random numbers of the tables' scale
(values a few hundredths, slopes smaller), smooth by construction (cubic
Hermite through values and derivatives).

* ``cluster``: one "molecule" of random carbon atoms in a small periodic box
  with 1-6 neighbours within the REBO cutoff, so every part of the bond
  order is active: N off the integers and beyond the table, the conjugation
  switch F(x) between 2 and 3, bonds in the cutoff switch.
* ``crystal``: an FCC C60 crystal with jittered atoms and a compressed cell,
  with many intermolecular pairs closer than 2^(1/6) sigma (the switched-LJ
  range) and bond orders b* around the switch window 0.77-0.81."""
from __future__ import annotations

import numpy as np

from fuller_md_en_b200 import Rebo2Knots, crystal


def random_knots(seed: int, pirc_shift: float = -0.05) -> Rebo2Knots:
    rng = np.random.default_rng(seed)
    pcc = np.zeros((5, 2))
    pcc[:, 0] = rng.uniform(-0.05, 0.05, 5)
    pcc[:, 1] = rng.uniform(-0.03, 0.03, 5)

    def tri(shift, amp):
        t = np.zeros((5, 5, 10, 8))
        t[..., 0] = rng.uniform(-amp, amp, (5, 5, 10)) + shift
        t[..., 1:4] = rng.uniform(-0.6 * amp, 0.6 * amp, (5, 5, 10, 3))
        t[..., 4:] = rng.uniform(-0.3 * amp, 0.3 * amp, (5, 5, 10, 4))
        return t

    return Rebo2Knots(pcc, tri(pirc_shift, 0.03), tri(0.0, 0.01))


def oracle_knots(k: Rebo2Knots):
    from oracle.fmd_oracle import Rebo2Knots as OK
    return OK.of(k.pcc, k.pirc, k.tcc)


def cluster(seed: int = 11, n: int = 64, edge: float = 9.0, dmin: float = 1.25) -> dict:
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < n:
        p = rng.uniform(0.0, edge, 3)
        if all(np.linalg.norm((p - q) - edge * np.round((p - q) / edge)) >= dmin for q in pts):
            pts.append(p)
    h = np.diag([edge, edge, edge]).reshape(-1).astype(np.float64)
    return {"pos": np.array(pts).reshape(-1), "h": h, "hi": crystal.inv9(h), "mol_id": np.zeros(n, np.int32),
            "na": n}


def crystal_case(seed: int = 7, jitter: float = 0.1, scale: float = 0.95) -> dict:
    s = crystal.atomistic(1, jitter=jitter, seed=seed, init_scale=scale)
    s["na"] = s["pos"].size // 3
    return s


def lists(oracle, s: dict, rc_lj: float = 3.0 * 3.4 + 1.0):
    """REBO rows (width 12, cutoff 2.3) and LJ half rows (width 400)."""
    na = s["na"]
    cr, lr, dr = oracle.nlist_intra(s["pos"], s["h"], s["hi"], na, s["mol_id"])
    cl, ll, dl = oracle.nlist_half(s["pos"], s["h"], s["hi"], na, s["mol_id"], rc_lj)
    assert dr == 0 and dl == 0
    return cr, lr, cl, ll


def strained(s: dict, a: int, b: int, eps: float):
    """Positions and cell under the homogeneous strain I + eps e_a e_b^T."""
    m = np.eye(3)
    m[a, b] += eps
    h = (m @ s["h"].reshape(3, 3)).reshape(-1)
    pos = (s["pos"].reshape(-1, 3) @ m.T).reshape(-1)
    return pos, h, crystal.inv9(h)
