"""Host-side set-up of synthetic fullerene crystals (not on the hot path).

* ``c60_ih(bond66, bond56)``: an icosahedral C60 built from the icosahedron
  by truncating every edge at fraction t, with t and the edge length chosen so
  the hexagon-hexagon (6:6) and pentagon-hexagon (5:6) bonds have the
  requested lengths (t*e = b56, (1-2t)*e = b66).
* lattice builders with the reference's site order (make_fcc/hcp/bcc,
  LJ:229-250) and default lattice constant (default_a0, LJ:251-254);
* atomistic and rigid-body systems with seeded velocities, quaternions and
  optional Gaussian jitter.

Velocities here use numpy's generator (synthetic inputs); the C++ drivers
reproduce the reference's std::mt19937 streams exactly.
"""
from __future__ import annotations

import math

import numpy as np

CONV = 9.64853321e-3
KB = 8.617333262e-5
MC = 12.011


def c60_ih(bond66: float = 1.39, bond56: float = 1.45) -> np.ndarray:
    """60 x 3 coordinates (centred) of an Ih C60 with the given bond lengths."""
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    ico = []
    for s1 in (-1.0, 1.0):
        for s2 in (-1.0, 1.0):
            ico += [(0.0, s1, s2 * phi), (s1, s2 * phi, 0.0), (s2 * phi, 0.0, s1)]
    ico = np.array(ico)
    d = np.linalg.norm(ico[:, None, :] - ico[None, :, :], axis=-1)
    edges = [(a, b) for a in range(12) for b in range(12) if a != b and abs(d[a, b] - 2.0) < 1e-9]
    # t e = b56 and (1 - 2t) e = b66  =>  t = b56 / (b66 + 2 b56)
    t = bond56 / (bond66 + 2.0 * bond56)
    e = bond56 / t
    pts = np.array([ico[a] + t * (ico[b] - ico[a]) for a, b in edges]) * (e / 2.0)
    pts -= pts.mean(axis=0)
    return pts


def bonds_from_geometry(coords: np.ndarray, cutoff: float = 1.6) -> np.ndarray:
    """Sorted unique (lo, hi) bond pairs closer than cutoff (as load_cc1 builds
    from the adjacency columns, MM:180-182)."""
    n = len(coords)
    out = []
    for i in range(n):
        for j in range(i + 1, n):
            if np.linalg.norm(coords[i] - coords[j]) < cutoff:
                out.append((i, j))
    return np.array(out, dtype=np.int32)


def mol_extent(coords: np.ndarray) -> tuple[float, float]:
    """(Rmol, Dmol) as load_cc1 computes them (LJ:194-200)."""
    r = np.sqrt((coords ** 2).sum(axis=1)).max()
    dm = np.sqrt(((coords[:, None, :] - coords[None, :, :]) ** 2).sum(-1)).max()
    return float(r), float(dm)


def default_a0(dmax: float, st: str = "FCC", s: float = 1.0) -> float:
    m = 1.4
    if st == "FCC":
        a0 = dmax * math.sqrt(2.0) * m
    elif st == "HCP":
        a0 = dmax * m
    else:
        a0 = dmax * 2.0 / math.sqrt(3.0) * m
    return a0 * s


def make_lattice(st: str, a: float, nc: int) -> tuple[np.ndarray, np.ndarray]:
    """Centres and cell matrix in the reference's order (LJ:229-250)."""
    pos = []
    h = np.zeros(9)
    if st == "FCC":
        bas = [(0, 0, 0), (.5 * a, .5 * a, 0), (.5 * a, 0, .5 * a), (0, .5 * a, .5 * a)]
        for x in range(nc):
            for y in range(nc):
                for z in range(nc):
                    for b in bas:
                        pos.append((a * x + b[0], a * y + b[1], a * z + b[2]))
        h[0] = h[4] = h[8] = nc * a
    elif st == "HCP":
        c = a * math.sqrt(8.0 / 3.0)
        a1, a2, a3 = (a, 0, 0), (a / 2, a * math.sqrt(3.0) / 2, 0), (0, 0, c)
        for x in range(nc):
            for y in range(nc):
                for z in range(nc):
                    for b in ((0, 0, 0), (1.0 / 3, 2.0 / 3, 0.5)):
                        fx, fy, fz = x + b[0], y + b[1], z + b[2]
                        pos.append(tuple(fx * a1[k] + fy * a2[k] + fz * a3[k] for k in range(3)))
        h[0] = nc * a1[0]; h[3] = nc * a1[1]; h[1] = nc * a2[0]; h[4] = nc * a2[1]; h[8] = nc * a3[2]
    else:
        for x in range(nc):
            for y in range(nc):
                for z in range(nc):
                    for b in ((0, 0, 0), (.5 * a, .5 * a, .5 * a)):
                        pos.append((a * x + b[0], a * y + b[1], a * z + b[2]))
        h[0] = h[4] = h[8] = nc * a
    return np.array(pos, dtype=np.float64), h


def inv9(h: np.ndarray) -> np.ndarray:
    """mat_inv9 with the reference's expression order (LJ:120-124)."""
    d = h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) + h[2] * (h[3] * h[7] - h[4] * h[6])
    i = 1.0 / d
    return np.array([i * (h[4] * h[8] - h[5] * h[7]), i * (h[2] * h[7] - h[1] * h[8]), i * (h[1] * h[5] - h[2] * h[4]),
                     i * (h[5] * h[6] - h[3] * h[8]), i * (h[0] * h[8] - h[2] * h[6]), i * (h[2] * h[3] - h[0] * h[5]),
                     i * (h[3] * h[7] - h[4] * h[6]), i * (h[1] * h[6] - h[0] * h[7]), i * (h[0] * h[4] - h[1] * h[3])])


def npt_atom(T: float, Pe: float, na: int) -> np.ndarray:
    """make_npt (AI:512-515) as {xi, Q, Vg[9], W, Pe, Tt, Nf}."""
    nf = 3 * na - 3
    Q = max(nf * KB * T * 100.0 * 100.0, 1e-20)
    W = max((nf + 9) * KB * T * 1000.0 * 1000.0, 1e-20)
    return np.array([0.0, Q] + [0.0] * 9 + [W, Pe, T, float(nf)])


def npt_rigid(T: float, Pe: float, n: int) -> np.ndarray:
    """make_npt (LJ:426-431)."""
    nf = 6 * n - 3
    Q = max(nf * KB * T * 100.0 * 100.0, 1e-20)
    W = max((nf + 9) * KB * T * 1000.0 * 1000.0, 1e-20)
    return np.array([0.0, Q] + [0.0] * 9 + [W, Pe, T, float(nf)])


def atomistic(nc: int, coords: np.ndarray | None = None, T: float = 300.0, seed: int = 42, jitter: float = 0.0,
              st: str = "FCC", init_scale: float = 1.0, mol_base: int = 1):
    """Flexible-atom crystal as the AIREBO/MM drivers build it (AI:781-786):
    every molecule a translated copy, mol_id = m + mol_base."""
    if coords is None:
        coords = c60_ih()
    natom = len(coords)
    _, dmol = mol_extent(coords)
    a0 = default_a0(dmol, st, init_scale)
    centres, h = make_lattice(st, a0, nc)
    nmol = len(centres)
    pos = (centres[:, None, :] + coords[None, :, :]).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    if jitter > 0:
        pos = pos + rng.normal(0.0, jitter, size=pos.shape)
    na = len(pos)
    mass = np.full(na, MC)
    mol_id = np.repeat(np.arange(nmol, dtype=np.int32) + mol_base, natom)
    sv = math.sqrt(KB * T * CONV / MC)
    vel = sv * rng.normal(size=(na, 3))
    vel -= vel.mean(axis=0)
    return {"pos": pos.reshape(-1).copy(), "vel": vel.reshape(-1).copy(), "mass": mass, "mol_id": mol_id,
            "h": h, "hi": inv9(h), "nmol": nmol, "natom": natom, "a0": a0}


def rigid(nc: int, coords: np.ndarray | None = None, T: float = 300.0, seed: int = 42, st: str = "FCC",
          a0: float | None = None, init_scale: float = 1.0):
    """Rigid-body crystal as the LJ driver builds it (LJ:754-801)."""
    if coords is None:
        coords = c60_ih()
    natom = len(coords)
    rmol, dmol = mol_extent(coords)
    if a0 is None:
        a0 = default_a0(dmol, st, init_scale)
    centres, h = make_lattice(st, a0, nc)
    n = len(centres)
    r2 = (coords ** 2).sum(axis=1)
    i0 = float((MC * (r2[:, None] - coords ** 2)).sum(axis=0).sum() / 3.0)
    mmol = natom * MC
    rng = np.random.default_rng(seed)
    sv = math.sqrt(KB * T * CONV / mmol)
    sw = math.sqrt(KB * T * CONV / i0)
    vel = sv * rng.normal(size=(n, 3))
    omg = sw * rng.normal(size=(n, 3))
    qv = rng.normal(size=(n, 4))
    qv /= np.linalg.norm(qv, axis=1, keepdims=True)
    vel -= vel.mean(axis=0)
    return {"pos": centres.reshape(-1).copy(), "vel": vel.reshape(-1).copy(), "omg": omg.reshape(-1).copy(),
            "qv": qv.reshape(-1).copy(), "body": coords.reshape(-1).copy(), "h": h, "hi": inv9(h), "n": n,
            "natom": natom, "I0": i0, "Mmol": mmol, "Rmol": rmol, "a0": a0}


KCAL2EV = 1.0 / 23.06054783          # MM:111


def _dihedral0(c, i, j, k, l) -> float:
    """Reference dihedral angle of four atoms (MM:240-252)."""
    b1 = [c[j][a] - c[i][a] for a in range(3)]
    b2 = [c[k][a] - c[j][a] for a in range(3)]
    b3 = [c[l][a] - c[k][a] for a in range(3)]
    mx, my, mz = b1[1] * b2[2] - b1[2] * b2[1], b1[2] * b2[0] - b1[0] * b2[2], b1[0] * b2[1] - b1[1] * b2[0]
    nx, ny, nz = b2[1] * b3[2] - b2[2] * b3[1], b2[2] * b3[0] - b2[0] * b3[2], b2[0] * b3[1] - b2[1] * b3[0]
    mm, nn = mx * mx + my * my + mz * mz, nx * nx + ny * ny + nz * nz
    if mm < 1e-20 or nn < 1e-20:
        return 0.0
    b2len = math.sqrt(b2[0] * b2[0] + b2[1] * b2[1] + b2[2] * b2[2])
    cp = (mx * nx + my * ny + mz * nz) / math.sqrt(mm * nn)
    cp = min(max(cp, -1.0), 1.0)
    sp = (mx * b3[0] + my * b3[1] + mz * b3[2]) * b2len / math.sqrt(mm * nn)
    return math.atan2(sp, cp)


def mm_topology(coords: np.ndarray, bonds: np.ndarray, nmol: int, kb: float = 469.0, kth: float = 63.0,
                v2: float = 14.5, kimp: float = 15.0) -> dict:
    """Flat MM topology of nmol copies of one molecule (build_flat_topology,
    MM:254-334): bonds from the sorted bond pairs with r0 from the geometry,
    angles i-j-k over each atom's neighbour pairs, dihedrals i-j-k-l over each
    bond, impropers on three-coordinated atoms, gamma = 2 phi0 + pi; force
    constants in kcal/mol converted to eV; copy m offsets indices by m natom."""
    c = [tuple(float(x) for x in row) for row in np.asarray(coords, np.float64).reshape(-1, 3)]
    na = len(c)
    bl = [(int(a), int(b)) for a, b in np.asarray(bonds, np.int64).reshape(-1, 2)]
    adj = [[] for _ in range(na)]
    for a, b in bl:
        adj[a].append(b)
        adj[b].append(a)
    # sqrt of the same left-to-right sum of squares as the reference
    br0 = [math.sqrt((c[a][0] - c[b][0]) * (c[a][0] - c[b][0]) + (c[a][1] - c[b][1]) * (c[a][1] - c[b][1]) +
                     (c[a][2] - c[b][2]) * (c[a][2] - c[b][2])) for a, b in bl]
    an, ath = [], []
    for j in range(na):
        for ii in range(len(adj[j])):
            for kk in range(ii + 1, len(adj[j])):
                i, k = adj[j][ii], adj[j][kk]
                u = [c[i][q] - c[j][q] for q in range(3)]
                v = [c[k][q] - c[j][q] for q in range(3)]
                du = math.sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
                dv = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
                ct = min(max((u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) / (du * dv), -1.0), 1.0)
                an.append((i, j, k))
                ath.append(math.acos(ct))
    dh, dg = [], []
    for bj, bk in bl:
        for i in adj[bj]:
            if i == bk:
                continue
            for l in adj[bk]:
                if l == bj or l == i:
                    continue
                dh.append((i, bj, bk, l))
                dg.append(2 * _dihedral0(c, i, bj, bk, l) + math.pi)
    im, ig = [], []
    for i in range(na):
        if len(adj[i]) == 3:
            j, k, l = adj[i]
            im.append((i, j, k, l))
            ig.append(2 * _dihedral0(c, j, i, k, l) + math.pi)
    shift = (np.arange(nmol, dtype=np.int32) * na)[:, None, None]

    def rep(a):                                      # copy m: indices + m na, copies in order
        base = np.asarray(a, np.int32).reshape(1, len(a), -1)
        return (base + shift).reshape(-1, base.shape[2]) if len(a) else np.zeros((0, 2), np.int32)

    tile = lambda a: np.tile(np.asarray(a, np.float64), nmol)
    return {"bonds": rep(bl), "kb": np.full(len(bl) * nmol, kb * KCAL2EV), "r0": tile(br0),
            "angles": rep(an), "kth": np.full(len(an) * nmol, kth * KCAL2EV), "th0": tile(ath),
            "dihedrals": rep(dh), "vn": np.full(len(dh) * nmol, v2 * KCAL2EV),
            "mult": np.full(len(dh) * nmol, 2, np.int32), "gamma": tile(dg),
            "impropers": rep(im), "ki": np.full(len(im) * nmol, kimp * KCAL2EV), "igamma": tile(ig),
            "mol_id": np.repeat(np.arange(nmol, dtype=np.int32), na)}
