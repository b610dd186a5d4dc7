"""Generates the golden fixtures in tests/golden/ by running the UNMODIFIED
reference routines (oracle/_ref, compiled from the reference sources by
oracle/Makefile) on seeded synthetic inputs.

The reference has no golden vectors of its own (its only test checks that a
run prints "Done"), so these fixtures are its outputs recorded here.  Inputs
are synthetic C60 crystals (fuller_md_en_b200.crystal); small lists are stored
in full, large ones as SHA-256 digests of their (count, row) contents.

Run:  make -C oracle && python tests/golden/gen_golden.py
"""
from __future__ import annotations

import ctypes
import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fuller_md_en_b200 import crystal  # noqa: E402
from oracle.fmd_oracle import Ref, d, i, ref_available  # noqa: E402

OUT = Path(__file__).resolve().parent


def list_digest(cnt, lst, cap):
    hsh = hashlib.sha256()
    hsh.update(np.ascontiguousarray(cnt, np.int32).tobytes())
    for k in range(len(cnt)):
        hsh.update(np.ascontiguousarray(lst[k * cap:k * cap + cnt[k]], np.int32).tobytes())
    return hsh.hexdigest()


def csr(cnt, lst, cap):
    return np.concatenate([lst[k * cap:k * cap + cnt[k]] for k in range(len(cnt))]).astype(np.int32)


def gen_airebo(R: Ref, nc: int, jitter: float, seed: int, full_lists: bool):
    s = crystal.atomistic(nc, jitter=jitter, seed=seed)
    pos, h, hi, mol = s["pos"], s["h"], s["hi"], s["mol_id"]
    na = pos.size // 3
    cr, lr, cl, ll = R.ai_lists(pos, h, hi, na, mol)
    E, F, W = R.ai_forces(pos, h, hi, cr, lr, cl, ll, na)
    er, Fr, Wr = R.ai_rebo(pos, h, hi, cr, lr, na)
    el, Fl, Wl = R.ai_lj(pos, h, hi, cl, ll, na)
    st = dict(pos=pos.copy(), vel=s["vel"].copy(), F=F.copy(), vir9=W.copy(), h=h.copy(), hi=hi.copy(),
              mass=s["mass"], npt=crystal.npt_atom(300.0, 0.0, na))
    step_in = {k: v.copy() for k, v in st.items()}
    out = R.ai_step(st, 0.5, cr, lr, cl, ll)
    rec = dict(pos=pos, vel=s["vel"], mass=s["mass"], mol_id=mol, h=h, hi=hi, npt0=step_in["npt"],
               E=E, F=F, W=W, E_rebo=er, F_rebo=Fr, W_rebo=Wr, E_lj=el, F_lj=Fl, W_lj=Wl,
               cnt_rebo=cr, csr_rebo=csr(cr, lr, 12), cnt_lj=cl,
               digest_lj=np.array(list_digest(cl, ll, 400)), digest_rebo=np.array(list_digest(cr, lr, 12)),
               step_out=out, step_pos=st["pos"], step_vel=st["vel"], step_F=st["F"], step_vir9=st["vir9"],
               step_h=st["h"], step_hi=st["hi"], step_npt=st["npt"])
    if full_lists:
        rec["csr_lj"] = csr(cl, ll, 400)
    np.savez_compressed(OUT / f"airebo_nc{nc}.npz", **rec)


def gen_rigid(R: Ref, nc: int, seed: int):
    s = crystal.rigid(nc, seed=seed)
    n, natom = s["n"], s["natom"]
    rmcut = 3.0 * 3.431 + 2 * s["Rmol"] + 1.0            # LJ:716
    cnt, lst = R.lj_nlist(s["pos"], s["h"], s["hi"], n, rmcut)
    e, F, T, W = R.lj_forces(s["pos"], s["qv"], s["body"], s["h"], s["hi"], cnt, lst, n, natom, rmcut * rmcut)
    st = dict(pos=s["pos"].copy(), vel=s["vel"].copy(), qv=s["qv"].copy(), omg=s["omg"].copy(), F=F.copy(),
              T=T.copy(), W9=W.copy(), h=s["h"].copy(), hi=s["hi"].copy(), npt=crystal.npt_rigid(300.0, 1.0, n))
    npt0 = st["npt"].copy()
    out = R.lj_step(st, s["body"], s["I0"], s["Mmol"], natom, rmcut * rmcut, 1.0, cnt, lst)
    np.savez_compressed(OUT / f"rigid_nc{nc}.npz", pos=s["pos"], vel=s["vel"], qv=s["qv"], omg=s["omg"],
                        body=s["body"], h=s["h"], hi=s["hi"], I0=s["I0"], Mmol=s["Mmol"], rmcut=rmcut,
                        cnt=cnt, csr=csr(cnt, lst, 80), E=e, F=F, T=T, W=W, npt0=npt0, step_out=out,
                        step_pos=st["pos"], step_vel=st["vel"], step_qv=st["qv"], step_omg=st["omg"],
                        step_F=st["F"], step_T=st["T"], step_W9=st["W9"], step_h=st["h"], step_hi=st["hi"],
                        step_npt=st["npt"])


def gen_core(R: Ref):
    coords = np.zeros(180)
    rd = np.zeros(3)
    R.core.ref_core_generate_c60(d(coords), d(rd))
    np.savez_compressed(OUT / "core_c60.npz", coords=coords, I0=rd[0], Mmol=rd[1], Rmol=rd[2],
                        rmcut=R.core.ref_core_rmcut())


def mm_topology(R: Ref, coords, bonds, nmol):
    L = R.mm
    natom, nb = len(coords), len(bonds)
    counts = np.zeros(4, np.int32)
    kcal2eV = 1.0 / 23.06054783
    args = [d(np.ascontiguousarray(coords.reshape(-1))), natom, i(np.ascontiguousarray(bonds.reshape(-1), np.int32)),
            nb, nmol, ctypes.c_double(469.0 * kcal2eV), ctypes.c_double(63.0 * kcal2eV),
            ctypes.c_double(14.5 * kcal2eV), ctypes.c_double(15.0 * kcal2eV), i(counts)]
    L.ref_mm_build_topology(*args, *([None] * 14))
    nb1, na1, nd1, ni1 = counts
    Nb, Na_, Nd, Ni = nb1 * nmol, na1 * nmol, nd1 * nmol, ni1 * nmol
    bi = np.zeros(2 * Nb, np.int32); bk = np.zeros(Nb); br = np.zeros(Nb)
    ai = np.zeros(3 * Na_, np.int32); ak = np.zeros(Na_); at = np.zeros(Na_)
    di = np.zeros(4 * Nd, np.int32); dv = np.zeros(Nd); dm = np.zeros(Nd, np.int32); dg = np.zeros(Nd)
    ii = np.zeros(4 * Ni, np.int32); ik = np.zeros(Ni); ig = np.zeros(Ni)
    mid = np.zeros(nmol * natom, np.int32)
    L.ref_mm_build_topology(*args, i(bi), d(bk), d(br), i(ai), d(ak), d(at), i(di), d(dv), i(dm), d(dg), i(ii),
                            d(ik), d(ig), i(mid))
    return dict(bonds=bi.reshape(2, -1).T.copy(), kb=bk, r0=br, angles=ai.reshape(3, -1).T.copy(), kth=ak, th0=at,
                dihedrals=di.reshape(4, -1).T.copy(), vn=dv, mult=dm, gamma=dg,
                impropers=ii.reshape(4, -1).T.copy(), ki=ik, igamma=ig, mol_id=mid, counts=counts)


def gen_mm(R: Ref, nc: int, seed: int):
    coords = crystal.c60_ih()
    bonds = crystal.bonds_from_geometry(coords)
    s = crystal.atomistic(nc, coords=coords, jitter=0.02, seed=seed, mol_base=0)
    pos, h, hi = s["pos"], s["h"], s["hi"]
    na, nmol = pos.size // 3, s["nmol"]
    t = mm_topology(R, coords, bonds, nmol)
    L = R.mm
    cnt = np.zeros(na, np.int32); lst = np.zeros(na * 400, np.int32)
    L.ref_mm_build_nlist_lj(d(pos), d(h), d(hi), na, i(t["mol_id"]), i(cnt), i(lst))

    def forces(charge, has_charge):
        F = np.zeros(3 * na); W = np.zeros(9); E = np.zeros(7)
        L.ref_mm_compute_forces(d(F), d(W), d(pos), d(h), d(hi), len(t["bonds"]), i(np.ascontiguousarray(t["bonds"].T.reshape(-1))),
                                d(t["kb"]), d(t["r0"]), len(t["angles"]), i(np.ascontiguousarray(t["angles"].T.reshape(-1))),
                                d(t["kth"]), d(t["th0"]), len(t["dihedrals"]),
                                i(np.ascontiguousarray(t["dihedrals"].T.reshape(-1))), d(t["vn"]), i(t["mult"]),
                                d(t["gamma"]), len(t["impropers"]), i(np.ascontiguousarray(t["impropers"].T.reshape(-1))),
                                d(t["ki"]), d(t["igamma"]), i(cnt), i(lst), d(charge), i(t["mol_id"]), has_charge, na,
                                d(E))
        return E, F, W

    zero_q = np.zeros(na)
    E, F, W = forces(zero_q, 0)
    rng = np.random.default_rng(seed + 1)
    q = rng.uniform(-0.05, 0.05, size=na)
    Eq, Fq, Wq = forces(q, 1)
    # one step (MM:811)
    st = dict(pos=pos.copy(), vel=s["vel"].copy(), F=F.copy(), vir9=W.copy(), h=h.copy(), hi=hi.copy(),
              npt=crystal.npt_atom(500.0, 1.0, na))
    npt0 = st["npt"].copy()
    out = np.zeros(8)
    L.ref_mm_step_npt(d(st["pos"]), d(st["vel"]), d(st["F"]), d(st["vir9"]), d(st["h"]), d(st["hi"]), na,
                      ctypes.c_double(0.1), d(st["npt"]), len(t["bonds"]), i(np.ascontiguousarray(t["bonds"].T.reshape(-1))),
                      d(t["kb"]), d(t["r0"]), len(t["angles"]), i(np.ascontiguousarray(t["angles"].T.reshape(-1))),
                      d(t["kth"]), d(t["th0"]), len(t["dihedrals"]), i(np.ascontiguousarray(t["dihedrals"].T.reshape(-1))),
                      d(t["vn"]), i(t["mult"]), d(t["gamma"]), len(t["impropers"]),
                      i(np.ascontiguousarray(t["impropers"].T.reshape(-1))), d(t["ki"]), d(t["igamma"]), i(cnt), i(lst),
                      d(zero_q), i(t["mol_id"]), 0, d(out))
    np.savez_compressed(OUT / f"mm_nc{nc}.npz", coords=coords, bonds_mol=bonds, pos=pos, vel=s["vel"], h=h, hi=hi,
                        charge=q, cnt=cnt, digest=np.array(list_digest(cnt, lst, 400)),
                        E=E, F=F, W=W, Eq=Eq, Fq=Fq, Wq=Wq, npt0=npt0, step_out=out, step_pos=st["pos"],
                        step_vel=st["vel"], step_F=st["F"], step_vir9=st["vir9"], step_h=st["h"], step_hi=st["hi"],
                        step_npt=st["npt"], **{f"topo_{k}": v for k, v in t.items()})


def main():
    if not ref_available():
        sys.exit("oracle/_ref is not built (needs the reference sources): make -C oracle")
    R = Ref()
    gen_airebo(R, 1, 0.05, 7, True)
    gen_airebo(R, 2, 0.01, 11, False)
    gen_rigid(R, 2, 3)
    gen_rigid(R, 3, 5)
    gen_core(R)
    gen_mm(R, 1, 13)
    for p in sorted(OUT.glob("*.npz")):
        print(f"{p.name:24s} {p.stat().st_size / 1024:8.1f} KiB")


if __name__ == "__main__":
    main()
