"""Pins the CPU oracle (oracle/fmd_oracle.c) to the reference's own outputs
recorded in tests/golden/ (see gen_golden.py).  Neighbour lists must match
bit for bit; forces, energies, virials and one NPT step must match to
round-off (the oracle follows the reference's operation order, so on the same
libm they agree exactly; 1e-12 leaves room for a different libm)."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import csr_rows, rel, rows, same_rows

TOL = 1e-12


def digest(cnt, lst, cap):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(cnt, np.int32).tobytes())
    for k in range(len(cnt)):
        h.update(np.ascontiguousarray(lst[k * cap:k * cap + cnt[k]], np.int32).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("nc", [1, 2])
def test_airebo_lists(oracle, golden, nc):
    g = golden(f"airebo_nc{nc}")
    na = g["pos"].size // 3
    cr, lr, _ = oracle.nlist_intra(g["pos"], g["h"], g["hi"], na, g["mol_id"])
    cl, ll, dropped = oracle.nlist_half(g["pos"], g["h"], g["hi"], na, g["mol_id"], 3.0 * 3.40 + 2.0)
    assert np.array_equal(cr, g["cnt_rebo"])
    assert same_rows(rows(cr, lr, 12), csr_rows(g["cnt_rebo"], g["csr_rebo"]))
    assert np.array_equal(cl, g["cnt_lj"])
    assert digest(cl, ll, 400) == str(g["digest_lj"])
    if "csr_lj" in g:
        assert same_rows(rows(cl, ll, 400), csr_rows(g["cnt_lj"], g["csr_lj"]))
    if nc == 2:
        assert dropped > 0 and (cl == 400).any(), "truncation at 400 must be exercised"
    # the row-split form used for the large-system tests gives the same list
    tc, tl, tdrop = oracle.nlist_half_threaded(g["pos"], g["h"], g["hi"], na, g["mol_id"], 3.0 * 3.40 + 2.0,
                                               threads=4, chunk=97)
    assert np.array_equal(tc, g["cnt_lj"]) and digest(tc, tl, 400) == str(g["digest_lj"]) and tdrop == dropped


def _lists(g, na):
    cr = g["cnt_rebo"]
    lr = np.zeros(na * 12, np.int32)
    for k, r in enumerate(csr_rows(cr, g["csr_rebo"])):
        lr[k * 12:k * 12 + len(r)] = r
    return cr, lr


@pytest.mark.parametrize("nc", [1, 2])
def test_airebo_forces_and_step(oracle, golden, nc):
    g = golden(f"airebo_nc{nc}")
    na = g["pos"].size // 3
    cr, lr = _lists(g, na)
    cl, ll, _ = oracle.nlist_half(g["pos"], g["h"], g["hi"], na, g["mol_id"], 3.0 * 3.40 + 2.0)
    E, F, W = oracle.airebo_forces(g["pos"], g["h"], g["hi"], cr, lr, cl, ll, na)
    assert rel(E, g["E"]) < TOL and rel(F, g["F"]) < TOL and rel(W, g["W"]) < TOL
    e, f, w = oracle.rebo(g["pos"], g["h"], g["hi"], cr, lr, na)
    assert abs(e - g["E_rebo"]) <= TOL * abs(g["E_rebo"]) and rel(f, g["F_rebo"]) < TOL and rel(w, g["W_rebo"]) < TOL
    e, f, w = oracle.lj(g["pos"], g["h"], g["hi"], cl, ll, na)
    assert abs(e - g["E_lj"]) <= TOL * abs(g["E_lj"]) and rel(f, g["F_lj"]) < TOL and rel(w, g["W_lj"]) < TOL
    st = dict(pos=g["pos"].copy(), vel=g["vel"].copy(), F=g["F"].copy(), vir9=g["W"].copy(), h=g["h"].copy(),
              hi=g["hi"].copy(), mass=g["mass"], npt=g["npt0"].copy())
    out = oracle.airebo_step(st, 0.5, cr, lr, cl, ll)
    assert rel(out, g["step_out"]) < TOL
    for k in ("pos", "vel", "F", "vir9", "h", "hi", "npt"):
        assert rel(st[k], g[f"step_{k}"]) < TOL, k


@pytest.mark.parametrize("nc", [2, 3])
def test_rigid(oracle, golden, nc):
    g = golden(f"rigid_nc{nc}")
    n = g["pos"].size // 3
    rmcut = float(g["rmcut"])
    c, l, _ = oracle.nlist_sym(g["pos"], g["h"], g["hi"], n, rmcut)
    assert np.array_equal(c, g["cnt"]) and same_rows(rows(c, l, 80), csr_rows(g["cnt"], g["csr"]))
    e, F, T, W = oracle.rigid_forces(g["pos"], g["qv"], g["body"], g["h"], g["hi"], c, l, n, 60, rmcut * rmcut)
    assert abs(e - g["E"]) <= TOL * abs(g["E"])
    assert rel(F, g["F"]) < TOL and rel(T, g["T"]) < TOL and rel(W, g["W"]) < TOL
    st = dict(pos=g["pos"].copy(), vel=g["vel"].copy(), qv=g["qv"].copy(), omg=g["omg"].copy(), F=F.copy(),
              T=T.copy(), W9=W.copy(), h=g["h"].copy(), hi=g["hi"].copy(), npt=g["npt0"].copy())
    out = oracle.rigid_step(st, g["body"], float(g["I0"]), float(g["Mmol"]), 60, rmcut * rmcut, 1.0, c, l)
    assert rel(out, g["step_out"]) < TOL
    for k in ("pos", "vel", "qv", "omg", "F", "T", "W9", "h", "hi", "npt"):
        assert rel(st[k], g[f"step_{k}"]) < TOL, k


def _mm_topo(g, nmol):
    t = {k[5:]: g[k] for k in g if k.startswith("topo_")}
    return t


def test_mm_topology(oracle, golden):
    g = golden("mm_nc1")
    t = _mm_topo(g, 4)
    mol = oracle.mm_topology_mol(g["coords"], g["bonds_mol"])
    counts = [len(mol["bonds"]), len(mol["angles"]), len(mol["dihedrals"]), len(mol["impropers"])]
    assert counts == list(t["counts"]) == [90, 180, 360, 60]
    natom = len(g["coords"])
    nb = counts[0]
    assert np.array_equal(mol["bonds"], t["bonds"][:nb])
    assert np.array_equal(mol["angles"], t["angles"][:counts[1]])
    assert np.array_equal(mol["dihedrals"], t["dihedrals"][:counts[2]])
    assert np.array_equal(mol["impropers"], t["impropers"][:counts[3]])
    assert rel(mol["r0"], t["r0"][:nb]) < TOL and rel(mol["th0"], t["th0"][:counts[1]]) < TOL
    assert rel(mol["gamma"], t["gamma"][:counts[2]]) < TOL and rel(mol["igamma"], t["igamma"][:counts[3]]) < TOL
    # replication with atom offsets (MM:315-331)
    assert np.array_equal(t["bonds"][nb:2 * nb], t["bonds"][:nb] + natom)


def test_mm_forces_and_step(oracle, golden):
    g = golden("mm_nc1")
    t = _mm_topo(g, 4)
    na = g["pos"].size // 3
    cnt, lst, _ = oracle.nlist_half(g["pos"], g["h"], g["hi"], na, t["mol_id"], 3.0 * 3.431 + 2.0)
    assert np.array_equal(cnt, g["cnt"]) and digest(cnt, lst, 400) == str(g["digest"])
    E, F, W = oracle.mm_forces(t, g["pos"], g["h"], g["hi"], cnt, lst, na)
    assert rel(E, g["E"]) < TOL and rel(F, g["F"]) < TOL and rel(W, g["W"]) < TOL
    Eq, Fq, Wq = oracle.mm_forces(t, g["pos"], g["h"], g["hi"], cnt, lst, na, charge=g["charge"],
                                  mol_id=t["mol_id"])
    assert abs(Eq[5]) > 0 and rel(Eq, g["Eq"]) < TOL and rel(Fq, g["Fq"]) < TOL
    st = dict(pos=g["pos"].copy(), vel=g["vel"].copy(), F=g["F"].copy(), vir9=g["W"].copy(), h=g["h"].copy(),
              hi=g["hi"].copy(), npt=g["npt0"].copy())
    out = oracle.mm_step(st, 0.1, t, cnt, lst)
    assert rel(out, g["step_out"]) < TOL
    for k in ("pos", "vel", "F", "vir9", "h", "hi", "npt"):
        assert rel(st[k], g[f"step_{k}"]) < TOL, k


def test_oracle_detects_planted_error(oracle, golden):
    """The comparison is sensitive: one flipped neighbour changes the digest
    and a 1e-9 nudge of one position moves the energy past the tolerance."""
    g = golden("airebo_nc1")
    na = g["pos"].size // 3
    cl, ll, _ = oracle.nlist_half(g["pos"], g["h"], g["hi"], na, g["mol_id"], 3.0 * 3.40 + 2.0)
    ll2 = ll.copy()
    ll2[0] = ll2[0] + 1
    assert digest(cl, ll2, 400) != str(g["digest_lj"])
    p = g["pos"].copy()
    p[0] += 1e-6
    cr, lr = _lists(g, na)
    E, F, W = oracle.airebo_forces(p, g["h"], g["hi"], cr, lr, cl, ll, na)
    assert rel(F, g["F"]) > TOL
