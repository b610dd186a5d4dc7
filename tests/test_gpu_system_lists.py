"""Neighbour lists built inside device-resident systems (the molecule-wise
builder for contiguous molecules, and the cell-grid builder it falls back to
on non-diagonal cells) against the reference builders, bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rows, same_rows
from fuller_md_en_b200 import RunConfig, System, crystal, mm_replica

pytestmark = pytest.mark.gpu

RC_AI = 3.0 * 3.40 + 2.0
RC_MM = 3.0 * 3.431 + 2.0


@pytest.mark.parametrize("nc,shear,jitter,seed", [(3, 0.0, 0.01, 1), (2, 0.9, 0.05, 2), (3, 0.0, 0.35, 3),
                                                  (5, 0.0, 0.01, 4)])
def test_airebo_system_lists_match_reference(ctx, oracle, nc, shear, jitter, seed):
    s = crystal.atomistic(nc, jitter=jitter, seed=seed)
    na = s["pos"].size // 3
    h = s["h"].copy()
    h[1] += shear
    hi = crystal.inv9(h)
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=10, nlup=20, nc=nc, nmol=s["nmol"])
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], h, crystal.npt_atom(300.0, 0.0, na))
    sysd.init()                                  # lists from the unwrapped positions (AI:830-836)
    ca, la, cb, lb = sysd.lists(400, 12)
    oc, ol, _ = oracle.nlist_half(s["pos"], h, hi, na, s["mol_id"], RC_AI)
    orc, orl, _ = oracle.nlist_intra(s["pos"], h, hi, na, s["mol_id"])
    assert np.array_equal(ca, oc) and same_rows(rows(ca, la, 400), rows(oc, ol, 400))
    assert np.array_equal(cb, orc) and same_rows(rows(cb, lb, 12), rows(orc, orl, 12))
    if nc == 5:
        assert (oc == 400).any()                 # truncated rows are part of the check
    fc, fl = sysd.lj_full_rows()
    ec, el = full_rows(oc, ol, 400, na)
    assert np.array_equal(fc, ec)
    assert all(np.array_equal(fl[j, :fc[j]], el[j]) for j in range(na))
    sysd.close()


def full_rows(cnt, lst, cap, n):
    """The LJ gather's full rows from the reference's half rows: row j holds
    the atoms i whose row lists j, ascending, then j's own row."""
    src = np.repeat(np.arange(n), cnt)
    dst = np.concatenate([lst[k * cap:k * cap + cnt[k]] for k in range(n)])
    o = np.lexsort((src, dst))
    src, dst = src[o], dst[o]
    start = np.searchsorted(dst, np.arange(n + 1))
    rws = [np.concatenate([src[start[j]:start[j + 1]], lst[j * cap:j * cap + cnt[j]]]) for j in range(n)]
    return np.array([len(r) for r in rws], np.int32), rws


@pytest.mark.parametrize("natom", [28, 32, 45, 64])
def test_lists_for_other_molecule_sizes(ctx, oracle, natom):
    """Molecules of 28 atoms (flat candidate walk, full rows by the
    transpose), 32 (partner walk with idle upper slices), 45 and 64 (partner
    walk, full rows from the candidate bitmap; 64 fills both slices): half
    rows against the reference builder and full rows against the half rows."""
    c60 = crystal.c60_ih()
    coords = c60[:natom] if natom <= 60 else np.vstack([c60, 0.45 * c60[:natom - 60]])
    s = crystal.atomistic(3, coords=coords, jitter=0.02, seed=natom)
    na = s["pos"].size // 3
    h, hi = s["h"], crystal.inv9(s["h"])
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=4, nlup=20, nc=3, nmol=s["nmol"])
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], h, crystal.npt_atom(300.0, 0.0, na))
    sysd.init()
    ca, la, _, _ = sysd.lists(400)
    oc, ol, _ = oracle.nlist_half(s["pos"], h, hi, na, s["mol_id"], RC_AI)
    assert np.array_equal(ca, oc) and same_rows(rows(ca, la, 400), rows(oc, ol, 400))
    fc, fl = sysd.lj_full_rows()
    ec, el = full_rows(oc, ol, 400, na)
    assert np.array_equal(fc, ec)
    assert all(np.array_equal(fl[j, :fc[j]], el[j]) for j in range(na))
    sysd.close()


def test_full_rows_on_a_sequence_of_builds(ctx, oracle):
    """Full rows after several builds on a moving system (the molecule
    builder's acceptance masks are rewritten each build) equal those formed
    from the current half rows."""
    s = crystal.atomistic(3, jitter=0.02, seed=8, T=600.0)
    na = s["pos"].size // 3
    cfg = RunConfig(dt=0.5, T=600.0, Pe=0.0, nsteps=60, nlup=20, nc=3, nmol=s["nmol"])
    sysd = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], s["h"],
                         crystal.npt_atom(600.0, 0.0, na))
    sysd.init()
    for g0 in (1, 21, 41):
        sysd.run(g0, g0 + 19)                    # 20 steps: one list build
        ca, la, _, _ = sysd.lists(400)
        fc, fl = sysd.lj_full_rows()
        ec, el = full_rows(ca, la, 400, na)
        assert np.array_equal(fc, ec), g0
        assert all(np.array_equal(fl[j, :fc[j]], el[j]) for j in range(na)), g0
    sysd.close()


def test_mm_system_lists_match_reference(ctx, oracle):
    sysd = mm_replica(ctx, 3, 300.0, 0.0, seed=9, jitter=0.02)
    sysd.init()
    ca, la, _, _ = sysd.lists(400)
    s = crystal.atomistic(3, coords=crystal.c60_ih(), jitter=0.02, seed=9, T=300.0, mol_base=0)
    na = s["pos"].size // 3
    oc, ol, _ = oracle.nlist_half(s["pos"], s["h"], s["hi"], na, s["mol_id"], RC_MM)
    assert same_rows(rows(ca, la, 400), rows(oc, ol, 400))
    sysd.close()
