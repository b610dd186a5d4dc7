"""REBO inside a device-resident system with crowded rows cut at the
reference's 12 entries (AI:251-261), so that i lists j while j's row lacks
i.  The system path walks the occupied slots of the last list build and
takes each bond's partner slot from the table built with it; the result must
match the reference's compute_forces on the reference's own lists."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel
from fuller_md_en_b200 import RunConfig, System, crystal

pytestmark = pytest.mark.gpu

RC_AI = 3.0 * 3.40 + 2.0


@pytest.mark.parametrize("scale,seed", [(0.65, 77), (0.7, 5)])
def test_system_rebo_with_cut_rows_matches_reference(ctx, oracle, scale, seed):
    s = crystal.atomistic(2, coords=crystal.c60_ih() * scale, jitter=0.05, seed=seed)
    na = s["pos"].size // 3
    h, hi = s["h"], crystal.inv9(s["h"])
    # the reference: lists from the unwrapped positions, forces on the wrapped ones (AI:830-852)
    cr, lr, dr = oracle.nlist_intra(s["pos"], h, hi, na, s["mol_id"])
    cl, ll, _ = oracle.nlist_half(s["pos"], h, hi, na, s["mol_id"], RC_AI)
    if scale < 0.7:
        rowsets = [set(lr[k * 12:k * 12 + cr[k]]) for k in range(na)]
        assert dr > 0 and any(i not in rowsets[j] for i in range(na) for j in rowsets[i])
    pos = oracle.apply_pbc(s["pos"].copy(), h, hi)
    Er, Fr, Wr = oracle.airebo_forces(pos, h, hi, cr, lr, cl, ll, na)
    cfg = RunConfig(dt=0.5, T=300.0, Pe=0.0, nsteps=4, nlup=20, nc=2, nmol=s["nmol"])
    y = System.airebo(ctx, cfg, s["pos"], s["vel"], s["mass"], s["mol_id"], h, crystal.npt_atom(300.0, 0.0, na))
    y.init()
    F, _, E = y.forces()
    W, _ = y.virial()
    assert rel(F, Fr) < 1e-10
    for k in range(3):
        assert abs(E[k] - Er[k]) <= 1e-10 * max(1.0, abs(Er[k])), (k, E[k], Er[k])
    assert rel(W, Wr) < 1e-10
    y.close()
