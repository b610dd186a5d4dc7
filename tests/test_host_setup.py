"""Host-side set-up used by the product path (no GPU): the flat MM topology
builder in fuller_md_en_b200.crystal against the reference's
build_flat_topology (through the oracle)."""
from __future__ import annotations

import numpy as np

from fuller_md_en_b200 import crystal


def test_mm_topology_matches_reference(oracle):
    coords = crystal.c60_ih()
    bonds = crystal.bonds_from_geometry(coords)
    nmol = 3
    t = crystal.mm_topology(coords, bonds, nmol)
    m = oracle.mm_topology_mol(coords, bonds)
    na = len(coords)
    for key, per in (("bonds", 90), ("angles", 180), ("dihedrals", 360), ("impropers", 60)):
        got = np.asarray(t[key])
        ref = np.asarray(m[key])
        assert len(ref) == per and got.shape == (per * nmol, ref.shape[1])
        for k in range(nmol):
            assert np.array_equal(got[k * per:(k + 1) * per], ref + k * na), key
    for key, ref in (("r0", m["r0"]), ("th0", m["th0"]), ("gamma", m["gamma"]), ("igamma", m["igamma"])):
        assert np.array_equal(np.asarray(t[key]), np.tile(ref, nmol)), key     # bitwise
    assert np.array_equal(t["mol_id"], np.repeat(np.arange(nmol), na))
    assert np.allclose(t["kb"], 469.0 / 23.06054783, rtol=1e-15)
