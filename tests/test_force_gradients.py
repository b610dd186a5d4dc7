"""Which of the reference's forces are gradients of its energies, measured on
the CPU by central differences of the oracle's energies; this is the analysis
behind the opt-in physics corrections (fmd_system_set_physics), whose GPU
forces test_physics_gpu.py checks the same way.

* MM: bond and angle forces are +grad E (MM:389-398, MM:468-491); dihedral
  and improper forces are neither +grad E nor -grad E; the LJ force is
  -grad E.
* REBO: the forces are not -grad E (three-body terms); the oracle's
  gradient restatement (fmo_rebo_grad, not the reference's arithmetic) is,
  with rows cut at 12 entries included.
* Torsion: negating the two projection coefficients of the middle atoms
  (what FMD_PHYS_MM_BONDED does in the kernel) makes the force -grad E."""
from __future__ import annotations

import numpy as np
import pytest

from fuller_md_en_b200 import crystal

H = 1e-5
RC_MM = 3.0 * 3.431 + 2.0


def _fd(energy, F, x, comps):
    """Largest |F_k + dE/dx_k| and |F_k - dE/dx_k| over comps."""
    em = ep = 0.0
    for k in comps:
        p, m = x.copy(), x.copy()
        p[k] += H
        m[k] -= H
        g = (energy(p) - energy(m)) / (2 * H)
        em, ep = max(em, abs(F[k] + g)), max(ep, abs(F[k] - g))
    return em, ep


@pytest.fixture(scope="module")
def mm_case():
    coords = crystal.c60_ih()
    s = crystal.atomistic(1, coords=coords, jitter=0.04, seed=17, T=300.0, mol_base=0)
    t = crystal.mm_topology(coords, crystal.bonds_from_geometry(coords), s["nmol"])
    return s, t


def _only(t, kind):
    groups = {"bonds": ("bonds", "kb", "r0"), "angles": ("angles", "kth", "th0"),
              "dihedrals": ("dihedrals", "vn", "mult", "gamma"), "impropers": ("impropers", "ki", "igamma")}
    u = dict(t)
    for k, keys in groups.items():
        if k != kind:
            for kk in keys:
                u[kk] = u[kk][:0]
    return u


@pytest.mark.parametrize("kind,expect", [("bonds", "+"), ("angles", "+"), ("dihedrals", "neither"),
                                         ("impropers", "neither"), ("lj", "-")])
def test_mm_reference_force_terms(oracle, mm_case, kind, expect):
    s, t = mm_case
    na = s["pos"].size // 3
    h, hi = s["h"], crystal.inv9(s["h"])
    if kind == "lj":
        u = _only(t, "none")
        cnt, lst, _ = oracle.nlist_half(s["pos"], h, hi, na, s["mol_id"], RC_MM)
    else:
        u = _only(t, kind)
        cnt, lst = np.zeros(na, np.int32), np.zeros(na * 400, np.int32)
    E, F, _ = oracle.mm_forces(u, s["pos"], h, hi, cnt, lst, na)
    comps = np.random.default_rng(5).choice(s["pos"].size, 16, replace=False)
    em, ep = _fd(lambda p: oracle.mm_forces(u, p, h, hi, cnt, lst, na)[0][6], F, s["pos"], comps)
    fmax = np.max(np.abs(F))
    small, large = 1e-8 * fmax, 1e-2 * fmax
    if expect == "+":
        assert ep < small and em > large, (em, ep, fmax)
    elif expect == "-":
        assert em < small and ep > large, (em, ep, fmax)
    else:
        assert em > large and ep > large, (em, ep, fmax)


@pytest.mark.parametrize("scale,seed", [(1.0, 11), (0.65, 77), (0.7, 5)])
def test_rebo_gradient_restatement(oracle, scale, seed):
    s = crystal.atomistic(1, coords=crystal.c60_ih() * scale, jitter=0.05, seed=seed)
    na = s["pos"].size // 3
    h, hi = s["h"], crystal.inv9(s["h"])
    cr, lr, dropped = oracle.nlist_intra(s["pos"], h, hi, na, s["mol_id"])
    if scale < 0.7:
        assert dropped > 0                               # rows cut at 12 entries
    pos = oracle.apply_pbc(s["pos"].copy(), h, hi)
    none = (np.zeros(na, np.int32), np.zeros(na * 400, np.int32))
    E_ref, F_ref, _ = oracle.airebo_forces(pos, h, hi, cr, lr, *none, na)
    E, F = oracle.rebo_grad(pos, h, hi, cr, lr, na)
    assert E == E_ref[1]                                 # the same energy, bit for bit
    comps = np.random.default_rng(seed).choice(pos.size, 16, replace=False)
    energy = lambda p: oracle.rebo_grad(p, h, hi, cr, lr, na)[0]
    em, _ = _fd(energy, F, pos, comps)
    assert em < 1e-7 * np.max(np.abs(F)), em
    assert np.max(np.abs(F.reshape(-1, 3).sum(axis=0))) < 1e-10 * np.max(np.abs(F))
    if scale == 1.0:
        em_ref, _ = _fd(energy, F_ref, pos, comps)
        assert em_ref > 1e-2 * np.max(np.abs(F_ref))      # the reference's forces are not -grad E


def _torsion(r, sg, mult=2, vn=0.6, gamma=1.1):
    """Energy and forces of one torsion in the kernel's formulation (torsion()
    in mm.cu): sg = 1 the reference's middle-atom terms, -1 the corrected."""
    b1, b2, b3 = r[1] - r[0], r[2] - r[1], r[3] - r[2]
    m, n = np.cross(b1, b2), np.cross(b2, b3)
    mm, nn = m @ m, n @ n
    b2len = np.sqrt(b2 @ b2)
    rmn = np.sqrt(mm * nn)
    phi = np.arctan2((m @ b3) * b2len / rmn, np.clip(m @ n / rmn, -1, 1))
    e = 0.5 * vn * (1 + np.cos(mult * phi - gamma))
    dphi = -0.5 * vn * mult * np.sin(mult * phi - gamma)
    f1, f4 = dphi * b2len / mm * m, -dphi * b2len / nn * n
    ci, ck = sg * (b1 @ b2) / b2len ** 2, sg * (b2 @ b3) / b2len ** 2
    return e, np.array([f1, -f1 + ci * f1 - ck * f4, -f4 - ci * f1 + ck * f4, f4])


@pytest.mark.parametrize("seed", range(4))
def test_torsion_correction(seed):
    r = np.random.default_rng(seed).normal(size=(4, 3)) * 1.5
    for sg, grad in ((-1.0, True), (1.0, False)):
        _, F = _torsion(r, sg)
        x = r.reshape(-1)
        em, _ = _fd(lambda p: _torsion(p.reshape(4, 3), sg)[0], F.reshape(-1), x, range(12))
        assert (em < 1e-8) == grad, (sg, em)
