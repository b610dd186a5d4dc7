"""The factored FP64 LJ pair terms of the list gather (csrc/ljpair.cuh) against
the reference's expressions (AI:443-445), on the CPU in IEEE double.

The gather evaluates 24 eps (2 s^12 - s^6) / r^2 as 24 eps s^6 (2 s^6 - 1) / r^2
and 4 eps (s^12 - s^6) as 4 eps s^6 (s^6 - 1).  Both forms round differently;
this bounds the difference by a few units in the last place of the terms
being combined, over the r^2 range the gather sees (the clamp at 0.25 A^2 to
the cutoff), for the AIREBO and MM parameters.  The GPU parity tests check
the device arithmetic itself against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

EPS64 = np.finfo(np.float64).eps

PARAMS = {  # sigma, epsilon (AI:119-124, MM:113-116)
    "airebo": (3.40, 2.84e-3),
    "mm": (3.431, 2.635e-3),
}


@pytest.mark.parametrize("ff", sorted(PARAMS))
def test_factored_pair_terms_match_the_reference_form(ff):
    sig, eps = PARAMS[ff]
    rc2 = (3.0 * sig) ** 2
    r2 = np.concatenate([np.linspace(0.25, rc2, 200001), np.geomspace(0.25, rc2, 20001)])
    sig2, c4, c24 = sig * sig, 4 * eps, 24 * eps
    ri2 = 1.0 / r2
    # reference (AI:443-445)
    sr2 = sig2 * ri2
    sr6 = sr2 * sr2 * sr2
    sr12 = sr6 * sr6
    fm_ref = c24 * (2 * sr12 - sr6) * ri2
    e_ref = c4 * (sr12 - sr6)
    # factored form of the gather
    s6 = sr2 * sr2 * sr2
    fm_fac = (c24 * ri2 * s6) * (2.0 * s6 - 1.0)
    e_fac = c4 * s6 * (s6 - 1.0)
    # scale of the combined terms: the repulsive part dominates at short range
    f_scale = c24 * (2 * sr12 + sr6) * ri2
    e_scale = c4 * (sr12 + sr6)
    assert np.max(np.abs(fm_fac - fm_ref) / f_scale) < 8 * EPS64
    assert np.max(np.abs(e_fac - e_ref) / e_scale) < 8 * EPS64


def test_force_zero_crossing_is_kept():
    """Near r = 2^(1/6) sigma both forms cancel to a small force; the factored
    form keeps the sign change at the same place to within rounding."""
    sig, eps = PARAMS["airebo"]
    r0 = 2 ** (1 / 6) * sig
    r = np.linspace(r0 * (1 - 1e-6), r0 * (1 + 1e-6), 2001)
    r2 = r * r
    ri2 = 1.0 / r2
    s2 = sig * sig * ri2
    s6 = s2 * s2 * s2
    ref = 24 * eps * (2 * s6 * s6 - s6) * ri2
    fac = (24 * eps * ri2 * s6) * (2.0 * s6 - 1.0)
    # same sign everywhere except within a few ulp of the root
    scale = 24 * eps * 3 * ri2
    mism = np.sign(ref) != np.sign(fac)
    assert np.all(np.abs(ref[mism]) < 8 * EPS64 * scale[mism])
