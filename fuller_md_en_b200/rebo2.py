"""Spline knots of the REBO-II extension (fmd_rebo2_knots in
include/fullermd.h; no counterpart in the reference, whose REBO bond order is
b = (1 + sum f_c G)^-1/2 only, AI:301-323).

For carbon-only systems the extension needs three splines, each cubic Hermite
in every variable through values and derivatives given at integer knots
(Brenner et al., J. Phys.: Condens. Matter 14 (2002) 783, eqs. 8, 12, 17):

* ``pcc[n] = (P, dP/dN)`` of P_CC(N, N_H = 0) at N = n, n = 0..4;
* ``pirc[x, y, z]`` and ``tcc[x, y, z]`` = (f, f_x, f_y, f_z, f_xy, f_xz,
  f_yz, f_xyz) of pi^rc_CC and T_CC at N_ij = x, N_ji = y (0..4) and
  N_conj = z (0..9).

The published tables are not part of this package: the caller fills the
knots.  All-zero knots give the reference's bond order.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from ._lib import Rebo2Knots as _Raw


def _zeros(shape):
    return np.zeros(shape)


@dataclass
class Rebo2Knots:
    pcc: np.ndarray = field(default_factory=lambda: _zeros((5, 2)))
    pirc: np.ndarray = field(default_factory=lambda: _zeros((5, 5, 10, 8)))
    tcc: np.ndarray = field(default_factory=lambda: _zeros((5, 5, 10, 8)))

    def raw(self) -> _Raw:
        """The C struct (a fresh copy of the arrays)."""
        s = _Raw()
        for name, n, shape in (("pcc", 10, (5, 2)), ("pirc", 2000, (5, 5, 10, 8)), ("tcc", 2000, (5, 5, 10, 8))):
            a = np.ascontiguousarray(getattr(self, name), np.float64)
            if a.shape != shape:
                raise ValueError(f"Rebo2Knots.{name}: shape {a.shape}, expected {shape}")
            ctypes.memmove(getattr(s, name), a.ctypes.data, 8 * n)
        return s
