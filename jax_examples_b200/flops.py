"""Frozen algorithmic FLOP model of the two-electron path (FMA = 2 flops).

The model counts the McMurchie-Davidson work of one primitive quartet of
class (la lb | lc ld), L = la+lb+lc+ld, independent of how a kernel
schedules it (pair quantities and E-coefficient products are amortised per
pair and not counted):

  Boys:      20 + 3L
  R:         2 * (C(L+4, 4) - 1)                    (R_tuv^n recursion)
  stage 1:   sum over ket Cartesian pairs cd of 2 * N_ab * h_cd
             N_ab = C(la+lb+3, 3) bra Hermite functions,
             h_cd = (cx+dx+1)(cy+dy+1)(cz+dz+1)
  stage 2:   sum over bra Cartesian pairs ab of 2 * h_ab * n_cd
  prefactor: 10

Digestion adds 12 flops per contracted Cartesian integral (2 J and 4 K
updates, FMA each, per density).  The gradient is counted with the same
model on the l+1-shifted bra class.  Reference values: (ss|ss) 34,
(pp|pp) 1434, (dd|dd) 48754, (ds|ps) 353.

This module is the single source of the roofline numerator; it does not
change when kernels are tuned.
"""

from __future__ import annotations

from functools import lru_cache
from math import comb

from .core import cartesian_components, n_cartesian


def _h(c, d):
    return (c[0] + d[0] + 1) * (c[1] + d[1] + 1) * (c[2] + d[2] + 1)


@lru_cache(maxsize=None)
def _sum_h(la: int, lb: int) -> int:
    return sum(_h(a, b) for a in cartesian_components(la) for b in cartesian_components(lb))


@lru_cache(maxsize=None)
def prim_quartet_flops(la: int, lb: int, lc: int, ld: int) -> int:
    """Model flops for one primitive quartet of class (la lb|lc ld)."""
    L = la + lb + lc + ld
    boys = 20 + 3 * L
    r = 2 * (comb(L + 4, 4) - 1)
    n_ab_herm = comb(la + lb + 3, 3)
    stage1 = 2 * n_ab_herm * _sum_h(lc, ld)
    stage2 = 2 * _sum_h(la, lb) * n_cartesian(lc) * n_cartesian(ld)
    return boys + r + stage1 + stage2 + 10


def digestion_flops(la: int, lb: int, lc: int, ld: int, n_dens: int = 1) -> int:
    """12 flops per contracted Cartesian integral per density."""
    return 12 * n_dens * n_cartesian(la) * n_cartesian(lb) * n_cartesian(lc) * n_cartesian(ld)


def grad_prim_quartet_flops(la: int, lb: int, lc: int, ld: int) -> int:
    """Gradient model: the ERI model on the class with the bra raised by one
    (derivative integrals need l+1 on one centre), times the four centres
    less one by translational invariance."""
    return 3 * prim_quartet_flops(la + 1, lb, lc, ld)


assert prim_quartet_flops(0, 0, 0, 0) == 34
assert prim_quartet_flops(1, 1, 1, 1) == 1434
assert prim_quartet_flops(2, 2, 2, 2) == 48754
assert prim_quartet_flops(2, 0, 1, 0) == 353
