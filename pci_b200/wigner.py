"""Exact Wigner 3j symbols and the relativistic Gaunt table of CONF.GNT.

The table layout (index ``In``, value ``Gnt``, per-partial-wave counts) is the
one written by pCI's ``basc`` (src/breit.f90:48-106, ``Subroutine Gaunt``) and
read by ``pconf`` (src/pconf.F90:383-406).  The coefficient itself follows
``Gaun`` (src/breit.f90:108-128):

    Gaun(k, j1, m1, j2, m2) = (-1)^floor(|m1 + 1/2|) * sqrt((2j1+1)(2j2+1))
                              * (j1 j2 k; -m1 m2 q) * (j1 j2 k; 1/2 -1/2 0),
    q = m1 - m2.

The reference evaluates the 3j symbols with log-factorials in double
precision (``FJ3``, src/wigner.f90:13-124).  Here they are evaluated exactly
(Racah's closed formula over Python integers) and rounded once to float64, so
the table is an independent, exact restatement of the same quantity.
"""
from __future__ import annotations

import math
from fractions import Fraction
from functools import lru_cache

import numpy as np

__all__ = ["three_j", "six_j", "gaun", "gaunt_table", "gaunt_lut"]


def _is_int(x: Fraction) -> bool:
    return x.denominator == 1


@lru_cache(maxsize=None)
def _three_j_sq_sign(j1, j2, j3, m1, m2, m3):
    """Return (sign, value**2 as Fraction) of the 3j symbol; arguments are Fractions."""
    if m1 + m2 + m3 != 0:
        return 0, Fraction(0)
    for j, m in ((j1, m1), (j2, m2), (j3, m3)):
        if abs(m) > j or not _is_int(j - m):
            return 0, Fraction(0)
    if not (abs(j1 - j2) <= j3 <= j1 + j2) or not _is_int(j1 + j2 + j3):
        return 0, Fraction(0)
    f = math.factorial
    a = int(j1 + j2 - j3)
    b = int(j1 - j2 + j3)
    c = int(-j1 + j2 + j3)
    d = int(j1 + j2 + j3 + 1)
    tri = Fraction(f(a) * f(b) * f(c), f(d))
    pre = f(int(j1 + m1)) * f(int(j1 - m1)) * f(int(j2 + m2)) * f(int(j2 - m2)) \
        * f(int(j3 + m3)) * f(int(j3 - m3))
    kmin = max(0, int(j2 - j3 - m1), int(j1 - j3 + m2))
    kmax = min(a, int(j1 - m1), int(j2 + m2))
    s = Fraction(0)
    for k in range(kmin, kmax + 1):
        den = f(k) * f(a - k) * f(int(j1 - m1) - k) * f(int(j2 + m2) - k) \
            * f(int(j3 - j2 + m1) + k) * f(int(j3 - j1 - m2) + k)
        s += Fraction((-1) ** k, den)
    if s == 0:
        return 0, Fraction(0)
    phase = -1 if int(j1 - j2 - m3) % 2 else 1
    sign = phase * (1 if s > 0 else -1)
    return sign, tri * pre * s * s


def three_j(j1, j2, j3, m1, m2, m3) -> float:
    """Wigner 3j symbol (j1 j2 j3; m1 m2 m3), exact up to the final rounding."""
    args = tuple(Fraction(x).limit_denominator(2) for x in (j1, j2, j3, m1, m2, m3))
    sign, sq = _three_j_sq_sign(*args)
    if sign == 0:
        return 0.0
    # sqrt of an exact rational, correctly rounded via integer sqrt at 2^-120 scale
    num, den = sq.numerator, sq.denominator
    scale = 1 << 240
    root = math.isqrt(num * scale // den)
    return sign * (root / float(1 << 120))


def _tri_sq(a, b, c):
    """Delta(abc)^2 as a Fraction, or None when a, b, c break the triangle rule."""
    if not (abs(a - b) <= c <= a + b) or not _is_int(a + b + c):
        return None
    f = math.factorial
    return Fraction(f(int(a + b - c)) * f(int(a - b + c)) * f(int(-a + b + c)), f(int(a + b + c + 1)))


@lru_cache(maxsize=None)
def _six_j_exact(j1, j2, j3, j4, j5, j6):
    tris = [_tri_sq(j1, j2, j3), _tri_sq(j1, j5, j6), _tri_sq(j4, j2, j6), _tri_sq(j4, j5, j3)]
    if any(t is None for t in tris):
        return 0, Fraction(0)
    f = math.factorial
    a = [int(j1 + j2 + j3), int(j1 + j5 + j6), int(j4 + j2 + j6), int(j4 + j5 + j3)]
    b = [int(j1 + j2 + j4 + j5), int(j2 + j3 + j5 + j6), int(j3 + j1 + j6 + j4)]
    s = Fraction(0)
    for t in range(max(a), min(b) + 1):
        den = 1
        for x in a:
            den *= f(t - x)
        for y in b:
            den *= f(y - t)
        s += Fraction((-1) ** t * f(t + 1), den)
    if s == 0:
        return 0, Fraction(0)
    pre = tris[0] * tris[1] * tris[2] * tris[3]
    return (1 if s > 0 else -1), pre * s * s


def six_j(j1, j2, j3, j4, j5, j6) -> float:
    """Wigner 6j symbol {j1 j2 j3; j4 j5 j6}, Racah's closed formula over
    exact rationals, rounded once (the reference's Fj6 evaluates the same
    quantity in floating point)."""
    args = tuple(Fraction(x).limit_denominator(2) for x in (j1, j2, j3, j4, j5, j6))
    sign, sq = _six_j_exact(*args)
    if sign == 0:
        return 0.0
    num, den = sq.numerator, sq.denominator
    scale = 1 << 240
    root = math.isqrt(num * scale // den)
    return sign * (root / float(1 << 120))


def gaun(k: int, j1: float, m1: float, j2: float, m2: float) -> float:
    """Relativistic Gaunt coefficient, src/breit.f90:108-128."""
    is_ = int(abs(m1 + 0.5) + 0.1)
    sgn = -1.0 if is_ % 2 else 1.0
    q = m1 - m2
    return sgn * math.sqrt((2 * j1 + 1) * (2 * j2 + 1)) \
        * three_j(j1, j2, k, -m1, m2, q) * three_j(j1, j2, k, 0.5, -0.5, 0.0)


def gaunt_table(nlx: int):
    """Build (Nlx, In, Gnt, num_gaunts_per_partial_wave) in the CONF.GNT layout.

    Enumeration order and index formula follow src/breit.f90:62-94: j1 <= j2,
    k >= max(1, j2-j1) up to j1+j2, m1 > 0, all m2 with |m2-m1| <= k, and
    ``ind = jx*jx*(jx*jx*k + 2*jx*j1 + 2*j2) + jx*(j1+m1) + (j2+m2)``,
    jx = 2*Nlx+1.  Nlx is raised to at least 5 (src/breit.f90:55).
    """
    nlx = max(nlx, 5)
    lx = nlx + 1
    jx = 2 * lx - 1
    ins, gnts = [], []
    per_wave = np.zeros(nlx + 1, dtype=np.int32)
    for ij1 in range(1, lx + 1):
        j1 = ij1 - 0.5
        for ij2 in range(ij1, lx + 1):
            j2 = ij2 - 0.5
            jj2 = 2 * ij2
            kmin = max(ij2 - ij1 + 1, 2)
            kmax = ij1 + ij2
            if kmax < kmin:
                continue
            for kk in range(kmin, kmax + 1):
                k = kk - 1
                ind1 = int(jx * jx * k + 2 * jx * j1 + 2 * j2 + 0.1)
                for im1 in range(1, ij1 + 1):
                    m1 = im1 - 0.5
                    for im2 in range(1, jj2 + 1):
                        m2 = im2 - j2 - 1
                        if abs(int(m2 - m1)) > k:
                            continue
                        ind = int(jx * jx * ind1 + jx * (j1 + m1) + (j2 + m2) + 0.1)
                        ins.append(ind)
                        gnts.append(gaun(k, j1, m1, j2, m2))
                        per_wave[ij1 - 1] += 1
    return nlx, np.asarray(ins, dtype=np.int32), np.asarray(gnts, dtype=np.float64), per_wave


def gaunt_lut(ins: np.ndarray, gnts: np.ndarray) -> np.ndarray:
    """Direct-index LUT GauntLUT(0:max(In)), src/integrals.f90:702-715."""
    lut = np.zeros(int(ins.max()) + 1, dtype=np.float64)
    lut[ins] = gnts
    return lut
