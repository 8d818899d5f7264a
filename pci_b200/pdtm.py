"""pdtm's reduction of a one-particle density matrix (RdcDM,
src/pdtm.f90:2229-2441): the reduced density matrices of ranks 0, 1 and 2
between the relativistic shells, the number of electrons and the occupation
numbers of the (n, l) shells.

The density matrix comes from the device (pci_gpu_density, pdtm's FormDM);
this reduction is host work over O(shells^2 x 2j+1) numbers, as in the
reference, which runs it on its master rank.  The hyperfine constants A and B
and the g-factors that RdcDM forms next from these matrices need pdtm's
radial integrals of the operators (DTM.INT, from the orbitals' radial
functions); they are not formed here.

Wigner 3j symbols are the exact ones of pci_b200.wigner (the reference's
Fj3 evaluates the same quantity with log-factorials).
"""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

from .wigner import three_j


def _sgn(n: int) -> float:
    """The reference's Isgn, (-1)**n, which it only calls with n >= 0."""
    if n < 0:
        raise ValueError("Isgn of a negative argument")
    return -1.0 if n % 2 else 1.0


@lru_cache(maxsize=None)
def _tj(j2a: int, k: int, j2b: int, m2: int) -> float:
    """(ja k jb; -m 0 m) with ja = j2a/2, jb = j2b/2, m = m2/2."""
    return three_j(j2a / 2, k, j2b / 2, -m2 / 2, 0, m2 / 2)


def rdc_shells(nh, jz, jj, imin, imax):
    """RdcDM's division of the m-states imin..imax (0-based, inclusive) into
    shells: runs of one orbital's m-states in which only Jz changes (the
    first and last may be cut short).  As in the reference's loop
    (pdtm.f90:2255-2267), a shell that would start at imax itself is not
    formed.  Returns [(first, last)]."""
    shells = []
    i = imin
    while i < imax:
        no = int(nh[i]) - 1
        i2 = i + (int(jj[no]) - int(jz[i])) // 2
        if i2 > imax:
            i2 = imax
        shells.append((i, i2))
        i = i2 + 1
    return shells


def reduced_density(ro, basis, nh, jz, tj, mj2, imin=0, imax=None):
    """RdcDM for one level: ro the density matrix over the m-states
    ([i, j] = Ro(i+1, j+1), pci_gpu_density's layout), basis the orbitals
    (nn, ll, jj = 2j), nh the 1-based orbital of each m-state, jz its 2m, tj
    the level's J (from J_av; rounded to a half-integer as the reference
    does), mj2 = 2 M.

    For rank k = 0, 1, 2 and shells a, b of equal parity,
    Rro_k(a, b) = sum over m of (-1)^(j_b - m) (j_b k j_a; -m 0 m) Ro(a m, b m)
    / [(-1)^(J - M) (J k J; -M 0 M)], each side times sqrt(2j + 1) for
    k = 0; a rank whose denominator vanishes is None.  Returns dict shells
    ([(n, l, 2j, first, last)]), rro ([3] of kmax x kmax or None), nel (the
    trace of the rank-0 matrix: the number of electrons in imin..imax) and
    occ ([(n, l, occupation)] of consecutive shells with equal n and l)."""
    ro = np.asarray(ro, np.float64)
    nh = np.asarray(nh)
    jz = np.asarray(jz)
    nn, ll, jj = basis.nn, basis.ll, basis.jj
    if imax is None:
        imax = ro.shape[0] - 1
    jt = int(tj + tj + 0.1)
    tjr = jt / 2.0
    spans = rdc_shells(nh, jz, jj, imin, imax)
    shells = []
    for a, b in spans:
        no = int(nh[a]) - 1
        if int(nh[b]) - 1 != no:
            raise ValueError(f"RdcDM: shell {len(shells)} spans two orbitals")
        shells.append((int(nn[no]), int(ll[no]), int(jj[no]), a, b))
    kmax = len(shells)
    rro = [None, None, None]
    nel = 0.0
    occ = []
    for rank in range(3):
        c = _sgn((jt - mj2) // 2) * three_j(tjr, rank, tjr, -mj2 / 2, 0, mj2 / 2)
        if c == 0.0:
            continue
        if rank == 0:
            c *= math.sqrt(2 * tjr + 1)
        r = np.zeros((kmax, kmax))
        for k, (nk, lk, jk, ik1, ik2) in enumerate(shells):
            for q, (nq, lq, jq, il1, il2) in enumerate(shells):
                s = 0.0
                if (lk + lq) % 2 == 0:
                    for ik in range(ik1, ik2 + 1):
                        mk = int(jz[ik])
                        il = il1 + (mk - int(jz[il1])) // 2        # the same m in shell q
                        if il1 <= il <= il2:
                            x = ro[ik, il]
                            if x != 0.0:
                                s += _sgn((jq - mk) // 2) * _tj(jq, rank, jk, mk) * x
                    if rank == 0:
                        s *= math.sqrt(jk + 1)
                r[k, q] = s / c
            if rank == 0:
                nel += r[k, k]
                if occ and occ[-1][0] == nk and occ[-1][1] == lk:
                    occ[-1] = (nk, lk, occ[-1][2] + r[k, k])
                else:
                    occ.append((nk, lk, r[k, k]))
        rro[rank] = r
    return {"shells": shells, "rro": rro, "nel": nel, "occ": occ, "J": tjr, "M": mj2 / 2}
