"""pdtm's reductions of one-particle density and transition density
matrices: RdcDM (src/pdtm.f90:2229-2441), the reduced density matrices of
ranks 0, 1 and 2 between the relativistic shells, the number of electrons
and the occupation numbers of the (n, l) shells; RdcTM (1681-2104), the
reduced transition matrices of ranks 0 to 3 between two levels.

The matrices come from the device (pci_gpu_density and
pci_gpu_transition_density, pdtm's FormDM and FormTM); the reductions are
host work over O(shells^2 x (2j+1)^2) numbers, as in the reference, which
runs them on its master rank.  The amplitudes that pdtm forms next from the
reduced matrices (hyperfine A and B, g-factors, E1/E2/E3/M1/M2/M3, EDM, PNC,
anapole and magnetic-quadrupole amplitudes) need its radial integrals of
the operators (DTM.INT, from the orbitals' radial functions); they are not
formed here.

Wigner 3j symbols are the exact ones of pci_b200.wigner (the reference's
Fj3 evaluates the same quantity with log-factorials).
"""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np

from .wigner import six_j, three_j


def _sgn(n: int) -> float:
    """The reference's Isgn, (-1)**n, which it only calls with n >= 0."""
    if n < 0:
        raise ValueError("Isgn of a negative argument")
    return -1.0 if n % 2 else 1.0


@lru_cache(maxsize=None)
def _tj(j2a: int, k: int, j2b: int, m2: int) -> float:
    """(ja k jb; -m 0 m) with ja = j2a/2, jb = j2b/2, m = m2/2."""
    return three_j(j2a / 2, k, j2b / 2, -m2 / 2, 0, m2 / 2)


@lru_cache(maxsize=None)
def _tjq(j2a: int, k: int, j2b: int, ma2: int, q2: int, mb2: int) -> float:
    """(ja k jb; -ma q mb) from doubled ja, jb, ma, q, mb."""
    return three_j(j2a / 2, k, j2b / 2, -ma2 / 2, q2 / 2, mb2 / 2)


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


def transition_parity(ro, nh, ll, imin=0, imax=None):
    """FormTM's parity of a transition (src/pdtm.f90:1614-1630): +1 or -1
    from the orbitals of the largest |Ro| element (the first in row-major
    order among equal ones)."""
    ro = np.asarray(ro, np.float64)
    if imax is None:
        imax = ro.shape[0] - 1
    sub = np.abs(ro[imin:imax + 1, imin:imax + 1])
    if not sub.any():
        raise ValueError("the transition density is zero")
    i, k = np.unravel_index(int(np.argmax(sub)), sub.shape)
    li, lk = int(ll[int(nh[imin + i]) - 1]), int(ll[int(nh[imin + k]) - 1])
    return 1 - 2 * ((li + lk) % 2)


def reduced_transition(ro, basis, nh, jz, tj1, mj1_2, tj2, mj2_2, parity=None, imin=0, imax=None):
    """RdcTM for a transition from level 1 (J1 = tj1, 2 M1 = mj1_2) to level
    2 (tj2, mj2_2): ro the transition density ([i, k] = Ro(initial m-state
    i+1, final m-state k+1), pci_gpu_transition_density's layout); parity
    +1 / -1 (None: transition_parity).  J values are rounded to
    half-integers as RdcDM does.

    For rank t = 0..3 and shells a (initial), b (final) whose l_a + l_b has
    the transition's parity,
    Rro_t(a, b) = sum over m_a, m_b of (-1)^(j_b - m_b) (j_b t j_a; -m_b q m_a)
    Ro(a m_a, b m_b) / [(-1)^(J2 - M2) (J2 t J1; -M2 q M1)], q = M2 - M1,
    each side times sqrt(2 j_a + 1), sqrt(2 J1 + 1) for t = 0; a rank whose
    denominator vanishes is None.  Returns dict shells, rro ([4]), parity,
    trace (of ro over imin..imax)."""
    ro = np.asarray(ro, np.float64)
    nh = np.asarray(nh)
    jz = np.asarray(jz)
    nn, ll, jj = basis.nn, basis.ll, basis.jj
    if imax is None:
        imax = ro.shape[0] - 1
    if parity is None:
        parity = transition_parity(ro, nh, ll, imin, imax)
    j1 = int(tj1 + tj1 + 0.1)
    j2 = int(tj2 + tj2 + 0.1)
    q2 = mj2_2 - mj1_2
    spans = rdc_shells(nh, jz, jj, imin, imax)
    shells = []
    for a, b in spans:
        no = int(nh[a]) - 1
        if int(nh[b]) - 1 != no or np.any(np.diff(jz[a:b + 1]) != 2):
            raise ValueError(f"RdcTM: wrong definition of shell {len(shells)}")
        shells.append((int(nn[no]), int(ll[no]), int(jj[no]), a, b))
    want_odd = (1 - parity) // 2
    rro = [None, None, None, None]
    for rank in range(4):
        c = _sgn((j2 - mj2_2) // 2) * _tjq(j2, rank, j1, mj2_2, q2, mj1_2)
        if c == 0.0:
            continue
        if rank == 0:
            c *= math.sqrt(j1 + 1)
        r = np.zeros((len(shells), len(shells)))
        for k, (nk, lk, jk, ik1, ik2) in enumerate(shells):
            for q, (nq, lq, jq, il1, il2) in enumerate(shells):
                if (lk + lq) % 2 != want_odd:
                    continue
                s = 0.0
                for il in range(il1, il2 + 1):
                    ml = int(jz[il])
                    for ik in range(ik1, ik2 + 1):
                        x = ro[ik, il]
                        if x != 0.0:
                            s += _sgn((jq - ml) // 2) * _tjq(jq, rank, jk, ml, q2, int(jz[ik])) * x
                if rank == 0:
                    s *= math.sqrt(jk + 1)
                r[k, q] = s / c
        rro[rank] = r
    return {"shells": shells, "rro": rro, "parity": parity,
            "trace": float(np.trace(ro[imin:imax + 1, imin:imax + 1]))}


def e1_amplitude(rt, radial):
    """RdcTM's reduced E1 amplitude in the length gauge (the l1 = 2 branch
    for a transition of parity -1, src/pdtm.f90:1810-1818, with amp_ops'
    AmpE1, src/amp_ops.f90): for each initial shell a and final shell b of
    the rank-1 reduced transition matrix, Rro_1(a, b) * radial(b, a) *
    (-1)^k * sqrt((2 j_b + 1)(2 j_a + 1) l_max) * {l_b j_b 1/2; j_a l_a 1},
    k = floor(j_a + l_max + 1.51), summed.  rt is reduced_transition's
    result; radial(final, initial) returns pdtm's E1 radial integral
    (Fint(3, ...), from its DTM.INT tables, which this engine does not form)
    for orbitals given as (n, l, 2j).  0 when the transition is not odd or
    has no rank-1 matrix."""
    r = rt["rro"][1]
    if rt["parity"] != -1 or r is None:
        return 0.0
    shells = rt["shells"]
    total = 0.0
    for a, (na, la, ja2, *_) in enumerate(shells):
        for b, (nb, lb, jb2, *_) in enumerate(shells):
            tme = r[a, b]
            if tme == 0.0:
                continue
            al = tme * radial((nb, lb, jb2), (na, la, ja2))
            if al == 0.0:
                continue
            lx = max(la, lb)
            k = int(ja2 / 2 + lx + 1.51)
            sign = -1.0 if k % 2 else 1.0
            c = math.sqrt((jb2 + 1) * (ja2 + 1) * lx) * six_j(lb, jb2 / 2, 0.5, ja2 / 2, la, 1)
            total += sign * c * al
    return total


def e2_amplitude(rt, radial):
    """RdcTM's reduced E2 amplitude (the l1 = 3 branch of an even
    transition, src/pdtm.f90:1849-1851, with amp_ops' AmpE2): for initial
    shell a and final shell b with |j_b - j_a| <= 2 <= j_a + j_b, minus the
    sum of Rro_2(a, b) * radial(b, a) * (-1)^floor(j_a + 0.51) *
    sqrt((2j_b+1)(2j_a+1)(2l_b+1)(2l_a+1)) * (l_b l_a 2; 0 0 0) *
    {j_b j_a 2; l_a l_b 1/2}.  radial(final, initial) is pdtm's E2 radial
    integral (Fint(10, ...)) for orbitals given as (n, l, 2j).  0 when the
    transition is not even or has no rank-2 matrix."""
    r = rt["rro"][2]
    if rt["parity"] != 1 or r is None:
        return 0.0
    shells = rt["shells"]
    total = 0.0
    for a, (na, la, ja2, *_) in enumerate(shells):
        for b, (nb, lb, jb2, *_) in enumerate(shells):
            if abs(jb2 - ja2) > 4 or jb2 + ja2 < 4:
                continue
            tme = r[a, b]
            if tme == 0.0:
                continue
            ae = tme * radial((nb, lb, jb2), (na, la, ja2))
            if ae == 0.0:
                continue
            total -= ae * _ek_angular(2, jb2, ja2, lb, la)
    return total


def _gj1(x, l):
    """pdtm's Gj1 (src/pdtm.f90:1664-1671)."""
    return (x + 0.5) * math.sqrt((2 * x + 1) * (4 * x - 2 * l + 1) / (2 * l + 1))


def _gjj(kx, l):
    """pdtm's Gjj (src/pdtm.f90:1673-1679), kx = 2j."""
    return _sgn((kx + 1) // 2 + l) * math.sqrt(2.0 * l * (l + 1) / (2 * l + 1))


def g_factor_nr(rd, overlap=None):
    """RdcDM's non-relativistic M1 g-factor (K_M1 = 1, src/pdtm.f90:2340-2352
    and 2392): over the rank-1 reduced density matrix, for shells a, b of
    one l that are the same orbital or spin-orbit partners (j_a /= j_b),
    Rro_1(a, b) * overlap(b, a) * (Gj1(j_a, l) when j_a = j_b, else Gjj(2 j_b,
    l)), summed and divided by sqrt(J(J+1)(2J+1)).  overlap(b, a) is pdtm's
    radial overlap (Fint(9, ...)) of orbitals given as (n, l, 2j); by default
    1 for equal n and 0 otherwise.  rd is reduced_density's result; 0 when
    its rank-1 matrix is absent."""
    r = rd["rro"][1]
    if r is None:
        return 0.0
    if overlap is None:
        overlap = lambda b, a: 1.0 if b[0] == a[0] and b[1] == a[1] else 0.0
    shells = rd["shells"]
    g = 0.0
    for a, (na, la, ja2, fa, _) in enumerate(shells):
        for b, (nb, lb, jb2, fb, _) in enumerate(shells):
            if la != lb:
                continue
            same = (na, la, ja2) == (nb, lb, jb2)
            if not (same or ja2 != jb2):
                continue
            g1 = r[a, b] * overlap((nb, lb, jb2), (na, la, ja2))
            g1 *= _gj1(ja2 / 2, la) if ja2 == jb2 else _gjj(jb2, lb)
            g += g1
    J = rd["J"]
    return g / math.sqrt(J * (J + 1) * (2 * J + 1)) if g != 0.0 else 0.0


# Hartree in cm^-1 as pdtm writes it (src/pdtm.f90:1704)
HARTREE_CM = 219474.63


def e1_rate(ae1, e1, e2, tj1, tj2):
    """RdcTM's E1 transition rate (src/pdtm.f90:1933-1949): the wavelength
    wl = |1e7 / dE| nm with dE = (e2 - e1) * 219474.63 cm^-1 and A =
    2.02613e18 AE1^2 / ((2J_u + 1) (10 wl)^3) s^-1, J_u the upper level's J
    (level 1 when e2 > e1).  Energies in the sign convention of CONF.XIJ
    (binding energies: the larger is the lower level).  Returns (wl, A)."""
    de = (e2 - e1) * HARTREE_CM
    if de == 0.0:
        raise ValueError("the two levels have the same energy")
    wl = abs(1e7 / de)
    ju = tj1 if e2 > e1 else tj2
    return wl, 2.02613e18 / ((2 * ju + 1) * (wl * 10) ** 3) * ae1 ** 2


# physical constants the reference uses (src/params.f90:14-21)
DPCL = 137.0359922594      # speed of light, a.u.
DPAU = 6.5796839e15        # a.u. of energy in Hz
DPMP = 1836.153            # proton mass, a.u.
DPRB = 0.529177249e-8      # Bohr radius, cm


def _hfs_a_angular(jb2, ja2, la):
    """HfsA's factor (src/amp_ops.f90) for column shell b (j_b) and row shell a
    (j_a, l_a): the sign (-1)^floor(j_a + l_a + 1.51) times
    sqrt((2j_b+1)(2j_a+1)/(min(j_a, j_b)+1)) between spin-orbit partners and
    (2j+1) sqrt((2j+1)/(j(j+1))) within one j."""
    jb, ja = jb2 / 2, ja2 / 2
    sign = -1.0 if int(ja + la + 1.51) % 2 else 1.0
    if abs(ja - jb) > 0.1:
        return sign * math.sqrt((2 * jb + 1) * (2 * ja + 1) / (min(ja, jb) + 1))
    return sign * (2 * jb + 1) * math.sqrt((2 * jb + 1) / (jb * (jb + 1)))


def hfs_constants(rd, radial_a, radial_b=None, gnuc=1.0, qnuc=1.0):
    """RdcDM's hyperfine constants A and B in MHz (src/pdtm.f90:2325-2392
    with amp_ops' HfsA and HfsB): A sums Rro_1(a, b) * radial_a(b, a) * HfsA's
    angular factor over shell pairs, B sums Rro_2(a, b) * radial_b(b, a) *
    (-1)^floor(j_a + 0.51) * sqrt((2j_b+1)(2j_a+1)(2l_b+1)(2l_a+1)) *
    (l_b l_a 2; 0 0 0) * {j_b j_a 2; l_a l_b 1/2}; then
    A = -gnuc / (4 c m_p) / sqrt(J(J+1)(2J+1)) * sum * au[Hz] * 1e-6 and
    B = -2 qnuc sqrt(J(2J-1) / ((J+1)(2J+1)(2J+3))) * sum * au[Hz] / r_B^2 *
    1e-30.  radial_a / radial_b(b, a) are pdtm's hyperfine radial integrals
    (Fint(1, ...), Fint(2, ...)) for orbitals given as (n, l, 2j); gnuc and
    qnuc the nuclear g-factor and quadrupole moment of CONF.INP (Gnuc,
    Qnuc).  Returns (A, B)."""
    shells = rd["shells"]
    J = rd["J"]
    a_sum = b_sum = 0.0
    r1, r2 = rd["rro"][1], rd["rro"][2]
    for a, (na, la, ja2, *_) in enumerate(shells):
        for b, (nb, lb, jb2, *_) in enumerate(shells):
            if r1 is not None and r1[a, b] != 0.0:
                v = r1[a, b] * radial_a((nb, lb, jb2), (na, la, ja2))
                if v != 0.0:
                    a_sum += v * _hfs_a_angular(jb2, ja2, la)
            if radial_b is not None and r2 is not None and r2[a, b] != 0.0:
                v = r2[a, b] * radial_b((nb, lb, jb2), (na, la, ja2))
                if v != 0.0:
                    b_sum += v * _ek_angular(2, jb2, ja2, lb, la)
    A = B = 0.0
    if a_sum != 0.0:
        A = -gnuc / (DPCL * 4 * DPMP) / math.sqrt(J * (J + 1) * (2 * J + 1)) * a_sum * DPAU * 1e-6
    if b_sum != 0.0:
        B = -2 * qnuc * math.sqrt(J * (2 * J - 1) / ((J + 1) * (2 * J + 1) * (2 * J + 3))) * b_sum \
            * DPAU / (DPRB * DPRB) * 1e-30
    return A, B


def _ek_angular(k, jb2, ja2, lb, la):
    """AmpE2 / AmpE3 / HfsB's factor for rank k, final (column) shell b and
    initial (row) shell a: (-1)^floor(j_a + 0.51) *
    sqrt((2j_b+1)(2j_a+1)(2l_b+1)(2l_a+1)) * (l_b l_a k; 0 0 0) *
    {j_b j_a k; l_a l_b 1/2}."""
    sign = -1.0 if int(ja2 / 2 + 0.51) % 2 else 1.0
    return sign * math.sqrt((jb2 + 1) * (ja2 + 1) * (2 * lb + 1) * (2 * la + 1)) \
        * three_j(lb, la, k, 0, 0, 0) * six_j(jb2 / 2, ja2 / 2, k, la, lb, 0.5)


def e3_amplitude(rt, radial):
    """RdcTM's reduced E3 amplitude (the l1 = 4 branch of an odd transition,
    src/pdtm.f90:1822-1826, with amp_ops' AmpE3): over initial shell a and
    final shell b with |j_b - j_a| <= 3 <= j_a + j_b, the sum of
    Rro_3(a, b) * radial(b, a) * the rank-3 factor of AmpE2's form.
    radial(final, initial) is pdtm's E3 radial integral (Fint(11, ...)) for
    orbitals given as (n, l, 2j)."""
    r = rt["rro"][3]
    if rt["parity"] != -1 or r is None:
        return 0.0
    total = 0.0
    for a, (na, la, ja2, *_) in enumerate(rt["shells"]):
        for b, (nb, lb, jb2, *_) in enumerate(rt["shells"]):
            if abs(jb2 - ja2) > 6 or jb2 + ja2 < 6 or r[a, b] == 0.0:
                continue
            v = r[a, b] * radial((nb, lb, jb2), (na, la, ja2))
            if v != 0.0:
                total += v * _ek_angular(3, jb2, ja2, lb, la)
    return total
