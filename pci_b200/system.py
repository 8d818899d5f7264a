"""Seeded synthetic CI systems in the layout pconf hands to FormH/Diag4.

A system is what pCI's ``pconf`` holds in module globals after ``Input``,
``Init``, ``Rint``, ``Dinit``, ``Det_Number`` and ``Det_List``
(src/pconf.F90:130-143) and ``InitFormH`` (src/pconf.F90:1049-1158):

* the orbital basis ``Nn, Ll, Kk, Jj`` (1-based orbital index ``ni``),
* the m-state tables ``Jz`` (2m) and ``Nh`` (orbital of an m-state),
  built as ``Dinit`` does (src/determinants.f90:47-105),
* the configuration list and the determinant list ``Iarr(Ne,Nd)`` with the
  per-configuration counts ``Ndc``, enumerated in ``Ndet`` order and sorted
  as ``Det_List``/``sort_det`` do (src/determinants.f90:144-183, 350-437,
  811-836),
* ``HintLUT(Nx*Nx)`` (src/integrals.f90:663-674) and the two-electron
  radial integrals ``Rint2/Iint2/Iint3`` on the canonical key set that
  ``Gint`` queries (src/integrals.f90:153-293),
* the Gaunt table of CONF.GNT (src/breit.f90:48-106).

The integral values are seeded synthetic stand-ins for ``pbasc`` output:
h_aa = -1/(2 n_eff^2) with n_eff = n - U(0.5, 2); h_ab ~ N(0, 1e-2) for
kappa_a = kappa_b; R^k(abcd) ~ N(0, 0.05 * 0.5^k) per canonical key.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

from . import wigner

__all__ = ["Basis", "CISystem", "make_basis", "make_system", "sd_excitations",
           "enumerate_determinants", "canonical_integral_keys", "CONFIGS"]

NX_DEFAULT = 440  # IPx, src/params.f90:30 (pbasc uses nx = IPx, src/pbasc.f90:889)


@dataclass
class Basis:
    """Relativistic orbital basis, arrays indexed by ni-1 (ni is 1-based)."""
    nn: np.ndarray
    ll: np.ndarray
    kk: np.ndarray
    jj: np.ndarray          # 2j
    nso: int = 0

    @property
    def ns(self) -> int:
        return int(self.nn.size)

    def label(self, ni: int) -> str:
        i = ni - 1
        return f"{self.nn[i]}{'spdfghik'[self.ll[i]]}{self.jj[i]}/2"


def make_basis(shells) -> Basis:
    """shells: iterable of (n, l).  Each (n, l) gives j = l-1/2 (if l>0) then j = l+1/2.

    Orbitals are ordered by the given (n, l) order, j = l-1/2 first, which is the
    order the reference's CONF.DAT lists them in (src/pconf.F90:483-502).
    """
    nn, ll, kk, jj = [], [], [], []
    for n, l in shells:
        for j2 in ([2 * l - 1] if l > 0 else []) + [2 * l + 1]:
            nn.append(n)
            ll.append(l)
            jj.append(j2)
            # kappa = -(l+1) for j = l+1/2, +l for j = l-1/2 (src/pconf.F90:507-514)
            kk.append(-(l + 1) if j2 == 2 * l + 1 else l)
    a = lambda x: np.asarray(x, dtype=np.int32)
    return Basis(a(nn), a(ll), a(kk), a(jj))


def m_states(basis: Basis, nsu: int):
    """Jz(Nst), Nh(Nst) and Nf0(Ns) as in Dinit (src/determinants.f90:61-83).

    m-states of orbital ni are contiguous, ordered by m = -j..j; Jz holds 2m.
    """
    jz, nh, nf0 = [], [], []
    i0 = 0
    for ni in range(1, nsu + 1):
        j2 = int(basis.jj[ni - 1])
        nf0.append(i0)
        for m2 in range(-j2, j2 + 1, 2):
            jz.append(m2)
            nh.append(ni)
            i0 += 1
    return np.asarray(jz, np.int32), np.asarray(nh, np.int32), np.asarray(nf0, np.int32)


def enumerate_determinants(basis: Basis, configs, ne: int, mj: int):
    """Determinants with M = mj for every configuration, in reference order.

    ``configs`` is a list of configurations; each is a list of (ni, nq) shells in
    CONF.INP order.  ``Ndet`` (src/determinants.f90:350-437) runs an odometer over
    shells with the last shell fastest, each shell's electrons stepping through
    m-state combinations in lexicographic order starting from the lowest m-states;
    ``Det_List`` keeps those with M == Mj and sorts each with ``sort_det``.
    Returns (Iarr[Nd, Ne] int32 of 1-based m-state indices, Ndc[Nc] int32).
    """
    nsu = max(ni for c in configs for ni, _ in c)
    jz, _, nf0 = m_states(basis, nsu)
    dets, ndc = [], []
    combo_cache = {}
    for conf in configs:
        shell_arrays = []
        for ni, nq in conf:
            if nq == 0:
                continue
            key = (ni, nq)
            if key not in combo_cache:
                j2 = int(basis.jj[ni - 1])
                base = int(nf0[ni - 1]) + 1
                combos = np.asarray(list(itertools.combinations(range(j2 + 1), nq)),
                                    dtype=np.int32).reshape(-1, nq) + base
                combo_cache[key] = combos
            shell_arrays.append(combo_cache[key])
        # cartesian product, first shell slowest (itertools.product order)
        sizes = [a.shape[0] for a in shell_arrays]
        idx = np.indices(sizes, dtype=np.int64).reshape(len(sizes), -1)
        parts = [shell_arrays[s][idx[s]] for s in range(len(sizes))]
        d = np.concatenate(parts, axis=1)
        m = jz[d - 1].sum(axis=1)
        d = d[m == mj]
        d.sort(axis=1)
        dets.append(d)
        ndc.append(d.shape[0])
    iarr = np.concatenate(dets, axis=0).astype(np.int32) if dets else np.zeros((0, ne), np.int32)
    return np.ascontiguousarray(iarr), np.asarray(ndc, dtype=np.int32)


def _conf_parity(basis, conf):
    return sum(int(basis.ll[ni - 1]) * nq for ni, nq in conf) % 2


def _conf_mmax(basis, conf):
    """Largest 2M a configuration can reach."""
    tot = 0
    for ni, nq in conf:
        j2 = int(basis.jj[ni - 1])
        ms = list(range(j2, -j2 - 1, -2))[:nq]
        tot += sum(ms)
    return tot


def sd_excitations(basis: Basis, refs, parity: int, mj: int, level: int = 2,
                   orbitals=None):
    """All configurations within `level` excitations of any reference configuration.

    A configuration is a sorted tuple of (ni, nq).  References come first in the
    given order; the rest follow in ascending tuple order.  Only configurations
    of the requested parity whose largest M reaches mj are kept.  This stands in
    for pCI's ``add`` program, which is outside the pconf hot path.
    """
    if orbitals is None:
        orbitals = list(range(1, basis.ns + 1))
    cap = {ni: int(basis.jj[ni - 1]) + 1 for ni in orbitals}

    def norm(occ):
        return tuple(sorted((ni, q) for ni, q in occ.items() if q > 0))

    refs_n = []
    for r in refs:
        occ = {}
        for ni in r:
            occ[ni] = occ.get(ni, 0) + 1
        refs_n.append(norm(occ))
    seen = set(refs_n)
    out = []
    frontier = list(dict.fromkeys(refs_n))
    for _ in range(level):
        nxt = []
        for conf in frontier:
            occ = dict(conf)
            for ni_from in list(occ):
                occ[ni_from] -= 1
                for ni_to in orbitals:
                    if occ.get(ni_to, 0) >= cap[ni_to]:
                        continue
                    occ[ni_to] = occ.get(ni_to, 0) + 1
                    c = norm(occ)
                    if c not in seen:
                        seen.add(c)
                        nxt.append(c)
                    occ[ni_to] -= 1
                occ[ni_from] += 1
        frontier = nxt
        out.extend(nxt)
    keep = [c for c in out if _conf_parity(basis, c) == parity and _conf_mmax(basis, c) >= mj]
    keep.sort()
    refs_kept = [r for r in dict.fromkeys(refs_n)
                 if _conf_parity(basis, r) == parity and _conf_mmax(basis, r) >= mj]
    return [list(c) for c in refs_kept] + [list(c) for c in keep]


def canonical_integral_keys(basis: Basis, nsu: int, nx: int = NX_DEFAULT, kbrt: int = 0):
    """Every radial-integral key Gint can ask for, with its k.

    Gint canonicalises (na,nb,nc,nd) so that na<=nc, nb<=nd, na<=nb and, for
    na==nb, nc<=nd (src/integrals.f90:201-227); it needs la+lb+lc+ld even and
    visits k = max(|ja-jc|,|jb-jd|)/2 .. min(ja+jc, jb+jd)/2 with k+la+lc even
    unless Breit integrals are present (src/integrals.f90:235-251).  Keys are
    iac = Nx*Nx*k + Nx*(na-Nso-1) + (nc-Nso) and ibd = Nx*(nb-Nso-1) + (nd-Nso)
    (src/integrals.f90:233-234, 253).  Returns arrays (na, nb, nc, nd, k, iac, ibd).
    """
    nso = basis.nso
    ll = basis.ll.astype(np.int64)
    jj = basis.jj.astype(np.int64)
    orbs = np.arange(nso + 1, nsu + 1, dtype=np.int64)
    out = [[] for _ in range(5)]
    for na in orbs:
        for nb in orbs[orbs >= na]:
            nc, nd = np.meshgrid(orbs[orbs >= na], orbs[orbs >= nb], indexing="ij")
            nc = nc.ravel()
            nd = nd.ravel()
            if na == nb:
                sel = nc <= nd
                nc, nd = nc[sel], nd[sel]
            la, lb = ll[na - 1], ll[nb - 1]
            lc, ld = ll[nc - 1], ll[nd - 1]
            par = ((la + lb + lc + ld) % 2) == 0
            nc, nd, lc, ld = nc[par], nd[par], lc[par], ld[par]
            ja, jb = jj[na - 1], jj[nb - 1]
            jc, jd = jj[nc - 1], jj[nd - 1]
            kmin = np.maximum(np.abs(ja - jc) // 2, np.abs(jb - jd) // 2)
            kmax = np.minimum((ja + jc) // 2, (jb + jd) // 2)
            nk = np.maximum(kmax - kmin + 1, 0)
            rep = np.repeat(np.arange(nc.size), nk)
            if rep.size == 0:
                continue
            off = np.arange(rep.size) - np.repeat(np.cumsum(nk) - nk, nk)
            k = kmin[rep] + off
            if kbrt == 0:
                ok = ((k + la + lc[rep]) % 2) == 0
                rep, k = rep[ok], k[ok]
            out[0].append(np.full(rep.size, na))
            out[1].append(np.full(rep.size, nb))
            out[2].append(nc[rep])
            out[3].append(nd[rep])
            out[4].append(k)
    na, nb, nc, nd, k = (np.concatenate(x).astype(np.int64) for x in out)
    iac = nx * nx * k + nx * (na - nso - 1) + (nc - nso)
    ibd = nx * (nb - nso - 1) + (nd - nso)
    return na, nb, nc, nd, k, iac, ibd


@dataclass
class CISystem:
    """One pconf problem: basis, determinants, integrals and Davidson settings."""
    name: str
    basis: Basis
    ne: int
    mj: int                      # 2*M_J (pconf's Mj)
    configs: list
    iarr: np.ndarray             # [Nd, Ne] int32, 1-based m-state indices
    ndc: np.ndarray              # [Nc] int32
    jz: np.ndarray               # [Nst] int32 (2m)
    nh: np.ndarray               # [Nst] int32 (1-based orbital)
    nsu: int
    nx: int
    hint_lut: np.ndarray         # [Nx*Nx] float64, entry ind-1 holds HintLUT(ind)
    rint2: np.ndarray            # [Ngint] or [Ngint,2] float32/float64
    iint2: np.ndarray            # [Ngint] int32
    iint3: np.ndarray            # [Ngint] int32
    kbrt: int
    nlx: int
    gaunt_in: np.ndarray
    gaunt_gnt: np.ndarray
    gaunt_per_wave: np.ndarray
    gaunt_lut: np.ndarray
    gj: float = 0.0
    xj_av: float = 0.0
    ecore: float = 0.0
    params: dict = field(default_factory=dict)

    @property
    def nd(self) -> int:
        return int(self.iarr.shape[0])

    @property
    def nc(self) -> int:
        return int(self.ndc.size)

    @property
    def nst(self) -> int:
        return int(self.jz.size)

    @property
    def ngint(self) -> int:
        return int(self.iint2.size)

    @property
    def r2_is_f64(self) -> bool:
        return self.rint2.dtype == np.float64


def make_integrals(basis: Basis, nsu: int, seed: int, nx: int = NX_DEFAULT,
                   r2_dtype=np.float64, kbrt: int = 0):
    """Seeded synthetic HintLUT and Rint2/Iint2/Iint3 (see module docstring)."""
    rng = np.random.default_rng(seed)
    nso = basis.nso
    lut = np.zeros(nx * nx, dtype=np.float64)
    for na in range(nso + 1, nsu + 1):
        n_eff = basis.nn[na - 1] - rng.uniform(0.5, 2.0)
        lut[nx * (na - nso - 1) + (na - nso) - 1] = -1.0 / (2.0 * n_eff * n_eff)
    for na in range(nso + 1, nsu + 1):
        for nb in range(na + 1, nsu + 1):
            if basis.kk[na - 1] == basis.kk[nb - 1]:
                lut[nx * (na - nso - 1) + (nb - nso) - 1] = rng.normal(0.0, 1e-2)
    na, nb, nc, nd, k, iac, ibd = canonical_integral_keys(basis, nsu, nx, kbrt)
    sigma = 0.05 * np.power(0.5, k.astype(np.float64))
    vals = rng.standard_normal(k.size) * sigma
    if kbrt:
        br = rng.standard_normal(k.size) * sigma * 0.01
        rint2 = np.stack([vals, br], axis=1).astype(r2_dtype)
    else:
        rint2 = vals.astype(r2_dtype)
    return lut, rint2, iac.astype(np.int32), ibd.astype(np.int32)


def make_system(name: str, shells, ne: int, mj: int, parity: int, refs,
                seed: int, level: int = 2, r2_dtype=np.float64, kbrt: int = 0,
                orbitals=None, params=None, gj: float = 0.0, xj_av: float = 0.0,
                drop_empty: bool = True, max_nd=None, nso: int = 0) -> CISystem:
    """Build a seeded synthetic system.

    ``refs`` holds reference configurations as lists of orbital indices, one per
    electron (1-based).  Configurations are all excitations up to ``level`` of
    the references with the given parity; determinants have 2M = mj.  With
    ``max_nd`` the configuration list is cut after the first configuration at
    which the determinant count reaches ``max_nd``.  With ``nso`` the first
    nso orbitals are closed core shells (pconf's Nso): their m-states are
    numbered first, as Dinit numbers them, no determinant occupies them, and
    the integrals are keyed from orbital Nso + 1.
    """
    basis = make_basis(shells)
    basis.nso = int(nso)
    if nso and orbitals is None:
        orbitals = list(range(nso + 1, basis.ns + 1))
    configs = sd_excitations(basis, refs, parity, mj, level, orbitals)
    if max_nd is not None:
        configs = _truncate_configs(basis, configs, ne, mj, int(max_nd))
    iarr, ndc = enumerate_determinants(basis, configs, ne, mj)
    if drop_empty:
        keep = ndc > 0
        configs = [c for c, k in zip(configs, keep) if k]
        ndc = ndc[keep]
    nsu = max(ni for c in configs for ni, _ in c)
    jz, nh, _ = m_states(basis, nsu)
    lut, rint2, iint2, iint3 = make_integrals(basis, nsu, seed, NX_DEFAULT, r2_dtype, kbrt)
    lmax = int(basis.ll[:nsu].max())
    nlx, gin, ggnt, gper = wigner.gaunt_table(lmax)
    glut = wigner.gaunt_lut(gin, ggnt)
    p = dict(Nlv=6, N_it=200, Crt4=1e-8, Kl4=1, Kv=4, MaxNd0=3000, Nc4=len(configs),
             KXIJ=0, admix_crit=1e-6)
    if params:
        p.update(params)
    return CISystem(name=name, basis=basis, ne=ne, mj=mj, configs=configs, iarr=iarr,
                    ndc=ndc, jz=jz, nh=nh, nsu=nsu, nx=NX_DEFAULT, hint_lut=lut,
                    rint2=rint2, iint2=iint2, iint3=iint3, kbrt=kbrt, nlx=nlx,
                    gaunt_in=gin, gaunt_gnt=ggnt, gaunt_per_wave=gper, gaunt_lut=glut,
                    gj=gj, xj_av=xj_av, params=p)


def _truncate_configs(basis, configs, ne, mj, max_nd, chunk=256):
    """Leading configurations of ``configs`` whose determinant count first reaches max_nd."""
    total = 0
    for c0 in range(0, len(configs), chunk):
        part = configs[c0:c0 + chunk]
        _, ndc = enumerate_determinants(basis, part, ne, mj)
        csum = total + np.cumsum(ndc)
        hit = np.nonzero(csum >= max_nd)[0]
        if hit.size:
            return configs[:c0 + int(hit[0]) + 1]
        total = int(csum[-1]) if csum.size else total
    return configs


def _shells(lmax_n):
    """(n, l) list ordered by n then l, for l with n in the given inclusive ranges."""
    out = []
    for n in range(1, 40):
        for l, (nlo, nhi) in sorted(lmax_n.items()):
            if nlo <= n <= nhi:
                out.append((n, l))
    return out


# Workload definitions.  Each returns the keyword arguments of make_system.
CONFIGS = {}


def _register(fn):
    CONFIGS[fn.__name__] = fn
    return fn


@_register
def tiny(seed=11):
    """A few hundred determinants; used by unit tests."""
    shells = _shells({0: (3, 6), 1: (3, 5), 2: (3, 4)})
    b = make_basis(shells)
    refs = [[1, 2]]
    return dict(name="tiny", shells=shells, ne=2, mj=0, parity=0, refs=refs, seed=seed,
                params=dict(Nlv=4, MaxNd0=40))


@_register
def small3(seed=12):
    """Three electrons, odd parity, 2M = 1: a few thousand determinants."""
    shells = _shells({0: (3, 7), 1: (3, 6), 2: (3, 5), 3: (4, 4)})
    refs = [[1, 2, 2], [1, 1, 2], [1, 2, 4]]
    return dict(name="small3", shells=shells, ne=3, mj=1, parity=1, refs=refs, seed=seed,
                params=dict(Nlv=6, MaxNd0=300))


@_register
def small4(seed=13):
    """Four electrons, even parity, M = 0."""
    shells = _shells({0: (3, 5), 1: (3, 4), 2: (3, 4)})
    refs = [[1, 1, 2, 2], [1, 1, 3, 3], [1, 2, 2, 4]]
    return dict(name="small4", shells=shells, ne=4, mj=0, parity=0, refs=refs, seed=seed,
                params=dict(Nlv=6, MaxNd0=400))


@_register
def cfg1(seed=1):
    """Plain FP64 CI: 2 valence electrons over 40 relativistic orbitals (n <= 12, l <= 3),
    even parity, M_J = 0, all doubles from 5 reference configurations; 6 roots."""
    shells = _shells({0: (3, 12), 1: (3, 9), 2: (3, 8), 3: (4, 5)})
    refs = [[1, 1], [1, 3], [2, 2], [1, 4], [3, 3]]
    return dict(name="cfg1", shells=shells, ne=2, mj=0, parity=0, refs=refs, seed=seed,
                params=dict(Nlv=6, MaxNd0=3000))


# Small systems at the other electron counts the H-build is compiled for
# (one translation unit per Ne), used by the parity tests.
@_register
def ne1(seed=21):
    """One electron: every element is a one-electron (Hint) element."""
    shells = _shells({0: (3, 8), 1: (3, 6), 2: (3, 5)})
    return dict(name="ne1", shells=shells, ne=1, mj=1, parity=0, refs=[[1]], seed=seed,
                params=dict(Nlv=3, MaxNd0=6))


@_register
def ne5(seed=22):
    """Five electrons over eleven orbitals."""
    shells = _shells({0: (3, 5), 1: (3, 4), 2: (3, 4)})
    return dict(name="ne5", shells=shells, ne=5, mj=1, parity=1, refs=[[1, 1, 2, 3, 3]], seed=seed,
                params=dict(Nlv=3, MaxNd0=200))


@_register
def ne6(seed=23):
    """Six electrons over eight orbitals."""
    shells = _shells({0: (3, 4), 1: (3, 4), 2: (3, 3)})
    return dict(name="ne6", shells=shells, ne=6, mj=0, parity=0, refs=[[1, 1, 2, 2, 3, 3]], seed=seed,
                params=dict(Nlv=3, MaxNd0=200))


@_register
def ne8(seed=24):
    """Eight electrons over eight orbitals (the largest Ne compiled)."""
    shells = _shells({0: (3, 4), 1: (3, 4), 2: (3, 3)})
    return dict(name="ne8", shells=shells, ne=8, mj=0, parity=0, refs=[[1, 1, 2, 2, 3, 3, 4, 4]], seed=seed,
                params=dict(Nlv=3, MaxNd0=200))


def _random_refs(shells, ne, parity, n, nlow, seed):
    b = make_basis(shells)
    rng = np.random.default_rng(seed)
    cands = [list(c) for c in itertools.combinations(range(1, nlow + 1), ne)
             if sum(int(b.ll[i - 1]) for i in c) % 2 == parity]
    idx = rng.choice(len(cands), n, replace=False)
    return [cands[i] for i in sorted(idx)]


@_register
def cfg2(seed=2):
    """Plain FP64 at scale: 3 valence electrons, 120 orbitals (n <= 20, l <= 4), odd parity,
    M_J = 1/2, singles + doubles from 20 reference configurations; 10 roots."""
    shells = _shells({0: (3, 20), 1: (3, 17), 2: (3, 15), 3: (4, 14), 4: (5, 16)})
    refs = _random_refs(shells, 3, 1, 20, 28, seed)
    return dict(name="cfg2", shells=shells, ne=3, mj=1, parity=1, refs=refs, seed=seed,
                params=dict(Nlv=10, MaxNd0=3000))


@_register
def cfg3(seed=3, max_nd=1300000):
    """Precision-form system: 4 valence electrons, 140 orbitals (n <= 24, l <= 4), even
    parity, M_J = 0, singles + doubles from 8 reference configurations, 10 roots.  The
    full singles-and-doubles space (well over 5M determinants) holds a Hamiltonian far
    beyond one GPU, so the configuration list is cut at max_nd determinants: the largest
    system whose FP64 lower triangle (about 1.1e10 stored elements) fits one B200 beside
    the solver's buffers."""
    shells = _shells({0: (3, 24), 1: (3, 19), 2: (3, 17), 3: (4, 16), 4: (5, 18)})
    refs = _random_refs(shells, 4, 0, 8, 28, seed)
    return dict(name="cfg3", shells=shells, ne=4, mj=0, parity=0, refs=refs, seed=seed, max_nd=max_nd,
                params=dict(Nlv=10, MaxNd0=3000))


@_register
def mid(seed=2):
    """A config-2-like system at about 1/12 the size (3 electrons, 71 orbitals,
    ~86k determinants); used for profiling captures."""
    shells = _shells({0: (3, 12), 1: (3, 10), 2: (3, 9), 3: (4, 8), 4: (5, 7)})
    refs = _random_refs(shells, 3, 1, 6, 12, seed)
    return dict(name="mid", shells=shells, ne=3, mj=1, parity=1, refs=refs, seed=seed,
                params=dict(Nlv=10, MaxNd0=3000))


def _shells_count(norb, lmax):
    """Shells (n, l), n from l+1, ordered by n then l, cut where the number of
    relativistic orbitals (one for s, two otherwise) first reaches norb."""
    out, cnt = [], 0
    for n in range(1, 60):
        for l in range(0, min(lmax, n - 1) + 1):
            out.append((n, l))
            cnt += 1 if l == 0 else 2
            if cnt >= norb:
                return out
    return out


def batch_block(index, seed0=1000, nd_lo=2000, nd_hi=400000):
    """Block ``index`` of the batched workload: a synthetic ion with its own
    seed (seed0 + index) drawing a determinant count log-uniform in
    [nd_lo, nd_hi], 2-4 valence electrons (3-4 above 6000 determinants, 4
    above 60000, where fewer electrons cannot reach the count), 30-120
    orbitals (at least 60 for two electrons and 80 for four electrons above
    150000), l <= 2..4, parity and 2M (0/2 for even, 1/3 for odd electron
    counts); the configurations are the singles and doubles of two low-lying
    references, cut at that count."""
    seed = seed0 + index
    rng = np.random.default_rng(seed)
    nd_target = int(round(float(np.exp(rng.uniform(np.log(nd_lo), np.log(nd_hi))))))
    if nd_target <= 6000:
        ne = int(rng.integers(2, 5))
    elif nd_target <= 60000:
        ne = int(rng.integers(3, 5))
    else:
        ne = 4
    parity = int(rng.integers(0, 2))
    mj = int(rng.choice([0, 2])) if ne % 2 == 0 else int(rng.choice([1, 3]))
    nmin = 60 if ne == 2 else (80 if nd_target > 150000 else 30)
    norb = int(rng.integers(nmin, 121))
    lmax = int(rng.integers(2, 5))
    shells = _shells_count(norb, lmax)
    refs = _random_refs(shells, ne, parity, 2, ne + 6, seed)
    return dict(name=f"block{index}", shells=shells, ne=ne, mj=mj, parity=parity, refs=refs,
                seed=seed, max_nd=nd_target, params=dict(Nlv=6))


def batch_blocks(nblocks=64, seed0=1000, nd_lo=2000, nd_hi=400000):
    """make_system keyword arguments of every block of the batched workload."""
    return [batch_block(i, seed0, nd_lo, nd_hi) for i in range(nblocks)]


def _make_block(kw):
    return make_system(**kw)


def split_blocks(nds, world, rank):
    """Indices of the blocks rank `rank` of `world` solves: blocks taken largest
    first (by determinant count), each to the rank with the fewest determinants
    so far (lowest rank on ties).  Every rank computes the same split from the
    same counts, so no communication is needed; the ranks' sets partition the
    blocks."""
    order = sorted(range(len(nds)), key=lambda i: (-int(nds[i]), i))
    load = [0] * world
    mine = []
    for i in order:
        rk = min(range(world), key=lambda q: (load[q], q))
        load[rk] += int(nds[i])
        if rk == rank:
            mine.append(i)
    return mine


def squeeze_config(basis, conf):
    """conf_pt's Squeeze (src/conf_pt.f90:1266-1317): a configuration's shell
    list with adjacent relativistic shells of the same (n, l) merged, their
    occupations added: [((n, l), q), ...]."""
    out = []
    for ni, nq in conf:
        key = (int(basis.nn[ni - 1]), int(basis.ll[ni - 1]))
        if out and out[-1][0] == key:
            out[-1] = (key, out[-1][1] + int(nq))
        else:
            out.append((key, int(nq)))
    return out


def nr_layout(basis, configs, ndc):
    """conf_pt's NR_Init (src/conf_pt.f90:500-570): consecutive relativistic
    configurations with equal squeezed shell lists form one non-relativistic
    configuration.  Returns, per NR configuration (0-based), NRR (its first
    relativistic configuration), NRN (how many), Ndcnr (its determinants),
    Nvcnr (the shells of its relativistic configurations) and the
    determinant offsets (Ncnr + 1 entries: the reference's Ndic plus the
    end)."""
    ndc = np.asarray(ndc, np.int64)
    nrr, nrn, ndcnr, nvcnr = [], [], [], []
    prev = None
    for ic, conf in enumerate(configs):
        sq = squeeze_config(basis, conf)
        if prev is None or sq != prev:
            nrr.append(ic)
            nrn.append(0)
            ndcnr.append(0)
            nvcnr.append(0)
        nrn[-1] += 1
        ndcnr[-1] += int(ndc[ic])
        nvcnr[-1] += len(conf)
        prev = sq
    ndcnr = np.asarray(ndcnr, np.int64)
    return {"nrr": np.asarray(nrr, np.int64), "nrn": np.asarray(nrn, np.int64), "ndcnr": ndcnr,
            "nvcnr": np.asarray(nvcnr, np.int64), "offsets": np.concatenate([[0], np.cumsum(ndcnr)])}


def nr_configurations(basis, configs, ndc, nd1=None):
    """Determinant offsets of NR_Init's non-relativistic configurations
    (nr_layout's offsets).  With nd1, an NR configuration may not straddle
    the CI / PT boundary (NR_Init stops with an error there); ValueError."""
    offs = nr_layout(basis, configs, ndc)["offsets"]
    if nd1 is not None and int(nd1) not in set(offs.tolist()):
        raise ValueError("a non-relativistic configuration straddles the CI / PT boundary")
    return offs


def pt_row_ranges(ndc, nd1, parts):
    """conf_pt's PT space (the determinants from nd1, which ends a
    configuration, to the end of the list) cut into `parts` contiguous
    ranges of whole configurations with about equal determinant counts, as
    (row_lo, row_hi) pairs; empty ranges are dropped.  The second-order sums
    of the ranges add up to the whole PT space's (each PT row's terms are
    independent), so the ranges go to separate PT-block builds on one GPU
    or to separate ranks, with one sum of dE at the end."""
    ends = np.cumsum(np.asarray(ndc, np.int64))
    nd = int(ends[-1]) if len(ends) else 0
    if nd1 != 0 and nd1 not in set(ends.tolist()):
        raise ValueError("nd1 must end a configuration")
    out, lo = [], int(nd1)
    for p in range(1, parts + 1):
        target = nd1 + (nd - nd1) * p / parts
        k = int(np.searchsorted(ends, target))      # first end at or beyond the target
        hi = nd if p == parts else int(ends[min(k, len(ends) - 1)])
        if hi > lo:
            out.append((lo, hi))
            lo = hi
    return out


def make_batch(nblocks=64, seed0=1000, nd_lo=2000, nd_hi=400000, workers=None):
    """Every block of the batched workload as a CISystem, generated in a pool
    of spawned worker processes (safe to start after CUDA is initialised)."""
    import multiprocessing as mp
    import os
    kws = batch_blocks(nblocks, seed0, nd_lo, nd_hi)
    workers = workers or min(len(kws), os.cpu_count() or 1)
    if workers <= 1:
        return [make_system(**kw) for kw in kws]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_make_block, kws, chunksize=1)
