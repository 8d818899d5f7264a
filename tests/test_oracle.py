"""CPU checks of the oracle (the C restatement of FormH/Hmltn/Gint/Davidson).

The reference ships no tests or golden outputs and cannot be compiled here
(Fortran), so the oracle is checked against independent known answers:

* H from an explicit second-quantised Hamiltonian (creation/annihilation
  operators on sorted occupation lists) with two-electron integrals assembled
  from exact 3j symbols -- this checks Rspq's phases and index conventions,
  Hmltn's integral selection, Gint's canonicalisation and k rules and the
  Gaunt table's symmetry folds, all at once;
* the Ne = 1 known answer (H is the one-electron matrix);
* dense eigensolves of the assembled H against the Davidson restatement;
* J^2 eigenvalues 4J(J+1) and integer or half-integer J from J_av;
* the two reference compare paths (Rspq and the bit-string path).
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from conftest import get_system, oracle_h
from pci_b200 import system as S
from pci_b200 import wigner


def micro(ne, parity, mj, seed=5, shells=None, refs=None, level=2):
    shells = shells or S._shells({0: (3, 4), 1: (3, 4), 2: (3, 3)})
    b = S.make_basis(shells)
    if refs is None:
        refs = [[i for i in range(1, ne + 1)]]
    return S.make_system("micro", shells, ne, mj, parity, refs, seed, level=level,
                         params=dict(Nlv=3, MaxNd0=20))


# ---------------------------------------------------------------- 3j / Gaunt

def test_three_j_known_values():
    assert wigner.three_j(0.5, 0.5, 0, 0.5, -0.5, 0) == pytest.approx(2 ** -0.5, abs=1e-16)
    assert wigner.three_j(1, 1, 2, 1, -1, 0) == pytest.approx((1 / 30) ** 0.5, abs=1e-16)
    assert wigner.three_j(2, 2, 2, 0, 0, 0) == pytest.approx(-(2 / 35) ** 0.5, abs=1e-16)
    assert wigner.three_j(1, 1, 1, 0, 0, 0) == 0.0           # odd sum of j with m = 0
    assert wigner.three_j(1, 1, 3, 0, 0, 0) == 0.0           # triangle violated
    # orthogonality: sum_{m1,m2} (j1 j2 j3; m1 m2 m3)^2 = 1/(2j3+1)
    j1, j2, j3, m3 = 2.5, 1.5, 2, 1
    s = sum(wigner.three_j(j1, j2, j3, m1, -m1 - m3, m3) ** 2
            for m1 in np.arange(-j1, j1 + 1))
    assert s == pytest.approx(1 / (2 * j3 + 1), abs=1e-15)


def test_gaunt_table_layout():
    nlx, ins, gnt, per = wigner.gaunt_table(5)
    assert nlx == 5 and ins.size == gnt.size == per.sum()
    # Ngaunt for Nlx = 5 is the 2891 noted beside src/pconf.F90:391
    assert ins.size == 2891
    # The index formula of src/breit.f90:77-82 aliases entries whose j1 + m1
    # reaches jx = 2*Nlx+1, i.e. j1 = m1 = Nlx + 1/2; every other index is unique.
    uniq, counts = np.unique(ins, return_counts=True)
    assert int((counts > 1).sum()) == 35 and counts.max() == 2
    lut = wigner.gaunt_lut(ins, gnt)
    assert lut.size == ins.max() + 1


def test_gaunt_lut_folds_match_direct_formula():
    """Gaunt() reads only the j1<=j2, m1>0 half of the table; its phases must
    reproduce Gaun for every argument Gint calls it with.  Gint's k range keeps
    |j1-j2| <= k <= j1+j2 for both factors; outside that range the index can
    alias a j = Nlx+1/2 entry, so those arguments are not compared."""
    s = get_system("small3")
    o = O.Oracle(s)
    for k in range(0, 10):
        for j1 in np.arange(0.5, 5.0):
            for j2 in np.arange(0.5, 5.0):
                if not (abs(j1 - j2) <= k <= j1 + j2):
                    continue
                for m1 in np.arange(-j1, j1 + 1):
                    for m2 in np.arange(-j2, j2 + 1):
                        g = o.gaunt(k, j1, m1, j2, m2)
                        if k == 0:
                            ref = 1.0 if (j1 == j2 and m1 == m2) else 0.0
                        elif abs(m2 - m1) > k:
                            ref = 0.0
                        else:
                            ref = wigner.gaun(k, j1, m1, j2, m2)
                        assert g == pytest.approx(ref, abs=1e-14), (k, j1, m1, j2, m2)


# -------------------------------------------------------- second quantisation

def _apply_annih(state, x):
    if x not in state:
        return None, 0
    i = state.index(x)
    return state[:i] + state[i + 1:], (-1) ** i


def _apply_creat(state, x):
    if x in state:
        return None, 0
    i = sum(1 for y in state if y < x)
    return state[:i] + (x,) + state[i:], (-1) ** i


def second_quantised_h(s):
    """<n|H|k> for H = sum h_pq a+_p a_q + 1/2 sum V(pqrs) a+_p a+_q a_s a_r with
    V(p,q,r,s) = sum_k [k+lp+lr even][k+lq+ls even] c^k(p,r) c^k(s,q) R^k(pqrs),
    c^k from exact 3j symbols and R^k looked up by canonical key."""
    nst = s.nst
    jz, nh = s.jz, s.nh
    ll, jj, kk = s.basis.ll, s.basis.jj, s.basis.kk
    nx, nso = s.nx, s.basis.nso
    R = {}
    for v, a, b in zip(np.atleast_1d(s.rint2), s.iint2, s.iint3):
        R[(int(a), int(b))] = float(v)

    def radial(a, b, c, d, k):   # 1-based orbitals
        if a > c: a, c = c, a
        if b > d: b, d = d, b
        if a > b: a, b, c, d = b, a, d, c
        if a == b and c > d: c, d = d, c
        iac = nx * nx * k + nx * (a - nso - 1) + (c - nso)
        ibd = nx * (b - nso - 1) + (d - nso)
        return R[(iac, ibd)]

    def V(p, q, r, s_):          # 0-based m-states
        if jz[p] + jz[q] != jz[r] + jz[s_]:
            return 0.0
        a, b, c, d = nh[p], nh[q], nh[r], nh[s_]
        la, lb, lc, ld = (int(ll[x - 1]) for x in (a, b, c, d))
        if (la + lb + lc + ld) % 2:
            return 0.0
        ja, jb, jc, jd = (int(jj[x - 1]) for x in (a, b, c, d))
        kmin = max(abs(ja - jc), abs(jb - jd)) // 2
        kmax = min(ja + jc, jb + jd) // 2
        e = 0.0
        for k in range(kmin, kmax + 1):
            if (k + la + lc) % 2:
                continue
            if k == 0:
                g1 = 1.0 if (ja == jc and jz[p] == jz[r]) else 0.0
                g2 = 1.0 if (jd == jb and jz[s_] == jz[q]) else 0.0
            else:
                g1 = wigner.gaun(k, ja / 2, jz[p] / 2, jc / 2, jz[r] / 2) if abs(jz[r] - jz[p]) <= 2 * k else 0.0
                g2 = wigner.gaun(k, jd / 2, jz[s_] / 2, jb / 2, jz[q] / 2) if abs(jz[q] - jz[s_]) <= 2 * k else 0.0
            if g1 == 0.0 or g2 == 0.0:
                continue
            e += g1 * g2 * radial(a, b, c, d, k)
        return e

    def h1(p, q):
        if jz[p] != jz[q] or kk[nh[p] - 1] != kk[nh[q] - 1]:
            return 0.0
        a, b = sorted((nh[p], nh[q]))
        return float(s.hint_lut[nx * (a - nso - 1) + (b - nso) - 1])

    dets = [tuple(int(x) - 1 for x in row) for row in s.iarr]
    index = {d: i for i, d in enumerate(dets)}
    Hm = np.zeros((len(dets), len(dets)))
    for kidx, dk in enumerate(dets):
        for q in dk:
            st1, s1 = _apply_annih(dk, q)
            for p in range(nst):
                st2, s2 = _apply_creat(st1, p)
                if st2 is None or st2 not in index:
                    continue
                Hm[index[st2], kidx] += s1 * s2 * h1(p, q)
        for r in dk:
            for s_ in dk:
                if r == s_:
                    continue
                st1, s1 = _apply_annih(dk, r)
                st2, s2 = _apply_annih(st1, s_)
                for q in range(nst):
                    st3, s3 = _apply_creat(st2, q)
                    if st3 is None:
                        continue
                    for p in range(nst):
                        if jz[p] + jz[q] != jz[r] + jz[s_]:
                            continue
                        st4, s4 = _apply_creat(st3, p)
                        if st4 is None or st4 not in index:
                            continue
                        v = V(p, q, r, s_)
                        if v != 0.0:
                            Hm[index[st4], kidx] += 0.5 * s1 * s2 * s3 * s4 * v
    return Hm


@pytest.mark.parametrize("ne,parity,mj", [(2, 0, 0), (3, 1, 1), (2, 1, 2)])
def test_oracle_matches_second_quantisation(ne, parity, mj):
    s = micro(ne, parity, mj)
    assert 10 < s.nd < 400
    rp, col, val, nz, hmin, pairs = O.Oracle(s).form_h()
    A = O.csr_to_dense(s.nd, rp, col, val)
    B = second_quantised_h(s)
    assert np.allclose(B, B.T, atol=1e-13)
    assert np.max(np.abs(A - B)) < 1e-12 * max(1.0, np.max(np.abs(B)))


def test_one_electron_known_answer():
    """Ne = 1: H is the one-electron matrix; its spectrum is the union of the
    kappa blocks of h (the same for every m)."""
    shells = S._shells({0: (3, 8), 1: (3, 7)})
    s = S.make_system("one", shells, 1, 1, 0, [[1]], seed=3, level=1, params=dict(Nlv=3, MaxNd0=10))
    rp, col, val, nz, hmin, pairs = O.Oracle(s).form_h()
    A = O.csr_to_dense(s.nd, rp, col, val)
    w = np.linalg.eigvalsh(A)
    b = s.basis
    ref = []
    for kappa in sorted(set(b.kk[:s.nsu].tolist())):
        orbs = [i for i in range(s.nsu) if b.kk[i] == kappa and b.jj[i] >= 1]
        if not orbs or (b.ll[orbs[0]] % 2) != 0:
            continue
        hk = np.array([[s.hint_lut[s.nx * min(a, c) + max(a, c)] for c in orbs] for a in orbs])
        ref.extend(np.linalg.eigvalsh(hk).tolist())
    assert np.allclose(np.sort(w), np.sort(ref), atol=1e-13)


# ------------------------------------------------------------ Davidson ---

@pytest.mark.parametrize("name", ["tiny", "cfg1"])
def test_davidson_matches_dense(name):
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    A = O.csr_to_dense(s.nd, rp, col, val)
    w = np.linalg.eigvalsh(A)
    p = dict(s.params)
    p["admix_crit"] = 0.0
    res = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    nlv = res["Tk"].size
    assert res["converged"]
    assert np.allclose(np.sort(-res["Tk"]), w[:nlv], atol=1e-9)
    # J values are integers or half integers
    assert np.allclose(2 * res["Tj"], np.round(2 * res["Tj"]), atol=1e-6)


def test_reference_davidson_stalls_on_synthetic_small3():
    """On small3 with the synthetic integrals, the reference's restarted
    Davidson (subspace 2*Nlv) is still far from Crt4 after 60 iterations while
    the dense eigenvalues are well separated."""
    s = get_system("small3")
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h("small3")
    p = dict(s.params)
    p.update(admix_crit=0.0, N_it=60)
    res = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    assert not res["converged"] and res["cnorm"].max() > 1e-3


def test_j2_spectrum():
    s = get_system("small3")
    _, (jr, jc, jv) = oracle_h("small3")
    w = np.linalg.eigvalsh(O.csr_to_dense(s.nd, jr, jc, jv))
    # eigenvalues of J^2 in units of (2j)^2 are (2J)(2J+2) = 4J(J+1), J half-integer for odd Ne
    tj = 0.5 * (np.sqrt(1 + w) - 1)
    assert np.allclose(2 * tj, np.round(2 * tj), atol=1e-8)
    assert np.allclose((np.round(2 * tj) % 2), 1)


def test_h_symmetric_structure_and_zero_drop():
    s = get_system("small4")
    (rp, col, val, nz, hmin, pairs), _ = oracle_h("small4")
    assert np.all(val != 0.0)
    assert pairs == rp[-1] + nz
    rows = np.repeat(np.arange(1, s.nd + 1), np.diff(rp))
    assert np.all(col <= rows)
    # columns ascending inside each row, diagonal last when present
    for n in range(0, s.nd, 97):
        c = col[rp[n]:rp[n + 1]]
        assert np.all(np.diff(c) > 0)
    assert hmin == val.min()


def test_rspq_vs_bit_path():
    """Both reference compare paths on random determinant pairs inside one 32-bit
    word: same difference count and differing m-states; the bit-string sign of
    get_det_indexes agrees with Rspq on every double difference, and on single
    differences except when no empty m-state precedes the difference, where it
    takes +1 (e.g. {1,2} -> {2,3}: Rspq -1, bit path +1)."""
    rng = np.random.default_rng(7)
    L = O.lib()
    stats = {1: [0, 0], 2: [0, 0]}
    for _ in range(4000):
        ne = int(rng.integers(2, 5))
        d1 = np.sort(rng.choice(np.arange(1, 33), ne, replace=False)).astype(np.int32)
        d2 = d1.copy()
        nchg = int(rng.integers(0, 3))
        pool = np.setdiff1d(np.arange(1, 33), d1)
        pos = rng.choice(ne, nchg, replace=False)
        d2[pos] = rng.choice(pool, nchg, replace=False)
        d2 = np.sort(d2).astype(np.int32)
        is1, nf1 = C.c_int(), C.c_int()
        i3 = np.zeros(3, np.int32); j3 = np.zeros(3, np.int32)
        L.orc_rspq(d1.ctypes.data_as(C.c_void_p), d2.ctypes.data_as(C.c_void_p), ne, C.byref(is1), C.byref(nf1),
                   i3.ctypes.data_as(C.c_void_p), j3.ctypes.data_as(C.c_void_p))
        b1 = np.array([np.bitwise_or.reduce(1 << (d1 - 1))], np.int64).astype(np.uint32).view(np.int32)
        b2 = np.array([np.bitwise_or.reduce(1 << (d2 - 1))], np.int64).astype(np.uint32).view(np.int32)
        nd_, is2 = C.c_int(), C.c_int()
        a1 = np.zeros(3, np.int32); a2 = np.zeros(3, np.int32)
        L.orc_bit_compare(b1.ctypes.data_as(C.c_void_p), b2.ctypes.data_as(C.c_void_p), 1, C.byref(nd_), C.byref(is2),
                          a1.ctypes.data_as(C.c_void_p), a2.ctypes.data_as(C.c_void_p))
        assert nd_.value == nf1.value
        nf = nf1.value
        if nf in (1, 2):
            assert set(a1[1:1 + nf]) == set(i3[1:1 + nf])
            stats[nf][1] += 1
            if is2.value == is1.value:
                stats[nf][0] += 1
            else:
                # only a single difference with no empty m-state below it
                assert nf == 1
                lo = min(int(a1[1]), int(a2[1]))
                occ = set(d1.tolist()) | set(d2.tolist())
                first = min(occ)
                assert all(m in occ for m in range(first, lo))
    assert stats[2][0] == stats[2][1] > 500
    assert stats[1][0] >= 0.99 * stats[1][1]


@pytest.mark.parametrize("name", ["tiny", "small3", "cfg1"])
def test_j_terms_match_j2_spectrum(name):
    """Jt of Dinit's term analysis = the 2J values in the J^2 spectrum."""
    s = get_system(name)
    _, (jr, jc, jv) = oracle_h(name)
    w = np.linalg.eigvalsh(O.csr_to_dense(s.nd, jr, jc, jv))
    two_j = sorted(set(np.round(np.sqrt(1 + w) - 1).astype(int).tolist()))
    assert O.j_terms(s.basis, s.configs, s.mj) == two_j


def test_davidson_kv3_matches_j_subspace():
    """Kv = 3 (J-selected FormB0, AvgDiag, Prj_J) converges to the lowest
    levels of H inside the J = XJ_av subspace, with J exact."""
    name, xj = "tiny", 0.0
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    A = O.csr_to_dense(s.nd, rp, col, val)
    wj, vj = np.linalg.eigh(O.csr_to_dense(s.nd, jr, jc, jv))
    P = vj[:, np.abs(np.sqrt(1 + wj) - 1 - 2 * xj) < 1e-6]
    exact = np.linalg.eigvalsh(P.T @ A @ P)
    p = dict(s.params, Kv=3, XJ_av=xj, Nlv=3, admix_crit=0.0)
    res = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc, jt=O.j_terms(s.basis, s.configs, s.mj))
    assert res["converged"]
    assert np.allclose(np.sort(-res["Tk"]), exact[:3], atol=1e-9)
    assert np.allclose(res["Tj"], xj, atol=1e-8)


def test_davidson_kv3_rejects_zero_term_filter():
    """A J = 0 term with XJ_av /= 0 makes Prj_J divide by zero in the reference."""
    s = get_system("tiny")
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h("tiny")
    p = dict(s.params, Kv=3, XJ_av=1.0, Nlv=3)
    with pytest.raises(ValueError, match="divides by zero"):
        O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc, jt=O.j_terms(s.basis, s.configs, s.mj))


@pytest.mark.parametrize("ne,parity,mj", [(2, 0, 0), (3, 1, 1)])
def test_oracle_with_core_shells_matches_second_quantisation(ne, parity, mj):
    """Closed core orbitals (Nso = 2: 1s and 2s in front of the valence
    shells), as every real CONF.INP has: the m-states of the core come first,
    determinants occupy none of them, and the radial-integral keys start at
    orbital Nso + 1.  The oracle's H equals the second-quantised one."""
    shells = [(1, 0), (2, 0)] + S._shells({0: (3, 4), 1: (3, 4), 2: (3, 3)})
    refs = [[i for i in range(3, ne + 3)]]
    s = S.make_system("core", shells, ne, mj, parity, refs, 5, level=2, params=dict(Nlv=3, MaxNd0=20), nso=2)
    assert s.basis.nso == 2 and s.iarr.min() > 2                # the 1s, 2s m-states (1, 2) never occupied
    assert 10 < s.nd < 600
    rp, col, val, nz, hmin, pairs = O.Oracle(s).form_h()
    A = O.csr_to_dense(s.nd, rp, col, val)
    B = second_quantised_h(s)
    assert np.max(np.abs(A - B)) < 1e-12 * max(1.0, np.max(np.abs(B)))
