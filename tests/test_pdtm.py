"""pdtm's reduction of the density matrix (RdcDM, src/pdtm.f90:2229-2441)
in pci_b200/pdtm.py: a one-electron state's reduced matrices are 1 in every
rank (the Wigner-Eckart ratio of a state to itself), the rank-0 diagonal is
each shell's occupation and sums to Ne, the (n, l) occupations add the two
relativistic shells, and the GPU density feeds the same reduction as the
oracle's."""
import numpy as np
import pytest

from conftest import get_system, oracle_h

from pci_b200 import pdtm as D
from pci_b200 import system as S


def _one_electron(m2):
    """2p1/2 and 2p3/2 m-states; one electron in 2p3/2 with 2m = m2."""
    b = S.make_basis([(2, 1)])
    nh = np.array([1, 1, 2, 2, 2, 2])
    jz = np.array([-1, 1, -3, -1, 1, 3])
    ro = np.zeros((6, 6))
    ro[2 + (m2 + 3) // 2, 2 + (m2 + 3) // 2] = 1.0
    return b, nh, jz, ro


@pytest.mark.parametrize("m2", [1, 3, -1])
def test_one_electron_reduced_matrices_are_one(m2):
    b, nh, jz, ro = _one_electron(m2)
    r = D.reduced_density(ro, b, nh, jz, tj=1.5, mj2=m2)
    assert [(n, l, j2) for n, l, j2, *_ in r["shells"]] == [(2, 1, 1), (2, 1, 3)]
    assert r["rro"][0] == pytest.approx(np.diag([0.0, 1.0]), abs=1e-15)
    for rank in (1, 2):
        want = np.zeros((2, 2))
        want[1, 1] = 1.0
        assert np.allclose(r["rro"][rank], want, atol=1e-14)
    assert r["nel"] == pytest.approx(1.0)
    assert r["occ"] == [(2, 1, pytest.approx(1.0))]


def test_rank_with_vanishing_denominator_is_skipped():
    # J = 3/2 and M = 3/2 against rank 1 is fine; J = 1/2 has no rank-2 matrix
    b = S.make_basis([(2, 1)])
    nh = np.array([1, 1, 2, 2, 2, 2])
    jz = np.array([-1, 1, -3, -1, 1, 3])
    ro = np.zeros((6, 6))
    ro[1, 1] = 1.0                                       # 2p1/2, m = 1/2
    r = D.reduced_density(ro, b, nh, jz, tj=0.5, mj2=1)
    assert r["rro"][2] is None
    assert r["rro"][1][0, 0] == pytest.approx(1.0)


def test_isgn_refuses_negative_arguments():
    assert D._sgn(0) == 1.0 and D._sgn(3) == -1.0
    with pytest.raises(ValueError):
        D._sgn(-1)


@pytest.mark.parametrize("name", ["cfg1", "small3"])
def test_rank0_is_the_shell_occupation(name):
    import oracle as O
    s = get_system(name)
    (rp, col, val, *_), (jr, jc, jv) = oracle_h(name)
    H = O.csr_to_dense(s.nd, rp, col, val)
    w, V = np.linalg.eigh(H)
    x = V[:, 0]
    tj = O.j_av(jr, jc, jv, x, s.nd)
    ro = O.Oracle(s).density(x, trd=0.0)
    r = D.reduced_density(ro, s.basis, s.nh, s.jz, tj=tj, mj2=s.mj)
    assert r["nel"] == pytest.approx(s.ne, abs=1e-9)
    for k, (n, l, j2, a, b) in enumerate(r["shells"]):
        assert r["rro"][0][k, k] == pytest.approx(np.trace(ro[a:b + 1, a:b + 1]), abs=1e-12)
    assert sum(p for *_, p in r["occ"]) == pytest.approx(s.ne, abs=1e-9)
    # adjacent shells of one (n, l) are merged
    assert all((a[0], a[1]) != (b[0], b[1]) for a, b in zip(r["occ"][:-1], r["occ"][1:]))
    # ranks are symmetric in the shells up to the 3j phase: rank 0 is symmetric
    assert np.allclose(r["rro"][0], r["rro"][0].T, atol=1e-12)


@pytest.mark.gpu
def test_reduction_of_device_density():
    import oracle as O
    from pci_b200.capi import Engine
    s = get_system("small3")
    (rp, col, val, *_), (jr, jc, jv) = oracle_h("small3")
    H = O.csr_to_dense(s.nd, rp, col, val)
    w, V = np.linalg.eigh(H)
    x = V[:, :1]
    tj = O.j_av(jr, jc, jv, x[:, 0], s.nd)
    with Engine(0) as e:
        e.load_system(s)
        ro = e.density(x)[0]
    want = D.reduced_density(O.Oracle(s).density(x[:, 0]), s.basis, s.nh, s.jz, tj=tj, mj2=s.mj)
    got = D.reduced_density(ro, s.basis, s.nh, s.jz, tj=tj, mj2=s.mj)
    for rank in range(3):
        if want["rro"][rank] is None:
            assert got["rro"][rank] is None
        else:
            assert np.allclose(got["rro"][rank], want["rro"][rank], rtol=1e-10, atol=1e-12)


def _sp_basis():
    """2s, 2p1/2, 2p3/2 m-states."""
    b = S.make_basis([(2, 0), (2, 1)])
    nh = np.array([1, 1, 2, 2, 3, 3, 3, 3])
    jz = np.array([-1, 1, -1, 1, -3, -1, 1, 3])
    return b, nh, jz


@pytest.mark.parametrize("ia,ib", [(1, 7), (1, 6), (1, 5), (2, 4), (0, 3), (6, 6), (5, 2)])
def test_one_electron_transition_is_one(ia, ib):
    """One electron from m-state ia to ib (2s, 2p1/2, 2p3/2 m-states): every
    rank the 3j symbols allow (the parity of l_a + l_b selects the shell
    pairs) reduces to 1 on that shell pair, the others are None."""
    b, nh, jz = _sp_basis()
    ma2, mb2 = int(jz[ia]), int(jz[ib])
    ro = np.zeros((8, 8))
    ro[ia, ib] = 1.0
    ja, jb = b.jj[nh[ia] - 1] / 2, b.jj[nh[ib] - 1] / 2
    r = D.reduced_transition(ro, b, nh, jz, ja, ma2, jb, mb2)
    assert r["parity"] == (1 if (b.ll[nh[ia] - 1] + b.ll[nh[ib] - 1]) % 2 == 0 else -1)
    ka = [k for k, sh in enumerate(r["shells"]) if sh[3] <= ia <= sh[4]][0]
    kb = [k for k, sh in enumerate(r["shells"]) if sh[3] <= ib <= sh[4]][0]
    nonzero = 0
    for rank in range(4):
        if r["rro"][rank] is None:
            continue
        nonzero += 1
        want = np.zeros_like(r["rro"][rank])
        want[ka, kb] = 1.0
        assert np.allclose(r["rro"][rank], want, atol=1e-14), rank
    assert nonzero >= 1


@pytest.mark.parametrize("name", ["cfg1", "small3"])
def test_transition_to_itself_reduces_as_the_density(name):
    """RdcTM of a level to itself (q = 0, even parity) equals RdcDM's
    matrices in ranks 0-2."""
    import oracle as O
    s = get_system(name)
    (rp, col, val, *_), (jr, jc, jv) = oracle_h(name)
    H = O.csr_to_dense(s.nd, rp, col, val)
    w, V = np.linalg.eigh(H)
    x = V[:, 1]
    tj = O.j_av(jr, jc, jv, x, s.nd)
    o = O.Oracle(s)
    ro = o.density(x, trd=0.0)
    tm = o.transition_density(o, x, x, trd=0.0)
    dm = D.reduced_density(ro, s.basis, s.nh, s.jz, tj=tj, mj2=s.mj)
    tr = D.reduced_transition(tm, s.basis, s.nh, s.jz, tj, s.mj, tj, s.mj)
    assert tr["parity"] == 1
    for rank in range(3):
        if dm["rro"][rank] is None:
            assert tr["rro"][rank] is None
        else:
            assert np.allclose(tr["rro"][rank], dm["rro"][rank], atol=1e-12)


@pytest.mark.gpu
def test_reduction_of_device_transition_density():
    import oracle as O
    from pci_b200.capi import Engine
    from test_density import _flipped
    si, sf = get_system("small3"), _flipped("small3")
    rng = np.random.default_rng(8)
    bi = rng.standard_normal(si.nd); bi /= np.linalg.norm(bi)
    bf = rng.standard_normal(sf.nd); bf /= np.linalg.norm(bf)
    want_ro = O.Oracle(sf).transition_density(O.Oracle(si), bi, bf)
    with Engine(0) as ei, Engine(0) as ef:
        ei.load_system(si)
        ef.load_system(sf)
        got_ro = ef.transition_density(ei, bi, bf)
    args = (si.basis, si.nh, si.jz, 1.5, si.mj, 2.5, sf.mj)
    want = D.reduced_transition(want_ro, *args)
    got = D.reduced_transition(got_ro, *args)
    assert got["parity"] == want["parity"] == -1
    for rank in range(4):
        if want["rro"][rank] is None:
            assert got["rro"][rank] is None
        else:
            assert np.allclose(got["rro"][rank], want["rro"][rank], rtol=1e-10, atol=1e-12)


def test_six_j_known_values():
    from pci_b200 import wigner as W
    # {a b c; 0 c b} = (-1)^(a+b+c) / sqrt((2b+1)(2c+1))
    for a, b, c in [(1, 1, 1), (0.5, 1, 0.5), (2, 1.5, 2.5), (1, 2, 2)]:
        want = (-1) ** int(round(a + b + c)) / np.sqrt((2 * b + 1) * (2 * c + 1))
        assert W.six_j(a, b, c, 0, c, b) == pytest.approx(want, abs=1e-15)
    assert W.six_j(0.5, 0.5, 1, 0.5, 0.5, 0) == pytest.approx(0.5, abs=1e-15)
    assert W.six_j(1, 0.5, 0.5, 2.5, 2, 1) == 0.0              # triangle (1/2 5/2 1) broken
    # orthogonality: sum_x (2x+1)(2f+1) {a b x; c d f}{a b x; c d f'} = delta(f, f')
    a, b, c, d = 1.5, 1, 1.5, 1
    for f in (0.5, 1.5, 2.5):
        for g in (0.5, 1.5, 2.5):
            s = sum((2 * x + 1) * (2 * f + 1) * W.six_j(a, b, x, c, d, f) * W.six_j(a, b, x, c, d, g)
                    for x in (0.5, 1.5, 2.5))
            assert s == pytest.approx(1.0 if f == g else 0.0, abs=1e-14)


def _c1_reduced(ja, la, jb, lb):
    """<jb lb || C^1 || ja la> from a 3j symbol: (-1)^(jb+1/2) sqrt((2jb+1)(2ja+1))
    (jb 1 ja; -1/2 0 1/2), zero unless la + lb is odd."""
    from pci_b200 import wigner as W
    if (la + lb) % 2 == 0:
        return 0.0
    return (-1) ** int(round(jb + 0.5)) * np.sqrt((2 * jb + 1) * (2 * ja + 1)) * W.three_j(jb, 1, ja, -0.5, 0, 0.5)


@pytest.mark.parametrize("ia,ib", [(1, 3), (1, 6), (3, 1), (6, 1), (0, 5)])
def test_one_electron_e1_amplitude_is_the_c1_reduced_element(ia, ib):
    """One electron between s1/2 and p1/2 / p3/2: the rank-1 reduced
    transition matrix is 1 on the pair, so with a unit radial integral the
    E1 amplitude's size is the single-particle <j_b||C^1||j_a>, computed
    here independently from a 3j symbol."""
    b, nh, jz = _sp_basis()
    ro = np.zeros((8, 8))
    ro[ia, ib] = 1.0
    ja2, jb2 = int(b.jj[nh[ia] - 1]), int(b.jj[nh[ib] - 1])
    la, lb = int(b.ll[nh[ia] - 1]), int(b.ll[nh[ib] - 1])
    rt = D.reduced_transition(ro, b, nh, jz, ja2 / 2, int(jz[ia]), jb2 / 2, int(jz[ib]))
    if rt["rro"][1] is None:
        pytest.skip("rank 1 not allowed by the 3j denominator for these M")
    amp = D.e1_amplitude(rt, lambda f, i: 1.0)
    assert abs(amp) == pytest.approx(abs(_c1_reduced(ja2 / 2, la, jb2 / 2, lb)), rel=1e-13)
    # the radial integral scales it, and an even transition has none
    assert D.e1_amplitude(rt, lambda f, i: 2.5) == pytest.approx(2.5 * amp)
    even = dict(rt, parity=1)
    assert D.e1_amplitude(even, lambda f, i: 1.0) == 0.0


def _c2_reduced(ja, la, jb, lb):
    """<jb lb || C^2 || ja la> from a 3j symbol, zero unless la + lb is even."""
    from pci_b200 import wigner as W
    if (la + lb) % 2:
        return 0.0
    return (-1) ** int(round(jb + 0.5)) * np.sqrt((2 * jb + 1) * (2 * ja + 1)) * W.three_j(jb, 2, ja, -0.5, 0, 0.5)


@pytest.mark.parametrize("ia,ib", [(3, 6), (6, 3), (4, 6), (3, 5), (2, 5), (6, 2)])
def test_one_electron_e2_amplitude_is_the_c2_reduced_element(ia, ib):
    """One electron within 2p (p1/2 <-> p3/2, p3/2 <-> p3/2): with a unit
    radial integral the E2 amplitude's size is <j_b||C^2||j_a> from a 3j
    symbol; the odd s-p transitions and j = 1/2 pairs have none."""
    b, nh, jz = _sp_basis()
    ro = np.zeros((8, 8))
    ro[ia, ib] = 1.0
    ja2, jb2 = int(b.jj[nh[ia] - 1]), int(b.jj[nh[ib] - 1])
    la, lb = int(b.ll[nh[ia] - 1]), int(b.ll[nh[ib] - 1])
    rt = D.reduced_transition(ro, b, nh, jz, ja2 / 2, int(jz[ia]), jb2 / 2, int(jz[ib]))
    want = abs(_c2_reduced(ja2 / 2, la, jb2 / 2, lb))
    if rt["rro"][2] is None:
        pytest.skip("rank 2 not allowed by the 3j denominator for these M")
    amp = D.e2_amplitude(rt, lambda f, i: 1.0)
    assert abs(amp) == pytest.approx(want, rel=1e-13)
    assert want > 0


def test_e2_amplitude_of_odd_transition_is_zero():
    b, nh, jz = _sp_basis()
    ro = np.zeros((8, 8))
    ro[1, 6] = 1.0                                       # 2s -> 2p3/2
    rt = D.reduced_transition(ro, b, nh, jz, 0.5, 1, 1.5, 1)
    assert D.e2_amplitude(rt, lambda f, i: 1.0) == 0.0


@pytest.mark.parametrize("shells,orb,m2,want", [
    ([(2, 0)], 1, 1, 2.0),                    # s1/2
    ([(2, 1)], 1, -1, 2 / 3),                 # p1/2
    ([(2, 1)], 2, 3, 4 / 3),                  # p3/2
    ([(3, 2)], 1, 1, 4 / 5),                  # d3/2
    ([(3, 2)], 2, -3, 6 / 5),                 # d5/2
])
def test_g_factor_of_one_electron_is_lande(shells, orb, m2, want):
    """One electron in (n, l, j), J = j: RdcDM's non-relativistic g-factor
    is Lande's g_j = 1 + (j(j+1) - l(l+1) + 3/4) / (2j(j+1))."""
    b = S.make_basis(shells)
    jz, nh, _ = S.m_states(b, b.ns)
    ro = np.zeros((jz.size, jz.size))
    i = [k for k in range(jz.size) if nh[k] == orb and jz[k] == m2][0]
    ro[i, i] = 1.0
    j = b.jj[orb - 1] / 2
    rd = D.reduced_density(ro, b, nh, jz, tj=j, mj2=m2)
    assert D.g_factor_nr(rd) == pytest.approx(want, rel=1e-13)
    l = b.ll[orb - 1]
    assert want == pytest.approx(1 + (j * (j + 1) - l * (l + 1) + 0.75) / (2 * j * (j + 1)))


def test_e1_rate():
    # level 1 at 0.30 Ha binding, level 2 at 0.40 (more bound): 1 is the upper level
    wl, a = D.e1_rate(2.0, 0.30, 0.40, 1.5, 0.5)
    de = 0.10 * 219474.63
    assert wl == pytest.approx(1e7 / de)
    assert a == pytest.approx(2.02613e18 * 4.0 / (4 * (10 * wl) ** 3))
    # the other way round the upper level is 2
    wl2, a2 = D.e1_rate(2.0, 0.40, 0.30, 1.5, 0.5)
    assert wl2 == pytest.approx(wl) and a2 == pytest.approx(2.02613e18 * 4.0 / (2 * (10 * wl) ** 3))
    with pytest.raises(ValueError):
        D.e1_rate(1.0, 0.3, 0.3, 0.5, 0.5)


@pytest.mark.parametrize("shells,orb", [([(2, 0)], 1), ([(2, 1)], 1), ([(2, 1)], 2), ([(3, 2)], 1), ([(3, 2)], 2)])
def test_hfs_a_of_one_electron(shells, orb):
    """One electron in (n, l, j), M = J = j, unit radial integral: RdcDM's A
    sum over sqrt(j(j+1)(2j+1)) is 2|kappa| / (j(j+1)) in size, twice the
    textbook single-particle kappa / (j(j+1)) (pdtm's radial integral is
    the one of P Q, the textbook's of P Q + Q P); A follows with the
    reference's constants."""
    b = S.make_basis(shells)
    jz, nh, _ = S.m_states(b, b.ns)
    j2 = int(b.jj[orb - 1])
    ro = np.zeros((jz.size, jz.size))
    i = [k for k in range(jz.size) if nh[k] == orb and jz[k] == j2][0]
    ro[i, i] = 1.0
    j = j2 / 2
    rd = D.reduced_density(ro, b, nh, jz, tj=j, mj2=j2)
    A, B = D.hfs_constants(rd, lambda f, i_: 1.0, lambda f, i_: 1.0, gnuc=1.0, qnuc=1.0)
    kappa = int(b.kk[orb - 1])
    per = abs(A) / (1.0 / (D.DPCL * 4 * D.DPMP) * D.DPAU * 1e-6)
    assert per == pytest.approx(2 * abs(kappa) / (j * (j + 1)), rel=1e-13)
    if j < 1:
        assert B == 0.0                        # no quadrupole constant for J = 1/2
    else:
        # B's angular sum is <j||C^2||j> in size
        bsum = abs(B) / (2 * np.sqrt(j * (2 * j - 1) / ((j + 1) * (2 * j + 1) * (2 * j + 3)))
                         * D.DPAU / D.DPRB ** 2 * 1e-30)
        l = int(b.ll[orb - 1])
        assert bsum == pytest.approx(abs(_c2_reduced(j, l, j, l)), rel=1e-13)


def _c3_reduced(ja, la, jb, lb):
    from pci_b200 import wigner as W
    if (la + lb) % 2 == 0:
        return 0.0
    return (-1) ** int(round(jb + 0.5)) * np.sqrt((2 * jb + 1) * (2 * ja + 1)) * W.three_j(jb, 3, ja, -0.5, 0, 0.5)


@pytest.mark.parametrize("orb_a,orb_b", [(2, 4), (4, 2), (2, 3), (1, 4)])
def test_one_electron_e3_amplitude_is_the_c3_reduced_element(orb_a, orb_b):
    """One electron between 2p and 3d shells: with a unit radial integral
    the E3 amplitude's size is <j_b||C^3||j_a> from a 3j symbol (zero for
    p1/2 <-> d3/2, where j_a + j_b < 3)."""
    b = S.make_basis([(2, 1), (3, 2)])                      # 2p1/2 2p3/2 3d3/2 3d5/2
    jz, nh, _ = S.m_states(b, b.ns)
    ja2, jb2 = int(b.jj[orb_a - 1]), int(b.jj[orb_b - 1])
    la, lb = int(b.ll[orb_a - 1]), int(b.ll[orb_b - 1])
    want = abs(_c3_reduced(ja2 / 2, la, jb2 / 2, lb))
    found = False
    for ia in range(jz.size):
        for ib in range(jz.size):
            if nh[ia] != orb_a or nh[ib] != orb_b:
                continue
            ro = np.zeros((jz.size, jz.size))
            ro[ia, ib] = 1.0
            rt = D.reduced_transition(ro, b, nh, jz, ja2 / 2, int(jz[ia]), jb2 / 2, int(jz[ib]))
            if rt["rro"][3] is None:
                continue
            found = True
            assert abs(D.e3_amplitude(rt, lambda f, i: 1.0)) == pytest.approx(want, rel=1e-13, abs=1e-15)
    assert found or want == 0.0
