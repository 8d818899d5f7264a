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
