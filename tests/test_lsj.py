"""LSJ (src/pconf.F90:2672-2962, the kLSJ = 1 step): J, L, S of each level.

CPU (oracle restatement, pinned by known answers): one electron gives J = j,
L = l, S = 1/2 of the orbital; J equals J_av over the J^2 matrix (the same
F_J2 terms, src/formj2.f90:13-46) for any vectors; a J = 0 level has L = S;
the sums over configuration ranges add up (calcLSJ's work split).
GPU: pci_gpu_lsj against the oracle on eigenvectors and random vectors."""
import numpy as np
import pytest

from conftest import get_system, oracle_h


def _dense(name):
    s = get_system(name)
    (rp, col, val, *_), (jr, jc, jv) = oracle_h(name)
    H = np.zeros((s.nd, s.nd))
    rows = np.repeat(np.arange(s.nd), np.diff(rp))
    H[rows, col - 1] = val
    H = H + H.T - np.diag(np.diag(H))
    w, V = np.linalg.eigh(H)
    return s, V, (jr, jc, jv)


def test_lsj_one_electron_known_answer():
    import oracle as O
    s, V, _ = _dense("ne1")
    o = O.Oracle(s)
    xj, xl, xs = o.lsj(V[:, :8])
    for v in range(8):
        n = int(np.argmax(np.abs(V[:, v])))
        orb = s.nh[s.iarr[n, 0] - 1] - 1
        assert abs(xj[v] - s.basis.jj[orb] / 2) < 1e-12
        assert abs(xl[v] - s.basis.ll[orb]) < 1e-12
        assert abs(xs[v] - 0.5) < 1e-12


@pytest.mark.parametrize("name", ["tiny", "cfg1", "small3", "small4"])
def test_lsj_j_equals_j_av(name):
    import oracle as O
    s, V, (jr, jc, jv) = _dense(name)
    o = O.Oracle(s)
    rng = np.random.default_rng(4)
    X = np.concatenate([V[:, :6], rng.standard_normal((s.nd, 2))], axis=1)
    X /= np.linalg.norm(X, axis=0)
    xj, xl, xs = o.lsj(X)
    tj = np.array([O.j_av(jr, jc, jv, X[:, v], s.nd) for v in range(X.shape[1])])
    assert np.allclose(xj, tj, rtol=0, atol=1e-10)
    assert np.all(np.isfinite(xl)) and np.all(np.isfinite(xs))


@pytest.mark.parametrize("name", ["tiny", "cfg1"])
def test_lsj_j0_levels_have_l_equal_s(name):
    import oracle as O
    s, V, _ = _dense(name)
    xj, xl, xs = O.Oracle(s).lsj(V[:, :12])
    j0 = np.abs(xj) < 1e-8
    assert j0.any()
    assert np.allclose(xl[j0], xs[j0], atol=1e-9)


def test_lsj_configuration_ranges_add_up():
    import oracle as O
    s, V, _ = _dense("small3")
    o = O.Oracle(s)
    full = o.lsj_sums(V[:, :4])
    half = s.nc // 2
    parts = o.lsj_sums(V[:, :4], 1, half) + o.lsj_sums(V[:, :4], half + 1, s.nc)
    assert np.allclose(full, parts, rtol=1e-13, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ne1", "tiny", "cfg1", "small3", "small4", "ne5", "ne6", "ne8"])
def test_lsj_gpu_matches_oracle(name):
    import oracle as O
    from pci_b200.capi import Engine
    s = get_system(name)
    rng = np.random.default_rng(11)
    X = rng.standard_normal((s.nd, 10))
    X /= np.linalg.norm(X, axis=0)
    want = O.Oracle(s).lsj_sums(X)
    with Engine(0) as e:
        e.load_system(s)
        xj, xl, xs = e.lsj(X)
    got = np.stack([xj, xl, xs])
    ref = 0.5 * (np.sqrt(want + 1) - 1)
    assert np.allclose(got, ref, rtol=1e-11, atol=1e-11), (got, ref)


@pytest.mark.gpu
def test_lsj_gpu_eigenvectors_and_j_av():
    """Eigenvectors of cfg1 through the device: J from LSJ equals J_av's."""
    from pci_b200.capi import Engine
    s, V, _ = _dense("cfg1")
    X = V[:, :12]
    with Engine(0) as e:
        e.load_system(s)
        e.form_j()
        xj, xl, xs = e.lsj(X)
        tj = e.j_av(X)
    assert np.allclose(xj, tj, atol=1e-10)
    j0 = np.abs(xj) < 1e-8
    assert np.allclose(xl[j0], xs[j0], atol=1e-9)


@pytest.mark.gpu
def test_lsj_gpu_errors():
    from pci_b200.capi import Engine, PciError
    s = get_system("tiny")
    with Engine(0) as e:
        with pytest.raises(PciError):
            e.lsj(np.ones((s.nd, 1)))            # no basis
        e.load_system(s)
        with pytest.raises(PciError):
            e.lsj(np.ones((s.nd, 65)))           # more than 64 vectors
