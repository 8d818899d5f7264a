"""One-particle density matrices (pdtm's FormDM, src/pdtm.f90:1134-1336).

CPU (oracle restatement): the trace of Ro is Ne for a normalised vector;
Ro is symmetric; for a single determinant it is the projector on its
occupied m-states.  GPU: pci_gpu_density against the oracle."""
import numpy as np
import pytest

from conftest import get_system, oracle_h


def _vectors(name, nv=3):
    import oracle as O
    s = get_system(name)
    (rp, col, val, *_), _ = oracle_h(name)
    H = O.csr_to_dense(s.nd, rp, col, val)
    w, V = np.linalg.eigh(H)
    return s, V[:, :nv]


@pytest.mark.parametrize("name", ["tiny", "cfg1", "small3"])
def test_density_oracle_trace_and_symmetry(name):
    import oracle as O
    s, X = _vectors(name)
    o = O.Oracle(s)
    for v in range(X.shape[1]):
        ro = o.density(X[:, v], trd=0.0)               # no cut-off: the trace is exactly Ne
        assert abs(np.trace(ro) - s.ne) < 1e-10
        assert np.allclose(ro, ro.T, atol=1e-14)
        ev = np.linalg.eigvalsh(ro)
        assert ev.min() > -1e-10 and ev.max() < 1 + 1e-10        # occupations in [0, 1]


def test_density_oracle_single_determinant():
    import oracle as O
    s = get_system("small3")
    o = O.Oracle(s)
    b = np.zeros(s.nd)
    b[37] = 1.0
    ro = o.density(b)
    want = np.zeros((s.nst, s.nst))
    for m in s.iarr[37]:
        want[m - 1, m - 1] = 1.0
    assert np.array_equal(ro, want)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "cfg1", "small3", "small4", "ne5", "ne8"])
def test_density_gpu_matches_oracle(name):
    import oracle as O
    from pci_b200.capi import Engine
    s = get_system(name)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((s.nd, 3))
    X /= np.linalg.norm(X, axis=0)
    X[::17, 0] = 1e-12                                  # below the threshold: left out as the reference does
    o = O.Oracle(s)
    with Engine(0) as e:
        e.load_system(s)
        ro = e.density(X)
    for v in range(3):
        want = o.density(X[:, v])
        assert np.allclose(ro[v], want, rtol=1e-11, atol=1e-13)


def _flipped(name):
    from pci_b200 import system as S
    kw = dict(S.CONFIGS[name]())
    kw["parity"] = 1 - kw["parity"]
    return S.make_system(**kw)


def test_transition_density_oracle_same_level_is_density():
    """FormTM from a level to itself in the same basis equals FormDM."""
    import oracle as O
    s, X = _vectors("small3")
    o = O.Oracle(s)
    for v in range(2):
        tm = o.transition_density(o, X[:, v], X[:, v], trd=0.0)
        assert np.allclose(tm, o.density(X[:, v], trd=0.0), atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small3", "cfg1", "small4"])
def test_transition_density_gpu_matches_oracle(name):
    """Initial levels over one parity's basis, final levels over the other's."""
    import oracle as O
    from pci_b200.capi import Engine
    si, sf = get_system(name), _flipped(name)
    rng = np.random.default_rng(8)
    bi = rng.standard_normal(si.nd); bi /= np.linalg.norm(bi)
    bf = rng.standard_normal(sf.nd); bf /= np.linalg.norm(bf)
    want = O.Oracle(sf).transition_density(O.Oracle(si), bi, bf)
    with Engine(0) as ei, Engine(0) as ef:
        ei.load_system(si)
        ef.load_system(sf)
        got = ef.transition_density(ei, bi, bf)
        same = ei.transition_density(ei, bi, bi, trd=0.0)
        dm = ei.density(bi, trd=0.0)[0]
    assert np.abs(want).max() > 0
    assert np.allclose(got, want, rtol=1e-11, atol=1e-13)
    assert np.allclose(same, dm, atol=1e-12)
