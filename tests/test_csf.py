"""CSF basis (kCSF = 1: jbasis, formh_sym, unsym; src/csf.f90).

CPU (oracle restatement): the CSFs are orthonormal, and the CSF
Hamiltonian's eigenvalues are exactly the determinant Hamiltonian's
eigenvalues whose J has 2J = Mj (J from J_av).
GPU: pci_gpu_form_csf against the oracle (per-configuration CSF counts, the
spectrum of the CSF matrix), pci_gpu_csf_to_det (the determinant vectors of
CSF eigenvectors are eigenvectors of H with 2J = Mj), and the batched solver
on the CSF matrix."""
import numpy as np
import pytest

from conftest import get_system, oracle_h


def _oracle(name):
    import oracle as O
    s = get_system(name)
    (rp, col, val, *_), J = oracle_h(name)
    H = O.csr_to_dense(s.nd, rp, col, val)
    counts, C = O.csf_basis(s, J)
    return s, H, J, counts, C


@pytest.mark.parametrize("name", ["tiny", "cfg1", "small3"])
def test_csf_oracle_spectrum_is_the_2j_eq_m_spectrum(name):
    import oracle as O
    s, H, (jr, jc, jv), counts, C = _oracle(name)
    assert np.abs(C.T @ C - np.eye(C.shape[1])).max() < 1e-12
    ec = np.linalg.eigvalsh(O.csf_hamiltonian(H, C))
    w, V = np.linalg.eigh(H)
    tj = np.array([O.j_av(jr, jc, jv, V[:, i], s.nd) for i in range(s.nd)])
    keep = np.abs(2 * tj - s.mj) < 1e-6
    assert keep.sum() == C.shape[1] == counts.sum()
    assert np.abs(ec - w[keep]).max() < 1e-10


def _gpu_csf(e, s):
    e.load_system(s)
    e.form_h(64)
    e.form_j()
    return e.form_csf()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "cfg1", "small3", "small4", "ne5"])
def test_csf_gpu_matches_oracle(name):
    import oracle as O
    from pci_b200.capi import Engine
    s, H, J, counts, C = _oracle(name)
    with Engine(0) as e:
        ncsf, nnz = _gpu_csf(e, s)
        got_counts = e.csf_counts(s.nc)
        rp, col, val = e.get_csr(0)
    assert ncsf == C.shape[1]
    assert np.array_equal(got_counts, counts)
    Hc = O.csr_to_dense(ncsf, rp, col, val)
    want = np.linalg.eigvalsh(O.csf_hamiltonian(H, C))
    assert np.abs(np.linalg.eigvalsh(Hc) - want).max() < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cfg1", "small3"])
def test_csf_to_det_gives_eigenvectors(name):
    import oracle as O
    from pci_b200.capi import Engine
    s, H, (jr, jc, jv), counts, C = _oracle(name)
    with Engine(0) as e:
        ncsf, nnz = _gpu_csf(e, s)
        rp, col, val = e.get_csr(0)
        Hc = O.csr_to_dense(ncsf, rp, col, val)
        w, Y = np.linalg.eigh(Hc)
        X = e.csf_to_det(Y[:, :6])
    assert np.abs(np.linalg.norm(X, axis=0) - 1).max() < 1e-10
    assert np.linalg.norm(H @ X - X * w[:6], axis=0).max() < 1e-9
    tj = np.array([O.j_av(jr, jc, jv, X[:, v], s.nd) for v in range(6)])
    assert np.abs(2 * tj - s.mj).max() < 1e-8


@pytest.mark.gpu
def test_csf_batched_solve():
    """The CSF matrix solved by the batched block Davidson: the lowest roots
    equal the dense eigenvalues of the oracle's C^T H C."""
    import oracle as O
    from pci_b200.capi import Batch, Engine
    s, H, J, counts, C = _oracle("small3")
    want = np.linalg.eigvalsh(O.csf_hamiltonian(H, C))[:6]
    with Engine(0) as e, Batch(0) as b:
        _gpu_csf(e, s)
        b.set_value_prec(64)
        b.add_engine(e)
        r = b.davidson(nlv=6, max_sub=48, keep=24, max_it=400, tol=1e-8)
    assert r["status"][0] == 1
    assert np.abs(r["E"][0] - want).max() < 1e-9


@pytest.mark.gpu
def test_csf_errors():
    from pci_b200.capi import Engine, PciError
    s = get_system("tiny")
    with Engine(0) as e:
        e.load_system(s)
        e.form_h(64)
        with pytest.raises(PciError):
            e.form_csf()                          # no J^2 yet
        e.form_j()
        e.form_csf()
        with pytest.raises(PciError):
            e.davidson(s.nd, Nlv=2)               # the resident matrix is the CSF one
