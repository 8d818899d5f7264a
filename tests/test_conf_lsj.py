"""conf_lsj's level table (PrintLSJ, src/conf_lsj.f90:958-1093) and PTE's
result table (src/conf_pt.f90:909-925) on the host."""
import numpy as np
import pytest

from conftest import get_system, oracle_h

from pci_b200 import conf_lsj as L
from pci_b200 import conf_pt as P


def test_lande_g_known_terms():
    # 2S1/2: 2; 2P1/2: 2/3; 2P3/2: 4/3; 3P1: 3/2; 1P1: 1
    got = L.lande_g([0.5, 0.5, 1.5, 1.0, 1.0], [0, 1, 1, 1, 1], [0.5, 0.5, 0.5, 1.0, 0.0])
    assert np.allclose(got, [2.0, 2 / 3, 4 / 3, 1.5, 1.0])
    assert np.isnan(L.lande_g(0.0, 0.0, 0.0))


def test_config_weights_sum_to_one_and_match_blocks():
    s = get_system("small3")
    import oracle as O
    (rp, col, val, *_), _ = oracle_h("small3")
    H = O.csr_to_dense(s.nd, rp, col, val)
    w, V = np.linalg.eigh(H)
    W = L.config_weights(V[:, :4], s.ndc)
    assert W.shape == (s.nc, 4)
    assert np.allclose(W.sum(axis=0), 1.0)
    ends = np.concatenate([[0], np.cumsum(s.ndc)])
    ic = 7
    assert W[ic, 2] == pytest.approx(np.sum(V[ends[ic]:ends[ic + 1], 2] ** 2))
    with pytest.raises(ValueError):
        L.config_weights(V[:-1, :2], s.ndc)


def test_level_table():
    E = np.array([-1.0, -0.99, -0.9])
    J = np.array([0.5, 1.5, 0.5])
    rows = L.level_table(E, J, [1, 1, 0], [0.5, 0.5, 0.5], gj=0.1, ecore=-0.5)
    et = E + 0.4 * J * (J + 1)
    assert rows[1][0] == 2 and rows[1][4] == pytest.approx(4 / 3)
    assert rows[2][5] == pytest.approx(et[2]) and rows[2][6] == pytest.approx(et[2] + 0.5)
    assert rows[1][7] == pytest.approx((et[0] - et[1]) * 2 * L.DPRY)
    assert rows[0][7] == 0.0


def test_pt_level_table_signs():
    E = np.array([-2.0, -1.9])            # the engine's eigenvalues
    dE = np.array([-0.01, -0.02])         # the engine's pt2 (negative: the levels go down)
    rows = P.pt_level_table(E, dE, J=[0.5, 1.5])
    assert rows[0][2] == 2.0 and rows[0][4] == pytest.approx(0.01)
    assert rows[1][3] == pytest.approx((2.0 - 1.9) * 2 * L.DPRY)
    assert rows[1][6] == pytest.approx(rows[1][3] + (0.01 - 0.02) * 2 * L.DPRY)
    assert rows[1][5] == pytest.approx(1.9 + 0.02)
