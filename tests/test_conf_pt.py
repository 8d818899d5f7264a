"""conf_pt's host steps around PTE (src/conf_pt.f90: Weight_CI 573-654,
Weight_PT 991-1013, Cutoff 1015-1091, Sort 1093-1128, NewConfList
1130-1264), restated in pci_b200/conf_pt.py.  Known answers worked by hand
from the reference's loops, then the whole selection on a CI + PT split of a
test system with the oracle's per-NR-configuration sums."""
import numpy as np
import pytest

from conftest import get_system, oracle_h

from pci_b200 import conf_pt as P


def test_weight_ci_known_answer():
    # 3 NR configurations of 2, 1, 2 determinants (1, 1, 2 relativistic configurations)
    x0 = np.array([0.9, 0.3, 0.2, 0.2, np.sqrt(1 - 0.81 - 0.09 - 0.04 - 0.04)])
    x1 = np.array([0.1, 0.1, 0.97, 0.1, np.sqrt(1 - 0.01 - 0.01 - 0.9409 - 0.01)])
    X = np.stack([x0, x1], axis=1)
    r = P.weight_ci(X, [2, 1, 2], [1, 1, 2], cut0=0.05)
    # level 0: tails 0.10, 0.06, 0 -> below 0.05 after the third: Nd0 5
    # level 1: tails 0.98, 0.0391, 0 -> below after the second: Nd0 3
    assert r["nd0"] == 5 and r["nc0"] == 4 and r["ncnr0"] == 3
    assert r["wmax"] == pytest.approx(0.0391)               # the largest tail left out (level 1)
    assert np.allclose(r["dvnr"], [0.81 + 0.09 + 0.02, 0.04 + 0.9409, 0.04 + x0[4] ** 2 + 0.01 + x1[4] ** 2])
    # with cut0 = 0.5 level 0 stops after the first configuration (tail 0.1) and
    # level 1 after the second (0.0391): Nd0 = 3, the largest
    r = P.weight_ci(X, [2, 1, 2], [1, 1, 2], cut0=0.5)
    assert (r["nd0"], r["nc0"], r["ncnr0"]) == (3, 2, 2)
    assert r["wmax"] == pytest.approx(0.1)
    # ippt caps the zero-order space
    r = P.weight_ci(X, [2, 1, 2], [1, 1, 2], cut0=0.05, ippt=4)
    assert r["nd0"] == 3


def test_pt_nr_weights_and_weight_pt():
    dEg = np.array([[-1e-3, -2e-3], [-5e-4, 1e-5], [0.0, 0.0]])
    dVg = np.array([[1e-4, 2e-4], [3e-4, 1e-4], [0.0, 0.0]])
    r = P.pt_nr_weights(dEg, dVg)
    assert np.allclose(r["denr"], [2e-3, 5e-4, 0.0])
    assert np.allclose(r["dvnr"], [3e-4, 4e-4, 0.0])
    assert r["dvnrx"] == pytest.approx(4e-4) and r["ix"] == 1
    icci, icpt, dvnrn = P.weight_pt([0.9, 1e-5, 0.05], r["dvnr"], r["dvnrx"])
    assert (icci, icpt) == (1, 2) and dvnrn == pytest.approx(1e-5)


def test_cutoff_sort_new_list_known_answer():
    # 5 NR configurations, 2 of them the CI space; weights on a lg scale
    dvnr = np.array([0.8, 1e-6, 4e-3, 0.0, 5e-3])
    nrn = np.array([2, 1, 1, 1, 2])
    nrr = np.array([0, 2, 3, 4, 5])
    ndc = np.array([3, 3, 2, 4, 1, 2, 2])
    # ktf 1: threshold lg(5e-3 / 2); kept: 0.8, 4e-3, 5e-3
    c = P.cutoff(dvnr, nrn, 5e-3, ktf=1, kvar=1, ncnr0=1, ncnrci=2)
    assert c["nc_0"] == 0
    assert c["w"][:, 1].tolist() == [1, 0, 1, 0, 1]
    assert c["ncnew"] == 2 + 1 + 2
    assert c["w"][3, 0] == -99.0
    order = P.sort_nr(c["w"], c["nc_0"])
    assert order == [0, 4, 2, 1, 3]
    new = P.new_conf_list(order, c["w"], nrr, nrn, ndc, c["nc_0"], nc4=7, maxnd0=9, ncnrci=2)
    assert new["conf_order"] == [0, 1, 5, 6, 3, 2, 4]
    assert new["nci"] == c["ncnew"] == 5
    # Nc4: NR 0 (6 dets) fits in 9, NR 4 (4 more) does not
    assert new["nc4"] == 2 and new["kl4"] == 1
    assert new["weights"][0] == pytest.approx(0.8, rel=1e-6)
    # kvar 3 keeps the whole CI space in front, unsorted, and starts from the stored vectors
    c3 = P.cutoff(dvnr, nrn, 5e-3, ktf=1, kvar=3, ncnr0=1, ncnrci=2)
    assert c3["w"][:, 1].tolist() == [1, 1, 1, 0, 1]
    o3 = P.sort_nr(c3["w"], c3["nc_0"])
    assert o3[:2] == [0, 1] and o3[2:] == [4, 2, 3]
    n3 = P.new_conf_list(o3, c3["w"], nrr, nrn, ndc, c3["nc_0"], nc4=7, maxnd0=100, ncnrci=2)
    assert n3["kl4"] == 2 and n3["nci"] == c3["ncnew"] == 6 and n3["nc4"] == 7


def test_sort_is_the_reference_selection_sort():
    # equal weights: the first largest of the rest moves forward, swapping
    w = np.array([[-1.0, 1], [-2.0, 1], [-1.0, 1], [-1.0, 1]])
    assert P.sort_nr(w, 0) == [0, 2, 3, 1]


def test_select_configurations_on_a_ci_pt_split():
    """The whole selection on small3 with the first third of its NR
    configurations as the CI space, the lowest CI levels as X, and the
    oracle's per-NR-configuration sums as PTE's."""
    import oracle as O
    from pci_b200 import system as S
    s = get_system("small3")
    lay = S.nr_layout(s.basis, s.configs, s.ndc)
    offs = lay["offsets"]
    ncnrci = len(lay["nrn"]) // 3
    nd1 = int(offs[ncnrci])
    (rp, col, val, *_), _ = oracle_h("small3")
    H = O.csr_to_dense(s.nd, rp, col, val)
    w, V = np.linalg.eigh(H[:nd1, :nd1])
    X = V[:, :3]
    r0 = P.weight_ci(X, lay["ndcnr"][:ncnrci], lay["nrn"][:ncnrci], cut0=1e-3)
    nd0 = r0["nd0"]
    assert 0 < nd0 <= nd1 and nd0 in set(offs.tolist())
    dEg, dVg = O.pt2_groups(H, nd1, nd0, X[:nd0], w[:3], offs[ncnrci:], s.ndc)
    r = P.select_configurations(lay, ncnrci, s.ndc, X, dEg, dVg, cut0=1e-3, ktf=5, kvar=1)
    order = r["conf_order"]
    assert sorted(order) == list(range(s.nc))                     # a permutation of all configurations
    kept = r["cutoff"]["w"][:, 1] == 1
    lgw = r["cutoff"]["w"][:, 0]
    assert np.array_equal(kept, lgw > r["cutoff"]["ctf"])
    # the new CI space is the kept NR configurations, heaviest first
    nr_order = r["nr_order"]
    nkept = int(kept.sum())
    assert all(kept[k] for k in nr_order[:nkept]) and not any(kept[k] for k in nr_order[nkept:])
    assert np.all(np.diff(lgw[nr_order]) <= 0)
    assert r["nci"] == int(lay["nrn"][kept].sum())
    assert r["pt"]["dvnrx"] == pytest.approx(float(dVg.sum(axis=1).max()))


@pytest.mark.gpu
def test_select_configurations_from_device_sums():
    """The same selection fed by pci_gpu_pt2_groups on the PT block of the
    device: the new configuration order equals the one from the oracle's
    sums (no weight sits within 1e-9 of the threshold here)."""
    import oracle as O
    from pci_b200 import system as S
    from pci_b200.capi import Engine
    s = get_system("small3")
    lay = S.nr_layout(s.basis, s.configs, s.ndc)
    offs = lay["offsets"]
    ncnrci = len(lay["nrn"]) // 3
    nd1 = int(offs[ncnrci])
    (rp, col, val, *_), _ = oracle_h("small3")
    H = O.csr_to_dense(s.nd, rp, col, val)
    w, V = np.linalg.eigh(H[:nd1, :nd1])
    X = V[:, :3]
    nd0 = P.weight_ci(X, lay["ndcnr"][:ncnrci], lay["nrn"][:ncnrci], cut0=1e-3)["nd0"]
    want_eg, want_vg = O.pt2_groups(H, nd1, nd0, X[:nd0], w[:3], offs[ncnrci:], s.ndc)
    with Engine(0) as e:
        e.load_system(s)
        e.form_h_pt(nd1, nd0)
        _, eg, vg = e.pt2_groups(nd1, X[:nd0], w[:3], offs[ncnrci:])
    assert np.allclose(vg, want_vg, rtol=1e-9, atol=1e-15)
    want = P.select_configurations(lay, ncnrci, s.ndc, X, want_eg, want_vg, cut0=1e-3)
    got = P.select_configurations(lay, ncnrci, s.ndc, X, eg, vg, cut0=1e-3)
    lgw, ctf = want["cutoff"]["w"][:, 0], want["cutoff"]["ctf"]
    if np.min(np.abs(lgw - ctf)) < 1e-9:
        pytest.skip("a weight sits on the threshold")
    assert got["conf_order"] == want["conf_order"]
    assert (got["nci"], got["nc4"], got["kl4"]) == (want["nci"], want["nc4"], want["kl4"])


def test_save_vectors_signs_and_layout(tmp_path):
    """SaveVectors' CONF_PT.XIJ: CI part then first-order part, normalised,
    energies and J as read; the PT part follows PTE's own formula
    (ci = x / (e0 - ei), e0 = En, ei = -Diag(i), conf_pt.f90:865-874) with
    the CONF.XIJ energy En = -E, which is -1 times the engine's
    coefficient."""
    import oracle as O
    from pci_b200 import files
    s = get_system("small3")
    (rp, col, val, *_), _ = oracle_h("small3")
    H = O.csr_to_dense(s.nd, rp, col, val)
    cs = np.concatenate([[0], np.cumsum(s.ndc)])
    nd1 = int(cs[10])
    w, V = np.linalg.eigh(H[:nd1, :nd1])
    X_ci, E = V[:, :2], w[:2]
    dE, C = O.pt2(H, nd1, nd1, X_ci, E)
    En = -E                                                 # CONF.XIJ's energies
    ref = np.zeros((s.nd, 2))
    for i in range(nd1, s.nd):
        x = H[i, :nd1] @ X_ci
        ref[i] = x / (En - (-H[i, i]))                      # PTE's ci
    assert np.allclose(ref[nd1:], -C[nd1:], rtol=1e-12, atol=1e-15)
    X = P.save_vectors(tmp_path / "CONF_PT.XIJ", En, [0.5, 1.5], X_ci, C, nd1)
    Tk, Tj, Xr = files.read_xij(tmp_path / "CONF_PT.XIJ", s.nd)
    assert np.allclose(Tk, En) and np.allclose(Tj, [0.5, 1.5])
    assert np.allclose(Xr, X) and np.allclose(np.linalg.norm(Xr, axis=0), 1.0)
    norm = np.sqrt(1.0 + np.sum(ref[nd1:] ** 2, axis=0))
    assert np.allclose(Xr[:nd1] * norm, X_ci) and np.allclose(Xr[nd1:] * norm, ref[nd1:])
