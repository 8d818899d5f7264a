"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Bar: the non-zero pattern (row pointers and 1-based columns), numzero and Hmin
are identical; FP64 values are bit-identical (both sides evaluate Hmltn/Gint
in the reference's operation order without fused multiply-adds); FP32 storage
equals the FP64 oracle value rounded to float32.  Davidson eigenvalues agree
with the oracle's restatement of Diag4 to 1e-8 Ha (|delta E| <= 1e-8).
"""
import numpy as np
import pytest

import oracle as O
from conftest import get_system, oracle_h
from pci_b200 import system as S

pytestmark = pytest.mark.gpu

SYSTEMS = ["tiny", "small3", "small4", "cfg1"]


@pytest.fixture(scope="module")
def engine():
    from pci_b200.capi import Engine
    e = Engine(0)
    yield e
    e.close()


def _load(engine, s):
    engine.load_system(s)


@pytest.mark.parametrize("build", ["padded", "exact"])
@pytest.mark.parametrize("name", SYSTEMS)
def test_form_h_bit_exact(engine, name, build, monkeypatch):
    """Both FormH builds: single evaluation into padded rows + compaction,
    and the two-pass count/fill build."""
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), _ = oracle_h(name)
    _load(engine, s)
    monkeypatch.setenv("PCI_FORMH", build)
    numh, numzero, ghmin = engine.form_h(64)
    st = engine.stats()
    assert st["formh_single_eval"] == (1.0 if build == "padded" else 0.0)
    if build == "padded":
        # the configuration bound covers every candidate pair (values evaluated = NumH + zeros)
        assert st["formh_slots"] >= numh + numzero
    grp, gcol, gval = engine.get_csr(0)
    assert numh == rp[-1]
    assert numzero == nz
    assert ghmin == hmin
    assert np.array_equal(grp, rp)
    assert np.array_equal(gcol, col)
    assert np.array_equal(gval.view(np.int64), val.view(np.int64))   # bit-identical


@pytest.mark.parametrize("build", ["padded", "exact"])
@pytest.mark.parametrize("name", ["small3", "small4"])
def test_form_h_fp32_storage(engine, name, build, monkeypatch):
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), _ = oracle_h(name)
    _load(engine, s)
    monkeypatch.setenv("PCI_FORMH", build)
    numh, numzero, ghmin = engine.form_h(32)
    grp, gcol, gval = engine.get_csr(0)
    assert np.array_equal(grp, rp) and np.array_equal(gcol, col)
    assert np.array_equal(gval, val.astype(np.float32).astype(np.float64))
    assert ghmin == float(np.float32(hmin))


@pytest.mark.parametrize("name", SYSTEMS)
def test_form_j_bit_exact(engine, name):
    s = get_system(name)
    _, (jr, jc, jv) = oracle_h(name)
    _load(engine, s)
    numj = engine.form_j()
    grp, gcol, gval = engine.get_csr(1)
    assert numj == jr[-1]
    assert np.array_equal(grp, jr) and np.array_equal(gcol, jc)
    assert np.array_equal(gval, jv)


def test_breit_and_gj_paths(engine):
    """kbrt = 1 (two radial values per key, Breit phase is_br) and Gj /= 0
    (the J^2 penalty inside Hmltn) on a small system."""
    kw = S.CONFIGS["small3"]()
    kw.update(kbrt=1, gj=0.05)
    s = S.make_system(**kw)
    rp, col, val, nz, hmin, pairs = O.Oracle(s).form_h()
    _load(engine, s)
    numh, numzero, ghmin = engine.form_h(64)
    grp, gcol, gval = engine.get_csr(0)
    assert np.array_equal(grp, rp) and np.array_equal(gcol, col)
    assert np.array_equal(gval.view(np.int64), val.view(np.int64))
    assert numzero == nz and ghmin == hmin


def test_fp32_integrals(engine):
    """Rint2 as float32 (the reference's default type2_real)."""
    kw = S.CONFIGS["small4"]()
    kw.update(r2_dtype=np.float32)
    s = S.make_system(**kw)
    rp, col, val, nz, hmin, pairs = O.Oracle(s).form_h()
    _load(engine, s)
    engine.form_h(64)
    grp, gcol, gval = engine.get_csr(0)
    assert np.array_equal(grp, rp) and np.array_equal(gcol, col)
    assert np.array_equal(gval.view(np.int64), val.view(np.int64))


@pytest.mark.parametrize("name", ["tiny", "cfg1"])
def test_davidson_converged_levels(engine, name):
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    p = dict(s.params)
    ref = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    _load(engine, s)
    engine.form_h(64)
    engine.form_j()
    res = engine.davidson(s.nd, Nlv=p["Nlv"], N_it=p["N_it"], Crt4=p["Crt4"], MaxNd0=p["MaxNd0"],
                          admix_crit=p["admix_crit"])
    assert res["iterations"] == ref["iterations"]
    assert np.max(np.abs(res["Tk"] - ref["Tk"])) <= 1e-8
    assert np.allclose(res["Tj"], ref["Tj"], atol=1e-6)
    # eigenvectors agree up to sign
    ov = np.abs(np.sum(res["X"] * ref["X"], axis=0))
    assert np.all(ov > 1 - 1e-6)


def test_davidson_trajectory_small3(engine):
    """A slowly converging case: after the same number of iterations of the same
    algorithm both sides hold the same Ritz values."""
    name = "small3"
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    p = dict(s.params)
    p.update(N_it=25, admix_crit=0.0)
    ref = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    _load(engine, s)
    engine.form_h(64)
    engine.form_j()
    res = engine.davidson(s.nd, Nlv=p["Nlv"], N_it=25, Crt4=p["Crt4"], MaxNd0=p["MaxNd0"], admix_crit=0.0)
    assert res["iterations"] == ref["iterations"] == 25
    assert np.max(np.abs(res["Tk"] - ref["Tk"])) <= 1e-8
    assert np.allclose(res["resid"], ref["cnorm"], rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("name", ["tiny", "small3", "small4", "cfg1"])
def test_jterms_match_oracle(engine, name):
    """Jt computed in set_basis from the configurations' M distributions
    equals the oracle's enumeration of Dinit's term analysis."""
    s = get_system(name)
    _load(engine, s)
    assert engine.jterms() == O.j_terms(s.basis, s.configs, s.mj)


@pytest.mark.parametrize("name,xj,nlv,n_it", [("tiny", 0.0, 3, 200), ("small3", 1.5, 6, 20)])
def test_davidson_kv3(engine, name, xj, nlv, n_it):
    """Kv = 3 against the oracle: the same iterations of J-selected FormB0,
    AvgDiag and Prj_J give the same Ritz values (1e-8) and J = XJ_av."""
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    p = dict(s.params, Kv=3, XJ_av=xj, Nlv=nlv, N_it=n_it, admix_crit=0.0)
    ref = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc, jt=O.j_terms(s.basis, s.configs, s.mj))
    _load(engine, s)
    engine.form_h(64)
    engine.form_j()
    res = engine.davidson(s.nd, Nlv=nlv, N_it=n_it, Crt4=p["Crt4"], Kv=3, XJ_av=xj, MaxNd0=p["MaxNd0"],
                          admix_crit=0.0)
    n = ref["Tk"].size
    assert res["iterations"] == ref["iterations"]
    assert np.max(np.abs(res["Tk"][:n] - ref["Tk"])) <= 1e-8
    assert np.allclose(res["Tj"][:n], xj, atol=1e-6)
    assert np.all(res["Iconverge"][n:] == -1)


def test_davidson_kv3_zero_term_is_rejected(engine):
    from pci_b200.capi import PciError
    s = get_system("tiny")
    _load(engine, s)
    engine.form_h(64)
    engine.form_j()
    with pytest.raises(PciError) as ei:
        engine.davidson(s.nd, Nlv=3, Kv=3, XJ_av=1.0)
    assert ei.value.code == 1 and "divides by zero" in str(ei.value)


@pytest.mark.parametrize("name,spmm", [("tiny", "full"), ("cfg1", "full"), ("cfg1", "lower")])
def test_davidson_fp32_form(name, spmm, monkeypatch):
    """Precision form: H stored in FP32 and FP32 SpMM (FP32 accumulate), FP64
    elsewhere.  Its levels match the FP64 oracle's to FP32 accuracy: within
    2e-6 Ha per level (stated per level in the assertion message)."""
    from pci_b200.capi import Engine
    monkeypatch.setenv("PCI_SPMM", spmm)
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    p = dict(s.params)
    ref = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    with Engine(0) as e:
        e.load_system(s)
        e.form_h(32)
        e.form_j()
        res = e.davidson(s.nd, Nlv=p["Nlv"], N_it=p["N_it"], Crt4=1e-6, mode=1, MaxNd0=p["MaxNd0"],
                         admix_crit=0.0)
        assert e.stats()["spmm_calls"] > 0
    err = np.abs(res["Tk"] - ref["Tk"])
    assert np.all(err <= 2e-6), f"per-level |dE| vs FP64: {err}"
    assert np.allclose(res["Tj"], ref["Tj"], atol=1e-4)


def test_fp32_form_needs_fp32_h(engine):
    from pci_b200.capi import PciError
    s = get_system("tiny")
    _load(engine, s)
    engine.form_h(64)
    engine.form_j()
    with pytest.raises(PciError) as ei:
        engine.davidson(s.nd, Nlv=3, mode=1)
    assert ei.value.code == 1


@pytest.mark.parametrize("build", ["padded", "exact"])
@pytest.mark.parametrize("name", ["tiny", "cfg1", "small3"])
def test_form_h_matches_golden(engine, name, build, monkeypatch):
    """The CUDA FormH against the committed fixtures (independent of the
    oracle code): CSR SHA-256, NumH, numzero and Hmin; then the Davidson
    levels over the fixture's iterations."""
    import hashlib
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))
    s = get_system(name)
    _load(engine, s)
    monkeypatch.setenv("PCI_FORMH", build)
    numh, numzero, hmin = engine.form_h(64)
    rp, col, val = engine.get_csr(0)
    h = hashlib.sha256()
    for a, t in ((rp, np.int64), (col, np.int32), (val, np.float64)):
        h.update(np.ascontiguousarray(a, t).tobytes())
    assert (numh, numzero, hmin) == (int(g["numh"]), int(g["numzero"]), float(g["hmin"]))
    assert h.hexdigest() == str(g["h_sha"])
    assert engine.jterms() == g["jterms"].tolist()
    engine.form_j()
    p = dict(s.params)
    n_it = int(g["n_it"]) if int(g["n_it"]) > 0 else p["N_it"]
    crit = 0.0 if int(g["n_it"]) > 0 else p["admix_crit"]
    res = engine.davidson(s.nd, Nlv=p["Nlv"], N_it=n_it, Crt4=p["Crt4"], MaxNd0=p["MaxNd0"], admix_crit=crit)
    assert res["iterations"] == int(g["iterations"])
    assert np.max(np.abs(res["Tk"] - g["tk"])) <= 1e-8


@pytest.mark.parametrize("build", ["padded", "exact"])
@pytest.mark.parametrize("name", ["ne1", "ne5", "ne6", "ne8"])
def test_form_h_other_electron_counts(engine, name, build, monkeypatch):
    """The H-build units for Ne = 1, 5, 6 and 8 (one per electron count):
    pattern, values (bit for bit), numzero, Hmin and J^2 as the oracle."""
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    _load(engine, s)
    monkeypatch.setenv("PCI_FORMH", build)
    numh, numzero, ghmin = engine.form_h(64)
    grp, gcol, gval = engine.get_csr(0)
    assert numzero == nz and ghmin == hmin
    assert np.array_equal(grp, rp) and np.array_equal(gcol, col)
    assert np.array_equal(gval.view(np.int64), val.view(np.int64))
    engine.form_j()
    jrp, jcol, jval = engine.get_csr(1)
    assert np.array_equal(jrp, jr) and np.array_equal(jcol, jc) and np.array_equal(jval, jv)


@pytest.mark.parametrize("name", ["ne1", "ne5", "ne8"])
def test_davidson_other_electron_counts(engine, name):
    """Ten Davidson iterations (or convergence) give the oracle's levels."""
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    p = dict(s.params, N_it=10, admix_crit=0.0)
    ref = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    _load(engine, s)
    engine.form_h(64)
    engine.form_j()
    res = engine.davidson(s.nd, Nlv=p["Nlv"], N_it=10, Crt4=p["Crt4"], MaxNd0=p["MaxNd0"], admix_crit=0.0)
    assert res["iterations"] == ref["iterations"]
    assert np.max(np.abs(res["Tk"] - ref["Tk"])) <= 1e-8


def test_missing_integral_is_reported(engine):
    from pci_b200.capi import PciError
    kw = S.CONFIGS["tiny"]()
    s = S.make_system(**kw)
    # drop R^0(3s 3s; 3s 3s), which every 3s^2 diagonal element needs
    keep = ~((s.iint2 == 1) & (s.iint3 == 1))
    assert keep.sum() == s.ngint - 1
    s.rint2 = s.rint2[keep]
    s.iint2 = s.iint2[keep]
    s.iint3 = s.iint3[keep]
    _load(engine, s)
    with pytest.raises(PciError) as ei:
        engine.form_h(64)
    assert ei.value.code == 3


def test_bad_determinant_order_is_reported(engine):
    from pci_b200.capi import PciError
    s = get_system("tiny")
    bad = S.make_system(**S.CONFIGS["tiny"]())
    bad.iarr = bad.iarr.copy()
    bad.iarr[5] = bad.iarr[5][::-1]
    with pytest.raises(PciError) as ei:
        engine.set_basis(bad)
    assert ei.value.code == 1
    _load(engine, s)   # the handle stays usable
    engine.form_h(64)


@pytest.mark.parametrize("mode", ["lower", "lower-tiles", "lower-windows", "full", "set-csr"])
def test_davidson_spmm_paths(mode, monkeypatch):
    """The SpMM paths give the same Davidson levels: lower triangle with
    transpose reductions (default), along the configuration tiles and in
    column windows, the full symmetric copy, and an H round-tripped through
    get_csr/set_csr."""
    from pci_b200.capi import Engine
    monkeypatch.setenv("PCI_SPMM", "full" if mode == "full" else "lower")
    if mode in ("lower-tiles", "lower-windows"):
        monkeypatch.setenv("PCI_SPMM_LOWER", mode.split("-")[1])
    name = "small3"
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    p = dict(s.params)
    p.update(N_it=25, admix_crit=0.0)
    ref = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    with Engine(0) as e:
        e.load_system(s)
        numh, _, hm = e.form_h(64)
        e.form_j()
        if mode == "set-csr":
            rp2, col2, val2 = e.get_csr(0)
            e.set_csr(0, rp2, col2, val2, hm)
        res = e.davidson(s.nd, Nlv=p["Nlv"], N_it=25, Crt4=p["Crt4"], MaxNd0=p["MaxNd0"], admix_crit=0.0)
    assert np.max(np.abs(res["Tk"] - ref["Tk"])) <= 1e-8


@pytest.mark.parametrize("name", ["tiny", "small3"])
def test_j_av_matches_oracle(engine, name):
    """J_av over the resident J^2 against the oracle's restatement, full length and
    restricted to the first rows (the FormB0 use on the initial block)."""
    s = get_system(name)
    _, (jr, jc, jv) = oracle_h(name)
    _load(engine, s)
    engine.form_j()
    rng = np.random.default_rng(3)
    X = rng.standard_normal((s.nd, 5))
    X /= np.linalg.norm(X, axis=0)
    for nlim in (s.nd, s.nd // 3):
        got = engine.j_av(X, nlim)
        ref = np.array([O.j_av(jr, jc, jv, X[:, v], nlim) for v in range(5)])
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", ["small3", "cfg1"])
def test_hij_streamed_from_device(engine, name, tmp_path):
    """CONF.HIJ and CONF.JJJ (src/sort.f90:16-80) streamed from the resident
    matrices in row ranges (pci_gpu_get_csr_rows + pci_io_append_hij) are the
    same bytes as the stream written from the oracle's FormH / FormJ CSR."""
    from pci_b200 import files
    s = get_system(name)
    (rp, col, val, *_), (jr, jc, jv) = oracle_h(name)
    _load(engine, s)
    engine.form_h(64)
    engine.form_j()
    for which, (r, c, v) in ((0, (rp, col, val)), (1, (jr, jc, jv))):
        got, want = tmp_path / f"dev{which}.HIJ", tmp_path / f"orc{which}.HIJ"
        files.write_hij_from_engine(got, engine, which, rows_per_chunk=97)
        files.write_hij(want, np.asarray(r, np.int64), np.asarray(c, np.int32), np.asarray(v, np.float64))
        assert got.read_bytes() == want.read_bytes()


def test_form_h_with_core_shells_bit_exact(engine):
    """Closed core orbitals (Nso = 2, as every real CONF.INP has): the device
    keys the integrals from orbital Nso + 1 and numbers the core m-states
    first, as the oracle (checked against the second-quantised H) does."""
    shells = [(1, 0), (2, 0)] + S._shells({0: (3, 4), 1: (3, 4), 2: (3, 3)})
    s = S.make_system("core", shells, 3, 1, 1, [[3, 4, 5]], 5, level=2, params=dict(Nlv=3, MaxNd0=20), nso=2)
    o = O.Oracle(s)
    rp, col, val, nz, hmin, pairs = o.form_h()
    jr, jc, jv = o.form_j()
    _load(engine, s)
    numh, numzero, ghmin = engine.form_h(64)
    grp, gcol, gval = engine.get_csr(0)
    assert numh == rp[-1] and numzero == nz and ghmin == hmin
    assert np.array_equal(grp, rp) and np.array_equal(gcol, col)
    assert np.array_equal(gval.view(np.int64), val.view(np.int64))
    engine.form_j()
    gjr, gjc, gjv = engine.get_csr(1)
    assert np.array_equal(gjr, jr) and np.array_equal(gjc, jc) and np.array_equal(gjv, jv)
