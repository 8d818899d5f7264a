"""CONF.INP (src/conf_init.f90:37-135, 215-312; shell codes decoded as in
src/pconf.F90:506-529) read and written by pci_b200/conf_inp.py, and
conf_pt's CONF_new.INP (src/conf_pt.f90:1130-1264)."""
import numpy as np
import pytest

from conftest import get_system, oracle_h

from pci_b200 import conf_inp as C
from pci_b200 import conf_pt as P
from pci_b200 import system as S

SAMPLE = """ Cs test
Z = 55.0
Am = 132.9
J = 0.5
Jm = 0.5
Nso = 2
Nc = 3
Kv = 4
Nlv = 5
Ne = 3   # three valence electrons
Kl4 = 1
Nc4 = 2
Crt4 = 1.d-4
Cut0 = 2.5D-3

    -0.1001     0.2102
   1 0.2102    -0.2101
   2 0.2101
     0.3001     0.3101
   3
     0.3002    -0.3101
"""


def test_shell_codes():
    assert C.decode_qnl(0.2102) == (2, 1, 3, -2, 2)          # 2p3/2, two electrons
    assert C.decode_qnl(-0.2101) == (2, 1, 1, 1, 1)          # 2p1/2, one electron
    assert C.decode_qnl(-0.1001) == (1, 0, -1, 0, 1)         # as pconf decodes a minus on an s shell
    assert C.decode_qnl(0.4012) == (4, 0, 1, -1, 12)
    for n, l, j2, q in [(2, 1, 3, 2), (3, 2, 3, 4), (5, 0, 1, 1), (4, 3, 7, 8)]:
        assert C.decode_qnl(C.encode_qnl(n, l, j2, q))[:3] == (n, l, j2)
        assert C.decode_qnl(C.encode_qnl(n, l, j2, q))[4] == q
    with pytest.raises(ValueError):
        C.encode_qnl(2, 1, 5, 1)


def test_read_sample():
    r = C.read_conf_inp(SAMPLE)
    assert r["name"].strip() == "Cs test"
    p = r["params"]
    assert (p["Z"], p["NSO"], p["NC"], p["NE"], p["KL4"], p["NC4"]) == (55.0, 2, 3, 3, 1, 2)
    assert p["CRT4"] == pytest.approx(1e-4) and p["KBRT"] == 0 and p["CUT0"] == pytest.approx(2.5e-3)
    assert r["core"] == [pytest.approx(-0.1001), pytest.approx(0.2102)]
    # configuration 2 runs over two lines until it holds Ne = 3 electrons;
    # configuration 3's first line is blank apart from its number
    got = [[round(x, 4) for x in c] for c in r["configs"]]
    assert got == [[0.2102, -0.2101], [0.2101, 0.3001, 0.3101], [0.3002, -0.3101]]


def test_write_read_round_trip_of_a_system():
    s = get_system("small3")
    codes = C.configs_to_qnl(s.basis, s.configs)
    params = {"Z": 55.0, "AM": 133.0, "J": 0.5, "JM": s.mj / 2, "NSO": 0, "NC": len(codes), "KV": 4,
              "NLV": 6, "NE": s.ne}
    r = C.read_conf_inp(C.write_conf_inp("small3", params, [], codes))
    assert r["params"]["NC"] == s.nc and r["params"]["NE"] == s.ne
    assert C.configs_from_qnl(s.basis, r["configs"]) == [[(int(a), int(b)) for a, b in c] for c in s.configs]


def test_new_conf_inp_reads_back_as_the_new_ci_space():
    import oracle as O
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
    dEg, dVg = O.pt2_groups(H, nd1, nd0, X[:nd0], w[:3], offs[ncnrci:], s.ndc)
    sel = P.select_configurations(lay, ncnrci, s.ndc, X, dEg, dVg, cut0=1e-3, nc4=40)
    codes = C.configs_to_qnl(s.basis, s.configs)
    params = {"Z": 55.0, "AM": 133.0, "J": 0.5, "JM": s.mj / 2, "NSO": 0, "NC": s.nc, "KV": 4, "NLV": 6,
              "NE": s.ne, "KL4": 1, "NC4": 40}
    parsed = C.read_conf_inp(C.write_conf_inp("small3", params, [], codes))
    text = C.new_conf_inp(parsed, sel, lay)
    assert "<CI<" in text and "(reordered)" in text.splitlines()[0]
    back = C.read_conf_inp(text)
    assert back["name"].strip() == "small3"
    assert back["params"]["NC"] == sel["nci"]
    assert (back["params"]["KL4"], back["params"]["NC4"]) == (sel["kl4"], sel["nc4"])
    want = [[(int(a), int(b)) for a, b in s.configs[ic]] for ic in sel["conf_order"][:sel["nci"]]]
    assert C.configs_from_qnl(s.basis, back["configs"]) == want
    # the whole list, read with Nc = all configurations, is every configuration in the new order
    full = C.read_conf_inp(text.replace(f"NC = {sel['nci']}", f"NC = {s.nc}"))
    assert len(full["configs"]) == s.nc
    assert C.configs_from_qnl(s.basis, full["configs"]) == [[(int(a), int(b)) for a, b in s.configs[ic]]
                                                           for ic in sel["conf_order"]]


def test_reference_documented_sample():
    """The head of the CONF.INP that the reference's pconf documentation
    shows (Ir17+, even parity; tests/golden/conf_inp_doc_head.txt, made by
    make_conf_inp_fixture.py): header keys with comments, 14 core shells over
    three lines, and eight configurations, each preceded by lines carrying
    only a number (the reader takes them as empty).  Core and valence
    electrons add up to Ir17+'s 60."""
    import pathlib
    text = (pathlib.Path(__file__).parent / "golden" / "conf_inp_doc_head.txt").read_text()
    text = text.replace("Nc = 481", "Nc =   8")          # the documentation shows the first 8
    r = C.read_conf_inp(text)
    assert r["name"].strip() == "Ir17+_even"
    p = r["params"]
    assert (p["Z"], p["AM"], p["J"], p["JM"]) == (77.0, 193.0, 2.0, 2.0)
    assert (p["NSO"], p["NC"], p["KV"], p["NLV"], p["NE"], p["KL4"], p["NC4"]) == (14, 8, 4, 5, 14, 1, 28)
    assert (p["KOUT"], p["NCPT"], p["N_IT"], p["KBRT"], p["K_IS"]) == (0, 1132, 100, 1, 0)
    assert p["CRT4"] == pytest.approx(1e-4) and p["CUT0"] == pytest.approx(1e-4)
    assert p["GNUC"] == pytest.approx(1.07) and p["C_IS"] == 0.0
    core = [C.decode_qnl(x) for x in r["core"]]
    assert len(core) == 14
    assert [(n, l, j2) for n, l, j2, _, _ in core[:4]] == [(1, 0, 1), (2, 0, 1), (2, 1, 1), (2, 1, 3)]
    assert sum(q for *_, q in core) == 46
    assert len(r["configs"]) == 8
    for conf in r["configs"]:
        assert sum(C.decode_qnl(x)[4] for x in conf) == p["NE"]
    assert sum(q for *_, q in core) + p["NE"] == 77 - 17
    # configuration 1 is 4f5/2^6 4f7/2^8; configuration 5 has a 5p1/2 electron
    assert [C.decode_qnl(x)[:3] + (C.decode_qnl(x)[4],) for x in r["configs"][0]] == [(4, 3, 5, 6), (4, 3, 7, 8)]
    assert C.decode_qnl(r["configs"][4][2])[:3] == (5, 1, 1)
    # written back in this module's layout and read again: the same shells
    again = C.read_conf_inp(C.write_conf_inp(r["name"], p, r["core"], r["configs"]))
    assert again["configs"] == [[pytest.approx(x) for x in c] for c in r["configs"]]
    assert again["core"] == [pytest.approx(x) for x in r["core"]]


def test_reference_pylib_written_configurations():
    """Configuration lines that the reference's own py-lib (orbitals.py, as
    create_conf_inp.py uses it) wrote for six non-relativistic
    configurations (tests/golden/conf_inp_pylib.txt, made by
    make_conf_inp_pylib_fixture.py): the reader finds the 30 relativistic
    configurations, each shell decodes to what py-lib's own decoder says
    (n = 10 included), and NR_Init's grouping of them (squeeze of adjacent
    shells of one n, l) gives py-lib's expansion groups back."""
    import json
    import pathlib
    g = pathlib.Path(__file__).parent / "golden"
    r = C.read_conf_inp((g / "conf_inp_pylib.txt").read_text())
    want = json.loads((g / "conf_inp_pylib.json").read_text())
    assert len(r["configs"]) == len(want["configs"]) == r["params"]["NC"] == 30
    lname = "spdfghikl"
    for conf, exp in zip(r["configs"], want["configs"]):
        got = []
        for x in conf:
            n, l, j2, kappa, q = C.decode_qnl(x)
            got.append([f"{n}{lname[l]}", f"{j2}/2", q])
        assert got == exp
        assert sum(q for *_, q in exp) == r["params"]["NE"]
    basis = S.make_basis([(4, 3), (5, 2), (6, 0), (6, 1), (10, 0)])
    configs = C.configs_from_qnl(basis, r["configs"])
    lay = S.nr_layout(basis, configs, [1] * len(configs))
    assert lay["nrn"].tolist() == want["group_sizes"]
    # and this module writes the same shell codes back
    again = C.read_conf_inp(C.write_conf_inp("again", r["params"], [], C.configs_to_qnl(basis, configs)))
    assert again["configs"] == [[pytest.approx(x) for x in c] for c in r["configs"]]


def _write_inputs(tmp_path, s, core_codes=(), nso=0):
    """CONF.INP, CONF.INT and CONF.GNT of a system, as the reference's
    programs would leave them."""
    from pci_b200 import files
    b = s.basis
    nz = np.nonzero(s.hint_lut)[0]
    orb = np.stack([b.nn[:s.nsu], b.kk[:s.nsu], b.ll[:s.nsu], b.jj[:s.nsu]], axis=1)
    files.write_int(tmp_path / "CONF.INT", ns=s.nsu, nso=nso, nsp=len(core_codes) + 3, ecore=-7.5, orbitals=orb,
                    rint1=s.hint_lut[nz], iint1=(nz + 1).astype(np.int32), rint2=s.rint2, iint2=s.iint2,
                    iint3=s.iint3, kbrt=s.kbrt, nlist=4, nx=s.nx)
    files.write_gnt(tmp_path / "CONF.GNT", s.nlx, s.gaunt_per_wave, s.gaunt_in, s.gaunt_gnt)
    params = {"Z": 20.0, "AM": 40.0, "J": 0.5, "JM": s.mj / 2, "NSO": nso, "NC": s.nc, "KV": 4, "NLV": 6,
              "NE": s.ne, "KL4": 1, "NC4": 5, "CRT4": 1e-6, "N_IT": 50, "GJ": 0.0}
    text = C.write_conf_inp("from files", params, list(core_codes), C.configs_to_qnl(b, s.configs))
    (tmp_path / "CONF.INP").write_text(text)


@pytest.mark.parametrize("name", ["tiny", "small3"])
def test_system_from_reference_files(tmp_path, name):
    """A system written out as the reference's inputs (CONF.INP, CONF.INT,
    CONF.GNT) and read back through system_from_files is the same system:
    determinants, m-states, integrals and Gaunt factors equal."""
    s = get_system(name)
    _write_inputs(tmp_path, s)
    r = C.system_from_files(tmp_path / "CONF.INP", tmp_path / "CONF.INT", tmp_path / "CONF.GNT")
    assert (r.ne, r.mj, r.nsu, r.nx, r.kbrt) == (s.ne, s.mj, s.nsu, s.nx, s.kbrt)
    assert np.array_equal(r.iarr, s.iarr) and np.array_equal(r.ndc, s.ndc)
    assert np.array_equal(r.jz, s.jz) and np.array_equal(r.nh, s.nh)
    assert np.array_equal(r.hint_lut, s.hint_lut) and np.array_equal(r.rint2, s.rint2)
    assert np.array_equal(r.iint2, s.iint2) and np.array_equal(r.iint3, s.iint3)
    assert np.array_equal(r.gaunt_lut, s.gaunt_lut)
    assert r.ecore == -7.5 and r.params["Nc4"] == 5 and r.params["N_it"] == 50
    # without CONF.GNT the exact 3j table stands in
    r2 = C.system_from_files(tmp_path / "CONF.INP", tmp_path / "CONF.INT")
    assert np.allclose(r2.gaunt_lut, s.gaunt_lut, rtol=0, atol=1e-15)


def test_system_from_files_checks_nso(tmp_path):
    s = get_system("tiny")
    _write_inputs(tmp_path, s)
    text = (tmp_path / "CONF.INP").read_text().replace("NSO = 0", "NSO = 1\n     0.1002", 1)
    (tmp_path / "CONF.INP").write_text(text)
    with pytest.raises(ValueError):
        C.system_from_files(tmp_path / "CONF.INP", tmp_path / "CONF.INT")


def test_system_from_files_refuses_isotope_shift(tmp_path):
    """K_is with a non-negligible C_is would add the reference's SMS / VS
    terms to H, which this engine does not: refused, not silently dropped;
    |C_is| < 1e-6 switches the operator off, as pconf does."""
    s = get_system("tiny")
    _write_inputs(tmp_path, s)
    base = (tmp_path / "CONF.INP").read_text()
    (tmp_path / "CONF.INP").write_text(base.replace("GJ = 0", "GJ = 0\nK_IS = 2\nC_IS = 1.0", 1))
    with pytest.raises(ValueError):
        C.system_from_files(tmp_path / "CONF.INP", tmp_path / "CONF.INT")
    (tmp_path / "CONF.INP").write_text(base.replace("GJ = 0", "GJ = 0\nK_IS = 2\nC_IS = 0.0", 1))
    assert C.system_from_files(tmp_path / "CONF.INP", tmp_path / "CONF.INT").nd == s.nd


def test_system_from_files_checks_kbrt(tmp_path):
    """As the reference's Rint: CONF.INP's Kbrt must be the one CONF.INT's
    integrals were made for."""
    s = get_system("tiny")
    _write_inputs(tmp_path, s)
    base = (tmp_path / "CONF.INP").read_text()
    (tmp_path / "CONF.INP").write_text(base.replace("GJ = 0", "GJ = 0\nKBRT = 1", 1))
    with pytest.raises(ValueError):
        C.system_from_files(tmp_path / "CONF.INP", tmp_path / "CONF.INT")
