"""pconf file formats through the C ABI of include/pci_io.h (no GPU).

Every writer is checked twice: by its own reader (round trip) and by an
independent parse of the bytes that follows the layouts of the reference's
writers -- WriteMatrixCSR (src/matrix_io.f90:689-799) for pCONF.HIJ, the
sort program's record stream (src/sort.f90:16-80, read by ReadHIJ,
src/pol.f90:766-797) for CONF.HIJ,
WriteFinalXIJ (src/pconf.F90:2566-2602) for CONF.XIJ, PrintEnergies
(src/pconf.F90:3152-3242) for CONF.RES, Wdet (src/determinants.f90:448-460)
for CONF.DET, the CONF.GNT records of src/breit.f90:96-101 and the CONF.INT
records Rint reads (src/integrals.f90:35-106).
"""
import os
import struct

import numpy as np
import pytest

from conftest import get_system
from pci_b200 import capi, files

H = os.path.join(os.path.dirname(__file__), "..", "include", "pci_io.h")


def _records(path):
    """Fortran unformatted sequential records (4-byte markers, no subrecords)."""
    out = []
    b = open(path, "rb").read()
    i = 0
    while i < len(b):
        (n,) = struct.unpack_from("<i", b, i)
        assert n >= 0
        rec = b[i + 4:i + 4 + n]
        (m,) = struct.unpack_from("<i", b, i + 4 + n)
        assert m == n
        out.append(rec)
        i += 8 + n
    return out


def _csr(seed, nd=57, dtype=np.float64):
    rng = np.random.default_rng(seed)
    cnt = rng.integers(0, 9, nd)
    rowptr = np.zeros(nd + 1, np.int64)
    rowptr[1:] = np.cumsum(cnt)
    col = np.concatenate([np.sort(rng.choice(np.arange(1, r + 2), size=min(c, r + 1), replace=False))
                          for r, c in enumerate(cnt)]).astype(np.int32) if cnt.sum() else np.zeros(0, np.int32)
    rowptr[1:] = np.cumsum([min(c, r + 1) for r, c in enumerate(cnt)])
    val = rng.standard_normal(col.size).astype(dtype)
    return rowptr, col, val


def test_exports_match_header():
    import re
    names = re.findall(r"\b(pci_io_\w+)\s*\(", open(H).read())
    assert sorted(set(names)) == sorted(files.EXPORTS)
    L = capi.load()
    for n in files.EXPORTS:
        assert hasattr(L, n)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_csr_stream(tmp_path, dtype):
    rowptr, col, val = _csr(3, dtype=dtype)
    p = tmp_path / "pCONF.HIJ"
    files.write_csr(p, rowptr, col, val)
    b = open(p, "rb").read()
    nd, nnz = struct.unpack_from("<qq", b, 0)
    assert (nd, nnz) == (rowptr.size - 1, col.size)
    o = 16
    assert np.array_equal(np.frombuffer(b, np.int64, nd + 1, o), rowptr)
    o += (nd + 1) * 8
    assert np.array_equal(np.frombuffer(b, np.int32, nnz, o), col)
    o += nnz * 4
    assert np.array_equal(np.frombuffer(b, dtype, nnz, o), val)
    assert len(b) == o + nnz * np.dtype(dtype).itemsize
    r2, c2, v2 = files.read_csr(p)
    assert np.array_equal(r2, rowptr) and np.array_equal(c2, col)
    assert v2.dtype == dtype and np.array_equal(v2, val)


def test_csr_stream_errors(tmp_path):
    rowptr, col, val = _csr(4)
    p = tmp_path / "bad.HIJ"
    bad = rowptr.copy()
    bad[-1] += 1
    with pytest.raises(capi.PciError):
        files.write_csr(p, bad, col, val)
    files.write_csr(p, rowptr, col, val)
    with open(p, "r+b") as f:            # a file whose length fits no value size
        f.truncate(os.path.getsize(p) - 3)
    with pytest.raises(capi.PciError):
        files.read_csr(p)


def _hij_parse(path):
    """The CONF.HIJ bytes as ReadHIJ reads them: int64 count, then (int32, int32, real64) records."""
    b = open(path, "rb").read()
    (n,) = struct.unpack_from("<q", b, 0)
    assert len(b) == 8 + 16 * n
    rec = np.frombuffer(b, np.dtype([("r", "<i4"), ("c", "<i4"), ("v", "<f8")]), n, 8)
    return n, rec


def test_hij_stream(tmp_path):
    """Whole-matrix and row-range writers give the same bytes: rows ascending,
    columns ascending within a row (the order sort.f90's quicksort leaves),
    exact zeros dropped, column <= row."""
    rowptr, col, val = _csr(5)
    val[::7] = 0.0
    p1, p2 = tmp_path / "CONF.HIJ", tmp_path / "CONF2.HIJ"
    files.write_hij(p1, rowptr, col, val)
    n, rec = _hij_parse(p1)
    rows = np.repeat(np.arange(1, rowptr.size), np.diff(rowptr))
    keep = val != 0.0
    assert n == keep.sum()
    assert np.array_equal(rec["r"], rows[keep]) and np.array_equal(rec["c"], col[keep])
    assert np.array_equal(rec["v"], val[keep])
    assert np.all(rec["c"] <= rec["r"])
    key = rec["r"].astype(np.int64) * (1 << 32) + rec["c"]
    assert np.all(np.diff(key) > 0)
    # the same stream in row ranges of 10
    nd = rowptr.size - 1
    L = files.lib()
    for r0 in range(0, nd, 10):
        r1 = min(nd, r0 + 10)
        rp = rowptr[r0:r1 + 1]
        files._call(L.pci_io_append_hij, files._path(p2), r0, r1 - r0, files._p(np.ascontiguousarray(rp)),
                    files._p(col[rp[0]:]), files._p(val[rp[0]:]))
    assert open(p1, "rb").read() == open(p2, "rb").read()
    r, c, v = files.read_hij(p1)
    assert np.array_equal(r, rec["r"]) and np.array_equal(c, rec["c"]) and np.array_equal(v, rec["v"])


def test_xij(tmp_path):
    rng = np.random.default_rng(5)
    nd, nlv = 101, 4
    X = rng.standard_normal((nd, nlv))
    Tk = -rng.random(nlv)
    Tj = np.array([0.5, 1.5, 0.5, 2.5])
    p = tmp_path / "CONF.XIJ"
    files.write_xij(p, Tk, Tj, X)
    recs = _records(p)
    assert len(recs) == nlv
    for n, r in enumerate(recs):
        assert len(r) == 8 + 8 + 4 + 8 * nd
        tk, tj, ndr = struct.unpack_from("<ddi", r, 0)
        assert (tk, tj, ndr) == (Tk[n], Tj[n], nd)
        assert np.array_equal(np.frombuffer(r, np.float64, nd, 20), X[:, n])
    tk2, tj2, x2 = files.read_xij(p, nd)
    assert np.array_equal(tk2, Tk) and np.array_equal(tj2, Tj) and np.array_equal(x2, X)
    with pytest.raises(capi.PciError):
        files.read_xij(p, nd + 1)


def test_res(tmp_path):
    Tj = np.array([0.5, 1.5, 2.5000001])
    Tk = np.array([-1.2345678901, -1.20, -0.9])
    p = tmp_path / "CONF.RES"
    files.write_res(p, kbrt=0, nc=1234, nd=56789, gj=0.0, Tj=Tj, Tk=Tk, ecore=-10.0)
    lines = open(p).read().splitlines()
    assert lines[0] == " " + "=" * 80 and lines[-1] == " " + "=" * 80
    assert lines[1] == "    Energy levels (COULOMB Nc=   1234 Nd=    56789); Gj = 0.0000"
    assert lines[2] == "    N" + " " * 6 + "JTOT" + " " * 12 + "EV" + " " * 16 + "ET" + " " * 9 + "DEL(CM**-1)"
    assert lines[3] == " " + "-" * 80
    dpry = 109737.315709
    for j in range(3):
        want = "   %3d%14.9f%14.8f%18.6f%15.2f" % (j + 1, Tj[j], Tk[j], Tk[j] + 10.0, (Tk[0] - Tk[j]) * 2 * dpry)
        assert lines[4 + j] == want
    assert lines[4] == "     1   0.500000000   -1.23456789          8.765432           0.00"
    # Gj shifts EV by 4 Gj J(J+1); append adds a second table
    files.write_res(p, kbrt=2, nc=1, nd=2, gj=0.1, Tj=Tj[:1], Tk=Tk[:1], append=True)
    more = open(p).read().splitlines()[len(lines):]
    assert more[1].startswith("    Energy levels (BREIT   Nc=") and more[1].endswith("Gj = 0.1000")
    assert more[4] == "   %3d%14.9f%14.8f%18.6f%15.2f" % (1, 0.5, Tk[0] + 0.4 * 0.75, Tk[0] + 0.4 * 0.75, 0.0)


def test_det(tmp_path):
    s = get_system("tiny")
    p = tmp_path / "CONF.DET"
    files.write_det(p, s.iarr, s.nsu)
    recs = _records(p)
    assert struct.unpack("<ii", recs[0]) == (s.nd, s.nsu)
    assert len(recs) == s.nd + 1
    assert all(np.array_equal(np.frombuffer(r, np.int32), s.iarr[i]) for i, r in enumerate(recs[1:]))
    iarr, nsu = files.read_det(p)
    assert nsu == s.nsu and np.array_equal(iarr, s.iarr)
    with open(p, "r+b") as f:
        f.truncate(os.path.getsize(p) - 10)
    with pytest.raises(capi.PciError, match="premature end"):
        files.read_det(p)


def test_gnt(tmp_path):
    s = get_system("tiny")
    p = tmp_path / "CONF.GNT"
    files.write_gnt(p, s.nlx, s.gaunt_per_wave, s.gaunt_in, s.gaunt_gnt)
    recs = _records(p)
    assert struct.unpack("<ii", recs[0]) == (s.nlx, s.gaunt_in.size)
    assert np.array_equal(np.frombuffer(recs[1], np.int32), s.gaunt_per_wave)
    assert np.array_equal(np.frombuffer(recs[2], np.int32), s.gaunt_in)
    assert np.array_equal(np.frombuffer(recs[3], np.float64), s.gaunt_gnt)
    nlx, per, In, Gnt = files.read_gnt(p)
    assert nlx == s.nlx and np.array_equal(In, s.gaunt_in) and np.array_equal(Gnt, s.gaunt_gnt)
    lut = files.gaunt_lut(In, Gnt)
    assert np.array_equal(lut, s.gaunt_lut)
    # an older file without Nlx and the per-wave counts: Nlx defaults to 5
    q = tmp_path / "old.GNT"
    with open(q, "wb") as f:
        for payload in (struct.pack("<i", In.size), In.tobytes(), Gnt.tobytes()):
            f.write(struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload)))
    nlx, per, In2, Gnt2 = files.read_gnt(q)
    assert nlx == 5 and np.array_equal(In2, In) and np.array_equal(Gnt2, Gnt)


@pytest.mark.parametrize("r2", ["f64", "f32", "breit"])
def test_int(tmp_path, r2):
    s = get_system("tiny")
    nz = np.nonzero(s.hint_lut)[0]
    iint1 = (nz + 1).astype(np.int32)
    rint1 = s.hint_lut[nz]
    rint2 = s.rint2.astype(np.float32) if r2 == "f32" else s.rint2
    kbrt = 0
    if r2 == "breit":
        kbrt = 1
        rint2 = np.stack([s.rint2, 0.01 * s.rint2], axis=1)
    b = s.basis
    orb = np.stack([b.nn[:s.nsu], b.kk[:s.nsu], b.ll[:s.nsu], b.jj[:s.nsu]], axis=1)
    p = tmp_path / "CONF.INT"
    files.write_int(p, ns=s.nsu, nso=0, nsp=7, ecore=-3.25, orbitals=orb, rint1=rint1, iint1=iint1,
                    rint2=rint2, iint2=s.iint2, iint3=s.iint3, kbrt=kbrt, nlist=11, nx=s.nx)
    recs = _records(p)
    assert len(recs) == 11
    assert struct.unpack("<iiiid", recs[0]) == (s.nsu, 0, 7, s.nsu, -3.25)
    assert struct.unpack("<ii", recs[3]) == (rint1.size, kbrt)
    assert struct.unpack("<qii", recs[6]) == (s.ngint, 11, s.nx * s.nx)
    assert len(recs[7]) == rint2.nbytes
    c = files.read_int(p)
    assert c.header.r2_bytes == rint2.itemsize and c.header.ecore == -3.25
    assert np.array_equal(c.orbitals, orb) and np.array_equal(c.rint2, rint2)
    assert np.array_equal(c.iint2, s.iint2) and np.array_equal(c.iint3, s.iint3)
    assert np.array_equal(files.hint_lut(c.rint1, c.iint1, s.nx), s.hint_lut)
