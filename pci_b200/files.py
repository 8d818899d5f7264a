"""ctypes binding of include/pci_io.h: pconf's file formats.

pCONF.HIJ / pCONF.JJJ (CSR stream), CONF.XIJ (eigenvectors), CONF.RES
(energy table), CONF.DET (determinant list), CONF.GNT (Gaunt factors) and
CONF.INT (radial integrals), read and written by the C++ code in
libpci_gpu.so.  Nothing here needs a GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import capi

_ERRLEN = 512


class IntHeader(C.Structure):
    """pci_int_header of include/pci_io.h (the leading CONF.INT records)."""
    _fields_ = [("ns", C.c_int32), ("nso", C.c_int32), ("nsp", C.c_int32), ("nsx", C.c_int32),
                ("ecore", C.c_double), ("nhint", C.c_int32), ("kbrt", C.c_int32), ("ngint", C.c_int64),
                ("nlist", C.c_int32), ("nrd", C.c_int32), ("r2_bytes", C.c_int32)]


_L = None


def lib():
    global _L
    if _L is not None:
        return _L
    L = capi.load()
    P, i32, i64, f64, s = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_char_p
    sig = {
        "pci_io_write_csr": [s, i64, i64, P, P, P, i32, P, i32],
        "pci_io_read_csr_header": [s, P, P, P, P, i32],
        "pci_io_read_csr": [s, i64, i64, P, P, P, i32, P, i32],
        "pci_io_write_xij": [s, i32, i64, P, P, P, P, i32],
        "pci_io_read_xij": [s, i32, i64, P, P, P, P, P, i32],
        "pci_io_write_res": [s, i32, i32, i32, i64, f64, i32, P, P, f64, P, i32],
        "pci_io_write_det": [s, i32, i64, i32, P, P, i32],
        "pci_io_read_det_header": [s, P, P, P, P, i32],
        "pci_io_read_det": [s, i32, i64, P, P, i32],
        "pci_io_write_gnt": [s, i32, i32, P, P, P, P, i32],
        "pci_io_read_gnt_header": [s, P, P, P, i32],
        "pci_io_read_gnt": [s, i32, i32, P, P, P, P, i32],
        "pci_io_gaunt_lut": [i32, P, P, P, P],
        "pci_io_read_int_header": [s, C.POINTER(IntHeader), P, i32],
        "pci_io_read_int": [s, C.POINTER(IntHeader), P, P, P, P, P, P, P, P, i32],
        "pci_io_write_int": [s, C.POINTER(IntHeader), P, P, P, P, P, P, P, P, i32],
        "pci_io_hint_lut": [i32, P, P, i32, P],
        "pci_io_write_hij": [s, i64, P, P, P, P, i32],
        "pci_io_append_hij": [s, i64, i64, P, P, P, P, i32],
        "pci_io_read_hij": [s, i64, P, P, P, P, P, i32],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    _L = L
    return L


EXPORTS = ["pci_io_write_csr", "pci_io_read_csr_header", "pci_io_read_csr", "pci_io_write_xij",
           "pci_io_read_xij", "pci_io_write_res", "pci_io_write_det", "pci_io_read_det_header",
           "pci_io_read_det", "pci_io_write_gnt", "pci_io_read_gnt_header", "pci_io_read_gnt",
           "pci_io_gaunt_lut", "pci_io_read_int_header", "pci_io_read_int", "pci_io_write_int",
           "pci_io_hint_lut", "pci_io_write_hij", "pci_io_append_hij", "pci_io_read_hij"]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _call(fn, *args):
    err = C.create_string_buffer(_ERRLEN)
    rc = fn(*args, err, _ERRLEN)
    if rc != 0:
        raise capi.PciError(rc, err.value.decode(errors="replace"))


def _path(p):
    return os.fsencode(p)


def _i64(v=0):
    return C.c_int64(v)


# ------------------------------------------------------------------ CSR ---

def write_csr(path, rowptr, col, val):
    """pCONF.HIJ / pCONF.JJJ: rowptr int64 (Nd+1, 0-based), col int32
    (1-based), val float64 or float32."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val)
    if val.dtype not in (np.float64, np.float32):
        raise ValueError("val must be float64 or float32")
    _call(lib().pci_io_write_csr, _path(path), rowptr.size - 1, col.size, _p(rowptr), _p(col), _p(val),
          val.itemsize)


def read_csr(path):
    L = lib()
    nd, nnz, vb = C.c_int64(), C.c_int64(), C.c_int32()
    _call(L.pci_io_read_csr_header, _path(path), C.byref(nd), C.byref(nnz), C.byref(vb))
    rowptr = np.empty(nd.value + 1, np.int64)
    col = np.empty(nnz.value, np.int32)
    val = np.empty(nnz.value, np.float64 if vb.value == 8 else np.float32)
    _call(L.pci_io_read_csr, _path(path), nd.value, nnz.value, _p(rowptr), _p(col), _p(val), vb.value)
    return rowptr, col, val


# ------------------------------------------------------- CONF.HIJ / JJJ ---

def write_hij(path, rowptr, col, val):
    """CONF.HIJ / CONF.JJJ record stream from a lower-triangle CSR (0-based
    rowptr, 1-based col, float64 val)."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    _call(lib().pci_io_write_hij, _path(path), rowptr.size - 1, _p(rowptr), _p(col), _p(val))


def write_hij_from_engine(path, eng, which=0, rows_per_chunk=1 << 16):
    """CONF.HIJ (which 0) or CONF.JJJ (which 1) streamed from a device-resident
    matrix in row ranges, so the host never holds the whole matrix."""
    nd = eng.csr_info(which)[0]
    L = lib()
    for r0 in range(0, nd, rows_per_chunk):
        r1 = min(nd, r0 + rows_per_chunk)
        rp, col, val = eng.get_csr_rows(which, r0 + 1, r1)
        _call(L.pci_io_append_hij, _path(path), r0, r1 - r0, _p(rp), _p(col), _p(val))
    if nd == 0:
        write_hij(path, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))


def read_hij(path):
    """(row int32, col int32, val float64) records of a CONF.HIJ stream."""
    L = lib()
    n = C.c_int64()
    _call(L.pci_io_read_hij, _path(path), 0, None, None, None, C.byref(n))
    row = np.empty(n.value, np.int32)
    col = np.empty(n.value, np.int32)
    val = np.empty(n.value, np.float64)
    _call(L.pci_io_read_hij, _path(path), n.value, _p(row), _p(col), _p(val), C.byref(n))
    return row, col, val


# ------------------------------------------------------------------ XIJ ---

def write_xij(path, Tk, Tj, X):
    """CONF.XIJ: X is Nd x nlv (one column per level)."""
    X = np.asfortranarray(X, dtype=np.float64)
    Tk = np.ascontiguousarray(Tk, dtype=np.float64)
    Tj = np.ascontiguousarray(Tj, dtype=np.float64)
    _call(lib().pci_io_write_xij, _path(path), X.shape[1], X.shape[0], _p(Tk), _p(Tj), _p(X))


def read_xij(path, nd, nlv_max=64):
    Tk = np.empty(nlv_max)
    Tj = np.empty(nlv_max)
    X = np.empty((nd, nlv_max), order="F")
    n = C.c_int32()
    _call(lib().pci_io_read_xij, _path(path), nlv_max, nd, _p(Tk), _p(Tj), _p(X), C.byref(n))
    k = n.value
    return Tk[:k].copy(), Tj[:k].copy(), np.asfortranarray(X[:, :k])


# ------------------------------------------------------------------ RES ---

def write_res(path, *, kbrt, nc, nd, gj, Tj, Tk, ecore=0.0, append=False):
    Tj = np.ascontiguousarray(Tj, dtype=np.float64)
    Tk = np.ascontiguousarray(Tk, dtype=np.float64)
    _call(lib().pci_io_write_res, _path(path), int(append), kbrt, nc, nd, gj, Tj.size, _p(Tj), _p(Tk), ecore)


# ------------------------------------------------------------------ DET ---

def write_det(path, iarr, nsu):
    """CONF.DET from Iarr as [Nd, Ne] (row per determinant, 1-based)."""
    iarr = np.ascontiguousarray(iarr, dtype=np.int32)   # row-major [Nd, Ne] == column-major Ne x Nd
    _call(lib().pci_io_write_det, _path(path), iarr.shape[1], iarr.shape[0], nsu, _p(iarr))


def read_det(path):
    L = lib()
    nd, nsu, ne = C.c_int64(), C.c_int32(), C.c_int32()
    _call(L.pci_io_read_det_header, _path(path), C.byref(nd), C.byref(nsu), C.byref(ne))
    iarr = np.empty((nd.value, ne.value), np.int32)
    _call(L.pci_io_read_det, _path(path), ne.value, nd.value, _p(iarr))
    return iarr, nsu.value


# ------------------------------------------------------------------ GNT ---

def write_gnt(path, nlx, per_wave, In, Gnt):
    per_wave = np.ascontiguousarray(per_wave, dtype=np.int32)
    In = np.ascontiguousarray(In, dtype=np.int32)
    Gnt = np.ascontiguousarray(Gnt, dtype=np.float64)
    _call(lib().pci_io_write_gnt, _path(path), nlx, In.size, _p(per_wave), _p(In), _p(Gnt))


def read_gnt(path):
    L = lib()
    nlx, ng = C.c_int32(), C.c_int32()
    _call(L.pci_io_read_gnt_header, _path(path), C.byref(nlx), C.byref(ng))
    per_wave = np.zeros(nlx.value + 1, np.int32)
    In = np.empty(ng.value, np.int32)
    Gnt = np.empty(ng.value, np.float64)
    _call(L.pci_io_read_gnt, _path(path), nlx.value, ng.value, _p(per_wave), _p(In), _p(Gnt))
    return nlx.value, per_wave, In, Gnt


def gaunt_lut(In, Gnt):
    In = np.ascontiguousarray(In, dtype=np.int32)
    Gnt = np.ascontiguousarray(Gnt, dtype=np.float64)
    n = C.c_int64()
    L = lib()
    if L.pci_io_gaunt_lut(In.size, _p(In), _p(Gnt), None, C.byref(n)) != 0:
        raise capi.PciError(1, "gaunt_lut: negative index")
    lut = np.empty(n.value)
    L.pci_io_gaunt_lut(In.size, _p(In), _p(Gnt), _p(lut), None)
    return lut


# ------------------------------------------------------------------ INT ---

@dataclass
class ConfInt:
    header: IntHeader
    orbitals: np.ndarray   # [Nsx, 4] Nn, Kk, Ll, Jj
    rint1: np.ndarray
    iint1: np.ndarray
    rint2: np.ndarray      # [Ngint] or [Ngint, 2]
    iint2: np.ndarray
    iint3: np.ndarray
    intord: np.ndarray


def read_int(path) -> ConfInt:
    L = lib()
    h = IntHeader()
    _call(L.pci_io_read_int_header, _path(path), C.byref(h))
    orb = np.empty((h.nsx, 4), np.int32)
    r1 = np.empty(h.nhint)
    i1 = np.empty(h.nhint, np.int32)
    shape = (h.ngint, 2) if h.kbrt else (h.ngint,)
    r2 = np.empty(shape, np.float64 if h.r2_bytes == 8 else np.float32)
    i2 = np.empty(h.ngint, np.int32)
    i3 = np.empty(h.ngint, np.int32)
    io = np.empty(h.nrd, np.int64)
    _call(L.pci_io_read_int, _path(path), C.byref(h), _p(orb), _p(r1), _p(i1), _p(r2), _p(i2), _p(i3), _p(io))
    return ConfInt(h, orb, r1, i1, r2, i2, i3, io)


def write_int(path, *, ns, nso, nsp, ecore, orbitals, rint1, iint1, rint2, iint2, iint3, kbrt, nlist, nx,
              intord=None):
    orbitals = np.ascontiguousarray(orbitals, dtype=np.int32)
    rint1 = np.ascontiguousarray(rint1, dtype=np.float64)
    iint1 = np.ascontiguousarray(iint1, dtype=np.int32)
    rint2 = np.ascontiguousarray(rint2)
    iint2 = np.ascontiguousarray(iint2, dtype=np.int32)
    iint3 = np.ascontiguousarray(iint3, dtype=np.int32)
    nrd = nx * nx
    intord = np.zeros(nrd, np.int64) if intord is None else np.ascontiguousarray(intord, dtype=np.int64)
    h = IntHeader(ns=ns, nso=nso, nsp=nsp, nsx=orbitals.shape[0], ecore=ecore, nhint=rint1.size, kbrt=kbrt,
                  ngint=iint2.size, nlist=nlist, nrd=nrd, r2_bytes=rint2.itemsize)
    _call(lib().pci_io_write_int, _path(path), C.byref(h), _p(orbitals), _p(rint1), _p(iint1), _p(rint2),
          _p(iint2), _p(iint3), _p(intord))


def hint_lut(rint1, iint1, nx):
    rint1 = np.ascontiguousarray(rint1, dtype=np.float64)
    iint1 = np.ascontiguousarray(iint1, dtype=np.int32)
    lut = np.empty(nx * nx)
    if lib().pci_io_hint_lut(rint1.size, _p(rint1), _p(iint1), nx, _p(lut)) != 0:
        raise capi.PciError(1, "hint_lut: index outside 1..Nx^2")
    return lut
