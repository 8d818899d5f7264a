"""The bit-string path on the device (pci_gpu_form_barr, pci_gpu_bit_compare)
against the oracle's restatement of FormBarr, compare_bit_dets and
get_det_indexes (src/determinants.f90:839-864, 933-1034): Barr bit for bit,
and difference count, phase and differing m-states identical for every pair,
on pairs the Hamiltonian connects (difference <= 2) and on random pairs."""
import ctypes as C

import numpy as np
import pytest

from conftest import get_system, oracle_h

pytestmark = pytest.mark.gpu


def _barr_numpy(iarr, nst):
    nint = (nst + 31) // 32
    out = np.zeros((iarr.shape[0], nint), np.uint32)
    for e in range(iarr.shape[1]):
        m = iarr[:, e].astype(np.int64) - 1
        np.bitwise_or.at(out, (np.arange(iarr.shape[0]), m // 32), (np.uint32(1) << (m % 32).astype(np.uint32)))
    return out.view(np.int32)


@pytest.mark.parametrize("name", ["small3", "cfg1", "small4", "ne6"])
def test_bit_path_matches_oracle(name):
    import oracle as O
    from pci_b200.capi import Engine
    s = get_system(name)
    (rp, col, val, *_), _ = oracle_h(name)
    with Engine(0) as e:
        e.load_system(s)
        barr = e.form_barr()
        assert np.array_equal(barr, _barr_numpy(s.iarr, s.nst))
        rng = np.random.default_rng(7)
        rows = np.repeat(np.arange(1, s.nd + 1), np.diff(rp))
        pick = rng.choice(col.size, min(col.size, 20000), replace=False)
        connected = np.stack([rows[pick], col[pick]], axis=1)
        random = rng.integers(1, s.nd + 1, size=(5000, 2))
        pairs = np.concatenate([connected, random]).astype(np.int64)
        nf, isg, i1, i2 = e.bit_compare(pairs)
    L = O.lib()
    nint = barr.shape[1]
    want = np.zeros((pairs.shape[0], 8), np.int32)
    for t, (a, b) in enumerate(pairs):
        b1 = np.ascontiguousarray(barr[a - 1])
        b2 = np.ascontiguousarray(barr[b - 1])
        nd_, is_ = C.c_int(), C.c_int()
        d1 = np.zeros(3, np.int32)
        d2 = np.zeros(3, np.int32)
        L.orc_bit_compare(b1.ctypes.data_as(C.c_void_p), b2.ctypes.data_as(C.c_void_p), nint, C.byref(nd_),
                          C.byref(is_), d1.ctypes.data_as(C.c_void_p), d2.ctypes.data_as(C.c_void_p))
        want[t] = [nd_.value, is_.value, *d1, *d2]
    got = np.concatenate([nf[:, None], isg[:, None], i1, i2], axis=1)
    assert np.array_equal(got, want)
    assert np.all(nf[:len(connected)] <= 2)


def test_bit_compare_errors():
    from pci_b200.capi import Engine, PciError
    s = get_system("tiny")
    with Engine(0) as e:
        e.load_system(s)
        with pytest.raises(PciError):
            e.bit_compare(np.array([[1, 2]]))       # before form_barr
        e.form_barr(copy=False)
        with pytest.raises(PciError):
            e.bit_compare(np.array([[1, s.nd + 1]]))
