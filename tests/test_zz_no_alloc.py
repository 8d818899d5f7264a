"""pci_gpu_j_av_noalloc: the J_av entry point for callers that cannot allocate.

Callers that own all device memory themselves (their own pool, or a
framework's caching allocator) or that cannot afford cudaMalloc's implicit
synchronisation pass every array as device memory they already hold; the
entry point keeps its scratch in a static device array.  This test gives it
the J^2 matrix and vectors in caller-owned device buffers (allocated here by
torch, the caller's allocator) and checks two calls in a row against
pci_gpu_j_av on the same data, within 1e-12.  It runs in a file of its own,
collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import get_system

pytestmark = pytest.mark.gpu


def _noalloc(L, rowptr, col, val, X, nlim, nv, out, errbuf, stream=None):
    return L.pci_gpu_j_av_noalloc(C.c_void_p(rowptr.data_ptr()), C.c_void_p(col.data_ptr()),
                                  C.c_void_p(val.data_ptr()), rowptr.numel() - 1,
                                  C.c_void_p(X.data_ptr()), X.shape[1], nv, nlim,
                                  C.c_void_p(out.data_ptr()),
                                  None if stream is None else C.c_void_p(stream.cuda_stream),
                                  errbuf, len(errbuf))


@pytest.mark.parametrize("name,nv,half,use_stream", [
    ("tiny", 7, False, False),
    ("small3", 7, False, False),
    ("small3", 1, True, False),      # column filter k < nlim and row limit n < nlim
    ("small3", 64, True, True),      # the edge of the static scratch, on a side stream
    ("cfg1", 64, False, True),
])
def test_noalloc_matches_j_av(name, nv, half, use_stream):
    import torch
    from pci_b200.capi import Engine, load
    s = get_system(name)
    L = load()
    with Engine(0) as e:
        e.load_system(s)
        e.form_j()
        rp, col, val = e.get_csr(1)
        rng = np.random.default_rng(11)
        X = rng.standard_normal((s.nd, nv))
        X /= np.linalg.norm(X, axis=0)
        nlim = s.nd // 2 if half else s.nd
        ref = e.j_av(X, nlim)
    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(rp).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    d_X = torch.from_numpy(np.ascontiguousarray(X.T)).to(dev)   # column-major Nd x nv, ldx = Nd
    errbuf = C.create_string_buffer(256)
    stream = torch.cuda.Stream(device=dev) if use_stream else None
    torch.cuda.synchronize()
    for _ in range(2):
        out = torch.full((nv,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = _noalloc(L, d_rp, d_col, d_val, d_X, nlim, nv, out, errbuf, stream)
        assert rc == 0, errbuf.value
        if stream is not None:
            stream.synchronize()
        torch.cuda.synchronize()
        assert np.allclose(out.cpu().numpy(), ref, rtol=1e-12, atol=1e-12)


def test_noalloc_rejects_too_many_vectors():
    import torch
    from pci_b200.capi import load
    L = load()
    dev = torch.device("cuda:0")
    rp = torch.zeros(3, dtype=torch.int64, device=dev)
    col = torch.ones(1, dtype=torch.int32, device=dev)
    val = torch.ones(1, dtype=torch.float64, device=dev)
    X = torch.zeros((65, 2), dtype=torch.float64, device=dev)
    out = torch.zeros(65, dtype=torch.float64, device=dev)
    errbuf = C.create_string_buffer(256)
    rc = _noalloc(L, rp, col, val, X, 2, 65, out, errbuf)
    assert rc == 1
    assert b"1..64" in errbuf.value
