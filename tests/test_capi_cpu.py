"""The C-ABI library loads without a GPU and exports every entry point
declared in include/pci_gpu.h; the Python binding mirrors the header."""
import ctypes as C
import os
import re

from conftest import ROOT


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "pci_gpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(pci_(?:gpu|mlp)_\w+)\s*\(", hdr)))


def test_library_exports_header_symbols():
    from pci_b200 import build
    lib = build.build()
    L = C.CDLL(lib)
    syms = declared_symbols()
    assert len(syms) >= 10
    for name in syms:
        assert hasattr(L, name), name


def test_binding_covers_header():
    from pci_b200 import capi
    assert sorted(capi.EXPORTS) == declared_symbols()


def test_dvd_params_layout():
    """pci_dvd_params: 8 int32 then 3 doubles, no padding (ISO_C_BINDING friendly)."""
    from pci_b200.capi import DvdParams
    assert C.sizeof(DvdParams) == 8 * 4 + 3 * 8
    hdr = open(os.path.join(ROOT, "include", "pci_gpu.h")).read()
    body = hdr[hdr.index("typedef struct {"):hdr.index("} pci_dvd_params;")]
    fields = re.findall(r"(int32_t|double)\s+(\w+);", body)
    assert [f for _, f in fields] == [f for f, _ in DvdParams._fields_]


def test_no_device_is_reported_not_crashing():
    """Without a GPU (this container) creating a handle fails with PCI_E_CUDA and a message."""
    import torch
    if torch.cuda.is_available():
        return
    from pci_b200 import capi
    L = capi.load()
    h = C.c_void_p()
    rc = L.pci_gpu_create(0, C.byref(h))
    assert rc == 6
    assert b"CUDA" in L.pci_gpu_last_error(h)
    L.pci_gpu_destroy(h)


def batch_declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "pci_batch.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(pci_batch_\w+)\s*\(", hdr)))


def test_batch_header_exported_and_bound():
    from pci_b200 import build, capi
    L = C.CDLL(build.build())
    syms = batch_declared_symbols()
    assert sorted(capi.BATCH_EXPORTS) == syms
    for name in syms:
        assert hasattr(L, name), name


def test_batch_params_layout():
    """pci_batch_params: 4 int32, a double, 4 int32, a double, 2 int32 (56
    bytes, no padding), field for field as the header declares them."""
    from pci_b200.capi import BatchParams
    assert C.sizeof(BatchParams) == 56
    hdr = open(os.path.join(ROOT, "include", "pci_batch.h")).read()
    body = hdr[hdr.index("typedef struct {"):hdr.index("} pci_batch_params;")]
    fields = re.findall(r"(int32_t|double)\s+(\w+);", body)
    assert [f for _, f in fields] == [f for f, _ in BatchParams._fields_]


def test_batch_variants_and_no_device():
    """The SpMM variant table answers without a device; creating a batch
    without a GPU fails with PCI_E_CUDA and a message."""
    import torch
    from pci_b200 import capi
    assert capi.batch_variants() == [(s, c) for s in (32, 16, 8) for c in (4, 8, 16, 32)]
    if torch.cuda.is_available():
        return
    L = capi.load()
    b = C.c_void_p()
    rc = L.pci_batch_create(0, C.byref(b))
    assert rc == 6 and b"CUDA" in L.pci_batch_last_error(b)
    L.pci_batch_destroy(b)


def test_batch_sample_layout():
    """pci_batch_sample: 4 int32, an int64 and 5 doubles (64 bytes), in the
    order of the header, as the numpy record type of the binding reads it."""
    from pci_b200.capi import SAMPLE_DTYPE
    assert SAMPLE_DTYPE.itemsize == 64
    hdr = open(os.path.join(ROOT, "include", "pci_batch.h")).read()
    body = hdr[hdr.index("typedef struct {", hdr.index("} pci_batch_params;")):hdr.index("} pci_batch_sample;")]
    names = []
    for typ, rest in re.findall(r"(int32_t|int64_t|double)\s+([\w, ]+);", body):
        names += [x.strip() for x in rest.split(",")]
    assert names == list(SAMPLE_DTYPE.names)
