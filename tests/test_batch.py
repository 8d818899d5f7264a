"""The batched form (include/pci_batch.h): many CI blocks solved in one
device-resident Davidson, against dense eigensolutions of each block's
FP32-stored Hamiltonian built by the oracle."""
import numpy as np
import pytest

from conftest import get_system, oracle_h
from pci_b200 import system as S

pytestmark = pytest.mark.gpu

NAMES = ["tiny", "cfg1", "small3", "small4", "ne5"]
TOL = 1e-8


def _dense_f32(rowptr, col, val, nd):
    """Full symmetric matrix of an oracle lower-triangle CSR with FP32-rounded values."""
    H = np.zeros((nd, nd))
    v32 = np.asarray(val, np.float64).astype(np.float32).astype(np.float64)
    rows = np.repeat(np.arange(nd), np.diff(rowptr))
    H[rows, np.asarray(col) - 1] = v32
    return H + np.tril(H, -1).T


def _blocks():
    out = []
    for name in NAMES:
        s = get_system(name)
        (rp, col, val, *_), _ = oracle_h(name)
        out.append((name, s, rp, col, val))
    return out


@pytest.fixture(scope="module")
def blocks():
    return _blocks()


@pytest.fixture(scope="module")
def dense(blocks):
    return {name: np.linalg.eigh(_dense_f32(rp, col, val, s.nd)) for name, s, rp, col, val in blocks}


def _batch(blocks, names=None):
    from pci_b200.capi import Batch
    b = Batch(0)
    for name, s, rp, col, val in blocks:
        if names is None or name in names:
            b.add_csr(rp, col, val)
    return b


def test_batch_matches_dense(blocks, dense):
    nlv = 6
    with _batch(blocks) as b:
        nblk, rows, nnz = b.info()
        assert nblk == len(blocks) and rows == sum(s.nd for _, s, *_ in blocks)
        r = b.davidson(nlv=nlv, max_sub=48, max_it=400, tol=TOL)
        assert np.all(r["status"] == 1), r
        assert np.all(r["rnorm"] <= TOL)
        for i, (name, s, rp, col, val) in enumerate(blocks):
            w, U = dense[name]
            dE = np.abs(r["E"][i] - w[:nlv])
            assert dE.max() <= 1e-9, (name, dE)
            X = b.vectors(i)
            H = _dense_f32(rp, col, val, s.nd)
            assert np.abs(X.T @ X - np.eye(nlv)).max() <= 1e-10
            res = H @ X - X * r["E"][i]
            assert np.linalg.norm(res, axis=0).max() <= 2 * TOL, name
        st = b.stats()
        assert st["iterations"] == r["iters"].max() and st["launches_per_iteration"] == 25
        assert r["graph_launches"] >= (r["iters"].max() + 3) // 4


@pytest.mark.parametrize("storage", [1, 0])
def test_batch_block_alone_matches_batch(blocks, storage):
    """A block solved alone and inside the batch: every per-block step reads
    only the block's own rows, in the same order; what may differ is the
    order of the SpMM's global reductions (lower triangles, storage 0) or of
    the transposed elements within a row of a full copy (placed by atomic
    cursors when the copy is built, storage 1; these blocks all fit)."""
    nlv = 4
    with _batch(blocks) as b:
        b.set_storage(storage)
        full = b.davidson(nlv=nlv, max_sub=32, max_it=400, tol=TOL, spmm_variant=5)
        assert b.stats()["full_share"] == (1.0 if storage else 0.0)
    for i, (name, *_rest) in enumerate(blocks):
        with _batch(blocks, names=[name]) as b1:
            b1.set_storage(storage)
            one = b1.davidson(nlv=nlv, max_sub=32, max_it=400, tol=TOL, spmm_variant=5)
        assert np.abs(one["E"][0] - full["E"][i]).max() <= 1e-10, name
        assert abs(int(one["iters"][0]) - int(full["iters"][i])) <= 2, name


def test_batch_storage_forms_agree(blocks, dense):
    """Lower triangles with reductions and full copies give the same levels."""
    nlv = 6
    out = []
    for storage in (0, 1):
        with _batch(blocks) as b:
            b.set_storage(storage)
            out.append(b.davidson(nlv=nlv, max_it=400, tol=TOL))
    assert np.all(out[0]["status"] == 1) and np.all(out[1]["status"] == 1)
    assert np.abs(out[0]["E"] - out[1]["E"]).max() <= 1e-10


def test_batch_from_device_build_matches_oracle_csr(blocks):
    """Blocks whose H the device builds in FP32 (FormH) against the oracle's
    CSR rounded to FP32 on adding: the same FP32 matrix, so the same levels."""
    from pci_b200.capi import Batch
    nlv = 5
    with Batch(0) as b:
        for name, s, *_ in blocks:
            b.add_system(s, value_prec=32)
        dev = b.davidson(nlv=nlv, max_it=400, tol=TOL)
    with _batch(blocks) as b:
        ora = b.davidson(nlv=nlv, max_it=400, tol=TOL)
    assert np.abs(dev["E"] - ora["E"]).max() <= 1e-10


def test_batch_generated_blocks():
    """Small blocks of the batched workload's generator (mixed electron
    counts, parity and M) built on the device, against dense solutions."""
    from pci_b200.capi import Batch, Engine
    kws = S.batch_blocks(6, seed0=1000, nd_lo=300, nd_hi=1500)
    systems = [S.make_system(**kw) for kw in kws]
    nlv = 6
    with Batch(0) as b:
        Hs = []
        for s in systems:
            with Engine(0) as e:
                e.load_system(s)
                e.form_h(32)
                rp, col, val = e.get_csr()
                Hs.append(_dense_f32(rp, col, val, s.nd))
                b.add_engine(e)
        r = b.davidson(nlv=nlv, max_it=400, tol=TOL)
    assert np.all(r["status"] == 1)
    for i, H in enumerate(Hs):
        w = np.linalg.eigvalsh(H)[:nlv]
        assert np.abs(r["E"][i] - w).max() <= 1e-9, i


def test_batch_fp64_values_ten_roots(blocks):
    """FP64 values kept (pci_batch_set_value_prec 64) and ten roots per block:
    the levels of the unrounded oracle matrices."""
    from pci_b200.capi import Batch
    nlv = 10
    names = ["cfg1", "small3", "small4"]
    with Batch(0) as b:
        b.set_value_prec(64)
        Hs = []
        for name, s, rp, col, val in blocks:
            if name in names:
                b.add_csr(rp, col, val)
                H = np.zeros((s.nd, s.nd))
                rows = np.repeat(np.arange(s.nd), np.diff(rp))
                H[rows, np.asarray(col) - 1] = val
                Hs.append(H + np.tril(H, -1).T)
        r = b.davidson(nlv=nlv, max_sub=64, keep=24, max_it=400, tol=TOL)
        assert np.all(r["status"] == 1)
        for i, H in enumerate(Hs):
            w = np.linalg.eigvalsh(H)[:nlv]
            assert np.abs(r["E"][i] - w).max() <= 1e-9, names[i]
            X = b.vectors(i)
            assert np.linalg.norm(H @ X - X * r["E"][i], axis=0).max() <= 2 * TOL
        with pytest.raises(Exception):
            b.davidson(nlv=nlv, spmm_variant=8)    # 8 lanes per row cannot hold 10 vectors


def test_batch_iteration_limit(blocks):
    with _batch(blocks, names=["small3"]) as b:
        r = b.davidson(nlv=6, max_it=3, tol=TOL)
        assert r["status"][0] == 2 and r["iters"][0] == 3
        assert np.all(r["rnorm"][0] > TOL)


def test_batch_tune_and_cache(blocks, tmp_path):
    from pci_b200.capi import batch_variants
    cache = str(tmp_path / "tune.txt")
    nv = len(batch_variants())
    assert nv == 12
    with _batch(blocks) as b:
        v, ms, hit = b.tune(6, cache)
        assert 0 <= v < nv and ms > 0 and not hit
        v2, ms2, hit2 = b.tune(6, cache)
        assert hit2 and v2 == v and ms2 == pytest.approx(ms, rel=1e-6)
        r = b.davidson(nlv=6, max_it=400, tol=TOL)
        assert b.stats()["spmm_variant"] == v and np.all(r["status"] == 1)
    line = open(cache).read().split()
    assert line[0] == "pci_batch_spmm" and "|nv=6" in line[1]


def test_batch_errors(blocks):
    from pci_b200.capi import Batch, PciError
    with Batch(0) as b:
        with pytest.raises(PciError):
            b.davidson(nlv=4)                      # no blocks
    with _batch(blocks, names=["tiny"]) as b:
        with pytest.raises(PciError):
            b.davidson(nlv=13)                     # more roots than supported
        with pytest.raises(PciError):
            b.davidson(nlv=6, max_sub=10)          # subspace below 2*nlv
        with pytest.raises(PciError):
            b.davidson(nlv=6, max_sub=120)         # above PCI_BATCH_MAX_SUB
        with pytest.raises(PciError):
            b.davidson(nlv=4, spmm_variant=99)
        with pytest.raises(PciError):
            b.set_storage(2)
