"""The batched solver's forms beside plain FP64 (include/pci_batch.h):
mixed precision (FP32 SpMM phase, then FP64 on the hi/lo split of H), the
largest subspace, and the learned correction with its tensor-core network,
against dense FP64 eigensolutions of the oracle's Hamiltonians."""
import numpy as np
import pytest

from conftest import get_system, oracle_h

pytestmark = pytest.mark.gpu

TOL = 1e-8


def _dense(rp, col, val, nd):
    H = np.zeros((nd, nd))
    rows = np.repeat(np.arange(nd), np.diff(rp))
    H[rows, np.asarray(col) - 1] = val
    return H + np.tril(H, -1).T


@pytest.fixture(scope="module")
def systems():
    out = []
    for name in ["cfg1", "small3", "small4", "ne5"]:
        s = get_system(name)
        (rp, col, val, *_), _ = oracle_h(name)
        out.append((name, s, rp, col, val, _dense(rp, col, val, s.nd)))
    return out


def _batch(systems, value_prec):
    from pci_b200.capi import Batch
    b = Batch(0)
    b.set_value_prec(value_prec)
    for name, s, rp, col, val, H in systems:
        b.add_csr(rp, col, val)
    return b


def test_mixed_precision_matches_fp64_dense(systems):
    """PCI_BATCH_MIXED on split (hi + lo) blocks: every root converges to
    residual <= 1e-8 against the FP64 matrix and the levels equal the dense
    FP64 ones to 1e-9; blocks spend iterations in the FP32 phase and all
    reach the FP64 phase."""
    from pci_b200.capi import PCI_BATCH_MIXED
    nlv = 6
    with _batch(systems, 48) as b:
        r = b.davidson(nlv=nlv, max_sub=48, keep=24, max_it=400, tol=TOL, precision=PCI_BATCH_MIXED,
                       switch_tol=1e-5)
        st = b.stats()
        assert np.all(r["status"] == 1), r["status"]
        assert st["fp32_iterations"] >= 1 and st["switched_blocks"] == len(systems)
        assert st["spmm32_ms"] > 0 and st["launches_per_iteration"] == 26
        for i, (name, s, rp, col, val, H) in enumerate(systems):
            w = np.linalg.eigvalsh(H)[:nlv]
            assert np.abs(r["E"][i] - w).max() <= 1e-9, name
            X = b.vectors(i)
            assert np.linalg.norm(H @ X - X * r["E"][i], axis=0).max() <= 2 * TOL, name


def test_mixed_stall_switch(systems):
    """A switch residual below what FP32 sums can reach ends the FP32 phase
    through the stall rule, and the FP64 phase still converges."""
    from pci_b200.capi import PCI_BATCH_MIXED
    nlv = 4
    sub = [x for x in systems if x[0] in ("small3", "cfg1")]
    with _batch(sub, 48) as b:
        r = b.davidson(nlv=nlv, max_sub=32, max_it=500, tol=TOL, precision=PCI_BATCH_MIXED, switch_tol=1e-8,
                       stall_max=4)
        assert np.all(r["status"] == 1)
        assert b.stats()["switched_blocks"] == len(sub)
        for i, (name, s, rp, col, val, H) in enumerate(sub):
            assert np.abs(r["E"][i] - np.linalg.eigvalsh(H)[:nlv]).max() <= 1e-9, name


@pytest.mark.parametrize("msub,keep", [(96, 48), (112, 48), (112, 100)])
def test_largest_subspace_with_restarts(systems, msub, keep):
    """Subspaces up to PCI_BATCH_MAX_SUB (112: the kernels' shared-memory
    limits) with 12 roots, forcing restarts on small3, against the dense
    levels."""
    nlv = 12
    sub = [x for x in systems if x[0] in ("small3", "small4")]
    with _batch(sub, 64) as b:
        r = b.davidson(nlv=nlv, max_sub=msub, keep=keep, max_it=400, tol=TOL)
        assert np.all(r["status"] == 1)
        for i, (name, s, rp, col, val, H) in enumerate(sub):
            assert np.abs(r["E"][i] - np.linalg.eigvalsh(H)[:nlv]).max() <= 1e-9, name
            X = b.vectors(i)
            assert np.linalg.norm(H @ X - X * r["E"][i], axis=0).max() <= 2 * TOL
    assert r["iters"].max() * nlv > msub - nlv   # more directions than fit: restarted


def test_tensor_core_forward_matches_forward():
    """pci_mlp_forward_occ (mma.sync BF16 hidden layers, the solver's path)
    against pci_mlp_forward (FP32 activations) on the same inputs."""
    from pci_b200.capi import Mlp
    nin = 43
    m = Mlp(nin, 0, seed=5)
    rng = np.random.default_rng(3)
    n = 1000
    orbs = np.full((n, 8), 0xff, np.uint8)
    X = np.zeros((n, nin), np.float32)
    for i in range(n):
        ne = rng.integers(1, 9)
        o = rng.integers(0, nin - 3, ne)
        orbs[i, :ne] = o
        np.add.at(X[i], o, 1.0)
    f = rng.normal(0, 2, (n, 3)).astype(np.float32)
    X[:, nin - 3:] = f
    y = m.forward(X)
    yt = m.forward_occ(orbs, f)
    scale = np.abs(y).max()
    assert scale > 0
    assert np.abs(yt - y).max() <= 2e-2 * scale
    m.close()


def test_learned_correction_converges_and_falls_back():
    """The learned form on a held-out config-1 seed, with a network trained on
    samples harvested from the solver's own converged runs at other seeds:
    every root converges to the same levels as the diagonal form."""
    from pci_b200 import learned as LR
    from pci_b200 import system as S
    train_sys = [S.make_system(**S.CONFIGS["cfg1"](seed=sd)) for sd in (100, 101, 102)]
    F, T, info = LR.harvest(train_sys, nlv=6, rows_per_block=600)
    assert F.shape[0] > 10000 and np.isfinite(F).all() and np.isfinite(T).all()
    m, loss = LR.train(F, T, epochs=3)
    assert np.isfinite(loss)
    test_sys = [S.make_system(**S.CONFIGS["cfg1"](seed=1))]
    rd, _ = LR.solve(test_sys, 6, None, max_sub=48, keep=24, max_it=400, tol=TOL)
    rl, stl = LR.solve(test_sys, 6, m, max_sub=48, keep=24, max_it=400, tol=TOL)
    assert rd["status"][0] == 1 and rl["status"][0] == 1
    assert np.abs(rl["E"][0] - rd["E"][0]).max() <= 1e-9
    assert stl["launches_per_iteration"] == 26
    m.close()
