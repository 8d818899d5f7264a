"""The learned Davidson correction: the MLP kernels against a numpy
restatement (forward pass, loss and every gradient, with the weights rounded
to BF16 as the kernels read them), training, and the learned Davidson form
against the diagonal one."""
import numpy as np
import pytest

from conftest import get_system
from pci_b200 import system as S

pytestmark = pytest.mark.gpu

DIMS = [None, 128, 128, 128, 1]


def bf16(a):
    """Round float32 to bfloat16 (nearest, ties to even) and back."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p, nin):
    dims = [nin] + DIMS[1:]
    Ws, bs, o = [], [], 0
    for l in range(4):
        n = dims[l] * dims[l + 1]
        Ws.append(p[o:o + n].reshape(dims[l], dims[l + 1]))
        o += n
        bs.append(p[o:o + dims[l + 1]])
        o += dims[l + 1]
    return Ws, bs


def numpy_loss_grad(p, X, T):
    """Mean squared error and its gradient for the kernels' network: BF16
    weights, FP32 biases and activations, ReLU on the three hidden layers."""
    nin = X.shape[1]
    Ws, bs = unpack(p, nin)
    Wb = [bf16(W).astype(np.float64) for W in Ws]
    A, Zs, As = X.astype(np.float64), [], [X.astype(np.float64)]
    for l in range(4):
        Z = A @ Wb[l] + bs[l]
        Zs.append(Z)
        A = np.maximum(Z, 0.0) if l < 3 else Z
        As.append(A)
    y = A[:, 0]
    n = X.shape[0]
    loss = np.mean((y - T) ** 2)
    dZ = (2.0 * (y - T) / n)[:, None]
    gW, gb = [None] * 4, [None] * 4
    for l in range(3, -1, -1):
        gW[l] = As[l].T @ dZ
        gb[l] = dZ.sum(axis=0)
        if l > 0:
            dZ = (dZ @ Wb[l].T) * (Zs[l - 1] > 0)
    g = np.concatenate([np.concatenate([gW[l].ravel(), gb[l]]) for l in range(4)])
    return loss, g


def test_mlp_gradients_match_numpy():
    from pci_b200.capi import Mlp
    rng = np.random.default_rng(0)
    nin, n = 14, 300
    m = Mlp(nin, seed=1)
    X = rng.standard_normal((n, nin)).astype(np.float32)
    T = rng.standard_normal(n).astype(np.float32)
    p = m.params()
    loss, g = m.loss_grad(X, T)
    ref_loss, ref_g = numpy_loss_grad(p.astype(np.float64), X, T)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    scale = np.max(np.abs(ref_g))
    assert np.max(np.abs(g - ref_g)) <= 2e-3 * scale
    # the forward pass alone
    y = m.forward(X)
    Ws, bs = unpack(p.astype(np.float64), nin)
    A = X.astype(np.float64)
    for l in range(4):
        A = A @ bf16(Ws[l]).astype(np.float64) + bs[l]
        if l < 3:
            A = np.maximum(A, 0.0)
    assert np.max(np.abs(y - A[:, 0])) <= 1e-3 * max(1.0, np.max(np.abs(A)))
    m.close()


def test_mlp_training_fits_a_function():
    from pci_b200.capi import Mlp
    rng = np.random.default_rng(1)
    X = rng.uniform(-1, 1, (20000, 4)).astype(np.float32)
    T = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2]).astype(np.float32)
    m = Mlp(4, seed=2)
    l0, _ = m.loss_grad(X, T)
    loss = m.train(X, T, epochs=30, batch=1024, lr=2e-3, seed=3)
    l1, _ = m.loss_grad(X, T)
    assert l1 < 0.05 * l0 and loss < 0.05 * l0
    m.close()


def test_learned_correction_gains_over_diagonal():
    """Train on samples harvested from config-1 systems at other seeds (small
    initial block, reference vectors from a solve whose initial block holds
    every determinant), then solve a held-out config-1 system both ways for
    60 iterations.  The learned form's levels come closer to the exact ones
    (measured: max |dE| 0.009 Ha learned, 0.059 Ha diagonal); it must at least
    beat the diagonal correction."""
    from pci_b200.capi import Engine, Mlp, PCI_DVD_LEARNED
    nlv, small = 6, 150

    def solved(seed):
        s = S.make_system(**S.CONFIGS["cfg1"](seed=seed))
        e = Engine(0)
        e.load_system(s)
        e.form_h(64)
        e.form_j()
        exact = e.davidson(s.nd, Nlv=nlv, N_it=5, MaxNd0=s.nd + 1, admix_crit=0.0)
        assert exact["iterations"] == 1 and np.all(exact["Iconverge"] == 1)
        return s, e, exact

    feats, targs = [], []
    for seed in (101, 102):
        s, e, exact = solved(seed)
        f, t, info = e.davidson_harvest(s.nd, s.nsu, nlv, N_it=40, MaxNd0=small, Xref=exact["X"])
        assert info["count"] == len(t) > 0 and np.all(np.isfinite(f)) and np.all(np.isfinite(t))
        feats.append(f)
        targs.append(t)
        e.close()
    X, T = np.concatenate(feats), np.concatenate(targs)
    m = Mlp(X.shape[1], seed=3)
    l0, _ = m.loss_grad(X[:20000], T[:20000])
    m.train(X, T, epochs=20, batch=4096, lr=1e-3, seed=1)
    l1, _ = m.loss_grad(X[:20000], T[:20000])
    assert l1 < l0

    s, e, exact = solved(1)
    diag = e.davidson(s.nd, Nlv=nlv, N_it=60, MaxNd0=small, admix_crit=0.0)
    e.set_correction_model(m)
    learned = e.davidson(s.nd, Nlv=nlv, N_it=60, MaxNd0=small, admix_crit=0.0, mode=PCI_DVD_LEARNED)
    e.set_correction_model(None)
    e.close()
    d_diag = np.max(np.abs(diag["Tk"] - exact["Tk"]))
    d_learned = np.max(np.abs(learned["Tk"] - exact["Tk"]))
    print(f"max |dE| after 60 iterations: diagonal {d_diag:.3e}, learned {d_learned:.3e}")
    assert d_learned < d_diag, (d_learned, d_diag)
    assert np.all(np.isfinite(learned["Tk"])) and np.all(np.isfinite(learned["resid"]))
    m.close()


def test_learned_form_needs_a_matching_model():
    from pci_b200.capi import Engine, Mlp, PciError, PCI_DVD_LEARNED
    s = get_system("tiny")
    with Engine(0) as e:
        e.load_system(s)
        e.form_h(64)
        e.form_j()
        with pytest.raises(PciError):
            e.davidson(s.nd, Nlv=3, mode=PCI_DVD_LEARNED)          # no model
        m = Mlp(s.nsu + 5, seed=0)
        e.set_correction_model(m)
        with pytest.raises(PciError):
            e.davidson(s.nd, Nlv=3, mode=PCI_DVD_LEARNED)          # wrong input width
        e.set_correction_model(None)
        m.close()
