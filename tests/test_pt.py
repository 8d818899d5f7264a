"""Second-order CI+PT (conf_pt's PTE, src/conf_pt.f90:751-952).

CPU (oracle restatement): on a two-block matrix [[A, l B], [l B^T, D]] the
second-order energy reproduces the exact lowest eigenvalue to O(l^4) (the
third order vanishes when the coupling is off-diagonal), and scales as l^2;
average_diag changes only each PT configuration's last diagonal element.
GPU: pci_gpu_pt2 on the resident H of a CI + PT determinant list against the
oracle, with and without average_diag."""
import numpy as np
import pytest

from conftest import get_system, oracle_h


def test_pt2_oracle_known_answer():
    import oracle as O
    rng = np.random.default_rng(5)
    nci, npt = 20, 30
    A = rng.standard_normal((nci, nci)); A = (A + A.T) / 2
    D = rng.standard_normal((npt, npt)); D = (D + D.T) / 2 + 8 * np.eye(npt)   # PT space above the CI levels
    B = rng.standard_normal((nci, npt))
    w, V = np.linalg.eigh(A)
    errs = []
    for lam in (1e-2, 5e-3):
        H = np.block([[A, lam * B], [lam * B.T, np.diag(np.diag(D))]])
        dE, C = O.pt2(H, nci, nci, V[:, :1], w[:1])
        exact = np.linalg.eigvalsh(H)[0]
        errs.append(abs(exact - (w[0] + dE[0])))
        assert dE[0] < 0
        assert abs(dE[0] / lam**2 - O.pt2(np.block([[A, B], [B.T, np.diag(np.diag(D))]]), nci, nci,
                                          V[:, :1], w[:1])[0][0]) < 1e-9
    assert errs[0] < 1e-6 and errs[1] < errs[0] / 8          # fourth order in the coupling


def test_pt2_oracle_average_diag_last_determinant():
    import oracle as O
    s = get_system("small3")
    (rp, col, val, *_), _ = oracle_h("small3")
    H = O.csr_to_dense(s.nd, rp, col, val)
    cs = np.concatenate([[0], np.cumsum(s.ndc)])
    nd1 = int(cs[len(cs) // 2])
    X0 = np.linalg.eigh(H[:nd1, :nd1])[1][:, :2]
    E = np.linalg.eigvalsh(H[:nd1, :nd1])[:2]
    d0, c0 = O.pt2(H, nd1, nd1, X0, E)
    d1, c1 = O.pt2(H, nd1, nd1, X0, E, s.ndc, avg_diag=True)
    changed = np.flatnonzero(np.any(c0 != c1, axis=1))
    last = set((cs[1:] - 1)[cs[1:] > nd1].tolist())
    assert set(changed.tolist()) <= last


def _ci_pt(name, k_ci):
    import oracle as O
    s = get_system(name)
    (rp, col, val, *_), _ = oracle_h(name)
    H = O.csr_to_dense(s.nd, rp, col, val)
    cs = np.concatenate([[0], np.cumsum(s.ndc)])
    nd1 = int(cs[k_ci])
    w, V = np.linalg.eigh(H[:nd1, :nd1])
    return s, H, cs, nd1, V[:, :4], w[:4]


@pytest.mark.gpu
@pytest.mark.parametrize("name,frac", [("cfg1", 0.3), ("small3", 0.5), ("small4", 0.4)])
@pytest.mark.parametrize("avg", [False, True])
def test_pt2_gpu_matches_oracle(name, frac, avg):
    import oracle as O
    from pci_b200.capi import Engine
    s0 = get_system(name)
    s, H, cs, nd1, X0, E = _ci_pt(name, max(1, int(frac * len(s0.ndc))))
    k0 = max(1, int(np.searchsorted(cs, nd1)) // 2)
    nd0 = int(cs[k0])                                  # a smaller zero-order space
    want_de, want_c = O.pt2(H, nd1, nd0, X0[:nd0], E, s.ndc, avg_diag=avg)
    with Engine(0) as e:
        e.load_system(s)
        e.form_h(64)
        de, c = e.pt2(nd1, X0[:nd0], E, avg_diag=avg, want_vectors=True)
    assert np.allclose(de, want_de, rtol=1e-10, atol=1e-13)
    assert np.allclose(c, want_c, rtol=1e-9, atol=1e-12)


@pytest.mark.gpu
def test_pt2_gpu_errors():
    from pci_b200.capi import Engine, PciError
    s, H, cs, nd1, X0, E = _ci_pt("small3", 10)
    with Engine(0) as e:
        e.load_system(s)
        e.form_h(64)
        with pytest.raises(PciError):
            e.pt2(nd1 + 1, X0, E)                      # Nd1 inside a configuration
        with pytest.raises(PciError):
            e.pt2(nd1, np.zeros((nd1 + 1, 1)), E[:1])  # Nd0 > Nd1


def _pt_mask(ndc, nd1, nd0):
    """Positions of conf_pt's PT block in the symmetric dense H: rows beyond
    nd1 against columns below nd0, and each PT configuration's own block."""
    conf = np.repeat(np.arange(len(ndc)), ndc)
    nd = conf.size
    i = np.arange(nd)[:, None]
    k = np.arange(nd)[None, :]
    m = (i >= nd1) & ((k < nd0) | (conf[:, None] == conf[None, :]))
    return m | m.T


@pytest.mark.gpu
@pytest.mark.parametrize("name,frac", [("cfg1", 0.3), ("small3", 0.5), ("small4", 0.4)])
def test_pt_block_is_the_pt_part_of_h(name, frac):
    """pci_gpu_form_h_pt stores exactly the PT block's elements of the
    oracle's H, bit for bit, and pt2 on it equals pt2 on the whole H and the
    oracle."""
    import oracle as O
    from pci_b200.capi import Engine
    s0 = get_system(name)
    s, H, cs, nd1, X0, E = _ci_pt(name, max(1, int(frac * len(s0.ndc))))
    nd0 = int(cs[max(1, int(np.searchsorted(cs, nd1)) // 2)])
    want_de, want_c = O.pt2(H, nd1, nd0, X0[:nd0], E, s.ndc, avg_diag=True)
    with Engine(0) as e:
        e.load_system(s)
        e.form_h(64)
        de_full = e.pt2(nd1, X0[:nd0], E, avg_diag=True)
        nnz = e.form_h_pt(nd1, nd0)
        rp, col, val = e.get_csr(0)
        de, c = e.pt2(nd1, X0[:nd0], E, avg_diag=True, want_vectors=True)
    mask = _pt_mask(np.asarray(s.ndc), nd1, nd0)
    want = np.where(mask, H, 0.0)
    assert nnz == rp[-1] == np.count_nonzero(np.tril(want))
    assert np.array_equal(O.csr_to_dense(s.nd, rp, col, val), want)
    assert np.all(np.diff(rp)[:nd1] == 0)
    assert np.allclose(de, de_full, rtol=1e-12, atol=1e-15)
    assert np.allclose(de, want_de, rtol=1e-10, atol=1e-13)
    assert np.allclose(c, want_c, rtol=1e-9, atol=1e-12)


@pytest.mark.gpu
def test_pt2_more_than_16_vectors():
    """The SpMM takes 16 vectors a call; pt2 runs 20 in two."""
    import oracle as O
    from pci_b200.capi import Engine
    s, H, cs, nd1, X0, E = _ci_pt("small3", 10)
    nd0 = nd1
    rng = np.random.default_rng(11)
    Xr = rng.standard_normal((nd0, 20))
    Er = np.diag(H).min() - 1.0 - np.arange(20) * 0.1
    want_de, want_c = O.pt2(H, nd1, nd0, Xr, Er)
    with Engine(0) as e:
        e.load_system(s)
        e.form_h_pt(nd1, nd0)
        de, c = e.pt2(nd1, Xr, Er, want_vectors=True)
    assert np.allclose(de, want_de, rtol=1e-10, atol=1e-13)
    assert np.allclose(c, want_c, rtol=1e-9, atol=1e-12)


@pytest.mark.gpu
def test_pt_block_state():
    """The PT block is for pt2 alone: the solvers refuse it, pt2 refuses
    another Nd1 / Nd0, the density pass rebuilds the full adjacency, and
    FormH afterwards gives the whole H again."""
    from pci_b200.capi import Batch, Engine, PciError
    s, H, cs, nd1, X0, E = _ci_pt("small3", 10)
    nd0 = int(cs[5])
    rng = np.random.default_rng(3)
    Xd = rng.standard_normal((s.nd, 2))
    Xd /= np.linalg.norm(Xd, axis=0)
    with Engine(0) as e:
        e.load_system(s)
        nfull = e.form_h(64)[0]
        ro_full = e.density(Xd)
        e.form_h_pt(nd1, nd0)
        with pytest.raises(PciError):
            e.davidson(s.nd, Nlv=2)
        with pytest.raises(PciError):
            e.pt2(nd1, X0[:nd1], E)                # built for nd0, called with nd1
        with pytest.raises(PciError):
            e.form_h_pt(nd1 + 1, nd0)              # not a configuration end
        ro_pt = e.density(Xd)
        with Batch(0) as b:
            with pytest.raises(PciError):
                b.add_engine(e)
        assert e.form_h(64)[0] == nfull
    assert np.allclose(ro_pt, ro_full, rtol=0, atol=1e-13)   # atomics: summation order varies


def test_nr_configurations_known_answer():
    """NR_Init's grouping: 2p-1 2p+1 and 2p+2 squeeze to the same 2p^2 and
    are consecutive (one NR configuration); 2p-1 3p-1 differs; 2p-2 is 2p^2
    again but not consecutive with the first group, so it starts a new one."""
    from pci_b200 import system as S
    b = S.make_basis([(2, 1), (3, 1)])                   # 2p-, 2p+, 3p-, 3p+
    configs = [[(1, 1), (2, 1)], [(2, 2)], [(1, 1), (3, 1)], [(1, 2)]]
    assert S.squeeze_config(b, configs[0]) == S.squeeze_config(b, configs[1]) == [((2, 1), 2)]
    offs = S.nr_configurations(b, configs, [3, 2, 4, 1])
    assert offs.tolist() == [0, 5, 9, 10]
    assert S.nr_configurations(b, configs, [3, 2, 4, 1], nd1=5).tolist() == [0, 5, 9, 10]
    with pytest.raises(ValueError):
        S.nr_configurations(b, configs, [3, 2, 4, 1], nd1=3)   # inside the first NR configuration


@pytest.mark.parametrize("name", ["small3", "cfg1"])
def test_nr_configurations_partition(name):
    from pci_b200 import system as S
    s = get_system(name)
    offs = S.nr_configurations(s.basis, s.configs, s.ndc)
    ends = np.concatenate([[0], np.cumsum(s.ndc)])
    assert offs[0] == 0 and offs[-1] == s.nd and np.all(np.diff(offs) > 0)
    assert set(offs.tolist()) <= set(ends.tolist())
    # within a group the squeezed lists agree; across a boundary they differ
    conf_of = {int(e): i for i, e in enumerate(ends[:-1])}
    for a, b in zip(offs[:-1], offs[1:]):
        cs = [i for e, i in conf_of.items() if a <= e < b]
        sq = {tuple(S.squeeze_config(s.basis, s.configs[i])) for i in cs}
        assert len(sq) == 1


def test_pt2_groups_oracle_sum_to_pt2():
    import oracle as O
    from pci_b200 import system as S
    s, H, cs, nd1, X0, E = _ci_pt("small3", 10)
    offs = S.nr_configurations(s.basis, s.configs, s.ndc)
    groups = offs[offs >= nd1]
    if groups[0] != nd1:
        pytest.skip("CI / PT boundary inside an NR configuration")
    dEg, dVg = O.pt2_groups(H, nd1, nd1, X0, E, groups, s.ndc, avg_diag=True)
    dE, Cf = O.pt2(H, nd1, nd1, X0, E, s.ndc, avg_diag=True)
    assert np.allclose(dEg.sum(axis=0), dE, rtol=1e-12, atol=1e-15)
    assert np.allclose(dVg.sum(axis=0), (Cf ** 2).sum(axis=0), rtol=1e-12, atol=1e-15)


def test_pt_row_ranges():
    from pci_b200 import system as S
    s = get_system("small3")
    cs = np.concatenate([[0], np.cumsum(s.ndc)])
    nd1 = int(cs[10])
    for parts in (1, 2, 3, 7):
        r = S.pt_row_ranges(s.ndc, nd1, parts)
        assert r[0][0] == nd1 and r[-1][1] == s.nd
        assert all(a[1] == b[0] for a, b in zip(r[:-1], r[1:]))
        assert all(lo in set(cs.tolist()) and hi in set(cs.tolist()) for lo, hi in r)
        assert len(r) <= parts


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cfg1", "small3"])
def test_pt2_groups_gpu_matches_oracle(name):
    import oracle as O
    from pci_b200 import system as S
    from pci_b200.capi import Engine
    s0 = get_system(name)
    offs = S.nr_configurations(s0.basis, s0.configs, s0.ndc)
    k = int(np.searchsorted(np.concatenate([[0], np.cumsum(s0.ndc)]), offs[len(offs) // 3]))
    s, H, cs, nd1, X0, E = _ci_pt(name, k)                # the CI space ends an NR configuration
    groups = offs[offs >= nd1]
    want_eg, want_vg = O.pt2_groups(H, nd1, nd1, X0, E, groups, s.ndc, avg_diag=True)
    with Engine(0) as e:
        e.load_system(s)
        e.form_h_pt(nd1, nd1)
        de, eg, vg = e.pt2_groups(nd1, X0, E, groups, avg_diag=True)
    assert np.allclose(eg, want_eg, rtol=1e-10, atol=1e-14)
    assert np.allclose(vg, want_vg, rtol=1e-9, atol=1e-14)
    assert np.allclose(eg.sum(axis=0), de, rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
def test_pt2_row_ranges_add_up():
    """PT blocks over row ranges: their dE, first-order coefficients and
    group sums add up to the single block's."""
    from pci_b200 import system as S
    from pci_b200.capi import Engine
    s, H, cs, nd1, X0, E = _ci_pt("small3", 10)
    ranges = S.pt_row_ranges(s.ndc, nd1, 3)
    assert len(ranges) == 3
    with Engine(0) as e:
        e.load_system(s)
        e.form_h_pt(nd1, nd1)
        de, c = e.pt2(nd1, X0, E, avg_diag=True, want_vectors=True)
        de_r, c_r = e.pt2_ranges(nd1, X0, E, ranges, avg_diag=True, want_vectors=True)
        groups = np.array([nd1, ranges[0][1], s.nd], np.int64)
        e.form_h_pt(nd1, nd1, rows=ranges[0])
        _, eg0, _ = e.pt2_groups(nd1, X0, E, groups)
    assert np.allclose(de_r, de, rtol=1e-12, atol=1e-15)
    assert np.allclose(c_r, c, rtol=1e-12, atol=1e-15)
    assert np.all(eg0[1] == 0.0)                       # the other range's rows are not in this block


def _pt_rank_worker(rank, port, q):
    import os
    import torch
    import torch.distributed as dist
    import oracle as O
    from pci_b200 import system as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    s, H, cs, nd1, X0, E = _ci_pt("small3", 10)
    lo, hi = S.pt_row_ranges(s.ndc, nd1, 2)[rank]
    eg, _ = O.pt2_groups(H, nd1, nd1, X0, E, [lo, hi], s.ndc, avg_diag=True)
    t = torch.tensor(eg[0])
    dist.all_reduce(t)                                  # the one exchange: dE summed over ranks
    q.put((rank, t.numpy().copy()))
    dist.destroy_process_group()


def test_pt_ranges_two_gloo_ranks():
    """Two ranks take one PT row range each (pt_row_ranges) and compute their
    share with no exchange; one all-reduce of dE gives the whole PT space's."""
    import multiprocessing as mp
    import socket
    import oracle as O
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_pt_rank_worker, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    res = dict(q.get(timeout=10) for _ in range(2))
    s, H, cs, nd1, X0, E = _ci_pt("small3", 10)
    want, _ = O.pt2(H, nd1, nd1, X0, E, s.ndc, avg_diag=True)
    assert np.allclose(res[0], res[1], rtol=0, atol=0)
    assert np.allclose(res[0], want, rtol=1e-12, atol=1e-15)
