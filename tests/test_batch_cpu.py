"""The batched workload's block generator (no GPU): 64 seeded synthetic ions
with 2-4 valence electrons, 30-120 orbitals, mixed parity and M, and
determinant counts log-uniform in [2000, 400000]."""
import numpy as np

from pci_b200 import system as S


def test_batch_block_draws():
    kws = S.batch_blocks()
    assert len(kws) == 64
    assert [kw["seed"] for kw in kws] == list(range(1000, 1064))
    ne = np.array([kw["ne"] for kw in kws])
    assert set(ne) <= {2, 3, 4} and len(set(ne)) == 3
    assert len({kw["parity"] for kw in kws}) == 2
    for kw in kws:
        assert kw["mj"] % 2 == kw["ne"] % 2
        norb = sum(1 if l == 0 else 2 for _, l in kw["shells"])
        assert 30 <= norb <= 121
        assert 2000 <= kw["max_nd"] <= 400000
        assert kw["params"]["Nlv"] == 6
    t = np.log([kw["max_nd"] for kw in kws])
    # log-uniform: the logs spread over the whole range
    assert t.min() < np.log(4000) and t.max() > np.log(200000)
    assert S.batch_blocks() == kws                  # deterministic


def test_truncated_block_reaches_its_count():
    kw = S.batch_block(4)                           # a small block of the set
    s = S.make_system(**kw)
    assert s.nd >= kw["max_nd"]
    # cut right after the configuration that reaches the count
    assert s.nd - int(s.ndc[-1]) < kw["max_nd"]
    assert s.ne == kw["ne"] and s.mj == kw["mj"]
    assert s.nsu <= sum(1 if l == 0 else 2 for _, l in kw["shells"])


def test_split_blocks_partitions_and_balances():
    nds = [kw["max_nd"] for kw in S.batch_blocks()]
    for world in (1, 2, 4, 8):
        parts = [S.split_blocks(nds, world, r) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(nds)))              # every block once
        loads = [sum(nds[i] for i in p) for p in parts]
        # greedy largest-first: no rank exceeds the lightest by more than the largest block
        assert max(loads) - min(loads) <= max(nds)
    assert S.split_blocks(nds, 1, 0)[0] == int(np.argmax(nds))


def _split_worker(rank, port, q):
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    nds = [kw["max_nd"] for kw in S.batch_blocks()]
    mine = S.split_blocks(nds, 2, rank)
    got = [None, None]
    dist.all_gather_object(got, mine)
    q.put((rank, got))
    dist.destroy_process_group()


def test_split_blocks_two_gloo_ranks():
    """Two ranks compute their shares independently; gathered over gloo, the
    shares agree between ranks and partition the 64 blocks."""
    import multiprocessing as mp
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_split_worker, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res[0] == res[1]
    assert sorted(res[0][0] + res[0][1]) == list(range(64))
    assert not set(res[0][0]) & set(res[0][1])
