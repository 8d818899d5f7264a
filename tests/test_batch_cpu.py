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
