"""dcx_shard_texts: the size-balanced split of a batch of independent texts over
ranks (host-only C-ABI call, no GPU).  Checked against a plain restatement of
longest-first scheduling with the same tie rules, and for the balance the
batched workload gets from it."""
import heapq

import numpy as np
import pytest

from distributed_suffix_sorting_evaluation_b200 import DcxError, shard_texts
from distributed_suffix_sorting_evaluation_b200 import workloads as W


def lpt_restated(lengths, world):
    """Longest first; equal lengths in index order; the lightest rank, the lower
    rank on equal loads."""
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    heap = [(0, r) for r in range(world)]
    owner = [0] * len(lengths)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + int(lengths[i]), r))
    loads = [0] * world
    for load, r in heap:
        loads[r] = load
    return np.array(owner, np.uint32), np.array(loads, np.uint64)


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7, 8])
@pytest.mark.parametrize("case", ["random", "equal", "few", "skewed"])
def test_matches_restatement(world, case):
    rng = np.random.default_rng(world * 31 + len(case))
    lens = {
        "random": rng.integers(1, 1 << 24, 500),
        "equal": np.full(37, 4096),
        "few": rng.integers(1, 100, max(world - 1, 1)),
        "skewed": np.concatenate([[1 << 30], rng.integers(1, 1 << 12, 200)]),
    }[case].astype(np.uint64)
    owner, loads = shard_texts(lens, world)
    ref_owner, ref_loads = lpt_restated(lens, world)
    assert np.array_equal(owner, ref_owner)
    assert np.array_equal(loads, ref_loads)
    assert int(loads.sum()) == int(lens.sum())
    for r in range(world):
        assert int(lens[owner == r].sum()) == int(loads[r])
    # any greedy split: no rank above the mean plus the longest text
    assert int(loads.max()) <= int(lens.sum()) / world + int(lens.max())


def test_batched_workload_balance():
    lens = W.batch_lengths(20000, 1 << 10, 16 << 20, seed=5)
    for world in (2, 4, 8):
        owner, loads = shard_texts(lens, world)
        assert np.bincount(owner, minlength=world).min() > 0
        assert loads.max() / (lens.sum() / world) < 1.001


def test_edges():
    owner, loads = shard_texts(np.zeros(0, np.uint64), 4)
    assert owner.size == 0 and loads.tolist() == [0, 0, 0, 0]
    owner, _ = shard_texts([5, 5, 5], 8)  # more ranks than texts: one text each, lowest ranks
    assert owner.tolist() == [0, 1, 2]
    with pytest.raises(DcxError):
        shard_texts([1, 2], 0)


def test_deterministic():
    lens = np.random.default_rng(3).integers(1, 1 << 20, 5000)
    a, _ = shard_texts(lens, 8)
    b, _ = shard_texts(lens.copy(), 8)
    assert np.array_equal(a, b)


def test_bench_batch_chunks_and_share():
    """bench.py's chunking of a rank's texts (consecutive runs of about `cap`
    bytes, a longer text alone) and its share of the batch at N = 1."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    lens = np.array([5, 5, 20, 1, 1, 1, 7], np.int64)
    chunks = bench.batch_chunks(lens, 10)
    assert chunks == [(0, 2, 10), (2, 3, 20), (3, 7, 10)]
    assert sum(c[2] for c in chunks) == int(lens.sum())
    assert bench.batch_chunks(np.zeros(0, np.int64), 10) == []
    ids, shift, job, steps = bench.batch_share(lens, 1, 0, 10)
    assert ids.tolist() == list(range(lens.size)) and shift == 0 and job == int(lens.sum()) and steps == 3
