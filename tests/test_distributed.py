"""The multi-GPU single-text build (distributed.py) as real gloo processes on
CPU: 2, 3 and 4 ranks, every rank holding one block of the text, the local
calls supplied by tests/dist_cpu_ops.py.  The gathered suffix array must equal
libsais's (built from the reference tree) for every difference cover, for
random texts of several alphabets, for lengths that leave ranks with tiny or
empty blocks, and for repetitive texts that need recursion and large tie
groups.  A low base-case threshold forces the distributed path, including its
recursion, at these small sizes.  The host-only pieces (block owners, window
words, splitter comparison) are checked directly."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import sys
from datetime import timedelta
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np, torch, torch.distributed as dist
dist.init_process_group("gloo", timeout=timedelta(seconds=120))
from distributed_suffix_sorting_evaluation_b200 import distributed as Dd
from dist_cpu_ops import CpuOps
from oracle import oracle as O
r, p = dist.get_rank(), dist.get_world_size()
rng = np.random.default_rng(5)
cases = [np.zeros(0, np.uint8)]
for n in (1, 3, 37, 301, 2500):
    for sig in (1, 2, 4, 20, 256):
        t = rng.integers(0, 256, n).astype(np.uint8) if sig == 256 else rng.integers(65, 65 + sig, n).astype(np.uint8)
        cases.append(t)
base = rng.integers(65, 69, 600).astype(np.uint8)
cases.append(np.concatenate([base, base, base[:100], rng.integers(65, 69, 50).astype(np.uint8), base]))
cases.append(np.tile(np.frombuffer(b"abcab", np.uint8), 400))
cases.append(np.full(1500, 66, np.uint8))
bad = []
for X in (3, 7, 13, 39):
    for ci, t in enumerate(cases):
        n = t.size
        blk = torch.from_numpy(t[r * n // p:(r + 1) * n // p].copy())
        for thr in (16, 1 << 20):
            loc = Dd.build_sa_distributed(blk, n, dc=X, ops=CpuOps(), base_threshold=thr)
            full = Dd.gather_sa(loc)
            if r == 0 and not np.array_equal(full.numpy(), O.libsais(t).astype(np.int64)):
                bad.append((X, ci, n, thr))
if r == 0:
    print("mismatches", bad, flush=True)
    assert not bad
dist.barrier()
dist.destroy_process_group()
print("rank", r, "ok", flush=True)
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3, 4])
def test_distributed_build_equals_libsais(world):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                   RANK=str(rank), LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
        src = WORKER.format(root=ROOT, tests=os.path.join(ROOT, "tests"))
        procs.append(subprocess.Popen([sys.executable, "-c", src], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=600)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("gloo ranks did not finish")
        outs.append(out)
    for rank, (p, out) in enumerate(zip(procs, outs)):
        assert p.returncode == 0, out[-3000:]
        assert f"rank {rank} ok" in out


def test_block_owners_and_windows():
    from distributed_suffix_sorting_evaluation_b200 import distributed as Dd
    for n, p in ((10, 3), (2, 4), (0, 2), (1000, 8)):
        starts = Dd._starts(n, p)
        st = torch.tensor(starts, dtype=torch.int64)
        pos = torch.arange(n + 1)
        own = Dd._owner(pos, st)
        for q, o in zip(pos.tolist(), own.tolist()):
            hi = starts[o + 1] if o + 1 < p else n + 1
            assert starts[o] <= q < hi, (n, p, q, o)
    # windows: base-B words (least significant first) order like the character tuples
    rng = np.random.default_rng(3)
    for B, L in ((5, 39), (257, 13), (1 << 20, 3), (3, 7)):
        cpw = Dd._chars_per_word(B)
        assert B ** cpw <= 1 << 32 < B ** (cpw + 1)
        ext = torch.from_numpy(rng.integers(0, min(B, 4), 200 + L).astype(np.int64))
        idx = torch.arange(200)
        words = Dd._window_words(ext, idx, L, B)
        packed = [tuple(int(w[i]) for w in reversed(words)) for i in range(200)]
        chars = [tuple(ext[i:i + L].tolist()) for i in range(200)]
        order_w = sorted(range(200), key=lambda i: (packed[i], i))
        order_c = sorted(range(200), key=lambda i: (chars[i], i))
        assert order_w == order_c
        assert all((packed[i] == packed[j]) == (chars[i] == chars[j]) for i in range(0, 200, 7) for j in range(200))
    rows = [torch.tensor([5, 1, 7]), torch.tensor([2, 2, 2])]  # least significant word first
    gt = Dd._rows_greater(rows, [1, 2])
    assert gt.tolist() == [True, False, True]
