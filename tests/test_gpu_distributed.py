"""The local GPU calls of the multi-GPU single-text build, through the C ABI:
dcx_sort_u32 (stable radix sort of key/value pairs) against numpy's stable
lexicographic sort, dcx_build_sa_u32 (SA of a 32-bit string) against a
prefix-doubling restatement, and the whole distributed build as one NCCL rank
on cuda:0 against libsais (this run has one GPU: the exchanges then stay on
the rank; their multi-rank form is covered by the gloo tests)."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch

from dist_cpu_ops import CpuOps

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("kw", [1, 2, 3])
def test_sort_u32_equals_stable_lexsort(ctx, kw):
    rng = np.random.default_rng(kw)
    for n in (0, 1, 7, 5000, 300_001):
        keys = [rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(kw)]
        keys[-1] &= 0xFF  # many equal top words: stability matters
        vals = np.arange(n, dtype=np.uint32)
        dk = [torch.from_numpy(k.view(np.int32)).cuda() for k in keys]
        dv = torch.from_numpy(vals.view(np.int32)).cuda()
        torch.cuda.synchronize()
        ctx.sort_u32_device([k.data_ptr() for k in dk], dv.data_ptr(), n)
        order = np.lexsort(keys) if n else np.zeros(0, np.int64)
        assert np.array_equal(dv.cpu().numpy().view(np.uint32), vals[order])
        for k, d in zip(keys, dk):
            assert np.array_equal(d.cpu().numpy().view(np.uint32), k[order])


def test_sort_u32_rejects_bad_arguments(ctx):
    from distributed_suffix_sorting_evaluation_b200 import DcxError
    k = torch.zeros(16, dtype=torch.int32, device="cuda")
    v = torch.zeros(16, dtype=torch.int32, device="cuda")
    with pytest.raises(DcxError):
        ctx.sort_u32_device([k.data_ptr()] * 4, v.data_ptr(), 16)  # four key words
    with pytest.raises(DcxError):
        ctx.sort_u32_device([k.data_ptr() + 4], v.data_ptr(), 8)  # not 16-byte aligned


@pytest.mark.parametrize("X", [3, 7, 39])
def test_build_sa_u32_equals_restatement(ctx, X):
    rng = np.random.default_rng(X)
    for n, sigma in ((1, 1), (100, 3), (5000, 1000), (70_000, 70_000), (40_000, 2)):
        s = rng.integers(1, sigma + 1, n).astype(np.int64)
        if n >= 40_000:
            s[n // 2: n // 2 + 10_000] = s[:10_000]  # long repeat: recursion
        d = torch.from_numpy(s.astype(np.int32)).cuda()
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        ctx.build_sa_u32_device(d.data_ptr(), n, int(s.max()), out.data_ptr(), dc=X, sa_width=32)
        want = CpuOps().suffix_array(torch.from_numpy(s), int(s.max())).numpy()
        assert np.array_equal(out.cpu().numpy().astype(np.int64), want)


WORKER = r"""
import sys
from datetime import timedelta
sys.path.insert(0, {root!r})
import numpy as np, torch, torch.distributed as dist
torch.cuda.set_device(0)
dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", 0))
from distributed_suffix_sorting_evaluation_b200 import distributed as Dd, workloads as W
from oracle import oracle as O
rng = np.random.default_rng(9)
base = rng.integers(65, 69, 30_000).astype(np.uint8)
cases = [W.markov_dna(1 << 20, seed=2), np.concatenate([base, base, base[:5000], base]),
         rng.integers(0, 256, 100_000).astype(np.uint8), np.full(3000, 66, np.uint8)]
for X in (3, 39):
    for t in cases:
        loc = Dd.build_sa_distributed(torch.from_numpy(t).cuda(), t.size, dc=X, base_threshold=4096)
        full = Dd.gather_sa(loc).cpu().numpy()
        assert np.array_equal(full, O.libsais(t).astype(np.int64)), (X, t.size)
dist.destroy_process_group()
print("distributed ok", flush=True)
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_distributed_build_one_nccl_rank():
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), WORLD_SIZE="1", RANK="0",
               LOCAL_RANK="0", NCCL_NVLS_ENABLE="0")
    p = subprocess.run([sys.executable, "-c", WORKER.format(root=ROOT)], env=env, cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, (p.stdout + p.stderr)[-3000:]
    assert "distributed ok" in p.stdout
