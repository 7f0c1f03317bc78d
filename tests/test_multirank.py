"""The multi-rank path of bench.py on CPU: two ranks over gloo.

`bench.py --gpus N` runs N independent replicas (one text per rank, no
data-path collective); the only cross-rank steps are the barrier around the
timed region and the max over ranks of the measured times.  These tests run
those steps as two real processes on the gloo backend, plus the rank handling
of the reference arm (rank 0 alone measures and prints; the others exit 0)."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import contextlib, io, json, sys
from datetime import timedelta
sys.path.insert(0, {root!r})
import numpy as np
import torch.distributed as dist
import bench
from distributed_suffix_sorting_evaluation_b200 import workloads as W

world, rank, local = bench._dist()
assert (world, local) == (2, rank), (world, rank, local)
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
# the job's time is the slowest rank's
got = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
assert got == 15.0, got
dist.barrier()
# each rank builds its own text: the generator seed is offset by the rank
w = W.WORKLOADS[bench.DEFAULT_WORKLOAD]
mine = getattr(W, w["gen"])(1 << 16, seed=w["seed"] + 1000 * rank)
gathered = [None, None]
dist.all_gather_object(gathered, mine.tobytes()[:4096])
assert gathered[0] != gathered[1]
# the batched workload: each rank computes the size-balanced split by itself;
# together the ranks build every text once and step through the same barriers
lens = W.batch_lengths(2000, 1 << 10, 16 << 20, seed=5)
cap = 256 << 20
ids, shift, job, steps = bench.batch_share(lens, world, rank, cap)
parts = [None, None]
dist.all_gather_object(parts, ids.tolist())
assert sorted(parts[0] + parts[1]) == list(range(lens.size))
assert shift == 0 and job == int(lens.sum())
assert steps == max(len(bench.batch_chunks(lens[np.array(p)], cap)) for p in parts)
ids_r, shift_r, job_r, _ = bench.batch_share(lens, world, rank, cap, "replicas")
assert ids_r.size == lens.size and shift_r == 7919 * rank and job_r == 2 * int(lens.sum())
# the reference arm: ranks other than 0 return 0 without output or work
if rank != 0:
    args = bench.argparse.Namespace(workload=bench.DEFAULT_WORKLOAD, steps=1, warmup=0,
                                    ref_sample_mib=1, batch_count=4, serve_requests=4)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.run_reference(args, world, rank) == 0
        assert bench.run_reference_batch(args, world, rank) == 0
        assert bench.run_reference_serve(args, world, rank) == 0
    assert buf.getvalue() == "", buf.getvalue()
dist.barrier()
dist.destroy_process_group()
print("rank", rank, "ok", flush=True)
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_reduce_and_split_work():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                   RANK=str(rank), LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(root=ROOT)], env=env,
                                      cwd=ROOT, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("gloo ranks did not finish")
        outs.append(out)
    for rank, (p, out) in enumerate(zip(procs, outs)):
        assert p.returncode == 0, out
        assert f"rank {rank} ok" in out


def test_max_over_ranks_is_identity_alone():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1) == 3.25
    assert bench._dist() == (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                             int(os.environ.get("LOCAL_RANK", "0")))
