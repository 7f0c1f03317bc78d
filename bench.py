#!/usr/bin/env python
"""Benchmark of the B200 DCX suffix-array build.

Workload (one step = one suffix-array build of one text):
  cfg2_dc39_markov_dna_1GiB -- 1 GiB order-3 Markov DNA with 5% repeats, DC39 with
  char packing, 40-bit SA output (seeded synthetic; no public corpus).
Metric: SA build GiB/s of input text on 1 B200 (bit-exact output).

  value   text already in HBM, SA left in HBM (40-bit), device time by CUDA events
          recorded on the library's own stream around exactly K builds
  e2e     the same through the public C ABI with pinned host buffers: text H2D,
          build, 40-bit SA D2H inside each timed step (events on the library
          stream around every step; the median step, with the mean beside it)
Inputs are larger than L2 (1 GiB vs 126 MB), so no flush is needed between steps.

--impl reference times the CPU reference implementation instead (libsais 2.10
built from the reference tree, OpenMP over all host threads) on the same whole
text (--ref-sample-mib bounds it to a prefix).  The built SA is checked on the
GPU after the timed region (--no-verify skips it).  N > 1: one process per GPU, each rank builds its own
text (independent replicas, weak scaling); the reference arm runs on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# the seeded text generators run OpenMP loops; idle OpenMP workers must sleep,
# not spin on the host cores the timed builds need for their kernel launches
os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")

GiB = float(1 << 30)
DEFAULT_WORKLOAD = "cfg2_dc39_markov_dna_1GiB"
RADIX_KERNEL = "k_onesweep"


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, world: int, device="cpu") -> float:
    """Largest value over the ranks of the process group (the job's time is its
    slowest rank's); the value itself when running alone.  `device` is where the
    backend reduces: the rank's GPU for NCCL, "cpu" for gloo."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _traffic_per_launch(kernel: str, alg_bytes_per_launch: float):
    """DRAM bytes per launch of the dominant kernel.  profiles/traffic.json holds
    the DRAM read + write bytes per element-word (one carried 32-bit word of one
    element: a pass reads and writes each once, 8 algorithmic bytes) that a
    small-case ncu capture of the same kernel measured; a launch here moves
    alg_bytes_per_launch / 8 element-words."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        e = json.load(f).get(kernel)
    if not isinstance(e, dict) or "dram_bytes_per_element_word" not in e:
        return None
    return int(e["dram_bytes_per_element_word"] * alg_bytes_per_launch / 8)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(text: np.ndarray, sample_bytes: int, threads: int):
    """libsais64_omp (reference tree sources) on the first `sample_bytes` of the text."""
    from oracle import oracle as O
    s = np.ascontiguousarray(text[:sample_bytes])
    O.libsais(s[: 1 << 20], threads=threads)  # warm the library and threads
    t0 = time.perf_counter()
    O.libsais(s, threads=threads)
    dt = time.perf_counter() - t0
    return s.size / GiB / dt, dt


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    from distributed_suffix_sorting_evaluation_b200 import workloads as W
    w = W.WORKLOADS[args.workload]
    text = W.make(args.workload)
    threads = os.cpu_count() or 1
    sample = min(text.size, args.ref_sample_mib << 20) if args.ref_sample_mib else text.size
    for _ in range(args.warmup):
        cpu_baseline(text, min(sample, 64 << 20), threads)
    vals = []
    for _ in range(args.steps):
        v, _ = cpu_baseline(text, sample, threads)
        vals.append(v)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "SA build GiB/s", "value": round(value, 4), "unit": "GiB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(sample / GiB / value * 1000, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": args.workload, "text_bytes": int(w["n"]), "dc": w["dc"], "sa_width": w["sa_width"],
                   "timed_text_bytes": int(sample), "same_text": bool(sample == text.size)},
        "cpu_baseline": {"value": round(value, 4), "unit": "GiB/s", "cores": threads, "kind": "reference",
                         "sample": (f"libsais64_omp on the whole {sample >> 20} MiB workload text"
                                    if sample == text.size else
                                    f"libsais64_omp on the first {sample >> 20} MiB of the workload text")
                                   + f", {threads} threads"},
        "e2e": {"value": round(value, 4), "unit": "GiB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_batch(args, world, rank):
    """Reference arm of the batched workload: libsais64_omp per text over a
    bounded sample of the batch's texts (the first texts in batch order up to
    --ref-sample-mib of text), all host threads."""
    if rank != 0:
        return 0
    from distributed_suffix_sorting_evaluation_b200 import workloads as W
    from oracle import oracle as O
    lens = W.batch_lengths(args.batch_count, 1 << 10, 16 << 20, seed=5)
    threads = os.cpu_count() or 1
    cap = (args.ref_sample_mib or 256) << 20
    texts, tot = [], 0
    for j in range(lens.size):
        if texts and tot + int(lens[j]) > cap:
            break
        texts.append(W.iid(int(lens[j]), b"ACGT", seed=1_000_000 + j))
        tot += int(lens[j])
    O.libsais(texts[0], threads=threads)
    vals = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        for t in texts:
            O.libsais(t, threads=threads)
        vals.append(tot / GiB / (time.perf_counter() - t0))
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "batched SA build GiB/s", "value": round(value, 4), "unit": "GiB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tot / GiB / value * 1000, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "cfg4_batch", "texts": int(lens.size), "text_bytes": int(lens.sum()), "sa_width": 32},
        "cpu_baseline": {"value": round(value, 4), "unit": "GiB/s", "cores": threads, "kind": "reference",
                         "sample": f"libsais64_omp per text on the first {len(texts)} texts "
                                   f"({tot >> 20} MiB), {threads} threads"},
        "e2e": {"value": round(value, 4), "unit": "GiB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_serve(args, world, rank):
    """Reference arm of the serving workload: libsais64_omp per request, in
    arrival order, over the first requests up to --ref-sample-mib of text."""
    if rank != 0:
        return 0
    from distributed_suffix_sorting_evaluation_b200 import workloads as W
    from oracle import oracle as O
    base_n = 1 << 30
    lens = W.batch_lengths(args.serve_requests, 4 << 10, 256 << 20, seed=6).astype(np.int64)
    rng = np.random.default_rng(7)
    offs = (rng.random(lens.size) * (base_n - lens)).astype(np.int64)
    base = W.markov_dna(base_n, seed=2)
    threads = os.cpu_count() or 1
    cap = (args.ref_sample_mib or 256) << 20
    k, tot = 0, 0
    while k < lens.size and (k == 0 or tot + int(lens[k]) <= cap):
        tot += int(lens[k])
        k += 1
    O.libsais(base[: 1 << 20], threads=threads)
    vals = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        for i in range(k):
            O.libsais(base[offs[i]:offs[i] + lens[i]], threads=threads)
        vals.append(tot / GiB / (time.perf_counter() - t0))
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": "served SA build GiB/s", "value": round(value, 4), "unit": "GiB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(tot / GiB / value * 1000, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "cfg5_serve", "lengths": "log-uniform 4 KiB-256 MiB", "sa_width": 32},
        "cpu_baseline": {"value": round(value, 4), "unit": "GiB/s", "cores": threads, "kind": "reference",
                         "sample": f"libsais64_omp per request on the first {k} requests "
                                   f"({tot >> 20} MiB), {threads} threads"},
        "e2e": {"value": round(value, 4), "unit": "GiB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def gsa_sample_check(d_set, d_gsa, pairs: int, seed: int) -> str:
    """Checks a generalized SA built on the device: a permutation of 0..n-1
    (device sort), and `pairs` random adjacent entries in the order of the
    string-set convention (suffixes compared through their separator, the 0 that
    ends each string, which is smaller than every character; suffixes equal
    through their separators ordered by string).  Raises on a violation."""
    import torch
    n = d_set.numel()
    srt, _ = torch.sort(d_gsa.to(torch.int64))
    if not torch.equal(srt, torch.arange(n, device=srt.device)):
        raise SystemExit("the generalized SA is not a permutation")
    del srt
    t = d_set.cpu().numpy()
    g = d_gsa.cpu().numpy().astype(np.int64)
    zpos = np.flatnonzero(t == 0)
    rng = np.random.default_rng(seed)
    for k in rng.integers(1, n, pairs):
        i, j = int(g[k - 1]), int(g[k])
        ei, ej = int(zpos[np.searchsorted(zpos, i)]), int(zpos[np.searchsorted(zpos, j)])
        a, b = t[i:ei + 1], t[j:ej + 1]
        m = min(a.size, b.size)
        d = np.flatnonzero(a[:m] != b[:m])
        if d.size:
            ok = a[d[0]] < b[d[0]]
        else:  # equal through the shorter one's separator: only possible when both end together
            ok = a.size == b.size and ei < ej
        if not ok:
            raise SystemExit(f"generalized SA out of order at entry {int(k)}")
    return f"permutation + {pairs} sampled adjacent pairs in order"


def run_split(args, world, rank, local):
    """One text spread over all ranks (--split-text): rank r holds the block
    T[r*n//N, (r+1)*n//N) and the ranks build the one suffix array together
    with the distributed sample sort of distributed.py (NCCL exchanges; strong
    scaling: the whole job builds one text).  value: text bytes / slowest
    rank's device time of the whole collective build, block already on the
    GPU.  e2e: the same with the block copied from pinned host memory and the
    rank's SA slice copied back inside each step."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from distributed_suffix_sorting_evaluation_b200 import Context, workloads as W
    from distributed_suffix_sorting_evaluation_b200 import distributed as Dd

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world == 1:  # one rank without torchrun: a local rendezvous
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", str(29500 + os.getpid() % 1000))
    if not dist.is_initialized():
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev,
                                world_size=world, rank=rank)
    w, gen_kw, label = _single_workload(args)
    n = int(w["n"])
    text = getattr(W, w["gen"])(n, seed=w["seed"], **gen_kw)  # the same text on every rank
    lo, hi = rank * n // world, (rank + 1) * n // world
    h_block = torch.from_numpy(text[lo:hi].copy()).pin_memory()
    d_block = h_block.to(dev)
    ctx = Context(local)
    ops = Dd.DeviceOps(ctx, dev)

    def step(block):
        return Dd.build_sa_distributed(block, n, dc=w["dc"], ops=ops)

    for _ in range(args.warmup):
        step(d_block)
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            loc = step(d_block)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    clock = clocks.summary()
    ms = max_over_ranks(ms, world, dev)
    ms_step = ms / args.steps
    verified = None
    if args.verify:
        full = Dd.gather_sa(loc)
        if rank == 0:
            ok = ctx.check_sa_device(torch.from_numpy(text).to(dev).data_ptr(), n,
                                     full.to(torch.int64).contiguous().data_ptr(), 64)
            verified = bool(ok)
            if not ok:
                raise SystemExit("the distributed suffix array failed the GPU check")
        del full
    # end to end: pinned block in, SA slice out
    e2e_ms = []
    for _ in range(max(1, min(args.steps, args.e2e_steps))):
        dist.barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        sl = step(h_block.to(dev, non_blocking=True))
        host_sa = sl.cpu()
        b.record()
        torch.cuda.synchronize()
        e2e_ms.append(max_over_ranks(a.elapsed_time(b), world, dev))
    ms_e2e = statistics.median(e2e_ms)
    if rank == 0:
        line = {
            "metric": "SA build GiB/s", "value": round(n / GiB / (ms_step / 1000.0), 4), "unit": "GiB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
            "data": W.DESCRIPTIONS[args.workload],
            "config": {"workload": label,
                       "text_bytes": n, "dc": w["dc"], "sa_width": 64,
                       "l2_flush": "inputs larger than L2", "parallelism": f"split text over {world} ranks"},
            "e2e": {"value": round(n / GiB / (ms_e2e / 1000.0), 4), "unit": "GiB/s",
                    "h2d_bytes_per_step": int(hi - lo), "d2h_bytes_per_step": int(host_sa.numel() * 8),
                    "statistic": "median step, max over ranks"},
            "verified": verified, "clocks": clock,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    dist.destroy_process_group()
    return 0


def run_gpu(args, world, rank, local):
    import torch
    from distributed_suffix_sorting_evaluation_b200 import Context, workloads as W

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    w, gen_kw, label = _single_workload(args)
    n = int(w["n"])
    dc, width = w["dc"], w["sa_width"]
    wb = width // 8
    host_text = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    getattr(W, w["gen"])(n, seed=w["seed"] + 1000 * rank, out=host_text.numpy(), **gen_kw)
    d_text = host_text.to(f"cuda:{local}")
    d_sa = torch.empty(n * wb, dtype=torch.uint8, device=f"cuda:{local}")
    host_sa = torch.empty(n * wb, dtype=torch.uint8, pin_memory=True)
    ctx = Context(local)
    if args.recursion_dc:
        ctx.set_option("recursion_dc", args.recursion_dc)
    for kv in args.option:
        k, v = kv.split("=", 1)
        ctx.set_option(k, float(v))
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    torch.cuda.synchronize()

    def step_device():
        ctx.build_sa_device(d_text.data_ptr(), n, d_sa.data_ptr(), dc=dc, sa_width=width)

    def step_e2e():
        ctx.build_sa_hostptr(host_text.data_ptr(), n, host_sa.data_ptr(), dc=dc, sa_width=width)

    for _ in range(args.warmup):
        step_device()
    # device-resident timing: exactly K builds between two events on the library stream
    stats = []
    with ClockSampler(local) as clocks:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step_device()
            stats.append(ctx.stats())
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    clock = clocks.summary()
    verified = None
    if args.verify:  # size-independent check of the last SA on the GPU (permutation + order conditions)
        verified = ctx.check_sa_device(d_text.data_ptr(), n, d_sa.data_ptr(), width)
        if not verified:
            raise SystemExit("the suffix array failed the GPU check")
    ms = max_over_ranks(ms, world, f"cuda:{local}")
    ms_step = ms / args.steps
    value = world * n / GiB / (ms_step / 1000.0)

    lcp_line = None
    if args.lcp:  # LCP of the built SA, device-resident (Phi + chunked Kasai)
        d_lcp = torch.empty(n, dtype=torch.int32, device=f"cuda:{local}")
        ctx.build_lcp_device(d_text.data_ptr(), n, d_sa.data_ptr(), width, d_lcp.data_ptr(), 32)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(3):
            ctx.build_lcp_device(d_text.data_ptr(), n, d_sa.data_ptr(), width, d_lcp.data_ptr(), 32)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_lcp = e0.elapsed_time(e1) / 3
        lcp_line = {"value": round(n / GiB / (ms_lcp / 1000.0), 4), "unit": "GiB/s", "ms": round(ms_lcp, 3),
                    "call": "dcx_build_lcp, device pointers, uint32 LCP"}
        del d_lcp

    bwt_line = None
    if args.bwt:  # BWT of the built SA, device-resident (primary-index scan + gather)
        d_bwt = torch.empty(n, dtype=torch.uint8, device=f"cuda:{local}")
        ctx.build_bwt_device(d_text.data_ptr(), n, d_sa.data_ptr(), width, d_bwt.data_ptr())
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(3):
            ctx.build_bwt_device(d_text.data_ptr(), n, d_sa.data_ptr(), width, d_bwt.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        ms_bwt = e0.elapsed_time(e1) / 3
        bwt_line = {"value": round(n / GiB / (ms_bwt / 1000.0), 4), "unit": "GiB/s", "ms": round(ms_bwt, 3),
                    "call": "dcx_build_bwt, device pointers"}
        del d_bwt

    safile_line = None
    if args.safile:  # SA file stream: device SA -> file (the reference's raw layout) -> device, checked
        import shutil
        sdir = args.safile_dir or tempfile.gettempdir()
        nbytes = n * wb
        free = shutil.disk_usage(sdir).free
        if free < nbytes + (4 << 30):
            safile_line = {"skipped": f"{free >> 30} GiB free in {sdir}; the SA file takes {nbytes >> 30} GiB"}
        else:
            path = os.path.join(sdir, f"dcx_sa_{os.getpid()}.bin")
            try:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ctx.write_sa_file(path, d_sa.data_ptr(), n, width)
                t1 = time.perf_counter()
                d_back = torch.empty_like(d_sa)
                torch.cuda.synchronize()
                t2 = time.perf_counter()
                ctx.read_sa_file(path, d_back.data_ptr(), n, width)
                torch.cuda.synchronize()
                t3 = time.perf_counter()
                same = bool(torch.equal(d_back, d_sa))
                del d_back
                safile_line = {"write_gb_per_s": round(nbytes / (t1 - t0) / 1e9, 3),
                               "read_gb_per_s": round(nbytes / (t3 - t2) / 1e9, 3), "bytes": nbytes,
                               "round_trip_equal": same,
                               "call": "dcx_write_sa_file then dcx_read_sa_file of the built SA, wall clock, "
                                       "one file in " + sdir}
            finally:
                if os.path.exists(path):
                    os.remove(path)

    gsa_line = None
    if args.gsa:  # generalized SA of the workload text cut into 1 MiB strings (a 0 ends each)
        d_set = d_text.clone()
        d_set[d_set == 0] = 1  # a 0 inside a string would end it early (Zipf texts hold 0 bytes)
        d_set[(1 << 20) - 1::1 << 20] = 0
        if n >= 2 and (n - 2) % (1 << 20) == (1 << 20) - 1:
            d_set[n - 2] = 1  # no empty last string
        d_set[n - 1] = 0
        d_gsa = torch.empty(n, dtype=torch.int32, device=f"cuda:{local}")
        ctx.build_gsa_device(d_set.data_ptr(), n, d_gsa.data_ptr(), dc=dc, sa_width=32)
        torch.cuda.synchronize()
        e0.record(stream)
        ctx.build_gsa_device(d_set.data_ptr(), n, d_gsa.data_ptr(), dc=dc, sa_width=32)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_gsa = e0.elapsed_time(e1)
        gsa_checked = gsa_sample_check(d_set, d_gsa, pairs=2000, seed=rank)
        gsa_line = {"value": round(n / GiB / (ms_gsa / 1000.0), 4), "unit": "GiB/s", "ms": round(ms_gsa, 3),
                    "call": "dcx_build_gsa, device pointers, 1 MiB strings, uint32 GSA",
                    "checked": gsa_checked}
        del d_set, d_gsa

    # end-to-end through the public call with host buffers; the device-resident
    # buffers of the runs above are released first, so the host-pointer build
    # has the device memory a caller of that path would have
    del d_text, d_sa
    torch.cuda.empty_cache()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    step_e2e()
    step_e2e()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # each step between two events on the library stream (H2D, build, D2H);
    # the line's value uses the median step, robust to stalls of the shared host
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(e2e_steps)]
    e2e_trace = []
    for a, b in ev:
        a.record(stream)
        step_e2e()
        b.record(stream)
        st = ctx.stats()
        e2e_trace.append(round(st["ms_total"], 1))
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms_e2e = statistics.median(step_ms)
    e2e_stats = ctx.stats()
    ms_e2e = max_over_ranks(ms_e2e, world, f"cuda:{local}")
    e2e_value = world * n / GiB / (ms_e2e / 1000.0)
    e2e_mean = world * n / GiB / (sum(step_ms) / len(step_ms) / 1000.0)

    # roofline of the dominant kernel (onesweep radix pass)
    s_last = stats[-1]
    bytes_radix = sum(s["bytes_radix"] for s in stats)
    ms_radix = sum(s["ms_radix"] for s in stats)
    passes = sum(s["radix_passes"] for s in stats)
    peak, peak_kind = _peaks()
    achieved = bytes_radix / (ms_radix / 1000.0) / 1e9 if ms_radix > 0 else 0.0
    launches = sum(s["kernel_launches"] for s in stats)

    if rank == 0:
        line = {
            "metric": "SA build GiB/s", "value": round(value, 4), "unit": "GiB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": W.DESCRIPTIONS[args.workload],
            "config": {"workload": label,
                       "text_bytes": n, "dc": dc, "packing": True, "sa_width": width,
                       "l2_flush": "inputs larger than L2 (1 GiB text)",
                       "parallelism": "replicas" if world > 1 else "single-gpu"},
            "e2e": {"value": round(e2e_value, 4), "unit": "GiB/s", "h2d_bytes_per_step": n,
                    "d2h_bytes_per_step": n * wb, "steps": e2e_steps,
                    "ms_h2d": round(e2e_stats["ms_h2d"], 2), "ms_build": round(e2e_stats["ms_total"], 2),
                    "ms_d2h": round(e2e_stats["ms_d2h"], 2), "statistic": "median step",
                    "mean_value": round(e2e_mean, 4), "step_ms": [round(x, 1) for x in step_ms],
                    "build_ms": e2e_trace},
            "gpu_launches": int(launches),
            "verified": verified,
            "roofline": {"kernel": f"{RADIX_KERNEL} (8-bit LSD radix pass)", "bound": "hbm",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "bytes_per_launch": int(bytes_radix / max(passes, 1)),
                         "launches": int(passes),
                         "traffic": _traffic_per_launch(RADIX_KERNEL, bytes_radix / max(passes, 1)),
                         "traffic_source": "profiles/traffic.json (ncu DRAM bytes per element-word of a small-case "
                                           "capture, scaled to this launch's element-words)"},
            "build_stats": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in s_last.items()},
            "clocks": clock,
        }
        if lcp_line:
            line["lcp"] = lcp_line
        if bwt_line:
            line["bwt"] = bwt_line
        if gsa_line:
            line["gsa"] = gsa_line
        if safile_line:
            line["safile"] = safile_line
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            sample = min(n, args.cpu_sample_mib << 20) if args.cpu_sample_mib else n
            v, dt = cpu_baseline(host_text.numpy(), sample, threads)
            line["cpu_baseline"] = {"value": round(v, 4), "unit": "GiB/s", "cores": threads, "kind": "reference",
                                    "sample": (f"libsais64_omp on the whole {sample >> 20} MiB text" if sample == n
                                               else f"libsais64_omp on the first {sample >> 20} MiB of the same text")
                                              + f" ({dt:.2f} s), {threads} threads"}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def batch_share(lens, world, rank, cap, split="lpt"):
    """This rank's part of the batched workload: (indices of its texts in batch
    order, seed offset of its texts, bytes the whole job builds, chunks of the
    rank with the most chunks).  "lpt" splits the texts by size, longest first
    (every rank computes the same split, no collective); "replicas" gives every
    rank all texts with its own seeds.  Every rank steps through the largest
    chunk count so that all ranks enter the same barriers."""
    if world <= 1 or split == "replicas":
        shift = 7919 * rank if world > 1 else 0
        return np.arange(lens.size), shift, world * int(lens.sum()), len(batch_chunks(lens, cap))
    from distributed_suffix_sorting_evaluation_b200 import shard_texts
    owner, _ = shard_texts(lens, world)
    steps = max(len(batch_chunks(lens[owner == r], cap)) for r in range(world))
    return np.flatnonzero(owner == rank), 0, int(lens.sum()), steps


def batch_chunks(lens, cap):
    """Consecutive runs of texts of about `cap` bytes each: (first, end, bytes)."""
    chunks, s0 = [], 0
    while s0 < lens.size:
        s1, tot = s0, 0
        while s1 < lens.size and (s1 == s0 or tot + int(lens[s1]) <= cap):
            tot += int(lens[s1])
            s1 += 1
        chunks.append((s0, s1, tot))
        s0 = s1
    return chunks


def run_batch(args, world, rank, local):
    """Batched workload: `count` independent i.i.d. {A,C,G,T} texts, lengths
    log-uniform in [1 KiB, 16 MiB] (seeded), one uint32 SA per text.  The texts
    are staged on the device a chunk (about --batch-chunk-mib of text) at a time;
    the timed region is the batched call over every chunk with the chunk's text
    already in HBM.  Beside it, the plain single-text call is looped over the
    same texts (whole chunks, while --loop-budget-s lasts) and the batched time
    of exactly those chunks gives the speed-up.  Under torchrun the texts are
    split over the ranks by size, longest first (--batch-split lpt, strong
    scaling: the same 20,000 texts in total), or every rank builds its own
    copy of the batch (--batch-split replicas, weak scaling)."""
    import torch
    from distributed_suffix_sorting_evaluation_b200 import Context, workloads as W

    if args.batch_count < world:
        raise SystemExit("the batched workload needs at least one text per rank")
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = f"cuda:{local}"
    all_lens = W.batch_lengths(args.batch_count, 1 << 10, 16 << 20, seed=5)
    ids, seed_shift, job_bytes, nsteps = batch_share(all_lens, world, rank, args.batch_chunk_mib << 20,
                                                     args.batch_split)
    lens = all_lens[ids]
    total = int(lens.sum())
    chunks = batch_chunks(lens, args.batch_chunk_mib << 20)
    big = max(c[2] for c in chunks)
    d_text = torch.empty(big + 16, dtype=torch.uint8, device=dev)
    d_sa = torch.empty(big + 16, dtype=torch.int32, device=dev)
    h_text = torch.empty(big + 16, dtype=torch.uint8, pin_memory=True)
    ctx = Context(local)
    tuned = None
    if args.batch_autotune:
        # size-class DCs from a sample of the workload's own distribution (other
        # seeds), tuned before the timed region
        slens = W.batch_lengths(400, 1 << 10, 16 << 20, seed=11)
        sample = [W.iid(int(m), b"ACGT", seed=2_000_000 + i) for i, m in enumerate(slens)]
        bounds = [16 << 10, 256 << 10, 2 << 20, 16 << 20]
        chosen, ms_tab = ctx.autotune_batch(sample, bounds, candidates=(3, 7, 13, 21, 39), repeats=2)
        tuned = {"classes_max_len": bounds, "dc": chosen, "ms": ms_tab.round(3).tolist(),
                 "radix_tile": ctx.batch_tile_table()}
        del sample
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def stage(ci):
        a, b, tot = chunks[ci]
        offs = np.zeros(b - a + 1, np.uint64)
        offs[1:] = np.cumsum(lens[a:b], dtype=np.uint64)
        hv = h_text.numpy()
        for j in range(a, b):
            o = int(offs[j - a])
            W.iid(int(lens[j]), b"ACGT", seed=1_000_000 + int(ids[j]) + seed_shift, out=hv[o:o + int(lens[j])])
        d_text[:tot].copy_(h_text[:tot], non_blocking=True)
        torch.cuda.synchronize()
        return offs

    def batched(offs):
        ctx.build_sa_batch_raw(d_text.data_ptr(), offs.ctypes.data, offs.size - 1, d_sa.data_ptr(), dc=0,
                               sa_width=32, device=True)

    def looped(offs):
        for k in range(offs.size - 1):
            b, n = int(offs[k]), int(offs[k + 1] - offs[k])
            ctx.build_sa_device(d_text.data_ptr() + b, n, d_sa.data_ptr() + 4 * b, dc=39, sa_width=32)

    offs0 = stage(0)
    for _ in range(max(1, args.warmup)):
        batched(offs0)
    torch.cuda.synchronize()
    batch_ms, loop_ms, loop_batch_ms = [], 0.0, 0.0
    loop_texts = loop_bytes = 0
    launches = 0
    verified = 0
    loop_open = args.loop_budget_s > 0
    with ClockSampler(local) as clocks:
        for ci in range(nsteps):
            if ci >= len(chunks):  # another rank still has chunks: meet its barriers
                torch.distributed.barrier()
                continue
            offs = offs0 if ci == 0 else stage(ci)
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            e0.record(stream)
            batched(offs)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            batch_ms.append(ms)
            last_stats = ctx.stats()
            launches += last_stats["kernel_launches"]
            if args.verify:
                a, b, tot = chunks[ci]
                for k in sorted({0, (b - a) // 2, b - a - 1}):
                    o, n = int(offs[k]), int(offs[k + 1] - offs[k])
                    t = h_text.numpy()[o:o + n].copy()
                    raw = d_sa[o:o + n].cpu().numpy().view(np.uint8)
                    if not ctx.check_sa(t, raw, 32):
                        raise SystemExit(f"batched SA of text {int(ids[a + k])} failed the check")
                    verified += 1
            if loop_open:
                e0.record(stream)
                looped(offs)
                e1.record(stream)
                torch.cuda.synchronize()
                loop_ms += e0.elapsed_time(e1)
                loop_batch_ms += ms
                loop_texts += chunks[ci][1] - chunks[ci][0]
                loop_bytes += chunks[ci][2]
                loop_open = loop_ms < args.loop_budget_s * 1000.0
    clock = clocks.summary()
    ms_total = sum(batch_ms)
    ms_total = max_over_ranks(ms_total, world, dev)
    value = job_bytes / GiB / (ms_total / 1000.0)
    split = args.batch_split if world > 1 else "single-gpu"
    if rank == 0:
        loop_v = loop_bytes / GiB / (loop_ms / 1000.0) if loop_ms > 0 else None
        same_v = loop_bytes / GiB / (loop_batch_ms / 1000.0) if loop_batch_ms > 0 else None
        line = {
            "metric": "batched SA build GiB/s", "value": round(value, 4), "unit": "GiB/s", "n_gpus": world,
            "steps": len(chunks), "warmup": max(1, args.warmup), "ms_per_step": round(ms_total / len(chunks), 3),
            "higher_is_better": True, "scaling": "strong" if split == "lpt" else "weak", "vs_baseline": None,
            "dtype": "u8",
            "data": "synthetic (seeded i.i.d. {A,C,G,T} texts, log-uniform lengths 1 KiB-16 MiB)",
            "config": {"workload": "cfg4_batch", "texts": int(all_lens.size), "text_bytes": int(all_lens.sum()),
                       "job_bytes": int(job_bytes), "rank0_texts": int(lens.size), "rank0_bytes": total,
                       "chunk_mib": args.batch_chunk_mib,
                       "dc": tuned if tuned else "DC39 above the in-CTA base case (2048 chars)", "sa_width": 32,
                       "l2_flush": "each chunk's text and SAs are larger than L2",
                       "parallelism": split},
            "seconds": round(ms_total / 1000.0, 3),
            "loop": {"value": None if loop_v is None else round(loop_v, 4), "unit": "GiB/s", "texts": loop_texts,
                     "bytes": loop_bytes, "call": "dcx_build_sa per text, DC39, device pointers",
                     "batched_same_texts": None if same_v is None else round(same_v, 4),
                     "speedup": None if not (loop_v and same_v) else round(same_v / loop_v, 3)},
            "verified_texts": verified,
            "gpu_launches": int(launches),
            "build_stats_last_chunk": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in last_stats.items()},
            "clocks": clock,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_serve(args, world, rank, local):
    """Serving workload: SA requests with lengths log-uniform in [4 KiB, 256 MiB]
    (seeded), each a distinct slice of a 1 GiB order-3 Markov DNA text (5%
    repeats), DC39, 32-bit SA, under a 150 GB serving budget.
      capacity  closed loop: the first requests (about --serve-cap-gib of text)
                submitted back to back, time until the last is done;
      served    open loop: Poisson arrivals at 80% of that capacity for
                --serve-seconds; p50/p99 of submit -> done latency (SA complete
                in HBM) and the sustained GiB/s of finished requests;
      plain     the per-request path on the capacity run's requests: one
                dcx_build_sa per request on its slice already in HBM (no
                upload), while --loop-budget-s lasts.
    Requests borrow slices of a pinned host copy of the text (zero-copy
    submission; --serve-copy makes the server copy each text at submission);
    the server's upload of each text is inside the latency."""
    import torch
    from distributed_suffix_sorting_evaluation_b200 import Context, SERVE_DONE, workloads as W

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=torch.device("cuda", local))
    base_n = 1 << 30
    base = W.markov_dna(base_n, seed=2 + 1000 * rank)
    count = args.serve_requests
    lens = W.batch_lengths(count, 4 << 10, 256 << 20, seed=6).astype(np.int64)
    rng = np.random.default_rng(7 + rank)
    offs = (rng.random(count) * (base_n - lens)).astype(np.int64)
    h_base = torch.from_numpy(base).pin_memory()
    ctx = Context(local)
    ctx.set_option("serve_budget", args.serve_budget_gb * 1e9)
    ctx.set_option("serve_lanes", args.serve_lanes)
    ctx.set_option("serve_express_priority", args.serve_express_priority)
    borrow = not args.serve_copy

    def submit(i):
        # borrow: requests point into the pinned host text (zero-copy submission);
        # copy: the server copies each text at submission (pinned arena)
        return ctx.serve_submit(None, dc=39, sa_width=32, text_ptr=h_base.data_ptr() + int(offs[i]),
                                n=int(lens[i]), borrow=borrow)

    # warm-up: a few requests of every size class through all lanes
    wids = [submit(i) for i in range(min(count, 3 * args.serve_lanes))]
    ctx.serve_drain()
    for r in wids:
        ctx.serve_release(r)

    # 1. capacity (closed loop): all submitted back to back, released as they finish
    cap_bytes = args.serve_cap_gib << 30
    k, tot = 0, 0
    while k < count and tot < cap_bytes:
        tot += int(lens[k])
        k += 1
    t0 = time.perf_counter()
    ids = [submit(i) for i in range(k)]
    t_sub = time.perf_counter() - t0
    for r in ids:
        while True:
            st, _ = ctx.serve_poll(r)
            if st == SERVE_DONE or st < 0:
                break
            time.sleep(0.0002)
        if st < 0:
            raise SystemExit(f"request failed: {st}")
        ctx.serve_release(r)
    t_cap = time.perf_counter() - t0
    capacity = tot / GiB / t_cap

    # 2. open loop: Poisson arrivals at 80% of capacity
    mean_len = float(lens.mean())
    rate = 0.8 * capacity * GiB / mean_len  # requests per second
    arr = np.cumsum(rng.exponential(1.0 / rate, size=count))
    n_req = int(np.searchsorted(arr, args.serve_seconds))
    n_req = max(1, min(n_req, count))
    lat, last_done, failed = [], [0.0], []
    nonlocal_done = [0]
    pending = {}
    lock = threading.Lock()
    stop = threading.Event()

    def poller():
        while not (stop.is_set() and not pending):
            with lock:
                items = list(pending.items())
            finished = []
            for rid, n in items:
                st, ms = ctx.serve_poll(rid)
                if st < 0:
                    failed.append(st)
                if st == SERVE_DONE or st < 0:
                    finished.append((rid, n, ms))
            for rid, n, ms in finished:
                ctx.serve_release(rid)
                with lock:
                    del pending[rid]
                lat.append((n, ms))
                nonlocal_done[0] += n
                last_done[0] = time.perf_counter()
            if not finished:
                time.sleep(0.0002)

    th = threading.Thread(target=poller)
    with ClockSampler(local) as clocks:
        start = time.perf_counter()
        th.start()
        for i in range(n_req):
            wait = start + float(arr[i]) - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            rid = submit(i % count)
            with lock:
                pending[rid] = int(lens[i % count])
        stop.set()
        th.join()
    clock = clocks.summary()
    if failed:
        raise SystemExit(f"{len(failed)} serving requests failed (first code {failed[0]})")
    served_s = last_done[0] - start
    done_bytes = nonlocal_done[0]
    sustained = done_bytes / GiB / served_s
    sstats = ctx.serve_stats()
    lat_n = np.array([x[0] for x in lat])
    lat_a = np.array([x[1] for x in lat])

    # 3. plain per-request path: one dcx_build_sa per request.
    #    (a) device only: the request's slice already in HBM, device time;
    #    (b) as a server: the same Poisson arrivals handled one at a time, each
    #        request uploaded from pinned host memory then built; latency =
    #        arrival -> SA complete in HBM, wall clock.
    d_base = torch.from_numpy(base).to(f"cuda:{local}")
    d_text = torch.empty(int(lens.max()) + 16, dtype=torch.uint8, device=f"cuda:{local}")
    d_sa = torch.empty(int(lens.max()) + 16, dtype=torch.int32, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    ctx.build_sa_device(d_base.data_ptr() + int(offs[0]), int(lens[0]), d_sa.data_ptr(), dc=39, sa_width=32)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    plain_ms, plain_bytes, j = 0.0, 0, 0
    while j < k and plain_ms < args.loop_budget_s * 1000.0:
        e0.record(stream)
        ctx.build_sa_device(d_base.data_ptr() + int(offs[j]), int(lens[j]), d_sa.data_ptr(), dc=39, sa_width=32)
        e1.record(stream)
        torch.cuda.synchronize()
        plain_ms += e0.elapsed_time(e1)
        plain_bytes += int(lens[j])
        j += 1
    plain = plain_bytes / GiB / (plain_ms / 1000.0)
    del d_base
    # plain capacity as a server would see it: upload + build per request, wall clock
    cur = torch.cuda.current_stream()
    t0 = time.perf_counter()
    for i in range(j):
        n_i, o_i = int(lens[i]), int(offs[i])
        d_text[:n_i].copy_(h_base[o_i:o_i + n_i], non_blocking=True)
        cur.synchronize()
        ctx.build_sa_device(d_text.data_ptr(), n_i, d_sa.data_ptr(), dc=39, sa_width=32)
    plain_wall = plain_bytes / GiB / (time.perf_counter() - t0)
    p_lat, p_n, p_bytes = [], [], 0
    cur = torch.cuda.current_stream()
    start = time.perf_counter()
    for i in range(n_req):
        t_arr = start + float(arr[i])
        wait = t_arr - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        n_i, o_i = int(lens[i % count]), int(offs[i % count])
        d_text[:n_i].copy_(h_base[o_i:o_i + n_i], non_blocking=True)
        cur.synchronize()
        ctx.build_sa_device(d_text.data_ptr(), n_i, d_sa.data_ptr(), dc=39, sa_width=32)
        p_lat.append((time.perf_counter() - t_arr) * 1000.0)
        p_n.append(n_i)
        p_bytes += n_i
    p_end = time.perf_counter()
    p_lat = np.array(p_lat)
    p_n = np.array(p_n)
    torch.cuda.synchronize()
    del d_text, d_sa, stream

    small = 4 << 20

    def pct(a, sel):
        a = a[sel]
        if a.size == 0:
            return None
        return {"p50": round(float(np.percentile(a, 50)), 2), "p99": round(float(np.percentile(a, 99)), 2),
                "requests": int(a.size)}

    if rank == 0:
        line = {
            "metric": "served SA build GiB/s", "value": round(sustained, 4), "unit": "GiB/s", "n_gpus": world,
            "steps": n_req, "warmup": len(wids), "ms_per_step": round(served_s * 1000 / n_req, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (slices of a seeded 1 GiB order-3 Markov DNA text, 5% repeats)",
            "config": {"workload": "cfg5_serve", "lengths": "log-uniform 4 KiB-256 MiB", "dc": 39, "sa_width": 32,
                       "budget_gb": args.serve_budget_gb, "lanes": args.serve_lanes,
                       "express_priority": args.serve_express_priority,
                       "submission": "borrow (zero-copy from pinned host text)" if borrow
                       else "copy at submission (pinned arena)",
                       "arrivals": "Poisson at 80% of measured capacity",
                       "l2_flush": "batches up to 1 GiB of text, larger than L2",
                       "parallelism": "replicas" if world > 1 else "single-gpu"},
            "latency_ms": {"p50": round(float(np.percentile(lat_a, 50)), 2),
                           "p99": round(float(np.percentile(lat_a, 99)), 2),
                           "max": round(float(lat_a.max()), 2), "requests": int(lat_a.size),
                           "definition": "submit -> SA complete in HBM, including queueing and upload",
                           "requests_le_4MiB": pct(lat_a, lat_n <= small),
                           "requests_gt_4MiB": pct(lat_a, lat_n > small)},
            "offered": {"requests_per_s": round(rate, 2), "gib_per_s": round(0.8 * capacity, 4),
                        "seconds": round(served_s, 2), "bytes": int(done_bytes)},
            "capacity": {"value": round(capacity, 4), "unit": "GiB/s", "requests": k, "bytes": int(tot),
                         "seconds": round(t_cap, 3), "submit_seconds": round(t_sub, 3)},
            "plain": {"value": round(plain, 4), "unit": "GiB/s", "requests": j, "bytes": plain_bytes,
                      "call": "dcx_build_sa per request on the capacity run's requests, device pointers, "
                              "text resident, device time",
                      "wall_with_upload": round(plain_wall, 4),
                      "capacity_over_plain_wall": round(capacity / plain_wall, 3)},
            "plain_served": {"value": round(p_bytes / GiB / (p_end - start), 4), "unit": "GiB/s",
                             "latency_ms": {"p50": round(float(np.percentile(p_lat, 50)), 2),
                                           "p99": round(float(np.percentile(p_lat, 99)), 2),
                                           "max": round(float(p_lat.max()), 2),
                                           "requests_le_4MiB": pct(p_lat, p_n <= small),
                                           "requests_gt_4MiB": pct(p_lat, p_n > small)},
                             "requests": int(p_lat.size),
                             "call": "same arrivals, one request at a time: pinned H2D + dcx_build_sa, "
                                     "arrival -> SA in HBM, wall clock"},
            "serve_stats": sstats,
            "clocks": clock,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def _single_workload(args):
    """The single-text workload's parameters, generator arguments and name,
    with the size overrides of profiling captures applied."""
    from distributed_suffix_sorting_evaluation_b200 import workloads as W
    w = dict(W.WORKLOADS[args.workload])
    label = args.workload
    if args.text_mib:
        w["n"] = args.text_mib << 20
        label += f"@{args.text_mib}MiB"
    gen_kw = {}
    if args.base_kib and w["gen"] == "pangenome":
        gen_kw["base_len"] = args.base_kib << 10
        label += f",base{args.base_kib}KiB"
    return w, gen_kw, label


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--text-mib", type=int, default=0, help="override the text size (profiling captures)")
    ap.add_argument("--base-kib", type=int, default=0,
                    help="pangenome base length (a smaller text with the full-size copy count, for profiling captures)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-sample-mib", type=int, default=0,
                    help="text prefix the CPU baseline builds (0 = the whole text)")
    ap.add_argument("--ref-sample-mib", type=int, default=0,
                    help="text prefix the reference arm builds (0 = the whole text; cfg4/cfg5: 256 MiB)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lcp", action="store_true", help="also time the LCP array of the built SA")
    ap.add_argument("--bwt", action="store_true", help="also time the BWT of the built SA")
    ap.add_argument("--safile", action="store_true",
                    help="also time writing the built SA to a file and reading it back (dcx_write/read_sa_file)")
    ap.add_argument("--safile-dir", default="", help="directory of that file (default: the temp directory)")
    ap.add_argument("--gsa", action="store_true",
                    help="also time the generalized SA of the text cut into 1 MiB strings")
    ap.add_argument("--recursion-dc", type=int, default=0, help="difference cover of the recursion levels")
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="context option (dcx_set_option) for the single-text workloads")
    ap.add_argument("--batch-count", type=int, default=20000, help="texts of the batched workload")
    ap.add_argument("--batch-chunk-mib", type=int, default=2048, help="text staged on the device per batched call")
    ap.add_argument("--batch-autotune", action="store_true",
                    help="tune the DC and radix tile per size class (dcx_autotune_batch) before the batched timing")
    ap.add_argument("--batch-split", default="lpt", choices=["lpt", "replicas"],
                    help="how the batched workload is split over ranks under torchrun")
    ap.add_argument("--loop-budget-s", type=float, default=60.0, help="device time for the per-text loop leg")
    ap.add_argument("--split-text", action="store_true",
                    help="build ONE text over all ranks with the distributed sample sort (strong scaling)")
    ap.add_argument("--verify", action=argparse.BooleanOptionalAction, default=True,
                    help="check the SA (batched: three SAs per chunk) on the GPU after the timed region")
    ap.add_argument("--serve-requests", type=int, default=20000, help="request pool of the serving workload")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="open-loop arrival window")
    ap.add_argument("--serve-cap-gib", type=int, default=16, help="text of the closed-loop capacity run")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-lanes", type=int, default=1)
    ap.add_argument("--serve-copy", action="store_true", help="copy texts at submission instead of borrowing")
    ap.add_argument("--serve-express-priority", type=int, default=1)
    args = ap.parse_args()
    world, rank, local = _dist()
    if args.workload == "cfg5_serve":
        if args.impl == "reference":
            return run_reference_serve(args, world, rank)
        return run_serve(args, world, rank, local)
    if args.workload == "cfg4_batch":
        if args.impl == "reference":
            return run_reference_batch(args, world, rank)
        return run_batch(args, world, rank, local)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.split_text:
        return run_split(args, world, rank, local)
    return run_gpu(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
