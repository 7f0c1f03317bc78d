#!/usr/bin/env python
"""Benchmark of the B200 DCX suffix-array build.

Workload (one step = one suffix-array build of one text):
  cfg2_dc39_markov_dna_1GiB -- 1 GiB order-3 Markov DNA with 5% repeats, DC39 with
  char packing, 40-bit SA output (seeded synthetic; no public corpus).
Metric: SA build GiB/s of input text on 1 B200 (bit-exact output).

  value   text already in HBM, SA left in HBM (40-bit), device time by CUDA events
          recorded on the library's own stream around exactly K builds
  e2e     the same through the public C ABI with pinned host buffers: text H2D,
          build, 40-bit SA D2H inside the timed region
Inputs are larger than L2 (1 GiB vs 126 MB), so no flush is needed between steps.

--impl reference times the CPU reference implementation instead (libsais 2.10
built from the reference tree, OpenMP over all host threads) on a bounded prefix
sample of the same text.  N > 1: one process per GPU, each rank builds its own
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

GiB = float(1 << 30)
DEFAULT_WORKLOAD = "cfg2_dc39_markov_dna_1GiB"


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _traffic_per_launch(kernel: str):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return j.get(kernel)
    return None


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
    """libsais64_omp (reference tree sources) on a prefix sample of the text."""
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
    sample = min(text.size, args.ref_sample_mib << 20)
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
        "config": {"workload": args.workload, "text_bytes": int(w["n"]), "dc": w["dc"], "sa_width": w["sa_width"]},
        "cpu_baseline": {"value": round(value, 4), "unit": "GiB/s", "cores": threads, "kind": "reference",
                         "sample": f"libsais64_omp on the first {sample >> 20} MiB of the workload text, "
                                   f"{threads} threads"},
        "e2e": {"value": round(value, 4), "unit": "GiB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gpu(args, world, rank, local):
    import torch
    from distributed_suffix_sorting_evaluation_b200 import Context, workloads as W

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    w = dict(W.WORKLOADS[args.workload])
    if args.text_mib:
        w["n"] = args.text_mib << 20
    n = int(w["n"])
    dc, width = w["dc"], w["sa_width"]
    wb = width // 8
    host_text = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    getattr(W, w["gen"])(n, seed=w["seed"] + 1000 * rank, out=host_text.numpy())
    d_text = host_text.to(f"cuda:{local}")
    d_sa = torch.empty(n * wb, dtype=torch.uint8, device=f"cuda:{local}")
    host_sa = torch.empty(n * wb, dtype=torch.uint8, pin_memory=True)
    ctx = Context(local)
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
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = world * n / GiB / (ms_step / 1000.0)

    # end-to-end through the public call with host buffers
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    step_e2e()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(e2e_steps):
        step_e2e()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    e2e_stats = ctx.stats()
    if world > 1:
        t = torch.tensor([ms_e2e], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_value = world * n / GiB / (ms_e2e / e2e_steps / 1000.0)

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
            "data": "synthetic (seeded order-3 Markov DNA + 5% repeats; no public corpus)",
            "config": {"workload": args.workload if not args.text_mib else f"{args.workload}@{args.text_mib}MiB",
                       "text_bytes": n, "dc": dc, "packing": True, "sa_width": width,
                       "l2_flush": "inputs larger than L2 (1 GiB text)",
                       "parallelism": "replicas" if world > 1 else "single-gpu"},
            "e2e": {"value": round(e2e_value, 4), "unit": "GiB/s", "h2d_bytes_per_step": n,
                    "d2h_bytes_per_step": n * wb, "steps": e2e_steps,
                    "ms_h2d": round(e2e_stats["ms_h2d"], 2), "ms_build": round(e2e_stats["ms_total"], 2),
                    "ms_d2h": round(e2e_stats["ms_d2h"], 2)},
            "gpu_launches": int(launches),
            "roofline": {"kernel": "k_onesweep (8-bit LSD radix pass)", "bound": "hbm",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "bytes_per_launch": int(bytes_radix / max(passes, 1)),
                         "launches": int(passes),
                         "traffic": _traffic_per_launch("k_onesweep")},
            "build_stats": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in s_last.items()},
            "clocks": clock,
        }
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            sample = min(n, args.cpu_sample_mib << 20)
            v, dt = cpu_baseline(host_text.numpy(), sample, threads)
            line["cpu_baseline"] = {"value": round(v, 4), "unit": "GiB/s", "cores": threads, "kind": "reference",
                                    "sample": f"libsais64_omp on the first {sample >> 20} MiB of the same text "
                                              f"({dt:.2f} s), {threads} threads"}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--text-mib", type=int, default=0, help="override the text size (profiling captures)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-mib", type=int, default=256)
    ap.add_argument("--ref-sample-mib", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = _dist()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_gpu(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
