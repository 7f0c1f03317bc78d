"""The LCP, BWT and generalized-SA kernels run on the CPU: their source
(csrc/lcp.cuh, bwt.cuh, gsa.cuh), unchanged, is compiled as host C++ through a
small shim of the CUDA builtins they use and launched sequentially
(tests/kernel_host/), then compared with libsais built from the reference tree
on random inputs, the reference's psac GSA test sets and the inputs the library
refuses.  This checks the kernels' index arithmetic and edge cases without a
GPU; the GPU suites check the same functions on the device."""
import ctypes
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import PSAC_GSA_CASES, flat_positions, psac_gsa_case, psac_glcp_case, set_bytes

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "distributed_suffix_sorting_evaluation_b200", "csrc")


@pytest.fixture(scope="module")
def kh(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    d = tmp_path_factory.mktemp("kernel_host")
    inc = d / "inc"
    inc.mkdir()
    for f in ("lcp.cuh", "bwt.cuh", "gsa.cuh"):
        shutil.copy(os.path.join(CSRC, f), inc / f)
    common = open(os.path.join(CSRC, "common.cuh")).read()
    m = re.search(r"__device__ __forceinline__ void store_sa_entry\(.*?\n}\n", common, re.S)
    assert m, "store_sa_entry not found in common.cuh"
    (inc / "common.cuh").write_text('#pragma once\n#include "cuda_shim.h"\nnamespace dcx {\n' + m.group(0) + "}\n")
    shutil.copy(os.path.join(HERE, "kernel_host", "cuda_shim.h"), inc / "cuda_shim.h")
    so = d / "libkernelhost.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(so),
                    os.path.join(HERE, "kernel_host", "harness.cpp"), f"-I{inc}"], check=True)
    lib = ctypes.CDLL(str(so))
    vp, u64 = ctypes.c_void_p, ctypes.c_uint64
    lib.kshim_bwt.argtypes = [vp, u64, vp, ctypes.c_int, vp, ctypes.POINTER(u64)]
    lib.kshim_gsa.argtypes = [vp, u64, vp, vp]
    lib.kshim_lcp.argtypes = [vp, u64, vp, ctypes.c_int, vp]
    lib.kshim_sa_to_u32.argtypes = [vp, ctypes.c_int, u64, vp]
    lib.kshim_store_sa.argtypes = [vp, u64, vp, ctypes.c_int]
    return lib


def _pack(sa, width):
    sa = np.asarray(sa, np.uint64)
    if width == 32:
        return sa.astype(np.uint32).view(np.uint8).copy()
    if width == 64:
        return sa.view(np.uint8).copy()
    b = np.zeros((sa.size, 5), np.uint8)
    for i in range(5):
        b[:, i] = (sa >> np.uint64(8 * i)) & np.uint64(255)
    return b.reshape(-1).copy()


def _bwt(lib, t, sa, width):
    out = np.zeros(max(t.size, 1), np.uint8)
    p = ctypes.c_uint64()
    raw = _pack(sa, width) if t.size else np.zeros(8, np.uint8)
    rc = lib.kshim_bwt(t.ctypes.data, t.size, raw.ctypes.data, width, out.ctypes.data, ctypes.byref(p))
    return rc, out[: t.size], p.value


def _gsa(lib, oracle, t):
    sa = oracle.libsais(t).astype(np.uint32) if t.size else np.zeros(1, np.uint32)
    out = np.zeros(max(t.size, 1), np.uint32)
    rc = lib.kshim_gsa(t.ctypes.data, t.size, sa.ctypes.data, out.ctypes.data)
    return rc, out[: t.size].astype(np.int64)


def _lcp(lib, t, sa, gsa):
    s = np.ascontiguousarray(np.asarray(sa, np.uint32))
    out = np.zeros(max(t.size, 1), np.uint32)
    rc = lib.kshim_lcp(t.ctypes.data, t.size, s.ctypes.data, int(gsa), out.ctypes.data)
    return rc, out[: t.size].astype(np.int64)


def _string_set(rng, k, sigma, base):
    parts = []
    for _ in range(k):
        m = rng.integers(0, 3)
        if m == 0:
            s = rng.integers(1, 1 + sigma, rng.integers(1, 60))
        elif m == 1:
            s = base[rng.integers(0, base.size):]
        else:
            s = base
        parts.append(np.concatenate([s, [0]]))
    return np.concatenate(parts).astype(np.uint8)


def test_bwt_kernels(kh, oracle):
    rng = np.random.default_rng(7)
    for trial in range(120):
        n = int(rng.integers(1, 3000))
        t = rng.integers(0, int(rng.integers(1, 256)) + 1, n).astype(np.uint8)
        if trial % 5 == 0:  # periodic: long repeats
            t = np.tile(t[: max(1, n // 7)], 8)[:n].copy()
        sa = oracle.libsais(t)
        want, p = oracle.libsais_bwt(t)
        for width in (32, 40, 64):
            rc, got, q = _bwt(kh, t, sa, width)
            assert rc == 0 and q == p and np.array_equal(got, want), (trial, width)
    t = rng.integers(65, 69, 500).astype(np.uint8)
    sa = oracle.libsais(t)
    bad = sa.copy()
    bad[3] = t.size
    assert _bwt(kh, t, bad, 64)[0] == -1
    bad = sa.copy()
    bad[bad == 1] = 0
    assert _bwt(kh, t, bad, 64)[0] == -1
    assert _bwt(kh, np.zeros(0, np.uint8), np.zeros(0, np.int64), 64)[2] == 0


def test_gsa_and_gsa_lcp_kernels(kh, oracle):
    rng = np.random.default_rng(8)
    for trial in range(150):
        base = rng.integers(1, 4 if trial % 2 else 255, rng.integers(1, 200))
        t = _string_set(rng, int(rng.integers(1, 60)), 3 if trial % 2 else 254, base)
        rc, got = _gsa(kh, oracle, t)
        want = oracle.libsais_gsa(t)
        assert rc == 0 and np.array_equal(got, want), trial
        rc, lcp = _lcp(kh, t, want, True)
        assert rc == 0 and np.array_equal(lcp, oracle.libsais_lcp_gsa(t, want)[1]), trial
    for seq, reps in PSAC_GSA_CASES:
        strings, expected = psac_gsa_case(seq, reps)
        t = set_bytes(strings)
        _, got = _gsa(kh, oracle, t)
        assert flat_positions(t, got) == expected
        _, lcp = _lcp(kh, t, got, True)
        assert lcp[t[got] != 0].tolist() == psac_glcp_case(seq, reps)
    for bad in (b"ab", b"a\0\0", b"\0a\0"):
        assert _gsa(kh, oracle, np.frombuffer(bad, np.uint8).copy())[0] == -1
    assert _gsa(kh, oracle, np.zeros(1, np.uint8))[1].tolist() == [0]


def test_plain_lcp_kernel(kh, oracle):
    rng = np.random.default_rng(9)
    for _ in range(60):
        t = rng.integers(0, 5, int(rng.integers(1, 4000))).astype(np.uint8)
        sa = oracle.libsais(t)
        rc, lcp = _lcp(kh, t, sa, False)
        assert rc == 0 and np.array_equal(lcp, oracle.libsais_lcp(t, sa)[1])


def test_sa_width_decode_kernel(kh):
    """k_sa_to_u32 (the LCP path's reader of 32/40/64-bit SAs; 40-bit entries
    four at a time from aligned words, the tail one by one)."""
    rng = np.random.default_rng(10)
    for n in (1, 2, 3, 4, 5, 7, 8, 9, 1000, 4097):
        sa = rng.permutation(n).astype(np.uint64) + np.uint64(rng.integers(0, 1 << 31))
        for width in (32, 40, 64):
            raw = _pack(sa, width)
            buf = np.zeros(raw.size + 8, np.uint8)  # 8-byte aligned base, as device buffers are
            buf[: raw.size] = raw
            out = np.zeros(n, np.uint32)
            kh.kshim_sa_to_u32(buf.ctypes.data, width, n, out.ctypes.data)
            assert np.array_equal(out, sa.astype(np.uint32)), (n, width)
            s32 = np.ascontiguousarray(sa.astype(np.uint32))
            back = np.zeros(raw.size, np.uint8)
            kh.kshim_store_sa(s32.ctypes.data, n, back.ctypes.data, width)
            assert back.tobytes() == raw.tobytes(), (n, width)
