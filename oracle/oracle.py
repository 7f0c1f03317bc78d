"""ctypes loader for the CPU checkers.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The GPU product never imports it.

Two checkers are exposed:
  * ``dcx_sa``   -- the restatement of lightweight_dcx's PDCX (oracle/cpu_dcx.cpp),
                    which also reports level-0 names / unique flags;
  * ``libsais``  -- libsais 2.10 compiled from the reference tree's own sources
                    (oracle/_ref/libsais.so), the suffix array every build must equal.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CPU_LIB = os.path.join(HERE, "lib", "libcpudcx.so")
SAIS_LIB = os.path.join(HERE, "_ref", "libsais.so")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)


class _Trace(ctypes.Structure):
    _fields_ = [
        ("m", ctypes.c_uint64),
        ("last_rank", ctypes.c_uint64),
        ("sample_chars", ctypes.c_uint64),
        ("merge_chars", ctypes.c_uint64),
        ("recursion", ctypes.c_int),
        ("max_depth", ctypes.c_int),
        ("base_case", ctypes.c_int),
        ("reduction", ctypes.c_double),
        ("capacity", ctypes.c_uint64),
        ("names", _u64p),
        ("unique", _u8p),
    ]


@dataclass
class Trace:
    m: int
    last_rank: int
    sample_chars: int
    merge_chars: int
    recursion: int
    max_depth: int
    base_case: int
    reduction: float
    names: np.ndarray | None
    unique: np.ndarray | None


_cpu = None
_sais = None


def build() -> None:
    """Compile the checkers with oracle/Makefile (needs the reference tree only
    for libsais; a prebuilt oracle/_ref/libsais.so is kept as is)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load_cpu():
    global _cpu
    if _cpu is None:
        if not os.path.exists(CPU_LIB):
            build()
        lib = ctypes.CDLL(CPU_LIB)
        lib.cpu_dcx_sa.argtypes = [_u8p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_uint64, ctypes.c_uint32, _u64p,
                                   ctypes.POINTER(_Trace)]
        lib.cpu_dcx_sa.restype = ctypes.c_int
        lib.cpu_compress_alphabet.argtypes = [_u8p, ctypes.c_uint64, _u32p]
        lib.cpu_compress_alphabet.restype = ctypes.c_int
        lib.cpu_dcx_table.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u8p, _u32p, _u32p]
        lib.cpu_dcx_table.restype = ctypes.c_int
        lib.cpu_packing_for_sigma.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p]
        lib.cpu_slow_sa.argtypes = [_u8p, ctypes.c_uint64, _u64p]
        lib.cpu_dcx_threads.restype = ctypes.c_int
        _cpu = lib
    return _cpu


def _load_sais():
    global _sais
    if _sais is None:
        if not os.path.exists(SAIS_LIB):
            build()
        lib = ctypes.CDLL(SAIS_LIB)
        lib.libsais64.argtypes = [_u8p, _i64p, ctypes.c_int64, ctypes.c_int64, _i64p]
        lib.libsais64.restype = ctypes.c_int64
        lib.libsais64_omp.argtypes = [_u8p, _i64p, ctypes.c_int64, ctypes.c_int64, _i64p, ctypes.c_int64]
        lib.libsais64_omp.restype = ctypes.c_int64
        lib.libsais64_plcp.argtypes = [_u8p, _i64p, _i64p, ctypes.c_int64]
        lib.libsais64_plcp.restype = ctypes.c_int64
        lib.libsais64_lcp.argtypes = [_i64p, _i64p, _i64p, ctypes.c_int64]
        lib.libsais64_lcp.restype = ctypes.c_int64
        lib.libsais64_bwt.argtypes = [_u8p, _u8p, _i64p, ctypes.c_int64, ctypes.c_int64, _i64p]
        lib.libsais64_bwt.restype = ctypes.c_int64
        lib.libsais64_gsa.argtypes = [_u8p, _i64p, ctypes.c_int64, ctypes.c_int64, _i64p]
        lib.libsais64_gsa.restype = ctypes.c_int64
        lib.libsais64_plcp_gsa.argtypes = [_u8p, _i64p, _i64p, ctypes.c_int64]
        lib.libsais64_plcp_gsa.restype = ctypes.c_int64
        _sais = lib
    return _sais


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def dc_table(X: int):
    """(DC, IN_DC, NEXT_RANK, cmpDepthRanks[X][X][3]) generated in closed form."""
    lib = _load_cpu()
    D = ctypes.c_uint32()
    dc = np.zeros(32, np.uint32)
    in_dc = np.zeros(X, np.uint8)
    nr = np.zeros(X, np.uint32)
    cmp = np.zeros(X * X * 3, np.uint32)
    rc = lib.cpu_dcx_table(X, ctypes.byref(D), _ptr(dc, _u32p), _ptr(in_dc, _u8p), _ptr(nr, _u32p),
                           _ptr(cmp, _u32p))
    if rc != 0:
        raise ValueError(f"no difference cover for X={X}")
    return dc[: D.value].copy(), in_dc, nr, cmp.reshape(X, X, 3)


def compress_alphabet(text: np.ndarray):
    """Remap bytes to 1..sigma (cli.cpp:417-463). Returns (remapped, sigma); raises on sigma == 256."""
    lib = _load_cpu()
    t = np.ascontiguousarray(text, dtype=np.uint8).copy()
    sigma = ctypes.c_uint32()
    rc = lib.cpu_compress_alphabet(_ptr(t, _u8p), t.size, ctypes.byref(sigma))
    if rc != 0:
        raise ValueError("alphabet of 256 symbols: 0 is reserved for padding")
    return t, sigma.value


def packing_for_sigma(X: int, sigma: int):
    lib = _load_cpu()
    b, w = ctypes.c_uint32(), ctypes.c_uint32()
    lib.cpu_packing_for_sigma(X, sigma, ctypes.byref(b), ctypes.byref(w))
    return b.value, w.value


def dcx_sa(text: np.ndarray, X: int = 39, packing: bool = True, discarding_threshold: float = 0.7,
           base_case_threshold: int = 10000, remap: bool = True, want_trace: bool = False):
    """Suffix array by the PDCX restatement.  ``text`` is raw bytes; when ``remap``
    it is passed through compress_alphabet first, as the reference cli does."""
    lib = _load_cpu()
    t = np.ascontiguousarray(text, dtype=np.uint8)
    if remap:
        t, sigma = compress_alphabet(t)
    else:
        sigma = int(t.max()) if t.size else 0
    n = t.size
    sa = np.zeros(max(n, 1), np.uint64)
    tr = _Trace()
    names = unique = None
    if want_trace:
        cap = n + 64
        names = np.zeros(cap, np.uint64)
        unique = np.zeros(cap, np.uint8)
        tr.capacity = cap
        tr.names = _ptr(names, _u64p)
        tr.unique = _ptr(unique, _u8p)
    if n == 0:
        return (np.zeros(0, np.uint64), None) if want_trace else np.zeros(0, np.uint64)
    rc = lib.cpu_dcx_sa(_ptr(t, _u8p), n, X, int(packing), int(packing), discarding_threshold,
                        base_case_threshold, sigma, _ptr(sa, _u64p), ctypes.byref(tr))
    if rc != 0:
        raise ValueError(f"cpu_dcx_sa failed: {rc}")
    sa = sa[:n]
    if not want_trace:
        return sa
    m = tr.m
    trace = Trace(tr.m, tr.last_rank, tr.sample_chars, tr.merge_chars, tr.recursion, tr.max_depth,
                  tr.base_case, tr.reduction,
                  names[:m].copy() if m else None, unique[:m].copy() if m else None)
    return sa, trace


def libsais(text: np.ndarray, threads: int = 1) -> np.ndarray:
    """SA of ``text`` (bytes, any values) by libsais64 / libsais64_omp."""
    lib = _load_sais()
    t = np.ascontiguousarray(text, dtype=np.uint8)
    n = t.size
    if n == 0:
        return np.zeros(0, np.int64)
    sa = np.zeros(n, np.int64)
    if threads == 1:
        rc = lib.libsais64(_ptr(t, _u8p), _ptr(sa, _i64p), n, 0, None)
    else:
        rc = lib.libsais64_omp(_ptr(t, _u8p), _ptr(sa, _i64p), n, 0, None, threads)
    if rc != 0:
        raise RuntimeError(f"libsais failed: {rc}")
    return sa


def libsais_lcp(text: np.ndarray, sa: np.ndarray | None = None):
    """(PLCP, LCP) of ``text`` by libsais64_plcp / libsais64_lcp (SA from libsais
    unless given)."""
    lib = _load_sais()
    t = np.ascontiguousarray(text, dtype=np.uint8)
    n = t.size
    if n == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    s = libsais(t) if sa is None else np.ascontiguousarray(sa, dtype=np.int64)
    plcp = np.zeros(n, np.int64)
    lcp = np.zeros(n, np.int64)
    if lib.libsais64_plcp(_ptr(t, _u8p), _ptr(s, _i64p), _ptr(plcp, _i64p), n) != 0:
        raise RuntimeError("libsais64_plcp failed")
    if lib.libsais64_lcp(_ptr(plcp, _i64p), _ptr(s, _i64p), _ptr(lcp, _i64p), n) != 0:
        raise RuntimeError("libsais64_lcp failed")
    return plcp, lcp


def libsais_bwt(text: np.ndarray):
    """(U, primary index) of ``text`` by libsais64_bwt
    (libsais/include/libsais64.h:125-135): U is the BWT without the sentinel
    row, the primary index is where that row would stand."""
    lib = _load_sais()
    t = np.ascontiguousarray(text, dtype=np.uint8)
    n = t.size
    u = np.zeros(max(n, 1), np.uint8)
    a = np.zeros(max(n, 1), np.int64)
    p = lib.libsais64_bwt(_ptr(t if n else u, _u8p), _ptr(u, _u8p), _ptr(a, _i64p), n, 0, None)
    if p < 0:
        raise RuntimeError(f"libsais64_bwt failed: {p}")
    return u[:n].copy(), int(p)


def libsais_gsa(text: np.ndarray) -> np.ndarray:
    """Generalized SA of a string set (each string followed by a 0 byte) by
    libsais64_gsa (libsais/include/libsais64.h:63-72)."""
    lib = _load_sais()
    t = np.ascontiguousarray(text, dtype=np.uint8)
    n = t.size
    sa = np.zeros(max(n, 1), np.int64)
    rc = lib.libsais64_gsa(_ptr(t if n else np.zeros(1, np.uint8), _u8p), _ptr(sa, _i64p), n, 0, None)
    if rc != 0:
        raise RuntimeError(f"libsais64_gsa refused the set: {rc}")
    return sa[:n].copy()


def libsais_lcp_gsa(text: np.ndarray, gsa: np.ndarray | None = None):
    """(PLCP, LCP) of a string set and its generalized SA by libsais64_plcp_gsa
    / libsais64_lcp: separators are distinct symbols and never match."""
    lib = _load_sais()
    t = np.ascontiguousarray(text, dtype=np.uint8)
    n = t.size
    if n == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    g = libsais_gsa(t) if gsa is None else np.ascontiguousarray(gsa, dtype=np.int64)
    plcp = np.zeros(n, np.int64)
    lcp = np.zeros(n, np.int64)
    if lib.libsais64_plcp_gsa(_ptr(t, _u8p), _ptr(g, _i64p), _ptr(plcp, _i64p), n) != 0:
        raise RuntimeError("libsais64_plcp_gsa failed")
    if lib.libsais64_lcp(_ptr(plcp, _i64p), _ptr(g, _i64p), _ptr(lcp, _i64p), n) != 0:
        raise RuntimeError("libsais64_lcp failed")
    return plcp, lcp


def gsa_from_sa(text: np.ndarray) -> np.ndarray:
    """The same order restated from the plain SA of the set: runs of plain-SA
    neighbours whose LCP reaches through the suffix's separator, each sorted by
    position (the construction the GPU follows)."""
    t = np.ascontiguousarray(text, dtype=np.uint8)
    n = t.size
    if n <= 1:
        return np.zeros(n, np.int64)
    sa = libsais(t).astype(np.int64)
    _, lcp = libsais_lcp(t, sa)
    zpos = np.flatnonzero(t == 0)
    to_sep = zpos[np.searchsorted(zpos, np.arange(n))] - np.arange(n) + 1
    joins = np.zeros(n, bool)
    joins[1:] = lcp[1:] >= to_sep[sa[1:]]
    run = np.cumsum(~joins)  # run number of each plain-SA entry
    return sa[np.lexsort((sa, run))]


def bwt_from_sa(text: np.ndarray, sa: np.ndarray):
    """The same (U, primary index) restated from a suffix array: U[0] = T[n-1],
    then T[SA[k]-1] for every SA[k] != 0 in SA order; primary = 1 + the k with
    SA[k] = 0 (0 for the empty text)."""
    t = np.ascontiguousarray(text, dtype=np.uint8)
    n = t.size
    if n == 0:
        return np.zeros(0, np.uint8), 0
    s = np.asarray(sa, dtype=np.int64)
    z = int(np.flatnonzero(s == 0)[0])
    rest = s[s != 0]
    return np.concatenate([t[n - 1:], t[rest - 1]]).astype(np.uint8), z + 1


def slow_sa(text: np.ndarray) -> np.ndarray:
    lib = _load_cpu()
    t = np.ascontiguousarray(text, dtype=np.uint8)
    sa = np.zeros(max(t.size, 1), np.uint64)
    lib.cpu_slow_sa(_ptr(t, _u8p), t.size, _ptr(sa, _u64p))
    return sa[: t.size]


def threads() -> int:
    return int(_load_cpu().cpu_dcx_threads())
