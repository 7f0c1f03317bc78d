"""Seeded synthetic inputs with the shapes, sizes and value distributions of the
benchmark configurations (no public corpus is named or used).

  iid_dna(n, seed)            config 1: i.i.d. uniform {A,C,G,T}
  markov_dna(n, seed)         config 2: order-3 Markov {A,C,G,T} (rows ~ Dirichlet(4),
                              about 1.87 bits per base), 5% of positions
                              covered by copies of earlier segments (log-uniform
                              1 KiB-100 KiB) with 1% substitutions
  pangenome(n, seed)          config 3a: copies of a 10 MiB i.i.d. base with 0.1%
                              substitutions and 0.01% indels (1-10), '$'-joined
  zipf256(n, seed)            config 3b: i.i.d. Zipf(1.1) over 256 byte values
  batch_lengths(count, ...)   config 4: log-uniform text lengths
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

_lib = None


def _gen():
    global _lib
    if _lib is None:
        p = os.path.join(_build.LIB, "libtextgen.so")
        if not os.path.exists(p):
            _build.build()
        lib = ctypes.CDLL(p)
        vp, u64, u32, dbl = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double
        lib.tg_iid.argtypes = [vp, u64, vp, u32, u64]
        lib.tg_markov.argtypes = [vp, u64, u64]
        lib.tg_repeats.argtypes = [vp, u64, dbl, u64, u64, dbl, u64]
        lib.tg_repeats.restype = u64
        lib.tg_pangenome.argtypes = [vp, u64, u64, dbl, dbl, u64]
        lib.tg_zipf.argtypes = [vp, u64, dbl, u64]
        lib.tg_loguniform_lengths.argtypes = [vp, u64, u64, u64, u64]
        lib.tg_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def _alloc(n, out=None):
    if out is None:
        out = np.empty(n, np.uint8)
    assert out.dtype == np.uint8 and out.flags.c_contiguous and out.size >= n
    return out


def iid(n: int, alphabet: bytes, seed: int = 1, out=None) -> np.ndarray:
    out = _alloc(n, out)
    a = np.frombuffer(alphabet, np.uint8).copy()
    _gen().tg_iid(out.ctypes.data, n, a.ctypes.data, a.size, seed)
    return out[:n]


def iid_dna(n: int, seed: int = 1, out=None) -> np.ndarray:
    return iid(n, b"ACGT", seed, out)


def markov_dna(n: int, seed: int = 2, repeat_frac: float = 0.05, out=None) -> np.ndarray:
    out = _alloc(n, out)
    lib = _gen()
    lib.tg_markov(out.ctypes.data, n, seed)
    if repeat_frac > 0:
        lib.tg_repeats(out.ctypes.data, n, repeat_frac, 1024, 100 * 1024, 0.01, seed)
    return out[:n]


def pangenome(n: int, seed: int = 3, base_len: int = 10 << 20, out=None) -> np.ndarray:
    out = _alloc(n, out)
    _gen().tg_pangenome(out.ctypes.data, n, min(base_len, max(n, 1)), 0.001, 0.0001, seed)
    return out[:n]


def zipf256(n: int, seed: int = 4, s: float = 1.1, out=None) -> np.ndarray:
    out = _alloc(n, out)
    _gen().tg_zipf(out.ctypes.data, n, s, seed)
    return out[:n]


def batch_lengths(count: int, lmin: int = 1 << 10, lmax: int = 16 << 20, seed: int = 5) -> np.ndarray:
    out = np.empty(count, np.uint64)
    _gen().tg_loguniform_lengths(out.ctypes.data, count, lmin, lmax, seed)
    return out


DESCRIPTIONS = {
    "cfg1_dc3_iid_dna_64MiB": "synthetic (seeded i.i.d. uniform {A,C,G,T})",
    "cfg2_dc39_markov_dna_1GiB": "synthetic (seeded order-3 Markov DNA + 5% repeats; no public corpus)",
    "cfg3a_dc39_pangenome_2GiB": "synthetic (200 mutated copies of a seeded 10 MiB {A,C,G,T} base, '$'-separated)",
    "cfg3b_dc39_zipf256_1GiB": "synthetic (seeded Zipf(s=1.1) over 256 byte values)",
}

WORKLOADS = {
    "cfg1_dc3_iid_dna_64MiB": dict(gen="iid_dna", n=64 << 20, dc=3, sa_width=64, seed=1),
    "cfg2_dc39_markov_dna_1GiB": dict(gen="markov_dna", n=1 << 30, dc=39, sa_width=40, seed=2),
    "cfg3a_dc39_pangenome_2GiB": dict(gen="pangenome", n=1 << 31, dc=39, sa_width=40, seed=3),
    "cfg3b_dc39_zipf256_1GiB": dict(gen="zipf256", n=1 << 30, dc=39, sa_width=40, seed=4),
}


def make(name: str, n: int | None = None, out=None) -> np.ndarray:
    w = WORKLOADS[name]
    fn = globals()[w["gen"]]
    return fn(n or w["n"], seed=w["seed"], out=out)
