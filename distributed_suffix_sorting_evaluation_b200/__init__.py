"""B200 DCX suffix-array builder: Python mirror of the reference's construction path.

The reference (lightweight_dcx) builds a suffix array through
``PDCX<char, index, DC>::compute_sa(std::vector<char>&) -> std::vector<index>``
(lightweight_dcx/src/pdcx/pdcx.hpp:529), configured by ``PDCXConfig``
(pdcx/config.hpp:27-60) and selected by the cli's ``--dcx`` flag
(executables/cli.cpp:598-653).  This module exposes the same operation over the
C ABI of ``lib/libdcxgpu.so`` (include/dcx_gpu.h):

    from distributed_suffix_sorting_evaluation_b200 import PDCX, PDCXConfig
    sa = PDCX(PDCXConfig(dc=39)).compute_sa(text_bytes)          # numpy uint64

Errors are raised as ``DcxError`` carrying the C status code (the reference
exits the process instead; the library never does).  There is no CPU fallback:
without the compiled library or a GPU every call raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libdcxgpu.so")

DCX_OK = 0
DCX_ERR_ARG = -1
DCX_ERR_ALPHABET = -2
DCX_ERR_OOM = -3
DCX_ERR_BUDGET = -4
DCX_ERR_TIMEOUT = -5
DCX_ERR_CUDA = -6
DCX_ERR_INTERNAL = -7
DCX_ERR_BUSY = -8
DCX_ERR_NOTFOUND = -9
DCX_ERR_IO = -10

DCX_HOST_PTRS = 0
DCX_DEVICE_PTRS = 1
DCX_NO_PACKING = 2
DCX_NO_REMAP = 4
DCX_SERVE_BORROW = 8
DCX_LCP_PERMUTED = 16
DCX_LCP_GSA = 32

SUPPORTED_DC = (3, 7, 13, 21, 31, 39, 57, 73, 91, 95, 133)

# Every exported symbol of include/dcx_gpu.h (checked by the CPU test suite).
EXPORTED = (
    "dcx_ctx_create", "dcx_ctx_destroy", "dcx_set_option", "dcx_build_sa", "dcx_build_sa_strict",
    "dcx_get_stream", "dcx_get_stats", "dcx_get_trace", "dcx_build_sa_batch", "dcx_serve_submit", "dcx_serve_poll",
    "dcx_serve_release", "dcx_serve_drain", "dcx_strerror", "dcx_dc_table", "dcx_version",
    "dcx_build_sa_noalloc", "dcx_check_sa", "dcx_serve_result_device", "dcx_serve_get_stats",
    "dcx_serve_submit_ex", "dcx_build_lcp", "dcx_shard_texts", "dcx_build_bwt",
    "dcx_build_gsa", "dcx_set_batch_dc_table", "dcx_get_batch_dc_table", "dcx_get_batch_tile_table", "dcx_autotune_batch",
    "dcx_write_sa_file", "dcx_read_sa_file", "dcx_check_sa_file", "dcx_bwt", "dcx_sort_u32", "dcx_build_sa_u32",
)

# serving request states (dcx_serve_poll)
SERVE_QUEUED, SERVE_RUNNING, SERVE_DONE = 0, 1, 2


class DcxError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"dcx error {code}: {what}")


class DcxStats(ctypes.Structure):
    _fields_ = [
        ("ms_total", ctypes.c_double), ("ms_phase0", ctypes.c_double), ("ms_phase12", ctypes.c_double),
        ("ms_phase3", ctypes.c_double), ("ms_phase4", ctypes.c_double), ("ms_h2d", ctypes.c_double),
        ("ms_d2h", ctypes.c_double), ("bytes_alg", ctypes.c_uint64), ("bytes_radix", ctypes.c_uint64),
        ("ms_radix", ctypes.c_double), ("radix_passes", ctypes.c_uint64), ("radix_keys", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint64), ("peak_bytes", ctypes.c_uint64), ("levels", ctypes.c_uint32),
        ("sigma", ctypes.c_uint32), ("level0_samples", ctypes.c_uint64), ("level0_last_rank", ctypes.c_uint64),
        ("level0_recursion", ctypes.c_int), ("level0_reduction", ctypes.c_double),
        ("tie_groups", ctypes.c_uint64), ("tie_elements", ctypes.c_uint64),
        ("lookback_gave_up", ctypes.c_uint64), ("pool_growth_bytes", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeStats(ctypes.Structure):
    _fields_ = [
        ("lanes", ctypes.c_uint32), ("budget_bytes", ctypes.c_uint64), ("reserved_bytes", ctypes.c_uint64),
        ("peak_reserved_bytes", ctypes.c_uint64), ("peak_lane_bytes", ctypes.c_uint64),
        ("submitted", ctypes.c_uint64), ("done", ctypes.c_uint64), ("failed", ctypes.c_uint64),
        ("done_bytes", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("max_batch_texts", ctypes.c_uint64),
        ("queued", ctypes.c_uint64), ("running_batches", ctypes.c_uint32),
        ("ms_upload", ctypes.c_double), ("ms_build", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load_library(path: str | None = None):
    """Loads lib/libdcxgpu.so (building it first when absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        from . import build as _b
        _b.build()
    lib = ctypes.CDLL(p)
    vp, u64, u32, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int
    lib.dcx_ctx_create.argtypes = [ctypes.POINTER(vp), i32, u64]
    lib.dcx_ctx_destroy.argtypes = [vp]
    lib.dcx_set_option.argtypes = [vp, ctypes.c_char_p, ctypes.c_double]
    lib.dcx_build_sa.argtypes = [vp, vp, u64, i32, i32, vp, u32]
    lib.dcx_build_sa_strict.argtypes = [vp, vp, u64, i32, i32, vp, u32]
    lib.dcx_get_stats.argtypes = [vp, ctypes.POINTER(DcxStats)]
    lib.dcx_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.dcx_get_trace.argtypes = [vp, ctypes.POINTER(u64), vp, vp, u64]
    lib.dcx_build_sa_batch.argtypes = [vp, vp, vp, u32, i32, i32, vp, u32]
    lib.dcx_serve_submit.argtypes = [vp, vp, u64, i32, i32, ctypes.POINTER(u64)]
    lib.dcx_serve_submit_ex.argtypes = [vp, vp, u64, i32, i32, u32, ctypes.POINTER(u64)]
    lib.dcx_serve_poll.argtypes = [vp, u64, vp, ctypes.POINTER(i32), ctypes.POINTER(ctypes.c_double)]
    lib.dcx_serve_release.argtypes = [vp, u64]
    lib.dcx_serve_drain.argtypes = [vp]
    lib.dcx_serve_result_device.argtypes = [vp, u64, ctypes.POINTER(vp)]
    lib.dcx_serve_get_stats.argtypes = [vp, ctypes.POINTER(ServeStats)]
    lib.dcx_strerror.argtypes = [i32]
    lib.dcx_strerror.restype = ctypes.c_char_p
    lib.dcx_dc_table.argtypes = [i32, vp, vp, vp, vp]
    lib.dcx_version.restype = ctypes.c_char_p
    lib.dcx_build_sa_noalloc.argtypes = [vp, u64, vp, vp]
    lib.dcx_build_lcp.argtypes = [vp, vp, u64, vp, i32, vp, i32, u32]
    lib.dcx_check_sa.argtypes = [vp, vp, u64, vp, i32, u32, ctypes.POINTER(i32)]
    lib.dcx_shard_texts.argtypes = [vp, u32, u32, vp, vp]
    lib.dcx_build_bwt.argtypes = [vp, vp, u64, vp, i32, vp, ctypes.POINTER(u64), u32]
    lib.dcx_bwt.argtypes = [vp, vp, vp, u64, i32, ctypes.POINTER(u64), u32]
    lib.dcx_build_gsa.argtypes = [vp, vp, u64, i32, i32, vp, u32]
    lib.dcx_set_batch_dc_table.argtypes = [vp, vp, vp, u32]
    lib.dcx_get_batch_dc_table.argtypes = [vp, vp, vp, u32, ctypes.POINTER(u32)]
    lib.dcx_get_batch_tile_table.argtypes = [vp, vp, u32, ctypes.POINTER(u32)]
    lib.dcx_autotune_batch.argtypes = [vp, vp, vp, u32, vp, u32, vp, u32, u32, vp, vp]
    lib.dcx_write_sa_file.argtypes = [vp, ctypes.c_char_p, vp, u64, i32, u64]
    lib.dcx_read_sa_file.argtypes = [vp, ctypes.c_char_p, vp, u64, i32, u64]
    lib.dcx_check_sa_file.argtypes = [vp, vp, u64, ctypes.c_char_p, i32, u32, ctypes.POINTER(i32)]
    lib.dcx_sort_u32.argtypes = [vp, vp, u32, vp, u64]
    lib.dcx_build_sa_u32.argtypes = [vp, vp, u64, u64, i32, i32, vp]
    _lib = lib
    return lib


def _check(rc: int):
    if rc != DCX_OK:
        raise DcxError(rc, load_library().dcx_strerror(rc).decode())


def dc_table(X: int):
    """(DC, NEXT_RANK, cmpDepthRanks[X][X][3]) from the library (host-only call)."""
    lib = load_library()
    D = ctypes.c_uint32()
    dc = np.zeros(32, np.uint32)
    nr = np.zeros(X, np.uint32)
    cmp = np.zeros(X * X * 3, np.uint32)
    _check(lib.dcx_dc_table(X, ctypes.byref(D), dc.ctypes.data, nr.ctypes.data, cmp.ctypes.data))
    return dc[: D.value].copy(), nr, cmp.reshape(X, X, 3)


def shard_texts(lengths, world: int):
    """Size-balanced split of independent texts over `world` ranks, longest
    first (host-only call): (owner[i] = rank of text i, bytes per rank).  Every
    rank computes the same split from the same lengths."""
    lens = np.ascontiguousarray(lengths, dtype=np.uint64)
    if lens.size >= 1 << 32:
        raise ValueError("at most 2^32 - 1 texts")
    owner = np.zeros(lens.size, np.uint32)
    loads = np.zeros(max(int(world), 0), np.uint64)
    _check(load_library().dcx_shard_texts(lens.ctypes.data, lens.size, int(world), owner.ctypes.data,
                                          loads.ctypes.data if loads.size else None))
    return owner, loads


def sa_dtype_bytes(width: int) -> int:
    return {32: 4, 40: 5, 64: 8}[width]


def unpack_sa(raw: np.ndarray, width: int, n: int) -> np.ndarray:
    """Raw SA bytes of the given width -> uint64 array."""
    if width == 32:
        return raw.view(np.uint32)[:n].astype(np.uint64)
    if width == 64:
        return raw.view(np.uint64)[:n].copy()
    b = raw.view(np.uint8)[: 5 * n].reshape(n, 5).astype(np.uint64)
    return b[:, 0] | (b[:, 1] << 8) | (b[:, 2] << 16) | (b[:, 3] << 24) | (b[:, 4] << 32)


class Context:
    """One device context (streams, memory pool, look-back scratch, statistics)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        _check(self.lib.dcx_ctx_create(ctypes.byref(h), device, hbm_budget_bytes))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.dcx_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_option(self, name: str, value: float):
        _check(self.lib.dcx_set_option(self.h, name.encode(), float(value)))

    def build_sa_raw(self, text, dc: int = 39, sa_width: int = 40, packing: bool = True, strict: bool = False,
                     remap: bool = True) -> np.ndarray:
        """SA of host bytes; returns the raw little-endian bytes of sa_width bits per entry."""
        t = np.ascontiguousarray(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray))
                                 else np.asarray(text, dtype=np.uint8))
        n = t.size
        out = np.zeros(max(n, 1) * sa_dtype_bytes(sa_width), np.uint8)
        flags = DCX_HOST_PTRS | (0 if packing else DCX_NO_PACKING) | (0 if remap else DCX_NO_REMAP)
        fn = self.lib.dcx_build_sa_strict if strict else self.lib.dcx_build_sa
        _check(fn(self.h, t.ctypes.data if n else None, n, dc, sa_width, out.ctypes.data, flags))
        return out[: n * sa_dtype_bytes(sa_width)]

    def build_sa(self, text, dc: int = 39, sa_width: int = 64, **kw) -> np.ndarray:
        raw = self.build_sa_raw(text, dc=dc, sa_width=sa_width, **kw)
        n = raw.size // sa_dtype_bytes(sa_width)
        return unpack_sa(raw, sa_width, n)

    def build_sa_device(self, text_ptr: int, n: int, sa_ptr: int, dc: int = 39, sa_width: int = 32,
                        packing: bool = True):
        """SA of a device-resident text into a device buffer (both raw CUDA pointers)."""
        flags = DCX_DEVICE_PTRS | (0 if packing else DCX_NO_PACKING)
        _check(self.lib.dcx_build_sa(self.h, ctypes.c_void_p(text_ptr), n, dc, sa_width, ctypes.c_void_p(sa_ptr),
                                     flags))

    def build_sa_batch(self, texts, dc: int = 0, sa_width: int = 32, packing: bool = True):
        """One SA per text (list of byte strings / uint8 arrays); dc = 0 lets the
        library choose.  Returns a list of uint64 arrays."""
        arrs = [np.frombuffer(t, np.uint8) if isinstance(t, (bytes, bytearray)) else np.asarray(t, np.uint8)
                for t in texts]
        offs = np.zeros(len(arrs) + 1, np.uint64)
        offs[1:] = np.cumsum([a.size for a in arrs], dtype=np.uint64)
        cat = np.ascontiguousarray(np.concatenate(arrs) if arrs else np.zeros(0, np.uint8))
        wb = sa_dtype_bytes(sa_width)
        out = np.zeros(max(int(offs[-1]), 1) * wb, np.uint8)
        flags = DCX_HOST_PTRS | (0 if packing else DCX_NO_PACKING)
        _check(self.lib.dcx_build_sa_batch(self.h, cat.ctypes.data if cat.size else out.ctypes.data,
                                           offs.ctypes.data, len(arrs), dc, sa_width, out.ctypes.data, flags))
        res = []
        for i, a in enumerate(arrs):
            b = int(offs[i])
            res.append(unpack_sa(out[b * wb:(b + a.size) * wb], sa_width, a.size))
        return res

    def build_sa_batch_raw(self, cat_ptr: int, offs_ptr: int, count: int, out_ptr: int, dc: int = 0,
                           sa_width: int = 32, device: bool = False):
        """Batch call on raw pointers (host or device per `device`)."""
        flags = DCX_DEVICE_PTRS if device else DCX_HOST_PTRS
        _check(self.lib.dcx_build_sa_batch(self.h, ctypes.c_void_p(cat_ptr), ctypes.c_void_p(offs_ptr), count, dc,
                                           sa_width, ctypes.c_void_p(out_ptr), flags))

    def check_sa(self, text, sa_raw: np.ndarray, sa_width: int) -> bool:
        """GPU check that sa_raw (raw bytes, sa_width bits per entry) is the SA of text."""
        t = np.ascontiguousarray(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray))
                                 else np.asarray(text, dtype=np.uint8))
        raw = np.ascontiguousarray(sa_raw).view(np.uint8)
        ok = ctypes.c_int()
        _check(self.lib.dcx_check_sa(self.h, t.ctypes.data if t.size else None, t.size,
                                     raw.ctypes.data if raw.size else None, sa_width, DCX_HOST_PTRS,
                                     ctypes.byref(ok)))
        return bool(ok.value)

    def build_lcp(self, text, sa: np.ndarray, permuted: bool = False, gsa: bool = False) -> np.ndarray:
        """LCP array (or PLCP) of a host text and its SA (any integer array); with
        gsa=True, of a 0-separated string set and its generalized SA."""
        t = np.ascontiguousarray(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray))
                                 else np.asarray(text, dtype=np.uint8))
        s = np.ascontiguousarray(np.asarray(sa).astype(np.uint64))
        out = np.zeros(max(t.size, 1), np.uint64)
        flags = DCX_HOST_PTRS | (DCX_LCP_PERMUTED if permuted else 0) | (DCX_LCP_GSA if gsa else 0)
        if t.size:
            _check(self.lib.dcx_build_lcp(self.h, t.ctypes.data, t.size, s.ctypes.data, 64, out.ctypes.data, 64,
                                          flags))
        return out[: t.size]

    def build_lcp_device(self, text_ptr: int, n: int, sa_ptr: int, sa_width: int, lcp_ptr: int,
                         lcp_width: int = 32, permuted: bool = False):
        flags = DCX_DEVICE_PTRS | (DCX_LCP_PERMUTED if permuted else 0)
        _check(self.lib.dcx_build_lcp(self.h, ctypes.c_void_p(text_ptr), n, ctypes.c_void_p(sa_ptr), sa_width,
                                      ctypes.c_void_p(lcp_ptr), lcp_width, flags))

    def set_batch_dc_table(self, table):
        """[(longest text of the class, X), ...] ascending; [] restores DC39."""
        ml = np.ascontiguousarray([int(a) for a, _ in table], dtype=np.uint64)
        dc = np.ascontiguousarray([int(b) for _, b in table], dtype=np.int32)
        _check(self.lib.dcx_set_batch_dc_table(self.h, ml.ctypes.data if ml.size else None,
                                               dc.ctypes.data if dc.size else None, len(table)))

    def batch_dc_table(self):
        cnt = ctypes.c_uint32()
        _check(self.lib.dcx_get_batch_dc_table(self.h, None, None, 0, ctypes.byref(cnt)))
        ml = np.zeros(max(cnt.value, 1), np.uint64)
        dc = np.zeros(max(cnt.value, 1), np.int32)
        _check(self.lib.dcx_get_batch_dc_table(self.h, ml.ctypes.data, dc.ctypes.data, cnt.value, ctypes.byref(cnt)))
        return [(int(ml[i]), int(dc[i])) for i in range(cnt.value)]

    def batch_tile_table(self):
        """Radix tile (elements) of every class of the batch DC table."""
        cnt = ctypes.c_uint32()
        _check(self.lib.dcx_get_batch_tile_table(self.h, None, 0, ctypes.byref(cnt)))
        t = np.zeros(max(cnt.value, 1), np.uint32)
        _check(self.lib.dcx_get_batch_tile_table(self.h, t.ctypes.data, cnt.value, ctypes.byref(cnt)))
        return [int(t[i]) for i in range(cnt.value)]

    def autotune_batch(self, texts, class_max_len, candidates=(3, 7, 13, 21, 39), repeats: int = 3):
        """Times each candidate DC on the sample texts of each size class and
        installs the fastest per class; returns (chosen DC per class, median ms
        [class][candidate])."""
        ts = [np.ascontiguousarray(np.frombuffer(t, np.uint8) if isinstance(t, (bytes, bytearray))
                                   else np.asarray(t, dtype=np.uint8)) for t in texts]
        offs = np.zeros(len(ts) + 1, np.uint64)
        offs[1:] = np.cumsum([t.size for t in ts], dtype=np.uint64)
        cat = np.concatenate(ts) if ts else np.zeros(0, np.uint8)
        cat = np.ascontiguousarray(cat if cat.size else np.zeros(1, np.uint8))
        cm = np.ascontiguousarray(class_max_len, dtype=np.uint64)
        cd = np.ascontiguousarray(candidates, dtype=np.int32)
        chosen = np.zeros(cm.size, np.int32)
        ms = np.zeros(cm.size * cd.size, np.float64)
        _check(self.lib.dcx_autotune_batch(self.h, cat.ctypes.data, offs.ctypes.data, len(ts), cm.ctypes.data,
                                           cm.size, cd.ctypes.data, cd.size, repeats, chosen.ctypes.data,
                                           ms.ctypes.data))
        return chosen.tolist(), ms.reshape(cm.size, cd.size)

    def build_gsa(self, text, dc: int = 39, sa_width: int = 64) -> np.ndarray:
        """Generalized SA (uint64) of a string set given as a host byte array:
        each string followed by a 0 byte, as libsais64_gsa takes it."""
        t = np.ascontiguousarray(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray))
                                 else np.asarray(text, dtype=np.uint8))
        raw = np.zeros(max(t.size, 1) * sa_dtype_bytes(sa_width), np.uint8)
        _check(self.lib.dcx_build_gsa(self.h, t.ctypes.data if t.size else None, t.size, dc, sa_width,
                                      raw.ctypes.data, DCX_HOST_PTRS))
        return unpack_sa(raw, sa_width, t.size)

    def build_gsa_device(self, text_ptr: int, n: int, sa_ptr: int, dc: int = 39, sa_width: int = 32):
        _check(self.lib.dcx_build_gsa(self.h, ctypes.c_void_p(text_ptr), n, dc, sa_width, ctypes.c_void_p(sa_ptr),
                                      DCX_DEVICE_PTRS))

    def build_bwt(self, text, sa: np.ndarray):
        """(BWT without the sentinel row, primary index) of a host text and its SA
        (any integer array), as libsais64_bwt returns them."""
        t = np.ascontiguousarray(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray))
                                 else np.asarray(text, dtype=np.uint8))
        s = np.ascontiguousarray(np.asarray(sa).astype(np.uint64))
        out = np.zeros(max(t.size, 1), np.uint8)
        primary = ctypes.c_uint64()
        _check(self.lib.dcx_build_bwt(self.h, t.ctypes.data if t.size else None, t.size,
                                      s.ctypes.data if s.size else None, 64, out.ctypes.data,
                                      ctypes.byref(primary), DCX_HOST_PTRS))
        return out[: t.size], int(primary.value)

    def bwt(self, text, dc: int = 39):
        """(BWT, primary index) of a host text, SA built on the GPU: libsais64_bwt's result."""
        t = np.ascontiguousarray(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray))
                                 else np.asarray(text, dtype=np.uint8))
        out = np.zeros(max(t.size, 1), np.uint8)
        primary = ctypes.c_uint64()
        _check(self.lib.dcx_bwt(self.h, t.ctypes.data if t.size else None, out.ctypes.data, t.size, dc,
                                ctypes.byref(primary), DCX_HOST_PTRS))
        return out[: t.size], int(primary.value)

    def build_bwt_device(self, text_ptr: int, n: int, sa_ptr: int, sa_width: int, bwt_ptr: int) -> int:
        """BWT of a device-resident text and SA into device memory; returns the primary index."""
        primary = ctypes.c_uint64()
        _check(self.lib.dcx_build_bwt(self.h, ctypes.c_void_p(text_ptr), n, ctypes.c_void_p(sa_ptr), sa_width,
                                      ctypes.c_void_p(bwt_ptr), ctypes.byref(primary), DCX_DEVICE_PTRS))
        return int(primary.value)

    def write_sa_file(self, path: str, sa_ptr: int, n: int, sa_width: int, chunk_bytes: int = 0):
        """Device-resident SA -> file in the reference's raw layout (streamed)."""
        _check(self.lib.dcx_write_sa_file(self.h, os.fsencode(path), ctypes.c_void_p(sa_ptr), n, sa_width,
                                          chunk_bytes))

    def read_sa_file(self, path: str, sa_ptr: int, n: int, sa_width: int, chunk_bytes: int = 0):
        """SA file in the reference's raw layout -> device memory (streamed)."""
        _check(self.lib.dcx_read_sa_file(self.h, os.fsencode(path), ctypes.c_void_p(sa_ptr), n, sa_width,
                                         chunk_bytes))

    def check_sa_file(self, text, path: str, sa_width: int) -> bool:
        """GPU check of the SA stored in `path` against a host text."""
        t = np.ascontiguousarray(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray))
                                 else np.asarray(text, dtype=np.uint8))
        ok = ctypes.c_int()
        _check(self.lib.dcx_check_sa_file(self.h, t.ctypes.data if t.size else None, t.size, os.fsencode(path),
                                          sa_width, DCX_HOST_PTRS, ctypes.byref(ok)))
        return bool(ok.value)

    def check_sa_device(self, text_ptr: int, n: int, sa_ptr: int, sa_width: int) -> bool:
        """GPU check of a device-resident SA against a device-resident text."""
        ok = ctypes.c_int()
        _check(self.lib.dcx_check_sa(self.h, ctypes.c_void_p(text_ptr), n, ctypes.c_void_p(sa_ptr), sa_width,
                                     DCX_DEVICE_PTRS, ctypes.byref(ok)))
        return bool(ok.value)

    def sort_u32_device(self, key_ptrs, val_ptr: int, n: int):
        """Stable in-place sort of n (key words, value) pairs in device memory,
        key_ptrs[-1] the most significant uint32 word (1 to 3 words)."""
        arr = (ctypes.c_void_p * len(key_ptrs))(*[ctypes.c_void_p(p) for p in key_ptrs])
        _check(self.lib.dcx_sort_u32(self.h, arr, len(key_ptrs), ctypes.c_void_p(val_ptr), n))

    def build_sa_u32_device(self, text_ptr: int, n: int, sigma: int, sa_ptr: int, dc: int = 3, sa_width: int = 32):
        """SA of a device string of n uint32 symbols in [1, sigma] into a device buffer."""
        _check(self.lib.dcx_build_sa_u32(self.h, ctypes.c_void_p(text_ptr), n, sigma, dc, sa_width,
                                         ctypes.c_void_p(sa_ptr)))

    def stream_handle(self) -> int:
        """cudaStream_t of this context as an integer (for torch.cuda.ExternalStream)."""
        p = ctypes.c_void_p()
        _check(self.lib.dcx_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def build_sa_hostptr(self, text_ptr: int, n: int, sa_ptr: int, dc: int = 39, sa_width: int = 40,
                         packing: bool = True):
        """SA of a text in (pinned) host memory into host memory: the end-to-end call."""
        flags = DCX_HOST_PTRS | (0 if packing else DCX_NO_PACKING)
        _check(self.lib.dcx_build_sa(self.h, ctypes.c_void_p(text_ptr), n, dc, sa_width, ctypes.c_void_p(sa_ptr),
                                     flags))

    def stats(self) -> dict:
        s = DcxStats()
        _check(self.lib.dcx_get_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    # ---- serving -------------------------------------------------------------
    def serve_submit(self, text, dc: int = 0, sa_width: int = 32, text_ptr: int | None = None,
                     n: int | None = None, borrow: bool = False, device: bool = False) -> int:
        """Queues an SA request; returns its id.  Pass either `text` (bytes /
        uint8 array; copied) or a raw pointer and length.  borrow=True skips the
        copy: the buffer must stay valid until the request is done; device=True
        (with borrow) means a device pointer."""
        if text_ptr is None:
            if borrow:
                raise ValueError("borrow needs a raw pointer whose lifetime the caller controls")
            t = np.ascontiguousarray(np.frombuffer(text, np.uint8) if isinstance(text, (bytes, bytearray))
                                     else np.asarray(text, dtype=np.uint8))
            text_ptr, n = (t.ctypes.data if t.size else None), t.size
        flags = (DCX_SERVE_BORROW if borrow else 0) | (DCX_DEVICE_PTRS if device else 0)
        rid = ctypes.c_uint64()
        _check(self.lib.dcx_serve_submit_ex(self.h, ctypes.c_void_p(text_ptr) if text_ptr else None, n, dc,
                                            sa_width, flags, ctypes.byref(rid)))
        return rid.value

    def serve_poll(self, rid: int, out: np.ndarray | None = None):
        """(status, latency_ms); when done and `out` (uint8, n * sa_width/8 bytes)
        is given, the SA is copied into it."""
        st = ctypes.c_int()
        lat = ctypes.c_double()
        _check(self.lib.dcx_serve_poll(self.h, rid, out.ctypes.data if out is not None and out.size else None,
                                       ctypes.byref(st), ctypes.byref(lat)))
        return st.value, lat.value

    def serve_result_device(self, rid: int) -> int:
        p = ctypes.c_void_p()
        _check(self.lib.dcx_serve_result_device(self.h, rid, ctypes.byref(p)))
        return p.value or 0

    def serve_release(self, rid: int):
        _check(self.lib.dcx_serve_release(self.h, rid))

    def serve_drain(self):
        _check(self.lib.dcx_serve_drain(self.h))

    def serve_stats(self) -> dict:
        s = ServeStats()
        _check(self.lib.dcx_serve_get_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    def serve_result(self, rid: int, n: int, sa_width: int = 32) -> np.ndarray:
        """Waits for request `rid` (n chars) and returns its SA as uint64."""
        import time
        out = np.zeros(max(n, 1) * sa_dtype_bytes(sa_width), np.uint8)
        while True:
            st, _ = self.serve_poll(rid, out)
            if st == SERVE_DONE:
                return unpack_sa(out, sa_width, n)
            if st < 0:
                raise DcxError(st, "serving request failed")
            time.sleep(0.0005)

    def trace(self):
        """Level-0 names and unique flags of the last build with option trace=1."""
        m = ctypes.c_uint64()
        _check(self.lib.dcx_get_trace(self.h, ctypes.byref(m), None, None, 0))
        names = np.zeros(max(m.value, 1), np.uint32)
        uniq = np.zeros(max(m.value, 1), np.uint8)
        _check(self.lib.dcx_get_trace(self.h, ctypes.byref(m), names.ctypes.data, uniq.ctypes.data, names.size))
        return names[: m.value], uniq[: m.value]


@dataclass
class PDCXConfig:
    """The fields of the reference's PDCXConfig that change the GPU build's behaviour.
    Distribution/sorter knobs of the reference (atomic_sorter, buckets, splitters,
    chunks) have no meaning on one GPU; they are accepted by the cli and ignored."""
    dc: int = 39
    use_char_packing_samples: bool = True
    use_char_packing_merging: bool = True
    discarding_threshold: float = 0.7
    sa_width: int = 40
    device: int = 0
    recursion_dc: int = 3
    extra: dict = field(default_factory=dict)


class PDCX:
    """Mirror of PDCX<char_type, index_type, DC> for the construction call."""

    def __init__(self, config: PDCXConfig | None = None, context: Context | None = None):
        self.config = config or PDCXConfig()
        if self.config.dc not in SUPPORTED_DC:
            raise DcxError(DCX_ERR_ARG, f"unsupported DC X={self.config.dc}")
        self.ctx = context or Context(self.config.device)
        self.ctx.set_option("discarding_threshold", self.config.discarding_threshold)
        self.ctx.set_option("recursion_dc", self.config.recursion_dc)

    def compute_sa(self, local_string) -> np.ndarray:
        packing = self.config.use_char_packing_samples or self.config.use_char_packing_merging
        return self.ctx.build_sa(local_string, dc=self.config.dc, sa_width=64, packing=packing)

    def stats(self) -> dict:
        return self.ctx.stats()
