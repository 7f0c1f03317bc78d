"""Bit-exact parity at the benchmark configurations' own sizes.

Every case builds the workload text the bench builds (same generator, same
seed), through the C ABI with host buffers, and compares the raw SA bytes with
libsais64_omp built from the reference tree (oracle/_ref/libsais.so), entry by
entry, with no tolerance:

  cfg1   64 MiB i.i.d. {A,C,G,T}, DC3, uint64 SA                (full size)
  cfg2   1 GiB order-3 Markov DNA + 5% repeats, DC39, uint40 SA (full size)
  cfg3a  256 MiB of the pangenome generator ('$'-joined mutated copies), DC39, uint40
  cfg3b  256 MiB of the Zipf(1.1) byte generator (all 256 values), DC39, uint40
  cfg4   200 texts drawn from the batched workload's length distribution
         (log-uniform 1 KiB-16 MiB), one batched call, uint32 SAs

libsais needs 8 bytes of host memory per character for its int64 SA; the 1 GiB
case holds about 20 GiB of host memory at its peak.
"""
import os

import numpy as np
import pytest

from distributed_suffix_sorting_evaluation_b200 import workloads as W

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _as_width(sa64: np.ndarray, width: int) -> np.ndarray:
    """libsais's int64 SA as the raw little-endian bytes of `width` bits per entry."""
    b = sa64.astype(np.int64, copy=False).view(np.uint8).reshape(-1, 8)
    return b[:, : width // 8]


def _compare(ctx, oracle, text: np.ndarray, dc: int, width: int):
    raw = ctx.build_sa_raw(text, dc=dc, sa_width=width)
    ref = oracle.libsais(text, threads=THREADS)
    got = raw.reshape(-1, width // 8)
    want = _as_width(ref, width)
    assert got.shape == want.shape
    if not np.array_equal(got, want):
        bad = np.flatnonzero((got != want).any(axis=1))
        pytest.fail(f"n={text.size} DC{dc}: {bad.size} entries differ, first at {bad[:5]}")
    st = ctx.stats()
    return st


def test_cfg1_iid_dna_64MiB_dc3_uint64(ctx, oracle):
    text = W.make("cfg1_dc3_iid_dna_64MiB")
    assert text.size == 64 << 20
    _compare(ctx, oracle, text, 3, 64)


def test_cfg2_markov_dna_1GiB_dc39_uint40(ctx, oracle):
    text = W.make("cfg2_dc39_markov_dna_1GiB")
    assert text.size == 1 << 30
    st = _compare(ctx, oracle, text, 39, 40)
    assert st["sigma"] == 4


def test_cfg3a_pangenome_256MiB_dc39_uint40(ctx, oracle):
    text = W.pangenome(256 << 20, seed=3)
    assert (text == ord("$")).any()
    st = _compare(ctx, oracle, text, 39, 40)
    assert st["levels"] >= 2  # the copies force recursion


def test_cfg3b_zipf256_256MiB_dc39_uint40(ctx, oracle):
    text = W.zipf256(256 << 20, seed=4)
    assert np.unique(text).size == 256  # the alphabet the reference cli refuses
    _compare(ctx, oracle, text, 39, 40)


def test_cfg4_batch_200_texts(ctx, oracle):
    lens = W.batch_lengths(200, 1 << 10, 16 << 20, seed=5)
    texts = [W.iid(int(n), b"ACGT", seed=1_000_000 + j) for j, n in enumerate(lens)]
    got = ctx.build_sa_batch(texts, dc=0, sa_width=32)
    assert len(got) == len(texts)
    for j, (t, sa) in enumerate(zip(texts, got)):
        ref = oracle.libsais(t, threads=THREADS)
        assert np.array_equal(sa, ref.astype(np.uint64)), f"text {j} (n={t.size}) differs"
