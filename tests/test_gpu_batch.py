"""Batched builds (many texts of uneven length in one call, segmented DCX levels):
every SA equals libsais's and the single-text build's."""
import numpy as np
import pytest

from conftest import random_text

pytestmark = pytest.mark.gpu


def _texts(seed, count, lo, hi, sigma=4):
    rng = np.random.default_rng(seed)
    lens = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    return [random_text(int(n), sigma, seed=seed * 1000 + i) for i, n in enumerate(lens)]


@pytest.mark.parametrize("dc", [0, 3, 7, 39])
def test_batch_mixed_sizes(ctx, oracle, dc):
    texts = _texts(1, 60, 1, 60_000)
    texts += [np.zeros(0, np.uint8), np.frombuffer(b"A", np.uint8), np.frombuffer(b"AB", np.uint8)]
    for t, sa in zip(texts, ctx.build_sa_batch(texts, dc=dc, sa_width=32)):
        assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64)), t.size


def test_batch_repetitive_mixed_recursion(ctx, oracle):
    """Texts needing no recursion, direct recursion and discarding in one level."""
    rng = np.random.default_rng(4)
    base = rng.integers(65, 69, 9_000).astype(np.uint8)
    texts = [
        random_text(30_000, 4, seed=1),                                   # distinct names
        np.full(20_000, 66, np.uint8),                                    # deep recursion
        np.tile(np.frombuffer(b"ACGTTGCAAC", np.uint8), 3_000),           # periodic
        np.concatenate([base, base, rng.integers(65, 69, 12_000).astype(np.uint8)]),  # copies
        random_text(5_000, 2, seed=9),
    ]
    for dc in (3, 39):
        for t, sa in zip(texts, ctx.build_sa_batch(texts, dc=dc, sa_width=64)):
            assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64))


@pytest.mark.parametrize("width", [32, 40, 64])
def test_batch_widths_and_alphabets(ctx, oracle, width):
    texts = [random_text(7_000, s, seed=s) for s in (1, 2, 20, 200)]
    t256 = random_text(9_000, 256, seed=3, offset=0)
    t256[:256] = np.arange(256, dtype=np.uint8)
    texts.append(t256)  # the round's alphabet has all 256 byte values
    for t, sa in zip(texts, ctx.build_sa_batch(texts, dc=39, sa_width=width)):
        assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64))


def test_batch_multiple_rounds(ctx, oracle):
    texts = _texts(7, 40, 500, 40_000)
    ctx.set_option("batch_round_cap", 100_000)
    try:
        got = ctx.build_sa_batch(texts, dc=0, sa_width=32)
    finally:
        ctx.set_option("batch_round_cap", 0)
    for t, sa in zip(texts, got):
        assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64))


def test_batch_equals_single(ctx):
    texts = _texts(11, 12, 3_000, 200_000)
    batch = ctx.build_sa_batch(texts, dc=39, sa_width=64)
    for t, sa in zip(texts, batch):
        assert np.array_equal(sa, ctx.build_sa(t, dc=39, sa_width=64))
