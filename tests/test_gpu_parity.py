"""GPU suffix arrays through the C ABI, bit-exact against libsais (built from the
reference tree) and the PDCX restatement (level-0 names / unique flags)."""
import numpy as np
import pytest

from conftest import random_text

pytestmark = pytest.mark.gpu


def _check(ctx, oracle, t, X, packing=True, width=64):
    sa = ctx.build_sa(t, dc=X, sa_width=width, packing=packing)
    ref = oracle.libsais(t).astype(np.uint64)
    assert sa.shape == ref.shape
    bad = np.nonzero(sa != ref)[0]
    assert bad.size == 0, f"X={X} n={t.size} first mismatch at {bad[:5]}"
    return sa


@pytest.mark.parametrize("X", [3, 7, 13, 39])
@pytest.mark.parametrize("sigma", [1, 2, 4, 8, 32, 200])
def test_random_texts(ctx, oracle, X, sigma):
    for n in (1, 2, 3, 10, 100, 2047, 2048, 2049, 5000, 65_537):
        _check(ctx, oracle, random_text(n, sigma, seed=n + sigma), X)


@pytest.mark.parametrize("X", [3, 7, 13, 39])
def test_alignment_sweep(ctx, oracle, X):
    """n mod X over every residue (dummy-sample path), as main.cpp:101-123."""
    for sigma in (2, 8, 32):
        for d in range(X + 1):
            _check(ctx, oracle, random_text(3000 + d, sigma, seed=d), X)


@pytest.mark.parametrize("X", [3, 39])
def test_unpacked(ctx, oracle, X):
    for sigma in (4, 32):
        _check(ctx, oracle, random_text(20_000, sigma, seed=sigma), X, packing=False)


@pytest.mark.parametrize("width", [32, 40, 64])
def test_output_widths(ctx, oracle, width):
    _check(ctx, oracle, random_text(10_000, 4, seed=5), 39, width=width)


@pytest.mark.parametrize("X", [3, 7, 39])
def test_repetitive_texts(ctx, oracle, X):
    """All-equal, periodic and copied text: deep recursion, discarding, big tie groups."""
    rng = np.random.default_rng(11)
    cases = [
        np.full(50_000, 65, np.uint8),
        np.tile(np.frombuffer(b"abcab", np.uint8), 12_000),
        np.tile(np.frombuffer(b"ACGTTGCAAC", np.uint8), 9_000),
    ]
    base = rng.integers(65, 69, 20_000).astype(np.uint8)
    cases.append(np.concatenate([base, base, base[:7000], rng.integers(65, 69, 5000).astype(np.uint8), base]))
    for t in cases:
        _check(ctx, oracle, t, X)


def test_alphabet_256(ctx, oracle):
    rng = np.random.default_rng(2)
    t = rng.integers(0, 256, 100_000).astype(np.uint8)
    t[:256] = np.arange(256, dtype=np.uint8)
    _check(ctx, oracle, t, 39)
    from distributed_suffix_sorting_evaluation_b200 import DCX_ERR_ALPHABET, DcxError
    with pytest.raises(DcxError) as e:
        ctx.build_sa(t, dc=39, strict=True)
    assert e.value.code == DCX_ERR_ALPHABET


def test_empty_text(ctx):
    assert ctx.build_sa(np.zeros(0, np.uint8), dc=39).size == 0


@pytest.mark.parametrize("X", [3, 39])
def test_level0_names_match_oracle(ctx, oracle, X):
    """Level-0 lexicographic names and unique flags equal the PDCX restatement's."""
    ctx.set_option("trace", 1)
    try:
        rng = np.random.default_rng(7)
        base = rng.integers(65, 69, 30_000).astype(np.uint8)
        t = np.concatenate([base, base[:5000], rng.integers(65, 69, 10_000).astype(np.uint8)])
        sa = ctx.build_sa(t, dc=X, sa_width=64)
        names, uniq = ctx.trace()
        osa, tr = oracle.dcx_sa(t, X=X, base_case_threshold=0, want_trace=True)
        assert np.array_equal(sa, osa)
        assert names.size == tr.m
        assert np.array_equal(names.astype(np.uint64), tr.names)
        assert np.array_equal(uniq, tr.unique)
        st = ctx.stats()
        assert st["level0_last_rank"] == tr.last_rank
        assert st["level0_recursion"] == tr.recursion
    finally:
        ctx.set_option("trace", 0)


def test_deterministic(ctx):
    t = random_text(200_000, 4, seed=9)
    a = ctx.build_sa(t, dc=39)
    b = ctx.build_sa(t, dc=39)
    assert np.array_equal(a, b)


def test_large_random_dna(ctx, oracle):
    t = random_text(4_000_000, 4, seed=1, offset=0)
    _check(ctx, oracle, np.frombuffer(b"ACGT", np.uint8)[t], 39, width=40)
