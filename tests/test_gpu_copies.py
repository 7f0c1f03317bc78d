"""Texts made of many mutated copies of one sequence ('$'-joined, the
pangenome generator with a short base) put almost every suffix into tie
groups of one element per copy.  With 40..250 copies those groups hold
33..256 elements, the sizes the warp-per-group refinement (including its path
for groups where at most 32 windows differ from the first one, and the full
network when more differ) and the warp-per-group cover-rank tie break sort.
Every SA is compared with libsais built from the reference tree."""
import numpy as np
import pytest

from distributed_suffix_sorting_evaluation_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _copies(copies: int, base_len: int, sub: float, indel: float, seed: int) -> np.ndarray:
    n = copies * (base_len + 1)
    out = np.empty(n, np.uint8)
    W._gen().tg_pangenome(out.ctypes.data, n, base_len, sub, indel, seed)
    return out


@pytest.mark.parametrize("copies,sub,indel", [
    (40, 0.001, 0.0001),    # groups of 33-64
    (100, 0.001, 0.0001),   # 65-128
    (204, 0.001, 0.0001),   # 129-256, a few mutated windows per group
    (204, 0.03, 0.0),       # 129-256, most windows of a group differ: the full network
    (150, 0.0, 0.0),        # exact copies: every window of a group equal
])
@pytest.mark.parametrize("dc", [39, 13])
def test_copies_equal_libsais(ctx, oracle, copies, sub, indel, dc):
    text = _copies(copies, 6000, sub, indel, seed=copies + int(sub * 1000))
    got = ctx.build_sa(text, dc=dc, sa_width=32)
    want = oracle.libsais(text).astype(np.uint64)
    assert np.array_equal(got.astype(np.uint64), want), (copies, sub, dc)


def test_copies_refined_at_recursion_levels(ctx, oracle):
    """With a 2-word first sort at the recursion levels (rec_prefix_words = 2),
    the DC3 levels refine their tie groups by the third name: the 32-bit-char
    forms of the warp-per-group refinement."""
    # names past 2^21 (a 16 M-char random part) make three names wider than two
    # key words; 50 copies of a 50 K base give level-1 groups of about 50
    text = np.concatenate([W.iid(16 << 20, b"ACGT", seed=78), _copies(50, 50_000, 0.001, 0.0001, seed=77)])
    ctx.set_option("rec_prefix_words", 2)
    try:
        got = ctx.build_sa(text, dc=39, sa_width=32)
    finally:
        ctx.set_option("rec_prefix_words", 3)
    assert np.array_equal(got.astype(np.uint64), oracle.libsais(text).astype(np.uint64))


@pytest.mark.parametrize("dc", [3, 39])
def test_tie_groups_longer_than_the_walk(ctx, oracle, dc):
    """Round-0 tie groups of more than 65,536 elements: texts that are almost
    all tied (a run of one character, a short period) take the scan; a random
    text with one long run has few ties, so its groups are walked from their
    starts until the run's group outgrows the walk and the scan takes over."""
    rng = np.random.default_rng(21)
    with_run = np.concatenate([rng.integers(65, 69, 500_000), np.full(100_000, 65), rng.integers(65, 69, 500_000)])
    for text in (np.full(300_000, ord("A"), np.uint8), np.tile(np.frombuffer(b"ACGT", np.uint8), 100_000),
                 with_run.astype(np.uint8)):
        got = ctx.build_sa(text, dc=dc, sa_width=32)
        assert np.array_equal(got.astype(np.uint64), oracle.libsais(text).astype(np.uint64)), (text.size, dc)
