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
