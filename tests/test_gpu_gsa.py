"""Generalized suffix array of a string set on the GPU against libsais64_gsa
from the reference tree: exact equality."""
import numpy as np
import pytest

from distributed_suffix_sorting_evaluation_b200 import DcxError

pytestmark = pytest.mark.gpu


def _set_of(strings):
    return np.concatenate([np.concatenate([np.asarray(s, np.uint8), [0]]) for s in strings]).astype(np.uint8)


def _cases():
    rng = np.random.default_rng(17)
    out = [np.zeros(1, np.uint8), np.frombuffer(b"a\0", np.uint8), np.frombuffer(b"ab\0ab\0", np.uint8),
           np.frombuffer(b"banana\0ana\0", np.uint8)]
    # many short random strings over {1..4}
    out.append(_set_of([rng.integers(1, 5, rng.integers(1, 60)) for _ in range(3000)]))
    # identical strings: every suffix of one agrees with the same suffix of the others
    s = rng.integers(65, 69, 5000)
    out.append(_set_of([s] * 40))
    # suffixes and prefixes of one base string (long shared tails)
    base = rng.integers(1, 4, 20_000)
    out.append(_set_of([base[rng.integers(0, base.size):] for _ in range(50)] + [base[:rng.integers(1, base.size)]
                                                                               for _ in range(50)]))
    # raw bytes 1..255 and a few long strings
    out.append(_set_of([rng.integers(1, 256, rng.integers(1, 200_000)) for _ in range(8)]))
    # the batched workload's shape, smaller: log-uniform lengths
    lens = np.exp(rng.uniform(np.log(16), np.log(1 << 16), 300)).astype(np.int64)
    out.append(_set_of([rng.integers(1, 5, int(m)) for m in lens]))
    return out


@pytest.mark.parametrize("idx", range(9))
@pytest.mark.parametrize("dc", [3, 39])
def test_gsa_matches_libsais(ctx, oracle, idx, dc):
    t = _cases()[idx]
    want = oracle.libsais_gsa(t)
    got = ctx.build_gsa(t, dc=dc, sa_width=64)
    assert np.array_equal(got, want.astype(np.uint64))


def test_gsa_device_widths(ctx, oracle):
    import torch
    rng = np.random.default_rng(4)
    t = _set_of([rng.integers(1, 5, rng.integers(1, 3000)) for _ in range(500)])
    want = oracle.libsais_gsa(t).astype(np.uint64)
    d_text = torch.from_numpy(t).cuda()
    from distributed_suffix_sorting_evaluation_b200 import unpack_sa
    for width in (32, 40, 64):
        d_sa = torch.empty(t.size * width // 8, dtype=torch.uint8, device="cuda")
        ctx.build_gsa_device(d_text.data_ptr(), t.size, d_sa.data_ptr(), dc=39, sa_width=width)
        torch.cuda.synchronize()
        assert np.array_equal(unpack_sa(d_sa.cpu().numpy(), width, t.size), want)


def test_gsa_refuses_what_libsais_refuses(ctx):
    for bad in (b"ab", b"a\0\0", b"\0a\0"):
        with pytest.raises(DcxError):
            ctx.build_gsa(np.frombuffer(bad, np.uint8))
    assert ctx.build_gsa(np.zeros(0, np.uint8)).size == 0


def test_gsa_on_the_psac_test_sets(ctx):
    """The string sets of the reference's psac GSA tests, checked against the
    arrays those tests expect."""
    from conftest import PSAC_GSA_CASES, flat_positions, psac_gsa_case, set_bytes
    t = set_bytes(["abab", "baba"])
    assert flat_positions(t, ctx.build_gsa(t)) == [7, 2, 5, 0, 3, 6, 1, 4]
    for seq, reps in PSAC_GSA_CASES:
        strings, expected = psac_gsa_case(seq, reps)
        t = set_bytes(strings)
        assert flat_positions(t, ctx.build_gsa(t)) == expected


@pytest.mark.parametrize("idx", range(9))
def test_gsa_lcp_matches_libsais(ctx, oracle, idx):
    """LCP of a generalized SA (separators never match) against
    libsais64_plcp_gsa + libsais64_lcp, from the GPU-built GSA."""
    t = _cases()[idx]
    g = ctx.build_gsa(t)
    plcp, lcp = oracle.libsais_lcp_gsa(t, g.astype(np.int64))
    assert np.array_equal(ctx.build_lcp(t, g, gsa=True), lcp.astype(np.uint64))
    assert np.array_equal(ctx.build_lcp(t, g, permuted=True, gsa=True), plcp.astype(np.uint64))


def test_gsa_lcp_on_the_psac_test_sets(ctx):
    from conftest import PSAC_GSA_CASES, psac_gsa_case, psac_glcp_case, set_bytes
    for seq, reps in PSAC_GSA_CASES:
        strings, _ = psac_gsa_case(seq, reps)
        t = set_bytes(strings)
        g = ctx.build_gsa(t)
        lcp = ctx.build_lcp(t, g, gsa=True)
        assert lcp[t[g.astype(np.int64)] != 0].tolist() == psac_glcp_case(seq, reps)


@pytest.mark.parametrize("dc", [3, 39])
def test_gpu_gsa_matches_fixtures(ctx, dc):
    """The committed generalized-SA fixtures (libsais64_gsa and its LCP, built
    from the reference tree)."""
    from test_golden_fixtures import _gsa_fixtures
    for name, t, g, glcp in _gsa_fixtures():
        got = ctx.build_gsa(t, dc=dc, sa_width=64)
        assert np.array_equal(got, g), (name, dc)
        assert np.array_equal(ctx.build_lcp(t, got, gsa=True), glcp), (name, dc)
