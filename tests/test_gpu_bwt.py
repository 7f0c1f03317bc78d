"""BWT from a suffix array on the GPU against libsais64_bwt from the reference
tree: the same bytes and the same primary index."""
import numpy as np
import pytest

from conftest import random_text
from distributed_suffix_sorting_evaluation_b200 import DcxError

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(13)
    out = [np.zeros(0, np.uint8), np.frombuffer(b"A", np.uint8), np.frombuffer(b"banana", np.uint8),
           np.frombuffer(b"mississippi", np.uint8)]
    for n, sigma in [(2, 2), (65, 4), (5000, 4), (100_000, 4), (300_000, 200), (1 << 20, 4)]:
        out.append(random_text(n, sigma, seed=n + sigma))
    out.append(np.full(70_000, 67, np.uint8))                                # primary index n
    base = rng.integers(0, 256, 50_000).astype(np.uint8)                     # raw bytes incl. 0
    out.append(np.concatenate([base, base, base[:7_000]]))
    return out


@pytest.mark.parametrize("idx", range(12))
def test_bwt_matches_libsais(ctx, oracle, idx):
    t = _cases()[idx]
    want, p = oracle.libsais_bwt(t)
    sa = oracle.libsais(t) if t.size else np.zeros(0, np.int64)
    got, q = ctx.build_bwt(t, sa)
    assert q == p
    assert np.array_equal(got, want)


def test_bwt_of_gpu_sa_device(ctx, oracle):
    """SA built on the GPU, BWT from device buffers, for each SA width."""
    import torch
    t = random_text(1 << 21, 4, seed=9)
    t[700_000:1_000_000] = t[:300_000]
    want, p = oracle.libsais_bwt(t)
    d_text = torch.from_numpy(t).cuda()
    d_bwt = torch.empty(t.size, dtype=torch.uint8, device="cuda")
    for width in (32, 40, 64):
        d_sa = torch.empty(t.size * width // 8, dtype=torch.uint8, device="cuda")
        ctx.build_sa_device(d_text.data_ptr(), t.size, d_sa.data_ptr(), dc=39, sa_width=width)
        q = ctx.build_bwt_device(d_text.data_ptr(), t.size, d_sa.data_ptr(), width, d_bwt.data_ptr())
        torch.cuda.synchronize()
        assert q == p
        assert np.array_equal(d_bwt.cpu().numpy(), want)


def test_bwt_refuses_what_is_not_a_suffix_array(ctx, oracle):
    t = random_text(10_000, 4, seed=3)
    sa = oracle.libsais(t)
    bad = sa.copy()
    bad[17] = t.size                   # out of range
    with pytest.raises(DcxError):
        ctx.build_bwt(t, bad)
    bad = sa.copy()
    bad[bad == 1] = 0                  # two zeros
    with pytest.raises(DcxError):
        ctx.build_bwt(t, bad)
    got, q = ctx.build_bwt(t, sa)      # the context is still usable
    want, p = oracle.libsais_bwt(t)
    assert q == p and np.array_equal(got, want)


@pytest.mark.parametrize("idx", [1, 2, 3, 6, 9, 10])
def test_bwt_from_text_like_libsais(ctx, oracle, idx):
    """dcx_bwt: text in, BWT and primary index out, as libsais64_bwt."""
    t = _cases()[idx]
    want, p = oracle.libsais_bwt(t)
    for dc in (3, 39):
        got, q = ctx.bwt(t, dc=dc)
        assert q == p and np.array_equal(got, want)


def test_gpu_bwt_matches_fixtures(ctx):
    """The committed BWT fixtures (libsais64_bwt built from the reference tree)."""
    from test_golden_fixtures import _bwt_fixtures, _fixtures
    sa_of = {n: sa for n, _, sa, _ in _fixtures()}
    for name, t, u, p in _bwt_fixtures():
        got, q = ctx.build_bwt(t, sa_of[name])
        assert q == p and np.array_equal(got, u), name
        got, q = ctx.bwt(t, dc=39)
        assert q == p and np.array_equal(got, u), name
