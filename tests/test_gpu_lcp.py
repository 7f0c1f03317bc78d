"""LCP construction on the GPU (Phi + chunked Kasai) against libsais64_plcp /
libsais64_lcp from the reference tree: exact equality."""
import numpy as np
import pytest

from conftest import random_text

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(11)
    out = [np.zeros(0, np.uint8), np.frombuffer(b"A", np.uint8), np.frombuffer(b"mississippi", np.uint8)]
    for n, sigma in [(2, 2), (63, 1), (64, 2), (65, 4), (1000, 2), (5000, 4), (100_000, 4), (300_000, 200),
                     (1 << 20, 4)]:
        out.append(random_text(n, sigma, seed=n + sigma))
    out.append(np.full(200_000, 67, np.uint8))                               # LCP up to n - 1
    out.append(np.tile(np.frombuffer(b"ACGTTGCA", np.uint8), 40_000))        # periodic
    base = rng.integers(0, 256, 50_000).astype(np.uint8)                     # raw bytes incl. 0
    out.append(np.concatenate([base, base, base[:7_000]]))                   # long repeats
    return out


@pytest.mark.parametrize("idx", range(15))
def test_lcp_matches_libsais(ctx, oracle, idx):
    cases = _cases()
    if idx >= len(cases):
        pytest.skip("no such case")
    t = cases[idx]
    sa = oracle.libsais(t)
    plcp, lcp = oracle.libsais_lcp(t, sa)
    got = ctx.build_lcp(t, sa)
    assert np.array_equal(got, lcp.astype(np.uint64))
    gotp = ctx.build_lcp(t, sa, permuted=True)
    assert np.array_equal(gotp, plcp.astype(np.uint64))


def test_lcp_of_gpu_sa_device(ctx, oracle):
    """SA built on the GPU, LCP from device buffers (40-bit SA in, 32-bit LCP out)."""
    import torch
    t = random_text(2_000_000, 4, seed=5)
    t[500_000:900_000] = t[:400_000]  # a long repeat
    d_text = torch.from_numpy(t).cuda()
    d_sa = torch.empty(t.size * 5, dtype=torch.uint8, device="cuda")
    ctx.build_sa_device(d_text.data_ptr(), t.size, d_sa.data_ptr(), dc=39, sa_width=40)
    d_lcp = torch.empty(t.size, dtype=torch.int32, device="cuda")
    ctx.build_lcp_device(d_text.data_ptr(), t.size, d_sa.data_ptr(), 40, d_lcp.data_ptr(), 32)
    torch.cuda.synchronize()
    _, lcp = oracle.libsais_lcp(t)
    assert np.array_equal(d_lcp.cpu().numpy().astype(np.int64), lcp)


def test_lcp_long_text_two_step_phi(ctx, oracle):
    """Texts past 2^22 characters build Phi in two steps (records, one radix pass
    on the second-highest byte of SA[k], an L2-local scatter); the LCP and PLCP
    must still equal libsais's, as must the generalized SA and its LCP of a set
    that long."""
    t = random_text(6_000_000, 4, seed=77)
    t[3_000_000:3_500_000] = t[100_000:600_000]  # a long repeat
    sa = oracle.libsais(t)
    plcp, lcp = oracle.libsais_lcp(t, sa)
    assert np.array_equal(ctx.build_lcp(t, sa), lcp.astype(np.uint64))
    assert np.array_equal(ctx.build_lcp(t, sa, permuted=True), plcp.astype(np.uint64))
    s = random_text(5_000_000, 3, seed=78)
    s[(1 << 20) - 1::1 << 20] = 0  # strings of 1 MiB, each ended by a 0
    s[-1] = 0
    gsa = oracle.libsais_gsa(s)
    assert np.array_equal(ctx.build_gsa(s, dc=39, sa_width=64), gsa.astype(np.uint64))
    _, glcp = oracle.libsais_lcp_gsa(s, gsa)
    assert np.array_equal(ctx.build_lcp(s, gsa, gsa=True), glcp.astype(np.uint64))
