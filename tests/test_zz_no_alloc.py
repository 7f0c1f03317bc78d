"""dcx_build_sa_noalloc: the allocation-free entry point for callers that cannot
call cudaMalloc (stream capture, allocator callbacks, fully reserved memory).
Its output must equal dcx_build_sa's on the same text, on consecutive calls that
share the library's one scratch array.  Kept in a file of its own that pytest
collects last."""
import ctypes

import numpy as np
import pytest

from conftest import random_text

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, text: np.ndarray) -> np.ndarray:
    d_text = torch.from_numpy(text.copy()).cuda()
    d_sa = torch.empty(max(text.size, 1), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.dcx_build_sa_noalloc(ctypes.c_void_p(d_text.data_ptr()), text.size, ctypes.c_void_p(d_sa.data_ptr()),
                                  ctypes.c_void_p(0))
    assert rc == 0
    torch.cuda.synchronize()
    return d_sa.cpu().numpy().view(np.uint32)[: text.size].astype(np.uint64)


def test_noalloc_matches_build_sa_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from distributed_suffix_sorting_evaluation_b200 import Context, load_library
    lib = load_library()
    rng = np.random.default_rng(21)
    base = rng.integers(65, 69, 12_000).astype(np.uint8)
    texts = [
        np.concatenate([base, base[:9000], rng.integers(65, 69, 11_768).astype(np.uint8)]),  # 32768 chars
        random_text(20_011, 200, seed=3, offset=0),  # includes byte 0
    ]
    with Context(0) as ctx:
        for t in texts:  # two calls in a row over the same shared scratch
            got = _noalloc(lib, torch, t)
            want = ctx.build_sa(t, dc=39, sa_width=32)
            assert np.array_equal(got, want)


def test_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from distributed_suffix_sorting_evaluation_b200 import DCX_ERR_ARG, load_library
    lib = load_library()
    d = torch.zeros(32769, dtype=torch.uint8, device="cuda")
    out = torch.empty(32769, dtype=torch.int32, device="cuda")
    assert lib.dcx_build_sa_noalloc(ctypes.c_void_p(d.data_ptr()), 32769, ctypes.c_void_p(out.data_ptr()),
                                    None) == DCX_ERR_ARG
