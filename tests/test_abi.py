"""C ABI checks that need no GPU: the library loads, exports every function that
include/dcx_gpu.h declares, and its host-only calls agree with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "dcx_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(dcx_\w+)\s*\(", src, re.M)))


def test_header_matches_python_binding():
    import distributed_suffix_sorting_evaluation_b200 as pkg
    assert sorted(pkg.EXPORTED) == _declared()


def test_library_exports_every_declared_symbol():
    import distributed_suffix_sorting_evaluation_b200 as pkg
    lib = pkg.load_library()
    for name in _declared():
        assert hasattr(lib, name), name
    assert lib.dcx_version().decode().startswith("dcx-b200")
    assert lib.dcx_strerror(-2).decode().startswith("alphabet")


@pytest.mark.parametrize("X", [3, 7, 13, 21, 31, 39, 57, 73, 91, 95, 133])
def test_dc_tables_equal_oracle(X, oracle):
    import distributed_suffix_sorting_evaluation_b200 as pkg
    dc, nr, cmp = pkg.dc_table(X)
    odc, _, onr, ocmp = oracle.dc_table(X)
    assert np.array_equal(dc, odc) and np.array_equal(nr, onr) and np.array_equal(cmp, ocmp)


def test_unsupported_dc_rejected():
    import distributed_suffix_sorting_evaluation_b200 as pkg
    lib = pkg.load_library()
    assert lib.dcx_dc_table(5, None, None, None, None) == pkg.DCX_ERR_ARG
    with pytest.raises(pkg.DcxError):
        pkg.PDCX.__init__(object.__new__(pkg.PDCX), pkg.PDCXConfig(dc=5))


def test_null_context_rejected():
    import distributed_suffix_sorting_evaluation_b200 as pkg
    lib = pkg.load_library()
    assert lib.dcx_build_sa(None, None, 0, 39, 40, None, 0) == pkg.DCX_ERR_ARG
    assert lib.dcx_ctx_destroy(None) == pkg.DCX_ERR_ARG
    # every other context call checks its context before touching a device
    rid = ctypes.c_uint64()
    st = ctypes.c_int()
    ok = ctypes.c_int()
    assert lib.dcx_build_sa_batch(None, None, None, 0, 0, 32, None, 0) == pkg.DCX_ERR_ARG
    assert lib.dcx_build_lcp(None, None, 0, None, 32, None, 32, 0) == pkg.DCX_ERR_ARG
    assert lib.dcx_build_gsa(None, None, 0, 39, 32, None, 0) == pkg.DCX_ERR_ARG
    cnt = ctypes.c_uint32()
    assert lib.dcx_set_batch_dc_table(None, None, None, 0) == pkg.DCX_ERR_ARG
    assert lib.dcx_get_batch_dc_table(None, None, None, 0, ctypes.byref(cnt)) == pkg.DCX_ERR_ARG
    assert lib.dcx_autotune_batch(None, None, None, 0, None, 0, None, 0, 1, None, None) == pkg.DCX_ERR_ARG
    primary = ctypes.c_uint64()
    assert lib.dcx_build_bwt(None, None, 0, None, 32, None, ctypes.byref(primary), 0) == pkg.DCX_ERR_ARG
    assert lib.dcx_bwt(None, None, None, 0, 39, ctypes.byref(primary), 0) == pkg.DCX_ERR_ARG
    assert lib.dcx_check_sa(None, None, 0, None, 32, 0, ctypes.byref(ok)) == pkg.DCX_ERR_ARG
    assert lib.dcx_serve_submit(None, None, 0, 0, 32, ctypes.byref(rid)) == pkg.DCX_ERR_ARG
    assert lib.dcx_serve_submit_ex(None, None, 0, 0, 32, 0, ctypes.byref(rid)) == pkg.DCX_ERR_ARG
    assert lib.dcx_serve_poll(None, 1, None, ctypes.byref(st), None) == pkg.DCX_ERR_ARG
    assert lib.dcx_serve_release(None, 1) == pkg.DCX_ERR_ARG
    assert lib.dcx_serve_drain(None) == pkg.DCX_ERR_ARG
    assert lib.dcx_set_option(None, b"trace", 1.0) == pkg.DCX_ERR_ARG


def test_uint40_unpacking():
    import distributed_suffix_sorting_evaluation_b200 as pkg
    vals = np.array([0, 1, 255, 256, 2**32 - 1, 2**32, 2**40 - 1], np.uint64)
    raw = np.zeros(5 * vals.size, np.uint8)
    for i, v in enumerate(vals):
        raw[5 * i: 5 * i + 5] = [(int(v) >> (8 * b)) & 255 for b in range(5)]
    assert np.array_equal(pkg.unpack_sa(raw, 40, vals.size), vals)
