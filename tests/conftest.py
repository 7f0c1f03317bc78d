import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference tree (read in place for its golden files); DCX_REFERENCE_TREE
# points elsewhere when it is mounted at another path.
REFERENCE = os.environ.get("DCX_REFERENCE_TREE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libdcxgpu.so")


# Suites run in dependency order: the suffix-array build itself first, then
# what wraps it (batches, serving, the CLI), then what consumes its output
# (LCP, SA files, BWT, generalized SA) and the batched-DC tuning; the
# allocation-free entry point last, in a file of its own.  Under -x a failure
# in a consumer then never hides the state of the build it consumes.
_SUITE_ORDER = ["test_abi", "test_oracle", "test_golden_fixtures", "test_gpu_parity", "test_gpu_copies", "test_gpu_batch",
                "test_gpu_serve", "test_cli", "test_gpu_lcp", "test_gpu_safile", "test_gpu_bwt", "test_gpu_gsa",
                "test_gpu_batch_autotune", "test_gpu_timeout", "test_distributed", "test_gpu_distributed",
                "test_gpu_fullsize"]


def pytest_collection_modifyitems(config, items):
    def rank(item):
        name = os.path.splitext(os.path.basename(str(item.fspath)))[0]
        if name == "test_zz_no_alloc":
            return len(_SUITE_ORDER) + 1
        return _SUITE_ORDER.index(name) if name in _SUITE_ORDER else len(_SUITE_ORDER)

    items.sort(key=rank)  # stable: the order inside a file is kept


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    from distributed_suffix_sorting_evaluation_b200 import Context
    if not gpu_available():
        pytest.skip("no GPU")
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    return O


def reference_file(*parts):
    """Path of a file in the reference tree, or skip when the tree is absent."""
    p = os.path.join(REFERENCE, *parts)
    if not os.path.exists(p):
        pytest.skip("reference tree not mounted")
    return p


def random_text(n, sigma, seed, offset=65):
    rng = np.random.default_rng(seed)
    return rng.integers(offset, offset + sigma, n).astype(np.uint8)


def psac_gsa_case(seq: str, reps: int):
    """The string sets of the reference's generalized-SA tests
    (psac/test/test_gsa.cpp:24-30, 145-178): `reps` strings, the j-th being
    `seq` repeated j+1 times.  Returns (strings, expected GSA over the
    concatenation without separators) with the expectation restated from
    psac/test/test_gsa.cpp:32-50: for each offset i inside one copy of `seq`,
    and each string j whose copy holds the next smallest suffix, the suffix of
    string j at i, then that suffix's equal in every longer string, each one
    copy of `seq` (k*len(seq) positions) further along."""
    L = len(seq)
    strings = [seq * (j + 1) for j in range(reps)]
    expected = []
    for i in range(L):
        for j in range(reps):
            pos = i + L * (j * (j + 1) // 2)  # offset i in string j
            expected.append(pos)
            for k in range(j + 2, reps + 1):
                pos += k * L
                expected.append(pos)
    return strings, expected


PSAC_GSA_CASES = [("ab", 3), ("abc", 3), ("a", 20), ("abc", 10), ("abcdef", 50)]


def flat_positions(text: np.ndarray, gsa: np.ndarray) -> list:
    """A generalized SA over a 0-separated set, without the separators and with
    positions counted in the concatenation without separators (psac's layout)."""
    g = np.asarray(gsa, dtype=np.int64)
    sep_before = np.concatenate([[0], np.cumsum(text == 0)[:-1]])
    keep = text[g] != 0
    return (g[keep] - sep_before[g[keep]]).tolist()


def set_bytes(strings) -> np.ndarray:
    return np.frombuffer(b"".join(s.encode() + b"\0" for s in strings), np.uint8).copy()


def psac_glcp_case(seq: str, reps: int) -> list:
    """The LCP array psac's GSA tests expect beside psac_gsa_case's GSA
    (psac/test/test_gsa.cpp:52-67), restated: for each offset i inside one copy
    of `seq`, a 0 for the first suffix at i, then for j = 1 .. reps-1 the value
    j*len(seq) - i once for each of the reps+1-j suffixes sharing it."""
    L = len(seq)
    out = []
    for i in range(L):
        out.append(0)
        for j in range(1, reps):
            out.extend([j * L - i] * (reps + 1 - j))
    return out
