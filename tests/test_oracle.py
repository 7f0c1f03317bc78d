"""The CPU oracle (restatement of PDCX) pinned against the reference's own golden
vectors and tables, and against libsais built from the reference tree."""
import re

import numpy as np
import pytest

from conftest import random_text, reference_file


def test_golden_abracadabra(oracle):
    for name in ("abracadabra4", "abracadabra8"):
        text = np.fromfile(reference_file("B_DC_3_7_13", "src", "examples", name), np.uint8)
        gold = np.fromfile(reference_file("B_DC_3_7_13", "src", "examples", name + ".sa"), np.uint32)
        for X in (3, 7, 13, 39):
            sa = oracle.dcx_sa(text, X=X, base_case_threshold=0)
            assert np.array_equal(sa, gold.astype(np.uint64)), (name, X)
        assert np.array_equal(oracle.libsais(text), gold.astype(np.int64))


def test_golden_three_brothers(oracle):
    text = np.fromfile(reference_file("dPD", "tests", "test_data", "the_three_brothers.txt"), np.uint8)
    gold = np.fromfile(reference_file("dPD", "tests", "test_data", "the_three_brothers_size_t_sa"), np.uint64)
    assert np.array_equal(oracle.libsais(text).astype(np.uint64), gold)
    for X in (3, 7, 13, 39):
        for packing in (True, False):
            assert np.array_equal(oracle.dcx_sa(text, X=X, packing=packing, base_case_threshold=0), gold)


def test_text_only_edge_files(oracle):
    for rel in (("B_DC_3_7_13", "src", "examples", "aaa"), ("B_DC_3_7_13", "src", "examples", "mississippi"),
                ("dPD", "tests", "test_data", "small_text.txt")):
        text = np.fromfile(reference_file(*rel), np.uint8)
        ref = oracle.libsais(text).astype(np.uint64)
        for X in (3, 39):
            assert np.array_equal(oracle.dcx_sa(text, X=X, base_case_threshold=0), ref)


def _parse_reference_tables():
    src = open(reference_file("lightweight_dcx", "src", "pdcx", "difference_cover.hpp")).read()
    out = {}
    for m in re.finditer(r"struct DC(\d+)Param \{(.*?)\n\};", src, re.S):
        X = int(m.group(1))
        body = m.group(2)
        nums = lambda key: [int(v) for v in re.findall(r"\d+", re.search(key + r".*?=\s*(\{.*?\});", body, re.S).group(1))]
        out[X] = (nums(r"DC\[D\]"), nums(r"NEXT_RANK\[X\]"), nums(r"cmpDepthRanks\[X\]\[X\]\[3\]"))
    return out


def test_dc_tables_closed_form_equal_reference(oracle):
    ref = _parse_reference_tables()
    assert set(ref) == {3, 7, 13, 21, 31, 39, 57, 73, 91, 95, 133}
    for X, (dc, nr, cmp) in ref.items():
        odc, _, onr, ocmp = oracle.dc_table(X)
        assert list(odc) == dc
        assert list(onr) == nr
        assert list(ocmp.ravel()) == cmp, X


@pytest.mark.parametrize("X", [3, 7, 13, 39])
def test_difference_cover_property(oracle, X):
    dc, in_dc, _, _ = oracle.dc_table(X)
    diffs = {(int(a) - int(b)) % X for a in dc for b in dc}
    assert diffs == set(range(X))


@pytest.mark.parametrize("X", [3, 7, 13, 39])
def test_reference_test_matrix(oracle, X):
    """main.cpp:80-123 matrix (sigma in {2,8,32}) with a small base case so the DCX
    phases run, plus the alignment sweep n = 1000 + d."""
    for sigma in (2, 8, 32):
        for n, reps in ((100, 6), (1000, 3), (10000, 1)):
            for r in range(reps):
                t = random_text(n, sigma, seed=r * 7 + sigma)
                assert np.array_equal(oracle.dcx_sa(t, X=X, base_case_threshold=0),
                                      oracle.libsais(t).astype(np.uint64))
        for d in range(15):
            t = random_text(1000 + d, sigma, seed=d)
            assert np.array_equal(oracle.dcx_sa(t, X=X, base_case_threshold=0),
                                  oracle.libsais(t).astype(np.uint64))


def test_recursion_and_discarding_paths(oracle):
    t = np.tile(np.frombuffer(b"ACGTTGCAAC", np.uint8), 600)
    sa, tr = oracle.dcx_sa(t, X=39, base_case_threshold=0, want_trace=True)
    assert tr.recursion in (1, 2) and tr.max_depth > 1
    assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64))
    rng = np.random.default_rng(3)
    base = rng.integers(0, 4, 3000).astype(np.uint8) + 65
    t2 = np.concatenate([base, base[:2000], rng.integers(65, 69, 3000).astype(np.uint8)])
    sa2, tr2 = oracle.dcx_sa(t2, X=7, base_case_threshold=0, want_trace=True)
    assert tr2.recursion == 2 and tr2.reduction <= 0.7
    assert np.array_equal(sa2, oracle.libsais(t2).astype(np.uint64))


def test_alphabet_256_refused(oracle):
    t = np.arange(512, dtype=np.uint32).astype(np.uint8)
    with pytest.raises(ValueError):
        oracle.compress_alphabet(t)


def test_packing_choice(oracle):
    # cli.cpp:488-533: 3/5/8 bits, K = ceil(X / (64 / bits))
    assert oracle.packing_for_sigma(39, 4) == (3, 2)
    assert oracle.packing_for_sigma(3, 4) == (3, 1)
    assert oracle.packing_for_sigma(39, 20) == (5, 4)
    assert oracle.packing_for_sigma(39, 200) == (8, 5)


def test_libsais_lcp_known_answer(oracle):
    """mississippi: SA 10 7 4 1 0 9 8 6 3 5 2, LCP 0 1 1 4 0 0 1 0 2 1 3 (textbook values)."""
    t = np.frombuffer(b"mississippi", np.uint8)
    plcp, lcp = oracle.libsais_lcp(t)
    assert list(oracle.libsais(t)) == [10, 7, 4, 1, 0, 9, 8, 6, 3, 5, 2]
    assert list(lcp) == [0, 1, 1, 4, 0, 0, 1, 0, 2, 1, 3]
    sa = oracle.libsais(t)
    assert all(plcp[sa[k]] == lcp[k] for k in range(t.size))


def test_libsais_bwt_known_answer_and_restatement(oracle):
    """banana: BWT of banana$ is annb$aa, so libsais64_bwt returns annbaa with
    primary index 4 (textbook values); the SA-based restatement the GPU kernel
    follows agrees with libsais on these and on random texts."""
    t = np.frombuffer(b"banana", np.uint8)
    u, p = oracle.libsais_bwt(t)
    assert (u.tobytes(), p) == (b"annbaa", 4)
    u, p = oracle.libsais_bwt(np.frombuffer(b"mississippi", np.uint8))
    assert (u.tobytes(), p) == (b"ipssmpissii", 5)
    assert oracle.libsais_bwt(np.zeros(0, np.uint8))[1] == 0
    for seed, (n, sigma) in enumerate([(1, 2), (2, 2), (100, 2), (5000, 4), (20000, 255)]):
        t = random_text(n, sigma, seed=seed)
        u, p = oracle.libsais_bwt(t)
        u2, p2 = oracle.bwt_from_sa(t, oracle.libsais(t))
        assert p == p2 and np.array_equal(u, u2)


def _string_set(rng, k, sigma, base):
    parts = []
    for _ in range(k):
        m = rng.integers(0, 3)
        if m == 0:
            s = rng.integers(1, 1 + sigma, rng.integers(1, 40))
        elif m == 1:
            s = base[rng.integers(0, base.size):]
        else:
            s = base
        parts.append(np.concatenate([s, [0]]))
    return np.concatenate(parts).astype(np.uint8)


def test_libsais_gsa_known_answer_and_restatement(oracle):
    """libsais64_gsa orders the suffixes of a 0-separated string set as if each
    separator were its own symbol, smallest, in string order; the plain-SA
    regrouping the GPU follows gives the same array."""
    t = np.frombuffer(b"ab\0ab\0", np.uint8)
    assert oracle.libsais_gsa(t).tolist() == [2, 5, 0, 3, 1, 4]
    t = np.frombuffer(b"banana\0ana\0", np.uint8)
    assert oracle.libsais_gsa(t).tolist() == [6, 10, 5, 9, 3, 7, 1, 0, 4, 8, 2]
    with pytest.raises(RuntimeError):
        oracle.libsais_gsa(np.frombuffer(b"a\0\0", np.uint8))  # empty string
    rng = np.random.default_rng(2)
    for _ in range(200):
        base = rng.integers(1, 4, rng.integers(1, 50))
        t = _string_set(rng, int(rng.integers(1, 30)), 3, base)
        assert np.array_equal(oracle.gsa_from_sa(t), oracle.libsais_gsa(t))


@pytest.mark.parametrize("seq,reps", [("ab", 3), ("abc", 3), ("a", 20), ("abc", 10), ("abcdef", 50)])
def test_libsais_gsa_equals_psac_test_expectations(oracle, seq, reps):
    """The generalized SA the GPU reproduces (libsais64_gsa's) is, without its
    separator positions, the array the reference's psac GSA tests expect."""
    from conftest import flat_positions, psac_gsa_case, set_bytes
    strings, expected = psac_gsa_case(seq, reps)
    t = set_bytes(strings)
    assert flat_positions(t, oracle.libsais_gsa(t)) == expected
    from conftest import psac_glcp_case
    _, lcp = oracle.libsais_lcp_gsa(t)
    assert lcp[t[oracle.libsais_gsa(t)] != 0].tolist() == psac_glcp_case(seq, reps)
    t = set_bytes(["abab", "baba"])  # psac/test/test_gsa.cpp:71-101
    g = oracle.libsais_gsa(t)
    assert flat_positions(t, g) == [7, 2, 5, 0, 3, 6, 1, 4]
    assert oracle.libsais_lcp_gsa(t, g)[1][t[g] != 0].tolist() == [0, 1, 2, 3, 0, 1, 2, 3]
