"""Generates the committed fixtures, computed by libsais 2.10 compiled from the
reference tree's own sources (oracle/_ref/libsais.so, built by oracle/Makefile):

  sa_lcp_fixtures.npz   seeded texts with their suffix array and LCP array;
  bwt_gsa_fixtures.npz  the same texts' BWT (libsais64_bwt: U and the primary
                        index), and seeded 0-separated string sets with their
                        generalized SA (libsais64_gsa) and its LCP
                        (libsais64_plcp_gsa + libsais64_lcp).

The fixtures travel with the repository, so the GPU tests can check against
reference-computed answers on a machine without the reference tree.  Run from
the repository root:  python tests/golden/make_golden.py [sa_lcp|bwt_gsa]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def cases():
    rng = np.random.default_rng(20261203)
    out = {}
    out["single"] = np.frombuffer(b"A", np.uint8)
    out["pair"] = np.frombuffer(b"BA", np.uint8)
    for n, sigma, off in [(17, 2, 65), (100, 4, 65), (1000, 8, 97), (4097, 4, 65), (20000, 32, 60),
                          (12000, 256, 0)]:
        out[f"rand_{n}_{sigma}"] = rng.integers(off, off + sigma, n).astype(np.uint8) if sigma < 256 \
            else rng.integers(0, 256, n).astype(np.uint8)
    out["all_equal_5000"] = np.full(5000, 84, np.uint8)
    out["periodic_9000"] = np.tile(np.frombuffer(b"ACGTTGCAA", np.uint8), 1000)
    base = rng.integers(65, 69, 3000).astype(np.uint8)
    mut = base.copy()
    mut[::97] = 71
    out["repeats_9500"] = np.concatenate([base, mut, base, base[:500]])
    return out


def string_sets():
    rng = np.random.default_rng(20261204)
    sets = {"psac_tiny": [b"abab", b"baba"]}  # psac/test/test_gsa.cpp:71-101
    sets["copies"] = [b"ACGTACGTTT"] * 6 + [b"ACGTACG", b"TT"]
    base = rng.integers(65, 69, 400).astype(np.uint8).tobytes()
    sets["tails"] = [base[int(rng.integers(0, 400)):] for _ in range(30)] + [base[: int(rng.integers(1, 400))]
                                                                          for _ in range(30)]
    sets["random"] = [rng.integers(97, 101, int(rng.integers(1, 300))).astype(np.uint8).tobytes()
                      for _ in range(200)]
    return {k: np.frombuffer(b"".join(s + b"\0" for s in v), np.uint8).copy() for k, v in sets.items()}


def main_bwt_gsa():
    arrays = {}
    for name, t in cases().items():
        u, p = O.libsais_bwt(t)
        arrays[f"text_{name}"] = t
        arrays[f"bwt_{name}"] = u
        arrays[f"primary_{name}"] = np.array([p], np.uint64)
    for name, t in string_sets().items():
        g = O.libsais_gsa(t)
        _, lcp = O.libsais_lcp_gsa(t, g)
        arrays[f"set_{name}"] = t
        arrays[f"gsa_{name}"] = g.astype(np.uint32)
        arrays[f"glcp_{name}"] = lcp.astype(np.uint32)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bwt_gsa_fixtures.npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path}")


def main():
    arrays = {}
    for name, t in cases().items():
        sa = O.libsais(t)
        _, lcp = O.libsais_lcp(t, sa)
        arrays[f"text_{name}"] = t
        arrays[f"sa_{name}"] = sa.astype(np.uint32)
        arrays[f"lcp_{name}"] = lcp.astype(np.uint32)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sa_lcp_fixtures.npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path}: {len(arrays) // 3} texts")


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    if which in ("all", "sa_lcp"):
        main()
    if which in ("all", "bwt_gsa"):
        main_bwt_gsa()
