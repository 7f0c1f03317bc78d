"""Generates tests/golden/sa_lcp_fixtures.npz: seeded texts with the suffix
array and LCP array computed by libsais 2.10 compiled from the reference
tree's own sources (oracle/_ref/libsais.so, built by oracle/Makefile).

The fixtures travel with the repository, so the GPU tests can check against
reference-computed answers on a machine without the reference tree.  Run from
the repository root:  python tests/golden/make_golden.py
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
    main()
