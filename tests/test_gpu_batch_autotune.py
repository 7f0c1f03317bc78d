"""The size-class DC table of batched builds and its autotuner: any table gives
the same SAs (libsais's); the autotuner installs one X per class from its
candidates.  Runs on a context of its own, so the table does not reach the
other tests' context."""
import numpy as np
import pytest

from conftest import random_text
from distributed_suffix_sorting_evaluation_b200 import Context, DcxError

pytestmark = pytest.mark.gpu


def _texts(seed, count, lo, hi, sigma=4):
    rng = np.random.default_rng(seed)
    lens = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    return [random_text(int(n), sigma, seed=seed * 1000 + i) for i, n in enumerate(lens)]


@pytest.fixture(scope="module")
def tctx():
    c = Context(0)
    yield c
    c.close()


def test_table_mixed_dcs_bit_exact(tctx, oracle):
    texts = _texts(2, 80, 1, 400_000)
    texts.append(np.tile(np.frombuffer(b"ACGTTGCAAC", np.uint8), 20_000))  # periodic, 200 KB
    table = [(4096, 3), (65536, 7), (300_000, 13)]
    tctx.set_batch_dc_table(table)
    assert tctx.batch_dc_table() == table
    for t, sa in zip(texts, tctx.build_sa_batch(texts, dc=0, sa_width=32)):
        assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64)), t.size
    tctx.set_batch_dc_table([])
    assert tctx.batch_dc_table() == []


def test_table_rejects_bad_entries(tctx):
    with pytest.raises(DcxError):
        tctx.set_batch_dc_table([(65536, 7), (4096, 3)])  # bounds descend
    with pytest.raises(DcxError):
        tctx.set_batch_dc_table([(4096, 5)])  # no difference cover modulo 5 is built
    assert tctx.batch_dc_table() == []


def test_autotune_installs_a_table(tctx, oracle):
    sample = _texts(3, 40, 3000, 300_000)
    chosen, ms = tctx.autotune_batch(sample, [20_000, 300_000, 1 << 24], candidates=(3, 39), repeats=1)
    assert chosen[0] in (3, 39) and chosen[1] in (3, 39)
    assert chosen[2] == 0 and (ms[2] == -1).all()  # no sample text above 300 KB
    assert (ms[:2] > 0).all()
    assert tctx.batch_dc_table() == [(20_000, chosen[0]), (300_000, chosen[1])]
    tiles = tctx.batch_tile_table()  # the radix tile chosen beside each class's X
    assert len(tiles) == 2 and all(t in (3072, 4096) for t in tiles)
    texts = _texts(4, 30, 1, 500_000)
    for t, sa in zip(texts, tctx.build_sa_batch(texts, dc=0, sa_width=40)):
        assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64)), t.size
    tctx.set_batch_dc_table([])
    assert tctx.batch_tile_table() == []


def test_radix_tile_3072_bit_exact(tctx, oracle):
    """Every radix pass on 3072-element tiles (the tile the autotuner may pick):
    single texts with recursion and a batch give libsais's SAs."""
    tctx.set_option("radix_tile", 3072)
    try:
        rng = np.random.default_rng(11)
        base = rng.integers(65, 69, 200_000).astype(np.uint8)
        for t in (random_text(1_000_003, 4, seed=12), np.concatenate([base, base, base[:50_000], base]),
                  rng.integers(0, 256, 300_000).astype(np.uint8)):
            assert np.array_equal(tctx.build_sa(t, dc=39, sa_width=64), oracle.libsais(t).astype(np.uint64))
        texts = _texts(5, 30, 1, 400_000)
        for t, sa in zip(texts, tctx.build_sa_batch(texts, dc=0, sa_width=32)):
            assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64)), t.size
        with pytest.raises(DcxError):
            tctx.set_option("radix_tile", 2048)
    finally:
        tctx.set_option("radix_tile", 4096)
