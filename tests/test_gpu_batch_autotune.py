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
    texts = _texts(4, 30, 1, 500_000)
    for t, sa in zip(texts, tctx.build_sa_batch(texts, dc=0, sa_width=40)):
        assert np.array_equal(sa, oracle.libsais(t).astype(np.uint64)), t.size
    tctx.set_batch_dc_table([])
