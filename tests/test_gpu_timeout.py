"""Failure detection without a GPU fault: the onesweep look-back is the only
device-side wait, and it gives up after `spin_limit` polls.  The test makes the
wait run out on purpose: with the option "lookback_hold_tile" = 0, tile 0 of
every radix pass never publishes its status (a flag that nothing sets), so the
CTA of tile 1 polls until its limit, records DEV_ERR_TIMEOUT, keeps every write
in range and finishes.  The build must return DCX_ERR_TIMEOUT right after that
sort and report how many CTAs gave up; the context stays usable: the same text
then builds correctly with the hook off and the default limit."""
import numpy as np
import pytest

from conftest import random_text
from distributed_suffix_sorting_evaluation_b200 import DCX_ERR_TIMEOUT, Context, DcxError

pytestmark = pytest.mark.gpu


def test_lookback_gives_up_cleanly(oracle):
    t = random_text(16 << 20, 4, seed=31)  # ~5,500 tiles per pass
    want = oracle.libsais(t).astype(np.uint64)
    with Context(0) as c:
        c.set_option("spin_limit", 256)  # a few microseconds of polling
        c.set_option("lookback_hold_tile", 0)
        with pytest.raises(DcxError) as e:
            c.build_sa(t, dc=39, sa_width=32)
        assert e.value.code == DCX_ERR_TIMEOUT, e.value
        assert c.stats()["lookback_gave_up"] >= 1
        c.set_option("lookback_hold_tile", -1)
        c.set_option("spin_limit", 1 << 24)
        assert np.array_equal(c.build_sa(t, dc=39, sa_width=32), want)
        assert c.stats()["lookback_gave_up"] == 0


def test_timeout_hook_off_by_default(oracle):
    t = random_text(1 << 20, 4, seed=32)
    with Context(0) as c:
        assert np.array_equal(c.build_sa(t, dc=39, sa_width=32), oracle.libsais(t).astype(np.uint64))
        assert c.stats()["lookback_gave_up"] == 0
