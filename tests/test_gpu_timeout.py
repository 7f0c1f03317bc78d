"""Failure detection without a GPU fault: the onesweep look-back is the only
device-side wait, and it gives up after `spin_limit` polls.  With the limit at
0 a CTA that finds its predecessor unpublished gives up at once; the kernel
records DEV_ERR_TIMEOUT, keeps every write in range, and the build returns
DCX_ERR_TIMEOUT right after that sort.  The context stays usable: the same
text then builds correctly with the default limit."""
import numpy as np
import pytest

from conftest import random_text
from distributed_suffix_sorting_evaluation_b200 import DCX_ERR_TIMEOUT, Context, DcxError

pytestmark = pytest.mark.gpu


def test_lookback_gives_up_cleanly(oracle):
    t = random_text(16 << 20, 4, seed=31)  # ~5,500 tiles per pass
    want = oracle.libsais(t).astype(np.uint64)
    with Context(0) as c:
        c.set_option("spin_limit", 0)
        try:
            got = c.build_sa(t, dc=39, sa_width=32)
        except DcxError as e:
            assert e.code == DCX_ERR_TIMEOUT, e
        else:  # no CTA ever had to wait: then the result is simply right
            assert np.array_equal(got, want)
        c.set_option("spin_limit", 1 << 24)
        assert np.array_equal(c.build_sa(t, dc=39, sa_width=32), want)
