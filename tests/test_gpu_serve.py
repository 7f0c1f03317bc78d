"""Serving (continuous batching): requests submitted from several host threads
while other batches run; every result equals the same text's SA built alone
(exact: integer work, no tolerance) and libsais's."""
import threading
import time

import numpy as np
import pytest

from conftest import random_text

pytestmark = pytest.mark.gpu


@pytest.fixture()
def sctx():
    """A fresh context per test: the server starts with the first request and
    reads its options then."""
    from distributed_suffix_sorting_evaluation_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _mixed_requests(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1), np.log(400_000))))
        sigma = int(rng.choice([2, 4, 20, 200]))
        t = random_text(n, sigma, seed=seed * 10_000 + i)
        if i % 9 == 4:  # a repetitive text: recursion inside the mix
            t = np.tile(t[: max(1, n // 50)], 50)[:n]
        out.append(t)
    out += [np.zeros(0, np.uint8), np.frombuffer(b"A", np.uint8)]
    return out


def _wait(ctx, rid):
    from distributed_suffix_sorting_evaluation_b200 import SERVE_DONE
    while True:
        st, lat = ctx.serve_poll(rid)
        if st == SERVE_DONE or st < 0:
            return st, lat
        time.sleep(0.0005)


def test_serve_results_equal_solo(sctx, ctx, oracle):
    sctx.set_option("serve_lanes", 3)
    sctx.set_option("serve_batch_bytes", 600_000)  # several batches, overlapping on the lanes
    texts = _mixed_requests(3, 48)
    ids = [None] * len(texts)

    def submitter(part):
        rng = np.random.default_rng(part)
        for i in range(part, len(texts), 3):
            ids[i] = sctx.serve_submit(texts[i], dc=0, sa_width=32)
            time.sleep(float(rng.exponential(0.002)))

    th = [threading.Thread(target=submitter, args=(p,)) for p in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i, t in enumerate(texts):
        got = sctx.serve_result(ids[i], t.size, 32)
        solo = ctx.build_sa(t, dc=39, sa_width=32) if t.size else np.zeros(0, np.uint64)
        assert np.array_equal(got, solo), (i, t.size)
        assert np.array_equal(got, oracle.libsais(t).astype(np.uint64)), (i, t.size)
        sctx.serve_release(ids[i])
    s = sctx.serve_stats()
    assert s["done"] == len(texts) and s["failed"] == 0
    assert s["batches"] >= 2
    assert s["reserved_bytes"] == 0 and s["queued"] == 0


@pytest.mark.parametrize("width,dc", [(40, 39), (64, 3), (32, 7)])
def test_serve_widths_and_dcs(sctx, oracle, width, dc):
    from distributed_suffix_sorting_evaluation_b200 import unpack_sa
    texts = [random_text(n, 4, seed=n) for n in (10, 3_000, 70_000)]
    ids = [sctx.serve_submit(t, dc=dc, sa_width=width) for t in texts]
    sctx.serve_drain()
    for rid, t in zip(ids, texts):
        out = np.zeros(t.size * width // 8, np.uint8)
        st, lat = sctx.serve_poll(rid, out)
        assert st == 2 and lat > 0
        assert np.array_equal(unpack_sa(out, width, t.size), oracle.libsais(t).astype(np.uint64))
        sctx.serve_release(rid)


def test_serve_budget_admission(sctx, oracle):
    """A budget that holds about two requests at a time: later requests wait for
    releases, all finish, and the reservation never exceeds the budget."""
    from distributed_suffix_sorting_evaluation_b200 import DcxError
    n = 200_000
    budget = 2 * (48 * (n + 1) + (1 << 20) + 2 * n + 4 * n + 1024) + (1 << 20)
    sctx.set_option("serve_budget", budget)
    sctx.set_option("serve_lanes", 2)
    texts = [random_text(n, 4, seed=50 + i) for i in range(6)]
    with pytest.raises(DcxError) as e:
        sctx.serve_submit(np.zeros(10 * n, np.uint8) + 65, dc=0, sa_width=32)
    assert e.value.code == -4  # DCX_ERR_BUDGET: can never fit
    ids = [sctx.serve_submit(t, dc=0, sa_width=32) for t in texts]
    done = 0
    for rid, t in zip(ids, texts):  # release in order: frees room for the waiting requests
        got = sctx.serve_result(rid, n, 32)
        assert np.array_equal(got, oracle.libsais(t).astype(np.uint64))
        sctx.serve_release(rid)
        done += 1
    s = sctx.serve_stats()
    assert s["done"] == 6 and s["peak_reserved_bytes"] <= budget


def test_serve_errors(sctx):
    from distributed_suffix_sorting_evaluation_b200 import DcxError
    rid = sctx.serve_submit(b"ACGTACGT", dc=0, sa_width=32)
    with pytest.raises(DcxError):
        sctx.serve_submit(b"ACGT", dc=4, sa_width=32)  # no difference cover for X = 4
    with pytest.raises(DcxError):
        sctx.serve_submit(b"ACGT", dc=0, sa_width=48)
    st, _ = _wait(sctx, rid)
    assert st == 2
    sctx.serve_release(rid)
    with pytest.raises(DcxError) as e:
        sctx.serve_release(rid)
    assert e.value.code == -9  # DCX_ERR_NOTFOUND


def test_serve_result_device(sctx):
    """The device-resident result passes the GPU checker in place."""
    import torch
    t = random_text(50_000, 4, seed=77)
    rid = sctx.serve_submit(t, dc=0, sa_width=32)
    assert _wait(sctx, rid)[0] == 2
    p = sctx.serve_result_device(rid)
    assert p != 0
    d_text = torch.from_numpy(t).cuda()
    torch.cuda.synchronize()
    assert sctx.check_sa_device(d_text.data_ptr(), t.size, p, 32)
    sctx.serve_release(rid)


def test_serve_drain_reports_stall(sctx, oracle):
    """Unreleased results can hold the whole budget: drain then returns
    DCX_ERR_BUDGET instead of waiting forever, and releases unblock the queue."""
    from distributed_suffix_sorting_evaluation_b200 import DcxError
    n = 100_000
    fp = 48 * (n + 1) + (1 << 20) + ((n + 16 + 255) & ~255) + ((4 * n + 16 + 255) & ~255)
    sctx.set_option("serve_budget", fp + (1 << 20))
    sctx.set_option("serve_lanes", 1)
    texts = [random_text(n, 4, seed=90 + i) for i in range(5)]
    ids = [sctx.serve_submit(t, dc=0, sa_width=32) for t in texts]
    with pytest.raises(DcxError) as e:
        sctx.serve_drain()
    assert e.value.code == -4
    for rid, t in zip(ids[:3], texts[:3]):
        assert np.array_equal(sctx.serve_result(rid, n, 32), oracle.libsais(t).astype(np.uint64))
        sctx.serve_release(rid)
    sctx.serve_drain()
    for rid, t in zip(ids[3:], texts[3:]):
        assert np.array_equal(sctx.serve_result(rid, n, 32), oracle.libsais(t).astype(np.uint64))
        sctx.serve_release(rid)


def test_serve_borrowed_host_and_device(sctx, oracle):
    """Zero-copy submissions: borrowed host and device buffers give the same SAs."""
    import torch
    texts = [random_text(n, 4, seed=300 + n) for n in (5, 4_000, 120_000)]
    hbufs = [torch.from_numpy(t.copy()).pin_memory() for t in texts]
    dbufs = [torch.from_numpy(t.copy()).cuda() for t in texts]
    torch.cuda.synchronize()
    ids = [sctx.serve_submit(None, text_ptr=h.data_ptr(), n=h.numel(), borrow=True) for h in hbufs]
    ids += [sctx.serve_submit(None, text_ptr=d.data_ptr(), n=d.numel(), borrow=True, device=True) for d in dbufs]
    for rid, t in zip(ids, texts + texts):
        assert np.array_equal(sctx.serve_result(rid, t.size, 32), oracle.libsais(t).astype(np.uint64))
        sctx.serve_release(rid)
