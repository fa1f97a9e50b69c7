"""Serving (gsparc_serve_*) through the C ABI: continuous batching of
requests over resident operands, admission by HBM budget.

Every request's result must equal the same contraction run alone
(gsparc_sptc): keys, order and nnz bit-exact; values of both within the
FP64-oracle bar of tests/value_bar.py (max relative error <= 1e-5).
"""
import threading
import time

import numpy as np
import pytest

import gsparc_b200 as gb
import oracle_bind as ob
import value_bar
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu



@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def mixed():
    return synth.batched_instances(count=32, seed=21, max_nnz=20_000)


@pytest.fixture(scope="module")
def alone(ctx, mixed):
    out = []
    for X, Y, cx, cy in mixed:
        dx, dy = ctx.upload(X), ctx.upload(Y)
        out.append(gb.sptc(ctx, dx, dy, cx, cy))
        dx.free()
        dy.free()
    return out


def same_result(r, a, X, Y, cx, cy, oracle=False):
    assert r.stats["status"] == 0
    assert r.nnz == a.nnz and r.ir_nnz == a.ir_nnz
    assert np.array_equal(r.keys, a.keys)
    if oracle:
        z = ob.sptc(X, Y, cx, cy)
        assert np.array_equal(r.keys, z.keys)
        value_bar.max_rel_err(r.vals, z.vals)
        value_bar.max_rel_err(a.vals, z.vals)


def test_each_result_same_alone_and_in_the_mix(mixed, alone):
    with gb.Server(0, lanes=2) as srv:
        ops = [(srv.upload(X), srv.upload(Y)) for X, Y, _, _ in mixed]
        tickets = [srv.submit(dx, dy, cx, cy) for (dx, dy), (_, _, cx, cy) in zip(ops, mixed)]
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
        for i, (r, a, (X, Y, cx, cy)) in enumerate(zip(res, alone, mixed)):
            same_result(r, a, X, Y, cx, cy, oracle=i < 8)
        assert st["completed"] == len(mixed) and st["failed"] == 0
        assert st["ir_nnz"] == sum(a.ir_nnz for a in alone)
        assert st["nnz"] == sum(a.nnz for a in alone)
        # everything was queued before the lanes could drain it: batches formed
        assert st["batches"] < len(mixed)
        assert st["max_batch"] > 1
        assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]


def test_poisson_arrivals_overlap_and_match(mixed, alone):
    """Requests arrive from another thread while earlier ones run."""
    rng = np.random.default_rng(5)
    gaps = rng.exponential(1.0 / 2000.0, size=len(mixed))  # mean 2k requests/s
    with gb.Server(0, lanes=2) as srv:
        ops = [(srv.upload(X), srv.upload(Y)) for X, Y, _, _ in mixed]
        tickets = [None] * len(mixed)

        def client():
            for i, ((dx, dy), (_, _, cx, cy)) in enumerate(zip(ops, mixed)):
                time.sleep(gaps[i])
                tickets[i] = srv.submit(dx, dy, cx, cy)
        th = threading.Thread(target=client)
        th.start()
        th.join()
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
        for r, a, (X, Y, cx, cy) in zip(res, alone, mixed):
            same_result(r, a, X, Y, cx, cy)
        assert st["completed"] == len(mixed)
        assert st["products_per_s"] > 0 and st["wall_ms"] > 0


def test_output_larger_than_admitted_memory_streams_in_chunks(ctx):
    """A request whose output exceeds the server's whole budget is partitioned."""
    X, _, cx, cy = synth.plain_small(scale=1.0)
    dx = ctx.upload(X)
    a = gb.sptc(ctx, dx, dx, cx, cy)
    dx.free()
    out_bytes = 12 * a.nnz
    budget = 200 << 20
    assert out_bytes > budget // 2
    with gb.Server(0, hbm_budget=budget, lanes=1) as srv:
        sx = srv.upload(X)
        r = srv.wait(srv.submit(sx, sx, cx, cy))
        assert r.stats["chunks"] > 1
        same_result(r, a, X, X, cx, cy)
        assert srv.stats()["peak_reserved_bytes"] <= budget


def test_admission_respects_the_budget(mixed, alone):
    budget = 1 << 30
    with gb.Server(0, hbm_budget=budget, lanes=3, max_batch_jobs=4) as srv:
        ops = [(srv.upload(X), srv.upload(Y)) for X, Y, _, _ in mixed]
        tickets = [srv.submit(dx, dy, cx, cy) for (dx, dy), (_, _, cx, cy) in zip(ops, mixed)]
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
        assert st["max_batch"] <= 4
        assert st["peak_reserved_bytes"] + st["resident_bytes"] <= budget
        for r, a, (X, Y, cx, cy) in zip(res, alone, mixed):
            same_result(r, a, X, Y, cx, cy)


def test_failed_request_fails_alone(mixed, alone):
    X, Y, cx, cy = mixed[0]
    # contract modes of 1 bit against Y's contract modes of >= 6 bits: EINVAL
    bad = synth.make_tensor([4096, 2, 2], 500, ["uniform"] * 3, "u11", 9)
    with gb.Server(0) as srv:
        sx, sy, sb = srv.upload(X), srv.upload(Y), srv.upload(bad)
        t0 = srv.submit(sx, sy, cx, cy)
        t1 = srv.submit(sb, sy, [1, 2][:len(cx)], cy)
        t2 = srv.submit(sx, sy, cx, cy)
        r0 = srv.wait(t0)
        r1 = srv.wait(t1, raise_on_error=False)
        r2 = srv.wait(t2)
        assert r1.stats["status"] != 0
        same_result(r0, alone[0], X, Y, cx, cy)
        same_result(r2, alone[0], X, Y, cx, cy)
        assert srv.stats()["failed"] == 1


def test_release_waits_for_pending_requests(mixed, alone):
    X, Y, cx, cy = mixed[1]
    with gb.Server(0) as srv:
        sx, sy = srv.upload(X), srv.upload(Y)
        ts = [srv.submit(sx, sy, cx, cy) for _ in range(4)]
        sx.release()  # freed once the four requests are done
        for t in ts:
            same_result(srv.wait(t), alone[1], X, Y, cx, cy)
        with pytest.raises(gb.GsparcError):
            srv.submit(sx, sy, cx, cy)  # handle is gone
        before = srv.stats()["resident_bytes"]
        sy.release()
        assert srv.stats()["resident_bytes"] < before


def test_wait_timeout_and_unknown_ticket(mixed):
    with gb.Server(0) as srv:
        with pytest.raises(gb.GsparcError):
            srv.wait(12345, timeout_ms=1.0)
        X, Y, cx, cy = mixed[2]
        sx, sy = srv.upload(X), srv.upload(Y)
        t = srv.submit(sx, sy, cx, cy)
        r = srv.wait(t, timeout_ms=60_000.0)
        assert r.stats["status"] == 0


def test_small_requests_complete_before_the_batch_ends(ctx, mixed, alone):
    """A batch is cut at job boundaries: the small requests of a batch are
    delivered while its larger ones still run, with unchanged results."""
    big = [synth.esc_large(scale=0.06, seed=s) for s in (1, 2, 3)]
    big_alone = []
    for X, _, cx, cy in big:
        dx = ctx.upload(X)
        big_alone.append(gb.sptc(ctx, dx, dx, cx, cy))
        dx.free()
    with gb.Server(0, lanes=1) as srv:
        sb = [srv.upload(X) for X, _, _, _ in big]
        ss = [(srv.upload(X), srv.upload(Y)) for X, Y, _, _ in mixed[:5]]
        # hold the lane with one request so the rest queue up and form one batch
        t_hold = srv.submit(sb[0], sb[0], big[0][2], big[0][3])
        tb = [srv.submit(x, x, b[2], b[3]) for x, b in zip(sb, big)]
        ts = [srv.submit(dx, dy, m[2], m[3]) for (dx, dy), m in zip(ss, mixed[:5])]
        same_result(srv.wait(t_hold), big_alone[0], big[0][0], big[0][0], big[0][2], big[0][3])
        rb = [srv.wait(t) for t in tb]
        rs = [srv.wait(t) for t in ts]
        for r, a, b in zip(rb, big_alone, big):
            same_result(r, a, b[0], b[0], b[2], b[3])
        for r, a, m in zip(rs, alone[:5], mixed[:5]):
            same_result(r, a, *m)
        # the batch runs small requests first and is cut after the first
        # large one, so the small requests finish before the last large one
        assert max(r.stats["t_total_ms"] for r in rs) < max(r.stats["t_total_ms"] for r in rb)


def test_served_stream_orders_3_to_5_with_wide_keys(ctx):
    """The served workload's mix (operand orders 3-5, some operand keys over 64
    bits) through the server: every result equal to the contraction alone."""
    inst, arrive = synth.served_stream(count=24, seed=8, max_nnz=20_000, min_nnz=2_000)
    assert {X.order for X, _, _, _ in inst} | {Y.order for _, Y, _, _ in inst} >= {3, 4, 5}
    with gb.Server(0) as srv:
        ops = [(srv.upload(X), srv.upload(Y)) for X, Y, _, _ in inst]
        tickets = []
        t0 = time.perf_counter()
        for i, ((dx, dy), (_, _, cx, cy)) in enumerate(zip(ops, inst)):
            d = t0 + arrive[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(srv.submit(dx, dy, cx, cy))
        res = [srv.wait(t) for t in tickets]
    for r, (X, Y, cx, cy) in zip(res, inst):
        dx, dy = ctx.upload(X), ctx.upload(Y)
        a = gb.sptc(ctx, dx, dy, cx, cy)
        dx.free()
        dy.free()
        same_result(r, a, X, Y, cx, cy, oracle=X.nnz * Y.nnz < 4e8)
