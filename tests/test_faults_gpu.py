"""Failure paths driven by host-side fault injection (no GPU fault involved):
an allocator armed to fail its nth device allocation (gsparc_ctx_inject_alloc_
failure / gsparc_serve_inject_alloc_failure) makes the engine meet an
out-of-memory condition at every allocation site of a contraction in turn.

Checks: every injected failure returns GSPARC_ENOMEM (the reference exit()s
instead, src/gsparc/cuda_memory.cpp:78), leaves no device memory allocated,
and the next call on the same context gives the same result as before; in a
batch the failing group's jobs report ENOMEM and a later batch succeeds; a
served batch that meets the failure retries each of its requests alone, and
every request completes with the result it has alone.
"""
import numpy as np
import pytest

import gsparc_b200 as gb
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu


def _same_vals(a, b):
    """Two runs of the same contraction: atomics may add a row's products in
    another order, which the compensated sums absorb to within an ulp."""
    return np.allclose(np.asarray(a, np.float64), np.asarray(b, np.float64), rtol=1e-6, atol=0)

ENOMEM = 2


@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


def test_every_allocation_site_fails_cleanly(ctx):
    X, Y, cx, cy = synth.esc_large(scale=0.005)
    dx = ctx.upload(X)
    try:
        base = gb.sptc(ctx, dx, dx, cx, cy)
        in_use = ctx.memory()["in_use"]
        nth, failed = 1, 0
        while True:
            ctx.inject_alloc_failure(nth)
            try:
                r = gb.sptc(ctx, dx, dx, cx, cy)
            except gb.GsparcError as e:
                assert e.status == ENOMEM, e
                assert "injected" in str(e)
                failed += 1
                assert ctx.memory()["in_use"] == in_use, f"allocation {nth}: memory not returned"
                nth += 1
                assert nth < 400
                continue
            ctx.inject_alloc_failure(0)
            break
        assert failed >= 10  # a contraction allocates at many sites
        assert np.array_equal(r.keys, base.keys) and _same_vals(r.vals, base.vals)
        again = gb.sptc(ctx, dx, dx, cx, cy)
        assert np.array_equal(again.keys, base.keys) and _same_vals(again.vals, base.vals)
    finally:
        dx.free()


def test_batch_group_failure_reports_enomem_and_recovers(ctx):
    inst = synth.batched_instances(6, seed=41, max_nnz=20_000)
    dev = [(ctx.upload(X), ctx.upload(Y)) for X, Y, _, _ in inst]
    try:
        jobs = [(dx, dy, cx, cy) for (dx, dy), (_, _, cx, cy) in zip(dev, inst)]
        good, _ = gb.sptc_batch(ctx, jobs)
        ctx.inject_alloc_failure(3)
        res, _ = gb.sptc_batch(ctx, jobs, raise_on_error=False)
        assert any(r.stats["status"] == ENOMEM for r in res)
        assert all(r.stats["status"] in (0, ENOMEM) for r in res)
        for r, g in zip(res, good):
            if r.stats["status"] == 0:
                assert np.array_equal(r.keys, g.keys)
        after, _ = gb.sptc_batch(ctx, jobs)
        for r, g in zip(after, good):
            assert np.array_equal(r.keys, g.keys) and _same_vals(r.vals, g.vals)
    finally:
        for dx, dy in dev:
            dx.free()
            dy.free()


def test_served_batch_meeting_enomem_retries_each_request_alone(ctx):
    inst = synth.batched_instances(8, seed=43, max_nnz=20_000)
    alone = []
    for X, Y, cx, cy in inst:
        dx, dy = ctx.upload(X), ctx.upload(Y)
        alone.append(gb.sptc(ctx, dx, dy, cx, cy))
        dx.free()
        dy.free()
    with gb.Server(0, lanes=1) as srv:
        ops = [(srv.upload(X), srv.upload(Y)) for X, Y, _, _ in inst]
        srv.pause(True)
        tickets = [srv.submit(dx, dy, cx, cy) for (dx, dy), (_, _, cx, cy) in zip(ops, inst)]
        srv.inject_alloc_failure(2)  # the batch of all eight meets it; the retries do not
        srv.pause(False)
        results = [srv.wait(t, timeout_ms=120_000) for t in tickets]
        st = srv.stats()
    assert st["batches"] == 1 and st["max_batch"] == len(inst)
    assert 1 <= st["retries"] <= len(inst)  # the jobs of the group that met the failure
    assert st["completed"] == len(inst) and st["failed"] == 0
    for r, a in zip(results, alone):
        assert r.stats["status"] == 0
        assert np.array_equal(r.keys, a.keys) and _same_vals(r.vals, a.vals)


def test_pause_holds_requests_until_resumed():
    X, Y, cx, cy = synth.plain_small(scale=0.02)
    with gb.Server(0, lanes=2) as srv:
        dx = srv.upload(X)
        srv.pause(True)
        t = srv.submit(dx, dx, cx, cy)
        with pytest.raises(gb.GsparcError):
            srv.wait(t, timeout_ms=300)  # still queued
        srv.pause(False)
        r = srv.wait(t, timeout_ms=60_000)
        assert r.stats["status"] == 0 and r.nnz > 0
