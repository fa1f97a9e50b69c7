"""FP64 verification on the GPU (gsparc_ctx_set_verify): the max relative error
of every result against FP64 sums of its exact products, stated in the stats.

Checks: with a budget covering the whole contraction every output and every
product is verified, no product misses its output key, and the reported max
relative / absolute errors equal the ones computed on the host against the
FP64 oracle (the two FP64 sums differ only in summation order); both meet the
bar of tests/value_bar.py.  With a smaller budget a seeded sample of rows of
about that many products is verified.  Batched jobs, row shards, keys over 64
bits and every accumulator mode report their own figures; verification off
reports zeros and does not change the result.
"""
import numpy as np
import pytest

import golden_cases as gc
import gsparc_b200 as gb
import oracle_bind as ob
import value_bar
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu

ALL = (1 << 63)


@pytest.fixture
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


def host_errors(vals, z):
    v = np.asarray(vals, np.float64)
    err = np.abs(v - z.vals)
    nz = z.vals != 0
    rel = float(np.max(err[nz] / np.abs(z.vals[nz]))) if nz.any() else 0.0
    return rel, float(err.max()) if err.size else 0.0


def check_full(res, z):
    st = res.stats
    assert st["verified_nnz"] == res.nnz == z.nnz
    assert st["verified_products"] == res.ir_nnz == z.ir_nnz
    assert st["verify_mismatch"] == 0 and st["verify_skipped_rows"] == 0
    rel, ab = host_errors(res.vals, z)
    assert st["max_rel_err"] == pytest.approx(rel, rel=1e-6, abs=1e-12)
    assert st["max_abs_err"] == pytest.approx(ab, rel=1e-6, abs=1e-12)
    assert st["max_rel_err"] <= value_bar.REL
    value_bar.max_rel_err(res.vals, z.vals)


@pytest.mark.parametrize("accum", [0, -1, 1])
@pytest.mark.parametrize("case", ["plain_small", "esc_large", "dense_acc"])
def test_verified_errors_equal_host_errors(ctx, case, accum):
    scale = {"plain_small": 0.3, "esc_large": 0.01, "dense_acc": 0.005}[case]
    X, Y, cx, cy = synth.WORKLOADS[case](scale=scale)
    ctx.set_verify(ALL)
    res = gb.SpTC(X, Y, cx, cy, dense_accumulator=accum, ctx=ctx)
    check_full(res, ob.sptc(X, Y, cx, cy))
    print(f"{case} accum {accum}: max rel err {res.stats['max_rel_err']:.3e}, "
          f"max abs err {res.stats['max_abs_err']:.3e} over {res.nnz} outputs")


@pytest.mark.parametrize("name", [n for n in gc.names()])
def test_verified_on_every_fixture(ctx, name):
    X, Y, cx, cy, _, _ = gc.load(name)
    ctx.set_verify(ALL)
    res = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    check_full(res, ob.sptc(X, Y, cx, cy))


def test_exactly_cancelling_sum_is_verified_exact(ctx):
    X, Y, cx, cy, _, _ = gc.hand_case()
    ctx.set_verify(ALL)
    res = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    check_full(res, ob.sptc(X, Y, cx, cy))
    assert res.stats["max_abs_err"] == 0.0


def test_many_chunks_verified_like_one(ctx):
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    ctx.set_verify(ALL)
    a = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    b = gb.SpTC(X, Y, cx, cy, ctx=ctx, max_chunk_nnz=max(1, a.nnz // 23))
    assert b.stats["chunks"] > 10
    for k in ("verified_nnz", "verified_products", "verify_mismatch"):
        assert a.stats[k] == b.stats[k], k
    # the FP64 sums (double atomics) may add in another order: equal to ~1e-15
    for k in ("max_rel_err", "max_abs_err"):
        assert a.stats[k] == pytest.approx(b.stats[k], rel=1e-6, abs=1e-15), k


def test_sampled_rows_when_over_budget(ctx):
    X, Y, cx, cy = synth.esc_large(scale=0.05)
    ctx.set_verify(2_000_000)
    res = gb.SpTC(X, Y, cx, cy, ctx=ctx, sink="discard")
    st = res.stats
    assert res.ir_nnz > 20 * 2_000_000
    assert 500_000 <= st["verified_products"] <= 8_000_000, st["verified_products"]
    assert 0 < st["verified_nnz"] < res.nnz
    assert st["verify_mismatch"] == 0
    assert 0 < st["max_rel_err"] <= value_bar.REL


def test_off_by_default_and_result_unchanged(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.2)
    a = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    assert a.stats["verified_nnz"] == 0 and a.stats["max_rel_err"] == 0.0
    ctx.set_verify(ALL)
    b = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    ctx.set_verify(0)
    c = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    assert np.array_equal(a.keys, b.keys) and np.array_equal(a.vals, b.vals)
    assert np.array_equal(a.keys, c.keys) and c.stats["verified_nnz"] == 0


def test_batched_jobs_report_their_own_errors(ctx):
    inst = synth.batched_instances(12, seed=31, max_nnz=20_000)
    dev = [(ctx.upload(X), ctx.upload(Y)) for X, Y, _, _ in inst]
    try:
        ctx.set_verify(ALL)
        jobs = [(dx, dy, cx, cy) for (dx, dy), (_, _, cx, cy) in zip(dev, inst)]
        res, bst = gb.sptc_batch(ctx, jobs)
        worst = 0.0
        for r, (X, Y, cx, cy) in zip(res, inst):
            z = ob.sptc(X, Y, cx, cy)
            check_full(r, z)
            worst = max(worst, r.stats["max_rel_err"])
        assert bst["max_rel_err"] == worst
        assert bst["verified_nnz"] == sum(r.nnz for r in res)
    finally:
        for dx, dy in dev:
            dx.free()
            dy.free()


def test_row_shards_are_verified(ctx):
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    dx = ctx.upload(X)
    try:
        ctx.set_verify(ALL)
        whole = gb.sptc(ctx, dx, dx, cx, cy)
        got = 0
        for k in range(3):
            r = gb.sptc(ctx, dx, dx, cx, cy, shard=k, nshards=3)
            assert r.stats["verified_nnz"] == r.nnz
            assert r.stats["verify_mismatch"] == 0
            assert r.stats["max_rel_err"] <= value_bar.REL
            got += r.stats["verified_products"]
        assert got == whole.ir_nnz
    finally:
        dx.free()


def test_keys_over_64_bits_are_verified(ctx):
    X, Y, cx, cy, _, _ = gc.load("wide_keys")
    ctx.set_verify(ALL)
    res = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    check_full(res, ob.sptc(X, Y, cx, cy))
