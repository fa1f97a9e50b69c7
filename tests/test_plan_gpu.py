"""Plans (gsparc_plan_*) through the C ABI: the coordinate-only work done once,
the numeric pass executed many times, also replayed from a CUDA graph.

Every execution must give the result gsparc_sptc gives for the operands'
current values: keys, order and nnz bit-exact; values within the FP64-oracle
bar of tests/value_bar.py (max relative error <= 1e-5).
"""
import numpy as np
import pytest
import torch

import gsparc_b200 as gb
import oracle_bind as ob
import value_bar
from gsparc_b200 import synth
from gsparc_b200.synth import CooTensor

pytestmark = pytest.mark.gpu



@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


def run_plan(plan, stream=0):
    """All chunks of a plan into one pair of device arrays; returns host copies."""
    keys = torch.empty(max(plan.total, 1), dtype=torch.int64, device="cuda")
    vals = torch.empty(max(plan.total, 1), dtype=torch.float32, device="cuda")
    for k in range(plan.nchunks):
        f, n = plan.chunk(k)
        plan.execute(k, keys[f:f + n], vals[f:f + n], stream=stream)
    torch.cuda.synchronize()
    plan.check()
    return keys[:plan.total].cpu().numpy().view(np.uint64), vals[:plan.total].cpu().numpy()


def check_oracle(keys, vals, X, Y, cx, cy):
    z = ob.sptc(X, Y, cx, cy)
    assert keys.shape[0] == z.nnz
    assert np.array_equal(keys, z.keys)
    value_bar.max_rel_err(vals, z.vals)


@pytest.mark.parametrize("make", [lambda: synth.plain_small(scale=0.2), lambda: synth.esc_large(scale=0.005),
                                  lambda: synth.dense_acc(scale=0.002)])
def test_plan_equals_sptc_and_oracle(ctx, make):
    X, Y, cx, cy = make()
    dx = ctx.upload(X)
    dy = dx if Y is X else ctx.upload(Y)
    plan = gb.Plan(ctx, [(dx, dy, cx, cy)])
    keys, vals = run_plan(plan)
    ref = gb.sptc(ctx, dx, dy, cx, cy)
    assert plan.total == ref.nnz
    assert np.array_equal(keys, ref.keys)
    check_oracle(keys, vals, X, Y, cx, cy)
    # executing again gives the same result
    k2, v2 = run_plan(plan)
    assert np.array_equal(k2, keys) and np.allclose(v2, vals, rtol=1e-6, atol=0)
    plan.close()


def test_plan_in_chunks_equals_one_chunk(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.3)
    dx = ctx.upload(X)
    whole = gb.Plan(ctx, [(dx, dx, cx, cy)])
    parts = gb.Plan(ctx, [(dx, dx, cx, cy)], max_chunk_nnz=max(1, whole.total // 5))
    assert parts.nchunks > 1 and parts.total == whole.total
    k1, v1 = run_plan(whole)
    k2, v2 = run_plan(parts)
    assert np.array_equal(k1, k2)
    assert np.allclose(v1, v2, rtol=1e-6, atol=0)
    whole.close()
    parts.close()


def test_batch_plan_with_wide_keys(ctx):
    d = 1 << 17
    wide = (synth.make_tensor([d, d, d, d], 2000, ["uniform", "uniform", ("zipf", 1.3), ("zipf", 1.3)], "u11", 71),
            synth.make_tensor([d, d, 300], 2000, [("zipf", 1.3), ("zipf", 1.3), "uniform"], "u11", 72), [2, 3], [0, 1])
    inst = synth.batched_instances(10, seed=31, max_nnz=10_000) + [wide]
    dev = [(ctx.upload(X), ctx.upload(Y)) for X, Y, _, _ in inst]
    plan = gb.Plan(ctx, [(dx, dy, cx, cy) for (dx, dy), (_, _, cx, cy) in zip(dev, inst)])
    keys, vals = run_plan(plan)
    for j, (X, Y, cx, cy) in enumerate(inst):
        f, n = plan.job_output(j)
        check_oracle(keys[f:f + n], vals[f:f + n], X, Y, cx, cy)
    plan.close()


def test_plan_picks_up_new_values(ctx):
    X, Y, cx, cy = synth.dense_acc(scale=0.002)
    dx, dy = ctx.upload(X), ctx.upload(Y)
    plan = gb.Plan(ctx, [(dx, dy, cx, cy)])
    rng = np.random.default_rng(3)
    for _ in range(2):
        xv = rng.standard_normal(X.nnz).astype(np.float32)
        yv = rng.standard_normal(Y.nnz).astype(np.float32)
        dx.set_values(xv)
        dy.set_values(yv)
        plan.refresh()
        keys, vals = run_plan(plan)
        check_oracle(keys, vals, CooTensor(X.dims, X.idx, xv), CooTensor(Y.dims, Y.idx, yv), cx, cy)
    plan.close()


def test_plan_replayed_from_a_cuda_graph(ctx):
    X, Y, cx, cy = synth.esc_large(scale=0.005)
    dx = ctx.upload(X)
    plan = gb.Plan(ctx, [(dx, dx, cx, cy)])
    assert plan.nchunks >= 1
    keys = torch.zeros(plan.total, dtype=torch.int64, device="cuda")
    vals = torch.zeros(plan.total, dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
        plan.refresh(stream=s.cuda_stream)
        for k in range(plan.nchunks):
            f, n = plan.chunk(k)
            plan.execute(k, keys[f:f + n], vals[f:f + n], stream=s.cuda_stream)
    ref = gb.sptc(ctx, dx, dx, cx, cy)
    for _ in range(2):
        keys.zero_()
        vals.zero_()
        g.replay()
        torch.cuda.synchronize()
        plan.check()
        assert np.array_equal(keys.cpu().numpy().view(np.uint64), ref.keys)
        check_oracle(keys.cpu().numpy().view(np.uint64), vals.cpu().numpy(), X, X, cx, cy)
    # new values, same graph
    xv = (np.random.default_rng(9).random(X.nnz, dtype=np.float32) - np.float32(0.5)).astype(np.float32)
    dx.set_values(xv)
    g.replay()
    torch.cuda.synchronize()
    Xn = CooTensor(X.dims, X.idx, xv)
    check_oracle(keys.cpu().numpy().view(np.uint64), vals.cpu().numpy(), Xn, Xn, cx, cy)
    del g
    plan.close()


def test_plan_rejects_small_output_arrays(ctx):
    X, _, cx, cy = synth.plain_small(scale=0.05)
    dx = ctx.upload(X)
    plan = gb.Plan(ctx, [(dx, dx, cx, cy)])
    f, n = plan.chunk(0)
    keys = torch.empty(max(n - 1, 1), dtype=torch.int64, device="cuda")
    vals = torch.empty(max(n - 1, 1), dtype=torch.float32, device="cuda")
    with pytest.raises(gb.GsparcError) as e:
        plan.execute(0, keys, vals)
    assert e.value.status == 1
    plan.close()
