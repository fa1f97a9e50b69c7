"""Contractions whose operand keys need more than 64 bits (the reference's
128-bit key path, include/gsparc/tensor_manager.tpp:301-406 and
include/gsparc/indexMatch.cuh:120-229), through the C ABI, against the FP64
oracle.  Bars as everywhere: coordinates, order and nnz bit-exact; values
|z - z64| <= 1e-5 * |z64| + 1e-7 * sum|products|.
"""
import numpy as np
import pytest

import gsparc_b200 as gb
import oracle_bind as ob
from gsparc_b200 import synth
from gsparc_b200.synth import CooTensor

pytestmark = pytest.mark.gpu

REL = 1e-5
ABS = 1e-7


@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


def check(res, X, Y, cx, cy):
    z = ob.sptc(X, Y, cx, cy)
    assert res.ir_nnz == z.ir_nnz
    assert res.nnz == z.nnz
    assert np.array_equal(res.keys, z.keys)
    tol = REL * np.abs(z.vals) + ABS * z.abs_sums
    assert np.all(np.abs(res.vals.astype(np.float64) - z.vals) <= tol)
    return z


def wide_contract(seed):
    # contract part of 66 bits (three 22-bit modes); X key 75 bits, Y key 74
    d = 1 << 22
    X = synth.make_tensor([300, d, d, d], 4000, ["uniform"] + [("zipf", 1.6)] * 3, "u11", seed)
    Y = synth.make_tensor([d, d, d, 200], 4000, [("zipf", 1.6)] * 3 + ["uniform"], "u11", seed + 1)
    return X, Y, [1, 2, 3], [0, 1, 2]


def wide_x_only(seed):
    # X key 17 * 4 = 68 bits, Y key 34 + 9 = 43 bits
    d = 1 << 17
    X = synth.make_tensor([d, d, d, d], 3000, ["uniform", "uniform", ("zipf", 1.3), ("zipf", 1.3)], "u11", seed)
    Y = synth.make_tensor([d, d, 400], 3000, [("zipf", 1.3), ("zipf", 1.3), "uniform"], "u11", seed + 1)
    return X, Y, [2, 3], [0, 1]


def wide_y_only(seed):
    X, Y, cx, cy = wide_x_only(seed)
    return Y, X, cy, cx  # Y's key is the wide one now


@pytest.mark.parametrize("make", [wide_contract, wide_x_only, wide_y_only])
@pytest.mark.parametrize("accum", [0, -1, 1])
def test_wide_keys_match_oracle(ctx, make, accum):
    X, Y, cx, cy = make(5)
    res = gb.SpTC(X, Y, cx, cy, dense_accumulator=accum, ctx=ctx)
    z = check(res, X, Y, cx, cy)
    assert z.ir_nnz > 0
    assert res.stats["nbits_x"] > 64 or res.stats["nbits_y"] > 64


def test_wide_chunked_output_equals_one_chunk(ctx):
    X, Y, cx, cy = wide_x_only(9)
    a = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    b = gb.SpTC(X, Y, cx, cy, ctx=ctx, max_chunk_nnz=max(1, a.nnz // 7))
    assert b.stats["chunks"] > 1
    assert np.array_equal(a.keys, b.keys)
    assert np.array_equal(a.vals, b.vals)


def test_wide_without_matches(ctx):
    d = 1 << 22
    X = CooTensor([8, d, d, d], np.array([[1], [1], [2], [3]], np.uint64), np.ones(1, np.float32))
    Y = CooTensor([d, d, d, 8], np.array([[1], [2], [4], [5]], np.uint64), np.ones(1, np.float32))
    X.idx[:, 0] = [7, d - 1, d - 1, d - 1]
    Y.idx[:, 0] = [d - 1, d - 1, d - 2, 7]
    res = gb.SpTC(X, Y, [1, 2, 3], [0, 1, 2], ctx=ctx)
    assert res.nnz == 0 and res.ir_nnz == 0


def test_wide_bad_index_fails(ctx):
    d = 1 << 22
    X = CooTensor([8, d, d, d], np.array([[1], [1], [2], [d]], np.uint64), np.ones(1, np.float32))
    Y = CooTensor([d, d, d, 8], np.array([[1], [2], [4], [5]], np.uint64), np.ones(1, np.float32))
    with pytest.raises(gb.GsparcError) as e:
        gb.SpTC(X, Y, [1, 2, 3], [0, 1, 2], ctx=ctx)
    assert e.value.status == 1


def test_wide_jobs_in_a_batch(ctx):
    inst = [wide_contract(11), synth.batched_instances(4, seed=13, max_nnz=5000)[0], wide_x_only(17),
            wide_y_only(19)] + synth.batched_instances(6, seed=23, max_nnz=5000)
    dev, jobs = [], []
    for X, Y, cx, cy in inst:
        dx, dy = ctx.upload(X), ctx.upload(Y)
        dev += [dx, dy]
        jobs.append((dx, dy, cx, cy))
    try:
        res, bst = gb.sptc_batch(ctx, jobs)
        assert bst["status"] == 0
        for r, (X, Y, cx, cy) in zip(res, inst):
            check(r, X, Y, cx, cy)
    finally:
        for d in dev:
            d.free()


def test_wide_request_served(ctx):
    X, Y, cx, cy = wide_contract(29)
    with gb.Server(0) as srv:
        sx, sy = srv.upload(X), srv.upload(Y)
        r = srv.wait(srv.submit(sx, sy, cx, cy))
        check(r, X, Y, cx, cy)
