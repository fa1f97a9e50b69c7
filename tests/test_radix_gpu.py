"""This library's own radix sort (radix.cu, gsparc_ctx_set_sort(ctx, 1)) against
CUB's and against a stable sort on the host.

The sort orders (key, value) pairs by the low nbits of the key and must be
stable: with values numbering the entries, equal digits must keep their input
order, so keys and values come out identical to numpy's stable argsort and to
CUB.  Sizes cover one entry, tile edges (2048 entries per tile), many tiles and
the headline workload's 3.1M entries; key widths cover a partial digit, whole
digits and all 64 bits, with keys drawn from a small range so that most are
repeated.  A whole contraction run with either sort gives bit-identical
results (both sorts are stable, so every later step sees the same order).
"""
import numpy as np
import pytest
import torch

import golden_cases as gc
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


def sorted_by(ctx, impl, keys, vals, nbits):
    ctx.set_sort(impl)
    try:
        k = torch.from_numpy(keys.view(np.int64).copy()).cuda()
        v = torch.from_numpy(vals.copy()).cuda()
        gb.sort_pairs(ctx, k, v, nbits)
        torch.cuda.synchronize()
        return k.cpu().numpy().view(np.uint64), v.cpu().numpy()
    finally:
        ctx.set_sort(0)


@pytest.mark.parametrize("n", [1, 2, 5, 2047, 2048, 2049, 6145, 100_003, 3_100_000])
@pytest.mark.parametrize("nbits,span", [(1, 2), (7, 50), (8, 256), (13, 3000), (40, 1 << 20), (64, 1 << 62)])
def test_own_sort_is_stable_and_equals_cub(ctx, n, nbits, span):
    rng = np.random.default_rng(n * 131 + nbits)
    keys = rng.integers(0, span, n, dtype=np.uint64)
    if nbits == 64:
        keys |= rng.integers(0, 2, n, dtype=np.uint64) << np.uint64(63)  # the top bit too
    else:
        keys |= rng.integers(0, 4, n, dtype=np.uint64) << np.uint64(nbits)  # bits above nbits ride along
    vals = np.arange(n, dtype=np.float32)  # entry numbers, exact below 2^24
    mask = np.uint64((1 << nbits) - 1) if nbits < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    order = np.argsort(keys & mask, kind="stable")
    k_own, v_own = sorted_by(ctx, 1, keys, vals, nbits)
    assert np.array_equal(v_own, vals[order])
    assert np.array_equal(k_own, keys[order])
    k_cub, v_cub = sorted_by(ctx, 0, keys, vals, nbits)
    assert np.array_equal(k_own, k_cub) and np.array_equal(v_own, v_cub)


def test_empty_and_zero_bits(ctx):
    keys = np.array([5, 3, 9], dtype=np.uint64)
    vals = np.array([0, 1, 2], dtype=np.float32)
    k, v = sorted_by(ctx, 1, keys, vals, 0)  # nothing to sort by: unchanged
    assert np.array_equal(k, keys) and np.array_equal(v, vals)
    k, v = sorted_by(ctx, 1, keys[:0], vals[:0], 8)
    assert k.size == 0


def test_switch_is_validated(ctx):
    assert gb.api.lib().gsparc_ctx_set_sort(ctx._h, 2) != 0  # GSPARC_EINVAL


def contract(ctx, impl, X, Y, cx, cy, accum=0):
    ctx.set_sort(impl)
    try:
        return gb.SpTC(X, Y, cx, cy, dense_accumulator=accum, ctx=ctx)
    finally:
        ctx.set_sort(0)


@pytest.mark.parametrize("name", gc.names())
def test_contraction_identical_with_either_sort(ctx, name):
    X, Y, cx, cy, _, _ = gc.load(name)
    a = contract(ctx, 0, X, Y, cx, cy)
    b = contract(ctx, 1, X, Y, cx, cy)
    assert a.nnz == b.nnz and a.ir_nnz == b.ir_nnz
    assert np.array_equal(a.keys, b.keys)
    assert np.array_equal(a.vals.view(np.uint32), b.vals.view(np.uint32))


@pytest.mark.parametrize("case,scale", [("esc_large", 0.01), ("plain_small", 0.3), ("dense_acc", 0.005)])
def test_workloads_identical_with_either_sort(ctx, case, scale):
    X, Y, cx, cy = synth.WORKLOADS[case](scale=scale)
    a = contract(ctx, 0, X, Y, cx, cy)
    b = contract(ctx, 1, X, Y, cx, cy)
    assert np.array_equal(a.keys, b.keys)
    assert np.array_equal(a.vals.view(np.uint32), b.vals.view(np.uint32))
    z = ob.sptc(X, Y, cx, cy)
    assert np.array_equal(b.keys, z.keys)
    value_bar.max_rel_err(b.vals, z.vals)


def test_batched_identical_with_either_sort(ctx):
    inst = synth.batched_instances(count=16, seed=11, max_nnz=20_000)
    jobs, dev = [], []
    for X, Y, cx, cy in (i[:4] for i in inst):
        dx, dy = ctx.upload(X), ctx.upload(Y)
        dev += [dx, dy]
        jobs.append((dx, dy, cx, cy, 0))
    try:
        a, _ = gb.sptc_batch(ctx, jobs)
        ctx.set_sort(1)
        b, _ = gb.sptc_batch(ctx, jobs)
    finally:
        ctx.set_sort(0)
        for d in dev:
            d.free()
    for ra, rb in zip(a, b):
        assert np.array_equal(ra.keys, rb.keys)
        assert np.array_equal(ra.vals.view(np.uint32), rb.vals.view(np.uint32))
