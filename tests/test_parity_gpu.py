"""Parity of the CUDA engine (through the C ABI) with the reference outputs and
the FP64 oracle.

Bars: output coordinates, order and nnz bit-exact; values: max relative error
    |z - z64| / |z64| <= 1e-5
against the FP64 oracle on every output whose FP64 value is nonzero, and
exactly 0 where it is 0 (sums that cancel exactly).  The engine's compensated
FP32 sums (TwoSum of every add plus each product's fma error) are within a few
units in the last place of the exact sum, so this holds with cancelling N(0,1)
sums too.
"""
import numpy as np
import pytest

import golden_cases as gc
import gsparc_b200 as gb
import oracle_bind as ob
from gsparc_b200 import synth
from gsparc_b200.synth import CooTensor

pytestmark = pytest.mark.gpu

REL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


def run(ctx, X, Y, cx, cy, accum=0, **kw):
    return gb.SpTC(X, Y, cx, cy, dense_accumulator=accum, ctx=ctx, **kw)


def check_vs_oracle(res, X, Y, cx, cy):
    z = ob.sptc(X, Y, cx, cy)
    assert res.ir_nnz == z.ir_nnz
    assert res.nnz == z.nnz
    assert np.array_equal(res.keys, z.keys)
    err = np.abs(res.vals.astype(np.float64) - z.vals)
    nz = z.vals != 0
    assert np.all(err[~nz] == 0), "an exactly cancelling sum is not exactly 0"
    rel = float(np.max(err[nz] / np.abs(z.vals[nz]))) if nz.any() else 0.0
    assert rel <= REL, rel
    return rel


@pytest.mark.parametrize("accum", [0, -1, 1])
@pytest.mark.parametrize("name", gc.names())
def test_matches_reference_cpu_sptc(ctx, name, accum):
    X, Y, cx, cy, zi, zv = gc.load(name)
    res = run(ctx, X, Y, cx, cy, accum)
    coords = gb.decode_keys(res.keys, X.dims, Y.dims, cx, cy)
    assert res.nnz == zi.shape[1]
    assert np.array_equal(coords, zi)
    check_vs_oracle(res, X, Y, cx, cy)


@pytest.mark.parametrize("accum", [0, 1])
def test_hand_case(ctx, accum):
    X, Y, cx, cy, zi, zv = gc.hand_case()
    res = run(ctx, X, Y, cx, cy, accum)
    assert np.array_equal(gb.decode_keys(res.keys, X.dims, Y.dims, cx, cy), zi)
    assert np.array_equal(res.vals.astype(np.float64), zv)
    assert res.ir_nnz == 13


@pytest.mark.parametrize("accum", [0, 1, -1])
@pytest.mark.parametrize("case", ["plain_small", "esc_large", "dense_acc"])
def test_workloads_reduced_scale(ctx, case, accum):
    scale = {"plain_small": 1.0, "esc_large": 0.02, "dense_acc": 0.01}[case]
    X, Y, cx, cy = synth.WORKLOADS[case](scale=scale)
    res = run(ctx, X, Y, cx, cy, accum)
    rel = check_vs_oracle(res, X, Y, cx, cy)
    print(f"{case} accum {accum}: max rel err vs FP64 {rel:.3e} over {res.nnz} outputs")


def test_many_output_chunks_equal_one_chunk(ctx):
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    a = run(ctx, X, Y, cx, cy)
    b = run(ctx, X, Y, cx, cy, max_chunk_nnz=max(1, a.nnz // 37))
    assert b.stats["chunks"] > 10
    assert np.array_equal(a.keys, b.keys) and np.array_equal(a.vals, b.vals)


def test_ring_sink_streams_every_chunk(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.3)
    a = run(ctx, X, Y, cx, cy)
    hk = np.zeros(1000, np.uint64)
    hv = np.zeros(1000, np.float32)
    got_k, got_v, firsts = [], [], []

    def on_chunk(k, v, n, first):
        got_k.append(k.copy()); got_v.append(v.copy()); firsts.append(first)
        return 0
    b = run(ctx, X, Y, cx, cy, sink="ring", host_keys=hk, host_vals=hv, on_chunk=on_chunk)
    assert b.nnz == a.nnz and len(firsts) > 1
    assert np.array_equal(np.concatenate(got_k), a.keys)
    assert np.array_equal(np.concatenate(got_v), a.vals)


def test_device_sink_digest(ctx):
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    a = run(ctx, X, Y, cx, cy)
    digs = []

    def on_chunk(k, v, n, first):
        digs.append((first, gb.digest_chunk(k, v, n)))
        return 0
    b = run(ctx, X, Y, cx, cy, sink="device", on_chunk=on_chunk, max_chunk_nnz=a.nnz // 5 + 1)
    assert b.nnz == a.nnz
    assert sum(d["n"] for _, d in digs) == a.nnz
    assert all(d["unsorted"] == 0 for _, d in digs)
    h = int(np.sum(gb.splitmix64(a.keys), dtype=np.uint64))
    assert sum(d["key_hash"] for _, d in digs) % (1 << 64) == h
    assert abs(sum(d["val_sum"] for _, d in digs) - float(np.sum(a.vals, dtype=np.float64))) < 1e-6 * a.nnz


def test_callback_stop_returns_status(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.2)
    with pytest.raises(gb.GsparcError) as e:
        run(ctx, X, Y, cx, cy, sink="device", on_chunk=lambda *a: 1)
    assert e.value.status == 8
    # the context stays usable
    run(ctx, X, Y, cx, cy)


def test_edge_cases(ctx):
    T = lambda dims, idx, val: CooTensor(dims, np.array(idx, np.uint64).reshape(len(dims), -1),
                                         np.array(val, np.float32))
    # empty X
    X = T([4, 5], [[], []], [])
    Y = T([5, 3], [[1, 2], [0, 2]], [1.0, 2.0])
    r = run(ctx, X, Y, [1], [0])
    assert r.nnz == 0 and r.ir_nnz == 0
    # no matching contract keys
    X = T([4, 5], [[0, 1], [0, 1]], [1.0, 2.0])
    Y = T([5, 3], [[3, 4], [0, 2]], [1.0, 2.0])
    r = run(ctx, X, Y, [1], [0])
    assert r.nnz == 0 and r.ir_nnz == 0
    # single nonzero each
    X = T([4, 5], [[3], [4]], [1.5])
    Y = T([5, 3], [[4], [2]], [-2.0])
    r = run(ctx, X, Y, [1], [0])
    assert r.nnz == 1 and r.vals[0] == np.float32(-3.0)
    # size-1 modes (0 bits) on both sides
    X = synth.make_tensor([30, 2, 20], 200, ["uniform"] * 3, "u11", 3)
    X = CooTensor([30, 1, 20], np.stack([X.idx[0], np.zeros_like(X.idx[1]), X.idx[2]]), X.val)
    Y = synth.make_tensor([20, 2, 7], 100, ["uniform", "uniform", "uniform"], "u11", 4)
    Y = CooTensor([20, 1, 7], np.stack([Y.idx[0], np.zeros_like(Y.idx[1]), Y.idx[2]]), Y.val)
    check_vs_oracle(run(ctx, X, Y, [2], [0]), X, Y, [2], [0])


def test_duplicate_coordinates_are_summed(ctx):
    X = synth.make_tensor([40, 60, 30], 3000, ["uniform"] * 3, "u11", 8)
    Y = synth.make_tensor([30, 50], 900, ["uniform"] * 2, "u11", 9)
    Xd = CooTensor(X.dims, np.concatenate([X.idx, X.idx[:, :500]], axis=1),
                   np.concatenate([X.val, X.val[:500] * np.float32(0.5)]))
    Yd = CooTensor(Y.dims, np.concatenate([Y.idx, Y.idx[:, :300]], axis=1),
                   np.concatenate([Y.val, Y.val[:300]]))
    for accum in (0, 1):
        check_vs_oracle(run(ctx, Xd, Yd, [2], [0], accum), Xd, Yd, [2], [0])


def test_64_bit_keys_and_wide_outputs(ctx):
    # X: 4 modes of 2^16 (64 key bits); output key 32 + 32 bits
    rng = np.random.default_rng(11)
    n = 4000
    dims = [1 << 16] * 4
    idx = np.stack([rng.integers(0, 1 << 16, n), rng.integers(0, 1 << 16, n),
                    rng.integers(0, 8, n), rng.integers(0, 8, n)]).astype(np.uint64)
    idx[:, 0] = [(1 << 16) - 1] * 4
    X = CooTensor(dims, idx, rng.random(n, dtype=np.float32))
    check_vs_oracle(run(ctx, X, X, [2, 3], [2, 3]), X, X, [2, 3], [2, 3])


def test_bad_inputs_return_status(ctx):
    X = CooTensor([4, 5], np.array([[0, 9], [0, 1]], np.uint64), np.ones(2, np.float32))
    Y = CooTensor([5, 3], np.array([[1], [2]], np.uint64), np.ones(1, np.float32))
    with pytest.raises(gb.GsparcError) as e:
        run(ctx, X, Y, [1], [0])
    assert e.value.status == 1
    Y2 = CooTensor([9, 3], np.array([[1], [2]], np.uint64), np.ones(1, np.float32))
    X2 = CooTensor([4, 5], np.array([[0], [1]], np.uint64), np.ones(1, np.float32))
    with pytest.raises(gb.GsparcError):
        run(ctx, X2, Y2, [1], [0])  # contract modes 5 vs 9: 3 vs 4 bits
    run(ctx, X2, CooTensor([5, 3], Y.idx, Y.val), [1], [0])


def test_same_result_alone_and_after_other_work(ctx):
    X, Y, cx, cy = synth.dense_acc(scale=0.003)
    a = run(ctx, X, Y, cx, cy)
    run(ctx, *synth.esc_large(scale=0.01))
    b = run(ctx, X, Y, cx, cy)
    assert np.array_equal(a.keys, b.keys)
    assert np.allclose(a.vals, b.vals, rtol=1e-6, atol=0)


def test_reserved_pool_gives_the_same_result(ctx):
    """gsparc_ctx_reserve maps the budget up front; results do not change."""
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    a = run(ctx, X, Y, cx, cy)
    with gb.Context(0, hbm_budget=4 << 30) as c2:
        c2.reserve()
        assert c2.memory()["in_use"] == 0
        b = run(c2, X, Y, cx, cy)
        c2.reserve(1 << 30)  # again, smaller: nothing changes
        c = run(c2, X, Y, cx, cy)
    assert np.array_equal(a.keys, b.keys) and np.array_equal(a.vals, b.vals)
    assert np.array_equal(a.keys, c.keys) and np.array_equal(a.vals, c.vals)
