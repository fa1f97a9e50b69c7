"""Batched contractions (gsparc_sptc_batch) through the C ABI.

Every job's result must equal the result of the same contraction run alone
(gsparc_sptc): keys, order and nnz bit-exact; values bit-exact where the
accumulation order is fixed and in every case within the FP64-oracle bar
(tests/value_bar.py: max relative error <= 1e-5).
"""
import numpy as np
import pytest

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


def upload_jobs(ctx, inst, accum=0):
    jobs, dev = [], []
    for item in inst:
        X, Y, cx, cy = item[:4]
        a = item[4] if len(item) > 4 else accum
        dx, dy = ctx.upload(X), ctx.upload(Y)
        dev += [dx, dy]
        jobs.append((dx, dy, cx, cy, a))
    return jobs, dev


def free_all(dev):
    for d in dev:
        d.free()


def check_oracle(res, X, Y, cx, cy):
    z = ob.sptc(X, Y, cx, cy)
    assert res.ir_nnz == z.ir_nnz
    assert res.nnz == z.nnz
    assert np.array_equal(res.keys, z.keys)
    value_bar.max_rel_err(res.vals, z.vals)


def check_same_as_alone(ctx, inst, jobs, results):
    for (item, job, r) in zip(inst, jobs, results):
        X, Y, cx, cy = item[:4]
        alone = gb.sptc(ctx, job[0], job[1], cx, cy, job[4])
        assert r.stats["status"] == 0
        assert r.nnz == alone.nnz and r.ir_nnz == alone.ir_nnz
        assert r.stats["rows"] == alone.stats["rows"]
        assert np.array_equal(r.keys, alone.keys)
        check_oracle(r, X, Y, cx, cy)


@pytest.fixture(scope="module")
def mixed():
    return synth.batched_instances(count=48, seed=11, max_nnz=20_000)


def test_batch_equals_each_job_alone(ctx, mixed):
    jobs, dev = upload_jobs(ctx, mixed)
    try:
        res, bst = gb.sptc_batch(ctx, jobs)
        assert bst["status"] == 0
        assert bst["ir_nnz"] == sum(r.ir_nnz for r in res)
        assert bst["nnz"] == sum(r.nnz for r in res)
        check_same_as_alone(ctx, mixed, jobs, res)
    finally:
        free_all(dev)


@pytest.mark.parametrize("accum", [-1, 1])
def test_batch_forced_accumulator(ctx, mixed, accum):
    inst = mixed[:16]
    jobs, dev = upload_jobs(ctx, inst, accum)
    try:
        res, _ = gb.sptc_batch(ctx, jobs)
        check_same_as_alone(ctx, inst, jobs, res)
    finally:
        free_all(dev)


def test_batch_light_values_bit_exact(ctx, mixed):
    # light rows sum each output in a fixed order, so the batched values equal
    # the values of the job run alone bit for bit when no row is heavy
    inst = [m for m in mixed if m[0].nnz < 3000][:12]
    jobs, dev = upload_jobs(ctx, inst, -1)
    try:
        res, _ = gb.sptc_batch(ctx, jobs)
        for job, r in zip(jobs, res):
            alone = gb.sptc(ctx, job[0], job[1], job[2], job[3], -1)
            if alone.stats["heavy_rows"] == 0:
                assert np.array_equal(r.vals, alone.vals)
    finally:
        free_all(dev)


def wide_instance(seed):
    # X keys of 64 bits (4 modes of 2^16): needs a group of its own
    d = 1 << 16
    X = synth.make_tensor([d, d, d, d], 3000, [("zipf", 1.2)] * 4, "u11", seed)
    Y = synth.make_tensor([d, d, 300], 3000, [("zipf", 1.2)] * 3, "u11", seed + 1)
    return (X, Y, [2, 3], [0, 1])


def test_batch_groups_for_wide_keys(ctx, mixed):
    inst = [wide_instance(5), mixed[0], wide_instance(7)] + list(mixed[1:10])
    jobs, dev = upload_jobs(ctx, inst)
    try:
        res, bst = gb.sptc_batch(ctx, jobs)
        assert bst["status"] == 0
        check_same_as_alone(ctx, inst, jobs, res)
    finally:
        free_all(dev)


def test_batch_many_chunks_equal_one_chunk(ctx, mixed):
    inst = mixed[:20]
    jobs, dev = upload_jobs(ctx, inst)
    try:
        a, ba = gb.sptc_batch(ctx, jobs)
        b, bb = gb.sptc_batch(ctx, jobs, max_chunk_nnz=max(1, ba["nnz"] // 23))
        assert bb["chunks"] > 10
        for x, y in zip(a, b):
            assert np.array_equal(x.keys, y.keys)
            assert x.nnz == y.nnz
        check_same_as_alone(ctx, inst, jobs, b)
    finally:
        free_all(dev)


def test_batch_small_staging_rings_each_job(ctx, mixed):
    inst = mixed[:10]
    jobs, dev = upload_jobs(ctx, inst)
    try:
        a, _ = gb.sptc_batch(ctx, jobs)
        b, _ = gb.sptc_batch(ctx, jobs, staging=97)
        for x, y in zip(a, b):
            assert np.array_equal(x.keys, y.keys)
            assert x.stats["nnz"] == y.stats["nnz"]
    finally:
        free_all(dev)


def test_batch_device_sink_per_job(ctx, mixed):
    inst = mixed[:12]
    jobs, dev = upload_jobs(ctx, inst)
    try:
        a, _ = gb.sptc_batch(ctx, jobs)
        got = {}

        def on_chunk(j, k, v, n, first):
            got.setdefault(j, []).append(gb.digest_chunk(k, v, n))
            return 0
        b, _ = gb.sptc_batch(ctx, jobs, sink="device", on_chunk=on_chunk)
        for j, r in enumerate(a):
            digs = got.get(j, [])
            assert sum(d["n"] for d in digs) == r.nnz
            h = int(np.sum(gb.splitmix64(r.keys), dtype=np.uint64))
            assert sum(d["key_hash"] for d in digs) % (1 << 64) == h
    finally:
        free_all(dev)


def test_batch_bad_job_fails_alone(ctx, mixed):
    good = list(mixed[:4])
    X, Y, cx, cy = mixed[4]
    assert cy[0] == 0 and cx[0] == len(X.dims) - len(cx)
    # a contract mode of Y with another bit width than X's: EINVAL on the host
    Yb = CooTensor([Y.dims[0] * 4 + 3] + list(Y.dims[1:]), Y.idx, Y.val)
    # an index outside its (free) mode: caught on the device
    Xo = CooTensor([max(1, X.dims[0] // 2)] + list(X.dims[1:]), X.idx, X.val)
    assert int(X.idx[0].max()) >= Xo.dims[0]
    inst = good[:2] + [(X, Yb, cx, cy)] + good[2:] + [(Xo, Y, cx, cy)]
    jobs, dev = upload_jobs(ctx, inst)
    try:
        res, bst = gb.sptc_batch(ctx, jobs, raise_on_error=False)
        assert bst["status"] == 1
        assert res[2].stats["status"] == 1 and res[2].keys is None
        assert res[-1].stats["status"] == 1 and res[-1].keys is None
        ok = [0, 1, 3, 4]
        check_same_as_alone(ctx, [inst[i] for i in ok], [jobs[i] for i in ok], [res[i] for i in ok])
    finally:
        free_all(dev)


def test_batch_empty_and_unmatched(ctx, mixed):
    res, bst = gb.sptc_batch(ctx, [])
    assert res == [] and bst["status"] == 0 and bst["nnz"] == 0
    X, Y, cx, cy = mixed[0]
    # Y whose contract indices never meet X's
    Yn = CooTensor(Y.dims, Y.idx.copy(), Y.val)
    for m in cy:
        Yn.idx[m] = np.uint64(Y.dims[m] - 1)
    Xn = CooTensor(X.dims, X.idx.copy(), X.val)
    for m in cx:
        Xn.idx[m] = np.uint64(0)
    inst = [(Xn, Yn, cx, cy), mixed[1]]
    jobs, dev = upload_jobs(ctx, inst)
    try:
        res, bst = gb.sptc_batch(ctx, jobs)
        assert res[0].nnz == 0 and res[0].ir_nnz == 0 and res[0].keys.size == 0
        check_same_as_alone(ctx, inst[1:], jobs[1:], res[1:])
    finally:
        free_all(dev)
