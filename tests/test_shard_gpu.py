"""Row shards of one contraction (gsparc_sptc_shard, the per-GPU partition
loop of the reference, include/gsparc/sptc.cuh:42-52), run one after another
on cuda:0 through the C ABI.

Each shard contracts a contiguous range of output rows (X free indices) of
about equal matched-product mass (gsparc_plan_shards); the shards' outputs are
disjoint and ordered by shard, so their concatenation must equal the whole
contraction (gsparc_sptc) and the FP64 oracle: keys and nnz exact, values
equal to the whole run's within an ulp (every row is computed the same way,
up to the order in which atomics add its products), and the shards' product
counts must add up.  The CLI's -g G -e (G shards on one
device) must print the same Result NNZ and write the same Z as -g 1.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import gsparc_b200 as gb
import oracle_bind as ob
import value_bar
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu


def _same_vals(a, b):
    """Two runs of the same contraction: atomics may add a row's products in
    another order, which the compensated sums absorb to within an ulp."""
    return np.allclose(np.asarray(a, np.float64), np.asarray(b, np.float64), rtol=1e-6, atol=0)


@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


CASES = {
    "esc_large_s002": lambda: synth.esc_large(scale=0.02),
    "plain_small_s03": lambda: synth.plain_small(scale=0.3),
    "dense_acc_s0005": lambda: synth.dense_acc(scale=0.005),
}


@pytest.mark.parametrize("nshards", [2, 3, 5])
@pytest.mark.parametrize("case", sorted(CASES))
def test_shards_concatenate_into_the_whole_contraction(ctx, case, nshards):
    X, Y, cx, cy = CASES[case]()
    dx = ctx.upload(X)
    dy = dx if Y is X else ctx.upload(Y)
    try:
        whole = gb.sptc(ctx, dx, dy, cx, cy)
        parts = [gb.sptc(ctx, dx, dy, cx, cy, shard=k, nshards=nshards) for k in range(nshards)]
    finally:
        dx.free()
        if dy is not dx:
            dy.free()
    keys = np.concatenate([p.keys for p in parts])
    vals = np.concatenate([p.vals for p in parts])
    assert sum(p.nnz for p in parts) == whole.nnz
    assert sum(p.ir_nnz for p in parts) == whole.ir_nnz
    assert np.array_equal(keys, whole.keys)
    assert _same_vals(vals, whole.vals)
    z = ob.sptc(X, Y, cx, cy)
    assert np.array_equal(keys, z.keys)
    value_bar.max_rel_err(vals, z.vals)
    # balance by product mass: no shard exceeds its share by more than one row's products
    share = whole.ir_nnz / nshards
    assert max(p.ir_nnz for p in parts) <= share + _max_row_products(X, Y, cx, cy)


def _max_row_products(X, Y, cx, cy):
    _, _, ncx, nfx = ob.layout(X.dims, cx)
    _, _, ncy, nfy = ob.layout(Y.dims, cy)
    xk, _ = ob.sort_pairs(ob.linearize(X, cx, 0), X.val, ncx + nfx)
    yk, _ = ob.sort_pairs(ob.linearize(Y, cy, 1), Y.val, ncy + nfy)
    _, cnt, _ = ob.index_match(xk, ncx, yk, nfy)
    _, inv = np.unique(xk >> np.uint64(ncx), return_inverse=True)
    return int(np.bincount(inv, weights=cnt.astype(np.float64)).max())


def test_more_shards_than_rows(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.01)
    dx = ctx.upload(X)
    try:
        whole = gb.sptc(ctx, dx, dx, cx, cy)
        n = whole.stats["rows"] + 7
        parts = [gb.sptc(ctx, dx, dx, cx, cy, shard=k, nshards=n) for k in range(n)]
    finally:
        dx.free()
    assert np.array_equal(np.concatenate([p.keys for p in parts]), whole.keys)
    assert sum(1 for p in parts if p.nnz == 0) >= 7


def test_bad_shard_arguments_return_statuses(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.01)
    dx = ctx.upload(X)
    try:
        for shard, n in ((2, 2), (-1, 2), (0, 0)):
            with pytest.raises(gb.GsparcError):
                gb.sptc(ctx, dx, dx, cx, cy, shard=shard, nshards=n)
        # the context still works
        assert gb.sptc(ctx, dx, dx, cx, cy).nnz > 0
    finally:
        dx.free()


def _cli(args):
    r = subprocess.run([gb.CLI_PATH, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return int(re.search(r"^Result NNZ: (\d+)$", r.stderr, re.M).group(1))


def test_cli_shards_on_one_device_equal_one_gpu(tmp_path):
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    xp = str(tmp_path / "x.tns")
    synth.write_tns(xp, X)
    base = ["-X", xp, "-Y", xp, "-c", "2", "-x", *map(str, cx), "-y", *map(str, cy)]
    z1, z3 = str(tmp_path / "z1.tns"), str(tmp_path / "z3.tns")
    n1 = _cli(base + ["-g", "1", "-o", z1])
    n3 = _cli(base + ["-g", "3", "-e", "-o", z3])
    assert n1 == n3 > 0
    assert open(z1).read() == open(z3).read()
