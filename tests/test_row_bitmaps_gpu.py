"""Heavy rows' column bitmaps kept from the symbolic to the numeric pass
(gsparc_ctx_set_row_bitmaps).

With the bitmaps kept, the numeric pass of a heavy row marks nothing: its
windows load the row's bitmap, end exactly after the window's capacity of
columns and find every run's part with that end.  Without them every window
marks its columns from the products.  Both must give the same output keys
(bit-exact, in the same order), the same nnz and matched products, and values
within the FP64 bar of tests/value_bar.py against the oracle.

Cases: the large-output ESC workload at reduced scale; rows with more runs
than one batch of the run search (512); rows whose ranks have gaps wider than
a window (empty windows) next to a row with a dense stretch; window capacity
256 (every window cut, the next one starting inside a bitmap word); batched
jobs; the golden fixtures.
"""
import numpy as np
import pytest

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


def both(ctx, X, Y, cx, cy, accum=0):
    dx = ctx.upload(X)
    dy = dx if Y is X else ctx.upload(Y)
    try:
        ctx.set_row_bitmaps(True)
        on = gb.sptc(ctx, dx, dy, cx, cy, accum)
        ctx.set_row_bitmaps(False)
        off = gb.sptc(ctx, dx, dy, cx, cy, accum)
    finally:
        ctx.set_row_bitmaps(True)
        dx.free()
        if dy is not dx:
            dy.free()
    return on, off


def check(on, off, X, Y, cx, cy):
    assert on.nnz == off.nnz and on.ir_nnz == off.ir_nnz
    assert np.array_equal(on.keys, off.keys)
    assert off.stats["kept_bitmap_bytes"] == 0
    z = ob.sptc(X, Y, cx, cy)
    assert on.nnz == z.nnz and on.ir_nnz == z.ir_nnz
    assert np.array_equal(on.keys, z.keys)
    value_bar.max_rel_err(on.vals, z.vals)
    value_bar.max_rel_err(off.vals, z.vals)


def many_runs(seed=3):
    """3 rows x 3000 contract keys; every Y run has 20 columns of 50,000."""
    rng = np.random.default_rng(seed)
    nc, nf, per = 3000, 50_000, 20
    f, c = np.meshgrid(np.arange(3), np.arange(nc), indexing="ij")
    X = synth.CooTensor([3, nc], np.stack([f.ravel(), c.ravel()]).astype(np.uint64),
                        rng.uniform(-1, 1, f.size).astype(np.float32))
    yc = np.repeat(np.arange(nc), per)
    yj = np.concatenate([rng.choice(nf, per, replace=False) for _ in range(nc)])
    Y = synth.CooTensor([nc, nf], np.stack([yc, yj]).astype(np.uint64),
                        rng.uniform(-1, 1, yc.size).astype(np.float32))
    return X, Y, [1], [0]


def gapped(seed=4):
    """Row 0 touches only the lowest and highest 100 ranks of 300,200 (a gap of
    300,000 ranks, wider than two windows); row 2 also takes the 300,000 middle
    ranks through one long run; row 1 has that run alone (a single-run row)."""
    rng = np.random.default_rng(seed)
    nf = 1_000_000
    ends = np.concatenate([np.arange(100), np.arange(nf - 100, nf)])
    yc = [np.repeat(np.arange(400), ends.size), np.full(300_000, 400)]
    yj = [np.tile(ends, 400), 100 + 3 * np.arange(300_000)]
    yc, yj = np.concatenate(yc), np.concatenate(yj)
    Y = synth.CooTensor([401, nf], np.stack([yc, yj]).astype(np.uint64),
                        rng.uniform(-1, 1, yc.size).astype(np.float32))
    xf = np.concatenate([np.zeros(400), [1], [2, 2]])
    xc = np.concatenate([np.arange(400), [400], [0, 400]])
    X = synth.CooTensor([3, 401], np.stack([xf, xc]).astype(np.uint64),
                        rng.uniform(-1, 1, xf.size).astype(np.float32))
    return X, Y, [1], [0]


@pytest.mark.parametrize("scale", [0.01, 0.03])
def test_esc_large_same_with_and_without_bitmaps(ctx, scale):
    X, _, cx, cy = synth.esc_large(scale=scale, seed=1)
    on, off = both(ctx, X, X, cx, cy)
    assert on.stats["kept_bitmap_bytes"] > 0
    check(on, off, X, X, cx, cy)
    print(f"scale {scale}: kept {on.stats['kept_bitmap_bytes']} B, windows {on.stats['heavy_windows']} "
          f"(marking: {off.stats['heavy_windows']})")


@pytest.mark.parametrize("accum", [0, 1])
def test_rows_with_more_runs_than_one_batch(ctx, accum):
    X, Y, cx, cy = many_runs()
    on, off = both(ctx, X, Y, cx, cy, accum)
    assert on.stats["heavy_rows"] == 3 and on.stats["kept_bitmap_bytes"] > 0
    check(on, off, X, Y, cx, cy)


def test_gaps_wider_than_a_window(ctx):
    X, Y, cx, cy = gapped()
    on, off = both(ctx, X, Y, cx, cy)
    assert on.stats["kept_bitmap_bytes"] > 0
    check(on, off, X, Y, cx, cy)


@pytest.mark.parametrize("case", ["esc", "many_runs", "gapped"])
def test_every_window_cut(ctx, case):
    if case == "esc":
        X, Y, cx, cy = synth.esc_large(scale=0.01, seed=2)[:4]
        Y = X
    else:
        X, Y, cx, cy = many_runs() if case == "many_runs" else gapped()
    ctx.set_tiles(0, 256)
    try:
        on, off = both(ctx, X, Y, cx, cy)
    finally:
        ctx.set_tiles(0, 0)
    check(on, off, X, Y, cx, cy)


def test_batched_jobs_same_with_and_without_bitmaps(ctx):
    inst = synth.batched_instances(count=24, seed=11, max_nnz=20_000)
    jobs, dev = [], []
    for X, Y, cx, cy in (i[:4] for i in inst):
        dx, dy = ctx.upload(X), ctx.upload(Y)
        dev += [dx, dy]
        jobs.append((dx, dy, cx, cy, 0))
    try:
        ctx.set_row_bitmaps(True)
        on, _ = gb.sptc_batch(ctx, jobs)
        ctx.set_row_bitmaps(False)
        off, _ = gb.sptc_batch(ctx, jobs)
    finally:
        ctx.set_row_bitmaps(True)
        for d in dev:
            d.free()
    for item, a, b in zip(inst, on, off):
        assert a.nnz == b.nnz and np.array_equal(a.keys, b.keys)
        z = ob.sptc(*item[:4])
        assert np.array_equal(a.keys, z.keys)
        value_bar.max_rel_err(a.vals, z.vals)


@pytest.mark.parametrize("name", gc.names())
def test_golden_fixtures_without_bitmaps(ctx, name):
    X, Y, cx, cy, _, _ = gc.load(name)
    on, off = both(ctx, X, Y, cx, cy)
    check(on, off, X, Y, cx, cy)


def test_switch_is_validated(ctx):
    assert gb.api.lib().gsparc_ctx_set_row_bitmaps(ctx._h, 2) != 0  # GSPARC_EINVAL
