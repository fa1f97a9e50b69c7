"""Operands that do not fit the HBM budget (gsparc_sptc_host), through the C ABI.

X is cut into output-row parts and Y into output-column parts, every pair is
contracted and Z must arrive whole and in key order: keys and nnz equal to the
contraction of the whole operands (gsparc_sptc on a context that holds them)
and to the FP64 oracle, values within the bar of tests/value_bar.py.  Parts are
forced by a cap on their size (several X parts, several Y parts, both) or
follow from a small budget on which the whole operands do not fit at all.
"""
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


def check(res, X, Y, cx, cy, whole=None):
    z = ob.sptc(X, Y, cx, cy)
    assert res.nnz == z.nnz and res.ir_nnz == z.ir_nnz
    assert np.array_equal(res.keys, z.keys)
    value_bar.max_rel_err(res.vals, z.vals)
    if whole is not None:
        assert np.array_equal(res.keys, whole.keys)


@pytest.mark.parametrize("split", [(4, 1), (1, 3), (4, 3), (7, 2)])
@pytest.mark.parametrize("case", ["esc_large", "dense_acc", "plain_small"])
def test_forced_parts_give_the_whole_result(ctx, case, split):
    scale = {"esc_large": 0.02, "dense_acc": 0.005, "plain_small": 0.3}[case]
    X, Y, cx, cy = synth.WORKLOADS[case](scale=scale)
    px, py = split
    res = gb.sptc_host(ctx, X, Y, cx, cy, max_part_nnz_x=(X.nnz + px - 1) // px,
                       max_part_nnz_y=(Y.nnz + py - 1) // py)
    st = res.stats
    assert st["x_parts"] >= px and st["y_parts"] >= py, (st["x_parts"], st["y_parts"])
    whole = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    check(res, X, Y, cx, cy, whole)


def test_one_part_each_when_everything_fits(ctx):
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    res = gb.sptc_host(ctx, X, Y, cx, cy)
    assert res.stats["x_parts"] == 1 and res.stats["y_parts"] == 1
    check(res, X, Y, cx, cy)


def test_budget_too_small_for_the_operands():
    X, Y, cx, cy = synth.dense_acc(scale=0.1)  # 1M + 1M nonzeros (56 MB resident), a 200 x 300 output
    with gb.Context(0, hbm_budget=48 << 20) as small:
        with pytest.raises(gb.GsparcError) as e:
            gb.SpTC(X, Y, cx, cy, ctx=small)
        assert e.value.status == 2  # ENOMEM: the whole operands do not fit
        res = gb.sptc_host(small, X, Y, cx, cy)
        assert res.stats["x_parts"] * res.stats["y_parts"] > 1
        assert small.memory()["peak"] <= 48 << 20
    check(res, X, Y, cx, cy)


def test_single_rows_larger_than_a_part_stay_whole(ctx):
    # a cap below the largest row: that row becomes a part of its own
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    res = gb.sptc_host(ctx, X, Y, cx, cy, max_part_nnz_x=16, max_part_nnz_y=X.nnz)
    assert res.stats["x_parts"] > 100
    check(res, X, Y, cx, cy)


def test_discard_sink_counts(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.2)
    res = gb.sptc_host(ctx, X, Y, cx, cy, max_part_nnz_x=X.nnz // 3, max_part_nnz_y=Y.nnz // 2, sink="discard")
    z = ob.sptc(X, Y, cx, cy)
    assert res.nnz == z.nnz and res.ir_nnz == z.ir_nnz and res.keys is None


def test_empty_and_unmatched_operands(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.05)
    E = synth.CooTensor(list(X.dims), np.zeros((X.order, 0), np.uint64), np.zeros(0, np.float32))
    res = gb.sptc_host(ctx, E, Y, cx, cy, max_part_nnz_y=Y.nnz // 2)
    assert res.nnz == 0 and res.ir_nnz == 0


def test_cli_parts_from_host_memory_equal_resident(tmp_path):
    import re
    import subprocess
    X, Y, cx, cy = synth.esc_large(scale=0.01)
    xp = str(tmp_path / "x.tns")
    synth.write_tns(xp, X)
    base = [gb.CLI_PATH, "-X", xp, "-Y", xp, "-c", "2", "-x", *map(str, cx), "-y", *map(str, cy)]
    outs = []
    for extra in ([], ["-P"]):
        zp = str(tmp_path / f"z{len(extra)}.tns")
        r = subprocess.run(base + extra + ["-o", zp], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append((int(re.search(r"^Result NNZ: (\d+)$", r.stderr, re.M).group(1)), open(zp).read()))
    assert outs[0][0] == outs[1][0] > 0
    assert outs[0][1] == outs[1][1]
