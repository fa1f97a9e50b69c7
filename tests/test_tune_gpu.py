"""The measured autotuner (gsparc_autotune) through the C ABI: it returns one of
the candidates it timed, remembers its choice per operand shape, and a
contraction run with the chosen settings (accumulator, tiles, output chunk)
gives the same result as the default (keys exact, values within the bar of
tests/value_bar.py against the FP64 oracle)."""
import subprocess

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


@pytest.mark.parametrize("make", [lambda: synth.plain_small(scale=0.3), lambda: synth.dense_acc(scale=0.002),
                                  lambda: synth.esc_large(scale=0.02)])
def test_autotune_choice_and_result(ctx, make):
    X, Y, cx, cy = make()
    dx = ctx.upload(X)
    dy = dx if Y is X else ctx.upload(Y)
    try:
        t = gb.autotune(ctx, dx, dy, cx, cy, retune=True)
        assert not t["cached"] and len(t["candidates"]) >= 2
        choice = (t["accum"], t["max_chunk_nnz"], t["ms"], t["light_row_max"], t["heavy_window_cap"])
        assert choice in [tuple(c) for c in t["candidates"]]
        assert t["ms"] == min(c[2] for c in t["candidates"])
        assert {c[0] for c in t["candidates"]} == {-1, 1}
        # tile candidates: the heavy window at half its outputs, and for ESC the on-chip row limit
        half = [c[4] for c in t["candidates"] if c[4]]
        assert half, t["candidates"]
        if t["accum"] == -1:
            assert {256, 2048} <= {c[3] for c in t["candidates"]}
        again = gb.autotune(ctx, dx, dy, cx, cy)
        assert again["cached"] and again["accum"] == t["accum"] and again["max_chunk_nnz"] == t["max_chunk_nnz"]
        base = gb.sptc(ctx, dx, dy, cx, cy)
        z = ob.sptc(X, Y, cx, cy)
        for light, cap in {(t["light_row_max"], t["heavy_window_cap"]), (256, 0), (2048, 0), (0, half[0]), (0, 256)}:
            ctx.set_tiles(light, cap)
            tuned = gb.sptc(ctx, dx, dy, cx, cy, t["accum"], max_chunk_nnz=t["max_chunk_nnz"])
            assert np.array_equal(tuned.keys, base.keys) and np.array_equal(tuned.keys, z.keys)
            value_bar.max_rel_err(tuned.vals, z.vals)
        ctx.set_tiles(0, 0)
    finally:
        dx.free()
        if dy is not dx:
            dy.free()


def test_cli_autotune_flag(tmp_path):
    X, _, cx, cy = synth.plain_small(scale=0.2)
    xp = tmp_path / "x.tns"
    synth.write_tns(str(xp), X)
    base = [gb.CLI_PATH, "-X", str(xp), "-Y", str(xp), "-c", "1", "-x", "2", "-y", "2"]
    r0 = subprocess.run(base, capture_output=True, text=True, timeout=300)
    r1 = subprocess.run(base + ["-t", "-n", "2"], capture_output=True, text=True, timeout=300)
    assert r0.returncode == 0 and r1.returncode == 0, r1.stderr
    assert "autotune: dense_accumulator" in r1.stderr
    nnz = [[l for l in r.stderr.splitlines() if l.startswith("Result NNZ:")][0] for r in (r0, r1)]
    assert nnz[0] == nnz[1]
