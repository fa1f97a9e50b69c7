"""Output keys over 64 bits (X's free bits + Y's free bits > 64), through the
C ABI with 128-bit keys (sink key_words = 2).

The reference truncates such keys to 64 bits (include/gsparc/contraction_extra.
cuh:149-151); with one key word the engine refuses them (GSPARC_EUNSUPPORTED),
with two it delivers every key as 128 bits, low word first.  Checked against a
coordinate-dictionary contraction in FP64 on the host (small inputs): output
coordinates decoded from the keys, their order and nnz exact, values within
the bar of tests/value_bar.py; for outputs of at most 64 bits the two-word keys
equal the one-word keys with a zero high word.
"""
from collections import defaultdict

import numpy as np
import pytest

import gsparc_b200 as gb
import value_bar
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu

EUNSUPPORTED = 6


@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


def dict_contraction(X, Y, cx, cy):
    fx = [m for m in range(X.order) if m not in cx]
    fy = [m for m in range(Y.order) if m not in cy]
    ymap = defaultdict(list)
    for k in range(Y.nnz):
        c = tuple(int(Y.idx[m][k]) for m in cy)
        ymap[c].append((tuple(int(Y.idx[m][k]) for m in fy), float(Y.val[k])))
    acc = defaultdict(float)
    for k in range(X.nnz):
        c = tuple(int(X.idx[m][k]) for m in cx)
        xf = tuple(int(X.idx[m][k]) for m in fx)
        xv = float(X.val[k])
        for yf, yv in ymap.get(c, ()):
            acc[xf + yf] += xv * yv
    keys = sorted(acc)
    coords = np.array(keys, np.uint64).T if keys else np.zeros((len(fx) + len(fy), 0), np.uint64)
    return coords, np.array([acc[k] for k in keys])


def wide_case(seed):
    # X free modes 2^20 x 2^21 (41 bits), Y free modes 2^21 x 2^20 (41 bits): 82-bit output keys
    X = synth.make_tensor([1 << 20, 1 << 21, 40], 3000, ["uniform", "uniform", ("zipf", 1.2)], "u11", seed)
    Y = synth.make_tensor([40, 1 << 21, 1 << 20], 3000, [("zipf", 1.2), "uniform", "uniform"], "u11", seed + 1)
    return X, Y, [2], [0]


@pytest.mark.parametrize("seed", [71, 73])
@pytest.mark.parametrize("accum", [0, 1])
def test_128_bit_output_keys_match_the_host_contraction(ctx, seed, accum):
    X, Y, cx, cy = wide_case(seed)
    bx = sum(synth._bits(d) for m, d in enumerate(X.dims) if m not in cx)
    by = sum(synth._bits(d) for m, d in enumerate(Y.dims) if m not in cy)
    assert bx + by > 64
    with pytest.raises(gb.GsparcError) as e:
        gb.SpTC(X, Y, cx, cy, ctx=ctx)
    assert e.value.status == EUNSUPPORTED
    res = gb.SpTC(X, Y, cx, cy, ctx=ctx, dense_accumulator=accum, key_words=2)
    zc, zv = dict_contraction(X, Y, cx, cy)
    assert res.keys.shape == (res.nnz, 2) and res.nnz == zc.shape[1] > 0
    coords = gb.decode_keys(res.keys, X.dims, Y.dims, cx, cy)
    assert np.array_equal(coords, zc)
    value_bar.max_rel_err(res.vals, zv)
    # strictly ascending as 128-bit numbers
    k = [(int(h) << 64) | int(l) for l, h in res.keys]
    assert all(a < b for a, b in zip(k, k[1:]))


def test_two_key_words_on_a_64_bit_output(ctx):
    X, Y, cx, cy = synth.plain_small(scale=0.05)
    one = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    two = gb.SpTC(X, Y, cx, cy, ctx=ctx, key_words=2)
    assert np.array_equal(two.keys[:, 0], one.keys) and not two.keys[:, 1].any()
    assert np.allclose(two.vals, one.vals, rtol=1e-6, atol=0)


def test_ring_sink_with_two_key_words(ctx):
    X, Y, cx, cy = wide_case(79)
    dx, dy = ctx.upload(X), ctx.upload(Y)
    try:
        whole = gb.sptc(ctx, dx, dy, cx, cy, key_words=2)
        hk = np.zeros(2 * 500, np.uint64)
        hv = np.zeros(500, np.float32)
        got = []

        def on_chunk(k, v, n, first):
            got.append((first, hk[: 2 * n].copy(), v[:n].copy()))
            return 0
        gb.sptc(ctx, dx, dy, cx, cy, sink="ring", host_keys=hk, host_vals=hv, on_chunk=on_chunk, key_words=2)
    finally:
        dx.free()
        dy.free()
    assert len(got) > 1
    keys = np.concatenate([g[1] for g in got]).reshape(-1, 2)
    assert np.array_equal(keys, whole.keys)
    assert np.allclose(np.concatenate([g[2] for g in got]), whole.vals, rtol=1e-6, atol=0)


def test_cli_writes_outputs_with_128_bit_keys(tmp_path):
    import subprocess
    X, Y, cx, cy = wide_case(83)
    xp, yp, zp = str(tmp_path / "x.tns"), str(tmp_path / "y.tns"), str(tmp_path / "z.tns")
    synth.write_tns(xp, X)
    synth.write_tns(yp, Y)
    r = subprocess.run([gb.CLI_PATH, "-X", xp, "-Y", yp, "-c", "1", "-x", "2", "-y", "0", "-o", zp],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    Z = gb.read_tns(zp)
    Xr, Yr = gb.read_tns(xp), gb.read_tns(yp)
    zc, zv = dict_contraction(Xr, Yr, cx, cy)
    assert np.array_equal(Z.idx, zc)
    assert np.allclose(Z.val, zv, rtol=1e-6, atol=1e-6)
