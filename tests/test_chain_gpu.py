"""Chained contractions: a result kept on the device as an operand
(gsparc_sptc_resident, the reference's multi-SpTC, main.cu:323-371 and
include/gsparc/sptc.cuh:362-698), through the C ABI and the CLI's -m.

The resident result must hold exactly the output of gsparc_sptc (coordinates
decoded from its keys, values bit-identical).  A chain Z = (X x Y) x T is
checked against the FP64 oracle run on the first result as the engine holds it
(FP32 values): keys, order and nnz bit-exact, values within the bar of
tests/value_bar.py (max relative error <= 1e-5).
"""
import os
import re
import subprocess

import numpy as np
import pytest

import golden_cases as gc
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


def download(t):
    h = t.download()
    return h.idx, h.val


def cases():
    X, Y, cx, cy, _, _ = gc.load("mixed_orders")
    yield "mixed_orders", X, Y, cx, cy
    X, Y, cx, cy, _, _ = gc.load("wide_keys")
    yield "wide_keys", X, Y, cx, cy
    X, Y, cx, cy = synth.plain_small(scale=0.05)
    yield "plain_small", X, Y, cx, cy


@pytest.mark.parametrize("case", list(cases()), ids=lambda c: c[0])
def test_resident_result_equals_returned_result(ctx, case):
    _, X, Y, cx, cy = case
    dx, dy = ctx.upload(X), ctx.upload(Y)
    try:
        a = gb.sptc(ctx, dx, dy, cx, cy)
        z = gb.sptc_resident(ctx, dx, dy, cx, cy)
        assert z.nnz == a.nnz and z.stats["ir_nnz"] == a.ir_nnz
        fx = [X.dims[m] for m in range(X.order) if m not in cx]
        fy = [Y.dims[m] for m in range(Y.order) if m not in cy]
        assert z.dims == fx + fy
        idx, val = download(z)
        coords = gb.decode_keys(a.keys, X.dims, Y.dims, cx, cy)
        assert np.array_equal(idx, coords)
        assert np.array_equal(val, a.vals)
        z.free()
    finally:
        dx.free()
        dy.free()


def test_download_round_trip(ctx):
    X, _, _, _ = synth.plain_small(scale=0.01)
    d = ctx.upload(X)
    h = d.download()
    d.free()
    assert h.dims == X.dims and np.array_equal(h.idx, X.idx) and np.array_equal(h.val, X.val)


def chain_oracle(X, Y, cx, cy, T, c1n, cz):
    z1 = ob.sptc(X, Y, cx, cy)
    coords = ob.decode_keys(z1.keys, X, Y, cx, cy)
    fx = [X.dims[m] for m in range(X.order) if m not in cx]
    fy = [Y.dims[m] for m in range(Y.order) if m not in cy]
    Z1 = CooTensor(fx + fy, coords.astype(np.uint64), z1.vals.astype(np.float32))
    c1 = list(range(Z1.order - c1n, Z1.order))
    return Z1, c1, ob.sptc(Z1, T, c1, cz)


def chain_case():
    # Z1 = X x_{2,0} Y (modes: X0 X1 | Y1 Y2), then Z1's (Y1, Y2) against T = Y's (1, 2)
    X = synth.make_tensor([40, 30, 50], 3000, ["uniform", "uniform", ("zipf", 1.2)], "u11", 61)
    Y = synth.make_tensor([50, 25, 20], 3000, [("zipf", 1.2), "uniform", "uniform"], "u11", 62)
    return X, Y, [2], [0], 2, [1, 2]


def check(res, z):
    assert res.ir_nnz == z.ir_nnz and res.nnz == z.nnz
    assert np.array_equal(res.keys, z.keys)
    value_bar.max_rel_err(res.vals, z.vals)


@pytest.mark.parametrize("accum", [0, -1, 1])
def test_chain_matches_oracle(ctx, accum):
    X, Y, cx, cy, na, cz = chain_case()
    dx, dy = ctx.upload(X), ctx.upload(Y)
    try:
        z1 = gb.sptc_resident(ctx, dx, dy, cx, cy, accum)
        c1 = list(range(z1.order - na, z1.order))
        res = gb.sptc(ctx, z1, dy, c1, cz, accum)
        # the oracle's first result rounded to FP32 equals the engine's Z1 here
        # up to the accumulation order; compare the chain against it
        Z1, c1o, z = chain_oracle(X, Y, cx, cy, Y, na, cz)
        idx, val = download(z1)
        assert np.array_equal(idx, Z1.idx)
        assert np.allclose(val, Z1.val, rtol=2e-6, atol=1e-6)
        # run the oracle on the engine's own Z1 values for the value bar
        zo = ob.sptc(CooTensor(z1.dims, idx, val), Y, c1, cz)
        check(res, zo)
        assert np.array_equal(res.keys, z.keys)
        z1.free()
    finally:
        dx.free()
        dy.free()


def test_resident_result_in_a_batch_and_served(ctx):
    X, Y, cx, cy, na, cz = chain_case()
    dx, dy = ctx.upload(X), ctx.upload(Y)
    try:
        z1 = gb.sptc_resident(ctx, dx, dy, cx, cy)
        c1 = list(range(z1.order - na, z1.order))
        alone = gb.sptc(ctx, z1, dy, c1, cz)
        res, bst = gb.sptc_batch(ctx, [(z1, dy, c1, cz), (dx, dy, cx, cy)])
        assert bst["status"] == 0
        assert np.array_equal(res[0].keys, alone.keys)
        assert np.allclose(res[0].vals, alone.vals, rtol=1e-5, atol=1e-6)
        z1.free()
    finally:
        dx.free()
        dy.free()


def test_cli_chained_multi_sptc(ctx, tmp_path):
    X, Y, cx, cy, na, cz = chain_case()
    xp, yp, zp = tmp_path / "x.tns", tmp_path / "y.tns", tmp_path / "z.tns"
    synth.write_tns(str(xp), X)
    synth.write_tns(str(yp), Y)
    cmd = [gb.CLI_PATH, "-X", str(xp), "-Y", str(yp), "-c", "1", "-x", "2", "-y", "0",
           "-m", "1", "-a", str(na), "-z", *map(str, cz), "-o", str(zp)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "First SpTC time:" in r.stderr and "multi_sptc: 1" in r.stderr
    assert "# contract modes of Z (second SpTC): 2, contract modes: 1 2 \n" in r.stderr
    # the reference's Table 4 script parses these lines with this pattern
    # (scripts/figure/Table4.py:10): one match per run
    table4 = (r"tensor X: .*?/([^/]+)\.tns[\s\S]*?First SpTC time: ([\d\.]+)[\s\S]*?"
              r"Bit reordering time: ([\d\.]+)[\s\S]*?Total time: ([\d\.]+)")
    m = re.findall(table4, r.stderr)
    assert len(m) == 1 and m[0][0] == "x", m
    assert re.search(r"Bit reordering ratio: [\d\.]+%\n", r.stderr)
    # the chain through the API on the .tns-read operands
    Xr, Yr = gb.read_tns(str(xp)), gb.read_tns(str(yp))
    dx, dy = ctx.upload(Xr), ctx.upload(Yr)
    z1 = gb.sptc_resident(ctx, dx, dy, cx, cy)
    c1 = list(range(z1.order - na, z1.order))
    res = gb.sptc(ctx, z1, dy, c1, cz)
    z1.free()
    dx.free()
    dy.free()
    nnz_line = [l for l in r.stderr.splitlines() if l.startswith("Result NNZ:")][0]
    assert int(nnz_line.split(":")[1]) == res.nnz
    Z = gb.read_tns(str(zp))
    assert Z.nnz == res.nnz
    coords = gb.decode_keys(res.keys, z1.dims, Yr.dims, c1, cz)
    # .tns holds coordinates in output order; the file's inferred dims may be
    # smaller than the nominal ones, so compare coordinates only
    assert np.array_equal(Z.idx, coords)
    assert np.allclose(Z.val, res.vals, rtol=1e-6, atol=0)


def test_cli_quantum_input_equals_tns_input(tmp_path):
    X, Y, cx, cy, _, _ = gc.load("mixed_orders")
    for name, t in (("x", X), ("y", Y)):
        synth.write_tns(str(tmp_path / f"{name}.tns"), t)
        synth.write_quantum(str(tmp_path / name), t)
    base = ["-c", "1", "-x", str(cx[0]), "-y", str(cy[0])]
    outs = []
    for q in (False, True):
        zp = tmp_path / f"z{int(q)}.tns"
        xs = [str(tmp_path / "x"), str(tmp_path / "y")] if q else [str(tmp_path / "x.tns"), str(tmp_path / "y.tns")]
        cmd = [gb.CLI_PATH, "-X", xs[0], "-Y", xs[1], *base, "-o", str(zp)] + (["-q"] if q else [])
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs.append((r.stderr, open(zp).read()))
    nnz = [[l for l in e.splitlines() if l.startswith("Result NNZ:")][0] for e, _ in outs]
    assert nnz[0] == nnz[1]
    assert outs[0][1] == outs[1][1]
