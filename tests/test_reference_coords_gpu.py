"""Output coordinates pinned against the reference GSPARC program itself, on the GPU.

oracle/_ref/gsparc_tap is the reference's main.cu and src/ compiled unmodified
for sm_100a and linked with oracle/esc_tap.cpp, which wraps the program's
device-to-host copy helper and digests the ESC output partitions the program
copies to the host and then drops (include/gsparc/contraction.cuh:540-555).
Its ESC mode (-d -1) is run on the same .tns files as ours; for every case:

* the nonzero count, the order-independent key hash (sum of splitmix64, the
  same definition as gsparc_digest_chunk), an order-sensitive hash of the
  concatenated keys, the first and last key and strict ascending order must be
  equal: output coordinates and their order are bit-exact with the reference;
* for the small cases the tap also dumps the reference's keys and values: the
  keys must equal ours element by element, and the reference's FP32 values
  (CUB ReduceByKey order, no compensation) must lie within the FP32 summation
  bound of the FP64 oracle (n * 2^-24 * sum|products| per output), while ours
  meet max relative error <= 1e-5 against the same FP64 oracle.

Inputs are ordinary ones only: non-empty operands with at least one matched
product and keys of at most 64 bits (the reference launches zero-size grids for
empty inputs and takes another code path for wider keys).
"""
import os
import re
import subprocess

import numpy as np
import pytest

import golden_cases as gc
import gsparc_b200 as gb
import oracle_bind as ob
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TAP_BIN = os.path.join(ROOT, "oracle", "_ref", "gsparc_tap")
REL = 1e-5

SYNTH = {
    "plain_small_full": lambda: synth.plain_small(scale=1.0),
    "esc_large_s005": lambda: synth.esc_large(scale=0.05),
    "dense_acc_s001": lambda: synth.dense_acc(scale=0.01),
    "esc_large_s01_seed4": lambda: synth.esc_large(scale=0.1, seed=4),
}
DUMP = set(n for n in gc.names() if n != "wide_keys") | {"hand", "dense_acc_s001"}
CASES = sorted(DUMP) + sorted(SYNTH)

TAP_RE = re.compile(r"^esc_tap: parts (\d+) nnz (\d+) key_hash (\d+) seq_hash (\d+) unsorted (\d+) "
                    r"first (\d+) last (\d+) val_sum (\S+)$", re.M)


def _load(case):
    if case in SYNTH:
        return SYNTH[case]()
    if case == "hand":
        X, Y, cx, cy, _, _ = gc.hand_case()
        return X, Y, cx, cy
    X, Y, cx, cy, _, _ = gc.load(case)
    return X, Y, cx, cy


def _seq_hash(keys: np.ndarray) -> int:
    """h = h * P + splitmix64(key) over the keys in order, mod 2^64 (the tap's definition)."""
    s = gb.splitmix64(keys)
    n = s.shape[0]
    with np.errstate(over="ignore"):
        pw = np.full(n, np.uint64(0x100000001B3), np.uint64)
        pw[-1] = np.uint64(1)
        pw = np.cumprod(pw[::-1], dtype=np.uint64)[::-1]  # P^(n-1-i)
        return int(np.sum(s * pw, dtype=np.uint64))


@pytest.mark.parametrize("case", CASES)
def test_output_coordinates_equal_reference_gsparc(case, tmp_path):
    if not os.path.exists(TAP_BIN):
        pytest.skip("tapped reference program not built (oracle/Makefile needs the reference tree)")
    X, Y, cx, cy = _load(case)
    xp, yp = str(tmp_path / "x.tns"), str(tmp_path / "y.tns")
    synth.write_tns(xp, X)
    synth.write_tns(yp, Y)
    Xr, Yr = gb.read_tns(xp), gb.read_tns(yp)
    assert sum(synth._bits(d) for d in Xr.dims) <= 64 and sum(synth._bits(d) for d in Yr.dims) <= 64
    env = dict(os.environ)
    dump = str(tmp_path / "ref") if case in DUMP else None
    if dump:
        env["GSPARC_ESC_TAP_DUMP"] = dump
    args = ["-X", xp, "-Y", yp, "-c", str(len(cx)), "-x", *map(str, cx), "-y", *map(str, cy), "-d", "-1"]
    ref = subprocess.run([TAP_BIN, *args], capture_output=True, text=True, timeout=600, env=env)
    assert ref.returncode == 0, ref.stderr[-2000:]
    m = TAP_RE.search(ref.stderr)
    assert m, ref.stderr[-2000:]
    parts, nnz, khash, shash, unsorted, first, last = (int(g) for g in m.groups()[:7])
    rnnz = int(re.search(r"^Result NNZ: (\d+)$", ref.stderr, re.M).group(1))
    assert nnz == rnnz and parts >= 1 and unsorted == 0

    with gb.Context(0) as ctx:
        res = gb.SpTC(Xr, Yr, cx, cy, ctx=ctx, dense_accumulator=-1)
    keys = np.asarray(res.keys, np.uint64)
    assert res.nnz == nnz == keys.shape[0]
    assert int(np.sum(gb.splitmix64(keys), dtype=np.uint64)) == khash
    assert _seq_hash(keys) == shash
    assert int(keys[0]) == first and int(keys[-1]) == last
    assert np.all(keys[1:] > keys[:-1])

    if dump:
        rk = np.fromfile(dump + ".keys", np.uint64)
        rv = np.fromfile(dump + ".vals", np.float32).astype(np.float64)
        assert np.array_equal(rk, keys)
        z = ob.sptc(Xr, Yr, cx, cy)
        assert np.array_equal(z.keys, keys)
        # the reference's plain FP32 sums: within the FP32 summation bound of FP64
        bound = np.maximum(z.nprod, 1) * 2.0 ** -24 * z.abs_sums
        assert np.all(np.abs(rv - z.vals) <= bound + 1e-30)
        # ours: max relative error against FP64
        ours = np.asarray(res.vals, np.float64)
        nz = z.vals != 0
        assert np.all(ours[~nz] == 0)
        rel = np.abs(ours[nz] - z.vals[nz]) / np.abs(z.vals[nz])
        assert rel.size == 0 or rel.max() <= REL, rel.max()
