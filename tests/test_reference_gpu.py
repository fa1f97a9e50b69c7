"""Output counts pinned against the reference GSPARC program itself, on the GPU.

oracle/_ref/gsparc is the reference's main.cu and src/ compiled unmodified for
sm_100a (oracle/Makefile, from the reference tree where it lies; the binary
travels with the repository, the sources do not).  The program reports only
the result's nonzero count ("Result NNZ", main.cu:428), never the result
itself, so that count is what is pinned here: the reference run in its ESC
mode (-d -1; its dense mode writes wrong keys when X_nfbits != Y_nfbits),
our CLI on the same .tns files, and the oracle must agree.  Coordinates and
values are pinned through the reference's CPU SpTC (tests/golden/) and the
oracle elsewhere.

Inputs are ordinary ones only: non-empty operands with at least one matched
product and keys of at most 64 bits (the reference launches zero-size grids
for empty inputs and takes another code path for wider keys).
"""
import os
import re
import subprocess

import pytest

import golden_cases as gc
import gsparc_b200 as gb
import oracle_bind as ob
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "gsparc")

SYNTH = {
    "plain_small_full": lambda: synth.plain_small(scale=1.0),
    "esc_large_s005": lambda: synth.esc_large(scale=0.05),
    "dense_acc_s001": lambda: synth.dense_acc(scale=0.01),
}
CASES = [n for n in gc.names() if n != "wide_keys"] + ["hand"] + sorted(SYNTH)


def _load(case):
    if case in SYNTH:
        return SYNTH[case]()
    if case == "hand":
        X, Y, cx, cy, _, _ = gc.hand_case()
        return X, Y, cx, cy
    X, Y, cx, cy, _, _ = gc.load(case)
    return X, Y, cx, cy


def _result_nnz(stderr):
    m = re.search(r"^Result NNZ: (\d+)$", stderr, re.M)
    assert m, stderr[-2000:]
    return int(m.group(1))


@pytest.mark.parametrize("case", CASES)
def test_result_nnz_equals_reference_gsparc(case, tmp_path):
    if not os.path.exists(REF_BIN):
        pytest.skip("reference program not built (oracle/Makefile needs the reference tree)")
    X, Y, cx, cy = _load(case)
    xp, yp = str(tmp_path / "x.tns"), str(tmp_path / "y.tns")
    synth.write_tns(xp, X)
    synth.write_tns(yp, Y)
    Xr, Yr = ob.read_tns(xp), ob.read_tns(yp)
    z = ob.sptc(Xr, Yr, cx, cy)
    assert z.ir_nnz > 0 and X.nnz > 0 and Y.nnz > 0
    assert sum(synth._bits(d) for d in Xr.dims) <= 64 and sum(synth._bits(d) for d in Yr.dims) <= 64
    args = ["-X", xp, "-Y", yp, "-c", str(len(cx)), "-x", *map(str, cx), "-y", *map(str, cy), "-d", "-1"]
    ref = subprocess.run([REF_BIN, *args], capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stderr[-2000:]
    ours = subprocess.run([gb.CLI_PATH, *args], capture_output=True, text=True, timeout=300)
    assert ours.returncode == 0, ours.stderr[-2000:]
    assert _result_nnz(ref.stderr) == _result_nnz(ours.stderr) == z.nnz
