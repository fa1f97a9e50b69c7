"""Generate the golden SpTC fixtures from the reference's own CPU SpTC.

The reference repository ships no tests or golden vectors.  Its CPU SpTC
baseline (baselines/Sparta: benchmark/ttt.c -> src/sptensor/tmul.c,
EXPERIMENT_MODES=3) is compiled from source by ``oracle/Makefile`` into
``oracle/_ref/ttt``.  This script runs it on small seeded inputs and stores
inputs plus Sparta's output tensor (0-based coordinates in lexicographic order,
values printed with 6 decimals; baselines/Sparta/src/sptensor/dump.c:29-49)
as compressed ``.npz`` fixtures next to this file.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gsparc_b200 import synth  # noqa: E402
from gsparc_b200.synth import CooTensor  # noqa: E402

TTT = os.path.join(ROOT, "oracle", "_ref", "ttt")


def hand_case():
    # 2x3x2 (X) contracted with 2x2x3 (Y) on X mode 2 / Y mode 0; the two
    # products landing on output (0,1,0,2) cancel to exactly zero (kept as a
    # nonzero by the ESC semantics), a duplicate-free tiny instance.
    X = CooTensor([2, 3, 2],
                  np.array([[0, 0, 1, 1, 0], [1, 1, 2, 0, 2], [0, 1, 1, 0, 1]], np.uint64),
                  np.array([0.5, -0.5, 2.0, 1.25, 3.0], np.float32))
    Y = CooTensor([2, 2, 3],
                  np.array([[0, 1, 1, 0, 1], [1, 1, 0, 0, 1], [2, 2, 1, 0, 0]], np.uint64),
                  np.array([2.0, 2.0, -1.0, 4.0, 0.75], np.float32))
    return X, Y, [2], [0]


def mixed_orders():
    X = synth.make_tensor([37, 50, 29], 500, ["uniform", ("zipf", 1.2), "uniform"], "u11", 11)
    Y = synth.make_tensor([29, 23, 11, 19], 300, [("zipf", 1.1), "uniform", "uniform", "uniform"],
                          "u11", 12)
    return X, Y, [2], [0]


def reordered_cmodes():
    X = synth.make_tensor([13, 40, 17], 1200, ["uniform", "uniform", "uniform"], "u01", 21)
    Y = synth.make_tensor([40, 17, 9, 31], 1500, ["uniform", "uniform", "uniform", "uniform"],
                          "u01", 22)
    # X mode 2 (size 17) pairs with Y mode 1, X mode 1 (size 40) with Y mode 0
    return X, Y, [2, 1], [1, 0]


def dense_like():
    # the dense-accumulator workload's structure at a size the CPU baseline
    # handles: small free spaces (20 x 30 output), Zipf contract modes.
    X = synth.make_tensor([20, 64, 64], 3000, ["uniform", ("zipf", 1.2), ("zipf", 1.2)], "normal", 31)
    Y = synth.make_tensor([64, 64, 30], 3000, [("zipf", 1.2), ("zipf", 1.2), "uniform"], "normal", 32)
    return X, Y, [1, 2], [0, 1]


def wide_keys():
    # X keys of 65 bits (free modes 2^17 x 2^17, contract modes 2^16 x 2^15):
    # the reference's 128-bit key path (ConvertTensor_extra); output keys of
    # 34 + 13 = 47 bits.  The contract space stays below 2^32 because the
    # baseline built here packs contract coordinates into 32-bit indices.
    X = synth.make_tensor([1 << 17, 1 << 17, 1 << 16, 1 << 15], 2000,
                          ["uniform", "uniform", ("zipf", 1.3), ("zipf", 1.3)], "u11", 41)
    Y = synth.make_tensor([1 << 16, 1 << 15, 5000], 2000, [("zipf", 1.3), ("zipf", 1.3), "uniform"], "u11", 42)
    return X, Y, [2, 3], [0, 1]


CASES = {
    "plain_small_s002": lambda: synth.plain_small(scale=0.02, seed=0),
    "esc_large_s0005": lambda: synth.esc_large(scale=0.0005, seed=1),
    "dense_like": dense_like,
    "mixed_orders": mixed_orders,
    "reordered_cmodes": reordered_cmodes,
    "wide_keys": wide_keys,
}


def run_sparta(X, Y, cx, cy, workdir):
    xp = os.path.join(workdir, "x.tns")
    yp = os.path.join(workdir, "y.tns")
    zp = os.path.join(workdir, "z.tns")
    synth.write_tns(xp, X)
    synth.write_tns(yp, Y)
    cmd = [TTT, "-X", xp, "-Y", yp, "-m", str(len(cx)), "-x", *map(str, cx),
           "-y", *map(str, cy), "-t", "1", "-Z", zp]
    env = dict(os.environ, EXPERIMENT_MODES="3")
    # The baseline binary is not robust on every input (it has been seen to hang
    # or crash on some shapes); bound each run and retry a few times.
    for attempt in range(12):
        try:
            r = subprocess.run(cmd, env=env, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                               timeout=15)
        except subprocess.TimeoutExpired:
            continue
        if r.returncode == 0 and os.path.exists(zp):
            break
    else:
        raise RuntimeError("baseline run did not complete: " + " ".join(cmd))
    with open(zp) as f:
        lines = f.read().split("\n")
    nmodes = int(lines[0])
    zdims = [int(t) for t in lines[1].split()]
    rows = [ln.split() for ln in lines[2:] if ln.strip()]
    zidx = np.array([[int(r[m]) for r in rows] for m in range(nmodes)], dtype=np.uint32).reshape(nmodes, len(rows))
    zval = np.array([float(r[-1]) for r in rows], dtype=np.float64)
    return zdims, zidx, zval


def main():
    if not os.path.exists(TTT):
        raise SystemExit("build oracle/_ref/ttt first: make -C oracle")
    only = set(sys.argv[1:])
    for name, fn in CASES.items():
        if only and name not in only:
            continue
        X, Y, cx, cy = fn()
        with tempfile.TemporaryDirectory() as td:
            zdims, zidx, zval = run_sparta(X, Y, cx, cy, td)
        out = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(out, x_dims=np.asarray(X.dims, np.uint64), x_idx=X.idx.astype(np.uint32),
                            x_val=X.val, y_dims=np.asarray(Y.dims, np.uint64),
                            y_idx=Y.idx.astype(np.uint32), y_val=Y.val,
                            cx=np.asarray(cx, np.int32), cy=np.asarray(cy, np.int32),
                            z_dims=np.asarray(zdims, np.uint64), z_idx=zidx, z_val=zval)
        print(f"{name}: X nnz {X.nnz} Y nnz {Y.nnz} Z nnz {zidx.shape[1]} -> {os.path.getsize(out)} B")


if __name__ == "__main__":
    main()
