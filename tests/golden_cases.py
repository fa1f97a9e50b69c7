"""Loading helpers for the golden fixtures in tests/golden/ (reference CPU SpTC outputs)."""
import glob
import os

import numpy as np

from gsparc_b200.synth import CooTensor

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


def load(name):
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    X = CooTensor([int(d) for d in z["x_dims"]], z["x_idx"].astype(np.uint64), z["x_val"].astype(np.float32))
    Y = CooTensor([int(d) for d in z["y_dims"]], z["y_idx"].astype(np.uint64), z["y_val"].astype(np.float32))
    return X, Y, [int(c) for c in z["cx"]], [int(c) for c in z["cy"]], z["z_idx"].astype(np.uint64), z["z_val"]


def hand_case():
    """Tiny case with an exactly cancelling output (kept, as ESC keeps it)."""
    X = CooTensor([2, 3, 2],
                  np.array([[0, 0, 1, 1, 0], [1, 1, 2, 0, 2], [0, 1, 1, 0, 1]], np.uint64),
                  np.array([0.5, -0.5, 2.0, 1.25, 3.0], np.float32))
    Y = CooTensor([2, 2, 3],
                  np.array([[0, 1, 1, 0, 1], [1, 1, 0, 0, 1], [2, 2, 1, 0, 0]], np.uint64),
                  np.array([2.0, 2.0, -1.0, 4.0, 0.75], np.float32))
    # expected Z (X free 0,1 then Y free 1,2), lexicographic, worked out by hand
    expect = [
        ((0, 1, 0, 0), 2.0), ((0, 1, 0, 1), 0.5), ((0, 1, 1, 0), -0.375), ((0, 1, 1, 2), 0.0),
        ((0, 2, 0, 1), -3.0), ((0, 2, 1, 0), 2.25), ((0, 2, 1, 2), 6.0), ((1, 0, 0, 0), 5.0),
        ((1, 0, 1, 2), 2.5), ((1, 2, 0, 1), -2.0), ((1, 2, 1, 0), 1.5), ((1, 2, 1, 2), 4.0),
    ]
    zi = np.array([e[0] for e in expect], np.uint64).T
    zv = np.array([e[1] for e in expect], np.float64)
    return X, Y, [2], [0], zi, zv
