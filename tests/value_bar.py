"""The value bar every engine test applies against FP64 sums.

Max relative error |z - z64| / |z64| <= 1e-5 on every output whose FP64 value
is nonzero, and exactly 0 where the FP64 value is exactly 0 (sums that cancel
exactly).  The engine's compensated FP32 accumulation (TwoSum of every add plus
each product's fma error, rounded once at the end) stays within a few units in
the last place of the exact sum, cancelling N(0,1) sums included.
"""
import numpy as np

REL = 1e-5


def max_rel_err(vals, z64) -> float:
    """Asserts the bar; returns the max relative error over nonzero FP64 values."""
    v = np.asarray(vals, np.float64)
    z = np.asarray(z64, np.float64)
    assert v.shape == z.shape, (v.shape, z.shape)
    err = np.abs(v - z)
    nz = z != 0
    assert np.all(err[~nz] == 0), "an exactly cancelling sum is not exactly 0"
    rel = float(np.max(err[nz] / np.abs(z[nz]))) if nz.any() else 0.0
    assert rel <= REL, f"max relative error {rel:.3e} > {REL}"
    return rel
