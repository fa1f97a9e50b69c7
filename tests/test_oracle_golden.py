"""The CPU oracle against the reference's own CPU SpTC outputs (tests/golden/)
and a hand-computed case.  Pins the oracle before it is used as the checker."""
import numpy as np
import pytest

import golden_cases as gc
import oracle_bind as ob


def _check(X, Y, cx, cy, zi, zv):
    z = ob.sptc(X, Y, cx, cy)
    coords = ob.decode_keys(z.keys, X, Y, cx, cy)
    assert z.nnz == zi.shape[1]
    assert np.array_equal(coords, zi), "coordinates / order differ from the reference"
    # reference values: FP32 sums printed with 6 decimals
    tol = 1e-6 + 2e-6 * z.abs_sums
    assert np.all(np.abs(z.vals - zv) <= tol)
    return z


@pytest.mark.parametrize("name", gc.names())
def test_oracle_matches_reference_cpu_sptc(name):
    X, Y, cx, cy, zi, zv = gc.load(name)
    _check(X, Y, cx, cy, zi, zv)


def test_oracle_hand_case_keeps_cancelled_sum():
    X, Y, cx, cy, zi, zv = gc.hand_case()
    z = _check(X, Y, cx, cy, zi, zv)
    assert z.ir_nnz == 13
    assert np.any(z.vals == 0.0)


def test_oracle_layout_follows_reference_mask_order():
    # 2482 x 2862 x 14036 x 17 with contract modes (2, 3): free modes 0,1 ->
    # mode 0 above mode 1; contract mode 2 above mode 3.
    shift, isc, ncb, nfb = ob.layout([2482, 2862, 14036, 17], [2, 3])
    assert (ncb, nfb) == (19, 24)
    assert list(shift) == [12, 0, 5, 0]
    assert list(isc) == [False, False, True, True]
    # contract modes listed out of order: the first listed sits highest
    shift, isc, ncb, nfb = ob.layout([13, 40, 17], [2, 1])
    assert ncb == 5 + 6 and shift[2] == 6 and shift[1] == 0


def test_oracle_size_one_mode_takes_zero_bits():
    assert ob.mode_bits(1) == 0 and ob.mode_bits(2) == 1 and ob.mode_bits(1024) == 10
    assert ob.mode_bits(1025) == 11 and ob.mode_bits(2**64 - 1) == 64


def test_oracle_wide_contract_keys_match_coordinate_sums():
    """Contract keys of 66 bits (the reference's 128-bit path): the oracle's
    128-bit keys against a plain dictionary contraction over coordinates."""
    from collections import defaultdict
    from gsparc_b200 import synth
    d = 1 << 22
    X = synth.make_tensor([300, d, d, d], 600, ["uniform"] + [("zipf", 1.6)] * 3, "u11", 3)
    Y = synth.make_tensor([d, d, d, 200], 600, [("zipf", 1.6)] * 3 + ["uniform"], "u11", 4)
    ymap = defaultdict(list)
    for k in range(Y.nnz):
        ymap[tuple(int(Y.idx[m][k]) for m in (0, 1, 2))].append((int(Y.idx[3][k]), float(Y.val[k])))
    ref = defaultdict(float)
    for k in range(X.nnz):
        for yf, yv in ymap.get(tuple(int(X.idx[m][k]) for m in (1, 2, 3)), []):
            ref[(int(X.idx[0][k]), yf)] += float(X.val[k]) * yv
    z = ob.sptc(X, Y, [1, 2, 3], [0, 1, 2])
    coords = ob.decode_keys(z.keys, X, Y, [1, 2, 3], [0, 1, 2])
    got = {(int(a), int(b)): v for a, b, v in zip(coords[0], coords[1], z.vals)}
    assert z.nnz == len(ref) > 0
    assert sorted(got) == sorted(ref)
    for k, v in ref.items():
        assert abs(got[k] - v) <= 1e-9 * max(1.0, abs(v))
