"""Stage entry points (linearise, sort, index match) against the oracle, bit-exact."""
import numpy as np
import pytest

import gsparc_b200 as gb
import oracle_bind as ob
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64) if a.dtype == np.uint64 else
                            np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("case", ["plain_small", "esc_large", "dense_acc"])
@pytest.mark.parametrize("role", [0, 1])
def test_linearize_bit_exact(case, role):
    X, Y, cx, cy = synth.WORKLOADS[case](scale=0.01)
    keys = gb.linearize(X.dims, cx, role, _dev(X.idx)).cpu().numpy().view(np.uint64)
    assert np.array_equal(keys, ob.linearize(X, cx, role))


def test_linearize_rejects_out_of_range():
    import torch
    idx = torch.tensor([[0, 5], [1, 1]], dtype=torch.int64, device="cuda")
    with pytest.raises(gb.GsparcError):
        gb.linearize([5, 2], [1], 0, idx)


@pytest.mark.parametrize("nbits", [10, 43, 64])
def test_sort_pairs_stable_bit_exact(ctx, nbits):
    rng = np.random.default_rng(nbits)
    n = 200_000
    hi = (1 << nbits) if nbits < 64 else None
    keys = rng.integers(0, 2**63, n, dtype=np.uint64) if hi is None else rng.integers(0, hi, n, dtype=np.uint64)
    keys[::7] = keys[0]  # many equal keys: stability shows in the payload order
    vals = np.arange(n, dtype=np.float32)
    k, v = _dev(keys), _dev(vals)
    gb.sort_pairs(ctx, k, v, nbits)
    ek, ev = ob.sort_pairs(keys, vals, nbits)
    assert np.array_equal(k.cpu().numpy().view(np.uint64), ek)
    assert np.array_equal(v.cpu().numpy(), ev)


@pytest.mark.parametrize("case", ["plain_small", "esc_large", "dense_acc"])
def test_index_match_bit_exact(ctx, case):
    X, Y, cx, cy = synth.WORKLOADS[case](scale=0.01)
    _, _, ncx, nfx = ob.layout(X.dims, cx)
    _, _, ncy, nfy = ob.layout(Y.dims, cy)
    xk, _ = ob.sort_pairs(ob.linearize(X, cx, 0), X.val, ncx + nfx)
    yk, _ = ob.sort_pairs(ob.linearize(Y, cy, 1), Y.val, ncy + nfy)
    pos, cnt, pre, ir = gb.index_match(ctx, _dev(xk), ncx, _dev(yk), nfy)
    epos, ecnt, epre = ob.index_match(xk, ncx, yk, nfy)
    assert ir == int(epre[-1])
    assert np.array_equal(cnt.cpu().numpy().view(np.uint64), ecnt)
    assert np.array_equal(pre.cpu().numpy().view(np.uint64), epre)
    m = ecnt > 0
    assert np.array_equal(pos.cpu().numpy().view(np.uint64)[m], epos[m])
