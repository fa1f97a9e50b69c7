"""gsparc_index_match_noalloc -- the index match for callers that cannot
allocate device memory (hosts whose own allocator owns all of the GPU's memory,
paths that must not enter the driver's allocator).  Its scratch is one
library-owned device array, shared by every call, so the checks are: the same
results as the allocating gsparc_index_match and as the oracle on the same
keys, on two calls in a row and on two different inputs back to back (nothing
may leak from one call into the next), the form that does not wait (ir NULL,
total left in prefix[nx]), and a clear refusal of inputs larger than that array.

Results are integers: compared exactly.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

import gsparc_b200 as gb
import oracle_bind as ob
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu


def _noalloc():
    f = gb.lib().gsparc_index_match_noalloc
    f.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _sorted_keys(case, scale):
    X, Y, cx, cy = synth.WORKLOADS[case](scale=scale)
    _, _, ncx, nfx = ob.layout(X.dims, cx)
    _, _, ncy, nfy = ob.layout(Y.dims, cy)
    xk, _ = ob.sort_pairs(ob.linearize(X, cx, 0), X.val, ncx + nfx)
    yk, _ = ob.sort_pairs(ob.linearize(Y, cy, 1), Y.val, ncy + nfy)
    return xk, ncx, yk, nfy


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _call_noalloc(xk, ncx, yk, nfy, want_total=True):
    import torch
    nx = xk.shape[0]
    pos = torch.full((nx,), -1, dtype=torch.int64, device="cuda")
    cnt = torch.full((nx,), -1, dtype=torch.int64, device="cuda")
    pre = torch.full((nx + 1,), -1, dtype=torch.int64, device="cuda")
    ir = np.zeros(1, np.uint64)
    st = _noalloc()(nx, xk.data_ptr(), ncx, yk.shape[0], yk.data_ptr(), nfy, pos.data_ptr(),
                    cnt.data_ptr(), pre.data_ptr(), ir.ctypes.data if want_total else None, None)
    assert st == 0, gb.lib().gsparc_last_error()
    pre_h = pre.cpu().numpy().view(np.uint64)
    total = int(ir[0]) if want_total else int(pre_h[nx])
    return (pos.cpu().numpy().view(np.uint64), cnt.cpu().numpy().view(np.uint64), pre_h, total)


def test_noalloc_index_match_equals_allocating_one_on_two_calls_in_a_row():
    with gb.Context(0) as ctx:
        for case, scale in (("esc_large", 0.05), ("dense_acc", 0.01)):
            xk, ncx, yk, nfy = _sorted_keys(case, scale)
            dx, dy = _dev(xk), _dev(yk)
            pos, cnt, pre, ir = gb.index_match(ctx, dx, ncx, dy, nfy)
            want_cnt = cnt.cpu().numpy().view(np.uint64)
            want_pre = pre.cpu().numpy().view(np.uint64)
            want_pos = pos.cpu().numpy().view(np.uint64)
            assert ir > 0
            o_pos, o_cnt, o_pre = ob.index_match(xk, ncx, yk, nfy)
            assert np.array_equal(o_cnt, want_cnt) and np.array_equal(o_pre, want_pre)
            hit = o_cnt > 0
            for want_total in (True, True, False):
                got_pos, got_cnt, got_pre, got_ir = _call_noalloc(dx, ncx, dy, nfy, want_total)
                assert got_ir == ir == int(o_pre[-1])
                assert np.array_equal(got_cnt, want_cnt)
                assert np.array_equal(got_pre, want_pre)
                assert np.array_equal(got_pos, want_pos)
                assert np.array_equal(got_pos[hit], o_pos[hit])


def test_noalloc_index_match_refuses_inputs_beyond_its_scratch():
    import torch
    ny = 6_000_000  # needs more than the 64 MiB the entry point owns
    yk = torch.arange(ny, dtype=torch.int64, device="cuda")
    xk = torch.arange(16, dtype=torch.int64, device="cuda")
    out = [torch.zeros(17, dtype=torch.int64, device="cuda") for _ in range(3)]
    ir = np.zeros(1, np.uint64)
    st = _noalloc()(16, xk.data_ptr(), 8, ny, yk.data_ptr(), 4, out[0].data_ptr(), out[1].data_ptr(),
                    out[2].data_ptr(), ir.ctypes.data, None)
    assert st == 1
    assert b"scratch" in gb.lib().gsparc_last_error()
    # a call within the limit still works afterwards
    xs, ncx, ys, nfy = _sorted_keys("plain_small", 0.05)
    assert _call_noalloc(_dev(xs), ncx, _dev(ys), nfy)[3] > 0
