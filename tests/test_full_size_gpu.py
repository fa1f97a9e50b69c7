"""Parity at the full sizes of the ESC and dense-accumulator workloads.

The FP64 oracle expands every product, so it cannot take these sizes whole;
they are checked through properties that do not depend on the size:

* esc_large (3.1M nonzeros, 1.75e10 products, 1.3e10 outputs, far more than
  the host can hold): the output streams through a device sink; every chunk is
  digested on the device (count, key hash, order, first and last key, value
  sums) and the whole output rows of a random sample of X rows, plus the
  heaviest row, are cut out of the stream and compared with the oracle run on
  exactly those X rows against the full Y (a row's output depends only on its
  own X nonzeros).  The product count is checked against the Y run lengths
  counted on the host, and a second run with every value doubled must give
  the same keys and four times the values (scaling by a power of two is exact
  in every step of the compensated sums).
* dense_acc (10M + 10M nonzeros, 7.6e8 products, a 200x300 output): every
  output is compared with an FP64 sparse matrix product (scipy) of the same
  operands, the structure and the product count with the product of their
  patterns.

Bars as everywhere: coordinates, order and nnz bit-exact; values within the
bar of tests/value_bar.py (max relative error <= 1e-5 against FP64).
"""
import numpy as np
import pytest

import gsparc_b200 as gb
import oracle_bind as ob
import value_bar
from gsparc_b200 import synth

pytestmark = pytest.mark.gpu



@pytest.fixture(scope="module")
def ctx():
    c = gb.Context(0)
    yield c
    c.close()


def _lin(T, modes):
    """Row-major linear index of the given modes (ordering only, not the key layout)."""
    k = np.zeros(T.nnz, np.int64)
    for m in modes:
        k = k * int(T.dims[m]) + T.idx[m].astype(np.int64)
    return k


def _run_lengths(X, Y, cx, cy):
    """Products of every X nonzero: the number of Y nonzeros with its contract index."""
    xc, yc = _lin(X, cx), _lin(Y, cy)
    uc, cnt = np.unique(yc, return_counts=True)
    pos = np.minimum(np.searchsorted(uc, xc), len(uc) - 1)
    return np.where(uc[pos] == xc, cnt[pos], 0).astype(np.int64)


class _DevArray:
    """A device pointer seen as a 1-D array (CUDA array interface) for torch."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3}


def _stream_rows(ctx, dx, dy, cx, cy, row_lo, row_hi):
    """Contract through a device sink: per-chunk digests, and the outputs whose
    keys fall in [row_lo[i], row_hi[i]) copied to the host."""
    import torch
    lo_d = torch.as_tensor(row_lo.astype(np.int64), device="cuda")
    hi_d = torch.as_tensor(row_hi.astype(np.int64), device="cuda")
    digs, cut_k, cut_v = [], [], []

    def on_chunk(k, v, n, first):
        digs.append((first, gb.digest_chunk(k, v, n)))
        keys = torch.as_tensor(_DevArray(k, n, "<i8"), device="cuda")
        vals = torch.as_tensor(_DevArray(v, n, "<f4"), device="cuda")
        a = torch.searchsorted(keys, lo_d).cpu().numpy()
        b = torch.searchsorted(keys, hi_d).cpu().numpy()
        for i, j in zip(a, b):
            if j > i:
                cut_k.append(keys[i:j].cpu().numpy().astype(np.uint64))
                cut_v.append(vals[i:j].cpu().numpy())
        torch.cuda.synchronize()
        return 0

    r = gb.sptc(ctx, dx, dy, cx, cy, sink="device", on_chunk=on_chunk)
    digs.sort(key=lambda t: t[0])
    keys = np.concatenate(cut_k) if cut_k else np.zeros(0, np.uint64)
    vals = np.concatenate(cut_v) if cut_v else np.zeros(0, np.float32)
    return r, [d for _, d in digs], keys, vals


def test_esc_large_full_size(ctx):
    X, Y, cx, cy = synth.esc_large(scale=1.0)
    runs = _run_lengths(X, Y, cx, cy)
    fx = [m for m in range(X.order) if m not in cx]
    xrow = _lin(X, fx)
    urow, inv = np.unique(xrow, return_inverse=True)
    row_prod = np.bincount(inv, weights=runs)
    rng = np.random.default_rng(11)
    pick = set(rng.choice(len(urow), size=24, replace=False).tolist())
    pick.add(int(np.argmax(row_prod)))
    sub = X.subset(np.isin(inv, sorted(pick)))
    z = ob.sptc(sub, Y, cx, cy, max_products=int(row_prod[sorted(pick)].sum()) + 1)
    assert z.nnz > 0 and int(z.keys.max()) < (1 << 63)
    rows = np.unique(z.keys >> np.uint64(z.y_nfbits))
    row_lo = rows << np.uint64(z.y_nfbits)
    row_hi = (rows + np.uint64(1)) << np.uint64(z.y_nfbits)

    dx = ctx.upload(X)
    try:
        r, digs, keys, vals = _stream_rows(ctx, dx, dx, cx, cy, row_lo, row_hi)
    finally:
        dx.free()
    # products and output count
    assert r.ir_nnz == int(runs.sum())
    assert sum(d["n"] for d in digs) == r.nnz
    assert r.stats["chunks"] == len(digs) > 1
    # global strict order: inside every chunk and across chunk boundaries
    assert all(d["unsorted"] == 0 for d in digs)
    assert all(p["last_key"] < q["first_key"] for p, q in zip(digs, digs[1:]))
    # the sampled rows, exactly as the oracle has them
    assert np.array_equal(keys, z.keys)
    rel = value_bar.max_rel_err(vals, z.vals)
    print(f"esc_large full size, sampled rows: max rel err vs FP64 {rel:.3e} over {vals.shape[0]} outputs")

    # linearity: every value doubled -> same keys, values times four
    X2 = synth.CooTensor(list(X.dims), X.idx, (X.val * np.float32(2)).astype(np.float32))
    dx2 = ctx.upload(X2)
    try:
        r2, digs2, keys2, vals2 = _stream_rows(ctx, dx2, dx2, cx, cy, row_lo, row_hi)
    finally:
        dx2.free()
    assert r2.nnz == r.nnz and r2.ir_nnz == r.ir_nnz
    assert sum(d["key_hash"] for d in digs2) % (1 << 64) == sum(d["key_hash"] for d in digs) % (1 << 64)
    s1 = sum(d["val_sum"] for d in digs)
    s2 = sum(d["val_sum"] for d in digs2)
    a1 = sum(d["val_abs_sum"] for d in digs)
    assert abs(s2 - 4 * s1) <= 4 * 1e-7 * a1
    assert np.array_equal(keys2, keys)
    value_bar.max_rel_err(vals2, 4 * z.vals)


def test_dense_acc_full_size(ctx):
    sp = pytest.importorskip("scipy.sparse")
    X, Y, cx, cy = synth.dense_acc(scale=1.0)
    r = gb.SpTC(X, Y, cx, cy, ctx=ctx)
    fx = [m for m in range(X.order) if m not in cx]
    fy = [m for m in range(Y.order) if m not in cy]
    nrow = int(np.prod([X.dims[m] for m in fx]))
    ncol = int(np.prod([Y.dims[m] for m in fy]))
    nmid = int(np.prod([X.dims[m] for m in cx]))
    xi, xj = _lin(X, fx), _lin(X, cx)
    yj, yk = _lin(Y, cy), _lin(Y, fy)
    A = sp.csr_matrix((X.val.astype(np.float64), (xi, xj)), shape=(nrow, nmid))
    B = sp.csr_matrix((Y.val.astype(np.float64), (yj, yk)), shape=(nmid, ncol))
    z64 = (A @ B).toarray()
    A.data[:] = 1.0
    B.data[:] = 1.0
    nprod = (A @ B).toarray()  # products per output, exact integers
    assert r.ir_nnz == int(nprod.sum())
    # one free mode per side: the output key is row << Y_nfbits | column
    ynf = synth._bits(ncol)
    i = (r.keys >> np.uint64(ynf)).astype(np.int64)
    k = (r.keys & np.uint64((1 << ynf) - 1)).astype(np.int64)
    assert np.all(np.diff(r.keys.astype(np.int64)) > 0)
    assert r.nnz == int(np.count_nonzero(nprod))
    assert np.all(nprod[i, k] > 0)
    rel = value_bar.max_rel_err(r.vals, z64[i, k])
    print(f"dense_acc full size: max rel err vs FP64 {rel:.3e} over {r.nnz} outputs")
