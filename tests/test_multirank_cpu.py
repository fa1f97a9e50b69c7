"""Multi-rank host logic on CPU (gloo, two ranks): row shards planned by the
library's gsparc_plan_shards agree across ranks, cover every output row once,
balance matched-product mass, and the shards' outputs (computed here with the
CPU oracle on each rank's rows) concatenate in rank order into the full Z.
Scalars (nnz, products) are combined with all_reduce as the benchmark does."""
import os
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

WORLD = 2


def _rows(X, cx):
    import oracle_bind as ob
    shift, isc, ncb, nfb = ob.layout(X.dims, cx)
    keys = ob.linearize(X, cx, 0)
    xf = keys >> np.uint64(ncb)
    return keys, xf, ncb


def _row_products(X, Y, cx, cy):
    import oracle_bind as ob
    _, _, ncx, nfx = ob.layout(X.dims, cx)
    _, _, ncy, nfy = ob.layout(Y.dims, cy)
    xk, _ = ob.sort_pairs(ob.linearize(X, cx, 0), X.val, ncx + nfx)
    yk, _ = ob.sort_pairs(ob.linearize(Y, cy, 1), Y.val, ncy + nfy)
    _, cnt, _ = ob.index_match(xk, ncx, yk, nfy)
    xf = xk >> np.uint64(ncx)
    rows, inv = np.unique(xf, return_inverse=True)
    return rows, np.bincount(inv, weights=cnt.astype(np.float64)).astype(np.uint64)


def _worker(rank, init_file, out_q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, here)
    import gsparc_b200 as gb
    import oracle_bind as ob
    from gsparc_b200 import synth

    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank, world_size=WORLD)
    try:
        X, Y, cx, cy = synth.esc_large(scale=0.003, seed=5)
        rows, row_prod = _row_products(X, Y, cx, cy)
        bounds = gb.plan_shards(row_prod, WORLD)
        # every rank planned the same shards
        gathered = [torch.zeros(WORLD + 1, dtype=torch.int64) for _ in range(WORLD)]
        dist.all_gather(gathered, torch.from_numpy(bounds.astype(np.int64)))
        assert all(torch.equal(g, gathered[0]) for g in gathered)
        ra, rb = int(bounds[rank]), int(bounds[rank + 1])
        # this rank's X nonzeros: rows [ra, rb)
        _, xf, _ = _rows(X, cx)
        mine = (xf >= rows[ra]) & (xf < (rows[rb] if rb < rows.shape[0] else np.uint64(2**64 - 1)))
        Xs = X.subset(mine)
        Xs.dims = list(X.dims)
        z = ob.sptc(Xs, Y, cx, cy) if Xs.nnz else None
        keys = z.keys if z is not None else np.zeros(0, np.uint64)
        vals = z.vals if z is not None else np.zeros(0)
        ir = z.ir_nnz if z is not None else 0
        assert ir == int(row_prod[ra:rb].sum())
        tot = torch.tensor([keys.shape[0], ir], dtype=torch.int64)
        dist.all_reduce(tot)
        out_q.put((rank, keys, vals, int(tot[0]), int(tot[1])))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_row_shards_concatenate_into_full_result():
    import oracle_bind as ob
    from gsparc_b200 import synth
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with tempfile.TemporaryDirectory() as td:
        init = os.path.join(td, "init")
        procs = [ctx.Process(target=_worker, args=(r, init, q)) for r in range(WORLD)]
        for p in procs:
            p.start()
        res = [q.get(timeout=240) for _ in range(WORLD)]
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
    res.sort(key=lambda r: r[0])
    X, Y, cx, cy = synth.esc_large(scale=0.003, seed=5)
    full = ob.sptc(X, Y, cx, cy)
    keys = np.concatenate([r[1] for r in res])
    vals = np.concatenate([r[2] for r in res])
    assert np.array_equal(keys, full.keys)          # disjoint, ordered by rank
    assert np.allclose(vals, full.vals, rtol=1e-12, atol=0)
    assert res[0][3] == full.nnz and res[0][4] == full.ir_nnz   # all_reduce'd totals


def test_plan_shards_is_deterministic_and_contiguous():
    import gsparc_b200 as gb
    rp = np.array([5, 0, 7, 100, 1, 1, 1, 50, 0, 3], np.uint64)
    for n in (1, 2, 3, 5, 10, 12):
        b = gb.plan_shards(rp, n)
        assert b[0] == 0 and b[-1] == rp.shape[0]
        assert np.all(np.diff(b.astype(np.int64)) >= 0)
        assert np.array_equal(b, gb.plan_shards(rp, n))
