"""Seeded synthetic sparse tensors for the SpTC workloads.

The reference measures on FROSTT / quantum tensors that are not shipped with
it (reference: scripts/download_data.sh).  These generators stand in for them
with the shapes, sizes and value distributions of the five workloads the
engine is measured on:

* ``plain_small``   1000x1000x1000, 100k nnz, uniform coordinates, U[0,1),
  seed 0, self-contraction on the last mode (``-c 1 -x 2 -y 2``).
* ``esc_large``     2482x2862x14036x17, 3.1M nnz, Zipf(s=1.1) per mode,
  U[0,1), self-contraction on modes 2,3 (``-c 2 -x 2 3 -y 2 3``).
* ``dense_acc``     X 200x4096x4096 and Y 4096x4096x300, 10M nnz each,
  contract modes Zipf(s=1.2), free modes uniform, N(0,1)
  (``-c 2 -x 1 2 -y 0 1``).
* ``batched_instances`` / ``served_stream``: mixed instances (orders 3-4 /
  3-5, the served ones with Poisson arrival times).

Rules shared by every generator (they make the inferred dims of the written
``.tns`` file equal the nominal dims, which the reference derives from the
largest index it reads, reference: include/gsparc/io_manager.tpp:213,250-256):

* coordinates are unique: samples are drawn in batches and a coordinate that
  was already drawn is rejected, until the stated nnz is reached;
* the first nonzero is planted at the largest coordinate of every mode;
* a bounded Zipf(s) over ranks 1..dim maps rank r to 0-based index r-1;
* values are float32 and are written with ``%.9g`` so that the reference's
  ``(float)std::stod`` reads back the identical float.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Callable, List, Optional, Sequence

import numpy as np

__all__ = [
    "CooTensor",
    "make_tensor",
    "plain_small",
    "esc_large",
    "dense_acc",
    "write_tns",
    "read_tns_py",
    "batched_instances",
    "served_stream",
    "write_quantum",
    "WORKLOADS",
]


@dataclasses.dataclass
class CooTensor:
    """SoA COO tensor: ``idx[m][k]`` 0-based uint64, ``val[k]`` float32."""

    dims: List[int]
    idx: np.ndarray  # (order, nnz) uint64
    val: np.ndarray  # (nnz,) float32

    @property
    def order(self) -> int:
        return len(self.dims)

    @property
    def nnz(self) -> int:
        return int(self.val.shape[0])

    def subset(self, sel) -> "CooTensor":
        return CooTensor(list(self.dims), np.ascontiguousarray(self.idx[:, sel]),
                         np.ascontiguousarray(self.val[sel]))


def _zipf_cdf(dim: int, s: float) -> np.ndarray:
    r = np.arange(1, dim + 1, dtype=np.float64)
    w = r ** (-s)
    c = np.cumsum(w)
    return c / c[-1]


def _draw_mode(rng: np.random.Generator, dim: int, dist, n: int) -> np.ndarray:
    if dist == "uniform":
        return rng.integers(0, dim, size=n, dtype=np.uint64)
    kind, s = dist
    assert kind == "zipf"
    cdf = _zipf_cdf(dim, float(s))
    u = rng.random(n)
    out = np.searchsorted(cdf, u, side="right")
    np.minimum(out, dim - 1, out=out)
    return out.astype(np.uint64)


def _bits(d: int) -> int:
    return 0 if d <= 1 else int(d - 1).bit_length()


def _pack_rows(coords: np.ndarray, dims: Sequence[int]) -> np.ndarray:
    """Pack rows of coordinates into sortable keys (uint64 or void rows)."""
    tot = sum(_bits(d) for d in dims)
    if tot <= 64:
        key = np.zeros(coords.shape[1], dtype=np.uint64)
        for m, d in enumerate(dims):
            key <<= np.uint64(_bits(d))
            key |= coords[m]
        return key
    # wide coordinates: compare whole rows
    rows = np.ascontiguousarray(coords.T)
    return rows.view(np.dtype((np.void, rows.dtype.itemsize * rows.shape[1]))).ravel()


def _first_occurrences(k: np.ndarray):
    """Positions (ascending) of the first occurrence of each distinct key."""
    order = np.argsort(k, kind="stable")
    ks = k[order]
    keep = np.ones(ks.shape[0], dtype=bool)
    if ks.shape[0] > 1:
        keep[1:] = ks[1:] != ks[:-1]
    first = np.sort(order[keep])
    return first, k[first]


def _sorted_contains(sorted_keys: np.ndarray, q: np.ndarray) -> np.ndarray:
    pos = np.searchsorted(sorted_keys, q)
    pos_c = np.minimum(pos, sorted_keys.shape[0] - 1)
    return (pos < sorted_keys.shape[0]) & (sorted_keys[pos_c] == q)


def make_tensor(dims: Sequence[int], nnz: int, mode_dists, values: str, seed: int,
                plant_max: bool = True) -> CooTensor:
    """Draw ``nnz`` unique coordinates (rejection sampling) and float32 values."""
    dims = [int(d) for d in dims]
    for d in dims:
        if d < 2:
            raise ValueError("size-1 modes are not generated")
    space = 1
    for d in dims:
        space *= d
    if nnz > space:
        raise ValueError("nnz exceeds the coordinate space")
    rng = np.random.default_rng(seed)
    order = len(dims)
    parts = []
    keys_seen = None
    count = 0
    if plant_max and nnz > 0:
        top = np.array([[d - 1] for d in dims], dtype=np.uint64)
        parts.append(top)
        keys_seen = np.sort(_pack_rows(top, dims))
        count = 1
    batch_min = 1 << 16
    while count < nnz:
        need = nnz - count
        n = max(batch_min, 2 * need)
        coords = np.stack([_draw_mode(rng, dims[m], mode_dists[m], n) for m in range(order)])
        k = _pack_rows(coords, dims)
        first, kf = _first_occurrences(k)
        if keys_seen is not None and keys_seen.size:
            fresh = ~_sorted_contains(keys_seen, kf)
            first = first[fresh]
            kf = kf[fresh]
        first = first[:need]
        kf = kf[:need]
        parts.append(coords[:, first])
        if keys_seen is None:
            keys_seen = np.sort(kf, kind="stable")
        else:
            keys_seen = np.sort(np.concatenate([keys_seen, np.sort(kf, kind="stable")]), kind="stable")
        count += first.size
        batch_min = min(batch_min * 2, 1 << 24)
    idx = np.concatenate(parts, axis=1) if parts else np.zeros((order, 0), np.uint64)
    if values == "u01":
        val = rng.random(nnz, dtype=np.float32)
    elif values == "normal":
        val = rng.standard_normal(nnz, dtype=np.float32)
    elif values == "u11":
        val = (rng.random(nnz, dtype=np.float32) * np.float32(2.0) - np.float32(1.0)).astype(np.float32)
    else:
        raise ValueError(values)
    return CooTensor(dims, np.ascontiguousarray(idx.astype(np.uint64)), val.astype(np.float32))


def plain_small(scale: float = 1.0, seed: int = 0):
    """X = 1000^3 with 100k uniform nnz; Z = X x_{2,2} X. Returns (X, Y, cx, cy)."""
    nnz = max(2, int(round(100_000 * scale)))
    X = make_tensor([1000, 1000, 1000], nnz, ["uniform"] * 3, "u01", seed)
    return X, X, [2], [2]


def esc_large(scale: float = 1.0, seed: int = 1):
    """X = 2482x2862x14036x17 Zipf(1.1), 3.1M nnz; Z = X x_{(2,3),(2,3)} X."""
    nnz = max(2, int(round(3_100_000 * scale)))
    X = make_tensor([2482, 2862, 14036, 17], nnz, [("zipf", 1.1)] * 4, "u01", seed)
    return X, X, [2, 3], [2, 3]


def dense_acc(scale: float = 1.0, seed: int = 2):
    """X 200x4096x4096, Y 4096x4096x300, 10M nnz each; contract the 4096 modes."""
    nnz = max(2, int(round(10_000_000 * scale)))
    X = make_tensor([200, 4096, 4096], nnz, ["uniform", ("zipf", 1.2), ("zipf", 1.2)],
                    "normal", seed)
    Y = make_tensor([4096, 4096, 300], nnz, [("zipf", 1.2), ("zipf", 1.2), "uniform"],
                    "normal", seed + 100)
    return X, Y, [1, 2], [0, 1]


def _make_pair(args):
    dx, dy, nnz_x, nnz_y, ox, oy, s, sx = args[:8]
    X = make_tensor(dx, nnz_x, [("zipf", s)] * ox, "u11", sx)
    Y = make_tensor(dy, nnz_y, [("zipf", s)] * oy, "u11", sx + 1)
    return X, Y


def batched_instances(count: int = 256, seed: int = 3, max_nnz: int = 1_000_000,
                      max_out_bits: int = 64, workers: int = 0):
    """Mixed instances: orders 3-4, modes log-uniform 64..100k, nnz log-uniform
    1e3..max_nnz, 1-2 contract modes, Zipf s in [1.0,1.4], U[-1,1).  Instances
    whose output key would need more than ``max_out_bits`` bits are redrawn.
    The tensors are drawn in ``workers`` spawned processes (0: one per core,
    up to 32); every instance has its own seed, so the result does not depend
    on the number of workers."""
    rng = np.random.default_rng(seed)
    params = []
    while len(params) < count:
        ox = int(rng.integers(3, 5))
        oy = int(rng.integers(3, 5))
        nc = int(rng.integers(1, 3))
        s = float(rng.uniform(1.0, 1.4))
        cdims = [int(round(math.exp(rng.uniform(math.log(64), math.log(100_000))))) for _ in range(nc)]
        fx = [int(round(math.exp(rng.uniform(math.log(64), math.log(100_000))))) for _ in range(ox - nc)]
        fy = [int(round(math.exp(rng.uniform(math.log(64), math.log(100_000))))) for _ in range(oy - nc)]
        if sum(_bits(d) for d in fx) + sum(_bits(d) for d in fy) > max_out_bits:
            continue
        if sum(_bits(d) for d in fx + cdims) > 64 or sum(_bits(d) for d in fy + cdims) > 64:
            continue
        nnz_x = int(round(math.exp(rng.uniform(math.log(1e3), math.log(max_nnz)))))
        nnz_y = int(round(math.exp(rng.uniform(math.log(1e3), math.log(max_nnz)))))
        # X: free modes first then contract modes; Y: contract modes first.
        dx = fx + cdims
        dy = cdims + fy
        cap_x = np.prod([float(d) for d in dx])
        cap_y = np.prod([float(d) for d in dy])
        nnz_x = int(min(nnz_x, cap_x // 4))
        nnz_y = int(min(nnz_y, cap_y // 4))
        sx = int(rng.integers(0, 2**31))
        params.append((dx, dy, nnz_x, nnz_y, ox, oy, s, sx, nc))
    return _build_pairs(params, workers)


def served_stream(count: int = 256, seed: int = 5, max_nnz: int = 2_000_000, min_nnz: int = 10_000,
                  nnz_s: float = 1.5, rate: float = 2000.0, max_out_bits: int = 64, workers: int = 0):
    """Requests of the served workload: operand orders 3-5, 1-2 contract modes,
    modes log-uniform 64..100k, operand nnz drawn from a power law
    p(n) ~ n^-nnz_s on [min_nnz, max_nnz] (inverse CDF), contract and free
    indices Zipf s in [1.0,1.4], U[-1,1) values, Poisson arrivals at ``rate``
    per second.  Operand keys may exceed 64 bits; instances whose output key
    would need more than ``max_out_bits`` bits are redrawn.  Returns
    ``(instances, arrival_seconds)``; instances are ``(X, Y, cx, cy)``."""
    rng = np.random.default_rng(seed)
    lo, hi, e = float(min_nnz), float(max_nnz), 1.0 - nnz_s

    def draw_nnz():
        u = rng.random()
        return int(round((lo ** e + u * (hi ** e - lo ** e)) ** (1.0 / e)))
    params = []
    while len(params) < count:
        ox = int(rng.integers(3, 6))
        oy = int(rng.integers(3, 6))
        nc = int(rng.integers(1, 3))
        s = float(rng.uniform(1.0, 1.4))
        logd = lambda: int(round(math.exp(rng.uniform(math.log(64), math.log(100_000)))))  # noqa: E731
        cdims = [logd() for _ in range(nc)]
        fx = [logd() for _ in range(ox - nc)]
        fy = [logd() for _ in range(oy - nc)]
        if sum(_bits(d) for d in fx) + sum(_bits(d) for d in fy) > max_out_bits:
            continue
        dx, dy = fx + cdims, cdims + fy
        nnz_x = int(min(draw_nnz(), np.prod([float(d) for d in dx]) // 4))
        nnz_y = int(min(draw_nnz(), np.prod([float(d) for d in dy]) // 4))
        params.append((dx, dy, nnz_x, nnz_y, ox, oy, s, int(rng.integers(0, 2**31)), nc))
    arrive = np.cumsum(rng.exponential(1.0 / rate, size=count))
    return _build_pairs(params, workers), arrive


def _build_pairs(params, workers: int):
    if workers == 0:
        workers = min(32, os.cpu_count() or 1)
    total = sum(p[2] + p[3] for p in params)
    if workers > 1 and total > 2_000_000:
        import concurrent.futures as cf
        import multiprocessing as mp
        with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            pairs = list(ex.map(_make_pair, params, chunksize=1))
    else:
        pairs = [_make_pair(p) for p in params]
    out = []
    for p, (X, Y) in zip(params, pairs):
        ox, nc = p[4], p[8]
        out.append((X, Y, list(range(ox - nc, ox)), list(range(nc))))
    return out


WORKLOADS = {
    "plain_small": plain_small,
    "esc_large": esc_large,
    "dense_acc": dense_acc,
}


def write_tns(path: str, t: CooTensor) -> None:
    """Write 1-based text COO, one nonzero per line, values as ``%.9g``."""
    cols = [np.char.mod("%d", (t.idx[m] + np.uint64(1)).astype(np.int64)) for m in range(t.order)]
    vals = np.char.mod("%.9g", t.val.astype(np.float64))
    with open(path, "w") as f:
        step = 1 << 20
        for s in range(0, t.nnz, step):
            e = min(t.nnz, s + step)
            rows = [" ".join(r) for r in zip(*[c[s:e] for c in cols], vals[s:e])]
            f.write("\n".join(rows))
            f.write("\n")


def write_quantum(path: str, t: CooTensor) -> None:
    """Write the quantum-chemistry directory format: ``path/indices.txt``, one
    line of 1-based indices per mode, and ``path/values.txt``, one value per
    line (``%.9g``)."""
    os.makedirs(path, exist_ok=True)
    with open(os.path.join(path, "indices.txt"), "w") as f:
        for m in range(t.order):
            f.write(" ".join(np.char.mod("%d", (t.idx[m] + np.uint64(1)).astype(np.int64))) + "\n")
    with open(os.path.join(path, "values.txt"), "w") as f:
        f.write("\n".join(np.char.mod("%.9g", t.val.astype(np.float64))) + "\n")


def read_tns_py(path: str) -> CooTensor:
    """Small pure-Python reader with the reference's dims rule (test helper)."""
    rows = []
    with open(path) as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            rows.append(tok)
    order = len(rows[0]) - 1
    idx = np.array([[int(r[m]) - 1 for r in rows] for m in range(order)], dtype=np.uint64)
    val = np.array([float(r[-1]) for r in rows], dtype=np.float64).astype(np.float32)
    dims = [int(idx[m].max()) + 1 for m in range(order)]
    return CooTensor(dims, idx, val)
