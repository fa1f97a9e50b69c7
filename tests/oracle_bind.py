"""ctypes binding of the CPU oracle (oracle/oracle.c).  Test infrastructure only:
the tests, the smoke check and the benchmark's CPU-baseline leg use it as the
checker; the engine never does."""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import Sequence

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")
SPARTA_TTT = os.path.join(ORACLE_DIR, "_ref", "ttt")

_lib = None


def build_oracle() -> None:
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(ORACLE_DIR, "oracle.c")):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "oracle"], check=True)


class _Result(ctypes.Structure):
    _fields_ = [
        ("ir_nnz", ctypes.c_uint64),
        ("nnz", ctypes.c_uint64),
        ("x_nfbits", ctypes.c_int),
        ("y_nfbits", ctypes.c_int),
        ("ncbits_x", ctypes.c_int),
        ("ncbits_y", ctypes.c_int),
        ("keys", ctypes.POINTER(ctypes.c_uint64)),
        ("vals", ctypes.POINTER(ctypes.c_double)),
        ("abs_sums", ctypes.POINTER(ctypes.c_double)),
        ("nprod", ctypes.POINTER(ctypes.c_uint64)),
    ]


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.oracle_mode_bits.argtypes = [ctypes.c_uint64]
        L.oracle_mode_bits.restype = ctypes.c_int
        L.oracle_layout.argtypes = [ctypes.c_int, P, ctypes.c_int, P, P, P, P, P, P]
        L.oracle_linearize.argtypes = [ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int,
                                       ctypes.c_uint64, P, P]
        L.oracle_sort_pairs.argtypes = [ctypes.c_uint64, P, P, ctypes.c_int]
        L.oracle_index_match.argtypes = [ctypes.c_uint64, P, ctypes.c_int, ctypes.c_uint64, P,
                                         ctypes.c_int, P, P, P]
        L.oracle_sptc.argtypes = [ctypes.c_int, P, ctypes.c_uint64, P, P,
                                  ctypes.c_int, P, ctypes.c_uint64, P, P,
                                  ctypes.c_int, P, P, ctypes.c_uint64,
                                  ctypes.POINTER(ctypes.POINTER(_Result))]
        L.oracle_free.argtypes = [ctypes.POINTER(_Result)]
        L.oracle_read_tns.argtypes = [ctypes.c_char_p, P, P, P, P, P]
        L.oracle_read_quantum.argtypes = [ctypes.c_char_p, P, P, P, P, P]
        L.oracle_free_buf.argtypes = [P]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def mode_bits(d: int) -> int:
    return lib().oracle_mode_bits(int(d))


def layout(dims: Sequence[int], cmodes: Sequence[int]):
    order = len(dims)
    d = np.asarray(dims, np.uint64)
    c = np.asarray(cmodes, np.int32)
    shift = np.zeros(64, np.int32)
    isc = np.zeros(64, np.int32)
    fpos = np.zeros(64, np.int32)
    ncb = np.zeros(1, np.int32)
    nfb = np.zeros(1, np.int32)
    st = lib().oracle_layout(order, _p(d), len(c), _p(c), _p(shift), _p(isc), _p(fpos),
                             _p(ncb), _p(nfb))
    if st:
        raise ValueError(f"oracle_layout status {st}")
    return shift[:order].copy(), isc[:order].astype(bool), int(ncb[0]), int(nfb[0])


def linearize(t, cmodes, role: int) -> np.ndarray:
    d = np.asarray(t.dims, np.uint64)
    c = np.asarray(cmodes, np.int32)
    idx = np.ascontiguousarray(t.idx, dtype=np.uint64)
    keys = np.zeros(t.nnz, np.uint64)
    st = lib().oracle_linearize(t.order, _p(d), len(c), _p(c), role, t.nnz, _p(idx), _p(keys))
    if st:
        raise ValueError(f"oracle_linearize status {st}")
    return keys


def sort_pairs(keys: np.ndarray, vals: np.ndarray, nbits: int):
    k = np.ascontiguousarray(keys, np.uint64).copy()
    v = np.ascontiguousarray(vals, np.float32).copy()
    st = lib().oracle_sort_pairs(k.shape[0], _p(k), _p(v), nbits)
    if st:
        raise MemoryError("oracle_sort_pairs")
    return k, v


def index_match(xkeys, x_ncbits, ykeys, y_nfbits):
    xk = np.ascontiguousarray(xkeys, np.uint64)
    yk = np.ascontiguousarray(ykeys, np.uint64)
    nx = xk.shape[0]
    pos = np.zeros(nx, np.uint64)
    cnt = np.zeros(nx, np.uint64)
    pre = np.zeros(nx + 1, np.uint64)
    lib().oracle_index_match(nx, _p(xk), x_ncbits, yk.shape[0], _p(yk), y_nfbits,
                             _p(pos), _p(cnt), _p(pre))
    return pos, cnt, pre


@dataclass
class OracleZ:
    ir_nnz: int
    nnz: int
    x_nfbits: int
    y_nfbits: int
    keys: np.ndarray
    vals: np.ndarray
    abs_sums: np.ndarray
    nprod: np.ndarray


def sptc(X, Y, cx, cy, max_products: int = 200_000_000) -> OracleZ:
    dx = np.asarray(X.dims, np.uint64)
    dy = np.asarray(Y.dims, np.uint64)
    ix = np.ascontiguousarray(X.idx, np.uint64)
    iy = np.ascontiguousarray(Y.idx, np.uint64)
    vx = np.ascontiguousarray(X.val, np.float32)
    vy = np.ascontiguousarray(Y.val, np.float32)
    c1 = np.asarray(cx, np.int32)
    c2 = np.asarray(cy, np.int32)
    out = ctypes.POINTER(_Result)()
    st = lib().oracle_sptc(X.order, _p(dx), X.nnz, _p(ix), _p(vx),
                           Y.order, _p(dy), Y.nnz, _p(iy), _p(vy),
                           len(c1), _p(c1), _p(c2), max_products, ctypes.byref(out))
    if st:
        raise ValueError(f"oracle_sptc status {st}")
    r = out.contents
    n = int(r.nnz)
    def arr(ptr, dt):
        if n == 0:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt).copy()
    z = OracleZ(int(r.ir_nnz), n, r.x_nfbits, r.y_nfbits, arr(r.keys, np.uint64),
                arr(r.vals, np.float64), arr(r.abs_sums, np.float64), arr(r.nprod, np.uint64))
    lib().oracle_free(out)
    return z


def read_tns(path: str):
    return _read(lib().oracle_read_tns, path)


def read_quantum(path: str):
    return _read(lib().oracle_read_quantum, path)


def _read(fn, path: str):
    from gsparc_b200.synth import CooTensor
    order = np.zeros(1, np.int32)
    nnz = np.zeros(1, np.uint64)
    dims = np.zeros(64, np.uint64)
    pidx = ctypes.c_void_p()
    pval = ctypes.c_void_p()
    st = fn(path.encode(), _p(order), _p(nnz), _p(dims), ctypes.byref(pidx), ctypes.byref(pval))
    if st:
        raise ValueError(f"oracle read status {st}")
    o = int(order[0]); n = int(nnz[0])
    idx = np.ctypeslib.as_array(ctypes.cast(pidx, ctypes.POINTER(ctypes.c_uint64)),
                                shape=(o * max(n, 1),))[: o * n].reshape(o, n).copy()
    val = np.ctypeslib.as_array(ctypes.cast(pval, ctypes.POINTER(ctypes.c_float)),
                                shape=(max(n, 1),))[:n].copy()
    lib().oracle_free_buf(pidx)
    lib().oracle_free_buf(pval)
    return CooTensor([int(d) for d in dims[:o]], idx, val)


def decode_keys(keys: np.ndarray, X, Y, cx, cy) -> np.ndarray:
    """Output keys -> coordinates (X free modes ascending, then Y free modes)."""
    shx, iscx, ncx, nfx = layout(X.dims, cx)
    shy, iscy, ncy, nfy = layout(Y.dims, cy)
    cols = []
    k = keys.astype(np.uint64)
    xf = k >> np.uint64(nfy) if nfy < 64 else np.zeros_like(k)
    yf = k & np.uint64((1 << nfy) - 1) if nfy < 64 else k
    for m in range(X.order):
        if not iscx[m]:
            b = mode_bits(X.dims[m])
            cols.append((xf >> np.uint64(shx[m])) & np.uint64((1 << b) - 1))
    for m in range(Y.order):
        if not iscy[m]:
            b = mode_bits(Y.dims[m])
            cols.append((yf >> np.uint64(shy[m])) & np.uint64((1 << b) - 1))
    return np.stack(cols) if cols else np.zeros((0, keys.shape[0]), np.uint64)
