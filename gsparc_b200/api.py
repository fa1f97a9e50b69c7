"""Python host interface over the engine's C ABI (include/gsparc_b200.h).

Mirrors the reference's SpTC interface for this path:

* :func:`SpTC` is ``gsparc::SpTC`` (reference include/gsparc/sptc.cuh:16-26) with
  the TensorManager steps that precede it in main.cu:293-321; its
  ``dense_accumulator`` argument is the reference's ``-d`` (1 dense, 0 auto,
  -1 ESC).
* :func:`read_tns` is ``IOManager::ParseFromFile`` (include/gsparc/io_manager.tpp:24-34).
* :func:`layout`, :func:`linearize`, :func:`sort_pairs`, :func:`index_match` are
  the stage functions ``compute_nbtis/setup_slitom``, ``ConvertTensor``,
  ``sort_64`` and ``IndexMatch``.

Errors raise :class:`GsparcError` carrying the library's status code; the
reference calls ``exit()`` instead.  There is no CPU fallback: the compiled
library must be present (``python -m gsparc_b200.build``).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from .synth import CooTensor

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libgsparc_b200.so")
CLI_PATH = os.path.join(_PKG, "bin", "gsparc")

ACCUM_ESC, ACCUM_AUTO, ACCUM_DENSE = -1, 0, 1
SINK_DISCARD, SINK_DEVICE, SINK_HOST = 0, 1, 2

STATUS = {0: "ok", 1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "EIO", 5: "ETIMEOUT",
          6: "EUNSUPPORTED", 7: "EINTERNAL", 8: "ECALLBACK"}


class GsparcError(RuntimeError):
    def __init__(self, status: int, what: str, msg: str):
        super().__init__(f"{what}: {STATUS.get(status, status)}: {msg}")
        self.status = status


class _Coo(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int), ("dims", ctypes.POINTER(ctypes.c_uint64)),
                ("nnz", ctypes.c_uint64), ("idx", ctypes.POINTER(ctypes.c_void_p)),
                ("val", ctypes.c_void_p), ("on_device", ctypes.c_int)]


CHUNK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int)


class _Sink(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("on_chunk", CHUNK_FN), ("user", ctypes.c_void_p),
                ("host_keys", ctypes.c_void_p), ("host_vals", ctypes.c_void_p),
                ("host_capacity", ctypes.c_uint64), ("max_chunk_nnz", ctypes.c_uint64),
                ("key_words", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("ir_nnz", ctypes.c_uint64), ("nnz", ctypes.c_uint64), ("nnz_x", ctypes.c_uint64),
                ("nnz_y", ctypes.c_uint64), ("rows", ctypes.c_uint64), ("heavy_rows", ctypes.c_uint64),
                ("chunks", ctypes.c_uint64), ("nbits_x", ctypes.c_int), ("nbits_y", ctypes.c_int),
                ("ncbits", ctypes.c_int), ("nfbits_x", ctypes.c_int), ("nfbits_y", ctypes.c_int),
                ("accumulator", ctypes.c_int), ("t_linearize_ms", ctypes.c_double),
                ("t_sort_ms", ctypes.c_double), ("t_match_ms", ctypes.c_double),
                ("t_plan_ms", ctypes.c_double), ("t_contract_ms", ctypes.c_double),
                ("t_output_ms", ctypes.c_double), ("t_total_ms", ctypes.c_double),
                ("bytes_h2d", ctypes.c_uint64), ("bytes_d2h", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64), ("t_numeric_kernel_ms", ctypes.c_double),
                ("heavy_windows", ctypes.c_uint64), ("stream_rows", ctypes.c_uint64),
                ("verified_nnz", ctypes.c_uint64), ("verified_products", ctypes.c_uint64),
                ("verify_mismatch", ctypes.c_uint64), ("verify_skipped_rows", ctypes.c_uint64),
                ("max_rel_err", ctypes.c_double), ("max_abs_err", ctypes.c_double),
                ("x_parts", ctypes.c_uint64), ("y_parts", ctypes.c_uint64),
                ("kept_bitmap_bytes", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

EXPORTS = [
    "gsparc_version", "gsparc_status_string", "gsparc_last_error", "gsparc_ctx_create", "gsparc_ctx_reserve",
    "gsparc_ctx_set_verify", "gsparc_ctx_set_tiles", "gsparc_ctx_set_row_bitmaps", "gsparc_ctx_set_sort", "gsparc_host_pin",
    "gsparc_host_unpin",
    "gsparc_ctx_destroy", "gsparc_ctx_memory", "gsparc_tensor_upload", "gsparc_tensor_free",
    "gsparc_tensor_info", "gsparc_sptc", "gsparc_sptc_shard", "gsparc_read_tns", "gsparc_write_tns",
    "gsparc_free_host", "gsparc_layout", "gsparc_plan_shards", "gsparc_linearize",
    "gsparc_sort_pairs", "gsparc_index_match", "gsparc_digest_chunk", "gsparc_sptc_batch",
    "gsparc_serve_create", "gsparc_serve_destroy", "gsparc_serve_upload", "gsparc_serve_release",
    "gsparc_serve_submit", "gsparc_serve_poll", "gsparc_serve_wait", "gsparc_serve_stats",
    "gsparc_serve_reset_stats", "gsparc_serve_pause", "gsparc_serve_inject_alloc_failure",
    "gsparc_ctx_inject_alloc_failure", "gsparc_sptc_host", "gsparc_sptc_resident", "gsparc_tensor_download",
    "gsparc_read_quantum", "gsparc_autotune", "gsparc_plan_create", "gsparc_plan_chunks", "gsparc_plan_chunk",
    "gsparc_plan_job_output", "gsparc_plan_refresh", "gsparc_plan_execute", "gsparc_plan_check",
    "gsparc_plan_destroy", "gsparc_tensor_set_values",
]


class _PartOpts(ctypes.Structure):
    _fields_ = [("max_part_nnz_x", ctypes.c_uint64), ("max_part_nnz_y", ctypes.c_uint64)]


class _Job(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("ncmodes", ctypes.c_int),
                ("cx", ctypes.c_void_p), ("cy", ctypes.c_void_p), ("accum", ctypes.c_int),
                ("sink", _Sink), ("stats", Stats), ("status", ctypes.c_int)]


class _ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("lanes", ctypes.c_int),
                ("max_batch_jobs", ctypes.c_int), ("max_batch_nnz", ctypes.c_uint64),
                ("fifo", ctypes.c_int), ("age_ms", ctypes.c_double), ("max_chunk_nnz", ctypes.c_uint64)]


class ServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("batches", ctypes.c_uint64), ("max_batch", ctypes.c_uint64), ("ir_nnz", ctypes.c_uint64),
                ("nnz", ctypes.c_uint64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("wall_ms", ctypes.c_double),
                ("products_per_s", ctypes.c_double), ("resident_bytes", ctypes.c_uint64),
                ("peak_reserved_bytes", ctypes.c_uint64), ("max_in_flight", ctypes.c_uint64),
                ("retries", ctypes.c_uint64), ("chunks", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("accum", ctypes.c_int), ("max_chunk_nnz", ctypes.c_uint64), ("ms", ctypes.c_double),
                ("cached", ctypes.c_int), ("ncandidates", ctypes.c_int), ("cand_accum", ctypes.c_int * 8),
                ("cand_chunk", ctypes.c_uint64 * 8), ("cand_ms", ctypes.c_double * 8),
                ("light_row_max", ctypes.c_uint64), ("heavy_window_cap", ctypes.c_uint32),
                ("cand_light", ctypes.c_uint64 * 8), ("cand_cap", ctypes.c_uint32 * 8)]

    def as_dict(self) -> dict:
        n = self.ncandidates
        return {"accum": self.accum, "max_chunk_nnz": self.max_chunk_nnz, "ms": self.ms,
                "light_row_max": self.light_row_max, "heavy_window_cap": self.heavy_window_cap,
                "cached": bool(self.cached),
                "candidates": [(self.cand_accum[i], self.cand_chunk[i], self.cand_ms[i], self.cand_light[i],
                                self.cand_cap[i]) for i in range(n)]}


class Digest(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("key_hash", ctypes.c_uint64), ("unsorted", ctypes.c_uint64),
                ("first_key", ctypes.c_uint64), ("last_key", ctypes.c_uint64),
                ("val_sum", ctypes.c_double), ("val_abs_sum", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib():
    """Load the compiled library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m gsparc_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P, U64, I = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
    L.gsparc_version.restype = ctypes.c_char_p
    L.gsparc_status_string.restype = ctypes.c_char_p
    L.gsparc_status_string.argtypes = [I]
    L.gsparc_last_error.restype = ctypes.c_char_p
    L.gsparc_ctx_create.argtypes = [I, U64, ctypes.POINTER(P)]
    L.gsparc_ctx_reserve.argtypes = [P, U64]
    L.gsparc_ctx_set_verify.argtypes = [P, U64]
    L.gsparc_ctx_set_tiles.argtypes = [P, U64, ctypes.c_uint32]
    L.gsparc_ctx_set_row_bitmaps.argtypes = [P, I]
    L.gsparc_ctx_set_sort.argtypes = [P, I]
    L.gsparc_host_pin.argtypes = [P, U64]
    L.gsparc_host_unpin.argtypes = [P]
    L.gsparc_ctx_destroy.argtypes = [P]
    L.gsparc_ctx_memory.argtypes = [P, P, P, P]
    L.gsparc_tensor_upload.argtypes = [P, ctypes.POINTER(_Coo), P, ctypes.POINTER(P)]
    L.gsparc_tensor_free.argtypes = [P, P]
    L.gsparc_tensor_info.argtypes = [P, P, P, P]
    L.gsparc_tensor_download.argtypes = [P, P, P, P]
    L.gsparc_sptc.argtypes = [P, P, P, I, P, P, I, ctypes.POINTER(_Sink), ctypes.POINTER(Stats), P]
    L.gsparc_sptc_shard.argtypes = [P, P, P, I, P, P, I, I, I, ctypes.POINTER(_Sink),
                                    ctypes.POINTER(Stats), P]
    L.gsparc_sptc_host.argtypes = [P, ctypes.POINTER(_Coo), ctypes.POINTER(_Coo), I, P, P, I,
                                   ctypes.POINTER(_PartOpts), ctypes.POINTER(_Sink), ctypes.POINTER(Stats), P]
    L.gsparc_read_tns.argtypes = [ctypes.c_char_p, I, P, P, P, ctypes.POINTER(P), ctypes.POINTER(P)]
    L.gsparc_read_quantum.argtypes = [ctypes.c_char_p, I, P, P, P, ctypes.POINTER(P), ctypes.POINTER(P)]
    L.gsparc_write_tns.argtypes = [ctypes.c_char_p, I, U64, P, P]
    L.gsparc_free_host.argtypes = [P]
    L.gsparc_layout.argtypes = [I, P, I, P, P, P, P, P, P]
    L.gsparc_plan_shards.argtypes = [P, U64, I, P]
    L.gsparc_linearize.argtypes = [I, P, I, P, I, U64, P, P, P]
    L.gsparc_sort_pairs.argtypes = [P, U64, P, P, I, P]
    L.gsparc_index_match.argtypes = [P, U64, P, I, U64, P, I, P, P, P, P, P]
    L.gsparc_digest_chunk.argtypes = [P, P, U64, ctypes.POINTER(Digest), P]
    L.gsparc_sptc_batch.argtypes = [P, P, I, U64, ctypes.POINTER(Stats), P]
    L.gsparc_plan_create.argtypes = [P, P, I, U64, ctypes.POINTER(P), ctypes.POINTER(U64), P]
    L.gsparc_plan_chunks.argtypes = [P, ctypes.POINTER(U64)]
    L.gsparc_plan_chunk.argtypes = [P, U64, ctypes.POINTER(U64), ctypes.POINTER(U64)]
    L.gsparc_plan_job_output.argtypes = [P, I, ctypes.POINTER(U64), ctypes.POINTER(U64)]
    L.gsparc_plan_refresh.argtypes = [P, P]
    L.gsparc_plan_execute.argtypes = [P, U64, P, P, U64, P]
    L.gsparc_plan_check.argtypes = [P, P]
    L.gsparc_plan_destroy.argtypes = [P]
    L.gsparc_tensor_set_values.argtypes = [P, P, P, I, P]
    L.gsparc_autotune.argtypes = [P, P, P, I, P, P, I, ctypes.POINTER(Tuning), P]
    L.gsparc_sptc_resident.argtypes = [P, P, P, I, P, P, I, ctypes.POINTER(P), ctypes.POINTER(Stats), P]
    L.gsparc_serve_create.argtypes = [I, ctypes.POINTER(_ServerOpts), ctypes.POINTER(P)]
    L.gsparc_serve_destroy.argtypes = [P]
    L.gsparc_serve_upload.argtypes = [P, ctypes.POINTER(_Coo), ctypes.POINTER(P)]
    L.gsparc_serve_release.argtypes = [P, P]
    L.gsparc_serve_submit.argtypes = [P, ctypes.POINTER(_Job), ctypes.POINTER(U64)]
    L.gsparc_serve_poll.argtypes = [P, U64, ctypes.POINTER(I), ctypes.POINTER(_Job)]
    L.gsparc_serve_wait.argtypes = [P, U64, ctypes.c_double, ctypes.POINTER(_Job)]
    L.gsparc_serve_stats.argtypes = [P, ctypes.POINTER(ServeStats)]
    L.gsparc_serve_reset_stats.argtypes = [P]
    L.gsparc_serve_pause.argtypes = [P, I]
    L.gsparc_serve_inject_alloc_failure.argtypes = [P, U64]
    L.gsparc_ctx_inject_alloc_failure.argtypes = [P, U64]
    for name in EXPORTS:
        getattr(L, name).restype = getattr(L, name).restype if name in (
            "gsparc_version", "gsparc_status_string", "gsparc_last_error") else (
            None if name == "gsparc_free_host" else ctypes.c_int)
    _lib = L
    return L


def _check(st: int, what: str) -> None:
    if st != 0:
        msg = lib().gsparc_last_error().decode(errors="replace")
        raise GsparcError(st, what, msg)


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def version() -> str:
    return lib().gsparc_version().decode()


# ------------------------------------------------------------------ host helpers
def layout(dims: Sequence[int], cmodes: Sequence[int]):
    """(bits, shift, is_contract, ncbits, nfbits) of one operand."""
    order = len(dims)
    d = np.asarray(dims, np.uint64)
    c = np.asarray(cmodes, np.int32)
    bits = np.zeros(order, np.int32)
    shift = np.zeros(order, np.int32)
    isc = np.zeros(order, np.int32)
    ncb = np.zeros(1, np.int32)
    nfb = np.zeros(1, np.int32)
    _check(lib().gsparc_layout(order, _p(d), len(c), _p(c), _p(bits), _p(shift), _p(isc),
                               _p(ncb), _p(nfb)), "layout")
    return bits, shift, isc.astype(bool), int(ncb[0]), int(nfb[0])


def read_tns(path: str, nthreads: int = 0) -> CooTensor:
    return _read(lib().gsparc_read_tns, path, nthreads)


def read_quantum(path: str, nthreads: int = 0) -> CooTensor:
    """Quantum-chemistry directory (indices.txt + values.txt), the reference's -q
    (IOManager::_ReadQuantumData, include/gsparc/io_manager.tpp:310-484)."""
    return _read(lib().gsparc_read_quantum, path, nthreads)


def _read(fn, path: str, nthreads: int) -> CooTensor:
    order = np.zeros(1, np.int32)
    dims = np.zeros(32, np.uint64)
    nnz = np.zeros(1, np.uint64)
    pidx, pval = ctypes.c_void_p(), ctypes.c_void_p()
    _check(fn(path.encode(), nthreads, _p(order), _p(dims), _p(nnz), ctypes.byref(pidx), ctypes.byref(pval)),
           f"read({path})")
    o, n = int(order[0]), int(nnz[0])
    try:
        idx = np.ctypeslib.as_array(ctypes.cast(pidx, ctypes.POINTER(ctypes.c_uint64)),
                                    shape=(max(o * n, 1),))[: o * n].reshape(o, n).copy()
        val = np.ctypeslib.as_array(ctypes.cast(pval, ctypes.POINTER(ctypes.c_float)),
                                    shape=(max(n, 1),))[:n].copy()
    finally:
        lib().gsparc_free_host(pidx)
        lib().gsparc_free_host(pval)
    return CooTensor([int(x) for x in dims[:o]], idx, val)


def write_tns(path: str, idx: np.ndarray, val: np.ndarray) -> None:
    idx = np.ascontiguousarray(idx, np.uint64)
    val = np.ascontiguousarray(val, np.float32)
    _check(lib().gsparc_write_tns(path.encode(), idx.shape[0], idx.shape[1], _p(idx), _p(val)),
           f"write_tns({path})")


def plan_shards(row_prod: np.ndarray, nshards: int) -> np.ndarray:
    rp = np.ascontiguousarray(row_prod, np.uint64)
    out = np.zeros(nshards + 1, np.uint64)
    _check(lib().gsparc_plan_shards(_p(rp), rp.shape[0], nshards, _p(out)), "plan_shards")
    return out


# ------------------------------------------------------------------ engine
class Context:
    """One device and an HBM budget (replaces CudaMemoryPool, src/gsparc/cuda_memory.cpp:17-30)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._h = ctypes.c_void_p()
        _check(lib().gsparc_ctx_create(device, hbm_budget, ctypes.byref(self._h)), "ctx_create")
        self.device = device

    @property
    def handle(self):
        return self._h

    def reserve(self, nbytes: int = 0):
        """Map nbytes (0 = the whole budget) into the context's pool now, so later
        contractions do not grow the pool inside their stages."""
        _check(lib().gsparc_ctx_reserve(self._h, nbytes), "ctx_reserve")

    def inject_alloc_failure(self, nth: int):
        """Host-side fault injection: the nth device allocation of this context
        from now (1 = the next) fails with GSPARC_ENOMEM, once; 0 disarms."""
        _check(lib().gsparc_ctx_inject_alloc_failure(self._h, nth), "ctx_inject_alloc_failure")

    def set_tiles(self, light_row_max: int = 0, heavy_window_cap: int = 0):
        """Accumulation tiles of later contractions (0 = defaults): rows of up to
        light_row_max products use the on-chip ESC (<= 2048), heavy windows hold
        at most heavy_window_cap outputs."""
        _check(lib().gsparc_ctx_set_tiles(self._h, light_row_max, heavy_window_cap), "ctx_set_tiles")

    def set_sort(self, impl: int = 0):
        """Sort of the operands' (key, value) pairs: 0 = CUB onesweep (default),
        1 = this library's own stable radix sort; results are identical."""
        _check(lib().gsparc_ctx_set_sort(self._h, impl), "ctx_set_sort")

    def set_row_bitmaps(self, on: bool = True):
        """Keep heavy rows' column bitmaps from the symbolic to the numeric pass
        (default on; results are identical either way)."""
        _check(lib().gsparc_ctx_set_row_bitmaps(self._h, 1 if on else 0), "ctx_set_row_bitmaps")

    def set_verify(self, max_products: int):
        """FP64 verification of later contractions' outputs on the GPU (all rows
        up to max_products matched products, a sample of rows above; 0 = off);
        results in the stats: max_rel_err, max_abs_err, verified_nnz, ..."""
        _check(lib().gsparc_ctx_set_verify(self._h, max_products), "ctx_set_verify")

    def memory(self):
        a = np.zeros(3, np.uint64)
        _check(lib().gsparc_ctx_memory(self._h, _p(a[0:1]), _p(a[1:2]), _p(a[2:3])), "ctx_memory")
        return {"in_use": int(a[0]), "peak": int(a[1]), "budget": int(a[2])}

    def close(self):
        if self._h:
            _check(lib().gsparc_ctx_destroy(self._h), "ctx_destroy")
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, t: CooTensor, stream: int = 0) -> "DeviceTensor":
        return DeviceTensor(self, t, stream)


class DeviceTensor:
    """A COO tensor resident in the context's HBM budget."""

    def __init__(self, ctx: Context, t, stream: int = 0):
        self.ctx = ctx
        self._h = ctypes.c_void_p()
        order = len(t.dims)
        self.dims = [int(d) for d in t.dims]
        self._dims = np.asarray(self.dims, np.uint64)
        on_device = 0
        if isinstance(t.val, np.ndarray):  # host COO (CooTensor or any object with dims/idx/val arrays)
            self._idx = np.ascontiguousarray(t.idx, np.uint64)
            self._val = np.ascontiguousarray(t.val, np.float32)
            nnz = self._val.shape[0]
            ptrs = [self._idx[m].ctypes.data for m in range(order)]
            vptr = self._val.ctypes.data
        else:  # (dims, idx_tensor[order, nnz] uint64/int64 cuda, val_tensor float32 cuda)
            dims, idx, val = t.dims, t.idx, t.val
            nnz = int(val.shape[0])
            ptrs = [idx[m].data_ptr() for m in range(order)]
            vptr = val.data_ptr()
            on_device = 1 if idx.is_cuda else 0
            self._keep = (idx, val)
        arr = (ctypes.c_void_p * max(order, 1))(*ptrs)
        coo = _Coo(order, self._dims.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), nnz, arr,
                   vptr, on_device)
        _check(lib().gsparc_tensor_upload(ctx.handle, ctypes.byref(coo), ctypes.c_void_p(stream),
                                          ctypes.byref(self._h)), "tensor_upload")
        self.nnz = nnz
        self.order = order
        self._idx = self._val = None

    @property
    def handle(self):
        return self._h

    def set_values(self, val: np.ndarray, stream: int = 0) -> None:
        """Overwrite the values (same order as the uploaded COO), coordinates unchanged."""
        v = np.ascontiguousarray(val, np.float32)
        if v.shape[0] != self.nnz:
            raise ValueError("need one value per nonzero")
        _check(lib().gsparc_tensor_set_values(self.ctx.handle, self._h, _p(v), 0, ctypes.c_void_p(stream)),
               "tensor_set_values")

    def download(self) -> CooTensor:
        """Copy the tensor back to host memory."""
        idx = np.zeros((self.order, self.nnz), np.uint64)
        val = np.zeros(self.nnz, np.float32)
        _check(lib().gsparc_tensor_download(self._h, _p(idx), _p(val), None), "tensor_download")
        return CooTensor(list(self.dims), idx, val)

    def free(self):
        if self._h:
            _check(lib().gsparc_tensor_free(self.ctx.handle, self._h), "tensor_free")
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


@dataclass
class SpTCResult:
    nnz: int
    ir_nnz: int
    keys: Optional[np.ndarray]
    vals: Optional[np.ndarray]
    stats: dict = field(default_factory=dict)


def sptc(ctx: Context, X: DeviceTensor, Y: DeviceTensor, cx: Sequence[int], cy: Sequence[int],
         dense_accumulator: int = ACCUM_AUTO, sink: str = "host", max_chunk_nnz: int = 0,
         shard: int = 0, nshards: int = 1, stream: int = 0, on_chunk=None,
         host_keys: Optional[np.ndarray] = None, host_vals: Optional[np.ndarray] = None,
         key_words: int = 1) -> SpTCResult:
    """Z = X x_{cx,cy} Y on resident operands.

    sink: "host" (Z copied into numpy arrays), "discard" (computed chunk-wise
    in HBM and dropped, like the reference), "device" (``on_chunk(keys_ptr,
    vals_ptr, n, first)`` gets device pointers per chunk) or "ring" (chunks
    stream through the given ``host_keys``/``host_vals`` arrays, ``on_chunk``
    sees numpy views).  key_words=2 delivers 128-bit keys (needed when X's
    and Y's free bits exceed 64 together): with the host sink, keys come back
    as an (n, 2) uint64 array, low word first.
    """
    if len(cx) != len(cy):
        raise ValueError("cx and cy must have the same length")
    c1 = np.asarray(cx, np.int32)
    c2 = np.asarray(cy, np.int32)
    st = Stats()
    s = _Sink()
    s.max_chunk_nnz = max_chunk_nnz
    s.key_words = key_words
    kw = 2 if key_words == 2 else 1
    keep = []
    keys = vals = None
    if sink == "discard":
        s.kind = SINK_DISCARD
    elif sink == "device":
        if on_chunk is None:
            raise ValueError("device sink needs on_chunk")
        s.kind = SINK_DEVICE

        def _cb(user, k, v, n, first, on_dev):
            return int(bool(on_chunk(k, v, n, first)))
        s.on_chunk = CHUNK_FN(_cb)
        keep.append(s.on_chunk)
    elif sink in ("host", "ring"):
        s.kind = SINK_HOST
        if sink == "host":
            # exact size is known only after the symbolic pass: collect chunks
            parts = []

            def _cbh(user, k, v, n, first, on_dev):
                if first and k == s.host_keys + 8 * kw * first:
                    return 0  # whole-Z mode: the chunk already sits at its final place
                kk = np.ctypeslib.as_array(ctypes.cast(k, ctypes.POINTER(ctypes.c_uint64)), shape=(kw * n,)).copy() if n else np.zeros(0, np.uint64)
                vv = np.ctypeslib.as_array(ctypes.cast(v, ctypes.POINTER(ctypes.c_float)), shape=(n,)).copy() if n else np.zeros(0, np.float32)
                parts.append((first, kk, vv))
                return 0
            cap = 1 << 22
            hk = np.zeros(kw * cap, np.uint64) if host_keys is None else host_keys
            hv = np.zeros(cap, np.float32) if host_vals is None else host_vals
            s.host_keys = hk.ctypes.data
            s.host_vals = hv.ctypes.data
            s.host_capacity = min(hk.shape[0] // kw, hv.shape[0])
            s.on_chunk = CHUNK_FN(_cbh)
            keep += [s.on_chunk, hk, hv]
        else:
            if host_keys is None or host_vals is None:
                raise ValueError("ring sink needs host_keys and host_vals")
            s.host_keys = host_keys.ctypes.data
            s.host_vals = host_vals.ctypes.data
            s.host_capacity = min(host_keys.shape[0] // kw, host_vals.shape[0])
            if on_chunk is not None:
                def _cbr(user, k, v, n, first, on_dev):
                    return int(bool(on_chunk(host_keys[: kw * n], host_vals[:n], n, first)))
                s.on_chunk = CHUNK_FN(_cbr)
                keep.append(s.on_chunk)
    else:
        raise ValueError(f"unknown sink {sink!r}")
    _check(lib().gsparc_sptc_shard(ctx.handle, X.handle, Y.handle, len(c1), _p(c1), _p(c2),
                                   int(dense_accumulator), shard, nshards, ctypes.byref(s),
                                   ctypes.byref(st), ctypes.c_void_p(stream)), "sptc")
    if sink == "host":
        parts.sort(key=lambda p: p[0])
        if st.nnz <= s.host_capacity:
            # whole Z fits the staging arrays: chunks landed in order
            keys = np.array(np.ctypeslib.as_array(ctypes.cast(s.host_keys, ctypes.POINTER(ctypes.c_uint64)), shape=(kw * s.host_capacity,))[: kw * st.nnz])
            vals = np.array(np.ctypeslib.as_array(ctypes.cast(s.host_vals, ctypes.POINTER(ctypes.c_float)), shape=(s.host_capacity,))[: st.nnz])
        else:
            keys = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0, np.uint64)
            vals = np.concatenate([p[2] for p in parts]) if parts else np.zeros(0, np.float32)
        if kw == 2:
            keys = keys.reshape(-1, 2)
    return SpTCResult(int(st.nnz), int(st.ir_nnz), keys, vals, st.as_dict())


def _host_coo(t: CooTensor):
    """A gsparc_coo over host arrays (and the arrays it points into)."""
    dims = np.asarray([int(d) for d in t.dims], np.uint64)
    idx = np.ascontiguousarray(t.idx, np.uint64)
    val = np.ascontiguousarray(t.val, np.float32)
    order = len(t.dims)
    arr = (ctypes.c_void_p * max(order, 1))(*[idx[m].ctypes.data for m in range(order)])
    coo = _Coo(order, dims.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), int(val.shape[0]), arr,
               val.ctypes.data, 0)
    return coo, (dims, idx, val, arr)


def sptc_host(ctx: Context, X: CooTensor, Y: CooTensor, cx: Sequence[int], cy: Sequence[int],
              dense_accumulator: int = ACCUM_AUTO, max_part_nnz_x: int = 0, max_part_nnz_y: int = 0,
              sink: str = "host", max_chunk_nnz: int = 0, stream: int = 0, staging: int = 1 << 22) -> SpTCResult:
    """Z = X x Y for host operands that need not fit the HBM budget
    (gsparc_sptc_host): X is cut into output-row parts and Y into
    output-column parts (of at most max_part_nnz_* nonzeros, or sized from the
    budget), every pair is contracted, Z arrives in key order.  sink: "host"
    (Z returned as numpy arrays) or "discard"."""
    if len(cx) != len(cy):
        raise ValueError("cx and cy must have the same length")
    c1 = np.asarray(cx, np.int32)
    c2 = np.asarray(cy, np.int32)
    cox, kx = _host_coo(X)
    coy, ky = _host_coo(Y)
    opts = _PartOpts(max_part_nnz_x, max_part_nnz_y)
    st = Stats()
    s = _Sink()
    s.max_chunk_nnz = max_chunk_nnz
    keep = [kx, ky]
    parts = []
    if sink == "discard":
        s.kind = SINK_DISCARD
    elif sink == "host":
        s.kind = SINK_HOST
        hk = np.zeros(staging, np.uint64)
        hv = np.zeros(staging, np.float32)

        def _cb(user, k, v, n, first, on_dev):
            kk = np.ctypeslib.as_array(ctypes.cast(k, ctypes.POINTER(ctypes.c_uint64)), shape=(n,)).copy() if n else np.zeros(0, np.uint64)
            vv = np.ctypeslib.as_array(ctypes.cast(v, ctypes.POINTER(ctypes.c_float)), shape=(n,)).copy() if n else np.zeros(0, np.float32)
            parts.append((first, kk, vv))
            return 0
        s.host_keys = hk.ctypes.data
        s.host_vals = hv.ctypes.data
        s.host_capacity = staging
        s.on_chunk = CHUNK_FN(_cb)
        keep += [hk, hv, s.on_chunk]
    else:
        raise ValueError(f"unknown sink {sink!r}")
    _check(lib().gsparc_sptc_host(ctx.handle, ctypes.byref(cox), ctypes.byref(coy), len(c1), _p(c1), _p(c2),
                                  int(dense_accumulator), ctypes.byref(opts), ctypes.byref(s), ctypes.byref(st),
                                  ctypes.c_void_p(stream)), "sptc_host")
    keys = vals = None
    if sink == "host":
        parts.sort(key=lambda p: p[0])
        keys = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0, np.uint64)
        vals = np.concatenate([p[2] for p in parts]) if parts else np.zeros(0, np.float32)
    return SpTCResult(int(st.nnz), int(st.ir_nnz), keys, vals, st.as_dict())


class ResidentResult(DeviceTensor):
    """A contraction result kept on the device (gsparc_sptc_resident): a
    COO operand whose modes are X's free modes then Y's free modes."""

    def __init__(self, ctx: Context, handle, stats: dict):
        self.ctx = ctx
        self._h = handle
        self.stats = stats
        order = ctypes.c_int()
        dims = np.zeros(32, np.uint64)
        nnz = ctypes.c_uint64()
        _check(lib().gsparc_tensor_info(handle, ctypes.byref(order), _p(dims), ctypes.byref(nnz)), "tensor_info")
        self.order = order.value
        self.dims = [int(d) for d in dims[: self.order]]
        self.nnz = nnz.value


class Plan:
    """Coordinate-only work of one or more contractions done once
    (gsparc_plan_*); ``execute(k, keys, vals)`` replays the numeric pass of
    output chunk k into device arrays (torch tensors or raw pointers) with
    launches only, so it can be captured in a CUDA graph.  ``refresh()`` picks
    up operand values changed with ``DeviceTensor.set_values``."""

    def __init__(self, ctx: Context, jobs, max_chunk_nnz: int = 0, stream: int = 0):
        self.ctx = ctx
        n = len(jobs)
        arr = (_Job * n)()
        self._keep = []
        for j, job in enumerate(jobs):
            X, Y, cx, cy = job[:4]
            c1 = np.asarray(cx, np.int32)
            c2 = np.asarray(cy, np.int32)
            self._keep += [c1, c2, X, Y]
            arr[j].x, arr[j].y = X.handle, Y.handle
            arr[j].ncmodes = len(c1)
            arr[j].cx, arr[j].cy = c1.ctypes.data, c2.ctypes.data
            arr[j].accum = int(job[4]) if len(job) > 4 else ACCUM_AUTO
        self._h = ctypes.c_void_p()
        tot = ctypes.c_uint64()
        _check(lib().gsparc_plan_create(ctx.handle, ctypes.cast(arr, ctypes.c_void_p), n, max_chunk_nnz,
                                        ctypes.byref(self._h), ctypes.byref(tot), ctypes.c_void_p(stream)),
               "plan_create")
        self.total = tot.value
        nc = ctypes.c_uint64()
        _check(lib().gsparc_plan_chunks(self._h, ctypes.byref(nc)), "plan_chunks")
        self.nchunks = nc.value
        self.njobs = n

    def chunk(self, k: int):
        f, m = ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().gsparc_plan_chunk(self._h, k, ctypes.byref(f), ctypes.byref(m)), "plan_chunk")
        return f.value, m.value

    def job_output(self, j: int):
        f, m = ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().gsparc_plan_job_output(self._h, j, ctypes.byref(f), ctypes.byref(m)), "plan_job_output")
        return f.value, m.value

    def refresh(self, stream: int = 0):
        _check(lib().gsparc_plan_refresh(self._h, ctypes.c_void_p(stream)), "plan_refresh")

    def execute(self, k: int, keys, vals, stream: int = 0):
        kp = keys.data_ptr() if hasattr(keys, "data_ptr") else int(keys)
        vp = vals.data_ptr() if hasattr(vals, "data_ptr") else int(vals)
        cap = min(keys.numel(), vals.numel()) if hasattr(keys, "numel") else self.chunk(k)[1]
        _check(lib().gsparc_plan_execute(self._h, k, ctypes.c_void_p(kp), ctypes.c_void_p(vp), cap,
                                         ctypes.c_void_p(stream)), "plan_execute")

    def check(self, stream: int = 0):
        _check(lib().gsparc_plan_check(self._h, ctypes.c_void_p(stream)), "plan_check")

    def close(self):
        if self._h:
            _check(lib().gsparc_plan_destroy(self._h), "plan_destroy")
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(ctx: Context, X: DeviceTensor, Y: DeviceTensor, cx: Sequence[int], cy: Sequence[int],
             retune: bool = False, stream: int = 0) -> dict:
    """Measured choice of accumulator, tiles and output chunk size for Z = X x Y
    (gsparc_autotune): {"accum", "max_chunk_nnz", "light_row_max",
    "heavy_window_cap", "ms", "cached", "candidates"}; candidates are
    (accum, max_chunk_nnz, ms, light_row_max, heavy_window_cap)."""
    if len(cx) != len(cy):
        raise ValueError("cx and cy must have the same length")
    c1 = np.asarray(cx, np.int32)
    c2 = np.asarray(cy, np.int32)
    t = Tuning()
    _check(lib().gsparc_autotune(ctx.handle, X.handle, Y.handle, len(c1), _p(c1), _p(c2), int(retune),
                                 ctypes.byref(t), ctypes.c_void_p(stream)), "autotune")
    return t.as_dict()


def sptc_resident(ctx: Context, X: DeviceTensor, Y: DeviceTensor, cx: Sequence[int], cy: Sequence[int],
                  dense_accumulator: int = ACCUM_AUTO, stream: int = 0) -> ResidentResult:
    """Z = X x_{cx,cy} Y kept resident, usable as an operand of further
    contractions (the reference's multi-SpTC chaining)."""
    if len(cx) != len(cy):
        raise ValueError("cx and cy must have the same length")
    c1 = np.asarray(cx, np.int32)
    c2 = np.asarray(cy, np.int32)
    st = Stats()
    h = ctypes.c_void_p()
    _check(lib().gsparc_sptc_resident(ctx.handle, X.handle, Y.handle, len(c1), _p(c1), _p(c2),
                                      int(dense_accumulator), ctypes.byref(h), ctypes.byref(st),
                                      ctypes.c_void_p(stream)), "sptc_resident")
    return ResidentResult(ctx, h, st.as_dict())


def sptc_batch(ctx: Context, jobs, sink: str = "host", max_chunk_nnz: int = 0, stream: int = 0,
               staging: int = 1 << 20, on_chunk=None, raise_on_error: bool = True):
    """Many contractions in one call (gsparc_sptc_batch).

    jobs: sequence of ``(X, Y, cx, cy)`` or ``(X, Y, cx, cy, accum)`` with
    resident DeviceTensors.  sink: "host" (every job's Z copied into numpy
    arrays through one shared staging buffer of ``staging`` entries),
    "discard", or "device" (``on_chunk(job, keys_ptr, vals_ptr, n, first)``
    with device pointers).  Returns ``(results, batch_stats)``; a failed job's
    result has ``keys is None`` and its status in ``stats["status"]``.
    """
    n = len(jobs)
    arr = (_Job * max(n, 1))()
    keep = []
    parts = [[] for _ in range(n)]
    hk = hv = None
    if sink == "host":
        hk = np.zeros(staging, np.uint64)
        hv = np.zeros(staging, np.float32)
        keep += [hk, hv]

        def _cbh(user, k, v, m, first, on_dev):
            j = int(user or 0)
            kk = np.ctypeslib.as_array(ctypes.cast(k, ctypes.POINTER(ctypes.c_uint64)), shape=(m,)).copy()
            vv = np.ctypeslib.as_array(ctypes.cast(v, ctypes.POINTER(ctypes.c_float)), shape=(m,)).copy()
            parts[j].append((first, kk, vv))
            return 0
        cb = CHUNK_FN(_cbh)
    elif sink == "device":
        if on_chunk is None:
            raise ValueError("device sink needs on_chunk")

        def _cbd(user, k, v, m, first, on_dev):
            return int(bool(on_chunk(int(user or 0), k, v, m, first)))
        cb = CHUNK_FN(_cbd)
    elif sink == "discard":
        cb = None
    else:
        raise ValueError(f"unknown sink {sink!r}")
    if cb is not None:
        keep.append(cb)
    for j, job in enumerate(jobs):
        X, Y, cx, cy = job[:4]
        accum = job[4] if len(job) > 4 else ACCUM_AUTO
        if len(cx) != len(cy):
            raise ValueError("cx and cy must have the same length")
        c1 = np.asarray(cx, np.int32)
        c2 = np.asarray(cy, np.int32)
        keep += [c1, c2]
        J = arr[j]
        J.x = X.handle
        J.y = Y.handle
        J.ncmodes = len(c1)
        J.cx = c1.ctypes.data
        J.cy = c2.ctypes.data
        J.accum = int(accum)
        J.sink.user = j
        if sink == "host":
            J.sink.kind = SINK_HOST
            J.sink.host_keys = hk.ctypes.data
            J.sink.host_vals = hv.ctypes.data
            J.sink.host_capacity = staging
            J.sink.on_chunk = cb
        elif sink == "device":
            J.sink.kind = SINK_DEVICE
            J.sink.on_chunk = cb
        else:
            J.sink.kind = SINK_DISCARD
    st = Stats()
    rc = lib().gsparc_sptc_batch(ctx.handle, ctypes.cast(arr, ctypes.c_void_p), n, max_chunk_nnz,
                                 ctypes.byref(st), ctypes.c_void_p(stream))
    if rc != 0 and raise_on_error:
        _check(rc, "sptc_batch")
    results = []
    for j in range(n):
        J = arr[j]
        d = J.stats.as_dict()
        d["status"] = int(J.status)
        keys = vals = None
        if J.status == 0 and sink == "host":
            ps = sorted(parts[j], key=lambda p: p[0])
            keys = np.concatenate([p[1] for p in ps]) if ps else np.zeros(0, np.uint64)
            vals = np.concatenate([p[2] for p in ps]) if ps else np.zeros(0, np.float32)
        results.append(SpTCResult(int(J.stats.nnz), int(J.stats.ir_nnz), keys, vals, d))
    bd = st.as_dict()
    bd["status"] = int(rc)
    return results, bd


class ServerTensor:
    """An operand resident in a :class:`Server`'s HBM budget."""

    def __init__(self, srv: "Server", t: CooTensor):
        self.srv = srv
        self._h = ctypes.c_void_p()
        self.dims = [int(d) for d in t.dims]
        self.order = len(self.dims)
        dims = np.asarray(self.dims, np.uint64)
        idx = np.ascontiguousarray(t.idx, np.uint64)
        val = np.ascontiguousarray(t.val, np.float32)
        self.nnz = int(val.shape[0])
        arr = (ctypes.c_void_p * max(self.order, 1))(*[idx[m].ctypes.data for m in range(self.order)])
        coo = _Coo(self.order, dims.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), self.nnz, arr,
                   val.ctypes.data, 0)
        _check(lib().gsparc_serve_upload(srv.handle, ctypes.byref(coo), ctypes.byref(self._h)), "serve_upload")

    @property
    def handle(self):
        return self._h

    def release(self):
        if self._h and self.srv.handle:
            _check(lib().gsparc_serve_release(self.srv.handle, self._h), "serve_release")
        self._h = ctypes.c_void_p()


class Server:
    """Request loop with continuous batching (gsparc_serve_*).

    ``submit`` queues a contraction of resident operands and returns a ticket;
    ``wait`` returns its :class:`SpTCResult`.  Free lanes take waiting
    requests (shortest first, or in arrival order once they waited longer
    than ``age_ms``; ``fifo`` keeps arrival order), as many as the HBM budget
    admits, and run them as one batch; lanes run concurrently on their own
    streams.
    """

    def __init__(self, device: int = 0, hbm_budget: int = 0, lanes: int = 0, max_batch_jobs: int = 0,
                 max_batch_nnz: int = 0, fifo: bool = False, age_ms: float = 0.0, max_chunk_nnz: int = 0):
        o = _ServerOpts(hbm_budget, lanes, max_batch_jobs, max_batch_nnz, int(fifo), age_ms, max_chunk_nnz)
        self._h = ctypes.c_void_p()
        _check(lib().gsparc_serve_create(device, ctypes.byref(o), ctypes.byref(self._h)), "serve_create")
        self._pending = {}

    @property
    def handle(self):
        return self._h

    def upload(self, t: CooTensor) -> ServerTensor:
        return ServerTensor(self, t)

    def submit(self, X: ServerTensor, Y: ServerTensor, cx: Sequence[int], cy: Sequence[int],
               dense_accumulator: int = ACCUM_AUTO, sink: str = "host", staging: int = 1 << 20) -> int:
        """Queue Z = X x_{cx,cy} Y; sink "host" (Z returned by wait) or "discard"."""
        if len(cx) != len(cy):
            raise ValueError("cx and cy must have the same length")
        c1 = np.asarray(cx, np.int32)
        c2 = np.asarray(cy, np.int32)
        J = _Job()
        J.x, J.y = X.handle, Y.handle
        J.ncmodes = len(c1)
        J.cx, J.cy = c1.ctypes.data, c2.ctypes.data
        J.accum = int(dense_accumulator)
        keep = [c1, c2]
        parts = []
        if sink == "host":
            hk = np.zeros(staging, np.uint64)
            hv = np.zeros(staging, np.float32)

            def _cbh(user, k, v, m, first, on_dev):
                kk = np.ctypeslib.as_array(ctypes.cast(k, ctypes.POINTER(ctypes.c_uint64)), shape=(m,)).copy()
                vv = np.ctypeslib.as_array(ctypes.cast(v, ctypes.POINTER(ctypes.c_float)), shape=(m,)).copy()
                parts.append((first, kk, vv))
                return 0
            cb = CHUNK_FN(_cbh)
            keep += [hk, hv, cb]
            J.sink.kind = SINK_HOST
            J.sink.host_keys = hk.ctypes.data
            J.sink.host_vals = hv.ctypes.data
            J.sink.host_capacity = staging
            J.sink.on_chunk = cb
        elif sink == "discard":
            J.sink.kind = SINK_DISCARD
        else:
            raise ValueError(f"unknown sink {sink!r}")
        t = ctypes.c_uint64()
        _check(lib().gsparc_serve_submit(self._h, ctypes.byref(J), ctypes.byref(t)), "serve_submit")
        self._pending[t.value] = (keep, parts, sink)
        return t.value

    def poll(self, ticket: int) -> bool:
        d = ctypes.c_int()
        _check(lib().gsparc_serve_poll(self._h, ticket, ctypes.byref(d), None), "serve_poll")
        return bool(d.value)

    def wait(self, ticket: int, timeout_ms: float = -1.0, raise_on_error: bool = True) -> SpTCResult:
        J = _Job()
        rc = lib().gsparc_serve_wait(self._h, ticket, timeout_ms, ctypes.byref(J))
        if rc == 5:  # ETIMEOUT: still pending
            _check(rc, "serve_wait")
        keep, parts, sink = self._pending.pop(ticket, (None, [], "discard"))
        if rc != 0 and raise_on_error:
            _check(rc, "serve_wait")
        d = J.stats.as_dict()
        d["status"] = int(J.status) if rc == 0 else int(rc)
        keys = vals = None
        if rc == 0 and sink == "host":
            ps = sorted(parts, key=lambda p: p[0])
            keys = np.concatenate([p[1] for p in ps]) if ps else np.zeros(0, np.uint64)
            vals = np.concatenate([p[2] for p in ps]) if ps else np.zeros(0, np.float32)
        return SpTCResult(int(J.stats.nnz), int(J.stats.ir_nnz), keys, vals, d)

    def stats(self) -> dict:
        st = ServeStats()
        _check(lib().gsparc_serve_stats(self._h, ctypes.byref(st)), "serve_stats")
        return st.as_dict()

    def reset_stats(self) -> None:
        _check(lib().gsparc_serve_reset_stats(self._h), "serve_reset_stats")

    def pause(self, paused: bool = True) -> None:
        """Hold the lanes (no new batch starts) or resume them."""
        _check(lib().gsparc_serve_pause(self._h, int(bool(paused))), "serve_pause")

    def inject_alloc_failure(self, nth: int) -> None:
        """Host-side fault injection: every lane's nth device allocation from
        now fails with GSPARC_ENOMEM, once (0 disarms)."""
        _check(lib().gsparc_serve_inject_alloc_failure(self._h, nth), "serve_inject_alloc_failure")

    def close(self) -> None:
        if self._h:
            _check(lib().gsparc_serve_destroy(self._h), "serve_destroy")
            self._h = ctypes.c_void_p()
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def SpTC(X: CooTensor, Y: CooTensor, cx: Sequence[int], cy: Sequence[int],
         dense_accumulator: int = ACCUM_AUTO, device: int = 0, ctx: Optional[Context] = None,
         **kw) -> SpTCResult:
    """One-shot contraction of two host COO tensors (uploads, contracts, frees)."""
    own = ctx is None
    ctx = ctx or Context(device)
    try:
        dx = ctx.upload(X)
        dy = dx if Y is X else ctx.upload(Y)
        try:
            return sptc(ctx, dx, dy, cx, cy, dense_accumulator, **kw)
        finally:
            dx.free()
            if dy is not dx:
                dy.free()
    finally:
        if own:
            ctx.close()


# ------------------------------------------------------------------ stage functions (torch device tensors)
def linearize(dims, cmodes, role: int, idx_dev, stream: int = 0):
    """Keys of one operand; idx_dev is a [order, nnz] int64/uint64 CUDA tensor."""
    import torch
    order, nnz = idx_dev.shape
    d = np.asarray(dims, np.uint64)
    c = np.asarray(cmodes, np.int32)
    keys = torch.empty(nnz, dtype=torch.int64, device=idx_dev.device)
    idx_dev = idx_dev.contiguous()
    _check(lib().gsparc_linearize(order, _p(d), len(c), _p(c), role, nnz,
                                  ctypes.c_void_p(idx_dev.data_ptr()), ctypes.c_void_p(keys.data_ptr()),
                                  ctypes.c_void_p(stream)), "linearize")
    return keys


def sort_pairs(ctx: Context, keys, vals, nbits: int, stream: int = 0):
    """In-place stable sort of CUDA tensors (int64 keys, float32 vals) by the low nbits."""
    _check(lib().gsparc_sort_pairs(ctx.handle, keys.shape[0], ctypes.c_void_p(keys.data_ptr()),
                                   ctypes.c_void_p(vals.data_ptr()), nbits, ctypes.c_void_p(stream)),
           "sort_pairs")
    return keys, vals


def index_match(ctx: Context, xkeys, x_ncbits: int, ykeys, y_nfbits: int, stream: int = 0):
    """(pos, cnt, prefix, ir) for sorted CUDA key tensors (int64)."""
    import torch
    nx = xkeys.shape[0]
    dev = xkeys.device
    pos = torch.zeros(nx, dtype=torch.int64, device=dev)
    cnt = torch.zeros(nx, dtype=torch.int64, device=dev)
    pre = torch.zeros(nx + 1, dtype=torch.int64, device=dev)
    ir = np.zeros(1, np.uint64)
    _check(lib().gsparc_index_match(ctx.handle, nx, ctypes.c_void_p(xkeys.data_ptr()), x_ncbits,
                                    ykeys.shape[0], ctypes.c_void_p(ykeys.data_ptr()), y_nfbits,
                                    ctypes.c_void_p(pos.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
                                    ctypes.c_void_p(pre.data_ptr()), _p(ir), ctypes.c_void_p(stream)),
           "index_match")
    return pos, cnt, pre, int(ir[0])


def digest_chunk(keys_ptr: int, vals_ptr: int, n: int, stream: int = 0) -> dict:
    """Verification digest of n output nonzeros at device pointers."""
    d = Digest()
    _check(lib().gsparc_digest_chunk(ctypes.c_void_p(keys_ptr), ctypes.c_void_p(vals_ptr), n,
                                     ctypes.byref(d), ctypes.c_void_p(stream)), "digest_chunk")
    return d.as_dict()


def splitmix64(k: np.ndarray) -> np.ndarray:
    """Host twin of the digest's key mix (mod 2^64)."""
    with np.errstate(over="ignore"):
        x = np.asarray(k, np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return x ^ (x >> np.uint64(31))


def decode_keys(keys: np.ndarray, x_dims, y_dims, cx, cy) -> np.ndarray:
    """Output keys -> coordinates [X free modes ascending, Y free modes ascending].
    keys: uint64 keys, or (n, 2) uint64 128-bit keys (low word first)."""
    bx, sx, icx, ncx, nfx = layout(x_dims, cx)
    by, sy, icy, ncy, nfy = layout(y_dims, cy)
    k = np.asarray(keys, np.uint64)
    if k.ndim == 2:  # 128-bit keys: x_f << nfy | y_f with x_f, y_f of at most 64 bits each
        lo, hi = k[:, 0], k[:, 1]
        if nfy == 0:
            xf, yf = lo, np.zeros_like(lo)
        elif nfy >= 64:
            xf, yf = hi, lo
        else:
            xf = (hi << np.uint64(64 - nfy)) | (lo >> np.uint64(nfy))
            yf = lo & np.uint64((1 << nfy) - 1)
        k = lo
    else:
        xf = k >> np.uint64(nfy) if nfy < 64 else np.zeros_like(k)
        yf = k & np.uint64((1 << nfy) - 1) if nfy < 64 else k
    cols = []
    for m in range(len(x_dims)):
        if not icx[m]:
            cols.append((xf >> np.uint64(sx[m])) & np.uint64((1 << int(bx[m])) - 1))
    for m in range(len(y_dims)):
        if not icy[m]:
            cols.append((yf >> np.uint64(sy[m])) & np.uint64((1 << int(by[m])) - 1))
    return np.stack(cols) if cols else np.zeros((0, k.shape[0]), np.uint64)
