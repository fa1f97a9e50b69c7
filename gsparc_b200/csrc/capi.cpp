// capi.cpp -- the C ABI (include/gsparc_b200.h): argument checks, exception to
// status translation, context and resident-tensor management.
#include <cstdlib>
#include <cstring>
#include <new>

#include "engine.h"
#include "kernels.cuh"

using gs::Error;

namespace {

template <class F>
gsparc_status guard(F &&f) {
    try {
        f();
        gs::set_last_error("");
        return GSPARC_OK;
    } catch (const Error &e) {
        gs::set_last_error(e.msg);
        return e.st;
    } catch (const std::bad_alloc &) {
        gs::set_last_error("host allocation failed");
        return GSPARC_ENOMEM;
    } catch (const std::exception &e) {
        gs::set_last_error(e.what());
        return GSPARC_EINTERNAL;
    }
}

struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) GS_CUDA(cudaSetDevice(dev));
    }
    ~DeviceScope() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" {

const char *gsparc_version(void) { return "gsparc-b200 0.1.0 (sm_100a)"; }

const char *gsparc_status_string(gsparc_status st) {
    switch (st) {
    case GSPARC_OK: return "ok";
    case GSPARC_EINVAL: return "invalid argument";
    case GSPARC_ENOMEM: return "out of memory";
    case GSPARC_ECUDA: return "CUDA error";
    case GSPARC_EIO: return "I/O error";
    case GSPARC_ETIMEOUT: return "device wait timed out";
    case GSPARC_EUNSUPPORTED: return "unsupported";
    case GSPARC_EINTERNAL: return "internal error";
    case GSPARC_ECALLBACK: return "stopped by callback";
    }
    return "unknown status";
}

const char *gsparc_last_error(void) { return gs::last_error(); }

gsparc_status gsparc_ctx_create(int device, uint64_t budget, gsparc_ctx **out) {
    return guard([&] {
        GS_REQUIRE(out, GSPARC_EINVAL, "out is null");
        *out = nullptr;
        int ndev = 0;
        GS_CUDA(cudaGetDeviceCount(&ndev));
        GS_REQUIRE(device >= 0 && device < ndev, GSPARC_EINVAL, "no such device");
        DeviceScope ds(device);
        auto *ctx = new gsparc_ctx();
        try {
            ctx->device = device;
            GS_CUDA(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
            size_t fr = 0, tot = 0;
            GS_CUDA(cudaMemGetInfo(&fr, &tot));
            if (budget == 0) budget = (uint64_t)(fr * 0.9);
            ctx->arena.init(device, budget);
            for (auto &e : ctx->ev) GS_CUDA(cudaEventCreate(&e));
            GS_CUDA(cudaMalloc(&ctx->d_flag, 64));
            GS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
            GS_CUDA(cudaStreamCreateWithFlags(&ctx->alt_stream, cudaStreamNonBlocking));
            GS_CUDA(cudaMemset(ctx->d_flag, 0, 64));
        } catch (...) {
            delete ctx;
            throw;
        }
        *out = ctx;
    });
}

gsparc_status gsparc_ctx_destroy(gsparc_ctx *ctx) {
    return guard([&] {
        if (!ctx) return;
        DeviceScope ds(ctx->device);
        cudaDeviceSynchronize();
        for (auto &e : ctx->ev)
            if (e) cudaEventDestroy(e);
        if (ctx->d_flag) cudaFree(ctx->d_flag);
        if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
        if (ctx->alt_stream) cudaStreamDestroy(ctx->alt_stream);
        delete ctx;
    });
}

gsparc_status gsparc_host_pin(void *p, uint64_t bytes) {
    return guard([&] {
        GS_REQUIRE(p || bytes == 0, GSPARC_EINVAL, "null buffer");
        if (bytes) GS_CUDA(cudaHostRegister(p, bytes, cudaHostRegisterDefault));
    });
}

gsparc_status gsparc_host_unpin(void *p) {
    return guard([&] {
        GS_REQUIRE(p, GSPARC_EINVAL, "null buffer");
        GS_CUDA(cudaHostUnregister(p));
    });
}

gsparc_status gsparc_ctx_inject_alloc_failure(gsparc_ctx *ctx, uint64_t nth) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        ctx->arena.inject_failure(nth);
    });
}

gsparc_status gsparc_ctx_set_tiles(gsparc_ctx *ctx, uint64_t light_row_max, uint32_t heavy_window_cap) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        GS_REQUIRE(light_row_max <= gs::kLightCap / 2, GSPARC_EINVAL,
                   "light_row_max above " + std::to_string(gs::kLightCap / 2));
        GS_REQUIRE(heavy_window_cap == 0 || (heavy_window_cap >= 256 && heavy_window_cap <= (uint32_t)gs::kHeavyCap),
                   GSPARC_EINVAL, "heavy_window_cap must be 0 or 256.." + std::to_string(gs::kHeavyCap));
        ctx->light_row_max = light_row_max;
        ctx->heavy_window_cap = heavy_window_cap;
    });
}

gsparc_status gsparc_ctx_set_sort(gsparc_ctx *ctx, int impl) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        GS_REQUIRE(impl == 0 || impl == 1, GSPARC_EINVAL, "impl must be 0 (CUB) or 1 (this library's radix sort)");
        ctx->sort_impl = impl;
    });
}

gsparc_status gsparc_ctx_set_row_bitmaps(gsparc_ctx *ctx, int on) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        GS_REQUIRE(on == 0 || on == 1, GSPARC_EINVAL, "on must be 0 or 1");
        ctx->keep_row_bitmaps = on;
    });
}

gsparc_status gsparc_ctx_set_verify(gsparc_ctx *ctx, uint64_t max_products) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        ctx->verify_budget = max_products;
    });
}

gsparc_status gsparc_ctx_reserve(gsparc_ctx *ctx, uint64_t bytes) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        DeviceScope ds(ctx->device);
        ctx->arena.reserve(bytes, ctx->copy_stream);
    });
}

gsparc_status gsparc_ctx_memory(gsparc_ctx *ctx, uint64_t *in_use, uint64_t *peak, uint64_t *budget) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        if (in_use) *in_use = ctx->arena.in_use();
        if (peak) *peak = ctx->arena.peak();
        if (budget) *budget = ctx->arena.budget();
    });
}

gsparc_status gsparc_tensor_upload(gsparc_ctx *ctx, const gsparc_coo *coo, void *stream,
                                   gsparc_tensor **out) {
    return guard([&] {
        GS_REQUIRE(ctx && coo && out, GSPARC_EINVAL, "null argument");
        *out = nullptr;
        GS_REQUIRE(coo->order >= 1 && coo->order <= gs::kMaxOrder, GSPARC_EINVAL, "order must be 1..32");
        GS_REQUIRE(coo->dims, GSPARC_EINVAL, "dims is null");
        GS_REQUIRE(coo->nnz == 0 || (coo->idx && coo->val), GSPARC_EINVAL, "idx/val is null");
        DeviceScope ds(ctx->device);
        cudaStream_t s = (cudaStream_t)stream;
        auto *t = new gsparc_tensor();
        try {
            t->order = coo->order;
            t->nnz = coo->nnz;
            for (int m = 0; m < coo->order; ++m) {
                GS_REQUIRE(coo->dims[m] >= 1, GSPARC_EINVAL, "mode size must be >= 1");
                t->dims[m] = coo->dims[m];
            }
            const uint64_t n = coo->nnz;
            const size_t ib = sizeof(uint64_t) * coo->order * (n ? n : 1);
            const size_t vb = sizeof(float) * (n ? n : 1);
            t->d_idx = (uint64_t *)ctx->arena.alloc(ib, s);
            t->d_val = (float *)ctx->arena.alloc(vb, s);
            cudaMemcpyKind kind = coo->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
            for (int m = 0; m < coo->order && n; ++m) {
                GS_REQUIRE(coo->idx[m], GSPARC_EINVAL, "idx[m] is null");
                GS_CUDA(cudaMemcpyAsync(t->d_idx + (uint64_t)m * n, coo->idx[m], 8 * n, kind, s));
            }
            if (n) GS_CUDA(cudaMemcpyAsync(t->d_val, coo->val, 4 * n, kind, s));
            GS_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            if (t->d_idx) ctx->arena.free(t->d_idx, s);
            if (t->d_val) ctx->arena.free(t->d_val, s);
            delete t;
            throw;
        }
        *out = t;
    });
}

gsparc_status gsparc_tensor_free(gsparc_ctx *ctx, gsparc_tensor *t) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        if (!t) return;
        DeviceScope ds(ctx->device);
        GS_CUDA(cudaDeviceSynchronize());
        ctx->arena.free(t->d_idx, nullptr);
        ctx->arena.free(t->d_val, nullptr);
        GS_CUDA(cudaDeviceSynchronize());
        delete t;
    });
}

gsparc_status gsparc_tensor_download(const gsparc_tensor *t, uint64_t *idx, float *val, void *stream) {
    return guard([&] {
        GS_REQUIRE(t && (t->nnz == 0 || (idx && val)), GSPARC_EINVAL, "null argument");
        cudaStream_t s = (cudaStream_t)stream;
        const uint64_t n = t->nnz;
        if (n) {
            GS_CUDA(cudaMemcpyAsync(idx, t->d_idx, 8 * (size_t)t->order * n, cudaMemcpyDeviceToHost, s));
            GS_CUDA(cudaMemcpyAsync(val, t->d_val, 4 * n, cudaMemcpyDeviceToHost, s));
        }
        GS_CUDA(cudaStreamSynchronize(s));
    });
}

gsparc_status gsparc_tensor_info(const gsparc_tensor *t, int *order, uint64_t *dims, uint64_t *nnz) {
    return guard([&] {
        GS_REQUIRE(t, GSPARC_EINVAL, "null tensor");
        if (order) *order = t->order;
        if (dims)
            for (int m = 0; m < t->order; ++m) dims[m] = t->dims[m];
        if (nnz) *nnz = t->nnz;
    });
}

gsparc_status gsparc_sptc(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y, int ncmodes,
                          const int *cx, const int *cy, int accum, const gsparc_sink *sink,
                          gsparc_stats *stats, void *stream) {
    return gsparc_sptc_shard(ctx, X, Y, ncmodes, cx, cy, accum, 0, 1, sink, stats, stream);
}

gsparc_status gsparc_sptc_shard(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y,
                                int ncmodes, const int *cx, const int *cy, int accum, int shard,
                                int nshards, const gsparc_sink *sink, gsparc_stats *stats,
                                void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        DeviceScope ds(ctx->device);
        // one contraction = a batch of one job
        gsparc_job job;
        std::memset(&job, 0, sizeof(job));
        job.x = X;
        job.y = Y;
        job.ncmodes = ncmodes;
        job.cx = cx;
        job.cy = cy;
        job.accum = accum;
        if (sink) job.sink = *sink;
        gsparc_stats bst;
        std::memset(&bst, 0, sizeof(bst));
        try {
            gs::sptc_batch(ctx, &job, 1, sink ? sink->max_chunk_nnz : 0, &bst, (cudaStream_t)stream, shard,
                           nshards);
        } catch (const gs::Error &e) {
            // the job's own status is the precise one
            throw gs::Error{job.status != GSPARC_OK ? job.status : e.st, e.msg};
        }
        if (stats) {
            gsparc_stats st = job.stats;
            st.chunks = bst.chunks;
            st.bytes_h2d = bst.bytes_h2d;
            st.bytes_d2h = bst.bytes_d2h;
            st.kernel_launches = bst.kernel_launches;
            st.t_numeric_kernel_ms = bst.t_numeric_kernel_ms;
            st.heavy_windows = bst.heavy_windows;
            st.stream_rows = bst.stream_rows;
            st.kept_bitmap_bytes = bst.kept_bitmap_bytes;
            *stats = st;
        }
    });
}

gsparc_status gsparc_sptc_host(gsparc_ctx *ctx, const gsparc_coo *X, const gsparc_coo *Y, int ncmodes,
                               const int *cx, const int *cy, int accum, const gsparc_part_opts *opts,
                               const gsparc_sink *sink, gsparc_stats *stats, void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        DeviceScope ds(ctx->device);
        gsparc_sink discard{};
        gs::sptc_partitioned(ctx, X, Y, ncmodes, cx, cy, accum, opts, sink ? sink : &discard, stats,
                             (cudaStream_t)stream);
    });
}

gsparc_status gsparc_sptc_resident(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y, int ncmodes,
                                   const int *cx, const int *cy, int accum, gsparc_tensor **Z,
                                   gsparc_stats *stats, void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        DeviceScope ds(ctx->device);
        gs::sptc_resident(ctx, X, Y, ncmodes, cx, cy, accum, Z, stats, (cudaStream_t)stream);
    });
}

gsparc_status gsparc_sptc_batch(gsparc_ctx *ctx, gsparc_job *jobs, int njobs, uint64_t max_chunk_nnz,
                                gsparc_stats *stats, void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        DeviceScope ds(ctx->device);
        gs::sptc_batch(ctx, jobs, njobs, max_chunk_nnz, stats, (cudaStream_t)stream);
    });
}

gsparc_status gsparc_plan_create(gsparc_ctx *ctx, const gsparc_job *jobs, int njobs, uint64_t max_chunk_nnz,
                                 gsparc_plan **out, uint64_t *total_nnz, void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
        DeviceScope ds(ctx->device);
        gs::plan_create(ctx, jobs, njobs, max_chunk_nnz, out, total_nnz, (cudaStream_t)stream);
    });
}

gsparc_status gsparc_plan_chunks(const gsparc_plan *plan, uint64_t *nchunks) {
    return guard([&] {
        GS_REQUIRE(plan && nchunks, GSPARC_EINVAL, "null argument");
        *nchunks = gs::plan_nchunks(plan);
    });
}

gsparc_status gsparc_plan_chunk(const gsparc_plan *plan, uint64_t k, uint64_t *first, uint64_t *nnz) {
    return guard([&] {
        GS_REQUIRE(plan, GSPARC_EINVAL, "null plan");
        gs::plan_chunk(plan, k, first, nnz);
    });
}

gsparc_status gsparc_plan_job_output(const gsparc_plan *plan, int job, uint64_t *first, uint64_t *nnz) {
    return guard([&] {
        GS_REQUIRE(plan, GSPARC_EINVAL, "null plan");
        gs::plan_job_output(plan, job, first, nnz);
    });
}

gsparc_status gsparc_plan_refresh(gsparc_plan *plan, void *stream) {
    return guard([&] { gs::plan_refresh(plan, (cudaStream_t)stream); });
}

gsparc_status gsparc_plan_execute(gsparc_plan *plan, uint64_t k, uint64_t *d_keys, float *d_vals,
                                  uint64_t capacity, void *stream) {
    return guard([&] { gs::plan_execute(plan, k, d_keys, d_vals, capacity, (cudaStream_t)stream); });
}

gsparc_status gsparc_plan_check(gsparc_plan *plan, void *stream) {
    return guard([&] { gs::plan_check(plan, (cudaStream_t)stream); });
}

gsparc_status gsparc_plan_destroy(gsparc_plan *plan) {
    return guard([&] { gs::plan_destroy(plan); });
}

gsparc_status gsparc_tensor_set_values(gsparc_ctx *ctx, gsparc_tensor *t, const float *val, int on_device,
                                       void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx && t && (t->nnz == 0 || val), GSPARC_EINVAL, "null argument");
        DeviceScope ds(ctx->device);
        cudaStream_t s = (cudaStream_t)stream;
        if (t->nnz)
            GS_CUDA(cudaMemcpyAsync(t->d_val, val, 4 * t->nnz,
                                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        GS_CUDA(cudaStreamSynchronize(s));
    });
}

gsparc_status gsparc_read_tns(const char *path, int nthreads, int *order, uint64_t *dims, uint64_t *nnz,
                              uint64_t **idx, float **val) {
    return guard([&] {
        GS_REQUIRE(path && order && dims && nnz && idx && val, GSPARC_EINVAL, "null argument");
        gs::read_tns(path, nthreads, order, dims, nnz, idx, val);
    });
}

gsparc_status gsparc_read_quantum(const char *dir, int nthreads, int *order, uint64_t *dims, uint64_t *nnz,
                                  uint64_t **idx, float **val) {
    return guard([&] {
        GS_REQUIRE(dir && order && dims && nnz && idx && val, GSPARC_EINVAL, "null argument");
        gs::read_quantum(dir, nthreads, order, dims, nnz, idx, val);
    });
}

gsparc_status gsparc_write_tns(const char *path, int order, uint64_t nnz, const uint64_t *idx,
                               const float *val) {
    return guard([&] {
        GS_REQUIRE(path && order >= 1 && order <= gs::kMaxOrder, GSPARC_EINVAL, "bad argument");
        GS_REQUIRE(nnz == 0 || (idx && val), GSPARC_EINVAL, "null data");
        gs::write_tns(path, order, nnz, idx, val);
    });
}

void gsparc_free_host(void *p) { std::free(p); }

gsparc_status gsparc_layout(int order, const uint64_t *dims, int ncmodes, const int *cmodes, int *bits,
                            int *shift, int *is_contract, int *ncbits, int *nfbits) {
    return guard([&] {
        GS_REQUIRE(dims && (ncmodes == 0 || cmodes), GSPARC_EINVAL, "null argument");
        gs::Layout L = gs::make_layout(order, dims, ncmodes, cmodes);
        for (int m = 0; m < order; ++m) {
            if (bits) bits[m] = L.bits[m];
            if (shift) shift[m] = L.shift[m];
            if (is_contract) is_contract[m] = L.is_c[m];
        }
        if (ncbits) *ncbits = L.ncbits;
        if (nfbits) *nfbits = L.nfbits;
    });
}

gsparc_status gsparc_plan_shards(const uint64_t *row_prod, uint64_t nrows, int nshards, uint64_t *bounds) {
    return guard([&] {
        GS_REQUIRE((row_prod || nrows == 0) && bounds, GSPARC_EINVAL, "null argument");
        gs::plan_shards(row_prod, nrows, nshards, bounds);
    });
}

gsparc_status gsparc_linearize(int order, const uint64_t *dims, int ncmodes, const int *cmodes, int role,
                               uint64_t nnz, const uint64_t *d_idx, uint64_t *d_keys, void *stream) {
    return guard([&] {
        GS_REQUIRE(dims && (ncmodes == 0 || cmodes) && (nnz == 0 || (d_idx && d_keys)), GSPARC_EINVAL,
                   "null argument");
        GS_REQUIRE(role == 0 || role == 1, GSPARC_EINVAL, "role must be 0 (X) or 1 (Y)");
        gs::Layout L = gs::make_layout(order, dims, ncmodes, cmodes);
        GS_REQUIRE(L.nbits() <= 64, GSPARC_EUNSUPPORTED, "keys wider than 64 bits");
        unsigned int *err = nullptr;
        GS_CUDA(cudaMalloc(&err, 4));
        cudaStream_t s = (cudaStream_t)stream;
        GS_CUDA(cudaMemsetAsync(err, 0, 4, s));
        gs::launch_linearize(gs::make_lin_params(L, dims, role), nnz, d_idx, nullptr, d_keys, nullptr, err, s);
        unsigned int h = 0;
        GS_CUDA(cudaMemcpyAsync(&h, err, 4, cudaMemcpyDeviceToHost, s));
        GS_CUDA(cudaStreamSynchronize(s));
        cudaFree(err);
        GS_REQUIRE(!h, GSPARC_EINVAL, "an index is not smaller than its mode size");
    });
}

gsparc_status gsparc_sort_pairs(gsparc_ctx *ctx, uint64_t n, uint64_t *d_keys, float *d_vals, int nbits,
                                void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx && (n == 0 || (d_keys && d_vals)), GSPARC_EINVAL, "null argument");
        GS_REQUIRE(nbits >= 0 && nbits <= 64, GSPARC_EINVAL, "nbits must be 0..64");
        DeviceScope ds(ctx->device);
        cudaStream_t s = (cudaStream_t)stream;
        gs::DBuf<uint64_t> k1(ctx->arena, n, s);
        gs::DBuf<float> v1(ctx->arena, n, s);
        int which = 0;
        unsigned int herr = 0;
        if (ctx->sort_impl) {
            gs::DBuf<unsigned int> err(ctx->arena, 1, s);
            GS_CUDA(cudaMemsetAsync(err.get(), 0, 4, s));
            gs::own_sort_pairs(ctx->arena, n, d_keys, k1, d_vals, v1, nbits, &which, err, s);
            GS_CUDA(cudaMemcpyAsync(&herr, err.get(), 4, cudaMemcpyDeviceToHost, s));
        } else {
            gs::sort_pairs(ctx->arena, n, d_keys, k1, d_vals, v1, nbits, &which, s);
        }
        if (which) {
            GS_CUDA(cudaMemcpyAsync(d_keys, k1.get(), 8 * n, cudaMemcpyDeviceToDevice, s));
            GS_CUDA(cudaMemcpyAsync(d_vals, v1.get(), 4 * n, cudaMemcpyDeviceToDevice, s));
        }
        GS_CUDA(cudaStreamSynchronize(s));
        GS_REQUIRE(!herr, GSPARC_EINTERNAL, "radix sort look-back gave up");
    });
}

gsparc_status gsparc_index_match(gsparc_ctx *ctx, uint64_t nx, const uint64_t *d_xkeys, int x_ncbits,
                                 uint64_t ny, const uint64_t *d_ykeys, int y_nfbits, uint64_t *d_pos,
                                 uint64_t *d_cnt, uint64_t *d_prefix, uint64_t *ir, void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx && d_prefix && (nx == 0 || (d_xkeys && d_pos && d_cnt)) && (ny == 0 || d_ykeys),
                   GSPARC_EINVAL, "null argument");
        GS_REQUIRE(x_ncbits >= 0 && x_ncbits <= 64 && y_nfbits >= 0 && y_nfbits <= 64, GSPARC_EINVAL,
                   "bit widths must be 0..64");
        DeviceScope ds(ctx->device);
        cudaStream_t s = (cudaStream_t)stream;
        gs::index_match_compat(ctx->arena, nx, d_xkeys, x_ncbits, ny, d_ykeys, y_nfbits, d_pos, d_cnt,
                               d_prefix, s);
        uint64_t h = 0;
        GS_CUDA(cudaMemcpyAsync(&h, d_prefix + nx, 8, cudaMemcpyDeviceToHost, s));
        GS_CUDA(cudaStreamSynchronize(s));
        if (ir) *ir = h;
    });
}

gsparc_status gsparc_digest_chunk(const uint64_t *d_keys, const float *d_vals, uint64_t n,
                                  gsparc_digest *out, void *stream) {
    return guard([&] {
        GS_REQUIRE(out && (n == 0 || (d_keys && d_vals)), GSPARC_EINVAL, "null argument");
        gs::digest_chunk(d_keys, d_vals, n, out, (cudaStream_t)stream);
    });
}

}  // extern "C"
