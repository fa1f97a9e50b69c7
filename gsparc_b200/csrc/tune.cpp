// tune.cpp -- measured choice of accumulator, tiles and output chunk size.
//
// The reference picks dense or ESC accumulation by a fixed rule on the
// output range and the free memory (include/gsparc/sptc.cuh:201-218) and
// partitions only when memory runs out (contraction.cuh:143-245).  Here the
// candidates are timed on the contraction itself: ESC for small rows (the
// on-chip sort path for rows of up to 1024 products, the windowed dense
// accumulator for the others) against the windowed dense accumulator for every
// row, each with the largest output chunk the budget allows, a quarter and a
// sixteenth of it (smaller chunks overlap delivery with compute sooner and
// hold less memory; larger ones launch less), and the tiles: rows of up to
// 256 or 2048 products on chip instead of 1024, heavy windows of half the
// outputs.  Choices are cached per operand shape.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "kernels.cuh"

namespace {

std::mutex g_mu;
std::map<std::string, gsparc_tuning> g_cache;

std::string shape_key(int device, const gsparc_tensor *X, const gsparc_tensor *Y, int nc, const int *cx,
                      const int *cy) {
    std::string k = std::to_string(device) + "|";
    for (const gsparc_tensor *t : {X, Y}) {
        k += std::to_string(t->order) + ":" + std::to_string(t->nnz) + ":";
        for (int m = 0; m < t->order; ++m) k += std::to_string(t->dims[m]) + ",";
        k += "|";
    }
    for (int i = 0; i < nc; ++i) k += std::to_string(cx[i]) + "-" + std::to_string(cy[i]) + ",";
    return k;
}

template <class F>
gsparc_status guard(F &&f) {
    try {
        f();
        gs::set_last_error("");
        return GSPARC_OK;
    } catch (const gs::Error &e) {
        gs::set_last_error(e.msg);
        return e.st;
    } catch (const std::bad_alloc &) {
        gs::set_last_error("host allocation failed");
        return GSPARC_ENOMEM;
    }
}

}  // namespace

extern "C" gsparc_status gsparc_autotune(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y,
                                         int nc, const int *cx, const int *cy, int retune, gsparc_tuning *out,
                                         void *stream) {
    return guard([&] {
        GS_REQUIRE(ctx && X && Y && out && cx && cy && nc >= 1, GSPARC_EINVAL, "null argument");
        int prev = -1;
        cudaGetDevice(&prev);
        if (prev != ctx->device) GS_CUDA(cudaSetDevice(ctx->device));
        const std::string key = shape_key(ctx->device, X, Y, nc, cx, cy);
        if (!retune) {
            std::lock_guard<std::mutex> lk(g_mu);
            auto it = g_cache.find(key);
            if (it != g_cache.end()) {
                *out = it->second;
                out->cached = 1;
                return;
            }
        }
        cudaStream_t s = (cudaStream_t)stream;
        cudaEvent_t e0, e1;
        GS_CUDA(cudaEventCreate(&e0));
        GS_CUDA(cudaEventCreate(&e1));
        gsparc_tuning t;
        std::memset(&t, 0, sizeof(t));
        t.ms = 1e300;
        uint64_t out_nnz = 0;
        const uint64_t light0 = ctx->light_row_max;
        const uint32_t cap0 = ctx->heavy_window_cap;
        auto run = [&](int accum, uint64_t chunk, uint64_t light, uint32_t cap) {
            gsparc_job job;
            std::memset(&job, 0, sizeof(job));
            job.x = X;
            job.y = Y;
            job.ncmodes = nc;
            job.cx = cx;
            job.cy = cy;
            job.accum = accum;
            job.sink.kind = GSPARC_SINK_DISCARD;
            gsparc_stats bst;
            std::memset(&bst, 0, sizeof(bst));
            ctx->light_row_max = light;
            ctx->heavy_window_cap = cap;
            GS_CUDA(cudaEventRecord(e0, s));
            gs::sptc_batch(ctx, &job, 1, chunk, &bst, s);
            GS_CUDA(cudaEventRecord(e1, s));
            GS_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            GS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            out_nnz = job.stats.nnz;
            const int i = t.ncandidates++;
            t.cand_accum[i] = accum;
            t.cand_chunk[i] = chunk;
            t.cand_light[i] = light;
            t.cand_cap[i] = cap;
            t.cand_ms[i] = ms;
            if (ms < t.ms) {
                t.ms = ms;
                t.accum = accum;
                t.max_chunk_nnz = chunk;
                t.light_row_max = light;
                t.heavy_window_cap = cap;
            }
        };
        try {
            run(GSPARC_ACCUM_ESC, 0, 0, 0);  // first run also warms the pool and learns nnz(Z)
            run(GSPARC_ACCUM_ESC, 0, 0, 0);
            run(GSPARC_ACCUM_DENSE, 0, 0, 0);
            const int acc = t.accum;
            // tiles: the on-chip ESC row limit (ESC only) and the heavy window
            if (acc == GSPARC_ACCUM_ESC) {
                run(acc, 0, 256, 0);
                run(acc, 0, 2048, 0);
            }
            run(acc, 0, t.light_row_max, (uint32_t)gs::kHeavyCap / 2);
            const uint64_t lb = t.light_row_max;
            const uint32_t cb = t.heavy_window_cap;
            for (uint64_t div : {4ull, 16ull}) {
                const uint64_t c = out_nnz / div;
                if (c >= (1ull << 20) && t.ncandidates < 8) run(acc, c, lb, cb);
            }
        } catch (...) {
            ctx->light_row_max = light0;
            ctx->heavy_window_cap = cap0;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        ctx->light_row_max = light0;
        ctx->heavy_window_cap = cap0;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        // the first run paid for warming up: drop it from the table
        for (int i = 1; i < t.ncandidates; ++i) {
            t.cand_accum[i - 1] = t.cand_accum[i];
            t.cand_chunk[i - 1] = t.cand_chunk[i];
            t.cand_light[i - 1] = t.cand_light[i];
            t.cand_cap[i - 1] = t.cand_cap[i];
            t.cand_ms[i - 1] = t.cand_ms[i];
        }
        t.ncandidates -= 1;
        t.ms = 1e300;
        for (int i = 0; i < t.ncandidates; ++i)
            if (t.cand_ms[i] < t.ms) {
                t.ms = t.cand_ms[i];
                t.accum = t.cand_accum[i];
                t.max_chunk_nnz = t.cand_chunk[i];
                t.light_row_max = t.cand_light[i];
                t.heavy_window_cap = t.cand_cap[i];
            }
        t.cached = 0;
        {
            std::lock_guard<std::mutex> lk(g_mu);
            g_cache[key] = t;
        }
        *out = t;
        if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    });
}
