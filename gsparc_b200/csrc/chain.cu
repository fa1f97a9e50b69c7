// chain.cu -- a contraction whose result stays on the device as an operand.
//
// The reference chains two contractions (multi-SpTC, main.cu:323-371 and
// include/gsparc/sptc.cuh:362-698): the first result's keys
// (x_f << Y_nfbits | y_f) stay in memory and are reused directly as the next
// contraction's X keys, the Y free part in the low bits playing the contract
// part.  Here the result is decoded on the device into a COO tensor whose
// modes are X's free modes (ascending) followed by Y's free modes
// (ascending): a resident operand like any uploaded one, so the next
// contraction may contract any of its modes, with any operand.
#include <cstring>
#include <memory>

#include "engine.h"
#include "kernels.cuh"

namespace gs {
namespace {

struct DecodeParams {
    int nz;                    // modes of Z
    int shift[2 * kMaxOrder];  // bit position of every Z mode inside the output key
    int bits[2 * kMaxOrder];
};

// key = x_f << Y_nfbits | y_f  ->  one index per Z mode (SoA)
__global__ void k_decode_keys(DecodeParams p, const uint64_t *__restrict__ keys, uint64_t n,
                              uint64_t *__restrict__ idx) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i];
        for (int m = 0; m < p.nz; ++m) {
            const int s = p.shift[m], b = p.bits[m];
            const uint64_t v = s >= 64 ? 0ull : (k >> s);
            idx[(uint64_t)m * n + i] = b >= 64 ? v : (v & ((1ull << b) - 1));
        }
    }
}

// Output chunks collected into one growing device buffer.
struct Collect {
    Arena *A = nullptr;
    cudaStream_t s = nullptr;
    DBuf<uint64_t> k;
    DBuf<float> v;
    uint64_t n = 0, cap = 0;
    Error err{GSPARC_OK, ""};
};

int collect_chunk(void *user, const uint64_t *keys, const float *vals, uint64_t n, uint64_t first, int) {
    Collect *c = static_cast<Collect *>(user);
    try {
        const uint64_t need = first + n;
        if (need > c->cap) {
            const uint64_t cap = std::max<uint64_t>(std::max<uint64_t>(need, 2 * c->cap), 1ull << 20);
            DBuf<uint64_t> k2(*c->A, cap, c->s);
            DBuf<float> v2(*c->A, cap, c->s);
            if (c->n) {
                GS_CUDA(cudaMemcpyAsync(k2.get(), c->k.get(), 8 * c->n, cudaMemcpyDeviceToDevice, c->s));
                GS_CUDA(cudaMemcpyAsync(v2.get(), c->v.get(), 4 * c->n, cudaMemcpyDeviceToDevice, c->s));
            }
            c->k = std::move(k2);
            c->v = std::move(v2);
            c->cap = cap;
        }
        // ordered on the engine's stream before the kernels of later chunks,
        // which are enqueued after this callback returns
        GS_CUDA(cudaMemcpyAsync(c->k.get() + first, keys, 8 * n, cudaMemcpyDeviceToDevice, c->s));
        GS_CUDA(cudaMemcpyAsync(c->v.get() + first, vals, 4 * n, cudaMemcpyDeviceToDevice, c->s));
        c->n = std::max(c->n, need);
        return 0;
    } catch (const Error &e) {
        c->err = e;
        return 1;
    }
}

}  // namespace

void sptc_resident(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y, int nc, const int *cx,
                   const int *cy, int accum, gsparc_tensor **out, gsparc_stats *stats, cudaStream_t s) {
    GS_REQUIRE(X && Y && out && cx && cy, GSPARC_EINVAL, "null argument");
    *out = nullptr;
    const Layout LX = make_layout(X->order, X->dims, nc, cx);
    const Layout LY = make_layout(Y->order, Y->dims, nc, cy);
    GS_REQUIRE(X->order - nc + Y->order - nc <= kMaxOrder, GSPARC_EUNSUPPORTED, "result has more than 32 modes");
    Collect c;
    c.A = &ctx->arena;
    c.s = s;
    gsparc_job job;
    std::memset(&job, 0, sizeof(job));
    job.x = X;
    job.y = Y;
    job.ncmodes = nc;
    job.cx = cx;
    job.cy = cy;
    job.accum = accum;
    job.sink.kind = GSPARC_SINK_DEVICE;
    job.sink.on_chunk = collect_chunk;
    job.sink.user = &c;
    gsparc_stats bst;
    std::memset(&bst, 0, sizeof(bst));
    try {
        sptc_batch(ctx, &job, 1, 0, &bst, s);
    } catch (const Error &e) {
        if (c.err.st != GSPARC_OK) throw c.err;
        throw Error{job.status != GSPARC_OK ? job.status : e.st, e.msg};
    }
    const uint64_t n = job.stats.nnz;
    GS_REQUIRE(c.n == n, GSPARC_EINTERNAL, "collected output does not match the result size");

    // Z modes: X free modes ascending, then Y free modes ascending
    DecodeParams p{};
    auto z = std::make_unique<gsparc_tensor>();
    int zm = 0;
    for (int m = 0; m < X->order; ++m)
        if (!LX.is_c[m]) {
            p.shift[zm] = LY.nfbits + LX.shift[m];
            p.bits[zm] = LX.bits[m];
            z->dims[zm++] = X->dims[m];
        }
    for (int m = 0; m < Y->order; ++m)
        if (!LY.is_c[m]) {
            p.shift[zm] = LY.shift[m];
            p.bits[zm] = LY.bits[m];
            z->dims[zm++] = Y->dims[m];
        }
    p.nz = zm;
    z->order = zm;
    z->nnz = n;
    z->d_idx = (uint64_t *)ctx->arena.alloc(8 * (size_t)zm * std::max<uint64_t>(n, 1), s);
    try {
        z->d_val = (float *)ctx->arena.alloc(4 * std::max<uint64_t>(n, 1), s);
        if (n) {
            const int grid = (int)std::min<uint64_t>((n + 255) / 256, 148ull * 32);
            k_decode_keys<<<grid, 256, 0, s>>>(p, c.k.get(), n, z->d_idx);
            count_launch();
            GS_CUDA(cudaGetLastError());
            GS_CUDA(cudaMemcpyAsync(z->d_val, c.v.get(), 4 * n, cudaMemcpyDeviceToDevice, s));
        }
        GS_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        ctx->arena.free(z->d_idx, s);
        if (z->d_val) ctx->arena.free(z->d_val, s);
        throw;
    }
    if (stats) {
        gsparc_stats st = job.stats;
        st.chunks = bst.chunks;
        st.kernel_launches = bst.kernel_launches + (n ? 1 : 0);
        st.t_numeric_kernel_ms = bst.t_numeric_kernel_ms;
        st.heavy_windows = bst.heavy_windows;
        st.stream_rows = bst.stream_rows;
        st.kept_bitmap_bytes = bst.kept_bitmap_bytes;
        *stats = st;
    }
    *out = z.release();
}

}  // namespace gs
