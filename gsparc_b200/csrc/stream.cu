// stream.cu -- output rows fed by a single matched Y run.
//
// When only one X nonzero of an output row matches, the row's products are
// that nonzero times one Y run.  When Y repeats no coordinate (the planner
// checks), the run's free indices are distinct and already ascending: the
// row's output is the run itself, one product per output, in order.  Its symbolic count is the run
// length, and the numeric pass is a copy with a multiply: no sort, no
// accumulator.  The value x*y rounded once is exactly what the compensated
// accumulators return for a single product (0 + p is exact and p + fma error
// rounds back to p), so the result is bit-identical to the general paths.
//
// The products of all such rows of a chunk form one flat index space.  A CTA
// takes a tile of kStreamTile consecutive products and stages, for the rows
// the tile touches (at most kRowBatch at a time), their flat start, first Y
// entry, X value, output slot and key prefix in shared memory, and the staged
// row of every product of the tile (each row marks its first product, a block
// max-scan carries the marks over the rest), so an output costs one shared
// lookup and two coalesced loads of the Y entry (its sorted key, whose low
// Y_nfbits bits are the output column y_f, and its value), with SU outputs'
// loads in flight per thread, and coalesced writes of the output.
#include <cstring>

#include "blockops.cuh"
#include "kernels.cuh"

namespace gs {

namespace {
using namespace dev;

constexpr int ST = 256;
constexpr int kStreamTile = 4096;

__device__ __forceinline__ uint64_t upper_bound_u64(const uint64_t *a, uint64_t lo, uint64_t hi, uint64_t v) {
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (a[mid] <= v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// The first i in [lo, hi) with a[i] > v (hi if none), given a[lo] <= v: steps
// of 1, 2, 4, ... forward from lo, then bisection of the last step, so a
// target k entries past lo costs about 2*log2(k) loads.
__device__ __forceinline__ uint64_t gallop_upper_u64(const uint64_t *a, uint64_t lo, uint64_t hi, uint64_t v) {
    uint64_t b = lo, e = hi, step = 1;
    for (;;) {
        const uint64_t q = b + step;
        if (q >= hi) break;
        if (a[q] > v) {
            e = q;
            break;
        }
        b = q;
        step <<= 1;
    }
    return upper_bound_u64(a, b + 1, e, v);
}

__device__ __forceinline__ uint64_t low_mask(int b) { return b >= 64 ? ~0ull : ((1ull << b) - 1); }

constexpr int kRowBatch = 512;  // rows whose parameters are staged at once
constexpr int SU = 4;           // outputs per thread with loads in flight

__global__ void __launch_bounds__(ST, 6) k_stream(AccArgs a) {
    __shared__ __align__(16) uint16_t s_row[kStreamTile];  // staged row of every output of the tile
    __shared__ uint32_t s_tmp[33];
    __shared__ uint64_t s_pre[kRowBatch + 1];  // flat start of every staged row (+ the end)
    __shared__ uint64_t s_xf[kRowBatch];       // x_f << Y_nfbits
    __shared__ uint64_t s_o0[kRowBatch];       // row's first slot in the chunk buffer
    __shared__ uint64_t s_ym[kRowBatch];       // mask of the y_f bits of a Y key
    __shared__ uint32_t s_j0[kRowBatch];       // row's first Y entry
    __shared__ float s_xv[kRowBatch];          // the row's X value
    __shared__ uint64_t s_k[2];
    const int tid = threadIdx.x;
    const uint64_t ns = a.nunits;
    const uint64_t P0 = a.sprefix[0];
    const uint64_t total = a.sprefix[ns] - P0;

    // a CTA takes a contiguous range of tiles, so each tile finds its rows by a
    // short forward search from the previous tile's last row
    const uint64_t ntiles = (total + kStreamTile - 1) / kStreamTile;
    const uint64_t per = (ntiles + gridDim.x - 1) / gridDim.x;
    const uint64_t tile_e = min(ntiles, (uint64_t)(blockIdx.x + 1) * per);
    uint64_t hint = 0;  // a row whose flat start is at or before this tile's first product
    for (uint64_t tile = (uint64_t)blockIdx.x * per; tile < tile_e; ++tile) {
        const uint64_t t0 = tile * kStreamTile;
        const uint64_t t1 = t0 + kStreamTile < total ? t0 + kStreamTile : total;
        // rows k0..k1 hold the tile's first and last product
        if (tid < 2) s_k[tid] = gallop_upper_u64(a.sprefix, hint, ns + 1, P0 + (tid ? t1 - 1 : t0)) - 1;
        __syncthreads();
        const uint64_t k0 = s_k[0], k1 = s_k[1];
        hint = k1;
        for (uint64_t kb = k0; kb <= k1; kb += kRowBatch) {
            const uint32_t nb = (uint32_t)(k1 - kb + 1 < (uint64_t)kRowBatch ? k1 - kb + 1 : (uint64_t)kRowBatch);
            for (uint32_t i = tid; i <= nb; i += ST) s_pre[i] = a.sprefix[kb + i] - P0;
            for (uint32_t i = tid; i < nb; i += ST) {
                const uint32_t row = a.units[kb + i];
                const uint32_t xi = a.row_xi[row];
                int y_nfbits;
                const uint64_t *cols;
                uint32_t ncols;
                row_job_params(a, row, y_nfbits, cols, ncols);
                s_xf[i] = shl(a.row_xf[row], y_nfbits);
                s_o0[i] = a.row_off[row] - a.chunk_base;
                s_ym[i] = low_mask(y_nfbits);
                s_j0[i] = a.pos[xi];
                s_xv[i] = a.xval[xi];
            }
            __syncthreads();
            const uint64_t b0 = t0 > s_pre[0] ? t0 : s_pre[0];
            const uint64_t b1 = t1 < s_pre[nb] ? t1 : s_pre[nb];
            // Row of every output of [b0, b1) (at most kStreamTile): each
            // staged row marks where it starts inside the range (the row
            // holding b0 marks 0), then a max-scan carries the marks forward.
            constexpr int PER = kStreamTile / ST;  // marks per thread, in 16-byte vectors
            static_assert(PER % 8 == 0, "whole uint4s of u16 marks per thread");
#pragma unroll
            for (int c = 0; c < PER; c += 8)
                *reinterpret_cast<uint4 *>(s_row + PER * tid + c) = make_uint4(0, 0, 0, 0);
            __syncthreads();
            for (uint32_t i = tid; i < nb; i += ST)
                if (s_pre[i + 1] > b0 && s_pre[i] < b1 && s_pre[i + 1] > s_pre[i])
                    s_row[(s_pre[i] > b0 ? s_pre[i] : b0) - b0] = (uint16_t)i;
            __syncthreads();
            {
                uint16_t m[PER];
#pragma unroll
                for (int c = 0; c < PER; c += 8) {
                    const uint4 v = *reinterpret_cast<const uint4 *>(s_row + PER * tid + c);
                    memcpy(m + c, &v, sizeof(v));
                }
                uint32_t run = 0;
#pragma unroll
                for (int k = 0; k < PER; ++k) run = max(run, (uint32_t)m[k]);
                run = block_excl_max_u32<ST>(run, s_tmp);
#pragma unroll
                for (int k = 0; k < PER; ++k) {
                    run = max(run, (uint32_t)m[k]);
                    m[k] = (uint16_t)run;
                }
#pragma unroll
                for (int c = 0; c < PER; c += 8) {
                    uint4 v;
                    memcpy(&v, m + c, sizeof(v));
                    *reinterpret_cast<uint4 *>(s_row + PER * tid + c) = v;
                }
            }
            __syncthreads();
            for (uint64_t tb = b0 + tid; tb < b1; tb += (uint64_t)ST * SU) {
                uint32_t li[SU], pp[SU];
                uint64_t yk[SU];
                float yv[SU];
#pragma unroll
                for (int u = 0; u < SU; ++u) {
                    const uint64_t t = tb + (uint64_t)u * ST;
                    li[u] = 0;
                    pp[u] = 0;
                    if (t < b1) {
                        const uint32_t lo = s_row[t - b0];  // largest i with s_pre[i] <= t
                        li[u] = lo;
                        pp[u] = (uint32_t)(t - s_pre[lo]);
                        const uint32_t j = s_j0[lo] + pp[u];
                        yk[u] = a.ykeys[j];
                        yv[u] = a.yval[j];
                    }
                }
#pragma unroll
                for (int u = 0; u < SU; ++u) {
                    const uint64_t t = tb + (uint64_t)u * ST;
                    if (t < b1) {
                        const uint32_t i = li[u];
                        const uint64_t o = s_o0[i] + pp[u];
                        if (o < a.out_cap) {
                            __stcs(a.out_keys + o, (unsigned long long)(s_xf[i] | (yk[u] & s_ym[i])));
                            __stcs(a.out_vals + o, s_xv[i] * yv[u]);
                        } else {
                            atomicOr(a.err, 4u);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
}

}  // namespace

void launch_stream(const AccArgs &a, int grid, cudaStream_t s) {
    if (a.nunits == 0) return;
    k_stream<<<grid, ST, 0, s>>>(a);
    count_launch();
    GS_CUDA(cudaGetLastError());
}

int stream_blocks_per_sm() {
    int n = 0;
    GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_stream, ST, 0));
    return n > 0 ? n : 1;
}

}  // namespace gs
