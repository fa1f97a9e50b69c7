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
// takes a tile of kStreamTile consecutive products, stages the product prefix
// of the rows that the tile touches in shared memory, and every thread maps
// its products to (row, offset) there.  Reads of the Y run and writes of the
// output are coalesced; the column table is read in ascending rank order.
#include "blockops.cuh"
#include "kernels.cuh"

namespace gs {

namespace {
using namespace dev;

constexpr int ST = 256;
constexpr int kStreamTile = 2048;

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

__global__ void __launch_bounds__(ST) k_stream(AccArgs a) {
    __shared__ uint64_t s_pre[kStreamTile + 2];
    __shared__ uint64_t s_k[2];
    const int tid = threadIdx.x;
    const uint64_t ns = a.nunits;
    const uint64_t P0 = a.sprefix[0];
    const uint64_t total = a.sprefix[ns] - P0;

    for (uint64_t t0 = (uint64_t)blockIdx.x * kStreamTile; t0 < total; t0 += (uint64_t)gridDim.x * kStreamTile) {
        const uint64_t t1 = t0 + kStreamTile < total ? t0 + kStreamTile : total;
        // rows k0..k1 hold the tile's first and last product
        if (tid < 2) s_k[tid] = upper_bound_u64(a.sprefix, 0, ns + 1, P0 + (tid ? t1 - 1 : t0)) - 1;
        __syncthreads();
        const uint64_t k0 = s_k[0], k1 = s_k[1];
        const uint32_t nk = (uint32_t)(k1 - k0 + 2);  // prefix entries k0 .. k1+1 (<= tile + 1)
        for (uint32_t i = tid; i < nk; i += ST) s_pre[i] = a.sprefix[k0 + i] - P0;
        __syncthreads();
        for (uint64_t t = t0 + tid; t < t1; t += ST) {
            uint32_t lo = 0, hi = nk - 1;  // largest i with s_pre[i] <= t
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_pre[mid] <= t)
                    lo = mid;
                else
                    hi = mid;
            }
            const uint64_t k = k0 + lo;
            const uint32_t p = (uint32_t)(t - s_pre[lo]);
            const uint32_t row = a.units[k];
            const uint32_t xi = a.row_xi[row];
            int y_nfbits;
            const uint64_t *cols;
            uint32_t ncols;
            row_job_params(a, row, y_nfbits, cols, ncols);
            const uint32_t j = a.pos[xi] + p;
            const uint64_t o = a.row_off[row] - a.chunk_base + p;
            if (o < a.out_cap) {
                __stcs(a.out_keys + o, (unsigned long long)(shl(a.row_xf[row], y_nfbits) | cols[a.yrank[j]]));
                __stcs(a.out_vals + o, a.xval[xi] * a.yval[j]);
            } else {
                atomicOr(a.err, 4u);
            }
        }
        __syncthreads();
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
