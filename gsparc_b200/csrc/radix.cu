// radix.cu -- this library's own stable LSD radix sort of (u64 key, f32 value)
// pairs, beside CUB's onesweep sort (the reference sorts with CUB too:
// include/gsparc/sort.cuh:90-108).  Selected per context by
// gsparc_ctx_set_sort; CUB stays the default.
//
// Onesweep form: 8 bits per pass over [0, nbits), the last pass masked to the
// bits below nbits.
//   1. k_os_hist reads every key once and counts the digits of all passes
//      (shared-memory counts per block, lanes of one digit aggregated by
//      __match_any_sync, then one global add per bin);
//   2. one k_os_pass per pass.  A CTA takes the next tile of kTile entries
//      from a counter, so every tile before it belongs to a CTA that is
//      already running.  It ranks its entries among those of the same digit
//      (a warp holds kPer entries per lane striped: entry 32*r + lane of its
//      stretch in round r, so rounds and lanes follow the input order;
//      __match_any_sync groups the lanes of one digit, a per-warp counter per
//      digit carries the rank across rounds, the warps' counts are then
//      prefixed), publishes its per-digit counts, and finds how many entries
//      of each digit the tiles before it hold by a decoupled look-back over
//      their published words (a count flagged as the tile's own or as the
//      inclusive prefix of every tile up to it; the look-back stops at the
//      first prefix).  The global start of each digit is an exclusive scan of
//      the pass's histogram.  The tile's entries are then placed in shared
//      memory in digit order and written out from there, so the entries of
//      one digit leave as consecutive addresses of consecutive threads.
// Equal digits keep their input order in every pass, so the sort is stable.
//
// The look-back waits only on tiles whose CTAs are resident and publish their
// counts before they wait on anything, so every wait ends; it is still
// bounded (kSpinLimit polls), and a wait that runs out, or a position outside
// the output, sets bit 8 of the caller's error word instead of writing.
#include <utility>

#include "kernels.cuh"

namespace gs {

namespace {

constexpr int kOsThreads = 256;
constexpr int kOsWarps = kOsThreads / 32;
constexpr int kPer = 8;                     // entries per lane
constexpr int kTile = kOsThreads * kPer;    // 2048 entries per tile
constexpr int kMaxPass = 8;                 // 64 bits
constexpr uint32_t FULL = 0xffffffffu;
constexpr uint32_t kAgg = 1u << 30;         // the word holds this tile's count
constexpr uint32_t kPrefix = 2u << 30;      // the word holds the count of every tile up to this one
constexpr uint32_t kCountMask = kAgg - 1u;  // counts stay below 2^30
constexpr uint32_t kSpinLimit = 1u << 20;   // look-back polls of one word before giving up
constexpr unsigned int kSortErr = 8u;

__device__ __forceinline__ uint32_t digit_of(uint64_t k, int shift, uint32_t dmask) {
    return (uint32_t)(k >> shift) & dmask;
}

__host__ __device__ __forceinline__ uint32_t pass_mask(int nbits, int shift) {
    return nbits - shift >= 8 ? 255u : (1u << (nbits - shift)) - 1u;
}

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Exclusive scan over the block's 256 threads (one value each); s_w holds
// kOsWarps words.
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t x, uint32_t *s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    uint32_t before = 0;
#pragma unroll
    for (int w = 0; w < kOsWarps; ++w)
        if (w < warp) before += s_w[w];
    __syncthreads();  // s_w may be reused by the caller
    return before + inc - x;
}

// Digit counts of every pass: gh[p * 256 + d].
__global__ void __launch_bounds__(kOsThreads) k_os_hist(const uint64_t *__restrict__ keys, uint64_t n, int nbits,
                                                        int npass, uint32_t *__restrict__ gh) {
    __shared__ uint32_t h[kMaxPass * 256];
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t lt = (1u << lane) - 1u;
    for (int j = tid; j < npass * 256; j += kOsThreads) h[j] = 0;
    __syncthreads();
    for (uint64_t i0 = (uint64_t)blockIdx.x * kOsThreads; i0 < n; i0 += (uint64_t)gridDim.x * kOsThreads) {
        const uint64_t i = i0 + tid;
        const bool ok = i < n;
        const uint64_t k = ok ? keys[i] : 0ull;
        for (int p = 0; p < npass; ++p) {
            const int shift = 8 * p;
            const uint32_t d = ok ? digit_of(k, shift, pass_mask(nbits, shift)) : 256u + (uint32_t)lane;
            const uint32_t peers = __match_any_sync(FULL, d);
            if (ok && (peers & lt) == 0) atomicAdd(&h[p * 256 + d], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    for (int j = tid; j < npass * 256; j += kOsThreads)
        if (h[j]) atomicAdd(&gh[j], h[j]);
}

// One pass: see the file comment.  status holds ntiles * 256 words and then
// the tile counter, all zero at launch.
__global__ void __launch_bounds__(kOsThreads, 4)
    k_os_pass(const uint64_t *__restrict__ keys_in, const float *__restrict__ vals_in, uint64_t n, int shift,
              uint32_t dmask, uint32_t ntiles, const uint32_t *__restrict__ gh, uint32_t *__restrict__ status,
              unsigned int *__restrict__ err, uint64_t *__restrict__ keys_out, float *__restrict__ vals_out) {
    extern __shared__ __align__(16) unsigned char os_smem[];
    uint64_t *s_k = reinterpret_cast<uint64_t *>(os_smem);                   // kTile keys in digit order
    float *s_v = reinterpret_cast<float *>(s_k + kTile);                      // kTile values
    uint32_t(*wcount)[256] = reinterpret_cast<uint32_t(*)[256]>(s_v + kTile);  // per warp and digit
    uint32_t *s_loc = &wcount[kOsWarps][0];                                   // tile-local digit starts
    uint32_t *s_base = s_loc + 256;                                           // global start of the tile's digits
    uint32_t *s_w = s_base + 256;                                             // scan scratch (kOsWarps words)
    uint32_t *s_tile = s_w + kOsWarps;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) *s_tile = atomicAdd(status + (uint64_t)ntiles * 256, 1u);
#pragma unroll
    for (int w = 0; w < kOsWarps; ++w) wcount[w][tid] = 0;
    __syncthreads();
    const uint32_t tile = *s_tile;
    const uint64_t first = (uint64_t)tile * kTile + (uint64_t)warp * (32 * kPer);

    uint64_t k[kPer];
    float v[kPer];
    uint32_t rank[kPer];
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
        const uint64_t i = first + 32 * r + lane;
        k[r] = i < n ? keys_in[i] : 0ull;
        v[r] = i < n ? vals_in[i] : 0.f;
    }
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
        const bool ok = first + 32 * r + lane < n;
        // lanes past the end get a digit of their own, so they join no group
        const uint32_t d = ok ? digit_of(k[r], shift, dmask) : 256u + (uint32_t)lane;
        const uint32_t peers = __match_any_sync(FULL, d);
        const uint32_t pre = ok ? wcount[warp][d] : 0u;
        __syncwarp();
        rank[r] = pre + __popc(peers & lt);
        if (ok && (peers & lt) == 0) wcount[warp][d] = pre + __popc(peers);  // the group's first lane
        __syncwarp();
    }
    __syncthreads();

    // digit tid: the counts of the warps before each warp, and the tile's count
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < kOsWarps; ++w) {
        const uint32_t t = wcount[w][tid];
        wcount[w][tid] = cnt;
        cnt += t;
    }
    uint32_t *my = status + (uint64_t)tile * 256 + tid;
    st_relaxed(my, (tile == 0 ? kPrefix : kAgg) | cnt);

    const uint32_t loc = block_excl_scan256(cnt, s_w);
    const uint32_t gstart = block_excl_scan256(gh[tid], s_w);

    // look-back: entries of digit tid in the tiles before this one
    uint32_t excl = 0;
    if (tile > 0) {
        int64_t t = (int64_t)tile - 1;
        uint32_t polls = 0;
        while (t >= 0) {
            const uint32_t w = ld_relaxed(status + (uint64_t)t * 256 + tid);
            if ((w & ~kCountMask) == 0) {
                if (++polls > kSpinLimit) {
                    atomicOr(err, kSortErr);
                    break;
                }
                __nanosleep(64);
                continue;
            }
            excl += w & kCountMask;
            if (w & kPrefix) break;
            --t;
        }
        st_relaxed(my, kPrefix | ((excl + cnt) & kCountMask));
    }
    s_loc[tid] = loc;
    s_base[tid] = gstart + excl;
    __syncthreads();

    // place the tile's entries in digit order
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
        if (first + 32 * r + lane < n) {
            const uint32_t d = digit_of(k[r], shift, dmask);
            const uint32_t j = s_loc[d] + wcount[warp][d] + rank[r];
            s_k[j] = k[r];
            s_v[j] = v[r];
        }
    }
    __syncthreads();

    // write them out: consecutive threads, consecutive entries of a digit
    const uint64_t t0 = (uint64_t)tile * kTile;
    const uint32_t m = (uint32_t)(n - t0 < (uint64_t)kTile ? n - t0 : (uint64_t)kTile);
    for (uint32_t j = tid; j < m; j += kOsThreads) {
        const uint64_t key = s_k[j];
        const uint32_t d = digit_of(key, shift, dmask);
        const uint64_t pos = (uint64_t)s_base[d] + (j - s_loc[d]);
        if (pos < n) {
            keys_out[pos] = key;
            vals_out[pos] = s_v[j];
        } else {
            atomicOr(err, kSortErr);
        }
    }
}

constexpr size_t kPassSmem = (size_t)kTile * (8 + 4) + 4 * (kOsWarps * 256 + 256 + 256 + kOsWarps + 1);

}  // namespace

void own_sort_pairs(Arena &a, uint64_t n, uint64_t *keys0, uint64_t *keys1, float *vals0, float *vals1, int nbits,
                    int *which, unsigned int *err, cudaStream_t s) {
    *which = 0;
    if (n <= 1 || nbits <= 0) return;
    GS_REQUIRE(n < (1ull << 30), GSPARC_EUNSUPPORTED, "own radix sort of 2^30 entries or more");
    GS_CUDA(cudaFuncSetAttribute(k_os_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPassSmem));
    const int npass = (nbits + 7) / 8;
    const uint32_t ntiles = (uint32_t)((n + kTile - 1) / kTile);
    DBuf<uint32_t> gh(a, (uint64_t)npass * 256, s), status(a, (uint64_t)ntiles * 256 + 1, s);
    GS_CUDA(cudaMemsetAsync(gh.get(), 0, 4ull * npass * 256, s));
    const uint64_t hblocks = std::min<uint64_t>((n + kOsThreads - 1) / kOsThreads, 148ull * 8);
    k_os_hist<<<(unsigned)hblocks, kOsThreads, 0, s>>>(keys0, n, nbits, npass, gh);
    count_launch();
    uint64_t *kin = keys0, *kout = keys1;
    float *vin = vals0, *vout = vals1;
    for (int p = 0; p < npass; ++p) {
        const int shift = 8 * p;
        GS_CUDA(cudaMemsetAsync(status.get(), 0, 4ull * ntiles * 256 + 4, s));
        k_os_pass<<<ntiles, kOsThreads, kPassSmem, s>>>(kin, vin, n, shift, pass_mask(nbits, shift), ntiles,
                                                        gh.get() + 256 * p, status, err, kout, vout);
        count_launch();
        std::swap(kin, kout);
        std::swap(vin, vout);
        *which ^= 1;
    }
    GS_CUDA(cudaGetLastError());
}

}  // namespace gs
