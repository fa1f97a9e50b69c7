// blockops.cuh -- small device helpers shared by the accumulation kernels.
#pragma once

#include <cstdint>

namespace gs {
namespace dev {

static __device__ __forceinline__ uint64_t shl(uint64_t v, int s) { return s >= 64 ? 0ull : (v << s); }

// 16-byte global -> shared copy that holds no register while in flight
// (cp.async, cached in L2 only); both addresses 16-byte aligned.
static __device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
static __device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Asks L2 to fetch [gmem, gmem + bytes) ahead of use (address 16-byte
// aligned, bytes a multiple of 16); no data comes back to the SM.
static __device__ __forceinline__ void prefetch_l2(const void *gmem, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(gmem), "r"(bytes) : "memory");
}

static __device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = a + b;
    float bp = s - a;
    e = (a - (s - bp)) + (b - bp);
}

template <int THREADS>
__device__ __forceinline__ uint32_t block_min_u32(uint32_t v, uint32_t *s_tmp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) s_tmp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < THREADS / 32 ? s_tmp[lane] : 0xffffffffu;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w = min(w, __shfl_xor_sync(0xffffffffu, w, o));
        if (lane == 0) s_tmp[32] = w;
    }
    __syncthreads();
    return s_tmp[32];
}

// Exclusive block scan of one value per thread; returns the exclusive prefix,
// *total gets the sum.
template <int THREADS>
__device__ __forceinline__ uint32_t block_excl_scan_u32(uint32_t v, uint32_t *s_tmp, uint32_t *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) s_tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < THREADS / 32 ? s_tmp[lane] : 0;
        uint32_t z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        s_tmp[lane] = z - w;  // exclusive warp offsets
        if (lane == 31) s_tmp[32] = z;
    }
    __syncthreads();
    *total = s_tmp[32];
    return s_tmp[warp] + x - v;
}

// Block sum of v and minimum of m, both returned to every thread, with two
// barriers (s_tmp holds at least 2 * THREADS / 32 words).
template <int THREADS>
__device__ __forceinline__ void block_sum_min_u32(uint32_t v, uint32_t m, uint32_t *s_tmp, uint32_t &sum,
                                                  uint32_t &mn) {
    constexpr int NW = THREADS / 32;
    static_assert(2 * NW <= 32, "sum and min of every warp fit s_tmp");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
        m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    __syncthreads();
    if (lane == 0) {
        s_tmp[warp] = v;
        s_tmp[NW + warp] = m;
    }
    __syncthreads();
    sum = 0;
    mn = 0xffffffffu;
#pragma unroll
    for (int i = 0; i < NW; ++i) {
        sum += s_tmp[i];
        mn = min(mn, s_tmp[NW + i]);
    }
}

// Exclusive block max-scan of one value per thread (0 for thread 0).
template <int THREADS>
__device__ __forceinline__ uint32_t block_excl_max_u32(uint32_t v, uint32_t *s_tmp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    uint32_t ex = __shfl_up_sync(0xffffffffu, x, 1);  // max over the lanes before this one
    if (lane == 0) ex = 0;
    __syncthreads();
    if (lane == 31) s_tmp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t z = lane < THREADS / 32 ? s_tmp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z = max(z, y);
        }
        const uint32_t zex = __shfl_up_sync(0xffffffffu, z, 1);
        s_tmp[lane] = lane ? zex : 0u;  // max over the warps before
    }
    __syncthreads();
    return max(s_tmp[warp], ex);
}


}  // namespace dev
}  // namespace gs
