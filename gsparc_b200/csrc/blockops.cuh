// blockops.cuh -- small device helpers shared by the accumulation kernels.
#pragma once

#include <cstdint>

namespace gs {
namespace dev {

static __device__ __forceinline__ uint64_t shl(uint64_t v, int s) { return s >= 64 ? 0ull : (v << s); }

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


}  // namespace dev
}  // namespace gs
