// accumulate.cu -- symbolic and numeric accumulation of matched products.
//
// Output row r is one X free index x_f (X is sorted free-major, so its
// nonzeros are contiguous).  Its products are the Y runs matched by the row's
// X nonzeros; every Y run is sorted by column (the Y free index, carried as a
// dense rank among Y's distinct free indices).  Two accumulators:
//
//  * heavy rows (many products): a dense window of kHeavyW columns in shared
//    memory sweeps the row's column range; each run keeps a cursor, so every
//    window takes exactly the run entries that fall inside it.  Sums are
//    compensated: the hardware add returns the old value, from which the exact
//    rounding error of that addition is rebuilt (TwoSum) and accumulated in a
//    second word; each product's own rounding error (fma) goes there too.
//    Touched cells are tracked in a bitmap so exact-zero sums still count
//    (the reference's ESC keeps them, include/gsparc/contraction.cuh:532-537).
//  * light rows (few products): units of consecutive rows are expanded,
//    sorted and compressed on chip (expand-sort-compress; reference ESC:
//    include/gsparc/contraction.cuh:100-141,506-537), with a compensated
//    sequential sum per output key.
//
// Both run twice: a symbolic pass that only counts each row's distinct
// columns, and a numeric pass that writes each row's sorted output at its
// final offset.
#include "kernels.cuh"

namespace gs {

namespace {

__device__ __forceinline__ uint64_t shl(uint64_t v, int s) { return s >= 64 ? 0ull : (v << s); }

__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
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

// ------------------------------------------------------------------ heavy
template <bool NUMERIC>
__global__ void __launch_bounds__(kHeavyThreads) k_heavy(AccArgs a) {
    constexpr int W = kHeavyW;
    constexpr int NW = W / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *hi = reinterpret_cast<float *>(smem_raw);
    float *lo = hi + W;
    uint32_t *bits = NUMERIC ? reinterpret_cast<uint32_t *>(lo + W) : reinterpret_cast<uint32_t *>(smem_raw);
    __shared__ uint32_t s_tmp[33];
    __shared__ uint32_t s_unit;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NWARPS = kHeavyThreads / 32;

    if (NUMERIC) {
        for (int i = tid; i < W; i += kHeavyThreads) {
            hi[i] = -0.0f;
            lo[i] = 0.0f;
        }
    }
    for (int i = tid; i < NW; i += kHeavyThreads) bits[i] = 0;
    __syncthreads();

    for (;;) {
        if (tid == 0) s_unit = atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t u = s_unit;
        if (u >= a.nunits) break;
        const uint32_t row = a.units[u];
        const uint32_t xs = a.row_start[row], xe = a.row_start[row + 1];
        const uint64_t xf_hi = shl(a.row_xf[row], a.y_nfbits);

        uint32_t mymin = 0xffffffffu;
        for (uint32_t i = xs + tid; i < xe; i += kHeavyThreads) {
            uint32_t p = a.pos[i];
            a.cursor[i] = p;
            if (a.cnt[i]) mymin = min(mymin, a.yrank[p]);
        }
        uint32_t B = block_min_u32<kHeavyThreads>(mymin, s_tmp);
        uint64_t out_pos = NUMERIC ? (a.row_off[row] - a.chunk_base) : 0;
        uint32_t row_total = 0;

        while (B != 0xffffffffu) {
            const uint32_t limit = B + (uint32_t)W;  // ranks < 2^31, no wrap
            uint32_t nextmin = 0xffffffffu;
            for (uint32_t i = xs + warp; i < xe; i += NWARPS) {
                uint32_t p = a.cursor[i];
                const uint32_t e = a.pos[i] + a.cnt[i];
                if (p >= e) continue;
                float xv = 0.f;
                if (NUMERIC) xv = a.xval[i];
                for (;;) {
                    const uint32_t idx = p + lane;
                    const uint32_t r = idx < e ? a.yrank[idx] : 0xffffffffu;
                    const bool in = r < limit;
                    if (in) {
                        const uint32_t cell = r - B;
                        const uint32_t m = 1u << (cell & 31);
                        if (NUMERIC) {
                            const float yv = a.yval[idx];
                            const float pr = xv * yv;
                            const float pe = fmaf(xv, yv, -pr);
                            const float old = atomicAdd(&hi[cell], pr);
                            if (__float_as_uint(old) == 0x80000000u) atomicOr(&bits[cell >> 5], m);
                            float s, err;
                            two_sum(old, pr, s, err);
                            atomicAdd(&lo[cell], err + pe);
                        } else {
                            if (!(bits[cell >> 5] & m)) atomicOr(&bits[cell >> 5], m);
                        }
                    }
                    const uint32_t bal = __ballot_sync(0xffffffffu, in);
                    const uint32_t n = __popc(bal);
                    if (n < 32) {
                        if (lane == (int)n) nextmin = min(nextmin, r);
                        p += n;
                        break;
                    }
                    p += 32;
                }
                if (lane == 0) a.cursor[i] = p;
            }
            const uint32_t Bnext = block_min_u32<kHeavyThreads>(nextmin, s_tmp);

            // extract the window in column order
            uint32_t w = 0;
            if (tid < NW) w = bits[tid];
            uint32_t tot;
            const uint32_t ex = block_excl_scan_u32<kHeavyThreads>(__popc(w), s_tmp, &tot);
            if (NUMERIC && w) {
                uint64_t o = out_pos + ex;
                uint32_t ww = w;
                while (ww) {
                    const int b = __ffs(ww) - 1;
                    ww &= ww - 1;
                    const uint32_t cell = (uint32_t)tid * 32 + b;
                    const float v = hi[cell] + lo[cell];
                    if (o < a.out_cap) {
                        a.out_keys[o] = xf_hi | a.cols[B + cell];
                        a.out_vals[o] = v;
                    } else {
                        atomicOr(a.err, 4u);
                    }
                    hi[cell] = -0.0f;
                    lo[cell] = 0.0f;
                    ++o;
                }
            }
            if (tid < NW) bits[tid] = 0;
            out_pos += tot;
            row_total += tot;
            __syncthreads();
            B = Bnext;
        }
        if (!NUMERIC && tid == 0) a.row_nnz[row] = row_total;
        __syncthreads();
    }
}

// ------------------------------------------------------------------ light
template <bool NUMERIC>
__global__ void __launch_bounds__(kLightThreads) k_light(AccArgs a) {
    constexpr int CAP = kLightCap;
    constexpr int PER = CAP / kLightThreads;  // scan elements per thread
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t *key = reinterpret_cast<uint64_t *>(smem_raw);
    uint32_t *pid = reinterpret_cast<uint32_t *>(key + CAP);
    uint32_t *hs = pid + CAP;
    float *pv = reinterpret_cast<float *>(hs + CAP);
    float *pe = pv + CAP;
    __shared__ uint32_t s_tmp[33];
    __shared__ uint32_t s_unit;
    const int tid = threadIdx.x;

    for (;;) {
        if (tid == 0) s_unit = atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t u = s_unit;
        if (u >= a.nunits) break;
        const uint32_t r0 = a.units[2 * u], r1 = a.units[2 * u + 1];
        const uint32_t xs = a.row_start[r0], xe = a.row_start[r1];
        const uint64_t P0 = a.xprefix[xs];
        const uint32_t P = (uint32_t)(a.xprefix[xe] - P0);
        if (P > CAP) {  // planner guarantees otherwise
            if (tid == 0) atomicOr(a.err, 2u);
            __syncthreads();
            continue;
        }
        uint32_t npad = 1;
        while (npad < P) npad <<= 1;

        // expand
        for (uint32_t t = tid; t < npad; t += kLightThreads) {
            if (t < P) {
                const uint64_t target = P0 + t;
                uint32_t lo = xs, hi = xe;  // largest i with xprefix[i] <= target
                while (hi - lo > 1) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (a.xprefix[mid] <= target)
                        lo = mid;
                    else
                        hi = mid;
                }
                const uint32_t i = lo;
                uint32_t rl = r0, rh = r1;  // largest r with row_start[r] <= i
                while (rh - rl > 1) {
                    uint32_t mid = (rl + rh) >> 1;
                    if (a.row_start[mid] <= i)
                        rl = mid;
                    else
                        rh = mid;
                }
                const uint32_t j = a.pos[i] + (uint32_t)(target - a.xprefix[i]);
                key[t] = ((uint64_t)(rl - r0) << 32) | a.yrank[j];
                pid[t] = t;
                if (NUMERIC) {
                    const float xv = a.xval[i], yv = a.yval[j];
                    const float pr = xv * yv;
                    pv[t] = pr;
                    pe[t] = fmaf(xv, yv, -pr);
                }
            } else {
                key[t] = ~0ull;
                pid[t] = t;
            }
        }
        __syncthreads();

        // bitonic sort of (key, pid) over npad entries
        for (uint32_t k = 2; k <= npad; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t t = tid; t < (npad >> 1); t += kLightThreads) {
                    const uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                    const uint32_t l = i | j;
                    const bool up = (i & k) == 0;
                    const uint64_t ki = key[i], kl = key[l];
                    if ((ki > kl) == up) {
                        key[i] = kl;
                        key[l] = ki;
                        const uint32_t pi = pid[i];
                        pid[i] = pid[l];
                        pid[l] = pi;
                    }
                }
                __syncthreads();
            }
        }

        // head flags and their exclusive scan (blocked: PER entries per thread)
        uint32_t local = 0;
        uint32_t hflag[PER];
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const uint32_t t = tid * PER + q;
            const uint32_t h = (t < P) && (t == 0 || key[t] != key[t - 1]);
            hflag[q] = h;
            local += h;
        }
        uint32_t total;
        uint32_t run = block_excl_scan_u32<kLightThreads>(local, s_tmp, &total);
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            hs[tid * PER + q] = run;
            run += hflag[q];
        }
        __syncthreads();

#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const uint32_t t = tid * PER + q;
            if (!hflag[q]) continue;
            const uint64_t k = key[t];
            const uint32_t rloc = (uint32_t)(k >> 32);
            const uint32_t row = r0 + rloc;
            if (!NUMERIC) {
                atomicAdd(&a.row_nnz[row], 1u);
                continue;
            }
            // first sorted entry of this row
            uint32_t lo = 0, hi = t;
            const uint64_t rk = (uint64_t)rloc << 32;
            while (lo < hi) {
                uint32_t mid = (lo + hi) >> 1;
                if (key[mid] < rk)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            const uint32_t rank_in_row = hs[t] - hs[lo];
            float s = 0.f, c = 0.f;
            uint32_t e = t;
            do {
                const uint32_t q2 = pid[e];
                float ns, err;
                two_sum(s, pv[q2], ns, err);
                s = ns;
                c += err + pe[q2];
                ++e;
            } while (e < P && key[e] == k);
            const uint64_t o = a.row_off[row] - a.chunk_base + rank_in_row;
            if (o < a.out_cap) {
                a.out_keys[o] = shl(a.row_xf[row], a.y_nfbits) | a.cols[(uint32_t)k];
                a.out_vals[o] = s + c;
            } else {
                atomicOr(a.err, 4u);
            }
        }
        __syncthreads();
    }
}

size_t heavy_smem(bool numeric) {
    return numeric ? (size_t)kHeavyW * 8 + kHeavyW / 8 : (size_t)kHeavyW / 8;
}
size_t light_smem(bool numeric) {
    return (size_t)kLightCap * (8 + 4 + 4) + (numeric ? (size_t)kLightCap * 8 : 0);
}

}  // namespace

int heavy_blocks_per_sm() { return 3; }
int light_blocks_per_sm() { return 2; }

void launch_heavy(const AccArgs &a, bool numeric, int grid, cudaStream_t s) {
    if (a.nunits == 0) return;
    size_t sm = heavy_smem(numeric);
    if (numeric) {
        GS_CUDA(cudaFuncSetAttribute(k_heavy<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_heavy<true><<<grid, kHeavyThreads, sm, s>>>(a);
        count_launch();
    } else {
        GS_CUDA(cudaFuncSetAttribute(k_heavy<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_heavy<false><<<grid, kHeavyThreads, sm, s>>>(a);
        count_launch();
    }
    GS_CUDA(cudaGetLastError());
}

void launch_light(const AccArgs &a, bool numeric, int grid, cudaStream_t s) {
    if (a.nunits == 0) return;
    size_t sm = light_smem(numeric);
    if (numeric) {
        GS_CUDA(cudaFuncSetAttribute(k_light<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_light<true><<<grid, kLightThreads, sm, s>>>(a);
        count_launch();
    } else {
        GS_CUDA(cudaFuncSetAttribute(k_light<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_light<false><<<grid, kLightThreads, sm, s>>>(a);
        count_launch();
    }
    GS_CUDA(cudaGetLastError());
}

}  // namespace gs
