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
#include "blockops.cuh"
#include "kernels.cuh"

namespace gs {

namespace {
using namespace dev;

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
                int y_nfbits;
                const uint64_t *cols;
                uint32_t ncols;
                row_job_params(a, row, y_nfbits, cols, ncols);
                a.out_keys[o] = shl(a.row_xf[row], y_nfbits) | cols[(uint32_t)k];
                a.out_vals[o] = s + c;
            } else {
                atomicOr(a.err, 4u);
            }
        }
        __syncthreads();
    }
}

size_t light_smem(bool numeric) {
    return (size_t)kLightCap * (8 + 4 + 4) + (numeric ? (size_t)kLightCap * 8 : 0);
}

}  // namespace

int light_blocks_per_sm() { return 2; }

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
