// verify.cu -- FP64 verification of output chunks on the device.
//
// With a verify budget set on the context (gsparc_ctx_set_verify), every
// output chunk is checked before it is delivered: for the chunk's rows (all of
// them when the contraction has at most `budget` matched products, otherwise a
// seeded sample of rows sized to about that many products) every matched
// product x*y is formed exactly in FP64 (two FP32 factors need 48 of double's
// 53 mantissa bits), added with a double atomic into the output slot whose key
// it belongs to (found by binary search in the row's sorted output keys), and
// each checked output's FP32 value is compared with that FP64 sum:
// max |z - z64| / |z64| (outputs with z64 != 0) and max |z - z64|, per job.
// A product whose key is missing from the row's output counts as a mismatch.
// This is the FP64 oracle on the GPU; the contraction itself never computes in
// FP64.  It is off by default and costs a pass over the sampled products.
#include "kernels.cuh"
#include "verify.h"

namespace gs {

namespace {

constexpr int VT = 256;

__device__ __forceinline__ uint64_t vshl(uint64_t v, int s) { return s >= 64 ? 0ull : (v << s); }

__device__ __forceinline__ uint64_t vmix(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ uint32_t row_job_of(const AccArgs &a, uint32_t r) { return a.row_job ? a.row_job[r] : 0u; }

// rows of the chunk [c0, c1) that are checked: listed with their slot range in acc
__global__ void k_vsel(AccArgs a, uint64_t nrows, uint64_t c0, uint64_t c1, uint64_t thr, uint64_t salt,
                       VerifyEntry *__restrict__ list, unsigned long long *__restrict__ cnt, uint64_t acc_cap,
                       VerifyOut *__restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += stride) {
        const uint64_t o0 = a.row_off[r], o1 = a.row_off[r + 1];
        if (o1 == o0 || o0 < c0 || o0 >= c1) continue;
        if (thr != ~0ull && (vmix(r ^ salt) >> 32) >= thr) continue;
        const uint64_t n = o1 - o0;
        const unsigned long long off = atomicAdd(&cnt[1], (unsigned long long)n);
        if (off + n > acc_cap) {
            atomicAdd(&out[row_job_of(a, (uint32_t)r)].skipped, 1ull);
            continue;
        }
        const unsigned long long e = atomicAdd(&cnt[0], 1ull);
        list[e] = VerifyEntry{(uint32_t)r, 0u, (uint64_t)off};
    }
}

__global__ void k_vzero(AccArgs a, const VerifyEntry *__restrict__ list, const unsigned long long *__restrict__ cnt,
                        double *__restrict__ acc) {
    const uint64_t ne = cnt[0];
    for (uint64_t e = blockIdx.x; e < ne; e += gridDim.x) {
        const VerifyEntry v = list[e];
        const uint64_t n = a.row_off[v.row + 1] - a.row_off[v.row];
        for (uint64_t s = threadIdx.x; s < n; s += blockDim.x) acc[v.off + s] = 0.0;
    }
}

// every product of a listed row, exact in FP64, into its output slot
__global__ void __launch_bounds__(VT) k_vacc(AccArgs a, uint64_t c0, const uint64_t *__restrict__ keys,
                                             const VerifyEntry *__restrict__ list,
                                             const unsigned long long *__restrict__ cnt, double *__restrict__ acc,
                                             VerifyOut *__restrict__ out) {
    const uint64_t ne = cnt[0];
    for (uint64_t e = blockIdx.x; e < ne; e += gridDim.x) {
        const VerifyEntry v = list[e];
        const uint32_t r = v.row;
        int ynf;
        const uint64_t *cols;
        uint32_t ncols;
        row_job_params(a, r, ynf, cols, ncols);
        const uint64_t xf = vshl(a.row_xf[r], ynf);
        const uint32_t xs = a.row_start[r], xe = a.row_start[r + 1];
        const uint64_t P0 = a.xprefix[xs], P = a.xprefix[xe] - P0;
        const uint64_t o0 = a.row_off[r] - c0, n = a.row_off[r + 1] - a.row_off[r];
        const uint64_t *rk = keys + o0;
        unsigned long long miss = 0;
        for (uint64_t t = threadIdx.x; t < P; t += blockDim.x) {
            const uint64_t q = P0 + t;
            uint32_t lo = xs, hi = xe;  // largest i in [xs, xe) with xprefix[i] <= q
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (a.xprefix[mid] <= q)
                    lo = mid;
                else
                    hi = mid;
            }
            const uint32_t j = a.pos[lo] + (uint32_t)(q - a.xprefix[lo]);
            const uint64_t key = xf | cols[a.yrank[j]];
            uint64_t l = 0, h = n;  // first output key >= key
            while (l < h) {
                const uint64_t mid = (l + h) >> 1;
                if (rk[mid] < key)
                    l = mid + 1;
                else
                    h = mid;
            }
            if (l < n && rk[l] == key)
                atomicAdd(&acc[v.off + l], (double)a.xval[lo] * (double)a.yval[j]);
            else
                ++miss;
        }
        const uint32_t job = row_job_of(a, r);
        if (miss) atomicAdd(&out[job].mismatch, miss);
        if (threadIdx.x == 0) {
            atomicAdd(&out[job].products, (unsigned long long)P);
            atomicAdd(&out[job].nnz, (unsigned long long)n);
        }
    }
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// FP32 output vs its FP64 sum
__global__ void __launch_bounds__(VT) k_vcmp(AccArgs a, uint64_t c0, const float *__restrict__ vals,
                                             const VerifyEntry *__restrict__ list,
                                             const unsigned long long *__restrict__ cnt,
                                             const double *__restrict__ acc, VerifyOut *__restrict__ out) {
    const uint64_t ne = cnt[0];
    for (uint64_t e = blockIdx.x; e < ne; e += gridDim.x) {
        const VerifyEntry v = list[e];
        const uint32_t r = v.row;
        const uint64_t o0 = a.row_off[r] - c0, n = a.row_off[r + 1] - a.row_off[r];
        double mrel = 0.0, mabs = 0.0;
        bool nan = false;
        for (uint64_t s = threadIdx.x; s < n; s += blockDim.x) {
            const double z = acc[v.off + s];
            const double f = (double)vals[o0 + s];
            const double d = fabs(f - z);
            nan |= d != d;
            mabs = fmax(mabs, d);
            if (z != 0.0) mrel = fmax(mrel, d / fabs(z));
        }
        mrel = warp_max(mrel);
        mabs = warp_max(mabs);
        const uint32_t job = row_job_of(a, r);
        if ((threadIdx.x & 31) == 0) {
            // non-negative doubles order like their bit patterns
            atomicMax(&out[job].max_rel_bits, (unsigned long long)__double_as_longlong(mrel));
            atomicMax(&out[job].max_abs_bits, (unsigned long long)__double_as_longlong(mabs));
        }
        if (nan) atomicAdd(&out[job].nan_values, 1ull);
    }
}

}  // namespace

uint64_t verify_threshold(uint64_t budget, uint64_t products) {
    if (budget == 0) return 0;
    if (products <= budget) return ~0ull;
    const double f = (double)budget / (double)products;
    return (uint64_t)(f * 4294967296.0);
}

void verify_chunk(const AccArgs &a, VerifyState &vs, uint64_t nrows, uint64_t c0, uint64_t c1,
                  const uint64_t *keys, const float *vals, cudaStream_t s) {
    if (nrows == 0 || c1 <= c0) return;
    GS_CUDA(cudaMemsetAsync(vs.cnt, 0, 2 * sizeof(unsigned long long), s));
    const int g1 = (int)std::min<uint64_t>((nrows + VT - 1) / VT, 148ull * 16);
    k_vsel<<<std::max(g1, 1), VT, 0, s>>>(a, nrows, c0, c1, vs.threshold, vs.salt, vs.list, vs.cnt, vs.acc_cap,
                                          vs.out);
    const int g2 = 148 * 8;
    k_vzero<<<g2, VT, 0, s>>>(a, vs.list, vs.cnt, vs.acc);
    k_vacc<<<g2, VT, 0, s>>>(a, c0, keys, vs.list, vs.cnt, vs.acc, vs.out);
    k_vcmp<<<g2, VT, 0, s>>>(a, c0, vals, vs.list, vs.cnt, vs.acc, vs.out);
    count_launch(4);
    GS_CUDA(cudaGetLastError());
}

void verify_fill_stats(const VerifyOut &o, gsparc_stats &st) {
    double rel, ab;
    static_assert(sizeof(double) == sizeof(unsigned long long), "double size");
    std::memcpy(&rel, &o.max_rel_bits, 8);
    std::memcpy(&ab, &o.max_abs_bits, 8);
    st.verified_nnz += o.nnz;
    st.verified_products += o.products;
    st.verify_mismatch += o.mismatch + o.nan_values;
    st.verify_skipped_rows += o.skipped;
    if (rel > st.max_rel_err || rel != rel) st.max_rel_err = rel;
    if (ab > st.max_abs_err || ab != ab) st.max_abs_err = ab;
}

}  // namespace gs
