// wide.cu -- operands whose keys need more than 64 bits.
//
// The reference switches to 128-bit keys when an operand's mode bits add up
// to more than 64 (ConvertTensor_extra, include/gsparc/tensor_manager.tpp:
// 301-406; IndexMatch_extra, include/gsparc/indexMatch.cuh:120-229;
// contraction_extra.cuh), with the same layouts, the match on the whole
// (up to 128-bit) contract key and 64-bit output keys (x_f << Y_nfbits | y_f).
//
// Here such a contraction is relabeled onto keys that fit 64 bits and then
// runs through the ordinary engine:
//
//   X'(F, C) = X,  Y'(C, G) = Y,
//
// F = rank of X's free part among X's distinct free parts, G = the same for
// Y, C = rank of the contract part among the distinct contract parts of X and
// Y together.  Ranks preserve order (F and G ascending in the original free
// values), so X' rows and Y' columns come in the original output order, and
// equal contract parts get equal ranks, so X' and Y' match exactly where X and
// Y do.  Every operand has fewer than 2^31 nonzeros, so F, G < 2^31 and
// C < 2^32 and the relabeled keys are at most 63 bits wide.  Output keys
// F << bits(G) | G are mapped back to x_f << Y_nfbits | y_f on every output
// chunk before it is delivered (order is unchanged by the map).
#include <cub/cub.cuh>

#include "engine.h"
#include "kernels.cuh"
#include "wide.h"

namespace gs {

namespace {

constexpr int kT = 256;

inline int grid_of(uint64_t n) {
    uint64_t g = (n + kT - 1) / kT;
    if (g < 1) g = 1;
    if (g > 148ull * 32) g = 148ull * 32;
    return (int)g;
}

struct PartParams {
    int order;
    int shift[kMaxOrder];
    int is_c[kMaxOrder];
    uint64_t dims[kMaxOrder];
};

// Free part (< 2^64) and contract part (hi:lo, < 2^128) of every nonzero, in
// the reference's layouts (free / contract modes concatenated, first mode in
// the highest bits).  Out-of-range indices set *err.
__global__ void k_wide_parts(PartParams p, uint64_t n, const uint64_t *__restrict__ idx,
                             uint64_t *__restrict__ f, uint64_t *__restrict__ chi, uint64_t *__restrict__ clo,
                             unsigned int *__restrict__ err) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        uint64_t fv = 0, hi = 0, lo = 0;
        bool bad = false;
        for (int m = 0; m < p.order; ++m) {
            const uint64_t v = idx[(uint64_t)m * n + k];
            bad |= v >= p.dims[m];
            const int s = p.shift[m];
            if (p.is_c[m]) {
                if (s >= 64) {
                    hi |= v << (s - 64);
                } else {
                    lo |= v << s;
                    if (s > 0) hi |= v >> (64 - s);
                }
            } else {
                fv |= s >= 64 ? 0ull : (v << s);
            }
        }
        if (bad) atomicOr(err, 1u);
        f[k] = fv;
        chi[k] = hi;
        clo[k] = lo;
    }
}

__global__ void k_iota(uint32_t *__restrict__ p, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = (uint32_t)i;
}

__global__ void k_gather_u64(const uint64_t *__restrict__ src, const uint32_t *__restrict__ perm, uint64_t n,
                             uint64_t *__restrict__ dst) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[perm[i]];
}

// head[i] = 1 where sorted value i differs from value i-1 (two words compared)
__global__ void k_heads(const uint64_t *__restrict__ a, const uint64_t *__restrict__ b, uint64_t n,
                        uint32_t *__restrict__ head) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        head[i] = (i == 0 || a[i] != a[i - 1] || (b && b[i] != b[i - 1])) ? 1u : 0u;
}

// rank[perm[i]] = scan[i] - 1 (scan: inclusive prefix of the head flags)
__global__ void k_scatter_rank(const uint32_t *__restrict__ scan, const uint32_t *__restrict__ perm, uint64_t n,
                               uint32_t *__restrict__ rank) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        rank[perm[i]] = scan[i] - 1u;
}

__global__ void k_pack2(const uint32_t *__restrict__ r0, const uint32_t *__restrict__ r1, uint64_t n,
                        uint64_t *__restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        out[i] = r0[i];
        out[n + i] = r1[i];
    }
}

__global__ void k_wide_remap(uint64_t *__restrict__ keys, uint64_t n, const uint64_t *__restrict__ xf,
                             const uint64_t *__restrict__ yf, int yb2, int nfbits_y) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t ymask = (1ull << yb2) - 1;  // yb2 <= 31
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i];
        const uint64_t x = xf[k >> yb2], y = yf[k & ymask];
        keys[i] = (nfbits_y >= 64 ? 0ull : (x << nfbits_y)) | y;
    }
}

// (x_f << nfbits_y) | y_f as 128 bits: x_f and y_f each fit 64 bits
__global__ void k_wide_remap128(const uint64_t *__restrict__ keys, uint64_t *__restrict__ out2, uint64_t n,
                                const uint64_t *__restrict__ xf, const uint64_t *__restrict__ yf, int yb2,
                                int nfbits_y) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t ymask = (1ull << yb2) - 1;  // yb2 <= 31
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i];
        const uint64_t x = xf[k >> yb2], y = yf[k & ymask];
        uint64_t lo, hi;
        if (nfbits_y == 0) {
            lo = x;
            hi = 0;
        } else if (nfbits_y >= 64) {
            lo = y;
            hi = x;
        } else {
            lo = (x << nfbits_y) | y;
            hi = x >> (64 - nfbits_y);
        }
        out2[2 * i] = lo;
        out2[2 * i + 1] = hi;
    }
}

template <class T>
void sort_pairs_u32(Arena &A, uint64_t n, const T *k_in, T *k_out, const uint32_t *v_in, uint32_t *v_out,
                    int bits, cudaStream_t s) {
    size_t tmp = 0;
    GS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k_in, k_out, v_in, v_out, (int)n, 0, bits, s));
    DBuf<uint8_t> t(A, tmp, s);
    GS_CUDA(cub::DeviceRadixSort::SortPairs(t.get(), tmp, k_in, k_out, v_in, v_out, (int)n, 0, bits, s));
}

// Dense ranks of n values given as (hi, lo) words (hi may be null: 64-bit
// values), hi_bits / lo_bits significant bits.  rank[i] = number of distinct
// values smaller than value i; for 64-bit values the distinct values,
// ascending, go to table_lo when it is non-null.  Returns the number of
// distinct values.
uint64_t dense_rank(Arena &A, uint64_t n, const uint64_t *hi, const uint64_t *lo, int hi_bits, int lo_bits,
                    uint32_t *rank, DBuf<uint64_t> *table_lo, cudaStream_t s) {
    if (n == 0) return 0;
    DBuf<uint32_t> p0(A, n, s), p1(A, n, s);
    DBuf<uint64_t> k0(A, n, s), k1(A, n, s);
    k_iota<<<grid_of(n), kT, 0, s>>>(p0, n);
    count_launch();
    // LSD over the two words: stable sort by lo, then (stable) by hi
    sort_pairs_u32<uint64_t>(A, n, lo, k0.get(), p0.get(), p1.get(), std::max(lo_bits, 1), s);
    const uint32_t *perm = p1.get();
    DBuf<uint64_t> shi, slo;
    if (hi && hi_bits > 0) {
        k_gather_u64<<<grid_of(n), kT, 0, s>>>(hi, p1, n, k1);
        count_launch();
        sort_pairs_u32<uint64_t>(A, n, k1.get(), k0.get(), p1.get(), p0.get(), hi_bits, s);
        perm = p0.get();
        shi.reset(A, n, s);
        slo.reset(A, n, s);
        k_gather_u64<<<grid_of(n), kT, 0, s>>>(hi, perm, n, shi);
        k_gather_u64<<<grid_of(n), kT, 0, s>>>(lo, perm, n, slo);
        count_launch(2);
    }
    const uint64_t *sa = shi.get() ? shi.get() : k0.get();  // sorted major word
    const uint64_t *sb = shi.get() ? slo.get() : nullptr;   // sorted minor word (128-bit values)
    DBuf<uint32_t> head(A, n, s), scan(A, n, s);
    k_heads<<<grid_of(n), kT, 0, s>>>(sa, sb, n, head);
    count_launch();
    {
        size_t tmp = 0;
        GS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, head.get(), scan.get(), (int)n, s));
        DBuf<uint8_t> t(A, tmp, s);
        GS_CUDA(cub::DeviceScan::InclusiveSum(t.get(), tmp, head.get(), scan.get(), (int)n, s));
    }
    k_scatter_rank<<<grid_of(n), kT, 0, s>>>(scan, perm, n, rank);
    count_launch();
    GS_CUDA(cudaGetLastError());
    uint32_t last = 0;
    GS_CUDA(cudaMemcpyAsync(&last, scan.get() + n - 1, 4, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    const uint64_t nu = last;
    if (table_lo) {
        // distinct values of a 64-bit key: the heads of the sorted keys
        table_lo->reset(A, nu, s);
        DBuf<uint64_t> cnt(A, 1, s);
        size_t tmp = 0;
        GS_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, sa, head.get(), table_lo->get(), cnt.get(), (int)n, s));
        DBuf<uint8_t> t(A, tmp, s);
        GS_CUDA(cub::DeviceSelect::Flagged(t.get(), tmp, sa, head.get(), table_lo->get(), cnt.get(), (int)n, s));
    }
    return nu;
}

PartParams part_params(const Layout &L, const uint64_t *dims) {
    PartParams p{};
    p.order = L.order;
    for (int m = 0; m < L.order; ++m) {
        p.shift[m] = L.shift[m];
        p.is_c[m] = L.is_c[m];
        p.dims[m] = dims[m];
    }
    return p;
}

}  // namespace

std::unique_ptr<WideMap> make_wide(Arena &A, const gsparc_tensor *X, const Layout &LX, const gsparc_tensor *Y,
                                   const Layout &LY, cudaStream_t s) {
    GS_REQUIRE(LX.ncbits <= 128 && LY.ncbits <= 128, GSPARC_EUNSUPPORTED, "contract keys wider than 128 bits");
    GS_REQUIRE(LX.nfbits <= 64 && LY.nfbits <= 64, GSPARC_EUNSUPPORTED, "free keys wider than 64 bits");
    auto w = std::make_unique<WideMap>();
    const uint64_t nx = X->nnz, ny = Y->nnz, nc = nx + ny;
    w->nfbits_y = LY.nfbits;
    DBuf<unsigned int> err(A, 1, s);
    GS_CUDA(cudaMemsetAsync(err.get(), 0, 4, s));
    DBuf<uint64_t> fx(A, nx, s), gy(A, ny, s), chi(A, nc, s), clo(A, nc, s);
    {
        if (nx) {
            k_wide_parts<<<grid_of(nx), kT, 0, s>>>(part_params(LX, X->dims), nx, X->d_idx, fx, chi, clo, err);
            count_launch();
        }
        if (ny) {
            k_wide_parts<<<grid_of(ny), kT, 0, s>>>(part_params(LY, Y->dims), ny, Y->d_idx, gy, chi.get() + nx,
                                                     clo.get() + nx, err);
            count_launch();
        }
        GS_CUDA(cudaGetLastError());
    }
    DBuf<uint32_t> rf(A, nx, s), rg(A, ny, s), rc(A, nc, s);
    const uint64_t nF = dense_rank(A, nx, nullptr, fx, 0, LX.nfbits, rf, &w->xf, s);
    const uint64_t nG = dense_rank(A, ny, nullptr, gy, 0, LY.nfbits, rg, &w->yf, s);
    const int cb = LX.ncbits;
    const uint64_t nC = dense_rank(A, nc, cb > 64 ? chi.get() : nullptr, clo, cb > 64 ? cb - 64 : 0,
                                   std::min(cb, 64), rc, nullptr, s);
    unsigned int herr = 0;
    GS_CUDA(cudaMemcpyAsync(&herr, err.get(), 4, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    GS_REQUIRE(!herr, GSPARC_EINVAL, "an index is not smaller than its mode size");

    w->x2idx.reset(A, 2 * std::max<uint64_t>(nx, 1), s);
    w->y2idx.reset(A, 2 * std::max<uint64_t>(ny, 1), s);
    if (nx) {
        k_pack2<<<grid_of(nx), kT, 0, s>>>(rf, rc, nx, w->x2idx);
        count_launch();
    }
    if (ny) {
        k_pack2<<<grid_of(ny), kT, 0, s>>>(rc.get() + nx, rg, ny, w->y2idx);
        count_launch();
    }
    GS_CUDA(cudaGetLastError());
    w->x2.order = 2;
    w->x2.nnz = nx;
    w->x2.dims[0] = std::max<uint64_t>(nF, 1);
    w->x2.dims[1] = std::max<uint64_t>(nC, 1);
    w->x2.d_idx = w->x2idx.get();
    w->x2.d_val = X->d_val;
    w->x2.owned = false;
    w->y2.order = 2;
    w->y2.nnz = ny;
    w->y2.dims[0] = std::max<uint64_t>(nC, 1);
    w->y2.dims[1] = std::max<uint64_t>(nG, 1);
    w->y2.d_idx = w->y2idx.get();
    w->y2.d_val = Y->d_val;
    w->y2.owned = false;
    w->yb2 = mode_bits(w->y2.dims[1]);
    return w;
}

void wide_remap_keys128(const WideMap &w, const uint64_t *keys, uint64_t *out2, uint64_t n, cudaStream_t s) {
    if (n == 0) return;
    k_wide_remap128<<<grid_of(n), kT, 0, s>>>(keys, out2, n, w.xf, w.yf, w.yb2, w.nfbits_y);
    count_launch();
    GS_CUDA(cudaGetLastError());
}

void wide_remap_keys(const WideMap &w, uint64_t *keys, uint64_t n, cudaStream_t s) {
    if (n == 0) return;
    k_wide_remap<<<grid_of(n), kT, 0, s>>>(keys, n, w.xf, w.yf, w.yb2, w.nfbits_y);
    count_launch();
    GS_CUDA(cudaGetLastError());
}

}  // namespace gs
