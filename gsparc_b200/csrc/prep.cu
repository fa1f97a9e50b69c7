// prep.cu -- linearise, sort, Y run table / column ranks, X match and row table.
#include <cub/cub.cuh>
#include <cstring>

#include "kernels.cuh"

namespace gs {

namespace {

constexpr int kThreads = 256;

inline int grid_for(uint64_t n, int threads = kThreads) {
    uint64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 148ull * 32) g = 148ull * 32;  // grid-stride beyond this
    return (int)g;
}

__device__ __forceinline__ uint64_t shl(uint64_t v, int s) { return s >= 64 ? 0ull : (v << s); }
__device__ __forceinline__ uint64_t shr(uint64_t v, int s) { return s >= 64 ? 0ull : (v >> s); }
__device__ __forceinline__ uint64_t low_mask(int b) { return b >= 64 ? ~0ull : ((1ull << b) - 1); }

// reference: include/gsparc/tensor_manager.tpp:249-268 (X) and :272-293 (Y).
// The contiguous per-mode masks make pdep a shift: mode m lands at shift[m]
// inside its free or contract part.
__global__ void k_linearize(LinParams p, uint64_t nnz, const uint64_t *__restrict__ idx,
                            const float *__restrict__ val, uint64_t *__restrict__ keys,
                            float *__restrict__ val_out, unsigned int *err) {
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        uint64_t f = 0, c = 0;
        bool bad = false;
        for (int m = 0; m < p.order; ++m) {
            uint64_t v = idx[(uint64_t)m * nnz + k];
            bad |= v >= p.dims[m];
            if (p.is_c[m])
                c |= shl(v, p.shift[m]);
            else
                f |= shl(v, p.shift[m]);
        }
        if (bad) atomicOr(err, 1u);
        keys[k] = p.role == 0 ? (shl(f, p.ncbits) | c) : (shl(c, p.nfbits) | f);
        if (val_out) val_out[k] = val[k];
    }
}

// Y: run boundaries of the contract key and the free index of every entry.
__global__ void k_y_split(const uint64_t *__restrict__ ykeys, uint64_t ny, int nfb,
                          uint8_t *__restrict__ run_flag, uint64_t *__restrict__ yf) {
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t fm = low_mask(nfb);
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ny; j += stride) {
        uint64_t k = ykeys[j];
        run_flag[j] = (j == 0) || (shr(k, nfb) != shr(ykeys[j - 1], nfb));
        yf[j] = k & fm;
    }
}

__global__ void k_y_rank(const uint64_t *__restrict__ ykeys, uint64_t ny, int nfb,
                         const uint64_t *__restrict__ cols, uint64_t ncols,
                         uint32_t *__restrict__ rank) {
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t fm = low_mask(nfb);
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ny; j += stride) {
        uint64_t f = ykeys[j] & fm;
        uint64_t lo = 0, hi = ncols;
        while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if (cols[mid] < f)
                lo = mid + 1;
            else
                hi = mid;
        }
        rank[j] = (uint32_t)lo;
    }
}

__global__ void k_run_keys(const uint64_t *__restrict__ ykeys, int nfb,
                           const uint32_t *__restrict__ run_start, uint64_t nruns, uint64_t ny,
                           uint64_t *__restrict__ run_key, uint32_t *__restrict__ run_start_out) {
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= nruns; r += stride) {
        if (r < nruns) run_key[r] = shr(ykeys[run_start[r]], nfb);
        else run_start_out[nruns] = (uint32_t)ny;
    }
}

__device__ __forceinline__ uint64_t lower_bound_u64(const uint64_t *a, uint64_t n, uint64_t v) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// reference: include/gsparc/indexMatch.cuh:67-118.  The run table turns the
// reference's binary search + linear run scan into a search over distinct
// contract keys and an O(1) run length.
__global__ void k_match(const uint64_t *__restrict__ xkeys, uint64_t nx, int ncb,
                        const uint64_t *__restrict__ run_key, const uint32_t *__restrict__ run_start,
                        uint64_t nruns, uint32_t *__restrict__ pos, uint32_t *__restrict__ cnt,
                        uint8_t *__restrict__ row_flag) {
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t cm = low_mask(ncb);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += stride) {
        uint64_t k = xkeys[i];
        uint64_t c = k & cm;
        uint64_t r = lower_bound_u64(run_key, nruns, c);
        uint32_t p = 0, n = 0;
        if (r < nruns && run_key[r] == c) {
            p = run_start[r];
            n = run_start[r + 1] - p;
        }
        pos[i] = p;
        cnt[i] = n;
        row_flag[i] = (i == 0) || (shr(k, ncb) != shr(xkeys[i - 1], ncb));
    }
}

__global__ void k_rows(const uint64_t *__restrict__ xkeys, int ncb, const uint32_t *__restrict__ rs,
                       uint64_t nrows, uint64_t nx, const uint64_t *__restrict__ xprefix,
                       uint32_t *__restrict__ row_start_out, uint64_t *__restrict__ row_xf,
                       uint64_t *__restrict__ row_prod) {
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= nrows; r += stride) {
        if (r == nrows) {
            row_start_out[nrows] = (uint32_t)nx;
            continue;
        }
        uint32_t a = rs[r];
        uint32_t b = (r + 1 < nrows) ? rs[r + 1] : (uint32_t)nx;
        row_start_out[r] = a;
        row_xf[r] = shr(xkeys[a], ncb);
        row_prod[r] = xprefix[b] - xprefix[a];
    }
}

struct CastU64 {
    __host__ __device__ uint64_t operator()(uint32_t v) const { return v; }
};

// u64 outputs for the reference-compatible stage entry point.
__global__ void k_match_compat(const uint64_t *__restrict__ xkeys, uint64_t nx, int ncb,
                               const uint64_t *__restrict__ run_key,
                               const uint32_t *__restrict__ run_start, uint64_t nruns,
                               uint64_t *__restrict__ pos, uint64_t *__restrict__ cnt) {
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t cm = low_mask(ncb);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += stride) {
        uint64_t c = xkeys[i] & cm;
        uint64_t r = lower_bound_u64(run_key, nruns, c);
        uint64_t p = 0, n = 0;
        if (r < nruns && run_key[r] == c) {
            p = run_start[r];
            n = run_start[r + 1] - p;
        }
        pos[i] = p;
        cnt[i] = n;
    }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Verification digest (device-side check of outputs too large for the host).
__global__ void k_digest(const uint64_t *__restrict__ keys, const float *__restrict__ vals, uint64_t n,
                         unsigned long long *acc_u, double *acc_d) {
    uint64_t h = 0, bad = 0;
    double sv = 0.0, sa = 0.0;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint64_t k = keys[i];
        h += splitmix64(k);
        if (i + 1 < n && k >= keys[i + 1]) ++bad;
        double v = vals[i];
        sv += v;
        sa += fabs(v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        h += __shfl_xor_sync(0xffffffffu, h, o);
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
        sv += __shfl_xor_sync(0xffffffffu, sv, o);
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc_u[0], (unsigned long long)h);
        atomicAdd(&acc_u[1], (unsigned long long)bad);
        atomicAdd(&acc_d[0], sv);
        atomicAdd(&acc_d[1], sa);
    }
}

}  // namespace

void digest_chunk(const uint64_t *keys, const float *vals, uint64_t n, gsparc_digest *out, cudaStream_t s) {
    std::memset(out, 0, sizeof(*out));
    out->n = n;
    if (n == 0) return;
    unsigned long long *acc = nullptr;
    GS_CUDA(cudaMallocAsync((void **)&acc, 64, s));
    GS_CUDA(cudaMemsetAsync(acc, 0, 64, s));
    k_digest<<<grid_for(n), kThreads, 0, s>>>(keys, vals, n, acc, reinterpret_cast<double *>(acc + 2));
    count_launch();
    GS_CUDA(cudaGetLastError());
    unsigned long long h[4];
    GS_CUDA(cudaMemcpyAsync(h, acc, 32, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaMemcpyAsync(&out->first_key, keys, 8, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaMemcpyAsync(&out->last_key, keys + n - 1, 8, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaFreeAsync(acc, s));
    GS_CUDA(cudaStreamSynchronize(s));
    out->key_hash = h[0];
    out->unsorted = h[1];
    std::memcpy(&out->val_sum, &h[2], 8);
    std::memcpy(&out->val_abs_sum, &h[3], 8);
}

LinParams make_lin_params(const Layout &L, const uint64_t *dims, int role) {
    LinParams p{};
    p.order = L.order;
    p.role = role;
    p.ncbits = L.ncbits;
    p.nfbits = L.nfbits;
    for (int m = 0; m < L.order; ++m) {
        p.shift[m] = L.shift[m];
        p.is_c[m] = L.is_c[m];
        p.dims[m] = dims[m];
    }
    return p;
}

void launch_linearize(const LinParams &p, uint64_t nnz, const uint64_t *idx, const float *val,
                      uint64_t *keys, float *val_out, unsigned int *err, cudaStream_t s) {
    if (nnz == 0) return;
    k_linearize<<<grid_for(nnz), kThreads, 0, s>>>(p, nnz, idx, val, keys, val_out, err);
    count_launch();
    GS_CUDA(cudaGetLastError());
}

void sort_pairs(Arena &a, uint64_t n, uint64_t *keys0, uint64_t *keys1, float *vals0, float *vals1,
                int nbits, int *which, cudaStream_t s) {
    *which = 0;
    if (n <= 1 || nbits <= 0) return;
    GS_REQUIRE(n < (1ull << 31), GSPARC_EUNSUPPORTED, "sort of more than 2^31 entries");
    cub::DoubleBuffer<uint64_t> kb(keys0, keys1);
    cub::DoubleBuffer<float> vb(vals0, vals1);
    size_t tmp = 0;
    GS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kb, vb, (int)n, 0, nbits, s));
    DBuf<uint8_t> t(a, tmp, s);
    GS_CUDA(cub::DeviceRadixSort::SortPairs(t.get(), tmp, kb, vb, (int)n, 0, nbits, s));
    *which = kb.selector;
}

void sort_keys(Arena &a, uint64_t n, uint64_t *keys0, uint64_t *keys1, int nbits, int *which,
               cudaStream_t s) {
    *which = 0;
    if (n <= 1 || nbits <= 0) return;
    GS_REQUIRE(n < (1ull << 31), GSPARC_EUNSUPPORTED, "sort of more than 2^31 entries");
    cub::DoubleBuffer<uint64_t> kb(keys0, keys1);
    size_t tmp = 0;
    GS_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, kb, (int)n, 0, nbits, s));
    DBuf<uint8_t> t(a, tmp, s);
    GS_CUDA(cub::DeviceRadixSort::SortKeys(t.get(), tmp, kb, (int)n, 0, nbits, s));
    *which = kb.selector;
}

static uint64_t read_u64(const uint64_t *d, cudaStream_t s) {
    uint64_t h = 0;
    GS_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    return h;
}

void prepare_y(Arena &a, const uint64_t *ykeys, uint64_t ny, int nfb, YPrep &out, cudaStream_t s) {
    out.ny = ny;
    GS_REQUIRE(ny < (1ull << 31), GSPARC_EUNSUPPORTED, "Y with more than 2^31 nonzeros");
    out.rank.reset(a, ny, s);
    if (ny == 0) {
        out.ncols = 0;
        out.nruns = 0;
        out.cols.reset(a, 1, s);
        out.run_key.reset(a, 1, s);
        out.run_start.reset(a, 1, s);
        GS_CUDA(cudaMemsetAsync(out.run_start.get(), 0, 4, s));
        return;
    }
    DBuf<uint8_t> flag(a, ny, s);
    DBuf<uint64_t> yf0(a, ny, s), yf1(a, ny, s);
    k_y_split<<<grid_for(ny), kThreads, 0, s>>>(ykeys, ny, nfb, flag, yf0);
    count_launch();
    GS_CUDA(cudaGetLastError());

    // distinct free indices (column space) and per-entry ranks
    int which = 0;
    sort_keys(a, ny, yf0, yf1, nfb, &which, s);
    uint64_t *sorted = which ? yf1.get() : yf0.get();
    uint64_t *uniq = which ? yf0.get() : yf1.get();
    DBuf<uint64_t> nsel(a, 1, s);
    size_t tmp = 0;
    GS_CUDA(cub::DeviceSelect::Unique(nullptr, tmp, sorted, uniq, nsel.get(), (int)ny, s));
    {
        DBuf<uint8_t> t(a, tmp, s);
        GS_CUDA(cub::DeviceSelect::Unique(t.get(), tmp, sorted, uniq, nsel.get(), (int)ny, s));
    }
    out.ncols = read_u64(nsel.get(), s);
    out.cols.reset(a, out.ncols, s);
    GS_CUDA(cudaMemcpyAsync(out.cols.get(), uniq, 8 * out.ncols, cudaMemcpyDeviceToDevice, s));
    k_y_rank<<<grid_for(ny), kThreads, 0, s>>>(ykeys, ny, nfb, out.cols, out.ncols, out.rank);
    count_launch();
    GS_CUDA(cudaGetLastError());

    // run table of contract keys
    DBuf<uint32_t> rs(a, ny + 1, s);
    tmp = 0;
    cub::CountingInputIterator<uint32_t> it(0);
    GS_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, it, flag.get(), rs.get(), nsel.get(), (int)ny, s));
    {
        DBuf<uint8_t> t(a, tmp, s);
        GS_CUDA(cub::DeviceSelect::Flagged(t.get(), tmp, it, flag.get(), rs.get(), nsel.get(), (int)ny, s));
    }
    out.nruns = read_u64(nsel.get(), s);
    out.run_key.reset(a, out.nruns, s);
    out.run_start = std::move(rs);
    k_run_keys<<<grid_for(out.nruns + 1), kThreads, 0, s>>>(ykeys, nfb, out.run_start, out.nruns, ny,
                                                             out.run_key, out.run_start);
    count_launch();
    GS_CUDA(cudaGetLastError());
}

void exclusive_scan_u32_to_u64(Arena &a, const uint32_t *in, uint64_t *out, uint64_t n,
                               cudaStream_t s) {
    GS_CUDA(cudaMemsetAsync(out, 0, 8, s));
    if (n == 0) return;
    cub::TransformInputIterator<uint64_t, CastU64, const uint32_t *> it(in, CastU64());
    size_t tmp = 0;
    GS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, it, out + 1, (int)n, s));
    DBuf<uint8_t> t(a, tmp, s);
    GS_CUDA(cub::DeviceScan::InclusiveSum(t.get(), tmp, it, out + 1, (int)n, s));
}

void match_x(Arena &a, const uint64_t *xkeys, uint64_t nx, int ncb, const YPrep &y, XMatch &out,
             cudaStream_t s) {
    out.nx = nx;
    GS_REQUIRE(nx < (1ull << 31), GSPARC_EUNSUPPORTED, "X with more than 2^31 nonzeros");
    out.pos.reset(a, nx, s);
    out.cnt.reset(a, nx, s);
    out.xprefix.reset(a, nx + 1, s);
    if (nx == 0) {
        out.nrows = 0;
        out.ir = 0;
        GS_CUDA(cudaMemsetAsync(out.xprefix.get(), 0, 8, s));
        out.row_start.reset(a, 1, s);
        GS_CUDA(cudaMemsetAsync(out.row_start.get(), 0, 4, s));
        out.row_xf.reset(a, 1, s);
        out.row_prod.reset(a, 1, s);
        return;
    }
    DBuf<uint8_t> rflag(a, nx, s);
    k_match<<<grid_for(nx), kThreads, 0, s>>>(xkeys, nx, ncb, y.run_key, y.run_start, y.nruns, out.pos,
                                               out.cnt, rflag);
    count_launch();
    GS_CUDA(cudaGetLastError());
    exclusive_scan_u32_to_u64(a, out.cnt, out.xprefix, nx, s);

    DBuf<uint32_t> rs(a, nx, s);
    DBuf<uint64_t> nsel(a, 1, s);
    size_t tmp = 0;
    cub::CountingInputIterator<uint32_t> it(0);
    GS_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, it, rflag.get(), rs.get(), nsel.get(), (int)nx, s));
    {
        DBuf<uint8_t> t(a, tmp, s);
        GS_CUDA(cub::DeviceSelect::Flagged(t.get(), tmp, it, rflag.get(), rs.get(), nsel.get(), (int)nx, s));
    }
    uint64_t hv[2];
    GS_CUDA(cudaMemcpyAsync(&hv[0], nsel.get(), 8, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaMemcpyAsync(&hv[1], out.xprefix.get() + nx, 8, cudaMemcpyDeviceToHost, s));
    GS_CUDA(cudaStreamSynchronize(s));
    out.nrows = hv[0];
    out.ir = hv[1];
    out.row_start.reset(a, out.nrows + 1, s);
    out.row_xf.reset(a, out.nrows, s);
    out.row_prod.reset(a, out.nrows, s);
    k_rows<<<grid_for(out.nrows + 1), kThreads, 0, s>>>(xkeys, ncb, rs, out.nrows, nx, out.xprefix,
                                                         out.row_start, out.row_xf, out.row_prod);
    count_launch();
    GS_CUDA(cudaGetLastError());
}

void index_match_compat(Arena &a, uint64_t nx, const uint64_t *xkeys, int x_ncbits, uint64_t ny,
                        const uint64_t *ykeys, int y_nfbits, uint64_t *pos, uint64_t *cnt,
                        uint64_t *prefix, cudaStream_t s) {
    YPrep y;
    prepare_y(a, ykeys, ny, y_nfbits, y, s);
    if (nx) {
        k_match_compat<<<grid_for(nx), kThreads, 0, s>>>(xkeys, nx, x_ncbits, y.run_key, y.run_start,
                                                          y.nruns, pos, cnt);
        count_launch();
        GS_CUDA(cudaGetLastError());
    }
    GS_CUDA(cudaMemsetAsync(prefix, 0, 8, s));
    if (nx) {
        size_t tmp = 0;
        GS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, cnt, prefix + 1, (int)nx, s));
        DBuf<uint8_t> t(a, tmp, s);
        GS_CUDA(cub::DeviceScan::InclusiveSum(t.get(), tmp, cnt, prefix + 1, (int)nx, s));
    }
}

}  // namespace gs
