// batch.cu -- many independent contractions run as one.
//
// The reference runs one gsparc::SpTC at a time (include/gsparc/sptc.cuh:16-360,
// driven from main.cu:293-376), so a stream of small contractions pays the
// fixed per-call cost (launches, host round trips) once per contraction.  Here
// the jobs of a batch are split into groups; inside a group every operand key
// carries its job id above the widest key of the group:
//
//     X key = job << kbx | (x_f << ncbits | c),   Y key = job << kby | (c << nfbits | y_f)
//
// so ONE linearise launch per side, ONE radix sort per side, ONE run table and
// ONE match serve every job of the group: sorting by the prefixed key sorts
// each job's keys exactly as the plain path does and keeps jobs apart.  Rows
// (distinct x_f) then know their job, and the accumulation kernels look up the
// job's column table and output key width per row (row_job_params), so ONE
// symbolic and ONE numeric persistent launch take the units of all jobs from
// one work counter.  Unit planning (light units, heavy rows) runs on the
// device, so a group needs two host round trips before its numeric launch
// whatever its number of jobs.  Each job's output is the contiguous range of
// the group's sorted output that belongs to it, delivered to the job's sink.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>

#include "engine.h"
#include "kernels.cuh"
#include "verify.h"
#include "wide.h"

namespace gs {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxGroupJobs = 65535;      // row_job is 16 bits
constexpr uint64_t kMaxGroupNnz = (1ull << 31) - 1;

inline int grid_for(uint64_t n) {
    uint64_t g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    if (g > 148ull * 32) g = 148ull * 32;
    return (int)g;
}

__device__ __forceinline__ uint64_t shl(uint64_t v, int s) { return s >= 64 ? 0ull : (v << s); }
__device__ __forceinline__ uint64_t shr(uint64_t v, int s) { return s >= 64 ? 0ull : (v >> s); }
__device__ __forceinline__ uint64_t low_mask(int b) { return b >= 64 ? ~0ull : ((1ull << b) - 1); }

template <class T>
__device__ __forceinline__ uint64_t lower_bound_dev(const T *a, uint64_t lo, uint64_t hi, T v) {
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// One operand of one job, for the batched linearise.
struct BLin {
    LinParams p;
    const uint64_t *idx;  // SoA idx[m * nnz + k]
    const float *val;
    uint64_t nnz;
};

// Per-job constants of the batched prep kernels.
struct BPrep {
    int x_ncbits;
    int y_nfbits;
    uint64_t light_max;  // rows with more products go to the windowed accumulator
};

// Per-job summary after the symbolic pass (entry g holds the totals).
struct JobOut {
    uint64_t row0;     // first row of the job
    uint64_t out_off;  // first output nonzero of the job
    uint64_t ir_off;   // matched products before the job
    uint64_t heavy0;   // heavy rows before the job
};

// reference: include/gsparc/tensor_manager.tpp:249-268 (X) and :272-293 (Y),
// once per job, with the job id above the group's widest key.  A key is masked
// to the group width, so an out-of-range index (flagged per job) can only
// damage its own job's keys.
__global__ void k_blin(const BLin *__restrict__ tab, const uint64_t *__restrict__ offs, int g,
                       uint64_t total, int kb, uint64_t *__restrict__ keys, float *__restrict__ vals,
                       unsigned int *__restrict__ jerr, int perm) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t km = low_mask(kb);
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += stride) {
        int lo = 0, hi = g;  // largest j with offs[j] <= k
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (offs[mid] <= k)
                lo = mid;
            else
                hi = mid;
        }
        const BLin &t = tab[lo];
        const uint64_t l = k - offs[lo];
        uint64_t f = 0, c = 0;
        bool bad = false;
        for (int m = 0; m < t.p.order; ++m) {
            const uint64_t v = t.idx[(uint64_t)m * t.nnz + l];
            bad |= v >= t.p.dims[m];
            if (t.p.is_c[m])
                c |= shl(v, t.p.shift[m]);
            else
                f |= shl(v, t.p.shift[m]);
        }
        if (bad) atomicOr(&jerr[lo], 1u);
        const uint64_t key = t.p.role == 0 ? (shl(f, t.p.ncbits) | c) : (shl(c, t.p.nfbits) | f);
        keys[k] = shl((uint64_t)lo, kb) | (key & km);
        // with perm the sort carries each entry's input position instead of its value
        vals[k] = perm ? __uint_as_float((unsigned int)k) : t.val[l];
    }
}

// The current values of sorted entries whose input positions the sort carried
// (k_blin with perm): vals[i] = the value at input position perm[i].
__global__ void k_bvals(const BLin *__restrict__ tab, const uint64_t *__restrict__ offs, int g, uint64_t total,
                        const float *__restrict__ perm, float *__restrict__ vals) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const uint64_t k = __float_as_uint(perm[i]);
        int lo = 0, hi = g;  // largest j with offs[j] <= k
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (offs[mid] <= k)
                lo = mid;
            else
                hi = mid;
        }
        vals[i] = tab[lo].val[k - offs[lo]];
    }
}

// Y: run boundaries of (job, contract key) and the prefixed free index.
// A job whose Y repeats a coordinate gets ydup[job] set: its runs may hold a
// free index twice, so none of its rows is streamed.
__global__ void k_by_split(const uint64_t *__restrict__ ykeys, uint64_t ny, int kby,
                           const BPrep *__restrict__ jobs, uint8_t *__restrict__ run_flag,
                           uint64_t *__restrict__ yfk, unsigned int *__restrict__ ydup) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t km = low_mask(kby);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ny; i += stride) {
        const uint64_t key = ykeys[i];
        const uint64_t j = shr(key, kby);
        const int nfb = jobs[j].y_nfbits;
        const uint64_t loc = key & km;
        const uint64_t c = shr(loc, nfb);
        uint8_t flag = 1;
        if (i > 0) {
            const uint64_t pk = ykeys[i - 1];
            flag = (shr(pk, kby) != j) || (shr(pk & km, nfb) != c);
            if (pk == key) atomicOr(&ydup[j], 1u);
        }
        run_flag[i] = flag;
        yfk[i] = shl(j, kby) | (loc & low_mask(nfb));
    }
}

// Distinct prefixed free indices -> plain free indices (the column tables).
__global__ void k_bcols(const uint64_t *__restrict__ uniq, const uint64_t *__restrict__ ncols_dev,
                        int kby, uint64_t *__restrict__ cols) {
    const uint64_t n = *ncols_dev;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t km = low_mask(kby);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        cols[i] = uniq[i] & km;
}

// Per-job column table range inside the group's table.
__global__ void k_bjobs(const uint64_t *__restrict__ uniq, const uint64_t *__restrict__ ncols_dev,
                        int kby, int g, const BPrep *__restrict__ jobs, BatchJob *__restrict__ acc) {
    const uint64_t n = *ncols_dev;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < g; j += gridDim.x * blockDim.x) {
        const uint64_t lo = lower_bound_dev<uint64_t>(uniq, 0, n, shl((uint64_t)j, kby));
        const uint64_t hi = (j + 1 == g) ? n : lower_bound_dev<uint64_t>(uniq, 0, n, shl((uint64_t)(j + 1), kby));
        BatchJob b;
        b.y_nfbits = jobs[j].y_nfbits;
        b.ncols = (uint32_t)(hi - lo);
        b.cols_off = lo;
        acc[j] = b;
    }
}

// Column rank of every Y entry inside its job's column table.
__global__ void k_brank(const uint64_t *__restrict__ ykeys, uint64_t ny, int kby,
                        const BPrep *__restrict__ jobs, const uint64_t *__restrict__ uniq,
                        const BatchJob *__restrict__ acc, uint32_t *__restrict__ rank) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t km = low_mask(kby);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ny; i += stride) {
        const uint64_t key = ykeys[i];
        const uint64_t j = shr(key, kby);
        const uint64_t f = key & km & low_mask(jobs[j].y_nfbits);
        const BatchJob b = acc[j];
        const uint64_t p = lower_bound_dev<uint64_t>(uniq, b.cols_off, b.cols_off + b.ncols, shl(j, kby) | f);
        rank[i] = (uint32_t)(p - b.cols_off);
    }
}

__global__ void k_bruns(const uint64_t *__restrict__ ykeys, int kby, const BPrep *__restrict__ jobs,
                        const uint32_t *__restrict__ rs, const uint64_t *__restrict__ nruns_dev,
                        uint64_t ny, uint64_t *__restrict__ run_key, uint32_t *__restrict__ run_start_out) {
    const uint64_t nr = *nruns_dev;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t km = low_mask(kby);
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= nr; r += stride) {
        if (r < nr) {
            const uint64_t key = ykeys[rs[r]];
            const uint64_t j = shr(key, kby);
            run_key[r] = shl(j, kby) | shr(key & km, jobs[j].y_nfbits);
        } else {
            run_start_out[nr] = (uint32_t)ny;
        }
    }
}

// reference: include/gsparc/indexMatch.cuh:67-118, over the run table of all
// jobs: the search key is (job, contract key).
__global__ void k_bmatch(const uint64_t *__restrict__ xkeys, uint64_t nx, int kbx, int kby,
                         const BPrep *__restrict__ jobs, const uint64_t *__restrict__ run_key,
                         const uint32_t *__restrict__ run_start, const uint64_t *__restrict__ nruns_dev,
                         uint32_t *__restrict__ pos, uint32_t *__restrict__ cnt,
                         uint8_t *__restrict__ row_flag) {
    const uint64_t nr = *nruns_dev;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t km = low_mask(kbx);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += stride) {
        const uint64_t key = xkeys[i];
        const uint64_t j = shr(key, kbx);
        const int ncb = jobs[j].x_ncbits;
        const uint64_t loc = key & km;
        const uint64_t target = shl(j, kby) | (loc & low_mask(ncb));
        const uint64_t r = lower_bound_dev<uint64_t>(run_key, 0, nr, target);
        uint32_t p = 0, n = 0;
        if (r < nr && run_key[r] == target) {
            p = run_start[r];
            n = run_start[r + 1] - p;
        }
        pos[i] = p;
        cnt[i] = n;
        uint8_t flag = 1;
        if (i > 0) {
            const uint64_t pk = xkeys[i - 1];
            flag = (shr(pk, kbx) != j) || (shr(pk & km, ncb) != shr(loc, ncb));
        }
        row_flag[i] = flag;
    }
}

// Row table: first X nonzero, free index, job and matched products of every
// row, the number of its X nonzeros that match (runs) and, for rows with one
// run, which nonzero that is.
__global__ void k_brows(const uint64_t *__restrict__ xkeys, int kbx, const BPrep *__restrict__ jobs,
                        const uint32_t *__restrict__ rs, const uint64_t *__restrict__ nrows_dev,
                        uint64_t nx, const uint64_t *__restrict__ xprefix, const uint32_t *__restrict__ mpre,
                        uint32_t *__restrict__ row_start, uint64_t *__restrict__ row_xf,
                        uint16_t *__restrict__ row_job, uint64_t *__restrict__ row_prod,
                        uint32_t *__restrict__ row_runs, uint32_t *__restrict__ row_xi) {
    const uint64_t nr = *nrows_dev;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t km = low_mask(kbx);
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= nr; r += stride) {
        if (r == nr) {
            row_start[nr] = (uint32_t)nx;
            continue;
        }
        const uint32_t a = rs[r];
        const uint32_t b = (r + 1 < nr) ? rs[r + 1] : (uint32_t)nx;
        const uint64_t key = xkeys[a];
        const uint64_t j = shr(key, kbx);
        row_start[r] = a;
        row_xf[r] = shr(key & km, jobs[j].x_ncbits);
        row_job[r] = (uint16_t)j;
        row_prod[r] = xprefix[b] - xprefix[a];
        const uint32_t runs = mpre[b] - mpre[a];
        row_runs[r] = runs;
        if (runs == 1) {
            // the nonzero i in [a, b) with mpre[i] == mpre[a] < mpre[i + 1]
            uint32_t lo = a, hi = b;  // first i in (a, b] with mpre[i] > mpre[a], minus one
            const uint32_t m0 = mpre[a];
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (mpre[mid + 1] <= m0)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            row_xi[r] = lo;
        }
    }
}

// Row classes: single-run rows of jobs without repeated Y coordinates stream
// (their output count is their product count), other rows with more than the job's light limit of products are
// heavy, the rest with products are light.  Rows outside [range[0],
// range[1]) (a shard) get no class and no output.
__global__ void k_bclass(const uint64_t *__restrict__ row_prod, const uint32_t *__restrict__ row_runs,
                         const uint16_t *__restrict__ row_job, const BPrep *__restrict__ jobs,
                         const unsigned int *__restrict__ ydup,
                         const uint64_t *__restrict__ nrows_dev, const uint64_t *__restrict__ range, uint64_t nx,
                         uint8_t *__restrict__ heavy, uint8_t *__restrict__ lnz, uint8_t *__restrict__ sflag,
                         uint8_t *__restrict__ brk, uint64_t *__restrict__ lp, uint32_t *__restrict__ row_nnz) {
    const uint64_t nr = *nrows_dev;
    const uint64_t r0 = range ? range[0] : 0, r1 = range ? range[1] : nr;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nx; r += stride) {
        uint8_t h = 0, l = 0, st = 0;
        uint64_t p = 0;
        if (r < nr && r >= r0 && r < r1) {
            p = row_prod[r];
            const uint16_t j = row_job[r];
            st = row_runs[r] == 1 && !ydup[j];
            h = !st && p > jobs[j].light_max;
            l = !st && !h && p > 0;
            if (st) row_nnz[r] = (uint32_t)p;
        }
        heavy[r] = h;
        lnz[r] = l;
        sflag[r] = st;
        brk[r] = h | st;
        lp[r] = l ? p : 0;
    }
}

// Row range of one shard of a single job: shard s starts at the first row
// whose product midpoint reaches s/n of the job's products, i.e. the first r
// with n * (P[r] + P[r+1]) >= 2 * s * P[nrows] (P = row product prefix), the
// exact-integer form of the host planner gs::plan_shards.
// range = {first row, end row, products of the shard}.
__device__ uint64_t shard_bound(const uint64_t *P, uint64_t nr, int s, int n) {
    if (s <= 0) return 0;
    if (s >= n) return nr;
    const unsigned __int128 target = (unsigned __int128)2 * (unsigned)s * P[nr];
    uint64_t lo = 0, hi = nr;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if ((unsigned __int128)(unsigned)n * ((unsigned __int128)P[mid] + P[mid + 1]) >= target)
            hi = mid;
        else
            lo = mid + 1;
    }
    return lo;
}

__global__ void k_shard_range(const uint64_t *__restrict__ P, const uint64_t *__restrict__ nrows_dev, int shard,
                              int nshards, uint64_t *__restrict__ range) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint64_t nr = *nrows_dev;
        const uint64_t a = shard_bound(P, nr, shard, nshards), b = shard_bound(P, nr, shard + 1, nshards);
        range[0] = a;
        range[1] = b;
        range[2] = P[b] - P[a];
    }
}

__global__ void k_sprod(const uint32_t *__restrict__ SR, const uint64_t *__restrict__ ns_dev, uint64_t nx,
                        const uint64_t *__restrict__ row_prod, uint64_t *__restrict__ sprod) {
    const uint64_t ns = *ns_dev;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nx; k += stride)
        sprod[k] = k < ns ? row_prod[SR[k]] : 0;
}

// A light unit is a maximal run of light rows with products whose first
// product falls in the same bin of `bin` products, with no heavy row between
// them (so it is a contiguous row range): its products stay below
// bin + light_max.
__global__ void k_bstart(const uint32_t *__restrict__ L, const uint64_t *__restrict__ nl_dev,
                         const uint64_t *__restrict__ lpre, const uint32_t *__restrict__ hc,
                         uint64_t bin, uint64_t nx, uint8_t *__restrict__ sf) {
    const uint64_t n = *nl_dev;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nx; k += stride) {
        uint8_t s = 0;
        if (k < n) {
            const uint32_t r = L[k];
            s = 1;
            if (k > 0) {
                const uint32_t q = L[k - 1];
                s = (hc[q] != hc[r]) || (lpre[q] / bin != lpre[r] / bin);
            }
        }
        sf[k] = s;
    }
}

// A light unit ends at the next unit start or at the next row of another
// class (heavy or stream: the breakers B, bc = breakers before each row).
__global__ void k_bunits(const uint32_t *__restrict__ L, const uint32_t *__restrict__ S,
                         const uint64_t *__restrict__ cnts, const uint32_t *__restrict__ H,
                         const uint32_t *__restrict__ hc, uint32_t *__restrict__ units) {
    const uint64_t nrows = cnts[2], nh = cnts[8], nu = cnts[5];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nu; u += stride) {
        const uint32_t r0 = L[S[u]];
        const uint64_t next = (u + 1 < nu) ? L[S[u + 1]] : nrows;
        const uint32_t h = hc[r0];
        const uint64_t nhv = h < nh ? H[h] : nrows;
        units[2 * u] = r0;
        units[2 * u + 1] = (uint32_t)(next < nhv ? next : nhv);
    }
}

__global__ void k_gather_prod(const uint32_t *__restrict__ H, uint64_t nh,
                              const uint64_t *__restrict__ row_prod, uint64_t *__restrict__ hp) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nh; k += stride)
        hp[k] = row_prod[H[k]];
}

__global__ void k_bjobout(const uint16_t *__restrict__ row_job, uint64_t nrows,
                          const uint64_t *__restrict__ row_off, const uint64_t *__restrict__ xprefix,
                          const uint32_t *__restrict__ hc, const uint64_t *__restrict__ xoffs, int g,
                          JobOut *__restrict__ out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= g; j += gridDim.x * blockDim.x) {
        const uint64_t r0 = (j == g) ? nrows : lower_bound_dev<uint16_t>(row_job, 0, nrows, (uint16_t)j);
        JobOut o;
        o.row0 = r0;
        o.out_off = row_off[r0];
        o.ir_off = xprefix[xoffs[j]];
        o.heavy0 = hc[r0];
        out[j] = o;
    }
}

// Light units first-row search: light units starting before row r.
__device__ __forceinline__ uint64_t light_before(const uint32_t *units, uint64_t nu, uint32_t r) {
    uint64_t lo = 0, hi = nu;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (units[2 * mid] < r)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// The three unit lists of a group, all in row order: light units (row
// pairs), heavy rows and single-run (stream) rows.
struct UnitLists {
    const uint32_t *units;
    uint64_t nu;
    const uint32_t *H;
    uint64_t nh;
    const uint32_t *SR;
    uint64_t ns;
    __device__ uint64_t size() const { return nu + nh + ns; }
    // first row of unit k of the concatenation light | heavy | stream
    __device__ uint32_t row(uint64_t k, uint32_t *last) const {
        if (k < nu) {
            *last = units[2 * k + 1];
            return units[2 * k];
        }
        const uint32_t r = k < nu + nh ? H[k - nu] : SR[k - nu - nh];
        *last = r + 1;
        return r;
    }
    // units of all three lists that start before row r
    __device__ uint64_t before(uint32_t r) const {
        return light_before(units, nu, r) + lower_bound_dev<uint32_t>(H, 0, nh, r) +
               lower_bound_dev<uint32_t>(SR, 0, ns, r);
    }
};

// Largest output of one unit.
__global__ void k_unit_max(UnitLists u, const uint64_t *__restrict__ row_off, uint64_t *__restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t m = 0;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < u.size(); k += stride) {
        uint32_t r1;
        const uint32_t r0 = u.row(k, &r1);
        const uint64_t v = row_off[r1] - row_off[r0];
        m = v > m ? v : m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t w = __shfl_xor_sync(0xffffffffu, m, o);
        m = w > m ? w : m;
    }
    if ((threadIdx.x & 31) == 0 && m) atomicMax((unsigned long long *)out, (unsigned long long)m);
}

// First row and first output of every unit, the three lists merged in row
// order (the lists are row-ordered and their rows are disjoint).
__global__ void k_merge_starts(UnitLists u, const uint64_t *__restrict__ row_off, uint32_t *__restrict__ urow,
                               uint64_t *__restrict__ uoff) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < u.size(); k += stride) {
        uint32_t r1;
        const uint32_t r = u.row(k, &r1);
        const uint64_t p = u.before(r);
        urow[p] = r;
        uoff[p] = row_off[r];
    }
}

// Chunk k starts at the first unit whose output starts at or after
// target[k] (target[0] = 0, increasing).  info[5k..5k+4] = first row, first
// output, first light unit, first heavy row (row-ordered index), first stream
// row of chunk k; entry K closes the last chunk.
constexpr int kChunkInfo = 5;
__global__ void k_chunk_bounds(const uint32_t *__restrict__ urow, const uint64_t *__restrict__ uoff, uint64_t M,
                               const uint64_t *__restrict__ target, uint64_t K, UnitLists u, uint64_t nrows,
                               uint64_t ntot, uint64_t *__restrict__ info) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k <= K; k += stride) {
        const uint64_t b = k == 0 ? 0 : (k == K ? M : lower_bound_dev<uint64_t>(uoff, 0, M, target[k]));
        const uint32_t row = (uint32_t)(b < M ? urow[b] : nrows);
        uint64_t *o = info + kChunkInfo * k;
        o[0] = row;
        o[1] = b < M ? uoff[b] : ntot;
        o[2] = light_before(u.units, u.nu, row);
        o[3] = lower_bound_dev<uint32_t>(u.H, 0, u.nh, row);
        o[4] = lower_bound_dev<uint32_t>(u.SR, 0, u.ns, row);
    }
}

// Sort key grouping heavy rows by chunk, largest first inside a chunk.
__global__ void k_heavy_chunk_keys(const uint32_t *__restrict__ Hs, uint64_t nh,
                                   const uint64_t *__restrict__ row_prod, const uint64_t *__restrict__ info,
                                   uint64_t K, uint64_t *__restrict__ keys) {
    constexpr uint64_t kProdMask = (1ull << 44) - 1;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nh; k += stride) {
        const uint32_t r = Hs[k];
        uint64_t lo = 0, hi = K;  // last chunk whose first row <= r
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) >> 1;
            if (info[kChunkInfo * mid] <= r)
                lo = mid;
            else
                hi = mid;
        }
        const uint64_t p = row_prod[r];
        keys[k] = (lo << 44) | (kProdMask - (p < kProdMask ? p : kProdMask));
    }
}

struct CastU32 {
    __host__ __device__ uint32_t operator()(uint8_t v) const { return v; }
};
struct CastU64 {
    __host__ __device__ uint64_t operator()(uint32_t v) const { return v; }
};
struct NonZero {
    __host__ __device__ uint32_t operator()(uint32_t v) const { return v != 0; }
};

template <class T>
void h2d(T *d, const T *h, size_t n, cudaStream_t s) {
    if (n) GS_CUDA(cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, s));
}
template <class T>
void d2h(T *h, const T *d, size_t n, cudaStream_t s) {
    if (n) GS_CUDA(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, s));
}

// Indices i < n with flag[i] != 0, ascending; the count goes to *count (device).
void select_idx(Arena &A, const uint8_t *flag, uint64_t n, uint32_t *out, uint64_t *count, cudaStream_t s) {
    if (n == 0) {
        GS_CUDA(cudaMemsetAsync(count, 0, 8, s));
        return;
    }
    cub::CountingInputIterator<uint32_t> it(0);
    size_t tmp = 0;
    GS_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, it, flag, out, count, (int)n, s));
    DBuf<uint8_t> t(A, tmp, s);
    GS_CUDA(cub::DeviceSelect::Flagged(t.get(), tmp, it, flag, out, count, (int)n, s));
}

// out[0] = 0, out[i+1] = in[0] + ... + in[i] (n + 1 entries).
template <class It, class T>
void prefix_sum(Arena &A, It in, T *out, uint64_t n, cudaStream_t s) {
    GS_CUDA(cudaMemsetAsync(out, 0, sizeof(T), s));
    if (n == 0) return;
    size_t tmp = 0;
    GS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, in, out + 1, (int)n, s));
    DBuf<uint8_t> t(A, tmp, s);
    GS_CUDA(cub::DeviceScan::InclusiveSum(t.get(), tmp, in, out + 1, (int)n, s));
}

inline int ceil_log2(uint64_t n) {
    int b = 0;
    while ((1ull << b) < n) ++b;
    return b;
}

struct Job {
    gsparc_job *job;
    const gsparc_tensor *tx, *ty;   // the operands the engine runs on (relabeled when wide)
    std::shared_ptr<WideMap> wide;  // set when the operand keys need more than 64 bits
    Layout LX, LY;
    uint64_t light_max;
    int width;          // widest operand key
    int key_words = 1;  // output key words delivered to the sink (2: 128-bit keys)
    bool done = false;  // reported through the completion callback
};

// First product count after which a job boundary closes a chunk when jobs
// complete one by one (about a millisecond of accumulation); each further cut
// waits for twice as many products, so a batch has O(log) extra chunks.
constexpr uint64_t kFirstCutProducts = 1ull << 26;

struct Times {
    double lin = 0, sort = 0, match = 0, plan = 0, contract = 0, out = 0, total = 0, numeric = 0;
};

// Everything the numeric pass of one group needs, kept on the device by a plan
// (gsparc_plan_*): the sorted operands' positions and current values, the run
// table, the match, the rows, the unit lists and the output offsets.
struct GroupPlan {
    int g = 0;
    uint64_t nx = 0, ny = 0, ntot = 0, nu = 0, nh = 0, nsr = 0;
    int gl = 1, gh = 1, gs_grid = 1;
    AccArgs aa{};
    std::vector<uint64_t> job_first;  // g + 1 group-local output offsets
    std::vector<Job *> jobs;
    DBuf<BLin> d_lx, d_ly;
    DBuf<uint64_t> d_xoffs, d_yoffs;
    DBuf<float> xperm, yperm, xvals, yvals;
    DBuf<uint64_t> ykeys;  // sorted Y keys (the single-run-row copy reads y_f from them)
    DBuf<BatchJob> d_acc;
    DBuf<uint32_t> rank, pos, cnt, row_start, units, H, H2, SR, row_xi, cursor, pend;
    DBuf<uint64_t> cols, xprefix, row_xf, sprefix, row_off;
    DBuf<uint16_t> row_job;
    DBuf<uint32_t> Hc;         // heavy rows grouped by chunk (several chunks only)
    DBuf<uint32_t> hbm, row_rb;  // heavy rows' kept column bitmaps (may be empty)
    DBuf<uint64_t> row_bmoff;
    DBuf<unsigned int> flags;  // error bits, work counter, windows swept, spare
    struct Chunk {
        uint64_t lu0, lu1, h0, h1, s0, s1, first, n;
    };
    std::vector<Chunk> chunks;
    const uint32_t *heavy_list() const { return Hc.get() ? Hc.get() : (H2.get() ? H2.get() : H.get()); }
};

// Delivers [dk, dk + n) of a job's output (first = offset inside the job);
// kw = key words per nonzero (2: 128-bit keys, dk holds 2n words).
void deliver_slice(gsparc_sink &sink, const uint64_t *dk, const float *dv, uint64_t n, uint64_t first,
                   uint64_t job_nnz, cudaStream_t s2, gsparc_stats &st, uint64_t &bytes_d2h, int kw = 1) {
    if (n == 0) return;
    if (sink.kind == GSPARC_SINK_DEVICE) {
        const uint64_t step = sink.max_chunk_nnz ? sink.max_chunk_nnz : n;
        for (uint64_t off = 0; off < n; off += step) {
            const uint64_t m = std::min(step, n - off);
            if (sink.on_chunk(sink.user, dk + kw * off, dv + off, m, first + off, 1))
                fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
        }
        ++st.chunks;
    } else if (sink.kind == GSPARC_SINK_HOST) {
        if (sink.host_capacity >= job_nnz) {
            d2h(sink.host_keys + kw * first, dk, kw * n, s2);
            d2h(sink.host_vals + first, dv, n, s2);
            bytes_d2h += (8 * kw + 4) * n;
            GS_CUDA(cudaStreamSynchronize(s2));
            if (sink.on_chunk &&
                sink.on_chunk(sink.user, sink.host_keys + kw * first, sink.host_vals + first, n, first, 0))
                fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
        } else {
            for (uint64_t off = 0; off < n; off += sink.host_capacity) {
                const uint64_t m = std::min<uint64_t>(sink.host_capacity, n - off);
                d2h(sink.host_keys, dk + kw * off, kw * m, s2);
                d2h(sink.host_vals, dv + off, m, s2);
                bytes_d2h += (8 * kw + 4) * m;
                GS_CUDA(cudaStreamSynchronize(s2));
                if (sink.on_chunk && sink.on_chunk(sink.user, sink.host_keys, sink.host_vals, m, first + off, 0))
                    fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
            }
        }
        ++st.chunks;
    }
}

void run_group(gsparc_ctx *ctx, std::vector<Job *> &G, uint64_t max_chunk_nnz, int shard, int nshards,
               Times &tm, gsparc_stats &bst, cudaStream_t s, const JobDoneFn *done_fn, GroupPlan *keep = nullptr) {
    Arena &A = ctx->arena;
    const int g = (int)G.size();
    const int jb = ceil_log2((uint64_t)g);
    int kbx = 0, kby = 0;
    uint64_t max_light = 0;
    for (Job *j : G) {
        kbx = std::max(kbx, j->LX.nbits());
        kby = std::max(kby, j->LY.nbits());
        max_light = std::max(max_light, j->light_max);
    }
    // light units hold rows whose first product falls in one bin of light_bin
    // products: fewer than light_bin + light_max <= kLightCap products
    const uint64_t light_bin = std::max<uint64_t>(
        1, std::min<uint64_t>(kLightUnitMax - kLightRowMax, (uint64_t)kLightCap - std::min<uint64_t>(max_light, kLightCap - 1)));
    GS_REQUIRE(kbx + jb <= 64 && kby + jb <= 64, GSPARC_EINTERNAL, "batch group keys wider than 64 bits");

    cudaEvent_t *ev = ctx->ev;
    auto mark = [&](int i) { GS_CUDA(cudaEventRecord(ev[i], s)); };
    auto ms = [&](int a, int b) {
        float t = 0.f;
        GS_CUDA(cudaEventElapsedTime(&t, ev[a], ev[b]));
        return (double)t;
    };
    mark(0);

    // ---- job tables ----
    std::vector<uint64_t> xoffs(g + 1, 0), yoffs(g + 1, 0);
    std::vector<BLin> lx(g), ly(g);
    std::vector<BPrep> bp(g);
    for (int j = 0; j < g; ++j) {
        const gsparc_job &J = *G[j]->job;
        const gsparc_tensor *tx = G[j]->tx, *ty = G[j]->ty;
        xoffs[j + 1] = xoffs[j] + tx->nnz;
        yoffs[j + 1] = yoffs[j] + ty->nnz;
        lx[j] = {make_lin_params(G[j]->LX, tx->dims, 0), tx->d_idx, tx->d_val, tx->nnz};
        ly[j] = {make_lin_params(G[j]->LY, ty->dims, 1), ty->d_idx, ty->d_val, ty->nnz};
        bp[j] = {G[j]->LX.ncbits, G[j]->LY.nfbits, G[j]->light_max};
    }
    const uint64_t nx = xoffs[g], ny = yoffs[g];
    DBuf<BLin> d_lx(A, g, s), d_ly(A, g, s);
    DBuf<BPrep> d_bp(A, g, s);
    DBuf<BatchJob> d_acc(A, g, s);
    DBuf<uint64_t> d_xoffs(A, g + 1, s), d_yoffs(A, g + 1, s);
    DBuf<unsigned int> d_jerr(A, g, s), d_ydup(A, g, s);
    // 0 ncols, 1 nruns, 2 nrows, 3 heavy rows, 4 light rows, 5 light units, 6 largest unit output,
    // 7 stream rows, 8 heavy + stream rows, 9..11 shard row range and products
    DBuf<uint64_t> cnts(A, 16, s);
    h2d(d_lx.get(), lx.data(), g, s);
    h2d(d_ly.get(), ly.data(), g, s);
    h2d(d_bp.get(), bp.data(), g, s);
    h2d(d_xoffs.get(), xoffs.data(), g + 1, s);
    h2d(d_yoffs.get(), yoffs.data(), g + 1, s);
    GS_CUDA(cudaMemsetAsync(d_jerr.get(), 0, 4 * g, s));
    GS_CUDA(cudaMemsetAsync(d_ydup.get(), 0, 4 * g, s));
    GS_CUDA(cudaMemsetAsync(cnts.get(), 0, 128, s));
    GS_CUDA(cudaMemsetAsync(ctx->d_flag, 0, 4 * 4, s));
    bst.bytes_h2d += (sizeof(BLin) * 2 + sizeof(BPrep) + 16) * g;

    // ---- linearise ----
    DBuf<uint64_t> xk0(A, nx, s), xk1(A, nx, s), yk0(A, ny, s), yk1(A, ny, s);
    DBuf<float> xv0(A, nx, s), xv1(A, nx, s), yv0(A, ny, s), yv1(A, ny, s);
    if (nx) {
        k_blin<<<grid_for(nx), kThreads, 0, s>>>(d_lx, d_xoffs, g, nx, kbx, xk0, xv0, d_jerr, keep != nullptr);
        count_launch();
        GS_CUDA(cudaGetLastError());
    }
    if (ny) {
        k_blin<<<grid_for(ny), kThreads, 0, s>>>(d_ly, d_yoffs, g, ny, kby, yk0, yv0, d_jerr, keep != nullptr);
        count_launch();
        GS_CUDA(cudaGetLastError());
    }
    mark(1);

    // ---- sort ----
    int wx = 0, wy = 0;
    if (ctx->sort_impl) {  // gsparc_ctx_set_sort; a failed look-back sets bit 8 of the error word
        own_sort_pairs(A, nx, xk0, xk1, xv0, xv1, kbx + jb, &wx, ctx->d_flag, s);
        own_sort_pairs(A, ny, yk0, yk1, yv0, yv1, kby + jb, &wy, ctx->d_flag, s);
    } else {
        sort_pairs(A, nx, xk0, xk1, xv0, xv1, kbx + jb, &wx, s);
        sort_pairs(A, ny, yk0, yk1, yv0, yv1, kby + jb, &wy, s);
    }
    const uint64_t *xkeys = wx ? xk1.get() : xk0.get();
    const float *xvals = wx ? xv1.get() : xv0.get();
    const uint64_t *ykeys = wy ? yk1.get() : yk0.get();
    const float *yvals = wy ? yv1.get() : yv0.get();
    if (wx) { xk0.release(); xv0.release(); } else { xk1.release(); xv1.release(); }
    if (wy) { yk0.release(); yv0.release(); } else { yk1.release(); yv1.release(); }
    if (keep) {
        // the sorted "values" are input positions: keep them, fetch the values
        keep->ykeys = wy ? std::move(yk1) : std::move(yk0);  // ykeys keeps pointing at it
        keep->xperm = wx ? std::move(xv1) : std::move(xv0);
        keep->yperm = wy ? std::move(yv1) : std::move(yv0);
        keep->xvals.reset(A, std::max<uint64_t>(nx, 1), s);
        keep->yvals.reset(A, std::max<uint64_t>(ny, 1), s);
        if (nx) k_bvals<<<grid_for(nx), kThreads, 0, s>>>(d_lx, d_xoffs, g, nx, keep->xperm, keep->xvals);
        if (ny) k_bvals<<<grid_for(ny), kThreads, 0, s>>>(d_ly, d_yoffs, g, ny, keep->yperm, keep->yvals);
        count_launch((nx ? 1 : 0) + (ny ? 1 : 0));
        GS_CUDA(cudaGetLastError());
        xvals = keep->xvals.get();
        yvals = keep->yvals.get();
    }
    mark(2);

    // ---- Y column tables, ranks and run table ----
    const uint64_t nyb = std::max<uint64_t>(ny, 1), nxb = std::max<uint64_t>(nx, 1);
    DBuf<uint32_t> rank(A, nyb, s);
    DBuf<uint64_t> cols(A, nyb, s), run_key(A, nyb, s);
    DBuf<uint32_t> run_start(A, ny + 1, s);
    {
        DBuf<uint8_t> flag(A, nyb, s);
        DBuf<uint64_t> yf0(A, nyb, s), yf1(A, nyb, s);
        if (ny) {
            k_by_split<<<grid_for(ny), kThreads, 0, s>>>(ykeys, ny, kby, d_bp, flag, yf0, d_ydup);
            count_launch();
            GS_CUDA(cudaGetLastError());
        }
        int which = 0;
        sort_keys(A, ny, yf0, yf1, kby + jb, &which, s);
        uint64_t *sorted = which ? yf1.get() : yf0.get();
        uint64_t *uniq = which ? yf0.get() : yf1.get();
        if (ny) {
            size_t tmp = 0;
            GS_CUDA(cub::DeviceSelect::Unique(nullptr, tmp, sorted, uniq, cnts.get() + 0, (int)ny, s));
            DBuf<uint8_t> t(A, tmp, s);
            GS_CUDA(cub::DeviceSelect::Unique(t.get(), tmp, sorted, uniq, cnts.get() + 0, (int)ny, s));
            k_bcols<<<grid_for(ny), kThreads, 0, s>>>(uniq, cnts.get() + 0, kby, cols);
            count_launch();
        }
        k_bjobs<<<grid_for(g), kThreads, 0, s>>>(uniq, cnts.get() + 0, kby, g, d_bp, d_acc);
        count_launch();
        GS_CUDA(cudaGetLastError());
        if (ny) {
            k_brank<<<grid_for(ny), kThreads, 0, s>>>(ykeys, ny, kby, d_bp, uniq, d_acc, rank);
            count_launch();
            GS_CUDA(cudaGetLastError());
        }
        select_idx(A, flag, ny, run_start, cnts.get() + 1, s);
        k_bruns<<<grid_for(ny + 1), kThreads, 0, s>>>(ykeys, kby, d_bp, run_start, cnts.get() + 1, ny, run_key,
                                                       run_start);
        count_launch();
        GS_CUDA(cudaGetLastError());
    }

    // ---- X match, row table and unit planning ----
    DBuf<uint32_t> pos(A, nxb, s), cnt(A, nxb, s);
    DBuf<uint64_t> xprefix(A, nx + 1, s);
    DBuf<uint32_t> row_start(A, nx + 1, s);
    DBuf<uint64_t> row_xf(A, nxb, s), row_prod(A, nxb, s);
    DBuf<uint16_t> row_job(A, nxb, s);
    DBuf<uint32_t> H(A, nxb, s), hc(A, nx + 1, s), units(A, 2 * nxb, s);
    DBuf<uint64_t> lpre(A, nx + 1, s);
    DBuf<uint32_t> mpre(A, nx + 1, s), row_runs(A, nxb, s), row_xi(A, nxb, s), SR(A, nxb, s);
    DBuf<uint64_t> sprefix(A, nx + 1, s);
    DBuf<uint32_t> row_nnz(A, nxb, s);
    GS_CUDA(cudaMemsetAsync(row_nnz.get(), 0, 4 * nxb, s));
    // heavy rows' kept column bitmaps: words of every heavy row and of the
    // dense ones only, their word offsets, each row's smallest rank
    const bool keep_bm = ctx->keep_row_bitmaps != 0;
    DBuf<uint32_t> bm_w_all, bm_w_dense, row_rb;
    DBuf<uint64_t> bm_off_all, bm_off_dense;
    if (keep_bm) {
        bm_w_all.reset(A, nxb, s);
        bm_w_dense.reset(A, nxb, s);
        row_rb.reset(A, nxb, s);
        bm_off_all.reset(A, nx + 1, s);
        bm_off_dense.reset(A, nx + 1, s);
    }
    {
        DBuf<uint8_t> rflag(A, nxb, s);
        if (nx) {
            k_bmatch<<<grid_for(nx), kThreads, 0, s>>>(xkeys, nx, kbx, kby, d_bp, run_key, run_start,
                                                        cnts.get() + 1, pos, cnt, rflag);
            count_launch();
            GS_CUDA(cudaGetLastError());
        }
        // 64-bit accumulation: a group's matched products can pass 2^32
        cub::TransformInputIterator<uint64_t, CastU64, const uint32_t *> cit(cnt.get(), CastU64());
        prefix_sum(A, cit, xprefix.get(), nx, s);
        cub::TransformInputIterator<uint32_t, NonZero, const uint32_t *> mit(cnt.get(), NonZero());
        prefix_sum(A, mit, mpre.get(), nx, s);
        DBuf<uint32_t> rsx(A, nxb, s);
        select_idx(A, rflag, nx, rsx, cnts.get() + 2, s);
        rflag.release();
        DBuf<uint8_t> heavy(A, nxb, s), lnz(A, nxb, s), sflag(A, nxb, s), brk(A, nxb, s);
        DBuf<uint64_t> lp(A, nxb, s);
        GS_CUDA(cudaMemsetAsync(row_prod.get(), 0, 8 * nxb, s));
        k_brows<<<grid_for(nx + 1), kThreads, 0, s>>>(xkeys, kbx, d_bp, rsx, cnts.get() + 2, nx, xprefix, mpre,
                                                       row_start, row_xf, row_job, row_prod, row_runs, row_xi);
        count_launch();
        GS_CUDA(cudaGetLastError());
        const uint64_t *range = nullptr;
        if (nshards > 1) {
            DBuf<uint64_t> rp(A, nx + 1, s);
            prefix_sum(A, row_prod.get(), rp.get(), nx, s);
            k_shard_range<<<1, 32, 0, s>>>(rp, cnts.get() + 2, shard, nshards, cnts.get() + 9);
            count_launch();
            GS_CUDA(cudaGetLastError());
            range = cnts.get() + 9;
        }
        if (nx) {
            k_bclass<<<grid_for(nx), kThreads, 0, s>>>(row_prod, row_runs, row_job, d_bp, d_ydup, cnts.get() + 2,
                                                        range, nx, heavy, lnz, sflag, brk, lp, row_nnz);
            count_launch();
            GS_CUDA(cudaGetLastError());
        }
        select_idx(A, sflag, nx, SR, cnts.get() + 7, s);
        {
            DBuf<uint64_t> sprod(A, nxb, s);
            if (nx) {
                k_sprod<<<grid_for(nx), kThreads, 0, s>>>(SR, cnts.get() + 7, nx, row_prod, sprod);
                count_launch();
                GS_CUDA(cudaGetLastError());
            }
            prefix_sum(A, sprod.get(), sprefix.get(), nx, s);
        }
        mark(3);
        prefix_sum(A, lp.get(), lpre.get(), nx, s);
        cub::TransformInputIterator<uint32_t, CastU32, const uint8_t *> hit(heavy.get(), CastU32());
        prefix_sum(A, hit, hc.get(), nx, s);
        select_idx(A, heavy, nx, H, cnts.get() + 3, s);
        DBuf<uint32_t> bc(A, nx + 1, s), B(A, nxb, s);
        cub::TransformInputIterator<uint32_t, CastU32, const uint8_t *> bit(brk.get(), CastU32());
        prefix_sum(A, bit, bc.get(), nx, s);
        select_idx(A, brk, nx, B, cnts.get() + 8, s);
        DBuf<uint32_t> L(A, nxb, s), S(A, nxb, s);
        select_idx(A, lnz, nx, L, cnts.get() + 4, s);
        if (nx) {
            k_bstart<<<grid_for(nx), kThreads, 0, s>>>(L, cnts.get() + 4, lpre, bc,
                                                        light_bin, nx, heavy);
            count_launch();
            GS_CUDA(cudaGetLastError());
        }
        select_idx(A, heavy, nx, S, cnts.get() + 5, s);  // `heavy` now holds the unit-start flags
        k_bunits<<<grid_for(nx), kThreads, 0, s>>>(L, S, cnts, B, bc, units);
        count_launch();
        GS_CUDA(cudaGetLastError());
        if (keep_bm) {
            launch_heavy_spans(H, cnts.get() + 3, nx, nx, row_start, pos, cnt, rank, row_prod, bm_w_all, bm_w_dense,
                               row_rb, s);
            exclusive_scan_u32_to_u64(A, bm_w_all, bm_off_all, nx, s);
            exclusive_scan_u32_to_u64(A, bm_w_dense, bm_off_dense, nx, s);
        }
    }
    uint64_t hc_cnt[16];
    std::vector<unsigned int> jerr(g);
    uint64_t ir = 0;
    d2h(hc_cnt, cnts.get(), 16, s);
    d2h(jerr.data(), d_jerr.get(), g, s);
    d2h(&ir, xprefix.get() + nx, 1, s);
    uint64_t bm_words_all = 0, bm_words_dense = 0;
    if (keep_bm) {
        d2h(&bm_words_all, bm_off_all.get() + nx, 1, s);
        d2h(&bm_words_dense, bm_off_dense.get() + nx, 1, s);
    }
    GS_CUDA(cudaStreamSynchronize(s));
    const uint64_t nrows = hc_cnt[2], nh = hc_cnt[3], nu = hc_cnt[5], nsr = hc_cnt[7];
    if (nshards > 1) ir = hc_cnt[11];  // the shard's products
    bst.ir_nnz += ir;
    bst.rows += nrows;
    bst.heavy_rows += nh;
    bst.stream_rows += nsr;

    // heavy rows largest first (H itself stays in row order for chunk planning)
    DBuf<uint32_t> H2;
    DBuf<uint64_t> hp0, hp1;
    const uint32_t *Hs = H.get();
    if (nh > 1) {
        hp0.reset(A, nh, s);
        hp1.reset(A, nh, s);
        H2.reset(A, nh, s);
        k_gather_prod<<<grid_for(nh), kThreads, 0, s>>>(H, nh, row_prod, hp0);
        count_launch();
        GS_CUDA(cudaGetLastError());
        const int bits = std::max(1, 64 - __builtin_clzll(std::max<uint64_t>(ir, 1)));
        size_t tmp = 0;
        GS_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, hp0.get(), hp1.get(), H.get(), H2.get(),
                                                          (int)nh, 0, bits, s));
        DBuf<uint8_t> t(A, tmp, s);
        GS_CUDA(cub::DeviceRadixSort::SortPairsDescending(t.get(), tmp, hp0.get(), hp1.get(), H.get(), H2.get(),
                                                          (int)nh, 0, bits, s));
        Hs = H2.get();
        hp0.release();
        hp1.release();
    }

    // ---- symbolic pass ----
    DBuf<uint32_t> cursor(A, nxb, s), pend(A, nxb, s);
    DBuf<uint64_t> row_off(A, nrows + 1, s);
    AccArgs aa{};
    aa.row_job = row_job;
    aa.jobs = d_acc;
    aa.row_start = row_start;
    aa.row_xf = row_xf;
    aa.pos = pos;
    aa.cnt = cnt;
    aa.xprefix = xprefix;
    aa.xval = xvals;
    aa.yrank = rank;
    aa.yval = yvals;
    aa.ykeys = ykeys;
    aa.cols = cols;
    aa.work_counter = ctx->d_flag + 1;
    aa.cursor = cursor;
    aa.pend = pend;
    aa.row_nnz = row_nnz;
    aa.row_off = row_off;
    aa.row_xi = row_xi;
    aa.err = ctx->d_flag;
    aa.heavy_cap = ctx->heavy_window_cap;
    // Kept bitmaps take at most an eighth of the memory left (the rest is for
    // the output chunks): those of the heavy rows of at most kKeepBitsMax bits
    // per product if they fit, else of the dense rows (at most
    // kKeepBitsPerProduct), else none; the other heavy rows mark their windows.
    DBuf<uint32_t> hbm;
    DBuf<uint64_t> *bm_off = nullptr;
    if (keep_bm && nh) {
        const uint64_t room = A.available() / 8;
        if (bm_words_all && bm_words_all * 4 <= room)
            bm_off = &bm_off_all;
        else if (bm_words_dense && bm_words_dense * 4 <= room)
            bm_off = &bm_off_dense;
    }
    if (bm_off) {
        const uint64_t words = bm_off == &bm_off_all ? bm_words_all : bm_words_dense;
        hbm.reset(A, words, s);
        aa.hbm = hbm;
        aa.row_bmoff = *bm_off;
        aa.row_rb = row_rb;
        bst.kept_bitmap_bytes += words * 4;
    }
    bm_w_all.release();
    bm_w_dense.release();
    if (bm_off != &bm_off_all) bm_off_all.release();
    if (bm_off != &bm_off_dense) bm_off_dense.release();
    const int ghs = std::max(1, ctx->sm_count * heavy_blocks_per_sm(false));
    const int gh = std::max(1, ctx->sm_count * heavy_blocks_per_sm(true));
    const int gl = std::max(1, ctx->sm_count * light_blocks_per_sm());
    const int gs_grid = std::max(1, ctx->sm_count * stream_blocks_per_sm());
    {
        AccArgs b = aa;
        b.units = units;
        b.nunits = (uint32_t)nu;
        GS_CUDA(cudaMemsetAsync(ctx->d_flag + 1, 0, 4, s));
        launch_light(b, false, (int)std::min<uint64_t>(gl, std::max<uint64_t>(1, nu)), s);
        b.units = Hs;
        b.nunits = (uint32_t)nh;
        GS_CUDA(cudaMemsetAsync(ctx->d_flag + 1, 0, 4, s));
        launch_heavy(b, false, (int)std::min<uint64_t>(ghs, std::max<uint64_t>(1, nh)), s);
    }
    exclusive_scan_u32_to_u64(A, row_nnz, row_off, nrows, s);
    DBuf<JobOut> d_jo(A, g + 1, s);
    k_bjobout<<<grid_for(g + 1), kThreads, 0, s>>>(row_job, nrows, row_off, xprefix, hc, d_xoffs, g, d_jo);
    count_launch();
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaMemsetAsync(cnts.get() + 6, 0, 8, s));
    const UnitLists ul{units, nu, H, nh, SR, nsr};
    if (nu + nh + nsr) {
        k_unit_max<<<grid_for(nu + nh + nsr), kThreads, 0, s>>>(ul, row_off, cnts.get() + 6);
        count_launch();
        GS_CUDA(cudaGetLastError());
    }
    std::vector<JobOut> jo(g + 1);
    unsigned int herr = 0;
    uint64_t max_unit = 0;
    d2h(jo.data(), d_jo.get(), g + 1, s);
    d2h(&herr, ctx->d_flag, 1, s);
    d2h(&max_unit, cnts.get() + 6, 1, s);
    GS_CUDA(cudaStreamSynchronize(s));
    bst.bytes_d2h += sizeof(JobOut) * (g + 1) + 64 + 4 * g + 8;
    GS_REQUIRE(!(herr & 2u), GSPARC_EINTERNAL, "light unit over capacity");
    GS_REQUIRE(!(herr & 8u), GSPARC_EINTERNAL, "radix sort look-back gave up");
    const uint64_t ntot = jo[g].out_off;
    bst.nnz += ntot;
    mark(4);

    // per-job counts; jobs with an out-of-range index fail alone
    std::vector<uint64_t> job_nnz(g);
    for (int j = 0; j < g; ++j) {
        gsparc_job &J = *G[j]->job;
        gsparc_stats &st = J.stats;
        st.ir_nnz = nshards > 1 ? ir : jo[j + 1].ir_off - jo[j].ir_off;
        st.nnz = jo[j + 1].out_off - jo[j].out_off;
        st.rows = jo[j + 1].row0 - jo[j].row0;
        st.heavy_rows = jo[j + 1].heavy0 - jo[j].heavy0;
        job_nnz[j] = st.nnz;
        if (jerr[j] & 1u) {
            J.status = GSPARC_EINVAL;
            set_last_error("an index is not smaller than its mode size");
        }
    }

    // ---- chunk plan (memory-aware partitioning of the output) ----
    // Units (light units, heavy rows) tile the output in row order.  A chunk
    // takes the units that start in [k*C, (k+1)*C) of the output; with units
    // of at most max_unit outputs and C >= max_unit every chunk is non-empty
    // and holds fewer than C + max_unit <= cap outputs.
    // a chunk's output buffers (two when chunks overlap delivery) must fit
    // the memory left; the caller's max_chunk_nnz can only lower that
    uint64_t cap = std::min<uint64_t>(A.available() / 3 / 12, 1ull << 31);
    if (max_chunk_nnz) cap = std::min(cap, max_chunk_nnz);
    cap = std::max<uint64_t>(cap, 1);
    struct Chunk {
        uint64_t lu0, lu1;  // light units [lu0, lu1)
        uint64_t h0, h1;    // heavy rows [h0, h1) of the chunk-grouped heavy list
        uint64_t s0, s1;    // stream rows [s0, s1)
        uint64_t first, n;
    };
    std::vector<Chunk> chunks;
    DBuf<uint32_t> Hc;  // heavy rows grouped by chunk, largest first inside a chunk
    const uint32_t *Hchunk = Hs;
    // Jobs that complete one by one get chunk cuts at job boundaries after
    // kFirstCutProducts, 2x that, 4x that, ... products.
    const bool progressive = done_fn && g > 1 && ntot > 0;
    if (ntot <= cap && !progressive) {
        if (ntot || nu || nh || nsr) chunks.push_back({0, nu, 0, nh, 0, nsr, 0, ntot});
    } else {
        uint64_t C = std::max(cap > max_unit ? cap - max_unit : 1, std::max<uint64_t>(max_unit, 1));
        C = std::max<uint64_t>(C, (ntot + (1ull << 20) - 1) >> 20);  // at most 2^20 uniform chunks
        GS_REQUIRE(2 * 12 * (C + max_unit) <= A.available(), GSPARC_ENOMEM,
                   "one output row does not fit the HBM budget");
        std::vector<uint64_t> target{0};
        if (!progressive) {
            for (uint64_t t = C; t < ntot; t += C) target.push_back(t);
        } else {
            uint64_t acc = 0, thr = kFirstCutProducts;
            for (int j = 0; j < g; ++j) {
                const uint64_t end = jo[j + 1].out_off;
                while (end - target.back() > C) target.push_back(target.back() + C);
                acc += jo[j + 1].ir_off - jo[j].ir_off;
                if (acc >= thr && j + 1 < g && end > target.back() && end < ntot) {
                    target.push_back(end);
                    acc = 0;
                    thr *= 2;
                }
            }
        }
        target.push_back(ntot);
        const uint64_t K = target.size() - 1;
        const uint64_t M = nu + nh + nsr;
        DBuf<uint32_t> urow(A, M, s);
        DBuf<uint64_t> uoff(A, M, s);
        k_merge_starts<<<grid_for(M), kThreads, 0, s>>>(ul, row_off, urow, uoff);
        count_launch();
        GS_CUDA(cudaGetLastError());
        DBuf<uint64_t> d_target(A, K + 1, s);
        h2d(d_target.get(), target.data(), K + 1, s);
        DBuf<uint64_t> cinfo(A, kChunkInfo * (K + 1), s);
        k_chunk_bounds<<<grid_for(K + 1), kThreads, 0, s>>>(urow, uoff, M, d_target, K, ul, nrows, ntot, cinfo);
        count_launch();
        GS_CUDA(cudaGetLastError());
        std::vector<uint64_t> ci(kChunkInfo * (K + 1));
        d2h(ci.data(), cinfo.get(), kChunkInfo * (K + 1), s);
        if (nh) {
            // heavy rows grouped by chunk (stable in the largest-first order)
            DBuf<uint64_t> hk0(A, nh, s), hk1(A, nh, s);
            Hc.reset(A, nh, s);
            k_heavy_chunk_keys<<<grid_for(nh), kThreads, 0, s>>>(Hs, nh, row_prod, cinfo, K, hk0);
            count_launch();
            GS_CUDA(cudaGetLastError());
            const int bits = 44 + ceil_log2(K);
            size_t tmp = 0;
            GS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, hk0.get(), hk1.get(), Hs, Hc.get(), (int)nh, 0,
                                                    bits, s));
            DBuf<uint8_t> t(A, tmp, s);
            GS_CUDA(cub::DeviceRadixSort::SortPairs(t.get(), tmp, hk0.get(), hk1.get(), Hs, Hc.get(), (int)nh, 0,
                                                    bits, s));
            Hchunk = Hc.get();
        }
        GS_CUDA(cudaStreamSynchronize(s));
        bst.bytes_d2h += 8 * kChunkInfo * (K + 1);
        for (uint64_t k = 0; k < K; ++k) {
            const uint64_t *a = &ci[kChunkInfo * k], *b = &ci[kChunkInfo * (k + 1)];
            if (b[1] > a[1]) chunks.push_back({a[2], b[2], a[3], b[3], a[4], b[4], a[1], b[1] - a[1]});
        }
    }
    bst.chunks += chunks.size();

    if (keep) {
        // a plan keeps what the numeric pass needs and stops here
        keep->g = g;
        keep->nx = nx;
        keep->ny = ny;
        keep->ntot = ntot;
        keep->nu = nu;
        keep->nh = nh;
        keep->nsr = nsr;
        keep->gl = gl;
        keep->gh = gh;
        keep->gs_grid = gs_grid;
        keep->job_first.resize(g + 1);
        for (int j = 0; j <= g; ++j) keep->job_first[j] = jo[j].out_off;
        keep->jobs = G;
        keep->d_lx = std::move(d_lx);
        keep->d_ly = std::move(d_ly);
        keep->d_xoffs = std::move(d_xoffs);
        keep->d_yoffs = std::move(d_yoffs);
        keep->d_acc = std::move(d_acc);
        keep->rank = std::move(rank);
        keep->pos = std::move(pos);
        keep->cnt = std::move(cnt);
        keep->row_start = std::move(row_start);
        keep->units = std::move(units);
        keep->H = std::move(H);
        keep->H2 = std::move(H2);
        keep->SR = std::move(SR);
        keep->row_xi = std::move(row_xi);
        keep->cursor = std::move(cursor);
        keep->pend = std::move(pend);
        keep->cols = std::move(cols);
        keep->xprefix = std::move(xprefix);
        keep->row_xf = std::move(row_xf);
        keep->sprefix = std::move(sprefix);
        keep->row_off = std::move(row_off);
        keep->row_job = std::move(row_job);
        keep->Hc = std::move(Hc);
        if (bm_off) {  // kept bitmaps are part of what the numeric pass reads
            keep->hbm = std::move(hbm);
            keep->row_rb = std::move(row_rb);
            keep->row_bmoff = std::move(*bm_off);
        }
        keep->chunks.clear();
        for (auto &c : chunks) keep->chunks.push_back({c.lu0, c.lu1, c.h0, c.h1, c.s0, c.s1, c.first, c.n});
        keep->flags.reset(A, 4, s);
        GS_CUDA(cudaMemsetAsync(keep->flags.get(), 0, 16, s));
        keep->aa = aa;  // the moved buffers keep their device addresses
        keep->aa.err = keep->flags.get();
        keep->aa.work_counter = keep->flags.get() + 1;
        keep->aa.row_nnz = nullptr;  // the symbolic counts are not kept
        GS_CUDA(cudaStreamSynchronize(s));
        tm.lin += ms(0, 1);
        tm.sort += ms(1, 2);
        tm.match += ms(2, 3);
        tm.plan += ms(3, 4);
        tm.total += ms(0, 4);
        return;
    }

    // ---- numeric pass, chunk by chunk, double-buffered against delivery ----
    const int nbuf = chunks.size() > 1 ? 2 : 1;
    uint64_t bufn = 0;
    for (auto &c : chunks) bufn = std::max(bufn, c.n);
    DBuf<uint64_t> out_k[2];
    DBuf<float> out_v[2];
    DBuf<uint64_t> out_k2[2];  // 128-bit keys of jobs whose sink asks for two key words
    bool any_kw2 = false;
    for (Job *q : G) any_kw2 |= q->key_words == 2;
    for (int i = 0; i < nbuf; ++i) {
        out_k[i].reset(A, std::max<uint64_t>(bufn, 1), s);
        out_v[i].reset(A, std::max<uint64_t>(bufn, 1), s);
        if (any_kw2) out_k2[i].reset(A, 2 * std::max<uint64_t>(bufn, 1), s);
    }
    std::vector<cudaEvent_t> kev(2 * chunks.size(), nullptr);
    for (auto &e : kev) GS_CUDA(cudaEventCreate(&e));
    cudaStream_t s2 = ctx->copy_stream;

    // FP64 verification of every chunk before delivery (off unless asked for)
    const bool verify = ctx->verify_budget != 0 && nrows > 0 && ntot > 0;
    VerifyState vs;
    DBuf<VerifyEntry> v_list;
    DBuf<unsigned long long> v_cnt;
    DBuf<double> v_acc;
    DBuf<VerifyOut> v_out;
    if (verify) {
        v_list.reset(A, nrows, s);
        v_cnt.reset(A, 2, s);
        v_out.reset(A, g, s);
        GS_CUDA(cudaMemsetAsync(v_out.get(), 0, sizeof(VerifyOut) * g, s));
        uint64_t cap = std::min<uint64_t>(bufn, 1ull << 25);
        cap = std::max<uint64_t>(1, std::min<uint64_t>(cap, A.available() / 2 / sizeof(double)));
        v_acc.reset(A, cap, s);
        vs.list = v_list.get();
        vs.cnt = v_cnt.get();
        vs.acc = v_acc.get();
        vs.acc_cap = cap;
        vs.out = v_out.get();
        vs.threshold = verify_threshold(ctx->verify_budget, ir);
        vs.salt = 0x5eed5eed5eedull;
        GS_CUDA(cudaStreamSynchronize(s));
    }
    double t_out = 0;
    std::vector<uint64_t> job_first(g + 1);
    for (int j = 0; j <= g; ++j) job_first[j] = jo[j].out_off;
    int next_done = 0;  // jobs before it were reported complete

    // Consecutive chunks go to two streams, so the next chunk's kernels start
    // on SMs the current chunk's kernels leave idle at their tails.  Each
    // stream has its own work counter; the buffer a chunk writes was delivered
    // (host-synchronously) before it is enqueued.  A device sink may enqueue
    // its own copies of a chunk on the engine's stream, which only orders them
    // before later chunks on that stream: groups with one stay on one stream.
    bool device_sink = false;
    for (Job *q : G) device_sink |= q->job->sink.kind == GSPARC_SINK_DEVICE;
    cudaStream_t sa = ctx->alt_stream && !device_sink && chunks.size() > 1 ? ctx->alt_stream : s;
    cudaEvent_t ev_ready = nullptr, ev_alt = nullptr;
    GS_CUDA(cudaEventCreateWithFlags(&ev_ready, cudaEventDisableTiming));
    GS_CUDA(cudaEventCreateWithFlags(&ev_alt, cudaEventDisableTiming));
    GS_CUDA(cudaEventRecord(ev_ready, s));
    GS_CUDA(cudaStreamWaitEvent(sa, ev_ready, 0));
    auto enqueue = [&](size_t ci) {
        const Chunk &c = chunks[ci];
        const int bi = (int)(ci % nbuf);
        const cudaStream_t sc = (ci & 1) ? sa : s;
        unsigned int *counter = ctx->d_flag + ((ci & 1) && sa != s ? 5 : 1);
        AccArgs b = aa;
        b.work_counter = counter;
        b.chunk_base = c.first;
        b.out_keys = out_k[bi];
        b.out_vals = out_v[bi];
        b.out_cap = c.n;
        b.units = units.get() + 2 * c.lu0;
        b.nunits = (uint32_t)(c.lu1 - c.lu0);
        GS_CUDA(cudaMemsetAsync(counter, 0, 4, sc));
        GS_CUDA(cudaEventRecord(kev[2 * ci], sc));
        launch_light(b, true, (int)std::min<uint64_t>(gl, std::max<uint64_t>(1, b.nunits)), sc);
        b.units = Hchunk + c.h0;
        b.nunits = (uint32_t)(c.h1 - c.h0);
        GS_CUDA(cudaMemsetAsync(counter, 0, 4, sc));
        launch_heavy(b, true, (int)std::min<uint64_t>(gh, std::max<uint64_t>(1, b.nunits)), sc);
        b.units = SR.get() + c.s0;
        b.nunits = (uint32_t)(c.s1 - c.s0);
        b.sprefix = sprefix.get() + c.s0;
        launch_stream(b, gs_grid, sc);
        GS_CUDA(cudaEventRecord(kev[2 * ci + 1], sc));
    };
    auto deliver = [&](size_t ci) {
        const Chunk &c = chunks[ci];
        const int bi = (int)(ci % nbuf);
        auto t0 = std::chrono::steady_clock::now();
        GS_CUDA(cudaStreamWaitEvent(s2, kev[2 * ci + 1], 0));
        GS_CUDA(cudaEventSynchronize(kev[2 * ci + 1]));
        const uint64_t c0 = c.first, c1 = c.first + c.n;
        if (verify) {
            // before any wide-key remap: the chunk still holds the engine's keys
            verify_chunk(aa, vs, nrows, c0, c1, out_k[bi].get(), out_v[bi].get(), s2);
            GS_CUDA(cudaStreamSynchronize(s2));  // the buffer is rewritten two chunks on
        }
        // jobs overlapping [c0, c1)
        int j = (int)(std::upper_bound(job_first.begin(), job_first.end(), c0) - job_first.begin()) - 1;
        for (j = std::max(j, 0); j < g && job_first[j] < c1; ++j) {
            gsparc_job &J = *G[j]->job;
            const uint64_t a0 = std::max(c0, job_first[j]), a1 = std::min(c1, job_first[j + 1]);
            if (a1 <= a0 || J.status != GSPARC_OK) continue;
            if (G[j]->wide && G[j]->key_words == 2) {
                // relabeled output keys back to x_f << Y_nfbits | y_f in 128 bits
                uint64_t *k2 = out_k2[bi].get() + 2 * (a0 - c0);
                wide_remap_keys128(*G[j]->wide, out_k[bi].get() + (a0 - c0), k2, a1 - a0, s2);
                GS_CUDA(cudaStreamSynchronize(s2));
                deliver_slice(J.sink, k2, out_v[bi].get() + (a0 - c0), a1 - a0, a0 - job_first[j], job_nnz[j],
                              s2, J.stats, bst.bytes_d2h, 2);
                continue;
            }
            if (G[j]->wide) {
                // relabeled output keys back to x_f << Y_nfbits | y_f
                wide_remap_keys(*G[j]->wide, out_k[bi].get() + (a0 - c0), a1 - a0, s2);
                GS_CUDA(cudaStreamSynchronize(s2));
            }
            deliver_slice(J.sink, out_k[bi].get() + (a0 - c0), out_v[bi].get() + (a0 - c0), a1 - a0,
                          a0 - job_first[j], job_nnz[j], s2, J.stats, bst.bytes_d2h);
        }
        t_out += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        // jobs whose whole output is now delivered are complete (unless a
        // device-side check of the chunk failed)
        if (done_fn && next_done < g && job_first[next_done + 1] <= c1) {
            unsigned int e = 0;
            d2h(&e, ctx->d_flag, 1, s2);
            GS_CUDA(cudaStreamSynchronize(s2));
            GS_REQUIRE(!(e & 6u), GSPARC_EINTERNAL, "numeric pass failed a device-side check");
        }
        if (done_fn)
            for (; next_done < g && job_first[next_done + 1] <= c1; ++next_done) {
                Job *q = G[next_done];
                if (!q->done && q->job->status == GSPARC_OK) {
                    q->done = true;
                    (*done_fn)(q->job);
                }
            }
    };
    try {
        for (size_t ci = 0; ci < chunks.size(); ++ci) {
            enqueue(ci);
            if (ci >= 1) deliver(ci - 1);
        }
        if (!chunks.empty()) deliver(chunks.size() - 1);
    } catch (...) {
        cudaStreamSynchronize(s2);
        cudaStreamSynchronize(sa);
        cudaStreamSynchronize(s);
        for (auto e : kev) cudaEventDestroy(e);
        cudaEventDestroy(ev_ready);
        cudaEventDestroy(ev_alt);
        throw;
    }
    GS_CUDA(cudaEventRecord(ev_alt, sa));
    GS_CUDA(cudaStreamWaitEvent(s, ev_alt, 0));
    cudaEventDestroy(ev_ready);
    cudaEventDestroy(ev_alt);
    if (verify) {
        std::vector<VerifyOut> vo(g);
        d2h(vo.data(), v_out.get(), g, s2);
        GS_CUDA(cudaStreamSynchronize(s2));
        for (int j = 0; j < g; ++j) {
            verify_fill_stats(vo[j], G[j]->job->stats);
            verify_fill_stats(vo[j], bst);
        }
    }
    mark(5);
    unsigned int hflags[4] = {0, 0, 0, 0};
    d2h(hflags, ctx->d_flag, 4, s);
    GS_CUDA(cudaStreamSynchronize(s));
    bst.heavy_windows += hflags[2];
    GS_REQUIRE(!(hflags[0] & 2u), GSPARC_EINTERNAL, "light unit over capacity");
    GS_REQUIRE(!(hflags[0] & 4u), GSPARC_EINTERNAL, "numeric pass wrote past its chunk (symbolic count mismatch)");
    tm.lin += ms(0, 1);
    tm.sort += ms(1, 2);
    tm.match += ms(2, 3);
    tm.plan += ms(3, 4);
    tm.contract += ms(4, 5);
    tm.total += ms(0, 5);
    tm.out += t_out;
    // numeric kernel time: first chunk's start to the last chunk's end (chunks
    // on the two streams overlap)
    {
        float span = 0.f;
        for (size_t i = 0; i + 1 < kev.size(); i += 2) {
            float t = 0.f;
            GS_CUDA(cudaEventElapsedTime(&t, kev[0], kev[i + 1]));
            span = std::max(span, t);
        }
        tm.numeric += span;
    }
    for (auto e : kev) cudaEventDestroy(e);
}

}  // namespace

// Checks every job on its own (a bad job fails alone: its status says why)
// and prepares the ones that pass: layouts, relabeling of keys over 64 bits.
void validate_jobs(gsparc_ctx *ctx, gsparc_job *jobs, int njobs, cudaStream_t s, std::vector<Job> &js,
                   gsparc_stats &bst) {
    js.reserve(njobs);
    for (int i = 0; i < njobs; ++i) {
        gsparc_job &J = jobs[i];
        std::memset(&J.stats, 0, sizeof(J.stats));
        J.status = GSPARC_OK;
        try {
            GS_REQUIRE(J.x && J.y, GSPARC_EINVAL, "null tensor");
            GS_REQUIRE(J.ncmodes >= 1 && J.ncmodes <= kMaxOrder && J.cx && J.cy, GSPARC_EINVAL, "bad contract modes");
            GS_REQUIRE(J.accum >= -1 && J.accum <= 1, GSPARC_EINVAL, "accum must be -1, 0 or 1");
            const gsparc_sink &k = J.sink;
            GS_REQUIRE(k.kind >= GSPARC_SINK_DISCARD && k.kind <= GSPARC_SINK_HOST, GSPARC_EINVAL, "bad sink kind");
            GS_REQUIRE(k.kind != GSPARC_SINK_HOST || (k.host_keys && k.host_vals && k.host_capacity), GSPARC_EINVAL,
                       "host sink needs host_keys, host_vals and host_capacity");
            GS_REQUIRE(k.kind != GSPARC_SINK_DEVICE || k.on_chunk, GSPARC_EINVAL, "device sink needs on_chunk");
            Job q;
            q.job = &J;
            q.tx = J.x;
            q.ty = J.y;
            q.LX = make_layout(J.x->order, J.x->dims, J.ncmodes, J.cx);
            q.LY = make_layout(J.y->order, J.y->dims, J.ncmodes, J.cy);
            GS_REQUIRE(J.x->order > J.ncmodes && J.y->order > J.ncmodes, GSPARC_EUNSUPPORTED,
                       "every operand needs at least one free mode");
            for (int m = 0; m < J.ncmodes; ++m)
                GS_REQUIRE(q.LX.bits[J.cx[m]] == q.LY.bits[J.cy[m]], GSPARC_EINVAL,
                           "contract modes of X and Y have different bit widths (mode sizes differ)");
            // a discarded output of more than 64 bits needs no key words at all:
            // run it on the 128-bit path and deliver nothing
            q.key_words = k.key_words ? k.key_words
                                      : (k.kind == GSPARC_SINK_DISCARD && q.LX.nfbits + q.LY.nfbits > 64 ? 2 : 1);
            GS_REQUIRE(q.key_words == 1 || q.key_words == 2, GSPARC_EINVAL, "sink key_words must be 0, 1 or 2");
            GS_REQUIRE(q.LX.nfbits + q.LY.nfbits <= 64 * q.key_words, GSPARC_EUNSUPPORTED,
                       "output key wider than 64 bits (X free bits + Y free bits > 64): set sink.key_words = 2");
            GS_REQUIRE(J.x->nnz < kMaxGroupNnz && J.y->nnz < kMaxGroupNnz, GSPARC_EUNSUPPORTED,
                       "operand with more than 2^31 nonzeros");
            const Layout LX0 = q.LX, LY0 = q.LY;
            if (q.LX.nbits() > 64 || q.LY.nbits() > 64 || q.key_words == 2) {
                // the reference's 128-bit key path: relabel onto 64-bit keys (128-bit
                // output keys are built from the rank tables at delivery)
                q.wide = make_wide(ctx->arena, J.x, q.LX, J.y, q.LY, s);
                q.tx = &q.wide->x2;
                q.ty = &q.wide->y2;
                q.LX = make_layout(2, q.tx->dims, 1, q.wide->cx2);
                q.LY = make_layout(2, q.ty->dims, 1, q.wide->cy2);
            }
            q.light_max = J.accum == GSPARC_ACCUM_DENSE ? 0 : (ctx->light_row_max ? ctx->light_row_max : kLightRowMax);
            q.width = std::max(q.LX.nbits(), q.LY.nbits());
            J.stats.nnz_x = J.x->nnz;
            J.stats.nnz_y = J.y->nnz;
            J.stats.nbits_x = LX0.nbits();
            J.stats.nbits_y = LY0.nbits();
            J.stats.ncbits = LX0.ncbits;
            J.stats.nfbits_x = LX0.nfbits;
            J.stats.nfbits_y = LY0.nfbits;
            J.stats.accumulator = J.accum;
            bst.nnz_x += J.x->nnz;
            bst.nnz_y += J.y->nnz;
            js.push_back(q);
        } catch (const Error &e) {
            J.status = e.st;
            set_last_error(e.msg);
        }
    }

}

// Groups of jobs whose keys, with the job id above them, fit 64 bits: widest
// keys first; a group of n jobs needs ceil(log2 n) id bits.
std::vector<std::vector<Job *>> make_groups(std::vector<Job> &js) {
    std::vector<Job *> order;
    for (auto &q : js) order.push_back(&q);
    std::stable_sort(order.begin(), order.end(), [](const Job *a, const Job *b) { return a->width > b->width; });
    std::vector<std::vector<Job *>> groups;
    {
        size_t i = 0;
        while (i < order.size()) {
            std::vector<Job *> G;
            uint64_t sx = 0, sy = 0;
            const int w = order[i]->width;  // widest of the group (sorted descending)
            while (i < order.size()) {
                Job *q = order[i];
                const uint64_t n1 = G.size() + 1;
                if (!G.empty() && (w + ceil_log2(n1) > 64 || (int)n1 > kMaxGroupJobs ||
                                   sx + q->job->x->nnz > kMaxGroupNnz || sy + q->job->y->nnz > kMaxGroupNnz))
                    break;
                G.push_back(q);
                sx += q->job->x->nnz;
                sy += q->job->y->nnz;
                ++i;
            }
            groups.push_back(std::move(G));
        }
    }

    return groups;
}

void sptc_batch(gsparc_ctx *ctx, gsparc_job *jobs, int njobs, uint64_t max_chunk_nnz, gsparc_stats *st_out,
                cudaStream_t s, int shard, int nshards, const JobDoneFn *done_fn) {
    GS_REQUIRE(ctx, GSPARC_EINVAL, "null context");
    GS_REQUIRE(njobs >= 0 && (njobs == 0 || jobs), GSPARC_EINVAL, "bad job array");
    GS_REQUIRE(nshards >= 1 && shard >= 0 && shard < nshards, GSPARC_EINVAL, "bad shard");
    GS_REQUIRE(nshards == 1 || njobs == 1, GSPARC_EINVAL, "row shards apply to a single contraction");
    gsparc_stats bst;
    std::memset(&bst, 0, sizeof(bst));
    const uint64_t launches0 = launch_count();

    std::vector<Job> js;
    validate_jobs(ctx, jobs, njobs, s, js, bst);
    std::vector<std::vector<Job *>> groups = make_groups(js);

    // completion reports: at most one per job, early ones from run_group
    std::vector<char> reported(njobs, 0);
    JobDoneFn report;
    const JobDoneFn *report_fn = nullptr;
    if (done_fn) {
        report = [&](gsparc_job *J) {
            reported[J - jobs] = 1;
            (*done_fn)(J);
        };
        report_fn = &report;
    }

    Times tm;
    for (auto &G : groups) {
        try {
            run_group(ctx, G, max_chunk_nnz, shard, nshards, tm, bst, s, report_fn);
        } catch (const Error &e) {
            // the group's jobs fail together (except those already complete);
            // later groups still run
            for (Job *q : G)
                if (!q->done && q->job->status == GSPARC_OK) q->job->status = e.st;
            set_last_error(e.msg);
            cudaStreamSynchronize(s);
        }
    }

    bst.t_linearize_ms = tm.lin;
    bst.t_sort_ms = tm.sort;
    bst.t_match_ms = tm.match;
    bst.t_plan_ms = tm.plan;
    bst.t_contract_ms = tm.contract;
    bst.t_output_ms = tm.out;
    bst.t_total_ms = tm.total;
    bst.t_numeric_kernel_ms = tm.numeric;
    bst.kernel_launches = launch_count() - launches0;
    bst.accumulator = GSPARC_ACCUM_AUTO;
    for (int i = 0; i < njobs; ++i) {
        gsparc_stats &st = jobs[i].stats;
        st.t_linearize_ms = tm.lin;
        st.t_sort_ms = tm.sort;
        st.t_match_ms = tm.match;
        st.t_plan_ms = tm.plan;
        st.t_contract_ms = tm.contract;
        st.t_output_ms = tm.out;
        st.t_total_ms = tm.total;
    }
    if (st_out) *st_out = bst;
    if (done_fn)
        for (int i = 0; i < njobs; ++i)
            if (!reported[i]) (*done_fn)(&jobs[i]);
    for (int i = 0; i < njobs; ++i)
        if (jobs[i].status != GSPARC_OK) {
            if (njobs == 1) fail(jobs[i].status, last_error());
            fail(jobs[i].status, std::string("job ") + std::to_string(i) + " failed (" +
                                     gsparc_status_string(jobs[i].status) + "); last message: " + last_error());
        }
}

}  // namespace gs

// ---- plans: the coordinate-only work done once, the numeric pass replayed ----

struct gsparc_plan {
    gsparc_ctx *ctx = nullptr;
    std::vector<gsparc_job> jobs;  // copies of the caller's jobs (modes copied too)
    std::vector<std::vector<int>> modes;
    std::vector<gs::Job> js;
    std::vector<std::unique_ptr<gs::GroupPlan>> groups;
    std::vector<uint64_t> group_off;               // first output of each group
    std::vector<std::pair<int, int>> chunk_of;     // plan chunk -> (group, group chunk)
    std::vector<uint64_t> job_first, job_nnz;      // per caller job
    uint64_t total = 0;
};

namespace gs {

void plan_create(gsparc_ctx *ctx, const gsparc_job *jobs, int njobs, uint64_t max_chunk_nnz, gsparc_plan **out,
                 uint64_t *total, cudaStream_t s) {
    GS_REQUIRE(ctx && out && njobs >= 1 && jobs, GSPARC_EINVAL, "bad argument");
    *out = nullptr;
    auto P = std::make_unique<gsparc_plan>();
    P->ctx = ctx;
    P->jobs.assign(jobs, jobs + njobs);
    P->modes.resize(njobs);
    for (int i = 0; i < njobs; ++i) {
        gsparc_job &J = P->jobs[i];
        GS_REQUIRE(J.ncmodes >= 1 && J.ncmodes <= kMaxOrder && J.cx && J.cy, GSPARC_EINVAL, "bad contract modes");
        auto &m = P->modes[i];
        m.assign(J.cx, J.cx + J.ncmodes);
        m.insert(m.end(), J.cy, J.cy + J.ncmodes);
        J.cx = m.data();
        J.cy = m.data() + J.ncmodes;
        J.sink = gsparc_sink{};
        J.sink.kind = GSPARC_SINK_DISCARD;
    }
    gsparc_stats bst;
    std::memset(&bst, 0, sizeof(bst));
    validate_jobs(ctx, P->jobs.data(), njobs, s, P->js, bst);
    for (int i = 0; i < njobs; ++i)
        if (P->jobs[i].status != GSPARC_OK)
            fail(P->jobs[i].status, "job " + std::to_string(i) + ": " + last_error());
    std::vector<std::vector<Job *>> groups = make_groups(P->js);
    Times tm;
    P->job_first.assign(njobs, 0);
    P->job_nnz.assign(njobs, 0);
    for (auto &G : groups) {
        auto gp = std::make_unique<GroupPlan>();
        run_group(ctx, G, max_chunk_nnz, 0, 1, tm, bst, s, nullptr, gp.get());
        for (Job *q : G)
            if (q->job->status != GSPARC_OK) fail(q->job->status, last_error());
        P->group_off.push_back(P->total);
        for (size_t c = 0; c < gp->chunks.size(); ++c) P->chunk_of.push_back({(int)P->groups.size(), (int)c});
        for (int j = 0; j < gp->g; ++j) {
            const int i = (int)(gp->jobs[j]->job - P->jobs.data());
            P->job_first[i] = P->total + gp->job_first[j];
            P->job_nnz[i] = gp->job_first[j + 1] - gp->job_first[j];
        }
        P->total += gp->ntot;
        P->groups.push_back(std::move(gp));
    }
    if (total) *total = P->total;
    *out = P.release();
}

// One chunk of a plan's output into keys/vals (first = the chunk's first
// output).  Launches only: memsets, value gathers, the numeric kernels and
// (for jobs with keys over 64 bits) the output key map.
void plan_execute(gsparc_plan *P, uint64_t chunk, uint64_t *keys, float *vals, uint64_t capacity,
                  cudaStream_t s) {
    GS_REQUIRE(P && chunk < P->chunk_of.size(), GSPARC_EINVAL, "no such chunk");
    const int gi = P->chunk_of[chunk].first, ci = P->chunk_of[chunk].second;
    GroupPlan &gp = *P->groups[gi];
    const GroupPlan::Chunk &c = gp.chunks[ci];
    GS_REQUIRE(c.n <= capacity && (c.n == 0 || (keys && vals)), GSPARC_EINVAL,
               "output arrays smaller than the chunk (gsparc_plan_chunk gives its size)");
    AccArgs b = gp.aa;
    b.chunk_base = c.first;
    b.out_keys = keys;
    b.out_vals = vals;
    b.out_cap = c.n;
    b.units = gp.units.get() + 2 * c.lu0;
    b.nunits = (uint32_t)(c.lu1 - c.lu0);
    GS_CUDA(cudaMemsetAsync(gp.flags.get() + 1, 0, 4, s));
    launch_light(b, true, (int)std::min<uint64_t>(gp.gl, std::max<uint64_t>(1, b.nunits)), s);
    b.units = gp.heavy_list() + c.h0;
    b.nunits = (uint32_t)(c.h1 - c.h0);
    GS_CUDA(cudaMemsetAsync(gp.flags.get() + 1, 0, 4, s));
    launch_heavy(b, true, (int)std::min<uint64_t>(gp.gh, std::max<uint64_t>(1, b.nunits)), s);
    b.units = gp.SR.get() + c.s0;
    b.nunits = (uint32_t)(c.s1 - c.s0);
    b.sprefix = gp.sprefix.get() + c.s0;
    launch_stream(b, gp.gs_grid, s);
    for (int j = 0; j < gp.g; ++j) {
        if (!gp.jobs[j]->wide) continue;
        const uint64_t a0 = std::max(c.first, gp.job_first[j]), a1 = std::min(c.first + c.n, gp.job_first[j + 1]);
        if (a1 > a0) wide_remap_keys(*gp.jobs[j]->wide, keys + (a0 - c.first), a1 - a0, s);
    }
}

// Fetches the operands' current values into the plan's sorted value arrays.
void plan_refresh(gsparc_plan *P, cudaStream_t s) {
    GS_REQUIRE(P, GSPARC_EINVAL, "null plan");
    for (auto &g : P->groups) {
        GroupPlan &gp = *g;
        if (gp.nx) {
            k_bvals<<<grid_for(gp.nx), kThreads, 0, s>>>(gp.d_lx, gp.d_xoffs, gp.g, gp.nx, gp.xperm, gp.xvals);
            count_launch();
        }
        if (gp.ny) {
            k_bvals<<<grid_for(gp.ny), kThreads, 0, s>>>(gp.d_ly, gp.d_yoffs, gp.g, gp.ny, gp.yperm, gp.yvals);
            count_launch();
        }
        GS_CUDA(cudaGetLastError());
    }
}

// Waits for `s`, reads and clears the device-side error words of every group.
void plan_check(gsparc_plan *P, cudaStream_t s) {
    GS_REQUIRE(P, GSPARC_EINVAL, "null plan");
    for (auto &gp : P->groups) {
        unsigned int f = 0;
        d2h(&f, gp->flags.get(), 1, s);
        GS_CUDA(cudaMemsetAsync(gp->flags.get(), 0, 4, s));
        GS_CUDA(cudaStreamSynchronize(s));
        GS_REQUIRE(!(f & 2u), GSPARC_EINTERNAL, "light unit over capacity");
        GS_REQUIRE(!(f & 4u), GSPARC_EINTERNAL, "numeric pass wrote past its chunk");
    }
}

void plan_destroy(gsparc_plan *P) {
    if (!P) return;
    const int dev = P->ctx->device;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
    cudaDeviceSynchronize();  // the buffers may still be read by executions in flight
    delete P;
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
}

uint64_t plan_nchunks(const gsparc_plan *P) { return P->chunk_of.size(); }

void plan_chunk(const gsparc_plan *P, uint64_t k, uint64_t *first, uint64_t *nnz) {
    GS_REQUIRE(k < P->chunk_of.size(), GSPARC_EINVAL, "no such chunk");
    const GroupPlan &gp = *P->groups[P->chunk_of[k].first];
    const GroupPlan::Chunk &c = gp.chunks[P->chunk_of[k].second];
    if (first) *first = P->group_off[P->chunk_of[k].first] + c.first;
    if (nnz) *nnz = c.n;
}

void plan_job_output(const gsparc_plan *P, int job, uint64_t *first, uint64_t *nnz) {
    GS_REQUIRE(job >= 0 && job < (int)P->job_first.size(), GSPARC_EINVAL, "no such job");
    if (first) *first = P->job_first[job];
    if (nnz) *nnz = P->job_nnz[job];
}

}  // namespace gs
