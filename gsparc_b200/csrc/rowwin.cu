// rowwin.cu -- windowed accumulation of heavy output rows.
//
// One CTA owns one output row (all products of one X free index).  The row's
// products are the matched Y runs of its X nonzeros; every run is sorted by
// column rank.  The CTA sweeps the column-rank axis in windows [R0, R0+rw):
//
//  A. each run's part inside the window is found by a search from the run's
//     cursor (a warp per run with a 32-way fan-out when runs are few, a thread
//     per run when they are many); parts that are empty are dropped;
//  B. a block scan flattens the remaining parts into one index space, so every
//     thread gets the same share of entries however uneven the runs are; a
//     warp maps its 32 entries to parts with a 5-step shuffle search;
//  1. touched columns are marked in a shared bitmap;
//  2. a word-wise prefix of the bitmap turns each touched column into a dense
//     output slot (slot = prefix[word] + popcount of lower bits), so the output
//     of the window is already in column order;
//  3. (numeric) every product is added into its slot with compensated FP32:
//     the hardware add returns the old value, from which TwoSum rebuilds the
//     exact rounding error of that add; errors (and the product's own fma
//     error) accumulate in a second word;
//  4. (numeric) a slot -> column table is built from the bitmap (a thread per
//     word), then every warp writes 32 consecutive slots per step.
//
// The window width adapts to the row's density: each window aims at fifteen
// sixteenths of kHeavyCap outputs at the density of the window before it (at
// most 4x wider per window); a window that overflows is cut at the
// kHeavyCap-th touched column and the rest is taken by the next window.  The
// symbolic pass (steps A, B and 1 on RW_SYM-wide windows: it keeps neither
// accumulators nor the word prefix) marks with atomics whose result it does not
// wait for and counts each window's columns by a popcount of its words, read
// anyway to store and clear them.
//
// Kept bitmaps: for the heavy rows whose column bitmap over their rank span
// costs at most kKeepBitsMax bits per product (kKeepBitsPerProduct when memory
// is short), the symbolic pass also stores the bitmap of every window in HBM
// (windows aligned to the bitmap's words, the words of skipped ranges
// cleared).  The numeric pass then marks nothing: each window copies its words
// to shared memory (cp.async, the next window's words prefetched into L2
// meanwhile), takes the word prefix, ends exactly where the kHeavyCap-th
// column is passed, and finds every run's part with that end, so windows are
// full and no product is read twice; the next window starts at the row's next
// column, so gaps are skipped.
#include "blockops.cuh"
#include "kernels.cuh"

namespace gs {

namespace {
using namespace dev;

constexpr int T = kHeavyThreads;
constexpr int NWARPS = T / 32;
constexpr int RW = kHeavyRW;
constexpr int NWORDS = RW / 32;
constexpr int CAP = kHeavyCap;
constexpr int MAXR = kHeavyMaxRuns;
// Numeric pass, words of the bitmap region: the bitmap (NWORDS words), then
// the word prefix (16-bit for a kept row's window, whose prefixes past the
// capacity are clamped, 32-bit for a marked window); step 4 then reuses the
// region as the slot -> column table (CAP words).
constexpr int AW = (2 * NWORDS > CAP ? 2 * NWORDS : CAP);
static_assert(CAP < 65535, "kept windows hold 16-bit prefixes");
constexpr int WPT_MAX = (NWORDS + T - 1) / T;
constexpr int RW_SYM = 262144;              // symbolic windows: no accumulators or word prefix kept
constexpr int NWORDS_SYM = RW_SYM / 32;
constexpr uint32_t INF = 0xffffffffu;
constexpr uint32_t FULL = 0xffffffffu;
static_assert(MAXR <= 2 * T, "run batch is scanned two per thread");

// First index in [p, e) whose rank is >= lim (e if none); *first_rank gets
// that entry's rank (INF if none).  All lanes of the warp call it with the
// same arguments.  Exponential search with a 32-way fan-out per step: the
// stride grows 32x while the window still holds the next 32 probes, then
// narrows 32x per step, so a part of length L costs about 2*log32(L) loads.
__device__ __forceinline__ uint32_t warp_gallop(const uint32_t *__restrict__ rank, uint32_t p, uint32_t e,
                                                uint32_t lim, uint32_t *first_rank) {
    const uint32_t lane = threadIdx.x & 31;
    uint64_t base = p;
    uint64_t s = 32;
    for (;;) {
        const uint64_t q = base + s * (lane + 1) - 1;
        const uint32_t r = q < e ? rank[q] : INF;
        const uint32_t bal = __ballot_sync(FULL, r >= lim);
        if (bal) {
            base += s * (uint64_t)(__ffs(bal) - 1);
            break;
        }
        base += s * 32;
        if (s < (1ull << 25)) s <<= 5;
    }
    // entries [p, base) are < lim and the entry at base + s - 1 is not
    uint32_t fr = INF;
    while (s > 1) {
        s >>= 5;
        const uint64_t q = base + s * (lane + 1) - 1;
        const uint32_t r = q < e ? rank[q] : INF;
        const uint32_t bal = __ballot_sync(FULL, r >= lim);
        const int f = __ffs(bal) - 1;
        base += s * (uint64_t)f;
        if (s == 1) fr = __shfl_sync(FULL, r, f);
    }
    *first_rank = fr;
    return base < e ? (uint32_t)base : e;
}

// Same search done by one thread: probe p, p+1, p+3, p+7, ... until a rank
// >= lim (or e), then bisect the last gap.  Cheap when the part is short.
__device__ __forceinline__ uint32_t thread_gallop(const uint32_t *__restrict__ rank, uint32_t p, uint32_t e,
                                                  uint32_t lim, uint32_t *first_rank) {
    uint32_t r = rank[p];
    if (r >= lim) {
        *first_rank = r;
        return p;
    }
    uint32_t lo = p, hi = e, fr = INF, step = 1;  // rank[lo] < lim; hi == e or rank[hi] >= lim
    for (;;) {
        const uint64_t q = (uint64_t)lo + step;
        if (q >= e) break;
        const uint32_t rq = rank[q];
        if (rq >= lim) {
            hi = (uint32_t)q;
            fr = rq;
            break;
        }
        lo = (uint32_t)q;
        step <<= 1;
    }
    while (hi - lo > 1) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        const uint32_t rm = rank[mid];
        if (rm >= lim) {
            hi = mid;
            fr = rm;
        } else {
            lo = mid;
        }
    }
    *first_rank = fr;
    return hi;
}

// In-place exclusive scan of v[0..n) (n <= 2*T); v[n] gets the total.
__device__ __forceinline__ void block_scan_inplace(uint32_t *v, uint32_t n, uint32_t *s_tmp) {
    const uint32_t i0 = 2u * threadIdx.x, i1 = i0 + 1u;
    const uint32_t a = i0 < n ? v[i0] : 0u;
    const uint32_t b = i1 < n ? v[i1] : 0u;
    uint32_t total;
    const uint32_t ex = block_excl_scan_u32<T>(a + b, s_tmp, &total);
    if (i0 < n) v[i0] = ex;
    if (i1 < n) v[i1] = ex + a;
    if (threadIdx.x == 0) v[n] = total;
    __syncthreads();
}

// The parts of runs [0, nb) sit uncompacted in the seg arrays (seg_off holds
// lengths).  Drop empty parts, then turn lengths into an exclusive prefix with
// the total at seg_off[ns].  Returns ns, the number of non-empty parts.
__device__ __forceinline__ uint32_t compact_parts(uint32_t nb, uint32_t *seg_start, uint32_t *seg_off,
                                                  uint32_t *seg_run, uint32_t *seg_cut, uint32_t *s_tmp) {
    if (nb <= 32u) {
        // at most 32 parts: warp 0 alone (a ballot and one shuffle scan)
        if (threadIdx.x < 32) {
            const uint32_t k = threadIdx.x;
            uint32_t st = 0, len = 0, rn = 0, ct = 0;
            if (k < nb) { st = seg_start[k]; len = seg_off[k]; rn = seg_run[k]; ct = seg_cut[k]; }
            const uint32_t bal = __ballot_sync(FULL, len != 0u);
            uint32_t x = len;  // empty parts (and lanes past nb) add nothing
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, x, o);
                if (k >= (uint32_t)o) x += y;
            }
            __syncwarp();  // every lane has read its part before any is overwritten
            if (len) {
                const uint32_t at = __popc(bal & ((1u << k) - 1u));
                seg_start[at] = st;
                seg_off[at] = x - len;
                seg_run[at] = rn;
                seg_cut[at] = ct;
            }
            if (k == 31) {
                seg_off[__popc(bal)] = x;
                s_tmp[32] = __popc(bal);
            }
        }
        __syncthreads();
        return s_tmp[32];
    }
    const uint32_t k0 = 2u * threadIdx.x, k1 = k0 + 1u;
    uint32_t s0 = 0, l0 = 0, r0 = 0, c0 = 0, s1 = 0, l1 = 0, r1 = 0, c1 = 0;
    if (k0 < nb) { s0 = seg_start[k0]; l0 = seg_off[k0]; r0 = seg_run[k0]; c0 = seg_cut[k0]; }
    if (k1 < nb) { s1 = seg_start[k1]; l1 = seg_off[k1]; r1 = seg_run[k1]; c1 = seg_cut[k1]; }
    const uint32_t f0 = (k0 < nb && l0) ? 1u : 0u, f1 = (k1 < nb && l1) ? 1u : 0u;
    uint32_t ns;
    const uint32_t at = block_excl_scan_u32<T>(f0 + f1, s_tmp, &ns);  // all reads done before it returns
    if (f0) { seg_start[at] = s0; seg_off[at] = l0; seg_run[at] = r0; seg_cut[at] = c0; }
    if (f1) { seg_start[at + f0] = s1; seg_off[at + f0] = l1; seg_run[at + f0] = r1; seg_cut[at + f0] = c1; }
    __syncthreads();
    block_scan_inplace(seg_off, ns, s_tmp);
    return ns;
}

// Flattened walk over the non-empty parts seg[0..ns): every entry idx of every
// part is visited once, entries spread evenly over the CTA's warps.  Warp w
// owns one contiguous stretch of the flattened index space; its lanes step
// through it 32 entries apart (coalesced loads), ILP steps at a time, so load
// runs for ILP entries before body runs for any of them and a warp keeps ILP
// independent memory loads in flight.  A lane finds the part of its first
// entry by binary search over the part offsets and then only moves forward:
// it advances to the next part whenever its entry passes the current part's
// end, so mapping an entry to (part, index) costs a compare and an add.
constexpr int ILP = 4;

template <class Item, class Load, class Body>
__device__ __forceinline__ void flat_for(const uint32_t *seg_start, const uint32_t *seg_off, uint32_t ns,
                                         Load &&load, Body &&body) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tot = seg_off[ns];
    constexpr uint32_t STEP = 32u * ILP;
    const uint32_t steps = (tot + STEP - 1) / STEP;       // warp steps in all
    const uint32_t per_warp = (steps + NWARPS - 1) / NWARPS;
    const uint32_t t0 = warp * per_warp * STEP + lane;    // this lane's first entry
    const uint32_t tend = min(tot, (warp + 1) * per_warp * STEP);
    if (t0 >= tend) return;
    // part holding t0: the last k with seg_off[k] <= t0 (seg_off[0] = 0, seg_off[ns] = tot > t0)
    uint32_t lo = 0, hi = ns;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (seg_off[mid] <= t0)
            lo = mid;
        else
            hi = mid;
    }
    uint32_t k = lo;
    uint32_t next = seg_off[k + 1];         // end of part k in the flattened space
    uint32_t base = seg_start[k] - seg_off[k];  // idx = base + t inside part k (mod 2^32)
    for (uint32_t t = t0; t < tend; t += STEP) {
        uint32_t kk[ILP], idx[ILP];
        bool ok[ILP];
#pragma unroll
        for (int u = 0; u < ILP; ++u) {
            const uint32_t tu = t + 32u * u;
            ok[u] = tu < tend;
            if (ok[u]) {
                while (tu >= next) {  // parts are non-empty and k + 1 < ns while tu < tot
                    ++k;
                    next = seg_off[k + 1];
                    base = seg_start[k] - seg_off[k];
                }
            }
            kk[u] = k;
            idx[u] = base + tu;
        }
        Item it[ILP];
#pragma unroll
        for (int u = 0; u < ILP; ++u)
            if (ok[u]) load(kk[u], idx[u], it[u]);
#pragma unroll
        for (int u = 0; u < ILP; ++u)
            if (ok[u]) body(kk[u], idx[u], it[u]);
    }
}

struct RankItem {
    uint32_t r;
};
struct ProdItem {
    uint32_t r;
    float xv, yv;
};

// Step A for runs b0 .. b0+nb-1 of the row: the part of each run from its
// cursor up to the first rank >= lim goes (uncompacted) to the seg arrays,
// its end to a.pend (END_TO = 1: the marking numeric pass reads the parts
// again) or straight to the run's cursor (END_TO = 2: the symbolic pass, which
// reads them once), or nowhere (0: the caller moves the cursors itself).
// Returns the smallest rank >= lim this thread saw (INF if none): the next
// window's start.
template <int END_TO>
__device__ __forceinline__ uint32_t find_parts(const AccArgs &a, uint32_t b0, uint32_t nb, uint32_t lim,
                                               uint32_t *seg_start, uint32_t *seg_off, uint32_t *seg_run,
                                               uint32_t *seg_cut) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t nextmin = INF;
    if (nb <= (uint32_t)kGallopWarpRuns) {
        // few runs, long parts: one warp per run, 32-way fan-out search
        for (uint32_t k = warp; k < nb; k += NWARPS) {
            const uint32_t i = b0 + k;
            const uint32_t p = a.cursor[i];
            const uint32_t e = a.pos[i] + a.cnt[i];
            uint32_t pe = p, fr = INF;
            if (p < e) pe = warp_gallop(a.yrank, p, e, lim, &fr);
            if (lane == 0) {
                seg_start[k] = p;
                seg_off[k] = pe - p;
                seg_run[k] = i;
                seg_cut[k] = pe;
                if (END_TO == 1) a.pend[i] = pe;
                if (END_TO == 2) a.cursor[i] = pe;
            }
            nextmin = min(nextmin, fr);
        }
    } else {
        // many runs, short parts: one thread per run, doubling then bisection
        for (uint32_t k = tid; k < nb; k += T) {
            const uint32_t i = b0 + k;
            const uint32_t p = a.cursor[i];
            const uint32_t e = a.pos[i] + a.cnt[i];
            uint32_t pe = p, fr = INF;
            if (p < e) pe = thread_gallop(a.yrank, p, e, lim, &fr);
            seg_start[k] = p;
            seg_off[k] = pe - p;
            seg_run[k] = i;
            seg_cut[k] = pe;
            if (END_TO == 1) a.pend[i] = pe;
            if (END_TO == 2) a.cursor[i] = pe;
            nextmin = min(nextmin, fr);
        }
    }
    return nextmin;
}

// Row constants kept in shared memory rather than registers (the numeric
// kernel runs at the register limit of two CTAs per SM).
struct RowConst {
    uint64_t xf_hi;         // x_f << Y_nfbits: the high part of every output key of the row
    const uint64_t *cols;   // the row's job's column table (rank -> y_f)
    const uint32_t *src;    // the row's kept bitmap (numeric)
    uint32_t rb;            // rank of the kept bitmap's bit 0
};

// Step 4: slot -> column table from the window's bitmap (nwu words from rank
// W0 at A, their prefixes at A + NWORDS: 16-bit when P16, else 32-bit; read
// into registers before the table overwrites the region), then coalesced
// writes of the window's `outputs` outputs and the reset of their
// accumulators.  Words go to threads cyclically (word tid + q*T), so a dense
// stretch of the bitmap spreads over many threads instead of a few.
template <bool P16>
__device__ __forceinline__ void write_window(const AccArgs &a, uint32_t *A, float *hi, float *lo, uint32_t nwu,
                                             uint32_t outputs, uint32_t W0, uint32_t out_pos, const RowConst &rc) {
    const uint32_t tid = threadIdx.x;
    uint32_t *ocol = A;
    const uint16_t *wp16 = reinterpret_cast<const uint16_t *>(A + NWORDS);
    uint32_t myw[WPT_MAX], myp[WPT_MAX];
#pragma unroll
    for (int q = 0; q < WPT_MAX; ++q) {
        const uint32_t w = tid + (uint32_t)q * T;
        myw[q] = w < nwu ? A[w] : 0u;
        myp[q] = w < nwu ? (P16 ? (uint32_t)wp16[w] : A[NWORDS + w]) : 0u;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < WPT_MAX; ++q) {
        uint32_t bw = myw[q];
        uint32_t slot = myp[q];
        const uint32_t cbase = W0 + 32u * (tid + (uint32_t)q * T);
        while (bw && slot < outputs) {
            ocol[slot++] = cbase + (uint32_t)(__ffs(bw) - 1);
            bw &= bw - 1;
        }
    }
    __syncthreads();
    // The stores stream past L2 so the output does not evict the Y operand.
    const uint64_t xf_hi = rc.xf_hi;
    const uint64_t *cols = rc.cols;
    for (uint32_t q = tid; q < outputs; q += T) {
        const uint64_t o = (uint64_t)out_pos + q;
        const float v = hi[q] + lo[q];
        if (o < a.out_cap) {
            __stcs(a.out_keys + o, (unsigned long long)(xf_hi | cols[ocol[q]]));
            __stcs(a.out_vals + o, v);
        } else {
            atomicOr(a.err, 4u);
        }
        hi[q] = 0.f;
        lo[q] = 0.f;
    }
}

template <bool NUMERIC>
__global__ void __launch_bounds__(T, NUMERIC ? 2 : 3) k_rowwin(AccArgs a) {  // numeric: two CTAs per SM, symbolic: three
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NWK = NUMERIC ? NWORDS : NWORDS_SYM;
    // numeric: region A (AW words, see AW); symbolic: the bitmap alone
    uint32_t *A = reinterpret_cast<uint32_t *>(smem_raw);
    uint32_t *bits = A;                                        // [NWK] bitmap
    uint32_t *wp = A + NWORDS;                                 // [NWORDS] word prefix (marked windows, numeric)
    uint16_t *wp16 = reinterpret_cast<uint16_t *>(A + NWORDS); // [NWORDS] word prefix (kept rows, numeric)
    uint32_t *seg_start = A + (NUMERIC ? AW : NWK);            // [MAXR]
    uint32_t *seg_off = seg_start + MAXR;                      // [MAXR + 4]
    uint32_t *seg_run = seg_off + MAXR + 4;                    // [MAXR]
    uint32_t *seg_cut = seg_run + MAXR;                        // [MAXR]
    float *seg_xv = reinterpret_cast<float *>(seg_cut + MAXR); // [MAXR]  (numeric) X value of each part
    float *hi = seg_xv + (NUMERIC ? MAXR : 0);                 // [CAP]   (numeric)
    float *lo = hi + CAP;                                      // [CAP]   (numeric)
    __shared__ uint32_t s_tmp[33];
    __shared__ uint32_t s_unit;
    __shared__ uint32_t s_cut;
    __shared__ uint32_t s_next;  // kept bitmaps: the smallest rank past the window (atomicMin)
    __shared__ RowConst s_rc;

    const int tid = threadIdx.x;
    // outputs per window: the compiled capacity, or a smaller tile chosen at run time
    const uint32_t cap = (a.heavy_cap && a.heavy_cap < (uint32_t)CAP) ? a.heavy_cap : (uint32_t)CAP;

    for (int i = tid; i < NWK; i += T) bits[i] = 0;
    if (NUMERIC)
        for (int i = tid; i < CAP; i += T) hi[i] = lo[i] = 0.f;
    __syncthreads();

    for (;;) {
        if (tid == 0) s_unit = atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t u = s_unit;
        if (u >= a.nunits) break;
        const uint32_t row = a.units[u];
        const uint32_t xs = a.row_start[row], xe = a.row_start[row + 1];
        // words of the row's kept column bitmap (0: none, the windows mark their columns)
        const uint32_t nwr = a.row_bmoff ? (uint32_t)(a.row_bmoff[row + 1] - a.row_bmoff[row]) : 0u;
        if (tid == 0) {  // read after the barriers of block_min_u32 below
            int y_nfbits;
            const uint64_t *cols;
            uint32_t ncols;
            row_job_params(a, row, y_nfbits, cols, ncols);
            s_rc.xf_hi = shl(a.row_xf[row], y_nfbits);
            s_rc.cols = cols;
            if (nwr) {
                s_rc.src = a.hbm + a.row_bmoff[row];
                s_rc.rb = a.row_rb[row];
            }
        }

        uint32_t mymin = INF;
        for (uint32_t i = xs + tid; i < xe; i += T) {
            const uint32_t p = a.pos[i];
            a.cursor[i] = p;
            if (a.cnt[i]) mymin = min(mymin, a.yrank[p]);
        }
        uint32_t R0 = block_min_u32<T>(mymin, s_tmp);

        // initial window width from the row's density (products vs columns)
        uint32_t rw = NUMERIC ? RW : RW_SYM;
        if (NUMERIC && !nwr) {
            const uint64_t P = a.xprefix[xe] - a.xprefix[xs];
            int y_nfbits;
            const uint64_t *cols;
            uint32_t ncols;
            row_job_params(a, row, y_nfbits, cols, ncols);
            const uint64_t est = (uint64_t)cap * ncols / (P ? P : 1);
            const uint64_t clamped = est < 32ull ? 32ull : (est > (uint64_t)RW ? (uint64_t)RW : est);
            rw = (uint32_t)clamped & ~31u;
        }
        // the row's first slot in the chunk buffer (a chunk holds fewer than 2^32 outputs)
        uint32_t out_pos = NUMERIC ? (uint32_t)(a.row_off[row] - a.chunk_base) : 0u;
        uint32_t row_total = 0;
        const bool one_batch = xe - xs <= (uint32_t)MAXR;  // parts from step A stay in place

        if (NUMERIC && nwr) {
            // ---- kept bitmap: windows are swept contiguously from the row's
            // smallest rank; each loads its words (from a 16-byte aligned word,
            // the ranks below R masked off), so nothing is marked and the window
            // ends exactly after its cap-th column.
            uint32_t R = R0;  // every column below R is written
            for (;;) {
                const uint32_t rb = s_rc.rb;
                if (R == INF) break;
                const uint32_t wo = ((R - rb) >> 7) << 2;
                if (wo >= nwr) break;
                const uint32_t W0 = rb + 32u * wo;
                const uint32_t nw = min((uint32_t)NWORDS, nwr - wo);
                const uint32_t skip = R - W0;  // < 128: ranks [W0, R) of words 0..3 are done
                __syncthreads();  // the previous window no longer reads bits, prefix, table or s_next
                for (uint32_t q = tid; q < (nw >> 2); q += T) cp_async16(bits + 4u * q, s_rc.src + wo + 4u * q);
                cp_async_wait_all();
                if (tid == 0) s_next = INF;
                __syncthreads();
                // word prefix: thread t owns wpt consecutive words (4 or 8, read as
                // 16-byte vectors; thread 0 clears the done ranks of words 0..3
                // and writes them back before any other thread reads them), the
                // 16-bit prefixes are written 4 at a time (clamped: slots past
                // the capacity are never used)
                const uint32_t wpt = ((nw + T - 1) / T + 3u) & ~3u;
                static_assert(NWORDS <= 8 * T, "at most 8 words per thread");
                const uint32_t w0 = (uint32_t)tid * wpt;
                const uint32_t w1 = min(w0 + wpt, nw);
                uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = make_uint4(0u, 0u, 0u, 0u);
                if (w0 < w1) v0 = *reinterpret_cast<const uint4 *>(bits + w0);
                if (w0 + 4u < w1) v1 = *reinterpret_cast<const uint4 *>(bits + w0 + 4u);
                if (w0 == 0 && skip) {
                    v0.x = skip >= 32u ? 0u : v0.x & (FULL << skip);
                    v0.y = skip >= 64u ? 0u : (skip <= 32u ? v0.y : v0.y & (FULL << (skip - 32u)));
                    v0.z = skip >= 96u ? 0u : (skip <= 64u ? v0.z : v0.z & (FULL << (skip - 64u)));
                    v0.w = skip <= 96u ? v0.w : v0.w & (FULL << (skip - 96u));
                    *reinterpret_cast<uint4 *>(bits) = v0;
                }
                const uint32_t loc = __popc(v0.x) + __popc(v0.y) + __popc(v0.z) + __popc(v0.w) + __popc(v1.x) +
                                     __popc(v1.y) + __popc(v1.z) + __popc(v1.w);
                uint32_t Dw;
                const uint32_t run0 = block_excl_scan_u32<T>(loc, s_tmp, &Dw);
                if (w0 < w1) {
                    // four 16-bit prefixes per 8-byte store
                    uint32_t p = run0;
                    auto pack = [&](uint32_t x, uint32_t y) {
                        const uint32_t a0 = min(p, 0xffffu);
                        p += __popc(x);
                        const uint32_t a1 = min(p, 0xffffu);
                        p += __popc(y);
                        return a0 | (a1 << 16);
                    };
                    const uint32_t h0 = pack(v0.x, v0.y);
                    const uint32_t h1 = pack(v0.z, v0.w);
                    *reinterpret_cast<uint2 *>(wp16 + w0) = make_uint2(h0, h1);
                    if (w0 + 4u < w1) {
                        const uint32_t h2 = pack(v1.x, v1.y);
                        const uint32_t h3 = pack(v1.z, v1.w);
                        *reinterpret_cast<uint2 *>(wp16 + w0 + 4u) = make_uint2(h2, h3);
                    }
                }
                if (Dw > cap && run0 <= cap && cap < run0 + loc) {
                    // this thread holds the cut: its word holding the (cap+1)-th column
                    for (uint32_t w = w0; w < w1; ++w) {
                        const uint32_t pw = wp16[w], b = bits[w];
                        if (pw <= cap && cap < pw + __popc(b))
                            s_cut = W0 + 32u * w + (uint32_t)__fns(b, 0u, (int)(cap - pw + 1));
                    }
                }
                uint32_t R1 = W0 + 32u * nw, outputs = Dw;
                if (Dw == 0) {  // a gap wider than the window (Dw is the same in every thread)
                    R = R1;
                    continue;
                }
                __syncthreads();
                if (Dw > cap) {
                    R1 = s_cut;
                    outputs = cap;
                }
                if (tid == 0) {
                    // the next window's words, fetched into L2 while this one is accumulated
                    const uint32_t wn = ((R1 - rb) >> 7) << 2;
                    if (wn < nwr) prefetch_l2(s_rc.src + wn, 4u * min((uint32_t)NWORDS, nwr - wn));
                }
                for (uint32_t b0 = xs; b0 < xe; b0 += MAXR) {
                    const uint32_t nb = min((uint32_t)MAXR, xe - b0);
                    const uint32_t nm = find_parts<0>(a, b0, nb, R1, seg_start, seg_off, seg_run, seg_cut);
                    if (nm != INF) atomicMin(&s_next, nm);
                    __syncthreads();
                    const uint32_t ns = compact_parts(nb, seg_start, seg_off, seg_run, seg_cut, s_tmp);
                    for (uint32_t k = tid; k < ns; k += T) seg_xv[k] = a.xval[seg_run[k]];
                    __syncthreads();
                    flat_for<ProdItem>(
                        seg_start, seg_off, ns,
                        [&](uint32_t k, uint32_t idx, ProdItem &it) {
                            it.r = a.yrank[idx];
                            it.yv = a.yval[idx];
                            it.xv = seg_xv[k];
                        },
                        [&](uint32_t, uint32_t, const ProdItem &it) {
                            const uint32_t c = it.r - W0;  // in [skip, 32*nw): parts end below R1
                            const uint32_t w = c >> 5;
                            const uint32_t slot =
                                w < nw ? wp16[w] + __popc(bits[w] & ((1u << (c & 31)) - 1u)) : outputs;
                            if (slot < outputs) {
                                const float pr = it.xv * it.yv;
                                const float pe = fmaf(it.xv, it.yv, -pr);
                                const float old = atomicAdd(&hi[slot], pr);
                                float sum, err;
                                two_sum(old, pr, sum, err);
                                atomicAdd(&lo[slot], err + pe);
                            } else {
                                atomicOr(a.err, 4u);  // the kept bitmap disagrees with the runs
                            }
                        });
                    __syncthreads();
                    for (uint32_t k = tid; k < ns; k += T) a.cursor[seg_run[k]] = seg_cut[k];
                    __syncthreads();
                }
                write_window<true>(a, A, hi, lo, nw, outputs, W0, out_pos, s_rc);
                if (tid == 0) atomicAdd(a.err + 2, 1u);  // windows swept (statistics)
                out_pos += outputs;
                row_total += outputs;
                // the next window starts at the row's next column (skipping a gap; INF: none left)
                R = max(R1, s_next);
            }
            R0 = INF;  // the row is done
        }

        while (R0 != INF) {
            // a kept row's symbolic windows start on a 16-byte boundary of its bitmap
            const uint32_t W0 = (!NUMERIC && nwr) ? R0 - ((R0 - s_rc.rb) & 127u) : R0;
            const uint32_t lim = W0 + rw;  // ranks < 2^31: no wrap
            const uint32_t nwu = rw >> 5;  // bitmap words in use
            uint32_t nextmin = INF;
            uint32_t ns = 0;
            uint32_t newcols = 0;  // symbolic: columns in this thread's words of the window
            if (NUMERIC) {
                // the region held the previous window's table (or a kept row's pairs): clear the bitmap
                __syncthreads();
                for (uint32_t w = 4u * tid; w < (uint32_t)NWORDS; w += 4u * T)
                    *reinterpret_cast<uint4 *>(bits + w) = make_uint4(0u, 0u, 0u, 0u);
                __syncthreads();
            }

            // ---- A, B, 1: parts of every run inside the window, marked in the bitmap
            for (uint32_t b0 = xs; b0 < xe; b0 += MAXR) {
                const uint32_t nb = min((uint32_t)MAXR, xe - b0);
                nextmin = min(nextmin, find_parts<NUMERIC ? 1 : 2>(a, b0, nb, lim, seg_start, seg_off, seg_run, seg_cut));
                __syncthreads();
                ns = compact_parts(nb, seg_start, seg_off, seg_run, seg_cut, s_tmp);
                if (NUMERIC)
                    for (uint32_t k = tid; k < ns; k += T) seg_xv[k] = a.xval[seg_run[k]];
                flat_for<RankItem>(
                    seg_start, seg_off, ns,
                    [&](uint32_t, uint32_t idx, RankItem &it) { it.r = a.yrank[idx]; },
                    [&](uint32_t, uint32_t, const RankItem &it) {
                        const uint32_t c = it.r - W0;
                        const uint32_t m = 1u << (c & 31);
                        if (!(bits[c >> 5] & m)) atomicOr(&bits[c >> 5], m);  // no return value needed
                    });
                __syncthreads();
            }

            if (!NUMERIC) {
                // a kept row's window goes to its bitmap (16-byte pieces, coalesced);
                // the bitmap is cleared for the next window either way
                static_assert(NWORDS_SYM % (4 * T) == 0, "whole 16-byte pieces per thread");
                uint32_t *dst = nwr ? a.hbm + a.row_bmoff[row] : nullptr;
                const uint32_t wo = nwr ? (W0 - s_rc.rb) >> 5 : 0u;  // a multiple of 4
                for (uint32_t q = 4u * tid; q < nwu; q += 4u * T) {
                    const uint4 v = *reinterpret_cast<const uint4 *>(bits + q);
                    newcols += __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
                    if (nwr && wo + q < nwr) *reinterpret_cast<uint4 *>(dst + wo + q) = v;
                    *reinterpret_cast<uint4 *>(bits + q) = make_uint4(0u, 0u, 0u, 0u);
                }
                // the window's new columns and the next window's start (the run
                // searches moved the cursors already)
                uint32_t Dw;
                block_sum_min_u32<T>(newcols, nextmin, s_tmp, Dw, R0);
                row_total += Dw;
                if (nwr) {
                    // the words up to the next window's (or the bitmap's end) hold no column
                    const uint32_t from = wo + nwu;
                    const uint32_t to = R0 == INF ? nwr : min(nwr, ((R0 - s_rc.rb) >> 7) << 2);
                    for (uint32_t q = from + 4u * tid; q < to; q += 4u * T)
                        *reinterpret_cast<uint4 *>(dst + q) = make_uint4(0u, 0u, 0u, 0u);
                }
                continue;
            }

            // ---- 2: word prefix of the bitmap
            // words in use are split in blocks of wpt consecutive words per thread
            const uint32_t wpt = (nwu + T - 1) / T;
            const uint32_t w0 = (uint32_t)tid * wpt;
            const uint32_t w1 = min(w0 + wpt, nwu);
            uint32_t loc = 0;
            for (uint32_t w = w0; w < w1; ++w) loc += __popc(bits[w]);
            uint32_t Dw;
            uint32_t run = block_excl_scan_u32<T>(loc, s_tmp, &Dw);
            for (uint32_t w = w0; w < w1; ++w) {
                wp[w] = run;
                run += __popc(bits[w]);
            }

            // ---- numeric: cut the window at the CAP-th touched column if needed
            const bool over = Dw > cap;
            uint32_t R1 = lim, outputs = Dw;
            if (over) {
                for (uint32_t w = w0; w < w1; ++w) {
                    const uint32_t pw = wp[w];
                    if (pw <= cap && cap < pw + __popc(bits[w])) {
                        const uint32_t b = __fns(bits[w], 0u, (int)(cap - pw + 1));
                        s_cut = R0 + 32u * w + b;
                    }
                }
                __syncthreads();
                R1 = s_cut;
                outputs = cap;
            }
            __syncthreads();

            // ---- 3: accumulate every product of the window into its slot
            for (uint32_t b0 = xs; b0 < xe; b0 += MAXR) {
                const uint32_t nb = min((uint32_t)MAXR, xe - b0);
                if (!one_batch) {
                    for (uint32_t k = tid; k < nb; k += T) {
                        const uint32_t i = b0 + k;
                        const uint32_t p = a.cursor[i];
                        const uint32_t pe = a.pend[i];
                        seg_start[k] = p;
                        seg_off[k] = pe - p;
                        seg_run[k] = i;
                        seg_cut[k] = pe;
                    }
                    __syncthreads();
                    ns = compact_parts(nb, seg_start, seg_off, seg_run, seg_cut, s_tmp);
                    for (uint32_t k = tid; k < ns; k += T) seg_xv[k] = a.xval[seg_run[k]];
                    __syncthreads();
                }
                flat_for<ProdItem>(
                    seg_start, seg_off, ns,
                    [&](uint32_t k, uint32_t idx, ProdItem &it) {
                        it.r = a.yrank[idx];
                        it.yv = a.yval[idx];
                        it.xv = seg_xv[k];
                    },
                    [&](uint32_t k, uint32_t idx, const ProdItem &it) {
                        if (it.r < R1) {
                            const uint32_t c = it.r - R0;
                            const uint32_t w = c >> 5;
                            const uint32_t slot = wp[w] + __popc(bits[w] & ((1u << (c & 31)) - 1u));
                            const float pr = it.xv * it.yv;
                            const float pe = fmaf(it.xv, it.yv, -pr);
                            const float old = atomicAdd(&hi[slot], pr);
                            float sum, err;
                            two_sum(old, pr, sum, err);
                            atomicAdd(&lo[slot], err + pe);
                        } else {
                            atomicMin(&seg_cut[k], idx);
                        }
                    });
                __syncthreads();
                for (uint32_t k = tid; k < ns; k += T) a.cursor[seg_run[k]] = seg_cut[k];
                __syncthreads();
            }

            // ---- 4: slot -> column table, then coalesced writes of the window
            write_window<false>(a, A, hi, lo, nwu, outputs, R0, out_pos, s_rc);
            if (tid == 0) atomicAdd(a.err + 2, 1u);  // windows swept (statistics)
            out_pos += outputs;
            row_total += outputs;
            // next width: fifteen sixteenths of the cap at the density just seen
            // (at most 4x wider per window)
            if (over) {
                rw = max(32u, ((R1 - R0) / 16u * 15u + 31u) & ~31u);
                __syncthreads();
                R0 = R1;
            } else {
                const uint64_t want = Dw ? (uint64_t)rw * (uint64_t)(15 * cap / 16) / Dw : (uint64_t)rw * 4u;
                uint64_t nr = want < (uint64_t)rw * 4u ? want : (uint64_t)rw * 4u;
                nr = nr > (uint64_t)RW ? (uint64_t)RW : (nr < 32u ? 32u : nr);
                rw = (uint32_t)nr & ~31u;
                R0 = block_min_u32<T>(nextmin, s_tmp);
            }
        }
        if (!NUMERIC && tid == 0) a.row_nnz[row] = row_total;
        __syncthreads();
    }
}

// Rank span of every heavy row: a warp per row (grid-stride over H, whose
// count is on the device); runs are sorted by rank, so a run's first and last
// entries bound it.
__global__ void k_hspan(const uint32_t *__restrict__ H, const uint64_t *__restrict__ nh,
                        const uint32_t *__restrict__ row_start, const uint32_t *__restrict__ pos,
                        const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ yrank,
                        const uint64_t *__restrict__ row_prod, uint32_t *__restrict__ w_all,
                        uint32_t *__restrict__ w_dense, uint32_t *__restrict__ row_rb) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t n = *nh;
    for (uint64_t k = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nwarps) {
        const uint32_t row = H[k];
        const uint32_t xs = row_start[row], xe = row_start[row + 1];
        uint32_t mn = INF, mx = 0;
        for (uint32_t i = xs + lane; i < xe; i += 32) {
            const uint32_t c = cnt[i];
            if (c) {
                const uint32_t p = pos[i];
                mn = min(mn, yrank[p]);
                mx = max(mx, yrank[p + c - 1]);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn = min(mn, __shfl_xor_sync(FULL, mn, o));
            mx = max(mx, __shfl_xor_sync(FULL, mx, o));
        }
        if (lane == 0 && mn != INF) {
            const uint64_t span = (uint64_t)mx - mn + 1;
            const uint32_t words = (uint32_t)(((span + 127) >> 7) << 2);
            w_all[row] = span <= kKeepBitsMax * row_prod[row] ? words : 0u;
            w_dense[row] = span <= kKeepBitsPerProduct * row_prod[row] ? words : 0u;
            row_rb[row] = mn;
        }
    }
}

size_t rowwin_smem(bool numeric) {
    const size_t words = (numeric ? (size_t)AW + MAXR : (size_t)NWORDS_SYM) + MAXR + (MAXR + 4) + MAXR + MAXR;
    return words * 4 + (numeric ? (size_t)CAP * 8 : 0);
}

}  // namespace

// Resident CTAs per SM of each instantiation (registers and shared memory
// decide: the symbolic pass needs no accumulators and fits more CTAs).
int heavy_blocks_per_sm(bool numeric) {
    int n = 0;
    const size_t sm = rowwin_smem(numeric);
    if (numeric) {
        GS_CUDA(cudaFuncSetAttribute(k_rowwin<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_rowwin<true>, T, sm));
    } else {
        GS_CUDA(cudaFuncSetAttribute(k_rowwin<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        GS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_rowwin<false>, T, sm));
    }
    return n > 0 ? n : 1;
}

void launch_heavy(const AccArgs &a, bool numeric, int grid, cudaStream_t s) {
    if (a.nunits == 0) return;
    const size_t sm = rowwin_smem(numeric);
    if (numeric) {
        GS_CUDA(cudaFuncSetAttribute(k_rowwin<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_rowwin<true><<<grid, T, sm, s>>>(a);
    } else {
        GS_CUDA(cudaFuncSetAttribute(k_rowwin<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_rowwin<false><<<grid, T, sm, s>>>(a);
    }
    count_launch();
    GS_CUDA(cudaGetLastError());
}

void launch_heavy_spans(const uint32_t *H, const uint64_t *nh, uint64_t nh_max, uint64_t nrows_max,
                        const uint32_t *row_start, const uint32_t *pos, const uint32_t *cnt,
                        const uint32_t *yrank, const uint64_t *row_prod, uint32_t *w_all, uint32_t *w_dense,
                        uint32_t *row_rb, cudaStream_t s) {
    if (nrows_max) {
        GS_CUDA(cudaMemsetAsync(w_all, 0, sizeof(uint32_t) * nrows_max, s));
        GS_CUDA(cudaMemsetAsync(w_dense, 0, sizeof(uint32_t) * nrows_max, s));
    }
    if (nh_max == 0) return;
    constexpr int B = 256;
    const uint64_t blocks = (nh_max * 32 + B - 1) / B;
    k_hspan<<<(unsigned)std::min<uint64_t>(blocks, 4096), B, 0, s>>>(H, nh, row_start, pos, cnt, yrank, row_prod,
                                                                     w_all, w_dense, row_rb);
    count_launch();
    GS_CUDA(cudaGetLastError());
}

}  // namespace gs
