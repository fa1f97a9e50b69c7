// kernels.cuh -- launch interfaces of the engine's device kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "internal.h"

namespace gs {

// ---- linearise (reference: include/gsparc/tensor_manager.tpp:246-294) ----
struct LinParams {
    int order;
    int role;       // 0: X layout f<<ncbits|c, 1: Y layout c<<nfbits|f
    int ncbits, nfbits;
    int shift[kMaxOrder];
    int is_c[kMaxOrder];
    uint64_t dims[kMaxOrder];
};
LinParams make_lin_params(const Layout &L, const uint64_t *dims, int role);
// keys[k] from SoA idx (idx[m*nnz+k]); optionally copies val -> val_out.
// Out-of-range indices set bit 0 of *err.
void launch_linearize(const LinParams &p, uint64_t nnz, const uint64_t *idx, const float *val,
                      uint64_t *keys, float *val_out, unsigned int *err, cudaStream_t s);

// ---- sort (CUB radix sort; reference: include/gsparc/sort.cuh:90-108) ----
// Sorts (keys, vals) by bits [0, nbits).  keys/vals are double buffers: on
// return *which tells which of the two holds the result (0 or 1).
void sort_pairs(Arena &a, uint64_t n, uint64_t *keys0, uint64_t *keys1, float *vals0, float *vals1,
                int nbits, int *which, cudaStream_t s);
void sort_keys(Arena &a, uint64_t n, uint64_t *keys0, uint64_t *keys1, int nbits, int *which,
               cudaStream_t s);
// This library's own stable onesweep radix sort of the same pairs (radix.cu),
// 8 bits per pass; same double-buffer contract as sort_pairs.  A look-back
// wait that runs out sets bit 8 of *err (the caller's device error word).
void own_sort_pairs(Arena &a, uint64_t n, uint64_t *keys0, uint64_t *keys1, float *vals0, float *vals1,
                    int nbits, int *which, unsigned int *err, cudaStream_t s);

// ---- Y preparation ----
// From sorted Y keys (c << nfbits | f): per-entry column rank among the
// distinct free indices, the distinct free indices, and the run table of
// contract keys (run r covers [run_start[r], run_start[r+1])).
struct YPrep {
    uint64_t ny = 0, ncols = 0, nruns = 0;
    DBuf<uint32_t> rank;      // [ny]
    DBuf<uint64_t> cols;      // [ncols] distinct y_f ascending
    DBuf<uint64_t> run_key;   // [nruns]
    DBuf<uint32_t> run_start; // [nruns+1]
};
void prepare_y(Arena &a, const uint64_t *ykeys, uint64_t ny, int y_nfbits, YPrep &out,
               cudaStream_t s);

// ---- X match + rows ----
struct XMatch {
    uint64_t nx = 0, nrows = 0, ir = 0;
    DBuf<uint32_t> pos;        // [nx] first Y index of the matching run
    DBuf<uint32_t> cnt;        // [nx] run length (0: no match)
    DBuf<uint64_t> xprefix;    // [nx+1] exclusive prefix of cnt
    DBuf<uint32_t> row_start;  // [nrows+1]
    DBuf<uint64_t> row_xf;     // [nrows]
    DBuf<uint64_t> row_prod;   // [nrows]
};
void match_x(Arena &a, const uint64_t *xkeys, uint64_t nx, int x_ncbits, const YPrep &y,
             XMatch &out, cudaStream_t s);

// ---- accumulation ----
// Per-job constants of a batch (gsparc_sptc_batch): rows of all jobs share
// the arrays below, each row knows its job.
struct BatchJob {
    int y_nfbits;       // the job's Y free bits (output key = x_f << y_nfbits | y_f)
    uint32_t ncols;     // the job's distinct Y free indices
    uint64_t cols_off;  // where the job's distinct Y free indices start in `cols`
};

struct AccArgs {
    // batch: job of every row (null for a single contraction) and job table
    const uint16_t *row_job;
    const BatchJob *jobs;
    // X side
    const uint32_t *row_start;
    const uint64_t *row_xf;
    const uint32_t *pos;
    const uint32_t *cnt;
    const uint64_t *xprefix;
    const float *xval;
    // Y side
    const uint32_t *yrank;
    const float *yval;
    const uint64_t *ykeys;     // sorted Y keys (c << nfbits | y_f, job id above): y_f without the column table
    const uint64_t *cols;
    int y_nfbits;
    // single-run rows (stream path): the matched X nonzero of every such row,
    // and the product prefix over the listed rows (nunits + 1 entries)
    const uint32_t *row_xi;
    const uint64_t *sprefix;
    // work
    const uint32_t *units;     // light: pairs (r0, r1); heavy and stream: row ids
    uint32_t nunits;
    unsigned int *work_counter;
    uint32_t *cursor;          // [nx] scratch (heavy path): next unprocessed Y entry per run
    uint32_t *pend;            // [nx] scratch (heavy path): end of the run's part in the window
    uint32_t ncols;            // distinct Y free indices (column ranks are < ncols)
    uint32_t heavy_cap;        // heavy rows: outputs per window (0 or > kHeavyCap: kHeavyCap)
    // heavy rows: column bitmaps the symbolic pass keeps for the numeric pass
    // (row_bmoff null: none kept).  A kept row's bitmap is the words
    // [row_bmoff[row], row_bmoff[row+1]) of hbm (a multiple of 4; none: the
    // row marks its windows), bit 0 = column rank row_rb[row], its smallest.
    uint32_t *hbm;
    const uint64_t *row_bmoff;  // [nrows + 1]
    const uint32_t *row_rb;     // [nrows]
    // symbolic output
    uint32_t *row_nnz;         // [nrows]
    // numeric output
    const uint64_t *row_off;   // [nrows] exclusive prefix of row_nnz
    uint64_t chunk_base;
    uint64_t out_cap;          // capacity of out_keys/out_vals (writes beyond are skipped, err bit 4)
    uint64_t *out_keys;
    float *out_vals;
    unsigned int *err;
};

constexpr int kHeavyThreads = 512;
constexpr int kHeavyRW = 1 << 17;  // column ranks covered by one window's touched bitmap
constexpr int kHeavyCap = 8192;    // output slots (compensated accumulators) per window
                                   // (sized so two CTAs fit one SM's shared memory)
constexpr int kHeavyMaxRuns = 512;   // runs flattened per batch
constexpr int kGallopWarpRuns = 64;  // up to this many runs per batch: one warp per run search
constexpr int kLightCap = 4096;    // on-chip ESC capacity (products per unit)
constexpr int kLightThreads = 512;
constexpr uint64_t kLightRowMax = 1024;   // rows with at most this many products are light
constexpr uint64_t kLightUnitMax = 3072;  // products per light unit

// Output-key width and column table of the job that owns `row`.
__device__ __forceinline__ void row_job_params(const AccArgs &a, uint32_t row, int &y_nfbits,
                                               const uint64_t *&cols, uint32_t &ncols) {
    if (a.row_job) {
        const BatchJob j = a.jobs[a.row_job[row]];
        y_nfbits = j.y_nfbits;
        cols = a.cols + j.cols_off;
        ncols = j.ncols;
    } else {
        y_nfbits = a.y_nfbits;
        cols = a.cols;
        ncols = a.ncols;
    }
}

void launch_heavy(const AccArgs &a, bool numeric, int grid, cudaStream_t s);
// For the heavy rows H[0..*nh) (nh on the device, at most nh_max): the words of
// a column bitmap over the row's rank span (a multiple of 4) in w_all for rows
// whose bitmap holds at most kKeepBitsMax bits per matched product, and in
// w_dense for those with at most kKeepBitsPerProduct; the row's smallest rank
// in row_rb.  Both word arrays are cleared first (nrows_max entries), so other
// rows have 0 words.
constexpr uint64_t kKeepBitsPerProduct = 32;
constexpr uint64_t kKeepBitsMax = 512;
void launch_heavy_spans(const uint32_t *H, const uint64_t *nh, uint64_t nh_max, uint64_t nrows_max,
                        const uint32_t *row_start, const uint32_t *pos, const uint32_t *cnt,
                        const uint32_t *yrank, const uint64_t *row_prod, uint32_t *w_all, uint32_t *w_dense,
                        uint32_t *row_rb, cudaStream_t s);
// numeric pass of single-run rows (their symbolic count is their product count)
void launch_stream(const AccArgs &a, int grid, cudaStream_t s);
int stream_blocks_per_sm();
void launch_light(const AccArgs &a, bool numeric, int grid, cudaStream_t s);
int heavy_blocks_per_sm(bool numeric);
int light_blocks_per_sm();

// ---- misc ----
void exclusive_scan_u32_to_u64(Arena &a, const uint32_t *in, uint64_t *out, uint64_t n,
                               cudaStream_t s);  // out has n+1 entries

void digest_chunk(const uint64_t *keys, const float *vals, uint64_t n, gsparc_digest *out,
                  cudaStream_t s);

// reference-compatible index match (u64 outputs) for the stage entry point
void index_match_compat(Arena &a, uint64_t nx, const uint64_t *xkeys, int x_ncbits, uint64_t ny,
                        const uint64_t *ykeys, int y_nfbits, uint64_t *pos, uint64_t *cnt,
                        uint64_t *prefix, cudaStream_t s);

}  // namespace gs
