/*
 * gsparc_b200.h -- C ABI of the B200-native sparse tensor contraction engine.
 *
 * Z = X x_{cx,cy} Y for two sparse COO tensors, computed the way the reference
 * (seohyeon0322/GSPARC) computes it: linearise each operand into 64-bit keys,
 * sort, match X and Y on their contract keys, accumulate matched products
 * into output keys (x_free << Y_nfbits) | y_free, memory-aware chunking of the
 * output.  Every function returns a status; none exits the process.
 *
 * Plain C: pointers and sizes only.  Streams are passed as `void *` holding a
 * cudaStream_t (NULL = the legacy default stream).
 *
 * Reference interfaces each entry point replaces are cited per declaration as
 * path:line inside the reference repository.
 */
#ifndef GSPARC_B200_H
#define GSPARC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference exits on every error
 * (src/common/cuda_helper.cpp:83-92, src/gsparc/cuda_memory.cpp:78,89,
 *  include/gsparc/sptc.cuh:209-210); these are returned instead. */
typedef enum {
    GSPARC_OK = 0,
    GSPARC_EINVAL = 1,       /* bad argument / malformed input            */
    GSPARC_ENOMEM = 2,       /* HBM budget or host memory exhausted        */
    GSPARC_ECUDA = 3,        /* CUDA runtime error                         */
    GSPARC_EIO = 4,          /* file could not be read / written           */
    GSPARC_ETIMEOUT = 5,     /* a bounded device wait ran out              */
    GSPARC_EUNSUPPORTED = 6, /* valid input outside the supported envelope */
    GSPARC_EINTERNAL = 7,    /* device-side consistency check failed       */
    GSPARC_ECALLBACK = 8     /* an output-sink callback asked to stop      */
} gsparc_status;

typedef struct gsparc_ctx gsparc_ctx;
typedef struct gsparc_tensor gsparc_tensor;

/* SoA COO tensor (0-based indices, float values).
 * Replaces gsparc::SparseTensor<uint64_t,float> (include/gsparc/sparse_tensor.hpp:12-44):
 * indices[m][k] / values[k]. */
typedef struct {
    int order;                   /* number of modes (1..32)                   */
    const uint64_t *dims;        /* [order] mode sizes (host memory)          */
    uint64_t nnz;
    const uint64_t *const *idx;  /* [order] pointers to nnz indices each      */
    const float *val;            /* [nnz]                                     */
    int on_device;               /* 0: idx/val are host pointers, 1: device   */
} gsparc_coo;

/* Accumulator selection, the reference's -d flag (src/gsparc/cmdline_opts.cpp:169-172,
 * include/gsparc/sptc.cuh:201-218). */
enum { GSPARC_ACCUM_ESC = -1, GSPARC_ACCUM_AUTO = 0, GSPARC_ACCUM_DENSE = 1 };

/* Output sink kinds. */
enum {
    GSPARC_SINK_DISCARD = 0, /* compute every chunk in HBM, then drop it      */
    GSPARC_SINK_DEVICE = 1,  /* call on_chunk with device pointers per chunk  */
    GSPARC_SINK_HOST = 2     /* copy chunks into host_keys/host_vals          */
};

/* Per-chunk callback.  keys/vals hold n output nonzeros in ascending key
 * order; first is the global index of the chunk's first nonzero.  on_device
 * tells where keys/vals live.  Return 0 to continue, nonzero to stop
 * (gsparc_sptc then returns GSPARC_ECALLBACK). */
typedef int (*gsparc_chunk_fn)(void *user, const uint64_t *keys, const float *vals,
                               uint64_t n, uint64_t first, int on_device);

/* Output sink.  The reference never returns Z: it copies each ESC chunk into
 * one reused pinned buffer and drops it (include/gsparc/contraction.cuh:554-561,596-597). */
typedef struct {
    int kind;
    gsparc_chunk_fn on_chunk; /* optional for DISCARD / HOST                   */
    void *user;
    /* HOST sink: destination arrays.  If host_capacity >= nnz(Z) the whole Z
     * lands there in order; otherwise every chunk overwrites the arrays from
     * index 0 and on_chunk is called after each copy (ring mode, like the
     * reference's reused pinned buffer).  Page-locked memory copies fastest. */
    uint64_t *host_keys;
    float *host_vals;
    uint64_t host_capacity;
    uint64_t max_chunk_nnz;   /* 0 = derive from the HBM budget                */
    /* Words per output key: 0 or 1 = one uint64 (x_f << Y_nfbits | y_f); 2 =
     * the same key in 128 bits, two uint64 per nonzero, low word first
     * (host_keys then holds 2 * host_capacity words, device chunks 2 * n).
     * Needed when X's free bits + Y's free bits exceed 64, where the
     * reference truncates the key (include/gsparc/contraction_extra.cuh:149-151)
     * and gsparc_sptc with one word returns GSPARC_EUNSUPPORTED. */
    int key_words;
} gsparc_sink;

/* Statistics of one contraction (the reference prints these to stderr,
 * main.cu:384-433). Times are milliseconds of device time per stage. */
typedef struct {
    uint64_t ir_nnz;          /* matched products (indexMatch.cuh:285)        */
    uint64_t nnz;             /* output nonzeros ("Result NNZ")               */
    uint64_t nnz_x, nnz_y;
    uint64_t rows;            /* distinct X free indices                      */
    uint64_t heavy_rows;      /* rows taken by the windowed dense accumulator */
    uint64_t chunks;          /* output chunks streamed                       */
    int nbits_x, nbits_y, ncbits, nfbits_x, nfbits_y;
    int accumulator;          /* accumulator actually used (GSPARC_ACCUM_*)   */
    double t_linearize_ms;    /* SLITOM construction (linearise)              */
    double t_sort_ms;         /* SLITOM sort                                  */
    double t_match_ms;        /* index match + row table                      */
    double t_plan_ms;         /* symbolic pass + chunk planning               */
    double t_contract_ms;     /* numeric accumulation                         */
    double t_output_ms;       /* output delivery (copies, callbacks)          */
    double t_total_ms;
    uint64_t bytes_h2d, bytes_d2h;
    uint64_t kernel_launches; /* this library's own kernels launched           */
    double t_numeric_kernel_ms; /* device time of the numeric accumulation kernels */
    uint64_t heavy_windows;   /* column windows swept by the heavy-row accumulator */
    uint64_t stream_rows;     /* rows with one matched run, copied without accumulation */
    /* FP64 verification (gsparc_ctx_set_verify; all zero when it is off):
     * outputs compared with the FP64 sums of their exact products, formed on
     * the GPU.  No counterpart in the reference, which never inspects Z. */
    uint64_t verified_nnz;      /* outputs checked                               */
    uint64_t verified_products; /* matched products summed in FP64              */
    uint64_t verify_mismatch;   /* products whose output key is missing, NaNs   */
    uint64_t verify_skipped_rows; /* sampled rows past the FP64 scratch (unchecked) */
    double max_rel_err;         /* max |z - z64| / |z64| over checked z64 != 0   */
    double max_abs_err;         /* max |z - z64| over checked outputs            */
    uint64_t x_parts, y_parts;  /* operand parts (gsparc_sptc_host; 0 otherwise) */
    uint64_t kept_bitmap_bytes; /* heavy rows' column bitmaps kept from the symbolic to the numeric pass */
} gsparc_stats;

/* ---- version / errors ---------------------------------------------------- */
const char *gsparc_version(void);
const char *gsparc_status_string(gsparc_status st);
/* Message of the last failing call on this thread (empty if none). */
const char *gsparc_last_error(void);

/* ---- context -------------------------------------------------------------- */
/* Replaces CudaMemoryPool(id) (src/gsparc/cuda_memory.cpp:17-30), which
 * claimed all free HBM minus 256 MiB; the context instead admits device
 * allocations up to hbm_budget_bytes (0 = 90% of the device's free memory). */
gsparc_status gsparc_ctx_create(int device, uint64_t hbm_budget_bytes, gsparc_ctx **out);
gsparc_status gsparc_ctx_destroy(gsparc_ctx *ctx);
/* Map `bytes` of device memory (0 = the whole budget) into the context's pool
 * now and keep it there, so later contractions draw on memory that is already
 * mapped instead of growing the pool inside their own stages.  The reference
 * does the same once per run when its CudaMemoryPool takes all free HBM
 * (src/gsparc/cuda_memory.cpp:17-28), before any stage is timed.  Admission
 * against the budget is unchanged. */
gsparc_status gsparc_ctx_reserve(gsparc_ctx *ctx, uint64_t bytes);
/* Tiles of the accumulation for later contractions on this context (0 = the
 * defaults): rows with at most light_row_max matched products (<= 2048,
 * default 1024) take the on-chip ESC, larger rows the windowed accumulator,
 * whose windows hold at most heavy_window_cap outputs (256..8192, default
 * 8192).  gsparc_autotune times candidates of both.  No counterpart in the
 * reference, whose ESC and dense kernels have fixed launch shapes
 * (include/gsparc/contraction.cuh:287-290,469-472). */
gsparc_status gsparc_ctx_set_tiles(gsparc_ctx *ctx, uint64_t light_row_max, uint32_t heavy_window_cap);
/* Column bitmaps of heavy rows kept from the symbolic to the numeric pass
 * (on = 1, the default; 0 = every heavy window marks its columns from the
 * products).  The bitmaps (one bit per column rank over each heavy row's
 * span) of the heavy rows costing at most 512 bits per matched product are
 * kept when they fit an eighth of the memory left, else those costing at most
 * 32 bits, else none; the bytes used are in gsparc_stats.kept_bitmap_bytes.
 * Results are identical either
 * way.  No counterpart in the reference, whose ESC re-expands every product
 * (include/gsparc/contraction.cuh:440-561). */
gsparc_status gsparc_ctx_set_row_bitmaps(gsparc_ctx *ctx, int on);
/* Sort used for the operands' (key, value) pairs by later contractions and by
 * gsparc_sort_pairs on this context: 0 = CUB's onesweep radix sort (the
 * default; the reference sorts with CUB, include/gsparc/sort.cuh:90-108),
 * 1 = this library's own stable LSD radix sort (8 bits per pass: a digit
 * histogram per tile, a scan of the digit-major counts, a scatter ranked with
 * warp match).  Both are stable, so results are identical either way. */
gsparc_status gsparc_ctx_set_sort(gsparc_ctx *ctx, int impl);
/* FP64 verification of every later contraction on this context: each output
 * chunk's values are compared, before delivery, with FP64 sums of their
 * matched products formed on the GPU, for all rows when a contraction has at
 * most max_products matched products, else for a seeded sample of rows of
 * about that many products; results in gsparc_stats (max_rel_err, ...).
 * 0 turns it off (the default).  Costs one extra pass over the sampled
 * products per chunk; a plan's replayed chunks are not verified. */
gsparc_status gsparc_ctx_set_verify(gsparc_ctx *ctx, uint64_t max_products);
/* Host-side fault injection (tests of the error paths; no counterpart in the
 * reference, which exit()s on exhaustion, src/gsparc/cuda_memory.cpp:78): the
 * nth device allocation of this context from now (1 = the next) fails with
 * GSPARC_ENOMEM, once; 0 disarms.  The device is not involved. */
gsparc_status gsparc_ctx_inject_alloc_failure(gsparc_ctx *ctx, uint64_t nth);
/* Bytes currently allocated by the context and its high-water mark. */
gsparc_status gsparc_ctx_memory(gsparc_ctx *ctx, uint64_t *in_use, uint64_t *peak,
                                uint64_t *budget);

/* ---- resident operands ---------------------------------------------------- */
/* Copy (or adopt, when on_device) a COO tensor into the context.  Replaces the
 * H2D copies of SortSlitomXY / SpTC (include/gsparc/sort.cuh:79-107,
 * include/gsparc/sptc.cuh:86-91,128-134).  The tensor stays resident until
 * gsparc_tensor_free. */
gsparc_status gsparc_tensor_upload(gsparc_ctx *ctx, const gsparc_coo *coo, void *stream,
                                   gsparc_tensor **out);
gsparc_status gsparc_tensor_free(gsparc_ctx *ctx, gsparc_tensor *t);
gsparc_status gsparc_tensor_info(const gsparc_tensor *t, int *order, uint64_t *dims /*[32]*/,
                                 uint64_t *nnz);
/* Copy a resident tensor to host memory: idx SoA (idx[m*nnz + k], order*nnz
 * entries), val nnz entries.  The reference copies its result keys to the
 * host the same way (include/gsparc/contraction.cuh:554-561). */
gsparc_status gsparc_tensor_download(const gsparc_tensor *t, uint64_t *idx, float *val, void *stream);

/* ---- the contraction ------------------------------------------------------ */
/* Z = X x_{cx,cy} Y.  Replaces gsparc::SpTC (include/gsparc/sptc.cuh:16-360)
 * together with the TensorManager steps main.cu:293-321 runs before it
 * (ConvertTensor, SortSlitomXY, Partition).  cx[i] of X is contracted with
 * cy[i] of Y.  accum is GSPARC_ACCUM_*.  Work is ordered on `stream`;
 * the call returns after the last chunk was delivered. */
gsparc_status gsparc_sptc(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y,
                          int ncmodes, const int *cx, const int *cy, int accum,
                          const gsparc_sink *sink, gsparc_stats *stats, void *stream);

/* Row-sharded form for multi-GPU runs: only the X free indices (output rows)
 * of shard `shard` of `nshards` are contracted.  Shards split the rows at
 * equal matched-product mass; the union of all shards is Z, and shard s's
 * output keys all precede shard s+1's.  Replaces the round-robin X partition
 * over GPUs of include/gsparc/sptc.cuh:42-45. */
gsparc_status gsparc_sptc_shard(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y,
                                int ncmodes, const int *cx, const int *cy, int accum,
                                int shard, int nshards,
                                const gsparc_sink *sink, gsparc_stats *stats, void *stream);

/* Measured choice of how to run one contraction.  No counterpart in the
 * reference, whose accumulator rule is fixed (include/gsparc/sptc.cuh:201-218).
 * gsparc_autotune runs the contraction (output discarded) with each candidate
 * -- accumulator ESC or DENSE (rows of up to 1024 products by the on-chip ESC,
 * or every row by the windowed dense accumulator); then, for the better one,
 * the tiles (light_row_max 256 or 2048 instead of 1024, a heavy window of half
 * the outputs) and output chunks of the size the HBM budget allows, a quarter
 * of it and a sixteenth -- times each with CUDA events on `stream` and returns
 * the fastest.  The choice is remembered per operand shape (orders, dims,
 * nnz, contract modes) for the life of the process; a later call for the same
 * shape returns it without running anything unless `retune` is set.  Pass
 * accum and max_chunk_nnz to gsparc_sptc / a job's sink and the tiles to
 * gsparc_ctx_set_tiles.  The context's tiles are left as they were. */
typedef struct {
    int accum;              /* GSPARC_ACCUM_ESC or GSPARC_ACCUM_DENSE        */
    uint64_t max_chunk_nnz; /* 0 = from the HBM budget                       */
    double ms;              /* measured time of the choice                   */
    int cached;             /* 1: taken from the cache, nothing was run      */
    int ncandidates;
    int cand_accum[8];
    uint64_t cand_chunk[8];
    double cand_ms[8];
    uint64_t light_row_max;     /* chosen tiles (gsparc_ctx_set_tiles)             */
    uint32_t heavy_window_cap;
    uint64_t cand_light[8];
    uint32_t cand_cap[8];
} gsparc_tuning;
gsparc_status gsparc_autotune(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y,
                              int ncmodes, const int *cx, const int *cy, int retune,
                              gsparc_tuning *out, void *stream);

/* Z = X x_{cx,cy} Y kept on the device as a resident COO tensor: its modes
 * are X's free modes (ascending) followed by Y's free modes (ascending), and
 * it can be an operand of any later contraction (free it with
 * gsparc_tensor_free).  Replaces the reference's multi-SpTC chaining
 * (main.cu:323-371, include/gsparc/sptc.cuh:362-698), which keeps the first
 * result's keys and reuses them as the next contraction's X keys.  Z must fit
 * the context's budget (12 B per output nonzero while collecting, then
 * 8 B per mode + 4 B per nonzero). */
gsparc_status gsparc_sptc_resident(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y,
                                   int ncmodes, const int *cx, const int *cy, int accum,
                                   gsparc_tensor **Z, gsparc_stats *stats, void *stream);

/* One contraction of a batch: the arguments of gsparc_sptc plus per-job
 * results. */
typedef struct {
    const gsparc_tensor *x, *y;
    int ncmodes;
    const int *cx, *cy;
    int accum;             /* GSPARC_ACCUM_*                                   */
    gsparc_sink sink;      /* this job's output; `first` counts from the job's
                            * first output nonzero.  max_chunk_nnz caps the
                            * pieces handed to a DEVICE sink's callback.      */
    gsparc_stats stats;    /* out: this job's counts; stage times are the
                            * batch's (the job's latency)                     */
    gsparc_status status;  /* out: GSPARC_OK or why this job failed           */
} gsparc_job;

/* Many independent contractions as one.  The reference runs gsparc::SpTC
 * (include/gsparc/sptc.cuh:16-360) once per contraction from main.cu:293-376;
 * here every job's keys carry the job id in their top bits, so a group of
 * jobs shares one linearise, one sort per side, one match and one symbolic +
 * one numeric persistent launch.  Each job's output (keys, values, nnz) is
 * exactly what gsparc_sptc returns for that job alone.  Jobs are grouped so
 * that every group's prefixed keys fit 64 bits.  A job that fails (bad
 * argument, out-of-range index) fails alone: its status says why and its sink
 * gets nothing; the call then returns the first failing job's status.
 * max_chunk_nnz (0 = from the HBM budget) bounds the output held in HBM at
 * once, across the jobs of a group. */
gsparc_status gsparc_sptc_batch(gsparc_ctx *ctx, gsparc_job *jobs, int njobs, uint64_t max_chunk_nnz,
                                gsparc_stats *stats, void *stream);

/* ---- plans: coordinates once, values many times -------------------------- */
/* No counterpart in the reference, which redoes every step per call.  A plan
 * does, once, everything of a set of contractions that depends only on the
 * operands' coordinates -- linearise, sort, run table, match, row planning,
 * the symbolic pass and the output chunks (at most max_chunk_nnz outputs each,
 * 0 = from the HBM budget) -- and keeps it on the device.  Executing a chunk
 * runs only the numeric pass into caller-provided device arrays: memsets and
 * kernel launches on `stream`, no allocation, no host synchronisation, so a
 * caller may capture its executions in a CUDA graph and replay them.
 * gsparc_plan_refresh fetches the operands' current values (after
 * gsparc_tensor_set_values); the coordinates must stay those the plan was
 * made from.  The plan holds the context's memory until destroyed; destroy it
 * before the context and the tensors.  The jobs' sinks are ignored; job i's
 * output is the range gsparc_plan_job_output gives of the plan's output,
 * whose chunks are consecutive. */
typedef struct gsparc_plan gsparc_plan;
gsparc_status gsparc_plan_create(gsparc_ctx *ctx, const gsparc_job *jobs, int njobs, uint64_t max_chunk_nnz,
                                 gsparc_plan **out, uint64_t *total_nnz, void *stream);
/* Number of output chunks, and chunk k's first output and size. */
gsparc_status gsparc_plan_chunks(const gsparc_plan *plan, uint64_t *nchunks);
gsparc_status gsparc_plan_chunk(const gsparc_plan *plan, uint64_t k, uint64_t *first, uint64_t *nnz);
/* Job i's output: `first` (in the plan's output) and nnz. */
gsparc_status gsparc_plan_job_output(const gsparc_plan *plan, int job, uint64_t *first, uint64_t *nnz);
gsparc_status gsparc_plan_refresh(gsparc_plan *plan, void *stream);
/* Chunk k into d_keys/d_vals (device arrays of at least the chunk's size). */
gsparc_status gsparc_plan_execute(gsparc_plan *plan, uint64_t k, uint64_t *d_keys, float *d_vals,
                                  uint64_t capacity, void *stream);
/* Waits for `stream`; reports (and clears) a device-side check that failed in
 * the executions since the last check. */
gsparc_status gsparc_plan_check(gsparc_plan *plan, void *stream);
gsparc_status gsparc_plan_destroy(gsparc_plan *plan);
/* Overwrite a resident tensor's values (nnz of them, in the order of the COO
 * it was uploaded from; host or device memory), coordinates unchanged. */
gsparc_status gsparc_tensor_set_values(gsparc_ctx *ctx, gsparc_tensor *t, const float *val, int on_device,
                                       void *stream);

/* ---- serving: a request loop over resident operands ----------------------- */
/* No counterpart in the reference, which runs one contraction per process
 * (main.cu:22-437).  A server owns one device, an HBM budget shared by its
 * resident operands and the working memory of the contractions in flight,
 * and `lanes` worker threads, each with its own CUDA stream.  A free lane
 * takes waiting requests, as many as the free budget and the batch limits
 * admit, and runs them as one gsparc_sptc_batch; requests that arrive
 * meanwhile wait for the next free lane, so batches of different lanes
 * overlap on the device.  Small requests go first unless one has waited
 * longer than age_ms (shortest first with ageing), so a small request is not
 * queued behind a large one that arrived just before it.  A request whose
 * output does not fit the HBM
 * budget streams it in chunks like gsparc_sptc.  Submit, poll, wait, stats
 * and upload may be called from any thread.  gsparc_serve_create maps the
 * whole budget into the server's memory pool once (as gsparc_ctx_reserve
 * does for a context), so no batch waits for the pool to grow. */
typedef struct gsparc_server gsparc_server;

typedef struct {
    uint64_t hbm_budget_bytes; /* resident operands + work in flight (0 = 90% of free HBM) */
    int lanes;                 /* worker threads / streams (0 = 2)                          */
    int max_batch_jobs;        /* requests per batch (0 = 256)                              */
    uint64_t max_batch_nnz;    /* operand nonzeros per batch, X + Y (0 = 2^24); a request
                                * larger than this runs in a batch of its own              */
    int fifo;                  /* 1: admit in arrival order.  0: requests that waited
                                * longer than age_ms first, in arrival order, then the
                                * others smallest first (fewest operand nonzeros)          */
    double age_ms;             /* 0 = 200 ms                                                */
    uint64_t max_chunk_nnz;    /* output nonzeros per chunk (0 = 2^28): bounds the output
                                * buffers a lane holds, larger outputs stream through     */
} gsparc_server_opts;

typedef struct {
    uint64_t submitted, completed, failed;
    uint64_t batches;          /* batches run                                               */
    uint64_t max_batch;        /* most requests in one batch                                */
    uint64_t ir_nnz, nnz;      /* matched products / output nonzeros of completed requests  */
    double p50_ms, p99_ms;     /* latency: submission to result delivered                   */
    double mean_ms, max_ms;
    double wall_ms;            /* first submission to last completion                       */
    double products_per_s;     /* ir_nnz / wall                                             */
    uint64_t resident_bytes;   /* operands held by the server                               */
    uint64_t peak_reserved_bytes; /* largest working memory admitted at once                */
    uint64_t max_in_flight;    /* most batches running at once                              */
    uint64_t retries;          /* requests rerun alone after their batch ran out of memory  */
    uint64_t chunks;           /* output chunks delivered, over all completed requests      */
} gsparc_server_stats;

gsparc_status gsparc_serve_create(int device, const gsparc_server_opts *opts, gsparc_server **out);
/* Waits for every submitted request, then stops the lanes and frees all
 * resident operands. */
gsparc_status gsparc_serve_destroy(gsparc_server *srv);
/* Upload an operand that stays resident in the server's budget; requests name
 * it by the returned handle.  Release frees it once no waiting or running
 * request uses it. */
gsparc_status gsparc_serve_upload(gsparc_server *srv, const gsparc_coo *coo, gsparc_tensor **out);
gsparc_status gsparc_serve_release(gsparc_server *srv, gsparc_tensor *t);
/* Queue one contraction.  The job is copied (cx/cy included); its sink, the
 * sink's buffers and callback must stay valid until the request completes.
 * The sink's callbacks run on a lane thread. */
gsparc_status gsparc_serve_submit(gsparc_server *srv, const gsparc_job *job, uint64_t *ticket);
/* done = 1 once the request completed; result (optional) then receives the
 * job with its status and stats.  Poll does not block. */
gsparc_status gsparc_serve_poll(gsparc_server *srv, uint64_t ticket, int *done, gsparc_job *result);
/* Block until the request completes or timeout_ms passes (< 0: no limit;
 * GSPARC_ETIMEOUT if it did not complete).  The ticket is retired after a
 * completed wait. */
gsparc_status gsparc_serve_wait(gsparc_server *srv, uint64_t ticket, double timeout_ms, gsparc_job *result);
gsparc_status gsparc_serve_stats(gsparc_server *srv, gsparc_server_stats *out);
/* Forget the latency samples and counters (after a warm-up). */
gsparc_status gsparc_serve_reset_stats(gsparc_server *srv);
/* Hold (paused != 0) or resume the lanes: while paused no lane starts a new
 * batch (running batches finish); submitted requests wait. */
gsparc_status gsparc_serve_pause(gsparc_server *srv, int paused);
/* Host-side fault injection: arms every lane's allocator so that its nth
 * device allocation from now fails with GSPARC_ENOMEM, once (0 disarms). */
gsparc_status gsparc_serve_inject_alloc_failure(gsparc_server *srv, uint64_t nth);

/* ---- host helpers (no GPU needed) ---------------------------------------- */
/* Parse a .tns file: 1-based text COO, one nonzero per line, order = tokens of
 * the first line minus one, dims[m] = largest index + 1.  Replaces
 * IOManager::ParseFromFile / parse_metadata_and_data
 * (include/gsparc/io_manager.tpp:24-34,75-259).  Arrays are malloc'd by the
 * library (free with gsparc_free_host); idx is SoA: idx[m*nnz + k]. */
gsparc_status gsparc_read_tns(const char *path, int nthreads, int *order, uint64_t *dims /*[32]*/,
                              uint64_t *nnz, uint64_t **idx, float **val);
/* Parse the quantum-chemistry directory format (the reference's -q):
 * <dir>/indices.txt holds one line per mode with the 1-based indices of all
 * nonzeros, <dir>/values.txt the values.  Replaces IOManager::_ReadQuantumData
 * (include/gsparc/io_manager.tpp:310-484).  Output arrays as gsparc_read_tns. */
gsparc_status gsparc_read_quantum(const char *dir, int nthreads, int *order, uint64_t *dims /*[32]*/,
                                  uint64_t *nnz, uint64_t **idx, float **val);
/* Write 1-based text COO with %.9g values. */
gsparc_status gsparc_write_tns(const char *path, int order, uint64_t nnz,
                               const uint64_t *idx /* SoA idx[m*nnz+k] */, const float *val);
void gsparc_free_host(void *p);
/* Page-lock an existing host buffer in place (gsparc_host_unpin releases it),
 * so uploads from it run at the full host-link rate.  The reference keeps its
 * converted operands in page-locked memory (cudaHostAlloc in
 * include/gsparc/tensor_manager.tpp:223-224); the CLI pins what it read. */
gsparc_status gsparc_host_pin(void *p, uint64_t bytes);
gsparc_status gsparc_host_unpin(void *p);

/* Bit layout of one operand.  Replaces TensorManager::compute_nbtis,
 * setup_slitom and create_mask (include/gsparc/tensor_manager.tpp:91-210):
 * bits[m] = 64 - clz(dims[m]-1) (0 for size-1 modes), free modes in
 * ascending order, the first free (contract) mode in the highest bits.
 * shift[m] is the position of mode m inside its part. */
gsparc_status gsparc_layout(int order, const uint64_t *dims, int ncmodes, const int *cmodes,
                            int *bits, int *shift, int *is_contract,
                            int *ncbits, int *nfbits);

/* Split rows into nshards ranges of near-equal product mass: row_prod[r] is
 * the matched products of row r; bounds gets nshards+1 row indices. */
gsparc_status gsparc_plan_shards(const uint64_t *row_prod, uint64_t nrows, int nshards,
                                 uint64_t *bounds);

/* ---- stage entry points (device pointers, for parity tests) -------------- */
/* Linearise one operand into 64-bit keys.  role 0 = X layout
 * (free << ncbits | contract), role 1 = Y layout (contract << nfbits | free).
 * Replaces TensorManager::ConvertTensor (include/gsparc/tensor_manager.tpp:213-298),
 * whose host pdep loop becomes a device kernel.  d_idx is SoA on the device:
 * d_idx[m*nnz + k]. */
gsparc_status gsparc_linearize(int order, const uint64_t *dims, int ncmodes, const int *cmodes,
                               int role, uint64_t nnz, const uint64_t *d_idx,
                               uint64_t *d_keys, void *stream);

/* Stable sort of (key, value) pairs by the low `nbits` bits of the key.
 * Replaces sort_64 (include/gsparc/sort.cuh:40-159).  In place. */
gsparc_status gsparc_sort_pairs(gsparc_ctx *ctx, uint64_t n, uint64_t *d_keys, float *d_vals,
                                int nbits, void *stream);

/* For sorted X keys and sorted Y keys: pos[i] = first Y index whose contract
 * key equals X[i]'s, cnt[i] = length of that run (0 and 0 if none),
 * prefix[0] = 0, prefix[i+1] = prefix[i] + cnt[i]; *ir = prefix[nx].
 * Replaces IndexMatch / compute_result_size_cuda
 * (include/gsparc/indexMatch.cuh:67-118,231-287). */
gsparc_status gsparc_index_match(gsparc_ctx *ctx, uint64_t nx, const uint64_t *d_xkeys,
                                 int x_ncbits, uint64_t ny, const uint64_t *d_ykeys,
                                 int y_nfbits, uint64_t *d_pos, uint64_t *d_cnt,
                                 uint64_t *d_prefix, uint64_t *ir, void *stream);

/* The same index match for callers that cannot allocate device memory:
 * hosts whose own allocator owns all of the GPU's memory and forbids other
 * allocations, and latency-critical paths that must not enter the driver's
 * allocator (which can synchronise the device).  It needs no context and
 * calls no cudaMalloc/cudaFree or other allocating routine: its scratch (Y's
 * run table and CUB's temporary storage) is one 64 MiB file-scope device
 * array that every GPU loading the library holds until exit.  A call needs
 * about 13 bytes per Y key plus CUB temporary storage that grows with nx
 * (Y up to roughly 4.9 million keys for small X); larger inputs return
 * GSPARC_EINVAL with the bytes needed in gsparc_last_error().  The first call
 * on each device looks the array's address up (cudaGetSymbolAddress) with
 * that device current.  `stream` must belong to the current device
 * (GSPARC_EINVAL otherwise).  With ir == NULL the call does not wait: the total stays in
 * d_prefix[nx]; otherwise it waits for the stream and stores the total.
 * All calls on a device share the array, so calls that overlap on the GPU
 * race and must be serialised by the caller; nothing is carried over between
 * calls.  No counterpart in the reference (its IndexMatch allocates from its
 * pool, include/gsparc/indexMatch.cuh:270-286). */
gsparc_status gsparc_index_match_noalloc(uint64_t nx, const uint64_t *d_xkeys, int x_ncbits,
                                         uint64_t ny, const uint64_t *d_ykeys, int y_nfbits,
                                         uint64_t *d_pos, uint64_t *d_cnt, uint64_t *d_prefix,
                                         uint64_t *ir, void *stream);

/* ---- operands larger than the HBM budget ---------------------------------- */
/* Part sizes for gsparc_sptc_host (0 = derived from the context's budget). */
typedef struct {
    uint64_t max_part_nnz_x;  /* at most this many X nonzeros per X part       */
    uint64_t max_part_nnz_y;  /* at most this many Y nonzeros per Y part       */
} gsparc_part_opts;
/* Z = X x Y for operands in HOST memory that need not fit the budget.  X is
 * cut into parts at output-row ranges (X free index), Y into parts at
 * output-column ranges (Y free index), each part gathered on the host and
 * uploaded with the operand's dims; every (X part, Y part) pair is contracted
 * and Z reaches the sink in key order (with several Y parts the outputs of
 * one X part are merged on the host).  A single row or column is never split.
 * Replaces FindPartitionNum / Partition / convert_and_sort and the part loop
 * of SpTC (include/gsparc/tensor_manager.tpp:33-61,634-886,
 * include/gsparc/sptc.cuh:42-139).  HOST sinks receive pieces in place while
 * Z fits their arrays, in ring mode beyond; stats count the parts. */
gsparc_status gsparc_sptc_host(gsparc_ctx *ctx, const gsparc_coo *X, const gsparc_coo *Y, int ncmodes,
                               const int *cx, const int *cy, int accum, const gsparc_part_opts *opts,
                               const gsparc_sink *sink, gsparc_stats *stats, void *stream);

/* ---- verification digest of an output chunk ------------------------------ */
/* Order-independent digest of n output nonzeros on the device: count, a sum
 * of mixed keys, how many neighbours are not strictly increasing, the first
 * and last key, and the values summed in double precision.  Used to verify
 * outputs too large to bring to the host.  No counterpart in the reference
 * (which never inspects its output). */
typedef struct {
    uint64_t n;
    uint64_t key_hash;      /* sum over keys of splitmix64(key), mod 2^64      */
    uint64_t unsorted;      /* #i with keys[i] >= keys[i+1]                    */
    uint64_t first_key, last_key;
    double val_sum;         /* sum of values (double)                         */
    double val_abs_sum;     /* sum of |values| (double)                       */
} gsparc_digest;
gsparc_status gsparc_digest_chunk(const uint64_t *d_keys, const float *d_vals, uint64_t n,
                                  gsparc_digest *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GSPARC_B200_H */
