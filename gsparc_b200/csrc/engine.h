// engine.h -- entry points of the contraction engine (C++ side of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <functional>

#include "internal.h"

namespace gs {

// Called once per job as soon as the job's whole output was delivered to its
// sink (or it failed); the job's status and counts are final by then.
using JobDoneFn = std::function<void(gsparc_job *)>;

// Many contractions as one (batch.cu).  A single contraction is a batch of one;
// shard/nshards restrict a single job to one row shard (multi-GPU runs).  With
// done_fn, jobs complete one by one: the numeric pass is cut into chunks at job
// boundaries of geometrically growing product counts, so a job finishes
// when the chunks holding its rows are delivered, not at the end of the batch.
void sptc_batch(gsparc_ctx *ctx, gsparc_job *jobs, int njobs, uint64_t max_chunk_nnz, gsparc_stats *st,
                cudaStream_t s, int shard = 0, int nshards = 1, const JobDoneFn *done_fn = nullptr);

// Z = X x Y with operands in host memory, cut into parts that fit the budget
// (partition.cpp).
void sptc_partitioned(gsparc_ctx *ctx, const gsparc_coo *X, const gsparc_coo *Y, int nc, const int *cx,
                      const int *cy, int accum, const gsparc_part_opts *opts, const gsparc_sink *sink,
                      gsparc_stats *stats, cudaStream_t s);

// Z = X x Y decoded into a resident COO tensor (chain.cu).
void sptc_resident(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y, int nc, const int *cx,
                   const int *cy, int accum, gsparc_tensor **out, gsparc_stats *stats, cudaStream_t s);

// Plans (batch.cu): coordinate-only work done once, the numeric pass replayed.
void plan_create(gsparc_ctx *ctx, const gsparc_job *jobs, int njobs, uint64_t max_chunk_nnz, gsparc_plan **out,
                 uint64_t *total, cudaStream_t s);
void plan_refresh(gsparc_plan *P, cudaStream_t s);
void plan_execute(gsparc_plan *P, uint64_t chunk, uint64_t *keys, float *vals, uint64_t capacity, cudaStream_t s);
void plan_check(gsparc_plan *P, cudaStream_t s);
void plan_destroy(gsparc_plan *P);
uint64_t plan_nchunks(const gsparc_plan *P);
void plan_chunk(const gsparc_plan *P, uint64_t k, uint64_t *first, uint64_t *nnz);
void plan_job_output(const gsparc_plan *P, int job, uint64_t *first, uint64_t *nnz);

void plan_shards(const uint64_t *row_prod, uint64_t nrows, int nshards, uint64_t *bounds);

// .tns text I/O (tns_io.cpp)
void read_tns(const char *path, int nthreads, int *order, uint64_t *dims, uint64_t *nnz,
              uint64_t **idx, float **val);
void write_tns(const char *path, int order, uint64_t nnz, const uint64_t *idx, const float *val);
void read_quantum(const char *dir, int nthreads, int *order, uint64_t *dims, uint64_t *nnz, uint64_t **idx,
                  float **val);

}  // namespace gs
