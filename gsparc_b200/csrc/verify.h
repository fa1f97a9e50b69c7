// verify.h -- FP64 verification of output chunks on the device (verify.cu).
#pragma once

#include <cstdint>
#include <cstring>

#include "kernels.cuh"

namespace gs {

struct VerifyEntry {
    uint32_t row;
    uint32_t pad;
    uint64_t off;  // first FP64 accumulator of the row
};

// Per-job results, accumulated over the job's chunks on the device.
struct VerifyOut {
    unsigned long long max_rel_bits, max_abs_bits;  // doubles (non-negative) as bits
    unsigned long long nnz, products, mismatch, skipped, nan_values, pad;
};

struct VerifyState {
    VerifyEntry *list = nullptr;     // [nrows]
    unsigned long long *cnt = nullptr;  // [0] listed rows, [1] accumulators handed out
    double *acc = nullptr;           // [acc_cap]
    uint64_t acc_cap = 0;
    VerifyOut *out = nullptr;        // [jobs of the group]
    uint64_t threshold = 0;          // rows with (mix(row ^ salt) >> 32) < threshold; ~0 = every row
    uint64_t salt = 0;
};

// The row-sampling threshold for a verify budget of `budget` products
// (0: off) on a contraction of `products` matched products.
uint64_t verify_threshold(uint64_t budget, uint64_t products);

// Checks the rows of output chunk [c0, c1) (keys/vals: the chunk buffer).
void verify_chunk(const AccArgs &a, VerifyState &vs, uint64_t nrows, uint64_t c0, uint64_t c1,
                  const uint64_t *keys, const float *vals, cudaStream_t s);

// Adds one job's results to its statistics.
void verify_fill_stats(const VerifyOut &o, gsparc_stats &st);

}  // namespace gs
