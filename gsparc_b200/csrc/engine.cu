// engine.cu -- host-side row-shard planning.
//
// The contraction itself (the reference's gsparc::SpTC, include/gsparc/sptc.cuh:16-360,
// plus the TensorManager steps main.cu:293-321) runs in batch.cu: a single
// contraction is a batch of one job.
#include "engine.h"

namespace gs {

// Shard s of n starts at the first row whose product midpoint reaches s/n of
// all products: the first r with n * (P[r] + P[r+1]) >= 2 * s * P[nrows], P
// the row product prefix.  Exact integer arithmetic, so the device planner of
// a sharded contraction (batch.cu, shard_bound) finds the same rows.
// Replaces the round-robin X partition over GPUs of include/gsparc/sptc.cuh:42-45.
void plan_shards(const uint64_t *row_prod, uint64_t nrows, int nshards, uint64_t *bounds) {
    GS_REQUIRE(nshards >= 1, GSPARC_EINVAL, "nshards must be >= 1");
    std::vector<uint64_t> P(nrows + 1, 0);
    for (uint64_t r = 0; r < nrows; ++r) P[r + 1] = P[r] + row_prod[r];
    bounds[0] = 0;
    for (int s = 1; s < nshards; ++s) {
        const unsigned __int128 target = (unsigned __int128)2 * (unsigned)s * P[nrows];
        uint64_t lo = 0, hi = nrows;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if ((unsigned __int128)(unsigned)nshards * ((unsigned __int128)P[mid] + P[mid + 1]) >= target)
                hi = mid;
            else
                lo = mid + 1;
        }
        bounds[s] = lo;
    }
    bounds[nshards] = nrows;
}

}  // namespace gs
