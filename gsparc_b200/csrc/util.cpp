// util.cpp -- errors, bit layout, budgeted device arena.
#include <atomic>
#include <cstring>
#include <mutex>

#include "internal.h"

namespace gs {

static thread_local std::string g_last_error;

void fail(gsparc_status st, const std::string &msg) { throw Error{st, msg}; }

static std::atomic<uint64_t> g_launches{0};
void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
void set_last_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

// reference: include/gsparc/tensor_manager.tpp:109 (64 - clz(dim-1)); a size-1
// mode takes 0 bits here (clz(0) is undefined in the reference).
int mode_bits(uint64_t dim) { return dim <= 1 ? 0 : 64 - __builtin_clzll(dim - 1); }

// reference: include/gsparc/tensor_manager.tpp:64-88 (free modes ascending) and
// :153-174 (the last free / contract mode in the lowest bits, the first one in
// the highest).
Layout make_layout(int order, const uint64_t *dims, int nc, const int *cmodes) {
    GS_REQUIRE(order >= 1 && order <= kMaxOrder, GSPARC_EINVAL, "order must be in 1..32");
    GS_REQUIRE(nc >= 0 && nc <= order, GSPARC_EINVAL, "bad number of contract modes");
    Layout L;
    L.order = order;
    L.nc = nc;
    for (int i = 0; i < nc; ++i) {
        int m = cmodes[i];
        GS_REQUIRE(m >= 0 && m < order, GSPARC_EINVAL, "contract mode out of range");
        GS_REQUIRE(!L.is_c[m], GSPARC_EINVAL, "contract mode listed twice");
        L.is_c[m] = 1;
        L.cpos[i] = m;
    }
    int fpos[kMaxOrder], nf = 0;
    for (int m = 0; m < order; ++m) {
        GS_REQUIRE(dims[m] >= 1, GSPARC_EINVAL, "mode size must be >= 1");
        L.bits[m] = mode_bits(dims[m]);
        if (!L.is_c[m]) fpos[nf++] = m;
    }
    int s = 0;
    for (int n = nf - 1; n >= 0; --n) {
        L.shift[fpos[n]] = s;
        s += L.bits[fpos[n]];
    }
    L.nfbits = s;
    s = 0;
    for (int n = nc - 1; n >= 0; --n) {
        L.shift[L.cpos[n]] = s;
        s += L.bits[L.cpos[n]];
    }
    L.ncbits = s;
    return L;
}

Arena::~Arena() {
    if (pool_ && owns_pool_) {
        // Outstanding buffers belong to objects that are being torn down too.
        cudaMemPoolDestroy(pool_);
    }
}

void Arena::init(int device, uint64_t budget) {
    device_ = device;
    budget_ = budget;
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    GS_CUDA(cudaMemPoolCreate(&pool_, &props));
    owns_pool_ = true;
    uint64_t thr = UINT64_MAX;
    GS_CUDA(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &thr));
}

void Arena::reserve(uint64_t bytes, cudaStream_t s) {
    uint64_t n = bytes ? std::min<uint64_t>(bytes, budget_) : budget_;
    n &= ~((uint64_t(1) << 21) - 1);
    if (n == 0) return;
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, n, pool_, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? GSPARC_ENOMEM : GSPARC_ECUDA,
             std::string("reserving ") + std::to_string(n) + " B failed: " + cudaGetErrorString(e));
    }
    GS_CUDA(cudaFreeAsync(p, s));
    GS_CUDA(cudaStreamSynchronize(s));
}

void Arena::init_shared(int device, cudaMemPool_t pool, uint64_t budget) {
    device_ = device;
    budget_ = budget;
    pool_ = pool;
    owns_pool_ = false;
}

void *Arena::alloc(size_t bytes, cudaStream_t s) {
    bytes = (bytes + 255) & ~size_t(255);
    for (uint64_t f = fail_in_.load(); f != 0;) {
        if (fail_in_.compare_exchange_weak(f, f - 1)) {
            if (f == 1) fail(GSPARC_ENOMEM, "injected allocation failure (" + std::to_string(bytes) + " B)");
            break;
        }
    }
    if (in_use_ + bytes > budget_)
        fail(GSPARC_ENOMEM, "HBM budget exhausted: need " + std::to_string(bytes) + " B, " +
                                std::to_string(available()) + " B left of " + std::to_string(budget_));
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool_, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? GSPARC_ENOMEM : GSPARC_ECUDA,
             std::string("device allocation of ") + std::to_string(bytes) + " B failed: " +
                 cudaGetErrorString(e));
    }
    sizes_[p] = bytes;
    in_use_ += bytes;
    if (in_use_ > peak_) peak_ = in_use_;
    return p;
}

void Arena::free(void *p, cudaStream_t s) {
    if (!p) return;
    auto it = sizes_.find(p);
    if (it == sizes_.end()) return;
    in_use_ -= it->second;
    sizes_.erase(it);
    cudaFreeAsync(p, s);
}

}  // namespace gs
