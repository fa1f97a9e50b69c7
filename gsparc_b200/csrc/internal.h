// internal.h -- host-side internals shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "gsparc_b200.h"

namespace gs {

constexpr int kMaxOrder = 32;

// Errors travel as exceptions inside the library and become status codes at
// the C ABI boundary (capi.cpp).
struct Error {
    gsparc_status st;
    std::string msg;
};

[[noreturn]] void fail(gsparc_status st, const std::string &msg);
// Count of this library's own kernel launches (process-wide).
void count_launch(uint64_t n = 1);
uint64_t launch_count();
void set_last_error(const std::string &msg);
const char *last_error();

#define GS_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            ::gs::fail(GSPARC_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define GS_REQUIRE(cond, st, msg)        \
    do {                                 \
        if (!(cond))                     \
            ::gs::fail((st), (msg));     \
    } while (0)

// Bit layout of one operand (reference: include/gsparc/tensor_manager.tpp:91-210).
struct Layout {
    int order = 0;
    int nc = 0;
    int bits[kMaxOrder] = {};
    int shift[kMaxOrder] = {};
    int is_c[kMaxOrder] = {};
    int cpos[kMaxOrder] = {};
    int ncbits = 0;
    int nfbits = 0;
    int nbits() const { return ncbits + nfbits; }
};

int mode_bits(uint64_t dim);
Layout make_layout(int order, const uint64_t *dims, int nc, const int *cmodes);

// Device memory admitted against a byte budget.  Backed by a private
// stream-ordered memory pool, so freeing a buffer on the stream that used it
// makes it reusable by later work on that stream without a device sync.
// (Replaces the reference's first-fit CudaMemoryPool, which grabbed all free
// HBM minus 256 MiB and exited on exhaustion: src/gsparc/cuda_memory.cpp:17-80.)
class Arena {
public:
    Arena() = default;
    ~Arena();
    void init(int device, uint64_t budget);
    // Draw from a pool owned elsewhere (several arenas on one pool, each with
    // its own budget); the pool outlives the arena.
    void init_shared(int device, cudaMemPool_t pool, uint64_t budget);
    void set_budget(uint64_t budget) { budget_ = budget; }
    // Map `bytes` (whole 2 MiB pages; 0 = the budget) into the pool now and keep
    // them there: one allocation of that size freed at once (the pool's release
    // threshold is unbounded), so later allocations carve mapped memory instead
    // of growing the pool in the middle of a contraction.
    void reserve(uint64_t bytes, cudaStream_t s);
    void reset_peak() { peak_ = in_use_; }
    void *alloc(size_t bytes, cudaStream_t s);
    void free(void *p, cudaStream_t s);
    uint64_t in_use() const { return in_use_; }
    uint64_t peak() const { return peak_; }
    uint64_t budget() const { return budget_; }
    // Host-side fault injection: the nth allocation from now (1 = the next)
    // fails with GSPARC_ENOMEM, once; 0 disarms.  Nothing touches the device.
    void inject_failure(uint64_t nth) { fail_in_.store(nth); }
    uint64_t available() const { return budget_ > in_use_ ? budget_ - in_use_ : 0; }
    int device() const { return device_; }
    cudaMemPool_t pool() const { return pool_; }

private:
    int device_ = -1;
    cudaMemPool_t pool_ = nullptr;
    bool owns_pool_ = false;
    uint64_t budget_ = 0, in_use_ = 0, peak_ = 0;
    std::unordered_map<void *, size_t> sizes_;
    std::atomic<uint64_t> fail_in_{0};
};

// RAII device buffer from an Arena.
template <class T>
class DBuf {
public:
    DBuf() = default;
    DBuf(Arena &a, size_t n, cudaStream_t s) { reset(a, n, s); }
    ~DBuf() { release(); }
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept { *this = std::move(o); }
    DBuf &operator=(DBuf &&o) noexcept {
        if (this != &o) {
            release();
            a_ = o.a_; p_ = o.p_; n_ = o.n_; s_ = o.s_;
            o.a_ = nullptr; o.p_ = nullptr; o.n_ = 0;
        }
        return *this;
    }
    void reset(Arena &a, size_t n, cudaStream_t s) {
        release();
        a_ = &a; s_ = s; n_ = n;
        p_ = static_cast<T *>(a.alloc(sizeof(T) * (n ? n : 1), s));
    }
    void release() {
        if (a_ && p_) a_->free(p_, s_);
        a_ = nullptr; p_ = nullptr; n_ = 0;
    }
    T *get() const { return p_; }
    size_t size() const { return n_; }
    operator T *() const { return p_; }

private:
    Arena *a_ = nullptr;
    T *p_ = nullptr;
    size_t n_ = 0;
    cudaStream_t s_ = nullptr;
};

}  // namespace gs

struct gsparc_ctx {
    int device = 0;
    gs::Arena arena;
    int sm_count = 148;
    cudaEvent_t ev[16] = {};
    unsigned int *d_flag = nullptr;  // device error / work counters
    cudaStream_t copy_stream = nullptr;  // output chunk copies (non-blocking)
    cudaStream_t alt_stream = nullptr;   // every other output chunk's kernels (non-blocking)
    uint64_t verify_budget = 0;          // FP64 verification of outputs (0: off)
    uint64_t light_row_max = 0;          // rows with at most this many products use the on-chip ESC (0: default)
    uint32_t heavy_window_cap = 0;       // heavy rows: outputs per window (0: the compiled capacity)
    int keep_row_bitmaps = 1;            // heavy rows: the symbolic pass keeps column bitmaps for the numeric pass
    int sort_impl = 0;                   // operand sorts: 0 CUB onesweep, 1 this library's radix sort (radix.cu)
};

struct gsparc_tensor {
    int order = 0;
    uint64_t dims[gs::kMaxOrder] = {};
    uint64_t nnz = 0;
    uint64_t *d_idx = nullptr;  // SoA, order * nnz
    float *d_val = nullptr;
    bool owned = true;
};
