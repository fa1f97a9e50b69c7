// noalloc.cu -- the index-match stage for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: hosts that hand the whole GPU memory to
// their own allocator and forbid any other allocation (a runtime that carves
// its arena at start-up and accounts every byte), and latency-critical paths
// that must not enter the driver's allocator, which can synchronise the device
// and take driver locks.  gsparc_index_match_noalloc does the same work as
// gsparc_index_match, but its scratch (the run table of Y's contract keys and
// CUB's temporary storage) lives in one file-scope __device__ array of
// kScratchBytes that every GPU loading this library holds until the process
// exits.  Inputs and outputs stay caller-owned.
//
// The array's host-side name is only a stand-in; its device address is looked
// up once per device with cudaGetSymbolAddress (with that device current) on
// the first call made on that device.  `stream` must belong to the current
// device (checked).
// Every call on a device shares the one array: calls whose work overlaps on
// the GPU (different streams, or different host threads) race on it and must
// be serialised by the caller.  No scratch content is carried from one call to
// the next: every byte a call reads is written by that call (the run count is
// cleared first).
#include <cub/cub.cuh>

#include <exception>
#include <mutex>
#include <new>
#include <string>

#include "internal.h"

namespace gs {
namespace {

constexpr size_t kScratchBytes = 64ull << 20;  // 64 MiB per device
constexpr int kThreads = 256;

static __device__ __align__(256) unsigned char g_match_scratch[kScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_addr[256] = {};

void *scratch_on_current_device() {
    int dev = -1;
    GS_CUDA(cudaGetDevice(&dev));
    GS_REQUIRE(dev >= 0 && dev < 256, GSPARC_EUNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        GS_CUDA(cudaGetSymbolAddress(&p, g_match_scratch));
        g_scratch_addr[dev] = p;
    }
    return g_scratch_addr[dev];
}

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

inline int grid_for(uint64_t n) {
    uint64_t g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    if (g > 148ull * 32) g = 148ull * 32;
    return (int)g;
}

__device__ __forceinline__ uint64_t shr(uint64_t v, int s) { return s >= 64 ? 0ull : (v >> s); }

// run boundaries of Y's contract key (ykeys sorted, contract key = key >> nfb)
__global__ void k_na_flags(const uint64_t *__restrict__ ykeys, uint64_t ny, int nfb, uint8_t *__restrict__ flag) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ny; j += stride)
        flag[j] = (j == 0) || (shr(ykeys[j], nfb) != shr(ykeys[j - 1], nfb));
}

__global__ void k_na_runkeys(const uint64_t *__restrict__ ykeys, int nfb, uint32_t *__restrict__ run_start,
                             const uint64_t *__restrict__ nruns_d, uint64_t ny, uint64_t *__restrict__ run_key) {
    const uint64_t nruns = *nruns_d;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= nruns; r += stride) {
        if (r < nruns)
            run_key[r] = shr(ykeys[run_start[r]], nfb);
        else
            run_start[nruns] = (uint32_t)ny;
    }
}

// pos/cnt of every X nonzero: the run of Y whose contract key equals x & cmask
__global__ void k_na_match(const uint64_t *__restrict__ xkeys, uint64_t nx, int ncb,
                           const uint64_t *__restrict__ run_key, const uint32_t *__restrict__ run_start,
                           const uint64_t *__restrict__ nruns_d, uint64_t *__restrict__ pos,
                           uint64_t *__restrict__ cnt) {
    const uint64_t nruns = *nruns_d;
    const uint64_t cm = ncb >= 64 ? ~0ull : ((1ull << ncb) - 1);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += stride) {
        const uint64_t c = xkeys[i] & cm;
        uint64_t lo = 0, hi = nruns;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (run_key[mid] < c)
                lo = mid + 1;
            else
                hi = mid;
        }
        uint64_t p = 0, n = 0;
        if (lo < nruns && run_key[lo] == c) {
            p = run_start[lo];
            n = run_start[lo + 1] - p;
        }
        pos[i] = p;
        cnt[i] = n;
    }
}

}  // namespace
}  // namespace gs

extern "C" gsparc_status gsparc_index_match_noalloc(uint64_t nx, const uint64_t *d_xkeys, int x_ncbits,
                                                    uint64_t ny, const uint64_t *d_ykeys, int y_nfbits,
                                                    uint64_t *d_pos, uint64_t *d_cnt, uint64_t *d_prefix,
                                                    uint64_t *ir, void *stream) {
    using namespace gs;
    try {
        GS_REQUIRE(d_prefix && (nx == 0 || (d_xkeys && d_pos && d_cnt)) && (ny == 0 || d_ykeys), GSPARC_EINVAL,
                   "null argument");
        GS_REQUIRE(x_ncbits >= 0 && x_ncbits <= 64 && y_nfbits >= 0 && y_nfbits <= 64, GSPARC_EINVAL,
                   "bit widths must be 0..64");
        GS_REQUIRE(nx < (1ull << 31) && ny < (1ull << 31), GSPARC_EINVAL, "more than 2^31 nonzeros");
        cudaStream_t s = (cudaStream_t)stream;
        int cur_dev = -1, stream_dev = -1;
        GS_CUDA(cudaGetDevice(&cur_dev));
        GS_CUDA(cudaStreamGetDevice(s, &stream_dev));
        GS_REQUIRE(stream_dev == cur_dev, GSPARC_EINVAL,
                   "stream belongs to device " + std::to_string(stream_dev) + ", the current device is " +
                       std::to_string(cur_dev));

        // scratch layout: flags[ny] | run_start[ny+1] | run_key[ny] | nruns | CUB temporary
        size_t t_sel = 0, t_scan = 0;
        cub::CountingInputIterator<uint32_t> it(0);
        if (ny)
            GS_CUDA(cub::DeviceSelect::Flagged(nullptr, t_sel, it, (uint8_t *)nullptr, (uint32_t *)nullptr,
                                               (uint64_t *)nullptr, (int)ny, s));
        if (nx)
            GS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, t_scan, (uint64_t *)nullptr, (uint64_t *)nullptr,
                                                  (int)nx, s));
        const size_t o_flag = 0;
        const size_t o_start = o_flag + align256(ny);
        const size_t o_key = o_start + align256(4 * (ny + 1));
        const size_t o_n = o_key + align256(8 * (ny ? ny : 1));
        const size_t o_tmp = o_n + 256;
        const size_t need = o_tmp + align256(t_sel > t_scan ? t_sel : t_scan);
        if (need > kScratchBytes)
            fail(GSPARC_EINVAL, "index match of " + std::to_string(nx) + " x " + std::to_string(ny) +
                                    " keys needs " + std::to_string(need) + " B of scratch; the no-allocation "
                                    "entry point holds " + std::to_string(kScratchBytes) +
                                    " B (about 13 B per Y key plus CUB temporary storage that grows "
                                    "with X)");

        unsigned char *sc = static_cast<unsigned char *>(scratch_on_current_device());
        uint8_t *flag = sc + o_flag;
        uint32_t *run_start = reinterpret_cast<uint32_t *>(sc + o_start);
        uint64_t *run_key = reinterpret_cast<uint64_t *>(sc + o_key);
        uint64_t *nruns = reinterpret_cast<uint64_t *>(sc + o_n);
        void *tmp = sc + o_tmp;

        GS_CUDA(cudaMemsetAsync(nruns, 0, 8, s));
        if (ny) {
            k_na_flags<<<grid_for(ny), kThreads, 0, s>>>(d_ykeys, ny, y_nfbits, flag);
            count_launch();
            GS_CUDA(cudaGetLastError());
            GS_CUDA(cub::DeviceSelect::Flagged(tmp, t_sel, it, flag, run_start, nruns, (int)ny, s));
            k_na_runkeys<<<grid_for(ny + 1), kThreads, 0, s>>>(d_ykeys, y_nfbits, run_start, nruns, ny, run_key);
            count_launch();
            GS_CUDA(cudaGetLastError());
        }
        if (nx) {
            k_na_match<<<grid_for(nx), kThreads, 0, s>>>(d_xkeys, nx, x_ncbits, run_key, run_start, nruns, d_pos,
                                                          d_cnt);
            count_launch();
            GS_CUDA(cudaGetLastError());
        }
        GS_CUDA(cudaMemsetAsync(d_prefix, 0, 8, s));
        if (nx) GS_CUDA(cub::DeviceScan::InclusiveSum(tmp, t_scan, d_cnt, d_prefix + 1, (int)nx, s));
        if (ir) {
            uint64_t h = 0;
            GS_CUDA(cudaMemcpyAsync(&h, d_prefix + nx, 8, cudaMemcpyDeviceToHost, s));
            GS_CUDA(cudaStreamSynchronize(s));
            *ir = h;
        }
        set_last_error("");
        return GSPARC_OK;
    } catch (const Error &e) {
        set_last_error(e.msg);
        return e.st;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return GSPARC_ENOMEM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return GSPARC_EINTERNAL;
    }
}
