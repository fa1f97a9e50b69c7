// serve.cpp -- a request loop with continuous batching over resident operands.
//
// The reference runs one contraction per process (main.cu:22-437); a service
// that answers a stream of contraction requests needs what it lacks: operands
// that stay in HBM between requests, admission against a memory budget, and
// batching of whatever is waiting.  A server holds:
//
//  * one stream-ordered memory pool for the device, shared by the resident
//    operands (an arena that owns the pool) and by every lane (arenas that draw
//    on it, each with the budget its current batch was admitted with);
//  * `lanes` worker threads, each with its own stream and engine context.
//
// A lane that is free takes the waiting requests in arrival order while the
// free budget (total budget - resident operands - working memory admitted to
// other lanes) covers their estimated working memory and the batch limits
// hold, and runs them as one gsparc_sptc_batch.  Requests arriving meanwhile
// queue up for the next free lane, so the batches of different lanes overlap
// on the device: one lane's host-side planning and output delivery run while
// another lane's kernels occupy the GPU.  A large batch (2^21 operand
// nonzeros or more) fills the GPU by itself and runs alone: overlapping it
// with others only made both slower (measured on the served workload).  A
// request whose output exceeds the
// memory it was admitted with streams its output in chunks (the engine's
// memory-aware partitioning), so admission only has to cover the operands'
// working set and a bounded output window.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    uint64_t ticket = 0;
    gsparc_job job{};
    int cx[gs::kMaxOrder] = {}, cy[gs::kMaxOrder] = {};
    Clock::time_point t_submit, t_done;
    uint64_t est = 0;  // working memory estimate of the operands' pipeline (bytes)
    uint64_t nz = 0;   // X + Y nonzeros
    bool taken = false;
    bool done = false;
};

struct Lane {
    gsparc_ctx ctx;
    cudaStream_t stream = nullptr;
    std::thread th;
};

// Peak working memory of one job's linearise / sort / run table / match /
// row planning, per operand nonzero, with headroom for CUB temporaries (the
// buffers run_group holds at its high-water mark: ~160 B per X nonzero and
// ~60 B per Y nonzero).
uint64_t job_estimate(const gsparc_job &J) {
    return 192ull * J.x->nnz + 96ull * J.y->nnz + (8ull << 20);
}

// Output window admitted with a batch: at least two output chunks of one
// full row of the widest job (a row has at most ny outputs), and otherwise
// half of what the batch leaves free.  The window only bounds the chunk size:
// chunk buffers are allocated for the output that exists, so a generous
// window costs nothing for small outputs and keeps large ones in few chunks.
// Batches with at least this many operand nonzeros (X + Y) run alone.
constexpr uint64_t kExclusiveNnz = 1ull << 21;

uint64_t output_window(uint64_t max_ny, uint64_t free_after) {
    const uint64_t w = std::max<uint64_t>(128ull << 20, 64ull * max_ny + (16ull << 20));
    return std::max(w, free_after / 2);
}

}  // namespace

struct gsparc_server {
    int device = 0;
    gsparc_server_opts opt{};
    uint64_t budget = 0;
    gs::Arena resident;  // owns the pool; resident operands only
    cudaStream_t up_stream = nullptr;
    std::vector<std::unique_ptr<Lane>> lanes;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
    std::unordered_map<const gsparc_tensor *, uint64_t> refs;  // waiting + running requests per tensor
    std::unordered_map<const gsparc_tensor *, bool> mine;      // uploaded here -> release asked
    uint64_t next_ticket = 1;
    uint64_t reserved = 0;  // working memory admitted to running batches
    int running = 0;
    bool stop = false;
    bool paused = false;  // gsparc_serve_pause: lanes take no new batch
    bool exclusive_running = false;  // a large batch runs alone

    // statistics
    std::vector<double> lat_ms;
    uint64_t submitted = 0, completed = 0, failed = 0, batches = 0, max_batch = 0;
    uint64_t ir = 0, nnz = 0, peak_reserved = 0, max_in_flight = 0, retries = 0, chunks = 0;
    Clock::time_point t_first, t_last;
    bool have_first = false;

    uint64_t free_bytes() const {
        const uint64_t used = resident.in_use() + reserved;
        return budget > used ? budget - used : 0;
    }
    void free_tensor_locked(gsparc_tensor *t) {
        resident.free(t->d_idx, up_stream);
        resident.free(t->d_val, up_stream);
        mine.erase(t);
        refs.erase(t);
        delete t;
    }
    void unref_locked(const gsparc_tensor *t) {
        auto it = refs.find(t);
        if (it == refs.end()) return;
        if (--it->second == 0) {
            refs.erase(it);
            auto m = mine.find(t);
            if (m != mine.end() && m->second) free_tensor_locked(const_cast<gsparc_tensor *>(t));
        }
    }
};

namespace {

// Marks a request complete with the job's final status and counts (lock
// held).  From then on a waiter may retire and delete the request, so the
// lane must not touch it again.
void complete_locked(gsparc_server *S, Req *r, const gsparc_job &J) {
    const auto now = Clock::now();
    r->job.status = J.status;
    r->job.stats = J.stats;
    r->t_done = now;
    r->done = true;
    r->job.stats.t_total_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
    S->lat_ms.push_back(r->job.stats.t_total_ms);
    S->completed += 1;
    if (J.status != GSPARC_OK) {
        S->failed += 1;
    } else {
        S->ir += J.stats.ir_nnz;
        S->nnz += J.stats.nnz;
    }
    S->unref_locked(r->job.x);
    S->unref_locked(r->job.y);
    S->t_last = now;
    S->cv_done.notify_all();
}

// Runs one admitted batch on the lane.  Jobs that succeed are reported
// complete as soon as their output is delivered (the engine cuts the numeric
// pass at job boundaries); failed jobs are settled after the batch.
void run_batch(gsparc_server *S, Lane *L, std::vector<Req *> &batch, uint64_t reserve) {
    L->ctx.arena.set_budget(reserve);
    // smallest first inside the batch: the engine's cuts at job boundaries
    // then deliver the small requests before the large ones finish
    std::stable_sort(batch.begin(), batch.end(), [](const Req *a, const Req *b) { return a->nz < b->nz; });
    std::vector<gsparc_job> jobs(batch.size());
    for (size_t i = 0; i < batch.size(); ++i) jobs[i] = batch[i]->job;
    std::vector<char> fin(batch.size(), 0);  // completed (the Req may be gone)
    gs::JobDoneFn on_done = [&](gsparc_job *J) {
        if (J->status != GSPARC_OK) return;
        const size_t i = (size_t)(J - jobs.data());
        std::lock_guard<std::mutex> lk(S->mu);
        if (fin[i]) return;
        fin[i] = 1;
        complete_locked(S, batch[i], *J);
    };
    gsparc_stats bst;
    std::memset(&bst, 0, sizeof(bst));
    try {
        gs::sptc_batch(&L->ctx, jobs.data(), (int)jobs.size(), S->opt.max_chunk_nnz, &bst, L->stream, 0, 1,
                       &on_done);
    } catch (const gs::Error &) {
        // per-job statuses say which jobs failed
    } catch (...) {
        for (auto &j : jobs)
            if (j.status == GSPARC_OK) j.status = GSPARC_EINTERNAL;
    }
    cudaStreamSynchronize(L->stream);
    // A job that ran out of its share of the batch's memory gets a second
    // chance alone, with all of the lane's admitted memory.
    if (jobs.size() > 1) {
        for (size_t i = 0; i < jobs.size(); ++i) {
            if (fin[i] || jobs[i].status != GSPARC_ENOMEM) continue;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                S->retries += 1;
            }
            jobs[i] = batch[i]->job;
            try {
                gsparc_stats rst;
                std::memset(&rst, 0, sizeof(rst));
                gs::sptc_batch(&L->ctx, &jobs[i], 1, S->opt.max_chunk_nnz, &rst, L->stream);
                bst.chunks += rst.chunks;
            } catch (...) {
            }
            cudaStreamSynchronize(L->stream);
        }
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->chunks += bst.chunks;
    for (size_t i = 0; i < batch.size(); ++i)
        if (!fin[i]) complete_locked(S, batch[i], jobs[i]);
}

void lane_main(gsparc_server *S, Lane *L) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_work.wait(lk, [&] { return S->stop || (!S->paused && !S->queue.empty()); });
        if (S->queue.empty() || S->paused) {
            if (S->stop) return;
            continue;
        }
        // ---- admission.  Candidates: requests that waited longer than age_ms
        // in arrival order, then the others smallest first (or all in arrival
        // order with fifo).  A batch takes candidates while the free budget
        // covers their working memory plus an output window, up to the batch
        // limits; a request larger than max_batch_nnz goes alone.
        const uint64_t free = S->free_bytes();
        const auto now = Clock::now();
        std::vector<Req *> cand(S->queue.begin(), S->queue.end());
        if (!S->opt.fifo) {
            const auto age = std::chrono::microseconds((int64_t)(S->opt.age_ms * 1e3));
            auto young = std::stable_partition(cand.begin(), cand.end(),
                                               [&](const Req *r) { return now - r->t_submit > age; });
            std::stable_sort(young, cand.end(), [](const Req *a, const Req *b) { return a->nz < b->nz; });
        }
        std::vector<Req *> batch;
        uint64_t need = 0, nz = 0, max_ny = 0, reserve = 0;
        for (Req *r : cand) {
            if ((int)batch.size() >= S->opt.max_batch_jobs) break;
            if (!batch.empty() && nz + r->nz > S->opt.max_batch_nnz) break;
            const uint64_t need2 = need + r->est;
            const uint64_t ny2 = std::max<uint64_t>(max_ny, r->job.y->nnz);
            const uint64_t res2 = need2 + output_window(ny2, free > need2 ? free - need2 : 0);
            if (res2 > free) {
                // The first candidate waits for memory held by other lanes; with
                // nothing running it takes all that is free and the engine
                // decides (it chunks the output, or fails the job with ENOMEM).
                if (batch.empty() && S->running == 0) {
                    batch.push_back(r);
                    reserve = free;
                }
                break;
            }
            batch.push_back(r);
            need = need2;
            nz += r->nz;
            max_ny = ny2;
            reserve = res2;
        }
        if (batch.empty()) {
            S->cv_work.wait(lk);  // a completion frees memory
            continue;
        }
        // Lane concurrency adapts to size: a large batch (at least
        // kExclusiveNnz operand nonzeros) fills the GPU by itself, so it runs
        // alone -- it waits for the running batches to finish and no other
        // batch starts beside it.  Small batches overlap freely.
        const bool exclusive = nz >= kExclusiveNnz;
        if (S->exclusive_running || (exclusive && S->running > 0)) {
            S->cv_work.wait(lk);
            continue;
        }
        for (Req *r : batch) r->taken = true;
        S->queue.erase(std::remove_if(S->queue.begin(), S->queue.end(), [](const Req *r) { return r->taken; }),
                       S->queue.end());
        S->reserved += reserve;
        S->running += 1;
        S->exclusive_running = exclusive;
        S->peak_reserved = std::max(S->peak_reserved, S->reserved);
        S->max_in_flight = std::max<uint64_t>(S->max_in_flight, S->running);
        S->batches += 1;
        S->max_batch = std::max<uint64_t>(S->max_batch, batch.size());
        lk.unlock();

        run_batch(S, L, batch, reserve);

        lk.lock();
        S->reserved -= reserve;
        S->running -= 1;
        if (exclusive) S->exclusive_running = false;
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

template <class F>
gsparc_status guard(F &&f) {
    try {
        f();
        gs::set_last_error("");
        return GSPARC_OK;
    } catch (const gs::Error &e) {
        gs::set_last_error(e.msg);
        return e.st;
    } catch (const std::bad_alloc &) {
        gs::set_last_error("host allocation failed");
        return GSPARC_ENOMEM;
    } catch (const std::exception &e) {
        gs::set_last_error(e.what());
        return GSPARC_EINTERNAL;
    }
}

void destroy_lane(Lane *L) {
    if (L->stream) cudaStreamDestroy(L->stream);
    for (auto &e : L->ctx.ev)
        if (e) cudaEventDestroy(e);
    if (L->ctx.d_flag) cudaFree(L->ctx.d_flag);
    if (L->ctx.copy_stream) cudaStreamDestroy(L->ctx.copy_stream);
    if (L->ctx.alt_stream) cudaStreamDestroy(L->ctx.alt_stream);
}

void stop_server(gsparc_server *S) {
    {
        std::unique_lock<std::mutex> lk(S->mu);
        S->cv_done.wait(lk, [&] { return S->queue.empty() && S->running == 0; });
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (auto &L : S->lanes)
        if (L->th.joinable()) L->th.join();
    for (auto &L : S->lanes) destroy_lane(L.get());
    S->lanes.clear();
    std::vector<gsparc_tensor *> ts;
    for (auto &kv : S->mine) ts.push_back(const_cast<gsparc_tensor *>(kv.first));
    for (auto *t : ts) S->free_tensor_locked(t);
    if (S->up_stream) {
        cudaStreamSynchronize(S->up_stream);
        cudaStreamDestroy(S->up_stream);
    }
}

}  // namespace

extern "C" {

gsparc_status gsparc_serve_create(int device, const gsparc_server_opts *opts, gsparc_server **out) {
    return guard([&] {
        GS_REQUIRE(out, GSPARC_EINVAL, "out is null");
        *out = nullptr;
        int ndev = 0;
        GS_CUDA(cudaGetDeviceCount(&ndev));
        GS_REQUIRE(device >= 0 && device < ndev, GSPARC_EINVAL, "no such device");
        GS_CUDA(cudaSetDevice(device));
        auto S = std::make_unique<gsparc_server>();
        S->device = device;
        if (opts) S->opt = *opts;
        GS_REQUIRE(S->opt.lanes >= 0 && S->opt.lanes <= 16, GSPARC_EINVAL, "lanes must be 0..16");
        GS_REQUIRE(S->opt.max_batch_jobs >= 0, GSPARC_EINVAL, "max_batch_jobs must be >= 0");
        if (S->opt.lanes == 0) S->opt.lanes = 2;
        if (S->opt.max_batch_jobs == 0) S->opt.max_batch_jobs = 256;
        if (S->opt.max_batch_nnz == 0) S->opt.max_batch_nnz = 1ull << 24;
        GS_REQUIRE(S->opt.age_ms >= 0, GSPARC_EINVAL, "age_ms must be >= 0");
        if (S->opt.age_ms == 0) S->opt.age_ms = 200.0;
        if (S->opt.max_chunk_nnz == 0) S->opt.max_chunk_nnz = 1ull << 28;
        size_t fr = 0, tot = 0;
        GS_CUDA(cudaMemGetInfo(&fr, &tot));
        S->budget = S->opt.hbm_budget_bytes ? S->opt.hbm_budget_bytes : (uint64_t)(fr * 0.9);
        S->resident.init(device, S->budget);
        GS_CUDA(cudaStreamCreateWithFlags(&S->up_stream, cudaStreamNonBlocking));
        // the budget is mapped into the shared pool once, before any request:
        // the lanes' working buffers (output chunks, kept row bitmaps) come and
        // go in sizes that change with every batch, and growing the pool for
        // one of them in the middle of a batch costs far more than the batch
        S->resident.reserve(0, S->up_stream);
        int sms = 148;
        GS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        for (int i = 0; i < S->opt.lanes; ++i) {
            auto L = std::make_unique<Lane>();
            L->ctx.device = device;
            L->ctx.sm_count = sms;
            L->ctx.arena.init_shared(device, S->resident.pool(), 0);
            try {
                for (auto &e : L->ctx.ev) GS_CUDA(cudaEventCreate(&e));
                GS_CUDA(cudaMalloc(&L->ctx.d_flag, 64));
                GS_CUDA(cudaMemset(L->ctx.d_flag, 0, 64));
                GS_CUDA(cudaStreamCreateWithFlags(&L->ctx.copy_stream, cudaStreamNonBlocking));
                GS_CUDA(cudaStreamCreateWithFlags(&L->ctx.alt_stream, cudaStreamNonBlocking));
                GS_CUDA(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking));
            } catch (...) {
                destroy_lane(L.get());
                for (auto &M : S->lanes) destroy_lane(M.get());
                throw;
            }
            S->lanes.push_back(std::move(L));
        }
        for (auto &L : S->lanes) L->th = std::thread(lane_main, S.get(), L.get());
        *out = S.release();
    });
}

gsparc_status gsparc_serve_destroy(gsparc_server *srv) {
    return guard([&] {
        if (!srv) return;
        cudaSetDevice(srv->device);
        stop_server(srv);
        delete srv;
    });
}

gsparc_status gsparc_serve_upload(gsparc_server *srv, const gsparc_coo *coo, gsparc_tensor **out) {
    return guard([&] {
        GS_REQUIRE(srv && coo && out, GSPARC_EINVAL, "null argument");
        *out = nullptr;
        GS_REQUIRE(coo->order >= 1 && coo->order <= gs::kMaxOrder, GSPARC_EINVAL, "order must be 1..32");
        GS_REQUIRE(coo->dims, GSPARC_EINVAL, "dims is null");
        GS_REQUIRE(coo->nnz == 0 || (coo->idx && coo->val), GSPARC_EINVAL, "idx/val is null");
        cudaSetDevice(srv->device);
        auto t = std::make_unique<gsparc_tensor>();
        t->order = coo->order;
        t->nnz = coo->nnz;
        for (int m = 0; m < coo->order; ++m) {
            GS_REQUIRE(coo->dims[m] >= 1, GSPARC_EINVAL, "mode size must be >= 1");
            t->dims[m] = coo->dims[m];
        }
        const uint64_t n = coo->nnz;
        const size_t ib = sizeof(uint64_t) * coo->order * (n ? n : 1);
        const size_t vb = sizeof(float) * (n ? n : 1);
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            // resident operands and admitted working memory share the budget
            srv->resident.set_budget(srv->budget > srv->reserved ? srv->budget - srv->reserved : 0);
            t->d_idx = (uint64_t *)srv->resident.alloc(ib, srv->up_stream);
            try {
                t->d_val = (float *)srv->resident.alloc(vb, srv->up_stream);
            } catch (...) {
                srv->resident.free(t->d_idx, srv->up_stream);
                throw;
            }
        }
        try {
            const cudaMemcpyKind kind = coo->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
            for (int m = 0; m < coo->order && n; ++m) {
                GS_REQUIRE(coo->idx[m], GSPARC_EINVAL, "idx[m] is null");
                GS_CUDA(cudaMemcpyAsync(t->d_idx + (uint64_t)m * n, coo->idx[m], 8 * n, kind, srv->up_stream));
            }
            if (n) GS_CUDA(cudaMemcpyAsync(t->d_val, coo->val, 4 * n, kind, srv->up_stream));
            GS_CUDA(cudaStreamSynchronize(srv->up_stream));
        } catch (...) {
            cudaStreamSynchronize(srv->up_stream);
            std::lock_guard<std::mutex> lk(srv->mu);
            srv->resident.free(t->d_idx, srv->up_stream);
            srv->resident.free(t->d_val, srv->up_stream);
            throw;
        }
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->mine[t.get()] = false;
        *out = t.release();
    });
}

gsparc_status gsparc_serve_release(gsparc_server *srv, gsparc_tensor *t) {
    return guard([&] {
        GS_REQUIRE(srv, GSPARC_EINVAL, "null server");
        if (!t) return;
        cudaSetDevice(srv->device);
        std::lock_guard<std::mutex> lk(srv->mu);
        auto m = srv->mine.find(t);
        GS_REQUIRE(m != srv->mine.end(), GSPARC_EINVAL, "tensor was not uploaded to this server");
        GS_REQUIRE(!m->second, GSPARC_EINVAL, "tensor already released");
        auto r = srv->refs.find(t);
        if (r == srv->refs.end() || r->second == 0)
            srv->free_tensor_locked(t);
        else
            m->second = true;  // freed by the lane that finishes its last request
    });
}

gsparc_status gsparc_serve_submit(gsparc_server *srv, const gsparc_job *job, uint64_t *ticket) {
    return guard([&] {
        GS_REQUIRE(srv && job && ticket, GSPARC_EINVAL, "null argument");
        GS_REQUIRE(job->x && job->y, GSPARC_EINVAL, "null tensor");
        GS_REQUIRE(job->ncmodes >= 1 && job->ncmodes <= gs::kMaxOrder && job->cx && job->cy, GSPARC_EINVAL,
                   "bad contract modes");
        auto r = std::make_unique<Req>();
        r->job = *job;
        for (int i = 0; i < job->ncmodes; ++i) {
            r->cx[i] = job->cx[i];
            r->cy[i] = job->cy[i];
        }
        r->job.cx = r->cx;
        r->job.cy = r->cy;
        r->job.status = GSPARC_OK;
        std::memset(&r->job.stats, 0, sizeof(r->job.stats));
        r->est = job_estimate(r->job);
        r->nz = job->x->nnz + job->y->nnz;
        std::lock_guard<std::mutex> lk(srv->mu);
        GS_REQUIRE(!srv->stop, GSPARC_EINVAL, "server is stopping");
        for (const gsparc_tensor *t : {job->x, job->y}) {
            auto m = srv->mine.find(t);
            GS_REQUIRE(m == srv->mine.end() || !m->second, GSPARC_EINVAL, "tensor was released");
        }
        srv->refs[job->x] += 1;
        srv->refs[job->y] += 1;
        r->ticket = srv->next_ticket++;
        r->t_submit = Clock::now();
        if (!srv->have_first) {
            srv->have_first = true;
            srv->t_first = r->t_submit;
        }
        srv->submitted += 1;
        *ticket = r->ticket;
        srv->queue.push_back(r.get());
        srv->reqs[r->ticket] = std::move(r);
        srv->cv_work.notify_one();
    });
}

gsparc_status gsparc_serve_poll(gsparc_server *srv, uint64_t ticket, int *done, gsparc_job *result) {
    return guard([&] {
        GS_REQUIRE(srv && done, GSPARC_EINVAL, "null argument");
        std::lock_guard<std::mutex> lk(srv->mu);
        auto it = srv->reqs.find(ticket);
        GS_REQUIRE(it != srv->reqs.end(), GSPARC_EINVAL, "unknown ticket");
        *done = it->second->done ? 1 : 0;
        if (*done && result) *result = it->second->job;
    });
}

gsparc_status gsparc_serve_wait(gsparc_server *srv, uint64_t ticket, double timeout_ms, gsparc_job *result) {
    return guard([&] {
        GS_REQUIRE(srv, GSPARC_EINVAL, "null server");
        std::unique_lock<std::mutex> lk(srv->mu);
        auto it = srv->reqs.find(ticket);
        GS_REQUIRE(it != srv->reqs.end(), GSPARC_EINVAL, "unknown ticket");
        Req *r = it->second.get();
        if (timeout_ms < 0) {
            srv->cv_done.wait(lk, [&] { return r->done; });
        } else {
            const auto until = Clock::now() + std::chrono::microseconds((int64_t)(timeout_ms * 1e3));
            if (!srv->cv_done.wait_until(lk, until, [&] { return r->done; }))
                gs::fail(GSPARC_ETIMEOUT, "request did not complete in time");
        }
        if (result) *result = r->job;
        const gsparc_status st = r->job.status;
        srv->reqs.erase(it);
        if (st != GSPARC_OK) gs::fail(st, "request failed: " + std::string(gsparc_status_string(st)));
    });
}

gsparc_status gsparc_serve_stats(gsparc_server *srv, gsparc_server_stats *out) {
    return guard([&] {
        GS_REQUIRE(srv && out, GSPARC_EINVAL, "null argument");
        std::lock_guard<std::mutex> lk(srv->mu);
        std::memset(out, 0, sizeof(*out));
        out->submitted = srv->submitted;
        out->completed = srv->completed;
        out->failed = srv->failed;
        out->batches = srv->batches;
        out->max_batch = srv->max_batch;
        out->ir_nnz = srv->ir;
        out->nnz = srv->nnz;
        out->resident_bytes = srv->resident.in_use();
        out->peak_reserved_bytes = srv->peak_reserved;
        out->max_in_flight = srv->max_in_flight;
        out->retries = srv->retries;
        out->chunks = srv->chunks;
        std::vector<double> v = srv->lat_ms;
        if (!v.empty()) {
            std::sort(v.begin(), v.end());
            // nearest-rank percentiles
            auto pct = [&](double p) {
                size_t k = (size_t)std::ceil(p / 100.0 * (double)v.size());
                if (k < 1) k = 1;
                return v[std::min(k, v.size()) - 1];
            };
            out->p50_ms = pct(50.0);
            out->p99_ms = pct(99.0);
            double s = 0;
            for (double x : v) s += x;
            out->mean_ms = s / (double)v.size();
            out->max_ms = v.back();
        }
        if (srv->have_first && srv->completed) {
            out->wall_ms = std::chrono::duration<double, std::milli>(srv->t_last - srv->t_first).count();
            if (out->wall_ms > 0) out->products_per_s = (double)srv->ir / (out->wall_ms / 1e3);
        }
    });
}

gsparc_status gsparc_serve_pause(gsparc_server *srv, int paused) {
    return guard([&] {
        GS_REQUIRE(srv, GSPARC_EINVAL, "null server");
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->paused = paused != 0;
        srv->cv_work.notify_all();
    });
}

gsparc_status gsparc_serve_inject_alloc_failure(gsparc_server *srv, uint64_t nth) {
    return guard([&] {
        GS_REQUIRE(srv, GSPARC_EINVAL, "null server");
        for (auto &L : srv->lanes) L->ctx.arena.inject_failure(nth);
    });
}

gsparc_status gsparc_serve_reset_stats(gsparc_server *srv) {
    return guard([&] {
        GS_REQUIRE(srv, GSPARC_EINVAL, "null server");
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->lat_ms.clear();
        srv->submitted = srv->completed = srv->failed = srv->batches = srv->max_batch = 0;
        srv->ir = srv->nnz = 0;
        srv->peak_reserved = srv->reserved;
        srv->max_in_flight = srv->running;
        srv->retries = srv->chunks = 0;
        srv->have_first = false;
    });
}

}  // extern "C"
