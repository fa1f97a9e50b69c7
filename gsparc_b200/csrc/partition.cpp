// partition.cpp -- contractions whose operands do not fit the HBM budget.
//
// The reference counts partitions from the operands' storage against half of
// its memory pool (include/gsparc/tensor_manager.tpp:33-61), splits X into
// near-equal parts at free-index group ends (:634-749), relays Y out by its
// free index and sorts it per part (:752-886), and runs every (X part, Y part)
// pair (include/gsparc/sptc.cuh:42-139).  Here the operands stay in host
// memory and the parts are planned the same way, by value ranges of the free
// part of the linearised key:
//
//   * X parts are ranges of x_f (output rows), Y parts ranges of y_f (output
//     columns), each holding at most max_part nonzeros (a single row or column
//     is never split);
//   * a part is gathered on the host (one counting-sort pass per operand) and
//     uploaded with the whole operand's dims, so every part has the operand's
//     bit layout and produces the same keys;
//   * the output of X part i and Y part j is Z restricted to those rows and
//     columns, and complete there (every product of an output lies in the one
//     Y part holding its column).  X parts run in row order, so with a single
//     Y part their outputs follow each other in Z's order; with several Y
//     parts the outputs of one X part (rows in order, columns of part j in
//     range j) are merged by key on the host before delivery.
//
// Part sizes follow the budget (a resident operand plus its working memory
// per nonzero, a third of the budget left for output chunks) unless the
// caller caps them.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "engine.h"
#include "kernels.cuh"

namespace gs {

namespace {

// Device bytes per operand nonzero while a part is contracted: the resident
// SoA copy plus the engine's working set (keys and values double-buffered for
// the sort, match and row tables); measured peaks stay below these.
uint64_t x_bytes_per_nnz(int order) { return 8ull * order + 4 + 192; }
uint64_t y_bytes_per_nnz(int order) { return 8ull * order + 4 + 96; }

int nthreads() {
    const unsigned h = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(h ? h : 1u, 32u));
}

template <class F>
void parallel_for(uint64_t n, F &&f) {
    const int T = (int)std::min<uint64_t>(nthreads(), std::max<uint64_t>(1, n / 65536));
    if (T <= 1) {
        f(0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t)
        th.emplace_back([&, t] { f(n * t / T, n * (t + 1) / T, t); });
    for (auto &x : th) x.join();
}

// Order-preserving 64-bit prefix of each nonzero's free part (the whole free
// part when it has at most 64 bits).
std::vector<uint64_t> free_prefix(const gsparc_coo &t, const Layout &L) {
    std::vector<uint64_t> v(t.nnz);
    const int drop = L.nfbits > 64 ? L.nfbits - 64 : 0;
    parallel_for(t.nnz, [&](uint64_t a, uint64_t b, int) {
        for (uint64_t k = a; k < b; ++k) {
            unsigned __int128 f = 0;
            for (int m = 0; m < t.order; ++m)
                if (!L.is_c[m]) f |= (unsigned __int128)t.idx[m][k] << L.shift[m];
            v[k] = (uint64_t)(f >> drop);
        }
    });
    return v;
}

// Value bounds b[0] = 0 < b[1] < ... < b[P] = max+1 such that every range
// [b[p], b[p+1]) holds at most max_part of the values, except a range of one
// value (a single row or column, which cannot be split).  Histograms over
// successively lower bits refine any bucket that is too large.
void split_values(const std::vector<uint64_t> &v, uint64_t lo, uint64_t hi, uint64_t max_part,
                  std::vector<uint64_t> &bounds) {
    // values in [lo, hi) only; bounds gets interior cut points in ascending order
    constexpr int B = 1 << 12;
    const unsigned __int128 width = (unsigned __int128)hi - lo;
    const unsigned __int128 step = (width + B - 1) / B;
    std::vector<uint64_t> h(B, 0);
    for (uint64_t x : v)
        if (x >= lo && x < hi) ++h[(size_t)((x - lo) / step)];
    uint64_t acc = 0;
    for (int b = 0; b < B; ++b) {
        const uint64_t b0 = lo + (uint64_t)(step * b);
        if (b0 >= hi) break;
        const unsigned __int128 e = (unsigned __int128)b0 + step;
        const uint64_t b1 = e > hi ? hi : (uint64_t)e;
        if (h[b] > max_part && b1 - b0 > 1) {
            if (acc) bounds.push_back(b0);
            acc = 0;
            // refine this bucket; its own cuts go in between
            split_values(v, b0, b1, max_part, bounds);
            bounds.push_back(b1);
            continue;
        }
        if (acc && acc + h[b] > max_part) {
            bounds.push_back(b0);
            acc = 0;
        }
        acc += h[b];
    }
}

// Parts of an operand: ranges of the free prefix, nonzeros grouped by part.
struct Parts {
    std::vector<uint64_t> bounds;  // P + 1 value bounds
    std::vector<uint64_t> start;   // P + 1 offsets into perm
    std::vector<uint64_t> perm;    // nonzero ids grouped by part, in input order inside a part
    int count() const { return (int)start.size() - 1; }
};

Parts plan_parts(const gsparc_coo &t, const Layout &L, uint64_t max_part) {
    Parts P;
    std::vector<uint64_t> v = free_prefix(t, L);
    uint64_t mx = 0;
    for (uint64_t x : v) mx = std::max(mx, x);
    std::vector<uint64_t> cuts;
    const uint64_t top = mx == ~0ull ? mx : mx + 1;
    if (t.nnz > max_part) split_values(v, 0, top, max_part, cuts);
    // drop duplicate or out-of-range cuts
    P.bounds.push_back(0);
    for (uint64_t c : cuts)
        if (c > P.bounds.back() && c < top) P.bounds.push_back(c);
    P.bounds.push_back(top);
    const int np = (int)P.bounds.size() - 1;
    // counting sort of nonzero ids by part (stable)
    std::vector<uint32_t> part(t.nnz);
    parallel_for(t.nnz, [&](uint64_t a, uint64_t b, int) {
        for (uint64_t k = a; k < b; ++k)
            part[k] = (uint32_t)(std::upper_bound(P.bounds.begin() + 1, P.bounds.end() - 1, v[k]) -
                                 (P.bounds.begin() + 1));
    });
    P.start.assign(np + 1, 0);
    for (uint64_t k = 0; k < t.nnz; ++k) ++P.start[part[k] + 1];
    for (int p = 0; p < np; ++p) P.start[p + 1] += P.start[p];
    P.perm.resize(t.nnz);
    std::vector<uint64_t> at(P.start.begin(), P.start.end() - 1);
    for (uint64_t k = 0; k < t.nnz; ++k) P.perm[at[part[k]]++] = k;
    return P;
}

// One part gathered into host SoA arrays and uploaded (the operand's dims).
gsparc_tensor *upload_part(gsparc_ctx *ctx, const gsparc_coo &t, const Parts &P, int p, cudaStream_t s,
                           uint64_t &bytes_h2d) {
    const uint64_t a = P.start[p], n = P.start[p + 1] - a;
    std::vector<uint64_t> idx((size_t)t.order * std::max<uint64_t>(n, 1));
    std::vector<float> val(std::max<uint64_t>(n, 1));
    parallel_for(n, [&](uint64_t i0, uint64_t i1, int) {
        for (uint64_t i = i0; i < i1; ++i) {
            const uint64_t k = P.perm[a + i];
            for (int m = 0; m < t.order; ++m) idx[(size_t)m * n + i] = t.idx[m][k];
            val[i] = t.val[k];
        }
    });
    std::vector<const uint64_t *> ptr(t.order);
    for (int m = 0; m < t.order; ++m) ptr[m] = idx.data() + (size_t)m * n;
    gsparc_coo c{t.order, t.dims, n, ptr.data(), val.data(), 0};
    gsparc_tensor *out = nullptr;
    const gsparc_status st = gsparc_tensor_upload(ctx, &c, s, &out);
    if (st) fail(st, std::string("uploading an operand part: ") + last_error());
    bytes_h2d += n * (8ull * t.order + 4);
    return out;
}

// Delivers output pieces to the caller's sink with global positions.
struct Deliver {
    const gsparc_sink *user;
    gsparc_ctx *ctx;
    cudaStream_t s;
    uint64_t offset = 0;  // outputs delivered so far
    uint64_t bytes_d2h = 0;
    uint64_t chunks = 0;

    // device-resident piece (from the engine's chunk)
    void device_piece(const uint64_t *dk, const float *dv, uint64_t n, uint64_t first_in_part) {
        const uint64_t first = offset + first_in_part;
        if (user->kind == GSPARC_SINK_DEVICE) {
            if (user->on_chunk(user->user, dk, dv, n, first, 1))
                fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
        } else if (user->kind == GSPARC_SINK_HOST) {
            host_copy(dk, dv, n, first, cudaMemcpyDeviceToHost);
        }
        ++chunks;
    }
    // host-resident piece (merged on the host)
    void host_piece(const uint64_t *hk, const float *hv, uint64_t n, uint64_t first) {
        if (user->kind == GSPARC_SINK_DEVICE) {
            DBuf<uint64_t> k(ctx->arena, std::max<uint64_t>(n, 1), s);
            DBuf<float> v(ctx->arena, std::max<uint64_t>(n, 1), s);
            GS_CUDA(cudaMemcpyAsync(k.get(), hk, 8 * n, cudaMemcpyHostToDevice, s));
            GS_CUDA(cudaMemcpyAsync(v.get(), hv, 4 * n, cudaMemcpyHostToDevice, s));
            GS_CUDA(cudaStreamSynchronize(s));
            if (user->on_chunk(user->user, k.get(), v.get(), n, first, 1))
                fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
        } else if (user->kind == GSPARC_SINK_HOST) {
            host_copy(hk, hv, n, first, cudaMemcpyHostToHost);
        }
        ++chunks;
    }
    // HOST sink: in place while the output fits the arrays, else ring mode
    // (each piece overwrites the arrays from index 0, on_chunk after each)
    void host_copy(const uint64_t *k, const float *v, uint64_t n, uint64_t first, cudaMemcpyKind kind) {
        const uint64_t cap = user->host_capacity;
        GS_REQUIRE(cap > 0 && user->host_keys && user->host_vals, GSPARC_EINVAL, "host sink without arrays");
        for (uint64_t o = 0; o < n;) {
            const bool in_place = first + n <= cap;
            const uint64_t m = in_place ? n : std::min(cap, n - o);
            uint64_t *dk = user->host_keys + (in_place ? first : 0);
            float *dv = user->host_vals + (in_place ? first : 0);
            GS_CUDA(cudaMemcpyAsync(dk, k + o, 8 * m, kind, s));
            GS_CUDA(cudaMemcpyAsync(dv, v + o, 4 * m, kind, s));
            GS_CUDA(cudaStreamSynchronize(s));
            if (kind == cudaMemcpyDeviceToHost) bytes_d2h += 12 * m;
            if (user->on_chunk && user->on_chunk(user->user, dk, dv, m, first + o, 0))
                fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
            o += m;
        }
    }
};

struct Collect {
    std::vector<uint64_t> keys;
    std::vector<float> vals;
    cudaStream_t s;
};

int collect_fn(void *u, const uint64_t *k, const float *v, uint64_t n, uint64_t first, int) {
    auto *c = static_cast<Collect *>(u);
    if (c->keys.size() < first + n) {
        c->keys.resize(first + n);
        c->vals.resize(first + n);
    }
    if (cudaMemcpyAsync(c->keys.data() + first, k, 8 * n, cudaMemcpyDeviceToHost, c->s) != cudaSuccess ||
        cudaMemcpyAsync(c->vals.data() + first, v, 4 * n, cudaMemcpyDeviceToHost, c->s) != cudaSuccess ||
        cudaStreamSynchronize(c->s) != cudaSuccess)
        return 1;
    return 0;
}

struct PassThrough {
    Deliver *d;
};

int pass_fn(void *u, const uint64_t *k, const float *v, uint64_t n, uint64_t first, int) {
    auto *p = static_cast<PassThrough *>(u);
    p->d->device_piece(k, v, n, first);
    return 0;
}

void add_stats(gsparc_stats &acc, const gsparc_stats &s) {
    acc.ir_nnz += s.ir_nnz;
    acc.nnz += s.nnz;
    acc.rows += s.rows;
    acc.heavy_rows += s.heavy_rows;
    acc.stream_rows += s.stream_rows;
    acc.t_linearize_ms += s.t_linearize_ms;
    acc.t_sort_ms += s.t_sort_ms;
    acc.t_match_ms += s.t_match_ms;
    acc.t_plan_ms += s.t_plan_ms;
    acc.t_contract_ms += s.t_contract_ms;
    acc.t_output_ms += s.t_output_ms;
    acc.t_total_ms += s.t_total_ms;
    acc.t_numeric_kernel_ms += s.t_numeric_kernel_ms;
    acc.heavy_windows += s.heavy_windows;
    acc.kept_bitmap_bytes = std::max(acc.kept_bitmap_bytes, s.kept_bitmap_bytes);  // parts run one at a time
    acc.verified_nnz += s.verified_nnz;
    acc.verified_products += s.verified_products;
    acc.verify_mismatch += s.verify_mismatch;
    acc.verify_skipped_rows += s.verify_skipped_rows;
    acc.max_rel_err = std::max(acc.max_rel_err, s.max_rel_err);
    acc.max_abs_err = std::max(acc.max_abs_err, s.max_abs_err);
    acc.accumulator = s.accumulator;
    acc.nbits_x = s.nbits_x;
    acc.nbits_y = s.nbits_y;
    acc.ncbits = s.ncbits;
    acc.nfbits_x = s.nfbits_x;
    acc.nfbits_y = s.nfbits_y;
}

}  // namespace

void sptc_partitioned(gsparc_ctx *ctx, const gsparc_coo *X, const gsparc_coo *Y, int nc, const int *cx,
                      const int *cy, int accum, const gsparc_part_opts *opts, const gsparc_sink *sink,
                      gsparc_stats *stats, cudaStream_t s) {
    GS_REQUIRE(ctx && X && Y && sink, GSPARC_EINVAL, "null argument");
    GS_REQUIRE(!X->on_device && !Y->on_device, GSPARC_EINVAL, "partitioned operands live in host memory");
    GS_REQUIRE(X->order >= 1 && X->order <= kMaxOrder && Y->order >= 1 && Y->order <= kMaxOrder, GSPARC_EINVAL,
               "order must be 1..32");
    GS_REQUIRE(nc >= 1 && cx && cy, GSPARC_EINVAL, "contract modes");
    GS_REQUIRE(sink->kind != GSPARC_SINK_DEVICE || sink->on_chunk, GSPARC_EINVAL, "device sink without on_chunk");
    GS_REQUIRE(X->nnz == 0 || (X->idx && X->val), GSPARC_EINVAL, "X idx/val is null");
    GS_REQUIRE(Y->nnz == 0 || (Y->idx && Y->val), GSPARC_EINVAL, "Y idx/val is null");
    const Layout LX = make_layout(X->order, X->dims, nc, cx);
    const Layout LY = make_layout(Y->order, Y->dims, nc, cy);

    // part sizes: X part and Y part resident with their working memory in two
    // thirds of what is free, the rest for output chunks
    const uint64_t free_b = ctx->arena.available();
    const uint64_t bx = x_bytes_per_nnz(X->order), by = y_bytes_per_nnz(Y->order);
    uint64_t max_x = opts && opts->max_part_nnz_x ? opts->max_part_nnz_x : 0;
    uint64_t max_y = opts && opts->max_part_nnz_y ? opts->max_part_nnz_y : 0;
    const uint64_t room = free_b / 3 * 2;
    if (!max_y) max_y = Y->nnz * by <= room / 2 ? std::max<uint64_t>(Y->nnz, 1) : std::max<uint64_t>(1, room / 2 / by);
    if (!max_x) {
        const uint64_t ybytes = std::min<uint64_t>(Y->nnz, max_y) * by;
        const uint64_t left = room > ybytes ? room - ybytes : room / 4;
        max_x = std::max<uint64_t>(1, left / bx);
    }

    Parts PX = plan_parts(*X, LX, max_x);
    Parts PY = plan_parts(*Y, LY, max_y);
    const int nx = PX.count(), ny = PY.count();

    gsparc_stats acc;
    std::memset(&acc, 0, sizeof(acc));
    acc.nnz_x = X->nnz;
    acc.nnz_y = Y->nnz;
    Deliver dl{sink, ctx, s};
    gsparc_tensor *ty_res = nullptr;  // the single Y part stays resident
    auto run_pair = [&](gsparc_tensor *tx, gsparc_tensor *ty, const gsparc_sink &sk) {
        gsparc_job job;
        std::memset(&job, 0, sizeof(job));
        job.x = tx;
        job.y = ty;
        job.ncmodes = nc;
        job.cx = cx;
        job.cy = cy;
        job.accum = accum;
        job.sink = sk;
        gsparc_stats bst;
        std::memset(&bst, 0, sizeof(bst));
        try {
            sptc_batch(ctx, &job, 1, sink->max_chunk_nnz, &bst, s);
        } catch (const Error &e) {
            throw Error{job.status != GSPARC_OK ? job.status : e.st, e.msg};
        }
        gsparc_stats st = job.stats;
        st.t_numeric_kernel_ms = bst.t_numeric_kernel_ms;
        st.heavy_windows = bst.heavy_windows;
        st.stream_rows = bst.stream_rows;
        st.kept_bitmap_bytes = bst.kept_bitmap_bytes;
        acc.chunks += bst.chunks;
        acc.kernel_launches += bst.kernel_launches;
        acc.bytes_h2d += bst.bytes_h2d;
        add_stats(acc, st);
        return st.nnz;
    };
    try {
        if (ny == 1) ty_res = upload_part(ctx, *Y, PY, 0, s, acc.bytes_h2d);
        for (int i = 0; i < nx; ++i) {
            if (PX.start[i + 1] == PX.start[i]) continue;
            gsparc_tensor *tx = upload_part(ctx, *X, PX, i, s, acc.bytes_h2d);
            try {
                if (ny == 1) {
                    PassThrough pt{&dl};
                    gsparc_sink sk{};
                    sk.kind = GSPARC_SINK_DEVICE;
                    sk.on_chunk = pass_fn;
                    sk.user = &pt;
                    dl.offset += run_pair(tx, ty_res, sk);
                } else {
                    // the parts' outputs for these rows, merged by key on the host
                    std::vector<Collect> got(ny);
                    for (int j = 0; j < ny; ++j) {
                        got[j].s = s;
                        if (PY.start[j + 1] == PY.start[j]) continue;
                        gsparc_tensor *ty = upload_part(ctx, *Y, PY, j, s, acc.bytes_h2d);
                        try {
                            gsparc_sink sk{};
                            sk.kind = GSPARC_SINK_DEVICE;
                            sk.on_chunk = collect_fn;
                            sk.user = &got[j];
                            run_pair(tx, ty, sk);
                        } catch (...) {
                            gsparc_tensor_free(ctx, ty);
                            throw;
                        }
                        gsparc_tensor_free(ctx, ty);
                        acc.bytes_d2h += 12ull * got[j].keys.size();
                    }
                    uint64_t total = 0;
                    for (auto &g : got) total += g.keys.size();
                    std::vector<uint64_t> mk(total);
                    std::vector<float> mv(total);
                    std::vector<size_t> pos(ny, 0);
                    for (uint64_t o = 0; o < total; ++o) {  // k-way merge (keys distinct across parts)
                        int best = -1;
                        for (int j = 0; j < ny; ++j)
                            if (pos[j] < got[j].keys.size() &&
                                (best < 0 || got[j].keys[pos[j]] < got[best].keys[pos[best]]))
                                best = j;
                        mk[o] = got[best].keys[pos[best]];
                        mv[o] = got[best].vals[pos[best]];
                        ++pos[best];
                    }
                    const uint64_t piece = sink->max_chunk_nnz ? sink->max_chunk_nnz : (1ull << 26);
                    for (uint64_t o = 0; o < total; o += piece)
                        dl.host_piece(mk.data() + o, mv.data() + o, std::min(piece, total - o), dl.offset + o);
                    dl.offset += total;
                }
            } catch (...) {
                gsparc_tensor_free(ctx, tx);
                throw;
            }
            gsparc_tensor_free(ctx, tx);
        }
    } catch (...) {
        if (ty_res) gsparc_tensor_free(ctx, ty_res);
        throw;
    }
    if (ty_res) gsparc_tensor_free(ctx, ty_res);
    acc.bytes_d2h += dl.bytes_d2h;
    acc.x_parts = (uint64_t)nx;
    acc.y_parts = (uint64_t)ny;
    acc.chunks = dl.chunks;
    acc.nnz = dl.offset;
    if (stats) *stats = acc;
}

}  // namespace gs
