// engine.cu -- orchestration of one contraction (the reference's gsparc::SpTC,
// include/gsparc/sptc.cuh:16-360, plus the TensorManager steps main.cu:293-321).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>

#include "engine.h"
#include "kernels.cuh"

namespace gs {

namespace {

struct Timeline {
    cudaEvent_t ev[8];
    explicit Timeline(gsparc_ctx *ctx) {
        for (int i = 0; i < 8; ++i) ev[i] = ctx->ev[i];
    }
    void mark(int i, cudaStream_t s) { GS_CUDA(cudaEventRecord(ev[i], s)); }
    double ms(int a, int b) {
        float t = 0.f;
        GS_CUDA(cudaEventElapsedTime(&t, ev[a], ev[b]));
        return t;
    }
};

template <class T>
void h2d(T *d, const T *h, size_t n, cudaStream_t s) {
    if (n) GS_CUDA(cudaMemcpyAsync(d, h, sizeof(T) * n, cudaMemcpyHostToDevice, s));
}
template <class T>
void d2h(T *h, const T *d, size_t n, cudaStream_t s) {
    if (n) GS_CUDA(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, s));
}

struct Unit {
    uint32_t r0, r1;
    bool heavy;
};

}  // namespace

void plan_shards(const uint64_t *row_prod, uint64_t nrows, int nshards, uint64_t *bounds) {
    GS_REQUIRE(nshards >= 1, GSPARC_EINVAL, "nshards must be >= 1");
    long double total = 0;
    for (uint64_t r = 0; r < nrows; ++r) total += (long double)row_prod[r];
    bounds[0] = 0;
    long double acc = 0;
    uint64_t r = 0;
    for (int s = 1; s < nshards; ++s) {
        long double target = total * s / nshards;
        while (r < nrows && acc + (long double)row_prod[r] / 2 < target) {
            acc += (long double)row_prod[r];
            ++r;
        }
        bounds[s] = r;
    }
    bounds[nshards] = nrows;
}

void sptc(gsparc_ctx *ctx, const gsparc_tensor *X, const gsparc_tensor *Y, int nc, const int *cx,
          const int *cy, int accum, int shard, int nshards, const gsparc_sink *sink_in,
          gsparc_stats *st_out, cudaStream_t s) {
    GS_REQUIRE(ctx && X && Y, GSPARC_EINVAL, "null context or tensor");
    GS_REQUIRE(nc >= 1 && nc <= kMaxOrder && cx && cy, GSPARC_EINVAL, "bad contract modes");
    GS_REQUIRE(nshards >= 1 && shard >= 0 && shard < nshards, GSPARC_EINVAL, "bad shard");
    GS_REQUIRE(accum >= -1 && accum <= 1, GSPARC_EINVAL, "accum must be -1, 0 or 1");
    gsparc_sink sink{};
    if (sink_in) sink = *sink_in;
    GS_REQUIRE(sink.kind >= GSPARC_SINK_DISCARD && sink.kind <= GSPARC_SINK_HOST, GSPARC_EINVAL,
               "bad sink kind");
    GS_REQUIRE(sink.kind != GSPARC_SINK_HOST || (sink.host_keys && sink.host_vals && sink.host_capacity),
               GSPARC_EINVAL, "host sink needs host_keys, host_vals and host_capacity");
    GS_REQUIRE(sink.kind != GSPARC_SINK_DEVICE || sink.on_chunk, GSPARC_EINVAL,
               "device sink needs on_chunk");

    Layout LX = make_layout(X->order, X->dims, nc, cx);
    Layout LY = make_layout(Y->order, Y->dims, nc, cy);
    GS_REQUIRE(X->order > nc && Y->order > nc, GSPARC_EUNSUPPORTED,
               "every operand needs at least one free mode");
    for (int i = 0; i < nc; ++i)
        GS_REQUIRE(LX.bits[cx[i]] == LY.bits[cy[i]], GSPARC_EINVAL,
                   "contract modes of X and Y have different bit widths (mode sizes differ)");
    GS_REQUIRE(LX.nbits() <= 64 && LY.nbits() <= 64, GSPARC_EUNSUPPORTED,
               "operand keys wider than 64 bits");
    GS_REQUIRE(LX.nfbits + LY.nfbits <= 64, GSPARC_EUNSUPPORTED,
               "output key wider than 64 bits (X free bits + Y free bits > 64)");

    Arena &A = ctx->arena;
    gsparc_stats st;
    std::memset(&st, 0, sizeof(st));
    st.nnz_x = X->nnz;
    st.nnz_y = Y->nnz;
    st.nbits_x = LX.nbits();
    st.nbits_y = LY.nbits();
    st.ncbits = LX.ncbits;
    st.nfbits_x = LX.nfbits;
    st.nfbits_y = LY.nfbits;
    st.accumulator = accum;

    Timeline tl(ctx);
    const uint64_t launches0 = launch_count();
    tl.mark(0, s);

    // ---- linearise (ConvertTensor) ----
    const uint64_t nx = X->nnz, ny = Y->nnz;
    DBuf<uint64_t> xk0(A, nx, s), xk1(A, nx, s), yk0(A, ny, s), yk1(A, ny, s);
    DBuf<float> xv0(A, nx, s), xv1(A, nx, s), yv0(A, ny, s), yv1(A, ny, s);
    GS_CUDA(cudaMemsetAsync(ctx->d_flag, 0, 4 * 4, s));
    launch_linearize(make_lin_params(LX, X->dims, 0), nx, X->d_idx, X->d_val, xk0, xv0, ctx->d_flag, s);
    launch_linearize(make_lin_params(LY, Y->dims, 1), ny, Y->d_idx, Y->d_val, yk0, yv0, ctx->d_flag, s);
    tl.mark(1, s);

    // ---- sort (SortSlitomXY) ----
    int wx = 0, wy = 0;
    sort_pairs(A, nx, xk0, xk1, xv0, xv1, LX.nbits(), &wx, s);
    sort_pairs(A, ny, yk0, yk1, yv0, yv1, LY.nbits(), &wy, s);
    const uint64_t *xkeys = wx ? xk1.get() : xk0.get();
    const float *xvals = wx ? xv1.get() : xv0.get();
    const uint64_t *ykeys = wy ? yk1.get() : yk0.get();
    const float *yvals = wy ? yv1.get() : yv0.get();
    tl.mark(2, s);

    // ---- match (IndexMatch) ----
    YPrep yp;
    prepare_y(A, ykeys, ny, LY.nfbits, yp, s);
    // the spare sort buffers of Y are no longer needed
    if (wy) { yk0.release(); yv0.release(); } else { yk1.release(); yv1.release(); }
    XMatch xm;
    match_x(A, xkeys, nx, LX.ncbits, yp, xm, s);
    if (wx) { xk0.release(); xv0.release(); } else { xk1.release(); xv1.release(); }
    unsigned int herr = 0;
    d2h(&herr, ctx->d_flag, 1, s);
    GS_CUDA(cudaStreamSynchronize(s));
    GS_REQUIRE(!(herr & 1u), GSPARC_EINVAL, "an index is not smaller than its mode size");
    st.ir_nnz = xm.ir;
    st.rows = xm.nrows;
    tl.mark(3, s);

    // ---- plan rows into units ----
    const uint64_t nrows = xm.nrows;
    std::vector<uint64_t> row_prod(nrows);
    d2h(row_prod.data(), xm.row_prod.get(), nrows, s);
    GS_CUDA(cudaStreamSynchronize(s));
    st.bytes_d2h += 8 * nrows;
    std::vector<uint64_t> bounds(nshards + 1);
    plan_shards(row_prod.data(), nrows, nshards, bounds.data());
    const uint64_t ra = bounds[shard], rb = bounds[shard + 1];
    if (nshards > 1) {
        st.ir_nnz = 0;
        for (uint64_t r = ra; r < rb; ++r) st.ir_nnz += row_prod[r];
    }

    std::vector<Unit> units;
    {
        uint64_t r = ra;
        while (r < rb) {
            if (row_prod[r] == 0) { ++r; continue; }
            bool heavy = accum == GSPARC_ACCUM_DENSE || row_prod[r] > kLightRowMax;
            if (heavy) {
                units.push_back({(uint32_t)r, (uint32_t)r + 1, true});
                ++r;
                continue;
            }
            uint64_t sum = 0;
            uint64_t r0 = r;
            while (r < rb && row_prod[r] <= kLightRowMax && sum + row_prod[r] <= kLightUnitMax &&
                   accum != GSPARC_ACCUM_DENSE) {
                sum += row_prod[r];
                ++r;
            }
            units.push_back({(uint32_t)r0, (uint32_t)r, false});
        }
    }
    for (auto &u : units) st.heavy_rows += u.heavy ? 1 : 0;

    std::vector<uint32_t> h_heavy, h_light;
    for (auto &u : units) {
        if (u.heavy) h_heavy.push_back(u.r0);
        else { h_light.push_back(u.r0); h_light.push_back(u.r1); }
    }
    DBuf<uint32_t> d_heavy(A, h_heavy.size(), s), d_light(A, h_light.size(), s);
    h2d(d_heavy.get(), h_heavy.data(), h_heavy.size(), s);
    h2d(d_light.get(), h_light.data(), h_light.size(), s);
    DBuf<uint32_t> cursor(A, nx, s), pend(A, nx, s);
    DBuf<uint32_t> row_nnz(A, nrows, s);
    DBuf<uint64_t> row_off(A, nrows + 1, s);
    GS_CUDA(cudaMemsetAsync(row_nnz.get(), 0, 4 * (nrows ? nrows : 1), s));

    AccArgs aa{};
    aa.row_start = xm.row_start;
    aa.row_xf = xm.row_xf;
    aa.pos = xm.pos;
    aa.cnt = xm.cnt;
    aa.xprefix = xm.xprefix;
    aa.xval = xvals;
    aa.yrank = yp.rank;
    aa.yval = yvals;
    aa.cols = yp.cols;
    aa.y_nfbits = LY.nfbits;
    aa.work_counter = ctx->d_flag + 1;
    aa.cursor = cursor;
    aa.pend = pend;
    aa.ncols = (uint32_t)yp.ncols;
    aa.row_nnz = row_nnz;
    aa.row_off = row_off;
    aa.err = ctx->d_flag;
    const int ghs = std::max(1, ctx->sm_count * heavy_blocks_per_sm(false));
    const int gh = std::max(1, ctx->sm_count * heavy_blocks_per_sm(true));
    const int gl = std::max(1, ctx->sm_count * light_blocks_per_sm());

    // ---- symbolic pass ----
    {
        AccArgs b = aa;
        b.units = d_light;
        b.nunits = (uint32_t)(h_light.size() / 2);
        GS_CUDA(cudaMemsetAsync(ctx->d_flag + 1, 0, 4, s));
        launch_light(b, false, std::min<int>(gl, (int)std::max<size_t>(1, b.nunits)), s);
        b.units = d_heavy;
        b.nunits = (uint32_t)h_heavy.size();
        GS_CUDA(cudaMemsetAsync(ctx->d_flag + 1, 0, 4, s));
        launch_heavy(b, false, std::min<int>(ghs, (int)std::max<size_t>(1, b.nunits)), s);
    }
    exclusive_scan_u32_to_u64(A, row_nnz, row_off, nrows, s);
    std::vector<uint64_t> h_off(nrows + 1);
    d2h(h_off.data(), row_off.get(), nrows + 1, s);
    d2h(&herr, ctx->d_flag, 1, s);
    GS_CUDA(cudaStreamSynchronize(s));
    st.bytes_d2h += 8 * (nrows + 1);
    GS_REQUIRE(!(herr & 2u), GSPARC_EINTERNAL, "light unit over capacity");
    const uint64_t nnz_total = h_off[rb] - h_off[ra];
    st.nnz = nnz_total;
    tl.mark(4, s);

    // ---- chunk plan (memory-aware partitioning of the output) ----
    uint64_t max_unit = 0;
    for (auto &u : units) max_unit = std::max(max_unit, h_off[u.r1] - h_off[u.r0]);
    uint64_t cap = sink.max_chunk_nnz;
    if (cap == 0) {
        uint64_t avail = A.available();
        cap = avail / 3 / 12;  // two chunk buffers (compute one, deliver the other), a third spare
        cap = std::min<uint64_t>(cap, 1ull << 31);
    }
    cap = std::max<uint64_t>(cap, 1);
    GS_REQUIRE(max_unit <= cap || sink.max_chunk_nnz == 0, GSPARC_EINVAL,
               "max_chunk_nnz is smaller than one output row");
    GS_REQUIRE(max_unit <= std::max<uint64_t>(cap, max_unit) && max_unit * 12 <= A.available(),
               GSPARC_ENOMEM, "one output row does not fit the HBM budget");
    cap = std::max(cap, max_unit);
    cap = std::min(cap, std::max<uint64_t>(nnz_total, 1));

    struct Chunk { size_t u0, u1; uint64_t first, n; };
    std::vector<Chunk> chunks;
    {
        size_t u = 0;
        while (u < units.size()) {
            size_t u0 = u;
            uint64_t first = h_off[units[u].r0] - h_off[ra];
            uint64_t n = 0;
            while (u < units.size()) {
                uint64_t un = h_off[units[u].r1] - h_off[units[u].r0];
                if (n && n + un > cap) break;
                n += un;
                ++u;
            }
            chunks.push_back({u0, u, first, n});
        }
    }
    st.chunks = chunks.size();

    // Two chunk buffers: chunk c+1 is computed on `s` while chunk c is handed to
    // the sink (device->host copies run on a second stream, ordered after the
    // chunk's kernels by an event).  A buffer is refilled only after its
    // delivery returned, so no device-side wait is needed for reuse.
    const int nbuf = chunks.size() > 1 ? 2 : 1;
    DBuf<uint64_t> out_k[2];
    DBuf<float> out_v[2];
    for (int i = 0; i < nbuf; ++i) {
        out_k[i].reset(A, nnz_total ? cap : 1, s);
        out_v[i].reset(A, nnz_total ? cap : 1, s);
    }
    double t_out = 0;
    std::vector<cudaEvent_t> kev(2 * chunks.size(), nullptr);
    for (auto &e : kev) GS_CUDA(cudaEventCreate(&e));
    std::vector<DBuf<uint32_t>> unit_bufs(2 * chunks.size());
    const bool host_whole = sink.kind == GSPARC_SINK_HOST && sink.host_capacity >= nnz_total;
    cudaStream_t s2 = ctx->copy_stream;

    auto enqueue = [&](size_t ci) {
        const Chunk &c = chunks[ci];
        const int bi = (int)(ci % nbuf);
        // per-chunk unit lists; heavy rows largest first
        std::vector<uint32_t> hh, hl;
        for (size_t u = c.u0; u < c.u1; ++u) {
            if (units[u].heavy) hh.push_back(units[u].r0);
            else { hl.push_back(units[u].r0); hl.push_back(units[u].r1); }
        }
        std::sort(hh.begin(), hh.end(), [&](uint32_t a, uint32_t b) { return row_prod[a] > row_prod[b]; });
        DBuf<uint32_t> &dh = unit_bufs[2 * ci], &dl = unit_bufs[2 * ci + 1];
        dh.reset(A, hh.size(), s);
        dl.reset(A, hl.size(), s);
        h2d(dh.get(), hh.data(), hh.size(), s);
        h2d(dl.get(), hl.data(), hl.size(), s);
        AccArgs b = aa;
        b.chunk_base = h_off[ra] + c.first;
        b.out_keys = out_k[bi];
        b.out_vals = out_v[bi];
        b.out_cap = c.n;
        b.units = dl;
        b.nunits = (uint32_t)(hl.size() / 2);
        GS_CUDA(cudaMemsetAsync(ctx->d_flag + 1, 0, 4, s));
        GS_CUDA(cudaEventRecord(kev[2 * ci], s));
        launch_light(b, true, std::min<int>(gl, (int)std::max<size_t>(1, b.nunits)), s);
        b.units = dh;
        b.nunits = (uint32_t)hh.size();
        GS_CUDA(cudaMemsetAsync(ctx->d_flag + 1, 0, 4, s));
        launch_heavy(b, true, std::min<int>(gh, (int)std::max<size_t>(1, b.nunits)), s);
        GS_CUDA(cudaEventRecord(kev[2 * ci + 1], s));
    };

    auto deliver = [&](size_t ci) {
        const Chunk &c = chunks[ci];
        const int bi = (int)(ci % nbuf);
        auto t0 = std::chrono::steady_clock::now();
        if (sink.kind == GSPARC_SINK_DEVICE) {
            GS_CUDA(cudaEventSynchronize(kev[2 * ci + 1]));
            if (sink.on_chunk(sink.user, out_k[bi].get(), out_v[bi].get(), c.n, c.first, 1))
                fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
        } else if (sink.kind == GSPARC_SINK_HOST) {
            GS_CUDA(cudaStreamWaitEvent(s2, kev[2 * ci + 1], 0));
            if (host_whole) {
                d2h(sink.host_keys + c.first, out_k[bi].get(), c.n, s2);
                d2h(sink.host_vals + c.first, out_v[bi].get(), c.n, s2);
                st.bytes_d2h += 12 * c.n;
                GS_CUDA(cudaStreamSynchronize(s2));
                if (sink.on_chunk && sink.on_chunk(sink.user, sink.host_keys + c.first, sink.host_vals + c.first,
                                                   c.n, c.first, 0))
                    fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
            } else {
                for (uint64_t off = 0; off < c.n; off += sink.host_capacity) {
                    const uint64_t n = std::min<uint64_t>(sink.host_capacity, c.n - off);
                    d2h(sink.host_keys, out_k[bi].get() + off, n, s2);
                    d2h(sink.host_vals, out_v[bi].get() + off, n, s2);
                    st.bytes_d2h += 12 * n;
                    GS_CUDA(cudaStreamSynchronize(s2));
                    if (sink.on_chunk &&
                        sink.on_chunk(sink.user, sink.host_keys, sink.host_vals, n, c.first + off, 0))
                        fail(GSPARC_ECALLBACK, "output callback stopped the contraction");
                }
            }
        }
        t_out += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };

    try {
        for (size_t ci = 0; ci < chunks.size(); ++ci) {
            enqueue(ci);
            if (ci >= 1) deliver(ci - 1);
        }
        if (!chunks.empty()) deliver(chunks.size() - 1);
    } catch (...) {
        cudaStreamSynchronize(s2);
        cudaStreamSynchronize(s);
        for (auto e : kev) cudaEventDestroy(e);
        throw;
    }
    tl.mark(5, s);
    unsigned int hflags[4] = {0, 0, 0, 0};
    d2h(hflags, ctx->d_flag, 4, s);
    GS_CUDA(cudaStreamSynchronize(s));
    herr = hflags[0];
    st.heavy_windows = hflags[2];
    GS_REQUIRE(!(herr & 2u), GSPARC_EINTERNAL, "light unit over capacity");
    GS_REQUIRE(!(herr & 4u), GSPARC_EINTERNAL, "numeric pass wrote past its chunk (symbolic count mismatch)");

    st.t_linearize_ms = tl.ms(0, 1);
    st.t_sort_ms = tl.ms(1, 2);
    st.t_match_ms = tl.ms(2, 3);
    st.t_plan_ms = tl.ms(3, 4);
    st.t_contract_ms = tl.ms(4, 5);
    st.t_output_ms = t_out;
    st.t_total_ms = tl.ms(0, 5);
    for (size_t i = 0; i + 1 < kev.size(); i += 2) {
        float t = 0.f;
        GS_CUDA(cudaEventElapsedTime(&t, kev[i], kev[i + 1]));
        st.t_numeric_kernel_ms += t;
    }
    for (auto e : kev) cudaEventDestroy(e);
    st.kernel_launches = launch_count() - launches0;
    if (st_out) *st_out = st;
}

}  // namespace gs
