// cli.cpp -- the `gsparc` command line, a thin program over the C ABI.
//
// Same options and stderr report as the reference binary
// (reference: src/gsparc/cmdline_opts.cpp:9-193, main.cu:22-437):
//   gsparc -X x.tns -Y y.tns -c N -x m1 .. mN -y m1 .. mN [-g G] [-n iters] [-d 1|0|-1]
// Extension: -o z.tns writes the output tensor (1-based, %.9g values).
// Chained multi-SpTC (-m 1 -a N -z m1 .. mN, main.cu:323-371): Z1 = X x Y stays
// on the device, then Z = Z1 x T with T the tensor of the -Y file (the
// reference parses it a second time for this, main.cu:42-48), contracting
// Z1's last N modes (Y's free modes, the low bits of the reference's Z1 keys
// that its second contraction matches on) with modes m1..mN of T.
// -t (extension) measures the accumulator and output chunk size first
// (gsparc_autotune) and runs the timed iterations with the fastest; it
// overrides -d.
// -q reads both operands from the quantum directory format (indices.txt +
// values.txt, io_manager.tpp:310-484).
#include <getopt.h>

#include <chrono>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "gsparc_b200.h"

namespace {

struct Opts {
    std::string X, Y, out;
    int nc = 0;
    std::vector<int> cx, cy;
    int gpus = 1, iters = 1, dense = 0;
    bool quantum = false;
    int multi = 0;
    bool host_copy = false;  // -H
    bool verify = false;     // -V
    bool one_device = false; // -e: the -g row shards one after another on device 0
    bool partition = false;  // -P: operands in parts from host memory (gsparc_sptc_host)
    int na = 0;
    std::vector<int> cz;
    bool tune = false;
};

[[noreturn]] void die(const char *what, gsparc_status st) {
    std::fprintf(stderr, "gsparc: %s: %s (%s)\n", what, gsparc_status_string(st), gsparc_last_error());
    std::exit(1);
}

void usage(const char *argv0) {
    std::fprintf(stderr,
                 "Usage: %s -X x.tns -Y y.tns -c N -x m1..mN -y m1..mN [-g G] [-n iters] [-d 1|0|-1] [-q]\n"
                 "          [-m 1 -a K -z t1..tK] [-t] [-o z.tns | -H] [-V] [-e] [-P]\n"
                 "  -H  copy every output chunk to page-locked host memory (and drop it there)\n"
                 "  -V  verify the values against FP64 sums on the GPU (all rows up to 2^28\n"
                 "      products, a seeded sample of rows above) and print the max errors\n"
                 "  -e  run the -g G row shards one after another on device 0 (their outputs\n"
                 "      concatenate into the same Z as on G devices)\n"
                 "  -P  contract from host memory in operand parts sized to the HBM budget (also\n"
                 "      taken when the whole operands do not fit, with one GPU)\n",
                 argv0);
}

struct Tensor {
    int order = 0;
    uint64_t dims[32] = {};
    uint64_t nnz = 0;
    uint64_t *idx = nullptr;
    float *val = nullptr;
};

struct OutCollect {
    std::vector<uint64_t> keys;  // kw words per nonzero (2: 128-bit keys, low word first)
    std::vector<float> vals;
    int kw = 1;
};

int collect_chunk(void *user, const uint64_t *k, const float *v, uint64_t n, uint64_t first, int on_device) {
    (void)on_device;
    auto *c = static_cast<OutCollect *>(user);
    if (c->vals.size() < first + n) {
        c->keys.resize(c->kw * (first + n));
        c->vals.resize(first + n);
    }
    std::memcpy(c->keys.data() + c->kw * first, k, 8 * c->kw * n);
    std::memcpy(c->vals.data() + first, v, 4 * n);
    return 0;
}

// The reference's stderr report (main.cu:415-432); times in seconds.
// reorder >= 0 (chained multi-SpTC only) adds the two bit-reordering lines of
// main.cu:422-426: the re-keying time of the first result per iteration and its
// share of the per-iteration total.
void print_report(double slitom, double idxmatch, double contraction, double dprtn, uint64_t result_nnz,
                  int iters, double reorder = -1.0) {
    const double partition = 0.0;
    const double n = iters;
    const double total = slitom + partition + idxmatch + contraction + dprtn;
    std::fprintf(stderr, "--------Break Down--------\n");
    std::fprintf(stderr, "SLITOM time: %f\n", slitom / n);
    std::fprintf(stderr, "Partition time: %f\n", partition / n);
    std::fprintf(stderr, "Idxmatch time: %f\n", idxmatch / n);
    std::fprintf(stderr, "Contraction time: %f\n", contraction / n);
    std::fprintf(stderr, "Dynamic Partition time: %f\n", dprtn / n);
    if (reorder >= 0.0) {
        std::fprintf(stderr, "Bit reordering time: %f\n", reorder / n);
        std::fprintf(stderr, "Bit reordering ratio: %f%%\n", total > 0 ? (reorder / total) * 100.0 : 0.0);
    }
    std::fprintf(stderr, "--------Elapsed Time--------\n");
    std::fprintf(stderr, "Result NNZ: %llu\n", (unsigned long long)(result_nnz / iters));
    std::fprintf(stderr, "SLITOM time: %f\n", slitom / n);
    std::fprintf(stderr, "Partition time: %f\n", partition / n);
    std::fprintf(stderr, "SpTC(IdxMatch + Contraction + Data Copy) time: %f\n", (idxmatch + contraction + dprtn) / n);
    std::fprintf(stderr, "Total time: %f\n", total / n);
    std::fprintf(stderr, "\n\n");
}

// Key words of the output: 2 when X's free bits + Y's free bits exceed 64.
int out_words(const Tensor &tx, const std::vector<int> &cx, const Tensor &ty, const std::vector<int> &cy, int nc) {
    int b[32], sh[32], ic[32], ncb, nfx, nfy;
    gsparc_layout(tx.order, tx.dims, nc, cx.data(), b, sh, ic, &ncb, &nfx);
    gsparc_layout(ty.order, ty.dims, nc, cy.data(), b, sh, ic, &ncb, &nfy);
    return nfx + nfy > 64 ? 2 : 1;
}

// Output keys -> coordinates (X free modes ascending, then Y free modes), written as .tns.
void write_output(const std::string &path, const OutCollect &out, int xo, const uint64_t *xd, const int *cx,
                  int yo, const uint64_t *yd, const int *cy, int nc) {
    int bx[32], shx[32], icx[32], ncx, nfx, by[32], shy[32], icy[32], ncy, nfy;
    gsparc_layout(xo, xd, nc, cx, bx, shx, icx, &ncx, &nfx);
    gsparc_layout(yo, yd, nc, cy, by, shy, icy, &ncy, &nfy);
    std::vector<int> fmx, fmy;
    for (int m = 0; m < xo; ++m) if (!icx[m]) fmx.push_back(m);
    for (int m = 0; m < yo; ++m) if (!icy[m]) fmy.push_back(m);
    const int zo = (int)(fmx.size() + fmy.size());
    const uint64_t zn = out.vals.size();
    std::vector<uint64_t> zi((size_t)zo * zn);
    for (uint64_t k = 0; k < zn; ++k) {
        // the key is x_f << nfy | y_f, in one word or (kw == 2) in two
        const unsigned __int128 key = out.kw == 2 ? ((unsigned __int128)out.keys[2 * k + 1] << 64) | out.keys[2 * k]
                                                  : (unsigned __int128)out.keys[k];
        uint64_t xf = (uint64_t)(key >> nfy);
        uint64_t yf = nfy >= 64 ? (uint64_t)key : (uint64_t)key & ((1ull << nfy) - 1);
        int z = 0;
        for (int m : fmx) zi[(size_t)(z++) * zn + k] = (xf >> shx[m]) & ((bx[m] >= 64) ? ~0ull : ((1ull << bx[m]) - 1));
        for (int m : fmy) zi[(size_t)(z++) * zn + k] = (yf >> shy[m]) & ((by[m] >= 64) ? ~0ull : ((1ull << by[m]) - 1));
    }
    gsparc_status st = gsparc_write_tns(path.c_str(), zo, zn, zi.data(), out.vals.data());
    if (st) die("writing Z", st);
}

// -m: Z1 = X x Y kept on the device, then Z = Z1 x T (T = the -Y tensor),
// Z1's last N modes against T's modes -z m1..mN.  One GPU.
int run_multi(const Opts &o, const Tensor &tx, const Tensor &ty) {
    if (o.gpus != 1) {
        std::fprintf(stderr, "gsparc: chained multi-SpTC (-m) runs on one GPU (-g 1)\n");
        return 1;
    }
    const int yfree = ty.order - o.nc;
    if (o.na < 1 || o.na > yfree || (int)o.cz.size() != o.na) {
        std::fprintf(stderr, "gsparc: -m needs -a N (1..%d, Y's free modes) and -z with N modes of the -Y tensor\n",
                     yfree);
        return 1;
    }
    double slitom = 0, idxmatch = 0, contraction = 0, dprtn = 0, first = 0, reorder = 0;
    uint64_t result_nnz = 0;
    OutCollect out;
    int z1o = 0;
    uint64_t z1d[32] = {};
    std::vector<int> cz1(o.na);
    gsparc_ctx *ctx = nullptr;
    gsparc_status s = gsparc_ctx_create(0, 0, &ctx);
    if (!s) s = gsparc_ctx_reserve(ctx, 0);
    if (s) die("context", s);
    for (int it = 0; it < o.iters; ++it) {
        const uint64_t *ix[32], *iy[32];
        for (int m = 0; m < tx.order; ++m) ix[m] = tx.idx + (size_t)m * tx.nnz;
        for (int m = 0; m < ty.order; ++m) iy[m] = ty.idx + (size_t)m * ty.nnz;
        gsparc_coo cx{tx.order, tx.dims, tx.nnz, ix, tx.val, 0};
        gsparc_coo cy{ty.order, ty.dims, ty.nnz, iy, ty.val, 0};
        gsparc_tensor *X = nullptr, *Y = nullptr, *Z1 = nullptr;
        auto t0 = std::chrono::steady_clock::now();
        if ((s = gsparc_tensor_upload(ctx, &cx, nullptr, &X)) || (s = gsparc_tensor_upload(ctx, &cy, nullptr, &Y)))
            die("upload", s);
        const double up = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        gsparc_stats s1{}, s2{};
        s = gsparc_sptc_resident(ctx, X, Y, o.nc, o.cx.data(), o.cy.data(), o.dense, &Z1, &s1, nullptr);
        if (s) die("first contraction", s);
        first += (up + s1.t_linearize_ms + s1.t_sort_ms + s1.t_match_ms + s1.t_plan_ms + s1.t_contract_ms) / 1e3;
        gsparc_tensor_info(Z1, &z1o, z1d, nullptr);
        for (int i = 0; i < o.na; ++i) cz1[i] = z1o - o.na + i;
        gsparc_sink sink{};
        sink.kind = GSPARC_SINK_DISCARD;
        std::vector<uint64_t> hk;
        std::vector<float> hv;
        if (!o.out.empty() && it == 0) {
            sink.kind = GSPARC_SINK_HOST;
            hk.resize(1 << 24);
            hv.resize(1 << 24);
            sink.host_keys = hk.data();
            sink.host_vals = hv.data();
            sink.host_capacity = hk.size();
            sink.on_chunk = collect_chunk;
            sink.user = &out;
        }
        s = gsparc_sptc(ctx, Z1, Y, o.na, cz1.data(), o.cz.data(), o.dense, &sink, &s2, nullptr);
        if (s) die("second contraction", s);
        result_nnz += s2.nnz;
        // the first result re-keyed as the second contraction's X (main.cu:351-358): its linearise
        reorder += s2.t_linearize_ms / 1e3;
        slitom += (up + s1.t_linearize_ms + s1.t_sort_ms + s2.t_linearize_ms + s2.t_sort_ms) / 1e3;
        idxmatch += (s1.t_match_ms + s2.t_match_ms) / 1e3;
        dprtn += (s1.t_plan_ms + s2.t_plan_ms) / 1e3;
        contraction += (s1.t_contract_ms + s2.t_contract_ms) / 1e3;
        gsparc_tensor_free(ctx, Z1);
        gsparc_tensor_free(ctx, X);
        gsparc_tensor_free(ctx, Y);
    }
    gsparc_ctx_destroy(ctx);
    std::fprintf(stderr, "First SpTC time: %f\n", first / o.iters);
    print_report(slitom, idxmatch, contraction, dprtn, result_nnz, o.iters, reorder);
    if (!o.out.empty()) write_output(o.out, out, z1o, z1d, cz1.data(), ty.order, ty.dims, o.cz.data(), o.na);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    Opts o;
    int c;
    while ((c = getopt(argc, argv, "X:Y:c:a:m:x:y:z:n:g:d:o:qbhvtHVeP")) != -1) {
        switch (c) {
        case 'X':
            std::fprintf(stderr, "tensor X: %s\n", optarg);
            o.X = optarg;
            break;
        case 'Y':
            std::fprintf(stderr, "tensor Y: %s\n", optarg);
            o.Y = optarg;
            break;
        case 'c':
            o.nc = std::atoi(optarg);
            break;
        case 'a':
            o.na = std::atoi(optarg);
            break;
        case 'x':
        case 'y':
        case 'z': {
            // the modes follow the flag as separate arguments (cmdline_opts.cpp:112-139,140-155)
            std::vector<int> &v = c == 'x' ? o.cx : (c == 'y' ? o.cy : o.cz);
            const int k = c == 'z' ? o.na : o.nc;
            if (c == 'z')
                std::fprintf(stderr, "# contract modes of Z (second SpTC): %d, contract modes: ", k);
            else
                std::fprintf(stderr, "# contract modes of %c: %d, contract modes: ", c == 'x' ? 'X' : 'Y', k);
            v.clear();
            for (int i = 0; i < k; ++i) {
                if (optind - 1 + i >= argc) {
                    std::fprintf(stderr, "\ngsparc: -%c needs %d modes\n", c, k);
                    return 1;
                }
                v.push_back(std::atoi(argv[optind - 1 + i]));
                std::fprintf(stderr, "%d ", v.back());
            }
            std::fprintf(stderr, "\n");
            optind += k - 1;
            break;
        }
        case 'g':
            o.gpus = std::atoi(optarg);
            std::fprintf(stderr, "num_gpus: %d\n", o.gpus);
            break;
        case 'n':
            o.iters = std::atoi(optarg);
            break;
        case 'd':
            o.dense = std::atoi(optarg);
            std::fprintf(stderr, "dense_accumulator: %d\n", o.dense);
            break;
        case 'o':
            o.out = optarg;
            break;
        case 'q':
            o.quantum = true;
            break;
        case 'm':
            o.multi = std::atoi(optarg);
            std::fprintf(stderr, "multi_sptc: %d\n", o.multi);
            break;
        case 't':
            o.tune = true;
            break;
        case 'H':
            o.host_copy = true;
            break;
        case 'V':
            o.verify = true;
            break;
        case 'e':
            o.one_device = true;
            break;
        case 'P':
            o.partition = true;
            break;
        case 'b':
        case 'v':
            break;
        case 'h':
            usage(argv[0]);
            return 0;
        default:
            usage(argv[0]);
            return 1;
        }
    }
    if (o.X.empty() || o.Y.empty() || o.nc < 1 || (int)o.cx.size() != o.nc || (int)o.cy.size() != o.nc ||
        o.gpus < 1 || o.iters < 1 || o.dense < -1 || o.dense > 1) {
        usage(argv[0]);
        return 1;
    }

    Tensor tx, ty;
    // -q: both operands in the quantum directory format (main.cu:44-48)
    auto rd = o.quantum ? gsparc_read_quantum : gsparc_read_tns;
    gsparc_status st = rd(o.X.c_str(), 0, &tx.order, tx.dims, &tx.nnz, &tx.idx, &tx.val);
    if (st) die("reading X", st);
    st = rd(o.Y.c_str(), 0, &ty.order, ty.dims, &ty.nnz, &ty.idx, &ty.val);
    if (st) die("reading Y", st);
    // page-locked operands upload at the full host-link rate (not timed, like
    // the reference's cudaHostAlloc of its converted operands); unpinned
    // memory still works if the host refuses to lock it
    void *const bufs[4] = {tx.idx, tx.val, ty.idx, ty.val};
    const uint64_t lens[4] = {8ull * tx.order * tx.nnz, 4ull * tx.nnz, 8ull * ty.order * ty.nnz, 4ull * ty.nnz};
    bool pinned[4];
    for (int i = 0; i < 4; ++i) pinned[i] = lens[i] && gsparc_host_pin(bufs[i], lens[i]) == GSPARC_OK;
    auto release = [&] {
        for (int i = 0; i < 4; ++i) {
            if (pinned[i]) gsparc_host_unpin(bufs[i]);
            gsparc_free_host(bufs[i]);
        }
    };
    if (o.multi) {
        const int rc = run_multi(o, tx, ty);
        release();
        return rc;
    }

    double slitom = 0, idxmatch = 0, contraction = 0, dprtn = 0;
    uint64_t result_nnz = 0;
    OutCollect out;
    gsparc_stats vsum{};  // -V: verification of the last iteration, over all GPUs

    // One context per GPU for the whole run, its pool mapped before any stage
    // is timed (the reference builds its memory pools once, main.cu:56-66).
    const int nctx = o.one_device ? 1 : o.gpus;
    std::vector<gsparc_ctx *> ctxs(nctx, nullptr);
    {
        std::vector<gsparc_status> cst(nctx, GSPARC_OK);
        std::vector<std::thread> th;
        for (int g = 0; g < nctx; ++g)
            th.emplace_back([&, g] {
                cst[g] = gsparc_ctx_create(g, 0, &ctxs[g]);
                if (!cst[g]) cst[g] = gsparc_ctx_reserve(ctxs[g], 0);
                if (!cst[g] && o.verify) cst[g] = gsparc_ctx_set_verify(ctxs[g], 1ull << 28);
            });
        for (auto &t : th) t.join();
        for (int g = 0; g < nctx; ++g)
            if (cst[g]) {
                for (auto c : ctxs)
                    if (c) gsparc_ctx_destroy(c);
                die("creating the device context", cst[g]);
            }
    }

    for (int it = 0; it < o.iters; ++it) {
        std::vector<gsparc_stats> stats(o.gpus);
        std::vector<gsparc_status> sts(o.gpus, GSPARC_OK);
        std::vector<double> upload_ms(o.gpus, 0.0);
        std::vector<OutCollect> parts(o.gpus);
        auto run = [&](int g) {
            gsparc_ctx *ctx = ctxs[o.one_device ? 0 : g];
            gsparc_status s = GSPARC_OK;
            const uint64_t *ix[32], *iy[32];
            for (int m = 0; m < tx.order; ++m) ix[m] = tx.idx + (size_t)m * tx.nnz;
            for (int m = 0; m < ty.order; ++m) iy[m] = ty.idx + (size_t)m * ty.nnz;
            gsparc_coo cx{tx.order, tx.dims, tx.nnz, ix, tx.val, 0};
            gsparc_coo cy{ty.order, ty.dims, ty.nnz, iy, ty.val, 0};
            gsparc_tensor *X = nullptr, *Y = nullptr;
            // operands in parts from host memory (FindPartitionNum / Partition,
            // tensor_manager.tpp:33-61,634-886): asked for, or when they do not fit
            auto run_parts = [&]() {
                gsparc_sink sink{};
                sink.kind = GSPARC_SINK_DISCARD;
                std::vector<uint64_t> hk;
                std::vector<float> hv;
                if (!o.out.empty()) {
                    sink.kind = GSPARC_SINK_HOST;
                    hk.resize(1 << 24);
                    hv.resize(1 << 24);
                    sink.host_keys = hk.data();
                    sink.host_vals = hv.data();
                    sink.host_capacity = hk.size();
                    sink.on_chunk = collect_chunk;
                    sink.user = &parts[g];
                }
                return gsparc_sptc_host(ctx, &cx, &cy, o.nc, o.cx.data(), o.cy.data(), o.dense, nullptr, &sink,
                                        &stats[g], nullptr);
            };
            if (o.partition) {
                sts[g] = run_parts();
                return;
            }
            auto t0 = std::chrono::steady_clock::now();
            if (!(s = gsparc_tensor_upload(ctx, &cx, nullptr, &X)) &&
                !(s = gsparc_tensor_upload(ctx, &cy, nullptr, &Y))) {
                upload_ms[g] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                gsparc_sink sink{};
                sink.kind = GSPARC_SINK_DISCARD;
                std::vector<uint64_t> hk;
                std::vector<float> hv;
                if (o.host_copy && o.out.empty()) {
                    // -H: every output chunk copied to a page-locked host ring and
                    // dropped there, as the reference copies each output partition to
                    // pinned host memory (contraction.cuh:554-555)
                    sink.kind = GSPARC_SINK_HOST;
                    hk.resize(1 << 26);
                    hv.resize(1 << 26);
                    sink.host_keys = hk.data();
                    sink.host_vals = hv.data();
                    sink.host_capacity = hk.size();
                    const bool pk = gsparc_host_pin(hk.data(), 8 * hk.size()) == GSPARC_OK;
                    const bool pv = gsparc_host_pin(hv.data(), 4 * hv.size()) == GSPARC_OK;
                    if (!s)
                        s = gsparc_sptc_shard(ctx, X, Y, o.nc, o.cx.data(), o.cy.data(), o.dense, g, o.gpus, &sink,
                                              &stats[g], nullptr);
                    if (pk) gsparc_host_unpin(hk.data());
                    if (pv) gsparc_host_unpin(hv.data());
                    if (X) gsparc_tensor_free(ctx, X);
                    if (Y) gsparc_tensor_free(ctx, Y);
                    sts[g] = s;
                    return;
                }
                if (!o.out.empty()) {
                    // output keys over 64 bits come as two words each
                    const int kw = out_words(tx, o.cx, ty, o.cy, o.nc);
                    parts[g].kw = kw;
                    sink.kind = GSPARC_SINK_HOST;
                    sink.key_words = kw;
                    hk.resize((size_t)kw << 24);
                    hv.resize(1 << 24);
                    sink.host_keys = hk.data();
                    sink.host_vals = hv.data();
                    sink.host_capacity = hv.size();
                    sink.on_chunk = collect_chunk;
                    sink.user = &parts[g];
                }
                int accum = o.dense;
                if (o.tune) {
                    // measured choice (cached per shape, so only the first iteration pays)
                    gsparc_tuning tn{};
                    s = gsparc_autotune(ctx, X, Y, o.nc, o.cx.data(), o.cy.data(), 0, &tn, nullptr);
                    if (!s) {
                        accum = tn.accum;
                        sink.max_chunk_nnz = tn.max_chunk_nnz;
                        s = gsparc_ctx_set_tiles(ctx, tn.light_row_max, tn.heavy_window_cap);
                        if (it == 0 && g == 0)
                            std::fprintf(stderr,
                                         "autotune: dense_accumulator %d, chunk %llu, light rows %llu, heavy window "
                                         "%u, %.3f ms\n",
                                         tn.accum, (unsigned long long)tn.max_chunk_nnz,
                                         (unsigned long long)tn.light_row_max, tn.heavy_window_cap, tn.ms);
                    }
                }
                if (!s)
                    s = gsparc_sptc_shard(ctx, X, Y, o.nc, o.cx.data(), o.cy.data(), accum, g, o.gpus, &sink,
                                          &stats[g], nullptr);
            }
            if (X) gsparc_tensor_free(ctx, X);
            if (Y) gsparc_tensor_free(ctx, Y);
            if (s == GSPARC_ENOMEM && o.gpus == 1 && !o.host_copy) {
                parts[g] = OutCollect{};
                stats[g] = gsparc_stats{};
                upload_ms[g] = 0;
                s = run_parts();
            }
            sts[g] = s;
        };
        std::vector<std::thread> th;
        for (int g = 0; g < o.gpus; ++g) {
            if (o.one_device)
                run(g);
            else
                th.emplace_back(run, g);
        }
        for (auto &t : th) t.join();
        for (int g = 0; g < o.gpus; ++g)
            if (sts[g]) {
                for (auto c : ctxs) gsparc_ctx_destroy(c);
                die("contraction", sts[g]);
            }
        vsum = gsparc_stats{};
        for (int g = 0; g < o.gpus; ++g) {
            const gsparc_stats &s = stats[g];
            vsum.verified_nnz += s.verified_nnz;
            vsum.verified_products += s.verified_products;
            vsum.verify_mismatch += s.verify_mismatch;
            vsum.max_rel_err = std::max(vsum.max_rel_err, s.max_rel_err);
            vsum.max_abs_err = std::max(vsum.max_abs_err, s.max_abs_err);
            if (s.accumulator == GSPARC_ACCUM_DENSE) std::fprintf(stderr, "Dense Accumulator\n");
            result_nnz += s.nnz;
            slitom += (upload_ms[g] + s.t_linearize_ms + s.t_sort_ms) / 1e3 / o.gpus;
            idxmatch += s.t_match_ms / 1e3 / o.gpus;
            dprtn += s.t_plan_ms / 1e3 / o.gpus;
            contraction += s.t_contract_ms / 1e3 / o.gpus;
        }
        if (it == 0 && !o.out.empty()) {
            uint64_t base = 0;
            for (int g = 0; g < o.gpus; ++g) {
                out.kw = parts[g].kw;
                out.keys.insert(out.keys.end(), parts[g].keys.begin(), parts[g].keys.end());
                out.vals.insert(out.vals.end(), parts[g].vals.begin(), parts[g].vals.end());
                base += parts[g].keys.size();
            }
        }
    }

    for (auto c : ctxs) gsparc_ctx_destroy(c);
    print_report(slitom, idxmatch, contraction, dprtn, result_nnz, o.iters);
    if (o.verify)
        std::fprintf(stderr,
                     "FP64 verification: %llu outputs, %llu products, %llu mismatches, max rel err %.3e, "
                     "max abs err %.3e\n",
                     (unsigned long long)vsum.verified_nnz, (unsigned long long)vsum.verified_products,
                     (unsigned long long)vsum.verify_mismatch, vsum.max_rel_err, vsum.max_abs_err);
    if (!o.out.empty()) write_output(o.out, out, tx.order, tx.dims, o.cx.data(), ty.order, ty.dims, o.cy.data(), o.nc);
    release();
    return 0;
}
