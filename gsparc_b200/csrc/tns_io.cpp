// tns_io.cpp -- parallel .tns reader / writer.
//
// Format (reference: include/gsparc/io_manager.tpp:75-259): text COO, one
// nonzero per line, `i_1 ... i_N value`, indices 1-based, tokens separated by
// spaces or tabs, no header.  The order is the number of tokens on the first
// line minus one; dims[m] is the largest index seen in mode m (so the 0-based
// mode size is max + 1 after the shift); values are parsed as double and
// narrowed to float.  Unlike the reference, which counts '\n' characters as
// nonzeros, blank lines are skipped and malformed lines are reported.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"

namespace gs {

namespace {

inline bool is_sep(char c) { return c == ' ' || c == '\t' || c == '\r'; }

struct Span {
    size_t b, e;
};

// Count lines that hold at least one token in [b, e).
uint64_t count_lines(const char *buf, size_t b, size_t e) {
    uint64_t n = 0;
    size_t i = b;
    while (i < e) {
        size_t j = i;
        bool tok = false;
        while (j < e && buf[j] != '\n') {
            if (!is_sep(buf[j])) tok = true;
            ++j;
        }
        n += tok;
        i = j + 1;
    }
    return n;
}

}  // namespace

void read_tns(const char *path, int nthreads, int *order_out, uint64_t *dims_out, uint64_t *nnz_out,
              uint64_t **idx_out, float **val_out) {
    FILE *f = std::fopen(path, "rb");
    if (!f) fail(GSPARC_EIO, std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::rewind(f);
    std::vector<char> data((size_t)std::max<long>(sz, 0) + 1);
    if (sz > 0 && std::fread(data.data(), 1, (size_t)sz, f) != (size_t)sz) {
        std::fclose(f);
        fail(GSPARC_EIO, std::string("short read of ") + path);
    }
    std::fclose(f);
    const size_t n = (size_t)std::max<long>(sz, 0);
    data[n] = '\0';
    const char *buf = data.data();

    // order from the first line holding tokens
    int ntok = 0;
    {
        size_t i = 0;
        while (i < n) {
            size_t j = i;
            int t = 0;
            while (j < n && buf[j] != '\n') {
                while (j < n && is_sep(buf[j])) ++j;
                if (j >= n || buf[j] == '\n') break;
                ++t;
                while (j < n && buf[j] != '\n' && !is_sep(buf[j])) ++j;
            }
            if (t) {
                ntok = t;
                break;
            }
            i = j + 1;
        }
    }
    GS_REQUIRE(ntok >= 2, GSPARC_EINVAL, std::string("no nonzero found in ") + path);
    const int order = ntok - 1;
    GS_REQUIRE(order <= kMaxOrder, GSPARC_EUNSUPPORTED, "more than 32 modes");

    int T = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
    T = std::max(1, std::min<int>(T, (int)(n / (1 << 16)) + 1));
    // cut the buffer at line starts
    std::vector<size_t> cut(T + 1, 0);
    cut[T] = n;
    for (int t = 1; t < T; ++t) {
        size_t p = std::max(n * (size_t)t / (size_t)T, cut[t - 1]);
        while (p > 0 && p < n && buf[p - 1] != '\n') ++p;
        cut[t] = p;
    }
    std::vector<Span> spans(T);
    for (int t = 0; t < T; ++t) spans[t] = {cut[t], cut[t + 1]};

    std::vector<uint64_t> cnt(T + 1, 0);
    {
        std::vector<std::thread> th;
        for (int t = 0; t < T; ++t)
            th.emplace_back([&, t] { cnt[t + 1] = count_lines(buf, spans[t].b, spans[t].e); });
        for (auto &x : th) x.join();
    }
    for (int t = 0; t < T; ++t) cnt[t + 1] += cnt[t];
    const uint64_t nnz = cnt[T];

    uint64_t *idx = (uint64_t *)std::malloc(sizeof(uint64_t) * (size_t)order * std::max<uint64_t>(nnz, 1));
    float *val = (float *)std::malloc(sizeof(float) * std::max<uint64_t>(nnz, 1));
    if (!idx || !val) {
        std::free(idx);
        std::free(val);
        fail(GSPARC_ENOMEM, "host allocation for the tensor failed");
    }
    std::vector<std::vector<uint64_t>> mx(T, std::vector<uint64_t>(order, 0));
    std::vector<std::string> errs(T);
    {
        std::vector<std::thread> th;
        for (int t = 0; t < T; ++t) {
            th.emplace_back([&, t] {
                uint64_t k = cnt[t];
                size_t i = spans[t].b;
                const size_t e = spans[t].e;
                while (i < e) {
                    size_t j = i;
                    while (j < e && buf[j] != '\n') ++j;
                    // parse [i, j)
                    size_t p = i;
                    while (p < j && is_sep(buf[p])) ++p;
                    if (p < j) {
                        for (int m = 0; m < order; ++m) {
                            while (p < j && is_sep(buf[p])) ++p;
                            uint64_t v = 0;
                            size_t q = p;
                            while (q < j && buf[q] >= '0' && buf[q] <= '9') {
                                v = v * 10 + (uint64_t)(buf[q] - '0');
                                ++q;
                            }
                            if (q == p || v == 0 || (q < j && !is_sep(buf[q]))) {
                                if (errs[t].empty())
                                    errs[t] = "malformed index on line " + std::to_string(k + 1);
                                v = 1;
                            }
                            idx[(size_t)m * nnz + k] = v - 1;
                            if (v > mx[t][m]) mx[t][m] = v;
                            p = q;
                        }
                        while (p < j && is_sep(buf[p])) ++p;
                        char *endp = nullptr;
                        double d = 0.0;
                        if (p < j) d = std::strtod(buf + p, &endp);
                        if (p >= j || endp == buf + p) {
                            if (errs[t].empty()) errs[t] = "missing value on line " + std::to_string(k + 1);
                        }
                        val[k] = (float)d;
                        ++k;
                    }
                    i = j + 1;
                }
            });
        }
        for (auto &x : th) x.join();
    }
    for (int t = 0; t < T; ++t) {
        if (!errs[t].empty()) {
            std::free(idx);
            std::free(val);
            fail(GSPARC_EINVAL, std::string(path) + ": " + errs[t]);
        }
    }
    for (int m = 0; m < order; ++m) {
        uint64_t d = 0;
        for (int t = 0; t < T; ++t) d = std::max(d, mx[t][m]);
        dims_out[m] = d;
    }
    *order_out = order;
    *nnz_out = nnz;
    *idx_out = idx;
    *val_out = val;
}

void write_tns(const char *path, int order, uint64_t nnz, const uint64_t *idx, const float *val) {
    FILE *f = std::fopen(path, "w");
    if (!f) fail(GSPARC_EIO, std::string("cannot open ") + path + " for writing");
    std::vector<char> line(64 * (order + 2));
    for (uint64_t k = 0; k < nnz; ++k) {
        int len = 0;
        for (int m = 0; m < order; ++m)
            len += std::snprintf(line.data() + len, line.size() - len, "%llu ",
                                 (unsigned long long)(idx[(size_t)m * nnz + k] + 1));
        len += std::snprintf(line.data() + len, line.size() - len, "%.9g\n", (double)val[k]);
        if (std::fwrite(line.data(), 1, (size_t)len, f) != (size_t)len) {
            std::fclose(f);
            fail(GSPARC_EIO, std::string("write to ") + path + " failed");
        }
    }
    if (std::fclose(f) != 0) fail(GSPARC_EIO, std::string("closing ") + path + " failed");
}

}  // namespace gs
