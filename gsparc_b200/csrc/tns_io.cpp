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

// Quantum-chemistry directory format (reference: include/gsparc/io_manager.tpp:
// 310-484, the -q flag): <dir>/indices.txt holds one line per mode with the
// 1-based indices of all nonzeros of that mode, <dir>/values.txt the nnz
// values.  The order is the number of index lines, nnz the number of tokens
// of a line, dims[m] the largest index of mode m.  Indices are parsed as
// numbers (the reference uses strtod, so "3.0" is index 3).  Unlike the
// reference, values are parsed as double and narrowed to float (it scans
// "%le" into a float slot), blank lines are skipped, and lines of different
// lengths, non-integral or non-positive indices and missing values are
// reported instead of being read past.
void read_quantum(const char *dir, int nthreads, int *order_out, uint64_t *dims_out, uint64_t *nnz_out,
                  uint64_t **idx_out, float **val_out) {
    auto slurp = [](const std::string &p) {
        FILE *f = std::fopen(p.c_str(), "rb");
        if (!f) fail(GSPARC_EIO, "cannot open " + p);
        std::fseek(f, 0, SEEK_END);
        long sz = std::ftell(f);
        std::rewind(f);
        std::vector<char> d((size_t)std::max<long>(sz, 0) + 1, '\0');
        if (sz > 0 && std::fread(d.data(), 1, (size_t)sz, f) != (size_t)sz) {
            std::fclose(f);
            fail(GSPARC_EIO, "short read of " + p);
        }
        std::fclose(f);
        d[(size_t)std::max<long>(sz, 0)] = '\0';
        return d;
    };
    const std::string base(dir);
    std::vector<char> ib = slurp(base + "/indices.txt");
    std::vector<char> vb = slurp(base + "/values.txt");
    // index lines holding a token
    std::vector<Span> lines;
    {
        const size_t n = ib.size() - 1;
        size_t i = 0;
        while (i < n) {
            size_t j = i;
            bool tok = false;
            while (j < n && ib[j] != '\n') {
                if (!is_sep(ib[j])) tok = true;
                ++j;
            }
            if (tok) lines.push_back({i, j});
            i = j + 1;
        }
    }
    const int order = (int)lines.size();
    GS_REQUIRE(order >= 1 && order <= kMaxOrder, GSPARC_EIO, "indices.txt must hold 1..32 non-empty lines");
    for (auto &l : lines) ib[l.e] = '\0';  // each line ends its own string
    std::vector<std::vector<uint64_t>> rows(order);
    std::vector<std::string> errs(order);
    auto parse_row = [&](int m) {
        const char *p = ib.data() + lines[m].b;
        std::vector<uint64_t> &r = rows[m];
        for (;;) {
            while (*p && is_sep(*p)) ++p;
            if (!*p) break;
            char *end = nullptr;
            errno = 0;
            const double v = std::strtod(p, &end);
            if (end == p || errno || !(v >= 1.0) || v != (double)(uint64_t)v || v > 9.007199254740992e15) {
                errs[m] = "bad index on line " + std::to_string(m + 1) + " of indices.txt";
                return;
            }
            r.push_back((uint64_t)v - 1);
            p = end;
        }
    };
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    {
        std::vector<std::thread> th;
        const int nt = std::min(nthreads, order);
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                for (int m = t; m < order; m += nt) parse_row(m);
            });
        for (auto &x : th) x.join();
    }
    for (int m = 0; m < order; ++m) GS_REQUIRE(errs[m].empty(), GSPARC_EIO, errs[m]);
    const uint64_t nnz = rows[0].size();
    for (int m = 1; m < order; ++m)
        GS_REQUIRE(rows[m].size() == nnz, GSPARC_EIO, "index lines of indices.txt differ in length");
    // values
    float *val = (float *)std::malloc(sizeof(float) * std::max<uint64_t>(nnz, 1));
    uint64_t *idx = (uint64_t *)std::malloc(sizeof(uint64_t) * std::max<uint64_t>((uint64_t)order * nnz, 1));
    if (!val || !idx) {
        std::free(val);
        std::free(idx);
        fail(GSPARC_ENOMEM, "host allocation failed");
    }
    {
        const char *p = vb.data();
        for (uint64_t k = 0; k < nnz; ++k) {
            while (*p && (is_sep(*p) || *p == '\n')) ++p;
            char *end = nullptr;
            const double v = *p ? std::strtod(p, &end) : 0.0;
            if (!*p || end == p) {
                std::free(val);
                std::free(idx);
                fail(GSPARC_EIO, "values.txt holds fewer values than there are nonzeros");
            }
            val[k] = (float)v;
            p = end;
        }
    }
    for (int m = 0; m < order; ++m) {
        uint64_t mx = 0;
        for (uint64_t k = 0; k < nnz; ++k) {
            idx[(uint64_t)m * nnz + k] = rows[m][k];
            mx = std::max(mx, rows[m][k] + 1);
        }
        dims_out[m] = mx;
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
