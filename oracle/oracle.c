/*
 * oracle.c -- CPU restatement of GSPARC's SpTC path.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the CUDA engine in gsparc_b200/: only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it.  The
 * product path never calls it.
 *
 * It restates, in plain C, the semantics of the reference's path
 * (seohyeon0322/GSPARC), step by step:
 *
 *   parse .tns          include/gsparc/io_manager.tpp:75-259 (dims = max idx + 1, :213,:250-256)
 *   mode bit widths     include/gsparc/tensor_manager.tpp:107-125 (64 - clz(dim-1))
 *   free-mode order     include/gsparc/tensor_manager.tpp:64-88
 *   masks / shifts      include/gsparc/tensor_manager.tpp:153-174 (first mode highest)
 *   linearise           include/gsparc/tensor_manager.tpp:246-268 (X: f<<ncbits|c)
 *                       include/gsparc/tensor_manager.tpp:270-294 (Y: c<<nfbits|f)
 *   stable sort by key  include/gsparc/sort.cuh:90-108 (CUB radix sort, stable)
 *   index match         include/gsparc/indexMatch.cuh:20-44,67-118,231-287
 *   ESC expand          include/gsparc/contraction.cuh:100-141 (key x_f<<Y_nfbits | y_f)
 *   sort + reduce       include/gsparc/contraction.cuh:506-537 (ascending keys, Sum)
 *   quantum input       include/gsparc/io_manager.tpp:310-484 (indices.txt + values.txt)
 *   keys over 64 bits   include/gsparc/tensor_manager.tpp:301-406 (ConvertTensor_extra:
 *                       the same layouts in a 128-bit key), include/gsparc/indexMatch.cuh:
 *                       120-229 (match on the full 128-bit contract key); output keys
 *                       stay 64-bit (include/gsparc/contraction_extra.cuh)
 *
 * nnz follows the ESC semantics: every distinct output key that received at
 * least one product counts, including sums that cancel to exactly zero.
 * Values are summed in double precision.  Mode widths of one bit-width 0 are
 * used for size-1 modes (the reference's clz(0) is undefined there).
 *
 * Parity status: the restatement is pinned against outputs of the
 * reference's own CPU SpTC (baselines/Sparta, built from source by
 * oracle/Makefile) through fixtures in tests/golden/.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define OR_OK 0
#define OR_EINVAL 1
#define OR_ENOMEM 2
#define OR_EIO 4

/* ------------------------------------------------------------------ bits */

/* tensor_manager.tpp:109 -- bits = 64 - clz(dim - 1); dim 1 gives 0 here. */
int oracle_mode_bits(uint64_t dim)
{
    if (dim <= 1)
        return 0;
    return 64 - __builtin_clzll(dim - 1);
}

/*
 * Layout of one operand: shift[m] for every mode m (position of the mode's
 * field inside its free or contract part), ncbits, nfbits.
 * Free modes are the non-contract modes in ascending order (tensor_manager.tpp:64-88);
 * the LAST free (contract) mode sits in the lowest bits and the first one in
 * the highest bits (tensor_manager.tpp:153-174).
 */
int oracle_layout(int order, const uint64_t *dims, int nc, const int *cpos,
                  int *shift, int *is_contract, int *fpos_out,
                  int *ncbits, int *nfbits)
{
    int fpos[64];
    int nf = 0;
    if (order <= 0 || order > 64 || nc < 0 || nc > order)
        return OR_EINVAL;
    for (int m = 0; m < order; ++m)
        is_contract[m] = 0;
    for (int i = 0; i < nc; ++i) {
        if (cpos[i] < 0 || cpos[i] >= order || is_contract[cpos[i]])
            return OR_EINVAL;
        is_contract[cpos[i]] = 1;
    }
    for (int m = 0; m < order; ++m)
        if (!is_contract[m])
            fpos[nf++] = m;
    int s = 0;
    for (int n = nf - 1; n >= 0; --n) {
        shift[fpos[n]] = s;
        s += oracle_mode_bits(dims[fpos[n]]);
    }
    *nfbits = s;
    s = 0;
    for (int n = nc - 1; n >= 0; --n) {
        shift[cpos[n]] = s;
        s += oracle_mode_bits(dims[cpos[n]]);
    }
    *ncbits = s;
    if (fpos_out)
        for (int i = 0; i < nf; ++i)
            fpos_out[i] = fpos[i];
    return OR_OK;
}

/*
 * Linearise one operand.  role 0 = X layout (f << ncbits | c),
 * role 1 = Y layout (c << nfbits | f).  idx is SoA: idx[m*nnz + k].
 */
int oracle_linearize(int order, const uint64_t *dims, int nc, const int *cpos,
                     int role, uint64_t nnz, const uint64_t *idx, uint64_t *keys)
{
    int shift[64], isc[64], ncb, nfb;
    int st = oracle_layout(order, dims, nc, cpos, shift, isc, NULL, &ncb, &nfb);
    if (st)
        return st;
    if (ncb + nfb > 64)
        return OR_EINVAL;
    for (uint64_t k = 0; k < nnz; ++k) {
        uint64_t f = 0, c = 0;
        for (int m = 0; m < order; ++m) {
            uint64_t v = idx[(uint64_t)m * nnz + k];
            if (isc[m])
                c |= v << shift[m];
            else
                f |= v << shift[m];
        }
        keys[k] = role == 0 ? ((ncb >= 64 ? 0 : (f << ncb)) | c)
                            : ((nfb >= 64 ? 0 : (c << nfb)) | f);
    }
    return OR_OK;
}

/*
 * 128-bit keys (tensor_manager.tpp:301-406): the layouts above, in a key of
 * up to 128 bits.  Used by oracle_sptc for every operand; keys of at most 64
 * bits come out identical to oracle_linearize's.
 */
typedef unsigned __int128 u128;

static void linearize128(int order, const int *shift, const int *isc, int ncb, int nfb,
                         int role, uint64_t nnz, const uint64_t *idx, u128 *keys)
{
    for (uint64_t k = 0; k < nnz; ++k) {
        u128 f = 0, c = 0;
        for (int m = 0; m < order; ++m) {
            u128 v = idx[(uint64_t)m * nnz + k];
            if (isc[m])
                c |= v << shift[m];
            else
                f |= v << shift[m];
        }
        keys[k] = role == 0 ? ((ncb >= 128 ? 0 : (f << ncb)) | c)
                            : ((nfb >= 128 ? 0 : (c << nfb)) | f);
    }
}

/* Stable LSD radix sort (16-bit digits) of 128-bit keys over their low nbits
 * bits; perm receives the sorted order. */
static int stable_sort_perm128(uint64_t n, const u128 *keys, int nbits, uint64_t *perm)
{
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    uint64_t *cnt = (uint64_t *)malloc(sizeof(uint64_t) * 65536);
    if (!tmp || !cnt) {
        free(tmp);
        free(cnt);
        return OR_ENOMEM;
    }
    for (uint64_t i = 0; i < n; ++i)
        perm[i] = i;
    uint64_t *a = perm, *b = tmp;
    for (int sh = 0; sh < nbits; sh += 16) {
        memset(cnt, 0, sizeof(uint64_t) * 65536);
        for (uint64_t i = 0; i < n; ++i)
            cnt[(uint64_t)(keys[a[i]] >> sh) & 0xFFFF]++;
        uint64_t run = 0;
        for (int d = 0; d < 65536; ++d) {
            uint64_t c = cnt[d];
            cnt[d] = run;
            run += c;
        }
        for (uint64_t i = 0; i < n; ++i)
            b[cnt[(uint64_t)(keys[a[i]] >> sh) & 0xFFFF]++] = a[i];
        uint64_t *t = a;
        a = b;
        b = t;
    }
    if (a != perm)
        memcpy(perm, a, sizeof(uint64_t) * n);
    free(tmp);
    free(cnt);
    return OR_OK;
}

/* ------------------------------------------------------------- sorting */

/* Stable LSD radix sort of keys with a permutation payload (16-bit digits). */
static int stable_sort_perm(uint64_t n, const uint64_t *keys, int nbits, uint64_t *perm)
{
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    uint64_t *cnt = (uint64_t *)malloc(sizeof(uint64_t) * 65536);
    if (!tmp || !cnt) {
        free(tmp);
        free(cnt);
        return OR_ENOMEM;
    }
    for (uint64_t i = 0; i < n; ++i)
        perm[i] = i;
    uint64_t *a = perm, *b = tmp;
    for (int sh = 0; sh < nbits; sh += 16) {
        memset(cnt, 0, sizeof(uint64_t) * 65536);
        for (uint64_t i = 0; i < n; ++i)
            cnt[(keys[a[i]] >> sh) & 0xFFFF]++;
        uint64_t run = 0;
        for (int d = 0; d < 65536; ++d) {
            uint64_t c = cnt[d];
            cnt[d] = run;
            run += c;
        }
        for (uint64_t i = 0; i < n; ++i)
            b[cnt[(keys[a[i]] >> sh) & 0xFFFF]++] = a[i];
        uint64_t *t = a;
        a = b;
        b = t;
    }
    if (a != perm)
        memcpy(perm, a, sizeof(uint64_t) * n);
    free(tmp);
    free(cnt);
    return OR_OK;
}

/* Sort (keys, vals) in place by key, stable (sort.cuh:90-108 semantics). */
int oracle_sort_pairs(uint64_t n, uint64_t *keys, float *vals, int nbits)
{
    uint64_t *perm = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    uint64_t *k2 = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    float *v2 = (float *)malloc(sizeof(float) * (n ? n : 1));
    if (!perm || !k2 || !v2) {
        free(perm);
        free(k2);
        free(v2);
        return OR_ENOMEM;
    }
    int st = stable_sort_perm(n, keys, nbits, perm);
    if (!st) {
        for (uint64_t i = 0; i < n; ++i) {
            k2[i] = keys[perm[i]];
            v2[i] = vals[perm[i]];
        }
        memcpy(keys, k2, sizeof(uint64_t) * n);
        memcpy(vals, v2, sizeof(float) * n);
    }
    free(perm);
    free(k2);
    free(v2);
    return st;
}

/* ------------------------------------------------------------ matching */

/*
 * indexMatch.cuh:20-44 + :67-118 -- for every X nonzero (sorted X keys), the
 * first Y position whose contract key (y >> fbits) equals x & cmask, and the
 * length of that run.  pos is left 0 and cnt 0 when there is no match
 * (the reference memsets both arrays, sptc.cuh:144-146).
 * prefix[0] = 0, prefix[i+1] = cnt[0] + ... + cnt[i] (indexMatch.cuh:275-285).
 */
int oracle_index_match(uint64_t nx, const uint64_t *xkeys, int x_ncbits,
                       uint64_t ny, const uint64_t *ykeys, int y_nfbits,
                       uint64_t *pos, uint64_t *cnt, uint64_t *prefix)
{
    uint64_t cmask = x_ncbits >= 64 ? ~0ull : ((1ull << x_ncbits) - 1);
    prefix[0] = 0;
    for (uint64_t i = 0; i < nx; ++i) {
        uint64_t c = xkeys[i] & cmask;
        uint64_t lo = 0, hi = ny;
        while (lo < hi) {
            uint64_t mid = lo + (hi - lo) / 2;
            uint64_t yc = y_nfbits >= 64 ? 0 : (ykeys[mid] >> y_nfbits);
            if (yc < c)
                lo = mid + 1;
            else
                hi = mid;
        }
        uint64_t n = 0;
        if (lo < ny && (y_nfbits >= 64 ? 0 : (ykeys[lo] >> y_nfbits)) == c) {
            pos[i] = lo;
            while (lo + n < ny && (y_nfbits >= 64 ? 0 : (ykeys[lo + n] >> y_nfbits)) == c)
                ++n;
        } else {
            pos[i] = 0;
        }
        cnt[i] = n;
        prefix[i + 1] = prefix[i] + n;
    }
    return OR_OK;
}

/* --------------------------------------------------------------- SpTC */

typedef struct {
    uint64_t ir_nnz;     /* matched products */
    uint64_t nnz;        /* distinct output keys */
    int x_nfbits, y_nfbits, ncbits_x, ncbits_y;
    uint64_t *keys;      /* [nnz] ascending output keys (x_f << y_nfbits | y_f) */
    double *vals;        /* [nnz] FP64 sums */
    double *abs_sums;    /* [nnz] sum of |products| (scale for tolerances) */
    uint64_t *nprod;     /* [nnz] products per key */
} oracle_result;

void oracle_free(oracle_result *r)
{
    if (!r)
        return;
    free(r->keys);
    free(r->vals);
    free(r->abs_sums);
    free(r->nprod);
    free(r);
}

/*
 * Full path: linearise X and Y, stable-sort both, match, expand every product
 * with key (x_f << Y_nfbits) | y_f (contraction.cuh:132-137), sort the products
 * by key and reduce equal keys.  idx arrays are SoA, 0-based.
 * max_products bounds the expansion (the oracle is for small cases).
 */
int oracle_sptc(int ox, const uint64_t *dx, uint64_t nx, const uint64_t *ix, const float *vx,
                int oy, const uint64_t *dy, uint64_t ny, const uint64_t *iy, const float *vy,
                int nc, const int *cx, const int *cy, uint64_t max_products,
                oracle_result **out)
{
    int shx[64], iscx[64], ncx, nfx, shy[64], iscy[64], ncy, nfy;
    int st;
    *out = NULL;
    if ((st = oracle_layout(ox, dx, nc, cx, shx, iscx, NULL, &ncx, &nfx)))
        return st;
    if ((st = oracle_layout(oy, dy, nc, cy, shy, iscy, NULL, &ncy, &nfy)))
        return st;
    for (int i = 0; i < nc; ++i)
        if (oracle_mode_bits(dx[cx[i]]) != oracle_mode_bits(dy[cy[i]]))
            return OR_EINVAL;
    /* operand keys of up to 128 bits (ConvertTensor_extra); output keys of 64 */
    if (ncx + nfx > 128 || ncy + nfy > 128 || nfx + nfy > 64)
        return OR_EINVAL;

    oracle_result *r = (oracle_result *)calloc(1, sizeof(oracle_result));
    u128 *kx = (u128 *)malloc(16 * (nx ? nx : 1));
    u128 *ky = (u128 *)malloc(16 * (ny ? ny : 1));
    u128 *kt = (u128 *)malloc(16 * ((nx > ny ? nx : ny) ? (nx > ny ? nx : ny) : 1));
    float *sx = (float *)malloc(4 * (nx ? nx : 1));
    float *sy = (float *)malloc(4 * (ny ? ny : 1));
    float *st_ = (float *)malloc(4 * ((nx > ny ? nx : ny) ? (nx > ny ? nx : ny) : 1));
    uint64_t *operm = (uint64_t *)malloc(8 * ((nx > ny ? nx : ny) ? (nx > ny ? nx : ny) : 1));
    uint64_t *pos = (uint64_t *)malloc(8 * (nx ? nx : 1));
    uint64_t *cnt = (uint64_t *)malloc(8 * (nx ? nx : 1));
    uint64_t *pre = (uint64_t *)malloc(8 * (nx + 1));
    if (!r || !kx || !ky || !kt || !sx || !sy || !st_ || !operm || !pos || !cnt || !pre) {
        st = OR_ENOMEM;
        goto fail;
    }
    r->x_nfbits = nfx;
    r->y_nfbits = nfy;
    r->ncbits_x = ncx;
    r->ncbits_y = ncy;
    linearize128(ox, shx, iscx, ncx, nfx, 0, nx, ix, kx);
    linearize128(oy, shy, iscy, ncy, nfy, 1, ny, iy, ky);
    /* stable sort of each operand by its full key (sort.cuh:90-108) */
    if ((st = stable_sort_perm128(nx, kx, ncx + nfx, operm)))
        goto fail;
    for (uint64_t i = 0; i < nx; ++i) {
        kt[i] = kx[operm[i]];
        st_[i] = vx[operm[i]];
    }
    memcpy(kx, kt, 16 * nx);
    memcpy(sx, st_, 4 * nx);
    if ((st = stable_sort_perm128(ny, ky, ncy + nfy, operm)))
        goto fail;
    for (uint64_t i = 0; i < ny; ++i) {
        kt[i] = ky[operm[i]];
        st_[i] = vy[operm[i]];
    }
    memcpy(ky, kt, 16 * ny);
    memcpy(sy, st_, 4 * ny);
    /* index match on the whole contract key (indexMatch.cuh:20-44,67-118,120-229) */
    {
        const u128 cmask = ncx >= 128 ? ~(u128)0 : (((u128)1 << ncx) - 1);
        pre[0] = 0;
        for (uint64_t i = 0; i < nx; ++i) {
            const u128 c = kx[i] & cmask;
            uint64_t lo = 0, hi = ny;
            while (lo < hi) {
                const uint64_t mid = lo + (hi - lo) / 2;
                const u128 yc = nfy >= 128 ? 0 : (ky[mid] >> nfy);
                if (yc < c)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            uint64_t n = 0;
            while (lo + n < ny && (nfy >= 128 ? 0 : (ky[lo + n] >> nfy)) == c)
                ++n;
            pos[i] = n ? lo : 0;
            cnt[i] = n;
            pre[i + 1] = pre[i] + n;
        }
    }
    uint64_t ir = pre[nx];
    r->ir_nnz = ir;
    if (ir > max_products) {
        st = OR_ENOMEM;
        goto fail;
    }
    {
        uint64_t *pk = (uint64_t *)malloc(8 * (ir ? ir : 1));
        double *pv = (double *)malloc(8 * (ir ? ir : 1));
        uint64_t *perm = (uint64_t *)malloc(8 * (ir ? ir : 1));
        if (!pk || !pv || !perm) {
            free(pk);
            free(pv);
            free(perm);
            st = OR_ENOMEM;
            goto fail;
        }
        uint64_t fmask = nfy >= 64 ? ~0ull : ((1ull << nfy) - 1);
        uint64_t p = 0;
        for (uint64_t i = 0; i < nx; ++i) {
            uint64_t xf = (uint64_t)(kx[i] >> ncx);  /* nfx <= 64 bits */
            for (uint64_t j = 0; j < cnt[i]; ++j) {
                uint64_t yk = (uint64_t)ky[pos[i] + j];
                pk[p] = (nfy >= 64 ? 0 : (xf << nfy)) | (yk & fmask);
                pv[p] = (double)sx[i] * (double)sy[pos[i] + j];
                ++p;
            }
        }
        st = stable_sort_perm(ir, pk, nfx + nfy, perm);
        if (st) {
            free(pk);
            free(pv);
            free(perm);
            goto fail;
        }
        uint64_t nz = 0;
        for (uint64_t q = 0; q < ir; ++q)
            if (q == 0 || pk[perm[q]] != pk[perm[q - 1]])
                ++nz;
        r->nnz = nz;
        r->keys = (uint64_t *)malloc(8 * (nz ? nz : 1));
        r->vals = (double *)malloc(8 * (nz ? nz : 1));
        r->abs_sums = (double *)malloc(8 * (nz ? nz : 1));
        r->nprod = (uint64_t *)malloc(8 * (nz ? nz : 1));
        if (!r->keys || !r->vals || !r->abs_sums || !r->nprod) {
            free(pk);
            free(pv);
            free(perm);
            st = OR_ENOMEM;
            goto fail;
        }
        int64_t o = -1;
        for (uint64_t q = 0; q < ir; ++q) {
            uint64_t k = pk[perm[q]];
            double v = pv[perm[q]];
            if (q == 0 || k != pk[perm[q - 1]]) {
                ++o;
                r->keys[o] = k;
                r->vals[o] = 0.0;
                r->abs_sums[o] = 0.0;
                r->nprod[o] = 0;
            }
            r->vals[o] += v;
            r->abs_sums[o] += fabs(v);
            r->nprod[o] += 1;
        }
        free(pk);
        free(pv);
        free(perm);
    }
    free(kx);
    free(ky);
    free(kt);
    free(sx);
    free(sy);
    free(st_);
    free(operm);
    free(pos);
    free(cnt);
    free(pre);
    *out = r;
    return OR_OK;
fail:
    free(kx);
    free(ky);
    free(kt);
    free(sx);
    free(sy);
    free(st_);
    free(operm);
    free(pos);
    free(cnt);
    free(pre);
    oracle_free(r);
    return st;
}

/* ---------------------------------------------------------- .tns input */

/*
 * io_manager.tpp:75-259: order = (#tokens of the first line) - 1; every line
 * holding tokens is one nonzero; indices are 1-based and stored 0-based;
 * dims[m] = max index + 1; values are parsed as double and cast to float.
 * Returns nnz and order via the out parameters; idx (SoA) and vals are
 * malloc'd and owned by the caller (free with oracle_free_buf).
 */
int oracle_read_tns(const char *path, int *order_out, uint64_t *nnz_out,
                    uint64_t *dims_out /* [64] */, uint64_t **idx_out, float **val_out)
{
    FILE *f = fopen(path, "rb");
    if (!f)
        return OR_EIO;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    rewind(f);
    char *buf = (char *)malloc((size_t)sz + 1);
    if (!buf) {
        fclose(f);
        return OR_ENOMEM;
    }
    if (fread(buf, 1, (size_t)sz, f) != (size_t)sz) {
        fclose(f);
        free(buf);
        return OR_EIO;
    }
    fclose(f);
    buf[sz] = '\0';
    /* order from the first line */
    int ntok = 0;
    {
        char *p = buf;
        while (*p && *p != '\n') {
            while (*p == ' ' || *p == '\t' || *p == '\r')
                ++p;
            if (!*p || *p == '\n')
                break;
            ++ntok;
            while (*p && *p != ' ' && *p != '\t' && *p != '\n' && *p != '\r')
                ++p;
        }
    }
    int order = ntok - 1;
    if (order <= 0 || order > 64) {
        free(buf);
        return OR_EINVAL;
    }
    uint64_t lines = 0;
    for (long i = 0; i < sz; ++i)
        if (buf[i] == '\n')
            ++lines;
    if (sz > 0 && buf[sz - 1] != '\n')
        ++lines;
    uint64_t *idx = (uint64_t *)malloc(8 * (size_t)order * (lines ? lines : 1));
    float *val = (float *)malloc(4 * (lines ? lines : 1));
    if (!idx || !val) {
        free(buf);
        free(idx);
        free(val);
        return OR_ENOMEM;
    }
    uint64_t *tmp = (uint64_t *)malloc(8 * (size_t)order * (lines ? lines : 1));
    float *tv = (float *)malloc(4 * (lines ? lines : 1));
    for (int m = 0; m < order; ++m)
        dims_out[m] = 0;
    uint64_t n = 0;
    char *p = buf;
    while (*p) {
        char *line = p;
        char *e = strchr(p, '\n');
        if (e) {
            *e = '\0';
            p = e + 1;
        } else {
            p = line + strlen(line);
        }
        char *s = line;
        while (*s == ' ' || *s == '\t' || *s == '\r')
            ++s;
        if (!*s)
            continue;
        int m = 0;
        char *q = s;
        for (; m < order; ++m) {
            char *endp;
            unsigned long long v = strtoull(q, &endp, 10);
            if (endp == q || v == 0) {
                free(buf); free(idx); free(val); free(tmp); free(tv);
                return OR_EINVAL;
            }
            tmp[(size_t)m * lines + n] = (uint64_t)(v - 1);
            if (v > dims_out[m])
                dims_out[m] = v;
            q = endp;
        }
        char *endp;
        double d = strtod(q, &endp);
        if (endp == q) {
            free(buf); free(idx); free(val); free(tmp); free(tv);
            return OR_EINVAL;
        }
        tv[n] = (float)d;
        ++n;
    }
    for (int m = 0; m < order; ++m)
        memcpy(idx + (size_t)m * n, tmp + (size_t)m * lines, 8 * n);
    memcpy(val, tv, 4 * n);
    free(tmp);
    free(tv);
    free(buf);
    *order_out = order;
    *nnz_out = n;
    *idx_out = idx;
    *val_out = val;
    return OR_OK;
}

/*
 * io_manager.tpp:310-484 (_ReadQuantumData, read_txt_dims_parallel,
 * read_txt_data_parallel): <dir>/indices.txt holds one line per mode, each
 * with the 1-based index of every nonzero (parsed with strtod); order = number
 * of lines, nnz = tokens per line, dims[m] = largest index of mode m;
 * <dir>/values.txt holds nnz values.  Values are read as double and narrowed
 * to float (the reference scans "%le" into its float array, which this
 * restatement does not copy).  Lines without a token are skipped.
 */
static char *slurp_text(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f)
        return NULL;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    rewind(f);
    char *b = (char *)malloc((size_t)(sz > 0 ? sz : 0) + 1);
    if (!b) {
        fclose(f);
        return NULL;
    }
    size_t r = sz > 0 ? fread(b, 1, (size_t)sz, f) : 0;
    fclose(f);
    b[r] = '\0';
    return b;
}

int oracle_read_quantum(const char *dir, int *order_out, uint64_t *nnz_out,
                        uint64_t *dims_out /* [64] */, uint64_t **idx_out, float **val_out)
{
    char path[4096];
    snprintf(path, sizeof path, "%s/indices.txt", dir);
    char *ib = slurp_text(path);
    snprintf(path, sizeof path, "%s/values.txt", dir);
    char *vb = slurp_text(path);
    if (!ib || !vb) {
        free(ib);
        free(vb);
        return OR_EIO;
    }
    /* pass 1: order and nnz (tokens of each non-empty line) */
    int order = 0;
    uint64_t nnz = 0;
    int bad = 0;
    for (char *p = ib; *p;) {
        char *e = strchr(p, '\n');
        char *end = e ? e : p + strlen(p);
        uint64_t cnt = 0;
        char *q = p;
        while (q < end) {
            while (q < end && (*q == ' ' || *q == '\t' || *q == '\r'))
                ++q;
            if (q >= end)
                break;
            ++cnt;
            while (q < end && !(*q == ' ' || *q == '\t' || *q == '\r'))
                ++q;
        }
        if (cnt) {
            if (order == 0)
                nnz = cnt;
            else if (cnt != nnz)
                bad = 1;
            ++order;
        }
        p = e ? e + 1 : end;
    }
    if (bad || order == 0 || order > 64) {
        free(ib);
        free(vb);
        return OR_EIO;
    }
    uint64_t *idx = (uint64_t *)malloc(8 * (size_t)order * (nnz ? nnz : 1));
    float *val = (float *)malloc(4 * (nnz ? nnz : 1));
    if (!idx || !val) {
        free(ib);
        free(vb);
        free(idx);
        free(val);
        return OR_ENOMEM;
    }
    /* pass 2: indices, row by row */
    int m = 0;
    for (char *p = ib; *p && m < order;) {
        char *e = strchr(p, '\n');
        if (e)
            *e = '\0';
        uint64_t k = 0, mx = 0;
        char *q = p;
        for (;;) {
            char *end;
            double v = strtod(q, &end);
            if (end == q)
                break;
            if (!(v >= 1.0) || v != (double)(uint64_t)v)
                bad = 1;
            uint64_t i0 = (uint64_t)v - 1;
            if (k < nnz)
                idx[(uint64_t)m * nnz + k] = i0;
            if (i0 + 1 > mx)
                mx = i0 + 1;
            ++k;
            q = end;
        }
        if (k) {
            dims_out[m] = mx;
            ++m;
        }
        p = e ? e + 1 : p + strlen(p);
    }
    /* values */
    char *q = vb;
    for (uint64_t k = 0; k < nnz; ++k) {
        char *end;
        double v = strtod(q, &end);
        if (end == q) {
            bad = 1;
            break;
        }
        val[k] = (float)v;
        q = end;
    }
    free(ib);
    free(vb);
    if (bad) {
        free(idx);
        free(val);
        return OR_EIO;
    }
    *order_out = order;
    *nnz_out = nnz;
    *idx_out = idx;
    *val_out = val;
    return OR_OK;
}

void oracle_free_buf(void *p) { free(p); }
