/*
 * Link shim for building the reference's CPU SpTC baseline (baselines/Sparta)
 * without libnuma or a BLAS.  TEST/BASELINE INFRASTRUCTURE ONLY.
 *
 * The SpTC driver (benchmark/ttt.c -> src/sptensor/tmul.c) allocates through
 * libnuma's node-placement calls; on a plain host those reduce to calloc /
 * realloc and a no-op preference.  libnuma hands out fresh anonymous pages,
 * which are zero-filled, and Sparta relies on that (its NUMA vector
 * constructors skip the memset), so the shim zero-fills too.  The BLAS/LAPACK entry points are only
 * referenced by Sparta's CPD code, which the SpTC driver never calls, so they
 * abort if reached.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void *numa_alloc_onnode(size_t size, int node)
{
    (void)node;
    return calloc(1, size ? size : 1);
}

void *numa_realloc(void *old_addr, size_t old_size, size_t new_size)
{
    char *p = (char *)realloc(old_addr, new_size ? new_size : 1);
    if (p && new_size > old_size)
        memset(p + old_size, 0, new_size - old_size);
    return p;
}

void numa_set_preferred(int node) { (void)node; }

static void blas_unavailable(const char *name)
{
    fprintf(stderr, "sparta_shim: %s is not available in this build\n", name);
    abort();
}

void ssyrk_(void) { blas_unavailable("ssyrk_"); }
void spotrf_(void) { blas_unavailable("spotrf_"); }
void spotrs_(void) { blas_unavailable("spotrs_"); }
void sgesv_(void) { blas_unavailable("sgesv_"); }

