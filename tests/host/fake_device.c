/*
 * CPU stand-in for the device layer (the kdg_* functions of kd_internal.h),
 * linked with the real host library kd_api.c by the host tests.  It keeps
 * each catalog's points on the host and counts exhaustively, so the host
 * code's own logic (argument checks, radius sorting and de-duplication,
 * cumulative sums, the reference's counter layout, batch concatenation, the
 * handle registry, error reporting) runs end to end without a GPU, under
 * ThreadSanitizer or AddressSanitizer.  Failures are injected on request.
 *
 * Differences from the device layer that the tests avoid: no deduplication
 * (a tree point's field is its own, so duplicates with mixed fields are not
 * modelled) and a dummy node array.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "kd_internal.h"

/* ---- failure injection (set by the test driver) */
int fake_fail_build = 0;  /* error code kdg_build returns, 0 = none */
int fake_fail_count = 0;  /* error code kdg_count_batch / kdg_count_static return */
int fake_fail_copy = 0;   /* error code of the node array copy (kdg_build_tree, or
                           * kdg_wait_nodes for a deferred build) */

typedef struct {
    double *xyz; /* n x 3 */
    int *f;      /* own field of every point */
} fake_pts;

int kdg_build(const double *h_xyz, const int *h_fields, int n, int num_fields, int query_only,
              kd_catalog *cat)
{
    int i, memsize = 2;
    fake_pts *fp;
    (void)query_only;
    if (fake_fail_build) {
        kd_set_error(fake_fail_build, "injected build failure");
        return fake_fail_build;
    }
    for (i = 0; i < n; i++)
        if (isnan(h_xyz[3 * i]) || isnan(h_xyz[3 * i + 1]) || isnan(h_xyz[3 * i + 2])) {
            kd_set_error(KD_ENAN, "NaN coordinate in tree points");
            return KD_ENAN;
        }
    while (memsize <= n) memsize *= 2;
    memset(cat, 0, sizeof *cat);
    fp = (fake_pts *)calloc(1, sizeof *fp);
    if (!fp) goto oom;
    fp->xyz = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    fp->f = (int *)malloc(sizeof(int) * (size_t)n);
    cat->d_nodes = calloc((size_t)memsize, sizeof(node_t));
    if (!fp->xyz || !fp->f || !cat->d_nodes) goto oom;
    memcpy(fp->xyz, h_xyz, sizeof(double) * 3 * (size_t)n);
    cat->n_raw = n;
    cat->n_u = n;
    cat->memsize = memsize;
    cat->num_fields = num_fields;
    cat->min_qf = 0;
    for (i = 0; i < n; i++) {
        fp->f[i] = h_fields ? h_fields[i] : 0;
        if (fp->f[i] > cat->max_qf) cat->max_qf = fp->f[i];
        if (i == 0 || fp->f[i] < cat->min_qf) cat->min_qf = fp->f[i];
        if ((fp->f[i] & 0xFF) > cat->max_tf) cat->max_tf = fp->f[i] & 0xFF;
    }
    cat->fields_split = cat->max_qf > 255;
    cat->d_x = (double *)fp; /* the fake keeps its points behind d_x */
    cat->nblocks = (n + KD_BLOCK_MAX - 1) / KD_BLOCK_MAX;
    return KD_OK;
oom:
    if (fp) {
        free(fp->xyz);
        free(fp->f);
    }
    free(fp);
    free(cat->d_nodes);
    cat->d_nodes = NULL;
    kd_set_error(KD_ENOMEM, "out of host memory");
    return KD_ENOMEM;
}

int kdg_build_tree(const double *h_xyz, const int *h_fields, int n, int num_fields,
                   kd_node_sink *sink, int deferred, kd_catalog *cat)
{
    int rc;
    void *host;
    sink->nodes = NULL;
    rc = kdg_build(h_xyz, h_fields, n, num_fields, 0, cat);
    if (rc != KD_OK) return rc;
    host = sink->alloc(sizeof(node_t) * (size_t)cat->memsize);
    if (!host || (fake_fail_copy && !deferred)) {
        if (host) sink->release(host);
        kdg_free(cat);
        rc = host ? fake_fail_copy : KD_ENOMEM;
        kd_set_error(rc, host ? "injected node copy failure" : "out of host memory");
        return rc;
    }
    memcpy(host, cat->d_nodes, sizeof(node_t) * (size_t)cat->memsize);
    free(cat->d_nodes);
    cat->d_nodes = NULL;
    sink->nodes = host;
    if (deferred) {
        /* the copy "still running": its outcome is reported by the wait */
        int *code = (int *)malloc(sizeof(int));
        if (!code) {
            sink->nodes = NULL;
            sink->release(host);
            kdg_free(cat);
            kd_set_error(KD_ENOMEM, "out of host memory");
            return KD_ENOMEM;
        }
        *code = fake_fail_copy;
        cat->pending = code;
    }
    return KD_OK;
}

int kdg_wait_nodes(kd_catalog *cat)
{
    int code = cat->pending ? *(int *)cat->pending : 0;
    if (code) kd_set_error(code, "injected node copy failure");
    return code;
}

int kdg_copy_inorder(const kd_catalog *cat, int *h_perm)
{
    int i;
    for (i = 0; i < cat->n_u; i++) h_perm[i] = i;
    return KD_OK;
}

void kdg_free(kd_catalog *cat)
{
    fake_pts *fp = (fake_pts *)cat->d_x;
    free(cat->pending);
    if (fp) {
        free(fp->xyz);
        free(fp->f);
        free(fp);
    }
    free(cat->d_nodes);
    memset(cat, 0, sizeof *cat);
}

/* d2 in the reference's order (kdquery.c:39-47 as compiled: dx*dx, then
 * fma(dy,dy,.), fma(dz,dz,.)) */
static double d2_ref(const double *t, const double *q)
{
    const double dx = t[0] - q[0], dy = t[1] - q[1], dz = t[2] - q[2];
    return fma(dz, dz, fma(dy, dy, dx * dx));
}

/* hist[e][qf][tf]: pairs with rsq[e-1] <= d2 < rsq[e] */
static void brute_hist(const kd_catalog *tc, const kd_catalog *qc, const double *rsq, int ne,
                       long long *hist)
{
    const fake_pts *tp = (const fake_pts *)tc->d_x, *qp = (const fake_pts *)qc->d_x;
    const size_t Fqe = (size_t)qc->max_qf + 1, Fte = (size_t)tc->max_tf + 1;
    int i, j;
    memset(hist, 0, sizeof(long long) * (size_t)(ne + 1) * Fqe * Fte);
    for (i = 0; i < qc->n_raw; i++)
        for (j = 0; j < tc->n_raw; j++) {
            const double d2 = d2_ref(tp->xyz + 3 * (size_t)j, qp->xyz + 3 * (size_t)i);
            int e = 0, hi = ne; /* first e with d2 < rsq[e] (NaN: none) */
            if (d2 != d2) e = ne;
            while (e < hi) {
                const int m = (e + hi) / 2;
                if (d2 < rsq[m]) hi = m;
                else e = m + 1;
            }
            if (e < ne) hist[((size_t)e * Fqe + (size_t)qp->f[i]) * Fte + (size_t)(tp->f[j] & 0xFF)]++;
        }
}

int kdg_count_batch(const kd_catalog *const *trees, const kd_catalog *const *queries, int njobs,
                    const double *rsq, int ne, int mode, int shard, int nshards,
                    long long *const *hists, kd_count_stats *stats)
{
    int j;
    (void)mode;
    if (fake_fail_count) {
        kd_set_error(fake_fail_count, "injected count failure");
        return fake_fail_count;
    }
    if (nshards < 1 || shard < 0 || shard >= nshards) {
        kd_set_error(KD_EINVAL, "shard %d of %d", shard, nshards);
        return KD_EINVAL;
    }
    /* the device counter's limit: the host library splits more radii into passes */
    if (ne < 1 || ne > KD_MAX_EDGES) {
        kd_set_error(KD_EINVAL, "fake device: %d distinct radii in one pass", ne);
        return KD_EINVAL;
    }
    for (j = 0; j < njobs; j++) {
        if (shard == 0) brute_hist(trees[j], queries[j], rsq, ne, hists[j]);
        else  /* every count on shard 0 in the fake */
            memset(hists[j], 0, sizeof(long long) * (size_t)(ne + 1) *
                                    ((size_t)queries[j]->max_qf + 1) * ((size_t)trees[j]->max_tf + 1));
    }
    if (stats) memset(stats, 0, sizeof *stats);
    return KD_OK;
}

int kdg_count(const kd_catalog *tree, const kd_catalog *query, const double *rsq, int ne,
              int mode, int shard, int nshards, long long *hist, kd_count_stats *stats)
{
    return kdg_count_batch(&tree, &query, 1, rsq, ne, mode, shard, nshards, &hist, stats);
}

int kdg_count_static(const kd_catalog *tree, int Ft, const kd_catalog *query, int Fq,
                     const double *rsq_sorted, int ne, const int *edge_of, int nradii, int mode,
                     long long *out)
{
    long long hist[(KD_MAX_EDGES + 1) * 16 * 16];
    const size_t Fqe = (size_t)query->max_qf + 1, Fte = (size_t)tree->max_tf + 1;
    int k, e;
    size_t a, b;
    (void)mode;
    if (fake_fail_count) {
        kd_set_error(fake_fail_count, "injected count failure");
        return fake_fail_count;
    }
    if (Fqe * Fte > 256) {
        kd_set_error(KD_EINVAL, "fake static count: at most 16 x 16 fields");
        return KD_EINVAL;
    }
    brute_hist(tree, query, rsq_sorted, ne, hist);
    memset(out, 0, sizeof(long long) * (size_t)nradii * (size_t)Fq * (size_t)Ft);
    for (k = 0; k < nradii; k++) {
        if (edge_of[k] < 0) continue;
        for (e = 0; e <= edge_of[k]; e++)
            for (a = 0; a < Fqe; a++)
                for (b = 0; b < Fte; b++)
                    out[(size_t)k * Fq * Ft + a * (size_t)Fq + b] += hist[((size_t)e * Fqe + a) * Fte + b];
    }
    return KD_OK;
}

int kdg_set_device(int device)
{
    if (device != 0) {
        kd_set_error(KD_ENODEV, "no CUDA device %d (fake: only 0)", device);
        return KD_ENODEV;
    }
    return KD_OK;
}
