/*
 * C host side of libkdtree.so: the reference ABI (tree_construct, pair_count,
 * destroy) and the additive kd_* entry points, on top of the GPU catalog
 * (kd_build.cu) and counter (kd_count.cu).
 *
 * Handles: tree_construct returns the reference's 64-byte kdtree_t by value
 * (kdbuild.c:513-536).  Its node_data is a host array of node_t, as the
 * reference returns; the device-side catalog behind it is found again from
 * that pointer through a registry, so a kdtree_t copied by value (ctypes,
 * C structs) keeps working.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <time.h>

#include "kd_internal.h"

/* ------------------------------------------------------------------ errors */

static __thread int g_code;
static __thread char g_msg[256];

void kd_set_error(int code, const char *fmt, ...)
{
    va_list ap;
    g_code = code;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
}

int kd_last_error(char *buf, int len)
{
    if (buf && len > 0) {
        strncpy(buf, g_code ? g_msg : "", (size_t)len - 1);
        buf[len - 1] = 0;
    }
    return g_code;
}

static void clear_error(void)
{
    g_code = 0;
    g_msg[0] = 0;
}

/* ---------------------------------------------------------------- registry */

typedef struct kd_handle {
    kd_catalog cat;
    node_t *nodes;
    struct kd_handle *next;
} kd_handle;

static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static kd_handle *g_handles;

static kd_handle *lookup(const kdtree_t *t)
{
    kd_handle *h;
    if (!t->node_data) return NULL;
    pthread_mutex_lock(&g_lock);
    for (h = g_handles; h; h = h->next)
        if (h->nodes == t->node_data) break;
    pthread_mutex_unlock(&g_lock);
    return h;
}

static kd_handle *lookup_or_fail(const kdtree_t *t, const char *what)
{
    kd_handle *h = lookup(t);
    if (!h) kd_set_error(KD_EINVAL, "%s: not a live tree from tree_construct", what);
    return h;
}

/* ---------------------------------------------------------------- ABI */

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

/* host memory for a node array: large ones (1.3 GB at 20M points) in 2 MB
 * pages where the kernel offers them, so that filling it takes a few hundred
 * page faults instead of hundreds of thousands */
static void *alloc_nodes(size_t nb)
{
    void *mem = NULL;
    if (nb >= ((size_t)64 << 20)) {
        if (posix_memalign(&mem, (size_t)2 << 20, nb) != 0) mem = NULL;
        if (mem) madvise(mem, nb, MADV_HUGEPAGE);
    } else {
        mem = malloc(nb);
    }
    return mem;
}

static void release_nodes(void *p) { free(p); }

static kdtree_t construct(double *xyz, int *fields, int length, int num_fields, int deferred,
                          const char *who)
{
    kdtree_t t;
    kd_handle *h;
    kd_node_sink sink;
    double t0 = now_ms();
    memset(&t, 0, sizeof t);
    clear_error();
    if (!xyz || length < 1) {
        kd_set_error(KD_EINVAL, "%s: need at least one point", who);
        return t;
    }
    if (length > KD_MAX_POINTS) {
        kd_set_error(KD_EINVAL, "%s: %d points, at most %d", who, length, KD_MAX_POINTS);
        return t;
    }
    h = (kd_handle *)calloc(1, sizeof *h);
    if (!h) {
        kd_set_error(KD_ENOMEM, "%s: out of host memory", who);
        return t;
    }
    /* every byte of the node array is written by the build's copy: empty
     * heap slots come zeroed from the device (as calloc leaves them in
     * kdbuild.c:516) */
    sink.alloc = alloc_nodes;
    sink.release = release_nodes;
    sink.nodes = NULL;
    if (kdg_build_tree(xyz, fields, length, num_fields, &sink, deferred, &h->cat) != KD_OK) {
        free(h);
        return t;
    }
    h->nodes = (node_t *)sink.nodes;
    h->cat.bstats.ms_total_host = now_ms() - t0;
    pthread_mutex_lock(&g_lock);
    h->next = g_handles;
    g_handles = h;
    pthread_mutex_unlock(&g_lock);
    t.node_data = h->nodes;
    t.size = h->cat.n_u;
    t.memsize = h->cat.memsize;
    t.num_fields = num_fields;
    return t;
}

kdtree_t tree_construct(double *xyz, int *fields, int length, int num_fields)
{
    return construct(xyz, fields, length, num_fields, 0, "tree_construct");
}

kdtree_t kd_tree_construct_deferred(double *xyz, int *fields, int length, int num_fields)
{
    return construct(xyz, fields, length, num_fields, 1, "kd_tree_construct_deferred");
}

int kd_tree_wait_nodes(kdtree_t t)
{
    kd_handle *h;
    clear_error();
    h = lookup_or_fail(&t, "kd_tree_wait_nodes");
    if (!h) return KD_EINVAL;
    return kdg_wait_nodes(&h->cat);
}

void destroy(kdtree_t t)
{
    kd_handle **pp, *h = NULL;
    if (!t.node_data) return;
    pthread_mutex_lock(&g_lock);
    for (pp = &g_handles; *pp; pp = &(*pp)->next)
        if ((*pp)->nodes == t.node_data) {
            h = *pp;
            *pp = h->next;
            break;
        }
    pthread_mutex_unlock(&g_lock);
    if (!h) return;
    kdg_free(&h->cat);
    free(h->nodes);
    free(h);
}

void kd_free_counts(long long *counts) { free(counts); }

int kd_tree_permutation(kdtree_t t, int *perm)
{
    kd_handle *h;
    clear_error();
    h = lookup_or_fail(&t, "kd_tree_permutation");
    if (!h) return KD_EINVAL;
    return kdg_copy_inorder(&h->cat, perm);
}

int kd_tree_build_stats(kdtree_t t, kd_build_stats *stats)
{
    kd_handle *h;
    clear_error();
    h = lookup_or_fail(&t, "kd_tree_build_stats");
    if (!h) return KD_EINVAL;
    if (!stats) {
        kd_set_error(KD_EINVAL, "kd_tree_build_stats: NULL output");
        return KD_EINVAL;
    }
    *stats = h->cat.bstats;
    return KD_OK;
}

int kd_set_device(int device)
{
    clear_error();
    return kdg_set_device(device);
}

int kd_tree_input_size(kdtree_t t)
{
    kd_handle *h = lookup(&t);
    return h ? h->cat.n_raw : -1;
}

/* ---------------------------------------------------------------- counting */

static int cmp_double(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* add a pass's statistics to the call's totals */
static void add_stats(kd_count_stats *to, const kd_count_stats *s)
{
    to->pairs_tested += s->pairs_tested;
    to->pairs_rechecked += s->pairs_rechecked;
    to->pairs_accepted += s->pairs_accepted;
    to->pairs_wide += s->pairs_wide;
    to->edge_pairs += s->edge_pairs;
    to->warp_tiles += s->warp_tiles;
    to->entries += s->entries;
    to->ms_traverse += s->ms_traverse;
    to->ms_tiles += s->ms_tiles;
    to->ms_total += s->ms_total;
    to->tile_launches += s->tile_launches;
    to->launches += s->launches;
    to->pairs_one_bin_multifield += s->pairs_one_bin_multifield;
}

/*
 * Count njobs (tree catalog, query catalog) pairs for all radii and write,
 * job after job, the reference's cumulative per-radius matrices
 * out[k][qf*Fq + tf] (kdquery.c:34: rows strided by the QUERY field count
 * Fq), nradii * Fq[j] * Ft[j] values per job.
 *
 * The distinct squared radii are counted in passes of at most KD_MAX_EDGES
 * (ascending), each one device batch over all jobs.  A pair's count at a
 * radius depends on that radius alone, so the passes are independent and any
 * number of radii gives the reference's counts (its drivers call pair_count
 * once per radius, clustering.py:218-230, whatever their number).
 */
static int count_jobs(const kd_catalog *const *tcs, const int *Fts, const kd_catalog *const *qcs,
                      const int *Fqs, int njobs, const double *radii, int nradii, int mode,
                      int shard, int nshards, long long *out, kd_count_stats *stats)
{
    double *rsq = NULL, *uniq = NULL;
    long long **hists = NULL, **cums = NULL;
    int j, k, ne = 0, rc = KD_OK;
    size_t total = 0;

    if (mode != KD_MODE_MIXED && mode != KD_MODE_FP64) {
        kd_set_error(KD_EINVAL, "unknown count mode %d", mode);
        return KD_EINVAL;
    }
    for (j = 0; j < njobs; j++) {
        const int Fq = Fqs[j], Ft = Fts[j];
        if (Fq < 1 || Ft < 1) {
            kd_set_error(KD_EFIELD, "field counts must be positive");
            return KD_EFIELD;
        }
        if (qcs[j]->min_qf < 0) {
            kd_set_error(KD_EFIELD, "negative query field id");
            return KD_EFIELD;
        }
        /* the reference would write outside its Fq*Ft counter (kdquery.c:34) */
        if ((long long)qcs[j]->max_qf * Fq + tcs[j]->max_tf >= (long long)Fq * Ft) {
            kd_set_error(KD_EFIELD, "field ids overflow the %d x %d counter (qfield*%d + tfield)",
                         Fq, Ft, Fq);
            return KD_EFIELD;
        }
        total += (size_t)Fq * (size_t)Ft * (size_t)nradii;
    }
    for (k = 0; k < nradii; k++)
        if (radii[k] < 0) {
            kd_set_error(KD_ERADIUS, "negative radius %g", radii[k]);
            return KD_ERADIUS;
        }
    if (total) memset(out, 0, sizeof(long long) * total);
    if (stats) memset(stats, 0, sizeof *stats);
    rsq = (double *)malloc(sizeof(double) * (size_t)(nradii + 1));
    uniq = (double *)malloc(sizeof(double) * (size_t)(nradii + 1));
    hists = (long long **)calloc((size_t)njobs, sizeof(long long *));
    cums = (long long **)calloc((size_t)njobs, sizeof(long long *));
    if (!rsq || !uniq || !hists || !cums) {
        kd_set_error(KD_ENOMEM, "out of host memory");
        rc = KD_ENOMEM;
        goto done;
    }
    /* squared radii exactly as kdquery.c:77 forms them; NaN counts nothing */
    for (k = 0; k < nradii; k++) rsq[k] = radii[k] * radii[k];
    for (k = 0; k < nradii; k++)
        if (rsq[k] == rsq[k]) uniq[ne++] = rsq[k];
    qsort(uniq, (size_t)ne, sizeof(double), cmp_double);
    {
        int w = 0;
        for (k = 0; k < ne; k++)
            if (w == 0 || uniq[k] != uniq[w - 1]) uniq[w++] = uniq[k];
        ne = w;
    }
    if (ne == 0) goto done;
    for (j = 0; j < njobs; j++) {
        const size_t hrow = ((size_t)qcs[j]->max_qf + 1) * ((size_t)tcs[j]->max_tf + 1);
        const int npass = ne < KD_MAX_EDGES ? ne : KD_MAX_EDGES;
        hists[j] = (long long *)calloc((size_t)(npass + 1) * hrow, sizeof(long long));
        cums[j] = (long long *)calloc((size_t)ne * hrow, sizeof(long long));
        if (!hists[j] || !cums[j]) {
            kd_set_error(KD_ENOMEM, "out of host memory");
            rc = KD_ENOMEM;
            goto done;
        }
    }
    {
        int e0;
        for (e0 = 0; e0 < ne; e0 += KD_MAX_EDGES) {
            const int n = ne - e0 < KD_MAX_EDGES ? ne - e0 : KD_MAX_EDGES;
            kd_count_stats ps;
            memset(&ps, 0, sizeof ps);
            if (e0 > 0)
                for (j = 0; j < njobs; j++)
                    memset(hists[j], 0, sizeof(long long) * (size_t)(n + 1) *
                                            ((size_t)qcs[j]->max_qf + 1) *
                                            ((size_t)tcs[j]->max_tf + 1));
            rc = kdg_count_batch(tcs, qcs, njobs, uniq + e0, n, mode, shard, nshards, hists,
                                 stats ? &ps : NULL);
            if (rc != KD_OK) goto done;
            if (stats) add_stats(stats, &ps);
            /* hist[e] holds the pairs with uniq[e0+e-1] <= d2 < uniq[e0+e]
             * (e = 0: every pair below uniq[e0]); cumulative sums give the
             * pairs with d2 < uniq[e0+e] */
            for (j = 0; j < njobs; j++) {
                const size_t hrow = ((size_t)qcs[j]->max_qf + 1) * ((size_t)tcs[j]->max_tf + 1);
                const long long *h = hists[j];
                long long *c = cums[j] + (size_t)e0 * hrow;
                size_t i;
                int e;
                for (i = 0; i < hrow; i++) c[i] = h[i];
                for (e = 1; e < n; e++)
                    for (i = 0; i < hrow; i++)
                        c[(size_t)e * hrow + i] = c[(size_t)(e - 1) * hrow + i] + h[(size_t)e * hrow + i];
            }
        }
    }
    for (j = 0; j < njobs; j++) {
        const size_t Fqe = (size_t)qcs[j]->max_qf + 1, Fte = (size_t)tcs[j]->max_tf + 1;
        const size_t hrow = Fqe * Fte, nrow = (size_t)Fqs[j] * (size_t)Fts[j];
        const long long *cum = cums[j];
        for (k = 0; k < nradii; k++) {
            int lo = 0, hi = ne;
            size_t qf, tf;
            long long *o = out + (size_t)k * nrow;
            if (rsq[k] != rsq[k]) continue;
            while (lo < hi) {
                int m = (lo + hi) / 2;
                if (uniq[m] < rsq[k]) lo = m + 1;
                else hi = m;
            }
            for (qf = 0; qf < Fqe; qf++)
                for (tf = 0; tf < Fte; tf++)
                    o[qf * (size_t)Fqs[j] + tf] += cum[(size_t)lo * hrow + qf * Fte + tf];
        }
        out += nrow * (size_t)nradii;
    }
done:
    if (hists)
        for (j = 0; j < njobs; j++) free(hists[j]);
    if (cums)
        for (j = 0; j < njobs; j++) free(cums[j]);
    free(hists);
    free(cums);
    free(rsq);
    free(uniq);
    return rc;
}

static int count_catalogs(const kd_catalog *tc, int Ft, const kd_catalog *qc, int Fq,
                          const double *radii, int nradii, int mode, int shard, int nshards,
                          long long *out, kd_count_stats *stats)
{
    return count_jobs(&tc, &Ft, &qc, &Fq, 1, radii, nradii, mode, shard, nshards, out, stats);
}

/* count_jobs' checks of the mode and the radii, for the calls that return
 * before counting (no query points) */
static int check_radii_mode(const double *radii, int nradii, int mode)
{
    int k;
    if (mode != KD_MODE_MIXED && mode != KD_MODE_FP64) {
        kd_set_error(KD_EINVAL, "unknown count mode %d", mode);
        return KD_EINVAL;
    }
    for (k = 0; k < nradii; k++)
        if (radii[k] < 0) {
            kd_set_error(KD_ERADIUS, "negative radius %g", radii[k]);
            return KD_ERADIUS;
        }
    return KD_OK;
}

/* query catalog from raw points; NaN rows are dropped (they count nothing in
 * the reference: every comparison with NaN is false, kdquery.c:33, :101-109) */
static int query_catalog(const double *xyz, const int *fields, int n, int Fq, kd_catalog *qc,
                         int *empty)
{
    int i, m = 0, rc;
    double *px = NULL;
    int *pf = NULL;
    const double *use_x = xyz;
    const int *use_f = fields;
    *empty = 0;
    for (i = 0; i < n; i++)
        if (isnan(xyz[3 * (size_t)i]) || isnan(xyz[3 * (size_t)i + 1]) || isnan(xyz[3 * (size_t)i + 2]))
            break;
    if (i < n) {
        px = (double *)malloc(sizeof(double) * 3 * (size_t)n);
        pf = fields ? (int *)malloc(sizeof(int) * (size_t)n) : NULL;
        if (!px || (fields && !pf)) {
            free(px);
            free(pf);
            kd_set_error(KD_ENOMEM, "out of host memory");
            return KD_ENOMEM;
        }
        for (i = 0; i < n; i++) {
            const double *p = xyz + 3 * (size_t)i;
            if (isnan(p[0]) || isnan(p[1]) || isnan(p[2])) continue;
            memcpy(px + 3 * (size_t)m, p, 3 * sizeof(double));
            if (pf) pf[m] = fields[i];
            m++;
        }
        use_x = px;
        use_f = pf;
        n = m;
    }
    if (n == 0) {
        *empty = 1;
        free(px);
        free(pf);
        return KD_OK;
    }
    rc = kdg_build(use_x, use_f, n, Fq, 1, qc);
    free(px);
    free(pf);
    return rc;
}

int kd_count_points(kdtree_t tree, const double *xyz, const int *fields, int length,
                    int num_fields, const double *radii, int nradii, int mode, long long *out,
                    kd_count_stats *stats)
{
    kd_handle *h;
    kd_catalog qc;
    int empty = 0, rc;
    clear_error();
    h = lookup_or_fail(&tree, "kd_count_points");
    if (!h) return KD_EINVAL;
    if (length < 0 || length > KD_MAX_POINTS || nradii < 0 || (length > 0 && !xyz) ||
        (nradii > 0 && (!radii || !out))) {
        kd_set_error(KD_EINVAL, "kd_count_points: bad arguments");
        return KD_EINVAL;
    }
    if (num_fields < 1 || tree.num_fields < 1) {
        kd_set_error(KD_EFIELD, "field counts must be positive");
        return KD_EFIELD;
    }
    if (length == 0) {
        if ((rc = check_radii_mode(radii, nradii, mode)) != KD_OK) return rc;
        if (nradii > 0)
            memset(out, 0, sizeof(long long) * (size_t)num_fields * (size_t)tree.num_fields *
                               (size_t)nradii);
        if (stats) memset(stats, 0, sizeof *stats);
        return KD_OK;
    }
    memset(&qc, 0, sizeof qc);
    rc = query_catalog(xyz, fields, length, num_fields, &qc, &empty);
    if (rc != KD_OK) return rc;
    if (empty) {
        if ((rc = check_radii_mode(radii, nradii, mode)) != KD_OK) return rc;
        if (nradii > 0)
            memset(out, 0, sizeof(long long) * (size_t)num_fields * (size_t)tree.num_fields *
                               (size_t)nradii);
        if (stats) memset(stats, 0, sizeof *stats);
        return KD_OK;
    }
    rc = count_catalogs(&h->cat, tree.num_fields, &qc, num_fields, radii, nradii, mode, 0, 1, out,
                        stats);
    kdg_free(&qc);
    return rc;
}

int kd_count_radii_shard(kdtree_t tree, kdtree_t query, const double *radii, int nradii,
                         int mode, int shard, int nshards, long long *out, kd_count_stats *stats)
{
    kd_handle *ht, *hq;
    clear_error();
    ht = lookup_or_fail(&tree, "kd_count_radii (tree)");
    if (!ht) return KD_EINVAL;
    hq = lookup_or_fail(&query, "kd_count_radii (query)");
    if (!hq) return KD_EINVAL;
    if (nshards < 1 || shard < 0 || shard >= nshards) {
        kd_set_error(KD_EINVAL, "kd_count_radii_shard: shard %d of %d", shard, nshards);
        return KD_EINVAL;
    }
    if (nradii < 0 || (nradii > 0 && (!radii || !out))) {
        kd_set_error(KD_EINVAL, "kd_count_radii: bad radius count or NULL array");
        return KD_EINVAL;
    }
    return count_catalogs(&ht->cat, tree.num_fields, &hq->cat, query.num_fields, radii, nradii,
                          mode, shard, nshards, out, stats);
}

int kd_count_radii(kdtree_t tree, kdtree_t query, const double *radii, int nradii, int mode,
                   long long *out, kd_count_stats *stats)
{
    return kd_count_radii_shard(tree, query, radii, nradii, mode, 0, 1, out, stats);
}

int kd_count_bins(kdtree_t tree, kdtree_t query, const double *edges, int nedges, int mode,
                  long long *out, kd_count_stats *stats)
{
    long long *cum;
    size_t nrow, k, j;
    int rc;
    clear_error();
    if (nedges < 1 || !edges || !out) {
        kd_set_error(KD_EINVAL, "kd_count_bins: need at least one edge");
        return KD_EINVAL;
    }
    nrow = (size_t)(query.num_fields > 0 ? query.num_fields : 0) *
           (size_t)(tree.num_fields > 0 ? tree.num_fields : 0);
    cum = (long long *)malloc(sizeof(long long) * (nrow ? nrow : 1) * (size_t)nedges);
    if (!cum) {
        kd_set_error(KD_ENOMEM, "out of host memory");
        return KD_ENOMEM;
    }
    rc = kd_count_radii(tree, query, edges, nedges, mode, cum, stats);
    if (rc == KD_OK)
        for (k = 0; k + 1 < (size_t)nedges; k++)
            for (j = 0; j < nrow; j++) out[k * nrow + j] = cum[(k + 1) * nrow + j] - cum[k * nrow + j];
    free(cum);
    return rc;
}

int kd_count_batch_shard(const kdtree_t *trees, const kdtree_t *queries, int njobs,
                         const double *radii, int nradii, int mode, int shard, int nshards,
                         long long *out, kd_count_stats *stats)
{
    const kd_catalog **tcs = NULL, **qcs = NULL;
    int *Fts = NULL, *Fqs = NULL;
    int j, rc = KD_OK;
    clear_error();
    if (njobs < 1 || !trees || !queries || nradii < 0 || (nradii > 0 && !radii) || !out) {
        kd_set_error(KD_EINVAL, "kd_count_batch: bad arguments");
        return KD_EINVAL;
    }
    if (nshards < 1 || shard < 0 || shard >= nshards) {
        kd_set_error(KD_EINVAL, "kd_count_batch: shard %d of %d", shard, nshards);
        return KD_EINVAL;
    }
    tcs = (const kd_catalog **)malloc(sizeof(*tcs) * (size_t)njobs);
    qcs = (const kd_catalog **)malloc(sizeof(*qcs) * (size_t)njobs);
    Fts = (int *)malloc(sizeof(int) * (size_t)njobs);
    Fqs = (int *)malloc(sizeof(int) * (size_t)njobs);
    if (!tcs || !qcs || !Fts || !Fqs) {
        kd_set_error(KD_ENOMEM, "out of host memory");
        rc = KD_ENOMEM;
        goto done;
    }
    for (j = 0; j < njobs; j++) {
        kd_handle *ht = lookup_or_fail(&trees[j], "kd_count_batch (tree)");
        kd_handle *hq = ht ? lookup_or_fail(&queries[j], "kd_count_batch (query)") : NULL;
        if (!ht || !hq) {
            rc = KD_EINVAL;
            goto done;
        }
        tcs[j] = &ht->cat;
        qcs[j] = &hq->cat;
        Fts[j] = trees[j].num_fields;
        Fqs[j] = queries[j].num_fields;
    }
    rc = count_jobs(tcs, Fts, qcs, Fqs, njobs, radii, nradii, mode, shard, nshards, out, stats);
done:
    free(tcs);
    free(qcs);
    free(Fts);
    free(Fqs);
    return rc;
}

int kd_count_batch(const kdtree_t *trees, const kdtree_t *queries, int njobs, const double *radii,
                   int nradii, int mode, long long *out, kd_count_stats *stats)
{
    return kd_count_batch_shard(trees, queries, njobs, radii, nradii, mode, 0, 1, out, stats);
}

int kd_count_radii_static(kdtree_t tree, kdtree_t query, const double *radii, int nradii,
                          int mode, long long *out)
{
    /* no heap: the radii are sorted in fixed arrays (insertion sort) */
    double uniq[KD_MAX_EDGES];
    int edge_of[KD_MAX_EDGES];
    int k, j, ne = 0;
    kd_handle *ht, *hq;
    clear_error();
    ht = lookup_or_fail(&tree, "kd_count_radii_static (tree)");
    if (!ht) return KD_EINVAL;
    hq = lookup_or_fail(&query, "kd_count_radii_static (query)");
    if (!hq) return KD_EINVAL;
    if (nradii < 0 || nradii > KD_MAX_EDGES || (nradii > 0 && (!radii || !out))) {
        kd_set_error(KD_EINVAL, "kd_count_radii_static: 0 to %d radii and an output array",
                     KD_MAX_EDGES);
        return KD_EINVAL;
    }
    if (mode != KD_MODE_MIXED && mode != KD_MODE_FP64) {
        kd_set_error(KD_EINVAL, "unknown count mode %d", mode);
        return KD_EINVAL;
    }
    if (query.num_fields < 1 || tree.num_fields < 1 || hq->cat.min_qf < 0 ||
        (long long)hq->cat.max_qf * query.num_fields + ht->cat.max_tf >=
            (long long)query.num_fields * tree.num_fields) {
        kd_set_error(KD_EFIELD, "field ids overflow the %d x %d counter (qfield*%d + tfield)",
                     query.num_fields, tree.num_fields, query.num_fields);
        return KD_EFIELD;
    }
    for (k = 0; k < nradii; k++) {
        double v = radii[k] * radii[k]; /* kdquery.c:77 */
        if (radii[k] < 0) {
            kd_set_error(KD_ERADIUS, "negative radius %g", radii[k]);
            return KD_ERADIUS;
        }
        if (v != v) continue;
        for (j = 0; j < ne && uniq[j] != v; j++)
            ;
        if (j < ne) continue;
        for (j = ne++; j > 0 && uniq[j - 1] > v; j--) uniq[j] = uniq[j - 1];
        uniq[j] = v;
    }
    for (k = 0; k < nradii; k++) {
        double v = radii[k] * radii[k];
        edge_of[k] = -1;
        for (j = 0; j < ne; j++)
            if (uniq[j] == v) edge_of[k] = j;
    }
    if (ne == 0) {
        if (nradii > 0)
            memset(out, 0, sizeof(long long) * (size_t)nradii * (size_t)query.num_fields *
                               (size_t)tree.num_fields);
        return KD_OK;
    }
    return kdg_count_static(&ht->cat, tree.num_fields, &hq->cat, query.num_fields, uniq, ne,
                            edge_of, nradii, mode, out);
}

/* mode used by pair_count on the calling thread (kd_set_precision) */
static __thread int g_pair_mode = KD_MODE_MIXED;

int kd_set_precision(int mode)
{
    clear_error();
    if (mode != KD_MODE_MIXED && mode != KD_MODE_FP64) {
        kd_set_error(KD_EINVAL, "kd_set_precision: unknown mode %d", mode);
        return KD_EINVAL;
    }
    g_pair_mode = mode;
    return KD_OK;
}

long long *pair_count(kdtree_t tree, double *data, int *fields, int length, int num_fields,
                      double r, int num_threads)
{
    long long *out;
    size_t nrow = (size_t)(num_fields > 0 ? num_fields : 0) * (size_t)(tree.num_fields > 0 ? tree.num_fields : 0);
    (void)num_threads;
    out = (long long *)calloc(nrow ? nrow : 1, sizeof(long long));
    if (!out) {
        kd_set_error(KD_ENOMEM, "out of host memory");
        return NULL;
    }
    if (kd_count_points(tree, data, fields, length, num_fields, &r, 1, g_pair_mode, out, NULL) !=
        KD_OK) {
        free(out);
        return NULL;
    }
    return out;
}
