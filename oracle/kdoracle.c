/*
 * CPU oracle for the corruscant pair-counting path -- TEST INFRASTRUCTURE ONLY.
 * See kdoracle.h.  Every function cites the reference lines it restates.
 *
 * Compiled with -ffp-contract=off: every fused multiply-add below is explicit,
 * mirroring the contractions gcc makes in the reference build
 * (oracle/Makefile explains which ones).
 */
#define _GNU_SOURCE
#include "kdoracle.h"

#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_err[256];

static int fail(int code, const char *msg)
{
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

const char *or_last_error(void) { return g_err; }

struct or_tree {
    int n_in;
    int n;          /* unique points */
    int memsize;
    int num_fields;
    double *u;      /* unique points, lexicographic order, interleaved xyz */
    int *ufield;    /* stored field (low 8 bits, as kdtree.h:15 keeps it) */
    int *uweight;
    int *urep;      /* input index of the representative (first occurrence) */
    int *npoint;    /* per heap slot: unique index, -1 when the slot is empty */
    unsigned char *nhas_l, *nhas_r, *ndim;
    int *inorder;   /* unique index at each in-order position */
};

/* ------------------------------------------------------------------ sorting */

/* Lexicographic (x,y,z) three-way compare with C '==' semantics, so that
 * -0.0 == +0.0.  Restates superkey_dupesafe, kdbuild.c:82-96. */
static int cmp_lex(const double *a, const double *b)
{
    for (int i = 0; i < 3; i++) {
        if (a[i] == b[i]) continue;
        return a[i] < b[i] ? -1 : 1;
    }
    return 0;
}

/* Cyclic superkey compare starting at dimension msd (kdbuild.c:59-80). */
static int cmp_super(const double *a, const double *b, int msd)
{
    for (int i = msd; i < msd + 3; i++) {
        int d = i % 3;
        if (a[d] == b[d]) continue;
        return a[d] < b[d] ? -1 : 1;
    }
    return 0;
}

typedef struct {
    const double *pts;
    int mode; /* -1: lexicographic, else superkey msd */
} sort_ctx;

static int ctx_cmp(const sort_ctx *c, int a, int b)
{
    const double *pa = c->pts + 3 * (size_t)a, *pb = c->pts + 3 * (size_t)b;
    return c->mode < 0 ? cmp_lex(pa, pb) : cmp_super(pa, pb, c->mode);
}

/* Stable bottom-up merge sort of an index array.  Stability reproduces the
 * reference mergesorts (kdbuild.c:98-152, 158-215): equal keys keep input
 * order, so the first occurrence of a duplicated point leads its run. */
static int stable_sort_idx(int *idx, int n, const sort_ctx *c)
{
    int *tmp = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!tmp) return OR_ENOMEM;
    for (int w = 1; w < n; w *= 2) {
        for (int lo = 0; lo < n; lo += 2 * w) {
            int mid = lo + w < n ? lo + w : n;
            int hi = lo + 2 * w < n ? lo + 2 * w : n;
            int i = lo, j = mid, k = lo;
            while (i < mid && j < hi) {
                if (ctx_cmp(c, idx[j], idx[i]) < 0) tmp[k++] = idx[j++];
                else tmp[k++] = idx[i++];
            }
            while (i < mid) tmp[k++] = idx[i++];
            while (j < hi) tmp[k++] = idx[j++];
        }
        memcpy(idx, tmp, sizeof(int) * (size_t)n);
    }
    free(tmp);
    return OR_OK;
}

/* ------------------------------------------------------------------- build */

typedef struct {
    or_tree_t *t;
    int *args[3];
    int *tmp;
    unsigned char *side;
} build_ctx;

/* max_variance_dim, kdbuild.c:308-351: per dimension a sequential sum in
 * args[j] order, mean by division, then a sequential sum of squared
 * deviations.  The reference build fuses the square into the accumulation
 * (one rounding per step), restated here with fma(). */
static int max_variance_dim(build_ctx *b, int l, int r)
{
    const double *u = b->t->u;
    double avg[3] = {0, 0, 0}, var[3] = {0, 0, 0};
    for (int j = 0; j < 3; j++)
        for (int i = l; i <= r; i++) avg[j] += u[3 * (size_t)b->args[j][i] + j];
    for (int j = 0; j < 3; j++) avg[j] /= (double)(r - l + 1);
    for (int j = 0; j < 3; j++)
        for (int i = l; i <= r; i++) {
            double d = u[3 * (size_t)b->args[j][i] + j] - avg[j];
            var[j] = fma(d, d, var[j]);
        }
    int dim = 0;
    double m = var[0];
    for (int j = 1; j < 3; j++)
        if (var[j] > m) { m = var[j]; dim = j; }
    return dim;
}

/* partition, kdbuild.c:251-291: for every dimension other than the split
 * dimension, a stable split of args[dim][l..r] into the points whose split
 * superkey is below the median's, then those above; the median is dropped.
 * The "below" set is exactly the points left of the median in
 * args[split][l..r], which is sorted by that superkey, so the sides are
 * marked from there instead of by comparing superkeys. */
static void partition(build_ctx *b, int l, int r, int split, int med)
{
    int *as = b->args[split];
    for (int i = l; i <= r; i++) b->side[as[i]] = i < med ? 0 : (i == med ? 2 : 1);
    for (int d = 0; d < 3; d++) {
        if (d == split) continue;
        int *a = b->args[d];
        int jl = 0, jr = med - l + 1;
        for (int i = l; i <= r; i++) {
            int p = a[i];
            if (b->side[p] == 2) continue;
            if (b->side[p] == 0) b->tmp[jl++] = p;
            else b->tmp[jr++] = p;
        }
        /* position med is never read again by the recursion; keep the
         * median there so every array stays a permutation */
        b->tmp[med - l] = as[med];
        memcpy(a + l, b->tmp, sizeof(int) * (size_t)(r - l + 1));
    }
}

/* build, kdbuild.c:373-433: median (l+r+1)/2 (kdbuild.c:52-55), split on the
 * max-variance dimension only for subtrees of 4+ points, sizes 1-3 are base
 * cases taken straight from args[0], children at heap slots 2p and 2p+1. */
static void build_rec(build_ctx *b, int p, int l, int r)
{
    or_tree_t *t = b->t;
    int med = (l + r + 1) / 2;
    int split = 0;
    if (r - l > 2) split = max_variance_dim(b, l, r);
    int pt = b->args[split][med];
    t->npoint[p] = pt;
    t->ndim[p] = (unsigned char)split;
    t->inorder[med] = pt;
    switch (r - l) {
    case 0:
        return;
    case 1:
        t->nhas_l[p] = 1;
        build_rec(b, 2 * p, l, l);
        return;
    case 2:
        t->nhas_l[p] = 1;
        t->nhas_r[p] = 1;
        build_rec(b, 2 * p, l, l);
        build_rec(b, 2 * p + 1, r, r);
        return;
    }
    partition(b, l, r, split, med);
    t->nhas_l[p] = 1;
    t->nhas_r[p] = 1;
    build_rec(b, 2 * p, l, med - 1);
    build_rec(b, 2 * p + 1, med + 1, r);
}

/* pow2ceil, kdbuild.c:435-449: 2^(floor(log2 n)+1) for n >= 1. */
static int heap_size(int n)
{
    int e = 1;
    while (n > 1) { n /= 2; e++; }
    return 1 << e;
}

void or_free(or_tree_t *t)
{
    if (!t) return;
    free(t->u); free(t->ufield); free(t->uweight); free(t->urep);
    free(t->npoint); free(t->nhas_l); free(t->nhas_r); free(t->ndim);
    free(t->inorder);
    free(t);
}

/* tree_construct, kdbuild.c:451-537. */
int or_build(const double *xyz, const int *fields, int n, int num_fields,
             or_tree_t **out)
{
    *out = NULL;
    if (n < 1) return fail(OR_EINVAL, "tree needs at least one point");
    for (size_t i = 0; i < 3 * (size_t)n; i++)
        if (isnan(xyz[i])) return fail(OR_ENAN, "NaN coordinate");

    or_tree_t *t = (or_tree_t *)calloc(1, sizeof *t);
    int *order = (int *)malloc(sizeof(int) * (size_t)n);
    if (!t || !order) { free(t); free(order); return fail(OR_ENOMEM, "oom"); }
    t->n_in = n;
    t->num_fields = num_fields;

    /* dedup: stable lexicographic sort, runs of '==' points merge into their
     * first occurrence, which keeps its field (kdbuild.c:479-499) */
    for (int i = 0; i < n; i++) order[i] = i;
    sort_ctx lc = {xyz, -1};
    if (stable_sort_idx(order, n, &lc)) { free(order); or_free(t); return fail(OR_ENOMEM, "oom"); }
    int nu = 0;
    for (int i = 0; i < n; i++)
        if (i == 0 || cmp_lex(xyz + 3 * (size_t)order[i - 1], xyz + 3 * (size_t)order[i]) != 0) nu++;
    t->n = nu;
    t->u = (double *)malloc(sizeof(double) * 3 * (size_t)nu);
    t->ufield = (int *)malloc(sizeof(int) * (size_t)nu);
    t->uweight = (int *)malloc(sizeof(int) * (size_t)nu);
    t->urep = (int *)malloc(sizeof(int) * (size_t)nu);
    if (!t->u || !t->ufield || !t->uweight || !t->urep) { free(order); or_free(t); return fail(OR_ENOMEM, "oom"); }
    int k = -1;
    for (int i = 0; i < n; i++) {
        int src = order[i];
        if (i == 0 || cmp_lex(xyz + 3 * (size_t)order[i - 1], xyz + 3 * (size_t)src) != 0) {
            k++;
            memcpy(t->u + 3 * (size_t)k, xyz + 3 * (size_t)src, 3 * sizeof(double));
            t->ufield[k] = fields ? (fields[src] & 0xFF) : 0;
            t->uweight[k] = 1;
            t->urep[k] = src;
        } else {
            t->uweight[k]++;
        }
    }
    free(order);
    for (int i = 0; i < nu; i++)
        if (t->uweight[i] > 255) {
            or_free(t);
            /* weight:8 (kdtree.h:16) wraps and the reference exits at
             * kdbuild.c:508-511 */
            return fail(OR_EDUP_OVERFLOW, "a point is repeated 256 or more times");
        }

    t->memsize = heap_size(nu);
    t->npoint = (int *)malloc(sizeof(int) * (size_t)t->memsize);
    t->nhas_l = (unsigned char *)calloc((size_t)t->memsize, 1);
    t->nhas_r = (unsigned char *)calloc((size_t)t->memsize, 1);
    t->ndim = (unsigned char *)calloc((size_t)t->memsize, 1);
    t->inorder = (int *)malloc(sizeof(int) * (size_t)nu);
    build_ctx b;
    memset(&b, 0, sizeof b);
    b.t = t;
    for (int d = 0; d < 3; d++) b.args[d] = (int *)malloc(sizeof(int) * (size_t)nu);
    b.tmp = (int *)malloc(sizeof(int) * (size_t)nu);
    b.side = (unsigned char *)malloc((size_t)nu);
    int ok = t->npoint && t->nhas_l && t->nhas_r && t->ndim && t->inorder &&
             b.args[0] && b.args[1] && b.args[2] && b.tmp && b.side;
    if (ok) {
        for (int i = 0; i < t->memsize; i++) t->npoint[i] = -1;
        /* superkey argsorts (kdbuild.c:221-243, 524-526) of the unique
         * points; the dedup order already is superkey-0 order */
        for (int d = 0; d < 3; d++) {
            for (int i = 0; i < nu; i++) b.args[d][i] = i;
            if (d > 0) {
                sort_ctx sc = {t->u, d};
                if (stable_sort_idx(b.args[d], nu, &sc)) ok = 0;
            }
        }
    }
    if (ok) build_rec(&b, 1, 0, nu - 1);
    for (int d = 0; d < 3; d++) free(b.args[d]);
    free(b.tmp);
    free(b.side);
    if (!ok) { or_free(t); return fail(OR_ENOMEM, "oom"); }
    *out = t;
    return OR_OK;
}

int or_tree_size(const or_tree_t *t) { return t->n; }
int or_tree_memsize(const or_tree_t *t) { return t->memsize; }
int or_tree_num_fields(const or_tree_t *t) { return t->num_fields; }

void or_tree_nodes(const or_tree_t *t, double *xyz, int *field, int *weight,
                   int *has_l, int *has_r, int *dim)
{
    for (int p = 0; p < t->memsize; p++) {
        int u = t->npoint[p];
        for (int d = 0; d < 3; d++) xyz[3 * (size_t)p + d] = u >= 0 ? t->u[3 * (size_t)u + d] : 0.0;
        field[p] = u >= 0 ? t->ufield[u] : 0;
        weight[p] = u >= 0 ? t->uweight[u] : 0;
        has_l[p] = t->nhas_l[p];
        has_r[p] = t->nhas_r[p];
        dim[p] = t->ndim[p];
    }
}

void or_tree_inorder(const or_tree_t *t, int *perm)
{
    for (int i = 0; i < t->n; i++) perm[i] = t->urep[t->inorder[i]];
}

void or_tree_unique(const or_tree_t *t, double *xyz, int *field, int *weight,
                    int *rep_index)
{
    memcpy(xyz, t->u, sizeof(double) * 3 * (size_t)t->n);
    memcpy(field, t->ufield, sizeof(int) * (size_t)t->n);
    memcpy(weight, t->uweight, sizeof(int) * (size_t)t->n);
    memcpy(rep_index, t->urep, sizeof(int) * (size_t)t->n);
}

/* ------------------------------------------------------------------ counting */

/* norm2, kdquery.c:39-47, as the reference build evaluates it: node minus
 * query per component, the first square rounded on its own, the other two
 * fused into the running sum. */
static inline double dist2_ref(const double *node, const double *q)
{
    double dx = node[0] - q[0], dy = node[1] - q[1], dz = node[2] - q[2];
    double s = dx * dx;
    s = fma(dy, dy, s);
    s = fma(dz, dz, s);
    return s;
}

/* Output index of the reference counter, kdquery.c:34 and :133-139: rows are
 * strided by the QUERY field count. */
static int check_layout(const or_tree_t *t, const int *qfields, int nq, int fq,
                        int nrow)
{
    int maxq = 0, minq = 0, maxt = 0;
    if (qfields)
        for (int i = 0; i < nq; i++) {
            if (qfields[i] > maxq) maxq = qfields[i];
            if (qfields[i] < minq) minq = qfields[i];
        }
    for (int i = 0; i < t->n; i++)
        if (t->ufield[i] > maxt) maxt = t->ufield[i];
    if (fq < 1 || t->num_fields < 1 || minq < 0) return OR_EFIELD;
    if ((long long)maxq * fq + maxt >= (long long)nrow) return OR_EFIELD;
    return OR_OK;
}

typedef struct {
    const or_tree_t *t;
    const double *q;
    const int *qf;
    int fq;
    int lo, hi;
    double rad, rsq;
    long long *cnt;
    long long visits;
    /* brute force */
    const double *rsq_sorted;
    const int *rank_of_sorted;
    int nsorted;
    long long *hist; /* (nsorted+1) * fq * ft */
} work_t;

/* radius, kdquery.c:62-113: distance tested at every visited node; prune on
 * the query coordinate +/- rad against the split value; a pruned node is not
 * counted; strict '<' against rad*rad. */
static void radius_rec(work_t *w, int p, const double *q, int qf)
{
    const or_tree_t *t = w->t;
    int u = t->npoint[p];
    const double *v = t->u + 3 * (size_t)u;
    w->visits++;
    double n2 = dist2_ref(v, q);
    int idx = qf * w->fq + t->ufield[u];
    if (!t->nhas_l[p]) {
        if (n2 < w->rsq) w->cnt[idx] += t->uweight[u];
        return;
    }
    if (!t->nhas_r[p]) {
        if (n2 < w->rsq) w->cnt[idx] += t->uweight[u];
        radius_rec(w, 2 * p, q, qf);
        return;
    }
    int d = t->ndim[p];
    double val = q[d];
    double upper = val + w->rad, lower = val - w->rad, point = v[d];
    if (upper < point) {
        radius_rec(w, 2 * p, q, qf);
    } else if (lower > point) {
        radius_rec(w, 2 * p + 1, q, qf);
    } else {
        if (n2 < w->rsq) w->cnt[idx] += t->uweight[u];
        radius_rec(w, 2 * p, q, qf);
        radius_rec(w, 2 * p + 1, q, qf);
    }
}

static void *radius_worker(void *arg)
{
    work_t *w = (work_t *)arg;
    for (int i = w->lo; i < w->hi; i++)
        radius_rec(w, 1, w->q + 3 * (size_t)i, w->qf ? w->qf[i] : 0);
    return NULL;
}

static int run_threads(work_t *ws, int nth, void *(*fn)(void *))
{
    pthread_t th[256];
    int started = 0;
    for (int i = 1; i < nth; i++)
        if (pthread_create(&th[i], NULL, fn, &ws[i]) == 0) started = i;
        else break;
    fn(&ws[0]);
    for (int i = started + 1; i < nth; i++) fn(&ws[i]);
    for (int i = 1; i <= started; i++) pthread_join(th[i], NULL);
    return OR_OK;
}

/* pair_count, kdquery.c:165-249, minus the thread pool: the per-thread
 * counter matrices are summed at the end exactly like kdquery.c:237-244. */
int or_pair_count(const or_tree_t *t, const double *q, const int *qfields,
                  int nq, int num_fields_q, double r, int nthreads,
                  long long *out, long long *visits)
{
    int nrow = num_fields_q * t->num_fields;
    if (nq < 0) return fail(OR_EINVAL, "negative query count");
    if (check_layout(t, qfields, nq, num_fields_q, nrow))
        return fail(OR_EFIELD, "field ids overflow the reference counter layout");
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 64) nthreads = 64;
    work_t ws[64];
    long long *cnt = (long long *)calloc((size_t)nthreads * (size_t)nrow, sizeof(long long));
    if (!cnt) return fail(OR_ENOMEM, "oom");
    for (int i = 0; i < nthreads; i++) {
        memset(&ws[i], 0, sizeof ws[i]);
        ws[i].t = t; ws[i].q = q; ws[i].qf = qfields; ws[i].fq = num_fields_q;
        ws[i].lo = (int)((long long)nq * i / nthreads);
        ws[i].hi = (int)((long long)nq * (i + 1) / nthreads);
        ws[i].rad = r; ws[i].rsq = r * r;
        ws[i].cnt = cnt + (size_t)i * (size_t)nrow;
    }
    run_threads(ws, nthreads, radius_worker);
    long long vis = 0;
    memset(out, 0, sizeof(long long) * (size_t)nrow);
    for (int i = 0; i < nthreads; i++) {
        for (int j = 0; j < nrow; j++) out[j] += ws[i].cnt[j];
        vis += ws[i].visits;
    }
    if (visits) *visits = vis;
    free(cnt);
    return OR_OK;
}

static void *brute_worker(void *arg)
{
    work_t *w = (work_t *)arg;
    const or_tree_t *t = w->t;
    int nrow = w->fq * t->num_fields;
    for (int i = w->lo; i < w->hi; i++) {
        const double *q = w->q + 3 * (size_t)i;
        int qf = w->qf ? w->qf[i] : 0;
        for (int u = 0; u < t->n; u++) {
            double d2 = dist2_ref(t->u + 3 * (size_t)u, q);
            /* first sorted edge with d2 < rsq; NaN d2 never counts */
            int lo = 0, hi = w->nsorted;
            while (lo < hi) {
                int mid = (lo + hi) / 2;
                if (d2 < w->rsq_sorted[mid]) hi = mid;
                else lo = mid + 1;
            }
            if (d2 != d2) lo = w->nsorted;
            w->hist[(size_t)lo * nrow + qf * w->fq + t->ufield[u]] += t->uweight[u];
        }
    }
    return NULL;
}

static int cmp_dbl(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

int or_brute_counts(const or_tree_t *t, const double *q, const int *qfields,
                    int nq, int num_fields_q, const double *radii, int nradii,
                    int nthreads, long long *out)
{
    int nrow = num_fields_q * t->num_fields;
    if (nq < 0 || nradii < 0) return fail(OR_EINVAL, "negative size");
    if (check_layout(t, qfields, nq, num_fields_q, nrow))
        return fail(OR_EFIELD, "field ids overflow the reference counter layout");
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 64) nthreads = 64;
    double *rs = (double *)malloc(sizeof(double) * (size_t)(nradii + 1));
    int ns = 0;
    for (int k = 0; k < nradii; k++) {
        double v = radii[k] * radii[k];
        if (v == v) rs[ns++] = v;
    }
    qsort(rs, (size_t)ns, sizeof(double), cmp_dbl);
    size_t hsz = (size_t)(ns + 1) * (size_t)nrow;
    long long *hist = (long long *)calloc((size_t)nthreads * hsz, sizeof(long long));
    if (!rs || !hist) { free(rs); free(hist); return fail(OR_ENOMEM, "oom"); }
    work_t ws[64];
    for (int i = 0; i < nthreads; i++) {
        memset(&ws[i], 0, sizeof ws[i]);
        ws[i].t = t; ws[i].q = q; ws[i].qf = qfields; ws[i].fq = num_fields_q;
        ws[i].lo = (int)((long long)nq * i / nthreads);
        ws[i].hi = (int)((long long)nq * (i + 1) / nthreads);
        ws[i].rsq_sorted = rs; ws[i].nsorted = ns;
        ws[i].hist = hist + (size_t)i * hsz;
    }
    run_threads(ws, nthreads, brute_worker);
    for (int i = 1; i < nthreads; i++)
        for (size_t j = 0; j < hsz; j++) hist[j] += hist[(size_t)i * hsz + j];
    for (int k = 0; k < nradii; k++) {
        double v = radii[k] * radii[k];
        long long *o = out + (size_t)k * nrow;
        memset(o, 0, sizeof(long long) * (size_t)nrow);
        if (v != v) continue;
        /* number of sorted edges <= v : pairs with d2 < v sit in bins
         * 0 .. (first sorted index with rs >= v) */
        int lo = 0, hi = ns;
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (rs[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        for (int b = 0; b <= lo && b < ns; b++)
            for (int j = 0; j < nrow; j++) o[j] += hist[(size_t)b * nrow + j];
    }
    free(rs);
    free(hist);
    return OR_OK;
}

/* Bin index of d2 among the sorted squared radii: the first with d2 < rsq
 * (nsorted when none; NaN never counts). */
static inline int bin_of(const work_t *w, double d2)
{
    int lo = 0, hi = w->nsorted;
    if (d2 != d2) return w->nsorted;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (d2 < w->rsq_sorted[mid]) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

/* The reference traversal (radius, kdquery.c:62-113) at radius w->rad, the
 * largest of the radii, binning every visited node's distance into all the
 * sorted radii at once.  The reference's prune at that radius never drops a
 * pair closer than it (if fl(q + rad) < split then every point of the right
 * subtree has fl(t - q) >= rad and so fl(d2) >= fl(rad*rad)), hence never one
 * closer than any smaller radius: the result is the exhaustive count. */
static void tree_bin_rec(work_t *w, int p, const double *q, int qf, int nrow)
{
    const or_tree_t *t = w->t;
    int u = t->npoint[p];
    const double *v = t->u + 3 * (size_t)u;
    double n2 = dist2_ref(v, q);
    w->hist[(size_t)bin_of(w, n2) * nrow + qf * w->fq + t->ufield[u]] += t->uweight[u];
    if (!t->nhas_l[p]) return;
    if (!t->nhas_r[p]) {
        tree_bin_rec(w, 2 * p, q, qf, nrow);
        return;
    }
    int d = t->ndim[p];
    double val = q[d];
    double upper = val + w->rad, lower = val - w->rad, point = v[d];
    if (upper < point) {
        tree_bin_rec(w, 2 * p, q, qf, nrow);
    } else if (lower > point) {
        tree_bin_rec(w, 2 * p + 1, q, qf, nrow);
    } else {
        tree_bin_rec(w, 2 * p, q, qf, nrow);
        tree_bin_rec(w, 2 * p + 1, q, qf, nrow);
    }
}

static void *tree_bin_worker(void *arg)
{
    work_t *w = (work_t *)arg;
    int nrow = w->fq * w->t->num_fields;
    for (int i = w->lo; i < w->hi; i++)
        tree_bin_rec(w, 1, w->q + 3 * (size_t)i, w->qf ? w->qf[i] : 0, nrow);
    return NULL;
}

int or_tree_counts(const or_tree_t *t, const double *q, const int *qfields,
                   int nq, int num_fields_q, const double *radii, int nradii,
                   int nthreads, long long *out)
{
    int nrow = num_fields_q * t->num_fields;
    double rmax = 0.0;
    if (nq < 0 || nradii < 0) return fail(OR_EINVAL, "negative size");
    for (int k = 0; k < nradii; k++) {
        double v = radii[k] * radii[k];
        if (radii[k] < 0) return fail(OR_EINVAL, "negative radius");
        if (v != v) continue;
        /* a squared radius of +inf counts every pair: no traversal prunes */
        if (v == INFINITY)
            return or_brute_counts(t, q, qfields, nq, num_fields_q, radii, nradii, nthreads, out);
        if (radii[k] > rmax) rmax = radii[k];
    }
    if (check_layout(t, qfields, nq, num_fields_q, nrow))
        return fail(OR_EFIELD, "field ids overflow the reference counter layout");
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 64) nthreads = 64;
    double *rs = (double *)malloc(sizeof(double) * (size_t)(nradii + 1));
    int ns = 0;
    if (!rs) return fail(OR_ENOMEM, "oom");
    for (int k = 0; k < nradii; k++) {
        double v = radii[k] * radii[k];
        if (v == v) rs[ns++] = v;
    }
    qsort(rs, (size_t)ns, sizeof(double), cmp_dbl);
    size_t hsz = (size_t)(ns + 1) * (size_t)nrow;
    long long *hist = (long long *)calloc((size_t)nthreads * hsz, sizeof(long long));
    if (!hist) { free(rs); return fail(OR_ENOMEM, "oom"); }
    work_t ws[64];
    for (int i = 0; i < nthreads; i++) {
        memset(&ws[i], 0, sizeof ws[i]);
        ws[i].t = t; ws[i].q = q; ws[i].qf = qfields; ws[i].fq = num_fields_q;
        ws[i].lo = (int)((long long)nq * i / nthreads);
        ws[i].hi = (int)((long long)nq * (i + 1) / nthreads);
        ws[i].rad = rmax;
        ws[i].rsq_sorted = rs; ws[i].nsorted = ns;
        ws[i].hist = hist + (size_t)i * hsz;
    }
    if (t->n > 0) run_threads(ws, nthreads, tree_bin_worker);
    for (int i = 1; i < nthreads; i++)
        for (size_t j = 0; j < hsz; j++) hist[j] += hist[(size_t)i * hsz + j];
    for (int k = 0; k < nradii; k++) {
        double v = radii[k] * radii[k];
        long long *o = out + (size_t)k * nrow;
        memset(o, 0, sizeof(long long) * (size_t)nrow);
        if (v != v) continue;
        int lo = 0, hi = ns;
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (rs[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        for (int b = 0; b <= lo && b < ns; b++)
            for (int j = 0; j < nrow; j++) o[j] += hist[(size_t)b * nrow + j];
    }
    free(rs);
    free(hist);
    return OR_OK;
}

/* ------------------------------------------------------------ visit count */

typedef struct {
    const double *nxyz;
    const int *has_l, *has_r, *dim;
    const double *q;
    int lo, hi;
    double r;
    long long visits;
} visit_t;

static void visit_rec(visit_t *v, int p, const double *q)
{
    v->visits++;
    if (!v->has_l[p]) return;
    if (!v->has_r[p]) {
        visit_rec(v, 2 * p, q);
        return;
    }
    int d = v->dim[p];
    double val = q[d], point = v->nxyz[3 * (size_t)p + d];
    if (val + v->r < point) visit_rec(v, 2 * p, q);
    else if (val - v->r > point) visit_rec(v, 2 * p + 1, q);
    else {
        visit_rec(v, 2 * p, q);
        visit_rec(v, 2 * p + 1, q);
    }
}

static void *visit_worker(void *arg)
{
    visit_t *v = (visit_t *)arg;
    for (int i = v->lo; i < v->hi; i++) visit_rec(v, 1, v->q + 3 * (size_t)i);
    return NULL;
}

long long or_count_visits(const double *nxyz, const int *has_l, const int *has_r,
                          const int *dim, int memsize, const double *q, int nq,
                          double r, int nthreads)
{
    (void)memsize;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 64) nthreads = 64;
    visit_t vs[64];
    pthread_t th[64];
    for (int i = 0; i < nthreads; i++) {
        vs[i] = (visit_t){nxyz, has_l, has_r, dim, q,
                          (int)((long long)nq * i / nthreads),
                          (int)((long long)nq * (i + 1) / nthreads), r, 0};
    }
    int started[64] = {0};
    for (int i = 1; i < nthreads; i++) started[i] = pthread_create(&th[i], NULL, visit_worker, &vs[i]) == 0;
    visit_worker(&vs[0]);
    long long tot = vs[0].visits;
    for (int i = 1; i < nthreads; i++) {
        if (started[i]) pthread_join(th[i], NULL);
        else visit_worker(&vs[i]);
        tot += vs[i].visits;
    }
    return tot;
}

/* ------------------------------------------------------------- coordinates */

#define OR_DEG2RAD (M_PI / 180.0) /* PI_OVER_180, coordmath.c:20 */

/* radec2cart64, coordmath.c:38-51 */
void or_radec2cart64(const double *ra, const double *dec, double *xyz, int n)
{
    for (int i = 0; i < n; i++) {
        double lon = ra[i] * OR_DEG2RAD, lat = dec[i] * OR_DEG2RAD;
        double c = cos(lat);
        xyz[3 * (size_t)i] = c * cos(lon);
        xyz[3 * (size_t)i + 1] = c * sin(lon);
        xyz[3 * (size_t)i + 2] = sin(lat);
    }
}

/* radecdist2cart64, coordmath.c:58-71 (left-to-right products) */
void or_radecdist2cart64(const double *ra, const double *dec,
                         const double *dist, double *xyz, int n)
{
    for (int i = 0; i < n; i++) {
        double lon = ra[i] * OR_DEG2RAD, lat = dec[i] * OR_DEG2RAD;
        double c = cos(lat);
        xyz[3 * (size_t)i] = dist[i] * c * cos(lon);
        xyz[3 * (size_t)i + 1] = dist[i] * c * sin(lon);
        xyz[3 * (size_t)i + 2] = dist[i] * sin(lat);
    }
}

/* radec2sph64, coordmath.c:73-80 */
void or_radec2sph64(const double *ra, const double *dec, double *theta,
                    double *phi, int n)
{
    for (int i = 0; i < n; i++) {
        theta[i] = (90.0 - dec[i]) * OR_DEG2RAD;
        phi[i] = ra[i] * OR_DEG2RAD;
    }
}
