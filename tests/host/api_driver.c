/*
 * Host-library driver for the sanitizer tests: the real kd_api.c linked with
 * the CPU stand-in of the device layer (fake_device.c).  Scenarios:
 *   count   - the C ABI's counts against an independent brute force here
 *             (radius order, repeats and NaN, query-major layout, batch
 *             concatenation, per-bin differences, pair_count, the static
 *             entry point);
 *   threads - several threads building, counting and destroying trees at
 *             once (run under ThreadSanitizer);
 *   faults  - argument errors, injected device-layer failures and an
 *             allocator that fails each allocation in turn (run under
 *             AddressSanitizer, which also reports leaks);
 *   coords  - the threaded RA/DEC conversion (coords_api.c), three callers
 *             at once, against a single-threaded evaluation;
 *   fuzz    - 4,000 calls of the counting entry points with random counts,
 *             radii, modes, field counts, NULL arrays and dead handles: each
 *             succeeds exactly when the argument rules say it must, and then
 *             with the brute-force counts (run under AddressSanitizer).
 * Prints PASS/FAIL lines; the exit status is the number of failures.
 */
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "coordmath.h"
#include "kdtree.h"

extern int fake_fail_build, fake_fail_count, fake_fail_copy;

/* ---- allocator that can fail (kd_api.c's malloc/calloc/posix_memalign) */
int fake_alloc_countdown = 0;
static pthread_mutex_t alloc_mu = PTHREAD_MUTEX_INITIALIZER;
static int alloc_should_fail(void)
{
    int fail = 0;
    pthread_mutex_lock(&alloc_mu);
    if (fake_alloc_countdown > 0 && --fake_alloc_countdown == 0) fail = 1;
    pthread_mutex_unlock(&alloc_mu);
    return fail;
}
void *fake_malloc(size_t n) { return alloc_should_fail() ? NULL : malloc(n); }
void *fake_calloc(size_t c, size_t s) { return alloc_should_fail() ? NULL : calloc(c, s); }
int fake_posix_memalign(void **p, size_t a, size_t n)
{
    if (alloc_should_fail()) return 12; /* ENOMEM */
    return posix_memalign(p, a, n);
}

static int failures = 0;
#define CHECK(cond, ...)                                  \
    do {                                                  \
        if (!(cond)) {                                    \
            failures++;                                   \
            printf("FAIL %s:%d: ", __FILE__, __LINE__);   \
            printf(__VA_ARGS__);                          \
            printf("\n");                                 \
        }                                                 \
    } while (0)

static unsigned long long rng = 88172645463325252ull;
static double urand(void)
{
    rng ^= rng << 13;
    rng ^= rng >> 7;
    rng ^= rng << 17;
    return (double)(rng >> 11) * (1.0 / 9007199254740992.0);
}

typedef struct {
    double *xyz;
    int *f;
    int n, nf;
} cat_t;

static cat_t make_cat(int n, int nf)
{
    cat_t c;
    int i;
    c.n = n;
    c.nf = nf;
    c.xyz = (double *)malloc(sizeof(double) * 3 * (size_t)n);
    c.f = (int *)malloc(sizeof(int) * (size_t)n);
    for (i = 0; i < 3 * n; i++) c.xyz[i] = urand();
    for (i = 0; i < n; i++) c.f[i] = (int)(c.xyz[3 * i] * nf) % nf;
    return c;
}

/* expected out[k][qf*Fq + tf] for radius k: the reference's pair_count */
static void brute(const cat_t *t, const cat_t *q, const double *radii, int nr, long long *out)
{
    int k, i, j;
    const int Fq = q->nf, Ft = t->nf;
    memset(out, 0, sizeof(long long) * (size_t)nr * Fq * Ft);
    for (k = 0; k < nr; k++) {
        const double rsq = radii[k] * radii[k];
        for (i = 0; i < q->n; i++)
            for (j = 0; j < t->n; j++) {
                const double *a = t->xyz + 3 * j, *b = q->xyz + 3 * i;
                const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
                const double d2 = fma(dz, dz, fma(dy, dy, dx * dx));
                if (d2 < rsq) out[(size_t)k * Fq * Ft + (size_t)q->f[i] * Fq + t->f[j]]++;
            }
    }
}

static int same(const long long *a, const long long *b, size_t n)
{
    return memcmp(a, b, sizeof(long long) * n) == 0;
}

static const double RADII[] = {0.3, 0.05, NAN, 0.2, 0.05, 0.0, INFINITY, 0.12};
#define NR ((int)(sizeof RADII / sizeof RADII[0]))

static void scenario_count(void)
{
    cat_t a = make_cat(300, 3), b = make_cat(500, 3);
    kdtree_t ta = tree_construct(a.xyz, a.f, a.n, a.nf), tb = tree_construct(b.xyz, b.f, b.n, b.nf);
    long long want[3][NR * 9], got[3 * NR * 9], cum[NR * 9];
    kdtree_t trees[3] = {ta, tb, tb}, queries[3] = {ta, ta, tb};
    const cat_t *tc[3] = {&a, &b, &b}, *qc[3] = {&a, &a, &b};
    int j, k;
    CHECK(ta.node_data && tb.node_data, "tree_construct failed");
    for (j = 0; j < 3; j++) {
        brute(tc[j], qc[j], RADII, NR, want[j]);
        CHECK(kd_count_radii(trees[j], queries[j], RADII, NR, KD_MODE_MIXED, got, NULL) == 0,
              "kd_count_radii");
        CHECK(same(got, want[j], NR * 9), "kd_count_radii job %d differs", j);
    }
    CHECK(kd_count_batch(trees, queries, 3, RADII, NR, KD_MODE_FP64, got, NULL) == 0,
          "kd_count_batch");
    for (j = 0; j < 3; j++) CHECK(same(got + j * NR * 9, want[j], NR * 9), "batch job %d", j);
    {
        const double edges[] = {0.0, 0.05, 0.12, 0.2, 0.3};
        long long bins[4 * 9], e_cum[5 * 9];
        brute(&b, &a, edges, 5, e_cum);
        CHECK(kd_count_bins(tb, ta, edges, 5, KD_MODE_MIXED, bins, NULL) == 0, "kd_count_bins");
        for (k = 0; k < 4 * 9; k++) CHECK(bins[k] == e_cum[k + 9] - e_cum[k], "bin %d", k);
    }
    {
        long long *p = pair_count(tb, a.xyz, a.f, a.n, 3, 0.2, 4);
        brute(&b, &a, (const double[]){0.2}, 1, cum);
        CHECK(p && same(p, cum, 9), "pair_count");
        kd_free_counts(p);
    }
    CHECK(kd_count_radii_static(tb, ta, RADII, NR, KD_MODE_MIXED, got) == 0, "static");
    CHECK(same(got, want[1], NR * 9), "static differs");
    destroy(ta);
    destroy(tb);
    destroy(ta); /* a second destroy of the same tree is a no-op */
    free(a.xyz), free(a.f), free(b.xyz), free(b.f);
    printf("PASS count\n");
}

/* ---- threads */
static cat_t g_cat;
static long long g_want[NR * 4];
static void *worker(void *arg)
{
    int it;
    (void)arg;
    for (it = 0; it < 40; it++) {
        long long got[NR * 4];
        char msg[128];
        kdtree_t t = tree_construct(g_cat.xyz, g_cat.f, g_cat.n, g_cat.nf);
        if (!t.node_data) {
            CHECK(0, "threaded tree_construct");
            continue;
        }
        CHECK(kd_count_radii(t, t, RADII, NR, it & 1, got, NULL) == 0, "threaded count");
        CHECK(same(got, g_want, NR * 4), "threaded count differs");
        /* errors stay per thread */
        CHECK(kd_count_radii(t, t, (const double[]){-1.0}, 1, 0, got, NULL) < 0, "neg radius");
        CHECK(kd_last_error(msg, sizeof msg) < 0 && strstr(msg, "negative"), "thread error: %s", msg);
        destroy(t);
    }
    return NULL;
}

static void scenario_threads(void)
{
    pthread_t th[8];
    int i;
    g_cat = make_cat(200, 2);
    brute(&g_cat, &g_cat, RADII, NR, g_want);
    for (i = 0; i < 8; i++) pthread_create(&th[i], NULL, worker, NULL);
    for (i = 0; i < 8; i++) pthread_join(th[i], NULL);
    free(g_cat.xyz), free(g_cat.f);
    printf("PASS threads\n");
}

/* ---- faults */
static int sequence(const cat_t *a)
{
    /* a whole use of the library; returns the number of calls that failed */
    int bad = 0;
    long long out[NR * 4], *p;
    kdtree_t t = tree_construct(a->xyz, a->f, a->n, a->nf), trees[2], qs[2];
    if (!t.node_data) return 1;
    bad += kd_count_radii(t, t, RADII, NR, 0, out, NULL) != 0;
    trees[0] = trees[1] = qs[0] = qs[1] = t;
    {
        long long big[2 * NR * 4];
        bad += kd_count_batch(trees, qs, 2, RADII, NR, 0, big, NULL) != 0;
    }
    p = pair_count(t, a->xyz, a->f, a->n, a->nf, 0.1, 1);
    bad += p == NULL;
    kd_free_counts(p);
    bad += kd_count_points(t, a->xyz, a->f, a->n, a->nf, RADII, NR, 0, out, NULL) != 0;
    destroy(t);
    return bad;
}

static void scenario_faults(void)
{
    cat_t a = make_cat(150, 2);
    long long out[NR * 4];
    kdtree_t t;
    int n, code, okruns = 0;
    char msg[128];

    /* argument errors */
    t = tree_construct(a.xyz, a.f, a.n, a.nf);
    CHECK(kd_count_radii(t, t, RADII, NR, 5, out, NULL) < 0, "bad mode");
    CHECK(kd_count_radii_shard(t, t, RADII, NR, 0, 2, 2, out, NULL) < 0, "bad shard");
    CHECK(kd_set_precision(9) < 0 && kd_set_precision(KD_MODE_FP64) == 0, "precision");
    kd_set_precision(KD_MODE_MIXED);
    CHECK(kd_set_device(3) < 0, "device");
    {
        /* any number of distinct radii (counted in passes of 64): 150 radii,
         * each count equal to the same radius counted on its own */
        double r[150];
        long long *o150 = (long long *)malloc(sizeof(long long) * 150 * 16);
        long long one[16];
        for (n = 0; n < 150; n++) r[n] = 0.004 * ((n * 37) % 150 + 1);
        CHECK(kd_count_radii(t, t, r, 150, 0, o150, NULL) == 0, "150 distinct radii refused");
        for (n = 0; n < 150; n += 7) {
            CHECK(kd_count_radii(t, t, r + n, 1, 0, one, NULL) == 0, "one radius");
            CHECK(memcmp(one, o150 + (size_t)n * a.nf * a.nf, sizeof(long long) * a.nf * a.nf) == 0,
                  "radius %d of 150 differs from its own count", n);
        }
        CHECK(kd_count_radii_static(t, t, r, 65, 0, o150) < 0, "static: 65 radii accepted");
        CHECK(kd_count_radii(t, t, (const double[]){0.1, -0.1}, 2, 0, o150, NULL) < 0, "neg");
        free(o150);
    }
    /* malformed counts and pointers are errors, never memory accesses */
    CHECK(kd_count_radii(t, t, RADII, -1, 0, out, NULL) == KD_EINVAL, "negative radius count");
    CHECK(kd_count_radii(t, t, NULL, 3, 0, out, NULL) == KD_EINVAL, "NULL radii");
    CHECK(kd_count_radii(t, t, RADII, NR, 0, NULL, NULL) == KD_EINVAL, "NULL output");
    CHECK(kd_count_batch(&t, &t, 1, RADII, -3, 0, out, NULL) == KD_EINVAL, "batch: negative count");
    CHECK(kd_count_points(t, a.xyz, a.f, 0, 0, RADII, NR, 0, out, NULL) == KD_EFIELD,
          "no queries, zero query fields");
    CHECK(kd_count_points(t, a.xyz, a.f, 0, -4, RADII, NR, 0, out, NULL) == KD_EFIELD,
          "no queries, negative query fields");
    CHECK(kd_count_points(t, a.xyz, a.f, 0, a.nf, RADII, NR, 0, NULL, NULL) == KD_EINVAL,
          "no queries, NULL output");
    CHECK(kd_count_points(t, a.xyz, a.f, 0, a.nf, NULL, NR, 0, out, NULL) == KD_EINVAL,
          "no queries, NULL radii");
    {
        double nanq[6] = {NAN, 0.1, 0.2, 0.3, NAN, 0.5};
        CHECK(kd_count_points(t, nanq, NULL, 2, 0, RADII, NR, 0, out, NULL) == KD_EFIELD,
              "NaN-only queries, zero query fields");
        CHECK(kd_count_points(t, nanq, NULL, 2, 1, RADII, 0, 0, NULL, NULL) == KD_OK,
              "no radii, no output array");
    }
    {
        /* the size check comes before any point is read (a.xyz holds 150) */
        kdtree_t big = tree_construct(a.xyz, a.f, KD_MAX_POINTS + 1, a.nf);
        CHECK(!big.node_data && kd_last_error(msg, sizeof msg) == KD_EINVAL &&
                  strstr(msg, "at most"), "2^30 points: %s", msg);
        CHECK(kd_count_points(t, a.xyz, a.f, KD_MAX_POINTS + 1, a.nf, RADII, NR, 0, out, NULL) ==
                  KD_EINVAL, "2^30 query points");
        CHECK(pair_count(t, a.xyz, a.f, KD_MAX_POINTS + 1, a.nf, 0.1, 1) == NULL,
              "pair_count with 2^30 points");
    }
    destroy(t);

    /* injected device-layer failures: clean errors, nothing leaks */
    fake_fail_build = -2;
    t = tree_construct(a.xyz, a.f, a.n, a.nf);
    code = kd_last_error(msg, sizeof msg);
    CHECK(!t.node_data && code == -2 && strstr(msg, "injected"), "build failure: %d %s", code, msg);
    fake_fail_build = 0;
    fake_fail_copy = -6;
    t = tree_construct(a.xyz, a.f, a.n, a.nf);
    CHECK(!t.node_data && kd_last_error(NULL, 0) == -6, "copy failure");
    fake_fail_copy = 0;
    /* deferred builds: counted before the wait; a copy failure is reported
     * by the wait, and destroy without a wait releases everything */
    {
        kdtree_t d = kd_tree_construct_deferred(a.xyz, a.f, a.n, a.nf);
        long long *want = (long long *)malloc(sizeof(long long) * NR * a.nf * a.nf);
        CHECK(d.node_data && want, "deferred build");
        t = tree_construct(a.xyz, a.f, a.n, a.nf);
        CHECK(kd_count_radii(t, t, RADII, NR, 0, want, NULL) == KD_OK &&
                  kd_count_radii(d, d, RADII, NR, 0, out, NULL) == KD_OK &&
                  !memcmp(want, out, sizeof(long long) * NR * a.nf * a.nf),
              "deferred tree counts");
        CHECK(kd_tree_wait_nodes(d) == KD_OK && kd_tree_wait_nodes(d) == KD_OK &&
                  kd_tree_wait_nodes(t) == KD_OK, "waits");
        destroy(d);
        CHECK(kd_tree_wait_nodes(d) == KD_EINVAL, "wait on a destroyed tree");
        destroy(t);
        free(want);
        fake_fail_copy = -6;
        d = kd_tree_construct_deferred(a.xyz, a.f, a.n, a.nf);
        CHECK(d.node_data && kd_tree_wait_nodes(d) == -6 &&
                  kd_last_error(msg, sizeof msg) == -6 && strstr(msg, "injected"),
              "deferred copy failure: %s", msg);
        destroy(d);
        d = kd_tree_construct_deferred(a.xyz, a.f, a.n, a.nf);
        CHECK(d.node_data, "deferred build");
        destroy(d); /* never waited for */
        fake_fail_copy = 0;
    }
    t = tree_construct(a.xyz, a.f, a.n, a.nf);
    fake_fail_count = -8;
    CHECK(kd_count_radii(t, t, RADII, NR, 0, out, NULL) == -8, "count failure");
    CHECK(pair_count(t, a.xyz, a.f, a.n, a.nf, 0.1, 1) == NULL, "pair_count failure");
    fake_fail_count = 0;
    destroy(t);

    /* every allocation of a whole sequence failing in turn */
    for (n = 1; n < 200; n++) {
        int bad;
        fake_alloc_countdown = n;
        bad = sequence(&a);
        if (fake_alloc_countdown > 0) { /* the n-th allocation was never reached */
            fake_alloc_countdown = 0;
            CHECK(bad == 0, "sequence failed without an injected failure");
            okruns++;
            break;
        }
        CHECK(bad > 0, "allocation %d failed but every call succeeded", n);
    }
    CHECK(okruns == 1 && n > 5, "allocation sweep ended after %d steps", n);
    free(a.xyz), free(a.f);
    printf("PASS faults (%d allocation points)\n", n - 1);
}

/* ---- coords: the threaded host conversion against a single-threaded
 * evaluation of the reference's formula (coordmath.c:38-51), from several
 * callers at once */
#define NC 1000000
static double *c_ra, *c_dec, *c_want;
static void *coord_worker(void *arg)
{
    double *xyz = (double *)malloc(sizeof(double) * 3 * NC);
    (void)arg;
    radec2cart64(c_ra, c_dec, xyz, NC);
    CHECK(memcmp(xyz, c_want, sizeof(double) * 3 * NC) == 0, "threaded radec2cart64 differs");
    free(xyz);
    return NULL;
}

static void scenario_coords(void)
{
    const double d2r = M_PI / 180.0;
    pthread_t th[3];
    int i;
    c_ra = (double *)malloc(sizeof(double) * NC);
    c_dec = (double *)malloc(sizeof(double) * NC);
    c_want = (double *)malloc(sizeof(double) * 3 * NC);
    for (i = 0; i < NC; i++) {
        double lon, lat, c;
        c_ra[i] = 360.0 * urand();
        c_dec[i] = 180.0 * urand() - 90.0;
        lon = c_ra[i] * d2r;
        lat = c_dec[i] * d2r;
        c = cos(lat);
        c_want[3 * i] = c * cos(lon);
        c_want[3 * i + 1] = c * sin(lon);
        c_want[3 * i + 2] = sin(lat);
    }
    for (i = 0; i < 3; i++) pthread_create(&th[i], NULL, coord_worker, NULL);
    for (i = 0; i < 3; i++) pthread_join(th[i], NULL);
    free(c_ra), free(c_dec), free(c_want);
    printf("PASS coords\n");
}

/* ---- fuzz: random arguments, valid and not, through every counting entry
 * point.  An independent statement of the argument rules predicts whether a
 * call must succeed; it must then give the brute-force counts, and otherwise
 * return a negative code.  Run under ASAN/UBSAN: no call may touch memory
 * it should not. */

/* distinct non-NaN squared radii among the first n, or -1 if one is negative */
static int distinct_edges(const double *r, int n)
{
    double u[160];
    int k, j, m = 0;
    for (k = 0; k < n; k++) {
        const double v = r[k] * r[k];
        if (r[k] < 0) return -1;
        if (v != v) continue;
        for (j = 0; j < m && u[j] != v; j++)
            ;
        if (j == m) u[m++] = v;
    }
    return m;
}

/* the reference's counter holds every (qfield, tfield) of these catalogs */
static int layout_ok(const cat_t *t, const cat_t *q)
{
    int i, mq = 0, mt = 0;
    for (i = 0; i < q->n; i++) mq = q->f[i] > mq ? q->f[i] : mq;
    for (i = 0; i < t->n; i++) mt = t->f[i] > mt ? t->f[i] : mt;
    return (long long)mq * q->nf + mt < (long long)q->nf * t->nf;
}

static void scenario_fuzz(void)
{
    cat_t a = make_cat(60, 2), b = make_cat(90, 3), c = make_cat(40, 1);
    cat_t *cats[3] = {&a, &b, &c};
    kdtree_t tr[3], dead;
    long long *out = (long long *)malloc(sizeof(long long) * 8192);
    long long *want = (long long *)malloc(sizeof(long long) * 8192);
    long long *cum = (long long *)malloc(sizeof(long long) * 8192);
    double radii[150];
    int it, i, k, succeeded = 0, refused = 0;
    for (i = 0; i < 3; i++)
        tr[i] = tree_construct(cats[i]->xyz, cats[i]->f, cats[i]->n, cats[i]->nf);
    memset(&dead, 0, sizeof dead);
    for (it = 0; it < 4000; it++) {
        const int ti = (int)(urand() * 3), qi = (int)(urand() * 3), which = (int)(urand() * 5);
        const cat_t *T = cats[ti], *Q = cats[qi];
        const int nr = (int)(urand() * 145) - 5; /* -5 .. 139: past one pass of 64 */
        const int mode = urand() < 0.9 ? (int)(urand() * 2) : (int)(urand() * 7) - 3;
        const int null_r = urand() < 0.05, null_o = urand() < 0.05, bad_tree = urand() < 0.03;
        const double *R = null_r ? NULL : radii;
        long long *O = null_o ? NULL : out;
        const kdtree_t tt = bad_tree ? dead : tr[ti];
        const int Fq = Q->nf, Ft = T->nf;
        int rc, ne, expect_ok;
        for (k = 0; k < 150; k++) {
            const double u = urand();
            radii[k] = u < 0.05 ? NAN : u < 0.08 ? INFINITY : urand() * 0.5;
        }
        if (urand() < 0.12) radii[(int)(urand() * (nr > 0 ? nr : 1))] = -0.1; /* one negative */
        ne = nr > 0 && !null_r ? distinct_edges(radii, nr) : 0;
        /* rules shared by every entry point */
        expect_ok = !bad_tree && nr >= 0 && (nr == 0 || (!null_r && !null_o)) &&
                    (mode == 0 || mode == 1) && ne >= 0;
        memset(out, 0x5a, sizeof(long long) * 8192);
        switch (which) {
        case 0: /* kd_count_radii */
            expect_ok = expect_ok && layout_ok(T, Q);
            rc = kd_count_radii(tt, tr[qi], R, nr, mode, O, NULL);
            if (rc == 0 && expect_ok) {
                brute(T, Q, radii, nr, want);
                CHECK(same(out, want, (size_t)nr * Fq * Ft), "fuzz %d radii counts", it);
            }
            break;
        case 1: { /* kd_count_points with a possibly bad length or field count */
            const double u = urand();
            const int len = u < 0.05 ? -3 : u < 0.12 ? 0 : Q->n;
            const int fq = urand() < 0.05 ? (int)(urand() * 3) - 2 : Fq;
            expect_ok = expect_ok && len >= 0 && fq >= 1 && (len == 0 || layout_ok(T, Q));
            rc = kd_count_points(tt, Q->xyz, Q->f, len, fq, R, nr, mode, O, NULL);
            if (rc == 0 && expect_ok) {
                if (len == 0) memset(want, 0, sizeof(long long) * (size_t)nr * Fq * Ft);
                else brute(T, Q, radii, nr, want);
                CHECK(same(out, want, (size_t)nr * Fq * Ft), "fuzz %d point counts", it);
            }
            break;
        }
        case 2: /* kd_count_bins: at least one edge, arrays required */
            expect_ok = expect_ok && nr >= 1 && !null_r && !null_o && layout_ok(T, Q);
            rc = kd_count_bins(tt, tr[qi], R, nr, mode, O, NULL);
            if (rc == 0 && expect_ok) {
                brute(T, Q, radii, nr, cum);
                for (k = 0; k + 1 < nr; k++)
                    for (i = 0; i < Fq * Ft; i++)
                        want[k * Fq * Ft + i] = cum[(k + 1) * Fq * Ft + i] - cum[k * Fq * Ft + i];
                CHECK(same(out, want, (size_t)(nr - 1) * Fq * Ft), "fuzz %d bins", it);
            }
            break;
        case 3: { /* kd_count_batch: jobs (T, Q) and (Q, T); output always required */
            const kdtree_t ts[2] = {tt, tr[qi]}, qs[2] = {tr[qi], tr[ti]};
            const int nj = urand() < 0.05 ? 0 : 2;
            expect_ok = expect_ok && nj == 2 && !null_o && layout_ok(T, Q) && layout_ok(Q, T);
            rc = kd_count_batch(ts, qs, nj, R, nr, mode, O, NULL);
            if (rc == 0 && expect_ok) {
                const size_t n0 = (size_t)nr * Fq * Ft;
                brute(T, Q, radii, nr, want);
                brute(Q, T, radii, nr, want + n0);
                CHECK(same(out, want, 2 * n0), "fuzz %d batch", it);
            }
            break;
        }
        default: /* kd_count_radii_static: at most 64 radii */
            expect_ok = expect_ok && nr <= 64 && layout_ok(T, Q);
            rc = kd_count_radii_static(tt, tr[qi], R, nr, mode, O);
            if (rc == 0 && expect_ok) {
                brute(T, Q, radii, nr, want);
                CHECK(same(out, want, (size_t)nr * Fq * Ft), "fuzz %d static", it);
            }
            break;
        }
        CHECK(rc <= 0, "fuzz %d: positive return %d", it, rc);
        CHECK((rc == 0) == (expect_ok != 0), "fuzz %d (entry %d, nr %d, mode %d, ne %d): rc %d", it,
              which, nr, mode, ne, rc);
        if (rc == 0) succeeded++;
        else refused++;
    }
    CHECK(succeeded > 1000 && refused > 500, "fuzz mix: %d succeeded, %d refused", succeeded,
          refused);
    for (i = 0; i < 3; i++) {
        destroy(tr[i]);
        free(cats[i]->xyz);
        free(cats[i]->f);
    }
    free(out);
    free(want);
    free(cum);
    printf("%s fuzz (%d calls succeeded, %d refused)\n", failures ? "FAIL" : "PASS", succeeded,
           refused);
}

int main(int argc, char **argv)
{
    int i;
    for (i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "count")) scenario_count();
        else if (!strcmp(argv[i], "threads")) scenario_threads();
        else if (!strcmp(argv[i], "faults")) scenario_faults();
        else if (!strcmp(argv[i], "coords")) scenario_coords();
        else if (!strcmp(argv[i], "fuzz")) scenario_fuzz();
    }
    printf("%d failures\n", failures);
    return failures;
}
