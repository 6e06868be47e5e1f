/*
 * Jackknife field division for libcoords.so (include/fields.h): the HEALPix
 * RING pixelisation and a weighted graph partition, the two pieces the
 * reference's corruscant/fields.py takes from healpy and pymetis.
 *
 * HEALPix, from its published definition (Gorski et al. 2005):
 *   - 12 base faces: four around the north pole, four on the equator, four
 *     around the south pole; face f has row f/4 and its centre at longitude
 *     (pi/4) * L_f with L_f = 2k+1 (polar rows) or 2k (equatorial row),
 *     k = f mod 4;
 *   - each face is an nside x nside grid of pixels; a point of the face has
 *     continuous coordinates (x, y) in [0, nside]^2, x growing to the
 *     north-east, y to the north-west, and lies on the continuous ring
 *     jr = (row + 2) * nside - x - y (0 at the north pole, 4 nside at the
 *     south pole) at longitude (pi/4) (L_f * nr + x - y) / nr, where nr is jr
 *     in the north cap (jr < nside), 4 nside - jr in the south cap and nside
 *     in the equatorial belt;
 *   - z = cos(theta) is 1 - jr^2 / (3 nside^2) in the north cap,
 *     (2 nside - jr) * 2 / (3 nside) in the belt, mirrored in the south;
 *   - RING numbering runs ring by ring from the north pole, each ring by
 *     increasing longitude: ring i has 4i pixels in the north cap (i < nside),
 *     4 nside in the belt, 4(4 nside - i) in the south cap, with centres at
 *     longitude (j + 1/2) pi / (2 nr), except that every other belt ring (the
 *     rings i with i + nside odd) starts at longitude 0.
 * ang2pix inverts this with the two families of pixel boundaries (in the
 * belt the lines nside (1/2 + t) -+ (3/4) nside z = integer, in the caps
 * t' sigma and (1 - t') sigma = integer with sigma = nside sqrt(3 (1 - |z|))
 * and t' the longitude within the quarter), as the paper describes.
 *
 * The partition is a recursive bisection written for this project: a
 * weighted greedy graph growing from a peripheral vertex (four starts, the
 * best kept), then Fiduccia-Mattheyses boundary refinement under a balance
 * tolerance of 1% of the weight (or the heaviest vertex).
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "fields.h"

#define HP_MAX_NSIDE (1 << 20)
#define HP_PI 3.141592653589793
#define HP_HALFPI 1.5707963267948966
#define HP_SQRT6 2.449489742783178

static int face_row(int f) { return f >> 2; }
static int face_lon(int f) { return face_row(f) == 1 ? 2 * (f & 3) : 2 * (f & 3) + 1; }

/* longitude in units of pi/2, in [0, 4) */
static double quarter_coord(double phi)
{
    double tt = fmod(phi / HP_HALFPI, 4.0);
    if (tt < 0.0) tt += 4.0;
    if (tt >= 4.0) tt -= 4.0;
    return tt;
}

/* nside * sqrt(3 (1 - |z|)), the polar-cap ring coordinate; near the poles
 * from sin(theta), which keeps its precision where 1 - |cos(theta)| does not */
static double cap_sigma(double ns, double theta, double za)
{
    if (theta < 0.01 || theta > HP_PI - 0.01) return ns * sin(theta) * sqrt(3.0 / (1.0 + za));
    return ns * sqrt(3.0 * (1.0 - za));
}

static long long ang2pix1(long long N, double theta, double phi)
{
    const double ns = (double)N, z = cos(theta), za = fabs(z), tt = quarter_coord(phi);
    if (za <= 2.0 / 3.0) {
        /* belt: indices of the two boundary families through the point */
        const double t1 = ns * (0.5 + tt), t2 = ns * z * 0.75;
        const long long jp = (long long)floor(t1 - t2), jm = (long long)floor(t1 + t2);
        const long long ir = N + 1 + jp - jm; /* 1 .. 2N+1, counted from z = 2/3 */
        const long long kshift = 1 - (ir & 1);
        const long long ip = ((jp + jm - N + kshift + 1) / 2) % (4 * N);
        return 2 * N * (N - 1) + (ir - 1) * 4 * N + ip;
    } else {
        const double tp = tt - floor(tt), s = cap_sigma(ns, theta, za);
        const long long jp = (long long)floor(tp * s), jm = (long long)floor((1.0 - tp) * s);
        const long long ir = jp + jm + 1; /* ring counted from the nearer pole */
        long long ip = (long long)floor(tt * (double)ir);
        if (ip >= 4 * ir) ip = 4 * ir - 1;
        return z > 0 ? 2 * ir * (ir - 1) + ip : 12 * N * N - 2 * ir * (ir + 1) + ip;
    }
}

/* largest i with 2 i (i - 1) <= q */
static long long ring_of_cap_index(long long q)
{
    long long i = (long long)((1.0 + sqrt(1.0 + 2.0 * (double)q)) / 2.0);
    while (i > 1 && 2 * i * (i - 1) > q) i--;
    while (2 * (i + 1) * i <= q) i++;
    return i;
}

static void pix2ang1(long long N, long long p, double *theta, double *phi)
{
    const double ns = (double)N;
    const long long ncap = 2 * N * (N - 1), npix = 12 * N * N;
    if (p < ncap) {
        const long long i = ring_of_cap_index(p), j = p - 2 * i * (i - 1);
        *theta = 2.0 * asin((double)i / (HP_SQRT6 * ns));
        *phi = ((double)j + 0.5) * HP_HALFPI / (double)i;
    } else if (p < npix - ncap) {
        const long long q = p - ncap, i = q / (4 * N) + N, j = q % (4 * N);
        *theta = acos((2.0 * ns - (double)i) * 2.0 / (3.0 * ns));
        *phi = ((double)j + (((i + N) & 1) ? 0.0 : 0.5)) * HP_HALFPI / ns;
    } else {
        /* south cap: ring i from the south pole starts at npix - 2 i (i + 1) */
        const long long i = ring_of_cap_index(npix - 1 - p) , j = p - (npix - 2 * i * (i + 1));
        *theta = HP_PI - 2.0 * asin((double)i / (HP_SQRT6 * ns));
        *phi = ((double)j + 0.5) * HP_HALFPI / (double)i;
    }
}

/* face chart: continuous face coordinates -> (theta, phi); points slightly
 * outside [0, nside]^2 extend the chart across the face's edges */
static void xyf2ang(long long N, int f, double x, double y, double *theta, double *phi)
{
    const double ns = (double)N, jr = (face_row(f) + 2) * ns - x - y;
    double nr, t;
    if (jr < ns) {
        nr = jr;
        *theta = 2.0 * asin(jr / (HP_SQRT6 * ns));
    } else if (jr > 3.0 * ns) {
        nr = 4.0 * ns - jr;
        *theta = HP_PI - 2.0 * asin(nr / (HP_SQRT6 * ns));
    } else {
        nr = ns;
        *theta = acos((2.0 * ns - jr) * 2.0 / (3.0 * ns));
    }
    t = nr > 1e-300 ? (face_lon(f) * nr + x - y) / nr : face_lon(f);
    t = fmod(t, 8.0);
    if (t < 0.0) t += 8.0;
    *phi = t * (HP_PI / 4.0);
}

/* the inverse chart: the face holding (theta, phi) and its continuous
 * coordinates there */
static void ang2xyf(long long N, double theta, double phi, int *face, double *x, double *y)
{
    const double ns = (double)N, z = cos(theta), za = fabs(z), tt = quarter_coord(phi);
    double jr, nr, d, xpy, xmy;
    int f;
    if (za <= 2.0 / 3.0) {
        const double jp = ns * (0.5 + tt - 0.75 * z), jm = ns * (0.5 + tt + 0.75 * z);
        const int ifp = (int)floor(jp / ns), ifm = (int)floor(jm / ns);
        f = ifp == ifm ? (ifp & 3) + 4 : (ifp < ifm ? (ifp & 3) : (ifm & 3) + 8);
        jr = ns * (2.0 - 1.5 * z);
        nr = ns;
    } else {
        int q = (int)tt;
        const double s = cap_sigma(ns, theta, za);
        if (q > 3) q = 3;
        f = z > 0 ? q : q + 8;
        jr = z > 0 ? s : 4.0 * ns - s;
        nr = s;
    }
    d = 2.0 * tt - face_lon(f); /* longitude from the face centre, units of pi/4 */
    d -= 8.0 * floor((d + 4.0) / 8.0);
    xpy = (face_row(f) + 2) * ns - jr;
    xmy = d * nr;
    *face = f;
    *x = 0.5 * (xpy + xmy);
    *y = 0.5 * (xpy - xmy);
}

/* ---------------------------------------------------------------- threads */

typedef struct {
    long long N, lo, hi;
    const double *theta, *phi;
    long long *pix;
    int bad;
} a2p_job;

static void *a2p_run(void *arg)
{
    a2p_job *j = (a2p_job *)arg;
    long long i;
    for (i = j->lo; i < j->hi; i++) {
        if (j->theta[i] != j->theta[i] || j->phi[i] != j->phi[i]) {
            j->bad = 1;
            j->pix[i] = -1;
            continue;
        }
        j->pix[i] = ang2pix1(j->N, j->theta[i], j->phi[i]);
    }
    return NULL;
}

int kd_healpix_ang2pix(int nside, const double *theta, const double *phi, long long n,
                       long long *pix)
{
    enum { MAXT = 64 };
    a2p_job jobs[MAXT];
    pthread_t th[MAXT];
    int started[MAXT];
    long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    long long nt = ncpu < 1 ? 1 : (ncpu > MAXT ? MAXT : ncpu), k;
    int bad = 0;
    if (nside < 1 || nside > HP_MAX_NSIDE || n < 0 || (n > 0 && (!theta || !phi || !pix)))
        return -1;
    if (n / 65536 + 1 < nt) nt = n / 65536 + 1;
    for (k = 0; k < nt; k++) {
        jobs[k].N = nside;
        jobs[k].lo = n * k / nt;
        jobs[k].hi = n * (k + 1) / nt;
        jobs[k].theta = theta;
        jobs[k].phi = phi;
        jobs[k].pix = pix;
        jobs[k].bad = 0;
    }
    for (k = 1; k < nt; k++) started[k] = pthread_create(&th[k], NULL, a2p_run, &jobs[k]) == 0;
    a2p_run(&jobs[0]);
    for (k = 1; k < nt; k++) {
        if (started[k]) pthread_join(th[k], NULL);
        else a2p_run(&jobs[k]);
    }
    for (k = 0; k < nt; k++) bad |= jobs[k].bad;
    return bad ? -1 : 0;
}

int kd_healpix_pix2ang(int nside, const long long *pix, long long n, double *theta, double *phi)
{
    const long long N = nside, npix = 12 * N * N;
    long long i;
    if (nside < 1 || nside > HP_MAX_NSIDE || n < 0 || (n > 0 && (!pix || !theta || !phi)))
        return -1;
    for (i = 0; i < n; i++)
        if (pix[i] < 0 || pix[i] >= npix) return -1;
    for (i = 0; i < n; i++) pix2ang1(N, pix[i], theta + i, phi + i);
    return 0;
}

int kd_healpix_edge_neighbours(int nside, long long *nb)
{
    /* south-west, north-west, north-east, south-east in face coordinates */
    static const int dx[4] = {-1, 0, 1, 0}, dy[4] = {0, 1, 0, -1};
    /* how far past the edge midpoint the probe goes, in pixels: well inside
     * the neighbour, far from its other edges */
    const double past = 0.52;
    const long long N = nside, npix = 12 * N * N;
    long long p;
    if (nside < 1 || nside > HP_MAX_NSIDE || !nb) return -1;
    for (p = 0; p < npix; p++) {
        double th, ph, x, y;
        int f, k;
        pix2ang1(N, p, &th, &ph);
        ang2xyf(N, th, ph, &f, &x, &y);
        x = floor(x) + 0.5; /* the centre, exactly */
        y = floor(y) + 0.5;
        for (k = 0; k < 4; k++) {
            double t2, p2;
            xyf2ang(N, f, x + dx[k] * past, y + dy[k] * past, &t2, &p2);
            nb[4 * p + k] = ang2pix1(N, t2, p2);
        }
    }
    return 0;
}

int kd_healpix_corners(int nside, long long pix, double *xyz)
{
    /* north (+x +y), west (+y), south, east (+x) corners of the pixel */
    static const double cx[4] = {1, 0, 0, 1}, cy[4] = {1, 1, 0, 0};
    const long long N = nside;
    double th, ph, x, y;
    int f, k;
    if (nside < 1 || nside > HP_MAX_NSIDE || pix < 0 || pix >= 12 * N * N || !xyz) return -1;
    pix2ang1(N, pix, &th, &ph);
    ang2xyf(N, th, ph, &f, &x, &y);
    x = floor(x);
    y = floor(y);
    for (k = 0; k < 4; k++) {
        double t2, p2;
        xyf2ang(N, f, x + cx[k], y + cy[k], &t2, &p2);
        xyz[3 * k] = sin(t2) * cos(p2);
        xyz[3 * k + 1] = sin(t2) * sin(p2);
        xyz[3 * k + 2] = cos(t2);
    }
    return 0;
}

/* ---------------------------------------------------------------- partition */

typedef struct {
    int nv;
    const int *xadj, *adjncy;
    const long long *vw, *ew;
    int *mark;     /* vertex -> generation of the subset it belongs to */
    int gen;
    char *side;    /* 0 / 1 during a bisection; 2 = not yet placed */
    long long *gain; /* refinement: cut weight saved by moving the vertex */
    int *queue;
    int *dist;
} pgraph;

/* cut weight of the subset's bisection (each cut edge once) */
static long long cut_weight(const pgraph *g, const int *vs, int n)
{
    long long c = 0;
    int i, e;
    for (i = 0; i < n; i++) {
        const int v = vs[i];
        for (e = g->xadj[v]; e < g->xadj[v + 1]; e++) {
            const int u = g->adjncy[e];
            if (u > v && g->mark[u] == g->gen && g->side[u] != g->side[v]) c += g->ew[e];
        }
    }
    return c;
}

/* breadth-first distances inside the subset from src; returns the last
 * vertex reached (a peripheral one) */
static int bfs_far(pgraph *g, int src)
{
    int head = 0, tail = 0, last = src, e;
    g->queue[tail++] = src;
    g->dist[src] = 0;
    while (head < tail) {
        const int v = g->queue[head++];
        last = v;
        for (e = g->xadj[v]; e < g->xadj[v + 1]; e++) {
            const int u = g->adjncy[e];
            if (g->mark[u] == g->gen && g->dist[u] < 0) {
                g->dist[u] = g->dist[v] + 1;
                g->queue[tail++] = u;
            }
        }
    }
    return last;
}

/* gain of moving v to side 0: edge weight to side-0 vertices minus edge
 * weight to the others (inside the subset) */
static long long gain_to0(const pgraph *g, int v)
{
    long long s = 0;
    int e;
    for (e = g->xadj[v]; e < g->xadj[v + 1]; e++) {
        const int u = g->adjncy[e];
        if (g->mark[u] != g->gen || u == v) continue;
        s += g->side[u] == 0 ? g->ew[e] : -g->ew[e];
    }
    return s;
}

/* grow side 0 from seed until it holds target weight: repeatedly add the
 * frontier vertex with the largest gain (the most edge weight into side 0),
 * restarting from an unplaced vertex when a component is exhausted */
static void grow(pgraph *g, const int *vs, int n, int seed, long long target)
{
    long long w0 = 0;
    int i, e, nfront = 0;
    int *front = g->queue; /* frontier list */
    for (i = 0; i < n; i++) g->side[vs[i]] = 2;
    g->side[seed] = 0;
    w0 = g->vw[seed];
    for (e = g->xadj[seed]; e < g->xadj[seed + 1]; e++) {
        const int u = g->adjncy[e];
        if (g->mark[u] == g->gen && g->side[u] == 2 && g->dist[u] != -2) {
            g->dist[u] = -2; /* on the frontier */
            front[nfront++] = u;
        }
    }
    while (w0 < target) {
        int best = -1, bi = -1;
        long long bg = 0;
        if (nfront == 0) {
            for (i = 0; i < n; i++)
                if (g->side[vs[i]] == 2) break;
            if (i == n) break;
            front[nfront++] = vs[i];
            g->dist[vs[i]] = -2;
        }
        for (i = 0; i < nfront; i++) {
            const int v = front[i];
            long long gv = 0;
            for (e = g->xadj[v]; e < g->xadj[v + 1]; e++) {
                const int u = g->adjncy[e];
                if (g->mark[u] != g->gen) continue;
                gv += g->side[u] == 0 ? g->ew[e] : -g->ew[e];
            }
            /* prefer overshooting the target least when gains tie */
            if (best < 0 || gv > bg || (gv == bg && g->vw[v] < g->vw[best])) {
                best = v;
                bg = gv;
                bi = i;
            }
        }
        front[bi] = front[--nfront];
        g->side[best] = 0;
        w0 += g->vw[best];
        for (e = g->xadj[best]; e < g->xadj[best + 1]; e++) {
            const int u = g->adjncy[e];
            if (g->mark[u] == g->gen && g->side[u] == 2 && g->dist[u] != -2) {
                g->dist[u] = -2;
                front[nfront++] = u;
            }
        }
    }
    for (i = 0; i < n; i++) {
        if (g->side[vs[i]] == 2) g->side[vs[i]] = 1;
        g->dist[vs[i]] = -1;
    }
}

/* boundary refinement (Fiduccia-Mattheyses passes): in each pass every
 * vertex may move once, always the unlocked one with the largest gain among
 * the moves that keep side 0's weight within tol of the target (or bring it
 * closer); negative gains are allowed so that the pass can climb out of a
 * local minimum, and the pass is rolled back to its best prefix */
static void refine(pgraph *g, const int *vs, int n, long long target, long long tol)
{
    long long w0 = 0;
    int i, e, pass;
    int *moved = (int *)malloc(sizeof(int) * (size_t)n);
    char *lock = (char *)calloc((size_t)n, 1);
    int *idx = g->queue + n; /* vertex -> position in vs (second half of queue) */
    if (!moved || !lock) {
        free(moved);
        free(lock);
        return;
    }
    for (i = 0; i < n; i++) {
        idx[vs[i]] = i;
        if (g->side[vs[i]] == 0) w0 += g->vw[vs[i]];
    }
    for (pass = 0; pass < 6; pass++) {
        long long cut_delta = 0, best_delta = 0, best_dev = llabs(w0 - target);
        int nm = 0, best_nm = 0, since_best = 0;
        memset(lock, 0, (size_t)n);
        for (i = 0; i < n; i++) g->gain[vs[i]] = 0;
        for (i = 0; i < n; i++) {
            const int v = vs[i];
            const long long g0 = gain_to0(g, v);
            g->gain[v] = g->side[v] == 0 ? -g0 : g0;
        }
        while (nm < n && since_best < 64) {
            int best = -1;
            long long bg = 0, bw0 = 0;
            for (i = 0; i < n; i++) {
                const int v = vs[i];
                long long nw0, dn;
                if (lock[i]) continue;
                nw0 = g->side[v] == 0 ? w0 - g->vw[v] : w0 + g->vw[v];
                dn = llabs(nw0 - target);
                if (dn > tol && dn >= llabs(w0 - target)) continue;
                if (best < 0 || g->gain[v] > bg) {
                    best = v;
                    bg = g->gain[v];
                    bw0 = nw0;
                }
            }
            if (best < 0) break;
            /* move it and update the gains of its neighbours */
            g->side[best] ^= 1;
            lock[idx[best]] = 1;
            w0 = bw0;
            cut_delta -= bg;
            g->gain[best] = -bg;
            for (e = g->xadj[best]; e < g->xadj[best + 1]; e++) {
                const int u = g->adjncy[e];
                if (g->mark[u] != g->gen || u == best) continue;
                /* the edge (u, best) was cut iff sides differed */
                g->gain[u] += g->side[u] == g->side[best] ? -2 * g->ew[e] : 2 * g->ew[e];
            }
            moved[nm++] = best;
            {
                const long long dev = llabs(w0 - target);
                const int ok = dev <= tol || dev < best_dev;
                if (ok && (cut_delta < best_delta || (cut_delta == best_delta && dev < best_dev))) {
                    best_delta = cut_delta;
                    best_dev = dev;
                    best_nm = nm;
                    since_best = 0;
                } else {
                    since_best++;
                }
            }
        }
        /* roll back the moves after the best prefix */
        while (nm > best_nm) {
            const int v = moved[--nm];
            g->side[v] ^= 1;
            w0 += g->side[v] == 0 ? g->vw[v] : -g->vw[v];
        }
        if (best_nm == 0) break;
    }
    free(moved);
    free(lock);
}

static void bisect(pgraph *g, const int *vs, int n, long long target, long long tol)
{
    /* a few growths from peripheral seeds; keep the least cut within the
     * balance, refined */
    char *best = (char *)malloc((size_t)n);
    long long bestc = -1, bestdev = 0;
    int trial, i, seed = vs[0];
    for (i = 0; i < n; i++) g->dist[vs[i]] = -1;
    for (trial = 0; trial < 4 && best; trial++) {
        long long w0 = 0, c, dev;
        int far;
        for (i = 0; i < n; i++) g->dist[vs[i]] = -1;
        far = bfs_far(g, seed);
        for (i = 0; i < n; i++) g->dist[vs[i]] = -1;
        grow(g, vs, n, far, target);
        refine(g, vs, n, target, tol);
        for (i = 0; i < n; i++)
            if (g->side[vs[i]] == 0) w0 += g->vw[vs[i]];
        c = cut_weight(g, vs, n);
        dev = llabs(w0 - target);
        if (bestc < 0 || (dev <= tol && (bestdev > tol || c < bestc)) ||
            (dev > tol && bestdev > tol && dev < bestdev)) {
            bestc = c;
            bestdev = dev;
            for (i = 0; i < n; i++) best[i] = g->side[vs[i]];
        }
        seed = vs[(int)(((long long)(trial + 1) * n) / 4) % n];
    }
    if (best) {
        for (i = 0; i < n; i++) g->side[vs[i]] = best[i];
        free(best);
    }
}

static void rec_part(pgraph *g, int *vs, int n, int nparts, int first, int *part, int *tmp)
{
    long long W = 0, vmax = 0, target, tol;
    int i, n0 = 0, k1;
    if (nparts <= 1 || n <= 1) {
        for (i = 0; i < n; i++) part[vs[i]] = first;
        return;
    }
    k1 = nparts / 2;
    g->gen++;
    for (i = 0; i < n; i++) {
        g->mark[vs[i]] = g->gen;
        W += g->vw[vs[i]];
        if (g->vw[vs[i]] > vmax) vmax = g->vw[vs[i]];
    }
    target = (long long)((double)W * k1 / nparts + 0.5);
    tol = W / 100 > vmax ? W / 100 : vmax;
    bisect(g, vs, n, target, tol);
    /* stable split of vs into side 0, then side 1 */
    for (i = 0; i < n; i++)
        if (g->side[vs[i]] == 0) tmp[n0++] = vs[i];
    {
        int m = n0;
        for (i = 0; i < n; i++)
            if (g->side[vs[i]] != 0) tmp[m++] = vs[i];
    }
    memcpy(vs, tmp, sizeof(int) * (size_t)n);
    rec_part(g, vs, n0, k1, first, part, tmp);
    rec_part(g, vs + n0, n - n0, nparts - k1, first + k1, part, tmp);
}

long long kd_partition_graph(int nv, const int *xadj, const int *adjncy, const long long *vwgt,
                             const long long *ewgt, int nparts, int *part)
{
    pgraph g;
    int *vs, *tmp, i, e;
    long long cut = 0;
    if (nv < 1 || nparts < 1 || !xadj || !adjncy || !vwgt || !ewgt || !part) return -1;
    for (i = 0; i < nv; i++) {
        if (xadj[i + 1] < xadj[i] || vwgt[i] < 0) return -1;
        for (e = xadj[i]; e < xadj[i + 1]; e++)
            if (adjncy[e] < 0 || adjncy[e] >= nv || ewgt[e] < 0) return -1;
    }
    memset(&g, 0, sizeof g);
    g.nv = nv;
    g.xadj = xadj;
    g.adjncy = adjncy;
    g.vw = vwgt;
    g.ew = ewgt;
    g.mark = (int *)calloc((size_t)nv, sizeof(int));
    g.side = (char *)calloc((size_t)nv, 1);
    g.queue = (int *)malloc(sizeof(int) * (size_t)nv * 2 + 16);
    g.dist = (int *)malloc(sizeof(int) * (size_t)nv);
    g.gain = (long long *)malloc(sizeof(long long) * (size_t)nv);
    vs = (int *)malloc(sizeof(int) * (size_t)nv);
    tmp = (int *)malloc(sizeof(int) * (size_t)nv);
    if (!g.mark || !g.side || !g.queue || !g.dist || !g.gain || !vs || !tmp) {
        cut = -1;
        goto done;
    }
    for (i = 0; i < nv; i++) {
        vs[i] = i;
        g.dist[i] = -1;
    }
    rec_part(&g, vs, nv, nparts, 0, part, tmp);
    for (i = 0; i < nv; i++)
        for (e = xadj[i]; e < xadj[i + 1]; e++)
            if (adjncy[e] > i && part[adjncy[e]] != part[i]) cut += ewgt[e];
done:
    free(g.mark);
    free(g.side);
    free(g.queue);
    free(g.dist);
    free(g.gain);
    free(vs);
    free(tmp);
    return cut;
}
