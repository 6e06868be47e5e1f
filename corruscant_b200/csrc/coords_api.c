/*
 * libcoords.so: RA/DEC conversions of the reference's src/coordmath.c,
 * element by element identical (same libm functions, same operation order:
 * angle = deg * (M_PI / 180.0), products evaluated left to right), split
 * across host threads for large inputs.  See include/coordmath.h for why
 * these stay on the host.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <unistd.h>

#include "coordmath.h"

#define DEG2RAD (M_PI / 180.0) /* the reference's PI_OVER_180, coordmath.c:20 */
#define MIN_PER_THREAD 65536
#define MAX_THREADS 64

typedef struct {
    const double *ra, *dec, *dist;
    double *out0, *out1;
    int lo, hi, kind;
} job_t;

static void run_range(const job_t *j)
{
    int i;
    if (j->kind == 0) {
        for (i = j->lo; i < j->hi; i++) {
            double lon = j->ra[i] * DEG2RAD, lat = j->dec[i] * DEG2RAD;
            double c = cos(lat);
            j->out0[3 * (size_t)i] = c * cos(lon);
            j->out0[3 * (size_t)i + 1] = c * sin(lon);
            j->out0[3 * (size_t)i + 2] = sin(lat);
        }
    } else if (j->kind == 1) {
        for (i = j->lo; i < j->hi; i++) {
            double lon = j->ra[i] * DEG2RAD, lat = j->dec[i] * DEG2RAD;
            double c = cos(lat);
            j->out0[3 * (size_t)i] = j->dist[i] * c * cos(lon);
            j->out0[3 * (size_t)i + 1] = j->dist[i] * c * sin(lon);
            j->out0[3 * (size_t)i + 2] = j->dist[i] * sin(lat);
        }
    } else {
        for (i = j->lo; i < j->hi; i++) {
            j->out0[i] = (90.0 - j->dec[i]) * DEG2RAD;
            j->out1[i] = j->ra[i] * DEG2RAD;
        }
    }
}

static void *worker(void *arg)
{
    run_range((const job_t *)arg);
    return NULL;
}

static void run(const double *ra, const double *dec, const double *dist, double *o0,
                double *o1, int n, int kind)
{
    job_t jobs[MAX_THREADS];
    pthread_t th[MAX_THREADS];
    long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    int nt = (int)(ncpu < 1 ? 1 : (ncpu > MAX_THREADS ? MAX_THREADS : ncpu));
    int k, started[MAX_THREADS];
    if (n <= 0) return;
    if (n / MIN_PER_THREAD + 1 < nt) nt = n / MIN_PER_THREAD + 1;
    for (k = 0; k < nt; k++) {
        jobs[k].ra = ra;
        jobs[k].dec = dec;
        jobs[k].dist = dist;
        jobs[k].out0 = o0;
        jobs[k].out1 = o1;
        jobs[k].lo = (int)((long long)n * k / nt);
        jobs[k].hi = (int)((long long)n * (k + 1) / nt);
        jobs[k].kind = kind;
    }
    for (k = 1; k < nt; k++) started[k] = pthread_create(&th[k], NULL, worker, &jobs[k]) == 0;
    run_range(&jobs[0]);
    for (k = 1; k < nt; k++) {
        if (started[k]) pthread_join(th[k], NULL);
        else run_range(&jobs[k]);
    }
}

void radec2cart64(double *ra, double *dec, double *xyz, int n)
{
    run(ra, dec, NULL, xyz, NULL, n, 0);
}

void radecdist2cart64(double *ra, double *dec, double *dist, double *xyz, int n)
{
    run(ra, dec, dist, xyz, NULL, n, 1);
}

void radec2sph64(double *ra, double *dec, double *theta, double *phi, int n)
{
    run(ra, dec, NULL, theta, phi, n, 2);
}
