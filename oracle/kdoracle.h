/*
 * CPU oracle for the corruscant pair-counting path.  TEST INFRASTRUCTURE ONLY:
 * the tests, the smoke check and the benchmark's CPU-baseline leg use it as the
 * checker; the product library never links, loads or calls it.
 *
 * It restates, in plain C, the reference algorithm:
 *   - tree build     : src/kdbuild.c:451-537 (dedup, superkey argsorts, median
 *                      build with max-variance split, kdbuild.c:308-433)
 *   - radius count   : src/kdquery.c:62-113 (single-tree traversal, strict <)
 *   - coordinates    : src/coordmath.c:38-80
 * plus an exhaustive FP64 brute-force bin counter that uses the reference's
 * distance operation order (kdquery.c:39-47 as compiled: fused multiply-adds).
 *
 * Parity is pinned against the reference itself, compiled from its sources by
 * oracle/Makefile into oracle/_ref/ (see tests/test_oracle_pin.py), and against
 * golden vectors generated from that build (tests/golden/).
 */
#ifndef KDORACLE_H
#define KDORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_tree or_tree_t;

/* error codes (negative) */
#define OR_OK 0
#define OR_EINVAL -1
#define OR_ENOMEM -2
#define OR_EDUP_OVERFLOW -3 /* >= 256 copies of one point: reference weight:8 wraps */
#define OR_ENAN -4
#define OR_EFIELD -5

const char *or_last_error(void);

/* Build.  xyz interleaved (n,3); fields may be NULL. */
int or_build(const double *xyz, const int *fields, int n, int num_fields,
             or_tree_t **out);
void or_free(or_tree_t *t);

int or_tree_size(const or_tree_t *t);     /* unique points */
int or_tree_memsize(const or_tree_t *t);  /* node array length */
int or_tree_num_fields(const or_tree_t *t);

/* Node array, semantic fields only, length memsize each (xyz: memsize*3).
 * Empty heap slots are all zero, like the reference's calloc'd array. */
void or_tree_nodes(const or_tree_t *t, double *xyz, int *field, int *weight,
                   int *has_l, int *has_r, int *dim);
/* In-order permutation: entry i = index (into the input array) of the
 * representative raw point stored at in-order position i. */
void or_tree_inorder(const or_tree_t *t, int *perm);
/* Unique points in dedup (lexicographic) order. */
void or_tree_unique(const or_tree_t *t, double *xyz, int *field, int *weight,
                    int *rep_index);

/* Reference-style count for one radius: out[qf*Fq + tf] (the reference's
 * counter indexing, kdquery.c:34).  visits (may be NULL) receives the number
 * of node distance evaluations the traversal performed. */
int or_pair_count(const or_tree_t *t, const double *q, const int *qfields,
                  int nq, int num_fields_q, double r, int nthreads,
                  long long *out, long long *visits);

/* Exhaustive FP64 count for many radii at once (any order, duplicates
 * allowed): out[k*Fq*Ft + qf*Fq + tf] = #{(q,t): fl(d2) < fl(r_k*r_k)}
 * weighted by the tree multiplicity. */
int or_brute_counts(const or_tree_t *t, const double *q, const int *qfields,
                    int nq, int num_fields_q, const double *radii, int nradii,
                    int nthreads, long long *out);

/* or_brute_counts' result from the reference traversal (kdquery.c:62-113)
 * run at the largest finite radius, every visited node's distance binned
 * into all radii: the same exhaustive counts, far fewer distances.  Falls
 * back to the exhaustive loop when a squared radius is +inf. */
int or_tree_counts(const or_tree_t *t, const double *q, const int *qfields,
                   int nq, int num_fields_q, const double *radii, int nradii,
                   int nthreads, long long *out);

/* Node distance evaluations the reference traversal (kdquery.c:62-113)
 * performs for nq queries at radius r, over a node array given by its
 * semantic fields (memsize entries; xyz interleaved).  This is the CPU
 * path's "pairs tested" count. */
long long or_count_visits(const double *nxyz, const int *has_l, const int *has_r,
                          const int *dim, int memsize, const double *q, int nq,
                          double r, int nthreads);

void or_radec2cart64(const double *ra, const double *dec, double *xyz, int n);
void or_radecdist2cart64(const double *ra, const double *dec,
                         const double *dist, double *xyz, int n);
void or_radec2sph64(const double *ra, const double *dec, double *theta,
                    double *phi, int n);

#ifdef __cplusplus
}
#endif
#endif
