/*
 * corruscant-b200: C ABI of the GPU pair-counting library (libkdtree.so).
 *
 * The first part is the reference's ABI, kept binary compatible so that the
 * reference's ctypes layer (corruscant/clustering.py:30-71) and C callers bind
 * unchanged.  The types have the reference's field order, widths and bitfield
 * layout (src/kdtree.h:11-41): a kdtree_t is 64 bytes, a node_t 40 bytes, and
 * node_data is a host array of memsize nodes in heap order (root at index 1,
 * children of p at 2p and 2p+1, empty slots all zero).
 *
 * The second part (kd_*) is additive: batched multi-radius counts, error
 * reporting and resource management the reference lacks.
 *
 * All entry points are reentrant: each call uses its own CUDA stream.  On the
 * GPU the library needs a CUDA device of compute capability 10.0 (B200); there
 * is no CPU fallback.
 */
#ifndef CORRUSCANT_B200_KDTREE_H
#define CORRUSCANT_B200_KDTREE_H

#ifdef __cplusplus
extern "C" {
#endif

#define NDIM 3

/* src/kdtree.h:13-17: a point; field and weight are 8-bit */
typedef struct datum {
    double value[NDIM];
    unsigned int field:8;
    unsigned int weight:8;
} datum_t;

/* src/kdtree.h:19-25: a heap node holding one point */
typedef struct node {
    datum_t data;
    unsigned int has_lchild:1;
    unsigned int has_rchild:1;
    unsigned int dim:8;
} node_t;

/* src/kdtree.h:27-31 (kept for source compatibility; unused by the ABI) */
typedef struct field_counter {
    long long total;
    long long *array;
    int num_fields;
} field_counter_t;

/* src/kdtree.h:33-41.  size = unique points; data, fields and args are NULL
 * (the reference frees them before returning, kdbuild.c:530-534). */
typedef struct kdtree {
    node_t *node_data;
    int size;
    int memsize;
    int num_fields;
    datum_t *data;
    int *fields;
    int *args[NDIM];
} kdtree_t;

/* ---------------------------------------------------------------- reference ABI */

/* Replaces tree_construct (src/kdtree.h:43, src/kdbuild.c:451-537).
 * xyz: n interleaved (x,y,z) doubles; fields: n ints or NULL; the tree stores
 * the low 8 bits of a field, like the reference's field:8.  Duplicated points
 * are merged into one node whose weight counts them and whose field is the
 * field of the first occurrence.  The node array is bit-identical in its
 * semantic fields to the reference build's.
 * On error (NaN coordinate, a point repeated 256+ times, n < 1, no device)
 * returns a tree with node_data == NULL and size == 0; kd_last_error() says
 * why.  The reference prints and exits in these cases (kdbuild.c:73-79,
 * :508-511). */
kdtree_t tree_construct(double *xyz, int *fields, int length, int num_fields);

/* Replaces pair_count (src/kdtree.h:45, src/kdquery.c:165-249).
 * Counts, for the `length` query points (interleaved xyz, NaN rows count
 * nothing), the tree points within distance r: fl(d2) < fl(r*r) with d2
 * evaluated in the reference's operation order, weighted by node weight.
 * Returns a malloc'd array of num_fields * tree.num_fields counts, indexed
 * qfield * num_fields + tfield as in kdquery.c:34 (free with kd_free_counts
 * or free()).  num_threads is accepted and ignored.  Returns NULL on error:
 * negative r (the reference's prune is undefined there), negative query
 * fields, field ids that would index outside the array, or a device error. */
long long *pair_count(kdtree_t tree, double *data, int *fields, int length,
                      int num_fields, double r, int num_threads);

/* Replaces destroy (src/kdbuild.c:303-306): releases the host node array and
 * the tree's device memory. */
void destroy(kdtree_t tree);

/* ---------------------------------------------------------------- additions */

#define KD_MODE_MIXED 0 /* FP32 distances + FP64 recheck near edges (default) */
#define KD_MODE_FP64 1  /* every distance in FP64 */

/* Status codes: 0 or negative.  Where the reference prints and exits
 * (kdbuild.c:73-79, :234-239, :508-511; kdquery.c:176-179) these calls
 * return a code, and kd_last_error() holds the message. */
#define KD_OK 0
#define KD_EINVAL -1      /* bad argument: count, pointer, mode, shard, handle */
#define KD_ENOMEM -2      /* host or device memory exhausted */
#define KD_EDUP -3        /* >= 256 copies of one point (weight:8 would wrap) */
#define KD_ENAN -4        /* NaN coordinate in a tree */
#define KD_EFIELD -5      /* field counts or ids do not fit the qfield*Fq + tfield counter */
#define KD_ECUDA -6       /* a CUDA call failed */
#define KD_ENODEV -7      /* no usable CUDA device */
#define KD_EINTERNAL -8   /* a device-side bound was hit (stack, sizes) */
#define KD_ERADIUS -9     /* negative radius (the reference's pruning is not defined there) */

/* Largest catalog, raw points (duplicates included): the node heap of
 * 2^(floor(log2 n) + 1) entries is indexed by int, as in the reference. */
#define KD_MAX_POINTS 1073741823

typedef struct kd_count_stats {
    long long pairs_tested;    /* distances evaluated in tiles */
    long long pairs_rechecked; /* pairs recomputed in FP64 after an FP32 band hit */
    long long pairs_accepted;  /* pairs binned by whole node pairs, no distance */
    long long pairs_wide;      /* pairs of tiles spanning more than 4 edges */
    long long edge_pairs;      /* sum over tested pairs of the edges each was binned against */
    long long warp_tiles;      /* (query block, tree run) tiles with distances computed */
    long long entries;         /* (query block, tree run) tiles listed */
    double ms_traverse;        /* device time: node-pair traversal */
    double ms_tiles;           /* device time: tile kernels */
    double ms_total;           /* device time: whole count */
    int tile_launches;
    int launches;              /* kernel launches of the count */
    long long pairs_one_bin_multifield; /* tested pairs of node pairs lying inside one
                                         * bin, tiled because a side holds several fields */
} kd_count_stats;

/* Where a tree_construct call spent its time (no counterpart in the
 * reference): device time of the build's phases, measured with events on
 * the build's stream, and host wall time of the whole call. */
typedef struct kd_build_stats {
    double ms_prep;       /* device: points to the device, keys, NaN check */
    double ms_dedup;      /* device: lexicographic sort, duplicate classes */
    double ms_argsort;    /* device: the two superkey orders */
    double ms_levels;     /* device: the level-by-level tree build */
    double ms_layout;     /* device: counting layout, runs, blocks, summaries */
    double ms_device;     /* device: first to last event of the build */
    double ms_node_copy;  /* host: node array to the returned host array, wall,
                           * from the start of the level loop (the copy follows
                           * the levels as they are built, then overlaps the
                           * counting layout) */
    double ms_node_wait;  /* host: how long the build then waited for that copy */
    double ms_total_host; /* host: the whole tree_construct call, wall */
    int levels;           /* tree levels built */
    int n_unique;         /* unique points */
} kd_build_stats;

/* Timing of the build that made `tree`.  Returns 0 or KD_EINVAL.  For a
 * deferred build (kd_tree_construct_deferred) ms_node_copy and ms_node_wait
 * are filled in by kd_tree_wait_nodes (0 until then) and ms_total_host is the
 * time until the construct call returned. */
int kd_tree_build_stats(kdtree_t tree, kd_build_stats *stats);

/* tree_construct (src/kdbuild.c:451-537) that returns before its node array
 * is complete: once the tree is built on the device, while a host thread is
 * still copying the node array into node_data.  The tree may be counted at
 * once (every kd_count_* entry point and pair_count read only the device
 * copy), which lets the count run while the 40-byte-per-slot node array
 * (1.3 GB at 20M points) drains to the host.  node_data must not be read
 * before kd_tree_wait_nodes has returned 0.  destroy waits for the copy
 * itself.  Errors of the build are returned as tree_construct returns them;
 * an error of the copy is returned by kd_tree_wait_nodes. */
kdtree_t kd_tree_construct_deferred(double *xyz, int *fields, int length, int num_fields);

/* Waits until the node array of `tree` is complete.  Returns 0 (at once for
 * a tree from tree_construct, or one already waited for), the copy's error
 * code with kd_last_error set, or KD_EINVAL for a tree that is not live. */
int kd_tree_wait_nodes(kdtree_t tree);

/* Last error of the calling thread: returns its code (0 = none) and copies
 * the message into buf (may be NULL). */
int kd_last_error(char *buf, int len);

/* Selects how pair_count counts on the calling thread: KD_MODE_MIXED (FP32
 * with exact FP64 rechecks near every edge, the default) or KD_MODE_FP64
 * (every distance in FP64).  Both give the reference's counts exactly.  The
 * reference's pair_count (src/kdquery.c:165) has no precision argument; this
 * keeps its signature unchanged.  Returns 0 or KD_EINVAL. */
int kd_set_precision(int mode);

/* Frees an array returned by pair_count. */
void kd_free_counts(long long *counts);

/* Multi-radius count with another tree's points as the queries (its raw
 * input points, duplicates included, each with its own field): for every
 * radius k, out[k*Fq*Ft + qf*Fq + tf] is what pair_count(tree,
 * query_points, query_fields, n, Fq, radii[k], .) returns, with
 * Fq = query.num_fields and Ft = tree.num_fields.  Any number of radii, in
 * any order, repeats and NaN included: up to 64 distinct squared radii are
 * counted in one pass over the node pairs, more in passes of 64 over the
 * same trees.  Replaces the per-edge pair_count loop of
 * clustering.py:218-230, :256-284.  mode: KD_MODE_MIXED or KD_MODE_FP64.
 * stats may be NULL.  Returns 0 or a negative error code. */
int kd_count_radii(kdtree_t tree, kdtree_t query, const double *radii,
                   int nradii, int mode, long long *out, kd_count_stats *stats);

/* One shard of kd_count_radii: only the query points of this shard's query
 * blocks are counted (the query tree's blocks of up to 128 spatially
 * adjacent points, taken in interleaved chunks of 32: chunk c belongs to
 * shard c mod nshards, which spreads early and late blocks evenly).  Summing
 * out over all shards gives kd_count_radii's result exactly; one shard per
 * GPU splits a count across devices with no exchange until that final sum. */
int kd_count_radii_shard(kdtree_t tree, kdtree_t query, const double *radii,
                         int nradii, int mode, int shard, int nshards,
                         long long *out, kd_count_stats *stats);

/* Per-bin counts: out[k*Fq*Ft + qf*Fq + tf] = (count at edges[k+1]) -
 * (count at edges[k]) for k = 0 .. nedges-2, exactly what the reference's
 * drivers compute with np.diff over one pair_count per edge
 * (clustering.py:218-230).  Edges in the caller's order (ascending for
 * ordinary bins).  Returns 0 or a negative error code. */
int kd_count_bins(kdtree_t tree, kdtree_t query, const double *edges, int nedges,
                  int mode, long long *out, kd_count_stats *stats);

/* kd_count_radii for njobs (trees[j], queries[j]) pairs sharing the radii
 * and mode, e.g. DD, DR and RR of an autocorrelation (clustering.py:218-230)
 * or the counts of many catalogs against one random catalog.  The query
 * blocks of all jobs are numbered consecutively and counted by one node-pair
 * traversal and one persistent tile launch over a shared work queue, so small
 * jobs do not each pay for launches and an underfilled GPU.  out receives,
 * job after job, each job's kd_count_radii result: nradii * Fq_j * Ft_j
 * counts (Fq_j = queries[j].num_fields, Ft_j = trees[j].num_fields).  stats
 * (may be NULL) totals the batch. */
int kd_count_batch(const kdtree_t *trees, const kdtree_t *queries, int njobs,
                   const double *radii, int nradii, int mode, long long *out,
                   kd_count_stats *stats);

/* One shard of kd_count_batch: the batch's query blocks (numbered job after
 * job) split into interleaved chunks of 32 as in kd_count_radii_shard.
 * Summing out over all shards gives kd_count_batch's result exactly. */
int kd_count_batch_shard(const kdtree_t *trees, const kdtree_t *queries, int njobs,
                         const double *radii, int nradii, int mode, int shard,
                         int nshards, long long *out, kd_count_stats *stats);

/* kd_count_radii for callers that cannot allocate device memory while they
 * count: a service whose device memory is owned by a fixed-budget pool, a
 * host that forbids cudaMalloc because it synchronizes the whole device and
 * would stall its other streams, or code that must not grow the process's
 * footprint mid-run.  No counterpart in the reference (which has no device
 * code).  Same inputs and output as kd_count_radii (trees from
 * tree_construct, host radii, host out array of nradii * Fq * Ft counts),
 * identical counts, no statistics.
 *
 * It allocates nothing, host or device, and creates no stream or event: its
 * buffers come from one fixed 32 MiB array in device memory that every GPU
 * holding the library keeps until the process exits; it runs on the legacy
 * default stream and returns when the counts are on the host.  Limits: at
 * most 64 radii; the bin histogram ((distinct radii + 1) x (max query field
 * + 1) x (max tree field + 1) x 8 bytes) plus 16 bytes per query block of up
 * to 128 points must leave room for tile records, and a single query block's
 * tile records must fit (a clear error otherwise); larger jobs run in more
 * batches, so this is slower than kd_count_radii.  The first call on a
 * device looks up the array's device address (keep that first call outside
 * any stream capture) and keeps it for the life of the process: a caller
 * that resets the device (cudaDeviceReset through this library's runtime)
 * must not call this entry point afterwards.  All calls share the array and
 * its contents persist between calls; each call clears what it needs, but
 * calls that overlap on the same GPU (other threads) race and must be
 * serialised by the caller. */
int kd_count_radii_static(kdtree_t tree, kdtree_t query, const double *radii,
                          int nradii, int mode, long long *out);

/* Same, with arbitrary query points (interleaved xyz, fields may be NULL). */
int kd_count_points(kdtree_t tree, const double *xyz, const int *fields,
                    int length, int num_fields, const double *radii,
                    int nradii, int mode, long long *out,
                    kd_count_stats *stats);

/* In-order permutation of the tree: perm[i] = index, in the input array
 * given to tree_construct, of the (first occurrence of the) point stored at
 * in-order position i.  perm holds tree.size ints. */
int kd_tree_permutation(kdtree_t tree, int *perm);

/* Selects the CUDA device used by later tree_construct calls of the calling
 * thread (default 0; the library has its own CUDA runtime, so a device
 * selected through another library does not apply).  Counts always run on
 * the device holding their trees.  Returns 0 or a negative error code. */
int kd_set_device(int device);

/* Raw (input) point count of a tree, duplicates included. */
int kd_tree_input_size(kdtree_t tree);

#ifdef __cplusplus
}
#endif
#endif
