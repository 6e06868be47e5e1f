/*
 * Internal interface between the C host library (kd_api.c) and the CUDA
 * translation units (kd_build.cu, kd_count.cu).  Plain C types only.
 *
 * A "catalog" is everything the GPU keeps for one tree_construct() call:
 *   - the reference-exact k-d tree (node_t array, heap order, root at 1) that
 *     kdbuild.c:451-537 would produce, plus its in-order permutation;
 *   - a counting layout of the RAW input points (duplicates kept, one entry
 *     each) ordered leaf by leaf along the top D levels of that same tree, with
 *     per-node bounding boxes, raw counts and single-field summaries, split
 *     into "runs" (<= KD_RUN_MAX consecutive points of one tree-side field) and
 *     "blocks" (<= KD_BLOCK_MAX consecutive points of one 16-leaf subtree,
 *     the query side of a tile).
 *
 * Every raw point carries two field ids: qf, its own field (what the
 * reference's query side reads, kdquery.c:67-70), and tf, the low 8 bits of
 * the field of the FIRST input occurrence of its coordinates (what the
 * reference's deduplicated tree node stores, kdbuild.c:472-499, kdtree.h:15).
 * Counting raw tree points with tf and weight 1 is identical to counting the
 * reference's unique nodes with their weight.
 */
#ifndef KD_INTERNAL_H
#define KD_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "kdtree.h" /* public ABI: node_t, kd_count_stats, KD_MODE_* */

#ifdef __cplusplus
extern "C" {
#endif

#define KD_RUN_MAX 64      /* points per tree-side run (shared-memory tile) */
#define KD_BLOCK_MAX 128   /* query points per block (one warp, 4 per lane) */
#define KD_QPL 4           /* query points per lane */
#define KD_LEAF_TARGET 64  /* unique points per counting leaf, upper bound */
#define KD_MAX_EDGES 64    /* distinct finite squared edges per count job */

/* the status codes (KD_OK, KD_EINVAL, ...) and KD_MAX_POINTS are public:
 * include/kdtree.h; the device error words use the same codes */

typedef struct kd_catalog {
    int device;
    int n_raw;        /* input points */
    int n_u;          /* unique points (tree size) */
    int memsize;      /* node array length */
    int num_fields;   /* as given to tree_construct */
    int max_qf;       /* largest own field id (0 without fields) */
    int max_tf;       /* largest stored tree field id */
    int min_qf;       /* smallest own field id */
    int fields_split; /* 1 when some raw point has qf != tf */
    double max_abs;   /* largest |coordinate| */

    /* reference-exact tree */
    void *d_nodes;    /* memsize node_t records (40 B), zero where empty */
    int *d_inorder_rep; /* n_u: input index of the point at in-order position */

    /* counting layout, n_raw entries each, in counting order */
    double *d_x, *d_y, *d_z;
    int *d_qf;        /* own field */
    int *d_tf;        /* tree field; aliases d_qf when fields_split == 0 */

    /* counting tree: heap ids 1 .. 2^(D+1)-1, leaves at depth D */
    int depth;        /* D */
    int nleaves;      /* 2^D */
    double *d_box;    /* 6 per heap id: lo x,y,z, hi x,y,z */
    int *d_ncount;    /* raw points per heap id */
    int *d_ntf;       /* single tree field of the node, -1 when mixed */
    int *d_nqf;       /* single own field of the node, -1 when mixed */
    int *d_leaf_run;  /* nleaves+1: first run of each leaf */
    int *d_leaf_pos;  /* nleaves+1: first raw position (counting order) of each leaf */

    int nruns;
    int *d_run_start, *d_run_len, *d_run_tf, *d_run_leaf;

    /* tree side in FP32: t = fl32(point - leaf box centre), stored as
     * float4 (-2 t.x, -2 t.y, -2 t.z, fl32(|t|^2)) */
    void *d_t4;
    double *d_leaf_c;  /* 3 per leaf: box centre */
    double leaf_hdiag; /* largest leaf box half-diagonal */

    int nblocks;
    int *d_blk_start, *d_blk_len;
    int *d_blk_qf;     /* single own field of the block, -1 when mixed */
    double *d_blk_box; /* 6 per block */

    size_t device_bytes;
    kd_build_stats bstats; /* phase timings of the build */
    void *pending;         /* deferred builds: the node copy still running */
} kd_catalog;

/* Build a catalog from host arrays (xyz interleaved (n,3), fields may be
 * NULL) to serve as the query side of counts only: a point may repeat 256 or
 * more times (only tree nodes store an 8-bit weight) and no node array is
 * returned.  Returns KD_OK or a negative status; on failure nothing is held. */
int kdg_build(const double *h_xyz, const int *h_fields, int n, int num_fields,
              int query_only, kd_catalog *cat);

/* Where a tree build puts the reference node array (tree_construct's
 * node_data): alloc gives host memory of the requested size (NULL when out
 * of memory), release frees it; on success nodes holds the filled array. */
typedef struct kd_node_sink {
    void *(*alloc)(size_t bytes);
    void (*release)(void *p);
    void *nodes;
} kd_node_sink;

/* kdg_build for a tree: the node array (memsize * 40 bytes) is copied into
 * sink's host array while the tree and the counting layout are built (the
 * device keeps no copy of it).  deferred = 0: returns once the host array is
 * complete.  deferred = 1: returns once the catalog is complete on the
 * device (it may be counted at once) while a host thread still fills the
 * host array; kdg_wait_nodes waits for that thread (KD_OK or the copy's
 * error, with the message set), and kdg_free waits for it first. */
int kdg_build_tree(const double *h_xyz, const int *h_fields, int n, int num_fields,
                   kd_node_sink *sink, int deferred, kd_catalog *cat);
int kdg_wait_nodes(kd_catalog *cat);
/* Copy the in-order permutation (input index of each in-order node). */
int kdg_copy_inorder(const kd_catalog *cat, int *h_perm);
void kdg_free(kd_catalog *cat);

/* Count pairs (query raw point, tree raw point) for every squared edge.
 *   rsq      : ne sorted distinct squared edges (may end with +inf)
 *   hist     : host output, (ne+1) x (max_qf+1) x (max_tf+1) int64:
 *              hist[e][qf][tf] = pairs whose FP64 squared distance d2
 *              satisfies rsq[e-1] <= d2 < rsq[e] (e = ne: beyond all edges,
 *              left zero)
 *   shard, nshards: count only this shard's query blocks (interleaved
 *              chunks of 32 blocks, chunk c on shard c mod nshards)
 */
int kdg_count(const kd_catalog *tree, const kd_catalog *query,
              const double *rsq, int ne, int mode, int shard, int nshards,
              long long *hist, kd_count_stats *stats);

/* kdg_count for njobs (trees[j], queries[j]) pairs at once: all their query
 * blocks are numbered consecutively (job after job) and counted by one
 * traversal and one persistent tile launch per record batch; hists[j] has
 * kdg_count's layout for job j.  shard/nshards split the global blocks. */
int kdg_count_batch(const kd_catalog *const *trees, const kd_catalog *const *queries,
                    int njobs, const double *rsq, int ne, int mode, int shard, int nshards,
                    long long *const *hists, kd_count_stats *stats);

/* Coordinates (libcoords). */
int kdg_radec2cart(const double *ra, const double *dec, const double *dist,
                   double *xyz, int n);

/* kdg_count without allocations: every buffer comes from a static device
 * array (kd_count.cu).  rsq_sorted: ne distinct sorted squared edges;
 * edge_of[k]: index in rsq_sorted of radius k, -1 for a NaN radius; out: host
 * array of nradii * Fq * Ft cumulative counts in the reference layout. */
int kdg_count_static(const kd_catalog *tree, int Ft, const kd_catalog *query, int Fq,
                     const double *rsq_sorted, int ne, const int *edge_of, int nradii,
                     int mode, long long *out);

/* cudaSetDevice for the calling thread, with the library's error reporting */
int kdg_set_device(int device);

void kd_set_error(int code, const char *fmt, ...);

#ifdef __cplusplus
}
#endif
#endif
