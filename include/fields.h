/*
 * corruscant-b200: C ABI of the jackknife field division (libcoords.so).
 *
 * Replaces the two third-party libraries the reference's
 * corruscant/fields.py imports (fields.py:22-26), which are not available
 * here: healpy for the HEALPix pixelisation of the sphere (ang2pix,
 * get_all_neighbours, boundaries) and pymetis for the weighted graph
 * partition of the pixels into fields (pymetis.part_graph, fields.py:123-126).
 *
 * HEALPix (Gorski et al. 2005, ApJ 622, 759), RING numbering, the scheme
 * healpy uses by default: 12 * nside^2 equal-area pixels in 4 * nside - 1
 * iso-latitude rings counted from the north pole; pixel p of ring i.  The
 * functions below are written from the published definition of the
 * projection (ring latitudes, pixel centres, the two families of pixel
 * boundaries), not from any HEALPix library.  nside is any positive integer
 * up to 2^20 (healpy's RING scheme takes any nside too).
 *
 * The partition is this project's own recursive bisection (greedy graph
 * growing and boundary refinement), minimising the weight of cut edges under
 * a vertex-weight balance; it fills the role of METIS's recursive partition
 * but does not reproduce METIS's heuristic choices.
 */
#ifndef CORRUSCANT_B200_FIELDS_H
#define CORRUSCANT_B200_FIELDS_H

#ifdef __cplusplus
extern "C" {
#endif

/* healpy.ang2pix(nside, theta, phi) (RING): theta colatitude in [0, pi],
 * phi longitude in radians (any value: taken modulo 2 pi).  Threaded over
 * large n.  Returns 0, or -1 for nside outside [1, 2^20] or a NaN angle. */
int kd_healpix_ang2pix(int nside, const double *theta, const double *phi, long long n,
                       long long *pix);

/* healpy.pix2ang(nside, pix) (RING): the pixel centres.  Returns 0 or -1
 * (bad nside or pixel index). */
int kd_healpix_pix2ang(int nside, const long long *pix, long long n, double *theta,
                       double *phi);

/* The four pixels sharing an edge with each pixel: nb[4*p + k] for
 * k = 0..3 in the directions south-west, north-west, north-east, south-east
 * (healpy.get_all_neighbours(nside, p)[::2], which fields.py:30 keeps).
 * nb holds 4 * 12 * nside^2 entries.  Returns 0 or -1. */
int kd_healpix_edge_neighbours(int nside, long long *nb);

/* Corners of a pixel as unit vectors (healpy.boundaries(nside, p), step 1):
 * xyz[3*k + d] for the corners k = 0..3 (north, west, south, east).
 * Returns 0 or -1. */
int kd_healpix_corners(int nside, long long pix, double *xyz);

/* Partition the graph of nv vertices (CSR: the neighbours of v are
 * adjncy[xadj[v] .. xadj[v+1]), with edge weights ewgt in the same layout,
 * and vertex weights vwgt) into nparts parts by recursive bisection: each
 * bisection splits the vertex weight in proportion to the parts on either
 * side and refines the boundary to cut as little edge weight as it can.
 * part[v] receives 0 .. nparts-1.  Returns the total weight of cut edges
 * (each edge counted once), or -1 for bad arguments. */
long long kd_partition_graph(int nv, const int *xadj, const int *adjncy, const long long *vwgt,
                             const long long *ewgt, int nparts, int *part);

#ifdef __cplusplus
}
#endif
#endif
