"""ctypes bindings of the in-tree native libraries (bin/libkdtree.so,
bin/libcoords.so).

The structure layouts are the reference's C ABI (src/kdtree.h:11-41).  Unlike
the reference's ctypes declaration (corruscant/clustering.py:36-45, where
``args`` is a single pointer and the struct is 48 bytes), ``KdTree`` declares
``args`` as three pointers, so it is the full 64-byte ``kdtree_t`` that
``tree_construct`` returns by value.

There is no fallback: if the library is missing or cannot find a CUDA device,
calls raise ``NativeError``.
"""
import ctypes
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_int, c_longlong, c_uint, c_void_p

import numpy as np

PROJECT_PATH = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(PROJECT_PATH, "bin")

KD_MODE_MIXED = 0
KD_MODE_FP64 = 1


class NativeError(RuntimeError):
    """An error reported by the native library (code and message)."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Datum(Structure):
    _fields_ = [("value", c_double * 3), ("field", c_uint, 8), ("weight", c_uint, 8)]


class Node(Structure):
    _fields_ = [("data", Datum), ("has_lchild", c_uint, 1), ("has_rchild", c_uint, 1),
                ("dim", c_uint, 8)]


class KdTree(Structure):
    _fields_ = [("node_data", POINTER(Node)), ("size", c_int), ("memsize", c_int),
                ("num_fields", c_int), ("data", POINTER(Datum)), ("fields", POINTER(c_int)),
                ("args", POINTER(c_int) * 3)]


class CountStats(Structure):
    _fields_ = [("pairs_tested", c_longlong), ("pairs_rechecked", c_longlong),
                ("pairs_accepted", c_longlong), ("pairs_wide", c_longlong),
                ("edge_pairs", c_longlong), ("warp_tiles", c_longlong), ("entries", c_longlong), ("ms_traverse", c_double), ("ms_tiles", c_double),
                ("ms_total", c_double), ("tile_launches", c_int), ("launches", c_int),
                ("pairs_one_bin_multifield", c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BuildStats(Structure):
    _fields_ = [(n, c_double) for n in ("ms_prep", "ms_dedup", "ms_argsort", "ms_levels",
                                        "ms_layout", "ms_device", "ms_node_copy",
                                        "ms_node_wait", "ms_total_host")] + \
               [("levels", c_int), ("n_unique", c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


assert ctypes.sizeof(KdTree) == 64
assert ctypes.sizeof(Node) == 40

_KD = None


def loadlib(name):
    """Load ``bin/<name>.so`` (the in-tree build)."""
    path = os.path.join(BIN, name + ".so")
    if not os.path.exists(path):
        raise OSError(f"{path} not found: build it with "
                      f"`python -c 'import __graft_entry__; __graft_entry__.build()'` "
                      f"or `make -C corruscant_b200/csrc`")
    return ctypes.CDLL(path)


def kdlib():
    global _KD
    if _KD is None:
        L = loadlib("libkdtree")
        L.tree_construct.restype = KdTree
        L.tree_construct.argtypes = [POINTER(c_double), POINTER(c_int), c_int, c_int]
        L.kd_tree_construct_deferred.restype = KdTree
        L.kd_tree_construct_deferred.argtypes = [POINTER(c_double), POINTER(c_int), c_int, c_int]
        L.kd_tree_wait_nodes.restype = c_int
        L.kd_tree_wait_nodes.argtypes = [KdTree]
        L.pair_count.restype = POINTER(c_longlong)
        L.pair_count.argtypes = [KdTree, POINTER(c_double), POINTER(c_int), c_int, c_int,
                                 c_double, c_int]
        L.destroy.restype = None
        L.destroy.argtypes = [KdTree]
        L.kd_last_error.restype = c_int
        L.kd_last_error.argtypes = [c_char_p, c_int]
        L.kd_free_counts.restype = None
        L.kd_free_counts.argtypes = [c_void_p]
        L.kd_count_radii.restype = c_int
        L.kd_count_radii.argtypes = [KdTree, KdTree, POINTER(c_double), c_int, c_int,
                                     POINTER(c_longlong), POINTER(CountStats)]
        L.kd_count_radii_shard.restype = c_int
        L.kd_count_radii_shard.argtypes = [KdTree, KdTree, POINTER(c_double), c_int, c_int, c_int,
                                           c_int, POINTER(c_longlong), POINTER(CountStats)]
        L.kd_count_bins.restype = c_int
        L.kd_count_bins.argtypes = [KdTree, KdTree, POINTER(c_double), c_int, c_int,
                                    POINTER(c_longlong), POINTER(CountStats)]
        L.kd_count_batch_shard.restype = c_int
        L.kd_count_batch_shard.argtypes = [POINTER(KdTree), POINTER(KdTree), c_int, POINTER(c_double),
                                           c_int, c_int, c_int, c_int, POINTER(c_longlong),
                                           POINTER(CountStats)]
        L.kd_count_batch.restype = c_int
        L.kd_count_batch.argtypes = [POINTER(KdTree), POINTER(KdTree), c_int, POINTER(c_double),
                                     c_int, c_int, POINTER(c_longlong), POINTER(CountStats)]
        L.kd_count_radii_static.restype = c_int
        L.kd_count_radii_static.argtypes = [KdTree, KdTree, POINTER(c_double), c_int, c_int,
                                            POINTER(c_longlong)]
        L.kd_count_points.restype = c_int
        L.kd_count_points.argtypes = [KdTree, POINTER(c_double), POINTER(c_int), c_int, c_int,
                                      POINTER(c_double), c_int, c_int, POINTER(c_longlong),
                                      POINTER(CountStats)]
        L.kd_tree_permutation.restype = c_int
        L.kd_tree_permutation.argtypes = [KdTree, POINTER(c_int)]
        L.kd_set_precision.restype = c_int
        L.kd_set_precision.argtypes = [c_int]
        L.kd_tree_build_stats.restype = c_int
        L.kd_tree_build_stats.argtypes = [KdTree, POINTER(BuildStats)]
        L.kd_set_device.restype = c_int
        L.kd_set_device.argtypes = [c_int]
        L.kd_tree_input_size.restype = c_int
        L.kd_tree_input_size.argtypes = [KdTree]
        _KD = L
    return _KD


def last_error():
    buf = ctypes.create_string_buffer(256)
    code = kdlib().kd_last_error(buf, 256)
    return code, buf.value.decode(errors="replace")


def raise_last(default="native call failed"):
    code, msg = last_error()
    raise NativeError(code or -1, msg or default)


def dptr(a):
    return a.ctypes.data_as(POINTER(c_double))


def iptr(a):
    return None if a is None else a.ctypes.data_as(POINTER(c_int))


def build_tree(points, fields, num_fields, deferred=False):
    """tree_construct on C-contiguous float64 (N,3) points and int32 fields.

    deferred: kd_tree_construct_deferred, which returns once the tree is on
    the device while its node array is still being copied to node_data; the
    tree can be counted at once, and wait_nodes(t) waits for the node array.
    """
    fn = kdlib().kd_tree_construct_deferred if deferred else kdlib().tree_construct
    t = fn(dptr(points), iptr(fields), c_int(points.shape[0]), c_int(num_fields))
    if not t.node_data:
        raise_last("tree_construct failed")
    return t


def wait_nodes(t):
    """kd_tree_wait_nodes: returns once t.node_data is complete."""
    if kdlib().kd_tree_wait_nodes(t) != 0:
        raise_last()


def node_fields(t):
    """Semantic node fields of a kdtree_t as numpy arrays (length memsize)."""
    wait_nodes(t)
    m = t.memsize
    raw = np.ctypeslib.as_array(ctypes.cast(t.node_data, POINTER(ctypes.c_uint8)),
                                shape=(m * 40,)).reshape(m, 40)
    xyz = raw[:, :24].copy().view(np.float64).reshape(m, 3)
    fw = raw[:, 24:28].copy().view(np.uint32).ravel().astype(np.int64)
    fl = raw[:, 32:36].copy().view(np.uint32).ravel().astype(np.int64)
    return dict(xyz=xyz, field=(fw & 0xFF).astype(np.int32),
                weight=((fw >> 8) & 0xFF).astype(np.int32),
                has_l=(fl & 1).astype(np.int32), has_r=((fl >> 1) & 1).astype(np.int32),
                dim=((fl >> 2) & 0xFF).astype(np.int32))


def count_radii(tree, query, radii, mode=KD_MODE_MIXED, with_stats=False):
    """Cumulative counts, shape (len(radii), Fq*Ft), for all radii in one pass."""
    radii = np.require(np.asarray(radii, dtype=np.float64), requirements="AC")
    out = np.zeros((len(radii), query.num_fields * tree.num_fields), dtype=np.int64)
    st = CountStats()
    rc = kdlib().kd_count_radii(tree, query, dptr(radii), c_int(len(radii)), c_int(mode),
                                out.ctypes.data_as(POINTER(c_longlong)), ctypes.byref(st))
    if rc != 0:
        raise_last()
    return (out, st.as_dict()) if with_stats else out


def count_radii_shard(tree, query, radii, shard, nshards, mode=KD_MODE_MIXED, with_stats=False):
    """One shard of count_radii (query blocks split evenly over nshards)."""
    radii = np.require(np.asarray(radii, dtype=np.float64), requirements="AC")
    out = np.zeros((len(radii), query.num_fields * tree.num_fields), dtype=np.int64)
    st = CountStats()
    rc = kdlib().kd_count_radii_shard(tree, query, dptr(radii), c_int(len(radii)), c_int(mode),
                                      c_int(shard), c_int(nshards),
                                      out.ctypes.data_as(POINTER(c_longlong)), ctypes.byref(st))
    if rc != 0:
        raise_last()
    return (out, st.as_dict()) if with_stats else out


def count_bins(tree, query, edges, mode=KD_MODE_MIXED):
    """kd_count_bins: (len(edges)-1, Fq*Ft) per-bin counts."""
    edges = np.require(np.asarray(edges, dtype=np.float64), requirements="AC")
    out = np.zeros((max(0, len(edges) - 1), query.num_fields * tree.num_fields), dtype=np.int64)
    rc = kdlib().kd_count_bins(tree, query, dptr(edges), c_int(len(edges)), c_int(mode),
                               out.ctypes.data_as(POINTER(c_longlong)), None)
    if rc != 0:
        raise_last()
    return out


def count_batch(jobs, radii, mode=KD_MODE_MIXED, with_stats=False, shard=0, nshards=1):
    """kd_count_batch: jobs is a sequence of (tree, query tree) pairs; returns
    one count_radii result per job (all jobs counted in one device batch)."""
    jobs = list(jobs)
    radii = np.require(np.asarray(radii, dtype=np.float64), requirements="AC")
    trees = (KdTree * len(jobs))(*[t for t, _ in jobs])
    queries = (KdTree * len(jobs))(*[q for _, q in jobs])
    sizes = [len(radii) * q.num_fields * t.num_fields for t, q in jobs]
    flat = np.zeros(max(1, sum(sizes)), dtype=np.int64)
    st = CountStats()
    rc = kdlib().kd_count_batch_shard(trees, queries, c_int(len(jobs)), dptr(radii),
                                      c_int(len(radii)), c_int(mode), c_int(shard), c_int(nshards),
                                      flat.ctypes.data_as(POINTER(c_longlong)), ctypes.byref(st))
    if rc != 0:
        raise_last()
    outs, at = [], 0
    for (t, q), n in zip(jobs, sizes):
        outs.append(flat[at:at + n].reshape(len(radii), q.num_fields * t.num_fields).copy())
        at += n
    return (outs, st.as_dict()) if with_stats else outs


def count_radii_static(tree, query, radii, mode=KD_MODE_MIXED):
    """count_radii through kd_count_radii_static (no allocation in the call)."""
    radii = np.require(np.asarray(radii, dtype=np.float64), requirements="AC")
    out = np.zeros((len(radii), query.num_fields * tree.num_fields), dtype=np.int64)
    rc = kdlib().kd_count_radii_static(tree, query, dptr(radii), c_int(len(radii)), c_int(mode),
                                       out.ctypes.data_as(POINTER(c_longlong)))
    if rc != 0:
        raise_last()
    return out


def count_points(tree, points, fields, num_fields, radii, mode=KD_MODE_MIXED, with_stats=False):
    points = np.require(points, dtype=np.float64, requirements="AC")
    fields = None if fields is None else np.require(fields, dtype=np.int32, requirements="AC")
    radii = np.require(np.asarray(radii, dtype=np.float64), requirements="AC")
    out = np.zeros((len(radii), num_fields * tree.num_fields), dtype=np.int64)
    st = CountStats()
    rc = kdlib().kd_count_points(tree, dptr(points), iptr(fields), c_int(points.shape[0]),
                                 c_int(num_fields), dptr(radii), c_int(len(radii)), c_int(mode),
                                 out.ctypes.data_as(POINTER(c_longlong)), ctypes.byref(st))
    if rc != 0:
        raise_last()
    return (out, st.as_dict()) if with_stats else out


def pair_count(tree, points, fields, num_fields, r):
    """The reference entry point: one radius, malloc'd result freed here."""
    points = np.require(points, dtype=np.float64, requirements="AC")
    fields = None if fields is None else np.require(fields, dtype=np.int32, requirements="AC")
    L = kdlib()
    p = L.pair_count(tree, dptr(points), iptr(fields), c_int(points.shape[0]),
                     c_int(num_fields), c_double(r), c_int(1))
    if not p:
        raise_last("pair_count failed")
    out = np.ctypeslib.as_array(p, shape=(num_fields * tree.num_fields,)).copy()
    L.kd_free_counts(ctypes.cast(p, c_void_p))
    return out


def permutation(tree):
    perm = np.zeros(tree.size, dtype=np.int32)
    if kdlib().kd_tree_permutation(tree, iptr(perm)) != 0:
        raise_last()
    return perm


def build_stats(tree):
    """kd_tree_build_stats: where the tree's build spent its time (ms)."""
    st = BuildStats()
    if kdlib().kd_tree_build_stats(tree, ctypes.byref(st)) != 0:
        raise_last()
    return st.as_dict()


def set_precision(mode):
    """Mode of pair_count on this thread (kd_set_precision)."""
    if kdlib().kd_set_precision(c_int(mode)) != 0:
        raise_last()


def set_device(device):
    """Device used by later tree builds of this thread (kd_set_device)."""
    if kdlib().kd_set_device(c_int(device)) != 0:
        raise_last()


def destroy(tree):
    kdlib().destroy(tree)


_CO = None


def coordlib():
    """bin/libcoords.so with the reference's signatures (coordmath.c:38-80)."""
    global _CO
    if _CO is None:
        L = loadlib("libcoords")
        L.radec2cart64.restype = None
        L.radec2cart64.argtypes = [POINTER(c_double)] * 3 + [c_int]
        L.radecdist2cart64.restype = None
        L.radecdist2cart64.argtypes = [POINTER(c_double)] * 4 + [c_int]
        L.radec2sph64.restype = None
        L.radec2sph64.argtypes = [POINTER(c_double)] * 4 + [c_int]
        # field division (include/fields.h)
        L.kd_healpix_ang2pix.restype = c_int
        L.kd_healpix_ang2pix.argtypes = [c_int, POINTER(c_double), POINTER(c_double), c_longlong,
                                         POINTER(c_longlong)]
        L.kd_healpix_pix2ang.restype = c_int
        L.kd_healpix_pix2ang.argtypes = [c_int, POINTER(c_longlong), c_longlong,
                                         POINTER(c_double), POINTER(c_double)]
        L.kd_healpix_edge_neighbours.restype = c_int
        L.kd_healpix_edge_neighbours.argtypes = [c_int, POINTER(c_longlong)]
        L.kd_healpix_corners.restype = c_int
        L.kd_healpix_corners.argtypes = [c_int, c_longlong, POINTER(c_double)]
        L.kd_partition_graph.restype = c_longlong
        L.kd_partition_graph.argtypes = [c_int, POINTER(c_int), POINTER(c_int),
                                         POINTER(c_longlong), POINTER(c_longlong), c_int,
                                         POINTER(c_int)]
        _CO = L
    return _CO


def _llp(a):
    return a.ctypes.data_as(POINTER(c_longlong))


def healpix_ang2pix(nside, theta, phi):
    """RING pixel of each (theta, phi) (healpy.ang2pix's default scheme)."""
    theta = np.require(np.asarray(theta, dtype=np.float64), requirements="AC")
    phi = np.require(np.asarray(phi, dtype=np.float64), requirements="AC")
    if theta.shape != phi.shape:
        raise ValueError("theta and phi must have the same shape")
    out = np.empty(theta.shape, dtype=np.int64)
    if coordlib().kd_healpix_ang2pix(int(nside), dptr(theta), dptr(phi), theta.size,
                                     _llp(out)) != 0:
        raise ValueError("ang2pix: nside must be in [1, 2^20] and angles not NaN")
    return out


def healpix_pix2ang(nside, pix):
    """Centres (theta, phi) of RING pixels."""
    pix = np.require(np.asarray(pix, dtype=np.int64), requirements="AC")
    th, ph = np.empty(pix.shape), np.empty(pix.shape)
    if coordlib().kd_healpix_pix2ang(int(nside), _llp(pix), pix.size, dptr(th), dptr(ph)) != 0:
        raise ValueError("pix2ang: bad nside or pixel index")
    return th, ph


def healpix_edge_neighbours(nside):
    """(12 nside^2, 4) int64: the south-west, north-west, north-east and
    south-east neighbour of every RING pixel."""
    npix = 12 * int(nside) ** 2
    out = np.empty((npix, 4), dtype=np.int64)
    if coordlib().kd_healpix_edge_neighbours(int(nside), _llp(out)) != 0:
        raise ValueError("bad nside")
    return out


def healpix_corners(nside, pix):
    """(3, 4) unit vectors of the pixel's north, west, south and east corners
    (the layout of healpy.boundaries)."""
    out = np.empty((4, 3))
    if coordlib().kd_healpix_corners(int(nside), int(pix), dptr(out)) != 0:
        raise ValueError("bad nside or pixel index")
    return out.T.copy()


def partition_graph(nparts, xadj, adjncy, vweights, eweights):
    """Recursive-bisection partition of a weighted graph in CSR form:
    (edge cut, part id of every vertex)."""
    xadj = np.require(np.asarray(xadj, dtype=np.int32), requirements="AC")
    adjncy = np.require(np.asarray(adjncy, dtype=np.int32), requirements="AC")
    vw = np.require(np.asarray(vweights, dtype=np.int64), requirements="AC")
    ew = np.require(np.asarray(eweights, dtype=np.int64), requirements="AC")
    nv = len(xadj) - 1
    if nv < 1 or len(vw) != nv or len(ew) != len(adjncy):
        raise ValueError("malformed graph")
    part = np.empty(nv, dtype=np.int32)
    cut = coordlib().kd_partition_graph(nv, iptr(xadj), iptr(adjncy), _llp(vw), _llp(ew),
                                        int(nparts), iptr(part))
    if cut < 0:
        raise ValueError("malformed graph or part count")
    return int(cut), part
