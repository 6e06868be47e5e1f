"""ctypes bindings for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the benchmark's CPU-baseline
leg import this module, and only as the checker.  The product
(``corruscant_b200``) never imports it.

``liboracle.so`` is this project's C restatement of the reference algorithm
(kdoracle.c).  ``RefLib`` binds the unmodified reference libraries that
``make -C oracle ref`` compiles from the reference sources into
``oracle/_ref/`` (present only where that build was made).
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_longlong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _dp(a):
    return a.ctypes.data_as(POINTER(c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(POINTER(c_int))


def lib():
    """Load (building on first use) oracle/liboracle.so."""
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
        L = ctypes.CDLL(path)
        L.or_last_error.restype = ctypes.c_char_p
        L.or_build.argtypes = [POINTER(c_double), POINTER(c_int), c_int, c_int,
                               POINTER(c_void_p)]
        L.or_free.argtypes = [c_void_p]
        for f in ("or_tree_size", "or_tree_memsize", "or_tree_num_fields"):
            getattr(L, f).argtypes = [c_void_p]
            getattr(L, f).restype = c_int
        L.or_tree_nodes.argtypes = [c_void_p, POINTER(c_double)] + [POINTER(c_int)] * 5
        L.or_tree_inorder.argtypes = [c_void_p, POINTER(c_int)]
        L.or_tree_unique.argtypes = [c_void_p, POINTER(c_double)] + [POINTER(c_int)] * 3
        L.or_pair_count.argtypes = [c_void_p, POINTER(c_double), POINTER(c_int), c_int,
                                    c_int, c_double, c_int, POINTER(c_longlong),
                                    POINTER(c_longlong)]
        L.or_brute_counts.argtypes = [c_void_p, POINTER(c_double), POINTER(c_int), c_int,
                                      c_int, POINTER(c_double), c_int, c_int,
                                      POINTER(c_longlong)]
        L.or_tree_counts.argtypes = [c_void_p, POINTER(c_double), POINTER(c_int), c_int,
                                     c_int, POINTER(c_double), c_int, c_int,
                                     POINTER(c_longlong)]
        L.or_count_visits.restype = c_longlong
        L.or_count_visits.argtypes = [POINTER(c_double)] + [POINTER(c_int)] * 3 + [
            c_int, POINTER(c_double), c_int, c_double, c_int]
        for f in ("or_radec2cart64",):
            getattr(L, f).argtypes = [POINTER(c_double)] * 3 + [c_int]
        L.or_radecdist2cart64.argtypes = [POINTER(c_double)] * 4 + [c_int]
        L.or_radec2sph64.argtypes = [POINTER(c_double)] * 4 + [c_int]
        _LIB = L
    return _LIB


class OracleError(RuntimeError):
    pass


class OracleTree:
    """The oracle's restatement of ``tree_construct`` (kdbuild.c:451-537)."""

    def __init__(self, points, fields=None, num_fields=None):
        L = lib()
        pts = np.require(points, dtype=np.float64, requirements="AC")
        self.n_in = pts.shape[0]
        f = None if fields is None else np.require(fields, dtype=np.int32, requirements="AC")
        if num_fields is None:
            num_fields = 1 if f is None else int(f.max()) + 1
        self.num_fields = num_fields
        h = c_void_p()
        rc = L.or_build(_dp(pts), _ip(f), c_int(self.n_in), c_int(num_fields), ctypes.byref(h))
        if rc != 0:
            raise OracleError(L.or_last_error().decode())
        self._h = h
        self.size = L.or_tree_size(h)
        self.memsize = L.or_tree_memsize(h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_free(self._h)
            self._h = None

    def nodes(self):
        """Semantic node fields: dict of arrays of length memsize."""
        m = self.memsize
        xyz = np.zeros((m, 3))
        arr = [np.zeros(m, dtype=np.int32) for _ in range(5)]
        lib().or_tree_nodes(self._h, _dp(xyz), *[_ip(a) for a in arr])
        return dict(xyz=xyz, field=arr[0], weight=arr[1], has_l=arr[2], has_r=arr[3],
                    dim=arr[4])

    def inorder(self):
        p = np.zeros(self.size, dtype=np.int32)
        lib().or_tree_inorder(self._h, _ip(p))
        return p

    def unique(self):
        n = self.size
        xyz = np.zeros((n, 3))
        f, w, r = (np.zeros(n, dtype=np.int32) for _ in range(3))
        lib().or_tree_unique(self._h, _dp(xyz), _ip(f), _ip(w), _ip(r))
        return xyz, f, w, r

    def pair_count(self, q, qfields=None, num_fields_q=1, r=0.1, nthreads=1,
                   return_visits=False):
        """Restated kdquery.c traversal; returns int64 (Fq*Ft,) flat counts."""
        q = np.require(q, dtype=np.float64, requirements="AC")
        qf = None if qfields is None else np.require(qfields, dtype=np.int32, requirements="AC")
        out = np.zeros(num_fields_q * self.num_fields, dtype=np.int64)
        vis = c_longlong(0)
        rc = lib().or_pair_count(self._h, _dp(q), _ip(qf), c_int(q.shape[0]),
                                 c_int(num_fields_q), c_double(r), c_int(nthreads),
                                 out.ctypes.data_as(POINTER(c_longlong)), ctypes.byref(vis))
        if rc != 0:
            raise OracleError(lib().or_last_error().decode())
        return (out, vis.value) if return_visits else out

    def brute_counts(self, q, qfields=None, num_fields_q=1, radii=(0.1,), nthreads=4):
        """Exhaustive FP64 cumulative counts, shape (len(radii), Fq*Ft)."""
        q = np.require(q, dtype=np.float64, requirements="AC")
        qf = None if qfields is None else np.require(qfields, dtype=np.int32, requirements="AC")
        radii = np.require(np.asarray(radii, dtype=np.float64), requirements="AC")
        out = np.zeros((len(radii), num_fields_q * self.num_fields), dtype=np.int64)
        rc = lib().or_brute_counts(self._h, _dp(q), _ip(qf), c_int(q.shape[0]),
                                   c_int(num_fields_q), _dp(radii), c_int(len(radii)),
                                   c_int(nthreads), out.ctypes.data_as(POINTER(c_longlong)))
        if rc != 0:
            raise OracleError(lib().or_last_error().decode())
        return out

    def tree_counts(self, q, qfields=None, num_fields_q=1, radii=(0.1,), nthreads=8):
        """brute_counts' result through the reference traversal pruned at the
        largest radius (or_tree_counts): exact, and fast enough for whole
        catalogs of a few hundred thousand points."""
        q = np.require(q, dtype=np.float64, requirements="AC")
        qf = None if qfields is None else np.require(qfields, dtype=np.int32, requirements="AC")
        radii = np.require(np.asarray(radii, dtype=np.float64), requirements="AC")
        out = np.zeros((len(radii), num_fields_q * self.num_fields), dtype=np.int64)
        rc = lib().or_tree_counts(self._h, _dp(q), _ip(qf), c_int(q.shape[0]),
                                  c_int(num_fields_q), _dp(radii), c_int(len(radii)),
                                  c_int(nthreads), out.ctypes.data_as(POINTER(c_longlong)))
        if rc != 0:
            raise OracleError(lib().or_last_error().decode())
        return out


def count_visits(nodes, q, r, nthreads=8):
    """Reference traversal node visits (its "pairs tested") over a node array
    given as the dict returned by OracleTree.nodes() / RefLib.nodes()."""
    xyz = np.require(nodes["xyz"], dtype=np.float64, requirements="AC")
    hl, hr, dm = (np.require(nodes[k], dtype=np.int32, requirements="AC")
                  for k in ("has_l", "has_r", "dim"))
    q = np.require(q, dtype=np.float64, requirements="AC")
    return lib().or_count_visits(_dp(xyz), _ip(hl), _ip(hr), _ip(dm), c_int(len(hl)), _dp(q),
                                 c_int(q.shape[0]), c_double(r), c_int(nthreads))


def radec2cart64(ra, dec):
    ra = np.require(ra, dtype=np.float64, requirements="AC")
    dec = np.require(dec, dtype=np.float64, requirements="AC")
    out = np.empty((ra.size, 3))
    lib().or_radec2cart64(_dp(ra), _dp(dec), _dp(out), c_int(ra.size))
    return out


def radecdist2cart64(ra, dec, dist):
    ra, dec, dist = (np.require(a, dtype=np.float64, requirements="AC") for a in (ra, dec, dist))
    out = np.empty((ra.size, 3))
    lib().or_radecdist2cart64(_dp(ra), _dp(dec), _dp(dist), _dp(out), c_int(ra.size))
    return out


def radec2sph64(ra, dec):
    ra = np.require(ra, dtype=np.float64, requirements="AC")
    dec = np.require(dec, dtype=np.float64, requirements="AC")
    th, ph = np.empty(ra.size), np.empty(ra.size)
    lib().or_radec2sph64(_dp(ra), _dp(dec), _dp(th), _dp(ph), c_int(ra.size))
    return th, ph


def reference_root():
    """The reference project's checkout (its ``src/`` and ``corruscant/``),
    read from the CORRUSCANT_REF environment variable, else the location this
    build's checker was set up against; None when neither exists.  This is
    the one place that names it: the build step, the golden generator and
    the side-by-side tests all ask here."""
    root = os.environ.get("CORRUSCANT_REF", "/root/reference")
    return root if os.path.isdir(os.path.join(root, "src")) else None


def ref_path():
    return os.path.join(HERE, "_ref")


def ref_available():
    return os.path.exists(os.path.join(ref_path(), "libkdtree.so"))


class _KdTreeStruct(ctypes.Structure):
    """kdtree_t as declared in the reference kdtree.h:33-41 (64 bytes)."""
    _fields_ = [("node_data", c_void_p), ("size", c_int), ("memsize", c_int),
                ("num_fields", c_int), ("data", c_void_p), ("fields", c_void_p),
                ("args", c_void_p * 3)]


class _NodeStruct(ctypes.Structure):
    """node_t, kdtree.h:13-25: datum (3 doubles + a word holding field:8 and
    weight:8) followed by a word holding has_lchild:1, has_rchild:1, dim:8."""
    _fields_ = [("value", c_double * 3), ("fw", ctypes.c_uint32), ("_pad0", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("_pad1", ctypes.c_uint32)]


class RefLib:
    """The unmodified reference library compiled from its sources (oracle/_ref)."""

    def __init__(self):
        p = ref_path()
        self.kd = ctypes.CDLL(os.path.join(p, "libkdtree.so"))
        self.co = ctypes.CDLL(os.path.join(p, "libcoords.so"))
        self.kd.tree_construct.restype = _KdTreeStruct
        self.kd.tree_construct.argtypes = [POINTER(c_double), POINTER(c_int), c_int, c_int]
        self.kd.pair_count.restype = POINTER(c_longlong)
        self.kd.pair_count.argtypes = [_KdTreeStruct, POINTER(c_double), POINTER(c_int),
                                       c_int, c_int, c_double, c_int]
        self.kd.destroy.argtypes = [_KdTreeStruct]
        self.kd.destroy.restype = None
        self.co.radec2cart64.argtypes = [POINTER(c_double)] * 3 + [c_int]
        self.co.radecdist2cart64.argtypes = [POINTER(c_double)] * 4 + [c_int]
        self.co.radec2sph64.argtypes = [POINTER(c_double)] * 4 + [c_int]
        self.libc = ctypes.CDLL(None)
        self.libc.free.argtypes = [c_void_p]

    def build(self, points, fields=None, num_fields=None):
        pts = np.require(points, dtype=np.float64, requirements="AC")
        f = None if fields is None else np.require(fields, dtype=np.int32, requirements="AC")
        if num_fields is None:
            num_fields = 1 if f is None else int(f.max()) + 1
        t = self.kd.tree_construct(_dp(pts), _ip(f), c_int(pts.shape[0]), c_int(num_fields))
        return t

    def nodes(self, t):
        """Semantic node fields of a reference tree, like OracleTree.nodes()."""
        m = t.memsize
        arr = (_NodeStruct * m).from_address(t.node_data)
        raw = np.ctypeslib.as_array(arr)
        xyz = np.array(raw["value"], dtype=np.float64).reshape(m, 3)
        fw = raw["fw"].astype(np.int64)
        fl = raw["flags"].astype(np.int64)
        return dict(xyz=xyz, field=(fw & 0xFF).astype(np.int32),
                    weight=((fw >> 8) & 0xFF).astype(np.int32),
                    has_l=(fl & 1).astype(np.int32), has_r=((fl >> 1) & 1).astype(np.int32),
                    dim=((fl >> 2) & 0xFF).astype(np.int32))

    def pair_count(self, t, q, qfields=None, num_fields_q=1, r=0.1, nthreads=1):
        q = np.require(q, dtype=np.float64, requirements="AC")
        qf = None if qfields is None else np.require(qfields, dtype=np.int32, requirements="AC")
        ptr = self.kd.pair_count(t, _dp(q), _ip(qf), c_int(q.shape[0]), c_int(num_fields_q),
                                 c_double(r), c_int(nthreads))
        n = num_fields_q * t.num_fields
        out = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        self.libc.free(ctypes.cast(ptr, c_void_p))
        return out

    def destroy(self, t):
        self.kd.destroy(t)

    def radec2cart64(self, ra, dec):
        ra = np.require(ra, dtype=np.float64, requirements="AC")
        dec = np.require(dec, dtype=np.float64, requirements="AC")
        out = np.empty((ra.size, 3))
        self.co.radec2cart64(_dp(ra), _dp(dec), _dp(out), c_int(ra.size))
        return out

    def radecdist2cart64(self, ra, dec, dist):
        ra, dec, dist = (np.require(a, dtype=np.float64, requirements="AC")
                         for a in (ra, dec, dist))
        out = np.empty((ra.size, 3))
        self.co.radecdist2cart64(_dp(ra), _dp(dec), _dp(dist), _dp(out), c_int(ra.size))
        return out

    def radec2sph64(self, ra, dec):
        """The reference's coordmath.c:73-80: (theta, phi) in radians."""
        ra = np.require(ra, dtype=np.float64, requirements="AC")
        dec = np.require(dec, dtype=np.float64, requirements="AC")
        theta, phi = np.empty(ra.size), np.empty(ra.size)
        self.co.radec2sph64(_dp(ra), _dp(dec), _dp(theta), _dp(phi), c_int(ra.size))
        return theta, phi
