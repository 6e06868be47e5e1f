"""Trees, auto/cross-correlation drivers and estimators.

User API of the reference module ``corruscant.clustering``
(corruscant/clustering.py): ``tree``, ``validate_points``,
``validate_fields``, the estimators ``est_standard``, ``est_hamilton``,
``est_landy_szalay`` and the result classes, with the same arguments, shapes
and error behaviour.

What changes is below the API: a ``tree`` is built on the GPU (bit-identical
node array), and ``_autocorr`` / ``_crosscorr`` count every bin edge of every
count type (DD, DR, RR, or the four cross counts) in one GPU batch
(``kd_count_batch``) instead of one ``pair_count`` call per edge and count
type (clustering.py:218-230, :256-284).  The per-edge cumulative
counts, their ``np.diff`` and everything downstream are the same numbers.

The estimator, error and covariance arithmetic is performed in the same
floating-point operation order as the reference (clustering.py:132-159,
:354-672), so estimates, errors and covariances agree with the reference to
0 ulp given the same counts.
"""
from __future__ import division, print_function

import warnings

import numpy as np

from . import _native

__all__ = ["tree", "validate_points", "validate_fields", "est_standard", "est_hamilton",
           "est_landy_szalay", "results", "autocorr_results", "crosscorr_results"]

#: counting precision used by the drivers: FP32 distances with FP64 recheck
#: (default) or every distance in FP64; both give identical counts
DEFAULT_MODE = _native.KD_MODE_MIXED

#: the C ABI's structures under the reference's ctypes names
#: (clustering.py:30-45; ``kdtree`` is the full 64-byte kdtree_t)
datum = _native.Datum
node = _native.Node
kdtree = _native.KdTree


def __getattr__(name):
    """``kdlib``: the loaded libkdtree (clustering.py:47-71), opened on first
    access."""
    if name == "kdlib":
        return _native.kdlib()
    raise AttributeError(name)


def validate_points(points):
    """(N,3) C-contiguous float array of points; a (3,N) array is transposed
    (clustering.py:92-114)."""
    points = np.array(points)
    n = max(points.shape)
    if points.shape != (n, 3):
        points = points.T
    if points.shape != (n, 3):
        raise ValueError("Array must be of shape (N, 3) or (3, N). The provided array has "
                         "shape {:s}".format(str(points.shape)))
    out = np.require(points, requirements="AC")
    if out is not points:
        warnings.warn("Data array is being copied to have shape {:s}".format(str(out.shape)),
                      RuntimeWarning)
    return out


def validate_fields(fields, points):
    """int32 field ids, one per point (clustering.py:116-130)."""
    fields = np.array(fields)
    n = max(points.shape)
    if fields.shape != (n,):
        raise ValueError("Field IDs must be a 1-d array of length equal to the number of "
                         "points")
    return np.require(fields, dtype="int32", requirements="AC")


# -------------------------------------------------------------- estimators

def _unpack(args):
    """(d1d2, d1r2, d2r1, r1r2) from 3 (auto: d2r1 = d1r2) or 4 arrays."""
    if len(args) == 3:
        d1d2, d1r2, r1r2 = args
        return d1d2, d1r2, d1r2, r1r2
    if len(args) == 4:
        return args
    raise TypeError("an estimator takes 3 (auto) or 4 (cross) count arrays")


def est_landy_szalay(*args):
    """(D1D2 - D1R2 - D2R1 + R1R2) / R1R2, evaluated left to right."""
    d1d2, d1r2, d2r1, r1r2 = _unpack(args)
    return (d1d2 - d1r2 - d2r1 + r1r2) / r1r2


def est_hamilton(*args):
    """D1D2 R1R2 / (D1R2 D2R1) - 1."""
    d1d2, d1r2, d2r1, r1r2 = _unpack(args)
    return (d1d2 * r1r2 / (d1r2 * d2r1)) - 1.


def est_standard(*args):
    """D1D2 / D1R2 - 1."""
    d1d2, d1r2, _, _ = _unpack(args)
    return d1d2 / d1r2 - 1.


_ESTIMATORS = {"landy-szalay": est_landy_szalay, "hamilton": est_hamilton,
               "standard": est_standard}


def _estimator(est_type):
    try:
        return _ESTIMATORS[est_type]
    except KeyError:
        raise ValueError("Estimator type for Xi \"{:s}\" not valid. Try \"standard\", "
                         "\"hamilton\", or \"landy-szalay\"".format(str(est_type)))


def _grid_sum(a, b):
    """sum over i, j of a[j] * b[i] (integer field-size products)."""
    return np.sum(np.multiply(*np.meshgrid(a, b)))


# ------------------------------------------------------------------- trees

class tree:
    """A k-d tree of points with optional jackknife field ids, built on the GPU.

    Same constructor and attributes as clustering.py:293-352: ``points``,
    ``fields`` (None or int32), ``N_fields``, ``field_sizes``, ``size``
    (unique points) and ``ctree`` (the 64-byte ``kdtree_t``).
    """

    def __init__(self, points, fields=None):
        points = validate_points(points)
        if fields is None:
            self.fields = None
            self.N_fields = 1
        else:
            fields = validate_fields(fields, points)
            ids = np.unique(fields)
            if not np.all(ids == range(np.max(fields) + 1)):
                raise ValueError("fields must be a 1-D array of integers from 0 to the number "
                                 "of unique fields minus one")
            self.N_fields = ids.size
            if self.N_fields < 2:
                raise ValueError("At least two unique field IDs must be provided if using "
                                 "error fields")
            self.fields = fields
            self.field_sizes = self._calc_field_sizes()
        self.points = np.require(points, dtype="float64", requirements="AC")
        self._make_tree()
        self.size = self._ct.size
        if fields is None:
            self.field_sizes = np.array(self.size)

    def _calc_field_sizes(self):
        """Points per field id 0 .. N_fields - 1 (clustering.py:336-338)."""
        return np.bincount(self.fields, minlength=self.N_fields)

    def _make_tree(self):
        """Build the GPU tree of ``points`` / ``fields`` (clustering.py:340-349).

        The build returns once the tree is on the device; its node array
        still drains to the host behind it, so counts can start at once.
        ``ctree`` waits for the node array before handing out the struct.
        """
        self._ct = _native.build_tree(self.points, self.fields, self.N_fields, deferred=True)
        self._nodes_ready = False

    @property
    def ctree(self):
        """The reference's ``kdtree_t``, its ``node_data`` complete."""
        if self._ct is not None and not self._nodes_ready:
            _native.wait_nodes(self._ct)
            self._nodes_ready = True
        return self._ct

    @ctree.setter
    def ctree(self, value):
        self._ct = value
        self._nodes_ready = True

    def __del__(self):
        ct = getattr(self, "_ct", None)
        if ct is not None and ct.node_data:
            _native.destroy(ct)
            self._ct = None


def _query_tree(tree_, points, radius, num_threads, fields=None, N_fields=1):
    """One radius through the reference entry point ``pair_count``
    (clustering.py:73-90): an (N_fields, tree.N_fields) int64 matrix."""
    del num_threads  # the GPU path has no thread count
    counts = _native.pair_count(tree_._ct, points, fields, N_fields, radius)
    return counts.reshape(N_fields, tree_.N_fields)


def _count_binned(tree_, query, radii, mode):
    """Per-bin (len(radii)-1, Fq, Ft) counts of ``query``'s points against
    ``tree_``: the np.diff over edges of the per-edge cumulative counts."""
    return _count_binned_batch([(tree_, query)], radii, mode)[0]


def _count_binned_batch(jobs, radii, mode):
    """_count_binned for several (tree, query) pairs, counted together in one
    device batch (``kd_count_batch``)."""
    cums = _native.count_batch([(t._ct, q._ct) for t, q in jobs], radii, mode=mode)
    return [np.diff(c.reshape(len(radii), q.N_fields, t.N_fields), axis=0)
            for (t, q), c in zip(jobs, cums)]


def _autocorr(data_tree, rand_tree, radii, est_type="landy-szalay", err_type="jackknife",
              num_threads=4, mode=None):
    """DD, DR, RR counts and an ``autocorr_results`` (clustering.py:161-235).
    ``err_type`` and ``num_threads`` are accepted for compatibility."""
    del err_type, num_threads
    if not data_tree.N_fields == rand_tree.N_fields:
        raise ValueError("data and random trees must have same number of fields")
    estimator = _estimator(est_type)
    mode = DEFAULT_MODE if mode is None else mode
    radii = np.asarray(radii, dtype="float64")
    dd, dr, rr = _count_binned_batch(
        [(data_tree, data_tree), (rand_tree, data_tree), (rand_tree, rand_tree)], radii, mode)
    return autocorr_results(dd, dr, rr, data_tree, rand_tree, estimator, radii)


def _crosscorr(data_tree_1, data_tree_2, rand_tree_1, rand_tree_2, radii,
               est_type="landy-szalay", num_threads=4, mode=None):
    """D1D2, D1R2, D2R1, R1R2 and a ``crosscorr_results`` (clustering.py:237-291).
    As in the reference, D1D2 and R1R2 query the larger (unique size) tree with
    the other catalog's points."""
    del num_threads
    if not (data_tree_1.N_fields == data_tree_2.N_fields == rand_tree_1.N_fields ==
            rand_tree_2.N_fields):
        raise ValueError("data and random trees must have same number of fields")
    estimator = _estimator(est_type)
    mode = DEFAULT_MODE if mode is None else mode
    radii = np.asarray(radii, dtype="float64")
    if data_tree_1.size > data_tree_2.size:
        dd_job = (data_tree_1, data_tree_2)
    else:
        dd_job = (data_tree_2, data_tree_1)
    if rand_tree_1.size > rand_tree_2.size:
        rr_job = (rand_tree_1, rand_tree_2)
    else:
        rr_job = (rand_tree_2, rand_tree_1)
    d1d2, d1r2, d2r1, r1r2 = _count_binned_batch(
        [dd_job, (rand_tree_2, data_tree_1), (rand_tree_1, data_tree_2), rr_job], radii, mode)
    return crosscorr_results(d1d2, d1r2, d2r1, r1r2, data_tree_1, data_tree_2, rand_tree_1,
                             rand_tree_2, estimator, radii)


# ----------------------------------------------------------------- results

class results(object):
    """Pair-count arrays (bins, F, F) with estimators and errors
    (clustering.py:354-634)."""

    def __init__(self, estimator, radii):
        self.estimator = estimator
        self.nbins = len(radii) - 1
        self.radii_euclidean = radii
        self.radii_nominal = None
        self.radii_units = None
        self.error_type = None

    # pair counts -----------------------------------------------------------
    def total_pair_counts(self, normalized):
        cts = [np.sum(arr, axis=(1, 2)) for arr in self.count_arrays]
        if normalized:
            cts = [arr.astype("float64") for arr in cts]
            for arr, (a, b) in zip(cts, self.count_sizes):
                arr /= _grid_sum(a, b)
        return cts

    def ftf_pair_counts(self, fid, normalized):
        cts = [np.copy(arr[:, fid, fid]) for arr in self.count_arrays]
        if normalized:
            cts = [arr.astype("float64") for arr in cts]
            for arr, (a, b) in zip(cts, self.count_sizes):
                arr /= float(a[fid] * b[fid])
        return cts

    def jackknife_pair_counts(self, fid, normalized):
        kept = []
        for arr in self.count_arrays:
            c = np.copy(arr)
            c[:, fid, :] = 0
            c[:, :, fid] = 0
            kept.append(np.sum(c, axis=(1, 2)))
        if normalized:
            kept = [arr.astype("float64") for arr in kept]
            for arr, (a, b) in zip(kept, self.count_sizes):
                a, b = np.copy(a), np.copy(b)
                a[fid] = 0
                b[fid] = 0
                arr /= _grid_sum(a, b).astype("float64")
        return kept

    def _jackknife_all(self, normalized):
        """``jackknife_pair_counts(f, normalized)`` for every field f at once,
        as (bins, F) arrays.  The counts kept without field f are total - row
        f - column f + cell (f, f), and the normalisation is the product of
        the field-size sums without f: both exact integers (int64), so every
        element equals the per-field method's, which zeroes a copy and sums
        it (clustering.py:457-491).  Integer count arrays only."""
        out = []
        for arr, (a, b) in zip(self.count_arrays, self.count_sizes):
            tot = np.sum(arr, axis=(1, 2))
            kept = (tot[:, np.newaxis] - np.sum(arr, axis=2) - np.sum(arr, axis=1) +
                    np.diagonal(arr, axis1=1, axis2=2))
            if normalized:
                a = np.asarray(a, dtype=np.int64)
                b = np.asarray(b, dtype=np.int64)
                den = (np.sum(a) - a) * (np.sum(b) - b)
                kept = kept.astype("float64") / den.astype("float64")[np.newaxis, :]
            out.append(kept)
        return out

    def bootstrap_pair_counts(self, N_trials):
        """Estimator inputs for N_trials field resamplings (numpy's global
        random state, as in clustering.py:416-455): (bins, N_trials) each."""
        nf = self.N_fields
        draws = np.random.randint(0, nf, N_trials * nf).reshape(N_trials, nf)
        hists = np.apply_along_axis(np.bincount, 1, draws, minlength=nf)
        freqs = np.apply_along_axis(lambda h: np.multiply(*np.meshgrid(h, h)), 1, hists)
        normed = [arr / _grid_sum(a, b).astype("float64")
                  for arr, (a, b) in zip(self.count_arrays, self.count_sizes)]
        return [np.tensordot(arr, freqs, axes=((1, 2), (1, 2))) for arr in normed]

    # errors ------------------------------------------------------------------
    def _need_fields(self, what):
        if self.N_fields <= 1:
            raise ValueError("{:s} cannot be calculated without data fields".format(what))

    def bootstrap_error(self, N_trials=1000):
        self._need_fields("Bootstrap error")
        est = self.estimator(*self.bootstrap_pair_counts(N_trials))
        return np.std(est, axis=1)

    def jackknife_error(self):
        self._need_fields("Jackknife error")
        return np.sqrt(np.diagonal(self.covariance("jackknife", normalized=False)))

    def ftf_error(self):
        self._need_fields("field-to-field error")
        return np.sqrt(np.diagonal(self.covariance("ftf", normalized=False)))

    def poisson_error(self):
        tot = self.total_pair_counts(normalized=False)
        with np.errstate(divide="ignore", invalid="ignore"):
            err = np.divide(1 + self.estimate(), np.sqrt(tot[0]))
            err[np.isneginf(err)] = np.nan
            err[np.isinf(err)] = np.nan
        return err

    def estimate(self):
        return self.estimator(*self.total_pair_counts(normalized=True))

    def covariance(self, error_type, normalized=False):
        """Jackknife or field-to-field covariance of the estimator
        (clustering.py:520-558): sum over fields of
        sqrt(RR_k / RR) (xi_k - xi) outer the same; ftf divides by F-1."""
        self._need_fields("Covariance matrix")
        jack = error_type in ("jackknife", "jk")
        ftf = error_type in ("field-to-field", "ftf")
        cov = np.zeros((self.nbins, self.nbins))
        xi = self.estimate()
        tot_rr = self.total_pair_counts(normalized=False)[-1].astype("float64")
        if jack and all(np.issubdtype(np.asarray(c).dtype, np.integer)
                        for c in self.count_arrays):
            # all fields at once (elementwise, so bit-identical to the loop
            # below); the sum over fields keeps its order
            est = self.estimator(*self._jackknife_all(normalized=True))
            raw = self._jackknife_all(normalized=False)[-1]
            diffs = est - xi[:, np.newaxis]
            ws = np.sqrt(raw / tot_rr[:, np.newaxis])
            for fid in range(self.N_fields):
                diff, w = diffs[:, fid], ws[:, fid]
                cov += (w * diff)[np.newaxis, :] * w[:, np.newaxis] * diff[:, np.newaxis]
            if normalized:
                sig = np.sqrt(np.diagonal(cov))
                return np.divide(cov, sig[np.newaxis, :] * sig[:, np.newaxis])
            return cov
        for fid in range(self.N_fields):
            if jack:
                norm = self.jackknife_pair_counts(fid, normalized=True)
                raw = self.jackknife_pair_counts(fid, normalized=False)
            elif ftf:
                norm = self.ftf_pair_counts(fid, normalized=True)
                raw = self.ftf_pair_counts(fid, normalized=False)
            diff = self.estimator(*norm) - xi
            w = np.sqrt(raw[-1] / tot_rr)
            # element (i, j) = ((w_j d_j) w_i) d_i, the reference's product order
            cov += (w * diff)[np.newaxis, :] * w[:, np.newaxis] * diff[:, np.newaxis]
        if ftf:
            cov /= float(self.N_fields - 1)
        if normalized:
            sig = np.sqrt(np.diagonal(cov))
            return np.divide(cov, sig[np.newaxis, :] * sig[:, np.newaxis])
        return cov

    def error(self, error_type):
        if error_type == "poisson":
            return self.poisson_error()
        if error_type in ("jackknife", "jk"):
            return self.jackknife_error()
        if error_type in ("field-to-field", "ftf"):
            return self.ftf_error()
        if error_type == "bootstrap":
            return self.bootstrap_error()
        return None

    def __str__(self):
        lo, hi = self.radii_nominal[:-1], self.radii_nominal[1:]
        cts = self.total_pair_counts(normalized=False)
        est = self.estimate()
        err = self.error(self.error_type)
        if err is None:
            err = [None] * len(est)
        widths = [max([len(str(c)) for c in ct] + [4]) + 2 for ct in cts]
        names = (["DD", "DR", "RR"] if len(cts) == 3 else ["D1D2", "D1R2", "D2R1", "R1R2"])
        labels = ["Bin L", "Bin R"] + names + ["Estimator", "Error"]
        sizes = [9, 9] + widths + [11, 10]
        lines = ["\n", "".join(l.ljust(s) for l, s in zip(labels, sizes)),
                 "{:^14}".format("({:s})".format(self.radii_units)), "-" * 79]
        for rl, ru, e, er, row in zip(lo, hi, est, err, zip(*cts)):
            cells = ["{:<9}".format("{:.2E}".format(rl)), "{:<9}".format("{:.2E}".format(ru))]
            cells += ["{:<{:d}}".format(c, w) for c, w in zip(row, widths)]
            cells += ["{:<11}".format("{:+.2E}".format(e)),
                      "{:<10}".format(str(None) if er is None else "{:.2E}".format(er))]
            lines.append("".join(cells))
        return "\n".join(lines)


class autocorr_results(results):
    """DD, DR, RR (clustering.py:636-651)."""

    def __init__(self, dd, dr, rr, dtree, rtree, estimator, radii):
        self.dd, self.dr, self.rr = dd, dr, rr
        self.N_fields = dtree.N_fields
        self.count_arrays = [self.dd, self.dr, self.rr]
        d, r = dtree.field_sizes, rtree.field_sizes
        self.count_sizes = [(np.copy(d), np.copy(d)), (np.copy(d), np.copy(r)),
                            (np.copy(r), np.copy(r))]
        super(autocorr_results, self).__init__(estimator, radii)


class crosscorr_results(results):
    """D1D2, D1R2, D2R1, R1R2 (clustering.py:653-672)."""

    def __init__(self, d1d2, d1r2, d2r1, r1r2, dtree_1, dtree_2, rtree_1, rtree_2, estimator,
                 radii):
        self.d1d2, self.d1r2, self.d2r1, self.r1r2 = d1d2, d1r2, d2r1, r1r2
        self.N_fields = dtree_1.N_fields
        self.count_arrays = [self.d1d2, self.d1r2, self.d2r1, self.r1r2]
        sz = [t.field_sizes for t in (dtree_1, dtree_2, rtree_1, rtree_2)]
        self.count_sizes = [(np.copy(sz[0]), np.copy(sz[1])), (np.copy(sz[0]), np.copy(sz[3])),
                            (np.copy(sz[1]), np.copy(sz[2])), (np.copy(sz[2]), np.copy(sz[3]))]
        super(crosscorr_results, self).__init__(estimator, radii)
