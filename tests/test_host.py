"""Host-side checks that need no GPU: the C ABI libraries load and export what
include/*.h declares, the estimator/error/covariance arithmetic matches the
reference's own outputs to 0 ulp, input validation behaves like the
reference, and the coordinate conversions are bit-identical."""
import ctypes
import os
import re
import types

import numpy as np
import pytest

from conftest import REPO
from corruscant_b200 import _native, clustering, twopoint


def _declared(header):
    """Function names declared in a C header (prototype lines)."""
    src = open(os.path.join(REPO, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "sizeof")))


@pytest.mark.parametrize("lib,header", [("libkdtree", "kdtree.h"), ("libcoords", "coordmath.h")])
def test_library_exports_every_declared_symbol(lib, header):
    names = _declared(header)
    assert names, header
    L = ctypes.CDLL(os.path.join(REPO, "corruscant_b200", "bin", lib + ".so"))
    for name in names:
        assert hasattr(L, name), (lib, name)


def test_reference_abi_struct_sizes():
    assert ctypes.sizeof(_native.KdTree) == 64
    assert ctypes.sizeof(_native.Node) == 40
    assert ctypes.sizeof(_native.Datum) == 32


def _fake_tree(fields, n_fields):
    return types.SimpleNamespace(N_fields=n_fields,
                                 field_sizes=np.array([np.sum(fields == i) for i in range(n_fields)]))


def _assert_bits(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.int64), b.view(np.int64)), (a, b)


def _check_estimators(res, g):
    _assert_bits(res.estimate(), g["xi"])
    _assert_bits(res.error("jackknife"), g["err_jackknife"])
    _assert_bits(res.error("ftf"), g["err_ftf"])
    _assert_bits(res.error("poisson"), g["err_poisson"])
    _assert_bits(res.covariance("jackknife"), g["cov_jackknife"])
    _assert_bits(res.covariance("jackknife", normalized=True), g["cov_jackknife_norm"])
    _assert_bits(res.covariance("ftf"), g["cov_ftf"])
    np.random.seed(11)
    _assert_bits(res.error("bootstrap"), g["err_bootstrap_seed11"])


def test_autocorr_estimators_match_reference_to_0ulp(golden):
    g = golden("config1.npz")
    np.random.seed(3)
    X = np.random.rand(4000, 3)
    Y = np.random.rand(80000, 3)
    fd = (X[:, 0] * 4).astype("int32")
    fr = (Y[:, 0] * 4).astype("int32")
    res = clustering.autocorr_results(g["dd"], g["dr"], g["rr"], _fake_tree(fd, 4),
                                      _fake_tree(fr, 4), clustering.est_landy_szalay, g["radii"])
    _check_estimators(res, g)
    for est in ("standard", "hamilton"):
        res.estimator = getattr(clustering, "est_" + est)
        _assert_bits(res.estimate(), g["xi_" + est])
        _assert_bits(res.error("jackknife"), g["err_jackknife_" + est])


def test_crosscorr_estimators_match_reference_to_0ulp(golden):
    g = golden("cross.npz")
    rs = np.random.RandomState(int(g["seed"]))
    cats = [rs.rand(int(n), 3) for n in g["sizes"]]
    fakes = [_fake_tree((c[:, 0] * 4).astype("int32"), 4) for c in cats]
    res = clustering.crosscorr_results(g["d1d2"], g["d1r2"], g["d2r1"], g["r1r2"], *fakes,
                                       clustering.est_landy_szalay, g["radii"])
    _check_estimators(res, g)


@pytest.mark.parametrize("est", ["landy-szalay", "hamilton", "standard"])
@pytest.mark.parametrize("cross", [False, True])
def test_jackknife_covariance_at_100_fields_equals_the_per_field_loop(est, cross):
    """The all-fields jackknife covariance (exact integer counts kept per
    field) is bit for bit the reference's loop over fields built on
    jackknife_pair_counts(f) (clustering.py:520-558), at F = 100."""
    rs = np.random.RandomState(21 + cross)
    F, nb = 100, 15
    arrays = [rs.randint(0, 10 ** k, (nb, F, F)).astype(np.int64) for k in (5, 6, 7, 8)]
    arrays = arrays if cross else arrays[:3]
    arrays[-1] += 1
    s = [rs.randint(1, 10 ** 5, F) for _ in range(4)]
    res = clustering.results.__new__(clustering.results)
    clustering.results.__init__(res, clustering._estimator(est), np.logspace(-3, 0, nb + 1))
    res.count_arrays, res.N_fields = arrays, F
    res.count_sizes = ([(s[0], s[1]), (s[0], s[3]), (s[1], s[2]), (s[2], s[3])] if cross
                       else [(s[0], s[0]), (s[0], s[1]), (s[1], s[1])])
    xi = res.estimate()
    tot_rr = res.total_pair_counts(normalized=False)[-1].astype("float64")
    want = np.zeros((nb, nb))
    for fid in range(F):
        diff = res.estimator(*res.jackknife_pair_counts(fid, normalized=True)) - xi
        w = np.sqrt(res.jackknife_pair_counts(fid, normalized=False)[-1] / tot_rr)
        want += (w * diff)[np.newaxis, :] * w[:, np.newaxis] * diff[:, np.newaxis]
    _assert_bits(res.covariance("jackknife"), want)
    sig = np.sqrt(np.diagonal(want))
    _assert_bits(res.covariance("jackknife", normalized=True),
                 np.divide(want, sig[np.newaxis, :] * sig[:, np.newaxis]))


def test_results_table_prints():
    dd = np.arange(1, 9).reshape(2, 2, 2)
    res = clustering.autocorr_results(dd, dd + 1, dd + 2, _fake_tree(np.array([0, 1]), 2),
                                      _fake_tree(np.array([0, 1]), 2),
                                      clustering.est_landy_szalay, np.array([0.1, 0.2, 0.3]))
    res.radii_nominal = res.radii_euclidean
    res.radii_units = "Data units"
    res.error_type = "jackknife"
    text = str(res)
    assert "Bin L" in text and "Estimator" in text and len(text.splitlines()) == 7


def test_validation_like_reference():
    with pytest.raises(ValueError):
        clustering.validate_points(np.zeros((5, 4)))
    with pytest.warns(RuntimeWarning):
        p = clustering.validate_points(np.zeros((3, 10)))
    assert p.shape == (10, 3)
    with pytest.raises(ValueError):
        clustering.validate_fields(np.zeros(9), p)
    assert clustering.validate_fields(np.zeros(10), p).dtype == np.int32
    with pytest.raises(ValueError):
        clustering._estimator("no-such-estimator")


def test_coordinates_bit_identical_to_reference(golden):
    c = golden("coords.npz")
    _assert_bits(twopoint.angular.cartesian(c["ra"], c["dec"]), c["xyz"])
    _assert_bits(twopoint.threedim.cartesian(c["ra"], c["dec"], c["dist"]), c["xyzd"])


def test_spherical_coordinates_bit_identical_to_reference(golden):
    """radec2sph64 (coordmath.c:73-80) of libcoords.so."""
    c = golden("coords.npz")
    ra = np.require(c["ra"], dtype=np.float64, requirements="AC")
    dec = np.require(c["dec"], dtype=np.float64, requirements="AC")
    theta, phi = np.empty(ra.size), np.empty(ra.size)
    _native.coordlib().radec2sph64(_native.dptr(ra), _native.dptr(dec), _native.dptr(theta),
                                   _native.dptr(phi), ra.size)
    _assert_bits(theta, c["theta"])
    _assert_bits(phi, c["phi"])


def test_cartesian_from_redshift_and_cosmology():
    """threedim.cartesian with z and a cosmology object (anything with
    comoving_distance, as astropy's; threedim.py:78-81) equals the call with
    those distances."""
    class Cosmology:
        def comoving_distance(self, z):
            return 2997.92458 * z / (1.0 + 0.3 * z)

    rs = np.random.RandomState(50)
    ra, dec, z = rs.rand(500) * 360, rs.rand(500) * 180 - 90, rs.rand(500) * 2
    _assert_bits(twopoint.threedim.cartesian(ra, dec, z=list(z), cosmology=Cosmology()),
                 twopoint.threedim.cartesian(ra, dec, Cosmology().comoving_distance(z)))
    # a given distance takes precedence over a redshift
    d = rs.rand(500) * 100
    _assert_bits(twopoint.threedim.cartesian(ra, dec, d, z=z, cosmology=Cosmology()),
                 twopoint.threedim.cartesian(ra, dec, d))


# every public name of the reference package (corruscant/__init__.py,
# clustering.py, twopoint/angular.py, twopoint/threedim.py) and the methods
# of its classes
REFERENCE_API = {
    "": ["PROJECT_PATH", "loadlib", "kdlib", "coordlib", "clustering", "twopoint"],
    "clustering": ["node", "datum", "kdtree", "kdlib", "_query_tree", "validate_points",
                   "validate_fields", "est_landy_szalay", "est_hamilton", "est_standard",
                   "_autocorr", "_crosscorr", "tree", "results", "autocorr_results",
                   "crosscorr_results"],
    "twopoint.angular": ["coordlib", "autocorr", "crosscorr", "cartesian"],
    "twopoint.threedim": ["coordlib", "autocorr", "crosscorr", "cartesian"],
}
REFERENCE_METHODS = {
    "tree": ["_calc_field_sizes", "_make_tree", "__del__"],
    "results": ["total_pair_counts", "ftf_pair_counts", "jackknife_pair_counts",
                "bootstrap_pair_counts", "bootstrap_error", "jackknife_error", "ftf_error",
                "poisson_error", "estimate", "covariance", "error", "__str__"],
}


def test_reference_api_names_exist():
    import importlib
    for mod, names in REFERENCE_API.items():
        m = importlib.import_module("corruscant_b200" + ("." + mod if mod else ""))
        for n in names:
            assert getattr(m, n, None) is not None, (mod, n)
    for cls, methods in REFERENCE_METHODS.items():
        for n in methods:
            assert callable(getattr(getattr(clustering, cls), n, None)), (cls, n)
    import corruscant_b200
    assert corruscant_b200.kdlib.tree_construct.restype is clustering.kdtree
    assert ctypes.sizeof(clustering.kdtree) == 64 and ctypes.sizeof(clustering.node) == 40
    assert corruscant_b200.coordlib is twopoint.angular.coordlib
    with pytest.raises(AttributeError):
        corruscant_b200.not_a_name


def test_chord_edges_are_the_reference_expression():
    deg = np.logspace(-3, np.log10(2.0), 16)
    _assert_bits(twopoint.angular.chord(deg), 2. * np.sin(deg * (np.pi / 180.) / 2.))


def test_set_precision_validates_mode():
    """kd_set_precision is host-only state for pair_count; unknown modes are
    refused with an error instead of being stored."""
    from corruscant_b200 import _native as N
    N.set_precision(N.KD_MODE_FP64)
    N.set_precision(N.KD_MODE_MIXED)
    with pytest.raises(N.NativeError):
        N.set_precision(7)
