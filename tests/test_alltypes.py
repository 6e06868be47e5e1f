"""The workloads of the reference's test/test_alltypes.py (3-D and angular,
auto and cross, with and without fields) and test/angular.py (10k / 200k
points on the sky, RA quadrants as fields): tests/golden/alltypes.npz, made
by tests/golden/make_golden.py from the reference itself.

On the CPU, the results classes fed the reference's counts give every
estimator x error type, the covariances and the printed results tables bit
for bit / character for character.  On the GPU, the whole user API (trees,
batched counts, results) gives the reference's counts and the same values."""
import importlib.util
import os
import types

import numpy as np
import pytest

from corruscant_b200 import clustering, twopoint

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden_module():
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


MG = _golden_module()
CASES = sorted(MG.ALLTYPES_CASES)


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


def _names(kind):
    return ("dd", "dr", "rr") if kind == "auto" else ("d1d2", "d1r2", "d2r1", "r1r2")


def _points(cats):
    return [c[1] if c[0] == "xyz" else twopoint.angular.cartesian(*c[1]) for c in cats]


def _check_values(g, case, res):
    """Every estimator x error type, covariance and table against the golden."""
    with_fields = MG.ALLTYPES_CASES[case]["nfields"] > 0
    for est in MG.ALLTYPES_ESTIMATORS:
        res.estimator = clustering._estimator(est)
        assert np.array_equal(_bits(res.estimate()), _bits(g[f"{case}/xi/{est}"])), est
        for err in MG.ALLTYPES_ERRORS if with_fields else (None, "poisson"):
            if err is not None:
                np.random.seed(11)
                assert np.array_equal(_bits(res.error(err)),
                                      _bits(g[f"{case}/err/{est}/{err}"])), (est, err)
            res.error_type = err
            np.random.seed(11)
            assert str(res) == str(g[f"{case}/table/{est}/{err}"]), (est, err)
        if with_fields:
            assert np.array_equal(_bits(res.covariance("jackknife")),
                                  _bits(g[f"{case}/cov_jackknife/{est}"])), est
            assert np.array_equal(_bits(res.covariance("ftf")),
                                  _bits(g[f"{case}/cov_ftf/{est}"])), est
    if not with_fields:
        for err in ("jackknife", "ftf", "bootstrap"):
            with pytest.raises(ValueError, match="without data fields"):
                res.error(err)


def _fake_tree(points, fields, nf):
    """The tree attributes the results classes read; without fields the
    field size is the unique size (all points are distinct here)."""
    if fields is None:
        return types.SimpleNamespace(N_fields=1, field_sizes=np.array(len(points)))
    return types.SimpleNamespace(N_fields=nf, field_sizes=np.bincount(fields, minlength=nf))


@pytest.mark.parametrize("case", CASES)
def test_alltypes_estimators_from_reference_counts(golden, case):
    g = golden("alltypes.npz")
    c = MG.ALLTYPES_CASES[case]
    kind, geom = c["kind"], c["geom"]
    cats, fields, nominal, radii = MG.alltypes_inputs(case)
    pts = _points(cats)
    assert MG._sha1(*pts, *fields) == str(g[f"{case}/inputs_sha1"])
    fakes = [_fake_tree(p, f, c["nfields"]) for p, f in zip(pts, fields)]
    arrays = [g[f"{case}/{k}"] for k in _names(kind)]
    est = clustering.est_landy_szalay
    if kind == "auto":
        res = clustering.autocorr_results(*arrays, *fakes, est, radii)
    else:
        res = clustering.crosscorr_results(*arrays, *fakes, est, radii)
    res.radii_nominal = radii if geom == "cube" else nominal
    res.radii_units = "Data units" if geom == "cube" else "degrees"
    _check_values(g, case, res)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_alltypes_case_through_the_api(golden, case):
    g = golden("alltypes.npz")
    c = MG.ALLTYPES_CASES[case]
    kind, geom = c["kind"], c["geom"]
    cats, fields, nominal, radii = MG.alltypes_inputs(case)
    pts = _points(cats)
    # the reference's inputs (for the sky, our conversion gives the
    # reference's coordinates bit for bit)
    assert MG._sha1(*pts, *fields) == str(g[f"{case}/inputs_sha1"])
    trees = [clustering.tree(p, f) for p, f in zip(pts, fields)]
    api = twopoint.threedim if geom == "cube" else twopoint.angular
    if kind == "auto":
        res = api.autocorr(*trees, nominal, num_threads=4)
    else:
        res = api.crosscorr(*trees, nominal, num_threads=4)
    assert np.array_equal(res.radii_euclidean, radii)
    for k in _names(kind):
        assert np.array_equal(getattr(res, k), g[f"{case}/{k}"]), k
    _check_values(g, case, res)
