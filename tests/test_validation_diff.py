"""The reference's own Python functions run side by side with ours (its
package imported from a temporary copy, as tests/golden/make_golden.py does;
skipped where the reference or its build is absent).

Input validation: same result arrays and dtypes, same copy warnings, same
exception types and messages, for well-formed and malformed inputs.
Results classes: random count arrays of several field and bin counts, auto
and cross, give the same estimates, errors (bootstrap seeded), covariances
and printed tables, bit for bit."""
import importlib.util
import os
import warnings

import numpy as np
import pytest

from corruscant_b200 import clustering
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = O.reference_root()

pytestmark = pytest.mark.skipif(
    not (O.ref_available() and REF_ROOT and os.path.isdir(os.path.join(REF_ROOT, "corruscant"))),
    reason="reference sources or oracle/_ref absent")


@pytest.fixture(scope="module")
def ref():
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg._ref_python(REF_ROOT)


def _outcome(fn, *args):
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        try:
            r = fn(*args)
            res = ("ok", np.asarray(r).dtype.str, np.asarray(r).shape, np.asarray(r).tobytes())
        except Exception as e:  # compared below
            res = ("raise", type(e).__name__, str(e))
    return res, sorted((x.category.__name__, str(x.message)) for x in w)


rs = np.random.RandomState(52)
POINTS = {
    "n3": rs.rand(10, 3),
    "3n": rs.rand(3, 10),
    "3x3": rs.rand(3, 3),
    "n4": rs.rand(10, 4),
    "fortran": np.asfortranarray(rs.rand(10, 3)),
    "strided": rs.rand(20, 3)[::2],
    "list": rs.rand(4, 3).tolist(),
    "int": rs.randint(0, 9, (6, 3)),
    "float32": rs.rand(6, 3).astype(np.float32),
    "one": rs.rand(1, 3),
    "flat": rs.rand(9),
}
FIELDS = {
    "ok": lambda n: (np.arange(n) % 3),
    "list": lambda n: [i % 2 for i in range(n)],
    "float": lambda n: np.arange(n) * 0.5,
    "short": lambda n: np.arange(max(n - 1, 0)),
    "2d": lambda n: np.zeros((n, 1)),
    "int64": lambda n: np.arange(n, dtype=np.int64) % 4,
}


@pytest.mark.parametrize("name", sorted(POINTS))
def test_validate_points_like_reference(ref, name):
    assert _outcome(clustering.validate_points, POINTS[name]) == \
        _outcome(ref.validate_points, POINTS[name])


@pytest.mark.parametrize("fname", sorted(FIELDS))
def test_validate_fields_like_reference(ref, fname):
    pts = np.ascontiguousarray(rs.rand(12, 3))
    f = FIELDS[fname](12)
    assert _outcome(clustering.validate_fields, f, pts) == _outcome(ref.validate_fields, f, pts)


def _tree_attrs(sizes):
    import types
    return types.SimpleNamespace(N_fields=len(sizes), field_sizes=np.asarray(sizes))


@pytest.mark.parametrize("F,nb,cross", [(2, 1, False), (5, 4, False), (13, 9, False),
                                        (3, 5, True), (8, 2, True)])
def test_results_like_reference(ref, F, nb, cross):
    """Random count arrays through our results classes and the reference's:
    every estimator x error type, covariances and tables, bit for bit."""
    g = np.random.RandomState(100 + F * 10 + nb)
    n = 4 if cross else 3
    arrays = [g.randint(0, 10 ** k, (nb, F, F)).astype(np.int64) for k in (4, 5, 6, 7)[:n]]
    arrays[-1] += 1
    sizes = [g.randint(1, 10 ** 4, F) for _ in range(4)]
    trees = [_tree_attrs(s) for s in sizes]
    radii = np.logspace(-2, -1, nb + 1)
    objs = []
    for mod in (clustering, ref):
        if cross:
            r = mod.crosscorr_results(*[a.copy() for a in arrays], *trees, mod.est_landy_szalay,
                                      radii)
        else:
            r = mod.autocorr_results(*[a.copy() for a in arrays], trees[0], trees[1],
                                     mod.est_landy_szalay, radii)
        r.radii_nominal, r.radii_units = radii, "Data units"
        objs.append((mod, r))
    for est in ("est_standard", "est_hamilton", "est_landy_szalay"):
        outs = []
        for mod, r in objs:
            r.estimator = getattr(mod, est)
            o = [_outcome(r.estimate)]
            for err in (None, "poisson", "ftf", "jackknife", "bootstrap"):
                np.random.seed(5)
                o.append(_outcome(r.error, err))
                r.error_type = err
                np.random.seed(5)
                o.append(_outcome(str, r))
            for kind in ("jackknife", "ftf"):
                for norm in (False, True):
                    o.append(_outcome(r.covariance, kind, norm))
            outs.append(o)
        assert outs[0] == outs[1], est
