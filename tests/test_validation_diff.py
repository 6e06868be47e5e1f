"""Input validation behaves like the reference's own functions, run side by
side (the reference's Python package imported from a temporary copy, as
tests/golden/make_golden.py does; skipped where the reference or its build
is absent): same result arrays and dtypes, same copy warnings, same
exception types and messages, for well-formed and malformed inputs."""
import importlib.util
import os
import warnings

import numpy as np
import pytest

from corruscant_b200 import clustering
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = "/root/reference"

pytestmark = pytest.mark.skipif(
    not (O.ref_available() and os.path.isdir(os.path.join(REF_ROOT, "corruscant"))),
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
