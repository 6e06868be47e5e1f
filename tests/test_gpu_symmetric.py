"""Autocorrelation counts (one tree on both sides) count each unordered pair
once and credit both orientations.  They must equal the ordered count of the
same points exactly; a second handle built from the same points is a
different catalog and is counted the ordered way."""
import numpy as np
import pytest

from corruscant_b200 import _native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = (N.KD_MODE_MIXED, N.KD_MODE_FP64)


def _fields(p, nf):
    return (p[:, 0] * nf).astype(np.int32).clip(0, nf - 1) if nf > 1 else None


def _pair(points, nf):
    points = np.ascontiguousarray(points, dtype=np.float64)
    f = _fields(points, nf)
    return N.build_tree(points, f, nf), N.build_tree(points, f, nf), f


def _clustered(rs, n, nparents, sigma):
    c = rs.rand(nparents, 3)
    return (c[rs.randint(0, nparents, n)] + rs.normal(0, sigma, (n, 3))) % 1.0


CASES = {
    "clustered_dups": lambda rs: np.concatenate([_clustered(rs, 60000, 300, 0.01)] * 2)[
        rs.permutation(120000)[:80000]],
    "uniform": lambda rs: rs.rand(150000, 3),
    "lattice": lambda rs: rs.randint(0, 48, (40000, 3)) / 48.0,
    "tiny": lambda rs: rs.rand(3, 3),
    "one_point_255_times": lambda rs: np.tile(rs.rand(1, 3), (255, 1)),
}


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", sorted(CASES))
def test_symmetric_equals_ordered(case, mode):
    rs = np.random.RandomState(31)
    pts = CASES[case](rs)
    nf = 1 if case.startswith("tiny") else 5
    radii = (np.sqrt(np.array([1, 2, 3, 5, 8, 13, 21, 50, 100])) / 48.0 if case == "lattice"
             else np.array([0.0, 0.003, 0.01, 0.02, 0.05, 0.1, np.inf]))
    a, b, f = _pair(pts, nf)
    try:
        got, st = N.count_radii(a, a, radii, mode=mode, with_stats=True)  # symmetric
        want, st2 = N.count_radii(a, b, radii, mode=mode, with_stats=True)  # ordered
        assert np.array_equal(got, want)
        if len(pts) > 1000:
            assert st["pairs_tested"] < 0.75 * st2["pairs_tested"]
        if len(pts) <= 40000:
            brute = O.OracleTree(pts, f, nf).brute_counts(pts, f, nf, radii, nthreads=8)
            assert np.array_equal(got, brute)
    finally:
        N.destroy(a)
        N.destroy(b)


def test_symmetric_shards_and_batch():
    rs = np.random.RandomState(32)
    p = _clustered(rs, 70000, 200, 0.02)
    a, b, _ = _pair(p, 4)
    r = rs.rand(90000, 3)
    fr = _fields(r, 4)
    t, t2 = N.build_tree(r, fr, 4), N.build_tree(r, fr, 4)
    radii = np.logspace(-2.5, -0.8, 9)
    try:
        want_dd = N.count_radii(a, b, radii)
        want_rr = N.count_radii(t, t2, radii)
        for nshards in (1, 3):
            dd = sum(N.count_radii_shard(a, a, radii, s, nshards) for s in range(nshards))
            assert np.array_equal(dd, want_dd), nshards
        dd, dr, rr = N.count_batch([(a, a), (t, a), (t, t)], radii)
        assert np.array_equal(dd, want_dd)
        assert np.array_equal(dr, N.count_radii(t, a, radii))
        assert np.array_equal(rr, want_rr)
    finally:
        for x in (a, b, t, t2):
            N.destroy(x)
