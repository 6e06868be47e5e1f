"""Limits, degenerate inputs, concurrency and medium-size properties of the
counts through the C ABI."""
import threading

import numpy as np
import pytest

from corruscant_b200 import _native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _clustered(rs, n, nparents, sigma):
    c = rs.rand(nparents, 3)
    return (c[rs.randint(0, nparents, n)] + rs.normal(0, sigma, (n, 3))) % 1.0


def test_64_distinct_edges_in_one_pass_65_in_two():
    rs = np.random.RandomState(41)
    p = rs.rand(20000, 3)
    t = N.build_tree(p, None, 1)
    try:
        radii = np.linspace(0.001, 0.2, 64)
        want = O.OracleTree(p).brute_counts(p, None, 1, radii, nthreads=8)
        for mode in (N.KD_MODE_MIXED, N.KD_MODE_FP64):
            assert np.array_equal(N.count_radii(t, t, radii, mode=mode), want)
        # repeated radii do not count toward the limit and get the same rows
        rep = np.concatenate([radii, radii[::7]])
        assert np.array_equal(N.count_radii(t, t, rep), np.concatenate([want, want[::7]]))
        # a 65th distinct radius takes a second pass over the trees
        r65 = np.linspace(0.001, 0.2, 65)
        got, st = N.count_radii(t, t, r65, with_stats=True)
        assert np.array_equal(got, O.OracleTree(p).brute_counts(p, None, 1, r65, nthreads=8))
        assert st["tile_launches"] >= 2
    finally:
        N.destroy(t)


def test_empty_and_degenerate_inputs():
    rs = np.random.RandomState(42)
    t = N.build_tree(rs.rand(500, 3), None, 1)
    one = N.build_tree(np.array([[0.3, 0.4, 0.5]]), None, 1)
    try:
        assert np.array_equal(N.count_points(t, np.empty((0, 3)), None, 1, [0.1]), [[0]])
        assert N.count_radii(t, t, []).shape == (0, 1)
        assert np.array_equal(N.count_radii(t, t, [np.nan, np.nan]), [[0], [0]])
        nan_q = np.full((3, 3), np.nan)
        assert np.array_equal(N.count_points(t, nan_q, None, 1, [0.5, np.inf]), [[0], [0]])
        # a single point against itself: d2 = 0 counts only where fl(r*r) > 0
        got = N.count_radii(one, one, [0.0, 1e-300, 1e-100, np.inf])
        assert np.array_equal(got, [[0], [0], [1], [1]])
    finally:
        N.destroy(t)
        N.destroy(one)


def test_concurrent_counts_from_threads():
    """The C ABI is reentrant (one stream per call): counts issued from several
    host threads at once equal the same counts issued one after another."""
    rs = np.random.RandomState(43)
    a = N.build_tree(_clustered(rs, 60000, 300, 0.01), None, 1)
    b = N.build_tree(rs.rand(120000, 3), None, 1)
    radii = np.logspace(-2.5, -1, 9)
    jobs = [(a, a), (b, a), (b, b), (a, b)] * 2
    try:
        want = [N.count_radii(t, q, radii) for t, q in jobs]
        got = [None] * len(jobs)
        errors = []

        def run(i):
            try:
                t, q = jobs[i]
                got[i] = N.count_radii(t, q, radii, mode=i % 2)
            except Exception as exc:  # reported below
                errors.append(exc)

        threads = [threading.Thread(target=run, args=(i,)) for i in range(len(jobs))]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        assert not errors
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
    finally:
        N.destroy(a)
        N.destroy(b)


@pytest.mark.parametrize("offset", [1.0e6, -3.0e4])
def test_far_from_origin(offset):
    """Coordinates of ~1e6 with separations of ~1e-4: FP32 values of the
    coordinates themselves would be useless here; the tile kernel works on
    block-relative coordinates and must still count exactly."""
    rs = np.random.RandomState(46)
    p = offset + rs.rand(20000, 3) * 0.01
    f = (rs.rand(len(p)) * 3).astype(np.int32)
    t = N.build_tree(p, f, 3)
    try:
        radii = np.array([1e-4, 3e-4, 1e-3, 2e-3, 5e-3])
        want = O.OracleTree(p, f, 3).brute_counts(p, f, 3, radii, nthreads=8)
        for mode in (N.KD_MODE_MIXED, N.KD_MODE_FP64):
            assert np.array_equal(N.count_radii(t, t, radii, mode=mode), want)
    finally:
        N.destroy(t)


def test_every_point_three_times():
    """The reference's test/test_duplicates.py shape: 30,000 points each
    repeated three times build a tree of 30,000 unique points (weight 3 each,
    kdbuild.c:472-511); counts of a query sample equal the oracle's."""
    from corruscant_b200 import clustering
    rs = np.random.RandomState(47)
    X = np.repeat(rs.rand(30000, 3), 3, axis=0)
    f = (X[:, 0] * 4).astype(np.int32)
    t = clustering.tree(X, f)
    assert t.size == 30000 and t.N_fields == 4
    assert np.array_equal(t.field_sizes, np.bincount(f, minlength=4))
    idx = np.sort(rs.choice(len(X), 500, replace=False))
    radii = np.array([0.0, 0.005, 0.02, 0.06])
    got = N.count_points(t.ctree, X[idx], f[idx], 4, radii)
    want = O.OracleTree(X, f, 4).brute_counts(X[idx], f[idx], 4, radii, nthreads=8)
    assert np.array_equal(got, want)
    assert np.all(got[1:].sum(axis=1) >= 3 * len(idx))  # each query meets its 3 copies


def test_fields_above_255_follow_the_reference():
    """The tree side keeps the low 8 bits of a field id (kdtree.h field:8), the
    query side the full id; an autocorrelation with such fields is counted the
    ordered way and matches the oracle."""
    rs = np.random.RandomState(44)
    p = rs.rand(30000, 3)
    f = rs.randint(0, 300, len(p)).astype(np.int32)
    t = N.build_tree(p, f, 300)
    try:
        radii = np.array([0.0, 0.01, 0.03, 0.08])
        want = O.OracleTree(p, f, 300).brute_counts(p, f, 300, radii, nthreads=8)
        assert np.array_equal(N.count_radii(t, t, radii), want)
    finally:
        N.destroy(t)


def test_medium_scale_properties():
    """100k clustered data and 2M randoms (the clustered workload at 1/10):
    mixed == FP64 for the whole DD + DR + RR batch, symmetric == ordered,
    shards sum to the batch, and a query sample equals the oracle's traversal."""
    rs = np.random.RandomState(45)
    d = _clustered(rs, 100000, 1000, 0.005)
    r = rs.rand(2_000_000, 3)

    def fields(x):
        return (16 * np.floor(4 * x[:, 0]) + 4 * np.floor(4 * x[:, 1]) +
                np.floor(4 * x[:, 2])).astype(np.int32)
    fd, fr = fields(d), fields(r)
    td, tr, tr2 = N.build_tree(d, fd, 64), N.build_tree(r, fr, 64), N.build_tree(r, fr, 64)
    radii = np.logspace(-3, -1, 21)
    jobs = [(td, td), (tr, td), (tr, tr)]
    try:
        mixed = N.count_batch(jobs, radii, mode=N.KD_MODE_MIXED)
        fp64 = N.count_batch(jobs, radii, mode=N.KD_MODE_FP64)
        for m, f in zip(mixed, fp64):
            assert np.array_equal(m, f)
        assert np.array_equal(mixed[2], N.count_radii(tr, tr2, radii))  # ordered RR
        parts = [N.count_batch(jobs, radii, shard=s, nshards=4) for s in range(4)]
        for j in range(3):
            assert np.array_equal(sum(p[j] for p in parts), mixed[j])
        idx = np.sort(rs.choice(len(r), 300, replace=False))
        ot = O.OracleTree(r, fr, 64)
        want = np.stack([ot.pair_count(r[idx], fr[idx], 64, x, nthreads=8) for x in radii])
        assert np.array_equal(N.count_points(tr, r[idx], fr[idx], 64, radii), want)
    finally:
        for x in (td, tr, tr2):
            N.destroy(x)
