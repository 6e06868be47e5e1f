"""Every benchmark workload, at a reduced scale, counted on the GPU and
checked count for count against the oracle; plus the ranges the workloads do
not reach: any number of radii, coordinates and radii from 1e15 to 1e300, and
a 5M-point tree node for node.

The workloads are the benchmark's own generators (bench.WORKLOADS): the
clustered 3-D autocorrelation, the angular sky patch with 100 quantile fields,
the batch of mock catalogs against shared randoms, and the lattice stress
cross-correlation with edges exactly on lattice distances and 10% duplicated
rows.  Each is counted as the benchmark counts it, every count of the
workload in one kd_count_batch (DD and RR symmetric), in both precisions, and
compared with the oracle's exhaustive counts (the reference traversal,
kdquery.c:62-113, pruned at the largest radius and binned into every radius:
or_tree_counts).  One count per workload is also compared with the
unmodified reference library (oracle/_ref) on a seeded query subset, one
pair_count per radius as clustering.py:218-230 drives it.
"""
import os

import numpy as np
import pytest

import bench
from corruscant_b200 import _native as N
from corruscant_b200 import clustering
from corruscant_b200.twopoint import threedim
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NTH = os.cpu_count() or 4
SCALES = {"clustered3d": 0.02, "angular": 0.02, "mocks": 0.02, "lattice": 0.05}


def _oracle_counts(w):
    trees, want = {}, {}
    for name, t, q in w.jobs:
        if t not in trees:
            trees[t] = O.OracleTree(*w.catalogs[t])
        p, f, nf = w.catalogs[q]
        want[name] = trees[t].tree_counts(p, f, nf, w.radii, nthreads=NTH)
    return want


@pytest.mark.parametrize("name", sorted(SCALES))
def test_workload_counts_equal_oracle(name):
    w = bench.WORKLOADS[name](SCALES[name])
    want = _oracle_counts(w)
    trees = {k: N.build_tree(p, f, nf) for k, (p, f, nf) in w.catalogs.items()}
    try:
        jobs = [(trees[t], trees[q]) for _, t, q in w.jobs]
        for mode in (N.KD_MODE_MIXED, N.KD_MODE_FP64):
            outs, st = N.count_batch(jobs, w.radii, mode=mode, with_stats=True)
            for (jn, _, _), got in zip(w.jobs, outs):
                assert np.array_equal(got, want[jn]), (name, mode, jn)
            if mode == N.KD_MODE_MIXED and name == "lattice":
                # pairs exactly on an edge: the FP64 recheck must have run
                assert st["pairs_rechecked"] > 0
        # the batch split over three shards sums to the same counts
        parts = [N.count_batch(jobs, w.radii, shard=s, nshards=3) for s in range(3)]
        for j, (jn, _, _) in enumerate(w.jobs):
            assert np.array_equal(sum(p[j] for p in parts), want[jn]), (name, "shards", jn)
    finally:
        for t in trees.values():
            N.destroy(t)


@pytest.mark.parametrize("name", sorted(SCALES))
def test_workload_query_subset_equals_reference_build(name):
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    w = bench.WORKLOADS[name](SCALES[name])
    R = O.RefLib()
    jn, tn, qn = max(w.jobs, key=lambda j: len(w.catalogs[j[2]][0]))
    (tp, tf, tnf), (qp, qf, qnf) = w.catalogs[tn], w.catalogs[qn]
    idx = np.sort(np.random.RandomState(5).choice(len(qp), size=min(400, len(qp)),
                                                  replace=False))
    rt = R.build(tp, tf, tnf)
    gt = N.build_tree(tp, tf, tnf)
    try:
        want = np.stack([R.pair_count(rt, qp[idx], qf[idx], qnf, r, 4) for r in w.radii])
        got = N.count_points(gt, qp[idx], qf[idx], qnf, w.radii)
        assert np.array_equal(got, want), (name, jn)
    finally:
        R.destroy(rt)
        N.destroy(gt)


def test_angular_workload_coordinates_are_the_oracles():
    # the sky catalogs are converted by libcoords; the oracle restates
    # coordmath.c:38-51 with the platform libm: bit for bit the same
    w = bench.WORKLOADS["angular"](SCALES["angular"])
    for name, (ra, dec) in w.radec.items():
        assert np.array_equal(w.catalogs[name][0].view(np.int64),
                              O.radec2cart64(ra, dec).view(np.int64))


def _clustered(seed, n, nf):
    rs = np.random.RandomState(seed)
    c = rs.rand(max(1, n // 50), 3)
    p = (c[rs.randint(0, len(c), n)] + rs.normal(0, 0.01, (n, 3))) % 1.0
    return np.ascontiguousarray(p), (p[:, 0] * nf).astype(np.int32).clip(0, nf - 1)


@pytest.mark.parametrize("nradii", [100, 257])
def test_any_number_of_radii(nradii):
    # more than 64 distinct radii run in passes of 64; repeats, NaN, 0 and an
    # unsorted order included
    d, fd = _clustered(31, 20_000, 4)
    r, fr = _clustered(32, 40_000, 4)
    rs = np.random.RandomState(nradii)
    radii = rs.permutation(np.concatenate([np.logspace(-3, -0.8, nradii - 4),
                                           [0.0, np.nan, 0.01, 0.01]]))
    ot = O.OracleTree(r, fr, 4)
    want = ot.tree_counts(d, fd, 4, radii, nthreads=NTH)
    t, q = N.build_tree(r, fr, 4), N.build_tree(d, fd, 4)
    try:
        for mode in (N.KD_MODE_MIXED, N.KD_MODE_FP64):
            got, st = N.count_radii(t, q, radii, mode=mode, with_stats=True)
            assert np.array_equal(got, want), mode
            assert st["launches"] >= 3 * ((nradii - 2 + 63) // 64)
        # the batch form (DD symmetric, DR ordered) over the same radii
        dd, dr = N.count_batch([(q, q), (t, q)], radii)
        assert np.array_equal(dr, want)
        assert np.array_equal(dd, O.OracleTree(d, fd, 4).tree_counts(d, fd, 4, radii,
                                                                      nthreads=NTH))
    finally:
        N.destroy(t)
        N.destroy(q)


def test_autocorr_with_101_edges():
    # the reference's drivers take any number of edges (one pair_count per
    # edge, clustering.py:218-230): DD, DR, RR per bin = np.diff of the
    # cumulative counts, for 101 log edges
    d, fd = _clustered(41, 15_000, 4)
    r, fr = _clustered(42, 30_000, 4)
    edges = np.logspace(-3, -1, 101)
    res = threedim.autocorr(clustering.tree(d, fd), clustering.tree(r, fr), edges)
    od, orr = O.OracleTree(d, fd, 4), O.OracleTree(r, fr, 4)

    def binned(tree_, q, qf):
        c = tree_.tree_counts(q, qf, 4, edges, nthreads=NTH)
        return np.diff(c.reshape(len(edges), 4, 4), axis=0)
    assert np.array_equal(res.dd, binned(od, d, fd))
    assert np.array_equal(res.dr, binned(orr, d, fd))
    assert np.array_equal(res.rr, binned(orr, r, fr))
    assert res.dd.shape == (100, 4, 4)


@pytest.mark.parametrize("extent,offset", [
    (1e20, 0.0),      # squared distances and edges past FP32 range: exact path
    (1e150, 0.0),     # squared distances near 1e300, still finite
    (1e200, 0.0),     # squared distances overflow to +inf (never below an edge)
    (1.0, 1e15),      # a unit catalog 1e15 from the origin
    (1e285, 1e300),   # far out, wide: coordinates near the top of FP64
])
def test_extreme_magnitudes(extent, offset):
    rs = np.random.RandomState(int(np.log10(extent) + 7 * np.log10(offset + 1)))
    n = 3000
    c = rs.rand(30, 3)
    p = offset + extent * ((c[rs.randint(0, 30, n)] + rs.normal(0, 0.02, (n, 3))) % 1.0)
    p[:200] = p[200:400]  # duplicates
    p = np.ascontiguousarray(p)
    f = (rs.rand(n) * 3).astype(np.int32)
    radii = extent * np.array([0.0, 0.003, 0.01, 0.03, 0.1, 0.3, 1.0, 3.0])
    ot = O.OracleTree(p, f, 3)
    want = ot.brute_counts(p, f, 3, radii, nthreads=NTH)
    t = N.build_tree(p, f, 3)
    try:
        nodes, onodes = N.node_fields(t), ot.nodes()
        for k in nodes:
            assert np.array_equal(nodes[k], onodes[k]), k
        for mode in (N.KD_MODE_MIXED, N.KD_MODE_FP64):
            assert np.array_equal(N.count_radii(t, t, radii, mode=mode), want), mode
            assert np.array_equal(N.count_batch([(t, t)], radii, mode=mode)[0], want), mode
    finally:
        N.destroy(t)


def test_five_million_point_tree_node_for_node():
    # the top levels of a large uniform tree take the parallel variance with
    # its interval check; every node must still be the reference's
    p = np.random.RandomState(51).rand(5_000_000, 3)
    f = (p[:, 2] * 8).astype(np.int32)
    ot = O.OracleTree(p, f, 8)
    t = N.build_tree(p, f, 8)
    try:
        nodes, onodes = N.node_fields(t), ot.nodes()
        for k in nodes:
            assert np.array_equal(nodes[k], onodes[k]), k
        assert np.array_equal(N.permutation(t), ot.inorder())
    finally:
        N.destroy(t)
