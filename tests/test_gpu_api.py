"""The user API end to end on the GPU (tree build, batched counts, estimators)
against the reference's golden outputs and the oracle."""
import numpy as np
import pytest

from corruscant_b200 import _native, clustering, twopoint
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.int64)


@pytest.mark.parametrize("mode", [_native.KD_MODE_MIXED, _native.KD_MODE_FP64])
def test_example_autocorr_end_to_end(golden, mode):
    """The reference's test/example.py workload through twopoint.threedim."""
    g = golden("config1.npz")
    np.random.seed(3)
    X = np.random.rand(4000, 3)
    Y = np.random.rand(80000, 3)
    dtree = clustering.tree(X, (X[:, 0] * 4).astype("int32"))
    rtree = clustering.tree(Y, (Y[:, 0] * 4).astype("int32"))
    res = twopoint.threedim.autocorr(dtree, rtree, np.logspace(-2.5, -1., 6),
                                     est_type="landy-szalay", num_threads=4, mode=mode)
    for k in ("dd", "dr", "rr"):
        assert np.array_equal(getattr(res, k), g[k]), k
    assert np.array_equal(_bits(res.estimate()), _bits(g["xi"]))
    assert np.array_equal(_bits(res.error("jackknife")), _bits(g["err_jackknife"]))
    res.error_type = "jackknife"
    assert "Estimator" in str(res)


def test_crosscorr_end_to_end(golden):
    g = golden("cross.npz")
    rs = np.random.RandomState(int(g["seed"]))
    cats = [rs.rand(int(n), 3) for n in g["sizes"]]
    trees = [clustering.tree(c, (c[:, 0] * 4).astype("int32")) for c in cats]
    res = twopoint.threedim.crosscorr(*trees, g["radii"])
    for k in ("d1d2", "d1r2", "d2r1", "r1r2"):
        assert np.array_equal(getattr(res, k), g[k]), k
    assert np.array_equal(_bits(res.estimate()), _bits(g["xi"]))
    assert np.array_equal(_bits(res.error("jackknife")), _bits(g["err_jackknife"]))


def test_reference_query_tree_entry_point_matches():
    """_query_tree goes through pair_count, one radius at a time, like the
    reference driver; it must agree with the batched counts."""
    rs = np.random.RandomState(2)
    X = rs.rand(3000, 3)
    f = (X[:, 1] * 3).astype("int32")
    t = clustering.tree(X, f)
    radii = np.array([0.01, 0.03, 0.08])
    batched = _native.count_radii(t.ctree, t.ctree, radii).reshape(3, 3, 3)
    for k, r in enumerate(radii):
        assert np.array_equal(clustering._query_tree(t, t.points, r, 4, t.fields, 3), batched[k])


def test_angular_autocorr_matches_oracle():
    rs = np.random.RandomState(4)
    n, m = 3000, 20000
    ra_d, ra_r = rs.rand(n) * 90, rs.rand(m) * 90
    dec_d = np.degrees(np.arcsin(rs.uniform(np.sin(np.radians(-10)), np.sin(np.radians(60)), n)))
    dec_r = np.degrees(np.arcsin(rs.uniform(np.sin(np.radians(-10)), np.sin(np.radians(60)), m)))
    Xd, Xr = twopoint.angular.cartesian(ra_d, dec_d), twopoint.angular.cartesian(ra_r, dec_r)
    fd, fr = (ra_d / 30).astype("int32"), (ra_r / 30).astype("int32")
    deg = np.logspace(-1, np.log10(5.0), 6)
    res = twopoint.angular.autocorr(clustering.tree(Xd, fd), clustering.tree(Xr, fr), deg)
    chords = twopoint.angular.chord(deg)
    od, orr = O.OracleTree(Xd, fd, 3), O.OracleTree(Xr, fr, 3)
    dd = np.diff(od.brute_counts(Xd, fd, 3, chords, nthreads=8), axis=0).reshape(-1, 3, 3)
    rr = np.diff(orr.brute_counts(Xr, fr, 3, chords, nthreads=8), axis=0).reshape(-1, 3, 3)
    assert np.array_equal(res.dd, dd)
    assert np.array_equal(res.rr, rr)
    assert res.radii_units == "degrees"


def test_build_statistics_and_overlapped_node_copy():
    """kd_tree_build_stats: every device phase timed, the node array copied
    while the layout was built; the copied array is the oracle's."""
    rs = np.random.RandomState(8)
    p = rs.rand(300_000, 3)
    f = (p[:, 0] * 4).astype(np.int32)
    t = _native.build_tree(p, f, 4)
    try:
        st = _native.build_stats(t)
        for k in ("ms_prep", "ms_dedup", "ms_argsort", "ms_levels", "ms_layout", "ms_device",
                  "ms_node_copy", "ms_total_host"):
            assert st[k] > 0, k
        assert st["ms_node_wait"] >= 0 and st["n_unique"] == 300_000 and st["levels"] >= 18
        parts = sum(st[k] for k in ("ms_prep", "ms_dedup", "ms_argsort", "ms_levels",
                                    "ms_layout"))
        assert abs(parts - st["ms_device"]) < 0.01 * st["ms_device"] + 0.05
        nodes, onodes = _native.node_fields(t), O.OracleTree(p, f, 4).nodes()
        for k in nodes:
            assert np.array_equal(nodes[k], onodes[k]), k
    finally:
        _native.destroy(t)


def test_deferred_build_counts_while_node_array_drains():
    """kd_tree_construct_deferred: the tree counts at once, its node array
    equals the oracle's after kd_tree_wait_nodes, the copy's timing is filled
    in by the wait, and a tree never waited for is destroyed cleanly."""
    rs = np.random.RandomState(9)
    p = rs.rand(3_000_000, 3)  # a 160 MB node array: several copy items
    f = (p[:, 1] * 4).astype(np.int32)
    q = rs.rand(20_000, 3)
    qf = (q[:, 1] * 4).astype(np.int32)
    radii = np.array([0.001, 0.004, 0.01])
    t = _native.build_tree(p, f, 4, deferred=True)
    tq = _native.build_tree(q, qf, 4, deferred=True)
    t2 = _native.build_tree(p, f, 4, deferred=True)
    try:
        got = _native.count_radii(t, tq, radii)
        _native.wait_nodes(t)
        _native.wait_nodes(t)  # a second wait returns at once
        st = _native.build_stats(t)
        assert st["ms_node_copy"] > 0 and st["ms_node_wait"] >= 0
        ot = O.OracleTree(p, f, 4)
        assert np.array_equal(got, ot.tree_counts(q, qf, 4, radii))
        nodes, onodes = _native.node_fields(t), ot.nodes()
        for k in nodes:
            assert np.array_equal(nodes[k], onodes[k]), k
        # the reference-facing tree object builds deferred and waits on ctree
        ct = clustering.tree(p[:100_000], f[:100_000])
        assert ct.ctree.size == 100_000 and ct._nodes_ready
        nodes = _native.node_fields(ct.ctree)
        onodes = O.OracleTree(p[:100_000], f[:100_000], 4).nodes()
        for k in nodes:
            assert np.array_equal(nodes[k], onodes[k]), k
    finally:
        _native.destroy(t)
        _native.destroy(tq)
        _native.destroy(t2)  # its copy may still be running


def test_many_deferred_builds_share_four_staging_pairs():
    """Twelve deferred builds whose node arrays (each above 4 MB) drain at
    once: at most four copies hold a pinned staging pair, the others wait
    for one; every node array arrives complete, from builds on one thread
    and on four threads at once."""
    from concurrent.futures import ThreadPoolExecutor
    rs = np.random.RandomState(10)
    cats = [rs.rand(int(n), 3) for n in rs.randint(150_000, 400_000, 12)]
    fields = [(c[:, 2] * 3).astype(np.int32) for c in cats]
    want = [O.OracleTree(c, f, 3).nodes() for c, f in zip(cats[:3], fields[:3])]
    for workers in (1, 4):
        def one(i):
            return _native.build_tree(cats[i], fields[i], 3, deferred=True)
        if workers == 1:
            trees = [one(i) for i in range(12)]
        else:
            with ThreadPoolExecutor(max_workers=workers) as ex:
                trees = list(ex.map(one, range(12)))
        try:
            for t in trees:
                _native.wait_nodes(t)
            for t, c, wn in zip(trees, cats, want):
                got = _native.node_fields(t)
                for k in got:
                    assert np.array_equal(got[k], wn[k]), k
            for t, c in zip(trees, cats):
                assert t.size == len(c)
        finally:
            for t in trees:
                _native.destroy(t)


def test_pinned_and_pageable_inputs_build_the_same_tree():
    """A catalog's points above 32 MB go to the device through pinned staging
    when they are pageable and in one copy when they are pinned: the same
    tree either way, and the oracle's."""
    torch = pytest.importorskip("torch")
    rs = np.random.RandomState(12)
    n = 2_000_000  # 48 MB of points
    p = rs.rand(n, 3)
    f = (p[:, 0] * 4).astype(np.int32)
    pin = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    pin.numpy()[...] = p
    pinf = torch.empty(n, dtype=torch.int32).pin_memory()
    pinf.numpy()[...] = f
    a = _native.build_tree(p, f, 4)
    b = _native.build_tree(pin.numpy(), pinf.numpy(), 4)
    try:
        na, nb = _native.node_fields(a), _native.node_fields(b)
        onodes = O.OracleTree(p, f, 4).nodes()
        for k in na:
            assert np.array_equal(na[k], nb[k]), k
            assert np.array_equal(na[k], onodes[k]), k
        assert np.array_equal(_native.permutation(a), _native.permutation(b))
    finally:
        _native.destroy(a)
        _native.destroy(b)
