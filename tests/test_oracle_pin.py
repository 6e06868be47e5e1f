"""Pin the CPU oracle to the reference before trusting it as the checker.

1. Golden vectors produced by the reference itself (tests/golden/, made by
   make_golden.py from the reference compiled from its sources): node arrays,
   pair counts at several radii (incl. 0 and inf), config-1 DD/DR/RR.
2. When oracle/_ref exists (this container), fresh random cases against the
   live reference build.
3. Internal consistency: the restated traversal equals the exhaustive FP64
   count, i.e. the reference's pruning is conservative.
"""
import numpy as np
import pytest

from conftest import golden_sets, none_if_empty, verify_heap
from oracle import oracle as O


def test_tree_nodes_match_reference_goldens(golden):
    sets = golden_sets(golden("trees.npz"))
    assert len(sets) >= 20
    for name, s in sets.items():
        f = none_if_empty(s["fields"])
        t = O.OracleTree(s["points"], f, int(s["num_fields"]))
        assert t.size == int(s["size"]), name
        nodes = t.nodes()
        for k in ("xyz", "field", "weight", "has_l", "has_r", "dim"):
            ref = s["node_" + k]
            got = nodes[k]
            if k == "xyz":
                # compare bit patterns: -0.0 vs +0.0 of the first occurrence
                assert np.array_equal(ref.view(np.int64), got.view(np.int64)), (name, k)
            else:
                assert np.array_equal(ref, got), (name, k)


def test_pair_counts_match_reference_goldens(golden):
    g = golden("counts.npz")
    radii = g["radii"]
    sets = golden_sets(g)
    trees = golden_sets(golden("trees.npz"))
    for name, s in sets.items():
        if name == "layout_q2_t3":
            t = O.OracleTree(s["points"], s["fields"].astype(np.int32), 3)
            fq = 2
        else:
            ts = trees[name]
            t = O.OracleTree(ts["points"], none_if_empty(ts["fields"]), int(ts["num_fields"]))
            fq = int(ts["num_fields"])
        qf = none_if_empty(s["qfields"])
        for k, r in enumerate(radii):
            got = t.pair_count(s["queries"], qf, fq, r)
            assert np.array_equal(got, s["counts"][k]), (name, r)


def test_traversal_equals_brute_force(golden):
    """kdquery.c's pruning never drops a pair: traversal == exhaustive FP64."""
    g = golden("counts.npz")
    radii = g["radii"]
    trees = golden_sets(golden("trees.npz"))
    for name in ("rand1000", "dup3", "dupmixed", "lattice8", "plane12", "signedzero", "w255",
                 "clustered_nofield"):
        ts = trees[name]
        f = none_if_empty(ts["fields"])
        nf = int(ts["num_fields"])
        t = O.OracleTree(ts["points"], f, nf)
        q = g[name + "/queries"]
        qf = none_if_empty(g[name + "/qfields"])
        brute = t.brute_counts(q, qf, nf, radii, nthreads=4)
        for k, r in enumerate(radii):
            assert np.array_equal(brute[k], t.pair_count(q, qf, nf, r)), (name, r)


def test_pruned_multi_radius_counter_equals_exhaustive(golden):
    """or_tree_counts (the traversal at the largest radius, every visited
    distance binned into all radii) == the exhaustive loop, on every golden
    set, a lattice with exact on-edge pairs and radii in any order; and equal
    to the live reference build, radius by radius."""
    g = golden("counts.npz")
    trees = golden_sets(golden("trees.npz"))
    radii = np.array([0.0, 0.02, np.nan, 0.05, 0.05, 0.5, 0.1, 0.25])
    for name in trees:
        ts = trees[name]
        f = none_if_empty(ts["fields"])
        nf = int(ts["num_fields"])
        t = O.OracleTree(ts["points"], f, nf)
        if name + "/queries" not in g:
            continue
        q = g[name + "/queries"]
        qf = none_if_empty(g[name + "/qfields"])
        assert np.array_equal(t.tree_counts(q, qf, nf, radii, nthreads=4),
                              t.brute_counts(q, qf, nf, radii, nthreads=4)), name
        # the goldens' own radii (0 and inf included: +inf squared falls back
        # to the exhaustive loop)
        gr = g["radii"]
        got = t.tree_counts(q, qf, nf, gr, nthreads=4)
        assert np.array_equal(got, t.brute_counts(q, qf, nf, gr, nthreads=4)), name
        # the reference build's counts at those radii
        assert np.array_equal(got, g[name + "/counts"].reshape(got.shape)), name
    rs = np.random.RandomState(5)
    lat = rs.randint(0, 64, (6000, 3)) / 64.0
    lat[:600] = lat[600:1200]
    t = O.OracleTree(lat, None, 1)
    edges = np.sqrt(np.array([1, 2, 3, 5, 9, 16, 25, 50])) / 64.0
    assert np.array_equal(t.tree_counts(lat, None, 1, edges[::-1]),
                          t.brute_counts(lat, None, 1, edges[::-1]))
    if O.ref_available():
        R = O.RefLib()
        rt = R.build(lat, None, 1)
        try:
            got = t.tree_counts(lat[:500], None, 1, edges)
            for k, r in enumerate(edges):
                assert np.array_equal(got[k], R.pair_count(rt, lat[:500], None, 1, r, 2))
        finally:
            R.destroy(rt)


def test_config1_counts_golden(golden):
    c1 = golden("config1.npz")
    assert c1["dd"].sum(axis=(1, 2)).tolist() == [12, 88, 896, 7130, 52570]
    assert c1["dr"].sum(axis=(1, 2)).tolist() == [286, 2240, 18017, 139246, 1039842]
    assert c1["rr"].sum(axis=(1, 2)).tolist() == [5892, 45782, 360228, 2772904, 20698426]
    np.random.seed(3)
    X = np.random.rand(4000, 3)
    Y = np.random.rand(80000, 3)
    fd = (X[:, 0] * 4).astype("int32")
    fr = (Y[:, 0] * 4).astype("int32")
    radii = c1["radii"]
    td = O.OracleTree(X, fd, 4)
    tr = O.OracleTree(Y, fr, 4)

    def binned(t, q, qf):
        return np.diff(np.array([t.pair_count(q, qf, 4, r, nthreads=4).reshape(4, 4)
                                 for r in radii]), axis=0)
    assert np.array_equal(binned(td, X, fd), c1["dd"])
    assert np.array_equal(binned(tr, X, fd), c1["dr"])
    assert np.array_equal(binned(tr, Y, fr), c1["rr"])


def test_coords_match_reference_goldens(golden):
    c = golden("coords.npz")
    xyz = O.radec2cart64(c["ra"], c["dec"])
    assert np.array_equal(xyz.view(np.int64), c["xyz"].view(np.int64))
    xyzd = O.radecdist2cart64(c["ra"], c["dec"], c["dist"])
    assert np.array_equal(xyzd.view(np.int64), c["xyzd"].view(np.int64))
    theta, phi = O.radec2sph64(c["ra"], c["dec"])
    assert np.array_equal(theta.view(np.int64), c["theta"].view(np.int64))
    assert np.array_equal(phi.view(np.int64), c["phi"].view(np.int64))


def test_weight_overflow_is_an_error():
    p = np.tile([[0.1, 0.2, 0.3]], (256, 1))
    with pytest.raises(O.OracleError):
        O.OracleTree(p)


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) absent")
def test_oracle_matches_live_reference_random():
    R = O.RefLib()
    rs = np.random.RandomState(123)
    for trial in range(6):
        n = int(rs.randint(50, 6000))
        if trial % 2:
            p = rs.randint(0, 16, size=(n, 3)) / 16.0      # lattice: ties, duplicates
        else:
            c = rs.rand(10, 3)
            p = (c[rs.randint(0, 10, n)] + rs.normal(0, 0.02, (n, 3))) % 1.0
        nf = int(rs.randint(1, 9))
        f = (rs.rand(n) * nf).astype(np.int32) if nf > 1 else None
        rt = R.build(p, f, nf)
        ot = O.OracleTree(p, f, nf)
        rn, on = R.nodes(rt), ot.nodes()
        for k in rn:
            assert np.array_equal(rn[k], on[k]), (trial, k)
        q = np.concatenate([p[:300], rs.rand(200, 3)])
        qf = None if f is None else np.concatenate([f[:300], (rs.rand(200) * nf).astype(np.int32)])
        for r in (0.0, 0.01, 0.07, 0.3):
            assert np.array_equal(R.pair_count(rt, q, qf, nf, r), ot.pair_count(q, qf, nf, r))
        R.destroy(rt)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("scale", [1e-300, 1e-150, 1e100, 1e154, 1e155, 1e200, 1e300, 1.7e308])
def test_oracle_matches_live_reference_at_extreme_magnitudes(scale):
    """Coordinates from 1e-300 to 1.7e308: the variance sums of the split
    choice underflow or overflow to inf (kdbuild.c:308-351) and the squared
    distances of the counts overflow; the oracle still builds the
    reference's node array and counts what the reference counts."""
    R = O.RefLib()
    rs = np.random.RandomState(51)
    p = (rs.rand(500, 3) - 0.5) * scale
    p[::7] *= 0.5 ** rs.randint(0, 40, len(p[::7]))[:, None]
    f = (rs.rand(len(p)) * 3).astype(np.int32)
    rt = R.build(p, f, 3)
    try:
        ot = O.OracleTree(p, f, 3)
        rn, on = R.nodes(rt), ot.nodes()
        assert np.array_equal(rn["xyz"].view(np.int64), on["xyz"].view(np.int64))
        for k in ("field", "weight", "has_l", "has_r", "dim"):
            assert np.array_equal(rn[k], on[k]), k
        q = np.concatenate([p[:100], (rs.rand(50, 3) - 0.5) * scale])
        qf = (rs.rand(len(q)) * 3).astype(np.int32)
        for r in (0.0, 0.01 * scale, 0.3 * scale, 2.0 * scale, np.inf):
            assert np.array_equal(R.pair_count(rt, q, qf, 3, r), ot.pair_count(q, qf, 3, r)), r
    finally:
        R.destroy(rt)


def test_heap_rule_holds_and_catches_a_planted_violation(golden):
    """The reference's verify_tree rule holds on oracle trees (golden sets
    and a 200k lattice with ties), and fails once a child is moved to the
    wrong side of its parent (the mistake is planted in the oracle's nodes)."""
    rs = np.random.RandomState(49)
    p = rs.randint(0, 32, (200_000, 3)) / 32.0
    nodes = O.OracleTree(p, (p[:, 1] * 2).astype(np.int32), 2).nodes()
    verify_heap(nodes)
    for name, s in golden_sets(golden("trees.npz")).items():
        f = none_if_empty(s["fields"])
        verify_heap(O.OracleTree(s["points"], f, int(s["num_fields"])).nodes())
    bad = {k: v.copy() for k, v in nodes.items()}
    i = int(np.nonzero(bad["has_l"][1:len(bad["dim"]) // 2])[0][100]) + 1
    d = int(bad["dim"][i])
    bad["xyz"][2 * i, d] = bad["xyz"][i, d] + 1.0
    with pytest.raises(AssertionError):
        verify_heap(bad)
