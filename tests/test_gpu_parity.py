"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

Bit-exact everywhere: node arrays (semantic fields, coordinates compared as
bit patterns), in-order permutation, and every pair count, in both the mixed
FP32 + FP64-recheck mode and the plain FP64 mode.
"""
import numpy as np
import pytest

from conftest import golden_sets, none_if_empty, verify_heap
from corruscant_b200 import _native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = (N.KD_MODE_MIXED, N.KD_MODE_FP64)


def _tree(points, fields, nf):
    return N.build_tree(np.require(points, dtype=np.float64, requirements="AC"),
                        None if fields is None else np.require(fields, dtype=np.int32,
                                                               requirements="AC"), nf)


def test_tree_nodes_match_reference_goldens(golden):
    for name, s in golden_sets(golden("trees.npz")).items():
        t = _tree(s["points"], none_if_empty(s["fields"]), int(s["num_fields"]))
        try:
            assert t.size == int(s["size"]), name
            assert t.memsize == len(s["node_dim"]), name
            nodes = N.node_fields(t)
            assert np.array_equal(nodes["xyz"].view(np.int64), s["node_xyz"].view(np.int64)), name
            for k in ("field", "weight", "has_l", "has_r", "dim"):
                assert np.array_equal(nodes[k], s["node_" + k]), (name, k)
        finally:
            N.destroy(t)


def test_permutation_matches_oracle(golden):
    sets = golden_sets(golden("trees.npz"))
    for name in ("rand1000", "dup3", "dupmixed", "lattice8", "plane12", "signedzero", "w255"):
        s = sets[name]
        f = none_if_empty(s["fields"])
        t = _tree(s["points"], f, int(s["num_fields"]))
        try:
            ot = O.OracleTree(s["points"], f, int(s["num_fields"]))
            assert np.array_equal(N.permutation(t), ot.inorder()), name
        finally:
            N.destroy(t)


def _large_set(kind):
    rs = np.random.RandomState(48)
    if kind == "clustered_1M":
        # the clustered workload's data catalog: Neyman-Scott, 10,000 parents
        parents = rs.rand(10000, 3)
        p = (np.repeat(parents, 100, axis=0) + rs.normal(0.0, 0.005, (1_000_000, 3))) % 1.0
        f = (16 * np.floor(4 * p[:, 0]) + 4 * np.floor(4 * p[:, 1]) +
             np.floor(4 * p[:, 2])).astype(np.int32)
        return p, f, 64
    # a 1/64 lattice: ties in every coordinate, about half the rows repeated
    p = rs.randint(0, 64, (400_000, 3)) / 64.0
    return p, (p[:, 0] * 3).astype(np.int32), 3


@pytest.mark.parametrize("kind", ["clustered_1M", "lattice_400k"])
def test_large_trees_match_the_oracle_node_for_node(kind):
    """Bit-exact node array and in-order permutation at the sizes the
    benchmarks build (the small sets are pinned to the reference itself; the
    oracle is pinned to it on those and on random lattice and clustered sets)."""
    p, f, nf = _large_set(kind)
    t = _tree(p, f, nf)
    try:
        ot = O.OracleTree(p, f, nf)
        assert t.size == ot.size and t.memsize == ot.memsize
        nodes, want = N.node_fields(t), ot.nodes()
        assert np.array_equal(nodes["xyz"].view(np.int64), want["xyz"].view(np.int64))
        for k in ("field", "weight", "has_l", "has_r", "dim"):
            assert np.array_equal(nodes[k], want[k]), k
        assert np.array_equal(N.permutation(t), ot.inorder())
        verify_heap(nodes)
    finally:
        N.destroy(t)


def test_pair_count_matches_reference_goldens(golden):
    g = golden("counts.npz")
    radii = g["radii"]
    trees = golden_sets(golden("trees.npz"))
    for name, s in golden_sets(g).items():
        if name == "layout_q2_t3":
            t = _tree(s["points"], s["fields"], 3)
            fq = 2
        else:
            ts = trees[name]
            t = _tree(ts["points"], none_if_empty(ts["fields"]), int(ts["num_fields"]))
            fq = int(ts["num_fields"])
        qf = none_if_empty(s["qfields"])
        try:
            for mode in MODES:  # the reference entry point in both precisions
                N.set_precision(mode)
                for k, r in enumerate(radii):
                    got = N.pair_count(t, s["queries"], qf, fq, r)
                    assert np.array_equal(got, s["counts"][k]), (name, r, mode)
            N.set_precision(N.KD_MODE_MIXED)
            for mode in MODES:
                got = N.count_points(t, s["queries"], qf, fq, radii, mode=mode)
                assert np.array_equal(got, s["counts"]), (name, mode)
        finally:
            N.destroy(t)


@pytest.mark.parametrize("mode", MODES)
def test_config1_landy_szalay_counts(golden, mode):
    c1 = golden("config1.npz")
    np.random.seed(3)
    X = np.random.rand(4000, 3)
    Y = np.random.rand(80000, 3)
    fd = (X[:, 0] * 4).astype("int32")
    fr = (Y[:, 0] * 4).astype("int32")
    td, tr = _tree(X, fd, 4), _tree(Y, fr, 4)
    try:
        for tree, query, key in ((td, td, "dd"), (tr, td, "dr"), (tr, tr, "rr")):
            cum = N.count_radii(tree, query, c1["radii"], mode=mode)
            assert np.array_equal(np.diff(cum, axis=0).reshape(-1, 4, 4), c1[key]), key
    finally:
        N.destroy(td)
        N.destroy(tr)


def _clustered(rs, n, nparents, sigma):
    c = rs.rand(nparents, 3)
    return (c[rs.randint(0, nparents, n)] + rs.normal(0, sigma, (n, 3))) % 1.0


@pytest.mark.parametrize("mode", MODES)
def test_random_catalogs_match_oracle(mode):
    rs = np.random.RandomState(99)
    radii = np.concatenate([[0.0], np.logspace(-3, -1, 21), [0.2, np.inf]])
    cases = [
        (_clustered(rs, 30000, 300, 0.005), _clustered(rs, 20000, 200, 0.01), 8),
        (rs.rand(25000, 3), rs.rand(3000, 3) * 2 - 0.5, 1),  # queries outside the tree box
    ]
    for pts, q, nf in cases:
        f = (pts[:, 0] * nf).astype(np.int32).clip(0, nf - 1) if nf > 1 else None
        qf = (np.abs(q[:, 1]) * nf).astype(np.int32).clip(0, nf - 1) if nf > 1 else None
        t = _tree(pts, f, nf)
        try:
            ot = O.OracleTree(pts, f, nf)
            want = ot.brute_counts(q, qf, nf, radii, nthreads=8)
            got = N.count_points(t, q, qf, nf, radii, mode=mode)
            assert np.array_equal(got, want)
        finally:
            N.destroy(t)


@pytest.mark.parametrize("mode", MODES)
def test_lattice_edges_exact(mode):
    """Points on a 1/64 lattice with edges at exact lattice distances: many
    pairs sit exactly on an edge, so the FP32 band must send them to FP64."""
    rs = np.random.RandomState(5)
    p = rs.randint(0, 64, size=(20000, 3)) / 64.0
    dup = rs.rand(len(p)) < 0.1
    p[dup] = p[rs.randint(0, len(p), dup.sum())]
    q = rs.randint(0, 64, size=(4000, 3)) / 64.0
    k = np.unique(np.geomspace(1, 900, 30).astype(int))
    radii = np.sqrt(k) / 64.0
    f = (p[:, 0] * 3).astype(np.int32)
    qf = (q[:, 0] * 3).astype(np.int32)
    t = _tree(p, f, 3)
    try:
        ot = O.OracleTree(p, f, 3)
        want = ot.brute_counts(q, qf, 3, radii, nthreads=8)
        got, st = N.count_points(t, q, qf, 3, radii, mode=mode, with_stats=True)
        assert np.array_equal(got, want)
        if mode == N.KD_MODE_MIXED:
            assert st["pairs_rechecked"] > 0
    finally:
        N.destroy(t)


def test_tree_as_queries_with_mixed_field_duplicates(golden):
    """DD-style count where duplicated points carry different fields: the
    query side keeps each copy's own field, the tree side the first one's."""
    s = golden_sets(golden("trees.npz"))["dupmixed"]
    f = s["fields"].astype(np.int32)
    t = _tree(s["points"], f, 3)
    try:
        ot = O.OracleTree(s["points"], f, 3)
        radii = np.array([0.0, 0.05, 0.1, 0.3, np.inf])
        want = ot.brute_counts(s["points"], f, 3, radii)
        for mode in MODES:
            assert np.array_equal(N.count_radii(t, t, radii, mode=mode), want)
    finally:
        N.destroy(t)


def test_errors_are_reported_not_fatal():
    p = np.random.RandomState(1).rand(100, 3)
    bad = p.copy()
    bad[7, 1] = np.nan
    with pytest.raises(N.NativeError):
        _tree(bad, None, 1)
    heavy = np.tile([[0.1, 0.2, 0.3]], (256, 1))
    with pytest.raises(N.NativeError):
        _tree(heavy, None, 1)
    t = _tree(p, None, 1)
    try:
        with pytest.raises(N.NativeError):
            N.count_points(t, p, None, 1, [-0.1])
        # NaN query rows and NaN radii count nothing, as in the reference
        q = p.copy()
        q[3] = np.nan
        got = N.count_points(t, q, None, 1, [np.nan, 0.3])
        want = O.OracleTree(p).brute_counts(q, None, 1, [np.nan, 0.3])
        assert np.array_equal(got, want)
        # a query point may repeat any number of times
        got = N.count_points(t, heavy, None, 1, [0.5])
        want = O.OracleTree(p).brute_counts(heavy, None, 1, [0.5])
        assert np.array_equal(got, want)
    finally:
        N.destroy(t)


def test_count_bins_is_the_diff_of_per_edge_counts(golden):
    """kd_count_bins gives the reference drivers' np.diff over per-edge counts
    (the config-1 goldens are those per-bin arrays)."""
    c1 = golden("config1.npz")
    np.random.seed(3)
    X = np.random.rand(4000, 3)
    Y = np.random.rand(80000, 3)
    td = _tree(X, (X[:, 0] * 4).astype("int32"), 4)
    tr = _tree(Y, (Y[:, 0] * 4).astype("int32"), 4)
    try:
        for tree, query, key in ((td, td, "dd"), (tr, td, "dr"), (tr, tr, "rr")):
            got = N.count_bins(tree, query, c1["radii"])
            assert np.array_equal(got.reshape(-1, 4, 4), c1[key]), key
        with pytest.raises(N.NativeError):
            N.count_bins(td, td, [])
    finally:
        N.destroy(td)
        N.destroy(tr)


def test_shards_sum_to_full_count():
    """kd_count_radii_shard: the shards of the query blocks partition the
    count exactly (the multi-GPU split, run here on one device)."""
    rs = np.random.RandomState(17)
    p = _clustered(rs, 40000, 200, 0.01)
    f = (p[:, 2] * 4).astype(np.int32)
    t = _tree(p, f, 4)
    radii = np.logspace(-2.5, -1, 7)
    try:
        full = N.count_radii(t, t, radii)
        for nshards in (2, 3, 8):
            parts = [N.count_radii_shard(t, t, radii, s, nshards) for s in range(nshards)]
            assert np.array_equal(sum(parts), full), nshards
    finally:
        N.destroy(t)
