"""kd_count_batch: many (tree, query tree) counts in one device batch.

Every job of a batch must give exactly what kd_count_radii gives for it
alone (and, for the small ones, what the exhaustive oracle gives), whatever
the mix of sizes, field counts and duplicates in the batch.
"""
import os

import numpy as np
import pytest

from corruscant_b200 import _native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = (N.KD_MODE_MIXED, N.KD_MODE_FP64)


def _clustered(rs, n, nparents, sigma):
    c = rs.rand(nparents, 3)
    return (c[rs.randint(0, nparents, n)] + rs.normal(0, sigma, (n, 3))) % 1.0


def _cat(points, nf, axis=0):
    points = np.ascontiguousarray(points, dtype=np.float64)
    f = (points[:, axis] * nf).astype(np.int32).clip(0, nf - 1) if nf > 1 else None
    return points, f, nf


@pytest.mark.parametrize("mode", MODES)
def test_batch_jobs_equal_single_counts_and_oracle(mode):
    rs = np.random.RandomState(21)
    dup = rs.rand(3000, 3)
    dup[1000:1400] = dup[:400]  # duplicates ...
    cats = {
        "A": _cat(_clustered(rs, 40000, 400, 0.01), 4),
        "B": _cat(rs.rand(90000, 3), 4, axis=1),
        "C": _cat(rs.rand(1, 3), 1),  # a one-point tree
        "D": _cat(dup, 3, axis=2),
        "E": _cat(_clustered(rs, 7000, 20, 0.02), 9),
    }
    fD = cats["D"][1].copy()
    fD[1000:1400] = (fD[1000:1400] + 1) % 3  # ... some of them with other fields
    cats["D"] = (cats["D"][0], fD, 3)
    trees = {k: N.build_tree(p, f, nf) for k, (p, f, nf) in cats.items()}
    # (tree, query) jobs; every one keeps qfield*Fq + tfield inside Fq*Ft, as
    # the reference's counter layout requires (kdquery.c:34)
    pairs = [("A", "A"), ("B", "A"), ("B", "B"), ("A", "C"), ("D", "D"), ("E", "B"),
             ("E", "E"), ("C", "C"), ("E", "C")]
    radii = np.array([0.0, 0.002, 0.01, np.nan, 0.03, 0.05, 0.05, 0.12, np.inf])
    try:
        jobs = [(trees[t], trees[q]) for t, q in pairs]
        got, st = N.count_batch(jobs, radii, mode=mode, with_stats=True)
        assert st["tile_launches"] >= 1 and st["launches"] <= 2 + 2 * st["tile_launches"]
        for (t, q), g in zip(pairs, got):
            want = N.count_radii(trees[t], trees[q], radii, mode=mode)
            assert np.array_equal(g, want), (t, q)
            if len(cats[t][0]) * len(cats[q][0]) <= 5e7:
                pt, ft, nft = cats[t]
                pq, fq, nfq = cats[q]
                brute = O.OracleTree(pt, ft, nft).brute_counts(pq, fq, nfq, radii, nthreads=8)
                assert np.array_equal(g, brute), (t, q)
    finally:
        for t in trees.values():
            N.destroy(t)


def test_batch_shards_sum_to_batch():
    rs = np.random.RandomState(22)
    a = N.build_tree(_clustered(rs, 30000, 100, 0.01), None, 1)
    b = N.build_tree(rs.rand(50000, 3), None, 1)
    radii = np.logspace(-2.5, -1, 8)
    jobs = [(a, a), (b, a), (b, b)]
    try:
        full = N.count_batch(jobs, radii)
        for nshards in (2, 5):
            parts = [N.count_batch(jobs, radii, shard=s, nshards=nshards) for s in range(nshards)]
            for j in range(len(jobs)):
                assert np.array_equal(sum(p[j] for p in parts), full[j]), (nshards, j)
    finally:
        N.destroy(a)
        N.destroy(b)


def test_mock_catalogs_against_shared_randoms():
    """The batched-mocks shape at reduced size: catalogs of log-uniform sizes,
    each with its DD and its cross count against one shared random catalog,
    all in one batch (16 fields on a 4x4 grid in x, y)."""
    rs = np.random.RandomState(23)
    sizes = np.exp(rs.uniform(np.log(2000), np.log(50000), 12)).astype(int)

    def fields(p):
        return (4 * np.floor(4 * p[:, 0]) + np.floor(4 * p[:, 1])).astype(np.int32)

    R = rs.rand(300000, 3)
    tr = N.build_tree(R, fields(R), 16)
    mocks = []
    for n in sizes:
        p = _clustered(rs, int(n), max(1, int(n) // 100), 0.005)
        mocks.append(N.build_tree(p, fields(p), 16))
    radii = np.logspace(np.log10(2e-3), -1, 13)
    try:
        jobs = [(m, m) for m in mocks] + [(tr, m) for m in mocks]
        got = N.count_batch(jobs, radii)
        for (t, q), g in zip(jobs, got):
            assert np.array_equal(g, N.count_radii(t, q, radii))
    finally:
        N.destroy(tr)
        for m in mocks:
            N.destroy(m)


def test_many_tiny_jobs_in_one_batch():
    """Hundreds of catalogs of 1..50 points in one batch (most jobs are a
    single query block): every job still gets exactly its own counts."""
    rs = np.random.RandomState(24)
    cats = []
    for i in range(300):
        n = int(rs.randint(1, 51))
        p = rs.rand(n, 3)
        nf = int(rs.randint(1, 4))
        f = (p[:, 0] * nf).astype(np.int32).clip(0, nf - 1) if nf > 1 else None
        cats.append((p, f, nf))
    trees = [N.build_tree(p, f, nf) for p, f, nf in cats]
    radii = np.array([0.0, 0.05, 0.2, 0.5, np.inf])
    try:
        pairs = [(i, i) for i in range(300)] + \
                [(i, (7 * i + 3) % 300) for i in range(0, 300, 3)
                 if cats[i][2] == cats[(7 * i + 3) % 300][2]]
        got = N.count_batch([(trees[ti], trees[qi]) for ti, qi in pairs], radii)
        assert len(got) == len(pairs)
        for (ti, qi), g in zip(pairs, got):
            pt, ft, nft = cats[ti]
            pq, fq, nfq = cats[qi]
            want = O.OracleTree(pt, ft, nft).brute_counts(pq, fq, nfq, radii, nthreads=1)
            assert np.array_equal(g, want), (ti, qi)
    finally:
        for t in trees:
            N.destroy(t)


def test_counts_split_over_many_record_batches():
    """With the tile-record buffer capped (KD_TILE_RECORD_CAP), a count runs
    as many traversal + tile batches; the counts equal the single-batch
    counts in both precisions, and every pair is still tested exactly once."""
    rs = np.random.RandomState(25)
    d, r = rs.rand(20000, 3), rs.rand(60000, 3)
    td = N.build_tree(d, (d[:, 0] * 4).astype(np.int32), 4)
    tr = N.build_tree(r, (r[:, 0] * 4).astype(np.int32), 4)
    radii = np.logspace(-2.5, -1, 8)
    jobs = [(td, td), (tr, td), (tr, tr)]
    try:
        want, s1 = N.count_batch(jobs, radii, with_stats=True)
        assert s1["tile_launches"] == 1
        # ~2e4 records (783 query blocks, tens of runs each) in batches of
        # 200 records, or of the largest block's records when that is more
        os.environ["KD_TILE_RECORD_CAP"] = "200"
        try:
            got, s2 = N.count_batch(jobs, radii, with_stats=True)
            got64 = N.count_batch(jobs, radii, mode=N.KD_MODE_FP64)
        finally:
            del os.environ["KD_TILE_RECORD_CAP"]
        assert s2["tile_launches"] >= 5 and s2["launches"] > s1["launches"]
        assert s2["pairs_tested"] == s1["pairs_tested"] and s2["entries"] == s1["entries"]
        for w, g, g64 in zip(want, got, got64):
            assert np.array_equal(g, w) and np.array_equal(g64, w)
    finally:
        N.destroy(td)
        N.destroy(tr)


def test_batch_argument_errors():
    rs = np.random.RandomState(1)
    t = N.build_tree(rs.rand(100, 3), None, 1)
    p4 = rs.rand(100, 3)
    t4 = N.build_tree(p4, (p4[:, 0] * 4).astype(np.int32), 4)
    try:
        with pytest.raises(N.NativeError):
            N.count_batch([(t, t)], [-1.0])
        with pytest.raises(N.NativeError):
            N.count_batch([(t, t)], [0.1], shard=2, nshards=2)
        # a 4-field query against a 1-field tree overflows the reference's
        # counter: the whole batch is refused, whatever the other jobs are
        with pytest.raises(N.NativeError, match="overflow"):
            N.count_batch([(t, t), (t, t4)], [0.1])
    finally:
        N.destroy(t)
        N.destroy(t4)
