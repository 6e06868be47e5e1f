"""The multi-rank plumbing of bench.py on the CPU: two gloo ranks split the
queries with bench.shard_items (the library's interleaved split), count their share (the oracle stands in for
the GPU counter here), SUM-reduce the int64 counts and MAX-reduce a timing.
The reduced counts must equal the single-process count."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    from oracle import oracle as O
    D = bench.Dist(backend="gloo")
    rs = np.random.RandomState(5)
    pts = rs.rand(3000, 3)
    f = (pts[:, 0] * 4).astype(np.int32)
    t = O.OracleTree(pts, f, 4)
    radii = np.logspace(-2, -0.8, 6)
    idx = bench.shard_items(len(pts), D.rank, D.world, chunk=100)
    part = t.brute_counts(pts[idx], f[idx], 4, radii, nthreads=2)
    total = D.reduce(part, "SUM")
    tmax = D.reduce([float(D.rank + 1)], "MAX")
    D.barrier()
    if D.rank == 0:
        np.savez(out_path, total=total, tmax=tmax,
                 full=t.brute_counts(pts, f, 4, radii, nthreads=2))
    D.close()


def test_two_gloo_ranks_reduce_exact_counts(tmp_path):
    out = str(tmp_path / "dist.npz")
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    r = np.load(out)
    assert np.array_equal(r["total"], r["full"])
    assert float(r["tmax"][0]) == 2.0


def test_shard_items_partition():
    import bench
    for n in (0, 1, 7, 33, 156250):
        for k in (1, 2, 3, 8):
            parts = [bench.shard_items(n, s, k) for s in range(k)]
            allidx = np.sort(np.concatenate(parts))
            assert np.array_equal(allidx, np.arange(n))  # disjoint and complete
            if n >= 32 * k * 4:  # interleaved: every shard within one chunk of n/k
                assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 32
