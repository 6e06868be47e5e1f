"""The benchmark's workloads (bench.py --workload ...) at tiny scale: the
shapes each one promises, and the reference CPU leg running on them against
the reference library built from its own sources."""
import numpy as np
import pytest

import bench
from oracle import oracle as O


@pytest.mark.parametrize("name,scale,ncat,njobs,nedges,nf", [
    ("clustered3d", 0.01, 2, 3, 21, 64),
    ("angular", 0.01, 2, 3, 16, 100),
    ("mocks", 0.02, 129, 257, 13, 16),
    ("lattice", 0.01, 2, 2, 30, 27),
])
def test_workload_shapes(name, scale, ncat, njobs, nedges, nf):
    w = bench.WORKLOADS[name](scale)
    assert len(w.catalogs) == ncat and len(w.jobs) == njobs and len(w.radii) == nedges
    assert np.all(np.diff(w.radii) > 0)
    for pts, f, F in w.catalogs.values():
        assert pts.dtype == np.float64 and pts.flags.c_contiguous and pts.shape[1] == 3
        assert F == nf and f.min() >= 0 and f.max() < nf
    for _, t, q in w.jobs:
        assert t in w.catalogs and q in w.catalogs


def test_lattice_edges_are_exact_lattice_distances():
    w = bench.wl_lattice(0.01)
    k = (w.radii * 1024) ** 2
    assert np.allclose(k, np.round(k)) and k[0] == 1 and round(k[-1]) == 10486
    pts = w.catalogs["D"][0]
    assert np.array_equal(pts * 1024, np.round(pts * 1024))
    assert len(np.unique(pts, axis=0)) < len(pts)  # duplicated rows


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,scale", [("clustered3d", 0.01), ("angular", 0.01),
                                        ("lattice", 0.01)])
def test_reference_leg_runs(name, scale):
    cb = bench.cpu_baseline(bench.WORKLOADS[name](scale), n_queries=200)
    assert cb["kind"] == "reference" and cb["value"] > 0 and cb["pairs_tested_per_sample"] > 0
    if name == "angular":
        assert cb["coordinates_bit_identical"]


class _FakeNative:
    """Stands in for corruscant_b200._native in bench._build_all: records the
    arguments of every build (from several threads at once)."""

    def __init__(self):
        import threading
        self.lock = threading.Lock()
        self.calls = []

    def build_tree(self, pts, f, nf, deferred=False):
        with self.lock:
            self.calls.append((len(pts), nf, deferred))
        return ("tree", len(pts))


@pytest.mark.parametrize("name,workers", [("clustered3d", 2), ("mocks", 4), ("angular", 2)])
def test_e2e_builds_every_catalog_once(name, workers):
    w = bench.WORKLOADS[name](0.01 if name != "mocks" else 0.02)
    assert bench._e2e_workers(w) == workers
    fake = _FakeNative()
    trees = bench._build_all(fake, w, convert=True, deferred=True, workers=workers)
    assert sorted(trees) == sorted(w.catalogs)
    assert len(fake.calls) == len(w.catalogs) and all(d for _, _, d in fake.calls)
    for name_, (pts, f, nf) in w.catalogs.items():
        assert trees[name_] == ("tree", len(pts))
    # one at a time, the largest catalog is built first
    fake1 = _FakeNative()
    bench._build_all(fake1, w, convert=True, deferred=True, workers=1)
    sizes = [n for n, _, _ in fake1.calls]
    assert sizes == sorted(sizes, reverse=True)
