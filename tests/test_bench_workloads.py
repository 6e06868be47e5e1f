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
