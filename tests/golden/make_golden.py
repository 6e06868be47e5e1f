"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs only where the reference sources are available: it needs
``make -C oracle ref`` (the reference C libraries compiled from their sources
into oracle/_ref/) and, for the estimator values, the reference's Python
package, which it imports from a temporary copy of the reference tree.

    python tests/golden/make_golden.py [/path/to/reference] [--only=PART,...]

(PART: trees, estimators, coords, alltypes; default all.)

Outputs (all small):
  trees.npz        inputs + reference node arrays (semantic fields) for small
                   and adversarial point sets
  counts.npz       reference pair_count outputs for those sets, several radii
  config1.npz      the 4,000 / 80,000-point unit-cube Landy-Szalay example
                   (numpy seed 3, 6 edges logspace(-2.5,-1), fields floor(4x)):
                   DD/DR/RR per bin and the reference estimator / error values
  cross.npz        a small cross-correlation with the reference's estimators
  coords.npz       reference radec2cart64 / radecdist2cart64 / radec2sph64 outputs
  alltypes.npz     the workloads of the reference's test/test_alltypes.py
                   (3-D and angular, auto and cross, with and without
                   fields; seeded inputs): counts, every estimator x error
                   type and the reference's printed results tables
"""
import atexit
import hashlib
import os
import shutil
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from oracle import oracle as O  # noqa: E402


def point_sets():
    """Named (points, fields, num_fields) inputs for the tree / count pins."""
    rs = np.random.RandomState(20240601)
    sets = {}
    for n in (1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 15, 16, 17, 31, 32, 33, 100, 257, 1000):
        p = rs.rand(n, 3)
        f = (p[:, 0] * 3).astype(np.int32)
        sets[f"rand{n}"] = (p, f, 3)
    # duplicates: every point three times, shuffled
    base = rs.rand(300, 3)
    p = np.repeat(base, 3, axis=0)
    perm = rs.permutation(len(p))
    p = p[perm]
    sets["dup3"] = (p, (p[:, 1] * 4).astype(np.int32), 4)
    # duplicates whose copies carry different fields: the first occurrence's
    # field must win on the tree side
    base = rs.rand(200, 3)
    p = np.concatenate([base, base[:120], base[:60]])
    f = np.concatenate([np.zeros(200), np.ones(120), np.full(60, 2)]).astype(np.int32)
    perm = rs.permutation(len(p))
    sets["dupmixed"] = (p[perm], f[perm], 3)
    # lattice with many exact ties in every coordinate and repeated points
    p = rs.randint(0, 8, size=(2000, 3)) / 8.0
    sets["lattice8"] = (p, (p[:, 2] * 2).astype(np.int32), 2)
    # a planar set (zero variance in z) on a square lattice: variance ties
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), indexing="ij"), -1).reshape(-1, 2)
    p = np.column_stack([g / 11.0, np.full(len(g), 0.5)])
    p = p[rs.permutation(len(p))]
    sets["plane12"] = (p, (p[:, 0] * 2).astype(np.int32).clip(0, 1), 2)
    # signed zeros: -0.0 and +0.0 compare equal and must dedup together
    p = rs.randint(-2, 3, size=(400, 3)).astype(np.float64) * 0.25
    neg = rs.rand(*p.shape) < 0.5
    p[(p == 0) & neg] = -0.0
    sets["signedzero"] = (p, (rs.rand(400) * 2).astype(np.int32), 2)
    # one point repeated 255 times (the largest weight the reference stores)
    p = np.concatenate([np.tile([[0.25, 0.5, 0.75]], (255, 1)), rs.rand(50, 3)])
    sets["w255"] = (p, None, 1)
    # no fields at all, clustered
    c = rs.rand(20, 3)
    p = (c[rs.randint(0, 20, 3000)] + rs.normal(0, 0.01, (3000, 3))) % 1.0
    sets["clustered_nofield"] = (p, None, 1)
    return sets


RADII = np.array([0.0, 1e-3, 0.02, 0.05, 0.1, 0.25, 0.5, np.inf])


def main():
    if not O.ref_available():
        sys.exit("build the reference first: make -C oracle ref")
    R = O.RefLib()
    args = [a for a in sys.argv[1:] if not a.startswith("--only=")]
    only = [a.split("=", 1)[1].split(",") for a in sys.argv[1:] if a.startswith("--only=")]
    parts = set(only[0]) if only else {"trees", "estimators", "coords", "alltypes"}
    ref_root = args[0] if args else O.reference_root()
    if ref_root is None:
        sys.exit("reference checkout not found: set CORRUSCANT_REF")
    if "trees" in parts:
        make_tree_goldens(R)
    if "estimators" in parts:
        make_estimator_goldens(R, ref_root)
    if "coords" in parts:
        make_coord_goldens(R)
    if "alltypes" in parts:
        make_alltypes_goldens(R, ref_root)


def make_tree_goldens(R):
    trees, counts = {}, {}
    rs = np.random.RandomState(7)
    for name, (p, f, nf) in point_sets().items():
        t = R.build(p, f, nf)
        nodes = R.nodes(t)
        trees[f"{name}/points"] = p
        trees[f"{name}/fields"] = np.array([]) if f is None else f
        trees[f"{name}/num_fields"] = np.array(nf)
        trees[f"{name}/size"] = np.array(t.size)
        for k, v in nodes.items():
            trees[f"{name}/node_{k}"] = v
        # queries: the points themselves plus fresh uniform points
        q = np.concatenate([p, rs.rand(64, 3)])
        qf = None if f is None else np.concatenate([f, (rs.rand(64) * nf).astype(np.int32)])
        counts[f"{name}/queries"] = q
        counts[f"{name}/qfields"] = np.array([]) if qf is None else qf
        out = np.stack([R.pair_count(t, q, qf, nf, r, 1) for r in RADII])
        counts[f"{name}/counts"] = out
        R.destroy(t)
    # the reference's query-major counter layout when Fq != Ft (kdquery.c:34)
    p = rs.rand(500, 3)
    tf = (p[:, 0] * 3).astype(np.int32)
    q = rs.rand(300, 3)
    qf = (q[:, 1] * 2).astype(np.int32)
    t = R.build(p, tf, 3)
    counts["layout_q2_t3/points"] = p
    counts["layout_q2_t3/fields"] = tf
    counts["layout_q2_t3/queries"] = q
    counts["layout_q2_t3/qfields"] = qf
    counts["layout_q2_t3/counts"] = np.stack([R.pair_count(t, q, qf, 2, r, 1) for r in RADII])
    R.destroy(t)
    # field ids beyond 255: the reference's node keeps only the low 8 bits
    # (kdtree.h: field:8) while the query side keeps the full id
    rs2 = np.random.RandomState(300)
    p = rs2.rand(600, 3)
    f = rs2.randint(0, 300, 600).astype(np.int32)
    t = R.build(p, f, 300)
    trees["fields300/points"] = p
    trees["fields300/fields"] = f
    trees["fields300/num_fields"] = np.array(300)
    trees["fields300/size"] = np.array(t.size)
    for k, v in R.nodes(t).items():
        trees[f"fields300/node_{k}"] = v
    q = np.concatenate([p, rs2.rand(64, 3)])
    qf = np.concatenate([f, rs2.randint(0, 300, 64).astype(np.int32)])
    counts["fields300/queries"] = q
    counts["fields300/qfields"] = qf
    counts["fields300/counts"] = np.stack([R.pair_count(t, q, qf, 300, r, 1) for r in RADII])
    R.destroy(t)
    counts["radii"] = RADII
    np.savez_compressed(os.path.join(HERE, "trees.npz"), **trees)
    np.savez_compressed(os.path.join(HERE, "counts.npz"), **counts)


_REF_PY = {}


def _ref_python(ref_root):
    """Import the reference's Python package from a temporary copy whose bin/
    holds the libraries compiled from the reference sources."""
    if "clustering" in _REF_PY:
        return _REF_PY["clustering"]
    tmp = tempfile.mkdtemp(prefix="refpy_")
    atexit.register(shutil.rmtree, tmp, True)
    shutil.copytree(os.path.join(ref_root, "corruscant"), os.path.join(tmp, "corruscant"))
    os.makedirs(os.path.join(tmp, "corruscant", "bin"), exist_ok=True)
    for lib in ("libkdtree.so", "libcoords.so"):
        shutil.copy(os.path.join(O.ref_path(), lib), os.path.join(tmp, "corruscant", "bin", lib))
    sys.path.insert(0, tmp)
    import corruscant.clustering as clustering  # noqa: E402
    _REF_PY["clustering"] = clustering
    return clustering


def _fake_tree(points, fields, n_fields):
    sizes = np.array([np.sum(fields == i) for i in range(n_fields)])
    return types.SimpleNamespace(N_fields=n_fields, field_sizes=sizes, points=points,
                                 fields=fields)


def _binned(R, tree, q, qf, nfq, radii):
    return np.diff(np.array([R.pair_count(tree, q, qf, nfq, r, 8).reshape(nfq, tree.num_fields)
                             for r in radii]), axis=0)


def _estimator_values(res):
    out = {"xi": res.estimate(), "err_jackknife": res.error("jackknife"),
           "err_ftf": res.error("ftf"), "err_poisson": res.error("poisson"),
           "cov_jackknife": res.covariance("jackknife"),
           "cov_jackknife_norm": res.covariance("jackknife", normalized=True),
           "cov_ftf": res.covariance("ftf")}
    np.random.seed(11)
    out["err_bootstrap_seed11"] = res.error("bootstrap")
    return out


def make_estimator_goldens(R, ref_root):
    clustering = _ref_python(ref_root)
    # config 1: test/example.py's workload
    np.random.seed(3)
    X = np.random.rand(4000, 3)
    Y = np.random.rand(80000, 3)
    radii = np.logspace(-2.5, -1.0, 6)
    fd = (X[:, 0] * 4).astype("int32")
    fr = (Y[:, 0] * 4).astype("int32")
    td, tr = R.build(X, fd, 4), R.build(Y, fr, 4)
    dd = _binned(R, td, X, fd, 4, radii)
    dr = _binned(R, tr, X, fd, 4, radii)
    rr = _binned(R, tr, Y, fr, 4, radii)
    res = clustering.autocorr_results(dd, dr, rr, _fake_tree(X, fd, 4), _fake_tree(Y, fr, 4),
                                      clustering.est_landy_szalay, radii)
    vals = _estimator_values(res)
    for est in ("standard", "hamilton"):
        res.estimator = getattr(clustering, "est_" + est)
        vals["xi_" + est] = res.estimate()
        vals["err_jackknife_" + est] = res.error("jackknife")
    np.savez_compressed(os.path.join(HERE, "config1.npz"), dd=dd, dr=dr, rr=rr,
                        radii=radii, **vals)
    R.destroy(td)
    R.destroy(tr)

    # a small cross-correlation, four trees, size-dependent orientation
    rs = np.random.RandomState(5)
    cats = [rs.rand(n, 3) for n in (1500, 1700, 30000, 28000)]
    flds = [(c[:, 0] * 4).astype("int32") for c in cats]
    trs = [R.build(c, f, 4) for c, f in zip(cats, flds)]
    d1, d2, r1, r2 = range(4)
    sz = [t.size for t in trs]
    radii = np.logspace(-2.0, -0.8, 5)
    a, b = (d1, d2) if sz[d1] > sz[d2] else (d2, d1)
    d1d2 = _binned(R, trs[a], cats[b], flds[b], 4, radii)
    d1r2 = _binned(R, trs[r2], cats[d1], flds[d1], 4, radii)
    d2r1 = _binned(R, trs[r1], cats[d2], flds[d2], 4, radii)
    a, b = (r1, r2) if sz[r1] > sz[r2] else (r2, r1)
    r1r2 = _binned(R, trs[a], cats[b], flds[b], 4, radii)
    fakes = [_fake_tree(c, f, 4) for c, f in zip(cats, flds)]
    res = clustering.crosscorr_results(d1d2, d1r2, d2r1, r1r2, *fakes,
                                       clustering.est_landy_szalay, radii)
    vals = _estimator_values(res)
    np.savez_compressed(os.path.join(HERE, "cross.npz"), seed=5, sizes=[1500, 1700, 30000, 28000],
                        radii=radii, d1d2=d1d2, d1r2=d1r2, d2r1=d2r1, r1r2=r1r2, **vals)
    for t in trs:
        R.destroy(t)


# ------------------------------------------------ test/test_alltypes.py cases

ALLTYPES_ESTIMATORS = ("standard", "hamilton", "landy-szalay")
ALLTYPES_ERRORS = (None, "poisson", "ftf", "jackknife", "bootstrap")
ALLTYPES_CASES = {
    # test/test_alltypes.py: 4k data, 20x randoms, eight fields (or none),
    # edges logspace(-2.5, -1, 6) in the cube, logspace(-1.5, 0.5, 6) degrees
    # on the sky
    "cube_nofield": dict(kind="auto", geom="cube", sizes=(4000, 80000), nfields=0, seed=41,
                         edges=(-2.5, -1.0)),
    "cube_fields": dict(kind="auto", geom="cube", sizes=(4000, 80000), nfields=8, seed=42,
                        edges=(-2.5, -1.0)),
    "cube_cross": dict(kind="cross", geom="cube", sizes=(4000, 4000, 80000, 80000), nfields=8,
                       seed=43, edges=(-2.5, -1.0)),
    "sphere_fields": dict(kind="auto", geom="sphere", sizes=(4000, 80000), nfields=8, seed=44,
                          edges=(-1.5, 0.5)),
    "sphere_cross": dict(kind="cross", geom="sphere", sizes=(4000, 4000, 80000, 80000),
                         nfields=8, seed=45, edges=(-1.5, 0.5)),
    # test/angular.py: 10k data, 200k randoms on the sky, RA quadrants as
    # fields, edges logspace(-2, 0, 6) degrees
    "sphere_quadrants": dict(kind="auto", geom="sphere", sizes=(10000, 200000), nfields=4,
                             seed=46, edges=(-2.0, 0.0)),
}


def alltypes_inputs(case):
    """Seeded inputs of one case, shaped like the reference's test scripts
    (testing.random_cube / random_sphere: unit cube, or the whole sky uniform
    in RA and sin DEC; fields are equal slices in x or in RA).  Returns the
    catalogs as ("xyz", points) or ("radec", (ra, dec)), their fields (or
    None), the nominal edges and the radii the reference's driver would pass
    to the counts (for the sky, chords of the angles in degrees, as
    angular.py:40 does)."""
    c = ALLTYPES_CASES[case]
    geom, nf = c["geom"], c["nfields"]
    rs = np.random.RandomState(c["seed"])
    cats, fields = [], []
    for n in c["sizes"]:
        if geom == "cube":
            p = rs.rand(n, 3)
            cats.append(("xyz", p))
            fields.append((p[:, 0] * nf).astype("int32") if nf else None)
        else:
            ra = rs.rand(n) * 360.0
            dec = np.arcsin(rs.rand(n) * 2.0 - 1.0) * 180.0 / np.pi
            cats.append(("radec", (ra, dec)))
            fields.append((ra / 360.0 * nf).astype("int32") if nf else None)
    nominal = np.logspace(c["edges"][0], c["edges"][1], 6)
    radii = nominal if geom == "cube" else 2.0 * np.sin(nominal * (np.pi / 180.0) / 2.0)
    return cats, fields, nominal, radii


def _sha1(*arrays):
    h = hashlib.sha1()
    for a in arrays:
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _fake_tree_sized(points, fields, n_fields, unique_size):
    """The reference tree's attributes that the results classes read
    (clustering.py:295-335): without fields, field_sizes is the unique size."""
    if fields is None:
        return types.SimpleNamespace(N_fields=1, field_sizes=np.array(unique_size),
                                     points=points, fields=None)
    return _fake_tree(points, fields, n_fields)


def make_alltypes_goldens(R, ref_root):
    clustering = _ref_python(ref_root)
    out = {}
    for case, c in ALLTYPES_CASES.items():
        kind, geom, with_fields = c["kind"], c["geom"], c["nfields"] > 0
        cats, fields, nominal, radii = alltypes_inputs(case)
        pts = [x[1] if x[0] == "xyz" else R.radec2cart64(*x[1]) for x in cats]
        nf = c["nfields"] if with_fields else 1
        trs = [R.build(p, f, nf) for p, f in zip(pts, fields)]
        fakes = [_fake_tree_sized(p, f, nf, t.size) for p, f, t in zip(pts, fields, trs)]
        out[f"{case}/inputs_sha1"] = np.array(_sha1(*pts, *fields))
        if kind == "auto":
            d, r = 0, 1
            arrays = {"dd": _binned(R, trs[d], pts[d], fields[d], nf, radii),
                      "dr": _binned(R, trs[r], pts[d], fields[d], nf, radii),
                      "rr": _binned(R, trs[r], pts[r], fields[r], nf, radii)}
            res = clustering.autocorr_results(arrays["dd"], arrays["dr"], arrays["rr"],
                                              fakes[d], fakes[r], clustering.est_landy_szalay,
                                              radii)
        else:
            d1, d2, r1, r2 = range(4)
            sz = [t.size for t in trs]
            a, b = (d1, d2) if sz[d1] > sz[d2] else (d2, d1)
            arrays = {"d1d2": _binned(R, trs[a], pts[b], fields[b], nf, radii),
                      "d1r2": _binned(R, trs[r2], pts[d1], fields[d1], nf, radii),
                      "d2r1": _binned(R, trs[r1], pts[d2], fields[d2], nf, radii)}
            a, b = (r1, r2) if sz[r1] > sz[r2] else (r2, r1)
            arrays["r1r2"] = _binned(R, trs[a], pts[b], fields[b], nf, radii)
            res = clustering.crosscorr_results(arrays["d1d2"], arrays["d1r2"], arrays["d2r1"],
                                               arrays["r1r2"], *fakes,
                                               clustering.est_landy_szalay, radii)
        for k, v in arrays.items():
            out[f"{case}/{k}"] = v
        # what twopoint.threedim / twopoint.angular set on the results
        res.radii_nominal = res.radii_euclidean if geom == "cube" else nominal
        res.radii_units = "Data units" if geom == "cube" else "degrees"
        for est in ALLTYPES_ESTIMATORS:
            res.estimator = getattr(clustering, "est_" + est.replace("-", "_"))
            out[f"{case}/xi/{est}"] = res.estimate()
            for err in ALLTYPES_ERRORS if with_fields else (None, "poisson"):
                if err is not None:
                    np.random.seed(11)
                    out[f"{case}/err/{est}/{err}"] = res.error(err)
                res.error_type = err
                np.random.seed(11)
                out[f"{case}/table/{est}/{err}"] = np.array(str(res))
            if with_fields:
                out[f"{case}/cov_jackknife/{est}"] = res.covariance("jackknife")
                out[f"{case}/cov_ftf/{est}"] = res.covariance("ftf")
        for t in trs:
            R.destroy(t)
    np.savez_compressed(os.path.join(HERE, "alltypes.npz"), **out)


def make_coord_goldens(R):
    rs = np.random.RandomState(9)
    n = 3000
    ra = rs.rand(n) * 360.0
    dec = np.degrees(np.arcsin(rs.rand(n) * 2 - 1))
    # awkward values: axes, poles, negatives, large angles
    special = np.array([0.0, -0.0, 90.0, -90.0, 180.0, 270.0, 360.0, 45.0, 30.0, 60.0,
                        1e-300, 5e-324, 720.5, -33.25, 89.999999999, 1e5])
    ra = np.concatenate([ra, special, rs.rand(16) * 90])
    dec = np.concatenate([dec, rs.rand(16) * 180 - 90, special.clip(-90, 90)])
    dist = rs.rand(ra.size) * 3000.0
    theta, phi = R.radec2sph64(ra, dec)
    np.savez_compressed(os.path.join(HERE, "coords.npz"), ra=ra, dec=dec, dist=dist,
                        xyz=R.radec2cart64(ra, dec), xyzd=R.radecdist2cart64(ra, dec, dist),
                        theta=theta, phi=phi)


if __name__ == "__main__":
    main()
