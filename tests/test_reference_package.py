"""The reference's own Python package, unmodified apart from the documented
kdtree_t declaration fix, driving this repository's C ABI.

The package (corruscant/, imported from a temporary copy of the reference
checkout) loads corruscant/bin/libkdtree* and libcoords* by name
(corruscant/__init__.py:9-20).  Here bin/ holds this repository's host
library kd_api.c -- built as libkdtree.so with the CPU stand-in of the
device layer (tests/host/fake_device.c), since this test needs no GPU -- and
this repository's libcoords.so.  The reference's test/example.py workload
(3-D autocorrelation, four x-slab fields) and an angular autocorrelation
(RA quadrants) run through the package's unchanged twopoint API, one
pair_count call per bin edge as its drivers make them
(clustering.py:218-230), and must give, bit for bit, what the same package
gives over the libraries compiled from the reference's own sources
(oracle/_ref): counts, estimates, every error type, covariances and the
printed results table.  Each side runs in its own process (the two copies
are both named ``corruscant``).  Skipped where the reference checkout,
oracle/_ref or gcc is absent.

The fix: the reference declares kdtree_t's last
member ``args`` as one pointer, 48 bytes against C's 64, so tree_construct's
returned struct is written past the ctypes buffer; declaring it as three
pointers makes the struct 64 bytes.
"""
import os
import shutil
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF = O.reference_root()

pytestmark = pytest.mark.skipif(
    not (REF and os.path.isdir(os.path.join(REF, "corruscant")) and O.ref_available()
         and shutil.which("gcc")),
    reason="reference checkout, oracle/_ref or gcc absent")

ARGS_DECL = '("args",POINTER(c_int)),'
ARGS_FIX = '("args",POINTER(c_int) * 3),'

DRIVER = textwrap.dedent("""
    import sys
    import numpy as np
    sys.path.insert(0, sys.argv[1])
    from corruscant import clustering, twopoint

    out = {}
    # test/example.py, smaller (the CPU stand-in counts exhaustively)
    np.random.seed(3)
    X = np.random.rand(1500, 3)
    Y = np.random.rand(6000, 3)
    radii = np.logspace(-2.5, -1.0, 6)
    fd = (X[:, 0] * 4).astype("int32")
    fr = (Y[:, 0] * 4).astype("int32")
    dtree = clustering.tree(X, fd)
    rtree = clustering.tree(Y, fr)
    res = twopoint.threedim.autocorr(dtree, rtree, radii, est_type="landy-szalay",
                                     num_threads=4)
    res.error_type = "jackknife"
    out["table3d"] = np.array(str(res))

    # angular: RA/DEC converted by libcoords, RA quadrants as fields
    rs = np.random.RandomState(9)
    ra_d, dec_d = rs.uniform(0, 360, 1200), np.degrees(np.arcsin(rs.uniform(-1, 1, 1200)))
    ra_r, dec_r = rs.uniform(0, 360, 4000), np.degrees(np.arcsin(rs.uniform(-1, 1, 4000)))
    pd = twopoint.angular.cartesian(ra_d, dec_d)
    pr = twopoint.angular.cartesian(ra_r, dec_r)
    out["pts_angular"] = pd
    ang = twopoint.angular.autocorr(
        clustering.tree(pd, (ra_d // 90).astype("int32")),
        clustering.tree(pr, (ra_r // 90).astype("int32")),
        np.logspace(-0.5, 1.2, 8), est_type="hamilton", num_threads=4)
    ang.error_type = "ftf"
    out["table_angular"] = np.array(str(ang))

    for tag, r in (("3d", res), ("ang", ang)):
        out["dd_" + tag], out["dr_" + tag], out["rr_" + tag] = r.dd, r.dr, r.rr
        out["xi_" + tag] = r.estimate()
        for e in ("jackknife", "ftf", "poisson"):
            out["err_%s_%s" % (e, tag)] = r.error(e)
        out["cov_" + tag] = r.covariance("jackknife")
        np.random.seed(11)
        out["boot_" + tag] = r.error("bootstrap")
    np.savez(sys.argv[2], **out)
""")


def _package(tmp, name, libkdtree):
    """A copy of the reference package with the kdtree_t fix and the given
    libkdtree.so (libcoords: this repository's, or the reference's)."""
    root = tmp / name
    shutil.copytree(os.path.join(REF, "corruscant"), root / "corruscant")
    cl = root / "corruscant" / "clustering.py"
    src = cl.read_text()
    assert src.count(ARGS_DECL) == 1, "the reference's kdtree_t declaration changed"
    cl.write_text(src.replace(ARGS_DECL, ARGS_FIX))
    binp = root / "corruscant" / "bin"
    binp.mkdir(exist_ok=True)
    shutil.copy(libkdtree, binp / "libkdtree.so")
    coords = (os.path.join(REPO, "corruscant_b200", "bin", "libcoords.so") if name == "ours"
              else os.path.join(O.ref_path(), "libcoords.so"))
    shutil.copy(coords, binp / "libcoords.so")
    return root


def _run(root, out):
    r = subprocess.run([sys.executable, "-c", DRIVER, str(root), str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return dict(np.load(out))


def test_reference_package_over_this_abi(tmp_path):
    csrc = os.path.join(REPO, "corruscant_b200", "csrc")
    ours = tmp_path / "libkdtree_host.so"
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-I" + os.path.join(REPO, "include"),
                    "-I" + csrc, os.path.join(csrc, "kd_api.c"),
                    os.path.join(HERE, "host", "fake_device.c"), "-o", str(ours),
                    "-lpthread", "-lm"], check=True)
    got = _run(_package(tmp_path, "ours", ours), tmp_path / "ours.npz")
    want = _run(_package(tmp_path, "ref", os.path.join(O.ref_path(), "libkdtree.so")),
                tmp_path / "ref.npz")
    assert set(got) == set(want)
    for k in want:
        assert np.array_equal(got[k].view(np.uint8) if got[k].dtype.kind == "f" else got[k],
                              want[k].view(np.uint8) if want[k].dtype.kind == "f" else want[k]), k
    assert want["dd_3d"].sum() > 0 and want["dd_ang"].sum() > 0
