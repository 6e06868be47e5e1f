"""Field division (corruscant_b200.fields, libcoords' HEALPix and partition
code) against the properties the reference's fields.py relies on.

healpy and pymetis, which the reference calls (fields.py:22-26), are not
installed, so nothing here is compared with them directly.  Instead:
HEALPix RING structure from its published definition (pixels per ring, ring
latitudes, equal areas, pixel centres mapping back to their pixels, the known
neighbours of the base pixels), edge neighbours that really share two
corners, and the partition's balance, cut and connectivity; then the
reference's create_fields acceptance rule, assign_fields and the colouring.
"""
import numpy as np
import pytest

from corruscant_b200 import _native as N
from corruscant_b200 import fields

NSIDES = [1, 2, 3, 4, 5, 8, 16, 33, 64]


@pytest.mark.parametrize("nside", NSIDES)
def test_pixel_centres_map_back_and_rings(nside):
    npix = 12 * nside * nside
    p = np.arange(npix)
    th, ph = N.healpix_pix2ang(nside, p)
    assert np.array_equal(N.healpix_ang2pix(nside, th, ph), p)
    # iso-latitude rings counted from the north pole: 4i pixels in the caps,
    # 4 nside in the belt; z = 1 - i^2/(3 nside^2) in the north cap
    z = np.cos(th)
    rings = np.split(z, np.flatnonzero(np.diff(z) != 0) + 1)
    sizes = [len(r) for r in rings]
    want = ([4 * i for i in range(1, nside)] + [4 * nside] * (2 * nside + 1) +
            [4 * i for i in range(nside - 1, 0, -1)])
    assert sizes == want
    for i in range(1, nside):
        assert abs(rings[i - 1][0] - (1 - i * i / (3.0 * nside * nside))) < 1e-12
    assert np.all(np.diff(z) <= 0)  # pixel ids run north to south


@pytest.mark.parametrize("nside", [1, 4, 16])
def test_equal_areas(nside):
    npix = 12 * nside * nside
    rs = np.random.RandomState(nside)
    m = 400 * npix
    cnt = np.bincount(N.healpix_ang2pix(nside, np.arccos(rs.uniform(-1, 1, m)),
                                        rs.uniform(-4 * np.pi, 4 * np.pi, m)), minlength=npix)
    chi2 = ((cnt - 400.0) ** 2 / 400.0).sum()
    assert chi2 < npix + 6 * np.sqrt(2 * npix)


def test_known_pixels():
    # Nside 1: four polar pixels around each pole, four on the equator
    assert list(N.healpix_ang2pix(1, [0.0, np.pi / 2, np.pi / 2, np.pi],
                                  [0.1, 0.0, np.pi / 2 + 0.1, 0.1])) == [0, 4, 5, 8]
    th, ph = N.healpix_pix2ang(1, np.arange(12))
    assert np.allclose(np.cos(th[:4]), 2 / 3) and np.allclose(ph[:4], np.pi / 4 * np.array([1, 3, 5, 7]))
    assert np.allclose(th[4:8], np.pi / 2) and np.allclose(ph[4:8], np.pi / 2 * np.arange(4))
    # edge neighbours (south-west, north-west, north-east, south-east) of the
    # equatorial base pixel 4 and the polar base pixel 0
    nb = N.healpix_edge_neighbours(1)
    assert list(nb[4]) == [11, 3, 0, 8]
    assert list(nb[0]) == [4, 3, 1, 5]
    with pytest.raises(ValueError):
        N.healpix_ang2pix(0, [0.1], [0.1])
    with pytest.raises(ValueError):
        N.healpix_ang2pix(4, [np.nan], [0.1])


@pytest.mark.parametrize("nside", [1, 2, 3, 8, 16])
def test_edge_neighbours_share_an_edge(nside):
    npix = 12 * nside * nside
    nb = N.healpix_edge_neighbours(nside)
    corners = np.stack([N.healpix_corners(nside, p).T for p in range(npix)])  # (npix, 4, 3)
    assert np.allclose(np.linalg.norm(corners, axis=2), 1.0)
    tol = 1e-9
    for p in range(npix):
        assert len(set(nb[p])) == 4 and p not in nb[p]
        for q in nb[p]:
            assert p in nb[q]
            # two corners in common: the shared edge
            d = np.linalg.norm(corners[p][:, None, :] - corners[q][None, :, :], axis=2)
            assert (d.min(axis=1) < tol).sum() == 2, (nside, p, q)


def _grid(nx, ny):
    adj = [[] for _ in range(nx * ny)]
    for i in range(nx):
        for j in range(ny):
            for a, b in ((i + 1, j), (i - 1, j), (i, j + 1), (i, j - 1)):
                if 0 <= a < nx and 0 <= b < ny:
                    adj[i * ny + j].append(a * ny + b)
    xadj = np.cumsum([0] + [len(a) for a in adj])
    return xadj, np.concatenate(adj)


def _connected(part, k, xadj, adjncy):
    verts = np.flatnonzero(part == k)
    if len(verts) == 0:
        return True
    seen, todo = {verts[0]}, [verts[0]]
    while todo:
        v = todo.pop()
        for u in adjncy[xadj[v]:xadj[v + 1]]:
            if part[u] == k and u not in seen:
                seen.add(u)
                todo.append(u)
    return len(seen) == len(verts)


@pytest.mark.parametrize("k", [2, 3, 7, 16])
def test_partition_of_a_grid(k):
    xadj, adjncy = _grid(40, 40)
    vw = np.ones(1600, np.int64)
    cut, part = N.partition_graph(k, xadj, adjncy, vw, np.ones(len(adjncy), np.int64))
    sizes = np.bincount(part, minlength=k)
    assert sizes.max() - sizes.min() <= 0.05 * 1600 / k + 1
    # within 1.5x of straight cuts of the square (sum of the part boundaries)
    straight = {2: 40, 3: 80, 7: 240, 16: 240}[k]
    assert cut <= 1.5 * straight, cut
    # the returned cut is the weight of edges between parts
    assert cut == sum(1 for v in range(1600) for u in adjncy[xadj[v]:xadj[v + 1]]
                      if u > v and part[u] != part[v])


def test_partition_cuts_through_light_edges():
    # two heavy 20x20 blocks joined by a light column: the bisection cuts the
    # light edges (weight 1) rather than heavy ones (weight 1000)
    nx, ny = 41, 20
    xadj, adjncy = _grid(nx, ny)
    col = np.repeat(np.arange(nx * ny) // ny, np.diff(xadj))
    ew = np.where((col == 20) | (adjncy // ny == 20), 1, 1000)
    vw = np.where(np.arange(nx * ny) // ny == 20, 0, 1)
    cut, part = N.partition_graph(2, xadj, adjncy, vw, ew)
    assert cut < 1000
    sizes = np.bincount(part, weights=vw)
    assert sizes[0] == sizes[1] == 400


def test_partition_arguments():
    xadj, adjncy = _grid(3, 3)
    with pytest.raises(ValueError):
        N.partition_graph(0, xadj, adjncy, np.ones(9), np.ones(len(adjncy)))
    bad = adjncy.copy()
    bad[0] = 99
    with pytest.raises(ValueError):
        N.partition_graph(2, xadj, bad, np.ones(9), np.ones(len(adjncy)))
    # more parts than vertices: ids stay in range (some parts empty)
    _, part = N.partition_graph(12, xadj, adjncy, np.ones(9), np.ones(len(adjncy)))
    assert part.min() >= 0 and part.max() < 12 and len(set(part)) > 1


def _sphere(n, seed=0):
    rs = np.random.RandomState(seed)
    return np.arccos(rs.uniform(-1, 1, n)), rs.uniform(0, 2 * np.pi, n)


def test_create_fields_on_the_sphere():
    # the reference's fields.py main(): 50,000 points, 20 fields, min_ratio 0.8
    theta, phi = _sphere(50_000)
    t = fields.template(20, theta, phi)
    ids = t.create_fields(min_ratio=0.8)
    h = np.bincount(ids, minlength=20)
    assert len(ids) == 50_000 and h.min() > 0 and h.min() / h.mean() >= 0.8
    assert np.array_equal(t.assign_fields(theta, phi), ids)
    # every field is one piece of sky
    nb = N.healpix_edge_neighbours(t.Nside)
    xadj = np.arange(0, nb.size + 1, 4)
    for k in range(20):
        assert _connected(t.fld_ids, k, xadj, nb.ravel())
    # touching fields get different colours
    colors = t.assign_colors()
    assert set(colors) == set(range(20))
    for p, nbs in t.adj_dict.items():
        for q in nbs:
            a, b = t.fld_ids[p], t.fld_ids[q]
            assert a == b or colors[a] != colors[b]


def test_create_fields_from_ra_dec_patch(capsys):
    rs = np.random.RandomState(14)
    ra = rs.uniform(0, 90, 100_000)
    dec = np.degrees(np.arcsin(rs.uniform(np.sin(np.radians(-10)), np.sin(np.radians(60)),
                                          100_000)))
    t = fields.template(50, ra=ra, dec=dec)
    ids = t.create_fields(min_ratio=0.5)
    h = np.bincount(ids, minlength=50)
    assert h.min() / h.mean() >= 0.5
    # the reference's messages as Nside grows
    assert "Trying Nside" in capsys.readouterr().out
    # radec2sph64 conventions: theta = (90 - dec) deg, phi = ra deg
    assert np.array_equal(t.theta, np.radians(90 - dec)) or np.allclose(
        t.theta, np.radians(90 - dec), rtol=0, atol=1e-15)
    assert np.array_equal(t.assign_fields(ra=ra, dec=dec), ids)
    p = fields.pixel(t.Nside, 5, 3)
    assert p.count == 3 and len(p.neighbors) == 4 and len(p.vertecies) == 4


def test_create_fields_rejects_unmeetable_ratio():
    theta, phi = _sphere(1000)
    with pytest.raises(ValueError):
        fields.template(4, theta, phi).create_fields(min_ratio=1.3)
    with pytest.raises(ValueError):
        fields.template(4, theta, phi[:10])
