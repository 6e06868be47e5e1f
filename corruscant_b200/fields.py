"""Jackknife field division on the sky (the reference's corruscant/fields.py).

Same classes, arguments and behaviour: ``template(N_fields, theta, phi)`` or
``template(N_fields, ra=..., dec=...)``, ``create_fields(Nside=1,
min_ratio=1.3)`` (HEALPix pixels of the data, a weighted pixel graph cut into
N_fields parts, Nside doubled until every field is populated and the
smallest holds at least min_ratio times the average, fields.py:66-144),
``assign_fields`` (the field of each point of another catalog, :146-166)
and ``assign_colors`` (Welsh-Powell colouring of the field adjacency graph,
:168-196); ``pixel`` keeps a pixel's id, count, edge neighbours and corners
(:28-34).

The reference takes the pixelisation from healpy and the graph partition
from pymetis (fields.py:22-26), neither of which is available here.  Both
are native code of this project in libcoords.so (include/fields.h): the
HEALPix RING scheme written from its published definition (the pixel a point
falls in, pixel centres, edge neighbours and corners are healpy's), and a
recursive-bisection partitioner of its own in place of METIS's.  The graph is
the reference's: every pixel a vertex weighted by its data count, joined to
its four edge neighbours, the edge weighing 1000 between two populated pixels
and 1 otherwise (so that cuts run through empty sky).  The partition is not
METIS's (its heuristics are its own), so field ids differ from the
reference's; the acceptance rule that decides Nside is the same.

Deviation: a min_ratio above 1 can never be met (the smallest field cannot
hold more than the average), and the reference then doubles Nside without
end; here such a call, or any search that passes Nside 8192, raises
ValueError.
"""
from __future__ import division, print_function

import numpy as np

from . import _native

__all__ = ["pixel", "template"]

MAX_NSIDE = 8192

_NEIGHBOURS = {}


def _edge_neighbours(Nside):
    nb = _NEIGHBOURS.get(Nside)
    if nb is None:
        nb = _native.healpix_edge_neighbours(Nside)
        _NEIGHBOURS.clear()  # one table at a time: they grow as 48 Nside^2 longs
        _NEIGHBOURS[Nside] = nb
    return nb


def _sph(ra, dec):
    """radec2sph64 (coordmath.c:73-80): theta = (90 - dec) deg, phi = ra deg."""
    ra = np.require(ra, requirements="AC", dtype="float64")
    dec = np.require(dec, requirements="AC", dtype="float64")
    theta, phi = np.empty(dec.size), np.empty(ra.size)
    _native.coordlib().radec2sph64(_native.dptr(ra), _native.dptr(dec), _native.dptr(theta),
                                   _native.dptr(phi), ra.size)
    return theta, phi


class pixel:
    """A HEALPix pixel: id, data count, its four edge neighbours
    (healpy.get_all_neighbours(Nside, id)[::2]) and its corners as unit
    vectors (healpy.boundaries), fields.py:28-34."""

    def __init__(self, Nside, id, count):
        self.id = id
        self.count = count
        self.Nside = Nside
        self.neighbors = set(int(n) for n in _edge_neighbours(Nside)[id])
        self.vertecies = set(map(tuple, _native.healpix_corners(Nside, id).T))


class template:
    """Field division of a data catalog, fields.py:36-64."""

    def __init__(self, N_fields, theta=None, phi=None, ra=None, dec=None):
        if theta is not None and phi is not None:
            self.theta = np.array(theta)
            self.phi = np.array(phi)
        else:
            self.theta, self.phi = _sph(ra, dec)
        if not (self.phi.shape == self.theta.shape):
            raise ValueError("Theta and phi arrays must be same size")
        self.N_fields = N_fields
        self.Nside = None
        # maps field IDs to color IDs
        self.color_dict = None
        self.filled_pix = None

    def create_fields(self, Nside=1, min_ratio=1.3):
        """Field id of every data point (fields.py:66-144)."""
        if min_ratio > 1:
            raise ValueError("min_ratio {:.3f} cannot be met: the smallest field holds at most "
                             "the average population".format(min_ratio))
        while True:
            if Nside > MAX_NSIDE:
                raise ValueError("no division into {:d} fields found up to Nside = {:d}"
                                 .format(self.N_fields, MAX_NSIDE))
            res = self._try_fields(Nside, min_ratio)
            if res is not None:
                return res
            Nside *= 2

    def _try_fields(self, Nside, min_ratio):
        pixels = _native.healpix_ang2pix(Nside, self.theta, self.phi)
        self.Nside = Nside
        nbins = 12 * Nside * Nside
        hist = np.bincount(pixels, minlength=nbins)

        self.filled_pix = [int(i) for i in np.flatnonzero(hist > 0)]
        npix_filled = len(self.filled_pix)
        if npix_filled < self.N_fields:
            print("Nside = {:d} too small for {:d} fields ({:d} pix with data). "
                  "Trying Nside = {:d}...".format(Nside, self.N_fields, npix_filled, 2 * Nside))
            return None

        self.pix_list = [pixel(Nside, i, hist[i]) for i in range(nbins)]
        nb = _edge_neighbours(Nside)
        # the reference's graph (fields.py:90-117): one vertex per pixel in id
        # order, its edge neighbours, weight 1000 between populated pixels
        adjncy = nb.ravel()
        xadj = np.arange(0, 4 * nbins + 1, 4)
        populated = hist > 0
        eweights = np.where(np.repeat(populated, 4) & populated[adjncy], 1000, 1)
        self.adj_dict = {i: [int(n) for n in nb[i]] for i in range(nbins)}

        _, fld_ids = _native.partition_graph(self.N_fields, xadj, adjncy, hist, eweights)

        # field id of every point
        fld_ids = np.array(fld_ids)
        pix_ids = fld_ids[np.array(pixels)]
        self.fld_ids = fld_ids

        counts = np.bincount(pix_ids, minlength=self.N_fields)
        if np.min(counts) == 0:
            print("At least one field has no population. "
                  "Trying Nside = {:d}...".format(2 * Nside))
            return None
        if float(np.min(counts)) / (np.average(counts)) < min_ratio:
            print("The smallest field has less than {:.3f} ".format(min_ratio) +
                  "times the average population. Trying "
                  "Nside = {:d}...".format(2 * Nside))
            return None
        return np.array(pix_ids)

    def assign_fields(self, theta=None, phi=None, ra=None, dec=None):
        """Field id of each point of another catalog (fields.py:146-166)."""
        if theta is not None and phi is not None:
            theta = np.array(theta)
            phi = np.array(phi)
        else:
            theta, phi = _sph(ra, dec)
        pix = _native.healpix_ang2pix(self.Nside, theta, phi)
        return self.fld_ids[pix]

    def assign_colors(self):
        """Colour ids of the fields such that touching fields differ: the
        Welsh-Powell greedy colouring (fields.py:168-196), fields taken by
        decreasing number of neighbouring fields."""
        field_graph = {}
        for key, nbs in self.adj_dict.items():
            f = self.fld_ids[key]
            for n in nbs:
                field_graph.setdefault(f, set()).add(self.fld_ids[n])
        for key in field_graph:
            field_graph[key].discard(key)

        order = sorted(field_graph, key=lambda x: len(field_graph[x]), reverse=True)
        color_dict = {}
        color = 0
        while order:
            same = []
            for key in order:
                if not any(n in same for n in field_graph[key]):
                    color_dict[key] = color
                    same.append(key)
            order = [k for k in order if k not in color_dict]
            color += 1
        self.color_dict = color_dict
        return color_dict
