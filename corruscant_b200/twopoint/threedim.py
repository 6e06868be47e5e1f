"""3-D correlation functions (corruscant/twopoint/threedim.py): radii in data
units, counts by the GPU drivers of ``clustering``."""
from __future__ import division, print_function

import numpy as np

from .. import _native, clustering

__all__ = ["autocorr", "crosscorr", "cartesian"]


def __getattr__(name):
    """``coordlib``: the loaded libcoords, as the reference module binds it
    (threedim.py:28-37), opened on first access."""
    if name == "coordlib":
        return _native.coordlib()
    raise AttributeError(name)


def autocorr(data_tree, rand_tree, radii, **kwargs):
    """DD/DR/RR estimator results for bin edges ``radii`` (threedim.py:39-46)."""
    res = clustering._autocorr(data_tree, rand_tree, radii, **kwargs)
    res.radii_nominal = res.radii_euclidean
    res.radii_units = "Data units"
    return res


def crosscorr(data_tree_1, data_tree_2, rand_tree_1, rand_tree_2, radii, **kwargs):
    """D1D2/D1R2/D2R1/R1R2 estimator results (threedim.py:48-56)."""
    res = clustering._crosscorr(data_tree_1, data_tree_2, rand_tree_1, rand_tree_2, radii,
                                **kwargs)
    res.radii_nominal = res.radii_euclidean
    res.radii_units = "Data units"
    return res


def cartesian(ra, dec, distance=None, z=None, cosmology=None):
    """(N,3) Cartesian points from RA, DEC (degrees) and a distance, or from a
    redshift and an astropy-style cosmology (threedim.py:58-113)."""
    if distance is None:
        distance = cosmology.comoving_distance(np.array(z))
    ra = np.require(ra, requirements="AC", dtype="float64")
    dec = np.require(dec, requirements="AC", dtype="float64")
    distance = np.require(distance, requirements="AC", dtype="float64")
    n = ra.size
    out = np.empty((n, 3), dtype="float64")
    _native.coordlib().radecdist2cart64(_native.dptr(ra), _native.dptr(dec),
                                        _native.dptr(distance), _native.dptr(out), n)
    return out
