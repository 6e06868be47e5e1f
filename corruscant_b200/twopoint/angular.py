"""Angular correlation functions (corruscant/twopoint/angular.py): bin edges in
degrees, converted on the host to chord lengths 2 sin(theta/2) of the unit
sphere, exactly the reference's numpy expression (angular.py:40, :54)."""
from __future__ import division, print_function

import numpy as np

from .. import _native, clustering

__all__ = ["autocorr", "crosscorr", "cartesian", "chord"]


def __getattr__(name):
    """``coordlib``: the loaded libcoords, as the reference module binds it
    (angular.py:27-35), opened on first access."""
    if name == "coordlib":
        return _native.coordlib()
    raise AttributeError(name)


def chord(radii_deg):
    """Chord length of angular separations given in degrees."""
    radii_deg = np.array(radii_deg)
    return 2. * np.sin(radii_deg * (np.pi / 180.) / 2.)


def autocorr(data_tree, rand_tree, radii_deg, **kwargs):
    radii_deg = np.array(radii_deg)
    res = clustering._autocorr(data_tree, rand_tree, chord(radii_deg), **kwargs)
    res.radii_nominal = radii_deg
    res.radii_units = "degrees"
    return res


def crosscorr(data_tree_1, data_tree_2, rand_tree_1, rand_tree_2, radii_deg, **kwargs):
    radii_deg = np.array(radii_deg)
    res = clustering._crosscorr(data_tree_1, data_tree_2, rand_tree_1, rand_tree_2,
                                chord(radii_deg), **kwargs)
    res.radii_nominal = radii_deg
    res.radii_units = "degrees"
    return res


def cartesian(ra, dec):
    """(N,3) unit vectors from RA, DEC in degrees (angular.py:64-107)."""
    n = np.size(ra)
    ra = np.require(ra, requirements="AC", dtype="float64")
    dec = np.require(dec, requirements="AC", dtype="float64")
    out = np.empty((n, 3), dtype="float64")
    _native.coordlib().radec2cart64(_native.dptr(ra), _native.dptr(dec), _native.dptr(out), n)
    return out
