"""corruscant_b200: B200-native pair counting behind corruscant's API.

Mirrors the reference package (corruscant/__init__.py:1-20): the native
libraries are loaded from ``bin/`` and the user API is ``clustering`` (trees,
auto/cross-correlation drivers, estimators) and ``twopoint.threedim`` /
``twopoint.angular``.  Importing the package loads nothing; the libraries are
opened on first use.
"""
from ._native import PROJECT_PATH, loadlib  # noqa: F401
from . import _native, clustering, twopoint  # noqa: F401

__all__ = ["clustering", "twopoint", "loadlib", "PROJECT_PATH"]


def __getattr__(name):
    """``kdlib`` and ``coordlib``: the loaded native libraries, as the
    reference package exposes them (corruscant/__init__.py:19-20), opened on
    first access."""
    if name == "kdlib":
        return _native.kdlib()
    if name == "coordlib":
        return _native.coordlib()
    raise AttributeError(name)
