"""corruscant_b200: B200-native pair counting behind corruscant's API.

Mirrors the reference package layout (corruscant/__init__.py:1-20): the
native libraries are loaded from ``bin/`` and the user API lives in
``clustering`` (trees, auto/cross correlation drivers, estimators) and
``twopoint.threedim`` / ``twopoint.angular``.
"""
from ._native import loadlib  # noqa: F401

__all__ = ["clustering", "twopoint"]
