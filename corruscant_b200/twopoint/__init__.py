"""Two-point correlation functions: ``threedim`` (Cartesian) and ``angular``
(RA/DEC on the unit sphere), as in the reference's corruscant.twopoint."""
from . import angular, threedim

__all__ = ["angular", "threedim"]
