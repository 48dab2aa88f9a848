"""B200-native single-block GRMHD step (PPM + HLL + constrained transport +
Noble inversion) behind a C ABI, with a Python mirror of the reference's
per-block interface."""
from .api import BC, Block, Geometry, build_geometry, ks_grid  # noqa: F401
from ._lib import HamrError, load  # noqa: F401
