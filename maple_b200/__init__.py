"""maple_b200: B200-native inverse-homogenization inner loop of MAPLE.

Periodic voxel FE solves (elastic 6 load cases, thermal 3) by matrix-free
multigrid-preconditioned CG on sm_100a, homogenized C^H / kappa^H, analytic
SIMP sensitivities, periodic box filter and OC update, behind the call
surface of the reference package ``maple.core`` (xing-yuu/MAPLE).
"""
from ._lib import MapleError  # noqa: F401

__version__ = "0.1.0"


def load_library():
    """Load libmaple_b200.so (raises ImportError when it is missing)."""
    from . import _lib
    return _lib.load()
