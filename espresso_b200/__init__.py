"""espresso_b200: B200-native (sm_100a) P3M electrostatics and short-range
pair engine behind the interface of ESPResSo's P3M / P3MGPU actors, and the
dipolar P3M actor (DipolarP3M) on the same mesh machinery.

The compute path is libp3mx.so (C ABI in include/p3mx.h); this package holds
the ctypes binding, the actor mirrors (``electrostatics``,
``magnetostatics``), a minimal
``System`` for scripting and tests, and the batched-replica driver.
"""
from . import electrostatics  # noqa: F401
from . import interactions  # noqa: F401
from . import magnetostatics  # noqa: F401
from ._lib import load as load_library  # noqa: F401
from .system import System  # noqa: F401

__all__ = ["System", "electrostatics", "interactions", "magnetostatics", "load_library"]
