"""B200-native d3-force tick engine.

The engine is the CUDA shared library ``_lib/libd3force_b200.so`` (built by
``build.py``) behind the C ABI of ``include/d3force_b200.h``; this package is
the host-side mirror of the d3-force API (``simulation.py``) plus the ctypes
binding (``core.py``). There is no CPU fallback: `cuda_core()` raises when the
library is missing or no CUDA device is usable.
"""

import os

from . import core
from .core import Core, CoreError
from .simulation import (Nodes, Simulation, d3_lcg, forceCenter, forceCollide, forceLink,
                         forceManyBody, forceRadial, forceSimulation, forceX, forceY)

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PACKAGE_DIR, "_lib", "libd3force_b200.so")

_cuda = None


def cuda_core():
    """The CUDA engine. Raises if the library is not built."""
    global _cuda
    if _cuda is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("CUDA engine not built: %s is missing (run build.py)" % LIB_PATH)
        _cuda = Core(LIB_PATH, "cuda")
    return _cuda


__all__ = [
    "Core", "CoreError", "Nodes", "Simulation", "core", "cuda_core", "d3_lcg", "forceCenter",
    "forceCollide", "forceLink", "forceManyBody", "forceRadial", "forceSimulation", "forceX",
    "forceY", "LIB_PATH",
]
