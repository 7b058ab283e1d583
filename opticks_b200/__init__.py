"""opticks_b200 : a B200-native (sm_100a) drop-in for the Opticks optical-photon simulate path.

The compute path is the in-tree shared library ``libphox.so`` (CUDA kernels + C ABI declared
in ``include/phox.h``).  Python here only prepares arrays and calls that ABI.
"""
from . import foundry, material, scenes  # noqa: F401  (pure numpy, no GPU needed)

__all__ = ["foundry", "material", "scenes", "engine_module"]


def engine_module():
    """import the ctypes-backed engine (loads libphox.so; raises ImportError if it is missing)"""
    from . import engine
    return engine
