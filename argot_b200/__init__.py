"""argot_b200: ARGOT's point-source radiative-transfer hot path on B200.

The compute lives in ``libargot_b200.so`` (CUDA for sm_100a, C ABI in
``include/argot_b200.h``); this package holds its ctypes binding, the ctypes
mirrors of the reference structs, a host driver of the device-resident path
and the seeded workload generators.
"""
from . import _lib  # noqa: F401

__all__ = ["_lib", "abi", "workload", "pipeline", "build"]
__version__ = "0.1"


def load():
    """Loads the CUDA library (raises if it is not built)."""
    return _lib.load()
