"""B200 (sm_100a) implementation of RELAX's per-time-step relaxation loop.

The compute path is ``relax_b200/librelax_b200.so`` (hand-written CUDA kernels
behind a C ABI, ``include/relax_b200.h``); this package is the thin host-side
mirror used by tests, the benchmark and Python callers.  Importing the
package does not load the library; ``relax_b200.lib()`` does, and raises if it
is missing.
"""
from .config import Simulation  # noqa: F401

__all__ = ["Simulation", "lib"]


def lib():
    from ._lib import load
    return load()
