"""cablegen_b200 -- B200-native generation and solve of 2048 endgame tablebases.

The engine (CUDA kernels + C ABI) is ``libcablegen_b200.so`` in this package
directory; it exports both the reference's C API (include/cablegen.h) and the
engine's own entry points (include/cablegen_b200.h).

* ``cablegen_b200.device``  -- device-level calls on torch CUDA tensors
* ``cablegen_b200.api``     -- the reference's C API (generate/solve/lookup ...)
* ``cablegen_b200.configs`` -- the seeded benchmark workloads
"""
from ._lib import LIB_PATH, CablegenError, ExtensionMissing  # noqa: F401

__all__ = ["LIB_PATH", "CablegenError", "ExtensionMissing"]
