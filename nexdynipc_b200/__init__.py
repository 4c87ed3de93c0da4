"""B200-native contact step for NexDynIPC-style rigid-body IPC.

The product is the CUDA library libnxd_b200.so (kernels + the C ABI of
include/nxd.h); this package binds it (runtime.py), describes its ABI
(abi.py) and generates the seeded synthetic scenes (scenes.py).
"""
from . import abi, scenes  # noqa: F401
from .runtime import Batch, Context, IPCSolver, NxdError, World, lib  # noqa: F401

__all__ = ["abi", "scenes", "Batch", "Context", "IPCSolver", "World", "NxdError", "lib"]
