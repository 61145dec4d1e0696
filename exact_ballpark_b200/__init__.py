"""exact-ballpark-b200: the batched destiny tick (exact-ballpark's flight-mode park) on NVIDIA B200, bit-exact.

The drop-in API is exact_ballpark.vec_modes / vec_modes_cuda's: `VecModesPark`, `tick`, `ModesGraph`,
`kernel_info`. The tick runs in the native library libebb.so (csrc/, C ABI in include/ebb.h).
"""

from .modes import (VecModesPark, ModesGraph, kernel_info, libm, tick, tick_plain, tick_tiled, tick_worlds)  # noqa: F401

__all__ = ["VecModesPark", "ModesGraph", "kernel_info", "libm", "tick", "tick_plain", "tick_tiled", "tick_worlds"]
