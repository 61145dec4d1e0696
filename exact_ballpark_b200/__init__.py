"""exact-ballpark-b200: exact-ballpark's batched destiny tick on NVIDIA B200, bit-exact.

The drop-in APIs are the reference's: exact_ballpark.vec_modes / vec_modes_cuda's flight-mode park (`VecModesPark`,
`tick`, `ModesGraph`, `kernel_info`) and exact_ballpark.vec_collide's collision park (`VecCollidePark`, gradient method
on spheres; `CollideGraph`) and exact_ballpark.vec_combat's combat park (`VecCombatPark`: missiles, formations,
cloaking) and
exact_ballpark.vec_composed's composed park (`VecComposedPark`: the combat park with collisions), with
exact_ballpark.vec_server's server layer over the flight park (`server.VecServer`, `server.ModesAdapter`). The ticks
run in the native library libebb.so (csrc/, C ABI in include/ebb.h).
"""

from .collide import CollideGraph, VecCollidePark  # noqa: F401
from .combat import CombatGraph, VecCombatPark  # noqa: F401
from . import server  # noqa: F401
from .composed import VecComposedPark  # noqa: F401
from .modes import (ModesGraph, VecModesPark, kernel_info, libm, tick, tick_plain, tick_tiled,  # noqa: F401
                    tick_worlds)

__all__ = ["VecModesPark", "ModesGraph", "kernel_info", "libm", "tick", "tick_plain", "tick_tiled", "tick_worlds",
           "VecCollidePark", "CollideGraph", "VecCombatPark", "CombatGraph", "VecComposedPark", "server"]
