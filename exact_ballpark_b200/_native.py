"""The package's native library (libebb.so, built in-tree from csrc/ by exact_ballpark_b200.build), loaded once a
process through ctypes, its entry points typed from include/ebb.h. There is no fallback: a missing or stale library
raises."""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libebb.so"
# the counting build (every IEEE operation counted; measurement only), loaded in place of the library when the process
# is started with EBB_COUNTING=1
if os.environ.get("EBB_COUNTING") == "1":
    LIB_PATH = HERE / "libebb_count.so"
ABI = 8
COLLIDE_MAX_SLOTS = 64          # include/ebb.h: EBB_COLLIDE_MAX_SLOTS
COLLIDE_MAX_STATICS = 64        # include/ebb.h: EBB_COLLIDE_MAX_STATICS
SPACE_MAX_SLOTS = 128           # include/ebb.h: EBB_SPACE_MAX_SLOTS
RAND_WORDS = 33                 # include/ebb.h: EBB_RAND_WORDS

_lib = None


class FlightState(ctypes.Structure):
    """include/ebb.h's EbbFlightState, field for field."""
    _fields_ = ([("n", ctypes.c_int64), ("friction", ctypes.c_double), ("dt", ctypes.c_double),
                 ("ffriction", ctypes.c_float), ("fdt", ctypes.c_float), ("new_orbit", ctypes.c_int32),
                 ("dynamical", ctypes.c_int32)]
                + [(k, ctypes.c_void_p) for k in (
                    "pos", "vel", "old_pos", "old_vel", "goto_pt", "last_g", "mass", "time_factor", "last_collision",
                    "radius", "max_vel", "agility", "speed_fraction", "follow_range", "max_ang_vel", "rot_agility",
                    "rot_roll", "rot", "old_rot", "ang_vel", "old_ang_vel", "torque", "ids", "effect_stamp",
                    "follow_id", "owner_id", "clock", "mode", "follow_ptr", "free_", "moribund", "massive",
                    "interactive", "sensor")])


class CombatState(ctypes.Structure):
    """include/ebb.h's EbbCombatState, field for field."""
    _fields_ = ([("flight", FlightState)]
                + [(k, ctypes.c_void_p) for k in (
                    "exists", "formation_id", "formation_slots", "owner_ptr", "hits_n", "ev_n", "ev_self", "bubble",
                    "cloaked", "flags", "formations", "formation_len")]
                + [("n_formations", ctypes.c_int64), ("max_slots", ctypes.c_int64), ("tick_ms", ctypes.c_int64),
                   ("do_missiles_off", ctypes.c_int32), ("master", ctypes.c_int32), ("active", ctypes.c_void_p)])


class ComposedState(ctypes.Structure):
    """include/ebb.h's EbbComposedState, field for field."""
    _fields_ = ([("combat", CombatState)]
                + [(k, ctypes.c_void_p) for k in ("world", "last_c", "level", "key", "mod", "hits")]
                + [("hit_cap", ctypes.c_int64)])


class ServerState(ctypes.Structure):
    """include/ebb.h's EbbServerState, field for field."""
    _fields_ = ([("flight", FlightState), ("worlds", ctypes.c_int64), ("width", ctypes.c_int64)]
                + [(k, ctypes.c_void_p) for k in ("world_rows", "world_ids", "pilot", "exists", "label", "cloaked",
                                                  "bubble", "refiled", "stamp_for_system", "bubble_time", "dead",
                                                  "settled", "fresh", "listed")]
                + [("neg_kdt", ctypes.c_double), ("master", ctypes.c_int32)])


class ServerQueue(ctypes.Structure):
    """include/ebb.h's EbbServerQueue, field for field."""
    _fields_ = ([("slots", ctypes.c_int64)]
                + [(k, ctypes.c_void_p) for k in ("kinds", "mask", "ball", "target", "n", "loc_in", "f", "ok", "row",
                                                  "trow", "loc", "route", "notice", "stamp", "clock", "has_character",
                                                  "gets_bubble")])


SPACE_SLOT_FIELDS = ("level", "key", "mod", "active", "bubble", "old_bubble", "seq", "my_box", "my_top")
SPACE_FLAG_FIELDS = ("in_park", "keep_alive", "dead", "dropped")
SPACE_BOX_FIELDS = ("box_level", "box_key", "box_balls", "box_kids", "box_bubble", "stack", "box_n", "free_boxes",
                    "box_hash", "box_free", "box_free_n")
SPACE_DICT_FIELDS = ("dict_bubble", "dict_n", "entry_bubble", "entry_id", "entry_value", "entry_n", "inter_bubble",
                     "inter_id", "inter_n", "keep_bubble", "keep_id", "keep_n", "bubble_id", "seq_next", "flags")


SPACE_SENSOR_FIELDS = ("srange", "speriod", "selapsed", "ntf_range", "trk_range", "trk", "cloaked", "sonly",
                       "has_prox", "ntf_in", "trk_in", "slist", "slen", "sbkt", "pmap", "pn", "pbkt", "ev", "evn", "rnd")


class SpaceState(ctypes.Structure):
    """include/ebb.h's EbbSpaceState, field for field."""
    _fields_ = ([(k, ctypes.c_int64) for k in ("worlds", "slots", "boxes", "dicts", "entries", "sets")]
                + [(k, ctypes.c_void_p) for k in ("rows",) + SPACE_SLOT_FIELDS + SPACE_FLAG_FIELDS + SPACE_BOX_FIELDS
                   + SPACE_DICT_FIELDS]
                + [("umap_cap", ctypes.c_int64), ("events", ctypes.c_int64)]
                + [(k, ctypes.c_void_p) for k in SPACE_SENSOR_FIELDS]
                + [("smask", ctypes.c_void_p), ("pmask", ctypes.c_void_p), ("lanes", ctypes.c_int64),
                   ("pitch", ctypes.c_int64)]
                + [(k, ctypes.c_void_p) for k in ("box_parent", "box_top", "box_home", "box_slot", "fbox")])


class SpaceQuery(ctypes.Structure):
    """include/ebb.h's EbbSpaceQuery, field for field."""
    _fields_ = [("kind", ctypes.c_int64)] + [(k, ctypes.c_void_p) for k in ("a", "b", "f", "out", "outd")]


class SpaceTape(ctypes.Structure):
    """include/ebb.h's EbbSpaceTape, field for field."""
    _fields_ = [("K", ctypes.c_int64), ("code", ctypes.c_void_p), ("a", ctypes.c_void_p), ("b", ctypes.c_void_p),
                ("f", ctypes.c_void_p)]


def lib() -> ctypes.CDLL:
    """The loaded library (loaded and checked on first use)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
                           " (the package has no CPU or library fallback)")
    L = ctypes.CDLL(str(LIB_PATH))
    if L.ebb_abi() != ABI:
        raise RuntimeError(f"{LIB_PATH}: ABI {L.ebb_abi()} is not {ABI}; rebuild it")
    p, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    if LIB_PATH.name == "libebb_count.so":
        for unit in ("flight", "space", "collide", "combat", "server"):
            getattr(L, "ebb_count_ops_" + unit).argtypes = [p, i32]
        L.ebb_count_sensor_paths.argtypes = [p, i32]
    L.ebb_error_string.restype = ctypes.c_char_p
    L.ebb_error_string.argtypes = [i32]
    L.ebb_flight_scratch_bytes.restype = i64
    L.ebb_flight_scratch_bytes.argtypes = [i64]
    L.ebb_flight_tick.argtypes = [ctypes.POINTER(FlightState), p, i64, p, i32]
    L.ebb_flight_tick_noalloc.argtypes = [ctypes.POINTER(FlightState), p, i32]
    L.ebb_flight_tick_tiled.argtypes = [ctypes.POINTER(FlightState), p, i64, i32, p, p, i32, i32]
    L.ebb_flight_tick_worlds.argtypes = [ctypes.POINTER(FlightState), p, p, i64, i32, p, p, p, i32, i32]
    L.ebb_plan_worlds.restype = i64
    L.ebb_plan_worlds.argtypes = [p, p, i64, i32, p, p]
    L.ebb_flight_move.argtypes = [ctypes.POINTER(FlightState), ctypes.POINTER(FlightState), p, p, i64, p, p, i32]
    L.ebb_collide_tick.argtypes = [p, p, p, p]
    L.ebb_collide_load.argtypes = [p, p, p]
    L.ebb_combat_tick.argtypes = [ctypes.POINTER(CombatState), p, i64, p, p, i32]
    L.ebb_composed_tick.argtypes = [ctypes.POINTER(ComposedState), p, i64, p, p, i32]
    L.ebb_composed_file.argtypes = [ctypes.POINTER(ComposedState), p, p, p, p, p]
    L.ebb_server_tick.argtypes = [ctypes.POINTER(ServerState), ctypes.POINTER(ServerQueue), i32, i64, i64, p, i32]
    L.ebb_space_query.argtypes = [ctypes.POINTER(FlightState), ctypes.POINTER(SpaceState), ctypes.POINTER(SpaceQuery),
                                  p, i32]
    L.ebb_space_tape.argtypes = [ctypes.POINTER(FlightState), ctypes.POINTER(SpaceState), ctypes.POINTER(SpaceTape), p,
                                 i32]
    L.ebb_glibc_srand.argtypes = [p, i64, p, p]
    L.ebb_glibc_rand.argtypes = [p, i64, i64, p, p]
    L.ebb_flight_snap.argtypes = [ctypes.POINTER(FlightState), p, i32, p, i32]
    L.ebb_flight_decay.argtypes = [ctypes.POINTER(FlightState), p, ctypes.c_double, p, i32]
    L.ebb_libm.argtypes = [i32, i64, p, p, p, p, i32]
    L.ebb_kernel_info.argtypes = [i32] + [ctypes.POINTER(i32)] * 5
    _lib = L
    return L


def check(rc: int, fn: str) -> None:
    """Raise RuntimeError for a nonzero return code of entry point `fn`."""
    if rc:
        msg = lib().ebb_error_string(rc).decode()
        raise RuntimeError(f"{fn} failed ({rc}: {msg})")
