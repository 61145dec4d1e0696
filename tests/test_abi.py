"""The C ABI without a GPU: libebb.so loads, exports every entry point include/ebb.h declares, reports its ABI
version, and refuses bad arguments before launching anything."""

import ctypes
import re

from exact_ballpark_b200 import _native
from golden_util import GOLDEN

HEADER = GOLDEN.parent.parent / "include" / "ebb.h"


def declared() -> list:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ebb_[a-z0-9_]+)\s*\(", text)))


def test_the_library_exports_every_declared_entry_point():
    lib = _native.lib()
    names = declared()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_scratch_size():
    lib = _native.lib()
    assert lib.ebb_abi() == _native.ABI == 8
    assert lib.ebb_flight_scratch_bytes(0) == 0
    b = lib.ebb_flight_scratch_bytes(1000)
    assert b >= 1000 * (8 * 7 + 1) and b % 256 == 0


def test_refused_arguments_launch_nothing():
    lib = _native.lib()
    s = _native.FlightState()
    s.n = 16
    assert lib.ebb_flight_tick(ctypes.byref(s), None, 0, None, 128) == -1          # no scratch
    assert lib.ebb_flight_tick(ctypes.byref(s), ctypes.c_void_p(256), 1 << 20, None, 100) == -1   # block % 32
    assert lib.ebb_flight_tick_tiled(ctypes.byref(s), None, 1, 128, None, None, 128, 1) == -1
    assert lib.ebb_libm(99, 4, ctypes.c_void_p(256), None, ctypes.c_void_p(512), None, 128) == -1
    assert lib.ebb_error_string(-1).decode().startswith("refused")
    s.n = 0
    assert lib.ebb_flight_tick(ctypes.byref(s), None, 0, None, 128) == 0             # nothing to do


def test_the_server_tick_refuses_bad_arguments_before_launching():
    lib = _native.lib()
    s, q = _native.ServerState(), _native.ServerQueue()
    s.worlds = 0
    call = lambda phase, j0=0, j1=0, block=128: lib.ebb_server_tick(ctypes.byref(s), ctypes.byref(q), phase, j0,  # noqa: E731
                                                                     j1, None, block)
    assert call(0) == 0                                   # no worlds: nothing to do
    assert call(7) == -1 and call(-1) == -1               # no such phase
    assert call(0, block=100) == -1 and call(0, block=256) == -1
    q.slots = 257
    assert call(0) == -1                                  # more than EBB_SERVER_MAX_SLOTS
    q.slots = 4
    assert call(2, 3, 2) == -1 and call(2, 0, 5) == -1    # a history range outside the queue
    s.worlds, s.width = 8, 4
    assert call(0) == -1                                  # no world table
    assert ctypes.sizeof(_native.ServerState) == ctypes.sizeof(_native.FlightState) + 16 + 14 * 8 + 16
    assert ctypes.sizeof(_native.ServerQueue) == 8 + 17 * 8


def test_the_space_tape_refuses_bad_arguments_before_launching():
    lib = _native.lib()
    p, s, t = _native.FlightState(), _native.SpaceState(), _native.SpaceTape()
    call = lambda block=128: lib.ebb_space_tape(ctypes.byref(p), ctypes.byref(s), ctypes.byref(t), None, block)  # noqa: E731
    s.worlds, s.slots, s.boxes, s.dicts, s.entries, s.sets, t.K = 4, 10, 64, 16, 16, 16, 1
    assert call(block=100) == -1 and call(block=256) == -1
    assert call() == -1                                   # no state buffers
    s.slots = 129
    assert call() == -1                                   # more than EBB_SPACE_MAX_SLOTS
    s.slots, s.boxes = 10, 0
    assert call() == -1                                   # no box table
    s.boxes, s.worlds = 64, 0
    assert call() == 0                                    # no worlds: nothing to do
    s.worlds, t.K = 4, 0
    assert call() == 0                                    # no operations


def test_the_space_tape_refuses_a_missing_box_index_before_launching():
    """Every buffer the tape writes through is checked: with one of the box table's index, free list or filing
    buffers missing the call is refused with EBB_EINVAL, nothing launched."""
    lib = _native.lib()
    p, s, t = _native.FlightState(), _native.SpaceState(), _native.SpaceTape()
    s.worlds, s.slots, s.boxes, s.dicts, s.entries, s.sets, t.K = 4, 10, 64, 16, 16, 16, 1
    s.umap_cap, s.events, s.lanes, s.pitch = 10, 16, 32, 1024     # valid: only the missing buffer refuses the call
    fake = 4096
    for st in (p, s, t):
        for name, kind in type(st)._fields_:
            if kind is ctypes.c_void_p:
                setattr(st, name, fake)
    for missing in ("box_hash", "box_free", "box_free_n", "my_box", "my_top", "box_parent", "box_top", "box_home",
                    "box_slot", "fbox"):
        keep = getattr(s, missing)
        setattr(s, missing, None)
        rc = lib.ebb_space_tape(ctypes.byref(p), ctypes.byref(s), ctypes.byref(t), None, 128)
        assert rc == -1, missing
        setattr(s, missing, keep)
