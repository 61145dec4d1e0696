"""The allocation-free tick, ebb_flight_tick_noalloc, through the C ABI.

Some callers cannot give the library device memory: an engine whose own allocator owns the GPU's memory, a loop that
must not allocate once it runs, or a binding from a language with no CUDA allocator at hand. For them the library
keeps the plain tick's records in a fixed buffer of its own (include/ebb.h: EBB_NOALLOC_MAX_ROWS rows) instead of
caller scratch. These tests hold that entry point to the regular one, ebb_flight_tick with caller scratch, bit for
bit (the tolerance every tick test here uses), over two calls in a row, and check the size limit.

This file is collected last on purpose; it passes alone in a fresh process as well as after the other tests.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

FIELDS = ("pos", "vel", "old_pos", "old_vel", "goto", "last_g", "ang_vel", "old_ang_vel", "torque", "rot", "old_rot",
          "speed_fraction", "follow_range", "last_collision", "rot_roll", "mode", "effect_stamp", "follow_id",
          "owner_id", "follow_ptr", "clock", "free", "massive", "interactive", "sensor")


def _same(a: np.ndarray, b: np.ndarray) -> bool:
    if a.dtype.kind == "f":
        a, b = a.astype(np.float64), b.astype(np.float64)
        return bool(((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))).all())
    return bool((a == b).all())


@pytest.mark.parametrize("worlds", [2048, 65536], ids=["8192_rows", "max_rows"])
def test_the_no_alloc_tick_equals_the_scratch_tick_twice(worlds):
    """Two calls in a row, on a small park and on one of exactly EBB_NOALLOC_MAX_ROWS rows (65,536 worlds of 4 ships),
    where the records' last plane ends at the buffer's end."""
    from exact_ballpark_b200 import VecModesPark, _native
    from exact_ballpark_b200.workloads import flight_worlds
    lib = _native.lib()
    w = flight_worlds(55, worlds, 4)
    assert worlds != 65536 or len(w.rows) == 262144
    parks = []
    for _ in range(2):
        p = VecModesPark(len(w.rows), device="cuda", dynamical_orientation=True, use_new_orbit=True)
        p.load(w.rows)
        w.apply(p)
        parks.append(p)
    with_scratch, without = parks
    scratch = with_scratch.scratch()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        rc = lib.ebb_flight_tick(ctypes.byref(with_scratch.state()), scratch.data_ptr(), scratch.numel(), stream, 256)
        assert rc == 0, lib.ebb_error_string(rc)
        rc = lib.ebb_flight_tick_noalloc(ctypes.byref(without.state()), stream, 256)
        assert rc == 0, lib.ebb_error_string(rc)
        torch.cuda.synchronize()
        for f in FIELDS:
            a = getattr(with_scratch, f).detach().cpu().numpy()
            b = getattr(without, f).detach().cpu().numpy()
            assert _same(a, b), f"call {call + 1}: {f} differs"


def test_the_no_alloc_tick_refuses_a_park_beyond_its_buffer():
    from exact_ballpark_b200 import _native
    lib = _native.lib()
    s = _native.FlightState()
    s.n = 262144 + 1                             # EBB_NOALLOC_MAX_ROWS + 1: refused before anything is launched
    rc = lib.ebb_flight_tick_noalloc(ctypes.byref(s), None, 256)
    assert rc == -2                              # EBB_ETOOBIG
    assert "EBB_NOALLOC_MAX_ROWS" in lib.ebb_error_string(rc).decode()
