"""TEST INFRASTRUCTURE, NOT THE PRODUCT. The CPU oracle of the master's partition and bubble partition of one world
(oracle/space.cpp): a stream of operations run on a fresh world, the state after each one as a text. Only tests/ use
it."""

from __future__ import annotations

import ctypes

import numpy as np

from .park import lib


def run(ops: np.ndarray, friction: float = 1.0e6, dt: float = 1.0, seed: int = 1) -> list:
    """The world's state after each operation ([n][16] doubles, oracle/space.cpp's codes), as texts; `seed` the world's
    srand seed."""
    ops = np.ascontiguousarray(ops, dtype=np.float64)
    L = lib()
    L.oracle_space_run.restype = ctypes.c_int64
    L.oracle_space_run.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64]
    n, stride = ops.shape
    need = L.oracle_space_run(ops.ctypes.data, n, stride, friction, dt, seed, None, 0)
    buf = ctypes.create_string_buffer(int(need) + 1)
    L.oracle_space_run(ops.ctypes.data, n, stride, friction, dt, seed, ctypes.addressof(buf), need + 1)
    return buf.raw[:need].decode().split("\x1e")[:-1]


def run_quiet(ops: np.ndarray, friction: float = 1.0e6, dt: float = 1.0, seed: int = 1) -> None:
    """The operations on a fresh world, no texts written (the benchmark's CPU baseline times this)."""
    ops = np.ascontiguousarray(ops, dtype=np.float64)
    L = lib()
    L.oracle_space_run.restype = ctypes.c_int64
    L.oracle_space_run.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64]
    n, stride = ops.shape
    L.oracle_space_run(ops.ctypes.data, n, stride, friction, dt, seed, None, -1)
