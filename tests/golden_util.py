"""Shared helpers of the tests: the golden fixtures' paths and a bit comparison."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
TRACES = ("trace_w0_do_new", "trace_w0_do_old", "trace_w0_nodo_new", "trace_mc1", "trace_mc2", "trace_fc1",
          "trace_fc2")
LIBM_CASES = (  # (function, input key, second input key or None, output key)
    ("sin", "sin_x", None, "sin_y"), ("cos", "sin_x", None, "cos_y"), ("sincos_sin", "sin_x", None, "sincos_s"),
    ("sincos_cos", "sin_x", None, "sincos_c"), ("log", "log_x", None, "log_y"), ("exp", "exp_x", None, "exp_y"),
    ("expf", "f_x", None, "expf_y"), ("sinf", "f_x", None, "sinf_y"), ("cosf", "f_x", None, "cosf_y"),
    ("atanf", "f_x", None, "atanf_y"), ("logf", "logf_x", None, "logf_y"), ("acosf", "acosf_x", None, "acosf_y"),
    ("atan2f", "f_x", "atan2f_y", "atan2f_out"), ("pow", "pow_x", "pow_y", "pow_out"),
    ("powf", "powf_x", "powf_y", "powf_out"))


def available_traces() -> list:
    return [t for t in TRACES if (GOLDEN / (t + ".npz")).exists()]


def bit_equal(a, b) -> np.ndarray:
    """Elementwise: the same float64 bits, or both NaN (the reference's comparison); integers equal."""
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind == "f" or b.dtype.kind == "f":
        a, b = a.astype(np.float64), b.astype(np.float64)
        return (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
    return a == b


F32_DIGEST_K = 0x9E3779B97F4A7C15


def f32_digest(arg_bits: np.ndarray, results: np.ndarray) -> np.uint64:
    """A chunk's digest of a float function's results: sum over the arguments, modulo 2^64, of (bits + 1) x (2 i + 1)
    x K, i the argument's binary32 pattern, bits the result's (every NaN as 0x7fc00000)."""
    y = np.asarray(results, dtype=np.float64).astype(np.float32)
    bits = y.view(np.uint32).astype(np.uint64)
    bits = np.where(np.isnan(y), np.uint64(0x7FC00000), bits)
    w = (np.asarray(arg_bits, dtype=np.uint64) * np.uint64(2) + np.uint64(1)) * np.uint64(F32_DIGEST_K)
    with np.errstate(over="ignore"):
        return np.uint64(np.sum((bits + np.uint64(1)) * w, dtype=np.uint64))
