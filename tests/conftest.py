"""The suite's configuration: the `gpu` marker (tests that need a CUDA GPU; `-m "not gpu"` runs the rest on a CPU
host), and the build of the native library and the CPU oracle before any test."""

from __future__ import annotations

import sys
from pathlib import Path

import torch  # noqa: F401  (first, before numpy)

ROOT = Path(__file__).resolve().parent.parent
for p in (str(ROOT), str(ROOT / "tests" / "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the native kernels")
    from exact_ballpark_b200.build import build_native
    from oracle.build import build as build_oracle
    build_oracle()
    try:
        build_native()
    except RuntimeError as e:                       # no nvcc: the ABI test reports it
        print(f"native build failed: {e}", file=sys.stderr)
