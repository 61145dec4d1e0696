"""TEST INFRASTRUCTURE. Builds the CPU oracle (oracle/liboracle.so) with g++: -O2 -ffp-contract=off (every
operation IEEE-rounded, nothing fused). Skipped when the library is newer than its sources."""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SOURCES = ("oracle_libm.cpp", "flight.cpp", "collide.cpp", "space.cpp")
DEPS = ("flight_state.h", "../exact_ballpark_b200/csrc/ebb_libm.cuh", "../exact_ballpark_b200/csrc/ebb_arith.cuh",
        "../exact_ballpark_b200/csrc/ebb_libm_tables.h")


def build(force: bool = False) -> Path:
    deps = [HERE / s for s in SOURCES] + [(HERE / d).resolve() for d in DEPS]
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    cxx = shutil.which("g++") or "g++"
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-o", str(tmp)]
    cmd += [str(HERE / s) for s in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed:\n{r.stderr[-4000:]}")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
