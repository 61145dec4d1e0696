"""Builds the package's native library in-tree: csrc/ -> exact_ballpark_b200/libebb.so for sm_100a.

nvcc -gencode arch=compute_100a,code=sm_100a with the exactness flags every kernel relies on: -fmad=false (no
contracted multiply-add), -prec-div=true, -prec-sqrt=true, -ftz=false, no fast math; the host side with
-ffp-contract=off. The build is skipped when the library is newer than every source.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
LIB = HERE / "libebb.so"
SOURCES = ("ebb_flight.cu", "ebb_collide.cu", "ebb_combat.cu", "ebb_server.cu", "ebb_space.cu", "ebb_rand.cu",
           "ebb_plan.cpp")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
              "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
              "-Xptxas", "-v", "-shared"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_native(force: bool = False, verbose: bool = False) -> Path:
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "ebb.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", str(tmp)] + [str(CSRC / s) for s in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stderr[-4000:]}")
    (HERE / "ptxas.txt").write_text(r.stderr)
    tmp.replace(LIB)
    if verbose:
        print(r.stderr)
    return LIB


if __name__ == "__main__":
    print(build_native(force=True))
