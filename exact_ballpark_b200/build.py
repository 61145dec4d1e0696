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
COUNT_LIB = HERE / "libebb_count.so"
SOURCES = ("ebb_flight.cu", "ebb_collide.cu", "ebb_combat.cu", "ebb_server.cu", "ebb_space.cu", "ebb_rand.cu",
           "ebb_plan.cpp")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
              "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
              "-Xptxas", "-v", "-shared"]
# per source: the space layer's program is long, branchy and latency-bound (a sequential program a world), and
# ptxas's -O1 schedule of it runs a few per cent faster on the B200 than -O3's (measured on the partition workload);
# the flight ticks' kernels are instruction-fetch-bound, and -O1's shorter code ran the tiled tick 7 % faster
# (65,536 worlds x 4 ships, dynamical orientation: 0.433 against 0.462 ms)
SOURCE_FLAGS = {"ebb_space.cu": ["-Xptxas", "-O1"], "ebb_flight.cu": ["-Xptxas", "-O1"]}


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


def build_native(force: bool = False, verbose: bool = False, counting: bool = False) -> Path:
    """Each source compiled to an object in parallel (no device code crosses files), then linked into the library.
    `counting`: the measurement build (EBB_COUNT_OPS: every IEEE operation counted) as libebb_count.so beside it."""
    from concurrent.futures import ThreadPoolExecutor
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "ebb.h"]
    target = COUNT_LIB if counting else LIB
    if not force and not _stale(target, deps):
        return target
    objdir = HERE / ("_build_count" if counting else "_build")
    objdir.mkdir(exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"] + (["-DEBB_COUNT_OPS"] if counting else [])

    def compile_one(src: str):
        obj = objdir / (src + ".o")
        r = subprocess.run([nvcc()] + compile_flags + SOURCE_FLAGS.get(src, []) + ["-c", "-o", str(obj), str(CSRC / src)],
                           capture_output=True, text=True)
        return src, obj, r

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    report = []
    for src, obj, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src} ({r.returncode}):\n{r.stderr[-4000:]}")
        report.append(r.stderr)
    tmp = target.with_suffix(".so.tmp")
    r = subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp)]
                       + [str(obj) for _, obj, _ in results], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{r.stderr[-4000:]}")
    if not counting:
        (HERE / "ptxas.txt").write_text("".join(report))
    tmp.replace(target)
    if verbose:
        print("".join(report))
    return target


if __name__ == "__main__":
    print(build_native(force=True))
