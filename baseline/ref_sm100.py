"""The reference's own CUDA kernels built for sm_100 and driven through the reference's own public API: the Blackwell
bar, timed on the same B200 as this package's kernels (bench.py's `ref_sm100` section).

The reference (exact-ballpark 0.1.0.dev0) is installed once, offline, into `baseline/_ref/`:

    python -m pip install --no-index --no-build-isolation --find-links /opt/wheelhouse --target baseline/_ref \
        --no-deps --ignore-requires-python <a copy of the reference checkout>

(its pyproject asks for Python 3.13, this image has 3.12; its one dependency, torch, is here). Its kernels are built
here by its own `build()` functions (`python baseline/ref_sm100.py`), from its sources as its compiler sees them,
with its FLAGS and its generated table headers, into `baseline/_ref/sm100/`, with two changes made in process (none
in its files):

- the "native" target list of every kernel module is sm_100 SASS alone (`compute_100` -> `sm_100`): the reference
  builds sm_90 and sm_100 SASS and compute_90 PTX, and a B200 runs the sm_100 SASS;
- the PTX read-back after each compile (`cuobjdump -ptx` and its regex check of the floating-point instructions) is
  not made, since this build reads no compiled code: `cuobjdump` is not run (it answers with an empty listing) and
  the check (`vec_orient_cuda.ptx_check`, which every other module calls, and `vec_collide_cuda.ptx_check`)
  answers that it was not made, which each library's manifest records under `ptx_check.not_read`. The flags that
  make the arithmetic exact (`-fmad=false -prec-div=true -prec-sqrt=true -ftz=false`) are the reference's own.

Two shims for Python 3.12: it has no `math.fma`, which the reference's scalar libm binds at import (dlibm.py,
dlibm_powf.py), so it gets an exact one (product and sum in rationals, rounded once) before the import (the kernels
do not use it); and its `Path.read_text` takes no `newline`, which `_cuda_build.SourcePath.read_text` passes on, so
that method reads the text without it (the same text: the argument is None there).

On the GPU box `install()` makes the same changes and points the reference's kernel cache at `baseline/_ref/sm100/`,
so its `load_library()` finds the libraries built here by their own build keys and compiles nothing.
"""

from __future__ import annotations

import importlib
import math
import os
import subprocess
import sys
from fractions import Fraction
from pathlib import Path

REF = Path(__file__).resolve().parent / "_ref"
CACHE = REF / "sm100"
SM100 = [("compute_100", "sm_100")]
NOT_READ = ("cuobjdump was not run: this build reads no compiled code, so the reference's PTX check of its "
            "floating-point instructions is not made; the compile flags are the reference's own")
# the reference's kernel modules, in dependency order
MODULES = ("vec_orient_cuda", "vec_modes_cuda", "vec_collide_cuda", "vec_combat_cuda", "vec_composed_cuda",
           "vec_server_cuda", "vec_space", "vec_server_space_cuda")
_done = False


def _fma(a: float, b: float, c: float) -> float:
    a, b, c = float(a), float(b), float(c)
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)):
        return a * b + c
    exact = Fraction(a) * Fraction(b) + Fraction(c)
    if exact == 0:
        p = a * b
        return p + c if p == 0.0 and c == 0.0 else 0.0
    return float(exact)


class _Subprocess:
    """The subprocess module as the reference's build modules see it: every command runs as asked, except
    cuobjdump, which is not run and answers with an empty listing."""

    def __getattr__(self, name):
        return getattr(subprocess, name)

    @staticmethod
    def run(cmd, *args, **kw):
        if Path(str(cmd[0])).name == "cuobjdump":
            text = kw.get("text") or kw.get("universal_newlines")
            return subprocess.CompletedProcess(cmd, 0, "" if text else b"", "" if text else b"")
        return subprocess.run(cmd, *args, **kw)


def _not_checked(ptx: str, *args, **kw) -> dict:
    """The PTX check's answer when the PTX is not read."""
    return {"fp_ops": {}, "refused": {}, "ok": True, "not_read": NOT_READ}


def unavailable() -> str | None:
    """Why the reference's kernels cannot run here (None when they can): the package or its built libraries are
    missing."""
    if not (REF / "exact_ballpark" / "vec_modes_cuda.py").is_file():
        return "the reference is not installed under baseline/_ref"
    if not CACHE.is_dir():
        return "the reference's sm_100 libraries are not built (python baseline/ref_sm100.py)"
    return None


def install() -> dict:
    """Make `exact_ballpark` (the reference) importable with its kernels built for sm_100 from `baseline/_ref/sm100`;
    returns the kernel modules by name."""
    global _done
    if not _done:
        if not hasattr(math, "fma"):
            math.fma = _fma
        os.environ["EXACT_BALLPARK_CACHE"] = str(CACHE)
        if Path("/usr/local/cuda/bin/nvcc").exists():
            os.environ.setdefault("EXACT_BALLPARK_NVCC", "/usr/local/cuda/bin/nvcc")
        for k in list(os.environ):
            if k.startswith("EXACT_BALLPARK_") and k.endswith("_CUDA_DIR"):
                del os.environ[k]                       # every library in the one cache
        if str(REF) not in sys.path:
            sys.path.insert(0, str(REF))
        _done = True
        build = importlib.import_module("exact_ballpark._cuda_build")
        if sys.version_info < (3, 13):
            def read_text(self, encoding=None, errors=None, newline=None):
                return build.expand(Path.read_text(self, encoding, errors), self.parent)
            build.SourcePath.read_text = read_text
    mods = {}
    shim = _Subprocess()
    for name in MODULES:
        m = importlib.import_module(f"exact_ballpark.{name}")
        targets = getattr(m, "TARGETS", None)
        if isinstance(targets, dict):
            targets["native"] = list(SM100)
        if hasattr(m, "subprocess"):
            m.subprocess = shim
        if callable(getattr(m, "ptx_check", None)):
            m.ptx_check = _not_checked
        mods[name] = m
    return mods


def build_all() -> list:
    """Build every library the timed parks load (the reference's own load_library calls them the same way);
    returns (library, registers and spills lines) pairs."""
    mods = install()
    out = []
    for name, kw in (("vec_orient_cuda", {}), ("vec_modes_cuda", {}), ("vec_collide_cuda", {}),
                     ("vec_collide_cuda", {"statics": True}), ("vec_collide_cuda", {"composed": True}),
                     ("vec_combat_cuda", {}), ("vec_composed_cuda", {}), ("vec_server_cuda", {}), ("vec_space", {}),
                     ("vec_server_space_cuda", {})):
        m = mods[name].build(**kw)
        out.append((m["library"], m.get("ptxas", [])))
    return out


if __name__ == "__main__":
    for lib, ptxas in build_all():
        print(lib)
        for line in ptxas:
            if "registers" in line or "spill" in line:
                print("   ", line)
