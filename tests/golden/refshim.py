"""Makes the reference's Python (exact_ballpark, read-only at a path given by EXACT_BALLPARK_REF) compute its own
arithmetic on this image, for the fixture generator only (tests/golden/make_golden.py).

Three differences between this image and the platform the reference was qualified on are shimmed, in process, before
`exact_ballpark` is imported:

1. Python 3.12 has no `math.fma`; the reference's libm transcriptions bind it at import (dlibm.py:41,
   dlibm_powf.py:40). The shim is exact: the product and sum in rationals, rounded once by `float()`.
2. torch 2.11's CPU float64 `sqrt` is not correctly rounded on x86 (about 0.7 % of arguments miss by an ulp). The
   tensor paths (vec_modes.py, vec_orient.py) need IEEE sqrt, so CPU float64/float32 tensors take numpy's, which is.
3. full.py binds the running C library's float functions through ctypes (full.py:131-133); on x86 glibc 2.39 the
   fdlibm ones (acosf, atanf, atan2f) differ from glibc 2.34 aarch64's. They are rebound to the reference's own
   transcriptions (vec_libm, dlibm_powf), which are glibc 2.34 aarch64's bit for bit.

Nothing here is imported by the package, the C oracle, bench.py or any GPU test: the reference does not exist where
those run.
"""

from __future__ import annotations

import math
import os
import sys
from fractions import Fraction

REF = os.environ.get("EXACT_BALLPARK_REF", "")
if not REF:
    raise SystemExit("set EXACT_BALLPARK_REF to a checkout of exact-ballpark: the fixtures are made by its own code")


def _fma(a: float, b: float, c: float) -> float:
    a, b, c = float(a), float(b), float(c)
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)):
        return a * b + c
    exact = Fraction(a) * Fraction(b) + Fraction(c)
    if exact == 0:
        # the sign of an exact zero: that of a*b + c under round-to-nearest
        p = a * b
        if p == 0.0 and c == 0.0:
            return p + c
        return 0.0
    return float(exact)


_installed = False


def install() -> None:
    """Install the three shims and put the reference's src/ and tests/ on sys.path (once)."""
    global _installed
    if _installed:
        return
    if not hasattr(math, "fma"):
        math.fma = _fma
    import numpy as np
    import torch

    real_sqrt = torch.sqrt

    def ieee_sqrt(x, *args, **kw):
        if isinstance(x, torch.Tensor) and x.device.type == "cpu" and x.dtype in (torch.float64, torch.float32) \
                and not args and not kw:
            return torch.from_numpy(np.sqrt(x.detach().numpy())).to(x.dtype)
        return real_sqrt(x, *args, **kw)

    torch.sqrt = ieee_sqrt
    real_method = torch.Tensor.sqrt

    def ieee_sqrt_method(self, *args, **kw):
        if self.device.type == "cpu" and self.dtype in (torch.float64, torch.float32) and not args and not kw:
            return torch.from_numpy(np.sqrt(self.detach().numpy())).to(self.dtype)
        return real_method(self, *args, **kw)

    torch.Tensor.sqrt = ieee_sqrt_method
    for p in (os.path.join(REF, "src"), os.path.join(REF, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import exact_ballpark.full as full
    from exact_ballpark import dlibm_powf, vec_libm

    def f1(fn):
        return lambda x: float(fn(torch.tensor([float(x)], dtype=torch.float64))[0])

    full._expf = f1(vec_libm.expf)
    full._logf = f1(vec_libm.logf)
    full._acosf = f1(vec_libm.acosf)
    full._sinf = f1(vec_libm.sinf)
    full._cosf = f1(vec_libm.cosf)
    full._atan2f = lambda y, x: float(vec_libm.atan2f(torch.tensor([float(y)], dtype=torch.float64),
                                                      torch.tensor([float(x)], dtype=torch.float64))[0])
    full._powf = lambda x, y: dlibm_powf.powf(float(x), float(y))
    _installed = True
