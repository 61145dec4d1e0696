"""Exhaustive golden digests of the float functions: every one of the 2^32 float arguments of expf, logf, sinf, cosf,
acosf and atanf through the reference's own transcriptions of glibc 2.34 aarch64 (exact_ballpark/vec_libm.py), the
results hashed in 256 chunks of 2^24 consecutive bit patterns, into tests/golden/libm_f32_digests.npz.

    EXACT_BALLPARK_REF=<checkout of exact-ballpark> python tests/golden/make_libm_digests.py [--only expf,...]

A chunk's digest (tests/golden_util.f32_digest) is the sum, modulo 2^64, of (bits + 1) x (2 i + 1) x K over its
arguments, i the argument's bit pattern and bits the result's binary32 pattern (every NaN as 0x7fc00000), K an odd
constant: a permutation, a one-bit change or a sign of zero anywhere in the chunk changes it. The device's results
are hashed the same way on the GPU (tests/test_gpu_libm.py)."""

from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent))

import refshim  # noqa: E402

FUNCS = ("expf", "logf", "sinf", "cosf", "acosf", "atanf")
CHUNK = 1 << 24


def main() -> None:
    refshim.install()
    import torch

    from exact_ballpark import vec_libm as L
    from golden_util import f32_digest
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=",".join(FUNCS))
    a = ap.parse_args()
    torch.set_num_threads(8)
    out_path = HERE / "libm_f32_digests.npz"
    have = dict(np.load(out_path)) if out_path.exists() else {}
    for fn in a.only.split(","):
        t0 = time.time()
        dig = np.zeros(1 << 8, dtype=np.uint64)
        for c in range(1 << 8):
            bits = np.arange(c * CHUNK, (c + 1) * CHUNK, dtype=np.uint64).astype(np.uint32)
            x = torch.from_numpy(bits.view(np.float32).astype(np.float64))
            y = getattr(L, fn)(x).numpy()
            dig[c] = f32_digest(bits, y)
        have[fn] = dig
        np.savez_compressed(out_path, **have)
        print(f"{fn}: {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main()
