"""The device libm (ebb_libm.cuh's sm_100a build) against the reference's transcriptions of glibc 2.34 aarch64
(tests/golden/libm.npz), bit for bit, through the C ABI's ebb_libm."""

import numpy as np
import pytest
import torch

from golden_util import GOLDEN, LIBM_CASES, bit_equal

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("fn,xk,yk,ok", LIBM_CASES, ids=[c[0] for c in LIBM_CASES])
def test_device_libm_matches_the_reference(fn, xk, yk, ok):
    from exact_ballpark_b200 import libm
    z = np.load(GOLDEN / "libm.npz")
    x = torch.tensor(z[xk], device="cuda")
    y = torch.tensor(z[yk], device="cuda") if yk else None
    got = libm(fn, x, y).cpu().numpy()
    eq = bit_equal(got, z[ok])
    assert eq.all(), f"{fn}: {(~eq).sum()} of {eq.size} differ, first at x={z[xk][~eq][:3]}"


F32_FUNCS = ("expf", "logf", "sinf", "cosf", "acosf", "atanf")


def _device_digests(fn: str) -> np.ndarray:
    """The device's results for every float argument, hashed as tests/golden_util.f32_digest hashes the reference's,
    256 chunks of 2^24 bit patterns (the sums wrap modulo 2^64 in int64 arithmetic)."""
    from exact_ballpark_b200 import libm
    from golden_util import F32_DIGEST_K
    K = F32_DIGEST_K - (1 << 64)                       # the same 64 bits as an int64
    chunk = 1 << 24
    out = np.zeros(256, dtype=np.uint64)
    base = torch.arange(chunk, dtype=torch.int64, device="cuda")
    for c in range(256):
        arg = base + c * chunk
        x = arg.to(torch.int32).view(torch.float32).to(torch.float64)
        y = libm(fn, x).to(torch.float32)
        bits = y.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
        bits = torch.where(torch.isnan(y), torch.full_like(bits, 0x7FC00000), bits)
        w = (arg * 2 + 1) * K
        out[c] = np.int64(((bits + 1) * w).sum().item()).view(np.uint64)
    return out


@pytest.mark.parametrize("fn", F32_FUNCS)
def test_device_float_libm_matches_the_reference_on_every_float(fn):
    """Exhaustive: all 2^32 float arguments of the function on the device against the reference's transcription
    (tests/golden/libm_f32_digests.npz, made by tests/golden/make_libm_digests.py), chunk by chunk."""
    path = GOLDEN / "libm_f32_digests.npz"
    z = np.load(path) if path.exists() else {}
    if fn not in z:
        pytest.skip(f"no exhaustive digests of {fn} recorded")
    got = _device_digests(fn)
    bad = np.nonzero(got != z[fn])[0]
    assert not len(bad), f"{fn}: {len(bad)} of 256 chunks of 2^24 arguments differ, first chunks {bad[:5]}"
