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
