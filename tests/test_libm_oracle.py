"""The oracle's libm (ebb_libm.cuh's host build, oracle/oracle_libm.cpp) against the reference's transcriptions of
glibc 2.34 aarch64 (golden vectors tests/golden/libm.npz and libm_dense.npz, made by tests/golden/make_golden.py from
exact_ballpark/dlibm.py, vec_exp.py and vec_libm.py): bit for bit on every argument, the edge cases included."""

import numpy as np
import pytest

from golden_util import GOLDEN, LIBM_CASES, bit_equal
from oracle.park import libm


@pytest.mark.parametrize("fn,xk,yk,ok", LIBM_CASES, ids=[c[0] for c in LIBM_CASES])
def test_oracle_libm_matches_the_reference(fn, xk, yk, ok):
    z = np.load(GOLDEN / "libm.npz")
    x = z[xk]
    y = z[yk] if yk else None
    got = libm(fn, x, y)
    eq = bit_equal(got, z[ok])
    assert eq.all(), f"{fn}: {(~eq).sum()} of {eq.size} differ, first at x={x[~eq][:3]}"


def test_a_planted_fault_is_caught():
    """A one-ulp change of one output is a failure of the comparison (the test can fail)."""
    z = np.load(GOLDEN / "libm.npz")
    got = libm("sin", z["sin_x"])
    got[17] = np.nextafter(got[17], np.inf)
    assert not bit_equal(got, z["sin_y"]).all()


@pytest.mark.parametrize("fn", ("expf", "logf", "sinf", "cosf", "acosf", "atanf"))
def test_oracle_float_libm_matches_the_exhaustive_digests_on_two_chunks(fn):
    """Two of the 256 exhaustive chunks (the arguments 0x3f000000-0x3fffffff, [0.5, 2), and their negatives) through
    the oracle's libm, hashed as the reference's were (the whole range runs on the device, tests/test_gpu_libm.py)."""
    from golden_util import f32_digest
    path = GOLDEN / "libm_f32_digests.npz"
    z = np.load(path) if path.exists() else {}
    if fn not in z:
        pytest.skip(f"no exhaustive digests of {fn} recorded")
    for c in (63, 191):
        bits = np.arange(c << 24, (c + 1) << 24, dtype=np.uint64).astype(np.uint32)
        y = libm(fn, bits.view(np.float32).astype(np.float64))
        assert f32_digest(bits, y) == z[fn][c], (fn, c)


DENSE_CASES = [c for c in LIBM_CASES if c[0] in ("sin", "cos", "sincos_sin", "sincos_cos", "log", "exp", "pow")]


@pytest.mark.parametrize("fn,xk,yk,ok", DENSE_CASES, ids=[c[0] for c in DENSE_CASES])
def test_oracle_double_libm_matches_the_reference_around_its_branch_bounds(fn, xk, yk, ok):
    """The double functions on arguments packed around glibc's branch bounds (representable neighbours and relative
    nudges either side; near multiples of pi/2 up to 10^8; exp's and pow's overflow, subnormal and underflow edges;
    log near 1 and through the subnormals): tests/golden/libm_dense.npz, from the reference's transcriptions."""
    z = np.load(GOLDEN / "libm_dense.npz")
    x = z[xk]
    y = z[yk] if yk else None
    got = libm(fn, x, y)
    eq = bit_equal(got, z[ok])
    assert eq.all(), f"{fn}: {(~eq).sum()} of {eq.size} differ, first at x={x[~eq][:3]}"
