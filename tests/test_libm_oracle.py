"""The oracle's libm (ebb_libm.cuh's host build, oracle/oracle_libm.cpp) against the reference's transcriptions of
glibc 2.34 aarch64 (golden vectors tests/golden/libm.npz, made by tests/golden/make_golden.py from
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
