"""TEST INFRASTRUCTURE, NOT THE PRODUCT. glibc 2.34's rand() after srand(seed) (random_r, TYPE_3), restated in Python
from glibc's published algorithm as the reference transcribes it (exact_ballpark/glibc_rand.py:14-45): the checker of
the device generator (exact_ballpark_b200.rand)."""

from __future__ import annotations


def _c_div(a: int, b: int) -> int:
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _i32(x: int) -> int:
    x &= 0xFFFFFFFF
    return x - (1 << 32) if x >= (1 << 31) else x


class Rand:
    def __init__(self, seed: int):
        seed &= 0xFFFFFFFF
        word = _i32(seed or 1)
        self.t = [word]
        for _ in range(30):
            hi = _c_div(word, 127773)
            lo = word - 127773 * hi
            word = 16807 * lo - 2836 * hi
            if word < 0:
                word += 2147483647
            self.t.append(word)
        self.f, self.r = 3, 0
        for _ in range(310):
            self.next()

    def next(self) -> int:
        val = (self.t[self.f] + self.t[self.r]) & 0xFFFFFFFF
        self.t[self.f] = _i32(val)
        self.f += 1
        if self.f >= 31:
            self.f, self.r = 0, self.r + 1
        else:
            self.r += 1
            if self.r >= 31:
                self.r = 0
        return val >> 1

    def state(self) -> list:
        return list(self.t) + [self.f, self.r]
