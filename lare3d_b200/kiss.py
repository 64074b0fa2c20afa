"""Marsaglia KISS generator as src/core/random_generator.f90 implements it.

Fortran INTEGER is 32-bit signed with wrap-around arithmetic; ISHFT is a
logical shift of the 32-bit pattern.  ``random()`` returns
(DBLE(kiss) + 2^31) / 2^32 in [0, 1) (random_generator.f90:31-53).
"""
from __future__ import annotations

import numpy as np

_M = 0xFFFFFFFF


def _s32(v: int) -> int:
    v &= _M
    return v - (1 << 32) if v & 0x80000000 else v


class Kiss:
    def __init__(self):
        # random_generator.f90:20 default seeds
        self.x, self.y, self.z, self.w = 123456789, 362436069, 521288629, 916191069

    def random(self) -> float:
        x = (69069 * self.x + 1327217885) & _M
        a1 = self.y & _M
        a2 = a1 ^ ((a1 << 13) & _M)
        a3 = a2 ^ (a2 >> 17)
        y = a3 ^ ((a3 << 5) & _M)
        z = (18000 * (self.z & 65535) + ((self.z & _M) >> 16)) & _M
        w = (30903 * (self.w & 65535) + ((self.w & _M) >> 16)) & _M
        self.x, self.y, self.z, self.w = _s32(x), _s32(y), _s32(z), _s32(w)
        kiss = _s32(x + y + ((z << 16) & _M) + w)
        return (float(kiss) + 2147483648.0) / 4294967296.0

    def init_local(self, seed: int):
        """random_init_local (random_generator.f90:57-73)."""
        self.x = _s32(self.x + seed)
        self.y = _s32(self.y + seed)
        self.z = _s32(self.z + seed)
        self.w = _s32(self.w + seed)
        for _ in range(1000):
            self.random()

    def uniform(self, n: int) -> np.ndarray:
        return np.array([self.random() for _ in range(n)], dtype=np.float64)


def seeded(seed: int) -> Kiss:
    k = Kiss()
    k.init_local(seed)
    return k
