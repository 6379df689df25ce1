"""java.util.Random restated (the 48-bit LCG its Javadoc specifies), so tests can
rebuild the exact random circuits and states the reference's JUnit tests draw with
`new Random(seed)` (e.g. StatevectorEngineTest.java:125-146, 462-495)."""
from __future__ import annotations

_MULT = 0x5DEECE66D
_ADD = 0xB
_MASK = (1 << 48) - 1


class JavaRandom:
    def __init__(self, seed: int):
        self.seed = (seed ^ _MULT) & _MASK

    def _next(self, bits: int) -> int:
        self.seed = (self.seed * _MULT + _ADD) & _MASK
        r = self.seed >> (48 - bits)
        if bits == 32 and r & (1 << 31):  # Java's (int) cast of a 32-bit pattern
            r -= 1 << 32
        return r

    def nextInt(self, bound: int | None = None) -> int:
        if bound is None:
            return self._next(32)
        if bound <= 0:
            raise ValueError("bound must be positive")
        r = self._next(31)
        m = bound - 1
        if bound & m == 0:
            return (bound * r) >> 31
        u = r
        while True:
            r = u % bound
            if u - r + m < (1 << 31):
                return r
            u = self._next(31)

    def nextBoolean(self) -> bool:
        return self._next(1) != 0

    def nextDouble(self) -> float:
        hi = self._next(26) & ((1 << 26) - 1)
        lo = self._next(27) & ((1 << 27) - 1)
        return ((hi << 27) + lo) * (1.0 / (1 << 53))
