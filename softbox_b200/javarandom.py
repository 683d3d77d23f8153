"""java.util.Random, restated from its published specification (Java SE API docs:
48-bit linear congruential generator, multiplier 0x5DEECE66D, addend 0xB). The
reference's scene builders (e.g. DenseContractileHarness.buildScene,
DenseContractileHarness.java:112-280) draw from it, so scenes built here match the
reference's placement order."""

_MULT = 0x5DEECE66D
_ADD = 0xB
_MASK = (1 << 48) - 1


class JavaRandom:
    def __init__(self, seed: int):
        self._seed = (seed ^ _MULT) & _MASK

    def _next(self, bits: int) -> int:
        self._seed = (self._seed * _MULT + _ADD) & _MASK
        r = self._seed >> (48 - bits)
        if r >= 1 << 31:
            r -= 1 << 32
        return r

    def next_int(self, bound=None) -> int:
        if bound is None:
            return self._next(32)
        if bound <= 0:
            raise ValueError("bound must be positive")
        r = self._next(31)
        m = bound - 1
        if (bound & m) == 0:
            return (bound * r) >> 31
        u = r
        while True:
            r = u % bound
            v = u - r + m
            if v < (1 << 31):          # int32 overflow in Java makes u - r + m negative
                return r
            u = self._next(31)

    def next_double(self) -> float:
        return ((self._next(26) << 27) + self._next(27)) * (1.0 / (1 << 53))
