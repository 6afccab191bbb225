"""java.util.Random, restated from its published algorithm, so the reference's
seeded test inputs can be regenerated without a JVM.

The reference's kernel tests draw every input from `new Random(seed)`
(e.g. kernels/src/test/java/io/vecruntime/kernels/GroupedAggregationTest.java:77,
TestData.java:42-153). The algorithms restated here are the ones the JDK
documents for java.util.Random: a 48-bit linear congruential generator
(multiplier 0x5DEECE66D, addend 0xB) with next(bits), nextInt(),
nextInt(bound) with rejection, nextLong(), nextBoolean(), nextDouble() and
nextBytes(); the bounded nextInt(origin, bound) / nextLong(origin, bound)
of java.util.random.RandomGenerator's default methods; and
java.math.BigInteger(numBits, Random) (random magnitude from nextBytes).

Bit-for-bit agreement with a JVM is not checked here (no JDK on this image);
the golden fixtures record a digest of every regenerated input so that any
change to this file shows up as a fixture mismatch.
"""
from __future__ import annotations

_MULT = 0x5DEECE66D
_ADD = 0xB
_MASK48 = (1 << 48) - 1


def i32(x: int) -> int:
    """Wraps to a signed 32-bit int (Java int arithmetic)."""
    x &= 0xFFFFFFFF
    return x - (1 << 32) if x & 0x80000000 else x


def i64(x: int) -> int:
    """Wraps to a signed 64-bit int (Java long arithmetic)."""
    x &= 0xFFFFFFFFFFFFFFFF
    return x - (1 << 64) if x & (1 << 63) else x


def string_hash(s: str) -> int:
    """String.hashCode(): s[0]*31^(n-1) + ... + s[n-1] in int arithmetic."""
    h = 0
    for ch in s:
        h = i32(31 * h + ord(ch))
    return h


class JavaRandom:
    def __init__(self, seed: int):
        self.seed = (seed ^ _MULT) & _MASK48

    def next(self, bits: int) -> int:
        self.seed = (self.seed * _MULT + _ADD) & _MASK48
        return i32(self.seed >> (48 - bits))

    def nextInt(self, *args) -> int:
        if not args:
            return self.next(32)
        if len(args) == 1:
            return self._next_int_bound(args[0])
        return self._bounded_int(args[0], args[1])

    def _next_int_bound(self, bound: int) -> int:
        if bound <= 0:
            raise ValueError("bound must be positive")
        r = self.next(31)
        m = bound - 1
        if bound & m == 0:  # a power of two: the high bits
            return i32((bound * r) >> 31)
        u = r
        while True:
            r = u % bound
            if i32(u - r + m) >= 0:
                return r
            u = self.next(31)

    def _bounded_int(self, origin: int, bound: int) -> int:
        if origin >= bound:
            raise ValueError("bound must be greater than origin")
        r = self.nextInt()
        n = i32(bound - origin)
        m = i32(n - 1)
        if n & m == 0:
            return i32((r & m) + origin)
        if n > 0:
            u = (r & 0xFFFFFFFF) >> 1
            while True:
                r = u % n
                if i32(u + m - r) >= 0:
                    return i32(r + origin)
                u = (self.nextInt() & 0xFFFFFFFF) >> 1
        while r < origin or r >= bound:
            r = self.nextInt()
        return r

    def nextLong(self, *args) -> int:
        if not args:
            return i64((self.next(32) << 32) + self.next(32))
        origin, bound = args
        if origin >= bound:
            raise ValueError("bound must be greater than origin")
        r = self.nextLong()
        n = i64(bound - origin)
        m = i64(n - 1)
        if n & m == 0:
            return i64((r & m) + origin)
        if n > 0:
            u = (r & 0xFFFFFFFFFFFFFFFF) >> 1
            while True:
                r = u % n
                if i64(u + m - r) >= 0:
                    return i64(r + origin)
                u = (self.nextLong() & 0xFFFFFFFFFFFFFFFF) >> 1
        while r < origin or r >= bound:
            r = self.nextLong()
        return r

    def nextBoolean(self) -> bool:
        return self.next(1) != 0

    def nextDouble(self) -> float:
        return ((self.next(26) << 27) + self.next(27)) * (1.0 / (1 << 53))

    def nextBytes(self, n: int) -> bytearray:
        out = bytearray(n)
        i = 0
        while i < n:
            rnd = self.nextInt()
            for _ in range(min(n - i, 4)):
                out[i] = rnd & 0xFF
                i += 1
                rnd >>= 8
        return out


def random_biginteger(num_bits: int, rnd: JavaRandom) -> int:
    """new BigInteger(numBits, rnd): a uniform magnitude in [0, 2^numBits)."""
    nbytes = (num_bits + 7) // 8
    if nbytes == 0:
        return 0
    b = rnd.nextBytes(nbytes)
    excess = 8 * nbytes - num_bits
    b[0] &= (1 << (8 - excess)) - 1
    return int.from_bytes(bytes(b), "big")


def bit_length(x: int) -> int:
    """BigInteger.bitLength(): two's-complement length without the sign bit."""
    return x.bit_length() if x >= 0 else (-x - 1).bit_length()
