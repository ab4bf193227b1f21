"""MT19937 + the VSL uniform mappings used by the reference's disorder generators.

Test infrastructure (see oracle/__init__.py).  Published algorithm: Matsumoto &
Nishimura, "Mersenne Twister", ACM TOMACS 8(1) 1998 (init_genrand seeding,
tempered 32-bit outputs).  The MKL calls it stands in for:

* ``vslNewStream(MT19937, seed)``   -- ``MT19937(seed)``
* ``vslSkipAheadStream(n)``         -- ``skip(n)``
* ``viRngUniformBits``              -- ``bits(n)``
* ``vdRngUniform(a, b)``            -- ``uniform(n, a, b)``: one 32-bit output x per
  value, ``a + (b - a) * (x * 2**-32)``.

The same mapping is used by oracle/shim/mkl.h (which the reference build links) and
by the product's host generator, so a seed gives the same disorder everywhere in
this repository; MKL's own mapping is not in the reference tree and stays unpinned.
"""
import numpy as np

_UPPER = np.uint32(0x80000000)
_LOWER = np.uint32(0x7FFFFFFF)
_MATRIX_A = np.uint32(0x9908B0DF)


class MT19937:
    def __init__(self, seed: int):
        mt = np.zeros(624, dtype=np.uint32)
        x = int(seed) & 0xFFFFFFFF
        mt[0] = x
        for i in range(1, 624):
            x = (1812433253 * (x ^ (x >> 30)) + i) & 0xFFFFFFFF
            mt[i] = x
        self.mt = mt
        self.out = np.empty(0, dtype=np.uint32)
        self.pos = 0

    def _twist(self):
        mt = self.mt
        # Sequential order: new mt[i] reads old mt[i+1] and mt[(i+397)%624], which is
        # old for i<227 and already new for i>=227.  These chunks keep that order.
        for lo, hi in ((0, 227), (227, 454), (454, 623), (623, 624)):
            i = np.arange(lo, hi)
            y = (mt[i] & _UPPER) | (mt[(i + 1) % 624] & _LOWER)
            v = mt[(i + 397) % 624] ^ (y >> np.uint32(1))
            v = np.where((y & np.uint32(1)) != 0, v ^ _MATRIX_A, v).astype(np.uint32)
            mt[lo:hi] = v
        y = mt.copy()
        y ^= y >> np.uint32(11)
        y ^= (y << np.uint32(7)) & np.uint32(0x9D2C5680)
        y ^= (y << np.uint32(15)) & np.uint32(0xEFC60000)
        y ^= y >> np.uint32(18)
        self.out = y
        self.pos = 0

    def bits(self, n: int) -> np.ndarray:
        res = np.empty(n, dtype=np.uint32)
        k = 0
        while k < n:
            if self.pos >= len(self.out):
                self._twist()
            take = min(n - k, len(self.out) - self.pos)
            res[k:k + take] = self.out[self.pos:self.pos + take]
            self.pos += take
            k += take
        return res

    def skip(self, n: int) -> None:
        while n > 0:
            if self.pos >= len(self.out):
                self._twist()
            take = min(n, len(self.out) - self.pos)
            self.pos += take
            n -= take

    def uniform(self, n: int, a: float, b: float) -> np.ndarray:
        u = self.bits(n).astype(np.float64) * (1.0 / 4294967296.0)
        return a + (b - a) * u


def rlm_disorder(impurity_num: int, L1: float, L2: float, seed: int, sample: int):
    """rlm/disorder_potential.cpp:3-21: a fresh stream per sample, skipped 3*N_imp*sample."""
    s = MT19937(seed)
    s.skip(3 * impurity_num * sample)
    x = s.uniform(impurity_num, 0.0, L1)
    y = s.uniform(impurity_num, 0.0, L2)
    bits = s.bits(impurity_num)
    strength = np.where(bits % 2 == 0, 1.0, -1.0)
    return x, y, strength


def hlm_potentials(seed: int, n_sites: int, n_sample: int) -> np.ndarray:
    """hlm/main_hlm_cpu.cpp:66-67,79: one run-long stream, n_sites draws in [-1,1) per sample."""
    s = MT19937(seed)
    return np.stack([s.uniform(n_sites, -1.0, 1.0) for _ in range(n_sample)]) if n_sample else \
        np.zeros((0, n_sites))
