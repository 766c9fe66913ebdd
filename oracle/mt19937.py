"""Default-seeded std::mt19937 + std::uniform_real_distribution<double>(a, b).

TEST INFRASTRUCTURE ONLY.  The reference's FFT and padding tests fill their
inputs from a default-constructed ``std::mt19937`` through
``std::uniform_real_distribution<real_t> dist(-1, 1)``
(test/azeban/operations/fft.cpp:198-213, test/azeban/operations/copy_to_padded.cpp:105-110).
This module regenerates those inputs so the parity tests use the same data.

The generator is the published MT19937 (Matsumoto & Nishimura 1998) with the
C++ default seed 5489.  libstdc++ draws a double from two 32-bit outputs:
x = (g1 + g2 * 2^32) / 2^64, clamped below 1, then a + (b - a) * x.
"""

from __future__ import annotations

import numpy as np

_N, _M = 624, 397
_MATRIX_A = 0x9908B0DF
_UPPER, _LOWER = 0x80000000, 0x7FFFFFFF


class MT19937:
    def __init__(self, seed: int = 5489):
        mt = [0] * _N
        mt[0] = seed & 0xFFFFFFFF
        for i in range(1, _N):
            mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.mt = np.array(mt, dtype=np.uint64)
        self.idx = _N

    def _twist(self):
        mt = self.mt
        for i in range(_N):
            y = (int(mt[i]) & _UPPER) | (int(mt[(i + 1) % _N]) & _LOWER)
            v = int(mt[(i + _M) % _N]) ^ (y >> 1)
            if y & 1:
                v ^= _MATRIX_A
            mt[i] = v
        self.idx = 0

    def next_block(self, count: int) -> np.ndarray:
        """``count`` consecutive 32-bit outputs as uint64."""
        out = np.empty(count, dtype=np.uint64)
        pos = 0
        while pos < count:
            if self.idx >= _N:
                self._twist()
            take = min(count - pos, _N - self.idx)
            y = self.mt[self.idx:self.idx + take].copy()
            y ^= y >> np.uint64(11)
            y ^= (y << np.uint64(7)) & np.uint64(0x9D2C5680)
            y ^= (y << np.uint64(15)) & np.uint64(0xEFC60000)
            y ^= y >> np.uint64(18)
            out[pos:pos + take] = y & np.uint64(0xFFFFFFFF)
            pos += take
            self.idx += take
        return out

    def uniform(self, a: float, b: float, count: int) -> np.ndarray:
        """``count`` draws of std::uniform_real_distribution<double>(a, b)."""
        raw = self.next_block(2 * count).astype(np.float64)
        x = (raw[0::2] + raw[1::2] * 4294967296.0) / 18446744073709551616.0
        x = np.where(x >= 1.0, np.nextafter(1.0, 0.0), x)
        return a + (b - a) * x
