"""The random draws of the reference's run configuration, on the host.

azeban's run seeds one std::mt19937 with the config's "seed"
(src/azeban/run_from_config.cpp:41-46) and its random variables draw from it
through std::uniform_real_distribution<double>
(include/azeban/random/uniform.hpp).  This module restates both: the
published MT19937 generator (M. Matsumoto, T. Nishimura, ACM TOMACS 8(1),
1998) and the libstdc++ mapping of two 32-bit outputs to a double in [0, 1),
(g1 + g2 * 2^32) / 2^64 (kept below 1), then a + (b - a) x.  Only the
initialisers' few parameters per sample are drawn here; the fields
themselves are generated on the device.
"""

from __future__ import annotations


class MT19937:
    """32-bit Mersenne Twister, seeded as std::mt19937(seed)."""

    N, M = 624, 397

    def __init__(self, seed: int = 5489):
        s = [seed & 0xFFFFFFFF]
        for i in range(1, self.N):
            s.append((1812433253 * (s[-1] ^ (s[-1] >> 30)) + i) & 0xFFFFFFFF)
        self.state = s
        self.pos = self.N

    def _regenerate(self) -> None:
        s = self.state
        for i in range(self.N):
            y = (s[i] & 0x80000000) | (s[(i + 1) % self.N] & 0x7FFFFFFF)
            v = s[(i + self.M) % self.N] ^ (y >> 1)
            s[i] = v ^ 0x9908B0DF if y & 1 else v
        self.pos = 0

    def __call__(self) -> int:
        if self.pos >= self.N:
            self._regenerate()
        y = self.state[self.pos]
        self.pos += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


_ONE_BELOW = 1.0 - 2.0 ** -53


def uniform_real(rng: MT19937, a: float, b: float) -> float:
    """One std::uniform_real_distribution<double>(a, b) draw (libstdc++)."""
    g1 = rng()
    g2 = rng()
    x = (float(g1) + float(g2) * 4294967296.0) / 18446744073709551616.0
    if x >= 1.0:
        x = _ONE_BELOW
    return (b - a) * x + a
