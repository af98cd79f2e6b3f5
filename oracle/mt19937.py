"""ORACLE (test infrastructure only) -- the reference's host random streams, restated.

SAFIRE's HostRandomGenerator (src/utilities/Random.hpp:37-51) is a std::mt19937 seeded with the
64-bit output of split_seed (src/utilities/Random.cpp:7-20) and sampled through
std::uniform_real_distribution<double>(0, 1).  execute.cpp:124-125 makes two of them from one seed:
stream 0 for the walkers (population control's comb draws one uniform per call,
population_control.hpp:34-42) and stream 1 for the auxiliary fields (assemble_X draws nwalk x nchol
uniforms per step, walker-major, AFQMCBasePropagator.cpp:708-716).

  * split_seed: the splitmix64 finalizer of (seed << 32 | stream << 24 | rank).
  * std::mt19937: the published MT19937 (Matsumoto & Nishimura 1998): seeding by the recurrence
    x[i] = 1812433253 * (x[i-1] ^ (x[i-1] >> 30)) + i on the low 32 bits of the seed, the twist
    and the tempering of the paper.  std::mt19937's result_type is 64 bits wide with libstdc++ on
    x86-64, and seeding reduces the seed modulo 2^32.
  * uniform_real_distribution<double>(0, 1) with libstdc++: generate_canonical<double, 53> takes
    k = 2 draws, u = (g1 + g2 * 2^32) / 2^64, and returns the largest double below 1 if the
    quotient rounds up to 1.

Pinned in the tests by the C++ standard's known answer (the 10000th output of a default-seeded
std::mt19937 is 4123659995) and by numpy's independent MT19937 (RandomState's integer seeding uses
the same init_genrand recurrence).
"""
import numpy as np

_N, _M = 624, 397
_MATRIX_A = 0x9908B0DF
_UPPER, _LOWER = 0x80000000, 0x7FFFFFFF
_M64 = (1 << 64) - 1


def split_seed(seed, rank=0, stream=0):
    """Random.cpp:7-20: distinct (seed, rank, stream) triples give distinct 64-bit seeds."""
    x = ((int(seed) & 0xFFFFFFFF) << 32 | (int(stream) & 0xFF) << 24 | (int(rank) & 0xFFFFFFFF)) & _M64
    x = (x + 0x9E3779B97F4A7C15) & _M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & _M64
    return x ^ (x >> 31)


class MT19937:
    """std::mt19937: 32-bit outputs, generated a state block (624 words) at a time."""

    def __init__(self, seed=5489):
        s = int(seed) & 0xFFFFFFFF
        mt = [0] * _N
        mt[0] = s
        for i in range(1, _N):
            mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.mt = np.array(mt, dtype=np.uint32)
        self.out = np.zeros(0, np.uint32)
        self.pos = _N  # the first draw twists

    def _twist(self):
        mt = self.mt.astype(np.uint64)
        # word i takes word i + 397 (mod 624); for i >= 227 that word was already replaced in this
        # pass, so the pass runs in slices of at most 227 words, in order, each reading only words
        # that are final
        for lo, hi in ((0, _N - _M), (_N - _M, 2 * (_N - _M)), (2 * (_N - _M), _N - 1)):
            y = (mt[lo:hi] & _UPPER) | (mt[lo + 1:hi + 1] & _LOWER)
            src = mt[lo + _M:hi + _M] if hi + _M <= _N else mt[lo + _M - _N:hi + _M - _N]
            mt[lo:hi] = src ^ (y >> 1) ^ np.where(y & 1, _MATRIX_A, 0).astype(np.uint64)
        y = (mt[_N - 1] & _UPPER) | (mt[0] & _LOWER)
        mt[_N - 1] = mt[_M - 1] ^ (y >> 1) ^ (_MATRIX_A if y & 1 else 0)
        self.mt = mt.astype(np.uint32)
        y = self.mt.astype(np.uint64)
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        self.out = (y & 0xFFFFFFFF).astype(np.uint32)
        self.pos = 0

    def raw(self, n):
        """The next n 32-bit outputs."""
        parts = []
        while n > 0:
            if self.pos >= _N:
                self._twist()
            take = min(n, _N - self.pos)
            parts.append(self.out[self.pos:self.pos + take])
            self.pos += take
            n -= take
        return np.concatenate(parts) if parts else np.zeros(0, np.uint32)


_ONE_BELOW = np.nextafter(1.0, 0.0)


class HostRandomGenerator:
    """HostRandomGenerator (Random.hpp:37-51): sampleUniformFields fills doubles on [0, 1)."""

    def __init__(self, seed64):
        self.mt = MT19937(seed64)

    def uniforms(self, n):
        g = self.mt.raw(2 * int(n)).astype(np.float64).reshape(-1, 2)
        # sum = g1 + g2 * 2^32 is exact in binary64 only up to 2^53: round it as the C++ sum does
        u = (g[:, 0] + g[:, 1] * 4294967296.0) / 18446744073709551616.0
        return np.where(u >= 1.0, _ONE_BELOW, u)
