"""ORACLE (test infrastructure only) -- Philox-4x32-10 counter-based generator in numpy.

This module is imported only by tests/, by the oracle itself, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``.  The CUDA kernels compute the same streams
in-kernel (``safire_b200/csrc/philox.cuh``); the two implementations are independent
restatements of the published algorithm (Salmon, Moraes, Dror, Shaw, "Parallel random
numbers: as easy as 1, 2, 3", SC'11) and must agree bit for bit.

The reference draws its auxiliary-field uniforms from std::mt19937 on the host or cuRAND
MT19937 on the device (src/utilities/Random.hpp:37-83) and injects them through
``sampleUniformFields`` (src/AFQMC/Propagators/AFQMCBasePropagator.cpp:709-716).  This build
replaces that generator with Philox so that every walker/step/vector draw is addressable
without sequential state; the injection point is the same.

Stream layout (shared with the CUDA side):
  key     = (seed & 0xffffffff, stream)
  counter = (pair_index, walker, step & 0xffffffff, step >> 32)
  one Philox call yields two uniforms: u0 from words (x0, x1), u1 from (x2, x3)
  u = ((x_a >> 6) * 2**26 + (x_b >> 6) + 0.5) * 2**-52    (exact, in the open interval (0,1))
"""
import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint64(0x9E3779B9)
W1 = np.uint64(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)

STREAM_WALKER = 0   # population-control comb draws
STREAM_FIELDS = 1   # auxiliary-field uniforms


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox-4x32 with 10 rounds; inputs broadcastable uint32-valued arrays."""
    c0 = np.asarray(c0, dtype=np.uint64) & MASK
    c1 = np.asarray(c1, dtype=np.uint64) & MASK
    c2 = np.asarray(c2, dtype=np.uint64) & MASK
    c3 = np.asarray(c3, dtype=np.uint64) & MASK
    k0 = np.asarray(k0, dtype=np.uint64) & MASK
    k1 = np.asarray(k1, dtype=np.uint64) & MASK
    for r in range(10):
        if r > 0:
            k0 = (k0 + W0) & MASK
            k1 = (k1 + W1) & MASK
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & MASK, lo1, (hi0 ^ c3 ^ k1) & MASK, lo0
    return c0, c1, c2, c3


def _u52(xa, xb):
    v = (xa >> np.uint64(6)) * np.uint64(1 << 26) + (xb >> np.uint64(6))
    return (v.astype(np.float64) + 0.5) * 2.0 ** -52


def uniforms(seed, stream, step, nwalk, nvec, walker0=0):
    """(nwalk, nvec) open-interval uniforms for one propagation step."""
    npair = (nvec + 1) // 2
    j = np.arange(npair, dtype=np.uint64)[None, :]
    w = (np.arange(nwalk, dtype=np.uint64) + np.uint64(walker0))[:, None]
    s = np.uint64(step)
    x0, x1, x2, x3 = philox4x32_10(j, w, s & MASK, s >> np.uint64(32),
                                   np.uint64(seed) & MASK, np.uint64(stream))
    out = np.empty((nwalk, 2 * npair), dtype=np.float64)
    out[:, 0::2] = _u52(x0, x1)
    out[:, 1::2] = _u52(x2, x3)
    return out[:, :nvec]


def comb_uniform(seed, call_index):
    """The single uniform drawn by each population-control comb call."""
    x0, x1, _, _ = philox4x32_10(0, 0, np.uint64(call_index) & MASK,
                                 np.uint64(call_index) >> np.uint64(32),
                                 np.uint64(seed) & MASK, STREAM_WALKER)
    return float(_u52(x0, x1))
