// Philox-4x32-10 (Salmon et al., SC'11) and the open-interval uniforms the auxiliary fields
// are drawn from.  Stream layout: key = (seed & 0xffffffff, stream),
// counter = (pair, walker, step & 0xffffffff, step >> 32); one call gives two uniforms.
// This replaces the mt19937/cuRAND generators of the reference
// (src/utilities/Random.hpp:37-83), consumed at the same place (sampleUniformFields).
#pragma once
#include <cstdint>

namespace sfq {

enum : uint32_t { kStreamWalker = 0, kStreamFields = 1 };

struct u32x4 {
  uint32_t v[4];
};

__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
  uint64_t p = uint64_t(a) * uint64_t(b);
  hi = uint32_t(p >> 32);
  lo = uint32_t(p);
}

__host__ __device__ __forceinline__ u32x4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                        uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, hi0, lo0);
    mulhilo32(0xCD9E8D57u, c2, hi1, lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  u32x4 o;
  o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
  return o;
}

// 52-bit mantissa uniform in (0,1): ((a>>6)*2^26 + (b>>6) + 0.5) * 2^-52, exact in double.
__host__ __device__ __forceinline__ double u52(uint32_t a, uint32_t b) {
  uint64_t v = (uint64_t(a >> 6) << 26) | uint64_t(b >> 6);
  return (double(v) + 0.5) * 2.220446049250313080847263336181640625e-16;
}

__host__ __device__ __forceinline__ void field_uniform_pair(uint64_t seed, uint64_t step, uint32_t walker,
                                                            uint32_t pair, double& u0, double& u1) {
  u32x4 r = philox4x32_10(pair, walker, uint32_t(step), uint32_t(step >> 32), uint32_t(seed), kStreamFields);
  u0 = u52(r.v[0], r.v[1]);
  u1 = u52(r.v[2], r.v[3]);
}

__host__ __device__ __forceinline__ double comb_uniform(uint64_t seed, uint64_t call) {
  u32x4 r = philox4x32_10(0, 0, uint32_t(call), uint32_t(call >> 32), uint32_t(seed), kStreamWalker);
  return u52(r.v[0], r.v[1]);
}

}  // namespace sfq
