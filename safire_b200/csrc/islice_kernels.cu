// Fixed-point int8 slices of the operands of the exact-accumulation products (see islice.cuh), and
// the elementwise steps between those products in the propagation.
//
// Row exponent: for a row whose largest |x| is m, e = floor(log2 m) - 6, plus one when 2^-e m > 126,
// so that y = 2^-e x has |y| <= 126.  Slices of y, each round to nearest (ties to even):
//   q1 = rint(y),  r = 256 (y - q1),  q2 = rint(r),  q3 = rint(256 (r - q2))   (|r| <= 128)
// then a q3 of +128 is carried into q2 and a q2 of +128 or more into q1, so every slice is int8
// (|q1| <= 127).  Every step is exact in FP64, so the slices are a function of x and e alone.
#include <cstdint>

#include "common.cuh"
#include "islice.cuh"

namespace sfq {
namespace {

__device__ __forceinline__ double pow2d(int e) {
  e = e < -1022 ? -1022 : (e > 1023 ? 1023 : e);
  return __longlong_as_double((long long)(e + 1023) << 52);
}

__device__ __forceinline__ int row_exponent(double m) {
  if (!(m > 0.0)) return 0;
  int ex = 0;
  frexp(m, &ex);  // m = f 2^ex, f in [0.5, 1)
  int e = ex - 7;  // 2^-e m in [64, 128)
  if (m * pow2d(-e) > 126.0) e += 1;
  return e;
}

// slices of x at scale 2^-e (passed as s = 2^-e)
__device__ __forceinline__ void slice_value(double x, double s, int ns, int& q1, int& q2, int& q3) {
  const double y = x * s;
  const double a = rint(y);
  const double r = (y - a) * 256.0;
  const double b = rint(r);
  int i1 = int(a), i2 = int(b), i3 = 0;
  if (ns > 2) {
    i3 = int(rint((r - b) * 256.0));
    if (i3 == 128) {
      i3 = -128;
      i2 += 1;
    }
  }
  if (i2 >= 128) {
    i2 -= 256;
    i1 += 1;
  }
  q1 = i1;
  q2 = i2;
  q3 = i3;
}

struct Q {
  int8_t* p[3];
};
Q qptrs(int8_t* const* q) {
  Q r;
  for (int s = 0; s < 3; ++s) r.p[s] = q[s];
  return r;
}

__device__ __forceinline__ void put(const Q& q, int ns, long idx, double x, double s) {
  int a, b, c;
  slice_value(x, s, ns, a, b, c);
  q.p[0][idx] = int8_t(a);
  if (ns > 1) q.p[1][idx] = int8_t(b);
  if (ns > 2) q.p[2][idx] = int8_t(c);
}

// the same slices for an FP32 value, in FP32 arithmetic: every step is exact for FP32 inputs (y has
// 24 significant bits and |y| <= 126, so y - q1, 256 r and r - q2 are representable), so these are
// the slices slice_value gives for the same value
__device__ __forceinline__ void slice_value_f(float x, float s, int ns, int& q1, int& q2, int& q3) {
  const float y = x * s;
  const float a = rintf(y);
  const float r = (y - a) * 256.f;
  const float b = rintf(r);
  int i1 = int(a), i2 = int(b), i3 = 0;
  if (ns > 2) {
    i3 = int(rintf((r - b) * 256.f));
    if (i3 == 128) {
      i3 = -128;
      i2 += 1;
    }
  }
  if (i2 >= 128) {
    i2 -= 256;
    i1 += 1;
  }
  q1 = i1;
  q2 = i2;
  q3 = i3;
}
// 2^-e as a float (e within the float exponent range; rows of FP32 values always are)
__device__ __forceinline__ float pow2f(int e) {
  e = e < -126 ? -126 : (e > 127 ? 127 : e);
  return __int_as_float((e + 127) << 23);
}
// four consecutive FP32 values -> one 4-byte word per slice at idx (a multiple of 4)
__device__ __forceinline__ void put4f(const Q& q, int ns, long idx, const float (&x)[4], float s) {
  int a[4], b[4], c[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) slice_value_f(x[u], s, ns, a[u], b[u], c[u]);
  *reinterpret_cast<char4*>(q.p[0] + idx) = make_char4(char(a[0]), char(a[1]), char(a[2]), char(a[3]));
  if (ns > 1) *reinterpret_cast<char4*>(q.p[1] + idx) = make_char4(char(b[0]), char(b[1]), char(b[2]), char(b[3]));
  if (ns > 2) *reinterpret_cast<char4*>(q.p[2] + idx) = make_char4(char(c[0]), char(c[1]), char(c[2]), char(c[3]));
}

// The slices of x and of -x at once: every step of slice_value_f is exact and symmetric under
// negation (rintf rounds half to even both ways), so -x has the negated slices before the carries,
// and only the carries (q3 = +128, q2 >= 128) differ.
__device__ __forceinline__ void slice_pm_f(float x, float s, int ns, int (&p)[3], int (&m)[3]) {
  const float y = x * s;
  const float a = rintf(y);
  const float r = (y - a) * 256.f;
  const float b = rintf(r);
  const int i1 = int(a), i2 = int(b), i3 = ns > 2 ? int(rintf((r - b) * 256.f)) : 0;
  int v[2][3] = {{i1, i2, i3}, {-i1, -i2, -i3}};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (ns > 2 && v[h][2] == 128) {
      v[h][2] = -128;
      v[h][1] += 1;
    }
    if (v[h][1] >= 128) {
      v[h][1] -= 256;
      v[h][0] += 1;
    }
  }
#pragma unroll
  for (int u = 0; u < 3; ++u) {
    p[u] = v[0][u];
    m[u] = v[1][u];
  }
}
// four consecutive FP32 values: their slices at idx and the slices of their negations at nidx
__device__ __forceinline__ void put4f_pm(const Q& q, int ns, long idx, long nidx, const float (&x)[4], float s) {
  int p[4][3], m[4][3];
#pragma unroll
  for (int u = 0; u < 4; ++u) slice_pm_f(x[u], s, ns, p[u], m[u]);
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    if (t < ns) {
      *reinterpret_cast<char4*>(q.p[t] + idx) = make_char4(char(p[0][t]), char(p[1][t]), char(p[2][t]), char(p[3][t]));
      *reinterpret_cast<char4*>(q.p[t] + nidx) = make_char4(char(m[0][t]), char(m[1][t]), char(m[2][t]), char(m[3][t]));
    }
  }
}

// scalar store of one FP32 value's slices
__device__ __forceinline__ void put1f(const Q& q, int ns, long idx, float x, float s) {
  int a, b, c;
  slice_value_f(x, s, ns, a, b, c);
  q.p[0][idx] = int8_t(a);
  if (ns > 1) q.p[1][idx] = int8_t(b);
  if (ns > 2) q.p[2][idx] = int8_t(c);
}

__device__ __forceinline__ double block_max(double v, double* sh) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double u = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o; o >>= 1) u = fmax(u, __shfl_xor_sync(0xffffffffu, u, o));
    if (threadIdx.x == 0) sh[0] = u;
  }
  __syncthreads();
  return sh[0];
}

// one block per row
__global__ void rows_real_kernel(const double* src, long K, long lds, int ns, Q q, long ld, int* e) {
  __shared__ double sh[32];
  const long r = blockIdx.x;
  const double* x = src + r * lds;
  double m = 0.0;
  for (long k = threadIdx.x; k < K; k += blockDim.x) m = fmax(m, fabs(x[k]));
  m = block_max(m, sh);
  const int ex = row_exponent(m);
  if (threadIdx.x == 0) e[r] = ex;
  const double s = pow2d(-ex);
  for (long k = threadIdx.x; k < ld; k += blockDim.x) put(q, ns, r * ld + k, k < K ? x[k] : 0.0, s);
}

// one block per complex row r: planar rows r (re) and R + r (im)
__global__ void rows_planar_kernel(const cplx* src, long R, long K, int ns, Q q, long ld, int* e, const cplx* sub) {
  __shared__ double sh[32];
  const long r = blockIdx.x;
  const cplx* x = src + r * K;
  double mr = 0.0, mi = 0.0;
  for (long k = threadIdx.x; k < K; k += blockDim.x) {
    const cplx z = sub ? csub(x[k], sub[k]) : x[k];
    mr = fmax(mr, fabs(z.x));
    mi = fmax(mi, fabs(z.y));
  }
  mr = block_max(mr, sh);
  mi = block_max(mi, sh);
  const int er = row_exponent(mr), ei = row_exponent(mi);
  if (threadIdx.x == 0) {
    e[r] = er;
    e[R + r] = ei;
  }
  const double sr = pow2d(-er), si = pow2d(-ei);
  for (long k = threadIdx.x; k < ld; k += blockDim.x) {
    const cplx z = k < K ? (sub ? csub(x[k], sub[k]) : x[k]) : mk(0.0, 0.0);
    put(q, ns, r * ld + k, z.x, sr);
    put(q, ns, (R + r) * ld + k, z.y, si);
  }
}

// long rows split over blocks: pass 1, each chunk's largest |re| and |im| into the row's maxima
// (non-negative doubles order like their bits, so a 64-bit atomic max is exact); pass 2 slices
constexpr long kPlanarChunk = 4096;
__global__ void __launch_bounds__(256) planar_max_kernel(const cplx* src, long R, long K, const cplx* sub,
                                                         unsigned long long* emax) {
  __shared__ double sh[32];
  const long r = blockIdx.y, k0 = blockIdx.x * kPlanarChunk;
  const long k1 = k0 + kPlanarChunk < K ? k0 + kPlanarChunk : K;
  const cplx* x = src + r * K;
  double mr = 0.0, mi = 0.0;
  for (long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    const cplx z = sub ? csub(x[k], sub[k]) : x[k];
    mr = fmax(mr, fabs(z.x));
    mi = fmax(mi, fabs(z.y));
  }
  mr = block_max(mr, sh);
  mi = block_max(mi, sh);
  if (threadIdx.x == 0) {
    atomicMax(emax + r, (unsigned long long)__double_as_longlong(mr));
    atomicMax(emax + R + r, (unsigned long long)__double_as_longlong(mi));
  }
}
__global__ void __launch_bounds__(256) planar_slice_kernel(const cplx* src, long R, long K, const cplx* sub,
                                                           const unsigned long long* emax, int ns, Q q, long ld,
                                                           int* e) {
  const long r = blockIdx.y, k0 = blockIdx.x * kPlanarChunk;
  const long k1 = k0 + kPlanarChunk < ld ? k0 + kPlanarChunk : ld;
  const int er = row_exponent(__longlong_as_double((long long)emax[r]));
  const int ei = row_exponent(__longlong_as_double((long long)emax[R + r]));
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    e[r] = er;
    e[R + r] = ei;
  }
  const double sr = pow2d(-er), si = pow2d(-ei);
  const cplx* x = src + r * K;
  for (long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    const cplx z = k < K ? (sub ? csub(x[k], sub[k]) : x[k]) : mk(0.0, 0.0);
    put(q, ns, r * ld + k, z.x, sr);
    put(q, ns, (R + r) * ld + k, z.y, si);
  }
}

// walkers: the largest |re|, |im| of each (w, a) over the orbitals (threads along a: coalesced)
__global__ void walkers_max_kernel(const cplx* SM, int M, int N, int* e) {
  __shared__ double sh[8][33];
  const int w = blockIdx.y, a = blockIdx.x * 32 + threadIdx.x;
  double m = 0.0;
  if (a < N)
    for (int j = threadIdx.y; j < M; j += blockDim.y) {
      const cplx z = SM[((long)w * M + j) * N + a];
      m = fmax(m, fmax(fabs(z.x), fabs(z.y)));
    }
  sh[threadIdx.y][threadIdx.x] = m;
  __syncthreads();
  if (threadIdx.y == 0 && a < N) {
    for (int y = 1; y < blockDim.y; ++y) m = fmax(m, sh[y][threadIdx.x]);
    e[(long)w * N + a] = row_exponent(m);
  }
}

// walkers -> rows (c, w, a) over j, 32 x 32 tiles through shared memory
__global__ void walkers_slice_kernel(const cplx* SM, int W, int M, int N, int ns, Q q, long ld, const int* e,
                                     float* planar) {
  __shared__ cplx tile[32][33];
  const int w = blockIdx.z, j0 = blockIdx.y * 32, a0 = blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, a = a0 + threadIdx.x;
    tile[r][threadIdx.x] = (j < M && a < N) ? SM[((long)w * M + j) * N + a] : mk(0.0, 0.0);
  }
  __syncthreads();
  const long R = (long)W * N;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int a = a0 + r, j = j0 + threadIdx.x;
    if (a >= N || j >= ld) continue;
    const long row = (long)w * N + a;
    const double s = pow2d(-e[row]);
    const cplx z = tile[threadIdx.x][r];
    put(q, ns, row * ld + j, z.x, s);
    put(q, ns, (R + row) * ld + j, z.y, s);
    if (planar && j < M) {
      planar[row * M + j] = float(z.x);
      planar[(R + row) * M + j] = float(z.y);
    }
  }
}

// Taylor update, one warp per row r of the planar walker-shaped arrays (FP32):
//   k = 0: S += C                    (S = W + (P1 - I) W = P1 W)
//   k > 0: T = (i / k) C (T_re = -C_im / k, T_im = C_re / k), S += T
// then the slices of S (SUM) or of T, one exponent per row over both parts.  Each lane holds QPL
// groups of four consecutive orbitals (lane + 32 t, t < QPL; QPL * 128 >= the slice row stride,
// at most kMaxQuads): every load of the row is issued before the first store, and the values stay
// in registers between the pass that updates S and finds the row's largest entry and the pass
// that slices.
constexpr int kMaxQuads = 8;
template <bool VEC>
__device__ __forceinline__ void ld4(const float* __restrict__ p, float (&v)[4], int valid) {
  if (VEC) {
    const float4 u = *reinterpret_cast<const float4*>(p);
    v[0] = u.x; v[1] = u.y; v[2] = u.z; v[3] = u.w;
  } else {
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = u < valid ? p[u] : 0.f;
  }
}
template <bool VEC>
__device__ __forceinline__ void st4(float* __restrict__ p, const float (&v)[4], int valid) {
  if (VEC) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (u < valid) p[u] = v[u];
  }
}
// 128 threads per block, at most 85 registers up to four groups per lane: 24 rows in flight per SM
// (measured 86 -> 70 us at M = 400, 25600 rows, against 92 registers and 256 threads)
template <bool SUM, bool VEC, int QPL>
__global__ void __launch_bounds__(128, (QPL <= 4 ? 6 : 1)) taylor_update_kernel(const float* __restrict__ C, float* __restrict__ S,
                                                            long R, int M, int k, int ns, Q q, long ld, int* e) {
  const long r = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= R) return;
  const int G4 = (M + 3) >> 2;
  float sr[QPL][4], si[QPL][4], vr[QPL][4], vi[QPL][4];
#pragma unroll
  for (int t = 0; t < QPL; ++t) {
    const int g = lane + 32 * t;
    const int valid = g < G4 ? (M - 4 * g < 4 ? M - 4 * g : 4) : 0;
    if (valid) {
      const long i0 = r * M + 4 * g, i1 = (R + r) * M + 4 * g;
      ld4<VEC>(S + i0, sr[t], valid);
      ld4<VEC>(S + i1, si[t], valid);
      ld4<VEC>(C + i0, vr[t], valid);
      ld4<VEC>(C + i1, vi[t], valid);
    } else {
#pragma unroll
      for (int u = 0; u < 4; ++u) sr[t][u] = si[t][u] = vr[t][u] = vi[t][u] = 0.f;
    }
  }
  float m = 0.f;
  const float fk = float(k);
#pragma unroll
  for (int t = 0; t < QPL; ++t) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      float tr = vr[t][u], ti = vi[t][u];
      if (k != 0) {
        tr = -vi[t][u] / fk;
        ti = vr[t][u] / fk;
      }
      sr[t][u] += tr;
      si[t][u] += ti;
      vr[t][u] = SUM ? sr[t][u] : tr;
      vi[t][u] = SUM ? si[t][u] : ti;
      m = fmaxf(m, fmaxf(fabsf(vr[t][u]), fabsf(vi[t][u])));
    }
  }
#pragma unroll
  for (int t = 0; t < QPL; ++t) {
    const int g = lane + 32 * t;
    const int valid = g < G4 ? (M - 4 * g < 4 ? M - 4 * g : 4) : 0;
    if (valid) {
      st4<VEC>(S + r * M + 4 * g, sr[t], valid);
      st4<VEC>(S + (R + r) * M + 4 * g, si[t], valid);
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int ex = row_exponent(double(m));
  if (lane == 0) e[r] = ex;
  const float sc = pow2f(-ex);
#pragma unroll
  for (int t = 0; t < QPL; ++t) {
    const int g = lane + 32 * t;
    if (4 * g >= ld) break;
    float xr[4], xi[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {  // zeros past M (the padding up to ld)
      const bool in = 4 * g + u < M;
      xr[u] = in ? vr[t][u] : 0.f;
      xi[u] = in ? vi[t][u] : 0.f;
    }
    put4f(q, ns, r * ld + 4 * g, xr, sc);
    put4f(q, ns, (R + r) * ld + 4 * g, xi, sc);
  }
}

template <int QPL>
void launch_taylor_update(const float* C, float* S, long R, int M, int k, bool slice_sum, int ns, const Q& q, long ld,
                          int* e, cudaStream_t st) {
  const int wpb = 4;
  const unsigned grid = unsigned((R + wpb - 1) / wpb);
  // four consecutive orbitals per group: 16-byte rows when M is a multiple of 4
  if (M % 4 == 0) {
    if (slice_sum) taylor_update_kernel<true, true, QPL><<<grid, 32 * wpb, 0, st>>>(C, S, R, M, k, ns, q, ld, e);
    else taylor_update_kernel<false, true, QPL><<<grid, 32 * wpb, 0, st>>>(C, S, R, M, k, ns, q, ld, e);
  } else {
    if (slice_sum) taylor_update_kernel<true, false, QPL><<<grid, 32 * wpb, 0, st>>>(C, S, R, M, k, ns, q, ld, e);
    else taylor_update_kernel<false, false, QPL><<<grid, 32 * wpb, 0, st>>>(C, S, R, M, k, ns, q, ld, e);
  }
}

// 4-byte asynchronous global -> shared copy (L1-allocating); no register holds the value, so a
// thread may have all of its copies in flight at once
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
  const unsigned s = unsigned(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// V slices from the packed vHS, one block per (walker, strip of rs <= 32 rows): both parts' full rows
// V[w][c][i][0..M) in shared memory, from the stored upper triangle (packed row i holds k >= i) and
// its mirror (k < i: packed row k, column i; the strip's columns lie side by side in every earlier
// packed row, so both are read in whole rows); each row's exponent from its maximum over both parts;
// then whole rows of the slices of Vr, Vi and -Vi (zeros past M up to ld), four orbitals per thread.
// The loads are asynchronous copies, every one of a block in flight together; the row stride lds is
// four times an odd number of floats, so the mirrored columns' 32 rows fall in 8 banks, not 2.
__global__ void __launch_bounds__(512) v_strip_kernel(const float* Cv, int W, int M, int rs, int lds, int ns, Q q,
                                                      long ld, int* e) {
  extern __shared__ float vs[];  // [2][rs][lds]
  __shared__ float scale[32];
  const int w = blockIdx.y, i0 = blockIdx.x * rs;
  const int rows = M - i0 < rs ? M - i0 : rs;
  const long P = (long)M * (M + 1) / 2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int c = 0; c < 2; ++c) {
    const float* src = Cv + ((long)c * W + w) * P;
    float* t = vs + c * rs * lds;
    for (int r = warp; r < rows; r += nw) {  // the strip's rows, k >= i
      const int i = i0 + r;
      const float* row = src + (long)i * M - (long)i * (i + 1) / 2;
      for (int k = i + lane; k < M; k += 32) cp_async4(t + r * lds + k, row + k);
    }
    // earlier rows k < i0: their columns i0 .. i0 + rows - 1
    if (lane < rows)
      for (int k = warp; k < i0; k += nw) cp_async4(t + lane * lds + k, src + (long)k * M - (long)k * (k + 1) / 2 + i0 + lane);
  }
  cp_async_wait_all();
  __syncthreads();
  for (int c = 0; c < 2; ++c) {  // the strip's own lower triangle, i0 <= k < i
    float* t = vs + c * rs * lds;
    for (int el = threadIdx.x; el < rows * rows; el += blockDim.x) {
      const int r = el / rows, rk = el - r * rows;
      if (rk < r) t[r * lds + i0 + rk] = t[rk * lds + i0 + r];
    }
  }
  __syncthreads();
  for (int r = warp; r < rows; r += nw) {
    float m = 0.f;
    for (int c = 0; c < 2; ++c)
      for (int k = lane; k < M; k += 32) m = fmaxf(m, fabsf(vs[(c * rs + r) * lds + k]));
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int ex = row_exponent(double(m));
    if (lane == 0) {
      e[(long)w * M + i0 + r] = ex;
      scale[r] = pow2f(-ex);
    }
  }
  __syncthreads();
  const long vb = (long)w * 3 * M * ld;
  for (int r = warp; r < rows; r += nw) {
    const long i = i0 + r;
    const float sc = scale[r];
    const float* tr = vs + r * lds;
    const float* ti = vs + (rs + r) * lds;
    for (int k = 4 * lane; k < ld; k += 128) {
      float xr[4], xi[4];
      if (k + 3 < M) {
        const float4 a = *reinterpret_cast<const float4*>(tr + k), b = *reinterpret_cast<const float4*>(ti + k);
        xr[0] = a.x; xr[1] = a.y; xr[2] = a.z; xr[3] = a.w;
        xi[0] = b.x; xi[1] = b.y; xi[2] = b.z; xi[3] = b.w;
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          xr[u] = k + u < M ? tr[k + u] : 0.f;
          xi[u] = k + u < M ? ti[k + u] : 0.f;
        }
      }
      put4f(q, ns, vb + i * ld + k, xr, sc);
      put4f_pm(q, ns, vb + ((long)M + i) * ld + k, vb + (2L * M + i) * ld + k, xi, sc);
    }
  }
}

__global__ void v_max_full_kernel(const float* Cv, int W, int M, int* emax) {
  const long row = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);  // (c * W + w) * M + i
  const int lane = threadIdx.x & 31;
  if (row >= 2L * W * M) return;
  const float* x = Cv + row * M;
  float m = 0.f;
  for (int k = lane; k < M; k += 32) m = fmaxf(m, fabsf(x[k]));
#pragma unroll
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  const long wc = row / M, i = row % M, w = wc % W;
  if (lane == 0) atomicMax(emax + w * M + i, __float_as_int(m));
}

__global__ void v_exponent_kernel(const int* emax, long n, int* e) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    e[t] = row_exponent(double(__int_as_float(emax[t])));
}

__global__ void v_slice_full_kernel(const float* Cv, int W, int M, int ns, Q q, long ld, const int* e) {
  const long n = 3L * W * M * ld;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const long k = t % ld, r = t / ld;  // r = (w * 3 + c) * M + i; block c = 2 is -Vi
    const long i = r % M, wc3 = r / M, c = wc3 % 3, w = wc3 / 3;
    const float v = k < M ? Cv[((c ? 1 : 0) * W + w) * (long)M * M + i * M + k] : 0.f;
    const float x = c == 2 ? -v : v;
    int a, b, d;
    slice_value_f(x, pow2f(-e[w * M + i]), ns, a, b, d);
    q.p[0][t] = int8_t(a);
    if (ns > 1) q.p[1][t] = int8_t(b);
    if (ns > 2) q.p[2][t] = int8_t(d);
  }
}

// planar FP32 C[c][w][a][j] -> SM[w][j][a] complex, 32 x 32 tiles through shared memory
__global__ void to_walkers_kernel(const float* C, const float* S, int W, int M, int N, cplx* SM) {
  __shared__ double2 tile[32][33];
  const int w = blockIdx.z, a0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  const long R = (long)W * N;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int a = a0 + r, j = j0 + threadIdx.x;
    if (a < N && j < M) {
      const long i = ((long)w * N + a) * M + j;
      double re = double(C[i]), im = double(C[R * M + i]);
      if (S) {
        re += double(S[i]);
        im += double(S[R * M + i]);
      }
      tile[r][threadIdx.x] = make_double2(re, im);
    }
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, a = a0 + threadIdx.x;
    if (a < N && j < M) {
      const double2 z = tile[threadIdx.x][r];
      SM[((long)w * M + j) * N + a] = mk(z.x, z.y);
    }
  }
}

inline int grid_for(long n) {
  long g = (n + 255) / 256;
  if (g > 148L * 32) g = 148L * 32;
  return int(g < 1 ? 1 : g);
}

int check_slices(int ns, int8_t* const* q, long ld) {
  if (ns < 2 || ns > 3) return record_error(SFQ_ERR_ARG, "islice: 2 or 3 slices");
  for (int s = 0; s < ns; ++s)
    if (!q[s]) return record_error(SFQ_ERR_ARG, "islice: slice %d missing", s);
  if (ld % 16) return record_error(SFQ_ERR_SHAPE, "islice: row stride %ld is not a multiple of 16", ld);
  return SFQ_OK;
}

}  // namespace

int islice_rows_real(const double* src, long R, long K, long lds, int nslices, int8_t* const* q, long ld, int* e,
                     cudaStream_t st) {
  if (int rc = check_slices(nslices, q, ld)) return rc;
  if (R <= 0) return SFQ_OK;
  if (ld < K || R > 2147483647L) return record_error(SFQ_ERR_SHAPE, "islice_rows_real: sizes");
  rows_real_kernel<<<unsigned(R), ld <= 512 ? 128 : 256, 0, st>>>(src, K, lds, nslices, qptrs(q), ld, e);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int islice_rows_planar(const cplx* src, long R, long K, int nslices, int8_t* const* q, long ld, int* e,
                       cudaStream_t st, const cplx* sub, unsigned long long* emax) {
  if (int rc = check_slices(nslices, q, ld)) return rc;
  if (R <= 0) return SFQ_OK;
  if (ld < K || R > 2147483647L) return record_error(SFQ_ERR_SHAPE, "islice_rows_planar: sizes");
  if (emax && K > 2 * kPlanarChunk && R <= 65535) {  // long rows: spread each row over blocks
    SFQ_CUDA_TRY(cudaMemsetAsync(emax, 0, sizeof(unsigned long long) * 2 * R, st));
    planar_max_kernel<<<dim3(unsigned((K + kPlanarChunk - 1) / kPlanarChunk), unsigned(R)), 256, 0, st>>>(src, R, K,
                                                                                                           sub, emax);
    SFQ_LAUNCHED();
    planar_slice_kernel<<<dim3(unsigned((ld + kPlanarChunk - 1) / kPlanarChunk), unsigned(R)), 256, 0, st>>>(
        src, R, K, sub, emax, nslices, qptrs(q), ld, e);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }
  rows_planar_kernel<<<unsigned(R), K >= 4096 ? 512 : 256, 0, st>>>(src, R, K, nslices, qptrs(q), ld, e, sub);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int islice_walkers(const cplx* SM, int W, int M, int N, int nslices, int8_t* const* q, long ld, int* e,
                   float* planar, cudaStream_t st) {
  if (int rc = check_slices(nslices, q, ld)) return rc;
  if (ld < M || W > 65535) return record_error(SFQ_ERR_SHAPE, "islice_walkers: sizes");
  walkers_max_kernel<<<dim3(unsigned((N + 31) / 32), unsigned(W)), dim3(32, 8), 0, st>>>(SM, M, N, e);
  SFQ_LAUNCHED();
  walkers_slice_kernel<<<dim3(unsigned((N + 31) / 32), unsigned((ld + 31) / 32), unsigned(W)), dim3(32, 8), 0, st>>>(
      SM, W, M, N, nslices, qptrs(q), ld, e, planar);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int islice_taylor_update(const float* C, float* S, long R, int M, int k, bool slice_sum, int nslices,
                         int8_t* const* q, long ld, int* e, cudaStream_t st) {
  if (int rc = check_slices(nslices, q, ld)) return rc;
  if (ld < M || ld > 128L * kMaxQuads) return record_error(SFQ_ERR_SHAPE, "islice_taylor_update: M=%d", M);
  if (!C || !S) return record_error(SFQ_ERR_ARG, "islice_taylor_update: product or sum missing");
  if (k == 0 && !slice_sum) return record_error(SFQ_ERR_ARG, "islice_taylor_update: k = 0 slices the sum");
  if (R <= 0) return SFQ_OK;
  const Q qq = qptrs(q);
  switch ((ld + 127) / 128) {  // quads per lane covering the slice row
    case 1: launch_taylor_update<1>(C, S, R, M, k, slice_sum, nslices, qq, ld, e, st); break;
    case 2: launch_taylor_update<2>(C, S, R, M, k, slice_sum, nslices, qq, ld, e, st); break;
    case 3: launch_taylor_update<3>(C, S, R, M, k, slice_sum, nslices, qq, ld, e, st); break;
    case 4: launch_taylor_update<4>(C, S, R, M, k, slice_sum, nslices, qq, ld, e, st); break;
    case 5: launch_taylor_update<5>(C, S, R, M, k, slice_sum, nslices, qq, ld, e, st); break;
    case 6: launch_taylor_update<6>(C, S, R, M, k, slice_sum, nslices, qq, ld, e, st); break;
    case 7: launch_taylor_update<7>(C, S, R, M, k, slice_sum, nslices, qq, ld, e, st); break;
    default: launch_taylor_update<8>(C, S, R, M, k, slice_sum, nslices, qq, ld, e, st); break;
  }
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int islice_build_v(const float* Cv, int W, int M, bool packed, int nslices, int8_t* const* q, long ld, int* e,
                   int* emax, cudaStream_t st) {
  if (int rc = check_slices(nslices, q, ld)) return rc;
  if (ld < M || 2L * W > 65535) return record_error(SFQ_ERR_SHAPE, "islice_build_v: sizes");
  if (packed) {
    // strips of up to 32 rows whose two parts fit 200 KB of shared memory; rows padded to four times
    // an odd number of floats (16-byte row starts for the slicing pass's vector reads, and the
    // mirrored columns' stores spread over 8 banks)
    const int l4 = (M + 3) / 4;
    const int lds = 4 * (l4 | 1);
    int rs = int((200L * 1024) / (2L * lds * sizeof(float)));
    if (rs > 32) rs = 32;
    if (rs < 1) return record_error(SFQ_ERR_SHAPE, "islice_build_v: nmo %d too large for a strip", M);
    const size_t smem = 2 * sizeof(float) * (size_t)rs * lds;
    SFQ_CUDA_TRY(cudaFuncSetAttribute(v_strip_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    v_strip_kernel<<<dim3(unsigned((M + rs - 1) / rs), unsigned(W)), 512, smem, st>>>(Cv, W, M, rs, lds, nslices,
                                                                                       qptrs(q), ld, e);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }
  SFQ_CUDA_TRY(cudaMemsetAsync(emax, 0, sizeof(int) * (size_t)W * M, st));
  v_max_full_kernel<<<unsigned((2L * W * M + 7) / 8), 256, 0, st>>>(Cv, W, M, emax);
  SFQ_LAUNCHED();
  v_exponent_kernel<<<grid_for((long)W * M), 256, 0, st>>>(emax, (long)W * M, e);
  SFQ_LAUNCHED();
  v_slice_full_kernel<<<grid_for(3L * W * M * ld), 256, 0, st>>>(Cv, W, M, nslices, qptrs(q), ld, e);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int islice_to_walkers(const float* C, const float* S, int W, int M, int N, cplx* SM, cudaStream_t st) {
  if (W > 65535) return record_error(SFQ_ERR_SHAPE, "islice_to_walkers: too many walkers");
  to_walkers_kernel<<<dim3(unsigned((M + 31) / 32), unsigned((N + 31) / 32), unsigned(W)), dim3(32, 8), 0, st>>>(
      C, S, W, M, N, SM);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

}  // namespace sfq
