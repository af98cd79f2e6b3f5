// Layout conversions of the mixed-precision propagation step.
//
// Working layouts (per walker w, orbitals i,k < M, electrons a < N, c = 0 real / 1 imaginary):
//   planar rows      P[c*W + w][e]               (split operands of the vbias / vHS GEMMs)
//   walker rows      WT[w][a][c*ldh + i]         (K = (c,i), each half padded to ldh, a multiple
//                                                 of 64, with zeros: Taylor / P1 A operand)
//   vHS planes       V[w][c][i][k] = Vr / Vi     (Taylor B operand; the tensor-core product forms
//                                                 [[Vr, -Vi], [Vi, Vr]] from them, negating Vi)
// so that the complex products become real K-major GEMMs on the tensor cores:
//   (V T)^T[a][(c,i)] = sum_(c',k) WT[a][(c',k)] [[Vr, -Vi], [Vi, Vr]][(c,i)][(c',k)],
//   (P1 W)^T[(a,c)][j] = sum_i WT[(a,c)][i] P1[j][i].
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.cuh"
#include "mixed.cuh"

namespace sfq {
namespace {

// operand planes: p0 = bf16(x), p1 = bf16(x - p0), p2 = bf16(x - p0 - p1) (null planes skipped)
struct Planes {
  __nv_bfloat16 *p0, *p1, *p2;
};

__device__ __forceinline__ void split_store(float x, const Planes& P, long idx) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(x);
  P.p0[idx] = h0;
  if (P.p1) {
    const float r1 = x - __bfloat162float(h0);
    const __nv_bfloat16 h1 = __float2bfloat16_rn(r1);
    P.p1[idx] = h1;
    if (P.p2) P.p2[idx] = __float2bfloat16_rn(r1 - __bfloat162float(h1));
  }
}
__device__ __forceinline__ void split_store_d(double x, const Planes& P, long idx) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(float(x));
  P.p0[idx] = h0;
  if (P.p1) {
    const double r1 = x - double(__bfloat162float(h0));
    const __nv_bfloat16 h1 = __float2bfloat16_rn(float(r1));
    P.p1[idx] = h1;
    if (P.p2) P.p2[idx] = __float2bfloat16_rn(float(r1 - double(__bfloat162float(h1))));
  }
}

Planes planes(void* const* pl) {
  Planes P;
  P.p0 = (__nv_bfloat16*)pl[0];
  P.p1 = (__nv_bfloat16*)pl[1];
  P.p2 = (__nv_bfloat16*)pl[2];
  return P;
}

inline int grid_for(long n) {
  long g = (n + 255) / 256;
  if (g > 148L * 32) g = 148L * 32;
  return int(g < 1 ? 1 : g);
}

// complex (W, E) -> planar split rows c*W + w
__global__ void split_planar_kernel(const cplx* src, int W, long E, Planes P) {
  const long total = (long)W * E;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long w = t / E, e = t % E;
    const cplx z = src[t];
    split_store_d(z.x, P, w * E + e);
    split_store_d(z.y, P, ((long)W + w) * E + e);
  }
}

// KS partial sums of planar fp32 rows (c*W + w), split s at C + s * sk -> complex fp64 (W, E),
// times alpha; the splits are added in order, in double precision
__global__ void reduce_planar_to_cplx_kernel(const float* C, int KS, long sk, int W, long E, double alpha,
                                             cplx* out, const cplx* add) {
  const long total = (long)W * E;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long w = t / E, e = t % E;
    const float* cr = C + w * E + e;
    const float* ci = C + ((long)W + w) * E + e;
    double re = 0.0, im = 0.0;
    int s = 0;
    for (; s + 4 <= KS; s += 4) {  // four splits' loads in flight, added in the same order
      float r[4], q[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        r[u] = cr[(s + u) * sk];
        q[u] = ci[(s + u) * sk];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        re += double(r[u]);
        im += double(q[u]);
      }
    }
    for (; s < KS; ++s) {
      re += double(cr[s * sk]);
      im += double(ci[s * sk]);
    }
    out[t] = add ? mk(add[e].x + alpha * re, add[e].y + alpha * im) : mk(alpha * re, alpha * im);
  }
}

// planar vHS (rows c*W + w, columns i*M + k, or the packed upper triangle when packed) ->
// V[w][c][i][k] split.  Each thread converts 4 consecutive elements of a row and stores each
// plane's 4 BF16 values as one 8-byte word (M is a multiple of 8, so a group never straddles the
// row end and is 8-byte aligned).
__device__ __forceinline__ void split_store4(const float (&x)[4], const Planes& P, long idx) {
  union U {
    __nv_bfloat162 h[2];
    uint2 u;
  };
  U q0;
  q0.h[0] = __floats2bfloat162_rn(x[0], x[1]);
  q0.h[1] = __floats2bfloat162_rn(x[2], x[3]);
  *reinterpret_cast<uint2*>(P.p0 + idx) = q0.u;
  if (!P.p1) return;
  float r[4];
  r[0] = x[0] - __low2float(q0.h[0]);
  r[1] = x[1] - __high2float(q0.h[0]);
  r[2] = x[2] - __low2float(q0.h[1]);
  r[3] = x[3] - __high2float(q0.h[1]);
  U q1;
  q1.h[0] = __floats2bfloat162_rn(r[0], r[1]);
  q1.h[1] = __floats2bfloat162_rn(r[2], r[3]);
  *reinterpret_cast<uint2*>(P.p1 + idx) = q1.u;
  if (!P.p2) return;
  U q2;
  q2.h[0] = __floats2bfloat162_rn(r[0] - __low2float(q1.h[0]), r[1] - __high2float(q1.h[0]));
  q2.h[1] = __floats2bfloat162_rn(r[2] - __low2float(q1.h[1]), r[3] - __high2float(q1.h[1]));
  *reinterpret_cast<uint2*>(P.p2 + idx) = q2.u;
}

// full M x M rows: float4 loads, 8-byte plane stores
__global__ void build_v_full_kernel(const float* Cv, int W, int M, Planes P) {
  const long MM = (long)M * M;
  const long groups = 2L * W * MM / 4;
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < groups; g += (long)gridDim.x * blockDim.x) {
    const long e = 4 * g;                 // element of the planar rows (c * W + w, i * M + k)
    const long wc = e / MM, ik = e - wc * MM;
    const long c = wc / W, w = wc - c * W;
    const float4 v = *reinterpret_cast<const float4*>(Cv + e);
    const float x[4] = {v.x, v.y, v.z, v.w};
    split_store4(x, P, (w * 2 + c) * MM + ik);
  }
}

// packed upper triangle: one block per 64 x 64 tile pair (ib <= kb) of one planar row; the tile is
// read once along the packed rows and written as V[i][k] and, off the diagonal, as its mirror
// V[k][i]
constexpr int kVT = 64;
__global__ void __launch_bounds__(256) build_v_packed_kernel(const float* Cv, int W, int M, int T, Planes P) {
  __shared__ float tile[kVT][kVT + 1];
  __shared__ long rowbase[kVT];
  const int wc = blockIdx.y;  // c * W + w
  const int c = wc / W, w = wc - c * W;
  int t = blockIdx.x, ib = 0;  // tile pair from the linear index: row ib holds kb = ib .. T-1
  while (ib < T && t >= T - ib) {
    t -= T - ib;
    ++ib;
  }
  const int kb = ib + t;
  const int i0 = ib * kVT, k0 = kb * kVT;
  const long MM = (long)M * M;
  const float* src = Cv + (long)wc * ((long)M * (M + 1) / 2);
  const long vbase = ((long)w * 2 + c) * MM;
  const int tid = threadIdx.x;
  if (tid < kVT) {
    const long i = i0 + tid;
    rowbase[tid] = i * M - i * (i + 1) / 2;  // packed index of (i, k) = rowbase + k, k >= i
  }
  __syncthreads();
  {
    // thread: column q of rows r0 + 4 s; all 16 loads issued before the first shared store
    const int q = tid % kVT, r0 = tid / kVT;
    float v[kVT / 4];
#pragma unroll
    for (int s = 0; s < kVT / 4; ++s) {
      const int r = r0 + 4 * s, i = i0 + r, k = k0 + q;
      v[s] = (i < M && k < M && i <= k) ? src[rowbase[r] + k] : 0.f;
    }
#pragma unroll
    for (int s = 0; s < kVT / 4; ++s) tile[r0 + 4 * s][q] = v[s];
  }
  __syncthreads();
  for (int e = tid; e < kVT * kVT / 4; e += 256) {
    const int r = e / (kVT / 4), g = 4 * (e % (kVT / 4));
    const int i = i0 + r, k = k0 + g;
    if (i >= M || k >= M) continue;
    float x[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) x[j] = (i <= k + j) ? tile[r][g + j] : tile[g + j][r];  // the diagonal tile's lower half mirrored
    split_store4(x, P, vbase + (long)i * M + k);
  }
  if (ib == kb) return;
  for (int e = tid; e < kVT * kVT / 4; e += 256) {
    const int r = e / (kVT / 4), g = 4 * (e % (kVT / 4));
    const int k = k0 + r, i = i0 + g;
    if (k >= M || i >= M) continue;
    float x[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) x[j] = tile[g + j][r];
    split_store4(x, P, vbase + (long)k * M + i);
  }
}

// split_store_d for 4 consecutive elements (residuals in double), each plane's 4 values as one
// 8-byte word (idx a multiple of 4)
__device__ __forceinline__ void split_store4_d(const double (&x)[4], const Planes& P, long idx) {
  union U {
    __nv_bfloat162 h[2];
    uint2 u;
  };
  U q0;
  q0.h[0] = __floats2bfloat162_rn(float(x[0]), float(x[1]));
  q0.h[1] = __floats2bfloat162_rn(float(x[2]), float(x[3]));
  *reinterpret_cast<uint2*>(P.p0 + idx) = q0.u;
  if (!P.p1) return;
  double r[4];
  r[0] = x[0] - double(__low2float(q0.h[0]));
  r[1] = x[1] - double(__high2float(q0.h[0]));
  r[2] = x[2] - double(__low2float(q0.h[1]));
  r[3] = x[3] - double(__high2float(q0.h[1]));
  U q1;
  q1.h[0] = __floats2bfloat162_rn(float(r[0]), float(r[1]));
  q1.h[1] = __floats2bfloat162_rn(float(r[2]), float(r[3]));
  *reinterpret_cast<uint2*>(P.p1 + idx) = q1.u;
  if (!P.p2) return;
  U q2;
  q2.h[0] = __floats2bfloat162_rn(float(r[0] - double(__low2float(q1.h[0]))), float(r[1] - double(__high2float(q1.h[0]))));
  q2.h[1] = __floats2bfloat162_rn(float(r[2] - double(__low2float(q1.h[1]))), float(r[3] - double(__high2float(q1.h[1]))));
  *reinterpret_cast<uint2*>(P.p2 + idx) = q2.u;
}

// inverse overlaps Tinv (W, N, N) complex -> the real block operand of G = (W Tinv)^T, rows
// (c, a), columns (b, c'): [[Tr, -Ti], [Ti, Tr]] at (Tinv[b][a]), split.  A 32 x 32 tile of Tinv
// goes through shared memory (read along a, written along b); each thread writes 4 consecutive
// columns (two b, both c') of one row as one 8-byte word per plane.  N is a multiple of 4.
__global__ void build_tblk_kernel(const cplx* Tinv, int W, int N, Planes P) {
  __shared__ cplx tile[32][33];
  const int w = blockIdx.z, b0 = blockIdx.y * 32, a0 = blockIdx.x * 32;
  const cplx* Tw = Tinv + (long)w * N * N;
  for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
    const int bb = e / 32, aa = e % 32;
    const int b = b0 + bb, a = a0 + aa;
    if (b < N && a < N) tile[bb][aa] = Tw[(long)b * N + a];
  }
  __syncthreads();
  const long N2 = 2L * N;
  for (int e = threadIdx.x; e < 2 * 32 * 16; e += blockDim.x) {
    const int c = e / (32 * 16), rem = e % (32 * 16);
    const int aa = rem / 16, bb = 2 * (rem % 16);
    const int a = a0 + aa, b = b0 + bb;
    if (a >= N || b >= N) continue;  // b even and N a multiple of 4: b + 1 < N too
    const cplx z0 = tile[bb][aa], z1 = tile[bb + 1][aa];
    double x[4];
    if (c == 0) {
      x[0] = z0.x; x[1] = -z0.y; x[2] = z1.x; x[3] = -z1.y;
    } else {
      x[0] = z0.y; x[1] = z0.x; x[2] = z1.y; x[3] = z1.x;
    }
    split_store4_d(x, P, ((long)w * N2 + (long)c * N + a) * N2 + 2L * b);
  }
}

// SM (W, M, N) complex fp64 -> WT[w][a][c][i] split, 32x32 tiles through shared memory
__global__ void walkers_to_wt_kernel(const cplx* SM, int M, int N, int ldh, Planes P) {
  __shared__ cplx tile[32][33];
  const int w = blockIdx.z;
  const int i0 = blockIdx.y * 32, a0 = blockIdx.x * 32;
  const cplx* S = SM + (long)w * M * N;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, a = a0 + threadIdx.x;
    if (i < M && a < N) tile[r][threadIdx.x] = S[(long)i * N + a];
  }
  __syncthreads();
  const long base = (long)w * N * 2 * ldh;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int a = a0 + r, i = i0 + threadIdx.x;
    if (i < M && a < N) {
      const cplx z = tile[threadIdx.x][r];
      split_store_d(z.x, P, base + ((long)a * 2 + 0) * ldh + i);
      split_store_d(z.y, P, base + ((long)a * 2 + 1) * ldh + i);
    }
  }
}

// the two operand layouts of the walkers in one pass over SM: the planes of SM read as reals (the G
// product's B operand, same layout) and WT[w][a][c * ldh + i] (the P1 product's A operand).  A
// 32 x 32 tile of SM goes through shared memory; every thread writes 4 consecutive values per plane
// as one 8-byte word (N is a multiple of 4, M of 8).
__global__ void walkers_split_both_kernel(const cplx* SM, int M, int N, int ldh, Planes PS, Planes PT) {
  __shared__ cplx tile[32][33];
  const int w = blockIdx.z;
  const int i0 = blockIdx.y * 32, a0 = blockIdx.x * 32;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const cplx* S = SM + (long)w * M * N;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, a = a0 + threadIdx.x;
    if (i < M && a < N) tile[r][threadIdx.x] = S[(long)i * N + a];
  }
  __syncthreads();
  // SM as reals: row i, electrons a, a + 1 -> 4 consecutive doubles
  for (int e = tid; e < 32 * 16; e += 256) {
    const int r = e / 16, aa = 2 * (e % 16);
    const int i = i0 + r, a = a0 + aa;
    if (i >= M || a >= N) continue;  // a even and N a multiple of 4: a + 1 < N too
    const cplx z0 = tile[r][aa], z1 = tile[r][aa + 1];
    const double x[4] = {z0.x, z0.y, z1.x, z1.y};
    split_store4_d(x, PS, 2 * (((long)w * M + i) * N + a));
  }
  // walker rows: electron a, part c, orbitals i .. i + 3
  const long base = (long)w * N * 2 * ldh;
  for (int e = tid; e < 32 * 2 * 8; e += 256) {
    const int aa = e / 16, c = (e / 8) % 2, ii = 4 * (e % 8);
    const int a = a0 + aa, i = i0 + ii;
    if (a >= N || i >= M) continue;  // i a multiple of 4 and M of 8: i + 3 < M too
    double x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) x[u] = c ? tile[ii + u][aa].y : tile[ii + u][aa].x;
    split_store4_d(x, PT, base + ((long)a * 2 + c) * ldh + i);
  }
}

}  // namespace

int mixed_walkers_split_both(const cplx* SM, int W, int M, int N, int ldh, void* const* ps, void* const* pt,
                             cudaStream_t st) {
  if (W > 65535) return record_error(SFQ_ERR_SHAPE, "walker split: too many walkers for one launch");
  dim3 grid((N + 31) / 32, (M + 31) / 32, W), block(32, 8);
  walkers_split_both_kernel<<<grid, block, 0, st>>>(SM, M, N, ldh, planes(ps), planes(pt));
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int mixed_split_planar(const cplx* src, int W, long E, void* const* pl, cudaStream_t st) {
  split_planar_kernel<<<grid_for((long)W * E), 256, 0, st>>>(src, W, E, planes(pl));
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int mixed_reduce_planar_to_cplx(const float* C, int KS, long sk, int W, long E, double alpha, cplx* out,
                                cudaStream_t st, const cplx* add) {
  reduce_planar_to_cplx_kernel<<<grid_for((long)W * E), 256, 0, st>>>(C, KS, sk, W, E, alpha, out, add);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int mixed_build_v(const float* Cv, int W, int M, bool packed, void* const* pl, cudaStream_t st) {
  if (M % 8) return record_error(SFQ_ERR_SHAPE, "build_v: M=%d is not a multiple of 8", M);
  if (!packed) {
    build_v_full_kernel<<<grid_for(2L * W * M * M / 4), 256, 0, st>>>(Cv, W, M, planes(pl));
    SFQ_LAUNCHED();
    return SFQ_OK;
  }
  if (2L * W > 65535) return record_error(SFQ_ERR_SHAPE, "build_v: too many walkers for one launch");
  const int T = (M + kVT - 1) / kVT;
  dim3 grid(unsigned(T * (T + 1) / 2), unsigned(2 * W));
  build_v_packed_kernel<<<grid, 256, 0, st>>>(Cv, W, M, T, planes(pl));
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int mixed_build_tblk(const cplx* Tinv, int W, int N, void* const* pl, cudaStream_t st) {
  if (N % 4) return record_error(SFQ_ERR_SHAPE, "build_tblk: N=%d is not a multiple of 4", N);
  if (W > 65535) return record_error(SFQ_ERR_SHAPE, "build_tblk: too many walkers for one launch");
  dim3 grid(unsigned((N + 31) / 32), unsigned((N + 31) / 32), unsigned(W));
  build_tblk_kernel<<<grid, 256, 0, st>>>(Tinv, W, N, planes(pl));
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int mixed_walkers_to_wt(const cplx* SM, int W, int M, int N, int ldh, void* const* pl, cudaStream_t st) {
  dim3 grid((N + 31) / 32, (M + 31) / 32, W), block(32, 8);
  walkers_to_wt_kernel<<<grid, block, 0, st>>>(SM, M, N, ldh, planes(pl));
  SFQ_LAUNCHED();
  return SFQ_OK;
}

}  // namespace sfq
