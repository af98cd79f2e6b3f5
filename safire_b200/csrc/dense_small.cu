// Per-walker small dense factorizations, one CTA per N x N matrix held in shared memory.
//
//  * lu_logdet_kernel: partial-pivot LU (pivot = first max of |re|+|im|, LAPACK izamax
//    semantics), log det = sum_i log(+-U_ii + tiny) folded to [-pi, pi]
//    (src/numerics/operations/determinants_impl.hpp:33-75), and optionally the inverse computed
//    the way zgetri does it (inv(U), then inv(A) L = inv(U), then column swaps), zeroed when
//    any U_ii == 0 (getri_or_zero, src/numerics/nda_functions.hpp:422-438).
//  * chol_rinv_kernel: S = R^H R (Cholesky, real positive diagonal) and R^-1, the small step
//    of CholeskyQR2; Q = W R^-1 has the positive-real-diagonal R that the reference produces
//    with geqrf + sign(Re R_ii) column scaling (orthogonalize.hpp:135-169).
#include "common.cuh"
#include "kernels.cuh"

namespace sfq {

namespace {

constexpr int LU_THREADS = 256;

__device__ __forceinline__ double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }

template <bool INVERT>
__global__ void __launch_bounds__(LU_THREADS) lu_logdet_kernel(cplx* T, long sT, int N, cplx* ovlp, int accumulate,
                                                               double post_scale) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  cplx* A = reinterpret_cast<cplx*>(sm_raw);
  cplx* work = A + N * N;
  int* piv = reinterpret_cast<int*>(work + N);
  __shared__ int s_p;
  __shared__ int s_info;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tx = lane, ty = warp, NY = LU_THREADS / 32;
  const long b = blockIdx.x;
  cplx* Tb = T + b * sT;

  for (int e = tid; e < N * N; e += LU_THREADS) A[e] = Tb[e];
  if (tid == 0) s_info = 0;
  __syncthreads();

  for (int j = 0; j < N; ++j) {
    if (warp == 0) {
      double best = -1.0;
      int bi = j;
      for (int i = j + lane; i < N; i += 32) {
        double v = cabs1(A[i * N + j]);
        if (v > best) { best = v; bi = i; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double ob = __shfl_down_sync(0xffffffffu, best, off);
        int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) {
        piv[j] = bi;
        s_p = bi;
        cplx d = A[bi * N + j];
        if (d.x == 0.0 && d.y == 0.0 && s_info == 0) s_info = j + 1;
      }
    }
    __syncthreads();
    const int p = s_p;
    if (p != j) {
      for (int k = tid; k < N; k += LU_THREADS) {
        cplx t = A[j * N + k];
        A[j * N + k] = A[p * N + k];
        A[p * N + k] = t;
      }
      __syncthreads();
    }
    const cplx d = A[j * N + j];
    if (d.x != 0.0 || d.y != 0.0) {
      const cplx r = cdiv(mk(1.0, 0.0), d);
      for (int i = j + 1 + tid; i < N; i += LU_THREADS) A[i * N + j] = cmul(A[i * N + j], r);
    }
    __syncthreads();
    for (int i = j + 1 + ty; i < N; i += NY) {
      const cplx l = A[i * N + j];
      for (int k = j + 1 + tx; k < N; k += 32) A[i * N + k] = csub(A[i * N + k], cmul(l, A[j * N + k]));
    }
    __syncthreads();
  }

  if (tid == 0) {
    cplx res = accumulate ? ovlp[b] : mk(0.0, 0.0);
    const double tiny = 2.2250738585072014e-308;
    for (int i = 0; i < N; ++i) {
      cplx dgl = A[i * N + i];
      cplx v = (piv[i] == i) ? dgl : mk(-dgl.x, -dgl.y);
      v.x += tiny;
      res = cadd(res, clog_(v));
    }
    const double pi = 3.141592653589793238462643383279502884;
    // bring the imaginary part to [-pi, pi]; |Im| <= N*pi, so the loops are bounded by N
    if (res.y > pi) {
      for (int it = 0; res.y > pi && it < 4 * N + 8; ++it) res.y -= 2 * pi;
    } else if (res.y < -pi) {
      for (int it = 0; res.y < -pi && it < 4 * N + 8; ++it) res.y += 2 * pi;
    }
    ovlp[b] = mk(res.x * post_scale, res.y * post_scale);
  }
  if (!INVERT) return;

  // singular (some U_ii == 0): getri reports info > 0 and the inverse is zeroed
  bool singular = false;
  for (int i = 0; i < N; ++i) {
    cplx dgl = A[i * N + i];
    if (dgl.x == 0.0 && dgl.y == 0.0) { singular = true; break; }
  }
  if (singular) {
    for (int e = tid; e < N * N; e += LU_THREADS) Tb[e] = mk(0.0, 0.0);
    return;
  }
  // inv(U) in place (ztrti2, upper, non-unit)
  for (int j = 0; j < N; ++j) {
    for (int i = tid; i < j; i += LU_THREADS) work[i] = A[i * N + j];
    __syncthreads();
    const cplx ujj = cdiv(mk(1.0, 0.0), A[j * N + j]);
    const cplx ajj = mk(-ujj.x, -ujj.y);
    for (int i = tid; i < j; i += LU_THREADS) {
      cplx s = mk(0.0, 0.0);
      for (int k = i; k < j; ++k) s = cadd(s, cmul(A[i * N + k], work[k]));
      A[i * N + j] = cmul(ajj, s);
    }
    __syncthreads();
    if (tid == 0) A[j * N + j] = ujj;
    __syncthreads();
  }
  // solve inv(A) * L = inv(U) (zgetri, unblocked)
  for (int j = N - 1; j >= 0; --j) {
    for (int i = j + 1 + tid; i < N; i += LU_THREADS) {
      work[i] = A[i * N + j];
      A[i * N + j] = mk(0.0, 0.0);
    }
    __syncthreads();
    if (j < N - 1) {
      for (int i = tid; i < N; i += LU_THREADS) {
        cplx s = mk(0.0, 0.0);
        for (int k = j + 1; k < N; ++k) s = cadd(s, cmul(A[i * N + k], work[k]));
        A[i * N + j] = csub(A[i * N + j], s);
      }
    }
    __syncthreads();
  }
  // column interchanges in reverse order
  for (int j = N - 2; j >= 0; --j) {
    const int jp = piv[j];
    if (jp != j) {
      for (int i = tid; i < N; i += LU_THREADS) {
        cplx t = A[i * N + j];
        A[i * N + j] = A[i * N + jp];
        A[i * N + jp] = t;
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < N * N; e += LU_THREADS) Tb[e] = A[e];
}

// Cholesky of the Hermitian positive definite S (N x N, upper storage used) into R (upper,
// S = R^H R), then R^-1 (upper) written over S.  status[b] = 0, or j+1 when the pivot j is not
// positive (the walker matrix lost rank).  again[b] = 1 when an upper bound of the condition
// number of R, sqrt(|R|_1 |R|_inf |R^-1|_1 |R^-1|_inf) with |z| <= |re| + |im|, exceeds
// kappa_max (one CholeskyQR pass leaves Q^H Q - I of order eps kappa^2: such walkers take a
// second pass).  Walkers with active[b] == 0 are skipped (active may be null).
// max over the block of v (all threads call it; red holds >= 32 doubles)
__device__ __forceinline__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double r = 0.0;
  for (int w = 0; w < int(blockDim.x >> 5); ++w) r = fmax(r, red[w]);
  return r;
}

// |A|_1 * |A|_inf of the upper triangle of A (N x N row-major), |z| as |re| + |im|
// position of (i, k), i <= k, in the packed upper triangle (rows of N - i entries)
__device__ __forceinline__ int pku(int i, int k, int N) { return i * N - ((i * (i - 1)) >> 1) + (k - i); }

// ||R||_1 * ||R||_inf of the packed upper-triangular R
__device__ double norm1_inf_upper(const cplx* A, int N, double* red) {
  double rmax = 0.0, cmax = 0.0;
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    double rs = 0.0, cs = 0.0;
    for (int k = t; k < N; ++k) rs += fabs(A[pku(t, k, N)].x) + fabs(A[pku(t, k, N)].y);
    for (int i = 0; i <= t; ++i) cs += fabs(A[pku(i, t, N)].x) + fabs(A[pku(i, t, N)].y);
    rmax = fmax(rmax, rs);
    cmax = fmax(cmax, cs);
  }
  const double r = block_max(rmax, red);
  const double c = block_max(cmax, red);
  return r * c;
}

// S = R^H R (right-looking upper Cholesky) and R^-1 for one Hermitian S per CTA, both on the packed
// upper triangle in shared memory (N(N+1)/2 entries: two CTAs share an SM at N = 100, where the
// barrier-bound sweeps of one CTA leave it mostly idle)
__global__ void __launch_bounds__(LU_THREADS) chol_rinv_kernel(cplx* S, long sS, int N, int* status, int* again,
                                                               const int* active, double kappa_max, cplx* Rout) {
  const long b = blockIdx.x;
  if (active && !active[b]) return;  // the whole CTA
  extern __shared__ __align__(16) unsigned char sm_raw[];
  cplx* A = reinterpret_cast<cplx*>(sm_raw);
  cplx* work = A + N * (N + 1) / 2;
  __shared__ double diag[kMaxSmallN];
  __shared__ double red[32];
  __shared__ int s_bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = LU_THREADS / 32;
  cplx* Sb = S + b * sS;
  for (int e = tid; e < N * N; e += LU_THREADS) {
    const int i = e / N, k = e % N;
    if (i <= k) A[pku(i, k, N)] = Sb[e];
  }
  if (tid == 0) s_bad = 0;
  __syncthreads();
  // right-looking upper Cholesky: for j: r_jj = sqrt(a_jj); row j /= r_jj; trailing -= r_j^H r_j
  for (int j = 0; j < N; ++j) {
    const double ajj = A[pku(j, j, N)].x;
    if (!(ajj > 0.0)) {
      if (tid == 0 && s_bad == 0) s_bad = j + 1;
      break;
    }
    const double rjj = sqrt(ajj);
    const double inv = 1.0 / rjj;
    __syncthreads();
    const int rj = pku(j, j, N);  // row j, column k at rj + (k - j)
    for (int k = j + tid; k < N; k += LU_THREADS) {
      A[rj + (k - j)] = (k == j) ? mk(rjj, 0.0) : cscale(A[rj + (k - j)], inv);
    }
    __syncthreads();
    // A[i][k] -= conj(R[j][i]) * R[j][k] for j < i <= k
    for (int i = j + 1 + warp; i < N; i += NW) {
      const cplx ci = cconj(A[rj + (i - j)]);
      const int ri = pku(i, i, N);
      for (int k = i + lane; k < N; k += 32) A[ri + (k - i)] = csub(A[ri + (k - i)], cmul(ci, A[rj + (k - j)]));
    }
    __syncthreads();
  }
  __syncthreads();
  if (s_bad) {
    if (tid == 0) {
      status[b] = s_bad;
      if (again) again[b] = 0;
    }
    return;
  }
  const double nR = norm1_inf_upper(A, N, red);
  if (Rout) {
    cplx* Rb = Rout + b * sS;
    for (int e = tid; e < N * N; e += LU_THREADS) {
      const int i = e / N, k = e % N;
      Rb[e] = (i > k) ? mk(0.0, 0.0) : A[pku(i, k, N)];
    }
    __syncthreads();  // every r_ii read before the diagonal below is replaced
  }
  // R^-1 by back substitution on all columns at once, right-looking and in place: going up
  // the rows, row k of R^-1 is the pending row k over r_kk, and its product with column k of R
  // leaves the rows above at once (one rank-1 update per row, parallel over the block).  The
  // diagonal of R moves to diag[] and the in-place diagonal becomes the identity's.
  for (int i = tid; i < N; i += LU_THREADS) {
    diag[i] = A[pku(i, i, N)].x;
    A[pku(i, i, N)] = mk(1.0, 0.0);
  }
  __syncthreads();
  for (int k = N - 1; k >= 0; --k) {
    const double xkk = 1.0 / diag[k];
    for (int i = tid; i < k; i += LU_THREADS) work[i] = A[pku(i, k, N)];  // column k of R, read once
    const int rk = pku(k, k, N);
    for (int jj = k + tid; jj < N; jj += LU_THREADS) A[rk + (jj - k)] = cscale(A[rk + (jj - k)], xkk);  // row k of R^-1
    __syncthreads();
    // pending rows above: P[i][j] -= R[i][k] X[k][j], where P[i][k] starts at 0 (the identity)
    for (int i = warp; i < k; i += NW) {
      const cplx rik = work[i];
      const int ri = pku(i, i, N);
      for (int jj = k + lane; jj < N; jj += 32) {
        const cplx base = (jj == k) ? mk(0.0, 0.0) : A[ri + (jj - i)];
        A[ri + (jj - i)] = csub(base, cmul(rik, A[rk + (jj - k)]));
      }
    }
    __syncthreads();
  }
  const double nX = norm1_inf_upper(A, N, red);
  // zero the strictly lower part (the GEMM W R^-1 reads the full square)
  for (int e = tid; e < N * N; e += LU_THREADS) {
    const int i = e / N, k = e % N;
    Sb[e] = (i > k) ? mk(0.0, 0.0) : A[pku(i, k, N)];
  }
  if (tid == 0) {
    status[b] = 0;
    if (again) again[b] = (sqrt(nR * nX) > kappa_max) ? 1 : 0;
  }
}

}  // namespace

size_t lu_smem_bytes(int N) { return size_t(N) * N * sizeof(cplx) + size_t(N) * sizeof(cplx) + size_t(N) * sizeof(int) + 16; }

int lu_logdet(cplx* T, long sT, int nbatch, int N, cplx* ovlp, bool accumulate, double post_scale, bool invert,
              cudaStream_t st) {
  if (nbatch <= 0) return SFQ_OK;
  if (N <= 0) return SFQ_OK;
  if (N > kMaxSmallN) return record_error(SFQ_ERR_UNSUPPORTED, "lu_logdet: N=%d exceeds %d", N, kMaxSmallN);
  // register-resident Gauss-Jordan for the sizes it covers; shared-memory LU + getri above that
  if (N <= kGjMaxLarge) return gj_logdet(T, sT, nbatch, N, ovlp, accumulate, post_scale, invert, st);
  const size_t sm = lu_smem_bytes(N);
  if (invert) {
    SFQ_CUDA_TRY(cudaFuncSetAttribute(lu_logdet_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    lu_logdet_kernel<true><<<nbatch, LU_THREADS, sm, st>>>(T, sT, N, ovlp, accumulate ? 1 : 0, post_scale);
  } else {
    SFQ_CUDA_TRY(cudaFuncSetAttribute(lu_logdet_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    lu_logdet_kernel<false><<<nbatch, LU_THREADS, sm, st>>>(T, sT, N, ovlp, accumulate ? 1 : 0, post_scale);
  }
  SFQ_LAUNCHED();
  return SFQ_OK;
}

int chol_rinv(cplx* S, long sS, int nbatch, int N, int* status, int* again, const int* active, double kappa_max,
              cudaStream_t st, cplx* Rout) {
  if (nbatch <= 0 || N <= 0) return SFQ_OK;
  if (N > kMaxSmallN) return record_error(SFQ_ERR_UNSUPPORTED, "chol_rinv: N=%d exceeds %d", N, kMaxSmallN);
  const size_t sm = size_t(N) * (N + 1) / 2 * sizeof(cplx) + size_t(N) * sizeof(cplx);  // packed R + work
  SFQ_CUDA_TRY(cudaFuncSetAttribute(chol_rinv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
  chol_rinv_kernel<<<nbatch, LU_THREADS, sm, st>>>(S, sS, N, status, again, active, kappa_max, Rout);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

}  // namespace sfq
