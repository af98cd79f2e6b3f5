// Register-resident Gauss-Jordan inverse + log det for the per-walker N x N overlap matrices.
//
// One CTA per matrix, 4*N threads.  Thread t owns column j = t / 4 and rows i = (t % 4) + 4 r,
// r < R: the matrix lives in registers, the four owners of a column are four adjacent lanes of one
// warp (the pivot search is a shuffle reduction), and an elimination step moves only the pivot row
// and pivot column through shared memory (double-buffered, two barriers per step).
//
// Pivoting reproduces LAPACK's partial pivoting (zgetrf): the pivot of column k is the first
// maximum of |re| + |im| over the rows not yet pivoted, "first" in the row order LAPACK has after
// its interchanges -- tracked as a position per row instead of moving rows.  The pivots are the U
// diagonal of LAPACK's LU, and the log determinant follows log_determinant_from_getrf
// (src/numerics/operations/determinants_impl.hpp:33-75): sum over k of log(+-U_kk + tiny), negated
// when the pivot came from another position, imaginary part folded into [-pi, pi].
// With INVERT the sweep is Gauss-Jordan in place and ends with A^-1[a][p_k] = B[p_a][k]
// (p_k: pivot row of step k), scattered straight to the output; without it only the trailing
// block is updated (an LU).  A zero pivot marks the matrix singular: the step is skipped and the
// inverse is written as zeros (getri_or_zero, src/numerics/nda_functions.hpp:422-438).
#include "common.cuh"
#include "kernels.cuh"

namespace sfq {
namespace {

constexpr int kGjMaxN = 128;

__device__ __forceinline__ double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }

template <int R, bool INVERT>
__global__ void __launch_bounds__(4 * 4 * R + 32)
    gj_kernel(cplx* T, long sT, int N, cplx* ovlp, int accumulate, double post_scale) {
  __shared__ cplx prow[2][kGjMaxN];
  __shared__ cplx pcol[2][kGjMaxN];
  __shared__ cplx diag[kGjMaxN];        // U_kk, for the log det
  __shared__ unsigned char flip[kGjMaxN];
  __shared__ int pos_of[kGjMaxN];       // LAPACK position of each physical row
  __shared__ int row_at[kGjMaxN];       // physical row at each LAPACK position
  __shared__ int step_of[kGjMaxN];      // step at which the row was the pivot
  __shared__ int piv_row[kGjMaxN];      // pivot row of each step
  __shared__ int s_p[2];
  __shared__ cplx s_pinv[2];
  __shared__ int s_singular;

  const int t = threadIdx.x;
  const int g = t & 3, j = t >> 2;
  const bool active = j < N;
  const long b = blockIdx.x;
  cplx* Tb = T + b * sT;

  cplx a[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = g + 4 * r;
    a[r] = (active && i < N) ? Tb[(long)i * N + j] : mk(0.0, 0.0);
  }
  unsigned pivoted = 0;  // bit r: row g + 4r already pivoted
  for (int i = t; i < N; i += blockDim.x) {
    pos_of[i] = i;
    row_at[i] = i;
  }
  if (t == 0) s_singular = 0;
  __syncthreads();

  for (int k = 0; k < N; ++k) {
    const int buf = k & 1;
    // (a) the warp holding column k: candidate per lane, shuffle reduction, winner bookkeeping
    if ((k >> 3) == (t >> 5)) {  // column k lives in lanes 4*(k%8) .. +3 of warp k/8
      const bool mine = (j == k);
      double best = -1.0;
      int brow = 1 << 30;
      cplx bz = mk(0.0, 0.0);
      if (mine) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = g + 4 * r;
          if (i < N) {
            pcol[buf][i] = a[r];
            if (!((pivoted >> r) & 1u)) {
              const double v = cabs1(a[r]);
              if (v > best) {
                best = v;
                brow = i;
                bz = a[r];
              } else if (v == best && pos_of[i] < pos_of[brow]) {
                brow = i;
                bz = a[r];
              }
            }
          }
        }
      }
      // reduce over the 4 owners (adjacent lanes, aligned to 4)
#pragma unroll
      for (int off = 1; off < 4; off <<= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int orow = __shfl_xor_sync(0xffffffffu, brow, off);
        const double ozx = __shfl_xor_sync(0xffffffffu, bz.x, off);
        const double ozy = __shfl_xor_sync(0xffffffffu, bz.y, off);
        bool take = ob > best;
        if (!take && ob == best && ob >= 0.0 && orow < N && brow < N) take = pos_of[orow] < pos_of[brow];
        if (take) {
          best = ob;
          brow = orow;
          bz = mk(ozx, ozy);
        }
      }
      if (mine && g == 0) {
        const int p = brow;
        const int ps = pos_of[p];
        flip[k] = ps != k ? 1 : 0;  // ipiv[k] != k: zgetrf swapped rows
        const int other = row_at[k];
        row_at[ps] = other;
        pos_of[other] = ps;
        row_at[k] = p;
        pos_of[p] = k;
        step_of[p] = k;
        piv_row[k] = p;
        diag[k] = bz;
        s_p[buf] = p;
        const double d = bz.x * bz.x + bz.y * bz.y;
        if (d == 0.0) {
          s_pinv[buf] = mk(0.0, 0.0);
          s_singular = 1;
        } else {
          const double inv = 1.0 / d;
          s_pinv[buf] = mk(bz.x * inv, -bz.y * inv);
        }
      }
    }
    __syncthreads();
    const int p = s_p[buf];
    const cplx pinv = s_pinv[buf];
    const bool skip = (pinv.x == 0.0 && pinv.y == 0.0);
    const int gp = p & 3, rp = p >> 2;
    if (g == gp) pivoted |= 1u << rp;
    // (b) the pivot row, normalised; column k carries the reciprocal pivot (in-place inverse)
    if (active && g == gp) {
      cplx v = mk(0.0, 0.0);
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (r == rp) v = a[r];
      prow[buf][j] = (j == k) ? pinv : cmul(v, pinv);
    }
    __syncthreads();
    // (c) eliminate column k (Gauss-Jordan: every other row; LU: the trailing block only)
    if (active && !skip && (INVERT || j > k)) {
      const cplx pr = prow[buf][j];
      const bool colk = (j == k);
      const cplx* pc = pcol[buf];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = g + 4 * r;
        const bool live = INVERT ? true : !((pivoted >> r) & 1u);
        if (i < N && live) {
          const cplx f = pc[i];
          const cplx base = colk ? mk(0.0, 0.0) : a[r];
          const cplx upd = csub(base, cmul(f, pr));
          a[r] = (i == p) ? pr : upd;
        }
        if ((r & 3) == 3) asm volatile("" ::: "memory");
      }
    }
  }
  __syncthreads();
  // log det: terms in parallel, summed in order by thread 0
  const double tiny = 2.2250738585072014e-308;
  if (t < N) {
    cplx u = diag[t];
    cplx v = flip[t] ? mk(-u.x, -u.y) : u;
    v.x += tiny;
    pcol[0][t] = clog_(v);
  }
  __syncthreads();
  if (t == 0) {
    cplx res = accumulate ? ovlp[b] : mk(0.0, 0.0);
    for (int k = 0; k < N; ++k) res = cadd(res, pcol[0][k]);
    const double pi = 3.141592653589793238462643383279502884;
    if (res.y > pi) {
      for (int it = 0; res.y > pi && it < 4 * N + 8; ++it) res.y -= 2 * pi;
    } else if (res.y < -pi) {
      for (int it = 0; res.y < -pi && it < 4 * N + 8; ++it) res.y += 2 * pi;
    }
    ovlp[b] = mk(res.x * post_scale, res.y * post_scale);
  }
  if (!INVERT) return;
  const bool singular = s_singular != 0;
  // A^-1[step_of[i]][piv_row[j]] = B[i][j]
  if (active) {
    const int col = piv_row[j];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = g + 4 * r;
      if (i < N) Tb[(long)step_of[i] * N + col] = singular ? mk(0.0, 0.0) : a[r];
    }
  }
}

template <int R>
int launch_gj(cplx* T, long sT, int nbatch, int N, cplx* ovlp, bool accumulate, double post_scale, bool invert,
              cudaStream_t st) {
  const int threads = ((4 * N + 31) / 32) * 32;
  if (invert)
    gj_kernel<R, true><<<nbatch, threads, 0, st>>>(T, sT, N, ovlp, accumulate ? 1 : 0, post_scale);
  else
    gj_kernel<R, false><<<nbatch, threads, 0, st>>>(T, sT, N, ovlp, accumulate ? 1 : 0, post_scale);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

}  // namespace

int gj_logdet(cplx* T, long sT, int nbatch, int N, cplx* ovlp, bool accumulate, double post_scale, bool invert,
              cudaStream_t st) {
  if (nbatch <= 0 || N <= 0) return SFQ_OK;
  if (N <= 32) return launch_gj<8>(T, sT, nbatch, N, ovlp, accumulate, post_scale, invert, st);
  if (N <= 64) return launch_gj<16>(T, sT, nbatch, N, ovlp, accumulate, post_scale, invert, st);
  if (N <= kGjMaxLarge) return launch_gj<25>(T, sT, nbatch, N, ovlp, accumulate, post_scale, invert, st);
  return record_error(SFQ_ERR_UNSUPPORTED, "gj_logdet: N=%d above %d", N, kGjMaxLarge);
}

}  // namespace sfq
