// Register-resident Gauss-Jordan inverse + log det for the per-walker N x N overlap matrices.
//
// One CTA per matrix, 4*N threads.  Thread t owns column j = t / 4 and rows i = (t % 4) + 4 r,
// r < R: the matrix lives in registers, the four owners of a column are four adjacent lanes of one
// warp (the pivot search is a shuffle reduction).  One block barrier per step: the pivot column
// and pivot go through shared memory (double-buffered), the pivot row by warp shuffles (each
// element is needed only by the owners of its column).  The warp that holds column k+1 starts its
// pivot search as soon as its own step-k elimination is done.  A step costs each thread one shared
// load and four FMAs per row it owns.
//
// Pivoting reproduces LAPACK's partial pivoting (zgetrf): the pivot of column k is the first
// maximum of |re| + |im| over the rows not yet pivoted, "first" in the row order LAPACK has after
// its interchanges -- tracked as a position per row instead of moving rows.  The pivots are the U
// diagonal of LAPACK's LU, and the log determinant follows log_determinant_from_getrf
// (src/numerics/operations/determinants_impl.hpp:33-75): sum over k of log(+-U_kk + tiny), negated
// when the pivot came from another position, imaginary part folded into [-pi, pi].
// The sweep is Gauss-Jordan in place with the pivot rows left unscaled until the end, where
// A^-1[a][p_k] = B[p_a][k] / U_aa (p_k: pivot row of step k) is scattered straight to the output
// with INVERT; without it only the log det is written.  A zero pivot marks the matrix singular: the step is skipped and the
// inverse is written as zeros (getri_or_zero, src/numerics/nda_functions.hpp:422-438).
#include "common.cuh"
#include "kernels.cuh"

namespace sfq {
namespace {

constexpr int kGjMaxN = 128;

__device__ __forceinline__ double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }

// Pivot candidates as integer keys: |re| + |im| of an unpivoted row as its bit pattern (a
// non-negative double orders like its bits, and integer compares are short and branch-free), -1
// for pivoted rows and NaN (never chosen, as no comparison with NaN succeeds).
__device__ __forceinline__ long long cand_key(cplx z, bool cand) {
  const long long bits = __double_as_longlong(fabs(z.x) + fabs(z.y));
  return (cand && bits <= 0x7ff0000000000000LL) ? bits : -1LL;
}

// the largest key of one owner and the bit mask of its rows that attain it, in one pass of NQ
// interleaved running maxima (dependent depth about R/NQ), with selects only: no branch, and no
// key kept beyond its own step (three chains at R = 25, whose matrix leaves few registers)
template <int R>
__device__ __forceinline__ void owner_max(const cplx (&a)[R], int g, int N, unsigned pivoted, long long& best,
                                          unsigned& mask) {
  constexpr int NQ = R > 16 ? 3 : 4;
  long long m[NQ];
  unsigned mk_[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    m[q] = -1LL;
    mk_[q] = 0u;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int q = r % NQ;
    const long long key = cand_key(a[r], g + 4 * r < N && !((pivoted >> r) & 1u));
    const bool gt = key > m[q], eq = key == m[q];
    mk_[q] = gt ? (1u << r) : (eq ? (mk_[q] | (1u << r)) : mk_[q]);
    m[q] = gt ? key : m[q];
  }
  best = m[0];
#pragma unroll
  for (int q = 1; q < NQ; ++q) best = m[q] > best ? m[q] : best;
  mask = 0u;
#pragma unroll
  for (int q = 0; q < NQ; ++q) mask |= (m[q] == best) ? mk_[q] : 0u;
}

template <int R, bool INVERT>
__global__ void __launch_bounds__(((16 * R + 31) / 32) * 32)
    gj_kernel(cplx* T, long sT, int N, cplx* ovlp, int accumulate, double post_scale) {
  __shared__ cplx prow[2][kGjMaxN];
  __shared__ cplx pcol[2][kGjMaxN];
  __shared__ cplx pinv_of[kGjMaxN];     // 1 / U_kk, for the deferred row scaling
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
  // rows N .. 4R-1 of the pivot column stay zero, so the padding rows stay zero without a test
  for (int i = N + t; i < 4 * R; i += blockDim.x) {
    pcol[0][i] = mk(0.0, 0.0);
    pcol[1][i] = mk(0.0, 0.0);
  }
  if (t == 0) s_singular = 0;
  __syncthreads();

  for (int k = 0; k < N; ++k) {
    const int buf = k & 1;
    // (a) the warp holding column k: candidate per lane, shuffle reduction, winner bookkeeping
    if ((k >> 3) == (t >> 5)) {  // column k lives in lanes 4*(k%8) .. +3 of warp k/8
      const bool mine = (j == k);
      if (mine) {
#pragma unroll
        for (int r = 0; r < R; ++r)
          if (g + 4 * r < N) pcol[buf][g + 4 * r] = a[r];
      }
      long long best = -1LL;
      unsigned mask = 0u;
      if (mine) owner_max<R>(a, g, N, pivoted, best, mask);
      int brow = (best >= 0) ? g + 4 * (__ffs(mask) - 1) : (1 << 30);
      bool tie = best >= 0 && __popc(mask) > 1;
      // reduce over the 4 owners (adjacent lanes, aligned to 4)
#pragma unroll
      for (int off = 1; off < 4; off <<= 1) {
        const long long ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int orow = __shfl_xor_sync(0xffffffffu, brow, off);
        const int otie = __shfl_xor_sync(0xffffffffu, int(tie), off);
        if (ob > best) {
          best = ob;
          brow = orow;
          tie = otie != 0;
        } else if (ob == best && ob >= 0) {
          tie = true;
        }
      }
      // only the four lanes of column k can see a tie: decide warp-uniformly, since the shuffles
      // below need every lane
      if (__any_sync(0xffffffffu, tie)) {
        // exact zgetrf rule among the tied maxima: the lowest LAPACK position
        int bpos = 1 << 30, prow_ = 1 << 30;
        if (mine && tie) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = g + 4 * r;
            if (i < N && cand_key(a[r], !((pivoted >> r) & 1u)) == best) {
              const int ps = pos_of[i];
              if (ps < bpos) {
                bpos = ps;
                prow_ = i;
              }
            }
          }
        }
#pragma unroll
        for (int off = 1; off < 4; off <<= 1) {
          const int opos = __shfl_xor_sync(0xffffffffu, bpos, off);
          const int orow = __shfl_xor_sync(0xffffffffu, prow_, off);
          if (opos < bpos) {
            bpos = opos;
            prow_ = orow;
          }
        }
        if (tie) brow = prow_;
      }
      __syncwarp();  // the column's stores to pcol[buf] come before their use below
      if (mine && g == 0) {
        // no candidate compares (a column of NaNs): take the row at position k; bz = 0 makes the
        // step singular
        const cplx bz = brow < N ? pcol[buf][brow] : mk(0.0, 0.0);
        const int p = brow < N ? brow : row_at[k];
        pcol[buf][p] = mk(0.0, 0.0);  // the pivot row itself is left as it is (scaled at the end)
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
          pinv_of[k] = mk(0.0, 0.0);
          s_singular = 1;
        } else {
          const double inv = __drcp_rn(d);
          s_pinv[buf] = mk(bz.x * inv, -bz.y * inv);
          pinv_of[k] = s_pinv[buf];
        }
      }
      // column k is now in pcol: its owners clear it, so that the sweep below leaves -a_ik / a_pk
      if (mine) {
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = mk(0.0, 0.0);
      }
    }
    __syncthreads();
    const int p = s_p[buf];
    const cplx pinv = s_pinv[buf];
    const bool skip = (pinv.x == 0.0 && pinv.y == 0.0);
    const int gp = p & 3, rp = p >> 2;
    if (g == gp) pivoted |= 1u << rp;
    // (b) the pivot row element of column j, normalised (column k: the reciprocal pivot); the
    // owner of row p in column j hands it to the other three owners through shared memory
    const int rsel = (active && g == gp) ? rp : -1;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (r == rsel) prow[buf][j] = a[r];
    __syncwarp();
    // (c) eliminate column k from every other row: a_ij -= a_ik pr_j.  Column k was cleared, so it
    // becomes -a_ik / a_pk; row p, whose pivot-column entry reads as 0, keeps its values:
    // pivot rows are normalised only when the result is written (times 1 / a_pk, and + 1 at
    // column k, where the clearing left 0 instead of a_pk / a_pk).  The LU variant runs the same
    // sweep: its trailing block, pivots and log det are the same numbers.
    if (active && !skip) {
      const cplx pr = (j == k) ? pinv : cmul(prow[buf][j], pinv);
      const cplx* pc = pcol[buf];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const cplx f = pc[g + 4 * r];
        a[r].x = fma(-f.x, pr.x, fma(f.y, pr.y, a[r].x));
        a[r].y = fma(-f.x, pr.y, fma(-f.y, pr.x, a[r].y));
        if ((r & 3) == 3) asm volatile("" ::: "memory");  // bounds the loads in flight (registers)
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
  // A^-1[step_of[i]][piv_row[j]] = (B[i][j] + [j == step_of[i]]) / a_(i, step_of[i])
  if (active) {
    const int col = piv_row[j];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = g + 4 * r;
      if (i < N) {
        const int si = step_of[i];
        cplx v = a[r];
        if (si == j) v.x += 1.0;
        Tb[(long)si * N + col] = singular ? mk(0.0, 0.0) : cmul(v, pinv_of[si]);
      }
      if ((r & 3) == 3) asm volatile("" ::: "memory");
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
