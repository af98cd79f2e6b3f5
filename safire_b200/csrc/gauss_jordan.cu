// Register-resident Gauss-Jordan inverse + log det for the per-walker N x N overlap matrices.
//
// One CTA per matrix: 4*N threads (rounded up to whole warps) hold the matrix, plus one pivot
// warp.  Thread t < 4N owns column j = t / 4 and rows i = (t % 4) + 4 r, r < R, in registers; the
// four owners of a column are four adjacent lanes of one warp.  One block barrier per step and no
// other wait: the pivot warp works on shared-memory copies only.
// Step k (pivot row p_k known): every owner takes its column's element of the pivot row (through
// shared memory, from the owner of row p_k in the same warp) and eliminates: one shared load of the
// pivot column and four FMAs per owned row.  Column k+1 is not in registers during step k: its
// owners wrote it to shared memory at the end of step k-1 and cleared it.  The pivot warp updates
// that copy (four rows per lane, the same FMAs the owners would make), finds the pivot of step k+1
// in its registers and publishes the column with the pivot row zeroed, while the owners sweep.  At
// the end of step k the owners of column k+2 move it to shared memory the same way.
//
// Pivoting reproduces LAPACK's partial pivoting (zgetrf): the pivot of column k is the first
// maximum of |re| + |im| over the rows not yet pivoted, "first" in the row order LAPACK has after
// its interchanges -- tracked as a position per row instead of moving rows.  The pivots are the U
// diagonal of LAPACK's LU, and the log determinant follows log_determinant_from_getrf
// (src/numerics/operations/determinants_impl.hpp:33-75): sum over k of log(+-U_kk + tiny), negated
// when the pivot came from another position, imaginary part folded into [-pi, pi].
// The sweep is Gauss-Jordan in place with the pivot rows left unscaled until the end, where
// A^-1[a][p_k] = B[p_a][k] / U_aa (p_k: pivot row of step k) is scattered straight to the output
// with INVERT; without it only the log det is written.  A zero pivot marks the matrix singular: the
// step is skipped and the inverse is written as zeros (getri_or_zero,
// src/numerics/nda_functions.hpp:422-438).
#include "common.cuh"
#include "kernels.cuh"

namespace sfq {
namespace {

constexpr int kGjMaxN = 128;

// Pivot candidates as integer keys: |re| + |im| of an unpivoted row as its bit pattern (a
// non-negative double orders like its bits, and integer compares are short and branch-free), -1
// for pivoted rows and NaN (never chosen, as no comparison with NaN succeeds).
__device__ __forceinline__ long long cand_key(cplx z, bool cand) {
  const long long bits = __double_as_longlong(fabs(z.x) + fabs(z.y));
  return (cand && bits <= 0x7ff0000000000000LL) ? bits : -1LL;
}

// The pivot of step k from column k held by the pivot warp (v[q]: row lane + 32 q; pmask bit q:
// that row already pivoted), then column k with the pivot row zeroed to pc (the sweep's
// multipliers; the pivot row is left as it is by the elimination and scaled at the end) and lane
// 0's bookkeeping: LAPACK positions, the pivot's reciprocal.
__device__ __forceinline__ void pivot_step(int k, int N, const cplx (&v)[kGjMaxN / 32], unsigned& pmask, cplx* pc,
                                           int* pos_of, int* row_at, int* step_of, int* piv_row, cplx* diag,
                                           unsigned char* flip, cplx* pinv_of, int* s_p, cplx* s_pinv,
                                           int* s_singular) {
  const int lane = threadIdx.x & 31;
  long long best = -1LL;
  int brow = 1 << 30;
  int cnt = 0;
#pragma unroll
  for (int q = 0; q < kGjMaxN / 32; ++q) {
    const int i = lane + 32 * q;
    if (i < N) {
      const long long key = cand_key(v[q], ((pmask >> q) & 1u) == 0u);
      if (key > best) {
        best = key;
        brow = i;
        cnt = 1;
      } else if (key == best && key >= 0) {
        ++cnt;
      }
    }
  }
  // the warp's largest key: keys + 1 as unsigned (no candidate, -1, becomes the least), reduced by
  // its high word, then by its low word among the lanes that hold the largest high word (two
  // redux.sync instead of a shuffle tree); the lanes holding the maximum are the ballot's
  {
    const unsigned long long u = (unsigned long long)(best + 1);
    const unsigned hi = unsigned(u >> 32), lo = unsigned(u);
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const unsigned win = __ballot_sync(0xffffffffu, hi == mhi && lo == mlo);
    best = (long long)(((unsigned long long)mhi << 32) | mlo) - 1;
    const bool any = best >= 0;
    // a tie: two lanes with the maximum, or one lane with it in two of its rows
    const bool tie = any && (__popc(win) > 1 || __any_sync(0xffffffffu, ((win >> lane) & 1u) && cnt > 1));
    brow = any ? __shfl_sync(0xffffffffu, brow, __ffs(win) - 1) : (1 << 30);
    cnt = tie ? 2 : 1;
  }
  if (cnt > 1) {
    // exact zgetrf rule among the tied maxima: the lowest LAPACK position
    int bpos = 1 << 30, prow_ = 1 << 30;
#pragma unroll
    for (int q = 0; q < kGjMaxN / 32; ++q) {
      const int i = lane + 32 * q;
      if (i < N && cand_key(v[q], ((pmask >> q) & 1u) == 0u) == best && pos_of[i] < bpos) {
        bpos = pos_of[i];
        prow_ = i;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const int opos = __shfl_xor_sync(0xffffffffu, bpos, off);
      const int orow = __shfl_xor_sync(0xffffffffu, prow_, off);
      if (opos < bpos) {
        bpos = opos;
        prow_ = orow;
      }
    }
    brow = prow_;
  }
  // brow is the same in every lane.  No candidate compares (a column of NaNs): take the row at
  // position k; bz = 0 makes the step singular
  const bool found = brow < N;
  const int p = found ? brow : row_at[k];
  const int qp = p >> 5;
  cplx vp = v[0];
#pragma unroll
  for (int q = 1; q < kGjMaxN / 32; ++q)
    if (q == qp) vp = v[q];
  vp.x = __shfl_sync(0xffffffffu, vp.x, p & 31);
  vp.y = __shfl_sync(0xffffffffu, vp.y, p & 31);
  const cplx bz = found ? vp : mk(0.0, 0.0);
#pragma unroll
  for (int q = 0; q < kGjMaxN / 32; ++q) {
    const int i = lane + 32 * q;
    if (i < N) pc[i] = (i == p) ? mk(0.0, 0.0) : v[q];
  }
  if (lane == (p & 31)) pmask |= 1u << qp;
  if (lane == 0) {
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
    *s_p = p;
    const double d = bz.x * bz.x + bz.y * bz.y;
    if (d == 0.0) {
      *s_pinv = mk(0.0, 0.0);
      pinv_of[k] = mk(0.0, 0.0);
      *s_singular = 1;
    } else {
      const double inv = __drcp_rn(d);
      *s_pinv = mk(bz.x * inv, -bz.y * inv);
      pinv_of[k] = *s_pinv;
    }
  }
}

// Block barrier that whole warps may reach from different places in the code (bar.sync counts
// threads; each warp executes it together)
__device__ __forceinline__ void block_barrier(unsigned nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// a[r] for a row index r that is the same in every thread (the pivot row's slot): one switch on a
// uniform value instead of R predicated stores per thread
template <int R>
__device__ __forceinline__ cplx pick_row(const cplx (&a)[R], int r) {
  static_assert(R <= 32, "rows per lane");
  cplx v = mk(0.0, 0.0);
  switch (r) {
#define SFQ_PICK(n) \
  case n:           \
    if (n < R) v = a[n < R ? n : 0]; \
    break;
    SFQ_PICK(0) SFQ_PICK(1) SFQ_PICK(2) SFQ_PICK(3) SFQ_PICK(4) SFQ_PICK(5) SFQ_PICK(6) SFQ_PICK(7)
    SFQ_PICK(8) SFQ_PICK(9) SFQ_PICK(10) SFQ_PICK(11) SFQ_PICK(12) SFQ_PICK(13) SFQ_PICK(14) SFQ_PICK(15)
    SFQ_PICK(16) SFQ_PICK(17) SFQ_PICK(18) SFQ_PICK(19) SFQ_PICK(20) SFQ_PICK(21) SFQ_PICK(22) SFQ_PICK(23)
    SFQ_PICK(24) SFQ_PICK(25) SFQ_PICK(26) SFQ_PICK(27) SFQ_PICK(28) SFQ_PICK(29) SFQ_PICK(30) SFQ_PICK(31)
#undef SFQ_PICK
    default:
      break;
  }
  return v;
}

template <int R, int LPC, bool INVERT>
__global__ void __launch_bounds__(((LPC * LPC * R + 31) / 32) * 32 + 32)
    gj_kernel(cplx* T, long sT, int N, cplx* ovlp, int accumulate, double post_scale) {
  static_assert(LPC == 4 || LPC == 8, "owners per column");
  __shared__ cplx prow[2][kGjMaxN];
  __shared__ cplx pcol[2][kGjMaxN];    // the pivot column of step k (pivot row zeroed): [k & 1]
  __shared__ cplx ncol[2][kGjMaxN];    // column k+1 before step k's sweep: [(k + 1) & 1]
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
  const int ncol_threads = ((LPC * N + 31) / 32) * 32;
  const bool pivot_warp = t >= ncol_threads;
  const int g = t % LPC, j = t / LPC;
  const bool active = !pivot_warp && j < N;
  const long b = blockIdx.x;
  cplx* Tb = T + b * sT;

  cplx a[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = g + LPC * r;
    a[r] = (active && i < N) ? Tb[(long)i * N + j] : mk(0.0, 0.0);
  }
  for (int i = t; i < N; i += blockDim.x) {
    pos_of[i] = i;
    row_at[i] = i;
  }
  // rows N .. 4R-1 of the pivot column stay zero, so the padding rows stay zero without a test
  for (int i = N + t; i < LPC * R; i += blockDim.x) {
    pcol[0][i] = mk(0.0, 0.0);
    pcol[1][i] = mk(0.0, 0.0);
  }
  if (t == 0) s_singular = 0;
  // column 0 for the first pivot search and column 1 for step 0 go to shared memory; their
  // registers start the sweep cleared (column 0 becomes -a_i0 / a_p0)
  if (active && j <= 1) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (g + LPC * r < N) (j == 0 ? pcol[0] : ncol[1])[g + LPC * r] = a[r];
      a[r] = mk(0.0, 0.0);
    }
  }
  __syncthreads();
  // From here the pivot warp and the column warps run separate loops that meet at the same number
  // of block barriers (one per step plus two); every warp is wholly on one side, so each barrier
  // instruction is executed by whole warps.
  const unsigned nthreads = blockDim.x;
  if (pivot_warp) {
    const int lane = t & 31;
    unsigned pmask = 0;  // bit q set once row lane + 32 q was a pivot
    {
      cplx v[kGjMaxN / 32];
#pragma unroll
      for (int q = 0; q < kGjMaxN / 32; ++q) v[q] = lane + 32 * q < N ? pcol[0][lane + 32 * q] : mk(0.0, 0.0);
      __syncwarp();
      pivot_step(0, N, v, pmask, pcol[0], pos_of, row_at, step_of, piv_row, diag, flip, pinv_of, &s_p[0],
                 &s_pinv[0], &s_singular);
    }
    block_barrier(nthreads);
    for (int k = 0; k < N; ++k) {
      const int buf = k & 1, nb = buf ^ 1;
      // column k+1: step k's update of the shared copy (the owners' FMAs), then the pivot of step k+1
      if (k + 1 < N) {
        const int p = s_p[buf];
        const cplx pinv = s_pinv[buf];
        const bool skip = (pinv.x == 0.0 && pinv.y == 0.0);
        const cplx* pc = pcol[buf];
        const cplx* nc = ncol[nb];
        const cplx pr = skip ? mk(0.0, 0.0) : cmul(nc[p], pinv);
        cplx v[kGjMaxN / 32];
#pragma unroll
        for (int q = 0; q < kGjMaxN / 32; ++q) {
          const int i = lane + 32 * q;
          v[q] = i < N ? nc[i] : mk(0.0, 0.0);
          if (!skip && i < N) {
            const cplx f = pc[i];
            v[q].x = fma(-f.x, pr.x, fma(f.y, pr.y, v[q].x));
            v[q].y = fma(-f.x, pr.y, fma(-f.y, pr.x, v[q].y));
          }
        }
        pivot_step(k + 1, N, v, pmask, pcol[nb], pos_of, row_at, step_of, piv_row, diag, flip, pinv_of, &s_p[nb],
                   &s_pinv[nb], &s_singular);
      }
      block_barrier(nthreads);
    }
    block_barrier(nthreads);  // the log det's barrier
    return;
  }
  block_barrier(nthreads);

  for (int k = 0; k < N; ++k) {
    const int buf = k & 1;
    const int p = s_p[buf];
    const cplx pinv = s_pinv[buf];
    const bool skip = (pinv.x == 0.0 && pinv.y == 0.0);
    const cplx* pc = pcol[buf];
    const int gp = p % LPC, rp = p / LPC;
    // (b) the pivot row element of column j, normalised (column k: the reciprocal pivot); the
    // owner of row p in column j hands it to the other three owners through shared memory
    {
      const cplx v = pick_row<R>(a, rp);  // rp is the same in every thread
      if (active && g == gp) prow[buf][j] = v;
    }
    __syncwarp();
    // (c) eliminate column k from every other row: a_ij -= a_ik pr_j.  Column k was cleared, so it
    // becomes -a_ik / a_pk; row p, whose pivot-column entry reads as 0, keeps its values: pivot rows
    // are normalised only when the result is written (times 1 / a_pk, and + 1 at column k, where
    // the clearing left 0 instead of a_pk / a_pk).  Column k+1 is the pivot warp's this step.  The
    // LU variant runs the same sweep: its trailing block, pivots and log det are the same numbers.
    if (active && !skip && j != k + 1) {
      const cplx pr = (j == k) ? pinv : cmul(prow[buf][j], pinv);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const cplx f = pc[g + LPC * r];
        a[r].x = fma(-f.x, pr.x, fma(f.y, pr.y, a[r].x));
        a[r].y = fma(-f.x, pr.y, fma(-f.y, pr.x, a[r].y));
        if ((r & 3) == 3) asm volatile("" ::: "memory");  // bounds the loads in flight (registers)
      }
    }
    // column k+2 to shared memory for the pivot warp's step k+1, cleared here
    if (active && j == k + 2) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (g + LPC * r < N) ncol[buf][g + LPC * r] = a[r];
        a[r] = mk(0.0, 0.0);
      }
    }
    block_barrier(nthreads);
  }
  // log det: terms in parallel, summed in order by thread 0
  const double tiny = 2.2250738585072014e-308;
  if (t < N) {
    cplx u = diag[t];
    cplx v = flip[t] ? mk(-u.x, -u.y) : u;
    v.x += tiny;
    pcol[0][t] = clog_(v);
  }
  block_barrier(nthreads);
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
      const int i = g + LPC * r;
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

template <int R, int LPC>
int launch_gj(cplx* T, long sT, int nbatch, int N, cplx* ovlp, bool accumulate, double post_scale, bool invert,
              cudaStream_t st) {
  const int threads = ((LPC * N + 31) / 32) * 32 + 32;  // column owners + the pivot warp
  if (invert)
    gj_kernel<R, LPC, true><<<nbatch, threads, 0, st>>>(T, sT, N, ovlp, accumulate ? 1 : 0, post_scale);
  else
    gj_kernel<R, LPC, false><<<nbatch, threads, 0, st>>>(T, sT, N, ovlp, accumulate ? 1 : 0, post_scale);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

}  // namespace

int gj_logdet(cplx* T, long sT, int nbatch, int N, cplx* ovlp, bool accumulate, double post_scale, bool invert,
              cudaStream_t st) {
  if (nbatch <= 0 || N <= 0) return SFQ_OK;
  if (N <= 32) return launch_gj<8, 4>(T, sT, nbatch, N, ovlp, accumulate, post_scale, invert, st);
  if (N <= 64) return launch_gj<16, 4>(T, sT, nbatch, N, ovlp, accumulate, post_scale, invert, st);
  if (N <= kGjMaxLarge) return launch_gj<13, 8>(T, sT, nbatch, N, ovlp, accumulate, post_scale, invert, st);
  return record_error(SFQ_ERR_UNSUPPORTED, "gj_logdet: N=%d above %d", N, kGjMaxLarge);
}

}  // namespace sfq
