// Register-resident Gauss-Jordan inverse + log det for the per-walker N x N overlap matrices.
//
// One CTA per matrix: 4*N threads (rounded up to whole warps) hold the matrix, plus one pivot
// warp.  Thread t < 4N owns column j = t / 4 and rows i = (t % 4) + 4 r, r < R, in registers; the
// four owners of a column are four adjacent lanes of one warp.  One block barrier per step.
// Step k: every owner takes its column's element of the pivot row (through shared memory, from
// the owner of row p_k in the same warp) and eliminates: one shared load of the pivot column and
// four FMAs per owned row.  The four owners of column k+1 do their rows first, publish the
// updated column to shared memory and signal the pivot warp (an mbarrier), which searches the
// pivot of step k+1 and does the bookkeeping while the other warps are still eliminating: the
// pivot search is off the critical path.
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
// src/numerics/nda_functions.hpp:422-438).  The pivot warp's wait for each column is bounded (2 s
// from the start of that wait); if one ever expired the matrix would be reported as singular with a
// NaN log det.
#include "common.cuh"
#include "kernels.cuh"

namespace sfq {
namespace {

constexpr int kGjMaxN = 128;
constexpr unsigned long long kGjWaitNs = 2000000000ull;

// Pivot candidates as integer keys: |re| + |im| of an unpivoted row as its bit pattern (a
// non-negative double orders like its bits, and integer compares are short and branch-free), -1
// for pivoted rows and NaN (never chosen, as no comparison with NaN succeeds).
__device__ __forceinline__ long long cand_key(cplx z, bool cand) {
  const long long bits = __double_as_longlong(fabs(z.x) + fabs(z.y));
  return (cand && bits <= 0x7ff0000000000000LL) ? bits : -1LL;
}

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// The pivot of step k from column k in pc (all 32 lanes of the pivot warp; rows lane + 32 q),
// then lane 0's bookkeeping: LAPACK positions, the pivot's reciprocal, and pc[p] = 0 (the pivot
// row is left as it is by the elimination and scaled at the end).
__device__ __forceinline__ void pivot_search(int k, int N, cplx* pc, unsigned char* prv, int* pos_of, int* row_at,
                                             int* step_of, int* piv_row, cplx* diag, unsigned char* flip,
                                             cplx* pinv_of, int* s_p, cplx* s_pinv, int* s_singular) {
  const int lane = threadIdx.x & 31;
  long long best = -1LL;
  int brow = 1 << 30;
  int cnt = 0;
#pragma unroll
  for (int q = 0; q < kGjMaxN / 32; ++q) {
    const int i = lane + 32 * q;
    if (i < N) {
      const long long key = cand_key(pc[i], prv[i] == 0);
      if (key > best) {
        best = key;
        brow = i;
        cnt = 1;
      } else if (key == best && key >= 0) {
        ++cnt;
      }
    }
  }
  bool tie = cnt > 1;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
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
  if (__any_sync(0xffffffffu, tie)) {
    // exact zgetrf rule among the tied maxima: the lowest LAPACK position
    int bpos = 1 << 30, prow_ = 1 << 30;
#pragma unroll
    for (int q = 0; q < kGjMaxN / 32; ++q) {
      const int i = lane + 32 * q;
      if (i < N && cand_key(pc[i], prv[i] == 0) == best && pos_of[i] < bpos) {
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
  if (lane == 0) {
    // no candidate compares (a column of NaNs): take the row at position k; bz = 0 makes the
    // step singular
    const int p = brow < N ? brow : row_at[k];
    const cplx bz = brow < N ? pc[p] : mk(0.0, 0.0);
    pc[p] = mk(0.0, 0.0);
    prv[p] = 1;
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

template <int R, int LPC, bool INVERT>
__global__ void __launch_bounds__(((LPC * LPC * R + 31) / 32) * 32 + 32)
    gj_kernel(cplx* T, long sT, int N, cplx* ovlp, int accumulate, double post_scale) {
  static_assert(LPC == 4 || LPC == 8, "owners per column");
  constexpr int CPW = 32 / LPC;  // columns per warp
  __shared__ cplx prow[2][kGjMaxN];
  __shared__ cplx pcol[2][kGjMaxN];
  __shared__ cplx pinv_of[kGjMaxN];     // 1 / U_kk, for the deferred row scaling
  __shared__ cplx diag[kGjMaxN];        // U_kk, for the log det
  __shared__ unsigned char flip[kGjMaxN];
  __shared__ unsigned char prv[kGjMaxN];  // row already pivoted
  __shared__ int pos_of[kGjMaxN];       // LAPACK position of each physical row
  __shared__ int row_at[kGjMaxN];       // physical row at each LAPACK position
  __shared__ int step_of[kGjMaxN];      // step at which the row was the pivot
  __shared__ int piv_row[kGjMaxN];      // pivot row of each step
  __shared__ int s_p[2];
  __shared__ cplx s_pinv[2];
  __shared__ int s_singular;
  __shared__ int s_timeout;
  __shared__ uint64_t col_ready;        // the next pivot column is in pcol (32 arrivals)

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
    prv[i] = 0;
  }
  // rows N .. 4R-1 of the pivot column stay zero, so the padding rows stay zero without a test
  for (int i = N + t; i < LPC * R; i += blockDim.x) {
    pcol[0][i] = mk(0.0, 0.0);
    pcol[1][i] = mk(0.0, 0.0);
  }
  if (t == 0) {
    s_singular = 0;
    s_timeout = 0;
    mbar_init(&col_ready, 32);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // column 0 to the pivot column buffer
  if (active && j == 0) {
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (g + LPC * r < N) pcol[0][g + LPC * r] = a[r];
  }
  __syncthreads();
  if (pivot_warp)
    pivot_search(0, N, pcol[0], prv, pos_of, row_at, step_of, piv_row, diag, flip, pinv_of, &s_p[0], &s_pinv[0],
                 &s_singular);
  if (active && j == 0) {  // column 0 is now in pcol: the sweep below turns it into -a_i0 / a_p0
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = mk(0.0, 0.0);
  }
  __syncthreads();

  for (int k = 0; k < N; ++k) {
    const int buf = k & 1, nb = buf ^ 1;
    const int p = s_p[buf];
    const cplx pinv = s_pinv[buf];
    const bool skip = (pinv.x == 0.0 && pinv.y == 0.0);
    const int gp = p % LPC, rp = p / LPC;
    // (b) the pivot row element of column j, normalised (column k: the reciprocal pivot); the
    // owner of row p in column j hands it to the other three owners through shared memory
    const int rsel = (active && g == gp) ? rp : -1;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (r == rsel) prow[buf][j] = a[r];
    __syncwarp();
    const cplx* pc = pcol[buf];
    const bool next_owner_warp = !pivot_warp && k + 1 < N && (t >> 5) == (k + 1) / CPW;
    if (next_owner_warp) {
      // column k+1 first: eliminate it, publish it for the pivot warp, then clear it
      if (j == k + 1) {
        if (!skip) {
          const cplx pr = cmul(prow[buf][j], pinv);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const cplx f = pc[g + LPC * r];
            a[r].x = fma(-f.x, pr.x, fma(f.y, pr.y, a[r].x));
            a[r].y = fma(-f.x, pr.y, fma(-f.y, pr.x, a[r].y));
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (g + LPC * r < N) pcol[nb][g + LPC * r] = a[r];
          a[r] = mk(0.0, 0.0);
        }
      }
      __syncwarp();
      mbar_arrive(&col_ready);
    }
    // (c) eliminate column k from every other row: a_ij -= a_ik pr_j.  Column k was cleared, so it
    // becomes -a_ik / a_pk; row p, whose pivot-column entry reads as 0, keeps its values: pivot rows
    // are normalised only when the result is written (times 1 / a_pk, and + 1 at column k, where
    // the clearing left 0 instead of a_pk / a_pk).  The LU variant runs the same sweep: its
    // trailing block, pivots and log det are the same numbers.
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
    if (pivot_warp && k + 1 < N) {
      // wait (bounded) for column k+1, then its pivot
      bool ok = true;
      if (!mbar_try_wait(&col_ready, uint32_t(k & 1))) {
        const unsigned long long deadline = gtimer() + kGjWaitNs;  // from the start of this wait
        uint32_t spins = 0;
        while (!mbar_try_wait(&col_ready, uint32_t(k & 1))) {
          if ((++spins & 255u) == 0u && gtimer() > deadline) {
            ok = false;
            break;
          }
        }
      }
      if (__all_sync(0xffffffffu, ok)) {
        pivot_search(k + 1, N, pcol[nb], prv, pos_of, row_at, step_of, piv_row, diag, flip, pinv_of, &s_p[nb],
                     &s_pinv[nb], &s_singular);
      } else if ((t & 31) == 0) {
        s_timeout = 1;
        s_singular = 1;
        s_p[nb] = k + 1;
        s_pinv[nb] = mk(0.0, 0.0);
      }
    }
    __syncthreads();
  }
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
    if (s_timeout) res = mk(__longlong_as_double(0x7ff8000000000000LL), 0.0);
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
  if (N <= kGjMaxLarge) return launch_gj<25, 4>(T, sT, nbatch, N, ovlp, accumulate, post_scale, invert, st);
  return record_error(SFQ_ERR_UNSUPPORTED, "gj_logdet: N=%d above %d", N, kGjMaxLarge);
}

}  // namespace sfq
