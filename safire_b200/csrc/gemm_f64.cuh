// Batched FP64 GEMM on the FP64 tensor pipe (DMMA, mma.sync.m8n8k4.f64) for the FP64 drop-in.
//
//   C[b] = alpha * op(A[b]) * B[b] + beta * C[b]        (optionally also  S[b] += alpha*A*B)
//
// A is M x K, B is K x N; either may be real (double) or complex (interleaved re,im: the
// layout of std::complex<double>); C is complex when any operand is.  Operands are described
// by element strides, so transposes, the walker-batched layouts (W, M, N) and the Cholesky
// layouts Likn (M, M, Nc) / Lnak (Nc, N, M) are all plain descriptors.  Each operand must be
// contiguous along K (".k") or along its outer dimension (".mn") -- a template parameter.
//
// Tiles: a CTA owns a BM x BN tile of C, K is consumed in slices of 16 staged through shared
// memory by cp.async (STAGES-deep ring).  Each warp owns a (BM/WM) x (BN/WN) sub-tile made of
// 8x8 DMMA fragments; complex products are four real DMMAs on split re/im fragments.
// Shared-memory row pitches are padded so every fragment load is bank-conflict free.
#pragma once
#include "common.cuh"

namespace sfq {

struct GemmDesc {
  int M = 0, N = 0, K = 0, batch = 1;
  const void* A = nullptr;
  long sAm = 0, sAk = 0, sAb = 0;  // element strides (complex elements count as one)
  const void* B = nullptr;
  long sBk = 0, sBn = 0, sBb = 0;
  void* C = nullptr;
  long sCm = 0, sCn = 0, sCb = 0;
  void* S = nullptr;  // optional second output: S += alpha*A*B (same strides as C)
  bool a_cplx = false, b_cplx = false, conj_a = false;
  cplx alpha = {1.0, 0.0};
  cplx beta = {0.0, 0.0};
  const int* mask = nullptr;  // optional: batch b is computed only where mask[b] != 0
  bool upper_only = false;    // C is needed on and above the diagonal only: tiles wholly below it are skipped
  bool b_upper = false;       // B is upper triangular: column n of C needs K <= n only
};

int gemm_f64(const GemmDesc& d, cudaStream_t stream);

namespace gemm_detail {

constexpr int BKT = 16;  // K slice per pipeline stage

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Pitch (in elements) of a smem tile row whose contiguous extent is `inner`.
template <bool CPLX>
__host__ __device__ constexpr int pitch(int inner, bool inner_is_k) {
  // real: pitch = 4 (mod 16) doubles; complex: pitch = 4 (mod 8) when the row is a K slice
  // (fragment lanes walk rows by 1 and k by 4), 2 (mod 8) when the row runs along M/N.
  return CPLX ? (inner_is_k ? inner + 4 : inner + 2) : inner + 4;
}

template <bool AC, bool BC, bool CONJA, bool AK, bool BK, int BM, int BN, int WM, int WN, int STAGES>
struct Cfg {
  static constexpr int THREADS = WM * WN * 32;
  static constexpr int TM = BM / WM, TN = BN / WN;  // warp tile
  static constexpr int FM = TM / 8, FN = TN / 8;    // fragments per warp
  static constexpr int A_ROWS = AK ? BM : BKT, A_INNER = AK ? BKT : BM;
  static constexpr int B_ROWS = BK ? BN : BKT, B_INNER = BK ? BKT : BN;
  static constexpr int A_PITCH = pitch<AC>(A_INNER, AK);
  static constexpr int B_PITCH = pitch<BC>(B_INNER, BK);
  static constexpr int A_ESZ = AC ? 16 : 8, B_ESZ = BC ? 16 : 8;
  static constexpr int A_STAGE_BYTES = A_ROWS * A_PITCH * A_ESZ;
  static constexpr int B_STAGE_BYTES = B_ROWS * B_PITCH * B_ESZ;
  static constexpr int STAGE_BYTES = A_STAGE_BYTES + B_STAGE_BYTES;
  static constexpr int SMEM = STAGES * STAGE_BYTES;
  static constexpr bool CC = AC || BC;
  static_assert(TM % 8 == 0 && TN % 8 == 0, "warp tile must be a multiple of 8");
};

template <bool AC, bool BC, bool CONJA, bool AK, bool BK, int BM, int BN, int WM, int WN, int STAGES>
__global__ void __launch_bounds__(WM* WN * 32)
    gemm_f64_kernel(GemmDesc d) {
  using C_ = Cfg<AC, BC, CONJA, AK, BK, BM, BN, WM, WN, STAGES>;
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp / WN, wn = warp % WN;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const long bz = blockIdx.z;
  if (d.mask && !d.mask[bz]) return;  // the whole CTA: batches left out by the mask
  if (d.upper_only && m0 >= n0 + BN) return;  // every row of the tile is below every column

  const unsigned char* Ab = (const unsigned char*)d.A + bz * d.sAb * C_::A_ESZ;
  const unsigned char* Bb = (const unsigned char*)d.B + bz * d.sBb * C_::B_ESZ;

  const int Keff = d.b_upper && n0 + BN < d.K ? n0 + BN : d.K;  // B[k][n] = 0 for k > n
  const int KT = (Keff + BKT - 1) / BKT;

  auto load_stage = [&](int stage, int kt) {
    unsigned char* As = smem + stage * C_::STAGE_BYTES;
    unsigned char* Bs = As + C_::A_STAGE_BYTES;
    const int k0 = kt * BKT;
    // A tile
    for (int e = tid; e < BM * BKT; e += C_::THREADS) {
      int r = e / C_::A_INNER, c = e % C_::A_INNER;  // r: row of the smem tile, c: contiguous
      int m = AK ? r : c, k = AK ? c : r;
      int gm = m0 + m, gk = k0 + k;
      bool ok = (gm < d.M) && (gk < d.K) && (kt < KT);
      const unsigned char* src = ok ? Ab + ((long)gm * d.sAm + (long)gk * d.sAk) * C_::A_ESZ : Ab;
      unsigned char* dst = As + (r * C_::A_PITCH + c) * C_::A_ESZ;
      if (AC) cp_async16(dst, src, ok); else cp_async8(dst, src, ok);
    }
    // B tile
    for (int e = tid; e < BN * BKT; e += C_::THREADS) {
      int r = e / C_::B_INNER, c = e % C_::B_INNER;
      int n = BK ? r : c, k = BK ? c : r;
      int gn = n0 + n, gk = k0 + k;
      bool ok = (gn < d.N) && (gk < d.K) && (kt < KT);
      const unsigned char* src = ok ? Bb + ((long)gk * d.sBk + (long)gn * d.sBn) * C_::B_ESZ : Bb;
      unsigned char* dst = Bs + (r * C_::B_PITCH + c) * C_::B_ESZ;
      if (BC) cp_async16(dst, src, ok); else cp_async8(dst, src, ok);
    }
  };

  double accr[C_::FM][C_::FN][2];
  double acci[C_::CC ? C_::FM : 1][C_::CC ? C_::FN : 1][2];
#pragma unroll
  for (int i = 0; i < C_::FM; ++i)
#pragma unroll
    for (int j = 0; j < C_::FN; ++j) {
      accr[i][j][0] = accr[i][j][1] = 0.0;
      if (C_::CC) acci[i][j][0] = acci[i][j][1] = 0.0;
    }

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    load_stage(s, s);
    cp_commit();
  }

  const int lr = lane >> 2, lc = lane & 3;
  for (int kt = 0; kt < KT; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    load_stage((kt + STAGES - 1) % STAGES, kt + STAGES - 1);
    cp_commit();

    const unsigned char* As = smem + (kt % STAGES) * C_::STAGE_BYTES;
    const unsigned char* Bs = As + C_::A_STAGE_BYTES;
#pragma unroll
    for (int kk = 0; kk < BKT; kk += 4) {
      double ar[C_::FM], ai[C_::FM], br[C_::FN], bi[C_::FN];
#pragma unroll
      for (int i = 0; i < C_::FM; ++i) {
        int m = wm * C_::TM + i * 8 + lr, k = kk + lc;
        int idx = AK ? (m * C_::A_PITCH + k) : (k * C_::A_PITCH + m);
        if (AC) {
          double2 v = reinterpret_cast<const double2*>(As)[idx];
          ar[i] = v.x;
          ai[i] = CONJA ? -v.y : v.y;
        } else {
          ar[i] = reinterpret_cast<const double*>(As)[idx];
          ai[i] = 0.0;
        }
      }
#pragma unroll
      for (int j = 0; j < C_::FN; ++j) {
        int n = wn * C_::TN + j * 8 + lr, k = kk + lc;
        int idx = BK ? (n * C_::B_PITCH + k) : (k * C_::B_PITCH + n);
        if (BC) {
          double2 v = reinterpret_cast<const double2*>(Bs)[idx];
          br[j] = v.x;
          bi[j] = v.y;
        } else {
          br[j] = reinterpret_cast<const double*>(Bs)[idx];
          bi[j] = 0.0;
        }
      }
#pragma unroll
      for (int i = 0; i < C_::FM; ++i) {
        double nai = -ai[i];
#pragma unroll
        for (int j = 0; j < C_::FN; ++j) {
          if (AC && BC) {
            dmma(accr[i][j][0], accr[i][j][1], ar[i], br[j]);
            dmma(accr[i][j][0], accr[i][j][1], nai, bi[j]);
            dmma(acci[i][j][0], acci[i][j][1], ar[i], bi[j]);
            dmma(acci[i][j][0], acci[i][j][1], ai[i], br[j]);
          } else if (AC) {
            dmma(accr[i][j][0], accr[i][j][1], ar[i], br[j]);
            dmma(acci[i][j][0], acci[i][j][1], ai[i], br[j]);
          } else if (BC) {
            dmma(accr[i][j][0], accr[i][j][1], ar[i], br[j]);
            dmma(acci[i][j][0], acci[i][j][1], ar[i], bi[j]);
          } else {
            dmma(accr[i][j][0], accr[i][j][1], ar[i], br[j]);
          }
        }
      }
    }
  }
  cp_wait<0>();

  // epilogue
  unsigned char* Cb = (unsigned char*)d.C + bz * d.sCb * (C_::CC ? 16 : 8);
  unsigned char* Sb = d.S ? (unsigned char*)d.S + bz * d.sCb * (C_::CC ? 16 : 8) : nullptr;
  const bool use_beta = (d.beta.x != 0.0) || (d.beta.y != 0.0);
#pragma unroll
  for (int i = 0; i < C_::FM; ++i) {
    int gm = m0 + wm * C_::TM + i * 8 + lr;
    if (gm >= d.M) continue;
#pragma unroll
    for (int j = 0; j < C_::FN; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int gn = n0 + wn * C_::TN + j * 8 + 2 * lc + h;
        if (gn >= d.N) continue;
        long off = (long)gm * d.sCm + (long)gn * d.sCn;
        if (C_::CC) {
          cplx acc = mk(accr[i][j][h], acci[i][j][h]);
          cplx v = cmul(d.alpha, acc);
          cplx* cp = reinterpret_cast<cplx*>(Cb) + off;
          if (use_beta) v = cadd(v, cmul(d.beta, *cp));
          *cp = v;
          if (Sb) {
            cplx* sp = reinterpret_cast<cplx*>(Sb) + off;
            cplx a2 = cmul(d.alpha, acc);
            *sp = cadd(*sp, a2);
          }
        } else {
          double v = d.alpha.x * accr[i][j][h];
          double* cp = reinterpret_cast<double*>(Cb) + off;
          if (use_beta) v += d.beta.x * (*cp);
          *cp = v;
          if (Sb) reinterpret_cast<double*>(Sb)[off] += d.alpha.x * accr[i][j][h];
        }
      }
    }
  }
}

}  // namespace gemm_detail
}  // namespace sfq
