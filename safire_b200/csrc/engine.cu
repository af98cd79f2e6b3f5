// The resident AFQMC engine: one system's Hamiltonian tensors, trial, walker set, propagator
// state and scratch, all in device memory on one GPU, driven on one CUDA stream.
//
// It plays the role of the objects execute_simulation builds (src/AFQMC/execute.cpp:107-206):
// Real3IndexFactorization (HamOps), NOMSD with ndet = 1 (trial), WalkerSet and
// AFQMCBasePropagator, for CLOSED walkers, and in FP64 for COLLINEAR walkers.
//
// A COLLINEAR walker is kept as one (M, nup + ndn) matrix, the up columns first, against the
// stacked trial [PsiT_up; PsiT_dn]: propagation, vHS, P1 and the half-rotated Lnak / haj are those
// of one N = nup + ndn matrix (the Hamiltonian is spin-independent), vbias sums both spins' rows.
// What is per spin -- the overlap matrix and its inverse and log det, the CholeskyQR Gram matrix,
// the exchange pairs -- keeps only the two diagonal spin blocks, which gives exactly the per-spin
// factorizations (with the pivots LAPACK would choose per spin) and the sum of the two log dets.
//
// A NONCOLLINEAR walker is one (2M, N) spinor matrix, the reference's layout, against PsiT (N, 2M):
// overlaps, G, vbias, the energy and the QR are those of a walker with Mr = 2M rows; P1 and vHS act
// on each component (the Hamiltonian is polarization-independent), and Lnak / haj are half-rotated
// per component.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "mixed.cuh"
#include "ops.cuh"
#include "umma_gemm.cuh"
#include "islice.cuh"

struct sfq_engine_s;

namespace sfq {

namespace {

constexpr int kNumProps = kWalkerProps;  // WEIGHT, PHASE, PSEUDO_ELOC_, E1_, EXX_, EJ_, OVLP, THETA
enum { P_WEIGHT = 0, P_PHASE, P_PSEUDO, P_E1, P_EXX, P_EJ, P_OVLP, P_THETA };
constexpr long kEnergyChunkElems = 1L << 27;

// weighted sums for the averages: out[0..1] = sum w e^{dt eloc}, out[2..3] = sum w,
// out[4..9] = sum w*E1, w*EXX, w*EJ (from E3 if given, else from the walker columns)
__global__ void averages_kernel(const cplx* props, int nwalk, double dt, const cplx* E3, double* out) {
  __shared__ double red[10][32];
  double acc[10];
  for (int i = 0; i < 10; ++i) acc[i] = 0.0;
  const cplx* w = props + (long)P_WEIGHT * nwalk;
  const cplx* el = props + (long)P_PSEUDO * nwalk;
  for (int i = threadIdx.x; i < nwalk; i += blockDim.x) {
    cplx wi = w[i];
    cplx ex = cexp_(cscale(el[i], dt));
    cplx a = cmul(wi, ex);
    acc[0] += a.x; acc[1] += a.y;
    acc[2] += wi.x; acc[3] += wi.y;
    cplx e1, e2, e3;
    if (E3) {
      e1 = E3[3 * i]; e2 = E3[3 * i + 1]; e3 = E3[3 * i + 2];
    } else {
      e1 = props[(long)P_E1 * nwalk + i]; e2 = props[(long)P_EXX * nwalk + i]; e3 = props[(long)P_EJ * nwalk + i];
    }
    cplx b1 = cmul(wi, e1), b2 = cmul(wi, e2), b3 = cmul(wi, e3);
    acc[4] += b1.x; acc[5] += b1.y; acc[6] += b2.x; acc[7] += b2.y; acc[8] += b3.x; acc[9] += b3.y;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < 10; ++k) {
    double v = acc[k];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < 10; ++k) {
      double s = 0.0;
      for (int i = 0; i < (int)(blockDim.x / 32); ++i) s += red[k][i];
      out[k] = s;
    }
  }
}

__global__ void seed_pseudo_kernel(cplx* props, const cplx* E3, const cplx* ov, int nwalk, int update_props) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwalk) return;
  if (update_props) {
    props[(long)P_E1 * nwalk + i] = E3[3 * i];
    props[(long)P_EXX * nwalk + i] = E3[3 * i + 1];
    props[(long)P_EJ * nwalk + i] = E3[3 * i + 2];
    props[(long)P_OVLP * nwalk + i] = ov[i];
  }
  if (update_props == 2) props[(long)P_PSEUDO * nwalk + i] = cadd(cadd(E3[3 * i], E3[3 * i + 1]), E3[3 * i + 2]);
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

// ---- the device-resident block driver's small kernels ------------------------------------
// Eshift += relax (log(Re(sum w e^{dt eloc} / sum w)) / dt - Eshift), from averages_kernel's sums
// (average_energy.hpp:37-48 and run_afqmc.cpp:91, on the device)
__global__ void eshift_relax_kernel(const double* red, double dt, double relax, double* eshift) {
  const double nr = red[0], ni = red[1], dr = red[2], di = red[3];
  const double re = (nr * dr + ni * di) / (dr * dr + di * di);
  const double pe = log(re) / dt;
  *eshift += relax * (pe - *eshift);
}
// MeasurementOutput (Measurements.hpp:96-142): the 10 numbers of sfq_engine_measure
__global__ void measure_kernel(const double* o, double* out) {
  const double d = o[2] * o[2] + o[3] * o[3];
  double r[6];
  for (int q = 0; q < 3; ++q) {
    const double ar = o[4 + 2 * q], ai = o[5 + 2 * q];
    r[2 * q] = (ar * o[2] + ai * o[3]) / d;
    r[2 * q + 1] = (ai * o[2] - ar * o[3]) / d;
  }
  out[0] = r[0] + r[2] + r[4];
  out[1] = r[1] + r[3] + r[5];
  for (int q = 0; q < 6; ++q) out[2 + q] = r[q];
  out[8] = o[2];
  out[9] = o[3];
}
__global__ void step_add_kernel(unsigned long long* step) { *step += 1ull; }
// back propagation in device-resident blocks: the history position lives in device memory (d_step[1])
__global__ void set_hist_kernel(unsigned long long* pos, unsigned long long v) { *pos = v; }
__global__ void hist_advance_kernel(unsigned long long* pos, int nhist) { *pos = (*pos + 1ull) % (unsigned long long)nhist; }
// storeFields into the ring slot pos % nbp: ring[w][slot][n] = X[w][n]
__global__ void store_fields_kernel(const cplx* X, cplx* ring, int nbp, int Nc, int W, const unsigned long long* pos) {
  const long slot = long(*pos % (unsigned long long)nbp);
  const long n = (long)W * Nc;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const long w = e / Nc, c = e % Nc;
    ring[(w * nbp + slot) * Nc + c] = X[e];
  }
}
__global__ void set_block_state_kernel(unsigned long long* step, unsigned long long s0, double* eshift, double e0) {
  *step = s0;
  *eshift = e0;
}
// a group member's block state from the group's input row: {step0, Eshift bits}
__global__ void load_block_state_kernel(const unsigned long long* in, unsigned long long* step, double* eshift) {
  *step = in[0];
  *eshift = __longlong_as_double((long long)in[1]);
}
// a group member's results into its output row: Eshift, population-control flag, product-timeout
// flag, then nm measurements of 10
__global__ void store_block_result_kernel(const double* eshift, const int* flag, const int* gerr, const double* meas,
                                          int nm, double* out) {
  if (threadIdx.x == 0) {
    out[0] = *eshift;
    out[1] = double(*flag);
    out[2] = gerr ? double(*gerr) : 0.0;
    out[3] = 0.0;
  }
  for (int i = threadIdx.x; i < 10 * nm; i += blockDim.x) out[4 + i] = meas[i];
}

// ---- multi-determinant NOMSD (NOMSD.cpp:184-216,238-331,466-512) ----------------------------
// Racc[w] (+)= wgt R[w], wsum[w] (+)= wgt with wgt = conj(ci) exp(ov[w] - lm[w]) (MixedDensityMatrix,
// ndet > 1: lm the walker's log overlap, which cancels in the ratio)
__global__ void md_accumulate_kernel(const cplx* R, const cplx* ov, const cplx* lm, cplx ci, cplx* Racc, cplx* wsum,
                                     long n, int first) {
  const long w = blockIdx.y;
  const cplx wg = cmul(cconj(ci), cexp_(csub(ov[w], lm[w])));
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const cplx v = cmul(wg, R[w * n + e]);
    Racc[w * n + e] = first ? v : cadd(Racc[w * n + e], v);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) wsum[w] = first ? wg : cadd(wsum[w], wg);
}
// the trial's own pair (q >= p): Racc += scl R, wsum += scl, scl = Re(conj(ci_q) ci_p exp(ov)) (vMF)
__global__ void md_pair_kernel(const cplx* R, const cplx* ov, cplx ciq, cplx cip, cplx* Racc, cplx* wsum, long n,
                               int first) {
  const double scl = cmul(cmul(cconj(ciq), cip), cexp_(ov[0])).x;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const cplx v = cscale(R[e], scl);
    Racc[e] = first ? v : cadd(Racc[e], v);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) wsum[0] = first ? mk(scl, 0.0) : cadd(wsum[0], mk(scl, 0.0));
}
__global__ void md_normalize_kernel(cplx* Racc, const cplx* wsum, long n) {
  const long w = blockIdx.y;
  const cplx s = wsum[w];
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    Racc[w * n + e] = cdiv(Racc[w * n + e], s);
}
// the position of the largest real part in a[d * W + w] over d, the first one on ties (max_element)
__device__ __forceinline__ int md_argmax(const cplx* a, int ndet, int W, int w) {
  int best = 0;
  for (int d = 1; d < ndet; ++d)
    if (a[(long)d * W + w].x > a[(long)best * W + w].x) best = d;
  return best;
}
// Log_Overlap, ndet > 1 (NOMSD.cpp:301-331): a_d = ov_d + log(conj ci_d); out = a_m + log sum exp(a_d - a_m)
__global__ void md_logsum_kernel(const cplx* ov, const cplx* lci, int ndet, int W, cplx* out) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  int m = 0;
  double best = 0.0;
  for (int d = 0; d < ndet; ++d) {
    const double r = ov[(long)d * W + w].x + lci[d].x;
    if (d == 0 || r > best) { best = r; m = d; }
  }
  const cplx am = cadd(ov[(long)m * W + w], lci[m]);
  cplx s = mk(0.0, 0.0);
  for (int d = 0; d < ndet; ++d) s = cadd(s, cexp_(csub(cadd(ov[(long)d * W + w], lci[d]), am)));
  out[w] = cadd(am, clog_(s));
}
// Energy, ndet > 1 (NOMSD.cpp:184-215): E = sum conj(ci_d) E_d exp(ov_d - ov_m) / deno, Ov = log deno + ov_m
__global__ void md_energy_kernel(const cplx* ov, const cplx* Ed, const cplx* cic, int ndet, int W, cplx* E3,
                                 cplx* Ov) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const int m = md_argmax(ov, ndet, W, w);
  const cplx om = ov[(long)m * W + w];
  cplx deno = mk(0.0, 0.0), s0 = mk(0.0, 0.0), s1 = mk(0.0, 0.0), s2 = mk(0.0, 0.0);
  for (int d = 0; d < ndet; ++d) {
    const cplx e = cmul(cic[d], cexp_(csub(ov[(long)d * W + w], om)));
    const cplx* E = Ed + ((long)d * W + w) * 3;
    s0 = cadd(s0, cmul(e, E[0]));
    s1 = cadd(s1, cmul(e, E[1]));
    s2 = cadd(s2, cmul(e, E[2]));
    deno = cadd(deno, e);
  }
  E3[3 * w] = cdiv(s0, deno);
  E3[3 * w + 1] = cdiv(s1, deno);
  E3[3 * w + 2] = cdiv(s2, deno);
  Ov[w] = cadd(clog_(deno), om);
}

// ---- back propagation (AFQMCBasePropagator.cpp:404-526, BackPropEstimator.hpp:170-230) -----
// refs[d][w] = PsiT_d^H for every walker (the references BackPropagate starts from)
__global__ void bp_init_refs_kernel(const cplx* PsiT, int ndet, int W, int Mr, int N, cplx* refs) {
  const long per = (long)Mr * N, total = (long)ndet * W * per;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long d = e / (W * per), r = e % per;
    const long i = r / N, a = r % N;
    refs[e] = cconj(PsiT[d * per + a * Mr + i]);
  }
}
// V[w] <- -V[w]^H in place: exp(i (-V^H)) = exp(-i V^H), the adjoint Taylor propagator (propagate.hpp:56-57)
// time-evolved back propagation helpers: X[b] = I (R x R) for every matrix b; out = conj(in)
// dst[c][r] = src[r * cols + c0 + c] for r < rows, c < nc: a block of columns of a row-major matrix,
// transposed through 32 x 32 shared-memory tiles
__global__ void transpose_cols_kernel(const double* src, long rows, long cols, long c0, int nc, double* dst) {
  __shared__ double tile[32][33];
  const long r0 = (long)blockIdx.x * 32;
  const int cb = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const long r = r0 + y;
    const int c = cb + threadIdx.x;
    tile[y][threadIdx.x] = (r < rows && c < nc) ? src[r * cols + c0 + c] : 0.0;
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = cb + y;
    const long r = r0 + threadIdx.x;
    if (c < nc && r < rows) dst[(long)c * rows + r] = tile[threadIdx.x][y];
  }
}

__global__ void set_identity_batched_kernel(cplx* X, long nmat, int R) {
  const long n = nmat * R * R;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const long k = e % ((long)R * R);
    X[e] = mk(k / R == k % R ? 1.0 : 0.0, 0.0);
  }
}
__global__ void conj_copy_kernel(const cplx* in, cplx* out, long n) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    out[e] = cconj(in[e]);
}
// V[w] <- V[w]^H (M x M, in place)
__global__ void adjoint_kernel(cplx* V, int M) {
  cplx* Vw = V + (long)blockIdx.y * M * M;
  const long npairs = (long)M * (M + 1) / 2;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < npairs; e += (long)gridDim.x * blockDim.x) {
    int i = int((sqrt(8.0 * e + 1.0) - 1.0) / 2.0);
    while ((long)i * (i + 1) / 2 > e) --i;
    while ((long)(i + 1) * (i + 2) / 2 <= e) ++i;
    const int j = int(e - (long)i * (i + 1) / 2);  // j <= i
    const cplx a = Vw[(long)i * M + j], b = Vw[(long)j * M + i];
    Vw[(long)i * M + j] = cconj(b);
    Vw[(long)j * M + i] = cconj(a);
  }
}

__global__ void neg_adjoint_kernel(cplx* V, int M) {
  cplx* Vw = V + (long)blockIdx.y * M * M;
  const long npairs = (long)M * (M + 1) / 2;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < npairs; e += (long)gridDim.x * blockDim.x) {
    int i = int((sqrt(8.0 * e + 1.0) - 1.0) / 2.0);
    while ((long)i * (i + 1) / 2 > e) --i;
    while ((long)(i + 1) * (i + 2) / 2 <= e) ++i;
    const int j = int(e - (long)i * (i + 1) / 2);  // j <= i
    const cplx a = Vw[(long)i * M + j], b = Vw[(long)j * M + i];
    Vw[(long)i * M + j] = mk(-b.x, b.y);
    Vw[(long)j * M + i] = mk(-a.x, a.y);
  }
}
// logdetR[d][w] -= mean over d (BackPropEstimator.hpp:183-186)
__global__ void bp_shift_kernel(cplx* ld, int ndet, int W) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  cplx s = mk(0.0, 0.0);
  for (int d = 0; d < ndet; ++d) s = cadd(s, ld[(long)d * W + w]);
  s = cscale(s, 1.0 / ndet);
  for (int d = 0; d < ndet; ++d) ld[(long)d * W + w] = csub(ld[(long)d * W + w], s);
}
// wt[w] *= wfac[w * stride]: one step of path restoration (BackPropEstimator.hpp:192-206)
__global__ void bp_restore_kernel(cplx* wt, const cplx* wfac, long stride, int W) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w < W) wt[w] = cmul(wt[w], wfac[(long)w * stride]);
}
// ov[w] = f ov[w] + conj(f ld[w]) (constructBPMeasurementInputs: CLOSED doubles both)
__global__ void bp_ov_kernel(cplx* ov, const cplx* ld, double f, int W) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w < W) ov[w] = cadd(cscale(ov[w], f), cconj(cscale(ld[w], f)));
}

// ---- TwoRDM, SpinCorr, PairCorr observables (Observables/twordm.hpp, spincorr.hpp, paircorr.hpp) ----
// XwG[w][s][x] = wc[w] Gf[w][s][x]
__global__ void scale_walker_rows_kernel(const cplx* Gf, const cplx* wc, long per_walker, int W, cplx* out) {
  const long n = per_walker * W;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    out[e] = cmul(wc[e / per_walker], Gf[e]);
}
// avg[i][k][j][l] += C[(i,k)][(j,l)] - [same spin] C[(i,l)][(j,k)], C = sum_w XwG_s[w] (x) G_s'[w]
// (twordm.hpp:57-71: (ikjl) = G_ik G_jl - G_il G_jk for one spin, G_ik G_jl across the spins)
__global__ void twordm_block_kernel(const cplx* C, int M, int same, cplx* avg) {
  const long MM = (long)M * M, n = MM * MM;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const long x = e / MM, y = e % MM;  // x = (i, k), y = (j, l)
    cplx v = C[e];
    if (same) {
      const long i = x / M, k = x % M, j = y / M, l = y % M;
      v = csub(v, C[(i * M + l) * MM + j * M + k]);
    }
    avg[e] = cadd(avg[e], v);
  }
}
// <S_i . S_j> for i <= j in the order i-major (spincorr.hpp:58-124): out[0] the XY channel, out[1] Z.
// kind 0 CLOSED (one block), 1 COLLINEAR (up, down blocks of M x M), 2 NONCOLLINEAR (one 2M x 2M block)
__global__ void spincorr_kernel(const cplx* Gf, const cplx* wc, int W, int M, int kind, cplx* out) {
  const int i = blockIdx.y, j = i + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const long P = (long)M * (M + 1) / 2;
  const long idx = (long)i * M - (long)i * (i - 1) / 2 + (j - i);
  const int R = kind == 2 ? 2 * M : M;
  const long blk = (long)R * R;
  const int ns = kind == 1 ? 2 : 1;
  cplx xy = mk(0.0, 0.0), z = mk(0.0, 0.0);
  const cplx one = mk(1.0, 0.0);
  for (int w = 0; w < W; ++w) {
    const cplx* G = Gf + (long)w * ns * blk;
    auto g = [&](int s, int a, int b) { return G[s * blk + (long)a * R + b]; };
    cplx cz, cxy;
    if (kind != 2) {
      const int d = kind == 1 ? 1 : 0;  // CLOSED: the down block is the up block
      if (j == i) {
        cz = cadd(cmul(g(0, i, i), csub(one, g(d, j, j))), cmul(g(d, i, i), csub(one, g(0, j, j))));
        cxy = cadd(cmul(g(0, i, j), csub(one, g(d, j, i))), cmul(g(d, i, j), csub(one, g(0, j, i))));
      } else {
        cz = csub(csub(cadd(cmul(g(0, i, i), csub(g(0, j, j), g(d, j, j))), cmul(g(d, i, i), csub(g(d, j, j), g(0, j, j)))),
                       cmul(g(0, i, j), g(0, j, i))),
                  cmul(g(d, i, j), g(d, j, i)));
        cxy = cadd(cmul(g(0, i, j), cscale(g(d, j, i), -1.0)), cmul(g(d, i, j), cscale(g(0, j, i), -1.0)));
      }
    } else {
      const int I = i + M, J = j + M;
      if (j == i) {
        cz = cadd(cadd(cmul(g(0, i, i), csub(one, g(0, J, J))), cmul(g(0, I, I), csub(one, g(0, j, j)))),
                  cadd(cmul(g(0, i, J), g(0, J, i)), cmul(g(0, I, j), g(0, j, I))));
        cxy = cadd(cadd(cmul(g(0, i, j), csub(one, g(0, J, I))), cmul(g(0, I, J), csub(one, g(0, j, i)))),
                   cadd(cmul(g(0, J, j), g(0, i, I)), cmul(g(0, j, J), g(0, I, i))));
      } else {
        cz = cadd(cmul(g(0, i, i), csub(g(0, j, j), g(0, J, J))), cmul(g(0, I, I), csub(g(0, J, J), g(0, j, j))));
        cz = csub(cz, cmul(g(0, i, j), g(0, j, i)));
        cz = csub(cz, cmul(g(0, I, J), g(0, J, I)));
        cz = cadd(cz, cmul(g(0, i, J), g(0, J, i)));
        cz = cadd(cz, cmul(g(0, I, j), g(0, j, I)));
        cxy = cadd(cmul(g(0, i, j), cscale(g(0, J, I), -1.0)), cmul(g(0, I, J), cscale(g(0, j, i), -1.0)));
        cxy = cadd(cxy, cadd(cmul(g(0, J, j), g(0, i, I)), cmul(g(0, j, J), g(0, I, i))));
      }
    }
    z = cadd(z, cmul(wc[w], cscale(cz, 0.25)));
    xy = cadd(xy, cmul(wc[w], cscale(cxy, 0.5)));
  }
  out[idx] = cadd(out[idx], xy);
  out[P + idx] = cadd(out[P + idx], z);
}
// P_ab(i, j) for the pair maps a, b (paircorr.hpp:80-135): kind 1 COLLINEAR (j > i), 2 NONCOLLINEAR
// (every j); maps (npair, M), a negative partner leaves the entry out; out (npair, npair, M, M)
__global__ void paircorr_kernel(const cplx* Gf, const cplx* wc, int W, int M, int kind, int npair, const int* maps,
                                cplx* out) {
  const long n = (long)npair * npair * M * M;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const int j = int(e % M), i = int((e / M) % M);
    const int b = int((e / ((long)M * M)) % npair), a = int(e / ((long)M * M * npair));
    if (kind == 1 && j <= i) continue;
    const int ib = maps[(long)a * M + i], jb = maps[(long)b * M + j];
    if (ib < 0 || jb < 0) continue;
    const int R = kind == 2 ? 2 * M : M;
    const long blk = (long)R * R;
    const int ns = kind == 1 ? 2 : 1;
    cplx acc = mk(0.0, 0.0);
    for (int w = 0; w < W; ++w) {
      const cplx* G = Gf + (long)w * ns * blk;
      auto g = [&](int s, int x, int y) { return G[s * blk + (long)x * R + y]; };
      cplx c;
      if (kind == 1) {
        c = cadd(cadd(cmul(g(0, i, j), g(1, ib, jb)), cmul(g(0, i, jb), g(1, ib, j))),
                 cadd(cmul(g(1, i, jb), g(0, ib, j)), cmul(g(1, i, j), g(0, ib, jb))));
      } else {
        c = csub(cmul(g(0, i, j), g(0, M + ib, M + jb)), cmul(g(0, i, M + jb), g(0, M + ib, j)));
        c = cadd(c, csub(cmul(g(0, i, jb), g(0, M + ib, M + j)), cmul(g(0, i, M + j), g(0, M + ib, jb))));
        c = cadd(c, csub(cmul(g(0, M + i, M + jb), g(0, ib, j)), cmul(g(0, M + i, j), g(0, ib, M + jb))));
        c = cadd(c, csub(cmul(g(0, M + i, M + j), g(0, ib, jb)), cmul(g(0, M + i, jb), g(0, ib, M + j))));
      }
      acc = cadd(acc, cmul(wc[w], cscale(c, 0.5)));
    }
    out[e] = cadd(out[e], acc);
  }
}

// ---- the mixed estimator's RDMs (MixedEstimator.hpp:37-147) ---------------------------------
// tot[w] = sum_d conj(ci_d) exp(ov_d[w] - shift[w]) over the reference determinants
__global__ void rdm_tot_kernel(const cplx* ov, const cplx* cic, const cplx* shift, int ndet, int W, cplx* tot) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  cplx s = mk(0.0, 0.0);
  const cplx sh = shift ? shift[w] : mk(0.0, 0.0);
  for (int d = 0; d < ndet; ++d) s = cadd(s, cmul(cic[d], cexp_(csub(ov[(long)d * W + w], sh))));
  tot[w] = s;
}
// wc[w] = weight[w] conj(ci_d) exp(ov_d[w] - shift[w]) / tot[w]
__global__ void rdm_coeff_kernel(const cplx* ov, cplx cic, const cplx* shift, const cplx* tot, const cplx* weight,
                                 int W, cplx* wc) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const cplx sh = shift ? shift[w] : mk(0.0, 0.0);
  wc[w] = cmul(weight[w], cdiv(cmul(cic, cexp_(csub(ov[w], sh))), tot[w]));
}
// diagonal two-body RDM blocks (Observables/diagonal_twordm.hpp:60-80), avg[b][i][j] += sum_w wc[w] (...):
// b = 2 s: G[s,i,i] G[s,j,j] - G[s,i,j] G[s,j,i] for each spin s; b = 1 (CLOSED, COLLINEAR):
// G[0,i,i] G[dn,j,j], dn the down block (CLOSED: the same)
__global__ void rdm_two_kernel(const cplx* Gf, const cplx* wc, int W, int nspin, int Mr, int nblk, cplx* avg) {
  const long MM = (long)Mr * Mr;
  const long total = nblk * MM;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int b = int(e / MM);
    const int i = int((e % MM) / Mr), j = int(e % Mr);
    cplx acc = mk(0.0, 0.0);
    for (int w = 0; w < W; ++w) {
      const cplx* Gw = Gf + (long)w * nspin * MM;
      cplx v;
      if (b == 1 && nblk > 1) {
        const cplx* Gd = Gw + (nspin == 2 ? MM : 0);
        v = cmul(Gw[(long)i * Mr + i], Gd[(long)j * Mr + j]);
      } else {
        const cplx* Gs = Gw + (long)(b / 2) * MM;
        v = csub(cmul(Gs[(long)i * Mr + i], Gs[(long)j * Mr + j]), cmul(Gs[(long)i * Mr + j], Gs[(long)j * Mr + i]));
      }
      acc = cadd(acc, cmul(wc[w], v));
    }
    avg[e] = cadd(avg[e], acc);
  }
}

}  // namespace

struct Engine {
  sfq_engine_params_t p{};
  int M = 0, N = 0, Nc = 0, W = 0;
  bool trial_real = true;
  // COLLINEAR walkers: N = nup + ndn columns, up first (CLOSED: collinear false, N = nup);
  // NONCOLLINEAR walkers: npol = 2, Mr = 2M rows (CLOSED, COLLINEAR: npol = 1, Mr = M)
  bool collinear = false;
  int nup = 0;
  int npol = 1, Mr = 0;
  bool closed() const { return !collinear && npol == 1; }
  // multi-determinant NOMSD trial (ndet > 1, FP64): PsiT, PsiTr, Lnak and haj hold the ndet
  // determinants one after the other (the names point at determinant 0); ci on the host
  int ndet = 1;
  std::vector<cplx> ci_h;
  cplx* md_ov = nullptr;   // (ndet, W) per-determinant log overlaps, without the ci terms
  cplx* md_E = nullptr;    // (ndet, W, 3) per-determinant local energies
  cplx* md_lci = nullptr;  // (ndet) log(conj ci), 1e-12 for a vanishing ci (NOMSD.cpp:312)
  cplx* md_cic = nullptr;  // (ndet) conj ci
  cplx* Rd = nullptr;      // (W, M, M) one determinant's full G summed over the spin / polarization blocks
  cplx* Racc = nullptr;    // (W, M, M) their ci-weighted mixture
  cplx* wsum = nullptr;    // (W) the mixture's weights
  long det_elems() const { return (long)N * Mr; }
  size_t lnak_esz() const { return trial_real ? sizeof(double) : sizeof(cplx); }
  // the exchange's spin split (and the CLOSED marker -1); a NONCOLLINEAR walker is one sector
  int spin_split() const { return collinear ? nup : (npol == 2 ? N : -1); }
  double ov_scale() const { return closed() ? 2.0 : 1.0; }  // NOMSD.cpp:285-290: CLOSED counts its determinant twice
  double vb_scale() const { return (closed() ? 2.0 : 1.0) * std::sqrt(p.dt); }  // Real3IndexFactorization.hpp:349
  cudaStream_t st = nullptr;
  // host-buffer steps: the field uniforms go in on a copy stream while the step's density and force
  // bias run; the fields kernel waits for uni_wait (cleared once waited on)
  cudaStream_t cst = nullptr;
  cudaEvent_t uni_ready = nullptr, uni_free = nullptr, uni_wait = nullptr;
  // arena
  unsigned char* arena = nullptr;
  size_t arena_bytes = 0;
  // Hamiltonian / trial
  double* hcore = nullptr;
  double* Likn = nullptr;
  cplx* PsiT = nullptr;
  double* PsiTr = nullptr;
  void* Lnak = nullptr;
  cplx* haj = nullptr;
  double* v0 = nullptr;
  double* vmf = nullptr;
  double* P1 = nullptr;
  double* H1m = nullptr;    // -1/2 herm(H1): P1 = exp(H1m)
  double* P1inv = nullptr;  // exp(-H1m), built when the time-evolved back propagation is enabled
  // walkers
  cplx* SM = nullptr;
  cplx* props = nullptr;
  // scratch
  cplx *SM2 = nullptr, *T = nullptr, *G = nullptr, *X = nullptr, *V = nullptr;
  cplx *TMN = nullptr, *T1 = nullptr, *T2 = nullptr;
  cplx *hw = nullptr, *mf = nullptr, *newov = nullptr, *E3 = nullptr, *ovtmp = nullptr;
  cplx *Tchunk = nullptr, *exxn = nullptr, *kl = nullptr;
  long tchunk_elems = 0;
  int* status = nullptr;
  double* red = nullptr;       // 16 doubles
  double* uni = nullptr;       // (W, Nc) staging for injected uniforms
  unsigned long long* stats = nullptr;  // 5 counters
  PopWork pw{};
  // mixed precision: split-BF16 planes and fp32 accumulators
  bool mixed = false;
  // symmetric Cholesky vectors (checked bit for bit at setup): vHS comes from the packed upper
  // triangle, P = M(M+1)/2 columns instead of M*M, and is mirrored afterwards
  bool sym = false;
  long P = 0;
  double* Lp = nullptr;  // (P, Nc), FP64 engines
  cplx* Vp = nullptr;    // (W, P), FP64 engines
  // T holds the inverse overlap matrices (PsiT W)^-1 of the current walkers and inv_ov their log
  // overlaps whenever inv_cached is set: the log overlap taken after a propagation or an
  // orthogonalization factors exactly the matrix the next Green's function needs, so that step
  // reuses it (same GEMM, same pivots, bit-identical G).  Every change to SM clears the flag.
  bool inv_cached = false;
  const cplx* inv_ov = nullptr;
  int nplanes = 3;  // bf16 planes per operand (2: ~16-bit products, 3: FP32-class)
  void* Likn_p[3] = {};
  void* Lnak_p[3] = {};
  void* P1_p[3] = {};
  void* Gs_p[3] = {};
  void* Xs_p[3] = {};
  void* Vb_p[3] = {};
  void* Wt_p[3] = {};
  void* Wt2_p[3] = {};  // second walker-operand buffer: a product's epilogue writes the next A here
  void* Tb_p[3] = {};   // block operand [[Tr, -Ti], [Ti, Tr]] of the inverse overlaps, (W, 2N, 2N)
  void* Ws_p[3] = {};   // the walkers read as reals, (W, M, 2N): the other operand of G
  float *Cvb = nullptr, *Cv = nullptr, *Sacc = nullptr;
  int vb_ks = 1;        // K splits of the vbias product (partial sums, reduced in a fixed order)
  int vb_ks_max = 1;    // the most any vbias tile width can take (the partial-sum buffer's size)
  // tile widths of the products (0: the built-in choice), set by autotune() or set_tiles()
  int vb_bn = 128, vhs_bn = 0, p1_bn = 0, g_bn = 0;
  int vb_ks_req = 0;  // a force-bias K split asked for (0: planned from the tile width)
  int tay_half = 0;     // orbitals per Taylor tile (tile width 2 * tay_half, re and im halves)
  int tay_req = 0;      // a Taylor tile asked for (0: the least padding)
  long vb_rows = 0;     // output columns of a Taylor product: ceil(M / tay_half) * 2 * tay_half
  int ldh = 0;          // padded half of the walker operand rows (re, im): M rounded up to 64
  int* gemm_err = nullptr;
  // exact-accumulation mode (nslices > 0): int8 fixed-point slices of every tensor-core operand, one
  // exponent per row (islice.cuh); rows of the walker-shaped arrays are r = (w npol + q) N + a (the
  // spinor components q of a NONCOLLINEAR walker are two (M, N) blocks that V and P1 act on alike),
  // and k runs over the Mr = npol M rows of the G-shaped arrays
  int nslices = 0;
  long ld_m = 0, ld_mr = 0, ld_nm = 0, ld_nc = 0;  // slice row strides (bytes): M, Mr, N*Mr, Nc rounded up to 64
  int8_t* Lv_q[3] = {};  int* Lv_e = nullptr;   // Lnak, rows n over (a, k): the force bias's B
  int8_t* Le_q[3] = {};  int* Le_e = nullptr;   // Lnak, rows (n, a) over k: the exchange tensor's B (per determinant)
  // multi-determinant trials: the force bias contracts the ci-weighted full G (M x M) with L
  int8_t* Lf_q[3] = {};  int* Lf_e = nullptr;   // L, rows n over (i, k)
  int8_t* Gf_q[3] = {};  int* Gf_e = nullptr;   // full G minus the trial's, planar rows (c, w) over (i, k)
  cplx* RT_md = nullptr;                         // the trial's ci-weighted full G (M x M), FP64
  long ld_mm = 0;
  int i8_md_ks = 1;                              // K splits of that product (exact int32 per range)
  int8_t* Lh_q[3] = {};  int* Lh_e = nullptr;   // L, rows (i, k) (packed pairs when symmetric) over n: vHS's B
  int8_t* P1_q[3] = {};  int* P1_e = nullptr;   // P1, rows j over i
  int8_t* Gv_q[3] = {};  int* Gv_e = nullptr;   // G, planar rows (c, w) over (a, k)
  int8_t* Ge_q[3] = {};  int* Ge_e = nullptr;   // G, planar rows (c, w, a) over k
  int8_t* Xq_q[3] = {};  int* Xq_e = nullptr;   // fields, planar rows (c, w) over n
  int8_t* V_q[3] = {};   int* V_e = nullptr;  int* V_emax = nullptr;  // V[w][c][i][k]: Vr, Vi, -Vi; e per (w, i)
  int8_t* A_q[2][3] = {};  int* A_e[2] = {};  // walker operand: rows (c, r)
  unsigned long long* pl_emax = nullptr;  // 2W scratch row maxima for slicing G - G_T
  cplx* GT_c = nullptr;  // the trial's own G (N, Mr) and force bias (Nc), FP64
  cplx* vbT = nullptr;
  float* Cp = nullptr;  // FP32 output of the walker-shaped products, planar (2 W N, M)
  int i8_vb_bn = 160, i8_vb_ks = 1, i8_bn = 160, i8_half = 80, i8_half_req = 0;
  double* h_pinned = nullptr;  // pinned host staging for e2e calls
  size_t h_pinned_bytes = 0;
  // device-resident block driver: Eshift, the step counter and the block's measurements in device
  // memory; one CUDA graph per block schedule, replayed
  static constexpr int kMeasCap = 64;
  bool dev_mode = false;  // steps read the step and Eshift from d_step / d_eshift
  double* d_eshift = nullptr;
  unsigned long long* d_step = nullptr;
  double* d_meas = nullptr;  // kMeasCap x 10
  struct BlockGraph {
    cudaGraphExec_t exec = nullptr;
    bool inv_after = false;
    const cplx* inv_ov_after = nullptr;
    int nmeas = 0;
  };
  std::map<std::string, BlockGraph> graphs;
  // results of the last block, staged in pinned memory: Eshift, status flags, measurements
  double* blk_host = nullptr;  // 4 + 10 kMeasCap doubles
  cudaEvent_t blk_done = nullptr;
  int blk_nmeas = 0;

  // optional per-phase CUDA-event timing on the engine stream
  static constexpr int NPH = SFQ_NUM_PHASES;
  bool profile = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[NPH];
  std::vector<cudaEvent_t> pool;
  cudaEvent_t open_ev[NPH] = {};
  cudaEvent_t take_event() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  void ph_begin(int ph) {
    if (!profile) return;
    open_ev[ph] = take_event();
    cudaEventRecord(open_ev[ph], st);
  }
  void ph_end(int ph) {
    if (!profile || !open_ev[ph]) return;
    cudaEvent_t e = take_event();
    cudaEventRecord(e, st);
    ev[ph].push_back({open_ev[ph], e});
    open_ev[ph] = nullptr;
  }
  int phase_times(double* ms, int* counts, int n) {
    SFQ_CUDA_TRY(cudaStreamSynchronize(st));
    for (int ph = 0; ph < NPH; ++ph) {
      double acc = 0.0;
      for (auto& pr : ev[ph]) {
        float t = 0.f;
        SFQ_CUDA_TRY(cudaEventElapsedTime(&t, pr.first, pr.second));
        acc += t;
        pool.push_back(pr.first);
        pool.push_back(pr.second);
      }
      if (ph < n) {
        if (ms) ms[ph] = acc;
        if (counts) counts[ph] = int(ev[ph].size());
      }
      ev[ph].clear();
    }
    return SFQ_OK;
  }
  void release_events() {
    for (int ph = 0; ph < NPH; ++ph) {
      for (auto& pr : ev[ph]) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
      ev[ph].clear();
    }
    for (auto e : pool) cudaEventDestroy(e);
    pool.clear();
  }

  WalkerProps wprops() const {
    WalkerProps w;
    w.weight = props + (long)P_WEIGHT * W;
    w.phase = props + (long)P_PHASE * W;
    w.pseudo_eloc = props + (long)P_PSEUDO * W;
    w.e1 = props + (long)P_E1 * W;
    w.exx = props + (long)P_EXX * W;
    w.ej = props + (long)P_EJ * W;
    w.ovlp = props + (long)P_OVLP * W;
    w.theta = props + (long)P_THETA * W;
    return w;
  }
  const void* lnak_ptr() const { return Lnak; }
  double target_pop() const { return p.target_population > 0 ? p.target_population : W; }

  int allocate() {
    const size_t c = sizeof(cplx), d = sizeof(double);
    const long MN = (long)M * N, NN = (long)N * N, MM = (long)M * M;
    const long RN = (long)Mr * N;  // a walker's elements
    tchunk_elems = (long)W * N * ops::energy_chunk(W, N, Nc, kEnergyChunkElems) * N;
    struct Item { void** ptr; size_t bytes; };
    std::vector<Item> items = {
        {(void**)&hcore, d * MM},
        {(void**)&Likn, d * MM * Nc},
        {(void**)&PsiT, c * ndet * RN},
        {(void**)&PsiTr, d * ndet * RN},
        {(void**)&Lnak, (trial_real ? d : c) * (size_t)ndet * Nc * RN},
        {(void**)&haj, c * ndet * RN},
        {(void**)&v0, d * MM},
        {(void**)&vmf, d * Nc},
        {(void**)&P1, d * MM},
        {(void**)&SM, c * W * RN},
        {(void**)&props, c * kNumProps * W},
        {(void**)&SM2, c * W * RN},
        {(void**)&T, c * W * NN},
        {(void**)&G, c * W * RN},
        {(void**)&X, c * (size_t)W * Nc},
        {(void**)&V, c * W * MM},
        {(void**)&TMN, c * W * RN},
        {(void**)&T1, c * W * RN},
        {(void**)&T2, c * W * RN},
        {(void**)&hw, c * W},
        {(void**)&mf, c * W},
        {(void**)&newov, c * W},
        {(void**)&E3, c * 3 * W},
        {(void**)&ovtmp, c * W},
        {(void**)&Tchunk, c * tchunk_elems},
        {(void**)&exxn, c * (size_t)W * Nc},
        {(void**)&kl, c * (size_t)W * Nc},
        {(void**)&status, sizeof(int) * 2 * W},
        {(void**)&red, d * 16},
        {(void**)&uni, d * (size_t)W * Nc},
        {(void**)&stats, sizeof(unsigned long long) * 8},
        {(void**)&pw.offspring, sizeof(int) * W},
        {(void**)&pw.pairs, sizeof(int) * 2 * W},
        {(void**)&pw.npairs, sizeof(int) * 4},
        {(void**)&pw.cum, d * W},
        {(void**)&pw.flag, sizeof(int) * 4},
        {(void**)&d_eshift, sizeof(double) * 2},
        {(void**)&d_step, sizeof(unsigned long long) * 2},
        {(void**)&d_meas, sizeof(double) * 10 * kMeasCap},
    };
    if (ndet > 1) {
      std::vector<Item> md = {
          {(void**)&md_ov, c * ndet * W}, {(void**)&md_E, c * ndet * W * 3}, {(void**)&md_lci, c * ndet},
          {(void**)&md_cic, c * ndet},    {(void**)&Rd, c * W * MM},          {(void**)&Racc, c * W * MM},
          {(void**)&wsum, c * W},
      };
      items.insert(items.end(), md.begin(), md.end());
    }
    if (mixed && nslices) {
      plan_i8();
      const long R = (long)W * npol * N, RG = (long)W * N, vrows = sym ? P : MM;
      const bool md = ndet > 1;  // the force bias from the full G: no slices of Lnak over (a, k) nor of G
      const long lp = trial_real ? 1 : 2;  // a complex trial's Lnak: planar rows, real parts then imaginary
      std::vector<Item> mx;
      for (int q = 0; q < nslices; ++q) {
        mx.push_back({(void**)&Lv_q[q], md ? 0 : (size_t)lp * Nc * ld_nm});
        mx.push_back({(void**)&Le_q[q], (size_t)lp * ndet * Nc * N * ld_mr});
        if (md) {
          mx.push_back({(void**)&Lf_q[q], (size_t)Nc * ld_mm});
          mx.push_back({(void**)&Gf_q[q], (size_t)2 * W * ld_mm});
        }
        mx.push_back({(void**)&Lh_q[q], (size_t)vrows * ld_nc});
        mx.push_back({(void**)&P1_q[q], (size_t)M * ld_m});
        mx.push_back({(void**)&Gv_q[q], md ? 0 : (size_t)2 * W * ld_nm});
        mx.push_back({(void**)&Ge_q[q], (size_t)2 * RG * ld_mr});
        mx.push_back({(void**)&Xq_q[q], (size_t)2 * W * ld_nc});
        mx.push_back({(void**)&V_q[q], (size_t)W * 3 * M * ld_m});
        for (int b = 0; b < 2; ++b) mx.push_back({(void**)&A_q[b][q], (size_t)2 * R * ld_m});
      }
      const size_t ie = sizeof(int);
      std::vector<Item> mx2 = {
          {(void**)&Lv_e, ie * lp * Nc}, {(void**)&Le_e, ie * lp * ndet * Nc * N}, {(void**)&Lh_e, ie * vrows},
          {(void**)&P1_e, ie * M}, {(void**)&Gv_e, ie * 2 * W}, {(void**)&Ge_e, ie * 2 * RG},
          {(void**)&Xq_e, ie * 2 * W}, {(void**)&V_e, ie * W * M}, {(void**)&V_emax, ie * W * M},
          {(void**)&A_e[0], ie * R}, {(void**)&A_e[1], ie * R},
          {(void**)&GT_c, c * (size_t)N * Mr}, {(void**)&vbT, c * (size_t)Nc},
          {(void**)&pl_emax, sizeof(unsigned long long) * 2 * (size_t)W},
          {(void**)&Cvb, sizeof(float) * std::max(i8_vb_ks, i8_md_ks) * 2 * (size_t)W * Nc},
          {(void**)&Cv, sizeof(float) * 2 * W * vrows},
          {(void**)&Sacc, sizeof(float) * 2 * R * M},
          {(void**)&Cp, sizeof(float) * 2 * R * M},
          {(void**)&gemm_err, sizeof(int) * 4},
      };
      if (md) {
        std::vector<Item> mx3 = {{(void**)&Lf_e, ie * Nc}, {(void**)&Gf_e, ie * 2 * W}, {(void**)&RT_md, c * MM}};
        mx2.insert(mx2.end(), mx3.begin(), mx3.end());
      }
      items.insert(items.end(), mx.begin(), mx.end());
      items.insert(items.end(), mx2.begin(), mx2.end());
    } else if (mixed) {
      const size_t b = 2;  // bf16
      const long MN2 = 2L * M * N;
      plan_mixed();
      std::vector<Item> mx;
      for (int q = 0; q < nplanes; ++q) {
        mx.push_back({&Likn_p[q], b * MM * Nc});
        mx.push_back({&Lnak_p[q], b * (size_t)Nc * N * M});
        mx.push_back({&P1_p[q], b * MM});
        mx.push_back({&Gs_p[q], b * 2 * W * MN});
        mx.push_back({&Xs_p[q], b * 2 * (size_t)W * Nc});
        mx.push_back({&Vb_p[q], b * W * 2 * MM});
        mx.push_back({&Wt_p[q], b * W * 2L * N * ldh});
        mx.push_back({&Wt2_p[q], b * W * 2L * N * ldh});
        mx.push_back({&Tb_p[q], b * W * 4 * NN});
        mx.push_back({&Ws_p[q], b * W * 2 * MN});
      }
      std::vector<Item> mx2 = {
          {(void**)&Cvb, sizeof(float) * vb_ks_max * 2 * (size_t)W * Nc},
          {(void**)&Cv, sizeof(float) * 2 * W * MM},
          {(void**)&Sacc, sizeof(float) * W * MN2},
          {(void**)&gemm_err, sizeof(int) * 4},
      };
      items.insert(items.end(), mx.begin(), mx.end());
      items.insert(items.end(), mx2.begin(), mx2.end());
    }
    size_t total = 0;
    for (auto& it : items) total += a256(it.bytes);
    SFQ_CUDA_TRY(cudaMalloc(&arena, total));
    arena_bytes = total;
    size_t off = 0;
    for (auto& it : items) {
      *it.ptr = arena + off;
      off += a256(it.bytes);
    }
    SFQ_CUDA_TRY(cudaMemsetAsync(arena, 0, total, st));
    return SFQ_OK;
  }

  // --- setup: RealDenseHamiltonian::getHamiltonianOperations + NOMSD::vMF + generateP1 --------
  // the int8-slice setup shared by single- and multi-determinant trials: vHS's B (L over n, the
  // packed pairs when symmetric) and the P1 slices
  int setup_i8_common() {
    int rc;
    const long MM = (long)M * M;
    if (sym) {
      double* packed = nullptr;
      SFQ_CUDA_TRY(cudaMallocAsync(&packed, sizeof(double) * P * Nc, st));
      if ((rc = pack_upper(Likn, M, Nc, packed, st))) return rc;
      if ((rc = islice_rows_real(packed, P, Nc, Nc, nslices, Lh_q, ld_nc, Lh_e, st))) return rc;
      SFQ_CUDA_TRY(cudaFreeAsync(packed, st));
    } else {
      if ((rc = islice_rows_real(Likn, MM, Nc, Nc, nslices, Lh_q, ld_nc, Lh_e, st))) return rc;
    }
    // P1 = I + Q with Q of order dt: the slices hold Q (each row's entries at their own scale, not
    // at the diagonal's), and the identity part is added exactly where the products are used
    double* q1 = nullptr;
    SFQ_CUDA_TRY(cudaMallocAsync((void**)&q1, sizeof(double) * MM, st));
    SFQ_CUDA_TRY(cudaMemcpyAsync(q1, P1, sizeof(double) * MM, cudaMemcpyDeviceToDevice, st));
    if ((rc = add_identity(q1, M, -1.0, st))) return rc;
    if ((rc = islice_rows_real(q1, M, M, M, nslices, P1_q, ld_m, P1_e, st))) return rc;
    SFQ_CUDA_TRY(cudaFreeAsync(q1, st));
    SFQ_CUDA_TRY(cudaMemsetAsync(gemm_err, 0, sizeof(int) * 4, st));
    return SFQ_OK;
  }
  // multi-determinant trials in the int8-slice mode: the trial's ci-weighted full G (the reference
  // the walkers' full G is sliced against) and its force bias, the slices of L as rows n over (i, k)
  // (L transposed in blocks of Cholesky vectors), and every determinant's exchange slices
  int setup_i8_md(const cplx* h_PsiT) {
    int rc;
    const long MM = (long)M * M;
    if ((rc = md_trial_green(h_PsiT))) return rc;
    SFQ_CUDA_TRY(cudaMemcpyAsync(RT_md, Racc, sizeof(cplx) * MM, cudaMemcpyDeviceToDevice, st));
    if ((rc = vbias_full(RT_md, 1, X))) return rc;
    SFQ_CUDA_TRY(cudaMemcpyAsync(vbT, X, sizeof(cplx) * Nc, cudaMemcpyDeviceToDevice, st));
    const long cap = (64L << 20) / MM;  // Cholesky vectors per block: at most 512 MB of FP64
    const int blk = int(cap < 1 ? 1 : (cap > Nc ? Nc : cap));
    double* tmp = nullptr;
    SFQ_CUDA_TRY(cudaMallocAsync((void**)&tmp, sizeof(double) * blk * MM, st));
    for (int n0 = 0; n0 < Nc; n0 += blk) {
      const int nb = Nc - n0 < blk ? Nc - n0 : blk;
      transpose_cols_kernel<<<dim3(unsigned((MM + 31) / 32), unsigned((nb + 31) / 32)), dim3(32, 8), 0, st>>>(
          Likn, MM, Nc, n0, nb, tmp);
      SFQ_LAUNCHED();
      int8_t* q[3];
      for (int t = 0; t < 3; ++t) q[t] = Lf_q[t] ? Lf_q[t] + (long)n0 * ld_mm : nullptr;
      if ((rc = islice_rows_real(tmp, nb, MM, MM, nslices, q, ld_mm, Lf_e + n0, st))) {
        cudaFreeAsync(tmp, st);
        return rc;
      }
    }
    SFQ_CUDA_TRY(cudaFreeAsync(tmp, st));
    const long o = det_elems(), lp = trial_real ? 1 : 2;
    for (int d = 0; d < ndet; ++d) {  // determinant d's rows at d lp Nc N (planar for a complex trial)
      int8_t* q[3];
      for (int t = 0; t < 3; ++t) q[t] = Le_q[t] ? Le_q[t] + lp * d * Nc * N * ld_mr : nullptr;
      int* ed = Le_e + lp * d * Nc * N;
      if (trial_real) {
        const double* Ld = (const double*)Lnak + (size_t)d * Nc * o;
        if ((rc = islice_rows_real(Ld, (long)Nc * N, Mr, Mr, nslices, q, ld_mr, ed, st))) return rc;
      } else {
        const cplx* Ld = (const cplx*)Lnak + (size_t)d * Nc * o;
        if ((rc = islice_rows_planar(Ld, (long)Nc * N, Mr, nslices, q, ld_mr, ed, st))) return rc;
      }
    }
    SFQ_CUDA_TRY(cudaStreamSynchronize(st));
    return setup_i8_common();
  }

  int setup(const double* h_hcore, const double* h_Likn, const cplx* h_PsiT) {
    int rc;
    const long MM = (long)M * M;
    SFQ_CUDA_TRY(cudaMemcpyAsync(hcore, h_hcore, sizeof(double) * MM, cudaMemcpyHostToDevice, st));
    SFQ_CUDA_TRY(cudaMemcpyAsync(Likn, h_Likn, sizeof(double) * MM * Nc, cudaMemcpyHostToDevice, st));
    const long RN = det_elems();
    SFQ_CUDA_TRY(cudaMemcpyAsync(PsiT, h_PsiT, sizeof(cplx) * ndet * RN, cudaMemcpyHostToDevice, st));
    std::vector<double> pr(size_t(ndet) * RN);
    for (size_t i = 0; i < pr.size(); ++i) pr[i] = h_PsiT[i].x;
    SFQ_CUDA_TRY(cudaMemcpyAsync(PsiTr, pr.data(), sizeof(double) * ndet * RN, cudaMemcpyHostToDevice, st));
    if (ndet > 1) {
      std::vector<cplx> lci(ndet), cic(ndet);
      for (int k = 0; k < ndet; ++k) {
        const cplx c = ci_h[k];
        cic[k] = cconj(c);
        const double a = std::hypot(c.x, c.y);
        lci[k] = a < 1e-12 ? mk(std::log(1e-12), 0.0) : mk(std::log(a), std::atan2(-c.y, c.x));
      }
      SFQ_CUDA_TRY(cudaMemcpyAsync(md_lci, lci.data(), sizeof(cplx) * ndet, cudaMemcpyHostToDevice, st));
      SFQ_CUDA_TRY(cudaMemcpyAsync(md_cic, cic.data(), sizeof(cplx) * ndet, cudaMemcpyHostToDevice, st));
      SFQ_CUDA_TRY(cudaStreamSynchronize(st));
    }
    {
      int asym = 1;
      SFQ_CUDA_TRY(cudaMemsetAsync(pw.flag, 0, sizeof(int), st));
      if ((rc = check_symmetric(Likn, M, Nc, pw.flag, st))) return rc;
      SFQ_CUDA_TRY(cudaMemcpyAsync(&asym, pw.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
      SFQ_CUDA_TRY(cudaMemsetAsync(pw.flag, 0, sizeof(int), st));
      SFQ_CUDA_TRY(cudaStreamSynchronize(st));
      sym = asym == 0;
      P = (long)M * (M + 1) / 2;
      if (sym && !mixed) {
        SFQ_CUDA_TRY(cudaMalloc(&Lp, sizeof(double) * P * Nc));
        SFQ_CUDA_TRY(cudaMalloc(&Vp, sizeof(cplx) * P * W));
        if ((rc = pack_upper(Likn, M, Nc, Lp, st))) return rc;
      }
    }
    SFQ_CUDA_TRY(cudaStreamSynchronize(st));

    // Lnak[n][a][k] = sum_i PsiT[a][i] L[i][k][n]  via tmp[a][(k,n)] then a permute; NONCOLLINEAR:
    // Lnak[n][a][q M + k] from PsiT's component q (RealDenseHamiltonian.cpp:141-161 with npol = 2)
    {
      void* tmp = nullptr;
      void* lq = nullptr;
      const size_t esz = trial_real ? sizeof(double) : sizeof(cplx);
      SFQ_CUDA_TRY(cudaMallocAsync(&tmp, esz * (size_t)N * M * Nc, st));
      if (npol > 1) SFQ_CUDA_TRY(cudaMallocAsync(&lq, esz * (size_t)N * M * Nc, st));
      for (int det = 0; det < ndet; ++det)
      for (int q = 0; q < npol; ++q) {
        GemmDesc d;
        const long a0 = det * RN + (long)q * M;
        char* ldst = static_cast<char*>(Lnak) + (size_t)det * Nc * RN * esz;
        d.M = N; d.N = int((long)M * Nc); d.K = M;
        d.A = trial_real ? (const void*)(PsiTr + a0) : (const void*)(PsiT + a0);
        d.sAm = Mr; d.sAk = 1; d.a_cplx = !trial_real;
        d.B = Likn; d.sBk = (long)M * Nc; d.sBn = 1; d.b_cplx = false;
        d.C = tmp; d.sCm = (long)M * Nc; d.sCn = 1;
        if ((rc = gemm_f64(d, st))) return rc;
        if (npol == 1) {
          if ((rc = permute_lnak(tmp, ldst, N, M, Nc, int(esz), st))) return rc;
        } else {
          if ((rc = permute_lnak(tmp, lq, N, M, Nc, int(esz), st))) return rc;
          SFQ_CUDA_TRY(cudaMemcpy2DAsync(ldst + (size_t)q * M * esz, Mr * esz, lq, M * esz, M * esz, (size_t)Nc * N,
                                         cudaMemcpyDeviceToDevice, st));
        }
      }
      SFQ_CUDA_TRY(cudaFreeAsync(tmp, st));
      if (lq) SFQ_CUDA_TRY(cudaFreeAsync(lq, st));
    }
    // haj = PsiT * hcore  (one_body.hpp:124-153); NONCOLLINEAR: PsiT * blockdiag(hcore, hcore)
    for (int det = 0; det < ndet; ++det)
    for (int q = 0; q < npol; ++q) {
      GemmDesc d;
      d.M = N; d.N = M; d.K = M;
      d.A = PsiT + det * RN + (long)q * M; d.sAm = Mr; d.sAk = 1; d.a_cplx = true;
      d.B = hcore; d.sBk = M; d.sBn = 1; d.b_cplx = false;
      d.C = haj + det * RN + (long)q * M; d.sCm = Mr; d.sCn = 1;
      if ((rc = gemm_f64(d, st))) return rc;
    }
    // v0 = -1/2 L L^T over (j, n)   (RealDenseHamiltonian.cpp:165-180)
    {
      GemmDesc d;
      const long K = (long)M * Nc;
      d.M = M; d.N = M; d.K = int(K);
      d.A = Likn; d.sAm = K; d.sAk = 1;
      d.B = Likn; d.sBk = 1; d.sBn = K;
      d.C = v0; d.sCm = M; d.sCn = 1;
      d.alpha = mk(-0.5, 0.0);
      if ((rc = gemm_f64(d, st))) return rc;
    }
    // vMF = Re vbias(G_trial)  (NOMSD.cpp:437-466; AFQMCBasePropagator.cpp:107 zero_imag)
    if (p.subtractMF && ndet > 1) {
      if ((rc = mean_field_md(h_PsiT))) return rc;
    } else if (p.subtractMF) {
      std::vector<cplx> psi(size_t(Mr) * N);  // PsiT^H  (Mr x N)
      for (int a = 0; a < N; ++a)
        for (int i = 0; i < Mr; ++i) psi[size_t(i) * N + a] = cconj(h_PsiT[size_t(a) * Mr + i]);
      SFQ_CUDA_TRY(cudaMemcpyAsync(SM2, psi.data(), sizeof(cplx) * Mr * N, cudaMemcpyHostToDevice, st));
      if ((rc = ops::overlap_matrix(PsiT, true, SM2, T, 1, Mr, N, st))) return rc;
      if ((rc = ops::mask_cross_spin(T, 1, N, spin_split(), st))) return rc;
      if ((rc = lu_logdet(T, (long)N * N, 1, N, ovtmp, false, 1.0, true, st))) return rc;
      if ((rc = ops::green_compact(T, SM2, G, 1, Mr, N, st))) return rc;
      if ((rc = ops::vbias(G, Lnak, !trial_real, X, 1, N, Mr, Nc, vb_scale(), st))) return rc;
      if ((rc = real_of(X, vmf, Nc, st))) return rc;
      SFQ_CUDA_TRY(cudaStreamSynchronize(st));
    } else {
      SFQ_CUDA_TRY(cudaMemsetAsync(vmf, 0, sizeof(double) * Nc, st));
    }
    // H1 = -1/2 herm(dt h + dt v0 + vHS(vMF)); P1 = exp(H1)  (generateP1, one_body.hpp:65-85)
    {
      // X <- vMF as a complex row
      std::vector<double> hv(Nc);
      SFQ_CUDA_TRY(cudaMemcpyAsync(hv.data(), vmf, sizeof(double) * Nc, cudaMemcpyDeviceToHost, st));
      SFQ_CUDA_TRY(cudaStreamSynchronize(st));
      std::vector<cplx> xv(Nc);
      for (int n = 0; n < Nc; ++n) xv[n] = mk(hv[n], 0.0);
      SFQ_CUDA_TRY(cudaMemcpyAsync(X, xv.data(), sizeof(cplx) * Nc, cudaMemcpyHostToDevice, st));
      if ((rc = ops::vhs(Likn, X, V, 1, M, Nc, std::sqrt(p.dt), st))) return rc;
      double* scr = nullptr;
      SFQ_CUDA_TRY(cudaMallocAsync((void**)&scr, sizeof(double) * 5 * MM, st));
      double* H = scr;
      double* Pa = H + MM;
      double* Pb = H + 2 * MM;
      double* term_a = H + 3 * MM;
      double* term_b = H + 4 * MM;
      if ((rc = build_h1(hcore, v0, V, p.dt, H, M, st))) return rc;
      std::vector<double> hh(MM);
      SFQ_CUDA_TRY(cudaMemcpyAsync(hh.data(), H, sizeof(double) * MM, cudaMemcpyDeviceToHost, st));
      SFQ_CUDA_TRY(cudaStreamSynchronize(st));
      double norm1 = 0.0;
      for (int k = 0; k < M; ++k) {
        double s = 0.0;
        for (int i = 0; i < M; ++i) s += std::fabs(hh[size_t(i) * M + k]);
        norm1 = std::fmax(norm1, s);
      }
      // scaling and squaring: exp(H) = exp(H / 2^s)^(2^s), ||H / 2^s||_1 <= 1/4, Taylor to order 18
      int sq = 0;
      while (norm1 / std::ldexp(1.0, sq) > 0.25) ++sq;
      const double scale = std::ldexp(1.0, -sq);
      SFQ_CUDA_TRY(cudaMemsetAsync(Pa, 0, sizeof(double) * MM, st));
      SFQ_CUDA_TRY(cudaMemsetAsync(term_a, 0, sizeof(double) * MM, st));
      if ((rc = add_identity(Pa, M, 1.0, st))) return rc;
      if ((rc = add_identity(term_a, M, 1.0, st))) return rc;
      for (int k = 1; k <= 18; ++k) {
        GemmDesc d;  // term_b = (scale/k) H term_a; Pa += term_b
        d.M = M; d.N = M; d.K = M;
        d.A = H; d.sAm = M; d.sAk = 1;
        d.B = term_a; d.sBk = M; d.sBn = 1;
        d.C = term_b; d.sCm = M; d.sCn = 1;
        d.S = Pa;
        d.alpha = mk(scale / double(k), 0.0);
        if ((rc = gemm_f64(d, st))) return rc;
        std::swap(term_a, term_b);
      }
      double* cur = Pa;
      double* nxt = Pb;
      for (int s = 0; s < sq; ++s) {
        GemmDesc d;
        d.M = M; d.N = M; d.K = M;
        d.A = cur; d.sAm = M; d.sAk = 1;
        d.B = cur; d.sBk = M; d.sBn = 1;
        d.C = nxt; d.sCm = M; d.sCn = 1;
        if ((rc = gemm_f64(d, st))) return rc;
        std::swap(cur, nxt);
      }
      SFQ_CUDA_TRY(cudaMemcpyAsync(P1, cur, sizeof(double) * MM, cudaMemcpyDeviceToDevice, st));
      if (!H1m) SFQ_CUDA_TRY(cudaMalloc(&H1m, sizeof(double) * MM));  // for P1^-1 (time-evolved BP)
      SFQ_CUDA_TRY(cudaMemcpyAsync(H1m, H, sizeof(double) * MM, cudaMemcpyDeviceToDevice, st));
      SFQ_CUDA_TRY(cudaFreeAsync(scr, st));
      if (!p.denseP1) {
        if ((rc = threshold_real(P1, MM, 1e-8, st))) return rc;
      }
    }
    // exact-accumulation mode: int8 slices of the resident real tensors, and the trial's own G and
    // force bias (NOMSD::vMF before its real part is taken)
    if (mixed && nslices && ndet > 1) {
      if ((rc = setup_i8_md(h_PsiT))) return rc;
    } else if (mixed && nslices) {
      const long NM = (long)N * Mr;
      {
        std::vector<cplx> psi(size_t(Mr) * N);  // PsiT^H (Mr x N)
        for (int a = 0; a < N; ++a)
          for (int i = 0; i < Mr; ++i) psi[size_t(i) * N + a] = cconj(h_PsiT[size_t(a) * Mr + i]);
        SFQ_CUDA_TRY(cudaMemcpyAsync(SM2, psi.data(), sizeof(cplx) * NM, cudaMemcpyHostToDevice, st));
        if ((rc = ops::overlap_matrix(PsiT, true, SM2, T, 1, Mr, N, st))) return rc;
        if (collinear && (rc = ops::mask_cross_spin(T, 1, N, spin_split(), st))) return rc;
        if ((rc = lu_logdet(T, (long)N * N, 1, N, ovtmp, false, 1.0, true, st))) return rc;
        if ((rc = ops::green_compact(T, SM2, G, 1, Mr, N, st))) return rc;
        SFQ_CUDA_TRY(cudaMemcpyAsync(GT_c, G, sizeof(cplx) * NM, cudaMemcpyDeviceToDevice, st));
        if ((rc = ops::vbias(G, Lnak, !trial_real, X, 1, N, Mr, Nc, vb_scale(), st))) return rc;
        SFQ_CUDA_TRY(cudaMemcpyAsync(vbT, X, sizeof(cplx) * Nc, cudaMemcpyDeviceToDevice, st));
        SFQ_CUDA_TRY(cudaStreamSynchronize(st));
      }
      if (trial_real) {
        const double* Ln = (const double*)Lnak;
        if ((rc = islice_rows_real(Ln, Nc, NM, NM, nslices, Lv_q, ld_nm, Lv_e, st))) return rc;
        if ((rc = islice_rows_real(Ln, (long)Nc * N, Mr, Mr, nslices, Le_q, ld_mr, Le_e, st))) return rc;
      } else {  // planar rows: Lr (rows r), Li (rows R + r)
        const cplx* Lc = (const cplx*)Lnak;
        if ((rc = islice_rows_planar(Lc, Nc, NM, nslices, Lv_q, ld_nm, Lv_e, st))) return rc;
        if ((rc = islice_rows_planar(Lc, (long)Nc * N, Mr, nslices, Le_q, ld_mr, Le_e, st))) return rc;
      }
      if ((rc = setup_i8_common())) return rc;
    } else if (mixed) {  // mixed precision: bf16 hi/lo planes of the resident real tensors
      if (sym) {
        double* packed = nullptr;
        SFQ_CUDA_TRY(cudaMallocAsync(&packed, sizeof(double) * P * Nc, st));
        if ((rc = pack_upper(Likn, M, Nc, packed, st))) return rc;
        if ((rc = split_bf16_f64(packed, P * Nc, Likn_p[0], Likn_p[1], Likn_p[2], st))) return rc;
        SFQ_CUDA_TRY(cudaFreeAsync(packed, st));
      } else {
        if ((rc = split_bf16_f64(Likn, MM * Nc, Likn_p[0], Likn_p[1], Likn_p[2], st))) return rc;
      }
      if ((rc = split_bf16_f64((const double*)Lnak, (long)Nc * N * M, Lnak_p[0], Lnak_p[1], Lnak_p[2], st))) return rc;
      if ((rc = split_bf16_f64(P1, MM, P1_p[0], P1_p[1], P1_p[2], st))) return rc;
      SFQ_CUDA_TRY(cudaMemsetAsync(gemm_err, 0, sizeof(int) * 4, st));
    }
    // walkers: copies of the trial, unit weight and phase
    {
      // NOMSD::initial_guess (NOMSD.cpp:132-153): the determinant of largest |ci|
      int d0 = 0;
      for (int k = 1; k < ndet; ++k)
        if (std::hypot(ci_h[k].x, ci_h[k].y) > std::hypot(ci_h[d0].x, ci_h[d0].y)) d0 = k;
      const cplx* ps = h_PsiT + (size_t)d0 * RN;
      std::vector<cplx> psi(size_t(Mr) * N);
      for (int a = 0; a < N; ++a)
        for (int i = 0; i < Mr; ++i) psi[size_t(i) * N + a] = cconj(ps[size_t(a) * Mr + i]);
      for (int w = 0; w < W; ++w)
        SFQ_CUDA_TRY(cudaMemcpyAsync(SM + (size_t)w * Mr * N, psi.data(), sizeof(cplx) * Mr * N,
                                     cudaMemcpyHostToDevice, st));
      SFQ_CUDA_TRY(cudaMemsetAsync(props, 0, sizeof(cplx) * kNumProps * W, st));
      if ((rc = fill_cplx(props + (long)P_WEIGHT * W, W, mk(1.0, 0.0), st))) return rc;
      if ((rc = fill_cplx(props + (long)P_PHASE * W, W, mk(1.0, 0.0), st))) return rc;
    }
    SFQ_CUDA_TRY(cudaMemsetAsync(stats, 0, sizeof(unsigned long long) * 8, st));
    SFQ_CUDA_TRY(cudaStreamSynchronize(st));
    return SFQ_OK;
  }

  // the inverse overlap matrices (PsiT W)^-1 of the current walkers in T, their log overlaps in
  // ov (W; may be null)
  int ensure_inverse(cplx* ov) {
    int rc;
    if (!inv_cached) {
      const void* A = trial_real ? (const void*)PsiTr : (const void*)PsiT;
      cplx* out = ov ? ov : ovtmp;
      if ((rc = ops::overlap_matrix(A, !trial_real, SM, T, W, Mr, N, st))) return rc;
      if ((rc = ops::mask_cross_spin(T, W, N, spin_split(), st))) return rc;
      if ((rc = lu_logdet(T, (long)N * N, W, N, out, false, ov_scale(), true, st))) return rc;
      inv_cached = true;
      inv_ov = out;
    } else if (ov && ov != inv_ov) {
      SFQ_CUDA_TRY(cudaMemcpyAsync(ov, inv_ov, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st));
    }
    return SFQ_OK;
  }

  // --- multi-determinant NOMSD (ndet > 1) -----------------------------------------------------
  // determinant d against the walkers B (nb of them): overlap matrices, their inverses in T and log
  // overlaps (times post, without the ci term) in ov
  int md_factor(int d, const cplx* B, int nb, cplx* ov, bool invert, double post) {
    int rc;
    const long o = d * det_elems();
    const void* A = trial_real ? (const void*)(PsiTr + o) : (const void*)(PsiT + o);
    if ((rc = ops::overlap_matrix(A, !trial_real, B, T, nb, Mr, N, st))) return rc;
    if ((rc = ops::mask_cross_spin(T, nb, N, spin_split(), st))) return rc;
    return lu_logdet(T, (long)N * N, nb, N, ov, false, post, invert, st);
  }
  // R[w][i][k] = sum_q sum_a PsiT_d[a][qM + i] Gc[w][a][qM + k]: determinant d's full G
  // (PsiT_d^T Gc, density_matrix.hpp:580-585) summed over the spin (rows of both spins) and
  // polarization (the diagonal component blocks) blocks, what vbias contracts with L
  int md_reduced_green(int d, const cplx* Gc, int nb, cplx* R) {
    int rc;
    for (int q = 0; q < npol; ++q) {
      GemmDesc g;
      g.M = M; g.N = M; g.K = N; g.batch = nb;
      g.A = PsiT + d * det_elems() + (long)q * M; g.sAm = 1; g.sAk = Mr; g.sAb = 0; g.a_cplx = true;
      g.B = Gc + (long)q * M; g.sBk = Mr; g.sBn = 1; g.sBb = det_elems(); g.b_cplx = true;
      g.C = R; g.sCm = M; g.sCn = 1; g.sCb = (long)M * M;
      if (q > 0) g.beta = mk(1.0, 0.0);
      if ((rc = gemm_f64(g, st))) return rc;
    }
    return SFQ_OK;
  }
  // vbias from a full G: out[w][n] = a sum_ik L[i][k][n] R[w][i][k] (Real3IndexFactorization.hpp:392-426)
  int vbias_full(const cplx* R, int nb, cplx* out) {
    GemmDesc g;
    g.M = nb; g.N = Nc; g.K = M * M; g.batch = 1;
    g.A = R; g.sAm = (long)M * M; g.sAk = 1; g.a_cplx = true;
    g.B = Likn; g.sBk = Nc; g.sBn = 1; g.b_cplx = false;
    g.C = out; g.sCm = Nc; g.sCn = 1;
    g.alpha = mk(vb_scale(), 0.0);
    return gemm_f64(g, st);
  }
  int md_grid(long n) const { return int(std::min<long>((n + 255) / 256, 64)); }
  // NOMSD::vMF, ndet > 1 (NOMSD.cpp:466-512): the pairs q >= p of the trial's own determinants
  int mean_field_md(const cplx* h_PsiT) {
    int rc;
    if ((rc = md_trial_green(h_PsiT))) return rc;
    if ((rc = vbias_full(Racc, 1, X))) return rc;
    if ((rc = real_of(X, vmf, Nc, st))) return rc;
    SFQ_CUDA_TRY(cudaStreamSynchronize(st));
    return SFQ_OK;
  }
  // the trial's own ci-weighted full G (M x M) into Racc (first walker slot): the pairs q >= p of
  // its determinants, normalised (NOMSD.cpp:466-512 before the force bias is taken)
  int md_trial_green(const cplx* h_PsiT) {
    int rc;
    const long MM = (long)M * M;
    bool first = true;
    std::vector<cplx> psi(size_t(Mr) * N);
    for (int pd = 0; pd < ndet; ++pd) {
      const cplx* ps = h_PsiT + (size_t)pd * det_elems();
      for (int a = 0; a < N; ++a)
        for (int i = 0; i < Mr; ++i) psi[size_t(i) * N + a] = cconj(ps[size_t(a) * Mr + i]);
      SFQ_CUDA_TRY(cudaMemcpyAsync(SM2, psi.data(), sizeof(cplx) * Mr * N, cudaMemcpyHostToDevice, st));
      for (int qd = pd; qd < ndet; ++qd) {
        // det_ops::MixedDensityMatrix as called there: the overlap not doubled for CLOSED
        if ((rc = md_factor(qd, SM2, 1, ovtmp, true, 1.0))) return rc;
        if ((rc = ops::green_compact(T, SM2, G, 1, Mr, N, st))) return rc;
        if ((rc = md_reduced_green(qd, G, 1, Rd))) return rc;
        md_pair_kernel<<<md_grid(MM), 256, 0, st>>>(Rd, ovtmp, ci_h[qd], ci_h[pd], Racc, wsum, MM, first ? 1 : 0);
        SFQ_LAUNCHED();
        first = false;
      }
      SFQ_CUDA_TRY(cudaStreamSynchronize(st));  // psi is refilled for the next p
    }
    md_normalize_kernel<<<dim3(md_grid(MM), 1), 256, 0, st>>>(Racc, wsum, MM);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }
  // NOMSD::vbias with ndet > 1 (NOMSD.cpp:39-61,238-278): the ci-weighted full G, then vbias on it
  int vbias_md(cplx* out) {
    int rc;
    if ((rc = md_full_green())) return rc;
    return vbias_full(Racc, W, out);
  }
  // every walker's ci-weighted full G (W, M, M) into Racc, the determinants' log overlaps in md_ov
  int md_full_green() {
    int rc;
    const long MM = (long)M * M;
    const cplx* lm = props + (long)P_OVLP * W;
    for (int d = 0; d < ndet; ++d) {
      if ((rc = md_factor(d, SM, W, md_ov + (long)d * W, true, ov_scale()))) return rc;
      if ((rc = ops::green_compact(T, SM, G, W, Mr, N, st))) return rc;
      if ((rc = md_reduced_green(d, G, W, Rd))) return rc;
      md_accumulate_kernel<<<dim3(md_grid(MM), W), 256, 0, st>>>(Rd, md_ov + (long)d * W, lm, ci_h[d], Racc, wsum,
                                                                 MM, d == 0 ? 1 : 0);
      SFQ_LAUNCHED();
    }
    md_normalize_kernel<<<dim3(md_grid(MM), W), 256, 0, st>>>(Racc, wsum, MM);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }
  // NOMSD::Log_Overlap with ndet > 1 into ov (W)
  int log_overlap_md(cplx* ov) {
    int rc;
    inv_cached = false;
    for (int d = 0; d < ndet; ++d)
      if ((rc = md_factor(d, SM, W, md_ov + (long)d * W, false, ov_scale()))) return rc;
    md_logsum_kernel<<<(W + 127) / 128, 128, 0, st>>>(md_ov, md_lci, ndet, W, ov);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }
  // NOMSD::Energy with ndet > 1: E3 and ovtmp
  int energy_md() {
    int rc;
    inv_cached = false;
    const long o = det_elems();
    for (int d = 0; d < ndet; ++d) {
      if ((rc = md_factor(d, SM, W, md_ov + (long)d * W, true, ov_scale()))) return rc;
      if ((rc = ops::green_compact(T, SM, G, W, Mr, N, st))) return rc;
      const void* Ld = static_cast<const char*>(Lnak) + (size_t)d * Nc * o * lnak_esz();
      if ((rc = ops::energy(md_E + (long)d * W * 3, G, haj + d * o, Ld, !trial_real, p.E0, W, N, Mr, Nc, 1, 1, 1,
                            Tchunk, tchunk_elems, exxn, kl, st, spin_split())))
        return rc;
    }
    md_energy_kernel<<<(W + 127) / 128, 128, 0, st>>>(md_ov, md_E, md_cic, ndet, W, E3, ovtmp);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }

  // the other observables of the mixed and back-propagated estimators, when asked for (results divided by the total weight)
  struct ObsSpec {
    bool two_rdm = false, spin_corr = false;
    int npair = 0;
    const int* maps = nullptr;  // host (npair, M)
    std::vector<cplx> two, spin, pair;
  };
  // --- time-evolved back propagation (TimeEvolvedBPEstimator.hpp, PropagateOperators
  // AFQMCBasePropagator.cpp:538-654) ----------------------------------------------------------
  // the operator states X (-> c^+), Y (-> c) and the stabilization sums M per spin and walker,
  // (ns, W, R, R) with R = npol M, evolved forward through the fields the back-propagation ring keeps
  cplx *te_X = nullptr, *te_Y = nullptr, *te_M = nullptr, *te_scr = nullptr;
  // out = exp(sgn H) by scaling and squaring (Taylor to order 18 at norm <= 1/4), as P1 is built
  int expm_real(const double* H, double sgn, double* out) {
    int rc;
    const long MM = (long)M * M;
    std::vector<double> hh(MM);
    SFQ_CUDA_TRY(cudaMemcpyAsync(hh.data(), H, sizeof(double) * MM, cudaMemcpyDeviceToHost, st));
    SFQ_CUDA_TRY(cudaStreamSynchronize(st));
    double norm1 = 0.0;
    for (int k = 0; k < M; ++k) {
      double a = 0.0;
      for (int i = 0; i < M; ++i) a += std::fabs(hh[size_t(i) * M + k]);
      norm1 = std::fmax(norm1, a);
    }
    int sq = 0;
    while (norm1 / std::ldexp(1.0, sq) > 0.25) ++sq;
    const double scale = sgn * std::ldexp(1.0, -sq);
    double* scr = nullptr;
    SFQ_CUDA_TRY(cudaMallocAsync((void**)&scr, sizeof(double) * 4 * MM, st));
    double *Pa = scr, *Pb = scr + MM, *ta = scr + 2 * MM, *tb = scr + 3 * MM;
    SFQ_CUDA_TRY(cudaMemsetAsync(Pa, 0, sizeof(double) * MM, st));
    SFQ_CUDA_TRY(cudaMemsetAsync(ta, 0, sizeof(double) * MM, st));
    if ((rc = add_identity(Pa, M, 1.0, st)) || (rc = add_identity(ta, M, 1.0, st))) return rc;
    for (int k = 1; k <= 18; ++k) {
      GemmDesc d;  // tb = (scale/k) H ta; Pa += tb
      d.M = M; d.N = M; d.K = M;
      d.A = H; d.sAm = M; d.sAk = 1;
      d.B = ta; d.sBk = M; d.sBn = 1;
      d.C = tb; d.sCm = M; d.sCn = 1;
      d.S = Pa;
      d.alpha = mk(scale / double(k), 0.0);
      if ((rc = gemm_f64(d, st))) return rc;
      std::swap(ta, tb);
    }
    double* cur = Pa;
    double* nxt = Pb;
    for (int q = 0; q < sq; ++q) {
      GemmDesc d;
      d.M = M; d.N = M; d.K = M;
      d.A = cur; d.sAm = M; d.sAk = 1;
      d.B = cur; d.sBk = M; d.sBn = 1;
      d.C = nxt; d.sCm = M; d.sCn = 1;
      if ((rc = gemm_f64(d, st))) return rc;
      std::swap(cur, nxt);
    }
    SFQ_CUDA_TRY(cudaMemcpyAsync(out, cur, sizeof(double) * MM, cudaMemcpyDeviceToDevice, st));
    SFQ_CUDA_TRY(cudaFreeAsync(scr, st));
    if (!p.denseP1 && (rc = threshold_real(out, MM, 1e-8, st))) return rc;
    return SFQ_OK;
  }
  int te_enable() {
    int rc;
    if (!nbp) return record_error(SFQ_ERR_ARG, "time-evolved back propagation needs the field ring: enable back propagation first");
    if (te_X) return SFQ_OK;
    const long RR = (long)Mr * Mr, nmat = (long)rdm_nspin() * W;
    SFQ_CUDA_TRY(cudaMalloc(&te_X, sizeof(cplx) * nmat * RR));
    SFQ_CUDA_TRY(cudaMalloc(&te_Y, sizeof(cplx) * nmat * RR));
    SFQ_CUDA_TRY(cudaMalloc(&te_M, sizeof(cplx) * nmat * RR));
    SFQ_CUDA_TRY(cudaMalloc(&te_scr, sizeof(cplx) * 4 * (size_t)W * RR));
    SFQ_CUDA_TRY(cudaMalloc(&P1inv, sizeof(double) * (size_t)M * M));
    if ((rc = expm_real(H1m, -1.0, P1inv))) return rc;  // generateP1(true): exp(+1/2 herm(H1))
    return te_anchor();
  }
  // setAnchor (TimeEvolvedBPEstimator.hpp:282-287): X = Y = I, M = 0
  int te_anchor() {
    if (!te_X) return record_error(SFQ_ERR_ARG, "time-evolved back propagation is not enabled");
    const long RR = (long)Mr * Mr, nmat = (long)rdm_nspin() * W;
    set_identity_batched_kernel<<<1184, 256, 0, st>>>(te_X, nmat, Mr);
    SFQ_LAUNCHED();
    set_identity_batched_kernel<<<1184, 256, 0, st>>>(te_Y, nmat, Mr);
    SFQ_LAUNCHED();
    SFQ_CUDA_TRY(cudaMemsetAsync(te_M, 0, sizeof(cplx) * nmat * RR, st));
    return SFQ_OK;
  }
  // columns [c0, c0 + nel) of the walkers' Slater matrices: the spin block s
  void spin_cols(int s, int& c0, int& nel) const {
    c0 = (collinear && s == 1) ? nup : 0;
    nel = collinear ? (s == 0 ? nup : N - nup) : N;
  }
  // PropagateOperators over the last nsteps stored fields, oldest first: X <- P1 e^{i vHS} P1 X,
  // Y <- P1^-1 e^{i vHS^H} P1^-1 Y (the adjoint of the inverse step), then per spin with the walkers'
  // Slater matrices S: Y <- S S^H Y, M += Y^H X, X <- X - S S^H X
  int te_evolve(int nsteps) {
    int rc;
    if (!te_X) return record_error(SFQ_ERR_ARG, "time-evolved back propagation is not enabled");
    if (nsteps <= 0 || nsteps > nbp) return record_error(SFQ_ERR_ARG, "operators evolved over %d steps (ring %d)", nsteps, nbp);
    const long MM = (long)M * M, RR = (long)Mr * Mr;
    const int ns = rdm_nspin();
    cplx* TM = te_scr;
    cplx* T1x = te_scr + (size_t)W * RR;
    cplx* T2x = te_scr + 2 * (size_t)W * RR;
    int slot = (hist_pos % nbp + nbp - nsteps) % nbp;
    for (int i = 0; i < nsteps; ++i, slot = (slot + 1) % nbp) {
      SFQ_CUDA_TRY(cudaMemcpy2DAsync(X, sizeof(cplx) * Nc, bp_fields + (long)slot * Nc, sizeof(cplx) * nbp * Nc,
                                     sizeof(cplx) * Nc, W, cudaMemcpyDeviceToDevice, st));
      if (sym) {
        if ((rc = ops::vhs_rows(Lp, P, X, Vp, W, Nc, std::sqrt(p.dt), st))) return rc;
        if ((rc = unpack_symmetric(Vp, W, M, V, st))) return rc;
      } else if ((rc = ops::vhs(Likn, X, V, W, M, Nc, std::sqrt(p.dt), st))) {
        return rc;
      }
      for (int q = 0; q < ns; ++q)
        if ((rc = ops::propagate(te_X + (size_t)q * W * RR, P1, false, V, W, M, Mr, p.taylor_order, TM, T1x, T2x, st,
                                 npol)))
          return rc;
      adjoint_kernel<<<dim3(md_grid(MM / 2 + M), W), 256, 0, st>>>(V, M);
      SFQ_LAUNCHED();
      for (int q = 0; q < ns; ++q)
        if ((rc = ops::propagate(te_Y + (size_t)q * W * RR, P1inv, false, V, W, M, Mr, p.taylor_order, TM, T1x, T2x,
                                 st, npol)))
          return rc;
    }
    for (int q = 0; q < ns; ++q) {
      int c0, nel;
      spin_cols(q, c0, nel);
      cplx* Xs = te_X + (size_t)q * W * RR;
      cplx* Ys = te_Y + (size_t)q * W * RR;
      cplx* Ms = te_M + (size_t)q * W * RR;
      if (nel == 0) {  // an empty sector: S S^H = 0
        SFQ_CUDA_TRY(cudaMemsetAsync(Ys, 0, sizeof(cplx) * W * RR, st));
        continue;
      }
      cplx* SY = TM;  // (W, nel, R)
      auto sh = [&](const cplx* B) {  // SY = S^H B
        GemmDesc g;
        g.M = nel; g.N = Mr; g.K = Mr; g.batch = W;
        g.A = SM + c0; g.sAm = 1; g.sAk = N; g.sAb = (long)Mr * N; g.a_cplx = true; g.conj_a = true;
        g.B = B; g.sBk = Mr; g.sBn = 1; g.sBb = RR; g.b_cplx = true;
        g.C = SY; g.sCm = Mr; g.sCn = 1; g.sCb = (long)nel * Mr;
        return gemm_f64(g, st);
      };
      auto s_sy = [&](cplx* C, cplx alpha, cplx beta) {  // C = alpha S SY + beta C
        GemmDesc g;
        g.M = Mr; g.N = Mr; g.K = nel; g.batch = W;
        g.A = SM + c0; g.sAm = N; g.sAk = 1; g.sAb = (long)Mr * N; g.a_cplx = true;
        g.B = SY; g.sBk = Mr; g.sBn = 1; g.sBb = (long)nel * Mr; g.b_cplx = true;
        g.C = C; g.sCm = Mr; g.sCn = 1; g.sCb = RR;
        g.alpha = alpha; g.beta = beta;
        return gemm_f64(g, st);
      };
      if ((rc = sh(Ys)) || (rc = s_sy(Ys, mk(1.0, 0.0), mk(0.0, 0.0)))) return rc;
      GemmDesc g;  // M += Y^H X
      g.M = Mr; g.N = Mr; g.K = Mr; g.batch = W;
      g.A = Ys; g.sAm = 1; g.sAk = Mr; g.sAb = RR; g.a_cplx = true; g.conj_a = true;
      g.B = Xs; g.sBk = Mr; g.sBn = 1; g.sBb = RR; g.b_cplx = true;
      g.C = Ms; g.sCm = Mr; g.sCn = 1; g.sCb = RR; g.beta = mk(1.0, 0.0);
      if ((rc = gemm_f64(g, st))) return rc;
      if ((rc = sh(Xs)) || (rc = s_sy(Xs, mk(-1.0, 0.0), mk(1.0, 0.0)))) return rc;
    }
    return SFQ_OK;
  }
  // the Green's functions the evolved operators dress (constructTimeEvolvedMeasurementInputs,
  // TimeEvolvedBPEstimator.hpp:42-140): Gf[w][s] = M_s + (PsiT_s X_s)^T (Gc_s conj(Y_s)), Gc the
  // walkers' compact mixed density matrix
  // det < 0: the single-determinant trial's G from density(); det >= 0: reference det's, its compact
  // G already in G (from its overlap factors) and its PsiT_d in the dressing
  int te_green(cplx* Gf, int det = -1) {
    int rc;
    const long RR = (long)Mr * Mr;
    const int ns = rdm_nspin();
    if (det < 0 && (rc = density(ovtmp))) return rc;
    const cplx* Pd = PsiT + (det < 0 ? 0 : (long)det * det_elems());
    cplx* Yc = te_scr;                        // conj(Y_s) (W, R, R)
    cplx* XR = te_scr + (size_t)W * RR;       // PsiT_s X_s (W, nel, R)
    cplx* GY = te_scr + 2 * (size_t)W * RR;   // Gc_s conj(Y_s) (W, nel, R)
    for (int q = 0; q < ns; ++q) {
      int c0, nel;
      spin_cols(q, c0, nel);
      SFQ_CUDA_TRY(cudaMemcpy2DAsync(Gf + q * RR, sizeof(cplx) * ns * RR, te_M + (size_t)q * W * RR,
                                     sizeof(cplx) * RR, sizeof(cplx) * RR, W, cudaMemcpyDeviceToDevice, st));
      if (nel == 0) continue;
      conj_copy_kernel<<<1184, 256, 0, st>>>(te_Y + (size_t)q * W * RR, Yc, (long)W * RR);
      SFQ_LAUNCHED();
      GemmDesc g;  // GY = Gc_s conj(Y_s)
      g.M = nel; g.N = Mr; g.K = Mr; g.batch = W;
      g.A = G + (long)c0 * Mr; g.sAm = Mr; g.sAk = 1; g.sAb = (long)N * Mr; g.a_cplx = true;
      g.B = Yc; g.sBk = Mr; g.sBn = 1; g.sBb = RR; g.b_cplx = true;
      g.C = GY; g.sCm = Mr; g.sCn = 1; g.sCb = (long)nel * Mr;
      if ((rc = gemm_f64(g, st))) return rc;
      GemmDesc h;  // XR = PsiT_s X_s
      h.M = nel; h.N = Mr; h.K = Mr; h.batch = W;
      h.A = Pd + (long)c0 * Mr; h.sAm = Mr; h.sAk = 1; h.sAb = 0; h.a_cplx = true;
      h.B = te_X + (size_t)q * W * RR; h.sBk = Mr; h.sBn = 1; h.sBb = RR; h.b_cplx = true;
      h.C = XR; h.sCm = Mr; h.sCn = 1; h.sCb = (long)nel * Mr;
      if ((rc = gemm_f64(h, st))) return rc;
      GemmDesc k;  // Gf_s += XR^T GY
      k.M = Mr; k.N = Mr; k.K = nel; k.batch = W;
      k.A = XR; k.sAm = 1; k.sAk = Mr; k.sAb = (long)nel * Mr; k.a_cplx = true;
      k.B = GY; k.sBk = Mr; k.sBn = 1; k.sBb = (long)nel * Mr; k.b_cplx = true;
      k.C = Gf + q * RR; k.sCm = Mr; k.sCn = 1; k.sCb = ns * RR; k.beta = mk(1.0, 0.0);
      if ((rc = gemm_f64(k, st))) return rc;
    }
    return SFQ_OK;
  }
  // the measurement: the weights restored over restore steps (TimeEvolvedBPEstimator.hpp:245-256),
  // the RDMs and observables of the dressed Green's functions, divided by their sum
  int te_measure(int restore, std::vector<cplx>& one, std::vector<cplx>& two, ObsSpec* obs) {
    if (!te_X) return record_error(SFQ_ERR_ARG, "time-evolved back propagation is not enabled");
    if (restore < 0 || restore > nhist) return record_error(SFQ_ERR_ARG, "weights restored over %d steps (history %d)", restore, nhist);
    inv_cached = false;
    SFQ_CUDA_TRY(cudaMemcpyAsync(bp_wt, props + (long)P_WEIGHT * W, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st));
    int h = hist_pos;
    for (int k = 0; k < restore; ++k) {
      h = h == 0 ? nhist - 1 : h - 1;
      bp_restore_kernel<<<(W + 127) / 128, 128, 0, st>>>(bp_wt, bp_wfac + h, nhist, W);
      SFQ_LAUNCHED();
    }
    return rdm_measure(bp_wt, false, one, two, obs, true);
  }

  // --- back propagation (WalkerSetBase::resize_bp, BackPropEstimator) ---------------------------
  // per walker: the anchored walkers, a ring of the last nbp steps' fields (slot hist_pos % nbp),
  // the weight factors of the last 3 nbp steps (slot hist_pos); all travel with population control
  int nbp = 0, nhist = 0, hist_pos = 0;
  cplx *bp_SMN = nullptr, *bp_fields = nullptr, *bp_wfac = nullptr;
  cplx *bp_refs = nullptr, *bp_ldet = nullptr, *bp_wt = nullptr;
  int enable_bp(int n) {
    if (mixed) return record_error(SFQ_ERR_UNSUPPORTED, "back propagation runs in FP64 engines");
    if (n <= 0) return record_error(SFQ_ERR_ARG, "back propagation needs nbp > 0");
    if (nbp) return record_error(SFQ_ERR_ARG, "back propagation is already enabled (nbp = %d)", nbp);
    nbp = n;
    nhist = 3 * n;
    hist_pos = 0;
    const long RN = det_elems();
    SFQ_CUDA_TRY(cudaMalloc(&bp_SMN, sizeof(cplx) * W * RN));
    SFQ_CUDA_TRY(cudaMalloc(&bp_fields, sizeof(cplx) * (size_t)W * nbp * Nc));
    SFQ_CUDA_TRY(cudaMalloc(&bp_wfac, sizeof(cplx) * (size_t)W * nhist));
    SFQ_CUDA_TRY(cudaMalloc(&bp_refs, sizeof(cplx) * (size_t)ndet * W * RN));
    SFQ_CUDA_TRY(cudaMalloc(&bp_ldet, sizeof(cplx) * (size_t)ndet * W));
    SFQ_CUDA_TRY(cudaMalloc(&bp_wt, sizeof(cplx) * W));
    SFQ_CUDA_TRY(cudaMemsetAsync(bp_fields, 0, sizeof(cplx) * (size_t)W * nbp * Nc, st));
    int rc;
    if ((rc = fill_cplx(bp_wfac, (long)W * nhist, mk(1.0, 0.0), st))) return rc;
    return bp_anchor();
  }
  int bp_anchor() {
    if (!nbp) return record_error(SFQ_ERR_ARG, "back propagation is not enabled");
    SFQ_CUDA_TRY(cudaMemcpyAsync(bp_SMN, SM, sizeof(cplx) * W * det_elems(), cudaMemcpyDeviceToDevice, st));
    return sync_checked();
  }
  // BackPropagate over the last nb steps and the BackPropEstimator's RDMs (one (nspin, Mr, Mr), two
  // before folding (nblk, Mr, Mr)), divided by the sum of the restored weights
  int measure_bp(int nb, int ortho, bool restore, std::vector<cplx>& one, std::vector<cplx>& two,
                 ObsSpec* obs = nullptr) {
    int rc;
    if (!nbp) return record_error(SFQ_ERR_ARG, "back propagation is not enabled");
    if (nb <= 0 || nb > nbp || ortho <= 0) return record_error(SFQ_ERR_ARG, "back propagation over %d steps (ring %d)", nb, nbp);
    const long RN = det_elems(), MM = (long)M * M;
    inv_cached = false;
    bp_init_refs_kernel<<<1184, 256, 0, st>>>(PsiT, ndet, W, Mr, N, bp_refs);
    SFQ_LAUNCHED();
    SFQ_CUDA_TRY(cudaMemsetAsync(bp_ldet, 0, sizeof(cplx) * (size_t)ndet * W, st));
    int slot = hist_pos % nbp;
    for (int ni = nb - 1; ni >= 0; --ni) {
      slot = slot == 0 ? nbp - 1 : slot - 1;
      SFQ_CUDA_TRY(cudaMemcpy2DAsync(X, sizeof(cplx) * Nc, bp_fields + (long)slot * Nc, sizeof(cplx) * nbp * Nc,
                                     sizeof(cplx) * Nc, W, cudaMemcpyDeviceToDevice, st));
      if (sym) {
        if ((rc = ops::vhs_rows(Lp, P, X, Vp, W, Nc, std::sqrt(p.dt), st))) return rc;
        if ((rc = unpack_symmetric(Vp, W, M, V, st))) return rc;
      } else if ((rc = ops::vhs(Likn, X, V, W, M, Nc, std::sqrt(p.dt), st))) {
        return rc;
      }
      neg_adjoint_kernel<<<dim3(md_grid(MM / 2 + M), W), 256, 0, st>>>(V, M);
      SFQ_LAUNCHED();
      for (int d = 0; d < ndet; ++d) {
        cplx* S = bp_refs + (long)d * W * RN;
        // P1 is real symmetric: P1^H = P1 (propagate.hpp:258-297 with TA = 'H')
        if ((rc = ops::propagate(S, P1, false, V, W, M, N, p.taylor_order, TMN, T1, T2, st, npol))) return rc;
        if (ni == 0 || ni % ortho == 0)
          if ((rc = ops::orthogonalize_logdet(S, SM2, T, Tchunk, status, bp_ldet + (long)d * W, W, Mr, N, st,
                                              spin_split())))
            return rc;
      }
    }
    bp_shift_kernel<<<(W + 127) / 128, 128, 0, st>>>(bp_ldet, ndet, W);
    SFQ_LAUNCHED();
    SFQ_CUDA_TRY(cudaMemcpyAsync(bp_wt, props + (long)P_WEIGHT * W, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st));
    if (restore) {
      int h = hist_pos;
      for (int k = 0; k < nb; ++k) {
        h = h == 0 ? nhist - 1 : h - 1;
        bp_restore_kernel<<<(W + 127) / 128, 128, 0, st>>>(bp_wt, bp_wfac + h, nhist, W);
        SFQ_LAUNCHED();
      }
    }
    return rdm_measure(bp_wt, true, one, two, obs);
  }

  // --- MixedEstimator with the OneRDM and DiagonalTwoRDM observables -------------------------
  cplx* rdm_buf = nullptr;  // Gf (W, nspin, Mr, Mr), one (nspin Mr Mr), two (nblk Mr Mr), wc, tot (W), ov (ndet W)
  int rdm_nspin() const { return collinear ? 2 : 1; }
  int rdm_nblk() const { return collinear ? 3 : (npol == 2 ? 1 : 2); }
  // one (rdm_nspin, Mr, Mr) and the diagonal two-body RDM before folding (rdm_nblk, Mr, Mr), both divided
  // by the total weight, on the host (MixedEstimator.hpp:37-147)
  int measure_rdm(std::vector<cplx>& one, std::vector<cplx>& two, ObsSpec* obs = nullptr) {
    if (mixed) return record_error(SFQ_ERR_UNSUPPORTED, "the mixed estimator's RDMs are measured in FP64 engines");
    inv_cached = false;
    return rdm_measure(props + (long)P_WEIGHT * W, false, one, two, obs);
  }
  // which observables this engine's walkers support, as the reference's constructors check them
  int check_obs(const ObsSpec& o) const {
    if (o.two_rdm && npol == 2)
      return record_error(SFQ_ERR_UNSUPPORTED, "TwoRDM is only implemented for closed and collinear walkers");
    if (o.two_rdm && (double)M * M * M * M * 16.0 > double(1L << 30))
      return record_error(SFQ_ERR_UNSUPPORTED, "TwoRDM of %d orbitals: more than 1 GiB per block", M);
    if (o.npair && closed())
      return record_error(SFQ_ERR_UNSUPPORTED, "PairCorr is not implemented for closed walkers");
    if (o.npair < 0 || (o.npair && !o.maps)) return record_error(SFQ_ERR_ARG, "PairCorr: %d maps", o.npair);
    for (long t = 0; t < (long)o.npair * M; ++t)
      if (o.maps[t] >= M) return record_error(SFQ_ERR_ARG, "PairCorr: partner %d of %d orbitals", o.maps[t], M);
    return SFQ_OK;
  }
  // the RDM reduction shared by the mixed estimator (bp false: the trial's references against the
  // walkers, coefficients relative to the walkers' log overlaps) and the back-propagated one (bp true:
  // each walker's propagated references against its anchored matrix, the overlaps with conj of the
  // references' QR log dets, constructBPMeasurementInputs, BackPropEstimator.hpp:36-110)
  int rdm_measure(const cplx* weight, bool bp, std::vector<cplx>& one, std::vector<cplx>& two,
                  ObsSpec* obs = nullptr, bool te = false) {
    int rc;
    if (obs && (rc = check_obs(*obs))) return rc;
    const int ns = rdm_nspin(), nb = rdm_nblk();
    const long MM = (long)Mr * Mr, RN = det_elems();
    const size_t elems = (size_t)W * ns * MM + ns * MM + nb * MM + 2 * (size_t)W + (size_t)ndet * W;
    if (!rdm_buf) SFQ_CUDA_TRY(cudaMalloc(&rdm_buf, sizeof(cplx) * elems));
    cplx* Gf = rdm_buf;
    cplx* o1 = Gf + (size_t)W * ns * MM;
    cplx* o2 = o1 + ns * MM;
    cplx* wc = o2 + nb * MM;
    cplx* tot = wc + W;
    cplx* ovd = tot + W;
    SFQ_CUDA_TRY(cudaMemsetAsync(o1, 0, sizeof(cplx) * (ns + nb) * MM, st));
    // observables' device buffers: TwoRDM (ns + 1 blocks of M^4) and its product scratch, the weighted
    // walker G's, SpinCorr (2, M(M+1)/2), PairCorr (npair^2 M^2) and the pair maps
    // (sized by the orbitals M: NONCOLLINEAR G blocks are 2M x 2M, the observables M x M)
    const int kind = npol == 2 ? 2 : (collinear ? 1 : 0);
    const long Mo2 = (long)M * M, M4 = Mo2 * Mo2, Ptri = (long)M * (M + 1) / 2;
    const long n2 = obs && obs->two_rdm ? (ns + 1) * M4 : 0, ns_sp = obs && obs->spin_corr ? 2 * Ptri : 0;
    const long npr = obs ? (long)obs->npair * obs->npair * Mo2 : 0;
    cplx *d_two = nullptr, *d_C = nullptr, *d_xwg = nullptr, *d_spin = nullptr, *d_pair = nullptr;
    int* d_maps = nullptr;
    if (n2) {
      SFQ_CUDA_TRY(cudaMallocAsync((void**)&d_two, sizeof(cplx) * n2, st));
      SFQ_CUDA_TRY(cudaMallocAsync((void**)&d_C, sizeof(cplx) * M4, st));
      SFQ_CUDA_TRY(cudaMallocAsync((void**)&d_xwg, sizeof(cplx) * (size_t)W * ns * MM, st));
      SFQ_CUDA_TRY(cudaMemsetAsync(d_two, 0, sizeof(cplx) * n2, st));
    }
    if (ns_sp) {
      SFQ_CUDA_TRY(cudaMallocAsync((void**)&d_spin, sizeof(cplx) * ns_sp, st));
      SFQ_CUDA_TRY(cudaMemsetAsync(d_spin, 0, sizeof(cplx) * ns_sp, st));
    }
    if (npr) {
      SFQ_CUDA_TRY(cudaMallocAsync((void**)&d_pair, sizeof(cplx) * npr, st));
      SFQ_CUDA_TRY(cudaMemsetAsync(d_pair, 0, sizeof(cplx) * npr, st));
      SFQ_CUDA_TRY(cudaMallocAsync((void**)&d_maps, sizeof(int) * (size_t)obs->npair * M, st));
      SFQ_CUDA_TRY(cudaMemcpyAsync(d_maps, obs->maps, sizeof(int) * (size_t)obs->npair * M, cudaMemcpyHostToDevice, st));
    }
    struct StreamFree {  // the observables' buffers go back to the pool on every way out
      cudaStream_t st;
      std::vector<void*> p;
      ~StreamFree() {
        for (void* q : p)
          if (q) cudaFreeAsync(q, st);
      }
    } obs_bufs{st, {d_two, d_C, d_xwg, d_spin, d_pair, d_maps}};
    const cplx* shift = bp ? nullptr : props + (long)P_OVLP * W;
    const cplx* B = bp ? bp_SMN : SM;
    std::vector<cplx> cic(ndet, mk(1.0, 0.0));
    for (int d = 0; d < ndet && ndet > 1; ++d) cic[d] = cconj(ci_h[d]);
    // determinant d's overlap matrices (one determinant per spin, not doubled; the time-evolved
    // estimator doubles CLOSED ones, TimeEvolvedBPEstimator.hpp:84-92), inverses in T
    const bool te_md = te && ndet > 1;
    auto factor = [&](int d, bool invert) -> int {
      if (!bp) return md_factor(d, SM, W, ovd + (long)d * W, invert, te ? ov_scale() : 1.0);
      GemmDesc g;  // T = Refs^H SMN, per walker (density_matrix.hpp:158-195)
      g.M = N; g.N = N; g.K = Mr; g.batch = W;
      g.A = bp_refs + (long)d * W * RN; g.sAm = 1; g.sAk = N; g.sAb = RN; g.a_cplx = true; g.conj_a = true;
      g.B = bp_SMN; g.sBk = N; g.sBn = 1; g.sBb = RN; g.b_cplx = true;
      g.C = T; g.sCm = N; g.sCn = 1; g.sCb = (long)N * N;
      int r;
      if ((r = gemm_f64(g, st))) return r;
      if ((r = ops::mask_cross_spin(T, W, N, spin_split(), st))) return r;
      if ((r = lu_logdet(T, (long)N * N, W, N, ovd + (long)d * W, false, 1.0, invert, st))) return r;
      bp_ov_kernel<<<(W + 127) / 128, 128, 0, st>>>(ovd + (long)d * W, bp_ldet + (long)d * W, ov_scale(), W);
      SFQ_LAUNCHED();
      return SFQ_OK;
    };
    for (int d = 0; d < ndet && (!te || te_md); ++d)
      if ((rc = factor(d, false))) return rc;
    if (!te || te_md) {
      cplx* dcic = nullptr;
      SFQ_CUDA_TRY(cudaMallocAsync((void**)&dcic, sizeof(cplx) * ndet, st));
      SFQ_CUDA_TRY(cudaMemcpyAsync(dcic, cic.data(), sizeof(cplx) * ndet, cudaMemcpyHostToDevice, st));
      rdm_tot_kernel<<<(W + 127) / 128, 128, 0, st>>>(ovd, dcic, shift, ndet, W, tot);
      SFQ_LAUNCHED();
      SFQ_CUDA_TRY(cudaFreeAsync(dcic, st));
      SFQ_CUDA_TRY(cudaStreamSynchronize(st));  // cic lives until the copy is done
    }
    for (int d = 0; d < ndet; ++d) {
      if (te && !te_md) {  // the operators' dressed G, a single determinant: coefficient 1
        if ((rc = te_green(Gf))) return rc;
        SFQ_CUDA_TRY(cudaMemcpyAsync(wc, weight, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st));
      }
      if ((!te || te_md) && (rc = factor(d, true))) return rc;
      if ((!te || te_md) && (rc = ops::green_compact(T, B, G, W, Mr, N, st))) return rc;
      if (te_md) {  // reference d's dressed G (constructTimeEvolvedMeasurementInputs) and coefficient
        if ((rc = te_green(Gf, d))) return rc;
        rdm_coeff_kernel<<<(W + 127) / 128, 128, 0, st>>>(ovd + (long)d * W, cic[d], shift, tot, weight, W, wc);
        SFQ_LAUNCHED();
      }
      // the full G of each spin block: Gf[w][s] = Aeff[rows s]^T Gc[w][rows s] (density_matrix.hpp:580-600),
      // Aeff = PsiT_d (shared) or the walker's conj(Refs^T)
      for (int s = 0; s < ns && !te; ++s) {
        const int r0 = collinear ? (s == 0 ? 0 : nup) : 0, r1 = collinear ? (s == 0 ? nup : N) : N;
        if (r1 == r0) {  // an empty spin sector has a zero G
          SFQ_CUDA_TRY(cudaMemset2DAsync(Gf + s * MM, sizeof(cplx) * ns * MM, 0, sizeof(cplx) * MM, W, st));
          continue;
        }
        GemmDesc g;
        g.M = Mr; g.N = Mr; g.K = r1 - r0; g.batch = W;
        if (bp) {
          g.A = bp_refs + (long)d * W * RN + r0; g.sAm = N; g.sAk = 1; g.sAb = RN; g.conj_a = true;
        } else {
          g.A = PsiT + d * RN + (long)r0 * Mr; g.sAm = 1; g.sAk = Mr; g.sAb = 0;
        }
        g.a_cplx = true;
        g.B = G + (long)r0 * Mr; g.sBk = Mr; g.sBn = 1; g.sBb = RN; g.b_cplx = true;
        g.C = Gf + s * MM; g.sCm = Mr; g.sCn = 1; g.sCb = ns * MM;
        if ((rc = gemm_f64(g, st))) return rc;
      }
      if (!te) {
        rdm_coeff_kernel<<<(W + 127) / 128, 128, 0, st>>>(ovd + (long)d * W, cic[d], shift, tot, weight, W, wc);
        SFQ_LAUNCHED();
      }
      GemmDesc g;  // one[s,i,j] += sum_w wc[w] Gf[w,s,i,j] (onerdm.hpp:56-61)
      g.M = 1; g.N = int(ns * MM); g.K = W; g.batch = 1;
      g.A = wc; g.sAm = W; g.sAk = 1; g.a_cplx = true;
      g.B = Gf; g.sBk = ns * MM; g.sBn = 1; g.b_cplx = true;
      g.C = o1; g.sCm = ns * MM; g.sCn = 1; g.beta = mk(1.0, 0.0);
      if ((rc = gemm_f64(g, st))) return rc;
      const long tot2 = nb * MM;
      rdm_two_kernel<<<int(std::min<long>((tot2 + 127) / 128, 1184)), 128, 0, st>>>(Gf, wc, W, ns, Mr, nb, o2);
      SFQ_LAUNCHED();
      if (n2) {  // avg blocks (a,a,a,a), (a,a,b,b), (b,b,b,b): C = sum_w (wc G_s)[w] (x) G_s'[w], one GEMM each
        scale_walker_rows_kernel<<<1184, 256, 0, st>>>(Gf, wc, ns * MM, W, d_xwg);
        SFQ_LAUNCHED();
        for (int blk = 0; blk <= ns; ++blk) {  // (TwoRDM runs for npol = 1 only: MM = M^2 here)
          const bool same = blk % 2 == 0;
          const int s1 = same ? blk / 2 : 0, s2 = same ? blk / 2 : ns - 1;
          GemmDesc g;
          g.M = int(MM); g.N = int(MM); g.K = W; g.batch = 1;
          g.A = d_xwg + s1 * MM; g.sAm = 1; g.sAk = ns * MM; g.a_cplx = true;
          g.B = Gf + s2 * MM; g.sBk = ns * MM; g.sBn = 1; g.b_cplx = true;
          g.C = d_C; g.sCm = MM; g.sCn = 1;
          if ((rc = gemm_f64(g, st))) return rc;
          twordm_block_kernel<<<1184, 256, 0, st>>>(d_C, M, same ? 1 : 0, d_two + blk * M4);
          SFQ_LAUNCHED();
        }
      }
      if (ns_sp) {
        spincorr_kernel<<<dim3((M + 127) / 128, M), 128, 0, st>>>(Gf, wc, W, M, kind, d_spin);
        SFQ_LAUNCHED();
      }
      if (npr) {
        paircorr_kernel<<<int(std::min<long>((npr + 127) / 128, 1184)), 128, 0, st>>>(Gf, wc, W, M, kind, obs->npair,
                                                                                       d_maps, d_pair);
        SFQ_LAUNCHED();
      }
    }
    if (obs) {
      obs->two.assign(n2, mk(0.0, 0.0));
      obs->spin.assign(ns_sp, mk(0.0, 0.0));
      obs->pair.assign(npr, mk(0.0, 0.0));
      if (n2) SFQ_CUDA_TRY(cudaMemcpyAsync(obs->two.data(), d_two, sizeof(cplx) * n2, cudaMemcpyDeviceToHost, st));
      if (ns_sp) SFQ_CUDA_TRY(cudaMemcpyAsync(obs->spin.data(), d_spin, sizeof(cplx) * ns_sp, cudaMemcpyDeviceToHost, st));
      if (npr) SFQ_CUDA_TRY(cudaMemcpyAsync(obs->pair.data(), d_pair, sizeof(cplx) * npr, cudaMemcpyDeviceToHost, st));
    }
    one.resize(ns * MM);
    two.resize(nb * MM);
    std::vector<cplx> pw(W);
    SFQ_CUDA_TRY(cudaMemcpyAsync(one.data(), o1, sizeof(cplx) * ns * MM, cudaMemcpyDeviceToHost, st));
    SFQ_CUDA_TRY(cudaMemcpyAsync(two.data(), o2, sizeof(cplx) * nb * MM, cudaMemcpyDeviceToHost, st));
    SFQ_CUDA_TRY(cudaMemcpyAsync(pw.data(), weight, sizeof(cplx) * W, cudaMemcpyDeviceToHost, st));
    if ((rc = sync_checked())) return rc;
    cplx den = mk(0.0, 0.0);
    for (int w = 0; w < W; ++w) den = mk(den.x + pw[w].x, den.y + pw[w].y);  // MeasurementOutput's denominator
    const double dd = den.x * den.x + den.y * den.y;
    auto divide = [&](std::vector<cplx>& v) {
      for (auto& z : v) z = mk((z.x * den.x + z.y * den.y) / dd, (z.y * den.x - z.x * den.y) / dd);
    };
    divide(one);
    divide(two);
    if (obs) {
      divide(obs->two);
      divide(obs->spin);
      divide(obs->pair);
    }
    return SFQ_OK;
  }

  // --- NOMSD::MixedDensityMatrix (compact, CLOSED: Ov x 2) into G, ov (W; may be null) ------
  int density(cplx* ov) {
    int rc;
    if ((rc = ensure_inverse(ov))) return rc;
    return ops::green_compact(T, SM, G, W, Mr, N, st);
  }

  // G for the force bias in the mixed mode: G[w][a][k] = sum_b Tinv[b][a] SM[k][b] as split-BF16
  // products, rows (c, a) of the block [[Tr, -Ti], [Ti, Tr]] against SM read as reals (K = (b, c')
  // interleaved), written straight into the planar planes of the vbias operand.  The FP64 G of
  // density() serves the energy; the force bias only ever saw G through these planes.
  bool mixed_green() const { return (N % 4) == 0; }
  int density_mixed() {
    int rc;
    if ((rc = ensure_inverse(nullptr))) return rc;
    if (!mixed_green()) {
      if ((rc = ops::green_compact(T, SM, G, W, M, N, st))) return rc;
      return mixed_split_planar(G, W, (long)N * M, Gs_p, st);
    }
    if ((rc = mixed_build_tblk(T, W, N, Tb_p, st))) return rc;
    // the walkers' planes for this product and, in the same pass, the walker rows of the P1
    // product later in the step (the walkers do not change in between)
    if ((rc = mixed_walkers_split_both(SM, W, M, N, ldh, Ws_p, Wt_p, st))) return rc;
    UmmaEpilogue eg;
    eg.kind = UMMA_EPI_PLANAR_SPLIT;
    eg.nel = N;
    eg.nmo = M;
    for (int q = 0; q < 3; ++q) eg.out[q] = Gs_p[q];
    eg.out_planes = nplanes;
    return tc_gemm(Tb_p, 2L * N, 4L * N * N, Ws_p, M, 2L * M * N, 2 * N, W, nullptr, 0, 0, 1.f, g_tile(), &eg);
  }

  // NOMSD::Overlap of the current walkers into ov; keeps their inverse overlap matrices in T
  int log_overlap(cplx* ov) {
    int rc;
    const void* A = trial_real ? (const void*)PsiTr : (const void*)PsiT;
    inv_cached = false;
    if ((rc = ops::overlap_matrix(A, !trial_real, SM, T, W, Mr, N, st))) return rc;
    if ((rc = ops::mask_cross_spin(T, W, N, spin_split(), st))) return rc;
    if ((rc = lu_logdet(T, (long)N * N, W, N, ov, false, ov_scale(), true, st))) return rc;
    inv_cached = true;
    inv_ov = ov;
    return SFQ_OK;
  }

  // --- AFQMCBasePropagator::Propagate (hybrid) ----------------------------------------------
  int propagate(double Eshift, unsigned long long step, const double* uniforms) {
    if (mixed) return propagate_mixed(Eshift, step, uniforms);
    int rc;
    if (ndet > 1) {
      ph_begin(SFQ_PH_VBIAS);
      if ((rc = vbias_md(X))) return rc;                                              // 1. G, vbias
      ph_end(SFQ_PH_VBIAS);
    } else {
      ph_begin(SFQ_PH_DENSITY);
      if ((rc = density(nullptr))) return rc;                                        // 1. G
      ph_end(SFQ_PH_DENSITY);
      ph_begin(SFQ_PH_VBIAS);
      if ((rc = ops::vbias(G, Lnak, !trial_real, X, W, N, Mr, Nc, vb_scale(), st))) return rc;
      ph_end(SFQ_PH_VBIAS);
    }
    ph_begin(SFQ_PH_FIELDS);
    FieldParams fp;                                                                   // 2. X
    fp.nwalk = W; fp.nchol = Nc; fp.vbias_bound = p.vbias_bound; fp.free_projection = p.free_projection;
    fp.seed = p.seed; fp.step = step; fp.uniforms = uniforms; fp.step_dev = dev_mode ? d_step : nullptr;
    if (uni_wait) {
      SFQ_CUDA_TRY(cudaStreamWaitEvent(st, uni_wait, 0));
      uni_wait = nullptr;
    }
    if ((rc = assemble_x(X, vmf, hw, mf, fp, st))) return rc;
    if (nbp && dev_mode) {  // storeFields (AFQMCBasePropagator.cpp:342-344): the fields into the ring slot
      store_fields_kernel<<<int(std::min<long>(((long)W * Nc + 255) / 256, 1184)), 256, 0, st>>>(X, bp_fields, nbp, Nc, W,
                                                                                                 d_step + 1);
      SFQ_LAUNCHED();
    } else if (nbp) {
      SFQ_CUDA_TRY(cudaMemcpy2DAsync(bp_fields + (long)(hist_pos % nbp) * Nc, sizeof(cplx) * nbp * Nc, X,
                                     sizeof(cplx) * Nc, sizeof(cplx) * Nc, W, cudaMemcpyDeviceToDevice, st));
    }
    ph_end(SFQ_PH_FIELDS);
    ph_begin(SFQ_PH_VHS);
    ph_begin(SFQ_PH_VHS_GEMM);
    if (sym) {                                                                        // 3. vHS
      if ((rc = ops::vhs_rows(Lp, P, X, Vp, W, Nc, std::sqrt(p.dt), st))) return rc;
    } else {
      if ((rc = ops::vhs(Likn, X, V, W, M, Nc, std::sqrt(p.dt), st))) return rc;
    }
    ph_end(SFQ_PH_VHS_GEMM);
    if (sym && (rc = unpack_symmetric(Vp, W, M, V, st))) return rc;
    ph_end(SFQ_PH_VHS);
    ph_begin(SFQ_PH_PROPAGATE);
    inv_cached = false;
    if ((rc = ops::propagate(SM, P1, false, V, W, M, N, p.taylor_order, TMN, T1, T2, st, npol))) return rc;  // 4.
    ph_end(SFQ_PH_PROPAGATE);
    ph_begin(SFQ_PH_OVERLAP);
    if ((rc = ndet > 1 ? log_overlap_md(newov) : log_overlap(newov))) return rc;      // 5.
    ph_end(SFQ_PH_OVERLAP);
    ph_begin(SFQ_PH_UPDATE);
    UpdateParams up;                                                                  // 6.+7.
    up.nwalk = W; up.dt = p.dt; up.Eshift = Eshift; up.E0 = p.E0;
    up.lower_cutoff = p.lower_cutoff_scale; up.upper_cutoff = p.upper_cutoff_scale;
    up.max_weight = std::fmax(p.weight_bound_floor, p.weight_bound_fraction * target_pop());
    up.hybrid = 1; up.free_projection = p.free_projection; up.use_cp_constraint = 0;
    up.Eshift_dev = dev_mode ? d_eshift : nullptr;
    if (nbp) {  // the step's weight factors into the history slot (WalkerSetUpdate.hpp:184-188)
      up.wfac = bp_wfac + (dev_mode ? 0 : hist_pos);
      up.wfac_pos = dev_mode ? d_step + 1 : nullptr;
      up.wfac_stride = nhist;
    }
    if ((rc = walker_update(wprops(), newov, mf, hw, E3, up, stats, st))) return rc;
    if (nbp && dev_mode) {  // advanceHistoryPos; a block's host position moves when it is launched
      hist_advance_kernel<<<1, 1, 0, st>>>(d_step + 1, nhist);
      SFQ_LAUNCHED();
    } else if (nbp) {
      hist_pos = (hist_pos + 1) % nhist;
    }
    ph_end(SFQ_PH_UPDATE);
    return SFQ_OK;
  }

  // tile shapes of the mixed products, fixed by the sizes
  void plan_mixed() {
    // Taylor tiles: `tay_half` orbitals, re and im halves side by side (tile width 2 * half, a
    // tile width the GEMM is built with); the least padding of M, then the widest tile
    int best = 0;
    long best_pad = 1L << 40;
    for (int h : {16, 32, 64, 80, 128}) {
      if (h == 128 && nplanes > 2) continue;
      if (tay_req && h != tay_req) continue;
      const long pad = (long)((M + h - 1) / h) * h;
      if (pad < best_pad || (pad == best_pad && h > best)) {
        best = h;
        best_pad = pad;
      }
    }
    tay_half = best;
    vb_rows = 2 * best_pad;
    ldh = (M + 63) / 64 * 64;
    vb_ks = vb_ks_req ? vb_ks_req : plan_ks(vb_bn);
    vb_ks_max = 1;
    for (int bn : {32, 64, 128, 160, 208, 256}) vb_ks_max = std::max(vb_ks_max, plan_ks(bn));  // every width set_tiles takes
  }

  // vbias: tiles of width bn over (2W, Nc), K = N*M split so that the work units fill whole waves
  // of SMs (K splits write partial sums, reduced in a fixed order)
  // (the smallest split reaching min_eff of whole waves when min_eff < 1: fewer partial sums to write
  // and add, a little wave quantization traded for it)
  int plan_ks(int bn, double min_eff = 0.999) const {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device);
    const long tiles = (long)((2 * W + 127) / 128) * ((Nc + bn - 1) / bn);
    const long kt = ((long)N * M + 63) / 64;
    double best_eff = 0.0;
    int best = 1;
    for (int ks = 1; ks <= 64 && ks * 8 <= kt; ++ks) {
      const double units = double(tiles) * ks;
      const double eff = units / (std::ceil(units / sms) * sms);
      if (eff > best_eff + 1e-9) {
        best_eff = eff;
        best = ks;
      }
      if (eff > min_eff) break;
    }
    return best;
  }

  // tile width of the P1 products (M columns): little padding, and a tile width built for the planes
  int p1_tile() const { return p1_bn ? p1_bn : (M <= 128 ? 128 : (nplanes > 2 ? 160 : 208)); }
  int g_tile() const { return g_bn ? g_bn : p1_tile(); }

  // C = alpha * A B^T on split planes (A: rows x K, B: cols x K, both K-major; rows a_ld apart,
  // K when 0)
  int tc_gemm(void* const* A, long a_rows, long a_bs, void* const* B, long b_rows, long b_bs, int K, int batch,
              float* C, long ldc, long sCb, float alpha, int bn = 0, const UmmaEpilogue* epi = nullptr,
              int ksplit = 1, long sCk = 0, long a_ld = 0) {
    UmmaGemmDesc d;
    d.M = int(a_rows); d.N = int(b_rows); d.K = K; d.batch = batch;
    for (int q = 0; q < 3; ++q) {
      d.A.p[q] = A[q];
      d.B.p[q] = B[q];
    }
    d.A.rows = a_rows; d.A.ld = a_ld ? a_ld : K; d.A.batch_stride = a_bs;
    d.B.rows = b_rows; d.B.ld = K; d.B.batch_stride = b_bs;
    d.C = C; d.ldc = ldc; d.sCb = sCb; d.alpha = alpha; d.nplanes = nplanes; d.bn = bn; d.err = gemm_err;
    d.ksplit = ksplit; d.sCk = sCk;
    if (epi) d.epi = *epi;
    return umma_gemm(d, st);
  }

  // ---- autotuner: the tile widths of the mixed products, timed on the engine's own operands ----
  // Product index: 0 G (density), 1 vbias (with its K-split reduction), 2 vHS, 3 one Taylor term,
  // 4 the two P1 products.  The choice changes only how the output is tiled, and for vbias in how
  // many K ranges the sum is split, so results of two engines with the same tiles are identical.
  static constexpr int kTunedProducts = 5;

  bool tile_built(int bn) const {
    if (bn == 32 || bn == 64 || bn == 128 || bn == 160) return true;
    return (bn == 208 || bn == 256) && nplanes <= 2;
  }
  bool half_ok(int h) const { return h == 16 || h == 32 || h == 64 || h == 80 || (h == 128 && nplanes <= 2); }

  // set the tiles (0: the built-in choice); the captured block graphs are dropped
  int set_tiles(int gbn, int vbbn, int vhsbn, int half, int p1bn, int vbks = 0) {
    if (!mixed) return record_error(SFQ_ERR_UNSUPPORTED, "tiles: only the mixed-precision products are tiled");
    if (nslices) return set_tiles_i8(gbn, vbbn, vhsbn, half, p1bn, vbks);
    for (int bn : {gbn, vbbn, vhsbn, p1bn})
      if (bn && !tile_built(bn))
        return record_error(SFQ_ERR_ARG, "tiles: width %d is not built for %d planes", bn, nplanes);
    if (half && !half_ok(half)) return record_error(SFQ_ERR_ARG, "tiles: Taylor half %d not built", half);
    const long kt = ((long)N * M + 63) / 64;
    if (vbks < 0 || vbks > vb_ks_max || vbks > kt)
      return record_error(SFQ_ERR_ARG, "tiles: force-bias K split %d outside 0..%d", vbks,
                          int(vb_ks_max < kt ? vb_ks_max : kt));
    vb_ks_req = vbks;
    g_bn = gbn;
    vb_bn = vbbn ? vbbn : 128;
    vhs_bn = vhsbn;
    p1_bn = p1bn;
    tay_req = half;
    plan_mixed();
    drop_graphs();
    return SFQ_OK;
  }

  void drop_graphs() {
    if (st) cudaStreamSynchronize(st);
    for (auto& kv : graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    graphs.clear();
  }

  // the int8-slice products: only the Taylor term's orbitals per tile are a choice (32, 64 or 80;
  // 0 = the planned one, the least padding of M); the other widths are fixed (0 or their value)
  int set_tiles_i8(int gbn, int vbbn, int vhsbn, int half, int p1bn, int vbks) {
    if (gbn || (vbbn && vbbn != i8_vb_bn) || (vhsbn && vhsbn != i8_bn) || (p1bn && p1bn != i8_bn) ||
        (vbks && vbks != i8_vb_ks))
      return record_error(SFQ_ERR_ARG, "tiles: the int8-slice products only tile the Taylor term (orbitals per tile)");
    if (half && half != 32 && half != 64 && half != 80)
      return record_error(SFQ_ERR_ARG, "tiles: Taylor half %d not built for int8 slices", half);
    i8_half_req = half;
    plan_i8();
    drop_graphs();
    return SFQ_OK;
  }

  void get_tiles(sfq_tiles_t* t) const {
    if (nslices) {
      t->g_bn = 0;  // G is FP64
      t->vbias_bn = i8_vb_bn;
      t->vhs_bn = i8_bn;
      t->taylor_half = i8_half;
      t->p1_bn = i8_bn;
      t->vbias_ksplit = i8_vb_ks;
      return;
    }
    t->g_bn = g_tile();
    t->vbias_bn = vb_bn;
    t->vhs_bn = vhs_bn ? vhs_bn : 128;
    t->taylor_half = tay_half;
    t->p1_bn = p1_tile();
    t->vbias_ksplit = vb_ks;
  }

  // median over `reps` launches of f (us), after two warm-up launches, by events on the engine stream
  template <class F>
  int time_median(F&& f, int reps, double* us) {
    int rc;
    for (int i = 0; i < 2; ++i)
      if ((rc = f())) return rc;
    std::vector<cudaEvent_t> ev(reps + 1, nullptr);
    cudaError_t ce = cudaSuccess;
    for (auto& x : ev)
      if (ce == cudaSuccess) ce = cudaEventCreate(&x);
    rc = ce == cudaSuccess ? SFQ_OK : record_cuda(ce, "cudaEventCreate", __FILE__, __LINE__);
    if (!rc) ce = cudaEventRecord(ev[0], st);
    for (int i = 0; i < reps && !rc && ce == cudaSuccess; ++i) {
      rc = f();
      if (!rc) ce = cudaEventRecord(ev[i + 1], st);
    }
    if (!rc && ce == cudaSuccess) ce = cudaEventSynchronize(ev[reps]);
    if (!rc && ce != cudaSuccess) rc = record_cuda(ce, "autotune events", __FILE__, __LINE__);
    std::vector<double> t(reps, 0.0);
    for (int i = 0; i < reps && !rc; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
      t[i] = 1e3 * ms;
    }
    for (auto& x : ev)
      if (x) cudaEventDestroy(x);
    if (rc) return rc;
    std::sort(t.begin(), t.end());
    *us = t[reps / 2];
    return SFQ_OK;
  }

  // the products with tile width bn (Taylor: half) on the operands the scratch buffers hold
  int tune_product(int which, int bn, int vbks = 0) {
    int rc;
    const long NM = (long)N * M, L2h = 2L * ldh, rows = 2L * W * N;
    switch (which) {
      case 0: {
        UmmaEpilogue eg;
        eg.kind = UMMA_EPI_PLANAR_SPLIT;
        eg.nel = N;
        eg.nmo = M;
        for (int q = 0; q < 3; ++q) eg.out[q] = Gs_p[q];
        eg.out_planes = nplanes;
        return tc_gemm(Tb_p, 2L * N, 4L * N * N, Ws_p, M, 2L * M * N, 2 * N, W, nullptr, 0, 0, 1.f, bn, &eg);
      }
      case 1: {
        const int ks = vbks ? vbks : plan_ks(bn);
        const long part = 2L * W * Nc;
        if ((rc = tc_gemm(Gs_p, 2L * W, 0, Lnak_p, Nc, 0, int(NM), 1, Cvb, Nc, 0, 1.f, bn, nullptr, ks, part)))
          return rc;
        return mixed_reduce_planar_to_cplx(Cvb, ks, part, W, Nc, 2.0 * std::sqrt(p.dt), X, st);
      }
      case 2: {
        const long vcols = sym ? P : (long)M * M;
        return tc_gemm(Xs_p, 2L * W, 0, Likn_p, vcols, 0, Nc, 1, Cv, vcols, 0, float(std::sqrt(p.dt)), bn);
      }
      case 3: {
        UmmaGemmDesc d;
        d.M = N; d.N = int(2L * ((M + bn - 1) / bn) * bn); d.K = int(L2h); d.batch = W;
        for (int q = 0; q < 3; ++q) {
          d.A.p[q] = Wt2_p[q];
          d.B.p[q] = Vb_p[q];
        }
        d.A.rows = N; d.A.ld = L2h; d.A.batch_stride = long(N) * L2h;
        d.B.rows = 2L * M; d.B.ld = M; d.B.batch_stride = 2L * M * M;
        d.cplx_half = bn; d.cplx_nmo = M; d.cplx_ldh = ldh;
        d.nplanes = nplanes; d.bn = 2 * bn; d.err = gemm_err;
        UmmaEpilogue& et = d.epi;
        et.kind = UMMA_EPI_TAYLOR;
        et.S = Sacc; et.nmo = M; et.ldh = ldh; et.half = bn; et.inv_k = 1.f;
        et.write = 1;
        for (int q = 0; q < 3; ++q) et.out[q] = Wt_p[q];
        et.out_planes = nplanes;
        return umma_gemm(d, st);
      }
      default: {
        UmmaEpilogue e1;
        e1.kind = UMMA_EPI_STORE_SPLIT;
        for (int q = 0; q < 3; ++q) e1.out[q] = Wt2_p[q];
        e1.out_planes = nplanes;
        e1.ldh = ldh;
        if ((rc = tc_gemm(Wt_p, rows, 0, P1_p, M, 0, M, 1, Sacc, M, 0, 1.f, bn, &e1, 1, 0, ldh))) return rc;
        UmmaEpilogue ew;  // into the scratch walker buffer: the walkers are not touched
        ew.kind = UMMA_EPI_TO_WALKERS;
        ew.SM = reinterpret_cast<double*>(SM2);
        ew.nel = N;
        return tc_gemm(Wt2_p, rows, 0, P1_p, M, 0, M, 1, nullptr, 0, 0, 1.f, bn, &ew, 1, 0, ldh);
      }
    }
  }

  // time every built tile width of each product on this engine's sizes and keep the fastest; the
  // walkers, their weights and overlaps are not modified (only scratch buffers are written)
  int autotune(int reps, sfq_tiles_t* out) {
    if (!mixed) return record_error(SFQ_ERR_UNSUPPORTED, "autotune: only the mixed-precision products are tiled");
    const bool prof = profile;
    profile = false;
    const int rc = nslices ? autotune_i8(reps < 1 ? 9 : reps, out) : autotune_run(reps < 1 ? 9 : reps, out);
    profile = prof;
    return rc;
  }

  // the int8-slice Taylor product at each built width (exact accumulation: every width gives the
  // same results bit for bit), on real operands: the step's stages up to the first Taylor term
  // (they write only per-step scratch, not the walkers or their properties)
  int autotune_i8(int reps, sfq_tiles_t* out) {
    int rc;
    IsliceGemmDesc d;
    bool more = true;
    for (int s = 0; more; ++s) {  // up to the first Taylor product
      if ((rc = propagate_i8_next(s, 0.0, 0, nullptr, &d, &more))) return rc;
      if (d.cplx_half > 0) break;
      if (more && (rc = islice_gemm(d, st))) return rc;
    }
    const int planned = i8_half;
    double t_cur = 0.0, best = 1e300;
    int chosen = planned;
    for (int h : {32, 64, 80}) {
      i8_half = h;
      const IsliceGemmDesc dt = i8_taylor(i8_cur);
      double us = 0.0;
      if ((rc = time_median([&] { return islice_gemm(dt, st); }, reps, &us))) {
        i8_half = planned;
        return rc;
      }
      if (h == planned) t_cur = us;
      if (us < best) {
        best = us;
        chosen = h;
      }
    }
    i8_half = planned;
    if ((rc = sync_checked())) return rc;
    if ((rc = set_tiles_i8(0, 0, 0, chosen, 0, 0))) return rc;
    if (out) {
      get_tiles(out);
      for (int i = 0; i < kTunedProducts; ++i) out->us_builtin[i] = out->us_tuned[i] = 0.0;
      out->us_builtin[3] = t_cur;
      out->us_tuned[3] = best;
    }
    return SFQ_OK;
  }

  int autotune_run(int reps, sfq_tiles_t* out) {
    int rc;
    // real operands in the scratch buffers: G planes, force bias, its planes, vHS and V, walker planes
    const double sdt = std::sqrt(p.dt);
    const long part = 2L * W * Nc;
    const long vcols = sym ? P : (long)M * M;
    if ((rc = density_mixed())) return rc;
    if ((rc = tc_gemm(Gs_p, 2L * W, 0, Lnak_p, Nc, 0, int((long)N * M), 1, Cvb, Nc, 0, 1.f, vb_bn, nullptr,
                      vb_ks, part)))
      return rc;
    if ((rc = mixed_reduce_planar_to_cplx(Cvb, vb_ks, part, W, Nc, 2.0 * sdt, X, st))) return rc;
    if ((rc = mixed_split_planar(X, W, Nc, Xs_p, st))) return rc;
    if ((rc = tc_gemm(Xs_p, 2L * W, 0, Likn_p, vcols, 0, Nc, 1, Cv, vcols, 0, float(sdt), vhs_bn))) return rc;
    if ((rc = mixed_build_v(Cv, W, M, sym, Vb_p, st))) return rc;
    if ((rc = mixed_walkers_to_wt(SM, W, M, N, ldh, Wt_p, st))) return rc;
    if ((rc = tune_product(4, p1_tile()))) return rc;
    sfq_tiles_t cur{};
    get_tiles(&cur);
    const int current[kTunedProducts] = {cur.g_bn, cur.vbias_bn, cur.vhs_bn, cur.taylor_half, cur.p1_bn};
    int chosen[kTunedProducts];
    int chosen_ks = cur.vbias_ksplit;
    double t_cur[kTunedProducts] = {}, t_best[kTunedProducts] = {};
    for (int which = 0; which < kTunedProducts; ++which) {
      // candidates (width, force-bias K split; 0 elsewhere)
      std::vector<std::pair<int, int>> cand;
      if (which == 3) {
        for (int h : {16, 32, 64, 80, 128})
          if (half_ok(h)) cand.push_back({h, 0});
      } else {
        for (int bn : {64, 128, 160, 208, 256}) {
          if (!tile_built(bn)) continue;
          if (which != 1) {
            cand.push_back({bn, 0});
            continue;
          }
          // the split that fills whole waves, and the smallest one within 6 % of it
          const int k1 = plan_ks(bn), k2 = plan_ks(bn, 0.94);
          cand.push_back({bn, k1});
          if (k2 != k1) cand.push_back({bn, k2});
        }
      }
      chosen[which] = current[which];
      if (which == 0 && !mixed_green()) continue;  // G comes from the FP64 density
      double best = 1e300;
      for (const auto& c : cand) {
        double us = 0.0;
        if ((rc = time_median([&] { return tune_product(which, c.first, c.second); }, reps, &us))) return rc;
        if (c.first == current[which] && (which != 1 || c.second == cur.vbias_ksplit)) t_cur[which] = us;
        if (us < best) {
          best = us;
          chosen[which] = c.first;
          if (which == 1) chosen_ks = c.second;
        }
      }
      t_best[which] = best;
    }
    if ((rc = sync_checked())) return rc;
    if ((rc = set_tiles(chosen[0], chosen[1], chosen[2], chosen[3], chosen[4], chosen_ks))) return rc;
    if (out) {
      get_tiles(out);
      for (int i = 0; i < kTunedProducts; ++i) {
        out->us_builtin[i] = t_cur[i];
        out->us_tuned[i] = t_best[i];
      }
    }
    return SFQ_OK;
  }

  // ---- exact-accumulation mode (int8 slices) ------------------------------------------------
  // slice rows start on 64-byte boundaries: a product's 64-byte K slice of a row is then exactly two
  // 32-byte sectors (rows 16 bytes apart made three of every such load)
  static long round64(long x) { return (x + 63) / 64 * 64; }
  // tile shapes of the int8-slice products: Taylor tiles of `half` orbitals (the least padding of
  // M, then the widest), the force bias split along K to fill whole waves of SMs
  void plan_i8() {
    ld_m = round64(M);
    ld_mr = round64(Mr);
    ld_nm = round64((long)N * Mr);
    ld_nc = round64(Nc);
    ld_mm = round64((long)M * M);
    int best = 0;
    long best_pad = 1L << 40;
    for (int h : {32, 64, 80}) {
      const long pad = (long)((M + h - 1) / h) * h;
      if (pad < best_pad || (pad == best_pad && h > best)) {
        best = h;
        best_pad = pad;
      }
    }
    i8_half = i8_half_req ? i8_half_req : best;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device);
    const long tiles = (long)((2 * W + 127) / 128) * ((Nc + i8_vb_bn - 1) / i8_vb_bn);
    const long kt = ((long)N * Mr + 127) / 128;
    double best_eff = 0.0;
    i8_vb_ks = 1;
    for (int ks = 1; ks <= 64 && ks * 4 <= kt; ++ks) {
      const double units = double(tiles) * ks;
      const double eff = units / (std::ceil(units / sms) * sms);
      if (eff > best_eff + 1e-9) {
        best_eff = eff;
        i8_vb_ks = ks;
      }
      if (eff > 0.999) break;
    }
    // multi-determinant force bias: K = M * M, split into ranges of at most 335 blocks of 128 (exact
    // int32 accumulation), then as for the single-determinant one to fill whole waves of SMs
    i8_md_ks = 1;
    if (ndet > 1) {
      const long ktm = ((long)M * M + 127) / 128;
      const int ks_min = int((ktm + 334) / 335);
      double be = -1.0;
      for (int ks = ks_min; ks <= 64 || ks == ks_min; ++ks) {
        const double units = double(tiles) * ks;
        const double eff = units / (std::ceil(units / sms) * sms);
        if (eff > be + 1e-9) {
          be = eff;
          i8_md_ks = ks;
        }
        if (eff > 0.999 || ks * 4 > ktm) break;
      }
    }
  }
  IsliceOperand i8_operand(int8_t* const* q, long rows, long ld, const int* e, long bstride = 0, long e_bs = 0,
                           long e_mod = 0) const {
    IsliceOperand o;
    for (int s2 = 0; s2 < 3; ++s2) o.q[s2] = q[s2];
    o.rows = rows; o.ld = ld; o.batch_stride = bstride; o.e = e; o.e_bs = e_bs; o.e_mod = e_mod;
    return o;
  }
  IsliceGemmDesc i8_desc() const {
    IsliceGemmDesc d;
    d.nslices = nslices;
    d.err = gemm_err;
    return d;
  }
  // C (2R, M) planar (+)= A (rows (c, r), one exponent per r) times (P1 - I)^T: the two P1 products,
  // whose identity part the caller adds
  IsliceGemmDesc i8_p1(int buf, float* C, bool accumulate) const {
    const long R = (long)W * npol * N;
    IsliceGemmDesc d = i8_desc();
    d.M = int(2 * R); d.N = M; d.K = M;
    d.A = i8_operand(A_q[buf], 2 * R, ld_m, A_e[buf], 0, 0, R);
    d.B = i8_operand(P1_q, M, ld_m, P1_e);
    d.bn = i8_bn;
    d.C = C; d.ldc = M; d.accumulate = accumulate;
    return d;
  }
  // one Taylor product of every walker: Cp = A [[Vr, -Vi], [Vi, Vr]]^T, planar [c][w][(q, a)][j]
  // (a NONCOLLINEAR walker's two components are one batch item of 2N rows against its V)
  IsliceGemmDesc i8_taylor(int buf) const {
    const long Nw = (long)npol * N, R = W * Nw;
    IsliceGemmDesc d = i8_desc();
    d.M = int(Nw); d.N = M; d.K = M; d.batch = W;
    d.A = i8_operand(A_q[buf], Nw, ld_m, A_e[buf], Nw * ld_m, Nw);
    for (int s2 = 0; s2 < 3; ++s2) d.a_im[s2] = A_q[buf][s2] ? A_q[buf][s2] + R * ld_m : nullptr;
    d.B = i8_operand(V_q, 3L * M, ld_m, V_e, 3L * M * ld_m, M);
    d.cplx_half = i8_half;
    d.C = Cp; d.ldc = M; d.sCc = R * M;
    return d;
  }

  // AFQMCBasePropagator::Propagate with the products from int8 slices (exact accumulation): force
  // bias, vHS, P1 and the Taylor terms on the tensor cores; the elementwise steps between them
  // (T = (i/k) C, S += T, slicing) round to nearest; G, LU / overlaps and the walker update in FP64.
  // The force bias is the trial's own (FP64, setup) plus that of G - G_trial from slices: G's rows
  // are dominated by entries near the trial's, which would set the fixed-point scale of the rest.
  //
  // Written as stages s = 0, 1, ...: stage s records its work on the stream and hands back, in *d,
  // the int8-slice product that follows it (not launched), *more = false after the last stage.  Run
  // alone, each product is launched right after its stage; a group of engines runs stage s of
  // every member, then all their products as one launch (Group::record_fused).
  int i8_cur = 0;  // Taylor operand buffer between stages
  // follow-up products of a stage, launched before the next stage: with a complex trial, Lnak's
  // imaginary rows Li make a force bias or exchange product C = [A_re; A_im] Lr^T complete only with
  // C_re -= A_im Li^T and C_im += A_re Li^T (accumulated into the same output, the same K splits)
  IsliceGemmDesc i8_queue[2];
  int i8_qn = 0, i8_qh = 0, i8_pst = 0, i8_est = 0;
  void i8_queue_cplx(const IsliceGemmDesc& d, long h, const IsliceOperand& Bi) {
    IsliceGemmDesc a = d, b = d;
    a.M = b.M = int(h);
    a.A.rows = b.A.rows = h;
    for (int t = 0; t < 3; ++t) a.A.q[t] = d.A.q[t] ? d.A.q[t] + h * d.A.ld : nullptr;  // A_im rows
    a.A.e = d.A.e + h;
    a.B = b.B = Bi;
    a.alpha = -d.alpha;
    a.accumulate = b.accumulate = true;
    b.C = d.C + h * d.ldc;
    i8_queue[0] = a;
    i8_queue[1] = b;
    i8_qh = 0;
    i8_qn = 2;
  }
  // the step's and the energy's products in order (stages and their follow-ups): call k = 0, 1, ...
  int propagate_i8_next(int k, double Eshift, unsigned long long step, const double* uniforms, IsliceGemmDesc* d,
                        bool* more) {
    if (k == 0) {
      i8_qn = 0;
      i8_pst = 0;
    }
    if (i8_qn > 0) {
      *d = i8_queue[i8_qh++];
      --i8_qn;
      *more = true;
      return SFQ_OK;
    }
    return propagate_i8_stage(i8_pst++, Eshift, step, uniforms, d, more);
  }
  int energy_i8_next(int k, IsliceGemmDesc* d, bool* more) {
    if (k == 0) {
      i8_qn = 0;
      i8_est = 0;
    }
    if (i8_qn > 0) {
      *d = i8_queue[i8_qh++];
      --i8_qn;
      *more = true;
      return SFQ_OK;
    }
    return energy_i8_stage(i8_est++, d, more);
  }
  int propagate_i8_stage(int s, double Eshift, unsigned long long step, const double* uniforms, IsliceGemmDesc* d,
                         bool* more) {
    int rc;
    const int Wb = W * npol;  // (M, N) walker blocks
    const long R = (long)Wb * N;
    const int order = p.taylor_order;
    *more = true;
    if (s == 0 && ndet > 1) {
      // NOMSD::vbias with ndet > 1: the ci-weighted full G (FP64), its difference from the trial's
      // sliced as planar rows over (i, k), against L; the trial's own force bias added back
      ph_begin(SFQ_PH_VBIAS);
      if ((rc = md_full_green())) return rc;
      if ((rc = islice_rows_planar(Racc, W, (long)M * M, nslices, Gf_q, ld_mm, Gf_e, st, RT_md, pl_emax))) return rc;
      *d = i8_desc();
      d->M = 2 * W; d->N = Nc; d->K = int((long)M * M);
      d->A = i8_operand(Gf_q, 2L * W, ld_mm, Gf_e);
      d->B = i8_operand(Lf_q, Nc, ld_mm, Lf_e);
      d->bn = i8_vb_bn; d->ksplit = i8_md_ks; d->sCk = 2L * W * Nc;
      d->C = Cvb; d->ldc = Nc;
      return SFQ_OK;
    }
    if (s == 0) {
      ph_begin(SFQ_PH_DENSITY);
      if ((rc = density(nullptr))) return rc;
      if ((rc = islice_rows_planar(G, W, (long)N * Mr, nslices, Gv_q, ld_nm, Gv_e, st, GT_c, pl_emax))) return rc;
      ph_end(SFQ_PH_DENSITY);
      ph_begin(SFQ_PH_VBIAS);
      *d = i8_desc();
      d->M = 2 * W; d->N = Nc; d->K = int((long)N * Mr);
      d->A = i8_operand(Gv_q, 2L * W, ld_nm, Gv_e);
      d->B = i8_operand(Lv_q, Nc, ld_nm, Lv_e);
      d->bn = i8_vb_bn; d->ksplit = i8_vb_ks; d->sCk = 2L * W * Nc;
      d->C = Cvb; d->ldc = Nc;
      if (!trial_real) {  // Lnak's imaginary rows follow its real ones
        int8_t* qi[3];
        for (int t = 0; t < 3; ++t) qi[t] = Lv_q[t] ? Lv_q[t] + (long)Nc * ld_nm : nullptr;
        i8_queue_cplx(*d, W, i8_operand(qi, Nc, ld_nm, Lv_e + Nc));
      }
      return SFQ_OK;
    }
    if (s == 1) {
      const int ks = ndet > 1 ? i8_md_ks : i8_vb_ks;
      if ((rc = mixed_reduce_planar_to_cplx(Cvb, ks, 2L * W * Nc, W, Nc, vb_scale(), X, st, vbT))) return rc;
      ph_end(SFQ_PH_VBIAS);
      ph_begin(SFQ_PH_FIELDS);
      FieldParams fp;
      fp.nwalk = W; fp.nchol = Nc; fp.vbias_bound = p.vbias_bound; fp.free_projection = p.free_projection;
      fp.seed = p.seed; fp.step = step; fp.uniforms = uniforms; fp.step_dev = dev_mode ? d_step : nullptr;
      if (uni_wait) {
        SFQ_CUDA_TRY(cudaStreamWaitEvent(st, uni_wait, 0));
        uni_wait = nullptr;
      }
      if ((rc = assemble_x(X, vmf, hw, mf, fp, st))) return rc;
      ph_end(SFQ_PH_FIELDS);
      ph_begin(SFQ_PH_VHS);
      if ((rc = islice_rows_planar(X, W, Nc, nslices, Xq_q, ld_nc, Xq_e, st))) return rc;
      ph_begin(SFQ_PH_VHS_GEMM);
      const long vcols = sym ? P : (long)M * M;
      *d = i8_desc();
      d->M = 2 * W; d->N = int(vcols); d->K = Nc;
      d->A = i8_operand(Xq_q, 2L * W, ld_nc, Xq_e);
      d->B = i8_operand(Lh_q, vcols, ld_nc, Lh_e);
      d->bn = i8_bn;
      d->C = Cv; d->ldc = vcols; d->alpha = std::sqrt(p.dt);
      return SFQ_OK;
    }
    if (s == 2) {
      ph_end(SFQ_PH_VHS_GEMM);
      if ((rc = islice_build_v(Cv, W, M, sym, nslices, V_q, ld_m, V_e, V_emax, st))) return rc;
      ph_end(SFQ_PH_VHS);
      ph_begin(SFQ_PH_PROPAGATE);
      inv_cached = false;
      // S = P1 W = W + (P1 - I) W; then T_k = (i/k) V T_{k-1}, S += T_k for k = 1..order; SM = S + (P1 - I) S
      if ((rc = islice_walkers(SM, Wb, M, N, nslices, A_q[0], ld_m, A_e[0], Sacc, st))) return rc;
      *d = i8_p1(0, Cp, false);
      return SFQ_OK;
    }
    if (s == 3) {
      if ((rc = islice_taylor_update(Cp, Sacc, R, M, 0, true, nslices, A_q[1], ld_m, A_e[1], st))) return rc;
      i8_cur = 1;
      ph_begin(SFQ_PH_TAYLOR_GEMM);
      *d = i8_taylor(i8_cur);  // T_1
      return SFQ_OK;
    }
    if (s <= 3 + order) {  // after the product of T_k, k = s - 3
      const int k = s - 3, cur = i8_cur;
      ph_end(SFQ_PH_TAYLOR_GEMM);
      const bool last = k == order;
      if ((rc = islice_taylor_update(Cp, Sacc, R, M, k, last, nslices, A_q[1 - cur], ld_m, A_e[1 - cur], st)))
        return rc;
      i8_cur = 1 - cur;
      if (last) {
        *d = i8_p1(i8_cur, Cp, false);
      } else {
        ph_begin(SFQ_PH_TAYLOR_GEMM);
        *d = i8_taylor(i8_cur);  // T_{k+1}
      }
      return SFQ_OK;
    }
    *more = false;
    if ((rc = islice_to_walkers(Cp, Sacc, Wb, M, N, SM, st))) return rc;
    ph_end(SFQ_PH_PROPAGATE);
    ph_begin(SFQ_PH_OVERLAP);
    if ((rc = ndet > 1 ? log_overlap_md(newov) : log_overlap(newov))) return rc;
    ph_end(SFQ_PH_OVERLAP);
    ph_begin(SFQ_PH_UPDATE);
    UpdateParams up;
    up.nwalk = W; up.dt = p.dt; up.Eshift = Eshift; up.E0 = p.E0;
    up.lower_cutoff = p.lower_cutoff_scale; up.upper_cutoff = p.upper_cutoff_scale;
    up.max_weight = std::fmax(p.weight_bound_floor, p.weight_bound_fraction * target_pop());
    up.hybrid = 1; up.free_projection = p.free_projection; up.use_cp_constraint = 0;
    up.Eshift_dev = dev_mode ? d_eshift : nullptr;
    if ((rc = walker_update(wprops(), newov, mf, hw, E3, up, stats, st))) return rc;
    ph_end(SFQ_PH_UPDATE);
    return SFQ_OK;
  }
  int propagate_i8(double Eshift, unsigned long long step, const double* uniforms) {
    int rc;
    IsliceGemmDesc d;
    bool more = true;
    for (int s = 0; more; ++s) {
      if ((rc = propagate_i8_next(s, Eshift, step, uniforms, &d, &more))) return rc;
      if (more && (rc = islice_gemm(d, st))) return rc;
    }
    return SFQ_OK;
  }

  // NOMSD::Energy in the exact-accumulation mode: E1 from the FP64 G; the exchange tensor
  // T[(c,w,b)][(n,a)] = sum_k G_c[w,b,k] Lnak[n,a,k] from int8 slices in chunks of Cholesky vectors
  // (FP32, one rounding), its contractions summed in FP64.  Stages as propagate_i8_stage: stage 0
  // ends in the product of the first chunk, stage s > 0 reduces chunk s - 1 and ends in the next.
  int i8_n0 = 0;  // first Cholesky vector of the chunk in flight
  long i8_chunk() const {
    const long per_n = 2L * W * N * N;
    long nv_max = (2L * tchunk_elems) / per_n;
    if (nv_max < 1) nv_max = 1;
    if (nv_max > Nc) nv_max = Nc;
    return nv_max;
  }
  void i8_exchange_desc(int n0, IsliceGemmDesc* d, int det = 0) {
    const long R = (long)W * N;
    const long nv_max = i8_chunk();
    const int nv = (Nc - n0) < nv_max ? (Nc - n0) : int(nv_max);
    const long ldc = (long)nv * N;
    const long lp = trial_real ? 1 : 2;
    const long row0 = lp * det * Nc * N + (long)n0 * N;  // determinant det's Lnak rows (n0, 0)
    int8_t* Lc[3];
    for (int q = 0; q < 3; ++q) Lc[q] = Le_q[q] ? Le_q[q] + row0 * ld_mr : nullptr;
    *d = i8_desc();
    d->M = int(2 * R); d->N = int(ldc); d->K = Mr;
    d->A = i8_operand(Ge_q, 2 * R, ld_mr, Ge_e);
    d->B = i8_operand(Lc, ldc, ld_mr, Le_e + row0);
    d->bn = i8_bn;
    d->C = reinterpret_cast<float*>(Tchunk); d->ldc = ldc;
    if (!trial_real) {  // the imaginary rows of these Lnak rows: Nc N rows further
      int8_t* qi[3];
      for (int q = 0; q < 3; ++q) qi[q] = Le_q[q] ? Le_q[q] + (row0 + (long)Nc * N) * ld_mr : nullptr;
      i8_queue_cplx(*d, R, i8_operand(qi, ldc, ld_mr, Le_e + row0 + (long)Nc * N));
    }
  }
  int i8_det = 0;  // multi-determinant trials: the determinant whose exchange is in flight
  // determinant det's G (FP64, its own overlap factors), one-body energy and G slices
  int energy_md_i8_prep(int det) {
    int rc;
    const long o = det_elems();
    const double scl = closed() ? 2.0 : 1.0;
    if ((rc = md_factor(det, SM, W, md_ov + (long)det * W, true, ov_scale()))) return rc;
    if ((rc = ops::green_compact(T, SM, G, W, Mr, N, st))) return rc;
    if ((rc = energy_e1(G, haj + det * o, md_E + (long)det * W * 3, W, N, Mr, p.E0, scl, 1, st))) return rc;
    return islice_rows_planar(G, (long)W * N, Mr, nslices, Ge_q, ld_mr, Ge_e, st);
  }
  // NOMSD::Energy with ndet > 1 in stages: each determinant's exchange chunks in turn (its G, one-body
  // energy and slices before its first chunk, its sums after its last), then the ci-weighted ratio
  int energy_md_i8_stage(int s, IsliceGemmDesc* d, bool* more) {
    int rc;
    const double scl = closed() ? 2.0 : 1.0;
    *more = true;
    if (s == 0) {
      ph_begin(SFQ_PH_ENERGY);
      inv_cached = false;
      i8_det = 0;
      i8_n0 = 0;
      if ((rc = energy_md_i8_prep(0))) return rc;
      i8_exchange_desc(0, d, 0);
      return SFQ_OK;
    }
    const long nv_max = i8_chunk();
    const int n0 = i8_n0;
    const int nv = (Nc - n0) < nv_max ? (Nc - n0) : int(nv_max);
    if ((rc = energy_exx_reduce_f32(reinterpret_cast<float*>(Tchunk), W, N, nv, n0, Nc, (long)nv * N, exxn, kl, st,
                                    spin_split())))
      return rc;
    i8_n0 = n0 + nv;
    if (i8_n0 < Nc) {
      i8_exchange_desc(i8_n0, d, i8_det);
      return SFQ_OK;
    }
    if ((rc = energy_finish(exxn, kl, md_E + (long)i8_det * W * 3, W, Nc, scl, 1, 1, st))) return rc;
    if (++i8_det < ndet) {
      i8_n0 = 0;
      if ((rc = energy_md_i8_prep(i8_det))) return rc;
      i8_exchange_desc(0, d, i8_det);
      return SFQ_OK;
    }
    *more = false;
    md_energy_kernel<<<(W + 127) / 128, 128, 0, st>>>(md_ov, md_E, md_cic, ndet, W, E3, ovtmp);
    SFQ_LAUNCHED();
    ph_end(SFQ_PH_ENERGY);
    return SFQ_OK;
  }
  int energy_i8_stage(int s, IsliceGemmDesc* d, bool* more) {
    if (ndet > 1) return energy_md_i8_stage(s, d, more);
    int rc;
    const double scl = closed() ? 2.0 : 1.0;  // CLOSED counts each orbital twice
    *more = true;
    if (s == 0) {
      ph_begin(SFQ_PH_ENERGY);
      if ((rc = density(ovtmp))) return rc;
      if ((rc = energy_e1(G, haj, E3, W, N, Mr, p.E0, scl, 1, st))) return rc;
      if ((rc = islice_rows_planar(G, (long)W * N, Mr, nslices, Ge_q, ld_mr, Ge_e, st))) return rc;
      i8_n0 = 0;
      i8_exchange_desc(0, d);
      return SFQ_OK;
    }
    const long nv_max = i8_chunk();
    const int n0 = i8_n0;
    const int nv = (Nc - n0) < nv_max ? (Nc - n0) : int(nv_max);
    if ((rc = energy_exx_reduce_f32(reinterpret_cast<float*>(Tchunk), W, N, nv, n0, Nc, (long)nv * N, exxn, kl, st,
                                    spin_split())))
      return rc;
    i8_n0 = n0 + nv;
    if (i8_n0 < Nc) {
      i8_exchange_desc(i8_n0, d);
      return SFQ_OK;
    }
    *more = false;
    if ((rc = energy_finish(exxn, kl, E3, W, Nc, scl, 1, 1, st))) return rc;
    ph_end(SFQ_PH_ENERGY);
    return SFQ_OK;
  }
  int energy_i8() {
    int rc;
    IsliceGemmDesc d;
    bool more = true;
    for (int s = 0; more; ++s) {
      if ((rc = energy_i8_next(s, &d, &more))) return rc;
      if (more && (rc = islice_gemm(d, st))) return rc;
    }
    return SFQ_OK;
  }

  // AFQMCBasePropagator::Propagate with the bulk products on the tensor cores (split BF16, FP32
  // accumulation); G, LU/log det, fields, overlaps and the walker update stay FP64.
  int propagate_mixed(double Eshift, unsigned long long step, const double* uniforms) {
    if (nslices) return propagate_i8(Eshift, step, uniforms);
    int rc;
    const long MM = (long)M * M, NM = (long)N * M, M2 = 2L * M;
    const double sdt = std::sqrt(p.dt);
    ph_begin(SFQ_PH_DENSITY);
    if ((rc = density_mixed())) return rc;
    ph_end(SFQ_PH_DENSITY);
    ph_begin(SFQ_PH_VBIAS);
    const long part = 2L * W * Nc;  // one K split's partial sums
    if ((rc = tc_gemm(Gs_p, 2L * W, 0, Lnak_p, Nc, 0, int(NM), 1, Cvb, Nc, 0, 1.f, vb_bn, nullptr, vb_ks, part)))
      return rc;
    if ((rc = mixed_reduce_planar_to_cplx(Cvb, vb_ks, part, W, Nc, 2.0 * sdt, X, st))) return rc;
    ph_end(SFQ_PH_VBIAS);
    ph_begin(SFQ_PH_FIELDS);
    FieldParams fp;
    fp.nwalk = W; fp.nchol = Nc; fp.vbias_bound = p.vbias_bound; fp.free_projection = p.free_projection;
    fp.seed = p.seed; fp.step = step; fp.uniforms = uniforms; fp.step_dev = dev_mode ? d_step : nullptr;
    if (uni_wait) {
      SFQ_CUDA_TRY(cudaStreamWaitEvent(st, uni_wait, 0));
      uni_wait = nullptr;
    }
    if ((rc = assemble_x(X, vmf, hw, mf, fp, st))) return rc;
    ph_end(SFQ_PH_FIELDS);
    ph_begin(SFQ_PH_VHS);
    if ((rc = mixed_split_planar(X, W, Nc, Xs_p, st))) return rc;
    ph_begin(SFQ_PH_VHS_GEMM);
    const long vcols = sym ? P : MM;
    if ((rc = tc_gemm(Xs_p, 2L * W, 0, Likn_p, vcols, 0, Nc, 1, Cv, vcols, 0, float(sdt), vhs_bn))) return rc;
    ph_end(SFQ_PH_VHS_GEMM);
    if ((rc = mixed_build_v(Cv, W, M, sym, Vb_p, st))) return rc;
    ph_end(SFQ_PH_VHS);
    ph_begin(SFQ_PH_PROPAGATE);
    inv_cached = false;
    // S = P1 W (fp32) and its planes T1 = S; then T_{k+1} = (i/k) VB T_k, S += T_{k+1} in the
    // Taylor products' epilogues, the operand planes alternating between the two buffers; the
    // last one leaves the planes of S for SM = P1 S, written straight back to the walkers
    const long rows = 2L * W * N;  // (w, a, c) rows of the walker operand
    if (!mixed_green() && (rc = mixed_walkers_to_wt(SM, W, M, N, ldh, Wt_p, st))) return rc;  // else done with G
    UmmaEpilogue e1;
    e1.kind = UMMA_EPI_STORE_SPLIT;
    for (int q = 0; q < 3; ++q) e1.out[q] = Wt2_p[q];
    e1.out_planes = nplanes;
    e1.ldh = ldh;
    if ((rc = tc_gemm(Wt_p, rows, 0, P1_p, M, 0, M, 1, Sacc, M, 0, 1.f, p1_tile(), &e1, 1, 0, ldh))) return rc;
    void** cur = Wt2_p;
    void** nxt = Wt_p;
    const long L2h = 2L * ldh;  // walker-operand row: [re | pad | im | pad]
    for (int k = 1; k <= p.taylor_order; ++k) {
      UmmaGemmDesc d;
      d.M = N; d.N = int(vb_rows); d.K = int(L2h); d.batch = W;
      for (int q = 0; q < 3; ++q) {
        d.A.p[q] = cur[q];
        d.B.p[q] = Vb_p[q];
      }
      d.A.rows = N; d.A.ld = L2h; d.A.batch_stride = long(N) * L2h;
      d.B.rows = M2; d.B.ld = M; d.B.batch_stride = M2 * M;
      d.cplx_half = tay_half; d.cplx_nmo = M; d.cplx_ldh = ldh;
      d.nplanes = nplanes; d.bn = 2 * tay_half; d.err = gemm_err;
      UmmaEpilogue& et = d.epi;
      et.kind = UMMA_EPI_TAYLOR;
      et.S = Sacc; et.nmo = M; et.ldh = ldh; et.half = tay_half; et.inv_k = 1.f / float(k);
      et.write = k < p.taylor_order ? 1 : 2;
      for (int q = 0; q < 3; ++q) et.out[q] = nxt[q];
      et.out_planes = nplanes;
      ph_begin(SFQ_PH_TAYLOR_GEMM);
      if ((rc = umma_gemm(d, st))) return rc;
      ph_end(SFQ_PH_TAYLOR_GEMM);
      std::swap(cur, nxt);
    }
    UmmaEpilogue ew;
    ew.kind = UMMA_EPI_TO_WALKERS;
    ew.SM = reinterpret_cast<double*>(SM);
    ew.nel = N;
    if ((rc = tc_gemm(cur, rows, 0, P1_p, M, 0, M, 1, nullptr, 0, 0, 1.f, p1_tile(), &ew, 1, 0, ldh))) return rc;
    ph_end(SFQ_PH_PROPAGATE);
    ph_begin(SFQ_PH_OVERLAP);
    if ((rc = log_overlap(newov))) return rc;
    ph_end(SFQ_PH_OVERLAP);
    ph_begin(SFQ_PH_UPDATE);
    UpdateParams up;
    up.nwalk = W; up.dt = p.dt; up.Eshift = Eshift; up.E0 = p.E0;
    up.lower_cutoff = p.lower_cutoff_scale; up.upper_cutoff = p.upper_cutoff_scale;
    up.max_weight = std::fmax(p.weight_bound_floor, p.weight_bound_fraction * target_pop());
    up.hybrid = 1; up.free_projection = p.free_projection; up.use_cp_constraint = 0;
    up.Eshift_dev = dev_mode ? d_eshift : nullptr;
    if ((rc = walker_update(wprops(), newov, mf, hw, E3, up, stats, st))) return rc;
    ph_end(SFQ_PH_UPDATE);
    return SFQ_OK;
  }

  int orthogonalize() {
    int rc;
    ph_begin(SFQ_PH_ORTHO);
    const long NN = (long)N * N;
    if (ndet == 1 && inv_cached && tchunk_elems >= 2L * W * NN) {
      // the cached inverse overlaps and log overlaps of the walkers ride through the QR, which
      // gives wfn->Log_Overlap(wset) of the orthogonalized walkers without a new factorization
      if (inv_ov != newov)
        SFQ_CUDA_TRY(cudaMemcpyAsync(newov, inv_ov, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st));
      if ((rc = ops::orthogonalize_carry(SM, SM2, Tchunk, Tchunk + W * NN, G, status, T, newov, ov_scale(), W, Mr, N,
                                         st, spin_split())))
        return rc;
      inv_ov = newov;
    } else {
      inv_cached = false;
      if ((rc = ops::orthogonalize(SM, SM2, T, status, nullptr, W, Mr, N, st, spin_split()))) return rc;
      if ((rc = ndet > 1 ? log_overlap_md(newov) : log_overlap(newov))) return rc;  // wfn->Log_Overlap(wset)
    }
    SFQ_CUDA_TRY(cudaMemcpyAsync(props + (long)P_OVLP * W, newov, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st));
    ph_end(SFQ_PH_ORTHO);
    return SFQ_OK;
  }

  // the comb's uniform: Philox(seed, call), or r itself when r >= 0 (a caller's generator)
  int population_control(unsigned long long call, double r = -1.0) {
    int rc;
    ph_begin(SFQ_PH_POPCONTROL);
    inv_cached = false;
    const bool own = r >= 0.0;
    if ((rc = sfq::population_control(SM, (long)Mr * N, wprops(), W, own ? r : 0.0, p.seed, call, own ? 0 : 1, pw, st,
                                      dev_mode && !own ? d_step : nullptr)))
      return rc;
    if (nbp) {  // copy_walker copies the back-propagation buffers too (WalkerSetBase.h:375-415)
      if ((rc = copy_walker_rows(bp_SMN, (long)Mr * N, pw, W, st))) return rc;
      if ((rc = copy_walker_rows(bp_fields, (long)nbp * Nc, pw, W, st))) return rc;
      if ((rc = copy_walker_rows(bp_wfac, nhist, pw, W, st))) return rc;
    }
    ph_end(SFQ_PH_POPCONTROL);
    if (dev_mode) return SFQ_OK;  // the collapse flag stays on the device until the block ends
    int flag = 0;
    SFQ_CUDA_TRY(cudaMemcpyAsync(&flag, pw.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    if ((rc = sync_checked())) return rc;
    if (flag == SFQ_ERR_WEIGHT_COLLAPSE) return record_error(flag, "The total walker weight collapsed.");
    if (flag) return record_error(flag, "population control: inconsistent copy plan");
    return SFQ_OK;
  }

  // NOMSD::Energy(wset, E, Ov): E3 and ovtmp
  int energy_only() {
    int rc;
    if (mixed) return energy_mixed();
    ph_begin(SFQ_PH_ENERGY);
    if (ndet > 1) {
      if ((rc = energy_md())) return rc;
      ph_end(SFQ_PH_ENERGY);
      return SFQ_OK;
    }
    if ((rc = density(ovtmp))) return rc;
    if ((rc = ops::energy(E3, G, haj, Lnak, !trial_real, p.E0, W, N, Mr, Nc, 1, 1, 1, Tchunk, tchunk_elems, exxn, kl,
                          st, spin_split())))
      return rc;
    ph_end(SFQ_PH_ENERGY);
    return SFQ_OK;
  }

  // the same in the mixed mode: E1 from the FP64 G, the exchange tensor T[(c,w,b)][(n,a)] =
  // sum_k G_c[w,b,k] Lnak[n,a,k] as split-BF16 tcgen05 products into FP32 (in chunks of Cholesky
  // vectors), its contractions summed in FP64
  int energy_mixed() {
    if (nslices) return energy_i8();
    int rc;
    ph_begin(SFQ_PH_ENERGY);
    if ((rc = density(ovtmp))) return rc;
    const double scl = 2.0;
    if ((rc = energy_e1(G, haj, E3, W, N, M, p.E0, scl, 1, st))) return rc;
    if ((rc = mixed_split_planar(G, W, (long)N * M, Gs_p, st))) return rc;
    // FP32 chunk of T in the FP64 chunk buffer: twice the elements
    const long per_n = 2L * W * N * N;  // FP32 values of T per Cholesky vector
    long nv_max = (2L * tchunk_elems) / per_n;
    if (nv_max < 1) nv_max = 1;
    if (nv_max > Nc) nv_max = Nc;
    float* Tf = reinterpret_cast<float*>(Tchunk);
    for (int n0 = 0; n0 < Nc; n0 += int(nv_max)) {
      const int nv = (Nc - n0) < nv_max ? (Nc - n0) : int(nv_max);
      void* Lc[3];
      for (int q = 0; q < 3; ++q)
        Lc[q] = Lnak_p[q] ? static_cast<void*>(static_cast<char*>(Lnak_p[q]) + 2L * n0 * N * M) : nullptr;
      const long ldc = (long)nv * N;
      if ((rc = tc_gemm(Gs_p, 2L * W * N, 0, Lc, ldc, 0, M, 1, Tf, ldc, 0, 1.f))) return rc;
      if ((rc = energy_exx_reduce_f32(Tf, W, N, nv, n0, Nc, ldc, exxn, kl, st))) return rc;
    }
    if ((rc = energy_finish(exxn, kl, E3, W, Nc, scl, 1, 1, st))) return rc;
    ph_end(SFQ_PH_ENERGY);
    return SFQ_OK;
  }

  int averages(const cplx* E, double* out10) {
    averages_kernel<<<1, 1024, 0, st>>>(props, W, p.dt, E, red);
    SFQ_LAUNCHED();
    SFQ_CUDA_TRY(cudaMemcpyAsync(out10, red, sizeof(double) * 10, cudaMemcpyDeviceToHost, st));
    return sync_checked();
  }

  // run_afqmc's loop (run_afqmc.cpp:69-113) over steps step0 .. step0+steps-1 as a string of
  // per-step codes: bit 0 orthogonalize, bit 1 population control, bit 2 Eshift relaxation,
  // bit 3 measurement; the schedule a block graph is captured for
  static std::string block_schedule(const sfq_run_params_t& rp) {
    std::string key;
    for (unsigned long long step = rp.step0; step < rp.step0 + (unsigned long long)rp.steps; ++step) {
      int c = 0;
      if (rp.walker_ortho_interval > 0 && step % rp.walker_ortho_interval == 0) c |= 1;
      if (rp.population_control_interval > 0 && step % rp.population_control_interval == 0) c |= 2;
      const bool equil = (long long)step < rp.equilibration_steps;
      if (equil || rp.steer_eshift) c |= 4;
      if (!equil && rp.measure_interval > 0 && step % rp.measure_interval == 0) c |= 8;
      key.push_back(char('a' + c));
    }
    return key;
  }

  // the block's work on the stream, in device mode (no host reads; captured into a graph)
  int record_block(const std::string& sched, double relax, int* nmeas) {
    int rc;
    inv_cached = false;  // the block starts from whatever walkers it is given
    int slot = 0;
    for (char ch : sched) {
      const int c = ch - 'a';
      if ((rc = propagate(0.0, 0, nullptr))) return rc;  // step and Eshift come from the device
      if ((rc = block_after_propagate(c))) return rc;
      if (c & 8) {
        if (slot >= kMeasCap) return record_error(SFQ_ERR_ARG, "block: more than %d measurements", kMeasCap);
        if ((rc = energy_only())) return rc;
        if ((rc = block_measure(&slot))) return rc;
      }
      if ((rc = block_step_end(c, relax))) return rc;
    }
    *nmeas = slot;
    return SFQ_OK;
  }
  // the pieces of one block step around the propagation and the energy (record_block's order)
  int block_after_propagate(int c) {
    int rc;
    if ((c & 1) && (rc = orthogonalize())) return rc;
    if ((c & 2) && (rc = population_control(0))) return rc;
    return SFQ_OK;
  }
  int block_measure(int* slot) {  // after the energy
    averages_kernel<<<1, 1024, 0, st>>>(props, W, p.dt, E3, red);
    SFQ_LAUNCHED();
    measure_kernel<<<1, 1, 0, st>>>(red, d_meas + 10 * *slot);
    SFQ_LAUNCHED();
    ++*slot;
    return SFQ_OK;
  }
  int block_step_end(int c, double relax) {
    if (c & 4) {
      averages_kernel<<<1, 1024, 0, st>>>(props, W, p.dt, nullptr, red);
      SFQ_LAUNCHED();
      eshift_relax_kernel<<<1, 1, 0, st>>>(red, p.dt, relax, d_eshift);
      SFQ_LAUNCHED();
    }
    step_add_kernel<<<1, 1, 0, st>>>(d_step);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }

  // run_afqmc's Eshift relaxation factor (run_afqmc.cpp:58-60) unless one is given
  static double block_relax(const sfq_run_params_t& rp) {
    double relax = rp.Eshift_relaxation_factor;
    if (!(relax > 0.0)) relax = rp.equilibration_steps > 1 ? 1.0 - std::exp(-10.0 / rp.equilibration_steps) : 1.0;
    return relax;
  }
  static std::string block_key(const sfq_run_params_t& rp) {
    char tail[64];
    std::snprintf(tail, sizeof(tail), "|%.17g", block_relax(rp));
    return block_schedule(rp) + tail;
  }

  // relative cost of one step, for balancing group lanes: the algorithmic flops of the products,
  // weighted by how much slower the FP64 path runs them
  double step_cost() const {
    const double f = double(W) * (8.0 * N * M * Nc + 4.0 * M * double(M) * Nc + 64.0 * M * double(M) * N);
    return mixed ? f : 6.0 * f;
  }

  // one member's part of a group block, recorded on the engine stream inside the group's capture:
  // the step counter and Eshift from the group's input row, the block, then the results into the
  // group's output row (4 + 10 kMeasCap doubles)
  int record_group_part(const sfq_run_params_t& rp, const unsigned long long* in, double* out, int* nmeas) {
    int rc = group_part_begin(in);
    if (!rc) rc = record_block(block_schedule(rp), block_relax(rp), nmeas);
    if (!rc) rc = group_part_results(out, *nmeas);
    group_part_end();
    return rc;
  }
  bool saved_profile = false;
  int group_part_begin(const unsigned long long* in) {
    saved_profile = profile;
    profile = false;
    dev_mode = true;
    inv_cached = false;
    load_block_state_kernel<<<1, 1, 0, st>>>(in, d_step, d_eshift);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }
  int group_part_results(double* out, int nmeas) {
    store_block_result_kernel<<<1, 128, 0, st>>>(d_eshift, pw.flag, mixed ? gemm_err : nullptr, d_meas, nmeas, out);
    SFQ_LAUNCHED();
    return SFQ_OK;
  }
  void group_part_end() {
    dev_mode = false;
    profile = saved_profile;
  }

  // enqueue one block: its graph (captured on first use of its schedule), then the copies of
  // its results into pinned memory and an event; block_result() waits for them
  int block_async(const sfq_run_params_t& rp, double Eshift) {
    int rc;
    if (rp.steps <= 0) return record_error(SFQ_ERR_ARG, "block: steps must be positive");
    const double relax = block_relax(rp);
    const std::string key = block_key(rp);
    auto it = graphs.find(key);
    if (it == graphs.end()) {
      BlockGraph bg;
      const bool prof = profile;
      profile = false;
      dev_mode = true;
      SFQ_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
      int nm = 0;
      rc = record_block(key.substr(0, rp.steps), relax, &nm);
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(st, &g);
      dev_mode = false;
      profile = prof;
      if (rc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc ? rc : record_cuda(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
      }
      const cudaError_t ie = cudaGraphInstantiate(&bg.exec, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) return record_cuda(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
      bg.inv_after = inv_cached;
      bg.inv_ov_after = inv_ov;
      bg.nmeas = nm;
      it = graphs.emplace(key, bg).first;
    }
    if (!blk_host) {
      SFQ_CUDA_TRY(cudaMallocHost(&blk_host, sizeof(double) * (4 + 10 * kMeasCap)));
      SFQ_CUDA_TRY(cudaEventCreateWithFlags(&blk_done, cudaEventDisableTiming));
    }
    const BlockGraph& bg = it->second;
    set_block_state_kernel<<<1, 1, 0, st>>>(d_step, rp.step0, d_eshift, Eshift);
    SFQ_LAUNCHED();
    if (nbp) {  // the block's steps store their fields and weight factors from here on
      set_hist_kernel<<<1, 1, 0, st>>>(d_step + 1, (unsigned long long)hist_pos);
      SFQ_LAUNCHED();
      hist_pos = int((hist_pos + (long)rp.steps) % nhist);
    }
    SFQ_CUDA_TRY(cudaGraphLaunch(bg.exec, st));
    inv_cached = bg.inv_after;
    inv_ov = bg.inv_ov_after;
    SFQ_CUDA_TRY(cudaMemcpyAsync(blk_host, d_eshift, sizeof(double), cudaMemcpyDeviceToHost, st));
    SFQ_CUDA_TRY(cudaMemcpyAsync(blk_host + 1, pw.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (mixed) SFQ_CUDA_TRY(cudaMemcpyAsync(blk_host + 2, gemm_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (bg.nmeas)
      SFQ_CUDA_TRY(cudaMemcpyAsync(blk_host + 4, d_meas, sizeof(double) * 10 * bg.nmeas, cudaMemcpyDeviceToHost, st));
    SFQ_CUDA_TRY(cudaEventRecord(blk_done, st));
    blk_nmeas = bg.nmeas;
    return SFQ_OK;
  }

  int block_query() {
    if (!blk_done) return 1;
    const cudaError_t q = cudaEventQuery(blk_done);
    if (q == cudaSuccess) return 1;
    if (q == cudaErrorNotReady) return 0;
    return -record_cuda(q, "cudaEventQuery", __FILE__, __LINE__);
  }

  int block_result(double* Eshift, double* meas, int max_meas, int* nmeas) {
    if (!blk_done) return record_error(SFQ_ERR_ARG, "block: no block was run");
    SFQ_CUDA_TRY(cudaEventSynchronize(blk_done));
    int flag = 0, gflag = 0;
    std::memcpy(&flag, blk_host + 1, sizeof(int));
    if (mixed) std::memcpy(&gflag, blk_host + 2, sizeof(int));
    if (gflag) {
      cudaMemsetAsync(gemm_err, 0, sizeof(int), st);
      return record_error(SFQ_ERR_TIMEOUT, "tensor-core product: a bounded wait expired in the block");
    }
    if (flag == SFQ_ERR_WEIGHT_COLLAPSE) return record_error(flag, "The total walker weight collapsed.");
    if (flag) return record_error(flag, "population control: inconsistent copy plan");
    if (Eshift) *Eshift = blk_host[0];
    const int n = blk_nmeas < max_meas ? blk_nmeas : max_meas;
    if (meas && n > 0) std::memcpy(meas, blk_host + 4, sizeof(double) * 10 * n);
    if (nmeas) *nmeas = blk_nmeas;
    return SFQ_OK;
  }

  // Synchronise the engine stream, then report a bounded wait of the tensor-core product that
  // expired since the last check (SFQ_ERR_TIMEOUT: the steps since then are invalid).
  int sync_checked() {
    int gflag = 0;
    if (mixed) SFQ_CUDA_TRY(cudaMemcpyAsync(&gflag, gemm_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SFQ_CUDA_TRY(cudaStreamSynchronize(st));
    if (gflag) {
      cudaMemsetAsync(gemm_err, 0, sizeof(int), st);
      return record_error(SFQ_ERR_TIMEOUT, "tensor-core product: a bounded wait expired; the steps since the "
                                           "last check are invalid");
    }
    return SFQ_OK;
  }
};

// ---- several systems advanced together ---------------------------------------------------------
// One block of every member as ONE CUDA graph: the members' block recordings (each on its own
// engine stream) form `lanes` branches forked from and joined back to the group stream; within a
// lane the members run one after another, the lanes side by side on the SMs.  Members go to lanes
// longest first, each to the lane with the least work so far (by step_cost x steps).  Per launch
// the group copies each member's {step0, Eshift} to the device once and reads all results back
// in one copy.
struct Group {
  static constexpr int kOut = 4 + 10 * Engine::kMeasCap;  // doubles per member's output row
  std::vector<Engine*> es;
  cudaStream_t gst = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_done = nullptr;
  std::vector<cudaEvent_t> ev_join, ev_pre;
  unsigned long long* d_in = nullptr;
  double* d_out = nullptr;
  unsigned long long* h_in = nullptr;
  double* h_out = nullptr;
  struct Captured {
    cudaGraphExec_t exec = nullptr;
    std::vector<char> inv_after;
    std::vector<const cplx*> inv_ov_after;
    std::vector<int> nmeas;
  };
  std::map<std::string, Captured> graphs;
  const Captured* pending = nullptr;
  int lanes = 0;  // 0: one lane per member
  // fused mode (int8-slice members on one block schedule): the members' steps interleaved stage by
  // stage, each stage's int8-slice products of all members as ONE grouped launch on the group
  // stream, the work between them on the members' streams side by side
  bool fused = false;
  struct Table {
    void* dev = nullptr;  // the grouped launch's table in device memory
    IsliceGroupPlan plan;
  };
  std::map<std::string, Table> tables;  // by stage and members; the same for every step and block
  std::vector<std::string> new_tables;  // created in the capture under way, to be copied to the device
  cudaEvent_t ev_prod = nullptr;        // after the last grouped launch
  std::vector<cudaEvent_t> ev_stage;

  // lane of each member, and the members of each lane in order
  std::vector<std::vector<int>> plan_lanes(const sfq_run_params_t* rps) const {
    const int n = int(es.size());
    const int L = (lanes <= 0 || lanes > n) ? n : lanes;
    std::vector<int> order(n);
    std::vector<double> cost(n);
    for (int i = 0; i < n; ++i) {
      order[i] = i;
      cost[i] = es[i]->step_cost() * rps[i].steps;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<std::vector<int>> out(L);
    std::vector<double> load(L, 0.0);
    for (int i : order) {
      int best = 0;
      for (int l = 1; l < L; ++l)
        if (load[l] < load[best]) best = l;
      out[best].push_back(i);
      load[best] += cost[i];
    }
    return out;
  }

  int init(const std::vector<Engine*>& members) {
    es = members;
    const size_t n = es.size();
    SFQ_CUDA_TRY(cudaSetDevice(es[0]->p.device));
    SFQ_CUDA_TRY(cudaStreamCreateWithFlags(&gst, cudaStreamNonBlocking));
    SFQ_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    SFQ_CUDA_TRY(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
    SFQ_CUDA_TRY(cudaEventCreateWithFlags(&ev_prod, cudaEventDisableTiming));
    ev_join.assign(n, nullptr);
    ev_pre.assign(n, nullptr);
    ev_stage.assign(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
      SFQ_CUDA_TRY(cudaEventCreateWithFlags(&ev_join[i], cudaEventDisableTiming));
      SFQ_CUDA_TRY(cudaEventCreateWithFlags(&ev_pre[i], cudaEventDisableTiming));
      SFQ_CUDA_TRY(cudaEventCreateWithFlags(&ev_stage[i], cudaEventDisableTiming));
    }
    SFQ_CUDA_TRY(cudaMalloc(&d_in, sizeof(unsigned long long) * 2 * n));
    SFQ_CUDA_TRY(cudaMalloc(&d_out, sizeof(double) * kOut * n));
    SFQ_CUDA_TRY(cudaMallocHost(&h_in, sizeof(unsigned long long) * 2 * n));
    SFQ_CUDA_TRY(cudaMallocHost(&h_out, sizeof(double) * kOut * n));
    return SFQ_OK;
  }

  void release() {
    if (gst) cudaStreamSynchronize(gst);
    for (auto& kv : graphs)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    graphs.clear();
    for (auto& kv : tables)
      if (kv.second.dev) cudaFree(kv.second.dev);
    tables.clear();
    for (auto* v : {&ev_join, &ev_pre, &ev_stage})
      for (auto& x : *v)
        if (x) cudaEventDestroy(x);
    if (ev_prod) cudaEventDestroy(ev_prod);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_done) cudaEventDestroy(ev_done);
    if (d_in) cudaFree(d_in);
    if (d_out) cudaFree(d_out);
    if (h_in) cudaFreeHost(h_in);
    if (h_out) cudaFreeHost(h_out);
    if (gst) cudaStreamDestroy(gst);
  }

  // capture the members' blocks as the lanes of one graph
  int capture(const sfq_run_params_t* rps, Captured* c) {
    const size_t n = es.size();
    c->nmeas.assign(n, 0);
    c->inv_after.assign(n, 0);
    c->inv_ov_after.assign(n, nullptr);
    const std::vector<std::vector<int>> plan = plan_lanes(rps);
    SFQ_CUDA_TRY(cudaStreamBeginCapture(gst, cudaStreamCaptureModeRelaxed));
    int rc = SFQ_OK;
    cudaError_t ce = cudaEventRecord(ev_fork, gst);
    for (const auto& lane : plan) {
      cudaEvent_t after = ev_fork;  // a member starts after the fork or after its lane predecessor
      for (int i : lane) {
        Engine& e = *es[i];
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e.st, after, 0);
        if (ce != cudaSuccess) break;
        if (!rc) rc = e.record_group_part(rps[i], d_in + 2 * i, d_out + (size_t)kOut * i, &c->nmeas[i]);
        c->inv_after[i] = e.inv_cached ? 1 : 0;
        c->inv_ov_after[i] = e.inv_ov;
        ce = cudaEventRecord(ev_join[i], e.st);  // close every forked branch, also after an error
        after = ev_join[i];
      }
      if (ce != cudaSuccess) break;
      ce = cudaStreamWaitEvent(gst, after, 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(gst, &g);
    if (rc || ce != cudaSuccess || ee != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      if (rc) return rc;
      return record_cuda(ce != cudaSuccess ? ce : ee, "group capture", __FILE__, __LINE__);
    }
    const cudaError_t ie = cudaGraphInstantiate(&c->exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return record_cuda(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
    return SFQ_OK;
  }

  int set_fused(bool on) {
    if (on) {
      for (Engine* e : es)
        if (!e->nslices || e->nslices != es[0]->nslices)
          return record_error(SFQ_ERR_UNSUPPORTED, "group: fused products need int8-slice members of one precision");
    }
    fused = on;
    return SFQ_OK;
  }

  // K slices of one output tile of a product (its tiles' length)
  static long tile_k(const IsliceGemmDesc& d) {
    const long kt = (d.K + 127) / 128;
    if (d.cplx_half > 0) return 2 * kt;
    const long ks = d.ksplit < 1 ? 1 : d.ksplit;
    return (kt + ks - 1) / ks;
  }

  // stage s = 0, 1, ... of every member still running: its work on its own stream (after the
  // previous grouped launch), then all their products as one launch on the group stream
  template <typename StageFn>
  int grouped_stages(const char* kind, StageFn stage) {
    const int n = int(es.size());
    std::vector<char> more(size_t(n), 1);
    for (int s = 0;; ++s) {
      std::vector<IsliceGemmDesc> ds;
      std::vector<int> who;
      for (int i = 0; i < n; ++i) {
        if (!more[size_t(i)]) continue;
        Engine& e = *es[size_t(i)];
        if (s > 0) SFQ_CUDA_TRY(cudaStreamWaitEvent(e.st, ev_prod, 0));
        IsliceGemmDesc d;
        bool m = false;
        int rc = stage(e, s, &d, &m);
        if (rc) return rc;
        more[size_t(i)] = m ? 1 : 0;
        if (!m) continue;
        ds.push_back(d);
        who.push_back(i);
        SFQ_CUDA_TRY(cudaEventRecord(ev_stage[size_t(i)], e.st));
        SFQ_CUDA_TRY(cudaStreamWaitEvent(gst, ev_stage[size_t(i)], 0));
      }
      if (ds.empty()) return SFQ_OK;
      // the longest tiles first: the persistent CTAs take the tiles in list order
      std::vector<size_t> ord(ds.size());
      for (size_t j = 0; j < ord.size(); ++j) ord[j] = j;
      std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return tile_k(ds[a]) > tile_k(ds[b]); });
      std::string key = std::string(kind) + std::to_string(s);
      for (size_t j : ord) key += "," + std::to_string(who[j]);
      auto it = tables.find(key);
      if (it == tables.end()) {
        std::vector<IsliceGemmDesc> sorted;
        for (size_t j : ord) sorted.push_back(ds[j]);
        Table t;
        int rc = islice_gemm_group_plan(sorted.data(), int(sorted.size()), &t.plan);
        if (rc) return rc;
        SFQ_CUDA_TRY(cudaMalloc(&t.dev, t.plan.image.size()));
        it = tables.emplace(key, std::move(t)).first;
        new_tables.push_back(key);
      }
      int rc = islice_gemm_group_launch(it->second.dev, it->second.plan, gst);
      if (rc) return rc;
      SFQ_CUDA_TRY(cudaEventRecord(ev_prod, gst));
    }
  }

  // the members' blocks as one graph in fused mode (the steps of record_block, stage by stage)
  int capture_fused(const sfq_run_params_t* rps, Captured* c) {
    const size_t n = es.size();
    const std::string sched = Engine::block_schedule(rps[0]);
    for (size_t i = 1; i < n; ++i)
      if (Engine::block_schedule(rps[i]) != sched)
        return record_error(SFQ_ERR_ARG, "group: fused products need every member on one block schedule");
    int nmeas = 0;
    for (char ch : sched)
      if ((ch - 'a') & 8) ++nmeas;
    if (nmeas > Engine::kMeasCap) return record_error(SFQ_ERR_ARG, "block: more than %d measurements", Engine::kMeasCap);
    c->nmeas.assign(n, 0);
    c->inv_after.assign(n, 0);
    c->inv_ov_after.assign(n, nullptr);
    new_tables.clear();
    SFQ_CUDA_TRY(cudaStreamBeginCapture(gst, cudaStreamCaptureModeRelaxed));
    int rc = SFQ_OK;
    cudaError_t ce = cudaEventRecord(ev_fork, gst);
    std::vector<char> forked(n, 0), begun(n, 0);
    for (size_t i = 0; i < n && ce == cudaSuccess; ++i) {
      ce = cudaStreamWaitEvent(es[i]->st, ev_fork, 0);
      if (ce != cudaSuccess) break;
      forked[i] = 1;
      if (!rc) {
        rc = es[i]->group_part_begin(d_in + 2 * i);
        begun[i] = 1;
      }
    }
    std::vector<int> slot(n, 0);
    for (char ch : sched) {
      if (rc || ce != cudaSuccess) break;
      const int cc = ch - 'a';
      rc = grouped_stages("p", [](Engine& e, int s, IsliceGemmDesc* d, bool* m) {
        return e.propagate_i8_next(s, 0.0, 0, nullptr, d, m);  // step and Eshift come from the device
      });
      for (size_t i = 0; i < n && !rc; ++i) rc = es[i]->block_after_propagate(cc);
      if (!rc && (cc & 8)) {
        rc = grouped_stages("e", [](Engine& e, int s, IsliceGemmDesc* d, bool* m) { return e.energy_i8_next(s, d, m); });
        for (size_t i = 0; i < n && !rc; ++i) rc = es[i]->block_measure(&slot[i]);
      }
      for (size_t i = 0; i < n && !rc; ++i) rc = es[i]->block_step_end(cc, Engine::block_relax(rps[i]));
    }
    for (size_t i = 0; i < n; ++i) {
      if (!rc && begun[i]) rc = es[i]->group_part_results(d_out + (size_t)kOut * i, slot[i]);
      c->nmeas[i] = slot[i];
      c->inv_after[i] = es[i]->inv_cached ? 1 : 0;
      c->inv_ov_after[i] = es[i]->inv_ov;
      if (begun[i]) es[i]->group_part_end();
      if (forked[i] && ce == cudaSuccess) {  // close every forked branch, also after an error
        ce = cudaEventRecord(ev_join[i], es[i]->st);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(gst, ev_join[i], 0);
      }
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(gst, &g);
    if (rc || ce != cudaSuccess || ee != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      for (const std::string& k : new_tables) {  // never copied: drop them
        auto it = tables.find(k);
        if (it != tables.end()) {
          cudaFree(it->second.dev);
          tables.erase(it);
        }
      }
      new_tables.clear();
      if (rc) return rc;
      return record_cuda(ce != cudaSuccess ? ce : ee, "group capture", __FILE__, __LINE__);
    }
    const cudaError_t ie = cudaGraphInstantiate(&c->exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return record_cuda(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
    // the new tables reach the device on the group stream, ahead of the graph's first launch there
    for (const std::string& k : new_tables) {
      const Table& t = tables[k];
      SFQ_CUDA_TRY(cudaMemcpyAsync(t.dev, t.plan.image.data(), t.plan.image.size(), cudaMemcpyHostToDevice, gst));
    }
    new_tables.clear();
    return SFQ_OK;
  }

  int block_async(const sfq_run_params_t* rps, const double* Eshift) {
    const size_t n = es.size();
    if (pending) return record_error(SFQ_ERR_ARG, "group: the previous block's results were not taken");
    std::string key = (fused ? std::string("F") : std::to_string(lanes)) + "#";
    for (size_t i = 0; i < n; ++i) {
      if (rps[i].steps <= 0) return record_error(SFQ_ERR_ARG, "group: steps must be positive");
      key += Engine::block_key(rps[i]);
      key += ';';
    }
    auto it = graphs.find(key);
    if (it == graphs.end()) {
      Captured c;
      int rc = fused ? capture_fused(rps, &c) : capture(rps, &c);
      if (rc) return rc;
      it = graphs.emplace(key, std::move(c)).first;
    }
    for (size_t i = 0; i < n; ++i) {
      h_in[2 * i] = rps[i].step0;
      std::memcpy(&h_in[2 * i + 1], &Eshift[i], sizeof(double));
    }
    // after every member's earlier work, one input copy, the graph, one output copy
    for (size_t i = 0; i < n; ++i) {
      SFQ_CUDA_TRY(cudaEventRecord(ev_pre[i], es[i]->st));
      SFQ_CUDA_TRY(cudaStreamWaitEvent(gst, ev_pre[i], 0));
    }
    SFQ_CUDA_TRY(cudaMemcpyAsync(d_in, h_in, sizeof(unsigned long long) * 2 * n, cudaMemcpyHostToDevice, gst));
    SFQ_CUDA_TRY(cudaGraphLaunch(it->second.exec, gst));
    SFQ_CUDA_TRY(cudaMemcpyAsync(h_out, d_out, sizeof(double) * kOut * n, cudaMemcpyDeviceToHost, gst));
    SFQ_CUDA_TRY(cudaEventRecord(ev_done, gst));
    for (size_t i = 0; i < n; ++i) {
      SFQ_CUDA_TRY(cudaStreamWaitEvent(es[i]->st, ev_done, 0));
      es[i]->inv_cached = it->second.inv_after[i] != 0;
      es[i]->inv_ov = it->second.inv_ov_after[i];
    }
    pending = &it->second;
    return SFQ_OK;
  }

  int block_query() {
    if (!pending) return 1;
    const cudaError_t q = cudaEventQuery(ev_done);
    if (q == cudaSuccess) return 1;
    if (q == cudaErrorNotReady) return 0;
    return -record_cuda(q, "cudaEventQuery", __FILE__, __LINE__);
  }

  // per member: Eshift, status (0, SFQ_ERR_WEIGHT_COLLAPSE, SFQ_ERR_TIMEOUT, ...), measurements
  int block_result(double* Eshift, int* status, double* meas, int max_meas, int* nmeas) {
    if (!pending) return record_error(SFQ_ERR_ARG, "group: no block was run");
    SFQ_CUDA_TRY(cudaEventSynchronize(ev_done));
    const Captured& c = *pending;
    pending = nullptr;
    int first = SFQ_OK;
    for (size_t i = 0; i < es.size(); ++i) {
      const double* o = h_out + (size_t)kOut * i;
      int s = SFQ_OK;
      if (o[2] != 0.0) {
        cudaMemsetAsync(es[i]->gemm_err, 0, sizeof(int), es[i]->st);
        s = SFQ_ERR_TIMEOUT;
      } else if (o[1] == double(SFQ_ERR_WEIGHT_COLLAPSE)) {
        s = SFQ_ERR_WEIGHT_COLLAPSE;
      } else if (o[1] != 0.0) {
        s = SFQ_ERR_INTERNAL;
      }
      if (status) status[i] = s;
      if (s && !first) first = s;
      if (Eshift) Eshift[i] = o[0];
      const int nm = c.nmeas[i] < max_meas ? c.nmeas[i] : max_meas;
      if (meas && nm > 0) std::memcpy(meas + (size_t)10 * max_meas * i, o + 4, sizeof(double) * 10 * nm);
      if (nmeas) nmeas[i] = c.nmeas[i];
    }
    if (first == SFQ_ERR_TIMEOUT)
      return record_error(first, "group: a tensor-core product's bounded wait expired in the block");
    if (first == SFQ_ERR_WEIGHT_COLLAPSE) return record_error(first, "group: a member's total walker weight collapsed.");
    if (first) return record_error(first, "group: population control: inconsistent copy plan");
    return SFQ_OK;
  }
};

}  // namespace sfq

struct sfq_engine_s {
  sfq::Engine e;
};

struct sfq_group_s {
  sfq::Group g;
};

using namespace sfq;

extern "C" {

void sfq_engine_params_default(sfq_engine_params_t* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->dt = 0.005;
  p->taylor_order = 6;
  p->vbias_bound = 50.0;
  p->lower_cutoff_scale = 1.0;
  p->upper_cutoff_scale = 10.0;
  p->weight_bound_floor = 100.0;
  p->weight_bound_fraction = 0.1;
  p->subtractMF = 1;
  p->denseP1 = 0;
  p->free_projection = 0;
  p->precision = SFQ_PRECISION_FP64;
  p->walker_type = SFQ_WALKER_CLOSED;
  p->nel_dn = 0;
}

int sfq_engine_create_nomsd(sfq_engine_t* out, const sfq_engine_params_t* p, const double* hcore, const double* Likn,
                            int ndet, const void* PsiT, const void* ci) {
  if (!out || !p || !hcore || !Likn || !PsiT || (ndet > 1 && !ci)) return record_error(SFQ_ERR_ARG, "null pointer");
  if (ndet < 1) return record_error(SFQ_ERR_SHAPE, "engine: ndet=%d", ndet);
  *out = nullptr;
  const int wt = p->walker_type == 0 ? SFQ_WALKER_CLOSED : p->walker_type;
  if (wt != SFQ_WALKER_CLOSED && wt != SFQ_WALKER_COLLINEAR && wt != SFQ_WALKER_NONCOLLINEAR)
    return record_error(SFQ_ERR_UNSUPPORTED, "engine: unknown walker type %d", p->walker_type);
  const bool coll = wt == SFQ_WALKER_COLLINEAR;
  const int npol = wt == SFQ_WALKER_NONCOLLINEAR ? 2 : 1;
  if (p->nmo <= 0 || p->nel <= 0 || p->nchol <= 0 || p->nwalk <= 0 || p->nel > npol * p->nmo ||
      (coll && (p->nel_dn < 0 || p->nel_dn > p->nmo)))
    return record_error(SFQ_ERR_SHAPE, "engine: invalid sizes nmo=%d nel=%d nel_dn=%d nchol=%d nwalk=%d", p->nmo,
                        p->nel, p->nel_dn, p->nchol, p->nwalk);
  const int ntot = p->nel + (coll ? p->nel_dn : 0);
  if (ntot > kMaxSmallN)
    return record_error(SFQ_ERR_UNSUPPORTED, "engine: %d electrons per walker exceed %d", ntot, kMaxSmallN);
  if (!(p->dt > 0.0)) return record_error(SFQ_ERR_ARG, "engine: dt must be positive");
  SFQ_CUDA_TRY(cudaSetDevice(p->device));
  auto* h = new sfq_engine_s();
  Engine& e = h->e;
  e.p = *p;
  e.M = p->nmo; e.N = ntot; e.Nc = p->nchol; e.W = p->nwalk;
  e.collinear = coll;
  e.nup = p->nel;
  e.npol = npol;
  e.Mr = npol * p->nmo;
  e.ndet = ndet;
  if (ndet > 1) {
    const cplx* c = reinterpret_cast<const cplx*>(ci);
    e.ci_h.assign(c, c + ndet);
  }
  const cplx* ps = reinterpret_cast<const cplx*>(PsiT);
  e.trial_real = true;
  for (long i = 0; i < (long)ndet * e.N * e.Mr; ++i)
    if (ps[i].y != 0.0) { e.trial_real = false; break; }
  e.nslices = p->precision == SFQ_PRECISION_INT8X3 ? 3 : p->precision == SFQ_PRECISION_INT8X2 ? 2 : 0;
  e.mixed = p->precision == SFQ_PRECISION_MIXED || p->precision == SFQ_PRECISION_MIXED_FP32 || e.nslices > 0;
  e.nplanes = p->precision == SFQ_PRECISION_MIXED_FP32 ? 3 : 2;
  if (p->precision != SFQ_PRECISION_FP64 && !e.mixed) {
    delete h;
    return record_error(SFQ_ERR_ARG, "engine: unknown precision %d", p->precision);
  }
  if (e.mixed && !e.nslices && (coll || npol > 1 || ndet > 1)) {
    delete h;
    return record_error(SFQ_ERR_UNSUPPORTED,
                        "engine: COLLINEAR and NONCOLLINEAR walkers and multi-determinant trials run in FP64 or the "
                        "int8-slice precisions");
  }
  if (e.nslices && e.M > 1024) {
    delete h;
    return record_error(SFQ_ERR_UNSUPPORTED, "engine: the int8-slice products need nmo <= 1024");
  }
  if (e.mixed && !e.nslices && (!e.trial_real || e.M % 8 || e.Nc % 8)) {
    delete h;
    return record_error(SFQ_ERR_UNSUPPORTED,
                        "engine: mixed precision needs a real trial and nmo, nchol multiples of 8 (nmo=%d nchol=%d)",
                        e.M, e.Nc);
  }
  int rc;
  cudaError_t ce = cudaStreamCreateWithFlags(&e.st, cudaStreamNonBlocking);
  if (ce != cudaSuccess) { delete h; return record_cuda(ce, "cudaStreamCreate", __FILE__, __LINE__); }
  if ((rc = e.allocate()) || (rc = e.setup(hcore, Likn, ps))) {
    sfq_engine_destroy(h);
    return rc;
  }
  *out = h;
  return SFQ_OK;
}

int sfq_engine_create(sfq_engine_t* out, const sfq_engine_params_t* p, const double* hcore, const double* Likn,
                      const void* PsiT) {
  return sfq_engine_create_nomsd(out, p, hcore, Likn, 1, PsiT, nullptr);
}

int sfq_engine_destroy(sfq_engine_t h) {
  if (!h) return SFQ_OK;
  Engine& e = h->e;
  if (e.st) cudaStreamSynchronize(e.st);
  e.release_events();
  e.drop_graphs();
  if (e.cst) cudaStreamSynchronize(e.cst);
  if (e.uni_ready) cudaEventDestroy(e.uni_ready);
  if (e.uni_free) cudaEventDestroy(e.uni_free);
  if (e.cst) cudaStreamDestroy(e.cst);
  if (e.blk_done) cudaEventDestroy(e.blk_done);
  if (e.blk_host) cudaFreeHost(e.blk_host);
  if (e.arena) cudaFree(e.arena);
  if (e.Lp) cudaFree(e.Lp);
  if (e.Vp) cudaFree(e.Vp);
  if (e.h_pinned) cudaFreeHost(e.h_pinned);
  if (e.rdm_buf) cudaFree(e.rdm_buf);
  for (void* q : {(void*)e.bp_SMN, (void*)e.bp_fields, (void*)e.bp_wfac, (void*)e.bp_refs, (void*)e.bp_ldet,
                  (void*)e.bp_wt, (void*)e.te_X, (void*)e.te_Y, (void*)e.te_M, (void*)e.te_scr, (void*)e.P1inv,
                  (void*)e.H1m})
    if (q) cudaFree(q);
  if (e.st) cudaStreamDestroy(e.st);
  delete h;
  return SFQ_OK;
}

int sfq_engine_synchronize(sfq_engine_t h) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.sync_checked();
}

void* sfq_engine_stream(sfq_engine_t h) { return h ? (void*)h->e.st : nullptr; }

int sfq_engine_set_walkers(sfq_engine_t h, const void* SM, const void* props) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  e.inv_cached = false;  // also the way to announce writes made through sfq_engine_info's SM pointer
  if (SM) SFQ_CUDA_TRY(cudaMemcpyAsync(e.SM, SM, sizeof(cplx) * e.W * e.Mr * e.N, cudaMemcpyHostToDevice, e.st));
  if (props) SFQ_CUDA_TRY(cudaMemcpyAsync(e.props, props, sizeof(cplx) * kNumProps * e.W, cudaMemcpyHostToDevice, e.st));
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  return SFQ_OK;
}

int sfq_engine_get_walkers(sfq_engine_t h, void* SM, void* props) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  if (SM) SFQ_CUDA_TRY(cudaMemcpyAsync(SM, e.SM, sizeof(cplx) * e.W * e.Mr * e.N, cudaMemcpyDeviceToHost, e.st));
  if (props) SFQ_CUDA_TRY(cudaMemcpyAsync(props, e.props, sizeof(cplx) * kNumProps * e.W, cudaMemcpyDeviceToHost, e.st));
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  return SFQ_OK;
}

int sfq_engine_export_walker_buffer(sfq_engine_t h, void* rows) {
  if (!h || !rows) return record_error(SFQ_ERR_ARG, "null pointer");
  Engine& e = h->e;
  const long mn = (long)e.Mr * e.N, rl = mn + 11;
  std::vector<cplx> sm(size_t(e.W) * mn), pr(size_t(kNumProps) * e.W);
  int rc;
  if ((rc = sfq_engine_get_walkers(h, sm.data(), pr.data()))) return rc;
  cplx* out = reinterpret_cast<cplx*>(rows);
  const int nu = e.collinear ? e.nup : e.N, nd = e.N - nu;
  for (int w = 0; w < e.W; ++w) {
    cplx* r = out + (size_t)w * rl;
    const cplx* s = sm.data() + (size_t)w * mn;
    if (nd == 0) {
      std::memcpy(r, s, sizeof(cplx) * mn);
    } else {  // the up block (M x nup) then the down block (M x ndn), WalkerSetBase.h:256-264
      for (int i = 0; i < e.M; ++i)
        for (int a = 0; a < e.N; ++a)
          r[a < nu ? (size_t)i * nu + a : (size_t)e.M * nu + (size_t)i * nd + (a - nu)] = s[(size_t)i * e.N + a];
    }
    // WEIGHT, PHASE, PSEUDO_ELOC_, E1_, EXX_, EJ_, OVLP, LOGSCL_UP, LOGSCL_DN, IS_UNITARY, THETA
    for (int k = 0; k < 7; ++k) r[mn + k] = pr[(size_t)k * e.W + w];
    r[mn + 7] = mk(0.0, 0.0);
    r[mn + 8] = mk(0.0, 0.0);
    r[mn + 9] = mk(0.0, 0.0);
    r[mn + 10] = pr[(size_t)P_THETA * e.W + w];
  }
  return SFQ_OK;
}

int sfq_engine_energy(sfq_engine_t h, int seed_pseudo, void* E3host) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  int rc;
  if ((rc = e.energy_only())) return rc;
  seed_pseudo_kernel<<<(e.W + 127) / 128, 128, 0, e.st>>>(e.props, e.E3, e.ovtmp, e.W, seed_pseudo ? 2 : 1);
  SFQ_LAUNCHED();
  if (E3host) SFQ_CUDA_TRY(cudaMemcpyAsync(E3host, e.E3, sizeof(cplx) * 3 * e.W, cudaMemcpyDeviceToHost, e.st));
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  return SFQ_OK;
}

int sfq_engine_propagate(sfq_engine_t h, double Eshift, unsigned long long step, const double* uniforms_dev) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.propagate(Eshift, step, uniforms_dev);
}

int sfq_engine_propagate_host(sfq_engine_t h, double Eshift, unsigned long long step, const double* uniforms_host,
                              void* props_host) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  int rc;
  const double* ud = nullptr;
  if (uniforms_host) {
    // the copy overlaps the step's density and force bias; it starts once earlier work on the
    // engine stream (a previous step's fields, which read the same buffer) is done
    if (!e.cst) {
      SFQ_CUDA_TRY(cudaStreamCreateWithFlags(&e.cst, cudaStreamNonBlocking));
      SFQ_CUDA_TRY(cudaEventCreateWithFlags(&e.uni_ready, cudaEventDisableTiming));
      SFQ_CUDA_TRY(cudaEventCreateWithFlags(&e.uni_free, cudaEventDisableTiming));
    }
    SFQ_CUDA_TRY(cudaEventRecord(e.uni_free, e.st));
    SFQ_CUDA_TRY(cudaStreamWaitEvent(e.cst, e.uni_free, 0));
    SFQ_CUDA_TRY(cudaMemcpyAsync(e.uni, uniforms_host, sizeof(double) * e.W * e.Nc, cudaMemcpyHostToDevice, e.cst));
    SFQ_CUDA_TRY(cudaEventRecord(e.uni_ready, e.cst));
    e.uni_wait = e.uni_ready;
    ud = e.uni;
  }
  rc = e.propagate(Eshift, step, ud);
  if (e.uni_wait) {  // not consumed (an error before the fields): keep the stream order anyway
    cudaStreamWaitEvent(e.st, e.uni_wait, 0);
    e.uni_wait = nullptr;
  }
  if (rc) return rc;
  if (props_host)
    SFQ_CUDA_TRY(cudaMemcpyAsync(props_host, e.props, sizeof(cplx) * kNumProps * e.W, cudaMemcpyDeviceToHost, e.st));
  return e.sync_checked();
}

int sfq_engine_orthogonalize(sfq_engine_t h) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.orthogonalize();
}

int sfq_engine_enable_back_propagation(sfq_engine_t h, int nbp) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.enable_bp(nbp);
}

int sfq_engine_enable_time_evolved_bp(sfq_engine_t h) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.te_enable();
}

int sfq_engine_te_anchor(sfq_engine_t h) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.te_anchor();
}

int sfq_engine_te_evolve(sfq_engine_t h, int nsteps) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.te_evolve(nsteps);
}

int sfq_engine_bp_anchor(sfq_engine_t h) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.bp_anchor();
}

static int fold_rdms(Engine& e, const std::vector<cplx>& one, const std::vector<cplx>& two, void* one_rdm,
                     void* diag_two_rdm);

int sfq_engine_measure_bp_rdm(sfq_engine_t h, int nsteps, int ortho_interval, int path_restoration, void* one_rdm,
                              void* diag_two_rdm) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  std::vector<cplx> one, two;
  int rc;
  if ((rc = e.measure_bp(nsteps, ortho_interval, path_restoration != 0, one, two))) return rc;
  return fold_rdms(e, one, two, one_rdm, diag_two_rdm);
}

int sfq_engine_measure_te_rdm(sfq_engine_t h, int restore_steps, void* one_rdm, void* diag_two_rdm) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  std::vector<cplx> one, two;
  int rc;
  if ((rc = e.te_measure(restore_steps, one, two, nullptr))) return rc;
  return fold_rdms(e, one, two, one_rdm, diag_two_rdm);
}

int sfq_engine_measure_rdm(sfq_engine_t h, void* one_rdm, void* diag_two_rdm) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  std::vector<cplx> one, two;
  int rc;
  if ((rc = e.measure_rdm(one, two))) return rc;
  return fold_rdms(e, one, two, one_rdm, diag_two_rdm);
}

namespace {
int obs_request(Engine& e, Engine::ObsSpec& o, void* two_rdm, void* spin_corr, int npair, const int* pair_maps,
                void* pair_corr) {
  o.two_rdm = two_rdm != nullptr;
  o.spin_corr = spin_corr != nullptr;
  o.npair = pair_corr ? npair : 0;
  o.maps = pair_maps;
  if (e.mixed) return record_error(SFQ_ERR_UNSUPPORTED, "the estimators' observables are measured in FP64 engines");
  return e.check_obs(o);
}
void obs_out(const Engine::ObsSpec& o, void* two_rdm, void* spin_corr, void* pair_corr) {
  if (two_rdm) std::memcpy(two_rdm, o.two.data(), sizeof(cplx) * o.two.size());
  if (spin_corr) std::memcpy(spin_corr, o.spin.data(), sizeof(cplx) * o.spin.size());
  if (pair_corr) std::memcpy(pair_corr, o.pair.data(), sizeof(cplx) * o.pair.size());
}
}  // namespace

int sfq_engine_measure_observables(sfq_engine_t h, void* two_rdm, void* spin_corr, int npair, const int* pair_maps,
                                   void* pair_corr) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  Engine::ObsSpec o;
  int rc;
  if ((rc = obs_request(e, o, two_rdm, spin_corr, npair, pair_maps, pair_corr))) return rc;
  std::vector<cplx> one, two;
  if ((rc = e.measure_rdm(one, two, &o))) return rc;
  obs_out(o, two_rdm, spin_corr, pair_corr);
  return SFQ_OK;
}

int sfq_engine_measure_bp_observables(sfq_engine_t h, int nsteps, int ortho_interval, int path_restoration,
                                      void* two_rdm, void* spin_corr, int npair, const int* pair_maps,
                                      void* pair_corr) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  Engine::ObsSpec o;
  int rc;
  if ((rc = obs_request(e, o, two_rdm, spin_corr, npair, pair_maps, pair_corr))) return rc;
  std::vector<cplx> one, two;
  if ((rc = e.measure_bp(nsteps, ortho_interval, path_restoration != 0, one, two, &o))) return rc;
  obs_out(o, two_rdm, spin_corr, pair_corr);
  return SFQ_OK;
}

int sfq_engine_measure_te_observables(sfq_engine_t h, int restore_steps, void* two_rdm, void* spin_corr, int npair,
                                      const int* pair_maps, void* pair_corr) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  Engine::ObsSpec o;
  int rc;
  if ((rc = obs_request(e, o, two_rdm, spin_corr, npair, pair_maps, pair_corr))) return rc;
  std::vector<cplx> one, two;
  if ((rc = e.te_measure(restore_steps, one, two, &o))) return rc;
  obs_out(o, two_rdm, spin_corr, pair_corr);
  return SFQ_OK;
}

static int fold_rdms(Engine& e, const std::vector<cplx>& one, const std::vector<cplx>& two, void* one_rdm,
                     void* diag_two_rdm) {
  if (one_rdm) std::memcpy(one_rdm, one.data(), sizeof(cplx) * one.size());
  if (!diag_two_rdm) return SFQ_OK;
  // fold the i <-> j symmetry (Observables/diagonal_twordm.hpp:104-140)
  cplx* out = static_cast<cplx*>(diag_two_rdm);
  const int M = e.M, R = e.Mr;
  auto at = [&](int b, int i, int j) { return two[((size_t)b * R + i) * R + j]; };
  auto half = [](cplx a, cplx b) { return mk(0.5 * (a.x + b.x), 0.5 * (a.y + b.y)); };
  long idx = 0;
  if (e.npol == 1) {
    for (int i = 0; i < M; ++i) {
      for (int j = i + 1; j < M; ++j) out[idx++] = half(at(0, i, j), at(0, j, i));
      for (int j = 0; j < M; ++j) out[idx++] = at(1, i, j);
    }
    if (e.collinear)
      for (int i = 0; i < M; ++i)
        for (int j = i + 1; j < M; ++j) out[idx++] = half(at(2, i, j), at(2, j, i));
  } else {
    for (int i = 0; i < 2 * M; ++i)
      for (int j = i + 1; j < 2 * M; ++j) out[idx++] = half(at(0, i, j), at(0, j, i));
  }
  return SFQ_OK;
}

int sfq_engine_population_control_uniform(sfq_engine_t h, double r) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  if (!(r >= 0.0 && r < 1.0)) return record_error(SFQ_ERR_ARG, "comb uniform %g outside [0, 1)", r);
  return h->e.population_control(0, r);
}

int sfq_engine_population_control(sfq_engine_t h, unsigned long long call) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.population_control(call);
}

int sfq_engine_averages(sfq_engine_t h, double* pseudo_energy, double* energy, double* total_weight) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  double o[10];
  int rc;
  if ((rc = h->e.averages(nullptr, o))) return rc;
  cplx num = mk(o[0], o[1]), den = mk(o[2], o[3]);
  // log(Re(sum w e^{dt eloc} / sum w)) / dt
  double re = (num.x * den.x + num.y * den.y) / (den.x * den.x + den.y * den.y);
  if (pseudo_energy) *pseudo_energy = std::log(re) / h->e.p.dt;
  if (energy) {
    cplx s = mk(o[4] + o[6] + o[8], o[5] + o[7] + o[9]);
    *energy = (s.x * den.x + s.y * den.y) / (den.x * den.x + den.y * den.y);
  }
  if (total_weight) *total_weight = den.x;
  return SFQ_OK;
}

int sfq_engine_measure(sfq_engine_t h, double* out10) {
  if (!h || !out10) return record_error(SFQ_ERR_ARG, "null pointer");
  Engine& e = h->e;
  int rc;
  if ((rc = e.energy_only())) return rc;
  double o[10];
  if ((rc = e.averages(e.E3, o))) return rc;
  // MeasurementOutput divides by sum_w (Measurements.hpp:101,120)
  auto div = [](double ar, double ai, double br, double bi, double* r) {
    double d = br * br + bi * bi;
    r[0] = (ar * br + ai * bi) / d;
    r[1] = (ai * br - ar * bi) / d;
  };
  double E1[2], EX[2], EJ[2];
  div(o[4], o[5], o[2], o[3], E1);
  div(o[6], o[7], o[2], o[3], EX);
  div(o[8], o[9], o[2], o[3], EJ);
  out10[0] = E1[0] + EX[0] + EJ[0];
  out10[1] = E1[1] + EX[1] + EJ[1];
  out10[2] = E1[0]; out10[3] = E1[1];
  out10[4] = EX[0]; out10[5] = EX[1];
  out10[6] = EJ[0]; out10[7] = EJ[1];
  out10[8] = o[2]; out10[9] = o[3];
  return SFQ_OK;
}

int sfq_engine_run(sfq_engine_t h, const sfq_run_params_t* rp, double* Eshift, double* meas, int max_meas,
                   int* nmeas) {
  if (!h || !rp || !Eshift) return record_error(SFQ_ERR_ARG, "null pointer");
  Engine& e = h->e;
  int rc;
  double relax = rp->Eshift_relaxation_factor;
  if (!(relax > 0.0)) relax = rp->equilibration_steps > 1 ? 1.0 - std::exp(-10.0 / rp->equilibration_steps) : 1.0;
  int nm = 0;
  for (unsigned long long step = rp->step0; step < rp->step0 + (unsigned long long)rp->steps; ++step) {
    if ((rc = e.propagate(*Eshift, step, nullptr))) return rc;
    if (rp->walker_ortho_interval > 0 && step % rp->walker_ortho_interval == 0)
      if ((rc = e.orthogonalize())) return rc;
    if (rp->population_control_interval > 0 && step % rp->population_control_interval == 0)
      if ((rc = e.population_control(step))) return rc;
    const bool equil = (long long)step < rp->equilibration_steps;
    if (!equil && rp->measure_interval > 0 && step % rp->measure_interval == 0) {
      double o[10];
      if ((rc = sfq_engine_measure(h, o))) return rc;
      if (meas && nm < max_meas) std::memcpy(meas + 10 * nm, o, sizeof(o));
      ++nm;
    }
    if (equil || rp->steer_eshift) {
      double pe;
      if ((rc = sfq_engine_averages(h, &pe, nullptr, nullptr))) return rc;
      *Eshift += relax * (pe - *Eshift);
    }
  }
  if (nmeas) *nmeas = nm;
  return e.sync_checked();
}

int sfq_engine_block(sfq_engine_t h, const sfq_run_params_t* rp, double* Eshift, double* meas, int max_meas,
                     int* nmeas) {
  if (!h || !rp || !Eshift) return record_error(SFQ_ERR_ARG, "null pointer");
  int rc;
  if ((rc = h->e.block_async(*rp, *Eshift))) return rc;
  return h->e.block_result(Eshift, meas, max_meas, nmeas);
}

int sfq_engine_block_async(sfq_engine_t h, const sfq_run_params_t* rp, double Eshift) {
  if (!h || !rp) return record_error(SFQ_ERR_ARG, "null pointer");
  return h->e.block_async(*rp, Eshift);
}

int sfq_engine_block_query(sfq_engine_t h) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.block_query();
}

int sfq_engine_block_result(sfq_engine_t h, double* Eshift, double* meas, int max_meas, int* nmeas) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.block_result(Eshift, meas, max_meas, nmeas);
}

int sfq_group_create(sfq_group_t* out, const sfq_engine_t* engines, int n) {
  if (!out || !engines || n <= 0) return record_error(SFQ_ERR_ARG, "group: no members");
  *out = nullptr;
  std::vector<Engine*> es;
  for (int i = 0; i < n; ++i) {
    if (!engines[i]) return record_error(SFQ_ERR_ARG, "group: null member %d", i);
    if (engines[i]->e.p.device != engines[0]->e.p.device)
      return record_error(SFQ_ERR_ARG, "group: members on different devices");
    for (int j = 0; j < i; ++j)
      if (engines[j] == engines[i]) return record_error(SFQ_ERR_ARG, "group: member %d repeated", i);
    if (engines[i]->e.nbp) return record_error(SFQ_ERR_UNSUPPORTED, "group: member %d keeps back propagation", i);
    es.push_back(&engines[i]->e);
  }
  sfq_group_t h = new sfq_group_s;
  const int rc = h->g.init(es);
  if (rc) {
    h->g.release();
    delete h;
    return rc;
  }
  *out = h;
  return SFQ_OK;
}

int sfq_group_destroy(sfq_group_t h) {
  if (!h) return SFQ_OK;
  h->g.release();
  delete h;
  return SFQ_OK;
}

int sfq_group_block_async(sfq_group_t h, const sfq_run_params_t* rps, const double* Eshift) {
  if (!h || !rps || !Eshift) return record_error(SFQ_ERR_ARG, "null pointer");
  return h->g.block_async(rps, Eshift);
}

int sfq_group_set_lanes(sfq_group_t h, int lanes) {
  if (!h) return record_error(SFQ_ERR_ARG, "null group");
  if (lanes < 0) return record_error(SFQ_ERR_ARG, "group: lanes must be >= 0");
  if (h->g.pending) return record_error(SFQ_ERR_ARG, "group: a block is running");
  h->g.lanes = lanes;
  return SFQ_OK;
}

int sfq_group_set_fused(sfq_group_t h, int fused) {
  if (!h) return record_error(SFQ_ERR_ARG, "null group");
  if (h->g.pending) return record_error(SFQ_ERR_ARG, "group: a block is running");
  return h->g.set_fused(fused != 0);
}

int sfq_group_block_query(sfq_group_t h) {
  if (!h) return record_error(SFQ_ERR_ARG, "null group");
  return h->g.block_query();
}

int sfq_group_block_result(sfq_group_t h, double* Eshift, int* status, double* meas, int max_meas, int* nmeas) {
  if (!h) return record_error(SFQ_ERR_ARG, "null group");
  return h->g.block_result(Eshift, status, meas, max_meas, nmeas);
}

int sfq_group_block(sfq_group_t h, const sfq_run_params_t* rps, double* Eshift, int* status, double* meas,
                    int max_meas, int* nmeas) {
  int rc;
  if ((rc = sfq_group_block_async(h, rps, Eshift))) return rc;
  return h->g.block_result(Eshift, status, meas, max_meas, nmeas);
}

int sfq_engine_autotune(sfq_engine_t h, int repeats, sfq_tiles_t* out) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.autotune(repeats, out);
}

int sfq_engine_set_tiles(sfq_engine_t h, const sfq_tiles_t* t) {
  if (!h || !t) return record_error(SFQ_ERR_ARG, "null pointer");
  return h->e.set_tiles(t->g_bn, t->vbias_bn, t->vhs_bn, t->taylor_half, t->p1_bn, t->vbias_ksplit);
}

int sfq_engine_tiles(sfq_engine_t h, sfq_tiles_t* t) {
  if (!h || !t) return record_error(SFQ_ERR_ARG, "null pointer");
  if (!h->e.mixed) return record_error(SFQ_ERR_UNSUPPORTED, "tiles: only the mixed-precision products are tiled");
  std::memset(t, 0, sizeof(*t));
  h->e.get_tiles(t);
  return SFQ_OK;
}

int sfq_engine_footprint(sfq_engine_t h, size_t* bytes) {
  if (!h || !bytes) return record_error(SFQ_ERR_ARG, "null pointer");
  const Engine& e = h->e;
  *bytes = e.arena_bytes + (e.Lp ? sizeof(double) * e.P * e.Nc : 0) + (e.Vp ? sizeof(cplx) * e.P * e.W : 0);
  return SFQ_OK;
}

int sfq_engine_profile(sfq_engine_t h, int enable) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  h->e.profile = enable != 0;
  return SFQ_OK;
}

int sfq_engine_phase_times(sfq_engine_t h, double* ms, int* counts, int nphase) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  return h->e.phase_times(ms, counts, nphase);
}

int sfq_engine_copy_walker(sfq_engine_t h, int from, int to) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  Engine& e = h->e;
  if (from < 0 || from >= e.W || to < 0 || to >= e.W)
    return record_error(SFQ_ERR_ARG, "copy_walker: slots %d, %d of %d", from, to, e.W);
  if (from == to) return SFQ_OK;
  const long mn = (long)e.Mr * e.N;
  SFQ_CUDA_TRY(cudaMemcpyAsync(e.SM + to * mn, e.SM + from * mn, sizeof(cplx) * mn, cudaMemcpyDeviceToDevice, e.st));
  SFQ_CUDA_TRY(cudaMemcpy2DAsync(e.props + to, sizeof(cplx) * e.W, e.props + from, sizeof(cplx) * e.W, sizeof(cplx),
                                 kNumProps, cudaMemcpyDeviceToDevice, e.st));
  e.inv_cached = false;
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  return SFQ_OK;
}

long sfq_engine_walker_row_elems(sfq_engine_t h) {
  if (!h) return -record_error(SFQ_ERR_ARG, "null engine");
  return (long)h->e.Mr * h->e.N + kNumProps;
}

namespace {
int exchange_checks(sfq_engine_t h, const void* list, int n, const void* rows, bool need_rows) {
  if (!h) return record_error(SFQ_ERR_ARG, "null engine");
  if (n < 0) return record_error(SFQ_ERR_ARG, "walker exchange: %d rows", n);
  if (n > 0 && (!list || (need_rows && !rows))) return record_error(SFQ_ERR_ARG, "walker exchange: null pointer");
  if (h->e.nbp)
    return record_error(SFQ_ERR_UNSUPPORTED, "walker exchange: the rows do not carry back-propagation history");
  return SFQ_OK;
}
}  // namespace

int sfq_engine_pack_walkers(sfq_engine_t h, const int* slots, int n, void* rows) {
  int rc;
  if ((rc = exchange_checks(h, slots, n, rows, true))) return rc;
  Engine& e = h->e;
  SFQ_CUDA_TRY(cudaSetDevice(e.p.device));
  if ((rc = pack_walker_rows(e.SM, e.props, e.W, (long)e.Mr * e.N, slots, n, static_cast<cplx*>(rows), e.st)))
    return record_error(rc, "pack_walkers: a slot outside [0, %d)", e.W);
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  return SFQ_OK;
}

int sfq_engine_unpack_walkers(sfq_engine_t h, const int* slots, int n, const void* rows) {
  int rc;
  if ((rc = exchange_checks(h, slots, n, rows, true))) return rc;
  Engine& e = h->e;
  SFQ_CUDA_TRY(cudaSetDevice(e.p.device));
  e.inv_cached = false;
  if ((rc = unpack_walker_rows(e.SM, e.props, e.W, (long)e.Mr * e.N, slots, n, static_cast<const cplx*>(rows), e.st)))
    return record_error(rc, "unpack_walkers: a slot outside [0, %d)", e.W);
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  return SFQ_OK;
}

int sfq_engine_copy_walkers(sfq_engine_t h, const int* pairs, int n, int normalize_weights) {
  int rc;
  if ((rc = exchange_checks(h, pairs, n, nullptr, false))) return rc;
  Engine& e = h->e;
  SFQ_CUDA_TRY(cudaSetDevice(e.p.device));
  e.inv_cached = false;
  if ((rc = copy_walker_pairs(e.SM, e.props, e.W, (long)e.Mr * e.N, pairs, n, normalize_weights, e.st)))
    return record_error(rc, "copy_walkers: pairs must lie in [0, %d), with distinct destinations that are no source",
                        e.W);
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  return SFQ_OK;
}

int sfq_engine_resize(sfq_engine_t* ph, int nwalk) {
  if (!ph || !*ph) return record_error(SFQ_ERR_ARG, "null engine");
  if (nwalk <= 0) return record_error(SFQ_ERR_ARG, "resize: %d walkers", nwalk);
  Engine& e = (*ph)->e;
  SFQ_CUDA_TRY(cudaSetDevice(e.p.device));
  if (nwalk == e.W) return SFQ_OK;
  // the inputs the engine was built from, back from the device
  const long MM = (long)e.M * e.M, RN = e.det_elems();
  std::vector<double> hc(MM), L(size_t(MM) * e.Nc);
  std::vector<cplx> ps(size_t(e.ndet) * RN);
  SFQ_CUDA_TRY(cudaMemcpyAsync(hc.data(), e.hcore, sizeof(double) * MM, cudaMemcpyDeviceToHost, e.st));
  SFQ_CUDA_TRY(cudaMemcpyAsync(L.data(), e.Likn, sizeof(double) * L.size(), cudaMemcpyDeviceToHost, e.st));
  SFQ_CUDA_TRY(cudaMemcpyAsync(ps.data(), e.PsiT, sizeof(cplx) * ps.size(), cudaMemcpyDeviceToHost, e.st));
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  sfq_engine_params_t p = e.p;
  p.nwalk = nwalk;
  sfq_engine_t nh = nullptr;
  int rc = e.ndet > 1 ? sfq_engine_create_nomsd(&nh, &p, hc.data(), L.data(), e.ndet, ps.data(), e.ci_h.data())
                      : sfq_engine_create(&nh, &p, hc.data(), L.data(), ps.data());
  if (rc) return rc;
  Engine& n = nh->e;
  const long mn = (long)e.Mr * e.N;
  for (int w = 0; w < nwalk && !rc; ++w) {  // slot w from slot w mod the old count
    const int src = w % e.W;
    cudaError_t ce = cudaMemcpyAsync(n.SM + w * mn, e.SM + src * mn, sizeof(cplx) * mn, cudaMemcpyDeviceToDevice, n.st);
    if (ce == cudaSuccess)
      ce = cudaMemcpy2DAsync(n.props + w, sizeof(cplx) * n.W, e.props + src, sizeof(cplx) * e.W, sizeof(cplx),
                             kNumProps, cudaMemcpyDeviceToDevice, n.st);
    if (ce != cudaSuccess) rc = record_cuda(ce, "resize: walker copy", __FILE__, __LINE__);
  }
  if (!rc) {
    const cudaError_t ce = cudaStreamSynchronize(n.st);
    if (ce != cudaSuccess) rc = record_cuda(ce, "resize", __FILE__, __LINE__);
  }
  if (rc) {
    sfq_engine_destroy(nh);
    return rc;
  }
  sfq_engine_destroy(*ph);
  *ph = nh;
  return SFQ_OK;
}

int sfq_engine_info(sfq_engine_t h, sfq_engine_info_t* info) {
  if (!h || !info) return record_error(SFQ_ERR_ARG, "null pointer");
  Engine& e = h->e;
  info->hcore = e.hcore;
  info->SM = e.SM;
  info->props = e.props;
  info->PsiT = e.PsiT;
  info->Lnak = e.Lnak;
  info->lnak_complex = e.trial_real ? 0 : 1;
  info->Likn = e.Likn;
  info->haj = e.haj;
  info->v0 = e.v0;
  info->vmf = e.vmf;
  info->P1 = e.P1;
  info->G = e.G;
  info->X = e.X;
  info->vHS = e.V;
  info->hw = e.hw;
  info->mf = e.mf;
  info->new_ovlp = e.newov;
  info->vhs_packed = e.sym ? 1 : 0;
  SFQ_CUDA_TRY(cudaMemcpyAsync(info->bound_stats, e.stats, sizeof(unsigned long long) * 5, cudaMemcpyDeviceToHost, e.st));
  SFQ_CUDA_TRY(cudaStreamSynchronize(e.st));
  return SFQ_OK;
}

}  // extern "C"
