// Composite device operations and the det_ops / HamOps C entry points.
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "ops.cuh"
#include <vector>
#include "umma_gemm.cuh"

namespace sfq {

// ---- error plumbing ------------------------------------------------------------------------
static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int record_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int record_cuda(cudaError_t e, const char* what, const char* file, int line) {
  if (e == cudaErrorMemoryAllocation)
    return record_error(SFQ_ERR_OOM, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  return record_error(SFQ_ERR_CUDA, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

namespace ops {

int overlap_matrix(const void* A, bool a_cplx, const cplx* B, cplx* T, int W, int M, int N, cudaStream_t st) {
  GemmDesc d;
  d.M = N; d.N = N; d.K = M; d.batch = W;
  d.A = A; d.sAm = M; d.sAk = 1; d.sAb = 0; d.a_cplx = a_cplx;
  d.B = B; d.sBk = N; d.sBn = 1; d.sBb = (long)M * N; d.b_cplx = true;
  d.C = T; d.sCm = N; d.sCn = 1; d.sCb = (long)N * N;
  return gemm_f64(d, st);
}

int green_compact(const cplx* Tinv, const cplx* B, cplx* G, int W, int M, int N, cudaStream_t st) {
  GemmDesc d;
  d.M = N; d.N = M; d.K = N; d.batch = W;
  d.A = Tinv; d.sAm = 1; d.sAk = N; d.sAb = (long)N * N; d.a_cplx = true;
  d.B = B; d.sBk = 1; d.sBn = N; d.sBb = (long)M * N; d.b_cplx = true;
  d.C = G; d.sCm = M; d.sCn = 1; d.sCb = (long)N * M;
  return gemm_f64(d, st);
}

int green_full(const void* A, bool a_cplx, const cplx* Gc, cplx* C, int W, int M, int N, cudaStream_t st) {
  GemmDesc d;
  d.M = M; d.N = M; d.K = N; d.batch = W;
  d.A = A; d.sAm = 1; d.sAk = M; d.sAb = 0; d.a_cplx = a_cplx;
  d.B = Gc; d.sBk = M; d.sBn = 1; d.sBb = (long)N * M; d.b_cplx = true;
  d.C = C; d.sCm = M; d.sCn = 1; d.sCb = (long)M * M;
  return gemm_f64(d, st);
}

int vbias(const cplx* G, const void* Lnak, bool l_cplx, cplx* v, int W, int N, int M, int Nc, double a,
          cudaStream_t st) {
  GemmDesc d;
  const long K = (long)N * M;
  d.M = W; d.N = Nc; d.K = int(K); d.batch = 1;
  d.A = G; d.sAm = K; d.sAk = 1; d.a_cplx = true;
  d.B = Lnak; d.sBk = 1; d.sBn = K; d.b_cplx = l_cplx;
  d.C = v; d.sCm = Nc; d.sCn = 1;
  d.alpha = mk(a, 0.0);
  return gemm_f64(d, st);
}

int vhs_rows(const double* L, long rows, const cplx* X, cplx* V, int W, int Nc, double a, cudaStream_t st) {
  GemmDesc d;
  d.M = W; d.N = int(rows); d.K = Nc; d.batch = 1;
  d.A = X; d.sAm = Nc; d.sAk = 1; d.a_cplx = true;
  d.B = L; d.sBk = 1; d.sBn = Nc; d.b_cplx = false;
  d.C = V; d.sCm = rows; d.sCn = 1;
  d.alpha = mk(a, 0.0);
  return gemm_f64(d, st);
}

int vhs(const double* Likn, const cplx* X, cplx* V, int W, int M, int Nc, double a, cudaStream_t st) {
  return vhs_rows(Likn, (long)M * M, X, V, W, Nc, a, st);
}

static int p1_apply(const void* P1, bool p_cplx, const cplx* in, cplx* out, int W, int M, int N, cudaStream_t st) {
  GemmDesc d;
  d.M = M; d.N = N; d.K = M; d.batch = W;
  d.A = P1; d.sAm = M; d.sAk = 1; d.sAb = 0; d.a_cplx = p_cplx;
  d.B = in; d.sBk = N; d.sBn = 1; d.sBb = (long)M * N; d.b_cplx = true;
  d.C = out; d.sCm = N; d.sCn = 1; d.sCb = (long)M * N;
  return gemm_f64(d, st);
}

int propagate(cplx* SM, const void* P1, bool p_cplx, const cplx* V, int W, int M, int N, int order, cplx* TMN,
              cplx* T1, cplx* T2, cudaStream_t st, int npol) {
  int rc;
  // npol = 2: spinor walkers (2M, N), the two components' M x N blocks one after the other; P1 and
  // V act on each component (propagate.hpp:247-298, polarization-independent vHS)
  const long n = (long)W * npol * M * N;
  // TMN = P1 * SM   (propagate.hpp:260)
  if ((rc = p1_apply(P1, p_cplx, SM, TMN, W * npol, M, N, st))) return rc;
  // apply_expM (propagate.hpp:45-70): T1 = S; T2 = (i/n) V T1; S += T2; swap
  SFQ_CUDA_TRY(cudaMemcpyAsync(T1, TMN, n * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
  cplx* a = T1;
  cplx* b = T2;
  const long MN = (long)M * N;
  for (int k = 1; k <= order; ++k) {
    for (int q = 0; q < npol; ++q) {
      GemmDesc d;
      d.M = M; d.N = N; d.K = M; d.batch = W;
      d.A = V; d.sAm = M; d.sAk = 1; d.sAb = (long)M * M; d.a_cplx = true;
      d.B = a + q * MN; d.sBk = N; d.sBn = 1; d.sBb = npol * MN; d.b_cplx = true;
      d.C = b + q * MN; d.sCm = N; d.sCn = 1; d.sCb = npol * MN;
      d.S = TMN + q * MN;
      d.alpha = mk(0.0, 1.0 / double(k));
      if ((rc = gemm_f64(d, st))) return rc;
    }
    cplx* t = a; a = b; b = t;
  }
  // SM = P1 * TMN   (propagate.hpp:297)
  return p1_apply(P1, p_cplx, TMN, SM, W * npol, M, N, st);
}

namespace {
// A[w][a][b] = 0 where a and b belong to different spins (a < nup <= b or b < nup <= a)
__global__ void mask_cross_spin_kernel(cplx* A, int N, int nup) {
  cplx* Aw = A + (long)blockIdx.x * N * N;
  const int ndn = N - nup;
  for (int e = threadIdx.x; e < nup * ndn; e += blockDim.x) {
    const int a = e / ndn, b = nup + e % ndn;
    Aw[(long)a * N + b] = mk(0.0, 0.0);
    Aw[(long)b * N + a] = mk(0.0, 0.0);
  }
}
}  // namespace

// COLLINEAR walkers (columns [0, nup) up, [nup, N) down): the per-walker N x N matrices keep only
// their two spin blocks; nothing to do unless both spins are occupied
int mask_cross_spin(cplx* A, int W, int N, int nup, cudaStream_t st) {
  if (nup <= 0 || nup >= N || W <= 0) return SFQ_OK;
  mask_cross_spin_kernel<<<W, 128, 0, st>>>(A, N, nup);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

// One CholeskyQR pass over the walkers selected by mask (all when null): S = Win^H Win = R^H R,
// Wout = Win R^-1; again[b] set from R's condition bound when again is not null.
// nup in (0, N): COLLINEAR walkers, columns [0, nup) up and [nup, N) down; the Gram matrix's
// cross-spin blocks are zeroed, so R, R^-1 and the new walkers are those of each spin on its own
// (orthogonalize.hpp:135-169 runs per spin).
static int cholqr_pass(const cplx* Win, cplx* Wout, cplx* S, int* status, int* again, const int* mask, int W, int M,
                       int N, cudaStream_t st, cplx* R = nullptr, int nup = -1) {
  int rc;
  GemmDesc d;  // S = Win^H Win
  d.M = N; d.N = N; d.K = M; d.batch = W;
  d.A = Win; d.sAm = 1; d.sAk = N; d.sAb = (long)M * N; d.a_cplx = true; d.conj_a = true;
  d.B = Win; d.sBk = N; d.sBn = 1; d.sBb = (long)M * N; d.b_cplx = true;
  d.C = S; d.sCm = N; d.sCn = 1; d.sCb = (long)N * N;
  d.mask = mask;
  d.upper_only = true;  // Hermitian: the Cholesky below reads the upper triangle only
  if ((rc = gemm_f64(d, st))) return rc;
  if ((rc = mask_cross_spin(S, W, N, nup, st))) return rc;
  if ((rc = chol_rinv(S, (long)N * N, W, N, status, again, mask, kCholQrKappa, st, R))) return rc;
  GemmDesc q;  // Wout = Win R^-1
  q.M = M; q.N = N; q.K = N; q.batch = W;
  q.A = Win; q.sAm = N; q.sAk = 1; q.sAb = (long)M * N; q.a_cplx = true;
  q.B = S; q.sBk = N; q.sBn = 1; q.sBb = (long)N * N; q.b_cplx = true;
  q.C = Wout; q.sCm = N; q.sCn = 1; q.sCb = (long)M * N;
  q.mask = mask;
  q.b_upper = true;  // R^-1 is upper triangular (its lower part stored as zeros)
  return gemm_f64(q, st);
}

// CholeskyQR2, with the second pass only where the first one's R was not well conditioned
// (kappa bound > kCholQrKappa: Q^H Q - I of one pass is of order eps kappa^2, <= 1e-12 below
// it).  status holds 2 W ints: the Cholesky status per walker, then the second-pass flags.
int orthogonalize(cplx* SM, cplx* SM2, cplx* S, int* status, cplx* log_detR, int W, int M, int N, cudaStream_t st,
                  int nup) {
  int rc;
  int* again = status + W;
  if ((rc = cholqr_pass(SM, SM2, S, status, again, nullptr, W, M, N, st, nullptr, nup))) return rc;
  if ((rc = cholqr_pass(SM2, SM, S, status, nullptr, again, W, M, N, st, nullptr, nup))) return rc;
  if ((rc = copy_walkers_where(SM, SM2, again, 0, W, (long)M * N, st))) return rc;  // one-pass walkers
  (void)log_detR;
  return SFQ_OK;
}

namespace {
// ov[w] -= scale * sum_i log r_ii over R[w] (real positive diagonal), one warp per walker, the sum
// in a fixed order; walkers with mask[w] == 0 are left alone (mask may be null)
__global__ void sub_logdiag_kernel(const cplx* R, int N, const int* mask, cplx* ov, double scale, int W) {
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= W || (mask && !mask[w])) return;
  const cplx* Rw = R + (long)w * N * N;
  double s = 0.0;
  for (int i = lane; i < N; i += 32) s += log(Rw[(long)i * N + i].x);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) ov[w].x -= scale * s;
}

// C[w] = R[w] Tin[w] (N x N complex, batch W; walkers with mask[w] == 0 skipped)
int rmul(const cplx* R, const cplx* Tin, cplx* C, const int* mask, int W, int N, cudaStream_t st) {
  GemmDesc d;
  d.M = N; d.N = N; d.K = N; d.batch = W;
  d.A = R; d.sAm = N; d.sAk = 1; d.sAb = (long)N * N; d.a_cplx = true;
  d.B = Tin; d.sBk = N; d.sBn = 1; d.sBb = (long)N * N; d.b_cplx = true;
  d.C = C; d.sCm = N; d.sCn = 1; d.sCb = (long)N * N;
  d.mask = mask;
  return gemm_f64(d, st);
}
}  // namespace

// orthogonalize() carrying the walkers' inverse overlap matrices and log overlaps through the
// QR instead of factoring the new overlaps again: with W' = W R^-1 (R = R2 R1 over the passes),
// (PsiT W')^-1 = R (PsiT W)^-1 and log det(PsiT W') = log det(PsiT W) - sum_i log r_ii, the r_ii
// real and positive (the phase is unchanged).  Tinv (W, N, N) and ov (W) in/out, scale = the
// number of identical determinants (2 for CLOSED walkers); S, R, Tw: (W, N, N) scratch.
int orthogonalize_carry(cplx* SM, cplx* SM2, cplx* S, cplx* R, cplx* Tw, int* status, cplx* Tinv, cplx* ov,
                        double scale, int W, int M, int N, cudaStream_t st, int nup) {
  int rc;
  int* again = status + W;
  const long NN = (long)N * N;
  if ((rc = cholqr_pass(SM, SM2, S, status, again, nullptr, W, M, N, st, R, nup))) return rc;
  if ((rc = rmul(R, Tinv, Tw, nullptr, W, N, st))) return rc;
  const int wpb = 8;
  sub_logdiag_kernel<<<(W + wpb - 1) / wpb, 32 * wpb, 0, st>>>(R, N, nullptr, ov, scale, W);
  SFQ_LAUNCHED();
  if ((rc = cholqr_pass(SM2, SM, S, status, nullptr, again, W, M, N, st, R, nup))) return rc;
  if ((rc = rmul(R, Tw, Tinv, again, W, N, st))) return rc;
  sub_logdiag_kernel<<<(W + wpb - 1) / wpb, 32 * wpb, 0, st>>>(R, N, again, ov, scale, W);
  SFQ_LAUNCHED();
  if ((rc = copy_walkers_where(SM, SM2, again, 0, W, (long)M * N, st))) return rc;  // one-pass walkers
  return copy_walkers_where(Tinv, Tw, again, 0, W, NN, st);
}

// orthogonalize() that also accumulates log det R = sum_i log r_ii of both passes into ldet (W):
// det_ops::orthogonalize(wset, ldet) with log_determinant_from_geqrf (orthogonalize.hpp:444-469;
// CholeskyQR's r_ii are real and positive, as Householder's after the sign fix)
int orthogonalize_logdet(cplx* SM, cplx* SM2, cplx* S, cplx* R, int* status, cplx* ldet, int W, int M, int N,
                         cudaStream_t st, int nup) {
  int rc;
  int* again = status + W;
  const int wpb = 8;
  if ((rc = cholqr_pass(SM, SM2, S, status, again, nullptr, W, M, N, st, R, nup))) return rc;
  sub_logdiag_kernel<<<(W + wpb - 1) / wpb, 32 * wpb, 0, st>>>(R, N, nullptr, ldet, -1.0, W);
  SFQ_LAUNCHED();
  if ((rc = cholqr_pass(SM2, SM, S, status, nullptr, again, W, M, N, st, R, nup))) return rc;
  sub_logdiag_kernel<<<(W + wpb - 1) / wpb, 32 * wpb, 0, st>>>(R, N, again, ldet, -1.0, W);
  SFQ_LAUNCHED();
  return copy_walkers_where(SM, SM2, again, 0, W, (long)M * N, st);  // one-pass walkers
}

int energy_chunk(int W, int N, int Nc, long max_elems) {
  long per = (long)W * N * N;
  long nv = per > 0 ? max_elems / per : Nc;
  if (nv < 1) nv = 1;
  if (nv > Nc) nv = Nc;
  return int(nv);
}

int energy(cplx* E3, const cplx* G, const cplx* haj, const void* Lnak, bool l_cplx, double E0, int W, int N, int M,
           int Nc, int addH1, int addEJ, int addEXX, cplx* Tchunk, long tchunk_elems, cplx* exxn, cplx* kl,
           cudaStream_t st, int nup) {
  int rc;
  const double scl = nup < 0 ? 2.0 : 1.0;  // CLOSED counts each orbital twice (energy, :148-173)
  if ((rc = energy_e1(G, haj, E3, W, N, M, E0, scl, addH1, st))) return rc;
  if (!addEXX && !addEJ) return SFQ_OK;
  const int nv_max = energy_chunk(W, N, Nc, tchunk_elems);
  const size_t esz = l_cplx ? sizeof(cplx) : sizeof(double);
  for (int n0 = 0; n0 < Nc; n0 += nv_max) {
    const int nv = (Nc - n0) < nv_max ? (Nc - n0) : nv_max;
    GemmDesc d;  // T[(w,b)][(n,a)] = sum_k G[w,b,k] Lnak[n0+n, a, k]
    d.M = W * N; d.N = nv * N; d.K = M; d.batch = 1;
    d.A = G; d.sAm = M; d.sAk = 1; d.a_cplx = true;
    d.B = (const unsigned char*)Lnak + (size_t)n0 * N * M * esz; d.sBk = 1; d.sBn = M; d.b_cplx = l_cplx;
    d.C = Tchunk; d.sCm = (long)nv * N; d.sCn = 1;
    if ((rc = gemm_f64(d, st))) return rc;
    if ((rc = energy_exx_reduce(Tchunk, W, N, nv, n0, Nc, exxn, kl, st, nup))) return rc;
  }
  return energy_finish(exxn, kl, E3, W, Nc, scl, addEXX, addEJ, st);
}

}  // namespace ops
}  // namespace sfq

// ============================================================================================
// C entry points: det_ops / HamiltonianOperations / propagator pieces
// ============================================================================================
using namespace sfq;

namespace {
inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
inline cudaStream_t S(void* p) { return reinterpret_cast<cudaStream_t>(p); }
constexpr long kEnergyChunkElems = 1L << 27;  // 2 GiB of complex T per chunk at most
}  // namespace

extern "C" {

int sfq_abi_version(void) { return 13; }

unsigned long long sfq_launch_count(void) { return g_launches.load(); }

int sfq_field_uniforms(double* out, unsigned long long seed, unsigned long long step, int nwalk, int nchol,
                       void* stream) {
  if (nwalk < 0 || nchol < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0 || nchol == 0) return SFQ_OK;
  if (!out) return record_error(SFQ_ERR_ARG, "null pointer");
  return field_uniforms(out, seed, step, nwalk, nchol, S(stream));
}

const char* sfq_last_error(void) { return g_last_error.c_str(); }

int sfq_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream) {
  if (bytes == 0) return SFQ_OK;
  if (!dst || !src) return record_error(SFQ_ERR_ARG, "null pointer");
  cudaMemcpyKind k = kind == 1 ? cudaMemcpyHostToDevice : kind == 2 ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  SFQ_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, k, S(stream)));
  SFQ_CUDA_TRY(cudaStreamSynchronize(S(stream)));
  return SFQ_OK;
}

size_t sfq_workspace_size(int op, int nwalk, int nmo, int nel, int nchol) {
  const size_t c = sizeof(cplx);
  switch (op) {
    case SFQ_OP_MIXED_DENSITY_MATRIX:
      return align256(c * nwalk * nel * nel) + align256(c * nwalk * nel * nmo);
    case SFQ_OP_LOG_OVERLAP:
      return align256(c * nwalk * nel * nel);
    case SFQ_OP_PROPAGATE:
      return 3 * align256(c * (size_t)nwalk * nmo * nel);
    case SFQ_OP_ORTHOGONALIZE:
      return align256(c * (size_t)nwalk * nmo * nel) + align256(c * nwalk * nel * nel) + align256(2 * sizeof(int) * nwalk);
    case SFQ_OP_ENERGY: {
      long nv = ops::energy_chunk(nwalk, nel, nchol, kEnergyChunkElems);
      return align256(c * (size_t)nwalk * nel * nv * nel) + 2 * align256(c * (size_t)nwalk * nchol);
    }
    case SFQ_OP_INVERSE_LOGDET:
      return 0;
    default:
      return 0;
  }
}

int sfq_mixed_density_matrix(const void* A, int a_complex, const void* B, void* C, void* ovlp, int nwalk, int nmo,
                             int nel, int compact, void* ws, size_t ws_bytes, void* stream) {
  if (nwalk < 0 || nmo < 0 || nel < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0) return SFQ_OK;
  if (nel == 0) {  // empty sector: overlap factor 1, G = 0 (density_matrix.hpp:563-566)
    if (!compact && nmo > 0)
      SFQ_CUDA_TRY(cudaMemsetAsync(C, 0, sizeof(cplx) * (size_t)nwalk * nmo * nmo, S(stream)));
    return SFQ_OK;
  }
  if (!A || !B || !C || !ovlp) return record_error(SFQ_ERR_ARG, "null pointer");
  if (ws_bytes < sfq_workspace_size(SFQ_OP_MIXED_DENSITY_MATRIX, nwalk, nmo, nel, 0))
    return record_error(SFQ_ERR_WORKSPACE, "mixed_density_matrix: workspace too small");
  cplx* T = (cplx*)ws;
  cplx* Gc = (cplx*)((char*)ws + align256(sizeof(cplx) * nwalk * nel * nel));
  int rc;
  if ((rc = ops::overlap_matrix(A, a_complex != 0, (const cplx*)B, T, nwalk, nmo, nel, S(stream)))) return rc;
  if ((rc = lu_logdet(T, (long)nel * nel, nwalk, nel, (cplx*)ovlp, true, 1.0, true, S(stream)))) return rc;
  if (compact) return ops::green_compact(T, (const cplx*)B, (cplx*)C, nwalk, nmo, nel, S(stream));
  if ((rc = ops::green_compact(T, (const cplx*)B, Gc, nwalk, nmo, nel, S(stream)))) return rc;
  return ops::green_full(A, a_complex != 0, Gc, (cplx*)C, nwalk, nmo, nel, S(stream));
}

int sfq_log_overlap(const void* A, int a_complex, const void* B, void* ovlp, int nwalk, int nmo, int nel, void* ws,
                    size_t ws_bytes, void* stream) {
  if (nwalk < 0 || nmo < 0 || nel < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0 || nel == 0) return SFQ_OK;
  if (!A || !B || !ovlp) return record_error(SFQ_ERR_ARG, "null pointer");
  if (ws_bytes < sfq_workspace_size(SFQ_OP_LOG_OVERLAP, nwalk, nmo, nel, 0))
    return record_error(SFQ_ERR_WORKSPACE, "log_overlap: workspace too small");
  cplx* T = (cplx*)ws;
  int rc;
  if ((rc = ops::overlap_matrix(A, a_complex != 0, (const cplx*)B, T, nwalk, nmo, nel, S(stream)))) return rc;
  return lu_logdet(T, (long)nel * nel, nwalk, nel, (cplx*)ovlp, true, 1.0, false, S(stream));
}

int sfq_inverse_logdet(const void* A, void* Ainv, void* logdet, int nbatch, int n, void* stream) {
  if (nbatch < 0 || n < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nbatch == 0 || n == 0) return SFQ_OK;
  if (!A || !Ainv || !logdet) return record_error(SFQ_ERR_ARG, "null pointer");
  SFQ_CUDA_TRY(cudaMemcpyAsync(Ainv, A, sizeof(cplx) * (size_t)nbatch * n * n, cudaMemcpyDeviceToDevice, S(stream)));
  return lu_logdet((cplx*)Ainv, (long)n * n, nbatch, n, (cplx*)logdet, true, 1.0, true, S(stream));
}

int sfq_propagate(void* SM, const void* P1, int p1_complex, const void* V, int nwalk, int nmo, int nel, int order,
                  void* ws, size_t ws_bytes, void* stream) {
  if (nwalk < 0 || nmo < 0 || nel < 0 || order < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0 || nel == 0 || nmo == 0) return SFQ_OK;
  if (!SM || !P1 || !V) return record_error(SFQ_ERR_ARG, "null pointer");
  if (ws_bytes < sfq_workspace_size(SFQ_OP_PROPAGATE, nwalk, nmo, nel, 0))
    return record_error(SFQ_ERR_WORKSPACE, "propagate: workspace too small");
  const size_t blk = align256(sizeof(cplx) * (size_t)nwalk * nmo * nel);
  cplx* TMN = (cplx*)ws;
  cplx* T1 = (cplx*)((char*)ws + blk);
  cplx* T2 = (cplx*)((char*)ws + 2 * blk);
  return ops::propagate((cplx*)SM, P1, p1_complex != 0, (const cplx*)V, nwalk, nmo, nel, order, TMN, T1, T2,
                        S(stream));
}

int sfq_orthogonalize(void* SM, void* log_detR, int nwalk, int nmo, int nel, void* ws, size_t ws_bytes,
                      void* stream) {
  if (nwalk < 0 || nmo < 0 || nel < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0 || nel == 0) return SFQ_OK;
  if (nel > nmo) return record_error(SFQ_ERR_SHAPE, "orthogonalize: nel > nmo");
  if (!SM) return record_error(SFQ_ERR_ARG, "null pointer");
  if (ws_bytes < sfq_workspace_size(SFQ_OP_ORTHOGONALIZE, nwalk, nmo, nel, 0))
    return record_error(SFQ_ERR_WORKSPACE, "orthogonalize: workspace too small");
  const size_t b1 = align256(sizeof(cplx) * (size_t)nwalk * nmo * nel);
  const size_t b2 = align256(sizeof(cplx) * (size_t)nwalk * nel * nel);
  cplx* SM2 = (cplx*)ws;
  cplx* Sb = (cplx*)((char*)ws + b1);
  int* status = (int*)((char*)ws + b1 + b2);
  return ops::orthogonalize((cplx*)SM, SM2, Sb, status, (cplx*)log_detR, nwalk, nmo, nel, S(stream));
}

int sfq_vbias(const void* G, const void* Lnak, int lnak_complex, void* v, int nwalk, int nel, int nmo, int nchol,
              double dt, int closed, void* stream) {
  if (nwalk < 0 || nel < 0 || nmo < 0 || nchol < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0 || nchol == 0) return SFQ_OK;
  if (!G || !Lnak || !v) return record_error(SFQ_ERR_ARG, "null pointer");
  const double a = std::sqrt(dt) * (closed ? 2.0 : 1.0);
  return ops::vbias((const cplx*)G, Lnak, lnak_complex != 0, (cplx*)v, nwalk, nel, nmo, nchol, a, S(stream));
}

int sfq_vhs(const double* Likn, const void* X, void* vHS, int nwalk, int nmo, int nchol, double dt, void* stream) {
  if (nwalk < 0 || nmo < 0 || nchol < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0 || nmo == 0) return SFQ_OK;
  if (!Likn || !X || !vHS) return record_error(SFQ_ERR_ARG, "null pointer");
  return ops::vhs(Likn, (const cplx*)X, (cplx*)vHS, nwalk, nmo, nchol, std::sqrt(dt), S(stream));
}

int sfq_one_body_matrix(const double* hcore, const double* v0, const double* Likn, const double* vMF, int nmo,
                        int nchol, double dt, double* H1, void* stream) {
  if (nmo <= 0 || nchol < 0) return record_error(SFQ_ERR_SHAPE, "one_body_matrix: sizes");
  if (!hcore || !v0 || !Likn || !H1 || (nchol > 0 && !vMF)) return record_error(SFQ_ERR_ARG, "null pointer");
  cudaStream_t st = S(stream);
  const long MM = (long)nmo * nmo;
  char* buf = nullptr;
  const size_t bx = (sizeof(cplx) * (nchol > 0 ? nchol : 1) + 255) & ~size_t(255);
  const size_t bv = (sizeof(cplx) * MM + 255) & ~size_t(255);
  SFQ_CUDA_TRY(cudaMallocAsync((void**)&buf, bx + bv + sizeof(double) * MM, st));
  cplx* X = reinterpret_cast<cplx*>(buf);
  cplx* V = reinterpret_cast<cplx*>(buf + bx);
  double* H = reinterpret_cast<double*>(buf + bx + bv);
  std::vector<cplx> xv(nchol > 0 ? nchol : 1);
  for (int n = 0; n < nchol; ++n) xv[n] = mk(vMF[n], 0.0);
  int rc = SFQ_OK;
  cudaError_t ce = cudaMemcpyAsync(X, xv.data(), sizeof(cplx) * xv.size(), cudaMemcpyHostToDevice, st);
  if (ce != cudaSuccess) rc = record_cuda(ce, "one_body_matrix: vMF", __FILE__, __LINE__);
  // the mean-field shift vHS(vMF) = sqrt(dt) sum_n L_n vMF_n (real for real Cholesky vectors)
  if (!rc && nchol > 0) rc = ops::vhs(Likn, X, V, 1, nmo, nchol, std::sqrt(dt), st);
  if (!rc && nchol == 0) {
    ce = cudaMemsetAsync(V, 0, sizeof(cplx) * MM, st);
    if (ce != cudaSuccess) rc = record_cuda(ce, "one_body_matrix", __FILE__, __LINE__);
  }
  if (!rc) rc = one_body_shift(hcore, v0, V, dt, H, nmo, st);
  if (!rc) {
    ce = cudaMemcpyAsync(H1, H, sizeof(double) * MM, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = record_cuda(ce, "one_body_matrix: H1", __FILE__, __LINE__);
  }
  cudaFreeAsync(buf, st);
  return rc;
}

int sfq_energy(void* E, const void* G, const void* haj, const void* Lnak, int lnak_complex, double E0, int nwalk,
               int nel, int nmo, int nchol, int addH1, int addEJ, int addEXX, void* ws, size_t ws_bytes,
               void* stream) {
  if (nwalk < 0 || nel < 0 || nmo < 0 || nchol < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0) return SFQ_OK;
  if (!E || !G || !haj || !Lnak) return record_error(SFQ_ERR_ARG, "null pointer");
  if (addEJ && !addEXX) return record_error(SFQ_ERR_UNSUPPORTED, "addEJ and not addEXX not yet implemented");
  if (ws_bytes < sfq_workspace_size(SFQ_OP_ENERGY, nwalk, nmo, nel, nchol))
    return record_error(SFQ_ERR_WORKSPACE, "energy: workspace too small");
  long nv = ops::energy_chunk(nwalk, nel, nchol, kEnergyChunkElems);
  const size_t bt = align256(sizeof(cplx) * (size_t)nwalk * nel * nv * nel);
  const size_t bk = align256(sizeof(cplx) * (size_t)nwalk * nchol);
  cplx* Tc = (cplx*)ws;
  cplx* exxn = (cplx*)((char*)ws + bt);
  cplx* kl = (cplx*)((char*)ws + bt + bk);
  return ops::energy((cplx*)E, (const cplx*)G, (const cplx*)haj, Lnak, lnak_complex != 0, E0, nwalk, nel, nmo, nchol,
                     addH1, addEJ, addEXX, Tc, (long)nwalk * nel * nv * nel, exxn, kl, S(stream));
}

int sfq_assemble_x(void* X, const double* vmf, void* hw, void* mf, const double* uniforms, unsigned long long seed,
                   unsigned long long step, int nwalk, int nchol, double vbias_bound, int free_projection,
                   void* stream) {
  if (nwalk < 0 || nchol < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0) return SFQ_OK;
  if (!X || !vmf || !hw || !mf) return record_error(SFQ_ERR_ARG, "null pointer");
  FieldParams p;
  p.nwalk = nwalk; p.nchol = nchol; p.vbias_bound = vbias_bound; p.free_projection = free_projection;
  p.seed = seed; p.step = step; p.uniforms = uniforms;
  return assemble_x((cplx*)X, vmf, (cplx*)hw, (cplx*)mf, p, S(stream));
}

int sfq_gemm_split_bf16(const double* A, const double* B, float* C, int M, int N, int K, int batch, int a_batched,
                        int b_batched, int nplanes, int tile_n, void* stream) {
  if (M < 0 || N < 0 || K < 0 || batch < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (!M || !N || !batch) return SFQ_OK;
  if (!A || !B || !C) return record_error(SFQ_ERR_ARG, "null pointer");
  if (K % 8) return record_error(SFQ_ERR_SHAPE, "sfq_gemm_split_bf16: K must be a multiple of 8");
  return gemm_split_bf16_f64(A, B, C, M, N, K, batch, a_batched, b_batched, nplanes, tile_n, S(stream));
}

int sfq_split_bf16(const double* src, long n, void* p0, void* p1, void* p2, void* stream) {
  if (n < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (n == 0) return SFQ_OK;
  if (!src || !p0) return record_error(SFQ_ERR_ARG, "null pointer");
  if (p2 && !p1) return record_error(SFQ_ERR_ARG, "plane 2 needs plane 1");
  return split_bf16_f64(src, n, p0, p1, p2, S(stream));
}

int sfq_gemm_bf16_planes(const void* const* A, const void* const* B, int nplanes, float* C, int M, int N, int K,
                         int batch, long a_batch_stride, long b_batch_stride, float alpha, float beta, int tile_n,
                         void* stream) {
  if (M < 0 || N < 0 || K < 0 || batch < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (!M || !N || !batch) return SFQ_OK;
  if (!A || !B || !C) return record_error(SFQ_ERR_ARG, "null pointer");
  if (nplanes < 1 || nplanes > 3) return record_error(SFQ_ERR_ARG, "nplanes must be 1, 2 or 3");
  UmmaGemmDesc d;
  d.M = M; d.N = N; d.K = K; d.batch = batch;
  for (int q = 0; q < nplanes; ++q) {
    d.A.p[q] = A[q];
    d.B.p[q] = B[q];
  }
  d.A.rows = M; d.A.ld = K; d.A.batch_stride = a_batch_stride;
  d.B.rows = N; d.B.ld = K; d.B.batch_stride = b_batch_stride;
  d.C = C; d.ldc = N; d.sCb = (long)M * N;
  d.alpha = alpha; d.beta = beta; d.nplanes = nplanes; d.bn = tile_n;
  return umma_gemm(d, S(stream));
}

int sfq_comb(const double* weights, double r, int nwalk, int* offspring, void* stream) {
  if (nwalk < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0) return SFQ_OK;
  if (!weights || !offspring) return record_error(SFQ_ERR_ARG, "null pointer");
  double* cum = nullptr;
  int* flag = nullptr;
  SFQ_CUDA_TRY(cudaMallocAsync((void**)&cum, sizeof(double) * nwalk + 256, S(stream)));
  flag = (int*)((char*)cum + ((sizeof(double) * nwalk + 15) & ~size_t(15)));
  int rc = comb_weights(weights, nwalk, r, offspring, cum, flag, S(stream));
  int h = 0;
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, S(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));
    if (e != cudaSuccess) rc = record_cuda(e, "sfq_comb", __FILE__, __LINE__);
  }
  cudaFreeAsync(cum, S(stream));
  if (rc) return rc;
  if (h == SFQ_ERR_WEIGHT_COLLAPSE) return record_error(h, "The total walker weight collapsed.");
  return h;
}

}  // extern "C"
