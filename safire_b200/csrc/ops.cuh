// Composite operations on device arrays (the bodies of the det_ops / HamOps entry points).
#pragma once
#include "common.cuh"
#include "gemm_f64.cuh"
#include "kernels.cuh"

namespace sfq {
namespace ops {

// T[w] = A * B[w]  (A: nel x nmo shared, real or complex; B: (W, nmo, nel) complex) -> (W, nel, nel)
int overlap_matrix(const void* A, bool a_cplx, const cplx* B, cplx* T, int W, int M, int N, cudaStream_t st);
// G[w] = Tinv[w]^T * B[w]^T -> (W, nel, nmo)
int green_compact(const cplx* Tinv, const cplx* B, cplx* G, int W, int M, int N, cudaStream_t st);
// C[w] = A^T * Gc[w] -> (W, nmo, nmo)   (non-compact, herm = true)
int green_full(const void* A, bool a_cplx, const cplx* Gc, cplx* C, int W, int M, int N, cudaStream_t st);
int vbias(const cplx* G, const void* Lnak, bool l_cplx, cplx* v, int W, int N, int M, int Nc, double a,
          cudaStream_t st);
int vhs(const double* Likn, const cplx* X, cplx* V, int W, int M, int Nc, double a, cudaStream_t st);
// V (W, rows) = a X L^T for L (rows, Nc): rows = M*M, or the packed upper triangle of symmetric L
int vhs_rows(const double* L, long rows, const cplx* X, cplx* V, int W, int Nc, double a, cudaStream_t st);
// SM <- P1 * Taylor(iV) * P1 * SM with scratch TMN, T1, T2 (each W*M*N complex)
int propagate(cplx* SM, const void* P1, bool p_cplx, const cplx* V, int W, int M, int N, int order, cplx* TMN,
              cplx* T1, cplx* T2, cudaStream_t st, int npol = 1);
// CholeskyQR2; SM2 (W*M*N), S (W*N*N) scratch, status (W) ints.  log_detR (W) accumulated if not null
// CholeskyQR2 in place on SM (SM2, S: scratch; status: 2 W ints)
// nup in (0, N) (here and below): COLLINEAR walkers, columns [0, nup) up and [nup, N) down, each spin
// on its own; -1: CLOSED
int orthogonalize(cplx* SM, cplx* SM2, cplx* S, int* status, cplx* log_detR, int W, int M, int N, cudaStream_t st,
                  int nup = -1);
// the same, carrying the inverse overlap matrices Tinv (W, N, N) and log overlaps ov (W) of the
// walkers through the QR ((PsiT W R^-1)^-1 = R (PsiT W)^-1, log det drops by scale * sum log r_ii);
// S, R, Tw: (W, N, N) scratch
int orthogonalize_carry(cplx* SM, cplx* SM2, cplx* S, cplx* R, cplx* Tw, int* status, cplx* Tinv, cplx* ov,
                        double scale, int W, int M, int N, cudaStream_t st, int nup = -1);
// the same QR accumulating log det R into ldet (W); S, R: (W, N, N) scratch
int orthogonalize_logdet(cplx* SM, cplx* SM2, cplx* S, cplx* R, int* status, cplx* ldet, int W, int M, int N,
                         cudaStream_t st, int nup = -1);
// zero the cross-spin blocks of W per-walker N x N matrices (a no-op unless 0 < nup < N)
int mask_cross_spin(cplx* A, int W, int N, int nup, cudaStream_t st);
// energy with chunked T; ws: T chunk (W*N*nv*N) + exxn (W*Nc) + kl (W*Nc)
// nup >= 0: COLLINEAR (scale 1, exchange within each spin, Coulomb 0.5 (sum of both spins' traces)^2);
// -1: CLOSED (scale 2)
int energy(cplx* E3, const cplx* G, const cplx* haj, const void* Lnak, bool l_cplx, double E0, int W, int N, int M,
           int Nc, int addH1, int addEJ, int addEXX, cplx* Tchunk, long tchunk_elems, cplx* exxn, cplx* kl,
           cudaStream_t st, int nup = -1);
int energy_chunk(int W, int N, int Nc, long max_elems);

}  // namespace ops
}  // namespace sfq
