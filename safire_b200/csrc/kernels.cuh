// Internal kernel launchers shared by the C ABI and the resident engine.
#pragma once
#include "common.cuh"

namespace sfq {

constexpr int kMaxSmallN = 118;  // N x N complex + work (+ static) fits in 227 KB of shared memory

size_t lu_smem_bytes(int N);
constexpr int kGjMaxLarge = 100;  // register-resident Gauss-Jordan up to this N
int gj_logdet(cplx* T, long sT, int nbatch, int N, cplx* ovlp, bool accumulate, double post_scale, bool invert,
              cudaStream_t st);
// T: nbatch matrices N x N (row-major, batch stride sT); ovlp[b] = post_scale * fold(acc + logdet)
int lu_logdet(cplx* T, long sT, int nbatch, int N, cplx* ovlp, bool accumulate, double post_scale, bool invert,
              cudaStream_t st);
// S = R^H R and R^-1 over S; again[b] = 1 when R's condition bound exceeds kappa_max (may be
// null); batches with active[b] == 0 are left alone (active may be null); R itself (upper, zeros
// below) into Rout when it is not null
int chol_rinv(cplx* S, long sS, int nbatch, int N, int* status, int* again, const int* active, double kappa_max,
              cudaStream_t st, cplx* Rout = nullptr);

struct FieldParams {
  int nwalk = 0, nchol = 0;
  double vbias_bound = 50.0;
  int free_projection = 0;
  unsigned long long seed = 0, step = 0;
  const double* uniforms = nullptr;  // optional injected (nwalk, nchol) buffer, else Philox
  const unsigned long long* step_dev = nullptr;  // when set, the step is read from device memory
};
int field_uniforms(double* out, unsigned long long seed, unsigned long long step, int nwalk, int nchol,
                   cudaStream_t st);
// X: in = vbias (nwalk, nchol) complex, out = fields; vmf (nchol) real; hw, mf (nwalk) complex
int assemble_x(cplx* X, const double* vmf, cplx* hw, cplx* mf, const FieldParams& p, cudaStream_t st);

struct UpdateParams {
  int nwalk = 0;
  double dt = 0.0, Eshift = 0.0, E0 = 0.0;
  double lower_cutoff = 1.0, upper_cutoff = 10.0;
  double max_weight = 100.0;  // max(floor, fraction * target population)
  int hybrid = 1, free_projection = 0, use_cp_constraint = 0;
  const double* Eshift_dev = nullptr;  // when set, Eshift is read from device memory
  // back propagation: the step's weight factor (phase over projection, WalkerSetUpdate.hpp:141-147)
  // of walker i goes to wfac[i * wfac_stride] when wfac is set
  cplx* wfac = nullptr;
  long wfac_stride = 1;
  const unsigned long long* wfac_pos = nullptr;  // when set, the history slot *wfac_pos is added to wfac
};
struct WalkerProps {  // columns of the walker set (SoA), each nwalk complex
  cplx *weight, *phase, *pseudo_eloc, *e1, *exx, *ej, *ovlp, *theta;
};
// stats: 5 counters (eloc total, eloc upper, eloc lower, weight total, weight upper)
int walker_update(const WalkerProps& w, const cplx* new_ovlp, const cplx* mf, const cplx* hw, const cplx* E3,
                  const UpdateParams& p, unsigned long long* stats, cudaStream_t st);

// population control: comb on |weight| with one Philox draw, then copy walkers into the
// slots left free, in the order swap_walkers_async fills them; weights -> w/|w|.
struct PopWork {
  int* offspring;   // nwalk
  int* pairs;       // 2 * nwalk (src, dst)
  int* npairs;      // 1
  double* cum;      // nwalk
  int* flag;        // 1: 0 ok, SFQ_ERR_WEIGHT_COLLAPSE
};
// the rows of A (elems per walker) copied along the population-control plan pw (after population_control)
int copy_walker_rows(cplx* A, long elems, const PopWork& pw, int nwalk, cudaStream_t st);
// property columns of a walker table: WEIGHT, PHASE, PSEUDO_ELOC_, E1_, EXX_, EJ_, OVLP, THETA
constexpr int kWalkerProps = 8;
// Walker rows of the sharded exchange: row r = [Slater matrix of walker slots[r] (elems complex),
// its kWalkerProps property values] (props (kWalkerProps, nwalk) column-major by walker).
// pack: rows[r] <- walker slots[r]; unpack: walker slots[r] <- rows[r]; slots are host values.
int pack_walker_rows(const cplx* SM, const cplx* props, int nwalk, long elems, const int* slots, int n, cplx* rows,
                     cudaStream_t st);
int unpack_walker_rows(cplx* SM, cplx* props, int nwalk, long elems, const int* slots, int n, const cplx* rows,
                       cudaStream_t st);
// every weight w <- w / |w| (normalize != 0), then walker pairs[2k+1] <- walker pairs[2k] (Slater matrix
// and properties) for k < n; pairs are host values, no destination may also be a source
int copy_walker_pairs(cplx* SM, cplx* props, int nwalk, long elems, const int* pairs, int n, int normalize,
                      cudaStream_t st);
// call_dev: when set, the comb's call index is read from device memory
int population_control(cplx* SM, long walker_elems, const WalkerProps& w, int nwalk, double r_uniform,
                       unsigned long long seed, unsigned long long call, int use_philox, const PopWork& pw,
                       cudaStream_t st, const unsigned long long* call_dev = nullptr);

int comb_weights(const double* wts, int nwalk, double r, int* offspring, double* cum, int* flag, cudaStream_t st);

// energy pieces
int energy_e1(const cplx* G, const cplx* haj, cplx* E3, int nwalk, int nel, int nmo, double E0, double scl,
              int addH1, cudaStream_t st);
// T chunk (nwalk, nel, nv, nel): exxn[w, n0+n] = sum_ab T[a,n,b]T[b,n,a]; kl[w, n0+n] = sum_a T[a,n,a]
// nup >= 0: COLLINEAR walkers, the exchange pairs orbitals of one spin only ([0, nup) and [nup, nel))
int energy_exx_reduce(const cplx* T, int nwalk, int nel, int nv, int n0, int nchol, cplx* exxn, cplx* kl,
                      cudaStream_t st, int nup = -1);
// the same from FP32 planar T of the split-BF16 product: rows (c*W + w)*nel + a, columns n*nel + b
int energy_exx_reduce_f32(const float* C, int nwalk, int nel, int nv, int n0, int nchol, long ldc, cplx* exxn,
                          cplx* kl, cudaStream_t st, int nup = -1);
// E3[:,1] += -0.5*scl*sum_n exxn; E3[:,2] += (CLOSED ? 2 : 0.5) * sum_n kl^2
int energy_finish(const cplx* exxn, const cplx* kl, cplx* E3, int nwalk, int nchol, double scl, int addEXX,
                  int addEJ, cudaStream_t st);

// misc
// [a][k][n] -> [n][a][k], complex or real (elements of esz bytes: 8 or 16)
int permute_lnak(const void* tmp, void* Lnak, int nel, int nmo, int nchol, int esz, cudaStream_t st);
// H[i][k] = -0.5 * herm(dt*h + dt*v0 + Re vhs)  (real symmetric one-body matrix of P1)
int build_h1(const double* h, const double* v0, const cplx* vhs, double dt, double* H, int nmo, cudaStream_t st);
int add_identity(double* P, int nmo, double v, cudaStream_t st);
// H = dt (h + v0) + Re vhs  (add_one_body_shifts)
int one_body_shift(const double* h, const double* v0, const cplx* vhs, double dt, double* H, int nmo,
                   cudaStream_t st);
int threshold_real(double* P, long n, double drop, cudaStream_t st);
int real_of(const cplx* z, double* r, long n, cudaStream_t st);
int fill_cplx(cplx* p, long n, cplx v, cudaStream_t st);
int copy_walkers_prop(cplx* dst, const cplx* src, long n, cudaStream_t st);
// dst walker w = src walker w (n elements each) where (mask[w] != 0) == want
int copy_walkers_where(cplx* dst, const cplx* src, const int* mask, int want, int W, long n, cudaStream_t st);
// condition bound below which one CholeskyQR pass is kept
constexpr double kCholQrKappa = 100.0;
int scale_cplx(cplx* p, long n, cplx s, cudaStream_t st);

// Symmetric Cholesky vectors, L[i][k][n] == L[k][i][n]: the upper triangle i <= k, row-major,
// holds everything, and vHS = sum_n X_n L_n is symmetric too.
__host__ __device__ inline long upper_index(long i, long k, long M) { return i * M - i * (i - 1) / 2 + (k - i); }
// flag |= 1 when some L[i][k][n] and L[k][i][n] differ in any bit
int check_symmetric(const double* L, int M, int Nc, int* flag, cudaStream_t st);
// Lp[upper_index(i, k)][n] = L[i][k][n], i <= k
int pack_upper(const double* L, int M, int Nc, double* Lp, cudaStream_t st);
// V[w][i][k] = V[w][k][i] = Vp[w][upper_index(min, max)]
int unpack_symmetric(const cplx* Vp, int W, int M, cplx* V, cudaStream_t st);

}  // namespace sfq
