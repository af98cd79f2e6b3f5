/*
 * SAFIRE-B200: C ABI for the AFQMC walker-propagation / local-energy path on one B200.
 *
 * The reference exposes this path as C++ templates (nda arrays parameterised by MEMORY_SPACE);
 * every entry point below replaces one of those calls for MEMORY_SPACE = DEVICE_MEMORY,
 * CLOSED walkers, a single-determinant trial and a dense real Cholesky Hamiltonian
 * (Real3IndexFactorization).  Reference paths are relative to the SAFIRE source tree.
 *
 * Conventions
 *  - complex numbers are interleaved (re, im) doubles, the layout of std::complex<double>;
 *  - arrays are C-ordered (row-major) exactly as the reference stores them;
 *  - "device" pointers are CUDA device addresses on the current device; `stream` is a
 *    cudaStream_t (NULL = legacy default stream);
 *  - functions return 0 (SFQ_OK) or an SFQ_ERR_* code and never throw; sfq_last_error()
 *    returns a description of the last failure on the calling thread.
 *  - workspace-taking functions need `ws_bytes >= sfq_workspace_size(...)` of device memory.
 */
#ifndef SAFIRE_B200_H
#define SAFIRE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SFQ_OK 0
#define SFQ_ERR_SHAPE 1           /* utils::check size mismatch (src/utilities/check.hpp:36-46) */
#define SFQ_ERR_ARG 2             /* invalid argument / null pointer */
#define SFQ_ERR_UNSUPPORTED 3     /* size or combination this build does not implement */
#define SFQ_ERR_CUDA 4            /* CUDA runtime error (cuda_check, src/arch/cuda_init.cpp:60-70) */
#define SFQ_ERR_OOM 5             /* device allocation failed */
#define SFQ_ERR_WEIGHT_COLLAPSE 6 /* comb: total weight <= 1e-6 (population_control.hpp:39) */
#define SFQ_ERR_NONFINITE 7       /* non-finite input where one is not allowed */
#define SFQ_ERR_TIMEOUT 8         /* bounded device wait expired */
#define SFQ_ERR_WORKSPACE 9       /* workspace smaller than sfq_workspace_size() */
#define SFQ_ERR_INTERNAL 10       /* internal consistency check failed */
#define SFQ_ERR_RANK 11           /* CholeskyQR: a walker lost rank (non-positive pivot) */

/* version of this ABI */
int sfq_abi_version(void); /* 13 */
const char* sfq_last_error(void);
/* kernels this library has launched in this process (all threads, all devices) */
unsigned long long sfq_launch_count(void);
/* cudaMemcpyAsync + stream synchronize (kind: 1 H2D, 2 D2H, 3 D2D), for callers without a CUDA runtime */
int sfq_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream);

/* ---------------------------------------------------------------------------------------
 * det_ops (src/AFQMC/SlaterDeterminantOperations/)
 * --------------------------------------------------------------------------------------- */
enum sfq_op {
  SFQ_OP_MIXED_DENSITY_MATRIX = 1,
  SFQ_OP_LOG_OVERLAP = 2,
  SFQ_OP_PROPAGATE = 3,
  SFQ_OP_ORTHOGONALIZE = 4,
  SFQ_OP_ENERGY = 5,
  SFQ_OP_INVERSE_LOGDET = 6
};
/* device bytes of scratch the op needs for these sizes */
size_t sfq_workspace_size(int op, int nwalk, int nmo, int nel, int nchol);

/* det_ops::MixedDensityMatrix(A, B, C, ovlp, compact, herm=true)
 *   density_matrix.hpp:544-601 (log_overlap_impl :120-156, getri_or_zero nda_functions.hpp:422-438)
 * A: trial PsiT (nel x nmo), complex if a_complex else real;  B: walkers (nwalk, nmo, nel) complex;
 * C: compact ? (nwalk, nel, nmo) : (nwalk, nmo, nmo) complex;  ovlp: (nwalk) complex, accumulated
 * (log det folded to [-pi, pi]).  A singular overlap gives a zero inverse, as in the reference. */
int sfq_mixed_density_matrix(const void* A, int a_complex, const void* B, void* C, void* ovlp, int nwalk, int nmo,
                             int nel, int compact, void* ws, size_t ws_bytes, void* stream);

/* Compact mixed density matrix with no allocation at all (no counterpart in the reference).
 * Same arguments and results as sfq_mixed_density_matrix(..., compact = 1, ...) but without a
 * workspace: for callers that cannot allocate device memory (a host program whose allocator owns
 * all of it, an FFI binding without a CUDA runtime, a loop that cannot afford cudaMalloc's
 * device-wide synchronisation).  Scratch is a fixed array of sfq_noalloc_scratch_bytes() (16 MiB)
 * compiled into the library and held on every GPU that loads it until the process exits; calls
 * with nwalk * nel * nel * 16 bytes above that return SFQ_ERR_WORKSPACE.  All calls on a device
 * share the array, so calls that overlap on the GPU race; the first call in each context looks up
 * the array's address and should come before any stream capture; the address is kept with the
 * context's id, so a context created anew (after cudaDeviceReset) is looked up again. */
int sfq_mixed_density_matrix_noalloc(const void* A, int a_complex, const void* B, void* C, void* ovlp, int nwalk,
                                     int nmo, int nel, void* stream);
size_t sfq_noalloc_scratch_bytes(void);

/* det_ops::Log_Overlap(A, B, ovlp, herm=true)   density_matrix.hpp:437-447 (accumulates into ovlp) */
int sfq_log_overlap(const void* A, int a_complex, const void* B, void* ovlp, int nwalk, int nmo, int nel, void* ws,
                    size_t ws_bytes, void* stream);

/* det_ops::detail::inverse_logdet(A, ovlp, TNN)   density_matrix.hpp:82-108
 * A (nbatch, n, n) complex (read only), Ainv (nbatch, n, n) complex out, logdet (nbatch) accumulated */
int sfq_inverse_logdet(const void* A, void* Ainv, void* logdet, int nbatch, int n, void* stream);

/* det_ops::Propagate<DEVICE,'N'>(wset, P1, V, order) for CLOSED walkers   propagate.hpp:247-298,391-408
 * SM (nwalk, nmo, nel) complex updated in place:  SM <- P1 * sum_k (i V)^k/k! * P1 * SM;
 * P1 (nmo, nmo) complex if p1_complex else real;  V (nwalk, nmo, nmo) complex */
int sfq_propagate(void* SM, const void* P1, int p1_complex, const void* V, int nwalk, int nmo, int nel, int order,
                  void* ws, size_t ws_bytes, void* stream);

/* det_ops::orthogonalize(A, log_detR)   orthogonalize.hpp:135-169
 * SM (nwalk, nmo, nel) complex replaced by Q with a positive real R diagonal (CholeskyQR2);
 * log_detR (nwalk) complex accumulated with sum_i log R_ii, may be NULL. */
int sfq_orthogonalize(void* SM, void* log_detR, int nwalk, int nmo, int nel, void* ws, size_t ws_bytes,
                      void* stream);

/* ---------------------------------------------------------------------------------------
 * HamiltonianOperations -> Real3IndexFactorization (src/AFQMC/HamiltonianOperations/)
 * --------------------------------------------------------------------------------------- */

/* vbias(G, v, dt)   Real3IndexFactorization.hpp:328-428 (ndet = 1, compact G)
 * v[w,n] = a * sum_{a,k} G[w,a,k] Lnak[n,a,k];  a = sqrt(dt) * (closed ? 2 : 1)
 * G (nwalk, nel*nmo) complex; Lnak (nchol, nel, nmo) complex if lnak_complex else real; v (nwalk, nchol) */
int sfq_vbias(const void* G, const void* Lnak, int lnak_complex, void* v, int nwalk, int nel, int nmo, int nchol,
              double dt, int closed, void* stream);

/* vHS(X, dt)   Real3IndexFactorization.hpp:282-326
 * vHS[w,i,k] = sqrt(dt) * sum_n Likn[i,k,n] X[w,n];  Likn (nmo, nmo, nchol) real; X (nwalk, nchol) complex;
 * vHS (nwalk, nmo, nmo) complex */
int sfq_vhs(const double* Likn, const void* X, void* vHS, int nwalk, int nmo, int nchol, double dt, void* stream);

/* energy(E, G, idet=0, addH1, addEJ, addEXX)   Real3IndexFactorization.hpp:138-174, energy_impl :476-590
 * E (nwalk, 3) complex out [E1, EXX, EJ]; G (nwalk, nel*nmo); haj (nel, nmo) complex; Lnak as in vbias;
 * CLOSED scaling (scl = 2, EJ factor 2). */
int sfq_energy(void* E, const void* G, const void* haj, const void* Lnak, int lnak_complex, double E0, int nwalk,
               int nel, int nmo, int nchol, int addH1, int addEJ, int addEXX, void* ws, size_t ws_bytes,
               void* stream);

/* ---------------------------------------------------------------------------------------
 * AFQMCBasePropagator pieces (src/AFQMC/Propagators/)
 * --------------------------------------------------------------------------------------- */

/* assemble_X + construct_X_impl + meanfield_factor   AFQMCBasePropagator.cpp:687-733,335-336;
 * construct_X_kernel.hpp:34-87.  X (nwalk, nchol) complex: in = vbias, out = fields;
 * vmf (nchol) real; hw, mf (nwalk) complex out.  uniforms (nwalk, nchol) doubles in (0,1) replace
 * sampleUniformFields when not NULL; otherwise Philox(seed, step) is drawn in-kernel. */
int sfq_assemble_x(void* X, const double* vmf, void* hw, void* mf, const double* uniforms, unsigned long long seed,
                   unsigned long long step, int nwalk, int nchol, double vbias_bound, int free_projection,
                   void* stream);

/* RandomGenerator_t::sampleUniformFields for one step (Random.hpp:37-83, replaced by Philox-4x32-10):
 * out (nwalk, nchol) doubles in (0,1), device; the same draws the engine makes in-kernel for (seed, step). */
int sfq_field_uniforms(double* out, unsigned long long seed, unsigned long long step, int nwalk, int nchol,
                       void* stream);

/* comb(rng, weights, num_target)   population_control.hpp:34-65
 * weights (nwalk) doubles (|w|), device;  offspring (nwalk) ints, device;  r: the comb's uniform.
 * Returns SFQ_ERR_WEIGHT_COLLAPSE when the total weight is <= 1e-6. */
int sfq_comb(const double* weights, double r, int nwalk, int* offspring, void* stream);

/* Population control over walkers sharded across ranks: host-only planning, no device needed
 * (population_control.hpp:34-255).  The global population is rank-major: rank r holds counts[r]
 * walkers, and its walker i is entry counts[0] + ... + counts[r-1] + i of weights / offspring.
 *
 * comb(rng, weights, num_target) on the root over the gathered |w| (host memory):
 * offspring (nwalk) receives the copies of each walker; SFQ_ERR_WEIGHT_COLLAPSE when the total
 * weight is <= 1e-6.  Same comparisons, in the same order, as sfq_comb. */
int sfq_comb_host(const double* weights, double r, int nwalk, int num_target, int* offspring);

/* plan_walker_exchange (population_control.hpp:73-133): the transfers realising offspring, as
 * (src rank, local walker on src, dst rank, copies dst ends with) quadruples in plan order.  Ranks
 * with excess export their walkers with the most copies first (ties in index order), filling the
 * ranks with a deficit in rank order.  Deterministic: every rank computes the same plan.
 * *ntransfers is set to the plan's length; SFQ_ERR_WORKSPACE when it exceeds capacity (at most
 * sum(counts) + nranks transfers).  SFQ_ERR_ARG when offspring does not preserve the population. */
int sfq_plan_walker_exchange(const int* offspring, const int* counts, int nranks, int* transfers, int capacity,
                             int* ntransfers);

/* rank's part of swap_walkers_async (population_control.hpp:143-209), all as (int, int) pairs:
 *   sends   (local walker, dst rank), in plan order          at most counts[rank] + nranks pairs
 *   recvs   (slot, src rank), in plan order                   at most counts[rank] pairs
 *   copies  (src slot, dst slot), made after the receives     at most counts[rank] pairs
 * max_sends, max_recvs and max_copies are the pairs each array has room for.  When one is too
 * small nothing is written, the three counts are set to the lengths needed and SFQ_ERR_WORKSPACE
 * is returned (a walker exported to several deficit ranks makes more sends than walkers).
 * A walker received into a slot replaces the walker that left it; local copies fill the remaining
 * free slots, the kept walkers' extra copies (in index order) first, then the received walkers'. */
int sfq_walker_moves(const int* offspring, const int* counts, int nranks, int rank, int* sends, int max_sends,
                     int* nsends, int* recvs, int max_recvs, int* nrecvs, int* copies, int max_copies, int* ncopies);

/* Mixed-precision tensor-core GEMM (tcgen05, split BF16, FP32 accumulation), no reference
 * counterpart: C[b] (M x N, fp32) = A[b] (M x K) * B[b] (N x K)^T with A, B fp64 on the device
 * (K contiguous), each split into nplanes bf16 planes x ~ p0 + p1 + p2 (p0 = bf16(x), p1 = bf16(x-p0),
 * ...); the product keeps the plane pairs of combined order < nplanes: 1 plane -> 1 tensor-core
 * product (8 bits), 2 -> 3 products (~16 bits), 3 -> 6 products (~24 bits, FP32 class).
 * a_batched / b_batched: 0 = one matrix shared by all batches.  tile_n: 0 auto, 64, 128 or 256 (256 only
 * with nplanes <= 2).  K must be a multiple of 8. */
int sfq_gemm_split_bf16(const double* A, const double* B, float* C, int M, int N, int K, int batch, int a_batched,
                        int b_batched, int nplanes, int tile_n, void* stream);

/* the same product on operands already held as bf16 planes (rows x K, K contiguous, 16-byte aligned,
 * K a multiple of 8); batch strides in elements (0 = shared); C = alpha * A B^T + beta * C (fp32). */
int sfq_gemm_bf16_planes(const void* const* A, const void* const* B, int nplanes, float* C, int M, int N, int K,
                         int batch, long a_batch_stride, long b_batch_stride, float alpha, float beta, int tile_n,
                         void* stream);
/* the planes of n doubles: p0 = bf16(x), p1 = bf16(x - p0), p2 = bf16(x - p0 - p1); p1, p2 may be NULL */
int sfq_split_bf16(const double* src, long n, void* p0, void* p1, void* p2, void* stream);

/* Exact-accumulation tensor-core products from int8 fixed-point slices (tcgen05 kind::i8), no
 * reference counterpart (the reference's products are FP64 BLAS calls): every row r of A (M x K)
 * and of B (N x K), device doubles, is held as 2^e_r (q1 + 2^-8 q2 + 2^-16 q3) with int8 slices
 * q, rounded to nearest from the row's largest entry (|q1| <= 127); the slice pairs of combined
 * order < nslices are multiplied and summed exactly in int32, combined exactly in FP64 and rounded
 * once: C = A B^T (FP32, M x N).  ksplit > 1 writes the partial products of ksplit K ranges at
 * C + s * M * N.  tile_n: 64, 128 or 160 (0: automatic). */
int sfq_gemm_int8_slices(const double* A, const double* B, float* C, int M, int N, int K, int nslices, int tile_n,
                         int ksplit, void* stream);
/* the Taylor term's product in the same arithmetic: C[c][w][a][j] = part c of sum_i A[w][a][i] V[w][j][i]
 * (A (W, N, M), V (W, M, M) complex doubles, taken through FP32 as the engine holds them; C planar
 * FP32 (2, W, N, M)); half: 32, 64 or 80 orbitals per tile. */
int sfq_gemm_int8_cplx_b(const void* A, const void* V, float* C, int W, int M, int N, int nslices, int half,
                         void* stream);
/* Failure-path self test of the tensor-core kernels' bounded waits, no reference counterpart: one
 * small int8-slice product whose loads are held back by a device flag nothing sets, every
 * mbarrier wait limited to wait_ns (1 ns .. 1 s).  Each wait expires; the kernel records
 * SFQ_ERR_TIMEOUT, has no copy or MMA in flight, frees its tensor memory and returns.  Returns the
 * status the kernel recorded (SFQ_ERR_TIMEOUT), or an error of its own. */
int sfq_selftest_wait_expiry(unsigned long long wait_ns, void* stream);

/* ---------------------------------------------------------------------------------------
 * Resident engine: HamiltonianOperations + NOMSD trial + WalkerSet + AFQMCBasePropagator
 * kept in device memory on one GPU (the drop-in for execute_simulation's objects).
 * --------------------------------------------------------------------------------------- */
typedef struct sfq_engine_s* sfq_engine_t;

typedef struct {
  int nmo, nel, nchol, nwalk;
  double dt;
  double E0;                     /* energy_offset() */
  int taylor_order;              /* PropagatorParameters::taylor_n (6) */
  double vbias_bound;            /* 50 */
  double lower_cutoff_scale;     /* 1 */
  double upper_cutoff_scale;     /* 10 */
  double weight_bound_floor;     /* 100 */
  double weight_bound_fraction;  /* 0.1 */
  int subtractMF;                /* 1 */
  int denseP1;                   /* 0: entries |P1| < 1e-8 dropped, as the CSR P1 does */
  int free_projection;           /* 0 */
  int target_population;         /* global target population (0 -> nwalk) */
  unsigned long long seed;       /* Philox key for fields and comb */
  int device;                    /* CUDA device ordinal */
  int precision;                 /* SFQ_PRECISION_FP64 (drop-in) or SFQ_PRECISION_MIXED */
  int walker_type;               /* SFQ_WALKER_CLOSED (0 reads as CLOSED), _COLLINEAR or _NONCOLLINEAR */
  int nel_dn;                    /* COLLINEAR: down electrons, may be 0 (nel = up electrons) */
} sfq_engine_params_t;

/* WALKER_TYPES (src/AFQMC/config.h:47-53).  COLLINEAR walkers carry an up and a down Slater matrix
 * against a trial with PsiT_up (nel, nmo) and PsiT_dn (nel_dn, nmo); the Hamiltonian is the same for
 * both spins.  Engine arrays then hold nel + nel_dn electrons per walker: PsiT is passed as the
 * stacked (nel + nel_dn, nmo) matrix [PsiT_up; PsiT_dn], a walker's SM is (nmo, nel + nel_dn) with
 * the up columns first, and sfq_engine_export_walker_buffer writes the reference's rows (the up
 * block nmo x nel, then the down block nmo x nel_dn).  NONCOLLINEAR walkers are (2 nmo, nel) spinor
 * matrices (the two components' rows one after the other) against PsiT (nel, 2 nmo), nel every
 * electron and nel_dn unused; the Hamiltonian acts on each component.  COLLINEAR and NONCOLLINEAR
 * run in SFQ_PRECISION_FP64. */
#define SFQ_WALKER_CLOSED 1
#define SFQ_WALKER_COLLINEAR 2
#define SFQ_WALKER_NONCOLLINEAR 3

/* SFQ_PRECISION_MIXED / _MIXED_FP32: vbias, vHS, the P1 products and the Taylor terms run on the tcgen05 tensor
 * cores as split-BF16 products (see sfq_gemm_split_bf16) with FP32 accumulation; the mixed density
 * matrix, LU / log det / phase, fields, overlaps, orthogonalization, walker update, population
 * control and energies stay FP64.  Needs a real trial and nmo, nchol multiples of 8. */
#define SFQ_PRECISION_FP64 0
#define SFQ_PRECISION_MIXED 1      /* 2 bf16 planes per operand: ~16-bit operands, 3 tensor-core products */
#define SFQ_PRECISION_MIXED_FP32 2 /* 3 bf16 planes per operand: ~24-bit operands, 6 tensor-core products */
/* SFQ_PRECISION_INT8X3 / _INT8X2: the same products from int8 fixed-point slices of every operand row
 * (x = 2^e (q1 + 2^-8 q2 + 2^-16 q3)), multiplied on the tensor cores (tcgen05 kind::i8) with exact
 * int32 accumulation and one round-to-nearest when the slice groups are combined.  The split-BF16
 * products above lose their low bits toward zero in the tensor cores' FP32 accumulation, which
 * biases every product by the same relative shrink; these carry no such bias.  The force bias, the
 * fields, vHS, the P1 products and Taylor terms, and the exchange tensor of the energy run this way;
 * the Green's function, LU / log det, overlaps, orthogonalization, walker update and all sums stay
 * FP64.  Needs nmo <= 1024; any nchol; CLOSED, COLLINEAR or NONCOLLINEAR walkers (a spinor walker's
 * two (nmo, nel) components share its vHS and P1); single- or multi-determinant trials (with ndet > 1
 * the force bias contracts the ci-weighted full G, minus the trial's, with L over (i, k), and each
 * determinant's exchange uses its own slices of its Lnak); real or complex trials (a complex trial's
 * Lnak adds the products with its imaginary rows to the force bias and the exchange tensor). */
#define SFQ_PRECISION_INT8X3 3     /* 3 slices: 2^-24 of each row's largest entry, 6 int8 products */
#define SFQ_PRECISION_INT8X2 4     /* 2 slices: 2^-16 of each row's largest entry, 3 int8 products */

/* fill *p with the reference's defaults (parameters.hpp:103-131, parameter_defaults.cpp:274-285) */
void sfq_engine_params_default(sfq_engine_params_t* p);

/* RealDenseHamiltonian::getHamiltonianOperations (RealDenseHamiltonian.cpp:53-185) + NOMSD ctor +
 * AFQMCBasePropagator ctor / generateP1 (AFQMCBasePropagator.cpp:43-214), from HOST arrays:
 * hcore (nmo, nmo) real; Likn (nmo, nmo, nchol) real; PsiT (nel, nmo) complex.
 * Walkers start as copies of the trial (PsiT^H) with unit weight. */
int sfq_engine_create(sfq_engine_t* out, const sfq_engine_params_t* p, const double* hcore, const double* Likn,
                      const void* PsiT);
/* the same with a multi-determinant NOMSD trial (NOMSD.cpp:159-331,466-512, ndet > 1): PsiT holds ndet
 * matrices of the walker type's shape one after the other, ci (ndet) complex the coefficients.  The
 * force bias comes from the ci-weighted full Green's function, overlaps and energies from the
 * determinants' own, the mean field from the trial's determinant pairs; walkers start as the
 * determinant of largest |ci|.  FP64 only; ndet = 1 is sfq_engine_create. */
int sfq_engine_create_nomsd(sfq_engine_t* out, const sfq_engine_params_t* p, const double* hcore, const double* Likn,
                            int ndet, const void* PsiT, const void* ci);
int sfq_engine_destroy(sfq_engine_t e);
/* waits for the engine stream; SFQ_ERR_TIMEOUT if a tensor-core product's bounded wait expired */
int sfq_engine_synchronize(sfq_engine_t e);
/* the stream the engine enqueues on (cudaStream_t) */
void* sfq_engine_stream(sfq_engine_t e);

/* walker set I/O (WalkerSetBase.h:320-481): SM (nwalk, nmo, nel) complex; props (8, nwalk) complex in the
 * order WEIGHT, PHASE, PSEUDO_ELOC_, E1_, EXX_, EJ_, OVLP, THETA.  Host pointers; NULL skips.
 * set_walkers also drops the inverse overlap matrices the engine keeps for the next step: call it
 * with both NULL after writing the walkers through sfq_engine_info's device pointer. */
int sfq_engine_set_walkers(sfq_engine_t e, const void* SM, const void* props);
int sfq_engine_get_walkers(sfq_engine_t e, void* SM, void* props);
/* the reference's walker_buffer rows (nwalk, nmo*nel + 11): SM, WEIGHT, PHASE, PSEUDO_ELOC_, E1_, EXX_,
 * EJ_, OVLP, LOGSCL_UP, LOGSCL_DN, IS_UNITARY, THETA (WalkerSetBase.cpp:44-124). Host pointer. */
int sfq_engine_export_walker_buffer(sfq_engine_t e, void* rows);

/* NOMSD::Energy(wset) (NOMSD.cpp:64-75,159-217): E1_/EXX_/EJ_/OVLP of every walker; with
 * seed_pseudo != 0 also seedPseudoEnergy (execute.cpp:46-53).  E3 (nwalk, 3) host out, may be NULL. */
int sfq_engine_energy(sfq_engine_t e, int seed_pseudo, void* E3);

/* AFQMCBasePropagator::Propagate(wset, Eshift) (AFQMCBasePropagator.cpp:290-392), hybrid, one step;
 * fields from Philox(seed, step) or, when uniforms_dev != NULL, from that (nwalk, nchol) device buffer. */
int sfq_engine_propagate(sfq_engine_t e, double Eshift, unsigned long long step, const double* uniforms_dev);
/* same step with HOST inputs and outputs: the field uniforms are copied in from uniforms_host (may be
 * NULL -> Philox) and the (8, nwalk) properties are copied back into props_host (may be NULL). */
int sfq_engine_propagate_host(sfq_engine_t e, double Eshift, unsigned long long step, const double* uniforms_host,
                              void* props_host);
/* AFQMCBasePropagator::Orthogonalize (AFQMCBasePropagator.cpp:736-741) */
int sfq_engine_orthogonalize(sfq_engine_t e);
/* population_control (population_control.hpp:219-255), single rank; the comb draws Philox(seed, call) */
int sfq_engine_population_control(sfq_engine_t e, unsigned long long call);
/* MixedEstimator::measure with the OneRDM and DiagonalTwoRDM observables (MixedEstimator.hpp:37-147,
 * Observables/onerdm.hpp, diagonal_twordm.hpp), FP64 engines: one_rdm (nspin, R, R) complex with
 * nspin 2 for COLLINEAR walkers, else 1, and R = 2 nmo for NONCOLLINEAR, else nmo; diag_two_rdm the
 * folded diagonal two-body RDM, nmo (2 nmo - 1) complex values (CLOSED: nmo (2 nmo - 1) - nmo (nmo - 1) / 2).
 * Both divided by the total weight, as recorded per measurement; host pointers, either may be NULL. */
int sfq_engine_measure_rdm(sfq_engine_t e, void* one_rdm, void* diag_two_rdm);

/* The other observables of MixedEstimator (sfq_engine_measure_observables) and BackPropEstimator
 * (sfq_engine_measure_bp_observables, the arguments of sfq_engine_measure_bp_rdm), FP64 engines, single- or
 * multi-determinant trials (summed over the references, each determinant's G with its coefficient, as
 * the reference's referenceLoop does), divided by the total weight as the RDMs are; host pointers,
 * NULL skips:
 *  - two_rdm: TwoRDM (Observables/twordm.hpp:29-77), (nspin + 1, nmo, nmo, nmo, nmo) complex as
 *    [block][i][k][j][l] = sum_w c_w (G_ik G_jl - G_il G_jk) within a spin, G_ik G_jl across, blocks
 *    (a,a,a,a), (a,a,b,b), (b,b,b,b) (CLOSED: the first two); CLOSED and COLLINEAR walkers, nmo^4 * 16
 *    bytes per block at most 1 GiB;
 *  - spin_corr: SpinCorr (Observables/spincorr.hpp:25-136), (2, nmo (nmo + 1) / 2) complex, the XY
 *    then the Z channel of <S_i . S_j> over i <= j, i-major; every walker type;
 *  - pair_corr: PairCorr (Observables/paircorr.hpp:31-152), (npair, npair, nmo, nmo) complex for the
 *    orbital pair maps pair_maps (npair, nmo) int (a negative partner leaves the orbital out);
 *    COLLINEAR (j > i) and NONCOLLINEAR (every j) walkers. */
int sfq_engine_measure_observables(sfq_engine_t e, void* two_rdm, void* spin_corr, int npair, const int* pair_maps,
                                   void* pair_corr);
int sfq_engine_measure_bp_observables(sfq_engine_t e, int nsteps, int ortho_interval, int path_restoration,
                                      void* two_rdm, void* spin_corr, int npair, const int* pair_maps,
                                      void* pair_corr);

/* TimeEvolvedBPEstimator (TimeEvolvedBPEstimator.hpp:42-300, PropagateOperators
 * AFQMCBasePropagator.cpp:538-654), FP64 engines, single- or multi-determinant trials; needs the back-propagation ring
 * (sfq_engine_enable_back_propagation with nbp >= the longest length).  Per walker and spin the
 * operator states X, Y (identity at the anchor) and M (zero) evolve forward: te_evolve(nsteps) replays
 * the last nsteps stored fields oldest first (X <- P1 e^{i vHS} P1 X, Y <- P1^-1 e^{i vHS^H} P1^-1 Y)
 * and regularizes against the walkers' current Slater matrices S (Y <- S S^H Y, M += Y^H X,
 * X <- X - S S^H X).  The measurements take the dressed Green's functions
 * M + (PsiT X)^T (Gc conj(Y)) (per reference determinant with its PsiT_d and Gc_d, weighted by
 * conj(c_d) exp(ov_d - OVLP) / sum, CLOSED overlaps counted twice) with the walker weights restored over restore_steps history steps
 * (the caller passes bp, or 2 bp with extra path restoration, or 0), and the output layouts of
 * sfq_engine_measure_rdm / sfq_engine_measure_observables.  The schedule (evolve the segment since
 * the previous length, measure, re-anchor after the longest) is the caller's, as the reference's
 * measure() does it. */
int sfq_engine_enable_time_evolved_bp(sfq_engine_t e);
int sfq_engine_te_anchor(sfq_engine_t e);
int sfq_engine_te_evolve(sfq_engine_t e, int nsteps);
int sfq_engine_measure_te_rdm(sfq_engine_t e, int restore_steps, void* one_rdm, void* diag_two_rdm);
int sfq_engine_measure_te_observables(sfq_engine_t e, int restore_steps, void* two_rdm, void* spin_corr, int npair,
                                      const int* pair_maps, void* pair_corr);

/* Back propagation (BackPropEstimator.hpp, AFQMCBasePropagator.cpp:404-526), FP64 engines.
 * enable: every later step keeps, per walker, its fields in a ring of nbp slots and its weight factor
 * (the step's phase over its projection, WalkerSetUpdate.hpp:141-147) in a history of 3 nbp slots,
 * copied with the walkers by population control (resize_bp); the anchored walkers start as the current
 * ones.  anchor: the anchored walkers become the current ones (setAnchor).  measure_bp_rdm: the trial's
 * references propagated backwards over the last nsteps <= nbp steps (adjoint propagator, QR every
 * ortho_interval steps and at the end), the weights restored by the last nsteps weight factors when
 * path_restoration, and the OneRDM / DiagonalTwoRDM between the references and the anchored walkers,
 * shaped as sfq_engine_measure_rdm's.  The caller keeps the estimator's schedule (measure at anchor +
 * nsteps, then re-anchor).  Device-resident blocks and groups refuse an engine with back propagation. */
int sfq_engine_enable_back_propagation(sfq_engine_t e, int nbp);
int sfq_engine_bp_anchor(sfq_engine_t e);
int sfq_engine_measure_bp_rdm(sfq_engine_t e, int nsteps, int ortho_interval, int path_restoration, void* one_rdm,
                              void* diag_two_rdm);
/* the same with the comb's uniform r in [0, 1) from the caller: the draw comb takes from the walker set's
 * generator (population_control.hpp:41-42, HostRandomGenerator::sampleUniformFields), so a caller that
 * owns the reference's stream replays its population control exactly */
int sfq_engine_population_control_uniform(sfq_engine_t e, double r);
/* averagePseudoEnergy / averageEnergy / total weight (average_energy.hpp:33-76); host scalars out */
int sfq_engine_averages(sfq_engine_t e, double* pseudo_energy, double* energy, double* total_weight);
/* EnergyEstimator::measure (EnergyEstimator.h:51-100): out[0..9] = Energy(re,im), Onebody(re,im),
 * Exchange(re,im), Coulomb(re,im), TotalWeight(re,im); walkers are not modified. */
int sfq_engine_measure(sfq_engine_t e, double* out10);

typedef struct {
  int steps;
  int walker_ortho_interval;        /* 10 */
  int population_control_interval;  /* 10 */
  int equilibration_steps;          /* 100 */
  int measure_interval;             /* 10 */
  double Eshift_relaxation_factor;  /* <= 0 -> 1 - exp(-10/equilibration_steps) */
  unsigned long long step0;
  int steer_eshift;  /* 1: Eshift keeps relaxing every step after equilibration too (measurements are taken
                        at their cadence, then Eshift relaxes); 0: run_afqmc's fixed Eshift */
} sfq_run_params_t;
/* run_afqmc's step loop (run_afqmc.cpp:69-113). *Eshift in/out.  Measurements (10 doubles each, see
 * sfq_engine_measure) are written to meas (capacity max_meas); *nmeas receives the count. */
int sfq_engine_run(sfq_engine_t e, const sfq_run_params_t* rp, double* Eshift, double* meas, int max_meas,
                   int* nmeas);

/* The same loop as one device-resident block: Eshift, the step counter and the measurements live in
 * device memory, every step's work (propagation, orthogonalization, population control, Eshift
 * relaxation, measurements at their cadence) is enqueued with no host round trip, and the block is
 * replayed from a CUDA graph captured the first time its schedule is seen.  At most 64
 * measurements per block.  sfq_engine_block runs it and waits; the _async form enqueues it on the
 * engine's stream, _query returns 1 once it has finished (0 while it runs, minus an SFQ_ERR_* code
 * on a CUDA error), _result waits for it
 * and returns its final Eshift and measurements (and its errors: SFQ_ERR_WEIGHT_COLLAPSE,
 * SFQ_ERR_TIMEOUT).  No counterpart in the reference, whose loop returns to the host every step. */
int sfq_engine_block(sfq_engine_t e, const sfq_run_params_t* rp, double* Eshift, double* meas, int max_meas,
                     int* nmeas);
int sfq_engine_block_async(sfq_engine_t e, const sfq_run_params_t* rp, double Eshift);
int sfq_engine_block_query(sfq_engine_t e);
int sfq_engine_block_result(sfq_engine_t e, double* Eshift, double* meas, int max_meas, int* nmeas);
/* bytes of device memory the engine holds (its arena and packed tensors) */
int sfq_engine_footprint(sfq_engine_t e, size_t* bytes);

/* ---- tile autotuner (the tensor-core precisions) -----------------------------------------------
 * The tensor-core products are tiled in output tiles of 128 rows by a width the kernel is built
 * for (64, 128, 160 with any plane count; 208, 256 with at most 2 planes).  sfq_engine_autotune
 * times every built width of each product on the engine's own operands (the current walkers; only
 * scratch buffers are written) and keeps the fastest: the G product, the force-bias product (its
 * width, and its K split: the one that fills whole waves of SMs or the smallest within 6 % of it,
 * fewer partial sums to add; longer K ranges accumulate more FP32 rounding in the force bias, about
 * as sqrt(K per range), so a caller that wants the tighter force bias sets the larger split), the
 * vHS product, the Taylor terms (taylor_half orbitals per
 * tile: 16, 32, 64, 80, or 128 with at most 2 planes) and the two P1 products.  The widths change
 * how the output is tiled and, for the force bias, how many partial sums are reduced, so two
 * engines given the same tiles (sfq_engine_set_tiles; 0 = the built-in choice) produce identical
 * results.  Setting tiles drops the engine's captured block graphs.  us_builtin / us_tuned: median
 * time of each product (G, force bias, vHS, one Taylor term, both P1 products) with the built-in
 * and the chosen tiles (0 when a product was not timed).  The int8-slice precisions tile only the
 * Taylor terms by choice (taylor_half 32, 64 or 80; the other widths are fixed and reported, g_bn = 0
 * as G is FP64): their exact integer accumulation gives the same results bit for bit at every
 * width, and the tuner times the three on the engine's operands.  No counterpart in the reference. */
typedef struct {
  int g_bn, vbias_bn, vhs_bn, taylor_half, p1_bn;
  int vbias_ksplit; /* force-bias K split; set_tiles: 0 = planned from vbias_bn */
  double us_builtin[5];
  double us_tuned[5];
} sfq_tiles_t;
int sfq_engine_autotune(sfq_engine_t e, int repeats, sfq_tiles_t* out);
int sfq_engine_set_tiles(sfq_engine_t e, const sfq_tiles_t* tiles);
int sfq_engine_tiles(sfq_engine_t e, sfq_tiles_t* tiles);

/* ---- several systems advanced together --------------------------------------------------------
 * A group of engines (systems of any M, N, Nchol, walker counts and precisions on one device)
 * advances by one block of every member per call: the members' blocks (sfq_engine_block
 * semantics, each with its own run parameters rps[i] and Eshift[i]) are captured, the first time a
 * combination of schedules is seen, as the branches of ONE CUDA graph, so that one graph launch
 * advances all systems and their kernels share the SMs.  sfq_group_set_lanes sets the schedule:
 * `lanes` chains of members run side by side, the members of a chain one after another (members
 * assigned longest first to the least loaded chain by their flops per block); 0 (the default)
 * gives every member its own chain, 1 runs them all in turn.  Results per member: Eshift[i] (in/out),
 * status[i] (0, SFQ_ERR_WEIGHT_COLLAPSE, SFQ_ERR_TIMEOUT), nmeas[i] measurements of 10 doubles at
 * meas + 10 * max_meas * i.  The call returns the first member error.  The engines stay usable on
 * their own between group blocks; one block of a group runs at a time (_async, then _result).
 * sfq_group_set_fused(g, 1) (members in one int8-slice precision, SFQ_PRECISION_INT8X3 or _INT8X2,
 * on one block schedule) instead interleaves the members' steps stage by stage: each stage's
 * tensor-core products of ALL members (force bias, vHS, the P1 products and Taylor terms, the
 * exchange tensor's chunks) run as ONE persistent grouped launch over their concatenated tile
 * lists, the work between them on the members' streams side by side.  Each tile is computed as the
 * member's own launch computes it: the results equal the members' blocks run alone, bit for bit.
 * No counterpart in the reference, which runs one system per process. */
typedef struct sfq_group_s* sfq_group_t;
int sfq_group_create(sfq_group_t* g, const sfq_engine_t* engines, int n);
int sfq_group_destroy(sfq_group_t g);
int sfq_group_block(sfq_group_t g, const sfq_run_params_t* rps, double* Eshift, int* status, double* meas,
                    int max_meas, int* nmeas);
int sfq_group_block_async(sfq_group_t g, const sfq_run_params_t* rps, const double* Eshift);
int sfq_group_block_query(sfq_group_t g);
int sfq_group_set_lanes(sfq_group_t g, int lanes);
int sfq_group_set_fused(sfq_group_t g, int fused);
int sfq_group_block_result(sfq_group_t g, double* Eshift, int* status, double* meas, int max_meas, int* nmeas);

/* ---- serving loop: continuous batching of propagation blocks over resident systems -----------
 * Systems are registered with their inputs (kept on the host); their engines are built on the
 * device when a request needs them and stay resident between blocks, under an HBM budget (the
 * least recently used idle systems are evicted, their walkers saved on the host and restored
 * when they are built again).  A request is one block (sfq_engine_block semantics; the server
 * continues each system's step count and Eshift).  sfq_server_progress retires finished blocks and
 * admits queued requests in arrival order as slots (max_inflight blocks on the GPU at once, one
 * per system) and memory free up; blocks of different systems run concurrently on their own
 * streams.  Times are seconds on sfq_server_clock.  No counterpart in the reference. */
typedef struct sfq_server_s* sfq_server_t;
typedef struct {
  size_t hbm_budget; /* bytes the resident engines may hold */
  int max_inflight;  /* blocks running at once */
  int device;
} sfq_server_params_t;
typedef struct {
  int status;        /* 1 queued, 2 running, 0 done, or an SFQ_ERR_* code */
  int system;
  double t_submit, t_start, t_finish;
  double Eshift;     /* after the block */
  int nmeas;
  unsigned long long step0; /* the system's step index the block started at */
  char message[128];  /* the error of a failed request */
} sfq_request_info_t;
int sfq_server_create(sfq_server_t* out, const sfq_server_params_t* p);
int sfq_server_destroy(sfq_server_t s);
int sfq_server_add_system(sfq_server_t s, const sfq_engine_params_t* p, const double* hcore, const double* Likn,
                          const void* PsiT, int* id);
/* build a system's engine now (e.g. before timing), evicting idle systems if the budget needs it */
int sfq_server_warm(sfq_server_t s, int system);
int sfq_server_submit(sfq_server_t s, int system, const sfq_run_params_t* rp, long long* request);
/* retire finished blocks and admit queued ones; *completed (may be NULL) = requests finished by this call */
int sfq_server_progress(sfq_server_t s, int* completed);
/* state and results of a request (meas: up to max_meas measurements of 10 doubles) */
int sfq_server_request(sfq_server_t s, long long request, sfq_request_info_t* info, double* meas, int max_meas);
/* resident bytes, resident systems, running and queued requests (any may be NULL) */
int sfq_server_stats(sfq_server_t s, size_t* used_bytes, int* resident, int* running, int* queued);
double sfq_server_clock(sfq_server_t s);

/* per-phase CUDA-event timing on the engine stream (AFQMCTimers analogue, AFQMCTimer.h:25-63) */
enum sfq_phase {
  SFQ_PH_DENSITY = 0,     /* overlap matrix + LU + mixed density matrix */
  SFQ_PH_VBIAS = 1,       /* force bias GEMM */
  SFQ_PH_FIELDS = 2,      /* assemble_X + meanfield factor */
  SFQ_PH_VHS = 3,         /* vHS GEMM */
  SFQ_PH_PROPAGATE = 4,   /* P1, Taylor exp, P1 */
  SFQ_PH_OVERLAP = 5,     /* post-propagation log overlap */
  SFQ_PH_UPDATE = 6,      /* walker_update + weight bound */
  SFQ_PH_ORTHO = 7,       /* orthogonalize + overlap refresh */
  SFQ_PH_POPCONTROL = 8,  /* comb + walker copies */
  SFQ_PH_ENERGY = 9,      /* local energy */
  SFQ_PH_VHS_GEMM = 10,   /* the vHS matrix product alone (inside SFQ_PH_VHS) */
  SFQ_PH_TAYLOR_GEMM = 11, /* the Taylor terms' matrix products alone (inside SFQ_PH_PROPAGATE), one per term */
  SFQ_NUM_PHASES = 12
};
int sfq_engine_profile(sfq_engine_t e, int enable);
/* synchronizes; ms[ph] = summed device time since the last call, counts[ph] = intervals (either may be NULL) */
int sfq_engine_phase_times(sfq_engine_t e, double* ms, int* counts, int nphase);

/* device addresses of the engine's resident arrays, for tests and zero-copy callers (writes to SM
 * through this pointer are announced with sfq_engine_set_walkers(e, NULL, NULL)) */
typedef struct {
  void* SM;           /* (nwalk, nmo, nel) complex */
  void* props;        /* (8, nwalk) complex */
  void* PsiT;         /* (nel, nmo) complex */
  void* Lnak;         /* (nchol, nel, nmo), real if lnak_complex == 0 */
  int lnak_complex;
  void* Likn;         /* (nmo, nmo, nchol) real */
  void* haj;          /* (nel, nmo) complex */
  void* v0;           /* (nmo, nmo) real */
  void* vmf;          /* (nchol) real */
  void* P1;           /* (nmo, nmo) real */
  void* G;            /* (nwalk, nel, nmo) complex, last mixed density matrix */
  void* X;            /* (nwalk, nchol) complex, last fields */
  void* vHS;          /* (nwalk, nmo, nmo) complex, last vHS */
  void* hw;           /* (nwalk) complex */
  void* mf;           /* (nwalk) complex */
  void* new_ovlp;     /* (nwalk) complex */
  unsigned long long bound_stats[5]; /* eloc total/upper/lower, weight total/upper */
  int vhs_packed;     /* 1: the Cholesky vectors are symmetric and vHS comes from their upper triangle */
  void* hcore;        /* (nmo, nmo) real */
} sfq_engine_info_t;
int sfq_engine_info(sfq_engine_t e, sfq_engine_info_t* info);

/* WalkerSet::copy_walker (WalkerSetBase.h:413-415): every field of the walker in slot `from` (its
 * Slater matrix and property columns) into slot `to`. */
int sfq_engine_copy_walker(sfq_engine_t e, int from, int to);
/* The sharded walker exchange on device buffers (swap_walkers_async, population_control.hpp:143-209;
 * the plan from sfq_walker_moves).  A row is one walker: its Slater matrix followed by its 8 property
 * values (the column order of sfq_engine_set_walkers), sfq_engine_walker_row_elems complex values in
 * all (negative: an error code).  pack writes walker slots[r] into row r of `rows` (device memory,
 * n rows), unpack writes row r into walker slots[r]; copy_walkers first sets every weight to
 * w / |w| when normalize_weights != 0 (population_control.hpp:238-241), then copies walker
 * pairs[2k] into walker pairs[2k+1], k < n (destinations distinct and none a source).  slots and
 * pairs are host arrays.  Each call runs on the engine stream and returns after it has finished, so
 * the rows are ready for a send on another stream.  Engines with back propagation on are refused
 * (the rows do not carry its history). */
long sfq_engine_walker_row_elems(sfq_engine_t e);
int sfq_engine_pack_walkers(sfq_engine_t e, const int* slots, int n, void* rows);
int sfq_engine_unpack_walkers(sfq_engine_t e, const int* slots, int n, const void* rows);
int sfq_engine_copy_walkers(sfq_engine_t e, const int* pairs, int n, int normalize_weights);
/* WalkerSet::resize (WalkerSetBase.h:195): the engine is rebuilt for nwalk walkers (the resident
 * tensors recomputed from its Hamiltonian and trial, tiles back to their defaults, back propagation
 * off), and its walkers are carried over, new slots filled from the existing walkers in
 * round-robin order, slot w from slot w mod the old count.  *e is replaced by the new engine. */
int sfq_engine_resize(sfq_engine_t* e, int nwalk);

/* HamiltonianOperations::getOneBodyPropagatorMatrix (Real3IndexFactorization.hpp:99-124,
 * add_one_body_shifts one_body.hpp:64-82): H1 = dt (hcore + v0) + sqrt(dt) sum_n L_n vMF_n, the
 * matrix generateP1 exponentiates.  hcore, v0 (nmo x nmo) and Likn (nmo, nmo, nchol) on the device;
 * vMF (nchol, the real mean field) and H1 (nmo x nmo, real) in host memory. */
int sfq_one_body_matrix(const double* hcore, const double* v0, const double* Likn, const double* vMF, int nmo,
                        int nchol, double dt, double* H1, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SAFIRE_B200_H */
