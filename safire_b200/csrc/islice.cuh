// Exact-accumulation tensor-core products from int8 fixed-point slices (tcgen05 kind::i8, sm_100a).
//
// The tensor cores' FP32 accumulation rounds toward zero: a split-BF16 product over K terms comes
// out shrunk by about (K / 16) * (products per step) * 2^-25 relative, the same sign for every
// element, and that bias moves the propagated walkers and the measured energies systematically.
// Integer products accumulate exactly.  Each operand row r is held in fixed point,
//
//   x[r][k] = 2^e[r] * (q1 + 2^-8 q2 + 2^-16 q3),   q1, q2, q3 int8 ("slices"),
//
// with e[r] chosen from the row's largest |x| so that |q1| <= 127; the slices are round-to-nearest
// digits, so the representation error is unbiased (2^-24 of the row maximum for 3 slices, 2^-16
// for 2).  A product keeps the slice pairs of combined order < slices, grouped by order g:
//
//   g = 0: q1 t1         g = 1: q1 t2 + q2 t1         g = 2: q1 t3 + q2 t2 + q3 t1
//
// each group summed exactly in int32 in tensor memory (|sum| < 3 * 2^14 * K < 2^31 for K <= 43000),
// and the epilogue forms 2^(eA + eB) * (acc0 + 2^-8 acc1 + 2^-16 acc2) exactly in FP64, times
// alpha, rounded once to FP32 (round to nearest).  3 slices: 6 int8 products (the work of 3 BF16
// products at twice the rate); 2 slices: 3.
//
// Persistent kernel: one CTA per SM walks a static list of 128 x BN output tiles; warp 0 issues
// TMA loads of K slices into a ring of stages (64 int8 elements per slice, 64-byte swizzle, where a
// tile's K range is short; 128 elements, 128-byte swizzle, half the stages, where it reaches 1024),
// one thread of warp 1 issues tcgen05.mma.kind::i8 (M = 128, N = BN, K = 32) and commits each
// stage, eight epilogue warps drain the group accumulators.  K tails are zero-filled by TMA and
// their MMA steps skipped; K splits fall on multiples of 128 elements at either slice width.
// Every mbarrier wait is bounded from its own start; on expiry the kernel records SFQ_ERR_TIMEOUT,
// waits for its own copies and MMAs, frees its tensor memory and returns.
//
// Complex B (cplx_half > 0), the Taylor product C = A [[Vr, -Vi], [Vi, Vr]]^T of one walker:
// B holds the rows Vr (i < nmo), Vi (nmo + i) and -Vi (2 nmo + i) sharing one exponent per
// orbital i; A has two arrays of the same shape, the real parts (a.q) and the imaginary parts
// (a_im), one exponent per row.  Output tile t holds [re | im] over orbitals t * half ... + half,
// two full-width MMAs per K step:  [re | im] += A_re [Vr; Vi]^T  and  [re | im] += A_im [-Vi; Vr]^T
// (int8 products have no negate bit, hence the negated rows of V), written planar:
// C[c * sCc + (batch * M + row) * ldc + i].
#pragma once
#include <cstdint>
#include <vector>

#include "common.cuh"

namespace sfq {

struct IsliceOperand {
  const int8_t* q[3] = {nullptr, nullptr, nullptr};  // slices (rows, K) per batch, K contiguous
  long rows = 0;           // rows per batch
  long ld = 0;             // bytes between rows (a multiple of 16, >= K)
  long batch_stride = 0;   // bytes between batches (0: shared by all batches)
  const int* e = nullptr;  // row exponents: e[batch * e_bs + (e_mod ? row % e_mod : row)]
  long e_bs = 0;
  long e_mod = 0;
};

struct IsliceGemmDesc {
  int M = 0, N = 0, K = 0, batch = 1;  // complex B: N = nmo orbitals, K = nmo
  int nslices = 3;                     // 2 or 3
  int bn = 0;                          // tile width (0: automatic); complex B: 2 * cplx_half
  int ksplit = 1;                      // K ranges, each writing its partial C at C + s * sCk
  long sCk = 0;
  IsliceOperand A, B;
  int cplx_half = 0;                   // complex B (see above): orbitals per tile
  const int8_t* a_im[3] = {nullptr, nullptr, nullptr};
  float* C = nullptr;                  // FP32 output, row-major: C[s*sCk + batch*sCb + row*ldc + col]
  long ldc = 0, sCb = 0, sCc = 0;      // sCc: complex B, elements between the re and im outputs
  double alpha = 1.0;
  bool accumulate = false;             // C += alpha A B^T (one FP32 round to nearest) instead of C =
  int* err = nullptr;                  // device flag: SFQ_ERR_TIMEOUT on an expired wait (may be null)
  unsigned long long wait_ns = 0;      // limit of one mbarrier wait without progress (0: 2 s)
  const int* hold = nullptr;           // if set, the loads start only once *hold != 0 (waits bounded)
};

int islice_gemm(const IsliceGemmDesc& d, cudaStream_t st);

// Several products (the same slice count; plain ones of tile width 160, complex-B ones of any
// half <= 80) as ONE persistent launch over the concatenated tile lists, each tile computed as its
// own product's launch computes it (the results are the same bit for bit).  The plan is a host
// image of the launch's table (per product: tensor maps and parameters; then the tile offsets)
// that the caller copies to device memory (128-byte aligned) before the launch runs, and keeps
// there for as long as the launch may run (a graph holding it may be replayed).
struct IsliceGroupPlan {
  std::vector<char> image;
  size_t start_off = 0;  // byte offset of the nprob + 1 tile offsets in the image
  int nprob = 0, nslices = 0;
  int bk = 64;  // K slice width of the launch
  long tiles = 0;
  unsigned long long wait_ns = 0;
};
int islice_gemm_group_plan(const IsliceGemmDesc* ds, int n, IsliceGroupPlan* out);
int islice_gemm_group_launch(const void* table, const IsliceGroupPlan& plan, cudaStream_t st);

// ---- slicing (islice_kernels.cu) ------------------------------------------------------------
// Every slicer writes nslices int8 arrays (rows, ld) at q[s] and one exponent per row (or per row
// group, where stated); elements k in [K, ld) of a row are written as zeros.

// real rows: x[r][k] = src[r * lds + k]
int islice_rows_real(const double* src, long R, long K, long lds, int nslices, int8_t* const* q, long ld, int* e,
                     cudaStream_t st);
// complex rows split into planar rows: row c * R + r holds part c (0 re, 1 im) of src[r * K + k]
// (minus sub[k] when sub is given), with its own exponent; with emax (2 R scratch values) rows longer
// than 8192 are spread over blocks (a max pass, then a slicing pass), else one block per row
int islice_rows_planar(const cplx* src, long R, long K, int nslices, int8_t* const* q, long ld, int* e,
                       cudaStream_t st, const cplx* sub = nullptr,
                       unsigned long long* emax = nullptr);
// walkers SM (W, M, N) complex -> rows (c, w, a) over orbitals j (the P1 product's A operand), one
// exponent per (w, a) for both parts: e[w * N + a]; planar (may be null): the same rows in FP32,
// row stride M
int islice_walkers(const cplx* SM, int W, int M, int N, int nslices, int8_t* const* q, long ld, int* e,
                   float* planar, cudaStream_t st);
// planar walker-shaped FP32 rows (r < R = W N, j < M, M <= 1024), the product C[c][r][j] into the
// sum S[c][r][j]: k = 0: S += C; k > 0: T = (i / k) C (T_re = -C_im / k, T_im = C_re / k) and
// S += T; then the slices of S (slice_sum; required for k = 0) or of T into q (rows (c, r)), one
// exponent per r
int islice_taylor_update(const float* C, float* S, long R, int M, int k, bool slice_sum, int nslices,
                         int8_t* const* q, long ld, int* e, cudaStream_t st);
// vHS (planar rows c * W + w over the packed upper triangle, or over M * M) -> V slices
// V[w][c][i][k], c = 0, 1, 2 for Vr, Vi, -Vi (the negation sliced as itself), with one exponent per
// (w, i) shared by the three rows; emax: W * M scratch ints (the full M * M form only)
int islice_build_v(const float* Cv, int W, int M, bool packed, int nslices, int8_t* const* q, long ld, int* e,
                   int* emax, cudaStream_t st);
// planar FP32 rows C[c][w][a][j] (+ S[c][w][a][j] when S is given, added in FP64) -> SM[w][j][a]
// (complex FP64)
int islice_to_walkers(const float* C, const float* S, int W, int M, int N, cplx* SM, cudaStream_t st);

}  // namespace sfq
