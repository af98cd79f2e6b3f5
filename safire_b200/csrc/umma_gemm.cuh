// Split-BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   C[b] (M x N, fp32) = alpha * sum_t A_t[b] (M x K) * B_t[b] (N x K)^T  (+ beta * C[b])
//
// Every operand is held as BF16 planes, x ~= p0 + p1 (+ p2) with p0 = bf16(x), p1 = bf16(x - p0),
// p2 = bf16(x - p0 - p1), and the product keeps the terms of combined order <= nplanes - 1:
//   1 plane : p0 q0                                   ( 8 significant bits)
//   2 planes: p0 q0 + p0 q1 + p1 q0                   (~16 bits, 3 tensor-core products)
//   3 planes: + p0 q2 + p1 q1 + p2 q0                 (~24 bits = FP32 class, 6 products)
// all accumulated in FP32 in tensor memory: the "complex FP32 from split-BF16" arithmetic of the
// mixed-precision propagation.
//
// Persistent kernel, one CTA per SM walking a static list of 128 x BN output tiles (M fastest, so
// the CTAs that share a B tile run together; optionally also split along K, each split writing
// its own partial C, for products with few output tiles and a long K).  Operands are K-major
// (K contiguous), loaded by TMA as 64-element (128-byte) K slices with the 128-byte swizzle into
// a ring of stages; one elected
// thread issues tcgen05.mma (M = 128, N = BN, K = 16) on the smem descriptors and commits each
// stage back to the TMA producer; the accumulator is double-buffered in tensor memory, so four
// epilogue warps drain tile i (tcgen05.ld) while the tensor core computes tile i + 1.  Every
// mbarrier wait is bounded, each from its own start (a launch that keeps making progress may run
// for any time): on expiry the kernel records SFQ_ERR_TIMEOUT in *err, waits for its own TMA
// loads and MMAs, frees its tensor memory and returns.
//
// The epilogue is selectable, so that the elementwise work around the products of the mixed
// propagation happens while the tile is still on chip:
//   STORE        C = alpha acc + beta C
//   STORE_SPLIT  C = alpha acc, and the BF16 planes of C (same layout) for a following product
//   TAYLOR       the tile's columns are [re | im] halves over `half` orbitals i (B rows ordered so);
//                T = (i / k) C, i.e. T_re = -C_im / k, T_im = C_re / k; S += T; planes of T (the
//                next term's A operand) or of the updated S (the final P1 product's A operand).
//                S uses [b][row][c * nmo + i], the planes [b][row][c * ldh + i].
//   TO_WALKERS   rows (w, a, c), columns j: SM[w][j][a].c = alpha acc (complex fp64 walkers)
//   PLANAR_SPLIT rows (c, a) of batch b (c < 2, a < nel), columns n: the BF16 planes of
//                alpha acc at row (c * batch + b) * nel + a, column n of an nmo-wide matrix (the
//                planar operand of a following product)
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace sfq {

struct UmmaOperand {
  const void* p[3] = {nullptr, nullptr, nullptr};  // bf16 planes (rows, K) per batch, K contiguous
  long rows = 0;             // rows per batch
  long ld = 0;               // elements between rows (>= K, multiple of 8)
  long batch_stride = 0;     // elements between batches (0: shared)
};

enum UmmaEpiKind {
  UMMA_EPI_STORE = 0,
  UMMA_EPI_STORE_SPLIT = 1,
  UMMA_EPI_TAYLOR = 2,
  UMMA_EPI_TO_WALKERS = 3,
  UMMA_EPI_PLANAR_SPLIT = 4
};

struct UmmaEpilogue {
  int kind = UMMA_EPI_STORE;
  void* out[3] = {nullptr, nullptr, nullptr};  // bf16 planes written by STORE_SPLIT and TAYLOR
  int out_planes = 0;                          // how many of them (1..3)
  // TAYLOR
  float* S = nullptr;     // [batch][M rows][2 * nmo]
  int nmo = 0;            // orbitals per half
  int ldh = 0;            // planes: [batch][M rows][2 * ldh], half c at c * ldh (0: ldh = nmo); STORE_SPLIT: row stride of the planes (0: ldc)
  int half = 0;           // orbitals per tile (BN = 2 * half, a multiple of 16)
  float inv_k = 0.f;      // 1 / k for T_{k+1} = (i / k) C
  int write = 0;          // 1: planes of T_{k+1}; 2: planes of the updated S; 0: none
  // TO_WALKERS
  double* SM = nullptr;   // (nwalk, nmo, nel) complex
  int nel = 0;
};

struct UmmaGemmDesc {
  int M = 0, N = 0, K = 0, batch = 1;
  UmmaOperand A, B;
  float* C = nullptr;
  long ldc = 0, sCb = 0;  // fp32 row-major output
  float alpha = 1.f, beta = 0.f;
  int nplanes = 2;        // 1, 2 or 3 (see above)
  int bn = 0;             // tile width: 0 = automatic, else 32, 64, 128, 160, 208 or 256
  int ksplit = 1;         // K split into this many ranges, each writing its partial C at C + s * sCk
  long sCk = 0;
  // Complex B (cplx_half > 0): B holds only Vr and Vi, rows (c, i) of 2 * cplx_nmo per batch, K = k
  // (cplx_nmo); A's K is (c', k) with each half padded to cplx_ldh (a multiple of 64).  Output
  // tile t has columns [re | im] over orbitals t * half .. + half, computed as
  //   re += A_re Vr^T - A_im Vi^T,   im += A_re Vi^T + A_im Vr^T
  // by two N = half MMAs per K slice (the -Vi through the instruction's negate-B bit): the
  // product with [[Vr, -Vi], [Vi, Vr]] without storing that block.  BN = 2 * half.
  int cplx_half = 0, cplx_nmo = 0, cplx_ldh = 0;
  UmmaEpilogue epi;
  int* err = nullptr;     // device flag, SFQ_ERR_TIMEOUT on an expired wait (may be null)
  unsigned long long wait_ns = 0;  // limit of one mbarrier wait without progress (0: 2 s)
};

int umma_gemm(const UmmaGemmDesc& d, cudaStream_t st);

int gemm_split_bf16_f64(const double* A, const double* B, float* C, int M, int N, int K, int batch, int a_batched,
                        int b_batched, int nplanes, int bn, cudaStream_t st);

// bf16 planes of an fp64 array: p0 = bf16(x), p1 = bf16(x - p0), p2 = bf16(x - p0 - p1); null planes skipped
int split_bf16_f64(const double* src, long n, void* p0, void* p1, void* p2, cudaStream_t st);

}  // namespace sfq
