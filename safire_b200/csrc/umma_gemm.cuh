// Split-BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   C[b] (M x N, fp32) = alpha * sum_t A_t[b] (M x K) * B_t[b] (N x K)^T  (+ beta * C[b])
//
// Every operand is held as two BF16 planes, x ~= hi + lo with hi = bf16(x), lo = bf16(x - hi),
// and the product is taken as hi*hi + hi*lo + lo*hi with FP32 accumulation in tensor memory:
// about 16 significant bits per operand, the "complex FP32 from split-BF16" arithmetic of the
// mixed-precision propagation.  nterms = 1 keeps hi*hi only.
//
// Operands are K-major (K contiguous), loaded by TMA as 64-element (128-byte) K slices with the
// 128-byte swizzle; one elected thread issues tcgen05.mma (M = 128, N = BN, K = 16) on the smem
// descriptors; tcgen05.commit releases each stage to the TMA producer; four epilogue warps read
// the accumulator with tcgen05.ld.  Every mbarrier wait is bounded: on expiry the kernel records
// SFQ_ERR_TIMEOUT in *err, drains its own TMA loads, frees its tensor memory and returns.
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace sfq {

struct UmmaOperand {
  const void* hi = nullptr;  // bf16 (rows, K) per batch, K contiguous
  const void* lo = nullptr;  // same layout; may be null when nterms == 1
  long rows = 0;             // rows per batch
  long ld = 0;               // elements between rows (>= K, multiple of 8)
  long batch_stride = 0;     // elements between batches (0: shared)
};

struct UmmaGemmDesc {
  int M = 0, N = 0, K = 0, batch = 1;
  UmmaOperand A, B;
  float* C = nullptr;
  long ldc = 0, sCb = 0;  // fp32 row-major output
  float alpha = 1.f, beta = 0.f;
  int nterms = 3;
  int bn = 0;             // tile width: 0 = automatic, else 64, 128 or 256
  int* err = nullptr;     // device flag, SFQ_ERR_TIMEOUT on an expired wait (may be null)
};

int umma_gemm(const UmmaGemmDesc& d, cudaStream_t st);

int gemm_split_bf16_f64(const double* A, const double* B, float* C, int M, int N, int K, int batch, int a_batched,
                        int b_batched, int nterms, int bn, cudaStream_t st);

// bf16 hi/lo planes of a strided fp64 / fp32 / complex source (elementwise helpers)
int split_bf16_f64(const double* src, long n, void* hi, void* lo, cudaStream_t st);

}  // namespace sfq
