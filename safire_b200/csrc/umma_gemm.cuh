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
  const void* p[3] = {nullptr, nullptr, nullptr};  // bf16 planes (rows, K) per batch, K contiguous
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
  int nplanes = 2;        // 1, 2 or 3 (see above)
  int bn = 0;             // tile width: 0 = automatic, else 64, 128 or 256 (256: nplanes <= 2)
  int* err = nullptr;     // device flag, SFQ_ERR_TIMEOUT on an expired wait (may be null)
};

int umma_gemm(const UmmaGemmDesc& d, cudaStream_t st);

int gemm_split_bf16_f64(const double* A, const double* B, float* C, int M, int N, int K, int batch, int a_batched,
                        int b_batched, int nplanes, int bn, cudaStream_t st);

// bf16 planes of an fp64 array: p0 = bf16(x), p1 = bf16(x - p0), p2 = bf16(x - p0 - p1); null planes skipped
int split_bf16_f64(const double* src, long n, void* p0, void* p1, void* p2, cudaStream_t st);

}  // namespace sfq
