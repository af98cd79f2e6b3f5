// Mixed-precision propagation helpers (layout conversions between the FP64 walker state and
// the split-BF16 operands of the tensor-core GEMMs).  See mixed_kernels.cu for the layouts.
#pragma once
#include "common.cuh"

namespace sfq {

// `pl` points at 3 plane pointers (p0, p1, p2); unused planes are null
int mixed_split_planar(const cplx* src, int W, long E, void* const* pl, cudaStream_t st);
int mixed_planar_to_cplx(const float* C, int W, long E, double alpha, cplx* out, cudaStream_t st);
// Cv: (2W, M*M) planar, or (2W, M(M+1)/2) with packed (upper triangle of a symmetric vHS)
int mixed_build_vblk(const float* Cv, int W, int M, bool packed, void* const* pl, cudaStream_t st);
int mixed_walkers_to_wt(const cplx* SM, int W, int M, int N, void* const* pl, cudaStream_t st);
int mixed_wt_to_walkers(const float* C2, int W, int M, int N, cplx* SM, cudaStream_t st);
// pl == null: only accumulate into S (last Taylor term)
int mixed_taylor_update(const float* C, long rows, int M, float inv_k, float* S, void* const* pl, cudaStream_t st);
int mixed_split_f32(const float* src, long n, void* const* pl, cudaStream_t st);

}  // namespace sfq
