// Mixed-precision propagation helpers (layout conversions between the FP64 walker state and
// the split-BF16 operands of the tensor-core GEMMs).  See mixed_kernels.cu for the layouts.
#pragma once
#include "common.cuh"

namespace sfq {

// `pl` points at 3 plane pointers (p0, p1, p2); unused planes are null
int mixed_split_planar(const cplx* src, int W, long E, void* const* pl, cudaStream_t st);
// out[w][e] = add[e] + alpha * (sum_s C_s[w][e], sum_s C_s[W + w][e]), the KS partial sums
// C_s = C + s * sk (add may be null)
int mixed_reduce_planar_to_cplx(const float* C, int KS, long sk, int W, long E, double alpha, cplx* out,
                                cudaStream_t st, const cplx* add = nullptr);
// Cv: (2W, M*M) planar, or (2W, M(M+1)/2) with packed (upper triangle of a symmetric vHS) ->
// split planes V[w][c][i][k] (Vr, Vi)
int mixed_build_v(const float* Cv, int W, int M, bool packed, void* const* pl, cudaStream_t st);
// Tinv (W, N, N) -> split planes of the block operand [[Tr, -Ti], [Ti, Tr]] (rows (c, a), columns (b, c'))
int mixed_build_tblk(const cplx* Tinv, int W, int N, void* const* pl, cudaStream_t st);
// SM (W, M, N) -> walker-operand planes WT[w][a][c * ldh + i]
int mixed_walkers_to_wt(const cplx* SM, int W, int M, int N, int ldh, void* const* pl, cudaStream_t st);
// one pass over SM: the planes of SM read as reals (ps, same layout) and the walker rows of
// mixed_walkers_to_wt (pt)
int mixed_walkers_split_both(const cplx* SM, int W, int M, int N, int ldh, void* const* ps, void* const* pt,
                             cudaStream_t st);

}  // namespace sfq
