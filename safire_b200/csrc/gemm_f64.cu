// Host dispatch for the FP64 DMMA GEMM: picks the instantiation from operand kinds/contiguity
// and the tile shape from the problem shape.
#include "gemm_f64.cuh"

namespace sfq {
using namespace gemm_detail;

namespace {

template <bool AC, bool BC, bool CONJA, bool AK, bool BK, int BM, int BN, int WM, int WN, int STAGES>
int launch(const GemmDesc& d, cudaStream_t st) {
  using C_ = Cfg<AC, BC, CONJA, AK, BK, BM, BN, WM, WN, STAGES>;
  auto k = gemm_f64_kernel<AC, BC, CONJA, AK, BK, BM, BN, WM, WN, STAGES>;
  static bool attr_set = false;  // one opt-in per instantiation (per process, device-agnostic)
  if (!attr_set) {
    SFQ_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, C_::SMEM));
    attr_set = true;
  }
  dim3 grid((d.N + BN - 1) / BN, (d.M + BM - 1) / BM, d.batch);
  if (grid.y > 65535u || grid.z > 65535u)
    return record_error(SFQ_ERR_SHAPE, "gemm_f64: grid (%u,%u,%u) too large", grid.x, grid.y, grid.z);
  k<<<grid, C_::THREADS, C_::SMEM, st>>>(d);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

template <bool AC, bool BC, bool CONJA, bool AK, bool BK>
int pick_tile(const GemmDesc& d, cudaStream_t st) {
  if constexpr (AC || BC) {
    if (d.N <= 32) return launch<AC, BC, CONJA, AK, BK, 128, 32, 4, 1, 3>(d, st);
    // per-walker products with 65-112 rows, a short K and many columns (the Green's function at
    // N = 100: 100 x 400 per walker, K = 100): one tile row of 104 or 112 pads 100 rows 1.04x or
    // 1.12x instead of the 1.28x of two 64-row tiles, 80 columns divide 400; one 8 x 40 warp
    // tile per warp.  At N = 100, 256 walkers: 386 us against 463 us with 64 x 64 tiles (same bits)
    if (d.batch > 1 && d.M > 64 && d.M <= 104 && d.N >= 160 && d.K <= 128)
      return launch<AC, BC, CONJA, AK, BK, 104, 80, 13, 2, 3>(d, st);
    if (d.batch > 1 && d.M > 64 && d.M <= 112 && d.N >= 160 && d.K <= 128)
      return launch<AC, BC, CONJA, AK, BK, 112, 80, 14, 2, 2>(d, st);
    // per-walker 65-112 square products of a real A over a long K (the overlap PsiT W with a real
    // trial at N = 100, K = 400): 56 x 56 tiles of 7 warps, four stages.  232 us against 256 us
    // with 64 x 64 tiles; with a complex A (W^H W) they were slower
    if (!AC && d.batch > 1 && d.M > 64 && d.M <= 112 && d.N > 64 && d.N <= 112 && d.K >= 256)
      return launch<AC, BC, CONJA, AK, BK, 56, 56, 7, 1, 4>(d, st);
    // per-walker products (overlaps, CholeskyQR, propagation, the Green's function): 8 warps per
    // 64 x 64 tile hide more of the DMMA latency on their short K loops (measured 4-6 % faster at
    // N = 100)
    if (d.batch > 1 && (d.N <= 128 || d.K <= 128)) return launch<AC, BC, CONJA, AK, BK, 64, 64, 4, 2, 3>(d, st);
    return launch<AC, BC, CONJA, AK, BK, 64, 64, 2, 2, 3>(d, st);
  } else {
    return launch<AC, BC, CONJA, AK, BK, 128, 64, 4, 2, 3>(d, st);
  }
}

}  // namespace

int gemm_f64(const GemmDesc& d, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || d.batch <= 0) return SFQ_OK;
  if (d.K <= 0) {
    if (d.beta.x != 0.0 || d.beta.y != 0.0)
      return record_error(SFQ_ERR_SHAPE, "gemm_f64: K=0 with beta != 0 is not supported");
  }
  const bool AK = d.sAk == 1, BK = d.sBk == 1;
  if (!AK && d.sAm != 1) return record_error(SFQ_ERR_SHAPE, "gemm_f64: A must be contiguous along K or M");
  if (!BK && d.sBn != 1) return record_error(SFQ_ERR_SHAPE, "gemm_f64: B must be contiguous along K or N");
  const bool AC = d.a_cplx, BC = d.b_cplx, CJ = d.conj_a && d.a_cplx;
  // instantiations used by the AFQMC path
  if (!AC && BC && !CJ && AK && !BK) return pick_tile<false, true, false, true, false>(d, st);
  if (AC && BC && !CJ && AK && !BK) return pick_tile<true, true, false, true, false>(d, st);
  if (AC && BC && !CJ && !AK && BK) return pick_tile<true, true, false, false, true>(d, st);
  if (AC && !BC && !CJ && AK && BK) return pick_tile<true, false, false, true, true>(d, st);
  if (AC && BC && !CJ && AK && BK) return pick_tile<true, true, false, true, true>(d, st);
  if (AC && BC && CJ && !AK && !BK) return pick_tile<true, true, true, false, false>(d, st);
  // conj(A) contiguous along K: the back-propagated references' full Green's function
  if (AC && BC && CJ && AK && !BK) return pick_tile<true, true, true, true, false>(d, st);
  if (!AC && !BC && !CJ && AK && !BK) return pick_tile<false, false, false, true, false>(d, st);
  if (AC && !BC && !CJ && AK && !BK) return pick_tile<true, false, false, true, false>(d, st);
  if (!AC && !BC && !CJ && AK && BK) return pick_tile<false, false, false, true, true>(d, st);
  if (AC && BC && !CJ && !AK && !BK) return pick_tile<true, true, false, false, false>(d, st);
  if (!AC && BC && !CJ && !AK && !BK) return pick_tile<false, true, false, false, false>(d, st);
  return record_error(SFQ_ERR_UNSUPPORTED, "gemm_f64: operand combination (ac=%d bc=%d conj=%d ak=%d bk=%d) not built",
                      int(AC), int(BC), int(CJ), int(AK), int(BK));
}

}  // namespace sfq
