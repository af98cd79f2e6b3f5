// tcgen05 split-BF16 GEMM (see umma_gemm.cuh).
#include <cuda_bf16.h>

#include <cstring>
#include <mutex>

#include "umma_gemm.cuh"

namespace sfq {
namespace umma {

constexpr int BM = 128;                  // UMMA M (one CTA, accumulator rows = TMEM lanes)
constexpr int BK = 64;                   // bf16 elements per K slice = one 128-byte swizzle row
constexpr int kWarps = 6;                // 0: TMA producer, 1: TMEM owner + MMA issuer, 2-5: epilogue
constexpr int kThreads = kWarps * 32;
constexpr unsigned long long kWaitNs = 2000000000ull;  // bounded waits: 2 s

struct KParams {
  int M, N, K;
  int a_batched, b_batched;
  float* C;
  long ldc, sCb;
  float alpha, beta;
  int nterms;
  int* err;
};

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for the phase with the given parity; false when the deadline passes.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long deadline) {
  uint32_t spins = 0;
  while (!mbar_try_wait(bar, parity)) {
    if ((++spins & 255u) == 0u && gtimer() > deadline) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(su32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(su32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major operand tile, 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc(const void* tile) {
  const uint64_t addr = su32(tile);
  uint64_t d = 0;
  d |= (addr & 0x3FFFFull) >> 4;        // start address
  d |= uint64_t(1) << 16;               // leading byte offset (unused for swizzled K-major)
  d |= uint64_t(1024 >> 4) << 32;       // stride byte offset: next 8-row group
  d |= uint64_t(1) << 46;               // descriptor version (sm_100)
  d |= uint64_t(2) << 61;               // SWIZZLE_128B
  return d;
}

template <int BN>
__host__ __device__ constexpr uint32_t instr_desc() {
  // kind::f16: D = F32, A = B = BF16, both K-major, N = BN, M = 128
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) | (uint32_t(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2),
        "r"(mask3));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int BN>
__host__ __device__ constexpr uint32_t tmem_cols() {
  return BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
}

template <int BN, int STAGES>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int BAR_OFF = STAGES * STAGE;
  static constexpr int TOTAL = BAR_OFF + (2 * STAGES + 1) * 8 + 16 + 1024;  // + alignment slack
  static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "tiles must keep 1024-byte alignment");
};

template <int BN, int STAGES>
__global__ void __launch_bounds__(kThreads, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
                     const __grid_constant__ CUtensorMap tBh, const __grid_constant__ CUtensorMap tBl, KParams p) {
  using L = Smem<BN, STAGES>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
  uint64_t* empty = full + STAGES;
  uint64_t* accum = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
  volatile int* s_abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN, bz = blockIdx.z;
  const int KT = (p.K + BK - 1) / BK;
  const bool three = p.nterms == 3;
  const uint32_t stage_tx = three ? uint32_t(2 * L::A_BYTES + 2 * L::B_BYTES) : uint32_t(L::A_BYTES + L::B_BYTES);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "r"(tmem_cols<BN>()));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const unsigned long long deadline = gtimer() + kWaitNs;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      int issued = 0;
      for (int kt = 0; kt < KT; ++kt) {
        const int s = kt % STAGES;
        const uint32_t ph = (kt / STAGES) & 1;
        if (!mbar_wait(&empty[s], ph ^ 1, deadline)) {
          *s_abort = 1;
          break;
        }
        if (*s_abort) break;
        unsigned char* st = smem + s * L::STAGE;
        mbar_expect_tx(&full[s], stage_tx);
        const int k0 = kt * BK;
        const int ab = p.a_batched ? bz : 0, bb = p.b_batched ? bz : 0;
        tma_load_3d(st, &tAh, &full[s], k0, m0, ab);
        tma_load_3d(st + 2 * L::A_BYTES, &tBh, &full[s], k0, n0, bb);
        if (three) {
          tma_load_3d(st + L::A_BYTES, &tAl, &full[s], k0, m0, ab);
          tma_load_3d(st + 2 * L::A_BYTES + L::B_BYTES, &tBl, &full[s], k0, n0, bb);
        }
        issued = kt + 1;
      }
      // drain: every issued stage must have landed before the CTA may exit
      for (int kt = (issued > STAGES ? issued - STAGES : 0); kt < issued; ++kt)
        mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1, gtimer() + kWaitNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc = instr_desc<BN>();
      for (int kt = 0; kt < KT; ++kt) {
        const int s = kt % STAGES;
        const uint32_t ph = (kt / STAGES) & 1;
        if (*s_abort || !mbar_wait(&full[s], ph, deadline)) {
          *s_abort = 1;
          break;
        }
        fence_after();
        unsigned char* st = smem + s * L::STAGE;
        const uint64_t ah = smem_desc(st), al = smem_desc(st + L::A_BYTES);
        const uint64_t bh = smem_desc(st + 2 * L::A_BYTES), bl = smem_desc(st + 2 * L::A_BYTES + L::B_BYTES);
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          const uint64_t off = uint64_t(kk * 32) >> 4;  // 16 bf16 = 32 bytes along the swizzled row
          umma_bf16(tmem, ah + off, bh + off, idesc, (kt | kk) ? 1u : 0u);
          if (three) {
            umma_bf16(tmem, ah + off, bl + off, idesc, 1u);
            umma_bf16(tmem, al + off, bh + off, idesc, 1u);
          }
        }
        umma_commit(&empty[s]);
      }
      umma_commit(accum);
    }
  } else {  // epilogue warps 2..5 -> TMEM lane quarters 2,3,0,1
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const bool ok = mbar_wait(accum, 0, deadline);
    fence_after();
    if (ok && !*s_abort) {
      const int gm = m0 + row;
      float* Cb = p.C + (long)bz * p.sCb;
#pragma unroll 1
      for (int c = 0; c < BN; c += 16) {
        float v[16];
        tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(c), v);
        if (gm < p.M) {
          float* crow = Cb + (long)gm * p.ldc;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int gn = n0 + c + j;
            if (gn < p.N) {
              float out = p.alpha * v[j];
              if (p.beta != 0.f) out += p.beta * crow[gn];
              crow[gn] = out;
            }
          }
        }
      }
    } else if (!ok) {
      *s_abort = 1;
    }
  }
  fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && *s_abort && p.err) atomicExch(p.err, SFQ_ERR_TIMEOUT);
  if (warp == 1) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols<BN>()));
  }
}

// ---- host side: tensor maps ---------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

int make_map(CUtensorMap* m, const void* base, long rows, long K, long ld, long batch, long bstride, int box_rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return record_error(SFQ_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 8) || (K % 8))
    return record_error(SFQ_ERR_SHAPE, "umma_gemm: operands need 16-byte alignment and K, ld multiples of 8");
  if (batch <= 1) {
    batch = 1;
    bstride = ((rows * ld) + 7) / 8 * 8;
  } else if (bstride % 8) {
    return record_error(SFQ_ERR_SHAPE, "umma_gemm: batch stride must be a multiple of 8 elements");
  }
  cuuint64_t dims[3] = {cuuint64_t(K), cuuint64_t(rows), cuuint64_t(batch)};
  cuuint64_t strides[2] = {cuuint64_t(ld) * 2, cuuint64_t(bstride) * 2};
  cuuint32_t box[3] = {cuuint32_t(BK), cuuint32_t(box_rows), 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return record_error(SFQ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", int(r));
  return SFQ_OK;
}

template <int BN, int STAGES>
int launch(const UmmaGemmDesc& d, cudaStream_t st) {
  using L = Smem<BN, STAGES>;
  CUtensorMap ah, al, bh, bl;
  int rc;
  const long ab = d.A.batch_stride ? d.batch : 1, bb = d.B.batch_stride ? d.batch : 1;
  if ((rc = make_map(&ah, d.A.hi, d.A.rows, d.K, d.A.ld, ab, d.A.batch_stride, BM))) return rc;
  if ((rc = make_map(&bh, d.B.hi, d.B.rows, d.K, d.B.ld, bb, d.B.batch_stride, BN))) return rc;
  if (d.nterms == 3) {
    if ((rc = make_map(&al, d.A.lo, d.A.rows, d.K, d.A.ld, ab, d.A.batch_stride, BM))) return rc;
    if ((rc = make_map(&bl, d.B.lo, d.B.rows, d.K, d.B.ld, bb, d.B.batch_stride, BN))) return rc;
  } else {
    al = ah;
    bl = bh;
  }
  KParams kp;
  kp.M = d.M; kp.N = d.N; kp.K = d.K;
  kp.a_batched = d.A.batch_stride != 0; kp.b_batched = d.B.batch_stride != 0;
  kp.C = d.C; kp.ldc = d.ldc; kp.sCb = d.sCb; kp.alpha = d.alpha; kp.beta = d.beta;
  kp.nterms = d.nterms; kp.err = d.err;
  auto k = umma_gemm_kernel<BN, STAGES>;
  SFQ_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L::TOTAL));
  dim3 grid((d.M + BM - 1) / BM, (d.N + BN - 1) / BN, d.batch);
  if (grid.y > 65535u || grid.z > 65535u) return record_error(SFQ_ERR_SHAPE, "umma_gemm: grid too large");
  k<<<grid, kThreads, L::TOTAL, st>>>(ah, al, bh, bl, kp);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

__global__ void split_f64_kernel(const double* src, long n, __nv_bfloat16* hi, __nv_bfloat16* lo) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const double x = src[e];
    const __nv_bfloat16 h = __float2bfloat16_rn(float(x));
    hi[e] = h;
    if (lo) lo[e] = __float2bfloat16_rn(float(x - double(__bfloat162float(h))));
  }
}

}  // namespace umma

int umma_gemm(const UmmaGemmDesc& d, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || d.batch <= 0) return SFQ_OK;
  if (d.K <= 0) return record_error(SFQ_ERR_SHAPE, "umma_gemm: K must be positive");
  if (d.nterms != 1 && d.nterms != 3) return record_error(SFQ_ERR_ARG, "umma_gemm: nterms must be 1 or 3");
  if (d.nterms == 3 && (!d.A.lo || !d.B.lo)) return record_error(SFQ_ERR_ARG, "umma_gemm: lo planes missing");
  const int bn = d.bn ? d.bn : (d.N <= 64 ? 64 : 128);
  switch (bn) {
    case 64: return umma::launch<64, 4>(d, st);
    case 128: return umma::launch<128, 3>(d, st);
    case 256: return umma::launch<256, 2>(d, st);
    default: return record_error(SFQ_ERR_ARG, "umma_gemm: tile width %d not built (64, 128, 256)", bn);
  }
}

// C ABI test/benchmark entry: fp64 operands split on the fly
int gemm_split_bf16_f64(const double* A, const double* B, float* C, int M, int N, int K, int batch, int a_batched,
                        int b_batched, int nterms, int bn, cudaStream_t st) {
  const long na = (long)M * K * (a_batched ? batch : 1), nb = (long)N * K * (b_batched ? batch : 1);
  void* buf = nullptr;
  const size_t bytes = size_t(2) * 2 * (na + nb) + 1024;
  SFQ_CUDA_TRY(cudaMallocAsync(&buf, bytes, st));
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  char* base = (char*)buf;
  void* ah = base;
  void* alo = base + al(2 * na);
  void* bh = base + 2 * al(2 * na);
  void* blo = base + 2 * al(2 * na) + al(2 * nb);
  int rc = split_bf16_f64(A, na, ah, alo, st);
  if (!rc) rc = split_bf16_f64(B, nb, bh, blo, st);
  if (!rc) {
    UmmaGemmDesc d;
    d.M = M; d.N = N; d.K = K; d.batch = batch;
    d.A.hi = ah; d.A.lo = alo; d.A.rows = M; d.A.ld = K; d.A.batch_stride = a_batched ? (long)M * K : 0;
    d.B.hi = bh; d.B.lo = blo; d.B.rows = N; d.B.ld = K; d.B.batch_stride = b_batched ? (long)N * K : 0;
    d.C = C; d.ldc = N; d.sCb = (long)M * N;
    d.nterms = nterms; d.bn = bn;
    rc = umma_gemm(d, st);
  }
  cudaFreeAsync(buf, st);
  return rc;
}

int split_bf16_f64(const double* src, long n, void* hi, void* lo, cudaStream_t st) {
  if (n <= 0) return SFQ_OK;
  long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  umma::split_f64_kernel<<<int(g), 256, 0, st>>>(src, n, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

}  // namespace sfq
