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
  int* err;
};

// products (plane of A, plane of B) kept for NP planes: the pairs of combined order < NP, listed
// so that NP = 1, 2, 3 use the first 1, 3, 6 entries
__host__ __device__ constexpr int n_terms(int np) { return np == 1 ? 1 : np == 2 ? 3 : 6; }
__host__ __device__ constexpr int term_a(int t) { return t < 2 ? 0 : t == 2 ? 1 : t == 3 ? 0 : t == 4 ? 1 : 2; }
__host__ __device__ constexpr int term_b(int t) { return t == 0 ? 0 : t == 1 ? 1 : t == 2 ? 0 : t == 3 ? 2 : t == 4 ? 1 : 0; }

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

template <int BN, int STAGES, int NP>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE = NP * (A_BYTES + B_BYTES);
  static constexpr int BAR_OFF = STAGES * STAGE;
  static constexpr int TOTAL = BAR_OFF + (2 * STAGES + 1) * 8 + 16 + 1024;  // + alignment slack
  static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "tiles must keep 1024-byte alignment");
};

struct Maps {
  CUtensorMap a[3], b[3];
};

template <int BN, int STAGES, int NP>
__global__ void __launch_bounds__(kThreads, 1) umma_gemm_kernel(const __grid_constant__ Maps maps, KParams p) {
  using L = Smem<BN, STAGES, NP>;
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
  const uint32_t stage_tx = uint32_t(L::STAGE);

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
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          tma_load_3d(st + q * L::A_BYTES, &maps.a[q], &full[s], k0, m0, ab);
          tma_load_3d(st + NP * L::A_BYTES + q * L::B_BYTES, &maps.b[q], &full[s], k0, n0, bb);
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
        uint64_t ad[NP], bd[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          ad[q] = smem_desc(st + q * L::A_BYTES);
          bd[q] = smem_desc(st + NP * L::A_BYTES + q * L::B_BYTES);
        }
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          const uint64_t off = uint64_t(kk * 32) >> 4;  // 16 bf16 = 32 bytes along the swizzled row
#pragma unroll
          for (int tt = 0; tt < n_terms(NP); ++tt)
            umma_bf16(tmem, ad[term_a(tt)] + off, bd[term_b(tt)] + off, idesc, (kt | kk | tt) ? 1u : 0u);
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

template <int BN, int STAGES, int NP>
int launch(const UmmaGemmDesc& d, cudaStream_t st) {
  using L = Smem<BN, STAGES, NP>;
  static_assert(L::TOTAL <= 232448, "shared memory budget");
  Maps maps;
  int rc;
  const long ab = d.A.batch_stride ? d.batch : 1, bb = d.B.batch_stride ? d.batch : 1;
  for (int q = 0; q < NP; ++q) {
    if (!d.A.p[q] || !d.B.p[q]) return record_error(SFQ_ERR_ARG, "umma_gemm: plane %d missing", q);
    if ((rc = make_map(&maps.a[q], d.A.p[q], d.A.rows, d.K, d.A.ld, ab, d.A.batch_stride, BM))) return rc;
    if ((rc = make_map(&maps.b[q], d.B.p[q], d.B.rows, d.K, d.B.ld, bb, d.B.batch_stride, BN))) return rc;
  }
  for (int q = NP; q < 3; ++q) {
    maps.a[q] = maps.a[0];
    maps.b[q] = maps.b[0];
  }
  KParams kp;
  kp.M = d.M; kp.N = d.N; kp.K = d.K;
  kp.a_batched = d.A.batch_stride != 0; kp.b_batched = d.B.batch_stride != 0;
  kp.C = d.C; kp.ldc = d.ldc; kp.sCb = d.sCb; kp.alpha = d.alpha; kp.beta = d.beta;
  kp.err = d.err;
  auto k = umma_gemm_kernel<BN, STAGES, NP>;
  SFQ_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L::TOTAL));
  dim3 grid((d.M + BM - 1) / BM, (d.N + BN - 1) / BN, d.batch);
  if (grid.y > 65535u || grid.z > 65535u) return record_error(SFQ_ERR_SHAPE, "umma_gemm: grid too large");
  k<<<grid, kThreads, L::TOTAL, st>>>(maps, kp);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

__global__ void split_f64_kernel(const double* src, long n, __nv_bfloat16* p0, __nv_bfloat16* p1,
                                 __nv_bfloat16* p2) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const double x = src[e];
    const __nv_bfloat16 h0 = __float2bfloat16_rn(float(x));
    p0[e] = h0;
    const double r1 = x - double(__bfloat162float(h0));
    const __nv_bfloat16 h1 = __float2bfloat16_rn(float(r1));
    if (p1) p1[e] = h1;
    if (p2) p2[e] = __float2bfloat16_rn(float(r1 - double(__bfloat162float(h1))));
  }
}

}  // namespace umma

int umma_gemm(const UmmaGemmDesc& d, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || d.batch <= 0) return SFQ_OK;
  if (d.K <= 0) return record_error(SFQ_ERR_SHAPE, "umma_gemm: K must be positive");
  const int bn = d.bn ? d.bn : (d.N <= 64 ? 64 : 128);
  switch (d.nplanes * 1000 + bn) {
    case 1064: return umma::launch<64, 6, 1>(d, st);
    case 1128: return umma::launch<128, 6, 1>(d, st);
    case 1256: return umma::launch<256, 4, 1>(d, st);
    case 2064: return umma::launch<64, 4, 2>(d, st);
    case 2128: return umma::launch<128, 3, 2>(d, st);
    case 2256: return umma::launch<256, 2, 2>(d, st);
    case 3064: return umma::launch<64, 3, 3>(d, st);
    case 3128: return umma::launch<128, 2, 3>(d, st);
    default:
      return record_error(SFQ_ERR_ARG, "umma_gemm: %d planes with tile width %d not built", d.nplanes, bn);
  }
}

// C ABI test/benchmark entry: fp64 operands split on the fly
int gemm_split_bf16_f64(const double* A, const double* B, float* C, int M, int N, int K, int batch, int a_batched,
                        int b_batched, int nplanes, int bn, cudaStream_t st) {
  if (nplanes < 1 || nplanes > 3) return record_error(SFQ_ERR_ARG, "nplanes must be 1, 2 or 3");
  const long na = (long)M * K * (a_batched ? batch : 1), nb = (long)N * K * (b_batched ? batch : 1);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t pa = al(2 * na), pb = al(2 * nb);
  void* buf = nullptr;
  SFQ_CUDA_TRY(cudaMallocAsync(&buf, nplanes * (pa + pb) + 256, st));
  char* base = (char*)buf;
  UmmaGemmDesc d;
  for (int q = 0; q < nplanes; ++q) {
    d.A.p[q] = base + q * pa;
    d.B.p[q] = base + nplanes * pa + q * pb;
  }
  int rc = split_bf16_f64(A, na, (void*)d.A.p[0], nplanes > 1 ? (void*)d.A.p[1] : nullptr,
                          nplanes > 2 ? (void*)d.A.p[2] : nullptr, st);
  if (!rc)
    rc = split_bf16_f64(B, nb, (void*)d.B.p[0], nplanes > 1 ? (void*)d.B.p[1] : nullptr,
                        nplanes > 2 ? (void*)d.B.p[2] : nullptr, st);
  if (!rc) {
    d.M = M; d.N = N; d.K = K; d.batch = batch;
    d.A.rows = M; d.A.ld = K; d.A.batch_stride = a_batched ? (long)M * K : 0;
    d.B.rows = N; d.B.ld = K; d.B.batch_stride = b_batched ? (long)N * K : 0;
    d.C = C; d.ldc = N; d.sCb = (long)M * N;
    d.nplanes = nplanes; d.bn = bn;
    rc = umma_gemm(d, st);
  }
  cudaFreeAsync(buf, st);
  return rc;
}

int split_bf16_f64(const double* src, long n, void* p0, void* p1, void* p2, cudaStream_t st) {
  if (n <= 0) return SFQ_OK;
  long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  umma::split_f64_kernel<<<int(g), 256, 0, st>>>(src, n, (__nv_bfloat16*)p0, (__nv_bfloat16*)p1,
                                                 (__nv_bfloat16*)p2);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

}  // namespace sfq
