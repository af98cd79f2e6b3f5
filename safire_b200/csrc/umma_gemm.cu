// tcgen05 split-BF16 GEMM (see umma_gemm.cuh).
#include <cuda_bf16.h>

#include <cstring>
#include <mutex>

#include "tc_common.cuh"
#include "umma_gemm.cuh"

namespace sfq {
namespace tc {
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

int sm_count() {
  static int counts[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!counts[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    counts[dev] = n;
  }
  return counts[dev];
}

}  // namespace tc

namespace umma {
using namespace tc;

constexpr int BM = 128;                  // UMMA M (one CTA, accumulator rows = TMEM lanes)
constexpr int BK = 64;                   // bf16 elements per K slice = one 128-byte swizzle row
constexpr int kWarps = 6;                // 0: TMA producer, 1: TMEM owner + MMA issuer, 2-5: epilogue
constexpr int kThreads = kWarps * 32;
constexpr unsigned long long kWaitNs = 2000000000ull;  // limit of one wait: 2 s without progress

struct KParams {
  int M, N, K;
  int a_batched, b_batched;
  int MT, NT, KS;  // tiles along M, N; K splits
  int batch;
  int cb_half, cb_nmo, cb_kth, cb_ldh;  // complex B (cb_half > 0): see UmmaGemmDesc
  long tiles;
  float* C;
  long ldc, sCb, sCk;  // sCk: elements between the partial outputs of the K splits
  float alpha, beta;
  UmmaEpilogue e;
  int* err;
  unsigned long long wait_ns;  // limit of one mbarrier wait
};

// products (plane of A, plane of B) kept for NP planes: the pairs of combined order < NP, listed
// so that NP = 1, 2, 3 use the first 1, 3, 6 entries
__host__ __device__ constexpr int n_terms(int np) { return np == 1 ? 1 : np == 2 ? 3 : 6; }
__host__ __device__ constexpr int term_a(int t) { return t < 2 ? 0 : t == 2 ? 1 : t == 3 ? 0 : t == 4 ? 1 : 2; }
__host__ __device__ constexpr int term_b(int t) { return t == 0 ? 0 : t == 1 ? 1 : t == 2 ? 0 : t == 3 ? 2 : t == 4 ? 1 : 0; }

template <int BN>
__host__ __device__ constexpr uint32_t instr_desc() {
  // kind::f16: D = F32, A = B = BF16, both K-major, N = BN, M = 128
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) | (uint32_t(BM >> 4) << 24);
}
__host__ __device__ inline uint32_t instr_desc_n(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | (uint32_t(BM >> 4) << 24);
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

template <int BN>
__host__ __device__ constexpr uint32_t tmem_cols() {
  return BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
}

// JOINT: complex-B products whose stage holds both halves of A (re and im parts of the walker
// operand at the same k) against one load of the tile's [Vr; Vi] rows
template <int BN, int STAGES, int NP, bool JOINT = false>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int A_SLOTS = JOINT ? 2 : 1;
  static constexpr int STAGE = NP * (A_SLOTS * A_BYTES + B_BYTES);
  static constexpr int BAR_OFF = STAGES * STAGE;
  static constexpr int NBAR = 2 * STAGES + 5;  // full, empty, acc_full[2], acc_empty[2], done
  static constexpr int TOTAL = BAR_OFF + NBAR * 8 + 16 + 1024;  // + alignment slack
  static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "tiles must keep 1024-byte alignment");
};

struct Maps {
  CUtensorMap a[3], b[3];
};

// tile t -> (M tile, N tile, batch, K split), M fastest, K split slowest
__device__ __forceinline__ void decode(const KParams& p, long t, int& mt, int& nt, int& bz, int& ks) {
  mt = int(t % p.MT);
  long r = t / p.MT;
  nt = int(r % p.NT);
  r /= p.NT;
  const long nb = p.tiles / ((long)p.MT * p.NT * p.KS);
  bz = int(r % nb);
  ks = int(r / nb);
}
// first K block of split s of KS over KT blocks (whole blocks, as even as they come)
__device__ __forceinline__ int k_begin(int KT, int KS, int s) { return int((long)KT * s / KS); }

// ---- epilogue helpers --------------------------------------------------------------------
// planes of x: p0 = bf16(x), p1 = bf16(x - p0), p2 = bf16(x - p0 - p1)
__device__ __forceinline__ void split3(float x, __nv_bfloat16& h0, __nv_bfloat16& h1, __nv_bfloat16& h2) {
  h0 = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h0);
  h1 = __float2bfloat16_rn(r1);
  h2 = __float2bfloat16_rn(r1 - __bfloat162float(h1));
}

// 16 consecutive values -> np planes at idx (vector stores when aligned: idx % 8 == 0)
__device__ __forceinline__ void put_planes16(const float* v, void* const* out, int np, long idx, bool vec, int valid) {
  __nv_bfloat16 h[3][16];
#pragma unroll
  for (int j = 0; j < 16; ++j) split3(v[j], h[0][j], h[1][j], h[2][j]);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q >= np) break;
    __nv_bfloat16* dst = static_cast<__nv_bfloat16*>(out[q]) + idx;
    if (vec) {
      uint4 w0, w1;
      memcpy(&w0, &h[q][0], 16);
      memcpy(&w1, &h[q][8], 16);
      reinterpret_cast<uint4*>(dst)[0] = w0;
      reinterpret_cast<uint4*>(dst)[1] = w1;
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (j < valid) dst[j] = h[q][j];
    }
  }
}

__device__ __forceinline__ void ld16f(const float* src, float* v, bool vec, int valid) {
  if (vec) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float4 x = reinterpret_cast<const float4*>(src)[j];
      v[4 * j] = x.x; v[4 * j + 1] = x.y; v[4 * j + 2] = x.z; v[4 * j + 3] = x.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = j < valid ? src[j] : 0.f;
  }
}
__device__ __forceinline__ void st16f(float* dst, const float* v, bool vec, int valid) {
  if (vec) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      reinterpret_cast<float4*>(dst)[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (j < valid) dst[j] = v[j];
  }
}

// the accumulator row `row` (TMEM lane) of one tile, at column base taddr, through the epilogue
template <int BN>
__device__ __forceinline__ void epilogue_tile(const KParams& p, uint32_t taddr, int row, int mt, int nt, int bz,
                                              int ks) {
  const int gm = mt * BM + row;  // row within the batch
  const bool live = gm < p.M;
  const UmmaEpilogue& e = p.e;
  if (e.kind == UMMA_EPI_TAYLOR) {
    const int h = e.half, nmo = e.nmo, ldh = e.ldh ? e.ldh : e.nmo;
    const long srow = ((long)bz * p.M + gm) * (2L * nmo);
    const long prow = ((long)bz * p.M + gm) * (2L * ldh);
#pragma unroll 1
    for (int c = 0; c < h; c += 16) {
      float re[16], im[16];
      __syncwarp();
      tmem_ld16(taddr + uint32_t(c), re);
      tmem_ld16(taddr + uint32_t(h + c), im);
      const int i0 = nt * h + c;
      if (live && i0 < nmo) {
      const int valid = nmo - i0 < 16 ? nmo - i0 : 16;
      const bool vec = valid == 16 && (nmo % 8) == 0;
      float tr[16], ti[16], s0[16], s1[16];
      float* S0 = e.S + srow + i0;
      float* S1 = S0 + nmo;
      ld16f(S0, s0, vec, valid);
      ld16f(S1, s1, vec, valid);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        tr[j] = -im[j] * e.inv_k;
        ti[j] = re[j] * e.inv_k;
        s0[j] += tr[j];
        s1[j] += ti[j];
      }
      st16f(S0, s0, vec, valid);
      st16f(S1, s1, vec, valid);
      const bool pvec = valid == 16 && (ldh % 8) == 0;
      if (e.write == 1) {
        put_planes16(tr, e.out, e.out_planes, prow + i0, pvec, valid);
        put_planes16(ti, e.out, e.out_planes, prow + ldh + i0, pvec, valid);
      } else if (e.write == 2) {
        put_planes16(s0, e.out, e.out_planes, prow + i0, pvec, valid);
        put_planes16(s1, e.out, e.out_planes, prow + ldh + i0, pvec, valid);
      }
      }
    }
    return;
  }
  if (e.kind == UMMA_EPI_PLANAR_SPLIT) {
    const int c = gm / e.nel, a = gm - c * e.nel;
    const long orow = ((long)c * p.batch + bz) * e.nel + a;
#pragma unroll 1
    for (int cc = 0; cc < BN; cc += 16) {
      float v[16];
      __syncwarp();
      tmem_ld16(taddr + uint32_t(cc), v);
      const int n0 = nt * BN + cc;
      if (live && n0 < p.N) {
        const int valid = p.N - n0 < 16 ? p.N - n0 : 16;
        const long idx = orow * e.nmo + n0;
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] *= p.alpha;
        put_planes16(v, e.out, e.out_planes, idx, valid == 16 && (idx % 8) == 0, valid);
      }
    }
    return;
  }
  if (e.kind == UMMA_EPI_TO_WALKERS) {
    // rows (w, a, c) of the walker operand, columns j
    const int w = gm / (2 * e.nel), a = (gm >> 1) % e.nel, cp = gm & 1;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      __syncwarp();
      tmem_ld16(taddr + uint32_t(c), v);
      if (live) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int gn = nt * BN + c + j;
          if (gn < p.N) e.SM[(((long)w * p.N + gn) * e.nel + a) * 2 + cp] = double(p.alpha * v[j]);
        }
      }
    }
    return;
  }
  // STORE / STORE_SPLIT
  const long rbase = (long)ks * p.sCk + (long)bz * p.sCb + (long)gm * p.ldc;
  float* crow = p.C + rbase;
#pragma unroll 1
  for (int c = 0; c < BN; c += 16) {
    float v[16];
    __syncwarp();
    tmem_ld16(taddr + uint32_t(c), v);
    const int n0 = nt * BN + c;
    if (!live || n0 >= p.N) continue;
    const int valid = p.N - n0 < 16 ? p.N - n0 : 16;
    const bool vec4 = valid == 16 && ((rbase + n0) % 4) == 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] *= p.alpha;
    if (p.beta != 0.f) {
      float o[16];
      ld16f(crow + n0, o, vec4, valid);
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] += p.beta * o[j];
    }
    st16f(crow + n0, v, vec4, valid);
    if (e.kind == UMMA_EPI_STORE_SPLIT) {
      const long pidx = (long)ks * p.sCk + (long)bz * p.sCb + (long)gm * (e.ldh ? e.ldh : p.ldc) + n0;
      put_planes16(v, e.out, e.out_planes, pidx, valid == 16 && (pidx % 8) == 0, valid);
    }
  }
}

template <int BN, int STAGES, int NP, bool JOINT>
__global__ void __launch_bounds__(kThreads, 1) umma_gemm_kernel(const __grid_constant__ Maps maps,
                                                                const __grid_constant__ KParams p) {
  using L = Smem<BN, STAGES, NP, JOINT>;
  constexpr uint32_t COLS = tmem_cols<BN>();  // one accumulator buffer; two are allocated
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;  // [2]
  uint64_t* acc_empty = acc_full + 2;   // [2]
  uint64_t* done = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* s_abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int KT = JOINT ? p.cb_kth : (p.K + BK - 1) / BK;  // JOINT: one stage per k slice of both halves
  const uint32_t stage_tx = uint32_t(L::STAGE);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 128);
    }
    mbar_init(done, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "r"(2 * COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const unsigned long long wait_ns = p.wait_ns;  // each wait may take this long from its own start

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      uint32_t it = 0;
      bool stop = false;
      for (long t = blockIdx.x; t < p.tiles && !stop; t += gridDim.x) {
        int mt, nt, bz, ks;
        decode(p, t, mt, nt, bz, ks);
        const int m0 = mt * BM, n0 = nt * BN;
        const int ab = p.a_batched ? bz : 0, bb = p.b_batched ? bz : 0;
        const int kb = k_begin(KT, p.KS, ks), ke = k_begin(KT, p.KS, ks + 1);
        for (int kt = kb; kt < ke; ++kt, ++it) {
          const int s = int(it % STAGES);
          const uint32_t ph = (it / STAGES) & 1;
          if (!mbar_wait_for(&empty[s], ph ^ 1, wait_ns) || *s_abort) {
            *s_abort = 1;
            stop = true;
            break;
          }
          unsigned char* st = smem + s * L::STAGE;
          mbar_expect_tx(&full[s], stage_tx);
          if constexpr (JOINT) {
            // k slice kt of both halves: A at k0 (re) and ldh + k0 (im), B the tile's [Vr; Vi] rows once
            const int k0 = kt * BK, i0 = nt * p.cb_half;
#pragma unroll
            for (int q = 0; q < NP; ++q) {
              unsigned char* aq = st + q * 2 * L::A_BYTES;
              unsigned char* bt = st + NP * 2 * L::A_BYTES + q * L::B_BYTES;
              tma_load_3d(aq, &maps.a[q], &full[s], k0, m0, ab);
              tma_load_3d(aq + L::A_BYTES, &maps.a[q], &full[s], p.cb_ldh + k0, m0, ab);
              tma_load_3d(bt, &maps.b[q], &full[s], k0, i0, bb);
              tma_load_3d(bt + p.cb_half * (BK * 2), &maps.b[q], &full[s], k0, p.cb_nmo + i0, bb);
            }
          } else if (p.cb_half) {
            // K slice kt = (c', k0): A at c' * ldh + k0; B: the Vr and Vi rows of the tile's orbitals,
            // [Vr; Vi] for c' = 0 and [Vi; Vr] for c' = 1 (each box half the tile)
            const int cp = kt / p.cb_kth, k0 = (kt - cp * p.cb_kth) * BK;
            const int i0 = nt * p.cb_half;
            const int r1 = (cp ? p.cb_nmo : 0) + i0, r2 = (cp ? 0 : p.cb_nmo) + i0;
#pragma unroll
            for (int q = 0; q < NP; ++q) {
              unsigned char* bt = st + NP * L::A_BYTES + q * L::B_BYTES;
              tma_load_3d(st + q * L::A_BYTES, &maps.a[q], &full[s], cp * p.cb_ldh + k0, m0, ab);
              tma_load_3d(bt, &maps.b[q], &full[s], k0, r1, bb);
              tma_load_3d(bt + p.cb_half * (BK * 2), &maps.b[q], &full[s], k0, r2, bb);
            }
          } else {
            const int k0 = kt * BK;
#pragma unroll
            for (int q = 0; q < NP; ++q) {
              tma_load_3d(st + q * L::A_BYTES, &maps.a[q], &full[s], k0, m0, ab);
              tma_load_3d(st + NP * L::A_BYTES + q * L::B_BYTES, &maps.b[q], &full[s], k0, n0, bb);
            }
          }
        }
      }
      // drain: every issued stage must have landed before the CTA may exit
      for (uint32_t j = (it > uint32_t(STAGES) ? it - STAGES : 0u); j < it; ++j)
        mbar_wait_for(&full[j % STAGES], (j / STAGES) & 1, kWaitNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc = instr_desc<BN>();
      uint32_t it = 0;
      int lt = 0;
      bool stop = false;
      for (long t = blockIdx.x; t < p.tiles && !stop; t += gridDim.x, ++lt) {
        const int b = lt & 1;
        const uint32_t aph = (uint32_t(lt) >> 1) & 1;
        if (*s_abort || !mbar_wait_for(&acc_empty[b], aph ^ 1, wait_ns)) {
          *s_abort = 1;
          break;
        }
        fence_after();
        const uint32_t d_tmem = tmem + uint32_t(b) * COLS;
        int mt, nt, bz, ks;
        decode(p, t, mt, nt, bz, ks);
        const int kb = k_begin(KT, p.KS, ks), ke = k_begin(KT, p.KS, ks + 1);
        for (int kt = kb; kt < ke; ++kt, ++it) {
          const int s = int(it % STAGES);
          const uint32_t ph = (it / STAGES) & 1;
          if (*s_abort || !mbar_wait_for(&full[s], ph, wait_ns)) {
            *s_abort = 1;
            stop = true;
            break;
          }
          fence_after();
          unsigned char* st = smem + s * L::STAGE;
          uint64_t ad[NP], bd[NP];
#pragma unroll
          for (int q = 0; q < NP; ++q) {
            ad[q] = smem_desc(st + q * L::A_SLOTS * L::A_BYTES);
            bd[q] = smem_desc(st + NP * L::A_SLOTS * L::A_BYTES + q * L::B_BYTES);
          }
          if constexpr (JOINT) {
            // [re | im] += A_re [Vr; Vi]^T (one N = BN product), re -= A_im Vi^T, im += A_im Vr^T
            const uint32_t h = uint32_t(p.cb_half);
            const uint32_t id_h = instr_desc_n(h), id_hneg = id_h | (1u << 14);  // bit 14: negate B
            const uint64_t boff = uint64_t(h * (BK * 2)) >> 4;
            const uint64_t aim = uint64_t(L::A_BYTES) >> 4;  // the im half, one A tile further
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
              const uint64_t off = uint64_t(kk * 32) >> 4;
#pragma unroll
              for (int tt = 0; tt < n_terms(NP); ++tt) {
                const uint64_t are = ad[term_a(tt)] + off, aimd = ad[term_a(tt)] + aim + off;
                umma_bf16(d_tmem, are, bd[term_b(tt)] + off, idesc, ((kt - kb) | kk | tt) ? 1u : 0u);
                umma_bf16(d_tmem, aimd, bd[term_b(tt)] + boff + off, id_hneg, 1u);
                umma_bf16(d_tmem + h, aimd, bd[term_b(tt)] + off, id_h, 1u);
              }
            }
          } else if (p.cb_half && kt < p.cb_kth) {
            // c' = 0: the boxes [Vr; Vi] lie in shared memory exactly as one 2 * half = BN row tile
            // (half is a multiple of 8, the swizzle atom), so [re | im] += A_re [Vr; Vi]^T is one
            // N = BN product
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
              const uint64_t off = uint64_t(kk * 32) >> 4;
#pragma unroll
              for (int tt = 0; tt < n_terms(NP); ++tt)
                umma_bf16(d_tmem, ad[term_a(tt)] + off, bd[term_b(tt)] + off, idesc, ((kt - kb) | kk | tt) ? 1u : 0u);
            }
          } else if (p.cb_half) {
            // c' = 1: two N = half products per slice, re half with -Vi (the instruction's negate-B
            // bit), im half with Vr, the second B box starting half * 128 bytes into the tile
            const uint32_t h = uint32_t(p.cb_half);
            const uint32_t id_h = instr_desc_n(h), id_hneg = id_h | (1u << 14);  // bit 14: negate B
            const uint64_t boff = uint64_t(h * (BK * 2)) >> 4;
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
              const uint64_t off = uint64_t(kk * 32) >> 4;
#pragma unroll
              for (int tt = 0; tt < n_terms(NP); ++tt) {
                const uint32_t acc = ((kt - kb) | kk | tt) ? 1u : 0u;
                umma_bf16(d_tmem, ad[term_a(tt)] + off, bd[term_b(tt)] + off, id_hneg, acc);
                umma_bf16(d_tmem + h, ad[term_a(tt)] + off, bd[term_b(tt)] + boff + off, id_h, acc);
              }
            }
          } else {
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
              const uint64_t off = uint64_t(kk * 32) >> 4;  // 16 bf16 = 32 bytes along the swizzled row
#pragma unroll
              for (int tt = 0; tt < n_terms(NP); ++tt)
                umma_bf16(d_tmem, ad[term_a(tt)] + off, bd[term_b(tt)] + off, idesc, ((kt - kb) | kk | tt) ? 1u : 0u);
            }
          }
          umma_commit(&empty[s]);
        }
        if (!stop) umma_commit(&acc_full[b]);
      }
      // every MMA issued has completed before the tensor memory may be released
      umma_commit(done);
      mbar_wait_for(done, 0, kWaitNs);
    }
  } else {  // epilogue warps 2..5 -> TMEM lane quarters 2,3,0,1
    const int q = warp & 3;
    const int row = q * 32 + lane;
    int lt = 0;
    for (long t = blockIdx.x; t < p.tiles; t += gridDim.x, ++lt) {
      const int b = lt & 1;
      const uint32_t aph = (uint32_t(lt) >> 1) & 1;
      const bool ok = mbar_wait_for(&acc_full[b], aph, wait_ns);
      // tcgen05.ld is warp-collective: the whole warp goes on, or stops, together
      const bool go = __all_sync(0xffffffffu, ok) && !__any_sync(0xffffffffu, *s_abort != 0);
      if (!go) {
        *s_abort = 1;
        break;
      }
      fence_after();
      int mt, nt, bz, ks;
      decode(p, t, mt, nt, bz, ks);
      epilogue_tile<BN>(p, tmem + (uint32_t(q * 32) << 16) + uint32_t(b) * COLS, row, mt, nt, bz, ks);
      fence_before();
      mbar_arrive(&acc_empty[b]);
    }
  }
  fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && *s_abort && p.err) atomicExch(p.err, SFQ_ERR_TIMEOUT);
  if (warp == 1) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * COLS));
  }
}

// ---- host side: tensor maps ---------------------------------------------------------------
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

template <int BN, int STAGES, int NP, bool JOINT = false>
int launch(const UmmaGemmDesc& d, cudaStream_t st) {
  using L = Smem<BN, STAGES, NP, JOINT>;
  static_assert(L::TOTAL <= 232448, "shared memory budget");
  static_assert(2 * tmem_cols<BN>() <= 512, "two accumulators must fit in tensor memory");
  Maps maps;
  int rc;
  const long ab = d.A.batch_stride ? d.batch : 1, bb = d.B.batch_stride ? d.batch : 1;
  const bool cb = d.cplx_half > 0;
  if (cb && (d.cplx_half * 2 != BN || d.cplx_half % 16 || d.cplx_ldh % BK || d.cplx_ldh < d.cplx_nmo ||
             d.K != 2 * d.cplx_ldh || d.B.rows != 2L * d.cplx_nmo))
    return record_error(SFQ_ERR_ARG, "umma_gemm: complex B needs BN = 2 half, K = 2 ldh, B rows = 2 nmo");
  for (int q = 0; q < NP; ++q) {
    if (!d.A.p[q] || !d.B.p[q]) return record_error(SFQ_ERR_ARG, "umma_gemm: plane %d missing", q);
    if ((rc = make_map(&maps.a[q], d.A.p[q], d.A.rows, d.K, d.A.ld, ab, d.A.batch_stride, BM))) return rc;
    if (cb) {
      if ((rc = make_map(&maps.b[q], d.B.p[q], d.B.rows, d.cplx_nmo, d.B.ld, bb, d.B.batch_stride, d.cplx_half)))
        return rc;
    } else if ((rc = make_map(&maps.b[q], d.B.p[q], d.B.rows, d.K, d.B.ld, bb, d.B.batch_stride, BN))) {
      return rc;
    }
  }
  for (int q = NP; q < 3; ++q) {
    maps.a[q] = maps.a[0];
    maps.b[q] = maps.b[0];
  }
  const UmmaEpilogue& e = d.epi;
  if (e.kind == UMMA_EPI_PLANAR_SPLIT && (e.nel <= 0 || d.M != 2 * e.nel || e.nmo < d.N))
    return record_error(SFQ_ERR_ARG, "umma_gemm: planar epilogue needs rows (c, a), 2 * nel of them");
  if (e.kind == UMMA_EPI_STORE_SPLIT || e.kind == UMMA_EPI_PLANAR_SPLIT || (e.kind == UMMA_EPI_TAYLOR && e.write)) {
    if (e.out_planes < 1 || e.out_planes > 3) return record_error(SFQ_ERR_ARG, "umma_gemm: output planes");
    for (int q = 0; q < e.out_planes; ++q)
      if (!e.out[q]) return record_error(SFQ_ERR_ARG, "umma_gemm: output plane %d missing", q);
  }
  if (e.kind == UMMA_EPI_TAYLOR) {
    const bool tile_ok = (BN % 32) == 0 && e.half * 2 == BN;  // two halves of whole 16-column chunks
    if (!tile_ok || !e.S || e.nmo <= 0)
      return record_error(SFQ_ERR_ARG, "umma_gemm: Taylor epilogue needs S and tile width 2 * half, half %% 16 == 0");
  }
  if (e.kind == UMMA_EPI_TO_WALKERS && (!e.SM || e.nel <= 0 || d.batch != 1 || d.M % (2 * e.nel)))
    return record_error(SFQ_ERR_ARG, "umma_gemm: walker epilogue needs rows (w, a, c) and one batch");
  if ((e.kind == UMMA_EPI_STORE || e.kind == UMMA_EPI_STORE_SPLIT) && !d.C)
    return record_error(SFQ_ERR_ARG, "umma_gemm: output missing");
  KParams kp;
  kp.M = d.M; kp.N = d.N; kp.K = d.K;
  kp.a_batched = d.A.batch_stride != 0; kp.b_batched = d.B.batch_stride != 0;
  kp.MT = (d.M + BM - 1) / BM;
  kp.NT = (d.N + BN - 1) / BN;
  const int KT = (d.K + BK - 1) / BK;
  kp.KS = d.ksplit < 1 ? 1 : (d.ksplit > KT ? KT : d.ksplit);
  if (kp.KS > 1 && (e.kind != UMMA_EPI_STORE || d.beta != 0.f || d.sCk <= 0))
    return record_error(SFQ_ERR_ARG, "umma_gemm: K splits write partial sums (plain store, beta = 0, sCk > 0)");
  kp.tiles = (long)kp.MT * kp.NT * d.batch * kp.KS;
  kp.batch = d.batch;
  kp.cb_half = cb ? d.cplx_half : 0;
  kp.cb_nmo = d.cplx_nmo;
  kp.cb_ldh = d.cplx_ldh;
  kp.cb_kth = cb ? d.cplx_ldh / BK : 0;
  if (cb && kp.KS != 1) return record_error(SFQ_ERR_ARG, "umma_gemm: complex B takes no K split");
  kp.C = d.C; kp.ldc = d.ldc; kp.sCb = d.sCb; kp.sCk = d.sCk; kp.alpha = d.alpha; kp.beta = d.beta;
  kp.e = e;
  kp.err = d.err;
  kp.wait_ns = d.wait_ns ? d.wait_ns : kWaitNs;
  if (JOINT && !cb) return record_error(SFQ_ERR_ARG, "umma_gemm: the joint layout is for complex B only");
  auto k = umma_gemm_kernel<BN, STAGES, NP, JOINT>;
  SFQ_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L::TOTAL));
  const long grid = kp.tiles < sm_count() ? kp.tiles : sm_count();
  k<<<unsigned(grid), kThreads, L::TOTAL, st>>>(maps, kp);
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
  // complex B with at most 2 planes and tiles up to 160 wide: the joint stage layout (both halves of
  // A against one load of [Vr; Vi]); two stages of it fit where three of the split layout did
  if (d.cplx_half > 0 && d.nplanes <= 2 && bn <= 160) {
    switch (d.nplanes * 1000 + bn) {
      case 1032: return umma::launch<32, 6, 1, true>(d, st);
      case 1064: return umma::launch<64, 5, 1, true>(d, st);
      case 1128: return umma::launch<128, 4, 1, true>(d, st);
      case 1160: return umma::launch<160, 4, 1, true>(d, st);
      case 2032: return umma::launch<32, 3, 2, true>(d, st);
      case 2064: return umma::launch<64, 2, 2, true>(d, st);
      case 2128: return umma::launch<128, 2, 2, true>(d, st);
      case 2160: return umma::launch<160, 2, 2, true>(d, st);
      default: break;
    }
  }
  switch (d.nplanes * 1000 + bn) {
    case 1032: return umma::launch<32, 8, 1>(d, st);
    case 1064: return umma::launch<64, 8, 1>(d, st);
    case 1128: return umma::launch<128, 6, 1>(d, st);
    case 1160: return umma::launch<160, 6, 1>(d, st);
    case 1208: return umma::launch<208, 4, 1>(d, st);
    case 1256: return umma::launch<256, 4, 1>(d, st);
    case 2032: return umma::launch<32, 5, 2>(d, st);
    case 2064: return umma::launch<64, 4, 2>(d, st);
    case 2128: return umma::launch<128, 3, 2>(d, st);
    case 2160: return umma::launch<160, 3, 2>(d, st);
    case 2208: return umma::launch<208, 2, 2>(d, st);
    case 2256: return umma::launch<256, 2, 2>(d, st);
    case 3032: return umma::launch<32, 3, 3>(d, st);
    case 3064: return umma::launch<64, 3, 3>(d, st);
    case 3128: return umma::launch<128, 2, 3>(d, st);
    case 3160: return umma::launch<160, 2, 3>(d, st);
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
