// Exact-accumulation int8-slice products on the tensor cores (see islice.cuh).
#include <cstddef>
#include <cstring>

#include "islice.cuh"
#include "tc_common.cuh"

namespace sfq {
namespace islice {
using namespace tc;

constexpr int BM = 128;                  // MMA M: accumulator rows = TMEM lanes
// int8 elements per K slice (BK, a template parameter): 64 (one 64-byte swizzle row) for products
// whose tiles run over short K ranges, 128 (one 128-byte swizzle row, half the stages) for long ones
constexpr int KSTEP = 32;                // K of one kind::i8 MMA
// warps: 0 TMA producer, 1 TMEM owner + MMA issuer, 2-9 epilogue (two per TMEM lane quarter, taking
// alternate 16-column chunks of the tile)
constexpr int kWarps = 10;
constexpr int kThreads = kWarps * 32;
constexpr int kEpiThreads = 256;
constexpr unsigned long long kWaitNs = 2000000000ull;  // limit of one wait: 2 s without progress

// slice pairs kept for NS slices, listed by group: g0 (0,0) | g1 (0,1) (1,0) | g2 (0,2) (1,1) (2,0)
__host__ __device__ constexpr int n_pairs(int ns) { return ns == 2 ? 3 : 6; }
__host__ __device__ constexpr int pair_a(int t) { return t == 0 ? 0 : t == 1 ? 0 : t == 2 ? 1 : t == 3 ? 0 : t == 4 ? 1 : 2; }
__host__ __device__ constexpr int pair_b(int t) { return t == 0 ? 0 : t == 1 ? 1 : t == 2 ? 0 : t == 3 ? 2 : t == 4 ? 1 : 0; }
__host__ __device__ constexpr int pair_g(int t) { return t == 0 ? 0 : t <= 2 ? 1 : 2; }
__host__ __device__ constexpr bool pair_first(int t) { return t == 0 || t == 1 || t == 3; }

// kind::i8: D = S32 (bits 4-5 = 2), A = B = signed 8-bit (bits 7-9, 10-12 = 1), both K-major, N, M = 128
__host__ __device__ constexpr uint32_t idesc_i8(uint32_t n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | (uint32_t(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2),
        "r"(mask3));
}

// K-major operand tile, BK-byte swizzle (64 or 128): rows of BK bytes (one K slice), 8-row groups
// 8 BK bytes apart
template <int BK>
__device__ __forceinline__ uint64_t smem_desc_k(const void* tile) {
  static_assert(BK == 64 || BK == 128, "K slice width");
  const uint64_t addr = su32(tile);
  uint64_t d = 0;
  d |= (addr & 0x3FFFFull) >> 4;                  // start address
  d |= uint64_t(1) << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= uint64_t((8 * BK) >> 4) << 32;             // stride byte offset: next 8-row group
  d |= uint64_t(1) << 46;                         // descriptor version (sm_100)
  d |= uint64_t(BK == 128 ? 2 : 4) << 61;         // SWIZZLE_128B or SWIZZLE_64B
  return d;
}

__host__ __device__ constexpr uint32_t pow2_ceil(uint32_t x) {
  return x <= 32 ? 32 : x <= 64 ? 64 : x <= 128 ? 128 : x <= 256 ? 256 : 512;
}

template <int BN, int STAGES, int NS, int BK>
struct Smem {
  static constexpr int A_BYTES = BM * BK;
  static constexpr int B_BYTES = BN * BK;
  static constexpr int STAGE = NS * (A_BYTES + B_BYTES);
  static constexpr int BAR_OFF = STAGES * STAGE;
  static constexpr int NBAR = 2 * STAGES + 5;  // full, empty, acc_full[2], acc_empty[2], done
  static constexpr int TOTAL = BAR_OFF + NBAR * 8 + 16 + 1024;
  static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "tiles must keep 1024-byte alignment");
};

struct Maps {
  CUtensorMap a[3], b[3], aim[3];
};

struct KParams {
  int M, N, K, batch;
  int a_batched, b_batched;
  int MT, NT, KS, KT;  // tiles along M, N; K splits; K slices (complex B: 2 per 128 orbitals)
  long tiles;
  int half;            // complex B: orbitals per tile (0: plain product)
  const int* ea; long ea_bs, ea_mod;
  const int* eb; long eb_bs, eb_mod;
  float* C;
  long ldc, sCb, sCc, sCk;
  double alpha;
  int accumulate;      // C += the product (one FP32 round to nearest) instead of C = the product
  int* err;
  unsigned long long wait_ns;
  const int* hold;
};

// a grouped launch: the products of several problems (the members of a group of systems) as one
// persistent tile list; problem i owns tiles [start[i], start[i+1]), its tensor maps and parameters
// in device memory (written before the launch)
struct alignas(128) GroupProb {
  Maps maps;
  KParams kp;
};
static_assert(sizeof(GroupProb) % 128 == 0 && offsetof(GroupProb, maps) == 0,
              "tensor maps in the table keep their 64-byte alignment");
struct GroupTab {
  const GroupProb* prob = nullptr;
  const long* start = nullptr;  // nprob + 1 tile offsets
  int nprob = 0;
  long tiles = 0;
};
__device__ __forceinline__ int find_prob(const GroupTab& g, long t) {
  int lo = 0, hi = g.nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (g.start[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
// the problem of tile t (global index) and its local tile index
template <bool GROUP>
__device__ __forceinline__ int locate(const GroupTab& g, long t, long& lt) {
  if (!GROUP) {
    lt = t;
    return 0;
  }
  const int pi = find_prob(g, t);
  lt = t - g.start[pi];
  return pi;
}
// a tensor map in device memory, written before the launch, is read by the tensor-map proxy
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(m))
               : "memory");
}

__device__ __forceinline__ void decode(const KParams& p, long t, int& mt, int& nt, int& bz, int& ks) {
  mt = int(t % p.MT);
  long r = t / p.MT;
  nt = int(r % p.NT);
  r /= p.NT;
  bz = int(r % p.batch);
  ks = int(r / p.batch);
}
// first K slice of split s of KS over KT slices of BK elements: the boundaries fall on multiples of
// 128 elements whatever BK, so a product's partial sums do not depend on the slice width
template <int BK>
__device__ __forceinline__ int k_begin(int KT, int KS, int s) {
  constexpr int per = 128 / BK;
  const int kt128 = (KT + per - 1) / per;
  const int b = int((long)kt128 * s / KS) * per;
  return b < KT ? b : KT;
}

__device__ __forceinline__ double pow2(int e) {
  e = e < -1022 ? -1022 : (e > 1023 ? 1023 : e);
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// tensor-memory loads of a chunk's groups issued back to back, then one wait; the wait names the
// registers so that nothing reads them before it
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld(uint32_t* r) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}

// first output column of the tile's chunk at accumulator column c (complex B: and its part, re or
// im); the same for the whole warp
template <int BN>
__device__ __forceinline__ int chunk_col0(const KParams& p, int nt, int c, int* part) {
  if (p.half) {  // complex B: [re | im] halves of `half` orbitals
    const int pt = c >= p.half ? 1 : 0;
    *part = pt;
    return nt * p.half + (c - pt * p.half);
  }
  *part = 0;
  return nt * BN + c;
}

// the 16-column chunks c0, c0 + 32, ... of one tile's accumulator groups at taddr (group g at column
// g * BN) -> FP32 output, row `row`
template <int BN, int NS>
__device__ __forceinline__ void epilogue_tile(const KParams& p, uint32_t taddr, int row, int mt, int nt, int bz,
                                              int ks, int c0) {
  const int gm = mt * BM + row;
  const bool live = gm < p.M;
  const int width = p.half ? 2 * p.half : BN;  // complex B: the [re | im] halves may be narrower than BN
  const int lane = threadIdx.x & 31;
  // the column exponents of all of this thread's chunks c0 + 32 j, loaded before the first one:
  // lanes 0-15 hold chunk 2m's 16 columns in eb2[m], lanes 16-31 chunk 2m + 1's
  constexpr int NPAIR = ((BN + 31) / 32 + 1) / 2;
  int eb2[NPAIR];
#pragma unroll
  for (int m = 0; m < NPAIR; ++m) {
    const int c = c0 + 32 * (2 * m + (lane >> 4));
    int e = 0;
    if (c < width) {
      int part;
      const int col0 = chunk_col0<BN>(p, nt, c, &part);
      if (col0 < p.N) {
        const int col = col0 + (lane & 15) < p.N ? col0 + (lane & 15) : p.N - 1;
        e = p.eb[(long)bz * p.eb_bs + (p.eb_mod ? col % p.eb_mod : col)];
      }
    }
    eb2[m] = e;
  }
  const int ea = live ? p.ea[(long)bz * p.ea_bs + (p.ea_mod ? gm % p.ea_mod : gm)] : 0;
#pragma unroll 1
  for (int j = 0;; ++j) {
    const int c = c0 + 32 * j;
    if (c >= width) break;
    uint32_t acc[3][16];
    __syncwarp();
#pragma unroll
    for (int g = 0; g < NS; ++g) tmem_ld16_nowait(taddr + uint32_t(g * BN + c), acc[g]);
#pragma unroll
    for (int g = 0; g < NS; ++g) tmem_wait_ld(acc[g]);
    int part;
    const int col0 = chunk_col0<BN>(p, nt, c, &part);
    if (col0 >= p.N) continue;
    const int valid = p.N - col0 < 16 ? p.N - col0 : 16;
    const long obase = p.half ? (long)part * p.sCc + ((long)bz * p.M + gm) * p.ldc + col0
                              : (long)ks * p.sCk + (long)bz * p.sCb + (long)gm * p.ldc + col0;
    // (col0 is the same for the whole warp; every lane takes part in the broadcast below, rows past
    // M included, whose results are dropped)
    int ebs = eb2[0];
#pragma unroll
    for (int m = 1; m < NPAIR; ++m)
      if ((j >> 1) == m) ebs = eb2[m];
    const int src = (j & 1) << 4;
    float v[16];
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
      const int eb = __shfl_sync(0xffffffffu, ebs, src + jj);
      // acc0 2^16 + acc1 2^8 + acc2: exact in int64 (< 2^48) and in its conversion to FP64 (< 2^53)
      long long sum = (long long)int(acc[0][jj]) << (8 * (NS - 1));
      if (NS > 1) sum += (long long)int(acc[1][jj]) << (8 * (NS - 2));
      if (NS > 2) sum += (long long)int(acc[2][jj]);
      v[jj] = __double2float_rn(double(sum) * pow2(ea + eb - 8 * (NS - 1)) * p.alpha);
    }
    if (!live) continue;
    float* out = p.C + obase;
    const bool vec = valid == 16 && (obase % 4) == 0;
    if (p.accumulate) {
#pragma unroll
      for (int jj = 0; jj < 16; ++jj)
        if (jj < valid) v[jj] = __fadd_rn(v[jj], out[jj]);
    }
    if (vec) {
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        reinterpret_cast<float4*>(out)[jj] = make_float4(v[4 * jj], v[4 * jj + 1], v[4 * jj + 2], v[4 * jj + 3]);
    } else {
#pragma unroll
      for (int jj = 0; jj < 16; ++jj)
        if (jj < valid) out[jj] = v[jj];
    }
  }
}

template <int BN, int STAGES, int NS, int BUFS, bool GROUP, int BK>
__global__ void __launch_bounds__(kThreads, 1) islice_gemm_kernel(const __grid_constant__ Maps maps0,
                                                                  const __grid_constant__ KParams p0,
                                                                  const __grid_constant__ GroupTab g) {
  using L = Smem<BN, STAGES, NS, BK>;
  constexpr uint32_t GCOLS = uint32_t(NS * BN);               // columns of one tile's groups
  constexpr uint32_t ALLOC = pow2_ceil(GCOLS * BUFS);
  constexpr int NP = n_pairs(NS);
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
  const long total = GROUP ? g.tiles : p0.tiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kEpiThreads);
    }
    mbar_init(done, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "r"(ALLOC));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const unsigned long long wait_ns = p0.wait_ns;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      uint32_t it = 0;
      bool stop = false;
      if (!GROUP && p0.hold) {  // start only once *hold is set (bounded like every wait)
        const unsigned long long t0 = gtimer();
        while (*reinterpret_cast<const volatile int*>(p0.hold) == 0) {
          if (gtimer() - t0 > wait_ns) {
            *s_abort = 1;
            stop = true;
            break;
          }
        }
      }
      int last_pi = -1;
      for (long t = blockIdx.x; t < total && !stop; t += gridDim.x) {
        long lt;
        const int pi = locate<GROUP>(g, t, lt);
        const KParams& p = GROUP ? g.prob[pi].kp : p0;
        const Maps& maps = GROUP ? g.prob[pi].maps : maps0;
        const bool cb = p.half > 0;
        if (GROUP && pi != last_pi) {
#pragma unroll
          for (int q = 0; q < NS; ++q) {
            tensormap_acquire(&maps.a[q]);
            tensormap_acquire(&maps.b[q]);
            if (cb) tensormap_acquire(&maps.aim[q]);
          }
          last_pi = pi;
        }
        // bytes of one stage: complex B loads two half-tiles of `half` rows of B
        const uint32_t stage_bytes = cb ? uint32_t(NS * (L::A_BYTES + 2 * p.half * BK)) : uint32_t(L::STAGE);
        int mt, nt, bz, ks;
        decode(p, lt, mt, nt, bz, ks);
        const int m0 = mt * BM;
        const int ab = p.a_batched ? bz : 0, bb = p.b_batched ? bz : 0;
        const int kb = k_begin<BK>(p.KT, p.KS, ks), ke = k_begin<BK>(p.KT, p.KS, ks + 1);
        for (int kt = kb; kt < ke; ++kt, ++it) {
          const int s = int(it % STAGES);
          const uint32_t ph = (it / STAGES) & 1;
          if (!mbar_wait_for(&empty[s], ph ^ 1, wait_ns) || *s_abort) {
            *s_abort = 1;
            stop = true;
            break;
          }
          unsigned char* stg = smem + s * L::STAGE;
          mbar_expect_tx(&full[s], stage_bytes);
          if (cb) {
            // part 0: A_re with the rows [Vr; Vi] of the tile's orbitals; part 1: A_im with [-Vi; Vr]
            const int part = kt & 1, k0 = (kt >> 1) * BK, i0 = nt * p.half;
#pragma unroll
            for (int q = 0; q < NS; ++q) {
              unsigned char* at = stg + q * L::A_BYTES;
              unsigned char* bt = stg + NS * L::A_BYTES + q * L::B_BYTES;
              tma_load_3d(at, part == 0 ? &maps.a[q] : &maps.aim[q], &full[s], k0, m0, ab);
              tma_load_3d(bt, &maps.b[q], &full[s], k0, (part == 0 ? 0 : 2 * p.N) + i0, bb);
              tma_load_3d(bt + p.half * BK, &maps.b[q], &full[s], k0, (part == 0 ? p.N : 0) + i0, bb);
            }
          } else {
            const int k0 = kt * BK, n0 = nt * BN;
#pragma unroll
            for (int q = 0; q < NS; ++q) {
              tma_load_3d(stg + q * L::A_BYTES, &maps.a[q], &full[s], k0, m0, ab);
              tma_load_3d(stg + NS * L::A_BYTES + q * L::B_BYTES, &maps.b[q], &full[s], k0, n0, bb);
            }
          }
        }
      }
      // every issued stage must have landed before the CTA may exit
      for (uint32_t j = (it > uint32_t(STAGES) ? it - STAGES : 0u); j < it; ++j)
        mbar_wait_for(&full[j % STAGES], (j / STAGES) & 1, kWaitNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      uint32_t it = 0;
      int lt_n = 0;
      bool stop = false;
      for (long t = blockIdx.x; t < total && !stop; t += gridDim.x, ++lt_n) {
        const int b = BUFS == 2 ? (lt_n & 1) : 0;
        const uint32_t aph = BUFS == 2 ? ((uint32_t(lt_n) >> 1) & 1) : (uint32_t(lt_n) & 1);
        if (*s_abort || !mbar_wait_for(&acc_empty[b], aph ^ 1, wait_ns)) {
          *s_abort = 1;
          break;
        }
        fence_after();
        const uint32_t d_tmem = tmem + uint32_t(b) * GCOLS;
        long lt;
        const int pi = locate<GROUP>(g, t, lt);
        const KParams& p = GROUP ? g.prob[pi].kp : p0;
        const bool cb = p.half > 0;
        const int Kv = cb ? p.N : p.K;  // valid K elements (complex B: the orbitals)
        int mt, nt, bz, ks;
        decode(p, lt, mt, nt, bz, ks);
        const int kb = k_begin<BK>(p.KT, p.KS, ks), ke = k_begin<BK>(p.KT, p.KS, ks + 1);
        const uint32_t idesc = idesc_i8(uint32_t(cb ? 2 * p.half : BN));
        for (int kt = kb; kt < ke; ++kt, ++it) {
          const int s = int(it % STAGES);
          const uint32_t ph = (it / STAGES) & 1;
          if (*s_abort || !mbar_wait_for(&full[s], ph, wait_ns)) {
            *s_abort = 1;
            stop = true;
            break;
          }
          fence_after();
          unsigned char* stg = smem + s * L::STAGE;
          uint64_t ad[NS], bd[NS];
#pragma unroll
          for (int q = 0; q < NS; ++q) {
            ad[q] = smem_desc_k<BK>(stg + q * L::A_BYTES);
            bd[q] = smem_desc_k<BK>(stg + NS * L::A_BYTES + q * L::B_BYTES);
          }
          const int k0 = cb ? (kt >> 1) * BK : kt * BK;
          const int rem = Kv - k0;
          const int nk = rem >= BK ? BK / KSTEP : (rem + KSTEP - 1) / KSTEP;  // K tail: skip all-zero steps
          const bool first_slice = kt == kb;  // complex B: part 0 of the first K block initialises
          for (int kk = 0; kk < nk; ++kk) {
            const uint64_t off = uint64_t(kk * KSTEP) >> 4;  // 32 bytes along the swizzled row
#pragma unroll
            for (int t2 = 0; t2 < NP; ++t2) {
              const uint32_t accum = (first_slice && kk == 0 && pair_first(t2)) ? 0u : 1u;
              umma_i8(d_tmem + uint32_t(pair_g(t2) * BN), ad[pair_a(t2)] + off, bd[pair_b(t2)] + off, idesc, accum);
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
  } else {  // epilogue warps 2..9 -> TMEM lane quarters 2,3,0,1 (a warp reaches only its quarter)
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const int c0 = 16 * ((warp - 2) >> 2);  // the two warps of a quarter take alternate 16-column chunks
    int lt_n = 0;
    for (long t = blockIdx.x; t < total; t += gridDim.x, ++lt_n) {
      const int b = BUFS == 2 ? (lt_n & 1) : 0;
      const uint32_t aph = BUFS == 2 ? ((uint32_t(lt_n) >> 1) & 1) : (uint32_t(lt_n) & 1);
      const bool ok = mbar_wait_for(&acc_full[b], aph, wait_ns);
      const bool go = __all_sync(0xffffffffu, ok) && !__any_sync(0xffffffffu, *s_abort != 0);
      if (!go) {
        *s_abort = 1;
        break;
      }
      fence_after();
      long lt;
      const int pi = locate<GROUP>(g, t, lt);
      const KParams& p = GROUP ? g.prob[pi].kp : p0;
      int mt, nt, bz, ks;
      decode(p, lt, mt, nt, bz, ks);
      epilogue_tile<BN, NS>(p, tmem + (uint32_t(q * 32) << 16) + uint32_t(b) * GCOLS, row, mt, nt, bz, ks, c0);
      fence_before();
      mbar_arrive(&acc_empty[b]);
    }
  }
  fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && *s_abort) {
    if (GROUP) {
      for (int i = 0; i < g.nprob; ++i)
        if (g.prob[i].kp.err) atomicExch(g.prob[i].kp.err, SFQ_ERR_TIMEOUT);
    } else if (p0.err) {
      atomicExch(p0.err, SFQ_ERR_TIMEOUT);
    }
  }
  if (warp == 1) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ALLOC));
  }
}

// ---- host side -------------------------------------------------------------------------------
int make_map_i8(CUtensorMap* m, const void* base, long rows, long K, long ld, long batch, long bstride, int box_rows,
                int bk) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return record_error(SFQ_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 16) || ld < K)
    return record_error(SFQ_ERR_SHAPE, "islice_gemm: slices need 16-byte alignment and a row stride >= K, a multiple of 16");
  if (batch <= 1) {
    batch = 1;
    bstride = (rows * ld + 15) / 16 * 16;
  } else if (bstride % 16) {
    return record_error(SFQ_ERR_SHAPE, "islice_gemm: batch stride must be a multiple of 16 bytes");
  }
  cuuint64_t dims[3] = {cuuint64_t(K), cuuint64_t(rows), cuuint64_t(batch)};
  cuuint64_t strides[2] = {cuuint64_t(ld), cuuint64_t(bstride)};
  cuuint32_t box[3] = {cuuint32_t(bk), cuuint32_t(box_rows), 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, bk == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return record_error(SFQ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", int(r));
  return SFQ_OK;
}

// the tensor maps and kernel parameters of one product; `group`: a member of a grouped launch of
// tile width BN, whose complex-B products may use narrower halves
template <int BN, int STAGES, int NS, int BK>
int prepare(const IsliceGemmDesc& d, Maps* maps, KParams* kp_out, bool group) {
  const bool cb = d.cplx_half > 0;
  int rc;
  const long ab = d.A.batch_stride ? d.batch : 1, bb = d.B.batch_stride ? d.batch : 1;
  for (int q = 0; q < NS; ++q) {
    if (!d.A.q[q] || !d.B.q[q]) return record_error(SFQ_ERR_ARG, "islice_gemm: slice %d missing", q);
    if ((rc = make_map_i8(&maps->a[q], d.A.q[q], d.A.rows, d.K, d.A.ld, ab, d.A.batch_stride, BM, BK))) return rc;
    if ((rc = make_map_i8(&maps->b[q], d.B.q[q], d.B.rows, d.K, d.B.ld, bb, d.B.batch_stride, cb ? d.cplx_half : BN,
                           BK)))
      return rc;
    if (cb) {
      if (!d.a_im[q]) return record_error(SFQ_ERR_ARG, "islice_gemm: complex B needs a_im");
      if ((rc = make_map_i8(&maps->aim[q], d.a_im[q], d.A.rows, d.K, d.A.ld, ab, d.A.batch_stride, BM, BK))) return rc;
    } else {
      maps->aim[q] = maps->a[q];
    }
  }
  for (int q = NS; q < 3; ++q) {
    maps->a[q] = maps->a[0];
    maps->b[q] = maps->b[0];
    maps->aim[q] = maps->aim[0];
  }
  if (!d.A.e || !d.B.e || !d.C) return record_error(SFQ_ERR_ARG, "islice_gemm: exponents and output required");
  KParams& kp = *kp_out;
  kp = KParams{};
  kp.M = d.M; kp.N = d.N; kp.K = d.K; kp.batch = d.batch;
  kp.a_batched = d.A.batch_stride != 0; kp.b_batched = d.B.batch_stride != 0;
  kp.MT = (d.M + BM - 1) / BM;
  if (cb) {
    const bool width_ok = group ? d.cplx_half * 2 <= BN : d.cplx_half * 2 == BN;
    if (!width_ok || d.cplx_half % 16 || d.K != d.N || d.B.rows != 3L * d.N || d.ksplit > 1)
      return record_error(SFQ_ERR_ARG, "islice_gemm: complex B needs BN = 2 half (a grouped launch: <=), half %% 16 "
                                       "== 0, K = N = nmo, B rows = 3 nmo and no K split");
    kp.NT = (d.N + d.cplx_half - 1) / d.cplx_half;
    kp.KT = 2 * ((d.K + BK - 1) / BK);
    kp.KS = 1;
  } else {
    kp.NT = (d.N + BN - 1) / BN;
    kp.KT = (d.K + BK - 1) / BK;
    const int kt128 = (d.K + 127) / 128;  // split boundaries fall on multiples of 128 elements
    kp.KS = d.ksplit < 1 ? 1 : (d.ksplit > kt128 ? kt128 : d.ksplit);
    if (kp.KS > 1 && d.sCk <= 0) return record_error(SFQ_ERR_ARG, "islice_gemm: K splits need a partial-sum stride");
  }
  // int32 exactness: a group sums at most 3 pairs of |q| <= 128 products over one K range (complex
  // B: each output sums both halves, 2 nmo terms)
  const long krange = cb ? 2L * d.K : (long)(((d.K + 127) / 128 + kp.KS - 1) / kp.KS) * 128;
  if (krange > 43000)
    return record_error(SFQ_ERR_SHAPE, "islice_gemm: K range of %ld too long for exact int32 accumulation", krange);
  kp.tiles = (long)kp.MT * kp.NT * d.batch * kp.KS;
  kp.half = cb ? d.cplx_half : 0;
  kp.ea = d.A.e; kp.ea_bs = d.A.e_bs; kp.ea_mod = d.A.e_mod;
  kp.eb = d.B.e; kp.eb_bs = d.B.e_bs; kp.eb_mod = cb ? 0 : d.B.e_mod;  // complex B: indexed by orbital
  kp.C = d.C; kp.ldc = d.ldc; kp.sCb = d.sCb; kp.sCc = d.sCc; kp.sCk = d.sCk;
  kp.alpha = d.alpha;
  kp.accumulate = d.accumulate ? 1 : 0;
  kp.err = d.err;
  kp.wait_ns = d.wait_ns ? d.wait_ns : kWaitNs;
  kp.hold = group ? nullptr : d.hold;
  return SFQ_OK;
}

template <int BN, int STAGES, int NS, int BK>
struct Config {
  using L = Smem<BN, STAGES, NS, BK>;
  static_assert(BN % 16 == 0, "the epilogue drains whole 16-column chunks");
  static constexpr int BUFS = (2 * NS * BN <= 512) ? 2 : 1;
  static_assert(L::TOTAL <= 232448, "shared memory budget");
  static_assert(NS * BN * BUFS <= 512, "accumulator groups must fit in tensor memory");
};

template <int BN, int STAGES, int NS, int BK>
int launch(const IsliceGemmDesc& d, cudaStream_t st) {
  using C = Config<BN, STAGES, NS, BK>;
  Maps maps;
  KParams kp;
  int rc;
  if ((rc = prepare<BN, STAGES, NS, BK>(d, &maps, &kp, false))) return rc;
  auto k = islice_gemm_kernel<BN, STAGES, NS, C::BUFS, false, BK>;
  SFQ_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, C::L::TOTAL));
  const long grid = kp.tiles < sm_count() ? kp.tiles : sm_count();
  k<<<unsigned(grid), kThreads, C::L::TOTAL, st>>>(maps, kp, GroupTab{});
  SFQ_LAUNCHED();
  return SFQ_OK;
}

// the grouped launches' tile widths: every plain product of a group has tile width kGroupBN
constexpr int kGroupBN = 160;
constexpr int group_stages(int ns, int bk) { return (ns == 2 ? 6 : 4) * 64 / bk; }

template <int NS, int BK>
int group_plan(const IsliceGemmDesc* ds, int n, IsliceGroupPlan* out) {
  constexpr int ST = group_stages(NS, BK);
  std::vector<GroupProb> probs(static_cast<size_t>(n));
  std::vector<long> start(size_t(n) + 1, 0);
  int rc;
  for (int i = 0; i < n; ++i) {
    const IsliceGemmDesc& d = ds[i];
    if (d.nslices != NS) return record_error(SFQ_ERR_ARG, "islice_gemm_group: members differ in slices");
    if (d.cplx_half == 0 && d.bn != kGroupBN)
      return record_error(SFQ_ERR_ARG, "islice_gemm_group: plain products need tile width %d", kGroupBN);
    if (d.hold) return record_error(SFQ_ERR_ARG, "islice_gemm_group: no held launches");
    if (d.M <= 0 || d.N <= 0 || d.batch <= 0 || d.K <= 0)
      return record_error(SFQ_ERR_SHAPE, "islice_gemm_group: empty member %d", i);
    GroupProb* pr = probs.data() + i;
    Maps* mp = &pr->maps;
    KParams* kq = &pr->kp;
    rc = prepare<kGroupBN, ST, NS, BK>(d, mp, kq, true);
    if (rc) return rc;
    start[size_t(i) + 1] = start[size_t(i)] + kq->tiles;
  }
  out->nprob = n;
  out->nslices = NS;
  out->bk = BK;
  out->tiles = start[size_t(n)];
  out->wait_ns = n ? probs[0].kp.wait_ns : kWaitNs;
  out->start_off = sizeof(GroupProb) * size_t(n);
  out->image.assign(out->start_off + sizeof(long) * (size_t(n) + 1), 0);
  std::memcpy(out->image.data(), probs.data(), out->start_off);
  std::memcpy(out->image.data() + out->start_off, start.data(), sizeof(long) * (size_t(n) + 1));
  return SFQ_OK;
}

template <int NS, int BK>
int group_launch(const void* table, const IsliceGroupPlan& plan, cudaStream_t st) {
  constexpr int ST = group_stages(NS, BK);
  using C = Config<kGroupBN, ST, NS, BK>;
  if (reinterpret_cast<uintptr_t>(table) & 127)
    return record_error(SFQ_ERR_ARG, "islice_gemm_group: the table needs 128-byte alignment");
  GroupTab g;
  g.prob = static_cast<const GroupProb*>(table);
  g.start = reinterpret_cast<const long*>(static_cast<const char*>(table) + plan.start_off);
  g.nprob = plan.nprob;
  g.tiles = plan.tiles;
  KParams kp{};
  kp.wait_ns = plan.wait_ns;
  auto k = islice_gemm_kernel<kGroupBN, ST, NS, C::BUFS, true, BK>;
  SFQ_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, C::L::TOTAL));
  const long grid = plan.tiles < sm_count() ? plan.tiles : sm_count();
  k<<<unsigned(grid), kThreads, C::L::TOTAL, st>>>(Maps{}, kp, g);
  SFQ_LAUNCHED();
  return SFQ_OK;
}

// the K slice width for a product: 128 elements where its tiles run over 1024 or more K elements
// (half as many stages, each twice as long), else 64
inline int k_slice_width(const IsliceGemmDesc& d) {
  const long k = d.cplx_half > 0 ? 2L * d.K : (d.K + (d.ksplit > 1 ? d.ksplit : 1) - 1) / (d.ksplit > 1 ? d.ksplit : 1);
  return k >= 1024 ? 128 : 64;
}

}  // namespace islice

int islice_gemm(const IsliceGemmDesc& d, cudaStream_t st) {
  if (d.M <= 0 || d.N <= 0 || d.batch <= 0) return SFQ_OK;
  if (d.K <= 0) return record_error(SFQ_ERR_SHAPE, "islice_gemm: K must be positive");
  const int bn = d.cplx_half > 0 ? 2 * d.cplx_half : (d.bn ? d.bn : (d.N <= 64 ? 64 : 128));
  const bool k128 = islice::k_slice_width(d) == 128;
  // stages: as many as about 216 KB of shared memory holds
  switch (d.nslices * 1000 + bn) {
    case 2064: return k128 ? islice::launch<64, 4, 2, 128>(d, st) : islice::launch<64, 8, 2, 64>(d, st);
    case 2128: return k128 ? islice::launch<128, 3, 2, 128>(d, st) : islice::launch<128, 6, 2, 64>(d, st);
    case 2160: return k128 ? islice::launch<160, 3, 2, 128>(d, st) : islice::launch<160, 6, 2, 64>(d, st);
    case 3064: return k128 ? islice::launch<64, 3, 3, 128>(d, st) : islice::launch<64, 6, 3, 64>(d, st);
    case 3080: return k128 ? islice::launch<80, 2, 3, 128>(d, st) : islice::launch<80, 5, 3, 64>(d, st);
    case 3128: return k128 ? islice::launch<128, 2, 3, 128>(d, st) : islice::launch<128, 4, 3, 64>(d, st);
    case 3160: return k128 ? islice::launch<160, 2, 3, 128>(d, st) : islice::launch<160, 4, 3, 64>(d, st);
    default:
      return record_error(SFQ_ERR_ARG, "islice_gemm: %d slices with tile width %d not built", d.nslices, bn);
  }
}

int islice_gemm_group_plan(const IsliceGemmDesc* ds, int n, IsliceGroupPlan* out) {
  if (n <= 0 || !ds || !out) return record_error(SFQ_ERR_ARG, "islice_gemm_group: no members");
  // one K slice width for the launch: the widest any member would take alone (the results do not
  // depend on it)
  bool k128 = false;
  for (int i = 0; i < n; ++i) k128 = k128 || islice::k_slice_width(ds[i]) == 128;
  if (ds[0].nslices == 2) return k128 ? islice::group_plan<2, 128>(ds, n, out) : islice::group_plan<2, 64>(ds, n, out);
  if (ds[0].nslices == 3) return k128 ? islice::group_plan<3, 128>(ds, n, out) : islice::group_plan<3, 64>(ds, n, out);
  return record_error(SFQ_ERR_ARG, "islice_gemm_group: %d slices not built", ds[0].nslices);
}

int islice_gemm_group_launch(const void* table, const IsliceGroupPlan& plan, cudaStream_t st) {
  if (plan.nprob <= 0 || plan.tiles <= 0) return SFQ_OK;
  const bool k128 = plan.bk == 128;
  if (plan.nslices == 2)
    return k128 ? islice::group_launch<2, 128>(table, plan, st) : islice::group_launch<2, 64>(table, plan, st);
  if (plan.nslices == 3)
    return k128 ? islice::group_launch<3, 128>(table, plan, st) : islice::group_launch<3, 64>(table, plan, st);
  return record_error(SFQ_ERR_ARG, "islice_gemm_group: %d slices not built", plan.nslices);
}

}  // namespace sfq

// ---- C ABI: the int8-slice products on caller operands (tests and benchmarks) ---------------
namespace sfq {
namespace {
template <typename T>
__global__ void cplx_to_planar_f32_kernel(const cplx* src, long n, T* re, T* im) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    re[t] = T(float(src[t].x));
    im[t] = T(float(src[t].y));
  }
}
}  // namespace
}  // namespace sfq

extern "C" {

int sfq_gemm_int8_slices(const double* A, const double* B, float* C, int M, int N, int K, int nslices, int tile_n,
                         int ksplit, void* stream) {
  using namespace sfq;
  if (nslices < 2 || nslices > 3) return record_error(SFQ_ERR_ARG, "nslices must be 2 or 3");
  if (M <= 0 || N <= 0 || K <= 0) return record_error(SFQ_ERR_SHAPE, "gemm_int8_slices: empty product");
  if (tile_n != 0 && tile_n != 64 && tile_n != 80 && tile_n != 128 && tile_n != 160)
    return record_error(SFQ_ERR_ARG, "gemm_int8_slices: tile width %d not built", tile_n);
  if (!A || !B || !C) return record_error(SFQ_ERR_ARG, "gemm_int8_slices: null operand");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long ld = (K + 63) / 64 * 64;  // slice rows on 64-byte boundaries, as the engine lays them out
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t qa = al((size_t)M * ld), qb = al((size_t)N * ld), ea = al(sizeof(int) * M), eb = al(sizeof(int) * N);
  const int ks = ksplit < 1 ? 1 : ksplit;
  const size_t cpart = al(sizeof(float) * (size_t)M * N);
  char* buf = nullptr;
  SFQ_CUDA_TRY(cudaMallocAsync((void**)&buf, nslices * (qa + qb) + ea + eb + (ks > 1 ? ks * cpart : 0), st));
  int8_t *aq[3] = {}, *bq[3] = {};
  for (int s = 0; s < nslices; ++s) {
    aq[s] = reinterpret_cast<int8_t*>(buf + s * qa);
    bq[s] = reinterpret_cast<int8_t*>(buf + nslices * qa + s * qb);
  }
  int* eA = reinterpret_cast<int*>(buf + nslices * (qa + qb));
  int* eB = reinterpret_cast<int*>(buf + nslices * (qa + qb) + ea);
  float* part = ks > 1 ? reinterpret_cast<float*>(buf + nslices * (qa + qb) + ea + eb) : nullptr;
  int rc = islice_rows_real(A, M, K, K, nslices, aq, ld, eA, st);
  if (!rc) rc = islice_rows_real(B, N, K, K, nslices, bq, ld, eB, st);
  if (!rc) {
    IsliceGemmDesc d;
    d.M = M; d.N = N; d.K = K; d.nslices = nslices; d.bn = tile_n; d.ksplit = ks;
    for (int s = 0; s < 3; ++s) {
      d.A.q[s] = aq[s];
      d.B.q[s] = bq[s];
    }
    d.A.rows = M; d.A.ld = ld; d.A.e = eA;
    d.B.rows = N; d.B.ld = ld; d.B.e = eB;
    d.C = ks > 1 ? part : C; d.ldc = N; d.sCk = (long)cpart / sizeof(float);
    rc = islice_gemm(d, st);
  }
  if (!rc && ks > 1) {  // the K ranges' partial products, written at C + s * M * N
    for (int s = 0; s < ks && !rc; ++s) {
      const cudaError_t ce = cudaMemcpyAsync(C + (size_t)s * M * N, reinterpret_cast<char*>(part) + s * cpart,
                                             sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToDevice, st);
      if (ce != cudaSuccess) rc = record_cuda(ce, "cudaMemcpyAsync", __FILE__, __LINE__);
    }
  }
  cudaFreeAsync(buf, st);
  return rc;
}

int sfq_selftest_wait_expiry(unsigned long long wait_ns, void* stream) {
  using namespace sfq;
  if (wait_ns == 0 || wait_ns > 1000000000ull) return record_error(SFQ_ERR_ARG, "selftest: wait of 1 ns .. 1 s");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  constexpr int n = 128;
  const size_t qb = (size_t)n * n, ebytes = sizeof(int) * n;
  char* buf = nullptr;
  const size_t total = 6 * qb + 2 * ebytes + sizeof(float) * n * n + 256;
  SFQ_CUDA_TRY(cudaMallocAsync((void**)&buf, total, st));
  SFQ_CUDA_TRY(cudaMemsetAsync(buf, 0, total, st));
  IsliceGemmDesc d;
  d.M = n; d.N = n; d.K = n; d.nslices = 3; d.bn = 128;
  for (int q = 0; q < 3; ++q) {
    d.A.q[q] = reinterpret_cast<int8_t*>(buf + q * qb);
    d.B.q[q] = reinterpret_cast<int8_t*>(buf + (3 + q) * qb);
  }
  d.A.rows = n; d.A.ld = n; d.A.e = reinterpret_cast<int*>(buf + 6 * qb);
  d.B.rows = n; d.B.ld = n; d.B.e = reinterpret_cast<int*>(buf + 6 * qb + ebytes);
  d.C = reinterpret_cast<float*>(buf + 6 * qb + 2 * ebytes);
  d.ldc = n;
  int* flags = reinterpret_cast<int*>(buf + total - 256);  // [0] the kernel's status, [1] the hold flag (0)
  d.err = flags;
  d.hold = flags + 1;
  d.wait_ns = wait_ns;
  int rc = islice_gemm(d, st);
  int status = SFQ_OK;
  if (!rc) {
    cudaError_t ce = cudaMemcpyAsync(&status, flags, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = record_cuda(ce, "selftest", __FILE__, __LINE__);
  }
  cudaFreeAsync(buf, st);
  return rc ? rc : status;
}

int sfq_gemm_int8_cplx_b(const void* A, const void* V, float* C, int W, int M, int N, int nslices, int half,
                         void* stream) {
  using namespace sfq;
  if (nslices < 2 || nslices > 3) return record_error(SFQ_ERR_ARG, "nslices must be 2 or 3");
  if (W <= 0 || M <= 0 || N <= 0) return record_error(SFQ_ERR_SHAPE, "gemm_int8_cplx_b: empty product");
  if (half != 32 && half != 64 && half != 80)
    return record_error(SFQ_ERR_ARG, "gemm_int8_cplx_b: %d orbitals per tile not built", half);
  if (!A || !V || !C) return record_error(SFQ_ERR_ARG, "gemm_int8_cplx_b: null operand");
  if (M > 1024) return record_error(SFQ_ERR_SHAPE, "gemm_int8_cplx_b: M=%d above 1024", M);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long ld = (M + 63) / 64 * 64, R = (long)W * N, MM = (long)M * M;  // 64-byte slice rows, as in the engine
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t sa = al(sizeof(float) * 2 * R * M), sz = al(sizeof(float) * 2 * R * M),
               sv = al(sizeof(float) * 2 * W * MM);
  const size_t qa = al((size_t)2 * R * ld), qv = al((size_t)W * 3 * M * ld);
  const size_t ea = al(sizeof(int) * R), ev = al(sizeof(int) * W * M);
  char* buf = nullptr;
  SFQ_CUDA_TRY(cudaMallocAsync((void**)&buf, sa + sz + sv + nslices * (qa + qv) + ea + 2 * ev, st));
  char* o = buf;
  float* S = reinterpret_cast<float*>(o); o += sa;
  float* Cz = reinterpret_cast<float*>(o); o += sz;
  float* Cv = reinterpret_cast<float*>(o); o += sv;
  int8_t *aq[3] = {}, *vq[3] = {};
  for (int s = 0; s < nslices; ++s) {
    aq[s] = reinterpret_cast<int8_t*>(o); o += qa;
    vq[s] = reinterpret_cast<int8_t*>(o); o += qv;
  }
  int* eA = reinterpret_cast<int*>(o); o += ea;
  int* eV = reinterpret_cast<int*>(o); o += ev;
  int* eVmax = reinterpret_cast<int*>(o);
  // A through FP32 as the planar rows (c, w, a) of a sum S (plus a zero product); V[w][j][i] as the
  // planar rows (c * W + w, j * M + i) of a full vHS
  cplx_to_planar_f32_kernel<<<148 * 8, 256, 0, st>>>(static_cast<const cplx*>(A), R * M, S, S + R * M);
  SFQ_LAUNCHED();
  SFQ_CUDA_TRY(cudaMemsetAsync(Cz, 0, sz, st));
  for (int w = 0; w < W; ++w) {
    cplx_to_planar_f32_kernel<<<148, 256, 0, st>>>(static_cast<const cplx*>(V) + w * MM, MM, Cv + w * MM,
                                                   Cv + (W + w) * MM);
    SFQ_LAUNCHED();
  }
  int rc = islice_taylor_update(Cz, S, R, M, 0, true, nslices, aq, ld, eA, st);
  if (!rc) rc = islice_build_v(Cv, W, M, false, nslices, vq, ld, eV, eVmax, st);
  if (!rc) {
    IsliceGemmDesc d;
    d.M = N; d.N = M; d.K = M; d.batch = W; d.nslices = nslices;
    for (int s = 0; s < 3; ++s) {
      d.A.q[s] = aq[s];
      d.a_im[s] = aq[s] ? aq[s] + R * ld : nullptr;
      d.B.q[s] = vq[s];
    }
    d.A.rows = N; d.A.ld = ld; d.A.batch_stride = (long)N * ld; d.A.e = eA; d.A.e_bs = N;
    d.B.rows = 3L * M; d.B.ld = ld; d.B.batch_stride = 3L * M * ld; d.B.e = eV; d.B.e_bs = M;
    d.cplx_half = half;
    d.C = C; d.ldc = M; d.sCc = R * M;
    rc = islice_gemm(d, st);
  }
  cudaFreeAsync(buf, st);
  return rc;
}

}  // extern "C"
