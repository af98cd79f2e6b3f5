// Mixed density matrix without any device allocation by the library or the caller.
//
// sfq_mixed_density_matrix needs a caller-provided workspace for the per-walker overlap
// matrices T = PsiT * W (nwalk * nel * nel complex).  Some callers cannot provide one: a host
// program whose allocator already owns every byte of device memory and hands out no extra
// buffers, a binding layer (an FFI from another language) that has no CUDA runtime of its own
// and so cannot size, allocate or free device memory, or a latency-bound loop that must not pay
// for cudaMalloc, which can synchronise the whole device.  This entry point serves them: the
// scratch lives in a fixed array compiled into the library, so neither side allocates.
//
// Limits and sharing rules (also stated next to the declaration in safire_b200.h):
//  * the array holds kNoAllocScratchBytes (16 MiB) on every GPU that loads the library, for the
//    life of the process; calls needing more (nwalk * nel * nel * 16 bytes) are rejected;
//  * every call on a device uses the same array and leaves its contents behind; nothing in it
//    has to start at zero, because the overlap GEMM overwrites the whole region it uses;
//  * two calls whose work overlaps on the GPU (different streams, or threads issuing at the same
//    time) race on the array: serialise them;
//  * the first call in each CUDA context looks up the array's device address
//    (cudaGetSymbolAddress with that device current); make that first call before any stream
//    capture.  The address is kept per device together with the context's unique id
//    (cuCtxGetId), so a context created anew on the device (after cudaDeviceReset, or after
//    the primary context was released) makes the next call look the address up again instead
//    of writing through one from the old context.
#include <mutex>

#include "ops.cuh"

namespace sfq {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

// Only device code may use this name as an address; host code uses the pointer looked up below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points (no link to libcuda).
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);

template <class Fn>
Fn driver_fn(const char* name) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<Fn>(p);
}

// Unique id of the calling thread's current context; 0 when there is none or the driver has no
// cuCtxGetId (the address is then looked up on every call).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    get_current = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
    get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
  });
  if (!get_current || !get_id) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

// Device address of g_noalloc_scratch in the current context, looked up once per context.
int scratch_address(void** out) {
  int dev = 0;
  SFQ_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return record_error(SFQ_ERR_UNSUPPORTED, "no-alloc scratch: device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  const unsigned long long ctx = current_context_id();
  if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return record_cuda(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    if (!p) return record_error(SFQ_ERR_INTERNAL, "no-alloc scratch: null device address");
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = current_context_id();  // the lookup made the primary context current
  }
  *out = g_scratch_addr[dev];
  return SFQ_OK;
}

}  // namespace
}  // namespace sfq

using namespace sfq;

extern "C" {

size_t sfq_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

int sfq_mixed_density_matrix_noalloc(const void* A, int a_complex, const void* B, void* C, void* ovlp, int nwalk,
                                     int nmo, int nel, void* stream) {
  if (nwalk < 0 || nmo < 0 || nel < 0) return record_error(SFQ_ERR_SHAPE, "negative size");
  if (nwalk == 0 || nel == 0) return SFQ_OK;
  if (!A || !B || !C || !ovlp) return record_error(SFQ_ERR_ARG, "null pointer");
  if (nel > kMaxSmallN) return record_error(SFQ_ERR_UNSUPPORTED, "nel=%d exceeds %d", nel, kMaxSmallN);
  const size_t need = sizeof(cplx) * (size_t)nwalk * nel * nel;
  if (need > kNoAllocScratchBytes)
    return record_error(SFQ_ERR_WORKSPACE,
                        "mixed_density_matrix_noalloc: nwalk*nel*nel*16 = %zu bytes exceeds the fixed %zu-byte "
                        "scratch; split the walkers into batches or use sfq_mixed_density_matrix",
                        need, kNoAllocScratchBytes);
  void* scratch = nullptr;
  int rc;
  if ((rc = scratch_address(&scratch))) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cplx* T = reinterpret_cast<cplx*>(scratch);
  if ((rc = ops::overlap_matrix(A, a_complex != 0, (const cplx*)B, T, nwalk, nmo, nel, st))) return rc;
  if ((rc = lu_logdet(T, (long)nel * nel, nwalk, nel, (cplx*)ovlp, true, 1.0, true, st))) return rc;
  return ops::green_compact(T, (const cplx*)B, (cplx*)C, nwalk, nmo, nel, st);
}

}  // extern "C"
