// Shared device/host helpers for the SAFIRE-B200 AFQMC kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#include "../../include/safire_b200.h"

namespace sfq {

// ---- complex double helpers (interleaved re,im -- the layout of std::complex<double>) -------
struct __align__(16) cplx {
  double x, y;
};

__host__ __device__ __forceinline__ cplx mk(double r, double i) { cplx c; c.x = r; c.y = i; return c; }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return mk(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ cplx cconj(cplx a) { return mk(a.x, -a.y); }
__device__ __forceinline__ double cabs_(cplx a) { return hypot(a.x, a.y); }
// Smith's algorithm for a/b
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + r * b.y;
    return mk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.y + r * b.x;
    return mk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
// principal complex log
__device__ __forceinline__ cplx clog_(cplx a) { return mk(log(hypot(a.x, a.y)), atan2(a.y, a.x)); }
__device__ __forceinline__ cplx cexp_(cplx a) {
  double e = exp(a.x);
  double s, c;
  sincos(a.y, &s, &c);
  return mk(e * c, e * s);
}

// ---- error reporting -------------------------------------------------------------------
#define SFQ_CUDA_TRY(expr)                                    \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) return ::sfq::record_cuda(_e, #expr, __FILE__, __LINE__); \
  } while (0)

int record_cuda(cudaError_t e, const char* what, const char* file, int line);
void count_launch();

// after every kernel launch: count it and surface launch-configuration errors
#define SFQ_LAUNCHED()                        \
  do {                                        \
    ::sfq::count_launch();                    \
    SFQ_CUDA_TRY(cudaGetLastError());         \
  } while (0)
int record_error(int code, const char* fmt, ...);

inline int ceil_div(long a, long b) { return int((a + b - 1) / b); }

}  // namespace sfq
