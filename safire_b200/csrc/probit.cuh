// Inverse normal CDF by P. J. Acklam's rational approximation (published algorithm, relative
// error < 1.15e-9).  Same branch points and coefficients as the reference's field sampler
// (src/AFQMC/Utilities/probit.h:58-136) so the Gaussian fields agree to rounding.
#pragma once
#include <math.h>

namespace sfq {

__host__ __device__ __forceinline__ double probit(double p) {
  const double a0 = -3.969683028665376e+01, a1 = 2.209460984245205e+02, a2 = -2.759285104469687e+02,
               a3 = 1.383577518672690e+02, a4 = -3.066479806614716e+01, a5 = 2.506628277459239e+00;
  const double b0 = -5.447609879822406e+01, b1 = 1.615858368580409e+02, b2 = -1.556989798598866e+02,
               b3 = 6.680131188771972e+01, b4 = -1.328068155288572e+01;
  const double c0 = -7.784894002430293e-03, c1 = -3.223964580411365e-01, c2 = -2.400758277161838e+00,
               c3 = -2.549732539343734e+00, c4 = 4.374664141464968e+00, c5 = 2.938163982698783e+00;
  const double d0 = 7.784695709041462e-03, d1 = 3.224671290700398e-01, d2 = 2.445134137142996e+00,
               d3 = 3.754408661907416e+00;
  const double plow = 0.02425, phigh = 0.97575;
  if (p < 0.0 || p > 1.0) return 0.0;
  if (p == 0.0) return -HUGE_VAL;
  if (p == 1.0) return HUGE_VAL;
  if (p < plow) {
    double q = sqrt(-2.0 * log(p));
    return (((((c0 * q + c1) * q + c2) * q + c3) * q + c4) * q + c5) /
           ((((d0 * q + d1) * q + d2) * q + d3) * q + 1.0);
  }
  if (p > phigh) {
    double q = sqrt(-2.0 * log(1.0 - p));
    return -(((((c0 * q + c1) * q + c2) * q + c3) * q + c4) * q + c5) /
           ((((d0 * q + d1) * q + d2) * q + d3) * q + 1.0);
  }
  double q = p - 0.5, r = q * q;
  return (((((a0 * r + a1) * r + a2) * r + a3) * r + a4) * r + a5) * q /
         (((((b0 * r + b1) * r + b2) * r + b3) * r + b4) * r + 1.0);
}

}  // namespace sfq
