// exp(x) in FP64 by P. T. P. Tang's table-driven method ("Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM Trans. Math. Softw. 15(2), 1989), for the sweep's
// Maxwellian values (x <= 0), from the mathematics:
//   x = (64 m + j) ln2/64 + r,  j = 0..63,  |r| <= ln2/128,
//   exp(x) = 2^m * 2^(j/64) * exp(r),
// with k = 64 m + j the integer nearest x*64/ln2 (rounded by adding and
// subtracting 1.5*2^52), r = x - k*ln2/64 by two fused multiply-adds with
// ln2/64 split into a 32-bit head and its remainder, and exp(r) - 1 by the
// Taylor polynomial of degree 5 (truncation error |r|^6/720 < 4e-17
// relative).  The table tab[j] = 2^(j/64) is the caller's (filled once per
// CTA); 2^m is applied by an integer add to the exponent field.  Below
// x = -707 (results under 1e-307) the value is flushed to +0; NaN stays NaN.
// Measured against long-double exp on the host (tests/test_exp_tang.py).
#pragma once
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define DGBGK_HD __host__ __device__ __forceinline__
#else
#define DGBGK_HD inline
#endif

namespace dgbgk {

constexpr int EXP_TAB = 64;

DGBGK_HD double dbl_from_bits(int64_t b) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)b);
#else
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
#endif
}
DGBGK_HD int64_t dbl_bits(double d) {
#if defined(__CUDA_ARCH__)
  return (int64_t)__double_as_longlong(d);
#else
  int64_t b;
  std::memcpy(&b, &d, sizeof b);
  return b;
#endif
}

DGBGK_HD double exp_tang(double x, const double* __restrict__ tab) {
  const double inv_step = 92.33248261689366;        // 64 / ln2
  const double step_hi = 0.01083042469326756;       // ln2/64, leading 32 bits
  const double step_lo = 2.9815858269852933e-12;    // ln2/64 - step_hi
  const double shift = 6755399441055744.0;          // 1.5 * 2^52
  const double ks = fma(x, inv_step, shift);        // k in the low word
  const double kd = ks - shift;
  const int k = (int)(uint32_t)dbl_bits(ks);
  double r = fma(-kd, step_hi, x);
  r = fma(-kd, step_lo, r);
  double p = fma(r, 1.0 / 120.0, 1.0 / 24.0);
  p = fma(r, p, 1.0 / 6.0);
  p = fma(r, p, 0.5);
  p = fma(r, p, 1.0);
  p = r * p;  // exp(r) - 1
  const double t = tab[k & (EXP_TAB - 1)];
  const double y = fma(t, p, t);
  const int64_t m = (int64_t)(k >> 6);  // floor(k / 64)
  // 2^m: m added to the exponent field (two's complement, shifted unsigned)
  const double v = dbl_from_bits((int64_t)((uint64_t)dbl_bits(y) + ((uint64_t)m << 52)));
  return x > -707.0 ? v : (x != x ? x : 0.0);
}

}  // namespace dgbgk
