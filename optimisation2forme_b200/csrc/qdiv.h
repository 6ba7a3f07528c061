// Correctly rounded FP64 quotients that share a divisor.
//
// The residual kernels divide many numerators by the same value (the cell
// volume V, the density rho): the reference computes each term as a/V with
// an IEEE division.  Here the reciprocal y = RN(1/b) is computed once, with
// an IEEE division, and each quotient is then obtained from y by
// multiply-add corrections (P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1),
// 1990; the quotient theorem as stated in Muller et al., Handbook of
// Floating-Point Arithmetic, ch. 4):
//
//   q0 = RN(a*y)               within 1.5 ulp of a/b
//   r0 = RN(a - b*q0)          (fma)
//   q1 = RN(q0 + r0*y)         within 1/2 ulp + 2^-51 ulp of a/b, so
//   r1 = a - b*q1              is exact (fma), and
//   q  = RN(q1 + r1*y)         is RN(a/b) (Markstein's theorem: y is within
//                              1/2 ulp of 1/b and q1 within 1 ulp of a/b).
//
// The result is bit-identical to a/b, which keeps the FP64 residual
// bit-identical to the reference.  The theorem needs every intermediate in
// the normal range; outside it the plain division is used:
//   * the divisor: recip_for_div returns NaN unless 2^-500 <= |b| <= 2^500,
//     and a NaN y sends every quotient of that divisor to a/b;
//   * the quotient: unless 2^-400 <= |q0| <= 2^400 (so zeros, signed zeros,
//     infinities, NaNs and extreme magnitudes) the result is a/b.
// Within both ranges |a| lies in [2^-901, 2^901], so r0 and r1 are normal.
//
// The helpers are __host__ __device__ so that the CPU test
// (tests/qdiv_check.cpp) runs this very code against IEEE division.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define O2F_QDIV_FN __host__ __device__ __forceinline__
#else
#define O2F_QDIV_FN inline
#endif

namespace o2f {

// y for qdiv: RN(1/b), or NaN when b is outside [2^-500, 2^500].
O2F_QDIV_FN double recip_for_div(double b) {
  const double m = fabs(b);
  return (m >= 0x1p-500 && m <= 0x1p+500) ? 1.0 / b : NAN;
}

// The same from an already computed inv_b = RN(1/b).
O2F_QDIV_FN double recip_for_div(double b, double inv_b) {
  const double m = fabs(b);
  return (m >= 0x1p-500 && m <= 0x1p+500) ? inv_b : NAN;
}

// RN(a/b) given y = recip_for_div(b).
O2F_QDIV_FN double qdiv(double a, double b, double y) {
  const double q0 = a * y;
  const double m = fabs(q0);
  if (!(m >= 0x1p-400 && m <= 0x1p+400)) return a / b;
  const double r0 = fma(-b, q0, a);
  const double q1 = fma(r0, y, q0);
  const double r1 = fma(-b, q1, a);
  return fma(r1, y, q1);
}

// The same without the fallback, for loops that divide many numerators by
// one value: `ok` is cleared when the quotient is outside the range above,
// and the caller then recomputes with plain division.
O2F_QDIV_FN double qdiv_flag(double a, double b, double y, bool& ok) {
  const double q0 = a * y;
  const double m = fabs(q0);
  ok &= (m >= 0x1p-400) & (m <= 0x1p+400);
  const double r0 = fma(-b, q0, a);
  const double q1 = fma(r0, y, q0);
  const double r1 = fma(-b, q1, a);
  return fma(r1, y, q1);
}

// FP32 instantiations (the mixed-precision path, which is not bit-exact by
// design): one reciprocal per divisor, each quotient a multiplication
// (within 1.5 ulp of a/b).
O2F_QDIV_FN float recip_for_div(float b) { return 1.0f / b; }
O2F_QDIV_FN float recip_for_div(float, float inv_b) { return inv_b; }
O2F_QDIV_FN float qdiv(float a, float, float y) { return a * y; }
O2F_QDIV_FN float qdiv_flag(float a, float, float y, bool&) { return a * y; }

}  // namespace o2f
