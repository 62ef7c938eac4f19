// Correctly rounded FP64 quotient p / m from a precomputed y = RN(1/m), by
// two Markstein corrections (P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34
// (1990) 111-119; also Muller et al., Handbook of Floating-Point
// Arithmetic, division with an FMA):
//   q0 = RN(p y)            within 2 ulp of p/m (|p y - p/m| <= 2^-53 |p/m|),
//   r0 = RN(p - m q0)       (a single rounding of a remainder of a few ulp),
//   q1 = RN(q0 + r0 y)      within 1 ulp: q0 + (p - m q0) y - p/m =
//                           (q0 - p/m)(1 - m y) with |1 - m y| <= 2^-53, and
//                           r0's rounding moves it by ~2^-52 ulp,
//   r1 = p - m q1           exact (q1 within one ulp of p/m),
//   q2 = RN(q1 + r1 y)      = RN(p/m) by Markstein's theorem (y within half
//                           an ulp of 1/m, q1 within one ulp of p/m).
// The error bounds need no underflow or overflow, so zero,
// tiny, huge and non-finite quotients take the correctly rounded division
// itself (which also keeps the sign of a zero).  The integrator divides
// every momentum by the same mass six times a step; this costs one
// reciprocal per atom and five FP64 operations per quotient.
#pragma once

namespace pb2 {

__device__ __forceinline__ double div_by(double p, double m, double y) {
  const double q0 = __dmul_rn(p, y);
  const double a = fabs(q0);
  if (!(a >= 0x1p-900 && a <= 0x1p+900)) return __ddiv_rn(p, m);
  const double r0 = __fma_rn(-m, q0, p);
  const double q1 = __fma_rn(r0, y, q0);
  const double r1 = __fma_rn(-m, q1, p);
  return __fma_rn(r1, y, q1);
}

}  // namespace pb2
