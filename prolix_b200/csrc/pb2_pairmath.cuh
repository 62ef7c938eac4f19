// FP32 pair arithmetic of the OBC2 descreening integral.
//
// I(r; rho, s) follows prolix physics/generalized_born.py:211-263 (OpenMM's
// CustomGBForce OBC2 form): L = max(rho, |r - s|), U = r + s,
//   I = 1/2 (1/L - 1/U) + 1/4 ln(L/U)/r + 1/8 (r - s^2/r)(1/U^2 - 1/L^2),
// zero unless r + s > rho, with floors of 1e-4 on L, U and r.
//
// Far field.  When r - s >= rho (so L = r - s) the expression simplifies,
// with t = s/r, to I = (1/(2r)) (t/(1 - t^2) - atanh t), whose Taylor series
//   I = (t^3 / r) sum_{k>=1} k/(2k+1) t^(2k-2),
//   dI/dr = -(t^3 / r^2) sum_{k>=1} 2k(k+1)/(2k+1) t^(2k-2)
// has only positive terms, and avoids both the logarithm and the
// cancellation between the O(1/r) terms of the closed form (whose sum is
// O(s^3/r^4)).  Nearer pairs use the closed form with an accurate logf.
//
// The pair kernels sort tiles into tiers by the smallest distance between
// the two blocks' bounding boxes, and evaluate the two sums there by minimax
// polynomials of 3 to 7 terms (pb2_obc_series.cuh, written by
// gen_obc_series.py), each within 2e-8 relative of the full series on its
// tier.  The closed-form helpers below take the Taylor series directly.
#pragma once

namespace pb2 {

constexpr float kSeriesU = 0.09f;      // closed-form helpers' series shortcut (9 terms)
constexpr float kSeriesUNear = 0.16f;  // per-pair test in near tiles (10 / 11 terms); 1/sqrt = 2.5

// sum_{k=1..K} k/(2k+1) u^(k-1), Horner; coefficients folded at compile time.
template <int K>
__device__ __forceinline__ float obc_series_val_n(float u) {
  float p = (float)((double)K / (double)(2 * K + 1));
#pragma unroll
  for (int k = K - 1; k >= 1; --k) p = fmaf(p, u, (float)((double)k / (double)(2 * k + 1)));
  return p;
}

// sum_{k=1..K} 2k(k+1)/(2k+1) u^(k-1).
template <int K>
__device__ __forceinline__ float obc_series_der_n(float u) {
  float p = (float)(2.0 * K * (K + 1) / (double)(2 * K + 1));
#pragma unroll
  for (int k = K - 1; k >= 1; --k) p = fmaf(p, u, (float)(2.0 * k * (k + 1) / (double)(2 * k + 1)));
  return p;
}

// I(r; rho, s).  inv_r = 1/r (already available to every caller).
__device__ __forceinline__ float obc_integral(float r, float inv_r, float rho, float s) {
  if (!(r + s > rho)) return 0.0f;
  const float t = s * inv_r;
  const float u = t * t;
  if (u <= kSeriesU && r - s >= rho) return t * u * inv_r * obc_series_val_n<9>(u);
  const float rs = fmaxf(r, 1e-4f);
  const float irs = 1.0f / rs;
  const float L = fmaxf(fmaxf(rho, fabsf(r - s)), 1e-4f);
  const float U = fmaxf(r + s, 1e-4f);
  const float il = 1.0f / L, iu = 1.0f / U;
  const float lg = logf(L * iu);
  return 0.5f * (il - iu) + 0.25f * lg * irs + 0.125f * (r - s * s * irs) * (iu * iu - il * il);
}

// dI/dr(r; rho, s).
__device__ __forceinline__ float obc_integral_dr(float r, float inv_r, float rho, float s) {
  if (!(r + s > rho)) return 0.0f;
  const float t = s * inv_r;
  const float u = t * t;
  if (u <= kSeriesU && r - s >= rho) return -t * u * inv_r * inv_r * obc_series_der_n<9>(u);
  const float rs = fmaxf(r, 1e-4f);
  const float drs = r > 1e-4f ? 1.0f : 0.0f;
  const float irs = 1.0f / rs;
  const float d = fabsf(r - s);
  const bool use_d = d > rho;
  const float Lraw = use_d ? d : rho;
  const float L = fmaxf(Lraw, 1e-4f);
  const float dL = (use_d && Lraw > 1e-4f) ? copysignf(1.0f, r - s) : 0.0f;
  const float Uraw = r + s;
  const float U = fmaxf(Uraw, 1e-4f);
  const float dU = Uraw > 1e-4f ? 1.0f : 0.0f;
  const float il = 1.0f / L, iu = 1.0f / U;
  const float lg = logf(L * iu);
  const float t1 = 0.5f * (-dL * il * il + dU * iu * iu);
  const float t2 = 0.25f * ((dL * il - dU * iu) * irs - lg * drs * irs * irs);
  const float a = r - s * s * irs;
  const float da = 1.0f + s * s * drs * irs * irs;
  const float b = iu * iu - il * il;
  const float db = -2.0f * dU * iu * iu * iu + 2.0f * dL * il * il * il;
  return t1 + t2 + 0.125f * (da * b + a * db);
}

}  // namespace pb2
