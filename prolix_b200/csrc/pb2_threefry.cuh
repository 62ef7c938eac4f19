// Counter-based noise for the Langevin O step, reproducing jax.random's
// threefry construction:
//  * threefry2x32, 20 rounds (Salmon et al., SC'11): rotations
//    (13,15,26,6),(17,29,16,24), key parity 0x1BD11BDA, a key injection after
//    every four rounds;
//  * split / random_bits in JAX's partitionable layout (element i of a shape
//    hashes the counter (hi32(i), lo32(i)); a 32-bit draw is the XOR of the
//    two output words) or the original layout (one iota split in halves);
//  * float32 uniform on [nextafter(-1,0), 1) from the top 23 bits, then
//    sqrt(2) * erfinv(u) with Giles' single-precision erfinv.
// Every float operation below is an explicitly rounded intrinsic (no
// contraction into FMA), in the same order as the CPU restatement, so the
// two produce identical bits.
#pragma once

#include <stdint.h>

namespace pb2 {

__device__ __forceinline__ uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

__device__ __forceinline__ void threefry2x32(uint32_t k0, uint32_t k1, uint32_t &x0,
                                             uint32_t &x1) {
  const uint32_t k2 = k0 ^ k1 ^ 0x1BD11BDAu;
  const uint32_t ks[3] = {k0, k1, k2};
  const int rot[8] = {13, 15, 26, 6, 17, 29, 16, 24};
  x0 += k0;
  x1 += k1;
#pragma unroll
  for (int r = 0; r < 20; ++r) {
    x0 += x1;
    x1 = rotl32(x1, rot[r & 7]);
    x1 ^= x0;
    if ((r & 3) == 3) {
      const int s = (r + 1) >> 2;
      x0 += ks[s % 3];
      x1 += ks[(s + 1) % 3] + (uint32_t)s;
    }
  }
}

// (new_key, sub) = jax.random.split(key)
__device__ __forceinline__ void split_key(uint32_t k0, uint32_t k1, bool partitionable,
                                          uint32_t out_key[2], uint32_t out_sub[2]) {
  if (partitionable) {
    uint32_t a0 = 0u, a1 = 0u, b0 = 0u, b1 = 1u;
    threefry2x32(k0, k1, a0, a1);
    threefry2x32(k0, k1, b0, b1);
    out_key[0] = a0; out_key[1] = a1;
    out_sub[0] = b0; out_sub[1] = b1;
  } else {
    // counts 0..3 split in halves: pairs (0,2) and (1,3); output [a0, a1, b0, b1]
    uint32_t a0 = 0u, b0 = 2u, a1 = 1u, b1 = 3u;
    threefry2x32(k0, k1, a0, b0);
    threefry2x32(k0, k1, a1, b1);
    out_key[0] = a0; out_key[1] = a1;
    out_sub[0] = b0; out_sub[1] = b1;
  }
}

// 32 random bits of element idx of a flat array of `count` elements.
__device__ __forceinline__ uint32_t random_bits32(const uint32_t key[2], uint32_t idx,
                                                  uint32_t count, bool partitionable) {
  if (partitionable) {
    uint32_t x0 = 0u, x1 = idx;
    threefry2x32(key[0], key[1], x0, x1);
    return x0 ^ x1;
  }
  const uint32_t half = (count + 1u) >> 1;
  uint32_t x0, x1;
  if (idx < half) {
    x0 = idx; x1 = idx + half;
    threefry2x32(key[0], key[1], x0, x1);
    return x0;
  }
  x0 = idx - half; x1 = idx;
  threefry2x32(key[0], key[1], x0, x1);
  return x1;
}

// log(1 + x) for x in (-1, 0]: own construction (argument reduction to
// m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1)) by its odd Taylor
// series to degree 15, e ln2 as a hi/lo pair, plus the rounding correction
// of 1 + x); cubic Taylor series for |x| < 2^-12.
__device__ __forceinline__ float log1p_own(float x) {
  const float one = 1.0f;
  const float u = __fadd_rn(one, x);
  const float c = __fdiv_rn(__fsub_rn(x, __fsub_rn(u, one)), u);
  const uint32_t bits = __float_as_uint(u);
  int e = (int)((bits >> 23) & 0xFFu) - 127;
  float m = __uint_as_float((bits & 0x7FFFFFu) | 0x3F800000u);
  if (m > __uint_as_float(1068827891u)) {  // 1.4142135f
    m = __fmul_rn(m, 0.5f);
    e += 1;
  }
  const float s = __fdiv_rn(__fsub_rn(m, one), __fadd_rn(m, one));
  const float s2 = __fmul_rn(s, s);
  float p = __uint_as_float(1032358025u);  // 1/15
  p = __fadd_rn(__fmul_rn(p, s2), __uint_as_float(1033734617u));  // 1/13
  p = __fadd_rn(__fmul_rn(p, s2), __uint_as_float(1035611788u));  // 1/11
  p = __fadd_rn(__fmul_rn(p, s2), __uint_as_float(1038323257u));  // 1/9
  p = __fadd_rn(__fmul_rn(p, s2), __uint_as_float(1041385765u));  // 1/7
  p = __fadd_rn(__fmul_rn(p, s2), __uint_as_float(1045220557u));  // 1/5
  p = __fadd_rn(__fmul_rn(p, s2), __uint_as_float(1051372203u));  // 1/3
  p = __fmul_rn(p, s2);
  const float two_s = __fmul_rn(2.0f, s);
  const float lm = __fadd_rn(two_s, __fmul_rn(two_s, p));
  const float ef = (float)e;
  const float ln2_hi = __uint_as_float(1060205056u);  // 0.693145751953125
  const float ln2_lo = __uint_as_float(901758606u);   // 1.4286068e-06
  const float r = __fadd_rn(__fmul_rn(ef, ln2_hi), __fadd_rn(lm, __fadd_rn(__fmul_rn(ef, ln2_lo), c)));
  if (fabsf(x) < 2.44140625e-4f) {  // 2^-12
    const float t = __fsub_rn(0.5f, __fmul_rn(x, __uint_as_float(1051372203u)));
    return __fmul_rn(x, __fsub_rn(one, __fmul_rn(x, t)));
  }
  return r;
}

// erfinv in float32: Giles (2011) single-precision polynomials in
// w - 2.5 (w < 5) or sqrt(w) - 3, w = -log(1 - x^2).
__device__ __forceinline__ float erfinv_f32(float x) {
  const float w = -log1p_own(-__fmul_rn(x, x));
  float p;
  if (w < 5.0f) {
    const float v = __fsub_rn(w, 2.5f);
    p = 2.81022636e-08f;
    p = __fadd_rn(3.43273939e-07f, __fmul_rn(p, v));
    p = __fadd_rn(-3.5233877e-06f, __fmul_rn(p, v));
    p = __fadd_rn(-4.39150654e-06f, __fmul_rn(p, v));
    p = __fadd_rn(0.00021858087f, __fmul_rn(p, v));
    p = __fadd_rn(-0.00125372503f, __fmul_rn(p, v));
    p = __fadd_rn(-0.00417768164f, __fmul_rn(p, v));
    p = __fadd_rn(0.246640727f, __fmul_rn(p, v));
    p = __fadd_rn(1.50140941f, __fmul_rn(p, v));
  } else {
    const float v = __fsub_rn(__fsqrt_rn(fmaxf(w, 0.0f)), 3.0f);
    p = -0.000200214257f;
    p = __fadd_rn(0.000100950558f, __fmul_rn(p, v));
    p = __fadd_rn(0.00134934322f, __fmul_rn(p, v));
    p = __fadd_rn(-0.00367342844f, __fmul_rn(p, v));
    p = __fadd_rn(0.00573950773f, __fmul_rn(p, v));
    p = __fadd_rn(-0.0076224613f, __fmul_rn(p, v));
    p = __fadd_rn(0.00943887047f, __fmul_rn(p, v));
    p = __fadd_rn(1.00167406f, __fmul_rn(p, v));
    p = __fadd_rn(2.83297682f, __fmul_rn(p, v));
  }
  if (fabsf(x) == 1.0f) return __fmul_rn(x, 3.402823466e+38f);
  return __fmul_rn(p, x);
}

// Standard normal (float32) from 32 random bits, as jax.random.normal.
__device__ __forceinline__ float normal_from_bits(uint32_t bits) {
  const float lo = __uint_as_float(0xBF7FFFFFu);  // nextafter(-1, 0)
  const float f = __fsub_rn(__uint_as_float((bits >> 9) | 0x3F800000u), 1.0f);
  float u = __fadd_rn(__fmul_rn(f, 2.0f), lo);  // span 1 - lo rounds to 2
  u = fmaxf(lo, u);
  return __fmul_rn(__uint_as_float(1068827891u), erfinv_f32(u));  // sqrt(2)
}

}  // namespace pb2
