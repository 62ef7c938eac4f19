// Pair kernels of the implicit-solvent force evaluation.
//
// Three warp-tiled passes visit every unique pair (i < j) of every system
// once (Newton's third law), in 32 x 32 tiles:
//   born  : descreening sums I_i += I(r; rho~_i, s_j), I_j += I(r; rho~_j, s_i)
//           (prolix physics/generalized_born.py:32-94, :266-337);
//   force : GB polar pair term, direct Coulomb and Lennard-Jones force, plus
//           dE_GB/dB for both atoms (generalized_born.py:97-208,
//           physics/optimization.py:21-297, analytical_forces.py:167-292);
//   chain : F -= (dE/dI_i dI_ij/dr + dE/dI_j dI_ji/dr) r^ , the Born-radius
//           chain rule (generalized_born.py:773-814).
// A per-atom pass between born and force turns the sums into Born radii and
// adds the self (q^2/B) and ACE terms.
//
// Mapping: one warp per work item (system, two consecutive i-blocks, range
// of j-blocks); lane l owns atom l of each i-block for the whole item; the
// j-block's data and j-side accumulators rotate through the lanes by
// shuffles, so lane l meets j-lane (l + k) mod 32 at step k of the 32-step
// loop, once for each of its two i atoms; the two pairs of a step run as
// packed f32x2 arithmetic.  Per tile, each lane's pair-validity and
// exclusion bit masks are rotated by its lane index once, so step k tests
// bit k (the sign bit of the bit-reversed mask shifted k times).  A
// per-block bounding box sorts tiles: tiles whose boxes are at least the
// far-field distance apart evaluate the OBC integral by a minimax
// polynomial of its far-field series (3 to 7 terms by separation,
// pb2_obc_series.cuh) without per-pair branches, and (with a cutoff) tiles
// beyond every cutoff are skipped.
//
// Arithmetic is FP32; per-tile partial sums are converted to 64-bit fixed
// point and combined with integer atomics, so results do not depend on
// scheduling order.
#include <algorithm>

#include "pb2_bonded.cuh"
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"
#include "pb2_obc_series.cuh"
#include "pb2_pairmath.cuh"

// Unroll factor of the 32-step rotation loop (code size against loop
// overhead; the instruction cache favours a partial unroll).
#ifndef PB2_UNROLL
#define PB2_UNROLL 2
#endif

namespace pb2 {

// The descreening / chain-rule loop is not unrolled: each kernel holds five
// tile variants (series lengths, near tiles) of two pairs per step, and
// unrolling them outgrows the instruction cache (unroll 2 cost 6 % and
// unroll 4 doubled the chain pass on B200).
#ifndef PB2_UNROLL_BC
#define PB2_UNROLL_BC 1
#endif

constexpr int kUnroll = PB2_UNROLL;
constexpr int kUnrollBC = PB2_UNROLL_BC;

__device__ __forceinline__ float shfl_next(float v, int src) { return __shfl_sync(kFull, v, src); }

__device__ __forceinline__ uint32_t rotr32(uint32_t x, int s) { return __funnelshift_r(x, x, s); }

// Squared distance between the bounding boxes of two blocks.
__device__ __forceinline__ float box_dist2(const float4 *bbox, int a, int b) {
  const float4 alo = bbox[2 * a], ahi = bbox[2 * a + 1];
  const float4 blo = bbox[2 * b], bhi = bbox[2 * b + 1];
  const float dx = fmaxf(0.f, fmaxf(alo.x - bhi.x, blo.x - ahi.x));
  const float dy = fmaxf(0.f, fmaxf(alo.y - bhi.y, blo.y - ahi.y));
  const float dz = fmaxf(0.f, fmaxf(alo.z - bhi.z, blo.z - ahi.z));
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}


struct PData {  // per-atom data a lane holds (its i atom, or the j atom passing through)
  float x, y, z, q, hs, se, ro, sr, B, iB, dedi;  // iB = sqrt(log2 e / 4) / B
  float rB;  // 1 / B
  float t2;  // (max(s / sqrt(kSeriesUNear), s + rho~_max))^2: series reach of this atom
  float s2, s3;  // s^2, s^3 of the scaled radius (far-field series)
};

// 4 / log2(e), and sqrt(log2(e) / 4): the force pass stores 1/B pre-scaled by
// sqrt(log2(e)/4) so that exp(-r^2 / (4 B_i B_j)) = exp2(-r^2 iB_i iB_j).
constexpr float kInvQuarterLog2e = 2.7725887222397811f;
constexpr float kSqrtQuarterLog2e = 0.60056120439322491f;
constexpr float kSixthRoot2 = 1.12246204830937298f;  // 2^(1/6)
constexpr float kSqrtHalf = 0.70710678118654752f;
struct Acc {
  float a0, a1, a2, a3;
};
struct TileConst {
  float cut2, gcut2, bcut2, pref, kcoul, lj14, coul14;  // bcut2: descreening / chain rule
  bool use_gb, use_lj, use_coul;
  int src, lane;
};

// The j-block's data of a tile, in shared memory, one warp's share: four
// float4 fields per atom, each holding two values as (v, v) pairs, so that
// a step reads a packed operand straight into a register pair.  Field-major
// (field, atom), so that the 32 lanes' 16-byte reads of one field are
// conflict-free.  Every atom is stored twice (entries a and a + 32): lane l
// reads entry l + k at step k, with no wrap-around arithmetic.  Force pass: (-x, -x, -y, -y), (-z, -z, q, q),
// (hs, hs, se, se), (B, B, iB, iB).  Descreening: (-x, -x, -y, -y),
// (-z, -z, s2, s2), (s3, s3, t2, t2).  Chain rule: the same with
// (s3, s3, dedi, dedi) and (t2, t2, 0, 0).
typedef float4 JTile[4][64];

// What a lane reads of its j atom at a step.
struct JF2 {  // force pass
  float2 mx, my, mz, q, hs, se, B, iB;
};
struct JD2 {  // descreening and chain rule
  float2 mx, my, mz, s2, s3, dedi;
  float t2;
};

__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

__device__ __forceinline__ JF2 load_jf(const JTile &t, int e) {
  const float4 a = t[0][e], b = t[1][e], c = t[2][e], d = t[3][e];
  return JF2{lo2(a), hi2(a), lo2(b), hi2(b), lo2(c), hi2(c), lo2(d), hi2(d)};
}

template <int PASS, bool FAR>
__device__ __forceinline__ JD2 load_jd(const JTile &t, int e) {
  const float4 a = t[0][e], b = t[1][e], c = t[2][e];
  JD2 j;
  j.mx = lo2(a); j.my = hi2(a); j.mz = lo2(b); j.s2 = hi2(b); j.s3 = lo2(c);
  j.dedi = make_float2(0.f, 0.f);
  j.t2 = 0.f;
  if (PASS == PASS_BORN) {
    if (!FAR) j.t2 = c.z;
  } else {
    j.dedi = hi2(c);
    if (!FAR) j.t2 = t[3][e].x;
  }
  return j;
}

// Store the lane's j atom into the warp's tile (after the previous tile's
// reads; the caller synchronises the warp before and after).
template <int PASS>
__device__ __forceinline__ void store_j(JTile &t, int lane, const PData &J) {
  float4 f[4];
  int nf = 3;
  f[0] = make_float4(-J.x, -J.x, -J.y, -J.y);
  if (PASS == PASS_FORCE) {
    f[1] = make_float4(-J.z, -J.z, J.q, J.q);
    f[2] = make_float4(J.hs, J.hs, J.se, J.se);
    f[3] = make_float4(J.B, J.B, J.iB, J.iB);
    nf = 4;
  } else if (PASS == PASS_BORN) {
    f[1] = make_float4(-J.z, -J.z, J.s2, J.s2);
    f[2] = make_float4(J.s3, J.s3, J.t2, J.t2);
  } else {
    f[1] = make_float4(-J.z, -J.z, J.s2, J.s2);
    f[2] = make_float4(J.s3, J.s3, J.dedi, J.dedi);
    f[3] = make_float4(J.t2, J.t2, 0.f, 0.f);
    nf = 4;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
    if (c < nf) {
      t[c][lane] = f[c];
      t[c][lane + 32] = f[c];
    }
}

// Force-pass rotation of the j-side sums but tj.a0.
__device__ __forceinline__ void rotate_force_rest(Acc &tj, int src, const TileConst &K) {
  tj.a1 = shfl_next(tj.a1, src); tj.a2 = shfl_next(tj.a2, src);
  if (K.use_gb) tj.a3 = shfl_next(tj.a3, src);
}

__device__ __forceinline__ void load_pdata(const PairArgs &a, int g, int pass, bool use_gb, float ro_max,
                                           PData &P) {
  const float4 p = a.posq[g], c = a.par[g];
  P.x = p.x; P.y = p.y; P.z = p.z; P.q = p.w;
  P.hs = c.x; P.se = c.y; P.ro = c.z; P.sr = c.w;
  const float t = fmaxf(P.sr * 2.5f, P.sr + ro_max);  // 2.5 = 1 / sqrt(kSeriesUNear)
  P.t2 = t * t;
  P.s2 = P.sr * P.sr;
  P.s3 = P.s2 * P.sr;
  P.B = P.iB = P.dedi = P.rB = 0.f;
  if ((pass == PASS_FORCE && use_gb) || pass == PASS_CHAIN) {
    const float4 b = a.born[g];
    P.B = b.x; P.iB = b.y * kSqrtQuarterLog2e; P.rB = b.y;
    if (pass == PASS_CHAIN) P.dedi = (float)((double)a.dedb_acc[g] * kForceInv) * b.z;
  }
  if (pass == PASS_FORCE) {  // the force pass's scaled per-atom factors (force_pair_step)
    P.hs *= kSixthRoot2;
    P.se *= kSqrtHalf;
    P.B *= 2.f;
  }
}

// ---------------------------------------------------------------- force pass
//
// The two pairs of a step run as packed f32x2 arithmetic (.x: i-block ib,
// .y: ib + 1), branch-free: invalid pairs are evaluated at r^2 = kFarR2,
// where every term underflows to zero; exclusions, 1-4 scales and cutoffs
// become per-component factors.

constexpr float kFarR2 = 1e30f;

struct FData2 {  // the lane's two i atoms, packed, for the force pass
  float2 x, y, z, hs, se, B, iB;
  float2 q2p;  // 2 P q_i: the GB factor A2 = 2 P q_i q_j / f^3 in one product
  float2 qk;   // k_C q_i
};
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

// The two lanes of a packed pair through the MUFU, written straight into one
// 64-bit register so that the packed operations that read the result find
// it in an aligned register pair (the same instructions rsqrtf and exp2f
// issue under -ftz).
__device__ __forceinline__ float2 unpack2(unsigned long long p) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(p));
  return r;
}
__device__ __forceinline__ float2 rsqrt2(float2 v) {
  unsigned long long p;
  asm("{\n\t.reg .f32 a, b;\n\trsqrt.approx.ftz.f32 a, %1;\n\trsqrt.approx.ftz.f32 b, %2;\n\tmov.b64 %0, {a, b};\n\t}"
      : "=l"(p) : "f"(v.x), "f"(v.y));
  return unpack2(p);
}
__device__ __forceinline__ float2 exp2neg2(float2 w) {  // 2^-w per lane
  unsigned long long p;
  asm("{\n\t.reg .f32 a, b;\n\tneg.f32 a, %1;\n\tneg.f32 b, %2;\n\tex2.approx.ftz.f32 a, a;\n\tex2.approx.ftz.f32 b, b;\n\tmov.b64 %0, {a, b};\n\t}"
      : "=l"(p) : "f"(w.x), "f"(w.y));
  return unpack2(p);
}
__device__ __forceinline__ float2 sel2(bool a, bool b, float va, float vb) {
  return make_float2(a ? va : vb, b ? va : vb);
}

struct Acc2F {
  float2 a0, a1, a2, a3;
};

// The masks of one packed pair of i-blocks (bit-reversed, tested through
// the sign bit and shifted once per step): pair validity, exclusion, 1-4.
struct ForceMasks {
  uint32_t R0, R1, X0, X1, Q0, Q1;
};
__device__ __forceinline__ ForceMasks force_masks(uint32_t V0, uint32_t V1, uint32_t E0, uint32_t E1, uint32_t S0,
                                                  uint32_t S1) {
  return ForceMasks{__brev(V0), __brev(V1), __brev(E0), __brev(E1), __brev(S0), __brev(S1)};
}

// One step of one packed pair of i-blocks against the j atom J: the i-side
// sums into ti, the j-side sums into tj (not rotated here).  Both the
// two-block and the four-block force kernels step through this function,
// so their sums are the same bit for bit.
template <bool CUT, bool FULL, bool EXCL>
__device__ __forceinline__ void force_pair_step(const FData2 &I, const JF2 &J, Acc2F &ti, Acc &tj, ForceMasks &M,
                                                const TileConst &K) {
  const float2 dx = __fadd2_rn(I.x, J.mx);
  const float2 dy = __fadd2_rn(I.y, J.my);
  const float2 dz = __fadd2_rn(I.z, J.mz);
  float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
  if (!FULL) {
    r2 = make_float2((int32_t)M.R0 < 0 ? r2.x : kFarR2, (int32_t)M.R1 < 0 ? r2.y : kFarR2);
    M.R0 <<= 1;
    M.R1 <<= 1;
  }
  float2 g = make_float2(0.f, 0.f);
  if (K.use_gb) {
    // E = P qq / f, f^2 = r^2 + B_i B_j e^(-r^2 / 4 B_i B_j); with
    // A2 = 2 P qq / f^3:  -dE/dr / r = A2 (1 - e / 4), and
    // dE/dB_i = -(A2 e / 2) (B_i B_j + r^2 / 4) / B_i, whose numerator is
    // the same for both atoms: h = A2 e (B_i B_j + r^2 / 4) is summed for
    // both, and each sum is scaled by -1 / (2 B) when it is flushed
    // No packed constants (each would be rematerialised into a register
    // pair): B is doubled per atom, so bb = 4 B_i B_j, and the MUFU returns
    // ex = e / 4 from the argument r^2 log2(e) / (4 B_i B_j) + 2, formed per
    // lane with the constant as an immediate; then f^2 = bb ex + r^2,
    // -dE/dr / r = A2 - A2 ex and h = A2 ex (bb + r^2).
    const float2 iBB = __fmul2_rn(I.iB, J.iB);
    const float2 ex = exp2neg2(make_float2(__fmaf_rn(r2.x, iBB.x, 2.f), __fmaf_rn(r2.y, iBB.y, 2.f)));
    const float2 bb = __fmul2_rn(I.B, J.B);
    const float2 f2 = __ffma2_rn(bb, ex, r2);
    const float2 inv_f = rsqrt2(f2);
    float2 A2 = __fmul2_rn(__fmul2_rn(I.q2p, J.q), __fmul2_rn(__fmul2_rn(inv_f, inv_f), inv_f));
    if (CUT && K.gcut2 != 0.f) A2 = __fmul2_rn(A2, sel2(r2.x < K.gcut2, r2.y < K.gcut2, 1.f, 0.f));
    const float2 A2e = __fmul2_rn(A2, ex);
    g = make_float2(__fsub_rn(A2.x, A2e.x), __fsub_rn(A2.y, A2e.y));
    const float2 h = __fmul2_rn(A2e, __fadd2_rn(bb, r2));
    ti.a3 = __fadd2_rn(ti.a3, h);
    tj.a3 = tj.a3 + h.x + h.y;
  }
  if (K.use_lj || K.use_coul) {
    const float2 inv_r = rsqrt2(r2);
    const float2 inv_r2 = __fmul2_rn(inv_r, inv_r);
    float2 sc_c = dup2(1.f), sc_l = dup2(1.f);  // exclusion and 1-4 factors
    if (EXCL) {
      const bool x0 = (int32_t)M.X0 < 0, x1 = (int32_t)M.X1 < 0, q0 = (int32_t)M.Q0 < 0, q1 = (int32_t)M.Q1 < 0;
      sc_c = make_float2(x0 ? 0.f : (q0 ? K.coul14 : 1.f), x1 ? 0.f : (q1 ? K.coul14 : 1.f));
      sc_l = make_float2(x0 ? 0.f : (q0 ? K.lj14 : 1.f), x1 ? 0.f : (q1 ? K.lj14 : 1.f));
      M.X0 <<= 1; M.X1 <<= 1; M.Q0 <<= 1; M.Q1 <<= 1;
    }
    float2 s = make_float2(0.f, 0.f);  // (-dE/dr) r for Coulomb and LJ
    if (K.use_coul) {
      s = __fmul2_rn(__fmul2_rn(I.qk, J.q), inv_r);
      if (EXCL) s = __fmul2_rn(s, sc_c);
    }
    if (K.use_lj) {
      const float2 sig = __fadd2_rn(I.hs, J.hs);
      const float2 sr2 = __fmul2_rn(__fmul2_rn(sig, sig), inv_r2);
      const float2 s6 = __fmul2_rn(__fmul2_rn(sr2, sr2), sr2);
      // sigma scaled by 2^(1/6) per atom: s6 = 2 (sigma / r)^6; se_i se_j =
      // 12 eps: e6 = 24 eps (sigma / r)^6, times 2 (sigma / r)^6 - 1 = s6 - 1
      float2 eps = __fmul2_rn(I.se, J.se);
      if (EXCL) eps = __fmul2_rn(eps, sc_l);
      s = __ffma2_rn(__fmul2_rn(eps, s6), make_float2(__fadd_rn(s6.x, -1.f), __fadd_rn(s6.y, -1.f)), s);
    }
    if (CUT && K.cut2 != 0.f) s = __fmul2_rn(s, sel2(r2.x < K.cut2, r2.y < K.cut2, 1.f, 0.f));
    g = __ffma2_rn(s, inv_r2, g);
  }
  ti.a0 = __ffma2_rn(g, dx, ti.a0);
  ti.a1 = __ffma2_rn(g, dy, ti.a1);
  ti.a2 = __ffma2_rn(g, dz, ti.a2);
  tj.a0 = fmaf(-g.x, dx.x, fmaf(-g.y, dx.y, tj.a0));
  tj.a1 = fmaf(-g.x, dy.x, fmaf(-g.y, dy.y, tj.a1));
  tj.a2 = fmaf(-g.x, dz.x, fmaf(-g.y, dz.y, tj.a2));
}

__device__ __forceinline__ void rotate_force(Acc &tj, int src, const TileConst &K) {
  tj.a0 = shfl_next(tj.a0, src);
  rotate_force_rest(tj, src, K);
}

template <bool CUT, bool FULL, bool EXCL>
__device__ __forceinline__ void run_force_tile2(const FData2 &I, const JTile &jt, Acc2F &ti, Acc &tj, uint32_t V0,
                                                uint32_t V1, uint32_t E0, uint32_t E1, uint32_t S0,
                                                uint32_t S1, const TileConst &K) {
  // step k tests the sign bits of the bit-reversed masks shifted left k times
  ForceMasks M = force_masks(V0, V1, E0, E1, S0, S1);
#pragma unroll kUnroll
  for (int k = 0; k < 32; ++k) {
    const JF2 J = load_jf(jt, K.lane + k);  // lane l meets j-lane (l + k) mod 32
    force_pair_step<CUT, FULL, EXCL>(I, J, ti, tj, M, K);
    rotate_force(tj, K.src, K);
  }
}

// Four i-blocks: two packed pairs share each step's j atom (one set of
// shared-memory loads for four pairs); each pair keeps its own j-side sums,
// so the sums are those of two two-block tiles.
template <bool CUT, bool FULL, bool EXCL>
__device__ __forceinline__ void run_force_tile4(const FData2 &Ia, const FData2 &Ib, const JTile &jt, Acc2F &ta,
                                                Acc2F &tb, Acc &tja, Acc &tjb, ForceMasks Ma, ForceMasks Mb,
                                                const TileConst &K) {
#pragma unroll 1
  for (int k = 0; k < 32; ++k) {
    const JF2 J = load_jf(jt, K.lane + k);
    force_pair_step<CUT, FULL, EXCL>(Ia, J, ta, tja, Ma, K);
    force_pair_step<CUT, FULL, EXCL>(Ib, J, tb, tjb, Mb, K);
    rotate_force(tja, K.src, K);
    rotate_force(tjb, K.src, K);
  }
}

// ------------------------------------------------ descreening and chain rule
//
// Both pairs of a step (the lane's atom of i-block ib and of ib + 1, against
// the same j atom) run the same arithmetic, so it is issued as packed FP32
// pairs (fma.rn.f32x2 and friends: .x = block ib, .y = block ib + 1), which
// halves the FP32 instructions of these passes.  Per component the results
// are those of the scalar fmaf / fmul / fadd.  The rsqrt and the j-side
// sums, to which both pairs add, stay scalar.

struct PData2 {  // the lane's two i atoms, packed
  float2 x, y, z, sr, ro, t2, s2, s3, dedi;
};
__device__ __forceinline__ PData2 pack2(const PData &a, const PData &b) {
  PData2 p;
  p.x = make_float2(a.x, b.x); p.y = make_float2(a.y, b.y); p.z = make_float2(a.z, b.z);
  p.sr = make_float2(a.sr, b.sr); p.ro = make_float2(a.ro, b.ro); p.t2 = make_float2(a.t2, b.t2);
  p.s2 = make_float2(a.s2, b.s2); p.s3 = make_float2(a.s3, b.s3); p.dedi = make_float2(a.dedi, b.dedi);
  return p;
}

// The near-tile domain (per-pair test against kSeriesUNear) is the widest
// tier of both polynomials.
static_assert((float)kValueTierU[3] == kSeriesUNear && (float)kDerivTierU[3] == kSeriesUNear,
              "series tiers");

struct Acc2 {
  float2 a0, a1, a2;
};

// Invalid pairs (padding lanes, j <= i on a diagonal, beyond the cutoff)
// are evaluated at r^2 = kFarR2: their radial factor underflows to exactly
// zero (1/r^4 = 1e-60), so they are summed without a select and never reach
// the closed form.

// Both pairs' geometry and both directions' integral terms.  The series
// keeps the radial factor apart: I = s^3 V(s^2/r^2) / r^4 and
// -(dI/dr) / r = s^3 D(s^2/r^2) / r^6, so vij, vji hold s^3 V (or s^3 D) and
// f the common 1/r^4 (or 1/r^6); a pair queued for the closed form has all
// three zeroed.
struct BCPair2 {
  float2 dx, dy, dz, r2, inv_r, vij, vji, f;
  bool ok0, ok1;
};

template <int PASS, bool CUT, bool FULL, int TIER>
__device__ __forceinline__ void bc_series2(const PData2 &I, const JD2 &J, bool ok0, bool ok1, BCPair2 &P,
                                           const TileConst &K) {
  P.dx = __fadd2_rn(I.x, J.mx);
  P.dy = __fadd2_rn(I.y, J.my);
  P.dz = __fadd2_rn(I.z, J.mz);
  const float2 r2 = __ffma2_rn(P.dx, P.dx, __ffma2_rn(P.dy, P.dy, __fmul2_rn(P.dz, P.dz)));
  if (CUT) {
    ok0 = ok0 && (K.bcut2 == 0.f || r2.x < K.bcut2);
    ok1 = ok1 && (K.bcut2 == 0.f || r2.y < K.bcut2);
  }
  P.ok0 = ok0;
  P.ok1 = ok1;
  // FULL: every pair of the tile exists (no cutoff): no select
  P.r2 = (FULL && !CUT) ? r2 : make_float2(ok0 ? r2.x : kFarR2, ok1 ? r2.y : kFarR2);
  // every lane evaluates, so the warp ballot that follows is reached by all lanes
  P.inv_r = rsqrt2(P.r2);
  const float2 inv_r2 = __fmul2_rn(P.inv_r, P.inv_r);
  const float2 inv_r4 = __fmul2_rn(inv_r2, inv_r2);
  if (PASS == PASS_BORN) {
    P.vij = __fmul2_rn(J.s3, ObcPoly<false, TIER>::eval2(__fmul2_rn(J.s2, inv_r2)));
    P.vji = __fmul2_rn(I.s3, ObcPoly<false, TIER>::eval2(__fmul2_rn(I.s2, inv_r2)));
    P.f = inv_r4;
  } else {
    P.vij = __fmul2_rn(J.s3, ObcPoly<true, TIER>::eval2(__fmul2_rn(J.s2, inv_r2)));
    P.vji = __fmul2_rn(I.s3, ObcPoly<true, TIER>::eval2(__fmul2_rn(I.s2, inv_r2)));
    P.f = __fmul2_rn(inv_r4, inv_r2);
  }
}

template <int PASS>
__device__ __forceinline__ void bc_accumulate2(const PData2 &I, const JD2 &J, const BCPair2 &P, Acc2 &ti,
                                               Acc &tj) {
  if (PASS == PASS_BORN) {
    ti.a0 = __ffma2_rn(P.vij, P.f, ti.a0);
    tj.a0 = fmaf(P.vji.x, P.f.x, fmaf(P.vji.y, P.f.y, tj.a0));
  } else {
    // h = -(dE/dI_i dI_ij/dr + dE/dI_j dI_ji/dr) / r; F_i += h d, F_j -= h d
    const float2 h = __fmul2_rn(__ffma2_rn(I.dedi, P.vij, __fmul2_rn(J.dedi, P.vji)), P.f);
    ti.a0 = __ffma2_rn(h, P.dx, ti.a0);
    ti.a1 = __ffma2_rn(h, P.dy, ti.a1);
    ti.a2 = __ffma2_rn(h, P.dz, ti.a2);
    tj.a0 = fmaf(-h.x, P.dx.x, fmaf(-h.y, P.dx.y, tj.a0));
    tj.a1 = fmaf(-h.x, P.dy.x, fmaf(-h.y, P.dy.y, tj.a1));
    tj.a2 = fmaf(-h.x, P.dz.x, fmaf(-h.y, P.dz.y, tj.a2));
  }
}

// Pairs of near tiles outside the series' domain take the closed form.
// Evaluated in place they would idle most of the warp at every step where
// one lane needs them (and a compact block of atoms holds many such pairs),
// so each warp queues them as (i, j) atom pairs in shared memory and
// evaluates them later, one pair per lane, adding each pair's two
// contributions to the fixed-point accumulators by itself.  A pair's
// contributions are the same whenever its queue is flushed, so results stay
// independent of scheduling.
constexpr int kCfCap = 256;  // queued pairs per warp (2 KB of shared memory)

struct CfArgs {
  const float4 *posq, *par, *born;
  const long long *dedb_acc;
  long long *born_acc, *fx, *fy, *fz;
};

__device__ __forceinline__ float dedi_of(const CfArgs &c, int g) {
  return (float)((double)c.dedb_acc[g] * kForceInv) * c.born[g].z;  // as load_pdata
}

// Evaluates the n queued pairs (warp-convergent; the caller synchronises
// the warp before and after): bc_series2's geometry, then the closed form
// of both directions (I or dI/dr), then bc_accumulate2's sums, per pair.
template <int PASS>
__device__ __forceinline__ void cf_flush(const CfArgs c, const int2 *q, int n, int lane, float bscale) {
  for (int e = lane; e < n; e += 32) {
    const int2 pr = q[e];  // (i, j) batch atom indices
    const float4 pi = c.posq[pr.x], pj = c.posq[pr.y];
    const float4 ci = c.par[pr.x], cj = c.par[pr.y];
    const float dx = pi.x + -pj.x, dy = pi.y + -pj.y, dz = pi.z + -pj.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float inv_r = rsqrtf(r2);
    const float r = r2 * inv_r;
    if (PASS == PASS_BORN) {
      atomic_add_fix(&c.born_acc[pr.x], to_fix_f(obc_integral(r, inv_r, ci.z, cj.w), bscale));
      atomic_add_fix(&c.born_acc[pr.y], to_fix_f(obc_integral(r, inv_r, cj.z, ci.w), bscale));
    } else {
      const float vij = obc_integral_dr(r, inv_r, ci.z, cj.w);
      const float vji = obc_integral_dr(r, inv_r, cj.z, ci.w);
      const float h = fmaf(dedi_of(c, pr.x), vij, dedi_of(c, pr.y) * vji) * -inv_r;
      const long long fx = to_fix_f(h * dx, bscale), fy = to_fix_f(h * dy, bscale),
                      fz = to_fix_f(h * dz, bscale);
      atomic_add_fix(&c.fx[pr.x], fx); atomic_add_fix(&c.fy[pr.x], fy); atomic_add_fix(&c.fz[pr.x], fz);
      atomic_add_fix(&c.fx[pr.y], -fx); atomic_add_fix(&c.fy[pr.y], -fy); atomic_add_fix(&c.fz[pr.y], -fz);
    }
  }
}

// The warp's closed-form queue and what a push needs to name its pairs.
struct CfQueue {
  CfArgs c;
  int2 *q;
  int n;              // warp-uniform
  int ig0, ig1, jg0;  // batch index of the lane's two i atoms; of the j-block's atom 0
  float bscale;
};

template <int PASS>
__device__ __forceinline__ void cf_drain(CfQueue &Q, int lane) {
  __syncwarp();  // the lanes' queue writes are visible to every lane
  cf_flush<PASS>(Q.c, Q.q, Q.n, lane, Q.bscale);
  __syncwarp();  // every lane has read its entries before the queue is reused
  Q.n = 0;
}

// FAR: both tiles lie in the series' domain (no per-pair test); otherwise
// each pair is tested, and those outside the domain go to the warp's
// closed-form queue with their series terms zeroed.
template <int PASS, bool FAR, bool CUT, bool FULL, int TIER>
__device__ __forceinline__ void run_bc_tile2(const PData2 &I, const JTile &jt, Acc2 &ti, Acc &tj, uint32_t V0,
                                             uint32_t V1, const TileConst &K, CfQueue &Q) {
  const int src = K.src;
  // step k tests the sign bit of the bit-reversed mask shifted left k times
  uint32_t R0 = __brev(V0), R1 = __brev(V1);
#pragma unroll kUnrollBC
  for (int k = 0; k < 32; ++k) {
    const JD2 J = load_jd<PASS, FAR>(jt, K.lane + k);  // lane l meets j-lane (l + k) mod 32
    BCPair2 P;
    bc_series2<PASS, CUT, FULL, TIER>(I, J, FULL || (int32_t)R0 < 0, FULL || (int32_t)R1 < 0, P, K);
    if (!FULL) {
      R0 <<= 1;
      R1 <<= 1;
    }
    if (!FAR) {
      // r >= t_i and r >= t_j give (s/r)^2 <= kSeriesUNear for both radii and
      // r - s >= rho~_max >= rho~ for both directions: a sufficient test in two
      // instructions (it sends about 1.3 % of near-tile pairs of compact
      // chains to the closed form, barely more than the exact test)
      const bool n0 = P.ok0 && !(P.r2.x >= fmaxf(I.t2.x, J.t2));
      const bool n1 = P.ok1 && !(P.r2.y >= fmaxf(I.t2.y, J.t2));
      const unsigned b0 = __ballot_sync(kFull, n0), b1 = __ballot_sync(kFull, n1);
      if (b0 | b1) {  // warp-uniform
        const int c0 = __popc(b0), cnt = c0 + __popc(b1);
        if (Q.n + cnt > kCfCap) cf_drain<PASS>(Q, K.lane);
        const unsigned lt = (1u << K.lane) - 1u;
        const int jg = Q.jg0 + ((K.lane + k) & 31);  // the j atom this lane holds at step k
        if (n0) {
          Q.q[Q.n + __popc(b0 & lt)] = make_int2(Q.ig0, jg);
          P.vij.x = 0.f; P.vji.x = 0.f; P.f.x = 0.f;
        }
        if (n1) {
          Q.q[Q.n + c0 + __popc(b1 & lt)] = make_int2(Q.ig1, jg);
          P.vij.y = 0.f; P.vji.y = 0.f; P.f.y = 0.f;
        }
        Q.n += cnt;
      }
    }
    bc_accumulate2<PASS>(I, J, P, ti, tj);
    tj.a0 = shfl_next(tj.a0, src);
    if (PASS == PASS_CHAIN) {
      tj.a1 = shfl_next(tj.a1, src); tj.a2 = shfl_next(tj.a2, src);
    }
  }
}

// One atom's Born radius from its descreening sum, and the per-atom GB
// self term and ACE as the initial dE/dB; clears the sum.
__device__ __forceinline__ void finalize_atom(const FinalizeArgs &a, int i, int s, const SysInfo &S) {
  const bool nl = S.clamp != 0;
  const double isum = (double)__ldcg(&a.born_acc[i]) * kBornInv;
  a.born_acc[i] = 0;
  const double r_in = a.radius[i];
  const double rad = nl ? fmax(r_in, 1e-6) : r_in;
  double ro = rad - kDielOffset;
  if (nl) ro = fmax(ro, 1e-4);
  const double psi = ro * isum;
  const double arg = kObcAlpha * psi - kObcBeta * psi * psi + kObcGamma * psi * psi * psi;
  const double th = tanh(arg);
  const double dr = nl ? fmax(rad, 1e-4) : rad;
  double inv_b = 1.0 / ro - th / dr;
  bool clamped = false;
  if (nl && inv_b < 1e-4) {
    inv_b = 1e-4;
    clamped = true;
  }
  const double B = 1.0 / inv_b;
  const double dpsi = (kObcAlpha - 2.0 * kObcBeta * psi + 3.0 * kObcGamma * psi * psi) * ro;
  const double dbdi = clamped ? 0.0 : B * B * (1.0 - th * th) / dr * dpsi;
  a.born[i] = make_float4((float)B, (float)inv_b, (float)dbdi, 0.f);
  if (a.born64) a.born64[i] = B;
  const double q = a.charge[i];
  const double r_nm = (r_in - kDielOffset) / 10.0 + 0.009;
  const double x = r_nm / (B / 10.0);
  const double x3 = x * x * x;
  const double ace = kAceCoeff * (r_nm + 0.14) * (r_nm + 0.14) * x3 * x3 * kKjToKcal;
  const double dedb = -S.pref_d * q * q * inv_b * inv_b - 6.0 * ace * inv_b;
  a.dedb_acc[i] = to_fix(dedb, kForceScale);
  if (a.energy_mode) {
    long long *e = a.energy + (size_t)s * PB2_NTERMS;
    atomic_add_fix(&e[PB2_TERM_GB], to_fix(S.pref_d * q * q * inv_b, kEnergyScale));
    atomic_add_fix(&e[PB2_TERM_NONPOLAR], to_fix(ace, kEnergyScale));
  }
}

// Spins of the bounded waits (each a 128 ns sleep and an L2 read): about a
// second at most; a wait for work in flight ends within one item (~0.1 ms).
constexpr int kWaitSpins = 1 << 20;

// Finalize chunk c (the batch's 32-atom block c) of the descreening pass:
// wait until every item of its system has been counted, then turn the
// block's sums into Born radii.  Every waited-for item was taken by a warp
// of this launch that is running, so the wait ends; it is bounded all the
// same, and a wait that gives up flags the system and skips the block.
__device__ __noinline__ void finalize_chunk(const PairArgs &a, int c, const int32_t *sys_items, int lane) {
  const int s = a.fin.blk_sys[c];
  if (a.fin.retired && a.fin.retired[s]) return;
  const SysInfo &S = a.sys[s];
  int ok = 1;
  if (lane == 0) {
    const int want = sys_items[s];
    const volatile int32_t *done = a.sys_done + s;
    for (int spin = 0; *done < want; ++spin) {
      if (spin >= kWaitSpins) {
        ok = 0;
        atomicOr(&a.fin.status[s], (uint32_t)PB2_STATUS_WAIT_TIMEOUT);
        break;
      }
      __nanosleep(128);
    }
  }
  ok = __shfl_sync(kFull, ok, 0);
  __threadfence();  // acquire: the counted items' sums are visible to every lane
  const int l = (c - S.blk_base) * 32 + lane;
  if (l < S.n) {
    if (ok) finalize_atom(a.fin, S.off + l, s, S);
    else a.fin.born_acc[S.off + l] = 0;  // the next evaluation starts from zero all the same
  }
  __syncwarp();
  if (lane == 0) {
    // the system's last chunk (all of them past their wait) resets the
    // counters for the next launch
    if (atomicAdd(&a.fin.sys_fin[s], 1) == S.nblk - 1) {
      a.sys_done[s] = 0;
      a.fin.sys_fin[s] = 0;
    }
  }
}

__global__ void born_finalize(const FinalizeArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    finalize_atom(a, i, s, a.sys[s]);
  }
}

// ------------------------------------------------------------------- kernel

// One warp per work item (system, even i-block ib, j-blocks [jb0, jb1)):
// lane l owns atom l of i-block ib and atom l of i-block ib + 1, and every
// j-block's data rotates once through the lanes, meeting both.  Tile
// (ib + 1, ib) lies below the diagonal and is skipped; (ib + 1, ib + 1) is
// the second block's diagonal tile.
//
// Items are handed out dynamically: each warp takes the next item from an
// atomic counter (items are sorted by cost, largest first), and the last
// warp to finish resets the counter for the next launch.
// ALL: GB, Coulomb and LJ all enabled (the term switches fold away).
// THREADS, MINB: the block shape (threads per block, and the blocks per SM
// the register budget is sized for); every pass is compiled for the shapes
// of kShapes and the autotuner picks one per pass at run time.
template <int PASS, bool CUT, bool ALL, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    tile2_kernel(const __grid_constant__ PairArgs a) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  TileConst K;
  K.use_gb = ALL || (a.terms & PB2_USE_GB) != 0;
  K.use_lj = ALL || (a.terms & PB2_USE_LJ) != 0;
  K.use_coul = ALL || (a.terms & PB2_USE_COULOMB) != 0;
  K.src = (lane + 1) & 31;
  K.lane = lane;
  // closed-form queues of the descreening and chain passes, one per warp
  constexpr int kWarps = THREADS / 32;
  __shared__ int2 s_cfq[PASS == PASS_FORCE ? 1 : kWarps][PASS == PASS_FORCE ? 1 : kCfCap];
  // the j-block of the current tile, one JTile per warp (4 KB)
  __shared__ JTile s_jt[kWarps];
  JTile &jt = s_jt[threadIdx.x >> 5];
  CfQueue Q;
  Q.c = {a.posq, a.par, a.born, a.dedb_acc, a.born_acc, a.fx, a.fy, a.fz};
  Q.q = s_cfq[PASS == PASS_FORCE ? 0 : (threadIdx.x >> 5)];
  Q.n = 0;
  Q.bscale = PASS == PASS_BORN ? (float)kBornScale : (float)kForceScale;
  const uint32_t diag_mask = lane == 31 ? 0u : (0xffffffffu << (lane + 1));
  const float bscale = PASS == PASS_BORN ? (float)kBornScale : (float)kForceScale;

  // a cutoff run with a pair list takes its items (and each item's j-blocks)
  // from the list; otherwise items are contiguous j-block ranges
  const bool plm = CUT && a.pl_ctl != nullptr;
  const TileItem *items = a.items;
  int n_items = a.item_count ? *a.item_count : a.n_items;
  const int32_t *sys_items = a.sys_items;
  if (plm) {
    const int cur = a.pl_ctl[PL_CUR];
    items = cur ? a.pl_items1 : a.pl_items0;
    n_items = a.pl_ctl[PL_COUNT0 + cur];
    if (sys_items) sys_items = cur ? a.pl_sys_items1 : a.pl_sys_items0;
  }
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(&a.sched[0], 1);
    it = __shfl_sync(kFull, it, 0);
    if (it >= n_items) {
      if constexpr (PASS == PASS_BORN) {
        // tail work: the Born radii of one 32-atom block, once its system's
        // items have all been summed
        const int c = it - n_items;
        if (sys_items && c < a.fin.n_blocks) {
          finalize_chunk(a, c, sys_items, lane);
          continue;
        }
      }
      if constexpr (PASS == PASS_CHAIN) {
        // tail work: a chunk of the bonded terms (FP64, their own forces)
        const int c = it - n_items;
        if (c < a.n_bonded_chunks) {
          const int t1 = min((c + 1) * kBondedChunk, bonded_total(a.bonded));
          for (int t = c * kBondedChunk + lane; t < t1; t += 32) bonded_term_call(a.bonded, t);
          continue;
        }
      }
      break;
    }
    const TileItem item = items[it];
    const SysInfo &S = a.sys[item.sys];
    const int n = S.n, off = S.off;
    K.cut2 = S.cutoff2; K.gcut2 = S.gb_cutoff2; K.bcut2 = S.born_cut2;
    K.pref = S.pref; K.kcoul = S.kcoul; K.lj14 = S.lj14; K.coul14 = S.coul14;
    const int ib0 = item.iblk, ib1 = item.iblk + 1;
    const bool has1 = ib1 < S.nblk;
    const int gib0 = S.blk_base + ib0, gib1 = S.blk_base + (has1 ? ib1 : ib0);
    const int il0 = ib0 * 32 + lane, il1 = ib1 * 32 + lane;
    const bool iv0 = il0 < n, iv1 = il1 < n;  // il1 >= n whenever !has1
    const int ig0 = off + (iv0 ? il0 : n - 1), ig1 = off + (iv1 ? il1 : n - 1);
    // largest distance at which this pass has any pair term (0: unbounded)
    float reach2 = 0.f;
    if (CUT) {
      if (PASS == PASS_FORCE) reach2 = (K.gcut2 == 0.f || K.cut2 == 0.f) ? 0.f : fmaxf(K.gcut2, K.cut2);
      else reach2 = K.bcut2;
    }
    PData I0, I1;
    load_pdata(a, ig0, PASS, K.use_gb, S.ro_max, I0);
    load_pdata(a, ig1, PASS, K.use_gb, S.ro_max, I1);
    const PData2 I2 = pack2(I0, I1);  // descreening / chain passes
    // exclusion entries: lanes 0-15 for block ib, lanes 16-31 for block ib + 1
    int2 ent = make_int2(-1, -1);
    if (PASS == PASS_FORCE) {
      if (lane < kExclPerBlock) ent = a.excl_ent[gib0 * kExclPerBlock + lane];
      else if (has1 && lane < 2 * kExclPerBlock) ent = a.excl_ent[gib1 * kExclPerBlock + lane - kExclPerBlock];
    }

    // the force pass's packed i-side data, once per item
    FData2 IF{};
    if constexpr (PASS == PASS_FORCE)
      IF = {make_float2(I0.x, I1.x), make_float2(I0.y, I1.y), make_float2(I0.z, I1.z),
            make_float2(I0.hs, I1.hs), make_float2(I0.se, I1.se),
            make_float2(I0.B, I1.B), make_float2(I0.iB, I1.iB),
            make_float2(2.f * K.pref * I0.q, 2.f * K.pref * I1.q),
            make_float2(K.kcoul * I0.q, K.kcoul * I1.q)};
    long long p0 = 0, p1 = 0, p2 = 0, p3 = 0, q0 = 0, q1 = 0, q2 = 0, q3 = 0;  // i-side sums
    for (int tt = item.jb0; tt < item.jb1; ++tt) {
      const int jb = plm ? a.pl_jlist[tt] : tt;
      const int gjb = S.blk_base + jb;
      // smallest bounding-box separation over the live tiles of the pair
      float d2 = 0.f;
      if (CUT || PASS != PASS_FORCE) {
        d2 = box_dist2(a.bbox, gib0, gjb);
        if (has1 && jb > ib0) d2 = fminf(d2, box_dist2(a.bbox, gib1, gjb));
      }
      if (CUT && reach2 > 0.f && d2 >= reach2) continue;  // no pair within reach
      const int jl0 = jb * 32;
      const int jl = jl0 + lane;
      const bool jvalid = jl < n;
      const int jg = off + (jvalid ? jl : n - 1);
      PData J;
      load_pdata(a, jg, PASS, K.use_gb, S.ro_max, J);
      __syncwarp();  // every lane is done with the previous tile's j data
      store_j<PASS>(jt, lane, J);
      __syncwarp();
      // pair validity of lane i with j-lane c: both exist, j > i on a diagonal
      const int nj = n - jl0;
      const uint32_t jmask = nj >= 32 ? 0xffffffffu : ((1u << nj) - 1u);
      uint32_t C0 = iv0 ? jmask : 0u, C1 = iv1 ? jmask : 0u;
      if (jb == ib0) {
        C0 &= diag_mask;
        C1 = 0u;
      } else if (jb == ib1) {
        C1 &= diag_mask;
      }
      const uint32_t V0 = rotr32(C0, lane), V1 = rotr32(C1, lane);

      Acc t0 = {0.f, 0.f, 0.f, 0.f}, t1 = {0.f, 0.f, 0.f, 0.f}, tj = {0.f, 0.f, 0.f, 0.f};
      if constexpr (PASS == PASS_FORCE) {
        const bool full = __all_sync(kFull, (C0 & C1) == 0xffffffffu);
        uint32_t E0 = 0u, S0 = 0u, E1 = 0u, S1 = 0u;
        const unsigned hit = __ballot_sync(kFull, ent.x == jb);
        static_assert(2 * kExclPerBlock == 32, "one exclusion entry per lane");
        const unsigned hit0 = hit & 0xffffu, hit1 = hit & 0xffff0000u;
        if (hit0) {
          const int roff = __shfl_sync(kFull, ent.y, __ffs(hit0) - 1);
          const ExclRow r = a.excl_rows[roff + lane];
          E0 = rotr32(r.excl, lane); S0 = rotr32(r.s14, lane);
        }
        if (hit1) {
          const int roff = __shfl_sync(kFull, ent.y, __ffs(hit1) - 1);
          const ExclRow r = a.excl_rows[roff + lane];
          E1 = rotr32(r.excl, lane); S1 = rotr32(r.s14, lane);
        }
        Acc2F tf = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        if (hit) run_force_tile2<CUT, false, true>(IF, jt, tf, tj, V0, V1, E0, E1, S0, S1, K);
        else if (!full) run_force_tile2<CUT, false, false>(IF, jt, tf, tj, V0, V1, E0, E1, S0, S1, K);
        else run_force_tile2<CUT, true, false>(IF, jt, tf, tj, V0, V1, E0, E1, S0, S1, K);
        t0.a0 = tf.a0.x; t0.a1 = tf.a1.x; t0.a2 = tf.a2.x; t0.a3 = tf.a3.x;
        t1.a0 = tf.a0.y; t1.a1 = tf.a1.y; t1.a2 = tf.a2.y; t1.a3 = tf.a3.y;
      } else {
        // series tier by the tiles' smallest separation
        const float *tier2 = S.tier2[PASS == PASS_BORN ? 0 : 1];
        Acc2 ti = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        Q.ig0 = ig0; Q.ig1 = ig1; Q.jg0 = off + jl0;
        // tiles whose 64 x 32 pairs all exist skip the validity masks
        const bool full = __all_sync(kFull, (C0 & C1) == 0xffffffffu);
        if (full) {
          if (d2 >= tier2[0]) run_bc_tile2<PASS, true, CUT, true, 0>(I2, jt, ti, tj, V0, V1, K, Q);
          else if (d2 >= tier2[1]) run_bc_tile2<PASS, true, CUT, true, 1>(I2, jt, ti, tj, V0, V1, K, Q);
          else if (d2 >= tier2[2]) run_bc_tile2<PASS, true, CUT, true, 2>(I2, jt, ti, tj, V0, V1, K, Q);
          else if (d2 >= S.far2) run_bc_tile2<PASS, true, CUT, true, 3>(I2, jt, ti, tj, V0, V1, K, Q);
          else run_bc_tile2<PASS, false, CUT, true, 3>(I2, jt, ti, tj, V0, V1, K, Q);
        } else {
          if (d2 >= tier2[0]) run_bc_tile2<PASS, true, CUT, false, 0>(I2, jt, ti, tj, V0, V1, K, Q);
          else if (d2 >= tier2[1]) run_bc_tile2<PASS, true, CUT, false, 1>(I2, jt, ti, tj, V0, V1, K, Q);
          else if (d2 >= tier2[2]) run_bc_tile2<PASS, true, CUT, false, 2>(I2, jt, ti, tj, V0, V1, K, Q);
          else if (d2 >= S.far2) run_bc_tile2<PASS, true, CUT, false, 3>(I2, jt, ti, tj, V0, V1, K, Q);
          else run_bc_tile2<PASS, false, CUT, false, 3>(I2, jt, ti, tj, V0, V1, K, Q);
        }
        if (Q.n >= 32) cf_drain<PASS>(Q, lane);  // a pair for every lane
        t0.a0 = ti.a0.x; t0.a1 = ti.a1.x; t0.a2 = ti.a2.x;
        t1.a0 = ti.a0.y; t1.a1 = ti.a1.y; t1.a2 = ti.a2.y;
      }

      // j partials are back in their home lanes: flush them
      if (jvalid) {
        if (PASS == PASS_BORN) {
          if (tj.a0 != 0.f) atomic_add_fix(&a.born_acc[jg], to_fix_f(tj.a0, bscale));
        } else {
          atomic_add_fix(&a.fx[jg], to_fix_f(tj.a0, bscale));
          atomic_add_fix(&a.fy[jg], to_fix_f(tj.a1, bscale));
          atomic_add_fix(&a.fz[jg], to_fix_f(tj.a2, bscale));
          if (PASS == PASS_FORCE && K.use_gb)
            atomic_add_fix(&a.dedb_acc[jg], to_fix_f(tj.a3 * (-0.5f * J.rB), bscale));
        }
      }
      p0 += to_fix_f(t0.a0, bscale);
      q0 += to_fix_f(t1.a0, bscale);
      if (PASS != PASS_BORN) {
        p1 += to_fix_f(t0.a1, bscale); p2 += to_fix_f(t0.a2, bscale);
        q1 += to_fix_f(t1.a1, bscale); q2 += to_fix_f(t1.a2, bscale);
      }
      if (PASS == PASS_FORCE) {
        p3 += to_fix_f(t0.a3 * (-0.5f * I0.rB), bscale);
        q3 += to_fix_f(t1.a3 * (-0.5f * I1.rB), bscale);
      }
    }

    if (PASS == PASS_BORN) {
      if (iv0 && p0 != 0) atomic_add_fix(&a.born_acc[ig0], p0);
      if (iv1 && q0 != 0) atomic_add_fix(&a.born_acc[ig1], q0);
      if (sys_items) {
        // count the item as summed: first the warp's queued closed-form
        // pairs, which may belong to it, then a release fence
        if (Q.n > 0) cf_drain<PASS>(Q, lane);
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicAdd(&a.sys_done[item.sys], 1);
      }
    } else {
      if (iv0) {
        atomic_add_fix(&a.fx[ig0], p0); atomic_add_fix(&a.fy[ig0], p1); atomic_add_fix(&a.fz[ig0], p2);
        if (PASS == PASS_FORCE && K.use_gb) atomic_add_fix(&a.dedb_acc[ig0], p3);
      }
      if (iv1) {
        atomic_add_fix(&a.fx[ig1], q0); atomic_add_fix(&a.fy[ig1], q1); atomic_add_fix(&a.fz[ig1], q2);
        if (PASS == PASS_FORCE && K.use_gb) atomic_add_fix(&a.dedb_acc[ig1], q3);
      }
    }
  }
  if constexpr (PASS != PASS_FORCE) {
    if (Q.n > 0) cf_drain<PASS>(Q, lane);
  }
  if (lane == 0 && atomicAdd(&a.sched[1], 1) == nwarps - 1) {
    // every warp has stopped taking items: reset for the next launch
    a.sched[0] = 0;
    a.sched[1] = 0;
  }
}

// The force pass with four i-blocks per warp: work items (system, i-block
// ib with ib % 4 == 0, j-blocks [jb0, jb1)); lane l owns atom l of blocks
// ib .. ib + 3, in two packed pairs (ib, ib + 1) and (ib + 2, ib + 3) that
// share every step's j atom.  Tiles below the diagonal (j-block before an
// i-block) are masked to zero, and each pair's sums, masks and exclusions
// are those of the two-block kernel's tile for the same blocks, so the
// forces and dE/dB are the same bit for bit (j-side sums of the two pairs
// are added in fixed point before their one atomic).
template <bool CUT, bool ALL, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) force4_kernel(const __grid_constant__ PairArgs a) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  TileConst K;
  K.use_gb = ALL || (a.terms & PB2_USE_GB) != 0;
  K.use_lj = ALL || (a.terms & PB2_USE_LJ) != 0;
  K.use_coul = ALL || (a.terms & PB2_USE_COULOMB) != 0;
  K.src = (lane + 1) & 31;
  K.lane = lane;
  constexpr int kWarps = THREADS / 32;
  __shared__ JTile s_jt[kWarps];
  __shared__ long long s_ps[kWarps][16][32];
  JTile &jt = s_jt[threadIdx.x >> 5];
  long long *ps = &s_ps[threadIdx.x >> 5][0][lane];
  const uint32_t diag_mask = lane == 31 ? 0u : (0xffffffffu << (lane + 1));
  const float bscale = (float)kForceScale;
  const int n_items = a.item_count ? *a.item_count : a.n_items;
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(&a.sched[0], 1);
    it = __shfl_sync(kFull, it, 0);
    if (it >= n_items) break;
    const TileItem item = a.items[it];
    const SysInfo &S = a.sys[item.sys];
    const int n = S.n, off = S.off;
    K.cut2 = S.cutoff2; K.gcut2 = S.gb_cutoff2; K.bcut2 = S.born_cut2;
    K.pref = S.pref; K.kcoul = S.kcoul; K.lj14 = S.lj14; K.coul14 = S.coul14;
    const int ib = item.iblk;
    int gib[4], ig[4];
    bool has[4], iv[4];
    PData I[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      has[k] = ib + k < S.nblk;
      gib[k] = S.blk_base + (has[k] ? ib + k : ib);
      const int il = (ib + k) * 32 + lane;
      iv[k] = il < n;  // false whenever !has[k]
      ig[k] = off + (iv[k] ? il : n - 1);
      load_pdata(a, ig[k], PASS_FORCE, K.use_gb, S.ro_max, I[k]);
    }
    const float reach2 = CUT ? ((K.gcut2 == 0.f || K.cut2 == 0.f) ? 0.f : fmaxf(K.gcut2, K.cut2)) : 0.f;
    FData2 IF[2];
    float rB[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) rB[k] = I[k].rB;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const PData &P0 = I[2 * h], &P1 = I[2 * h + 1];
      IF[h] = {make_float2(P0.x, P1.x), make_float2(P0.y, P1.y), make_float2(P0.z, P1.z),
               make_float2(P0.hs, P1.hs), make_float2(P0.se, P1.se),
               make_float2(P0.B, P1.B), make_float2(P0.iB, P1.iB),
               make_float2(2.f * K.pref * P0.q, 2.f * K.pref * P1.q),
               make_float2(K.kcoul * P0.q, K.kcoul * P1.q)};
    }
    // exclusion entries: ent[h], lanes 0-15 for block ib + 2h, 16-31 for ib + 2h + 1
    int2 ent[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      ent[h] = make_int2(-1, -1);
      if (lane < kExclPerBlock) {
        if (has[2 * h]) ent[h] = a.excl_ent[gib[2 * h] * kExclPerBlock + lane];
      } else if (has[2 * h + 1]) {
        ent[h] = a.excl_ent[gib[2 * h + 1] * kExclPerBlock + lane - kExclPerBlock];
      }
    }
    // i-side fixed-point sums, (block, component) x lane, in shared memory
    // (registers hold the two packed pairs' data and sums)
#pragma unroll
    for (int k = 0; k < 16; ++k) ps[32 * k] = 0;
    for (int jb = item.jb0; jb < item.jb1; ++jb) {
      const int gjb = S.blk_base + jb;
      if (CUT && reach2 > 0.f) {
        // smallest box separation over the blocks with a tile on or above the diagonal
        float d2 = box_dist2(a.bbox, gib[0], gjb);
#pragma unroll
        for (int k = 1; k < 4; ++k)
          if (has[k] && jb >= ib + k) d2 = fminf(d2, box_dist2(a.bbox, gib[k], gjb));
        if (d2 >= reach2) continue;  // no pair within reach
      }
      const int jl0 = jb * 32;
      const int jl = jl0 + lane;
      const bool jvalid = jl < n;
      const int jg = off + (jvalid ? jl : n - 1);
      PData J;
      load_pdata(a, jg, PASS_FORCE, K.use_gb, S.ro_max, J);
      __syncwarp();  // every lane is done with the previous tile's j data
      store_j<PASS_FORCE>(jt, lane, J);
      __syncwarp();
      const int nj = n - jl0;
      const uint32_t jmask = nj >= 32 ? 0xffffffffu : ((1u << nj) - 1u);
      uint32_t C[4], V[4];
      bool all_full = true;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        C[k] = iv[k] ? jmask : 0u;
        if (jb == ib + k) C[k] &= diag_mask;
        else if (jb < ib + k) C[k] = 0u;  // below the diagonal: another tile's pairs
        V[k] = rotr32(C[k], lane);
        all_full = all_full && C[k] == 0xffffffffu;
      }
      const bool full = __all_sync(kFull, all_full);
      uint32_t E[4] = {0u, 0u, 0u, 0u}, Sx[4] = {0u, 0u, 0u, 0u};
      bool any_hit = false;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const unsigned hit = __ballot_sync(kFull, ent[h].x == jb);
        const unsigned hit0 = hit & 0xffffu, hit1 = hit & 0xffff0000u;
        if (hit0) {
          const int roff = __shfl_sync(kFull, ent[h].y, __ffs(hit0) - 1);
          const ExclRow r = a.excl_rows[roff + lane];
          E[2 * h] = rotr32(r.excl, lane); Sx[2 * h] = rotr32(r.s14, lane);
        }
        if (hit1) {
          const int roff = __shfl_sync(kFull, ent[h].y, __ffs(hit1) - 1);
          const ExclRow r = a.excl_rows[roff + lane];
          E[2 * h + 1] = rotr32(r.excl, lane); Sx[2 * h + 1] = rotr32(r.s14, lane);
        }
        any_hit = any_hit || hit != 0u;
      }
      const ForceMasks Ma = force_masks(V[0], V[1], E[0], E[1], Sx[0], Sx[1]);
      const ForceMasks Mb = force_masks(V[2], V[3], E[2], E[3], Sx[2], Sx[3]);
      Acc2F tf[2];
#pragma unroll
      for (int h = 0; h < 2; ++h)
        tf[h] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      Acc tja = {0.f, 0.f, 0.f, 0.f}, tjb = {0.f, 0.f, 0.f, 0.f};
      if (any_hit) run_force_tile4<CUT, false, true>(IF[0], IF[1], jt, tf[0], tf[1], tja, tjb, Ma, Mb, K);
      else if (!full) run_force_tile4<CUT, false, false>(IF[0], IF[1], jt, tf[0], tf[1], tja, tjb, Ma, Mb, K);
      else run_force_tile4<CUT, true, false>(IF[0], IF[1], jt, tf[0], tf[1], tja, tjb, Ma, Mb, K);

      // j partials are back in their home lanes: both pairs' sums, added in
      // fixed point, in one atomic per component
      if (jvalid) {
        atomic_add_fix(&a.fx[jg], to_fix_f(tja.a0, bscale) + to_fix_f(tjb.a0, bscale));
        atomic_add_fix(&a.fy[jg], to_fix_f(tja.a1, bscale) + to_fix_f(tjb.a1, bscale));
        atomic_add_fix(&a.fz[jg], to_fix_f(tja.a2, bscale) + to_fix_f(tjb.a2, bscale));
        if (K.use_gb)
          atomic_add_fix(&a.dedb_acc[jg], to_fix_f(tja.a3 * (-0.5f * J.rB), bscale) +
                                              to_fix_f(tjb.a3 * (-0.5f * J.rB), bscale));
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        long long *p0 = ps + 32 * 4 * (2 * h), *p1 = ps + 32 * 4 * (2 * h + 1);
        p0[0] += to_fix_f(tf[h].a0.x, bscale); p0[32] += to_fix_f(tf[h].a1.x, bscale);
        p0[64] += to_fix_f(tf[h].a2.x, bscale); p0[96] += to_fix_f(tf[h].a3.x * (-0.5f * rB[2 * h]), bscale);
        p1[0] += to_fix_f(tf[h].a0.y, bscale); p1[32] += to_fix_f(tf[h].a1.y, bscale);
        p1[64] += to_fix_f(tf[h].a2.y, bscale); p1[96] += to_fix_f(tf[h].a3.y * (-0.5f * rB[2 * h + 1]), bscale);
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (iv[k]) {
        const long long *pk = ps + 32 * 4 * k;
        atomic_add_fix(&a.fx[ig[k]], pk[0]); atomic_add_fix(&a.fy[ig[k]], pk[32]);
        atomic_add_fix(&a.fz[ig[k]], pk[64]);
        if (K.use_gb) atomic_add_fix(&a.dedb_acc[ig[k]], pk[96]);
      }
    }
  }
  if (lane == 0 && atomicAdd(&a.sched[1], 1) == nwarps - 1) {
    a.sched[0] = 0;
    a.sched[1] = 0;
  }
}

// Per-block bounding boxes of the float32 positions: one warp per block.
__global__ void bbox_kernel(const SysInfo *sys, const int32_t *blk_sys, const float4 *posq,
                            float4 *bbox, int n_blocks, const float4 *pl_ref, int32_t *pl_ctl) {
  const int lane = threadIdx.x & 31;
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  bool moved = false;  // this lane saw an atom beyond skin / 2 of the pair list's reference
  for (int b = w; b < n_blocks; b += nw) {
    const SysInfo &S = sys[blk_sys[b]];
    const int lb = b - S.blk_base;
    const int l = lb * 32 + lane;
    const int i = S.off + (l < S.n ? l : lb * 32);
    const float4 p = posq[i];
    if (pl_ref) {
      const float4 r = pl_ref[i];
      const float dx = p.x - r.x, dy = p.y - r.y, dz = p.z - r.z;
      moved |= (double)fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > S.skin_half2;
    }
    float lo[3] = {p.x, p.y, p.z}, hi[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = fminf(lo[c], __shfl_xor_sync(kFull, lo[c], o));
        hi[c] = fmaxf(hi[c], __shfl_xor_sync(kFull, hi[c], o));
      }
    if (lane == 0) {
      bbox[2 * b] = make_float4(lo[0], lo[1], lo[2], 0.f);
      bbox[2 * b + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
    }
  }
  if (pl_ctl && __any_sync(kFull, moved) && lane == 0) atomicOr(&pl_ctl[PL_DIRTY], 1);
}

// Born radii from the descreening sums, plus the per-atom GB self term
// (q_i^2 / B_i, generalized_born.py:200-206, :410-413) and ACE
// (:600-648), written as the initial value of dE/dB.  Clears the sums.
// FP64: one evaluation per atom.


// --------------------------------------------------------------- launchers

// Block shapes compiled for each pass (threads, min blocks per SM); entry 0
// is the default.  The descreening pass holds fewer registers, so its
// shapes allow more resident blocks.
struct Shape {
  int threads, minb;
};
constexpr Shape kShapes[3][kShapesPerPass] = {
    {{256, 3}, {256, 2}, {128, 6}},   // descreening
    {{256, 2}, {128, 4}, {128, 5}},   // force
    {{256, 2}, {128, 4}, {128, 5}}};  // chain rule

template <int PASS, bool CUT, bool ALL, int SH>
static void launch_one(const PairArgs &a, int grid, cudaStream_t st) {
  constexpr Shape sh = kShapes[PASS][SH];
  tile2_kernel<PASS, CUT, ALL, sh.threads, sh.minb><<<grid, sh.threads, 0, st>>>(a);
}

template <int PASS, bool CUT, bool ALL>
static void launch_shaped(const PairArgs &a, int grid, int shape, cudaStream_t st) {
  switch (shape) {
    case 1: launch_one<PASS, CUT, ALL, 1>(a, grid, st); break;
    case 2: launch_one<PASS, CUT, ALL, 2>(a, grid, st); break;
    default: launch_one<PASS, CUT, ALL, 0>(a, grid, st);
  }
}

cudaError_t launch_tiles(int pass, const PairArgs &a, int grid, int shape, cudaStream_t st) {
  switch (pass) {
    case PASS_BORN:
      if (a.cut) launch_shaped<PASS_BORN, true, false>(a, grid, shape, st);
      else launch_shaped<PASS_BORN, false, false>(a, grid, shape, st);
      break;
    case PASS_CHAIN:
      if (a.cut) launch_shaped<PASS_CHAIN, true, false>(a, grid, shape, st);
      else launch_shaped<PASS_CHAIN, false, false>(a, grid, shape, st);
      break;
    default: {
      const int all_terms = PB2_USE_GB | PB2_USE_LJ | PB2_USE_COULOMB;
      const bool all = (a.terms & all_terms) == all_terms;
      if (a.cut) {
        if (all) launch_shaped<PASS_FORCE, true, true>(a, grid, shape, st);
        else launch_shaped<PASS_FORCE, true, false>(a, grid, shape, st);
      } else {
        if (all) launch_shaped<PASS_FORCE, false, true>(a, grid, shape, st);
        else launch_shaped<PASS_FORCE, false, false>(a, grid, shape, st);
      }
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_bbox(const SysInfo *sys, const int32_t *blk_sys, const float4 *posq, float4 *bbox,
                        int n_blocks, cudaStream_t st, const float4 *pl_ref, int32_t *pl_ctl) {
  if (n_blocks <= 0) return cudaSuccess;
  const int grid = (n_blocks + 7) / 8;
  bbox_kernel<<<grid, 256, 0, st>>>(sys, blk_sys, posq, bbox, n_blocks, pl_ref, pl_ctl);
  return cudaGetLastError();
}

cudaError_t launch_born_finalize(const FinalizeArgs &a, cudaStream_t st) {
  if (a.n_total <= 0) return cudaSuccess;
  const int grid = (a.n_total + 255) / 256;
  born_finalize<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

template <int PASS, bool CUT, bool ALL, int SH>
static int occ_one() {
  constexpr Shape sh = kShapes[PASS][SH];
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, tile2_kernel<PASS, CUT, ALL, sh.threads, sh.minb>,
                                                sh.threads, 0);
  return blocks;
}

template <int PASS, bool CUT, bool ALL>
static int occ_shaped(int shape) {
  switch (shape) {
    case 1: return occ_one<PASS, CUT, ALL, 1>();
    case 2: return occ_one<PASS, CUT, ALL, 2>();
    default: return occ_one<PASS, CUT, ALL, 0>();
  }
}

// Four-block force kernel: its own block shapes (more registers per thread
// for the four i atoms' data and sums).
constexpr Shape kShapes4[kShapesPerPass] = {{128, 3}, {128, 2}, {64, 5}};

template <bool CUT, bool ALL, int SH>
static void launch_force4_one(const PairArgs &a, int grid, cudaStream_t st) {
  constexpr Shape sh = kShapes4[SH];
  force4_kernel<CUT, ALL, sh.threads, sh.minb><<<grid, sh.threads, 0, st>>>(a);
}
template <bool CUT, bool ALL>
static void launch_force4_shaped(const PairArgs &a, int grid, int shape, cudaStream_t st) {
  switch (shape) {
    case 1: launch_force4_one<CUT, ALL, 1>(a, grid, st); break;
    case 2: launch_force4_one<CUT, ALL, 2>(a, grid, st); break;
    default: launch_force4_one<CUT, ALL, 0>(a, grid, st);
  }
}
cudaError_t launch_force4(const PairArgs &a, int grid, int shape, cudaStream_t st) {
  if (grid <= 0) return cudaSuccess;
  const bool all = (a.terms & (PB2_USE_GB | PB2_USE_LJ | PB2_USE_COULOMB)) ==
                   (PB2_USE_GB | PB2_USE_LJ | PB2_USE_COULOMB);
  if (a.cut) {
    if (all) launch_force4_shaped<true, true>(a, grid, shape, st);
    else launch_force4_shaped<true, false>(a, grid, shape, st);
  } else {
    if (all) launch_force4_shaped<false, true>(a, grid, shape, st);
    else launch_force4_shaped<false, false>(a, grid, shape, st);
  }
  return cudaGetLastError();
}
template <bool CUT, bool ALL, int SH>
static int occ_force4_one() {
  constexpr Shape sh = kShapes4[SH];
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, force4_kernel<CUT, ALL, sh.threads, sh.minb>, sh.threads, 0);
  return blocks;
}
template <bool CUT, bool ALL>
static int occ_force4_shaped(int shape) {
  switch (shape) {
    case 1: return occ_force4_one<CUT, ALL, 1>();
    case 2: return occ_force4_one<CUT, ALL, 2>();
    default: return occ_force4_one<CUT, ALL, 0>();
  }
}
int force4_occupancy(bool cut, int shape) {
  return cut ? std::min(occ_force4_shaped<true, true>(shape), occ_force4_shaped<true, false>(shape))
             : std::min(occ_force4_shaped<false, true>(shape), occ_force4_shaped<false, false>(shape));
}
int force4_shape(int shape, int *threads, int *min_blocks) {
  if (shape < 0 || shape >= kShapesPerPass) return -1;
  *threads = kShapes4[shape].threads;
  *min_blocks = kShapes4[shape].minb;
  return 0;
}

int tile_shape(int pass, int shape, int *threads, int *min_blocks) {
  if (pass < 0 || pass > 2 || shape < 0 || shape >= kShapesPerPass) return -1;
  *threads = kShapes[pass][shape].threads;
  *min_blocks = kShapes[pass][shape].minb;
  return 0;
}

int tile_kernel_warps(int pass, int shape) {
  int t = 256, m = 0;
  tile_shape(pass, shape, &t, &m);
  return t / 32;
}

int tile_kernel_occupancy(int pass, bool cut, int shape) {
  int blocks;
  if (pass == PASS_BORN)
    blocks = cut ? occ_shaped<PASS_BORN, true, false>(shape) : occ_shaped<PASS_BORN, false, false>(shape);
  else if (pass == PASS_CHAIN)
    blocks = cut ? occ_shaped<PASS_CHAIN, true, false>(shape) : occ_shaped<PASS_CHAIN, false, false>(shape);
  else if (cut)
    blocks = std::min(occ_shaped<PASS_FORCE, true, false>(shape), occ_shaped<PASS_FORCE, true, true>(shape));
  else
    blocks = std::min(occ_shaped<PASS_FORCE, false, false>(shape), occ_shaped<PASS_FORCE, false, true>(shape));
  return blocks > 0 ? blocks : 1;
}

}  // namespace pb2
