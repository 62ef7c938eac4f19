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
// Mapping: one warp per work item (system, i-block, range of j-blocks);
// lane l owns atom i = 32*iblk + l for the whole item; the j-block's data and
// j-side accumulators rotate through the lanes by shuffles, so lane l meets
// j-lane (l + k) mod 32 at step k of a fully unrolled 32-step loop.  Per
// tile, each lane's pair-validity and exclusion bit masks are rotated by its
// lane index once, so step k tests bit k.  A per-block bounding box sorts
// tiles: tiles whose boxes are at least the far-field distance apart
// evaluate the OBC integral by its series without per-pair branches, and
// (with a cutoff) tiles beyond every cutoff are skipped.
//
// Arithmetic is FP32; per-tile partial sums are converted to 64-bit fixed
// point and combined with integer atomics, so results do not depend on
// scheduling order.
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"
#include "pb2_pairmath.cuh"

// Unroll factor of the 32-step rotation loop (code size against loop
// overhead; the instruction cache favours a partial unroll).
#ifndef PB2_UNROLL
#define PB2_UNROLL 4
#endif
// Minimum resident blocks per SM asked of the register allocator (bounds
// registers per thread at 65536 / (256 * PB2_MINB)).
#ifndef PB2_MINB
#define PB2_MINB 3
#endif

namespace pb2 {

constexpr int kUnroll = PB2_UNROLL;

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

// Far-field OBC integral and derivative with K series terms (valid when
// r - s >= rho~ and (s/r)^2 is inside K's domain; the caller guarantees it).
template <int K>
__device__ __forceinline__ float obc_far_val(float s, float inv_r) {
  const float t = s * inv_r;
  const float u = t * t;
  return t * u * inv_r * obc_series_val_n<K>(u);
}
template <int K>
__device__ __forceinline__ float obc_far_der(float s, float inv_r, float inv_r2) {
  const float t = s * inv_r;
  const float u = t * t;
  return -t * u * inv_r2 * obc_series_der_n<K + 1>(u);
}

struct PData {  // per-atom data a lane holds (its i atom, or the j atom passing through)
  float x, y, z, q, hs, se, ro, sr, B, iB, dedi;  // iB = sqrt(log2 e / 4) / B
};

// Both directions of a pair inside the near-tile series' domain:
// r - s >= rho~ and (s/r)^2 <= kSeriesUNear.
__device__ __forceinline__ bool far_pair(float r, float r2, const PData &I, const PData &J) {
  const float lim = kSeriesUNear * r2;
  return (J.sr * J.sr <= lim) && (I.sr * I.sr <= lim) && (r - J.sr >= I.ro) && (r - I.sr >= J.ro);
}

// 4 / log2(e), and sqrt(log2(e) / 4): the force pass stores 1/B pre-scaled by
// sqrt(log2(e)/4) so that exp(-r^2 / (4 B_i B_j)) = exp2(-r^2 iB_i iB_j).
constexpr float kInvQuarterLog2e = 2.7725887222397811f;
constexpr float kSqrtQuarterLog2e = 0.60056120439322491f;
struct Acc {
  float a0, a1, a2, a3;
};
struct TileConst {
  float cut2, gcut2, pref, kcoul, lj14, coul14;
  bool use_gb, use_lj, use_coul;
  int src;
};

// One 32 x 32 tile.  V: rotated validity mask (bit k = pair at step k);
// E, S14: rotated exclusion / 1-4 masks.  FAR: series OBC without checks;
// NT: series terms (value; the derivative takes NT + 1).
template <int PASS, bool FAR, bool CUT, bool FULL, bool EXCL, int NT = 10>
__device__ __forceinline__ void run_tile(const PData &I, PData &J, Acc &ti, Acc &tj, uint32_t V,
                                         uint32_t E, uint32_t S14, const TileConst &K) {
  const int src = K.src;
#pragma unroll kUnroll
  for (int k = 0; k < 32; ++k) {
    bool ok = FULL ? true : ((V >> k) & 1u);
    const float dx = I.x - J.x, dy = I.y - J.y, dz = I.z - J.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (PASS != PASS_FORCE && CUT) ok = ok && (K.gcut2 == 0.f || r2 < K.gcut2);
    if (PASS == PASS_BORN || PASS == PASS_CHAIN) {
      // All lanes evaluate (results of invalid pairs are discarded), so the
      // warp vote below is reached by every lane of the warp.
      const float inv_r = rsqrtf(r2);
      const float inv_r2 = inv_r * inv_r;
      float vij, vji;
      if (PASS == PASS_BORN) {
        vij = obc_far_val<NT>(J.sr, inv_r);
        vji = obc_far_val<NT>(I.sr, inv_r);
      } else {
        vij = obc_far_der<NT>(J.sr, inv_r, inv_r2);
        vji = obc_far_der<NT>(I.sr, inv_r, inv_r2);
      }
      if (!FAR) {
        // near tile: the series holds for most pairs; the closed form runs
        // only for lanes whose pair lies inside the far-field bound
        const float r = r2 * inv_r;
        const bool need = ok && !far_pair(r, r2, I, J);
        if (__any_sync(kFull, need)) {
          if (need) {
            if (PASS == PASS_BORN) {
              vij = obc_integral(r, inv_r, I.ro, J.sr);
              vji = obc_integral(r, inv_r, J.ro, I.sr);
            } else {
              vij = obc_integral_dr(r, inv_r, I.ro, J.sr);
              vji = obc_integral_dr(r, inv_r, J.ro, I.sr);
            }
          }
        }
      }
      if (ok) {
        if (PASS == PASS_BORN) {
          ti.a0 += vij;
          tj.a0 += vji;
        } else {
          const float g = (I.dedi * vij + J.dedi * vji) * inv_r;
          ti.a0 -= g * dx; ti.a1 -= g * dy; ti.a2 -= g * dz;
          tj.a0 += g * dx; tj.a1 += g * dy; tj.a2 += g * dz;
        }
      }
    } else if (ok) {
      {
        float g = 0.f;
        const float qq = I.q * J.q;
        if (K.use_gb && (!CUT || K.gcut2 == 0.f || r2 < K.gcut2)) {
          const float w = r2 * (I.iB * J.iB);  // r^2 log2(e) / (4 B_i B_j)
          const float ex = exp2f(-w);
          const float f2 = fmaf(I.B * J.B, ex, r2);
          const float inv_f = rsqrtf(f2);
          const float inv_f3 = inv_f * inv_f * inv_f;
          const float pq = K.pref * qq;
          g = 2.0f * pq * (1.0f - 0.25f * ex) * inv_f3;
          const float c = -pq * ex * fmaf(w, kInvQuarterLog2e * 0.25f, 1.0f) * inv_f3;
          ti.a3 += c * J.B;
          tj.a3 += c * I.B;
        }
        const bool excluded = EXCL ? ((E >> k) & 1u) : false;
        if (!excluded && (K.use_lj || K.use_coul) && (!CUT || K.cut2 == 0.f || r2 < K.cut2)) {
          const bool is14 = EXCL ? ((S14 >> k) & 1u) : false;
          const float inv_r = rsqrtf(r2);
          const float inv_r2 = inv_r * inv_r;
          if (K.use_coul) {
            const float ec = K.kcoul * qq * (is14 ? K.coul14 : 1.0f) * inv_r;
            g += ec * inv_r2;
          }
          if (K.use_lj) {
            const float sig = I.hs + J.hs;
            const float eps = I.se * J.se * (is14 ? K.lj14 : 1.0f);
            const float sr2 = sig * sig * inv_r2;
            const float s6 = sr2 * sr2 * sr2;
            g += 24.0f * eps * s6 * (2.0f * s6 - 1.0f) * inv_r2;
          }
        }
        ti.a0 += g * dx; ti.a1 += g * dy; ti.a2 += g * dz;
        tj.a0 -= g * dx; tj.a1 -= g * dy; tj.a2 -= g * dz;
      }
    }
    // rotate the j data and j partials one lane down
    J.x = shfl_next(J.x, src); J.y = shfl_next(J.y, src); J.z = shfl_next(J.z, src);
    tj.a0 = shfl_next(tj.a0, src);
    if (PASS == PASS_BORN) {
      J.sr = shfl_next(J.sr, src);
      if (!FAR) J.ro = shfl_next(J.ro, src);
    } else if (PASS == PASS_CHAIN) {
      J.sr = shfl_next(J.sr, src);
      if (!FAR) J.ro = shfl_next(J.ro, src);
      J.dedi = shfl_next(J.dedi, src);
      tj.a1 = shfl_next(tj.a1, src); tj.a2 = shfl_next(tj.a2, src);
    } else {
      J.q = shfl_next(J.q, src);
      if (K.use_lj) { J.hs = shfl_next(J.hs, src); J.se = shfl_next(J.se, src); }
      tj.a1 = shfl_next(tj.a1, src); tj.a2 = shfl_next(tj.a2, src);
      if (K.use_gb) {
        J.B = shfl_next(J.B, src); J.iB = shfl_next(J.iB, src);
        tj.a3 = shfl_next(tj.a3, src);
      }
    }
  }
}

__device__ __forceinline__ void load_pdata(const PairArgs &a, int g, int pass, bool use_gb, PData &P) {
  const float4 p = a.posq[g], c = a.par[g];
  P.x = p.x; P.y = p.y; P.z = p.z; P.q = p.w;
  P.hs = c.x; P.se = c.y; P.ro = c.z; P.sr = c.w;
  P.B = P.iB = P.dedi = 0.f;
  if ((pass == PASS_FORCE && use_gb) || pass == PASS_CHAIN) {
    const float4 b = a.born[g];
    P.B = b.x; P.iB = b.y * kSqrtQuarterLog2e;
    if (pass == PASS_CHAIN) P.dedi = (float)((double)a.dedb_acc[g] * kForceInv) * b.z;
  }
}

// Work items are handed out dynamically: each warp takes the next item from
// an atomic counter (items are sorted by cost, largest first), and the last
// warp to finish resets the counter for the next launch.
template <int PASS, bool CUT>
__global__ void __launch_bounds__(256, PB2_MINB) tile_kernel(const PairArgs a) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  TileConst K;
  K.use_gb = (a.terms & PB2_USE_GB) != 0;
  K.use_lj = (a.terms & PB2_USE_LJ) != 0;
  K.use_coul = (a.terms & PB2_USE_COULOMB) != 0;
  K.src = (lane + 1) & 31;
  const uint32_t diag_mask = lane == 31 ? 0u : (0xffffffffu << (lane + 1));

  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(&a.sched[0], 1);
    it = __shfl_sync(kFull, it, 0);
    if (it >= a.n_items) break;
    const TileItem item = a.items[it];
    const SysInfo &S = a.sys[item.sys];
    const int n = S.n, off = S.off;
    K.cut2 = S.cutoff2; K.gcut2 = S.gb_cutoff2;
    K.pref = S.pref; K.kcoul = S.kcoul; K.lj14 = S.lj14; K.coul14 = S.coul14;
    const float far2 = S.far2, far2_k8 = S.far2_k8, far2_k6 = S.far2_k6, far2_k4 = S.far2_k4;
    const int gib = S.blk_base + item.iblk;
    const int il = item.iblk * 32 + lane;
    const bool ivalid = il < n;
    const int ig = off + (ivalid ? il : n - 1);
    // largest distance at which this pass has any pair term (0: unbounded)
    float reach2 = 0.f;
    if (CUT) {
      if (PASS == PASS_FORCE) reach2 = (K.gcut2 == 0.f || K.cut2 == 0.f) ? 0.f : fmaxf(K.gcut2, K.cut2);
      else reach2 = K.gcut2;
    }
    PData I;
    load_pdata(a, ig, PASS, K.use_gb, I);
    int2 ent = make_int2(-1, -1);
    if (PASS == PASS_FORCE && lane < kExclPerBlock) ent = a.excl_ent[gib * kExclPerBlock + lane];

    long long ai0 = 0, ai1 = 0, ai2 = 0, ai3 = 0;  // i-side fixed-point sums

    for (int jb = item.jb0; jb < item.jb1; ++jb) {
      const int gjb = S.blk_base + jb;
      const float d2 = (CUT || PASS != PASS_FORCE) ? box_dist2(a.bbox, gib, gjb) : 0.f;
      if (CUT && reach2 > 0.f && d2 >= reach2) continue;  // no pair within reach
      const int jl0 = jb * 32;
      const int jl = jl0 + lane;
      const bool jvalid = jl < n;
      const int jg = off + (jvalid ? jl : n - 1);
      PData J;
      load_pdata(a, jg, PASS, K.use_gb, J);
      // pair validity of lane i with j-lane c: both exist, j > i on the diagonal
      const int nj = n - jl0;
      const uint32_t jmask = nj >= 32 ? 0xffffffffu : ((1u << nj) - 1u);
      uint32_t C = ivalid ? jmask : 0u;
      if (jb == item.iblk) C &= diag_mask;
      const uint32_t V = rotr32(C, lane);
      const bool full = __all_sync(kFull, C == 0xffffffffu);

      uint32_t E = 0u, S14 = 0u;
      bool excl = false;
      if (PASS == PASS_FORCE) {
        const unsigned hit = __ballot_sync(kFull, ent.x == jb);
        if (hit) {
          const int roff = __shfl_sync(kFull, ent.y, __ffs(hit) - 1);
          const ExclRow r = a.excl_rows[roff + lane];
          E = rotr32(r.excl, lane);
          S14 = rotr32(r.s14, lane);
          excl = true;
        }
      }
      Acc ti = {0.f, 0.f, 0.f, 0.f}, tj = {0.f, 0.f, 0.f, 0.f};
      if (PASS == PASS_FORCE) {
        if (excl || !full) run_tile<PASS, false, CUT, false, true>(I, J, ti, tj, V, E, S14, K);
        else run_tile<PASS, false, CUT, true, false>(I, J, ti, tj, V, E, S14, K);
      } else if (d2 >= far2_k4) {  // series length by the tiles' smallest separation
        run_tile<PASS, true, CUT, false, false, 4>(I, J, ti, tj, V, E, S14, K);
      } else if (d2 >= far2_k6) {
        run_tile<PASS, true, CUT, false, false, 6>(I, J, ti, tj, V, E, S14, K);
      } else if (d2 >= far2_k8) {
        run_tile<PASS, true, CUT, false, false, 8>(I, J, ti, tj, V, E, S14, K);
      } else if (d2 >= far2) {
        run_tile<PASS, true, CUT, false, false, 10>(I, J, ti, tj, V, E, S14, K);
      } else {
        run_tile<PASS, false, CUT, false, false, 10>(I, J, ti, tj, V, E, S14, K);
      }

      // j partials are back in their home lanes: flush them
      if (jvalid) {
        if (PASS == PASS_BORN) {
          if (tj.a0 != 0.f) atomic_add_fix(&a.born_acc[jg], to_fix_f(tj.a0, (float)kBornScale));
        } else {
          atomic_add_fix(&a.fx[jg], to_fix_f(tj.a0, (float)kForceScale));
          atomic_add_fix(&a.fy[jg], to_fix_f(tj.a1, (float)kForceScale));
          atomic_add_fix(&a.fz[jg], to_fix_f(tj.a2, (float)kForceScale));
          if (PASS == PASS_FORCE && K.use_gb)
            atomic_add_fix(&a.dedb_acc[jg], to_fix_f(tj.a3, (float)kForceScale));
        }
      }
      if (PASS == PASS_BORN) {
        ai0 += to_fix_f(ti.a0, (float)kBornScale);
      } else {
        ai0 += to_fix_f(ti.a0, (float)kForceScale);
        ai1 += to_fix_f(ti.a1, (float)kForceScale);
        ai2 += to_fix_f(ti.a2, (float)kForceScale);
        if (PASS == PASS_FORCE) ai3 += to_fix_f(ti.a3, (float)kForceScale);
      }
    }

    if (ivalid) {
      if (PASS == PASS_BORN) {
        if (ai0 != 0) atomic_add_fix(&a.born_acc[ig], ai0);
      } else {
        atomic_add_fix(&a.fx[ig], ai0);
        atomic_add_fix(&a.fy[ig], ai1);
        atomic_add_fix(&a.fz[ig], ai2);
        if (PASS == PASS_FORCE && K.use_gb) atomic_add_fix(&a.dedb_acc[ig], ai3);
      }
    }
  }
  if (lane == 0 && atomicAdd(&a.sched[1], 1) == nwarps - 1) {
    // every warp has stopped taking items: reset for the next launch
    a.sched[0] = 0;
    a.sched[1] = 0;
  }
}

// Per-block bounding boxes of the float32 positions: one warp per block.
__global__ void bbox_kernel(const SysInfo *sys, const int32_t *blk_sys, const float4 *posq,
                            float4 *bbox, int n_blocks) {
  const int lane = threadIdx.x & 31;
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int b = w; b < n_blocks; b += nw) {
    const SysInfo &S = sys[blk_sys[b]];
    const int lb = b - S.blk_base;
    const int l = lb * 32 + lane;
    const int i = S.off + (l < S.n ? l : lb * 32);
    const float4 p = posq[i];
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
}

// Born radii from the descreening sums, plus the per-atom GB self term
// (q_i^2 / B_i, generalized_born.py:200-206, :410-413) and ACE
// (:600-648), written as the initial value of dE/dB.  Clears the sums.
// FP64: one evaluation per atom.

__global__ void born_finalize(const FinalizeArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    const SysInfo &S = a.sys[s];
    const bool nl = S.clamp != 0;
    const double isum = (double)a.born_acc[i] * kBornInv;
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
}

// --------------------------------------------------------------- launchers

cudaError_t launch_tiles(int pass, const PairArgs &a, int grid, cudaStream_t st) {
  if (a.n_items <= 0) return cudaSuccess;
  const bool cut = a.cut != 0;
  switch (pass) {
    case PASS_BORN:
      if (cut) tile_kernel<PASS_BORN, true><<<grid, 256, 0, st>>>(a);
      else tile_kernel<PASS_BORN, false><<<grid, 256, 0, st>>>(a);
      break;
    case PASS_CHAIN:
      if (cut) tile_kernel<PASS_CHAIN, true><<<grid, 256, 0, st>>>(a);
      else tile_kernel<PASS_CHAIN, false><<<grid, 256, 0, st>>>(a);
      break;
    default:
      if (cut) tile_kernel<PASS_FORCE, true><<<grid, 256, 0, st>>>(a);
      else tile_kernel<PASS_FORCE, false><<<grid, 256, 0, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_bbox(const SysInfo *sys, const int32_t *blk_sys, const float4 *posq, float4 *bbox,
                        int n_blocks, cudaStream_t st) {
  if (n_blocks <= 0) return cudaSuccess;
  const int grid = (n_blocks + 7) / 8;
  bbox_kernel<<<grid, 256, 0, st>>>(sys, blk_sys, posq, bbox, n_blocks);
  return cudaGetLastError();
}

cudaError_t launch_born_finalize(const FinalizeArgs &a, cudaStream_t st) {
  if (a.n_total <= 0) return cudaSuccess;
  const int grid = (a.n_total + 255) / 256;
  born_finalize<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

template <int PASS>
static int occ(bool cut) {
  int blocks = 0;
  if (cut) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, tile_kernel<PASS, true>, 256, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, tile_kernel<PASS, false>, 256, 0);
  return blocks;
}

int tile_kernel_occupancy(int pass, bool cut) {
  const int blocks = pass == PASS_BORN ? occ<PASS_BORN>(cut)
                     : (pass == PASS_CHAIN ? occ<PASS_CHAIN>(cut) : occ<PASS_FORCE>(cut));
  return blocks > 0 ? blocks : 1;
}

}  // namespace pb2
