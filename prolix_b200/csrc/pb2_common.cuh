// Shared device-side definitions: batch layout in HBM, fixed-point
// accumulation, and launch helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "prolix_b200.h"

namespace pb2 {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Fixed-point scales.  Forces and dE/dB use 2^32 (range +-2.1e9, resolution
// 2.3e-10); the descreening sums use 2^40 (range +-8.4e6).
constexpr double kForceScale = 4294967296.0;
constexpr double kForceInv = 1.0 / 4294967296.0;
constexpr double kBornScale = 1099511627776.0;
constexpr double kBornInv = 1.0 / 1099511627776.0;
// Energies: 2^24 (range +-5.5e11 kcal/mol, resolution 6e-8 kcal/mol).
constexpr double kEnergyScale = 16777216.0;
constexpr double kEnergyInv = 1.0 / 16777216.0;
constexpr double kFixMax = 9.0e18;  // below 2^63: values beyond are flagged

// OBC II constants (prolix physics/generalized_born.py:18-21) and ACE
// constants (:628-647).
constexpr double kObcAlpha = 1.0, kObcBeta = 0.8, kObcGamma = 4.85;
constexpr double kDielOffset = 0.09;
constexpr double kAceCoeff = 28.3919551, kKjToKcal = 0.239006;

constexpr int kExclPerBlock = 16;  // distinct j-blocks with exclusions per i-block

// Per-system constants, one 168-byte record per system.  Pair kernels see
// positions relative to the system origin (its initial centroid), which keeps
// float32 coordinates small.
struct SysInfo {
  int32_t n;          // atoms
  int32_t off;        // first atom in the batch arrays
  int32_t nblk;       // 32-atom blocks
  int32_t blk_base;   // first block in the batch-wide block numbering
  float pref;         // P = -0.5 k_gb (1/eps_in - 1/eps_out)
  float kcoul;        // direct Coulomb constant
  float lj14, coul14; // 1-4 scales
  float cutoff2;      // LJ / Coulomb cutoff^2; 0: all pairs
  float far2;         // tiles at least this far apart (squared) take the far-field series
                      // of the widest tier; nearer tiles test each pair
  float gb_cutoff2;   // GB / descreening cutoff^2; 0: all pairs
  int32_t clamp;      // neighbour-list clamps on Born radii (GB cutoff set)
  float ro_max;       // largest rho~ = radius - offset of the system
  float born_cut2;    // descreening / chain-rule cutoff^2; 0: all pairs
  float tier2[2][3];  // [value, derivative][tier 0-2]: tiles at least this far apart
                      // (squared) evaluate that tier's series polynomial
  double kcoul_d;     // direct Coulomb constant in double (energy path)
  double pref_d;      // P in double (self / energy terms)
  double dt, half_dt; // tau
  double c1, c2;      // exp(-gamma dt), sqrt(1 - c1^2)
  double kT;
  double skin_half2;  // (skin/2)^2
  double ox, oy, oz;  // origin subtracted before the float32 pair kernels
};
static_assert(sizeof(SysInfo) == 168, "SysInfo layout");

// Work item of the tile kernels: tiles (iblk, jb) for jb in [jb0, jb1) of
// system sys.  Block indices are local to the system.
struct TileItem {
  int32_t sys, iblk, jb0, jb1;
};

// One row of the pair list: the even i-block iblk (with iblk + 1) of system
// sys; its live j-blocks are stored from pair_list_j[jbase], room for
// nblk - iblk of them.
struct PlRow {
  int32_t sys, iblk, jbase, pad;
};

// Exclusion masks of one (i-block, j-block) tile: per i row, bit c set when
// (row, col c) is excluded (1-2/1-3) or 1-4 scaled.
struct ExclRow {
  uint32_t excl, s14;
};

// Fixed-point helpers.  Conversion rounds to nearest; out-of-range values
// saturate in the hardware conversion and are flagged by the integrator.
__device__ __forceinline__ long long to_fix(double v, double scale) {
  return __double2ll_rn(v * scale);
}
__device__ __forceinline__ long long to_fix_f(float v, float scale) {
  return __float2ll_rn(v * scale);
}
__device__ __forceinline__ void atomic_add_fix(long long *addr, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(addr), static_cast<unsigned long long>(v));
}

// Asynchronous global -> shared copies (cp.async): a thread's copies land in
// groups, in order; cp_async_wait<N>() waits until at most N groups are in
// flight.  Source and destination aligned to the copy's size.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

}  // namespace pb2
