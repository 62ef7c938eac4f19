// Pair kernels of the implicit-solvent force evaluation.
//
// Three warp-tiled passes visit every unique pair (i < j) of every system
// once (Newton's third law), in 32 x 32 tiles:
//   born  : descreening sums I_i += I(r; rho~_i, s_j), I_j += I(r; rho~_j, s_i)
//           (prolix physics/generalized_born.py:32-94, :266-337);
//   force : GB polar pair term, direct Coulomb and Lennard-Jones energy and
//           force, plus dE_GB/dB for both atoms (generalized_born.py:97-208,
//           physics/optimization.py:21-297, analytical_forces.py:167-292);
//   chain : F -= (dE/dI_i dI_ij/dr + dE/dI_j dI_ji/dr) r^ , the Born-radius
//           chain rule (generalized_born.py:773-814).
// A per-atom pass between born and force turns the sums into Born radii and
// adds the self (q^2/B) and ACE terms.
//
// Mapping: one warp per work item (system, i-block, range of j-blocks);
// lane l owns atom i = 32*iblk + l for the whole item, and the j-block's data
// and j-side accumulators rotate through the lanes by shuffles, so lane l
// meets j-lane (l + k) mod 32 at step k.  Arithmetic is FP32; per-tile
// partial sums are converted to 64-bit fixed point and combined with integer
// atomics, so results do not depend on scheduling order.
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"
#include "pb2_pairmath.cuh"

namespace pb2 {


__device__ __forceinline__ float shfl_next(float v, int lane) {
  return __shfl_sync(kFull, v, (lane + 1) & 31);
}

template <int PASS>
__global__ void __launch_bounds__(256) tile_kernel(const PairArgs a) {
  const int lane = threadIdx.x & 31;
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const bool use_gb = (a.terms & PB2_USE_GB) != 0;
  const bool use_lj = (a.terms & PB2_USE_LJ) != 0;
  const bool use_coul = (a.terms & PB2_USE_COULOMB) != 0;

  for (int it = warp; it < a.n_items; it += nwarps) {
    const TileItem item = a.items[it];
    const SysInfo &S = a.sys[item.sys];
    const int n = S.n, off = S.off;
    const float cut2 = S.cutoff2;
    const float pref = S.pref, kcoul = S.kcoul, lj14 = S.lj14, coul14 = S.coul14;
    const int il = item.iblk * 32 + lane;
    const bool ivalid = il < n;
    const int ig = off + (ivalid ? il : n - 1);

    const float4 pi = a.posq[ig];
    const float4 ci = a.par[ig];
    float4 bi = make_float4(0.f, 0.f, 0.f, 0.f);
    float dedi_i = 0.f;
    if (PASS == PASS_FORCE && use_gb) bi = a.born[ig];
    if (PASS == PASS_CHAIN) {
      bi = a.born[ig];
      dedi_i = (float)((double)a.dedb_acc[ig] * kForceInv) * bi.z;
    }

    int2 ent = make_int2(-1, -1);
    if (PASS == PASS_FORCE && lane < kExclPerBlock)
      ent = a.excl_ent[(S.blk_base + item.iblk) * kExclPerBlock + lane];

    long long ai0 = 0, ai1 = 0, ai2 = 0, ai3 = 0;  // i-side fixed-point sums

    for (int jb = item.jb0; jb < item.jb1; ++jb) {
      const int jl0 = jb * 32;
      const int jl = jl0 + lane;
      const bool jvalid = jl < n;
      const int jg = off + (jvalid ? jl : n - 1);
      float4 pj = a.posq[jg];
      float4 cj = a.par[jg];
      float bjB = 0.f, bjI = 0.f, dedi_j = 0.f;
      if (PASS == PASS_FORCE && use_gb) {
        const float4 b = a.born[jg];
        bjB = b.x;
        bjI = b.y;
      }
      if (PASS == PASS_CHAIN) {
        const float4 b = a.born[jg];
        dedi_j = (float)((double)a.dedb_acc[jg] * kForceInv) * b.z;
      }

      uint32_t exm = 0u, s14m = 0u;
      if (PASS == PASS_FORCE) {
        const unsigned hit = __ballot_sync(kFull, ent.x == jb);
        if (hit) {
          const int src = __ffs(hit) - 1;
          const int roff = __shfl_sync(kFull, ent.y, src);
          const ExclRow r = a.excl_rows[roff + lane];
          exm = r.excl;
          s14m = r.s14;
        }
      }
      const bool diag = (jb == item.iblk);

      float ti0 = 0.f, ti1 = 0.f, ti2 = 0.f, ti3 = 0.f;  // i partials of this tile
      float tj0 = 0.f, tj1 = 0.f, tj2 = 0.f, tj3 = 0.f;  // j partials (rotate)

#pragma unroll 4
      for (int k = 0; k < 32; ++k) {
        const int jc = (lane + k) & 31;
        bool ok = ivalid && (jl0 + jc < n) && (!diag || jc > lane);
        const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (cut2 > 0.f) ok = ok && (r2 < cut2);
        if (ok) {
          if (PASS == PASS_BORN) {
            const float inv_r = rsqrtf(r2);
            const float r = r2 * inv_r;
            ti0 += obc_integral(r, inv_r, ci.z, cj.w);
            tj0 += obc_integral(r, inv_r, cj.z, ci.w);
          } else if (PASS == PASS_CHAIN) {
            const float inv_r = rsqrtf(r2);
            const float r = r2 * inv_r;
            const float dij = obc_integral_dr(r, inv_r, ci.z, cj.w);
            const float dji = obc_integral_dr(r, inv_r, cj.z, ci.w);
            const float g = (dedi_i * dij + dedi_j * dji) * inv_r;
            ti0 -= g * dx; ti1 -= g * dy; ti2 -= g * dz;
            tj0 += g * dx; tj1 += g * dy; tj2 += g * dz;
          } else {
            float g = 0.f;
            const float qq = pi.w * pj.w;
            if (use_gb) {
              const float inv_d = bi.y * bjI;
              const float ex = expf(-0.25f * r2 * inv_d);
              const float f2 = fmaf(bi.x * bjB, ex, r2);
              const float inv_f = rsqrtf(f2);
              const float inv_f3 = inv_f * inv_f * inv_f;
              const float pq = pref * qq;
              g = 2.0f * pq * (1.0f - 0.25f * ex) * inv_f3;
              const float c = -pq * ex * fmaf(0.25f * r2, inv_d, 1.0f) * inv_f3;
              ti3 += c * bjB;
              tj3 += c * bi.x;
            }
            const bool excluded = (exm >> jc) & 1u;
            if (!excluded && (use_lj || use_coul)) {
              const bool is14 = (s14m >> jc) & 1u;
              const float inv_r = rsqrtf(r2);
              const float inv_r2 = inv_r * inv_r;
              if (use_coul) {
                const float ec = kcoul * qq * (is14 ? coul14 : 1.0f) * inv_r;
                g += ec * inv_r2;
              }
              if (use_lj) {
                const float sig = ci.x + cj.x;
                const float eps = ci.y * cj.y * (is14 ? lj14 : 1.0f);
                const float sr2 = sig * sig * inv_r2;
                const float s6 = sr2 * sr2 * sr2;
                g += 24.0f * eps * s6 * (2.0f * s6 - 1.0f) * inv_r2;
              }
            }
            ti0 += g * dx; ti1 += g * dy; ti2 += g * dz;
            tj0 -= g * dx; tj1 -= g * dy; tj2 -= g * dz;
          }
        }
        // rotate the j data and j partials one lane down
        pj.x = shfl_next(pj.x, lane); pj.y = shfl_next(pj.y, lane);
        pj.z = shfl_next(pj.z, lane);
        tj0 = shfl_next(tj0, lane);
        if (PASS == PASS_BORN) {
          cj.z = shfl_next(cj.z, lane); cj.w = shfl_next(cj.w, lane);
        } else if (PASS == PASS_CHAIN) {
          cj.z = shfl_next(cj.z, lane); cj.w = shfl_next(cj.w, lane);
          dedi_j = shfl_next(dedi_j, lane);
          tj1 = shfl_next(tj1, lane); tj2 = shfl_next(tj2, lane);
        } else {
          pj.w = shfl_next(pj.w, lane);
          cj.x = shfl_next(cj.x, lane); cj.y = shfl_next(cj.y, lane);
          tj1 = shfl_next(tj1, lane); tj2 = shfl_next(tj2, lane);
          if (use_gb) {
            bjB = shfl_next(bjB, lane); bjI = shfl_next(bjI, lane);
            tj3 = shfl_next(tj3, lane);
          }
        }
      }

      // j partials are back in their home lanes: flush them
      if (jvalid) {
        if (PASS == PASS_BORN) {
          if (tj0 != 0.f) atomic_add_fix(&a.born_acc[jg], to_fix_f(tj0, (float)kBornScale));
        } else {
          atomic_add_fix(&a.fx[jg], to_fix_f(tj0, (float)kForceScale));
          atomic_add_fix(&a.fy[jg], to_fix_f(tj1, (float)kForceScale));
          atomic_add_fix(&a.fz[jg], to_fix_f(tj2, (float)kForceScale));
          if (PASS == PASS_FORCE && use_gb)
            atomic_add_fix(&a.dedb_acc[jg], to_fix_f(tj3, (float)kForceScale));
        }
      }
      if (PASS == PASS_BORN) {
        ai0 += to_fix_f(ti0, (float)kBornScale);
      } else {
        ai0 += to_fix_f(ti0, (float)kForceScale);
        ai1 += to_fix_f(ti1, (float)kForceScale);
        ai2 += to_fix_f(ti2, (float)kForceScale);
        if (PASS == PASS_FORCE) ai3 += to_fix_f(ti3, (float)kForceScale);
      }
    }

    if (ivalid) {
      if (PASS == PASS_BORN) {
        if (ai0 != 0) atomic_add_fix(&a.born_acc[ig], ai0);
      } else {
        atomic_add_fix(&a.fx[ig], ai0);
        atomic_add_fix(&a.fy[ig], ai1);
        atomic_add_fix(&a.fz[ig], ai2);
        if (PASS == PASS_FORCE && use_gb) atomic_add_fix(&a.dedb_acc[ig], ai3);
      }
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
    const bool nl = S.cutoff2 > 0.f;
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
      atomic_add_fix(&e[PB2_TERM_GB], to_fix(S.pref_d * q * q * inv_b, kForceScale));
      atomic_add_fix(&e[PB2_TERM_NONPOLAR], to_fix(ace, kForceScale));
    }
  }
}

// --------------------------------------------------------------- launchers

cudaError_t launch_tiles(int pass, const PairArgs &a, int grid, cudaStream_t st) {
  if (a.n_items <= 0) return cudaSuccess;
  switch (pass) {
    case PASS_BORN: tile_kernel<PASS_BORN><<<grid, 256, 0, st>>>(a); break;
    case PASS_CHAIN: tile_kernel<PASS_CHAIN><<<grid, 256, 0, st>>>(a); break;
    default: tile_kernel<PASS_FORCE><<<grid, 256, 0, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_born_finalize(const FinalizeArgs &a, cudaStream_t st) {
  if (a.n_total <= 0) return cudaSuccess;
  const int grid = (a.n_total + 255) / 256;
  born_finalize<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

int tile_kernel_occupancy(int pass) {
  int blocks = 0;
  switch (pass) {
    case PASS_BORN:
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, tile_kernel<PASS_BORN>, 256, 0);
      break;
    case PASS_CHAIN:
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, tile_kernel<PASS_CHAIN>, 256, 0);
      break;
    default:
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, tile_kernel<PASS_FORCE>, 256, 0);
  }
  return blocks > 0 ? blocks : 1;
}

}  // namespace pb2
