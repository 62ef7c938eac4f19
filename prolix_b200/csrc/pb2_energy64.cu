// FP64 energy evaluation (energy reporting, NVE drift checks; never part of
// an MD step, which needs forces only).
//
// Float32 coordinates bound the accuracy of a pair energy: a Lennard-Jones
// term moves by 12 dr/r for a coordinate rounding dr, about 1e-6 relative in
// a 20 A system, so per-term energies to 1e-6 need FP64 distances.  These
// kernels use the same tiles and work items as the force kernels, read the
// FP64 state, and evaluate the same formulas in double:
//   born   : descreening sums (prolix physics/generalized_born.py:211-263);
//   energy : GB polar pair terms, Coulomb and LJ energies
//            (generalized_born.py:118-208, physics/optimization.py:21-297).
// The Born radii of this path come from the FP64 sums (finalize in
// pb2_pair.cu with the same per-atom code).
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"

namespace pb2 {

__device__ __forceinline__ double shfl_next_d(double v, int lane) {
  return __shfl_sync(kFull, v, (lane + 1) & 31);
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ double obc_integral_d(double r, double rho, double s) {
  if (!(r + s > rho)) return 0.0;
  const double L = fmax(fmax(rho, fabs(r - s)), 1e-4);
  const double U = fmax(r + s, 1e-4);
  const double rs = fmax(r, 1e-4);
  const double il = 1.0 / L, iu = 1.0 / U;
  return 0.5 * (il - iu) + 0.25 * log(L / U) / rs + 0.125 * (r - s * s / rs) * (iu * iu - il * il);
}

template <int PASS>
__global__ void __launch_bounds__(256) energy64_kernel(const Energy64Args a) {
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
    const double cut2 = (double)S.cutoff2, gcut2 = (double)S.gb_cutoff2, bcut2 = (double)S.born_cut2;
    const double pref = S.pref_d, kcoul = S.kcoul_d;
    const int il = item.iblk * 32 + lane;
    const bool ivalid = il < n;
    const int ig = off + (ivalid ? il : n - 1);
    const double xi = a.x[ig], yi = a.y[ig], zi = a.z[ig];
    const double qi = a.q[ig], hsi = a.hs[ig], sei = a.se[ig], roi = a.ro[ig], sri = a.sr[ig];
    const double bi = (PASS == 1 && use_gb) ? a.born64[ig] : 0.0;
    int2 ent = make_int2(-1, -1);
    if (PASS == 1 && lane < kExclPerBlock)
      ent = a.excl_ent[(S.blk_base + item.iblk) * kExclPerBlock + lane];
    double acc_i = 0.0, e_gb = 0.0, e_coul = 0.0, e_lj = 0.0;

    for (int jb = item.jb0; jb < item.jb1; ++jb) {
      const int jl0 = jb * 32;
      const int jl = jl0 + lane;
      const bool jvalid = jl < n;
      const int jg = off + (jvalid ? jl : n - 1);
      double xj = a.x[jg], yj = a.y[jg], zj = a.z[jg];
      double qj = a.q[jg], hsj = a.hs[jg], sej = a.se[jg], roj = a.ro[jg], srj = a.sr[jg];
      double bj = (PASS == 1 && use_gb) ? a.born64[jg] : 0.0;
      uint32_t exm = 0u, s14m = 0u;
      if (PASS == 1) {
        const unsigned hit = __ballot_sync(kFull, ent.x == jb);
        if (hit) {
          const int roff = __shfl_sync(kFull, ent.y, __ffs(hit) - 1);
          const ExclRow r = a.excl_rows[roff + lane];
          exm = r.excl;
          s14m = r.s14;
        }
      }
      const bool diag = (jb == item.iblk);
      double acc_j = 0.0;
      for (int k = 0; k < 32; ++k) {
        const int jc = (lane + k) & 31;
        bool ok = ivalid && (jl0 + jc < n) && (!diag || jc > lane);
        const double dx = xi - xj, dy = yi - yj, dz = zi - zj;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (PASS == 0 && bcut2 > 0.0) ok = ok && (r2 < bcut2);
        if (ok) {
          if (PASS == 0) {
            const double r = sqrt(r2 + 1e-12);
            acc_i += obc_integral_d(r, roi, srj);
            acc_j += obc_integral_d(r, roj, sri);
          } else {
            const double qq = qi * qj;
            if (use_gb && (gcut2 == 0.0 || r2 < gcut2)) {
              const double rg2 = r2 + 1e-12;
              const double d = bi * bj;
              const double f = sqrt(rg2 + d * exp(-rg2 / (4.0 * d)));
              e_gb += 2.0 * pref * qq / f;
            }
            if (!((exm >> jc) & 1u) && (use_lj || use_coul) && (cut2 == 0.0 || r2 < cut2)) {
              const bool is14 = (s14m >> jc) & 1u;
              const double r = sqrt(r2);
              if (use_coul) e_coul += kcoul * qq * (is14 ? (double)S.coul14 : 1.0) / r;
              if (use_lj) {
                const double sig = hsi + hsj;
                const double sr2 = sig * sig / r2;
                const double s6 = sr2 * sr2 * sr2;
                e_lj += 4.0 * sei * sej * (is14 ? (double)S.lj14 : 1.0) * (s6 * s6 - s6);
              }
            }
          }
        }
        xj = shfl_next_d(xj, lane); yj = shfl_next_d(yj, lane); zj = shfl_next_d(zj, lane);
        if (PASS == 0) {
          roj = shfl_next_d(roj, lane); srj = shfl_next_d(srj, lane);
          acc_j = shfl_next_d(acc_j, lane);
        } else {
          qj = shfl_next_d(qj, lane); hsj = shfl_next_d(hsj, lane); sej = shfl_next_d(sej, lane);
          bj = shfl_next_d(bj, lane);
        }
      }
      if (PASS == 0 && jvalid && acc_j != 0.0) atomic_add_fix(&a.born_acc[jg], to_fix(acc_j, kBornScale));
    }
    if (PASS == 0) {
      if (ivalid && acc_i != 0.0) atomic_add_fix(&a.born_acc[ig], to_fix(acc_i, kBornScale));
    } else {
      e_gb = warp_sum_d(e_gb);
      e_coul = warp_sum_d(e_coul);
      e_lj = warp_sum_d(e_lj);
      if (lane == 0) {
        long long *e = a.energy + (size_t)item.sys * PB2_NTERMS;
        atomic_add_fix(&e[PB2_TERM_GB], to_fix(e_gb, kEnergyScale));
        atomic_add_fix(&e[PB2_TERM_COULOMB], to_fix(e_coul, kEnergyScale));
        atomic_add_fix(&e[PB2_TERM_LJ], to_fix(e_lj, kEnergyScale));
      }
    }
  }
}

cudaError_t launch_energy64(int pass, const Energy64Args &a, int grid, cudaStream_t st) {
  if (a.n_items <= 0) return cudaSuccess;
  if (pass == 0) energy64_kernel<0><<<grid, 256, 0, st>>>(a);
  else energy64_kernel<1><<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace pb2
