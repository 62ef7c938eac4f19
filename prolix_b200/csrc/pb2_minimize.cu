// Batched energy minimisation: restrained steepest descent and FIRE, all
// systems of the batch at once (prolix batched_simulate.py:682-960,
// `batched_minimize`).
//
// Forces come from the same force kernels as the MD step (fixed-point
// accumulators F); the minimiser adds a harmonic position restraint
//   E = k/2 sum_i m_i |r_i - r0_i|^2   (batched_simulate.py:675-679)
// on a per-atom selection m (all atoms, heavy atoms or backbone atoms) and
// zeroes non-finite force components (the reference's NaN guard).
//
// Steepest descent (batched_simulate.py:748-791): dr = F dt, |dr| capped at
// max_dx per atom, r += dr.
//
// FIRE (Bitzek et al., PRL 97, 170201 (2006), as jax_md 0.2.27
// minimize.fire_descent applies it; the reference calls it at
// batched_simulate.py:818-878): a velocity-Verlet step on momenta
//   p += dt/2 F; r += dt p / m; F = force(r); p += dt/2 F,
// then per system, with P = sum F.p, |F| = sqrt(sum F^2 + 1e-6), |p|:
//   p = p + alpha (F |p| / |F| - p);
//   P >= 0: n_pos += 1, else n_pos = 0;
//   P > 0 and n_pos > 5: dt = min(1.1 dt, dt_max), alpha *= 0.99;
//   P < 0: dt *= 0.5, alpha = 0.1, p = 0.
// The reference then caps each atom's displacement of the step at max_disp
// (0.1 A), scales its momentum by the same factor, keeps the force of the
// uncapped position, and returns the positions of the lowest force RMS seen
// at the start of an iteration.  The same order is kept here.
//
// Per-system sums run in one thread block per system in a fixed order, so
// the trajectory does not depend on scheduling.
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"

namespace pb2 {

constexpr int kMinThreads = 256;

__device__ __forceinline__ double fix_d(long long v) { return (double)v * kForceInv; }

// Restraint selection of atom i for the kind in par[kMinKind].
__device__ __forceinline__ bool selected(const MinArgs &a, int i) {
  const int kind = (int)a.par[kMinKind];
  if (kind == 0) return true;
  return ((a.sel[i] >> (kind - 1)) & 1u) != 0;
}

// F (physical, fixed point) + restraint force at the current position.
__device__ __forceinline__ void total_force(const MinArgs &a, int i, double f[3]) {
  const double k = a.par[kMinK];
  const bool m = k != 0.0 && selected(a, i);
  const size_t N = a.n_total;
  f[0] = fix_d(a.fx[i]);
  f[1] = fix_d(a.fy[i]);
  f[2] = fix_d(a.fz[i]);
  if (m) {
    f[0] -= k * (a.x[i] - a.x0[i]);
    f[1] -= k * (a.y[i] - a.x0[N + i]);
    f[2] -= k * (a.z[i] - a.x0[2 * N + i]);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if (!isfinite(f[c])) f[c] = 0.0;
}

__device__ __forceinline__ void put_posq(const MinArgs &a, int i) {
  const SysInfo &S = a.sys[a.atom_sys[i]];
  a.posq[i] = make_float4((float)(a.x[i] - S.ox), (float)(a.y[i] - S.oy), (float)(a.z[i] - S.oz),
                          (float)a.charge[i]);
}

// Block-wide sums of up to three values (fixed order: deterministic).
__device__ __forceinline__ void block_sum3(double &v0, double &v1, double &v2) {
  __shared__ double sh[3][kMinThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_down_sync(kFull, v0, o);
    v1 += __shfl_down_sync(kFull, v1, o);
    v2 += __shfl_down_sync(kFull, v2, o);
  }
  if (lane == 0) { sh[0][w] = v0; sh[1][w] = v1; sh[2][w] = v2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int k = 0; k < kMinThreads / 32; ++k) { s0 += sh[0][k]; s1 += sh[1][k]; s2 += sh[2][k]; }
    sh[0][0] = s0; sh[1][0] = s1; sh[2][0] = s2;
  }
  __syncthreads();
  v0 = sh[0][0]; v1 = sh[1][0]; v2 = sh[2][0];
  __syncthreads();
}

// ----------------------------------------------------------- steepest descent

__global__ void min_sd_kernel(const MinArgs a) {
  const double dt = a.par[kMinSdDt], max_dx = a.par[kMinMaxDx];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    double f[3];
    total_force(a, i, f);
    double d[3] = {f[0] * dt, f[1] * dt, f[2] * dt};
    const double dm = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + 1e-30);
    const double sc = fmin(1.0, max_dx / dm);
    a.x[i] += d[0] * sc;
    a.y[i] += d[1] * sc;
    a.z[i] += d[2] * sc;
    a.fx[i] = 0; a.fy[i] = 0; a.fz[i] = 0;
    put_posq(a, i);
  }
}

// A system with any non-finite coordinate goes back to its reference
// positions (the reference's rollback after SD and after FIRE).
__global__ void min_rollback_kernel(const MinArgs a) {
  __shared__ int bad;
  const size_t N = a.n_total;
  for (int s = blockIdx.x; s < a.n_sys; s += gridDim.x) {
    const SysInfo &S = a.sys[s];
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x)
      if (!(isfinite(a.x[i]) && isfinite(a.y[i]) && isfinite(a.z[i]))) bad = 1;
    __syncthreads();
    if (bad) {
      for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
        a.x[i] = a.x0[i]; a.y[i] = a.x0[N + i]; a.z[i] = a.x0[2 * N + i];
        put_posq(a, i);
      }
      if (threadIdx.x == 0) atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NONFINITE);
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------- FIRE

// p = 0, state force = F + restraint, per-system scalars reset.
__global__ void min_fire_init_kernel(const MinArgs a) {
  const size_t N = a.n_total;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    double f[3];
    total_force(a, i, f);
    a.ft[i] = f[0]; a.ft[N + i] = f[1]; a.ft[2 * N + i] = f[2];
    a.px[i] = 0.0; a.py[i] = 0.0; a.pz[i] = 0.0;
    a.best[i] = a.x[i]; a.best[N + i] = a.y[i]; a.best[2 * N + i] = a.z[i];
  }
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < a.n_sys; s += gridDim.x * blockDim.x) {
    a.sys_dt[s] = a.par[kMinDtStart];
    a.sys_alpha[s] = kFireAlphaStart;
    a.sys_npos[s] = 0;
    a.sys_best[s] = 1e10;
  }
}

// Start of an iteration: RMS of the state force; keep the positions if it is
// the lowest so far.
__global__ void min_fire_begin_kernel(const MinArgs a) {
  __shared__ int better;
  const size_t N = a.n_total;
  for (int s = blockIdx.x; s < a.n_sys; s += gridDim.x) {
    const SysInfo &S = a.sys[s];
    double f2 = 0.0, z0 = 0.0, z1 = 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x)
      f2 += a.ft[i] * a.ft[i] + a.ft[N + i] * a.ft[N + i] + a.ft[2 * N + i] * a.ft[2 * N + i];
    block_sum3(f2, z0, z1);
    if (threadIdx.x == 0) {
      const double rms = sqrt(f2 / (double)S.n);
      better = rms < a.sys_best[s];
      if (better) a.sys_best[s] = rms;
    }
    __syncthreads();
    if (better)
      for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
        a.best[i] = a.x[i]; a.best[N + i] = a.y[i]; a.best[2 * N + i] = a.z[i];
      }
    __syncthreads();
  }
}

// First half kick and drift; remembers the positions for the displacement
// cap.  With a force cap (prolix simulate.py:613-621) the state force of
// each atom is scaled to at most that norm for this kick.
__global__ void min_fire_drift_kernel(const MinArgs a) {
  const size_t N = a.n_total;
  const double cap = a.par[kMinForceCap];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const double dt = a.sys_dt[a.atom_sys[i]], h = 0.5 * dt, m = a.mass[i];
    double f[3] = {a.ft[i], a.ft[N + i], a.ft[2 * N + i]};
    if (cap > 0.0) {
      const double sc = fmin(1.0, cap / (sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]) + 1e-8));
      f[0] *= sc; f[1] *= sc; f[2] *= sc;
    }
    const double px = a.px[i] + h * f[0], py = a.py[i] + h * f[1], pz = a.pz[i] + h * f[2];
    a.px[i] = px; a.py[i] = py; a.pz[i] = pz;
    a.xb[i] = a.x[i]; a.xb[N + i] = a.y[i]; a.xb[2 * N + i] = a.z[i];
    a.x[i] += dt * px / m;
    a.y[i] += dt * py / m;
    a.z[i] += dt * pz / m;
    a.fx[i] = 0; a.fy[i] = 0; a.fz[i] = 0;
    put_posq(a, i);
  }
}

// Second half kick with the new force, FIRE mixing and time-step control,
// then the displacement cap.
__global__ void min_fire_mix_kernel(const MinArgs a) {
  __shared__ double mix_f, mix_p;
  __shared__ int zero_p;
  const size_t N = a.n_total;
  const double max_disp = a.par[kMinMaxDisp], dt_max = a.par[kMinDtMax];
  for (int s = blockIdx.x; s < a.n_sys; s += gridDim.x) {
    const SysInfo &S = a.sys[s];
    const double h = 0.5 * a.sys_dt[s];
    double fp = 0.0, f2 = 0.0, p2 = 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
      double f[3];
      total_force(a, i, f);
      a.ft[i] = f[0]; a.ft[N + i] = f[1]; a.ft[2 * N + i] = f[2];
      const double px = a.px[i] + h * f[0], py = a.py[i] + h * f[1], pz = a.pz[i] + h * f[2];
      a.px[i] = px; a.py[i] = py; a.pz[i] = pz;
      fp += f[0] * px + f[1] * py + f[2] * pz;
      f2 += f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
      p2 += px * px + py * py + pz * pz;
    }
    block_sum3(fp, f2, p2);
    if (threadIdx.x == 0) {
      const double alpha = a.sys_alpha[s];
      const double fn = sqrt(f2 + 1e-6), pn = sqrt(p2);
      mix_f = alpha * pn / fn;
      mix_p = alpha;
      int npos = fp >= 0.0 ? a.sys_npos[s] + 1 : 0;
      double dt = a.sys_dt[s], al = alpha;
      if (fp > 0.0 && npos > kFireNmin) {
        dt = fmin(dt * kFireFinc, dt_max);
        al = al * kFireFalpha;
      }
      if (fp < 0.0) {
        dt = dt * kFireFdec;
        al = kFireAlphaStart;
      }
      zero_p = fp < 0.0;
      a.sys_npos[s] = npos;
      a.sys_dt[s] = dt;
      a.sys_alpha[s] = al;
    }
    __syncthreads();
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
      double p[3] = {a.px[i], a.py[i], a.pz[i]};
      const double f[3] = {a.ft[i], a.ft[N + i], a.ft[2 * N + i]};
#pragma unroll
      for (int c = 0; c < 3; ++c) p[c] = zero_p ? 0.0 : p[c] + (mix_f * f[c] - mix_p * p[c]);
      const double dx = a.x[i] - a.xb[i], dy = a.y[i] - a.xb[N + i], dz = a.z[i] - a.xb[2 * N + i];
      const double dm = sqrt(dx * dx + dy * dy + dz * dz + 1e-30);
      const double sc = max_disp > 0.0 ? fmin(1.0, max_disp / dm) : 1.0;  // 0: no cap
      a.x[i] = a.xb[i] + dx * sc;
      a.y[i] = a.xb[N + i] + dy * sc;
      a.z[i] = a.xb[2 * N + i] + dz * sc;
      a.px[i] = p[0] * sc; a.py[i] = p[1] * sc; a.pz[i] = p[2] * sc;
    }
    __syncthreads();
  }
}

// End of a FIRE stage: the best positions become the state.
__global__ void min_take_best_kernel(const MinArgs a) {
  const size_t N = a.n_total;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    a.x[i] = a.best[i]; a.y[i] = a.best[N + i]; a.z[i] = a.best[2 * N + i];
    put_posq(a, i);
  }
}

// RMS over atoms of the physical force (unrestrained), per system.
__global__ void min_rms_kernel(const MinArgs a, double *out) {
  for (int s = blockIdx.x; s < a.n_sys; s += gridDim.x) {
    const SysInfo &S = a.sys[s];
    double f2 = 0.0, z0 = 0.0, z1 = 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
      const double f[3] = {fix_d(a.fx[i]), fix_d(a.fy[i]), fix_d(a.fz[i])};
      f2 += f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
    }
    block_sum3(f2, z0, z1);
    if (threadIdx.x == 0) out[s] = sqrt(f2 / (double)S.n);
  }
}

// -------------------------------------------------------------------- L-BFGS
//
// Limited-memory BFGS (Nocedal & Wright, Numerical Optimization, alg. 7.4
// and 7.5) per system, the polish stage of the reference (jaxopt LBFGS,
// batched_simulate.py:885-936): history of the last m steps s = x' - x and
// gradient changes y = g' - g, two-loop recursion for d = -H g with
// H0 = (s.y / y.y) I of the newest pair, and a backtracking line search
// (x0 + t d, t from min(1, max_step) shrinking by 0.8: jaxopt's
// max_stepsize clips the step length) accepting the first t with
// E(t) <= E0 + 1e-4 t g.d and |g(t).d| <= 0.9 |g.d|, or the last of the
// trials.  The gradient is minus the force; energies come from the FP64
// energy path.

__device__ __forceinline__ double grad_c(const LbfgsArgs &a, int i, int c) {
  const long long *f = c == 0 ? a.m.fx : (c == 1 ? a.m.fy : a.m.fz);
  const double v = -fix_d(f[i]);
  return isfinite(v) ? v : 0.0;
}

// A block sums one product over the system's 3n coordinates.
__device__ __forceinline__ double sys_dot(const double *u, const double *v, const SysInfo &S, size_t N) {
  double acc = 0.0, z0 = 0.0, z1 = 0.0;
  for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x)
    acc += u[i] * v[i] + u[N + i] * v[N + i] + u[2 * N + i] * v[2 * N + i];
  block_sum3(acc, z0, z1);
  return acc;
}

// g <- gradient at the current positions, x0 <- positions, E0 <- energy,
// empty history.
__global__ void lbfgs_begin_kernel(const LbfgsArgs a) {
  const size_t N = a.m.n_total;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.m.n_total; i += gridDim.x * blockDim.x) {
    a.g[i] = grad_c(a, i, 0); a.g[N + i] = grad_c(a, i, 1); a.g[2 * N + i] = grad_c(a, i, 2);
    a.x0[i] = a.m.x[i]; a.x0[N + i] = a.m.y[i]; a.x0[2 * N + i] = a.m.z[i];
  }
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < a.m.n_sys; s += gridDim.x * blockDim.x) {
    a.e0[s] = a.energy[(size_t)s * PB2_NTERMS + PB2_TERM_TOTAL];
    a.count[s] = 0;
    a.head[s] = 0;
    a.flags[s] = 0;
  }
}

// Two-loop recursion: d = -H g; t = min(1, max_step); gd = g.d.
__global__ void lbfgs_direction_kernel(const LbfgsArgs a) {
  __shared__ double alpha[kLbfgsMaxHist];
  __shared__ double coef;
  const size_t N = a.m.n_total, H = 3 * N;
  for (int s = blockIdx.x; s < a.m.n_sys; s += gridDim.x) {
    const SysInfo &S = a.m.sys[s];
    if (a.flags[s] & kLbfgsDone) continue;  // uniform over the block
    const int cnt = a.count[s], head = a.head[s], m = a.hist;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
      a.d[i] = a.g[i]; a.d[N + i] = a.g[N + i]; a.d[2 * N + i] = a.g[2 * N + i];
    }
    __syncthreads();
    for (int k = 0; k < cnt; ++k) {  // newest to oldest
      const int h = (head - 1 - k + m) % m;
      const double *sh = a.hs + h * H, *yh = a.hy + h * H;
      const double al = a.rho[(size_t)h * a.m.n_sys + s] * sys_dot(sh, a.d, S, N);
      if (threadIdx.x == 0) alpha[k] = al;
      for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
        a.d[i] -= al * yh[i]; a.d[N + i] -= al * yh[N + i]; a.d[2 * N + i] -= al * yh[2 * N + i];
      }
      __syncthreads();
    }
    double gamma = 1.0;
    if (cnt > 0) {
      const int h = (head - 1 + m) % m;
      const double sy = sys_dot(a.hs + h * H, a.hy + h * H, S, N);
      const double yy = sys_dot(a.hy + h * H, a.hy + h * H, S, N);
      if (yy > 0.0) gamma = sy / yy;
    }
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
      a.d[i] *= gamma; a.d[N + i] *= gamma; a.d[2 * N + i] *= gamma;
    }
    __syncthreads();
    for (int k = cnt - 1; k >= 0; --k) {  // oldest to newest
      const int h = (head - 1 - k + m) % m;
      const double *sh = a.hs + h * H, *yh = a.hy + h * H;
      const double be = a.rho[(size_t)h * a.m.n_sys + s] * sys_dot(yh, a.d, S, N);
      const double c = alpha[k] - be;
      for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
        a.d[i] += c * sh[i]; a.d[N + i] += c * sh[N + i]; a.d[2 * N + i] += c * sh[2 * N + i];
      }
      __syncthreads();
    }
    // d = -r; not a descent direction (or empty history start): steepest descent
    double gd = -sys_dot(a.g, a.d, S, N);
    if (threadIdx.x == 0) coef = (gd < 0.0) ? -1.0 : 0.0;
    __syncthreads();
    const bool sd = coef == 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
      for (int c = 0; c < 3; ++c) {
        double &dv = a.d[c * N + i];
        dv = sd ? -a.g[c * N + i] : -dv;
      }
    }
    __syncthreads();
    if (sd) gd = -sys_dot(a.g, a.g, S, N);
    if (threadIdx.x == 0) {
      if (sd) a.count[s] = 0;
      a.gd[s] = gd;
      a.t[s] = fmin(1.0, a.max_step);
      a.flags[s] &= ~kLbfgsAccepted;
    }
    __syncthreads();
  }
}

// Trial positions x0 + t d for the systems still searching.
__global__ void lbfgs_trial_kernel(const LbfgsArgs a) {
  const size_t N = a.m.n_total;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.m.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.m.atom_sys[i];
    if (!(a.flags[s] & (kLbfgsDone | kLbfgsAccepted))) {
      const double t = a.t[s];
      a.m.x[i] = a.x0[i] + t * a.d[i];
      a.m.y[i] = a.x0[N + i] + t * a.d[N + i];
      a.m.z[i] = a.x0[2 * N + i] + t * a.d[2 * N + i];
    }
    a.m.fx[i] = 0; a.m.fy[i] = 0; a.m.fz[i] = 0;
    put_posq(a.m, i);
  }
}

// Line-search test; on acceptance (or the last trial) the history, gradient,
// energy and base positions advance and convergence is checked.
__global__ void lbfgs_check_kernel(const LbfgsArgs a, int last_trial) {
  __shared__ int take;
  const size_t N = a.m.n_total, H = 3 * N;
  for (int s = blockIdx.x; s < a.m.n_sys; s += gridDim.x) {
    const SysInfo &S = a.m.sys[s];
    if (a.flags[s] & (kLbfgsDone | kLbfgsAccepted)) continue;
    const double et = a.energy[(size_t)s * PB2_NTERMS + PB2_TERM_TOTAL];
    double gtd = 0.0, z0 = 0.0, z1 = 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x)
      gtd += grad_c(a, i, 0) * a.d[i] + grad_c(a, i, 1) * a.d[N + i] + grad_c(a, i, 2) * a.d[2 * N + i];
    block_sum3(gtd, z0, z1);
    if (threadIdx.x == 0) {
      const double t = a.t[s], gd = a.gd[s];
      const bool ok = isfinite(et) && et <= a.e0[s] + 1e-4 * t * gd && fabs(gtd) <= 0.9 * fabs(gd);
      take = ok || last_trial;
      if (!take) a.t[s] = t * 0.8;
    }
    __syncthreads();
    if (take) {
      const int m = a.hist, h = a.head[s];
      double *sh = a.hs + h * H, *yh = a.hy + h * H;
      double sy = 0.0, g2 = 0.0, z2 = 0.0;
      for (int i = S.off + threadIdx.x; i < S.off + S.n; i += blockDim.x) {
        const double xn[3] = {a.m.x[i], a.m.y[i], a.m.z[i]};
        for (int c = 0; c < 3; ++c) {
          const size_t k = c * N + i;
          const double gn = grad_c(a, i, c);
          sh[k] = xn[c] - a.x0[k];
          yh[k] = gn - a.g[k];
          sy += sh[k] * yh[k];
          g2 += gn * gn;
          a.g[k] = gn;
          a.x0[k] = xn[c];
        }
      }
      block_sum3(sy, g2, z2);
      if (threadIdx.x == 0) {
        if (sy > 1e-12) {  // keep the pair only with positive curvature
          a.rho[(size_t)h * a.m.n_sys + s] = 1.0 / sy;
          a.head[s] = (h + 1) % m;
          a.count[s] = min(a.count[s] + 1, m);
        }
        a.e0[s] = et;
        a.flags[s] |= kLbfgsAccepted;
        if (sqrt(g2) < a.tol) a.flags[s] |= kLbfgsDone;
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- launchers

static int atom_grid(int n) {
  const int g = (n + kMinThreads - 1) / kMinThreads;
  return g < 1 ? 1 : (g > 8192 ? 8192 : g);
}

cudaError_t launch_min(int op, const MinArgs &a, double *out, cudaStream_t st) {
  if (a.n_total <= 0) return cudaSuccess;
  const int ga = atom_grid(a.n_total), gs = a.n_sys;
  switch (op) {
    case kMinOpSd: min_sd_kernel<<<ga, kMinThreads, 0, st>>>(a); break;
    case kMinOpRollback: min_rollback_kernel<<<gs, kMinThreads, 0, st>>>(a); break;
    case kMinOpFireInit: min_fire_init_kernel<<<ga, kMinThreads, 0, st>>>(a); break;
    case kMinOpFireBegin: min_fire_begin_kernel<<<gs, kMinThreads, 0, st>>>(a); break;
    case kMinOpFireDrift: min_fire_drift_kernel<<<ga, kMinThreads, 0, st>>>(a); break;
    case kMinOpFireMix: min_fire_mix_kernel<<<gs, kMinThreads, 0, st>>>(a); break;
    case kMinOpTakeBest: min_take_best_kernel<<<ga, kMinThreads, 0, st>>>(a); break;
    case kMinOpRms: min_rms_kernel<<<gs, kMinThreads, 0, st>>>(a, out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_lbfgs(int op, const LbfgsArgs &a, int last_trial, cudaStream_t st) {
  if (a.m.n_total <= 0) return cudaSuccess;
  const int ga = atom_grid(a.m.n_total), gs = a.m.n_sys;
  switch (op) {
    case kLbfgsOpBegin: lbfgs_begin_kernel<<<ga, kMinThreads, 0, st>>>(a); break;
    case kLbfgsOpDirection: lbfgs_direction_kernel<<<gs, kMinThreads, 0, st>>>(a); break;
    case kLbfgsOpTrial: lbfgs_trial_kernel<<<ga, kMinThreads, 0, st>>>(a); break;
    case kLbfgsOpCheck: lbfgs_check_kernel<<<gs, kMinThreads, 0, st>>>(a, last_trial); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace pb2
