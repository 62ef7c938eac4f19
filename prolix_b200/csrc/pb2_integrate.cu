// BAOAB Langevin integrator, all systems of the batch, one thread per atom.
//
// Order and arithmetic follow prolix physics/settle.py:1698-1744 with the
// step helpers :2064-2087 (the jax_md nvt_langevin order):
//   p += dt/2 F; x += dt/2 p/m; (key, sub) = split(key);
//   p = c1 p + c2 sqrt(m kT) xi,  xi = normal(sub, (N, 3));
//   x += dt/2 p/m; F = force(x); p += dt/2 F.
// The state is FP64.  Every FP64 operation is an explicitly rounded
// intrinsic (no FMA contraction) in the order NumPy evaluates the same
// expressions, so with identical forces the update is bit-identical to the
// CPU restatement.
//
// Kernel boundaries: step_kernel applies the final half kick of the
// previous step (when finish_prev), the first half kick, A, O, A of the new
// step, converts the new positions for the float32 pair kernels and clears
// the force accumulators; the force kernels then run; finish_kernel applies
// the last half kick of a chunk.  Keys live in two buffers: a step reads
// buffer `parity` and writes the advanced key to the other.
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"
#include "pb2_threefry.cuh"

namespace pb2 {


__device__ __forceinline__ double fix_to_d(long long v) { return (double)v * kForceInv; }

__device__ __forceinline__ void check_fix(const IntArgs &a, int s, long long v) {
  if (v == LLONG_MAX || v == LLONG_MIN) atomicOr(&a.status[s], (uint32_t)PB2_STATUS_FORCE_RANGE);
}

__device__ __forceinline__ void write_posq(const IntArgs &a, int i, const SysInfo &S, double x,
                                           double y, double z) {
  a.posq[i] = make_float4((float)(x - S.ox), (float)(y - S.oy), (float)(z - S.oz), (float)a.charge[i]);
}

__global__ void step_kernel(const IntArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    const SysInfo &S = a.sys[s];
    const int loc = i - S.off;
    const int rnd = a.user[i] - S.off;  // the atom's index in the caller's order: its noise
    const double h = S.half_dt;
    const double m = a.mass[i];
    const long long lfx = a.fx[i], lfy = a.fy[i], lfz = a.fz[i];
    check_fix(a, s, lfx); check_fix(a, s, lfy); check_fix(a, s, lfz);
    const double f[3] = {fix_to_d(lfx), fix_to_d(lfy), fix_to_d(lfz)};
    a.fx[i] = 0; a.fy[i] = 0; a.fz[i] = 0;
    double p[3] = {a.px[i], a.py[i], a.pz[i]};
    double x[3] = {a.x[i], a.y[i], a.z[i]};
    const uint32_t *kin = a.keys + ((size_t)a.parity * a.n_sys + s) * 2;
    uint32_t knew[2], sub[2];
    split_key(kin[0], kin[1], a.partitionable != 0, knew, sub);
    const uint32_t count = 3u * (uint32_t)S.n;
    const double c1 = S.c1, sg = a.sigma[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (a.finish_prev) p[c] = __dadd_rn(p[c], __dmul_rn(h, f[c]));
      p[c] = __dadd_rn(p[c], __dmul_rn(h, f[c]));
      x[c] = __dadd_rn(x[c], __dmul_rn(h, __ddiv_rn(p[c], m)));
      const float xi = normal_from_bits(random_bits32(sub, 3u * (uint32_t)rnd + c, count, a.partitionable != 0));
      p[c] = __dadd_rn(__dmul_rn(c1, p[c]), __dmul_rn(sg, (double)xi));
      x[c] = __dadd_rn(x[c], __dmul_rn(h, __ddiv_rn(p[c], m)));
    }
    a.px[i] = p[0]; a.py[i] = p[1]; a.pz[i] = p[2];
    a.x[i] = x[0]; a.y[i] = x[1]; a.z[i] = x[2];
    write_posq(a, i, S, x[0], x[1], x[2]);
    if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]) && isfinite(p[0]) &&
          isfinite(p[1]) && isfinite(p[2])))
      atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NONFINITE);
    if (loc == 0) {
      uint32_t *kout = a.keys + ((size_t)(a.parity ^ 1) * a.n_sys + s) * 2;
      kout[0] = knew[0];
      kout[1] = knew[1];
      a.steps[s] += 1;
    }
  }
}

__global__ void finish_kernel(const IntArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    const double h = a.sys[s].half_dt;
    const long long lfx = a.fx[i], lfy = a.fy[i], lfz = a.fz[i];
    check_fix(a, s, lfx); check_fix(a, s, lfy); check_fix(a, s, lfz);
    const double px = __dadd_rn(a.px[i], __dmul_rn(h, fix_to_d(lfx)));
    const double py = __dadd_rn(a.py[i], __dmul_rn(h, fix_to_d(lfy)));
    const double pz = __dadd_rn(a.pz[i], __dmul_rn(h, fix_to_d(lfz)));
    a.px[i] = px; a.py[i] = py; a.pz[i] = pz;
    if (!(isfinite(px) && isfinite(py) && isfinite(pz)))
      atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NONFINITE);
  }
}

// p = sqrt(m kT) * normal(sub) with (key, sub) = split(key)  (settle.py:1676-1696)
__global__ void init_kernel(const IntArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    const SysInfo &S = a.sys[s];
    const int loc = i - S.off;
    const int rnd = a.user[i] - S.off;  // the atom's index in the caller's order: its noise
    const uint32_t *kin = a.keys + ((size_t)a.parity * a.n_sys + s) * 2;
    uint32_t knew[2], sub[2];
    split_key(kin[0], kin[1], a.partitionable != 0, knew, sub);
    const uint32_t count = 3u * (uint32_t)S.n;
    const double sd = __dsqrt_rn(__dmul_rn(a.mass[i], S.kT));
    double p[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float xi = normal_from_bits(random_bits32(sub, 3u * (uint32_t)rnd + c, count, a.partitionable != 0));
      p[c] = __dmul_rn(sd, (double)xi);
    }
    a.px[i] = p[0]; a.py[i] = p[1]; a.pz[i] = p[2];
    write_posq(a, i, S, a.x[i], a.y[i], a.z[i]);
    if (loc == 0) {
      uint32_t *kout = a.keys + ((size_t)(a.parity ^ 1) * a.n_sys + s) * 2;
      kout[0] = knew[0];
      kout[1] = knew[1];
    }
  }
}

// Refresh the float32 pair-kernel positions from the FP64 state.
__global__ void posq_kernel(const IntArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const SysInfo &S = a.sys[a.atom_sys[i]];
    write_posq(a, i, S, a.x[i], a.y[i], a.z[i]);
  }
}

static int grid_for(int n) {
  int g = (n + 255) / 256;
  return g > 0 ? g : 1;
}

cudaError_t launch_step(const IntArgs &a, cudaStream_t st) {
  step_kernel<<<grid_for(a.n_total), 256, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_finish(const IntArgs &a, cudaStream_t st) {
  finish_kernel<<<grid_for(a.n_total), 256, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_init(const IntArgs &a, cudaStream_t st) {
  init_kernel<<<grid_for(a.n_total), 256, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_posq(const IntArgs &a, cudaStream_t st) {
  posq_kernel<<<grid_for(a.n_total), 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace pb2
