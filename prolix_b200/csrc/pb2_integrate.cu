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
// step, converts the new positions for the float32 pair kernels, writes the
// 32-atom blocks' bounding boxes and clears the force accumulators; the
// force kernels then run; finish_kernel applies the last half kick of a
// chunk.  Keys live in two buffers: a step reads
// buffer `parity` and writes the advanced key to the other.
#include <algorithm>
#include <atomic>

#include "pb2_common.cuh"
#include "pb2_divide.cuh"
#include "pb2_kernels.cuh"
#include "pb2_threefry.cuh"

namespace pb2 {


__device__ __forceinline__ double fix_to_d(long long v) { return (double)v * kForceInv; }

__device__ __forceinline__ void check_fix(const IntArgs &a, int s, long long v) {
  if (v == LLONG_MAX || v == LLONG_MIN) atomicOr(&a.status[s], (uint32_t)PB2_STATUS_FORCE_RANGE);
}

__device__ __forceinline__ float4 posq_of(double x, double y, double z, const double3 &o, double charge) {
  return make_float4((float)(x - o.x), (float)(y - o.y), (float)(z - o.z), (float)charge);
}

__device__ __forceinline__ float4 write_posq(const IntArgs &a, int i, const SysInfo &S, double x,
                                             double y, double z) {
  const float4 q = posq_of(x, y, z, make_double3(S.ox, S.oy, S.oz), a.charge[i]);
  a.posq[i] = q;
  return q;
}

// The step kernels map one warp to one 32-atom block (lane l: atom l of the
// block), so that the block's bounding box of the new positions -- what the
// pair kernels cull tiles by -- comes out of the same launch, and so does
// the pair list's displacement test.  Lanes past a system's last atom take
// the block's first atom for the box.
__device__ __forceinline__ void block_box(const IntArgs &a, int b, int lane, bool valid, float4 q) {
  const float4 q0 = make_float4(__shfl_sync(kFull, q.x, 0), __shfl_sync(kFull, q.y, 0),
                                __shfl_sync(kFull, q.z, 0), 0.f);
  if (!valid) q = q0;
  float lo[3] = {q.x, q.y, q.z}, hi[3] = {q.x, q.y, q.z};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      lo[c] = fminf(lo[c], __shfl_xor_sync(kFull, lo[c], o));
      hi[c] = fmaxf(hi[c], __shfl_xor_sync(kFull, hi[c], o));
    }
  if (lane == 0) {
    a.bbox[2 * b] = make_float4(lo[0], lo[1], lo[2], 0.f);
    a.bbox[2 * b + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
  }
}

// The charge and the pair list's reference position, loaded before the
// step's stores: the FP64 stores could alias the charge and the posq store
// the reference, and a load ordered after them adds a memory latency at the
// end of every thread.
struct StepExtra {
  double charge;
  float4 ref;  // zero without a list
};
__device__ __forceinline__ StepExtra step_extra(const IntArgs &a, int i) {
  StepExtra e;
  e.charge = a.charge[i];
  e.ref = a.pl_ref ? a.pl_ref[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  return e;
}

__device__ __forceinline__ bool moved_past_half_skin(const IntArgs &a, const StepExtra &e, const SysInfo &S,
                                                     float4 q) {
  if (!a.pl_ref) return false;
  const float dx = q.x - e.ref.x, dy = q.y - e.ref.y, dz = q.z - e.ref.z;
  return (double)fmaf(dx, dx, fmaf(dy, dy, dz * dz)) > S.skin_half2;
}

// keys[parity ^ 1][s] = k, and its split for the step that will read it.
__device__ __forceinline__ void store_key(const IntArgs &a, int s, const uint32_t k[2]) {
  const size_t slot = (size_t)(a.parity ^ 1) * a.n_sys + s;
  a.keys[2 * slot] = k[0];
  a.keys[2 * slot + 1] = k[1];
  uint32_t k2[2], s2[2];
  split_key(k[0], k[1], a.partitionable != 0, k2, s2);
  reinterpret_cast<uint4 *>(a.splits)[slot] = make_uint4(k2[0], k2[1], s2[0], s2[1]);
}

// End of a step for system s (its first atom's thread): the advanced key,
// and the step counter.
__device__ __forceinline__ void advance_key(const IntArgs &a, int s, const uint32_t knew[2]) {
  store_key(a, s, knew);
  a.steps[s] += 1;
}

__global__ void key_splits_kernel(const IntArgs a) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < a.n_sys; s += gridDim.x * blockDim.x) {
    const size_t slot = (size_t)a.parity * a.n_sys + s;
    uint32_t k2[2], s2[2];
    split_key(a.keys[2 * slot], a.keys[2 * slot + 1], a.partitionable != 0, k2, s2);
    reinterpret_cast<uint4 *>(a.splits)[slot] = make_uint4(k2[0], k2[1], s2[0], s2[1]);
  }
}

// The plain step: a persistent grid (one resident wave) whose warps each
// take 32-atom blocks in turn (lane l: atom l of the block) and copy the
// next block's inputs into shared memory (cp.async, 8 bytes per lane and
// array) while they step the current one, so that a block's load latency
// hides behind the previous block's arithmetic.
struct StepIn {  // one block's inputs, [component][lane]
  double x[3][32], p[3][32];
  long long f[3][32];
  double m[32], sg[32], q[32];
  int user[32];
};
constexpr int kStepWarps = 4;  // warps per thread block of the plain step

// Block info (system, first atom, atoms): lanes past the block's last atom
// copy its first atom (never used).
__device__ __forceinline__ void issue_block(const IntArgs &a, int4 info, int lane, StepIn &B) {
  const int i = info.y + (lane < info.z ? lane : 0);
  cp_async8(&B.x[0][lane], a.x + i); cp_async8(&B.x[1][lane], a.y + i); cp_async8(&B.x[2][lane], a.z + i);
  cp_async8(&B.p[0][lane], a.px + i); cp_async8(&B.p[1][lane], a.py + i); cp_async8(&B.p[2][lane], a.pz + i);
  cp_async8(&B.f[0][lane], a.fx + i); cp_async8(&B.f[1][lane], a.fy + i); cp_async8(&B.f[2][lane], a.fz + i);
  cp_async8(&B.m[lane], a.mass + i); cp_async8(&B.sg[lane], a.sigma + i); cp_async8(&B.q[lane], a.charge + i);
  cp_async4(&B.user[lane], a.user + i);
}

// One atom's plain BAOAB step from its copied inputs; returns the float32
// position it wrote.
__device__ __forceinline__ float4 step_atom(const IntArgs &a, int i, int s, const SysInfo &S, const StepIn &B,
                                            int lane) {
  const int loc = i - S.off;
  const int rnd = B.user[lane] - S.off;  // the atom's index in the caller's order: its noise
  const double h = S.half_dt;
  const double m = B.m[lane];
  const double rm = __drcp_rn(m);  // p / m = div_by(p, m, rm), correctly rounded
  const long long lfx = B.f[0][lane], lfy = B.f[1][lane], lfz = B.f[2][lane];
  check_fix(a, s, lfx); check_fix(a, s, lfy); check_fix(a, s, lfz);
  const double f[3] = {fix_to_d(lfx), fix_to_d(lfy), fix_to_d(lfz)};
  a.fx[i] = 0; a.fy[i] = 0; a.fz[i] = 0;
  double p[3] = {B.p[0][lane], B.p[1][lane], B.p[2][lane]};
  double x[3] = {B.x[0][lane], B.x[1][lane], B.x[2][lane]};
  const uint4 sp = reinterpret_cast<const uint4 *>(a.splits)[(size_t)a.parity * a.n_sys + s];
  const uint32_t knew[2] = {sp.x, sp.y}, sub[2] = {sp.z, sp.w};
  const uint32_t count = 3u * (uint32_t)S.n;
  const double c1 = S.c1, sg = B.sg[lane];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (a.finish_prev) p[c] = __dadd_rn(p[c], __dmul_rn(h, f[c]));
    p[c] = __dadd_rn(p[c], __dmul_rn(h, f[c]));
    x[c] = __dadd_rn(x[c], __dmul_rn(h, div_by(p[c], m, rm)));
    const float xi = normal_from_bits(random_bits32(sub, 3u * (uint32_t)rnd + c, count, a.partitionable != 0));
    p[c] = __dadd_rn(__dmul_rn(c1, p[c]), __dmul_rn(sg, (double)xi));
    x[c] = __dadd_rn(x[c], __dmul_rn(h, div_by(p[c], m, rm)));
  }
  a.px[i] = p[0]; a.py[i] = p[1]; a.pz[i] = p[2];
  a.x[i] = x[0]; a.y[i] = x[1]; a.z[i] = x[2];
  const float4 q = posq_of(x[0], x[1], x[2], make_double3(S.ox, S.oy, S.oz), B.q[lane]);
  a.posq[i] = q;
  if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]) && isfinite(p[0]) &&
        isfinite(p[1]) && isfinite(p[2])))
    atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NONFINITE);
  if (loc == 0) advance_key(a, s, knew);
  return q;
}

// Six blocks of 128 threads per SM (80 registers): at eight (64 registers)
// the step spilled and ran slower.
__global__ void __launch_bounds__(32 * kStepWarps, 6) step_kernel(const IntArgs a) {
  __shared__ StepIn s_in[kStepWarps][2];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int nw = (int)gridDim.x * kStepWarps;
  int b = (int)blockIdx.x * kStepWarps + wl;
  bool moved = false;
  const int4 none = make_int4(0, 0, 0, 0);
  int4 info = b < a.n_blocks ? a.blk_info[b] : none;
  if (b < a.n_blocks) issue_block(a, info, lane, s_in[wl][0]);
  cp_async_commit();
  int4 info_next = b + nw < a.n_blocks ? a.blk_info[b + nw] : none;
  for (int it = 0; b < a.n_blocks; b += nw, ++it) {
    const int bn = b + nw;
    if (bn < a.n_blocks) issue_block(a, info_next, lane, s_in[wl][(it + 1) & 1]);
    cp_async_commit();
    const int4 cur = info;
    info = info_next;
    info_next = bn + nw < a.n_blocks ? a.blk_info[bn + nw] : none;
    cp_async_wait<1>();  // this block's copies (all but the newest group) have landed
    const int s = cur.x;
    if (!a.retired[s]) {  // a retired system keeps its state and box
      const SysInfo &S = a.sys[s];
      const bool valid = lane < cur.z;
      float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
      if (valid) {
        StepExtra e;  // the charge comes from the copied inputs
        e.ref = a.pl_ref ? a.pl_ref[cur.y + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
        q = step_atom(a, cur.y + lane, s, S, s_in[wl][it & 1], lane);
        moved |= moved_past_half_skin(a, e, S, q);
      }
      block_box(a, b, lane, valid, q);
    }
    __syncwarp();  // the buffer is read before the next block's copies refill it
  }
  cp_async_wait<0>();
  if (a.pl_ctl && __any_sync(kFull, moved) && lane == 0) atomicOr(&a.pl_ctl[PL_DIRTY], 1);
}

// Safeguarded step: prolix's batched Langevin step (batched_simulate.py:218-382)
// without constraints, in its order:
//   F <- F min(1, cap / sqrt(|F|^2 + 1e-12))     (a step's closing force, :336-340)
//   p += dt/2 F;  where |p/m| > vlimit: p *= min(1, vlimit / (|p/m| + 1e-30))   (:263-274)
//   x_old = x;  A;  O;  A                                                         (:277-288)
//   s = min(1, max_dx / |dx|), |dx| = sqrt(|x - x_old|^2 + 1e-30);
//   x = x_old + (x - x_old) s;  where |dx| > max_dx: p *= s                        (:290-305)
// and a per-system count of the steps in which each cap fired (:361-367).  The
// constraint projection of :307-324 is the identity without constraints.  The
// force that closes step n opens step n+1 capped as well (the reference stores
// the capped force in the state); a force that no step produced (after init or
// a state load) opens the next step as it is.
__device__ __forceinline__ double norm3(double a, double b, double c, double eps) {
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c)), eps));
}

// Scale a closing force to at most force_cap; true when it was above.
__device__ __forceinline__ bool cap_force(double f[3], double cap) {
  const double fm = norm3(f[0], f[1], f[2], 1e-12);
  const double sc = fmin(1.0, __ddiv_rn(cap, fm));
#pragma unroll
  for (int c = 0; c < 3; ++c) f[c] = __dmul_rn(f[c], sc);
  return fm > cap;
}

// The thread of a system's first atom adds the caps recorded by the previous
// launch (the other parity's flag word) to the system's counts and clears it.
__device__ __forceinline__ void fold_warns(const IntArgs &a, int s) {
  uint32_t *w = a.warn_flags + (size_t)(a.parity ^ 1) * a.n_sys + s;
  const uint32_t fl = *w;
  if (fl) {
#pragma unroll
    for (int k = 0; k < kWarnTypes; ++k)
      if (fl & (1u << k)) a.warn_counts[(size_t)s * kWarnTypes + k] += 1;
    *w = 0;
  }
}

// One atom's safeguarded step; returns the float32 position it wrote.
__device__ __forceinline__ float4 step_guarded_atom(const IntArgs &a, int i, int s, const SysInfo &S,
                                                    const StepExtra &e, bool cap_open) {
  {
    const int loc = i - S.off;
    const int rnd = a.user[i] - S.off;
    const double h = S.half_dt;
    const double m = a.mass[i];
    const double rm = __drcp_rn(m);  // p / m = div_by(p, m, rm), correctly rounded
    const long long lfx = a.fx[i], lfy = a.fy[i], lfz = a.fz[i];
    check_fix(a, s, lfx); check_fix(a, s, lfy); check_fix(a, s, lfz);
    double f[3] = {fix_to_d(lfx), fix_to_d(lfy), fix_to_d(lfz)};
    a.fx[i] = 0; a.fy[i] = 0; a.fz[i] = 0;
    uint32_t bits = 0;
    if (a.force_cap > 0.0 && cap_open && cap_force(f, a.force_cap) && a.finish_prev)
      bits |= 1u << kWarnForceCap;  // counted once, by the launch that closes the step
    double p[3] = {a.px[i], a.py[i], a.pz[i]};
    double x[3] = {a.x[i], a.y[i], a.z[i]};
    const double xo[3] = {x[0], x[1], x[2]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (a.finish_prev) p[c] = __dadd_rn(p[c], __dmul_rn(h, f[c]));
      p[c] = __dadd_rn(p[c], __dmul_rn(h, f[c]));
    }
    if (a.vlimit > 0.0) {
      const double vm = norm3(div_by(p[0], m, rm), div_by(p[1], m, rm), div_by(p[2], m, rm), 1e-30);
      if (vm > a.vlimit) {
        const double sc = fmin(1.0, __ddiv_rn(a.vlimit, __dadd_rn(vm, 1e-30)));
#pragma unroll
        for (int c = 0; c < 3; ++c) p[c] = __dmul_rn(p[c], sc);
        bits |= 1u << kWarnVlimit;
      }
    }
    const uint4 sp = reinterpret_cast<const uint4 *>(a.splits)[(size_t)a.parity * a.n_sys + s];
    const uint32_t knew[2] = {sp.x, sp.y}, sub[2] = {sp.z, sp.w};
    const uint32_t count = 3u * (uint32_t)S.n;
    const double c1 = S.c1, sg = a.sigma[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      x[c] = __dadd_rn(x[c], __dmul_rn(h, div_by(p[c], m, rm)));
      const float xi = normal_from_bits(random_bits32(sub, 3u * (uint32_t)rnd + c, count, a.partitionable != 0));
      p[c] = __dadd_rn(__dmul_rn(c1, p[c]), __dmul_rn(sg, (double)xi));
      x[c] = __dadd_rn(x[c], __dmul_rn(h, div_by(p[c], m, rm)));
    }
    if (a.max_dx > 0.0) {
      const double d[3] = {__dsub_rn(x[0], xo[0]), __dsub_rn(x[1], xo[1]), __dsub_rn(x[2], xo[2])};
      const double dm = norm3(d[0], d[1], d[2], 1e-30);
      const double sc = fmin(1.0, __ddiv_rn(a.max_dx, dm));
#pragma unroll
      for (int c = 0; c < 3; ++c) x[c] = __dadd_rn(xo[c], __dmul_rn(d[c], sc));
      if (dm > a.max_dx) {
#pragma unroll
        for (int c = 0; c < 3; ++c) p[c] = __dmul_rn(p[c], sc);
        bits |= 1u << kWarnDxCap;
      }
    }
    a.px[i] = p[0]; a.py[i] = p[1]; a.pz[i] = p[2];
    a.x[i] = x[0]; a.y[i] = x[1]; a.z[i] = x[2];
    const float4 q = posq_of(x[0], x[1], x[2], make_double3(S.ox, S.oy, S.oz), e.charge);
    a.posq[i] = q;
    if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]) && isfinite(p[0]) &&
          isfinite(p[1]) && isfinite(p[2])))
      atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NONFINITE);
    if (bits) atomicOr(&a.warn_flags[(size_t)a.parity * a.n_sys + s], bits);
    if (loc == 0) {
      advance_key(a, s, knew);
      fold_warns(a, s);
    }
    return q;
  }
}

__global__ void __launch_bounds__(256, 4) step_guarded_kernel(const IntArgs a) {
  const bool cap_open = a.finish_prev || *a.guard_end;
  const int lane = threadIdx.x & 31;
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  bool moved = false;
  for (int b = w; b < a.n_blocks; b += nw) {
    const int s = a.blk_sys[b];
    const SysInfo &S = a.sys[s];
    const int blk_base = S.blk_base, n = S.n;  // loaded beside the retired flag, not after it
    if (a.retired[s]) continue;  // a retired system keeps its state and box
    const int l = (b - blk_base) * 32 + lane;
    const bool valid = l < n;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
      const StepExtra e = step_extra(a, S.off + l);
      q = step_guarded_atom(a, S.off + l, s, S, e, cap_open);
      moved |= moved_past_half_skin(a, e, S, q);
    }
    block_box(a, b, lane, valid, q);
  }
  if (a.pl_ctl && __any_sync(kFull, moved) && lane == 0) atomicOr(&a.pl_ctl[PL_DIRTY], 1);
}

__global__ void finish_guarded_kernel(const IntArgs a) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.guard_end = 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    if (a.retired[s]) continue;
    const double h = a.sys[s].half_dt;
    const long long lfx = a.fx[i], lfy = a.fy[i], lfz = a.fz[i];
    check_fix(a, s, lfx); check_fix(a, s, lfy); check_fix(a, s, lfz);
    double f[3] = {fix_to_d(lfx), fix_to_d(lfy), fix_to_d(lfz)};
    if (a.force_cap > 0.0 && cap_force(f, a.force_cap))
      atomicOr(&a.warn_flags[(size_t)a.parity * a.n_sys + s], 1u << kWarnForceCap);
    const double px = __dadd_rn(a.px[i], __dmul_rn(h, f[0]));
    const double py = __dadd_rn(a.py[i], __dmul_rn(h, f[1]));
    const double pz = __dadd_rn(a.pz[i], __dmul_rn(h, f[2]));
    a.px[i] = px; a.py[i] = py; a.pz[i] = pz;
    if (!(isfinite(px) && isfinite(py) && isfinite(pz)))
      atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NONFINITE);
    if (i == a.sys[s].off) fold_warns(a, s);
  }
}

__global__ void finish_kernel(const IntArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    if (a.retired[s]) continue;
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
    if (loc == 0) store_key(a, s, knew);
  }
}

// Remove each system's mean momentum (jax_md's center_velocity at init,
// applied by prolix over real atoms only, physics/settle.py:1121-1142); a
// one-atom system keeps its momentum.  One block per system; the sums run
// in a fixed order, so the result is deterministic.
constexpr int kCenterThreads = 256;
__global__ void __launch_bounds__(kCenterThreads) center_kernel(const IntArgs a) {
  const SysInfo &S = a.sys[blockIdx.x];
  if (S.n <= 1) return;
  __shared__ double sh[3][kCenterThreads];
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int l = threadIdx.x; l < S.n; l += kCenterThreads) {
    const int i = S.off + l;
    sx += a.px[i];
    sy += a.py[i];
    sz += a.pz[i];
  }
  sh[0][threadIdx.x] = sx;
  sh[1][threadIdx.x] = sy;
  sh[2][threadIdx.x] = sz;
  __syncthreads();
  for (int w = kCenterThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
    __syncthreads();
  }
  const double mx = sh[0][0] / S.n, my = sh[1][0] / S.n, mz = sh[2][0] / S.n;
  for (int l = threadIdx.x; l < S.n; l += kCenterThreads) {
    const int i = S.off + l;
    a.px[i] -= mx;
    a.py[i] -= my;
    a.pz[i] -= mz;
  }
}

// Per-atom noise amplitude c2 sqrt(m kT) after new Langevin parameters, the
// same correctly rounded operations as at batch creation.
__global__ void noise_scale_kernel(const SysInfo *sys, const int32_t *atom_sys, const double *mass,
                                   double *sigma, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const SysInfo &S = sys[atom_sys[i]];
    sigma[i] = __dmul_rn(S.c2, __dsqrt_rn(__dmul_rn(mass[i], S.kT)));
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

static bool guarded(const IntArgs &a) { return a.vlimit > 0.0 || a.max_dx > 0.0 || a.force_cap > 0.0; }

// Resident thread blocks of the plain step on the current device.
static int step_grid(int n_blocks) {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  int g = cached[dev].load(std::memory_order_relaxed);
  if (g == 0) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, step_kernel, 32 * kStepWarps, 0);
    g = std::max(1, sms * std::max(per, 1));
    cached[dev].store(g, std::memory_order_relaxed);
  }
  return std::max(1, std::min((n_blocks + kStepWarps - 1) / kStepWarps, g));
}

void warm_step_launch(int n_blocks) { step_grid(n_blocks); }

cudaError_t launch_step(const IntArgs &a, cudaStream_t st) {
  const int grid = (a.n_blocks + 7) / 8;  // 8 warps, one 32-atom block each
  if (grid <= 0) return cudaSuccess;
  if (guarded(a))
    step_guarded_kernel<<<grid, 256, 0, st>>>(a);
  else
    step_kernel<<<step_grid(a.n_blocks), 32 * kStepWarps, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_finish(const IntArgs &a, cudaStream_t st) {
  if (guarded(a))
    finish_guarded_kernel<<<grid_for(a.n_total), 256, 0, st>>>(a);
  else
    finish_kernel<<<grid_for(a.n_total), 256, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_key_splits(const IntArgs &a, cudaStream_t st) {
  key_splits_kernel<<<(a.n_sys + 255) / 256, 256, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_init(const IntArgs &a, cudaStream_t st) {
  init_kernel<<<grid_for(a.n_total), 256, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_noise_scale(const SysInfo *sys, const int32_t *atom_sys, const double *mass,
                               double *sigma, int n, cudaStream_t st) {
  noise_scale_kernel<<<grid_for(n), 256, 0, st>>>(sys, atom_sys, mass, sigma, n);
  return cudaGetLastError();
}
cudaError_t launch_center(const IntArgs &a, cudaStream_t st) {
  center_kernel<<<a.n_sys, kCenterThreads, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_posq(const IntArgs &a, cudaStream_t st) {
  posq_kernel<<<grid_for(a.n_total), 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace pb2
