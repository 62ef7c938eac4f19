// Host <-> device state transfers.
//
// The C ABI exchanges (n_atoms, 3) row-major FP64 arrays, the layout of
// prolix's jax_md state (NVTLangevinState.position / momentum / force);
// the device keeps x, y, z (and forces as 64-bit fixed point) as separate
// arrays.  One contiguous copy moves the row-major array between the host
// buffer and a device staging buffer; these kernels convert on the device,
// so the host does no per-atom work and the copy runs at full PCIe speed
// when the caller's buffer is page-locked.
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"

namespace pb2 {

// In every kernel below, atom i of the batch's arrays is row user[i] of the
// caller's (n, 3) arrays (the batch stores each system's atoms in its own
// order).

__global__ void rows_to_soa(const double *__restrict__ rows, const int32_t *__restrict__ user, double *x,
                            double *y, double *z, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double *r = rows + 3 * (size_t)user[i];
    x[i] = r[0];
    y[i] = r[1];
    z[i] = r[2];
  }
}

__global__ void soa_to_rows(const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, const int32_t *__restrict__ user, double *rows, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double *r = rows + 3 * (size_t)user[i];
    r[0] = x[i];
    r[1] = y[i];
    r[2] = z[i];
  }
}

// Fixed point -> FP64 is exact for |F| < 2^21 kcal/mol/A (|v| < 2^53), so a
// get/set round trip restores the accumulators bit for bit.
__global__ void fix_to_rows(const long long *__restrict__ fx, const long long *__restrict__ fy,
                            const long long *__restrict__ fz, const int32_t *__restrict__ user, double *rows,
                            int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double *r = rows + 3 * (size_t)user[i];
    r[0] = (double)fx[i] * kForceInv;
    r[1] = (double)fy[i] * kForceInv;
    r[2] = (double)fz[i] * kForceInv;
  }
}

__global__ void rows_to_fix(const double *__restrict__ rows, const int32_t *__restrict__ user, long long *fx,
                            long long *fy, long long *fz, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double *r = rows + 3 * (size_t)user[i];
    fx[i] = to_fix(r[0], kForceScale);
    fy[i] = to_fix(r[1], kForceScale);
    fz[i] = to_fix(r[2], kForceScale);
  }
}

// Gather whole systems: slot s takes the state of slot perm[s] (systems of
// equal size and topology), atom by atom in the caller's order, since two
// systems may store their atoms in different orders.  src and dst are
// (n, 8-byte word) arrays.
__global__ void gather_systems(const SysInfo *sys, const int32_t *atom_sys, const int32_t *perm,
                               const int32_t *__restrict__ user, const int32_t *__restrict__ devidx,
                               const unsigned long long *__restrict__ src, unsigned long long *dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = atom_sys[i];
    const int u = user[i] - sys[s].off;  // the atom's index in the caller's order
    dst[i] = src[devidx[sys[perm[s]].off + u]];
  }
}

// Per-system term energies (2^-24 fixed point) to FP64, with the total
// summed in term order.
__global__ void energies_to_double(const long long *__restrict__ e, double *out, int n_sys) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_sys; s += gridDim.x * blockDim.x) {
    double tot = 0.0;
    for (int t = 0; t < PB2_TERM_TOTAL; ++t) {
      const double v = (double)e[(size_t)s * PB2_NTERMS + t] * kEnergyInv;
      out[(size_t)s * PB2_NTERMS + t] = v;
      tot += v;
    }
    out[(size_t)s * PB2_NTERMS + PB2_TERM_TOTAL] = tot;
  }
}

// Trajectory frame: float32 positions and velocities (p / m), (n, 3) each
// in the caller's atom order, plus every system's step counter.
__global__ void snapshot_frame(const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ px,
                               const double *__restrict__ py, const double *__restrict__ pz,
                               const double *__restrict__ mass, const long long *__restrict__ steps,
                               const int32_t *__restrict__ user, float *pos, float *vel, long long *frame_steps,
                               int n, int n_sys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double im = 1.0 / mass[i];
    const size_t r = 3 * (size_t)user[i];
    pos[r] = (float)x[i];
    pos[r + 1] = (float)y[i];
    pos[r + 2] = (float)z[i];
    vel[r] = (float)(px[i] * im);
    vel[r + 1] = (float)(py[i] * im);
    vel[r + 2] = (float)(pz[i] * im);
  }
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_sys; s += gridDim.x * blockDim.x)
    frame_steps[s] = steps[s];
}

// The whole BAOAB state (x, p, F) from three consecutive (n, 3) row arrays
// in one pass, and back: one launch on each side of a host round trip, so
// that the three copies of each direction run back to back.
__global__ void state_from_rows(const double *__restrict__ rows, const int32_t *__restrict__ user, double *x,
                                double *y, double *z, double *px, double *py, double *pz, long long *fx,
                                long long *fy, long long *fz, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const size_t u = user[i];
    const double *r = rows + 3 * u;
    const double *q = rows + 3 * ((size_t)n + u);
    const double *f = rows + 3 * (2 * (size_t)n + u);
    x[i] = r[0]; y[i] = r[1]; z[i] = r[2];
    px[i] = q[0]; py[i] = q[1]; pz[i] = q[2];
    fx[i] = to_fix(f[0], kForceScale); fy[i] = to_fix(f[1], kForceScale); fz[i] = to_fix(f[2], kForceScale);
  }
}

__global__ void state_to_rows(const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const double *__restrict__ px,
                              const double *__restrict__ py, const double *__restrict__ pz,
                              const long long *__restrict__ fx, const long long *__restrict__ fy,
                              const long long *__restrict__ fz, const int32_t *__restrict__ user, double *rows,
                              int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const size_t u = user[i];
    double *r = rows + 3 * u;
    double *q = rows + 3 * ((size_t)n + u);
    double *f = rows + 3 * (2 * (size_t)n + u);
    r[0] = x[i]; r[1] = y[i]; r[2] = z[i];
    q[0] = px[i]; q[1] = py[i]; q[2] = pz[i];
    f[0] = (double)fx[i] * kForceInv; f[1] = (double)fy[i] * kForceInv; f[2] = (double)fz[i] * kForceInv;
  }
}

static int grid_for(int n) {
  const int g = (n + 255) / 256;
  return g < 1 ? 1 : (g > 4096 ? 4096 : g);
}

cudaError_t launch_rows_to_soa(const double *rows, const int32_t *user, double *x, double *y, double *z, int n,
                               cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  rows_to_soa<<<grid_for(n), 256, 0, st>>>(rows, user, x, y, z, n);
  return cudaGetLastError();
}

cudaError_t launch_soa_to_rows(const double *x, const double *y, const double *z, const int32_t *user,
                               double *rows, int n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  soa_to_rows<<<grid_for(n), 256, 0, st>>>(x, y, z, user, rows, n);
  return cudaGetLastError();
}

cudaError_t launch_fix_to_rows(const long long *fx, const long long *fy, const long long *fz, const int32_t *user,
                               double *rows, int n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  fix_to_rows<<<grid_for(n), 256, 0, st>>>(fx, fy, fz, user, rows, n);
  return cudaGetLastError();
}

cudaError_t launch_rows_to_fix(const double *rows, const int32_t *user, long long *fx, long long *fy,
                               long long *fz, int n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  rows_to_fix<<<grid_for(n), 256, 0, st>>>(rows, user, fx, fy, fz, n);
  return cudaGetLastError();
}

cudaError_t launch_gather_systems(const SysInfo *sys, const int32_t *atom_sys, const int32_t *perm,
                                  const int32_t *user, const int32_t *devidx, const void *src, void *dst, int n,
                                  cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  gather_systems<<<grid_for(n), 256, 0, st>>>(sys, atom_sys, perm, user, devidx, (const unsigned long long *)src,
                                              (unsigned long long *)dst, n);
  return cudaGetLastError();
}

cudaError_t launch_energies_to_double(const long long *e, double *out, int n_sys, cudaStream_t st) {
  if (n_sys <= 0) return cudaSuccess;
  energies_to_double<<<grid_for(n_sys), 256, 0, st>>>(e, out, n_sys);
  return cudaGetLastError();
}

cudaError_t launch_snapshot(const double *x, const double *y, const double *z, const double *px,
                            const double *py, const double *pz, const double *mass, const long long *steps,
                            const int32_t *user, float *pos, float *vel, long long *frame_steps, int n, int n_sys,
                            cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  snapshot_frame<<<grid_for(n), 256, 0, st>>>(x, y, z, px, py, pz, mass, steps, user, pos, vel, frame_steps, n,
                                              n_sys);
  return cudaGetLastError();
}

cudaError_t launch_state_from_rows(const double *rows, const int32_t *user, double *x, double *y, double *z,
                                   double *px, double *py, double *pz, long long *fx, long long *fy,
                                   long long *fz, int n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  state_from_rows<<<grid_for(n), 256, 0, st>>>(rows, user, x, y, z, px, py, pz, fx, fy, fz, n);
  return cudaGetLastError();
}

cudaError_t launch_state_to_rows(const double *x, const double *y, const double *z, const double *px,
                                 const double *py, const double *pz, const long long *fx, const long long *fy,
                                 const long long *fz, const int32_t *user, double *rows, int n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  state_to_rows<<<grid_for(n), 256, 0, st>>>(x, y, z, px, py, pz, fx, fy, fz, user, rows, n);
  return cudaGetLastError();
}

}  // namespace pb2
