// Bonded terms: harmonic bonds, Urey-Bradley springs and angles, periodic
// torsions, periodic and harmonic impropers and CMAP, all systems of the
// batch in one launch, one thread per term.
//
// Reference: prolix physics/bonded.py:20-185 (bond via jax_md
// simple_spring_bond, E = k/2 (r - r0)^2, also for the Urey-Bradley 1-3
// springs of system.py:93-95; angle with the 1e-8 guard and the
// +-0.999999 clip; dihedral angle b0 = r_i - r_j, b1 = r_k - r_j,
// b2 = r_l - r_k, phi = atan2(y, x); torsion sum k (1 + cos(n phi - delta)),
// also for periodic impropers; harmonic impropers k d^2 with
// d = ((phi - phi0 + pi) mod 2 pi) - pi)
// and physics/cmap.py:316-376 (bicubic patch evaluation at angles mapped to
// [0, 2 pi); phi from row atoms 0-3, psi from 1-4, system.py:99-102), and the
// explicit 1-4 exception pairs of bonded.py:186-230.
//
// These terms are O(N) and stiff: a bond force k (r - r0) needs r - r0 to
// ~1e-7 A, which float32 coordinates cannot give, so the arithmetic is
// FP64 on the FP64 integrator positions.  Forces go to the same 2^32
// fixed-point accumulators as the pair kernels.
#include "pb2_bonded.cuh"

namespace pb2 {

__global__ void bonded_kernel(const BondedArgs a) {
  const int total = bonded_total(a);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) bonded_term(a, t);
}

cudaError_t launch_bonded(const BondedArgs &a, int grid_cap, cudaStream_t st) {
  const int total = a.n_bond + a.n_angle + a.n_tors + a.n_cmap + a.n_exc;
  if (total <= 0) return cudaSuccess;
  int grid = (total + 255) / 256;
  if (grid > grid_cap) grid = grid_cap;
  bonded_kernel<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace pb2
