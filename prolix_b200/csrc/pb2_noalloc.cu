// Born radii of one system without any device allocation.
//
// Who needs this: callers that cannot call cudaMalloc.  Examples are code
// running inside an XLA custom call, where the runtime owns every buffer
// and the handler gets only the operands and results it declared; code
// that runs while a CUDA stream is being captured into a graph, where
// cudaMalloc is not a legal stream operation; and embedded hosts that hand
// the library a fixed memory pool.  Those callers can still pass device
// buffers for inputs and outputs, so this entry point asks only for those.
//
// The descreening sums need 64-bit scratch per atom.  Here it lives in a
// file-scope __device__ array of PB2_NOALLOC_MAX_ATOMS entries (256 KiB),
// which every GPU that loads this library holds until the process exits.
// Host code reaches it only through cudaGetSymbolAddress: in host code the
// array's name is a host-side stand-in, not a device address.  The address
// is looked up once per device, on the first call made with that device
// current; make that first call before any stream capture.  After a
// cudaDeviceReset the cached address no longer names device memory and the
// next call looks it up again (so that call, too, belongs outside a
// capture).  Every buffer must be device memory of the current device, and
// with a context that device must be the context's.
//
// All calls share the one array and it keeps the last call's contents, so
// every call clears the part it uses first.  Calls whose kernels overlap on
// the GPU (different streams, or different host threads on one device)
// race on the array and give wrong results: serialise them.
#include <mutex>

#include "pb2_common.cuh"
#include "pb2_internal.h"
#include "pb2_kernels.cuh"
#include "pb2_pairmath.cuh"

namespace pb2 {

static __device__ __align__(256) long long g_noalloc_sum[PB2_NOALLOC_MAX_ATOMS];

__global__ void noalloc_clear(long long *acc, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[i] = 0;
}

// One warp per 32 x 32 tile (ib, jb), jb >= ib; both halves of each
// unique pair's descreening, as the batched born pass does.
__global__ void noalloc_born_tiles(const double *pos, const double *radii, const double *sr, int n,
                                   float cut2, int clamp, long long *acc) {
  const int lane = threadIdx.x & 31;
  const int nb = (n + 31) / 32;
  const long long n_tiles = (long long)nb * (nb + 1) / 2;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  // a fixed origin near the system keeps float32 coordinates small
  const double ox = rint(pos[0]), oy = rint(pos[1]), oz = rint(pos[2]);
  for (long long t = warp0; t < n_tiles; t += nwarps) {
    // row ib holds nb - ib tiles; find ib with start(ib) <= t < start(ib + 1)
    int ib = (int)((2.0 * nb + 1.0 - sqrt((2.0 * nb + 1.0) * (2.0 * nb + 1.0) - 8.0 * (double)t)) * 0.5);
    if (ib < 0) ib = 0;
    if (ib > nb - 1) ib = nb - 1;
    while (ib > 0 && (long long)ib * nb - (long long)ib * (ib - 1) / 2 > t) --ib;
    while (ib < nb - 1 && (long long)(ib + 1) * nb - (long long)(ib + 1) * ib / 2 <= t) ++ib;
    const int jb = ib + (int)(t - ((long long)ib * nb - (long long)ib * (ib - 1) / 2));
    const int il = ib * 32 + lane, jl = jb * 32 + lane;
    const bool ivalid = il < n, jvalid = jl < n;
    const int ic = ivalid ? il : n - 1, jc0 = jvalid ? jl : n - 1;
    const float xi = (float)(pos[3 * ic] - ox), yi = (float)(pos[3 * ic + 1] - oy),
                zi = (float)(pos[3 * ic + 2] - oz);
    double ri = radii[ic];
    double ro_i = ri - kDielOffset;
    if (clamp) ro_i = fmax(fmax(ri, 1e-6) - kDielOffset, 1e-4);
    const float roi = (float)ro_i, sri = (float)sr[ic];
    float xj = (float)(pos[3 * jc0] - ox), yj = (float)(pos[3 * jc0 + 1] - oy),
          zj = (float)(pos[3 * jc0 + 2] - oz);
    double rj = radii[jc0];
    double ro_j = rj - kDielOffset;
    if (clamp) ro_j = fmax(fmax(rj, 1e-6) - kDielOffset, 1e-4);
    float roj = (float)ro_j, srj = (float)sr[jc0];
    const bool diag = ib == jb;
    float ti = 0.f, tj = 0.f;
    for (int k = 0; k < 32; ++k) {
      const int jc = (lane + k) & 31;
      bool ok = ivalid && (jb * 32 + jc < n) && (!diag || jc > lane);
      const float dx = xi - xj, dy = yi - yj, dz = zi - zj;
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (cut2 > 0.f) ok = ok && r2 < cut2;
      if (ok) {
        const float inv_r = rsqrtf(r2);
        const float r = r2 * inv_r;
        ti += obc_integral(r, inv_r, roi, srj);
        tj += obc_integral(r, inv_r, roj, sri);
      }
      const int src = (lane + 1) & 31;
      xj = __shfl_sync(kFull, xj, src); yj = __shfl_sync(kFull, yj, src);
      zj = __shfl_sync(kFull, zj, src);
      roj = __shfl_sync(kFull, roj, src); srj = __shfl_sync(kFull, srj, src);
      tj = __shfl_sync(kFull, tj, src);
    }
    if (jvalid && tj != 0.f) atomic_add_fix(&acc[jl], to_fix_f(tj, (float)kBornScale));
    if (ivalid && ti != 0.f) atomic_add_fix(&acc[il], to_fix_f(ti, (float)kBornScale));
  }
}

// B_i = 1 / (1/rho~ - tanh(a Psi - b Psi^2 + c Psi^3) / rho), Psi = rho~ I
// (prolix physics/generalized_born.py:85-94; clamps of :300-337 when clamp).
__global__ void noalloc_born_finalize(const double *radii, const long long *acc, int n, int clamp,
                                      double *born) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double isum = (double)acc[i] * kBornInv;
    const double r_in = radii[i];
    const double rad = clamp ? fmax(r_in, 1e-6) : r_in;
    double ro = rad - kDielOffset;
    if (clamp) ro = fmax(ro, 1e-4);
    const double psi = ro * isum;
    const double th = tanh(kObcAlpha * psi - kObcBeta * psi * psi + kObcGamma * psi * psi * psi);
    const double dr = clamp ? fmax(rad, 1e-4) : rad;
    double inv_b = 1.0 / ro - th / dr;
    if (clamp) inv_b = fmax(inv_b, 1e-4);
    born[i] = 1.0 / inv_b;
  }
}

}  // namespace pb2

using namespace pb2;

static std::mutex g_noalloc_lock;
static long long *g_noalloc_addr[64];

// True when p is device (or managed) memory of device dev.
static bool on_device(const void *p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // an unknown pointer leaves an error behind on old runtimes
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

extern "C" int pb2_born_radii_noalloc(pb2_ctx *ctx, int32_t n_atoms, const double *positions,
                                      const double *radii, const double *scaled_radii,
                                      double cutoff, double *born, void *stream) {
  if (!positions || !radii || !scaled_radii || !born)
    return set_error(ctx, PB2_EINVAL, "pb2_born_radii_noalloc: NULL buffer");
  if (n_atoms <= 0 || n_atoms > PB2_NOALLOC_MAX_ATOMS)
    return set_error(ctx, PB2_EINVAL,
                     "pb2_born_radii_noalloc: n_atoms must be in 1..PB2_NOALLOC_MAX_ATOMS (32768)");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return set_error(ctx, PB2_ENODEV, "pb2_born_radii_noalloc: no current CUDA device");
  if (ctx && dev != ctx->device)
    return set_error(ctx, PB2_EINVAL,
                     "pb2_born_radii_noalloc: the current CUDA device is not the context's device");
  if (!on_device(positions, dev) || !on_device(radii, dev) || !on_device(scaled_radii, dev) ||
      !on_device(born, dev))
    return set_error(ctx, PB2_EINVAL,
                     "pb2_born_radii_noalloc: every buffer must be device memory of the current device");
  long long *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_lock);
    // looked up once per device; a cudaDeviceReset in between unloads the
    // module, the cached address stops being device memory, and it is
    // looked up again
    if (g_noalloc_addr[dev] && !on_device(g_noalloc_addr[dev], dev)) g_noalloc_addr[dev] = nullptr;
    if (!g_noalloc_addr[dev]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_sum);
      if (e != cudaSuccess || !p)
        return set_error(ctx, PB2_ECUDA, "pb2_born_radii_noalloc: cudaGetSymbolAddress failed");
      g_noalloc_addr[dev] = static_cast<long long *>(p);
    }
    scratch = g_noalloc_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int n = n_atoms;
  const int clamp = cutoff > 0.0 ? 1 : 0;
  const float cut2 = clamp ? (float)(cutoff * cutoff) : 0.f;
  const int nb = (n + 31) / 32;
  const long long tiles = (long long)nb * (nb + 1) / 2;
  const int grid_atoms = (n + 255) / 256;
  int grid_tiles = (int)((tiles + 7) / 8);
  if (grid_tiles > 4096) grid_tiles = 4096;
  cudaGetLastError();  // an earlier, unrelated launch error is not this call's
  noalloc_clear<<<grid_atoms, 256, 0, st>>>(scratch, n);
  noalloc_born_tiles<<<grid_tiles, 256, 0, st>>>(positions, radii, scaled_radii, n, cut2, clamp, scratch);
  noalloc_born_finalize<<<grid_atoms, 256, 0, st>>>(radii, scratch, n, clamp, born);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(ctx, PB2_ECUDA, cudaGetErrorString(e));
  return PB2_OK;
}
