// Pair list of the cutoff runs: for every pair of i-blocks (ib, ib + 1) of a
// system, the j-blocks (jb >= ib) whose bounding boxes come within
// cutoff + skin of either i-block, compacted, and the work items of the
// pair kernels over them.
//
// This is the skin-buffered neighbour list of prolix's production loop
// (jax_md partition.neighbor_list with dr_threshold, rebuilt when an atom
// has moved more than half the skin since the last build;
// batched_simulate.py:1429-1464, :1600-1622), at the granularity the pair
// kernels work in: 32-atom blocks of spatially sorted atoms, so a tile is
// kept or dropped whole.  Keeping every block pair within cutoff + skin at
// build time keeps every atom pair that comes within the cutoff before any
// atom has moved skin / 2 (a block's box moves by at most that much per
// side, so box separations shrink by at most the skin).  The pair kernels
// still skip listed tiles that are beyond the cutoff at the current step.
//
// Everything stays on the device: the step kernel (or, outside a step, the
// bounding-box kernel) raises the rebuild flag when an atom has moved more
// than skin/2 from the positions of the last build, and this kernel,
// launched every step of a cutoff run
// (inside the captured step graphs), returns at once unless the flag is
// set.  A rebuild writes the new items into the buffer the pair kernels
// are not reading, and the last warp to finish publishes it, so no launch
// needs the host.
#include "pb2_common.cuh"
#include "pb2_kernels.cuh"

namespace pb2 {

__device__ __forceinline__ float pl_box_dist2(const float4 *bbox, int a, int b) {
  const float4 alo = bbox[2 * a], ahi = bbox[2 * a + 1];
  const float4 blo = bbox[2 * b], bhi = bbox[2 * b + 1];
  const float dx = fmaxf(0.f, fmaxf(alo.x - bhi.x, blo.x - ahi.x));
  const float dy = fmaxf(0.f, fmaxf(alo.y - bhi.y, blo.y - ahi.y));
  const float dz = fmaxf(0.f, fmaxf(alo.z - bhi.z, blo.z - ahi.z));
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// One warp per list row (a pair of i-blocks).
__global__ void pl_update_kernel(const PlArgs a) {
  if (a.ctl[PL_DIRTY] == 0) return;  // the whole grid sees the same flag
  const int lane = threadIdx.x & 31;
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int nxt = a.ctl[PL_CUR] ^ 1;
  TileItem *out = nxt ? a.items1 : a.items0;
  for (int r = w; r < a.n_rows; r += nw) {
    const PlRow row = a.rows[r];
    if (a.retired[row.sys]) continue;  // a retired system lists no work
    const SysInfo &S = a.sys[row.sys];
    const int ib = row.iblk;
    const bool has1 = ib + 1 < S.nblk;
    const int gib0 = S.blk_base + ib, gib1 = gib0 + 1;
    // the new displacement reference of the row's atoms
    for (int k = lane; k < 64; k += 32) {
      const int l = ib * 32 + k;
      if (l < S.n) a.ref[S.off + l] = a.posq[S.off + l];
    }
    int cnt = 0;
    for (int j0 = ib; j0 < S.nblk; j0 += 32) {
      const int jb = j0 + lane;
      bool live = false;
      if (jb < S.nblk) {
        float d2 = pl_box_dist2(a.bbox, gib0, S.blk_base + jb);
        if (has1 && jb > ib) d2 = fminf(d2, pl_box_dist2(a.bbox, gib1, S.blk_base + jb));
        live = d2 < a.reach2;
      }
      const unsigned m = __ballot_sync(kFull, live);
      if (live) a.jlist[row.jbase + cnt + __popc(m & ((1u << lane) - 1u))] = jb;
      cnt += __popc(m);
    }
    const int nit = (cnt + a.seg - 1) / a.seg;
    int base = 0;
    if (lane == 0 && nit > 0) {
      base = atomicAdd(&a.ctl[PL_NEW], nit);
      atomicAdd(&(nxt ? a.sys_items1 : a.sys_items0)[row.sys], nit);
    }
    base = __shfl_sync(kFull, base, 0);
    for (int k = lane; k < nit; k += 32)
      out[base + k] = TileItem{row.sys, ib, row.jbase + k * a.seg, row.jbase + min((k + 1) * a.seg, cnt)};
  }
  // the last warp publishes the new list, clears the per-system counts of
  // the buffer the next build will write, and clears the flag
  __syncwarp();
  int last = 0;
  if (lane == 0) {
    __threadfence();
    last = atomicAdd(&a.ctl[PL_DONE], 1) == nw - 1;
  }
  if (__shfl_sync(kFull, last, 0)) {
    __threadfence();
    int32_t *old_counts = nxt ? a.sys_items0 : a.sys_items1;
    for (int s = lane; s < a.n_sys; s += 32) old_counts[s] = 0;
    if (lane == 0) {
      a.ctl[PL_COUNT0 + nxt] = atomicAdd(&a.ctl[PL_NEW], 0);
      a.ctl[PL_NEW] = 0;
      a.ctl[PL_DONE] = 0;
      a.ctl[PL_CUR] = nxt;
      a.ctl[PL_DIRTY] = 0;
    }
    __threadfence();
  }
}

cudaError_t launch_pl_update(const PlArgs &a, int grid, cudaStream_t st) {
  if (a.n_rows <= 0) return cudaSuccess;
  pl_update_kernel<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

// Retire a system and re-list the live work items: an ordered compaction
// of the full list by one thread block (the list is a few thousand items
// per thousand atoms; one block keeps the order without a second pass).
constexpr int kRetireThreads = 1024;
__global__ void __launch_bounds__(kRetireThreads) retire_kernel(int32_t sys, int8_t *retired, const TileItem *all,
                                                                 int n_all, TileItem *live, int32_t *count,
                                                                 int32_t *pl_ctl) {
  __shared__ int warp_sum[kRetireThreads / 32];
  __shared__ int base;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    if (sys >= 0) {
      retired[sys] = 1;
      if (pl_ctl) pl_ctl[PL_DIRTY] = 1;
    }
    base = 0;
  }
  __syncthreads();
  for (int k0 = 0; k0 < n_all; k0 += kRetireThreads) {
    const int k = k0 + threadIdx.x;
    TileItem t{};
    bool keep = false;
    if (k < n_all) {
      t = all[k];
      keep = retired[t.sys] == 0;
    }
    const unsigned m = __ballot_sync(kFull, keep);
    if (lane == 0) warp_sum[w] = __popc(m);
    __syncthreads();
    int before = base;
    for (int v = 0; v < w; ++v) before += warp_sum[v];
    if (keep) live[before + __popc(m & ((1u << lane) - 1u))] = t;
    __syncthreads();
    if (threadIdx.x == kRetireThreads - 1) base = before + __popc(m);
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = base;
}

cudaError_t launch_retire(int32_t sys, int8_t *retired, const TileItem *all, int n_all, TileItem *live,
                          int32_t *count, int32_t *pl_ctl, cudaStream_t st) {
  retire_kernel<<<1, kRetireThreads, 0, st>>>(sys, retired, all, n_all, live, count, pl_ctl);
  return cudaGetLastError();
}

}  // namespace pb2
