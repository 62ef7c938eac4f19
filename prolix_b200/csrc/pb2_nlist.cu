// Neighbour lists in jax_md's layout, built with a cell list on the GPU.
//
// Reference: jax_md partition.neighbor_list as prolix uses it
// (physics/neighbor_list.py:155-172; batched_simulate.py:1429-1464), the
// host cell list of physics/cell_list.py:102-242, and the skin rule of
// batched_simulate.py:1600-1622 (rebuild when an atom moved more than
// skin/2 since the last build).  Output: per atom, the local indices of all
// atoms within cutoff + skin (both (i, j) and (j, i) present), padded with
// the sentinel n_atoms of its system; capacity K per atom.
//
// Build, all systems of the batch at once:
//   1. each atom's cell on a per-system grid of cells of edge >= cutoff +
//      skin (atoms outside the grid are clamped to edge cells, which keeps
//      every pair within reach in adjacent cells); counts per cell;
//   2. exclusive scan of the counts; 3. scatter atoms to their cells;
//   4. sort each cell by atom index (so list order is deterministic);
//   5. one warp per atom scans the 27 neighbouring cells in a fixed order
//      and compacts the hits with a ballot into its row.
// The HBM traffic is dominated by step 5's row writes (4 B per entry).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pb2_common.cuh"
#include "pb2_internal.h"
#include "pb2_kernels.cuh"

namespace pb2 {

constexpr int kMaxCellSort = 4096;  // atoms per cell handled by the in-block sort

__global__ void nl_assign_kernel(const NlArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    const NlGrid g = a.grid[s];
    const float4 p = a.posq[i];
    int cx = (int)floorf((p.x - g.x0) * g.inv_cell);
    int cy = (int)floorf((p.y - g.y0) * g.inv_cell);
    int cz = (int)floorf((p.z - g.z0) * g.inv_cell);
    cx = min(max(cx, 0), g.nx - 1);
    cy = min(max(cy, 0), g.ny - 1);
    cz = min(max(cz, 0), g.nz - 1);
    const int c = g.cell_base + (cz * g.ny + cy) * g.nx + cx;
    a.atom_cell[i] = c;
    atomicAdd(&a.cell_count[c], 1);
  }
}

// Exclusive scan of cell_count into cell_start (single block, chunked);
// cell_start[n_cells] = total.  Also clears the scatter cursors.
__global__ void nl_scan_kernel(const NlArgs a) {
  __shared__ int buf[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < a.n_cells; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < a.n_cells ? a.cell_count[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const int t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
      __syncthreads();
      buf[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < a.n_cells) {
      a.cell_start[i] = carry + buf[threadIdx.x] - v;
      a.cell_cursor[i] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 1023) carry += buf[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.cell_start[a.n_cells] = carry;
}

__global__ void nl_scatter_kernel(const NlArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int c = a.atom_cell[i];
    const int slot = atomicAdd(&a.cell_cursor[c], 1);
    a.cell_atoms[a.cell_start[c] + slot] = i;
  }
}

// One block per cell: bitonic sort of the cell's atom indices in shared memory.
__global__ void nl_sort_kernel(const NlArgs a) {
  __shared__ int v[kMaxCellSort];
  for (int c = blockIdx.x; c < a.n_cells; c += gridDim.x) {
    const int start = a.cell_start[c];
    const int cnt = a.cell_start[c + 1] - start;
    if (cnt <= 1) continue;
    if (cnt > kMaxCellSort) {
      if (threadIdx.x == 0) atomicOr(a.error, 1u);
      continue;
    }
    int m = 1;
    while (m < cnt) m <<= 1;
    for (int t = threadIdx.x; t < m; t += blockDim.x) v[t] = t < cnt ? a.cell_atoms[start + t] : 0x7fffffff;
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int t = threadIdx.x; t < m; t += blockDim.x) {
          const int p = t ^ j;
          if (p > t) {
            const bool up = (t & k) == 0;
            const int x = v[t], y = v[p];
            if ((x > y) == up) { v[t] = y; v[p] = x; }
          }
        }
        __syncthreads();
      }
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) a.cell_atoms[start + t] = v[t];
    __syncthreads();
  }
}

// One warp per atom: scan the 27 cells around its cell, keep j != i within
// reach, write local indices; count beyond the capacity only counts.
__global__ void nl_rows_kernel(const NlArgs a) {
  const int lane = threadIdx.x & 31;
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int i = w; i < a.n_total; i += nw) {
    const int s = a.atom_sys[i];
    const NlGrid g = a.grid[s];
    const int off = g.atom_off;
    const float4 p = a.posq[i];
    const int lc = a.atom_cell[i] - g.cell_base;
    const int cx = lc % g.nx, cy = (lc / g.nx) % g.ny, cz = lc / (g.nx * g.ny);
    int count = 0;
    int *row = a.rows + (size_t)i * a.capacity;
    for (int dz = -1; dz <= 1; ++dz) {
      const int z = cz + dz;
      if (z < 0 || z >= g.nz) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = cy + dy;
        if (y < 0 || y >= g.ny) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = cx + dx;
          if (x < 0 || x >= g.nx) continue;
          const int c = g.cell_base + (z * g.ny + y) * g.nx + x;
          const int st = a.cell_start[c], en = a.cell_start[c + 1];
          for (int b = st; b < en; b += 32) {
            const int k = b + lane;
            int j = -1;
            bool hit = false;
            if (k < en) {
              j = a.cell_atoms[k];
              if (j != i) {
                const float4 q = a.posq[j];
                const float ex = p.x - q.x, ey = p.y - q.y, ez = p.z - q.z;
                hit = fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < g.reach2;
              }
            }
            const unsigned m = __ballot_sync(kFull, hit);
            if (hit) {
              const int slot = count + __popc(m & ((1u << lane) - 1u));
              if (slot < a.capacity) row[slot] = j - off;
            }
            count += __popc(m);
          }
        }
      }
    }
    for (int t = count + lane; t < a.capacity; t += 32) row[t] = g.n;  // sentinel
    if (lane == 0) {
      a.counts[i] = count;
      if (count > a.capacity) atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NLOVERFLOW);
    }
  }
}

// Largest squared displacement per system since the last build (FP64).
__global__ void nl_disp_kernel(const NlArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const double dx = a.x[i] - a.xref[i], dy = a.y[i] - a.xref[a.n_total + i],
                 dz = a.z[i] - a.xref[2 * (size_t)a.n_total + i];
    const float d2 = (float)(dx * dx + dy * dy + dz * dz);
    atomicMax(&a.max_disp2[a.atom_sys[i]], __float_as_int(d2));  // d2 >= 0: int order = float order
  }
}

__global__ void nl_ref_kernel(const NlArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    a.xref[i] = a.x[i];
    a.xref[a.n_total + i] = a.y[i];
    a.xref[2 * (size_t)a.n_total + i] = a.z[i];
  }
}

static int grid_for(int n, int per) { return std::max(1, std::min((n + per - 1) / per, 65535)); }

cudaError_t nl_launch_build(const NlArgs &a, cudaStream_t st) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(a.cell_count, 0, (size_t)a.n_cells * sizeof(int), st)) != cudaSuccess) return e;
  nl_assign_kernel<<<grid_for(a.n_total, 256), 256, 0, st>>>(a);
  nl_scan_kernel<<<1, 1024, 0, st>>>(a);
  nl_scatter_kernel<<<grid_for(a.n_total, 256), 256, 0, st>>>(a);
  nl_sort_kernel<<<grid_for(a.n_cells, 1), 256, 0, st>>>(a);
  nl_rows_kernel<<<grid_for(a.n_total, 8), 256, 0, st>>>(a);
  nl_ref_kernel<<<grid_for(a.n_total, 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t nl_launch_disp(const NlArgs &a, cudaStream_t st) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(a.max_disp2, 0, (size_t)a.n_sys * sizeof(int), st)) != cudaSuccess) return e;
  nl_disp_kernel<<<grid_for(a.n_total, 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace pb2

// ------------------------------------------------------------ host side

static double nl_reach(const pb2_batch *b) {
  const double c = std::max(b->params.cutoff, b->params.gb_cutoff < 0 ? b->params.cutoff
                                                                      : b->params.gb_cutoff);
  return c + std::max(b->params.skin, 0.0);
}

static NlArgs nl_args(pb2_batch *b) {
  NlArgs a;
  a.atom_sys = b->atom_sys;
  a.grid = b->nl_grid;
  a.posq = b->posq;
  a.x = b->x; a.y = b->y; a.z = b->z;
  a.xref = b->nl_xref;
  a.atom_cell = b->nl_atom_cell;
  a.cell_count = b->nl_cell_count;
  a.cell_start = b->nl_cell_start;
  a.cell_cursor = b->nl_cell_cursor;
  a.cell_atoms = b->nl_cell_atoms;
  a.rows = b->nl_rows;
  a.counts = b->nl_counts;
  a.capacity = b->nl_capacity;
  a.n_total = b->n_total;
  a.n_cells = b->nl_cells;
  a.n_sys = b->n_sys;
  a.status = b->status;
  a.error = b->nl_error;
  a.max_disp2 = b->nl_max_disp2;
  return a;
}

// Per-system grids from the current block bounding boxes; (re)allocates
// the cell arrays when the total cell count grows.
static int nl_setup(pb2_batch *b, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  const double reach = nl_reach(b);
  CUDA_TRY(ctx, launch_posq(int_args_for_nl(b), st));
  CUDA_TRY(ctx, launch_bbox(b->sys, b->blk_sys, b->posq, b->bbox, b->n_blocks, st));
  std::vector<float4> bb(2 * (size_t)b->n_blocks);
  CUDA_TRY(ctx, cudaMemcpyAsync(bb.data(), b->bbox, bb.size() * sizeof(float4), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  std::vector<NlGrid> grids(b->n_sys);
  int cells = 0;
  for (int s = 0; s < b->n_sys; ++s) {
    const SysInfo &S = b->sys_host[s];
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (int k = 0; k < S.nblk; ++k) {
      const float4 l = bb[2 * (size_t)(S.blk_base + k)], h = bb[2 * (size_t)(S.blk_base + k) + 1];
      lo[0] = std::min(lo[0], l.x); lo[1] = std::min(lo[1], l.y); lo[2] = std::min(lo[2], l.z);
      hi[0] = std::max(hi[0], h.x); hi[1] = std::max(hi[1], h.y); hi[2] = std::max(hi[2], h.z);
    }
    double cell = reach;
    const double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]}) + 2.0 * reach;
    if (ext / cell > 128.0) cell = ext / 128.0;
    NlGrid &g = grids[s];
    g.x0 = lo[0] - (float)reach; g.y0 = lo[1] - (float)reach; g.z0 = lo[2] - (float)reach;
    g.inv_cell = (float)(1.0 / cell);
    g.nx = std::max(1, (int)std::ceil((hi[0] - lo[0] + 2.0 * reach) / cell));
    g.ny = std::max(1, (int)std::ceil((hi[1] - lo[1] + 2.0 * reach) / cell));
    g.nz = std::max(1, (int)std::ceil((hi[2] - lo[2] + 2.0 * reach) / cell));
    g.cell_base = cells;
    g.n = S.n;
    g.atom_off = S.off;
    g.reach2 = (float)(reach * reach);
    g.pad = 0;
    cells += g.nx * g.ny * g.nz;
  }
  Dev &D = b->nl;
  if (!b->nl_grid) {
    b->nl_grid = D.alloc<NlGrid>(b->n_sys);
    b->nl_atom_cell = D.alloc<int>(b->n_total);
    b->nl_counts = D.alloc<int>(b->n_total);
    b->nl_xref = D.alloc<double>(3 * (size_t)b->n_total);
    b->nl_max_disp2 = D.alloc<int>(b->n_sys);
    b->nl_error = D.alloc<unsigned>(1);
    b->nl_cell_atoms = D.alloc<int>(b->n_total);
    if (!b->nl_grid || !b->nl_atom_cell || !b->nl_counts || !b->nl_xref || !b->nl_max_disp2 ||
        !b->nl_error || !b->nl_cell_atoms)
      return fail(ctx, PB2_ENOMEM, "neighbour-list allocation failed");
    CUDA_TRY(ctx, cudaMemsetAsync(b->nl_error, 0, sizeof(unsigned), st));
  }
  if (cells > b->nl_cells) {
    D.release(b->nl_cell_count);
    D.release(b->nl_cell_start);
    D.release(b->nl_cell_cursor);
    b->nl_cell_count = D.alloc<int>(cells);
    b->nl_cell_start = D.alloc<int>(cells + 1);
    b->nl_cell_cursor = D.alloc<int>(cells);
    if (!b->nl_cell_count || !b->nl_cell_start || !b->nl_cell_cursor)
      return fail(ctx, PB2_ENOMEM, "neighbour-list cell allocation failed");
  }
  b->nl_cells = cells;
  CUDA_TRY(ctx, cudaMemcpyAsync(b->nl_grid, grids.data(), grids.size() * sizeof(NlGrid),
                                cudaMemcpyHostToDevice, st));
  return PB2_OK;
}

static int nl_alloc_rows(pb2_batch *b, int capacity) {
  pb2_ctx *ctx = b->ctx;
  b->nl.release(b->nl_rows);
  b->nl_rows = b->nl.alloc<int>((size_t)b->n_total * std::max(capacity, 1));
  if (!b->nl_rows) return fail(ctx, PB2_ENOMEM, "neighbour-list rows allocation failed");
  b->nl_capacity = capacity;
  return PB2_OK;
}

static int nl_max_count(pb2_batch *b, cudaStream_t st, int *out) {
  pb2_ctx *ctx = b->ctx;
  std::vector<int> c(b->n_total);
  CUDA_TRY(ctx, cudaMemcpyAsync(c.data(), b->nl_counts, c.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  unsigned err = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&err, b->nl_error, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (err) return fail(ctx, PB2_ENLOVERFLOW, "a neighbour-list cell holds more than 4096 atoms");
  *out = c.empty() ? 0 : *std::max_element(c.begin(), c.end());
  return PB2_OK;
}

static int nl_build_all(pb2_batch *b, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  if (!(b->params.cutoff > 0.0 || b->params.gb_cutoff > 0.0))
    return fail(ctx, PB2_EINVAL, "a neighbour list needs cutoff > 0 (or gb_cutoff > 0)");
  int rc = nl_setup(b, st);
  if (rc) return rc;
  const int fixed = b->params.nl_capacity;
  if (!b->nl_rows) {
    rc = nl_alloc_rows(b, fixed > 0 ? fixed : 0);
    if (rc) return rc;
  }
  for (int attempt = 0; attempt < 4; ++attempt) {
    CUDA_TRY(ctx, nl_launch_build(nl_args(b), st));
    int maxc = 0;
    rc = nl_max_count(b, st, &maxc);
    if (rc) return rc;
    if (maxc <= b->nl_capacity) {
      b->nl_built = true;
      return PB2_OK;
    }
    if (fixed > 0) {
      char buf[160];
      snprintf(buf, sizeof buf, "neighbour-list capacity %d exceeded (an atom has %d neighbours)",
               fixed, maxc);
      return fail(ctx, PB2_ENLOVERFLOW, buf);
    }
    rc = nl_alloc_rows(b, ((maxc + maxc / 4 + 8 + 31) / 32) * 32);
    if (rc) return rc;
    // the overflow pass set the status bit; the rebuild supersedes it
    CUDA_TRY(ctx, cudaMemsetAsync(b->status, 0, b->n_sys * sizeof(uint32_t), st));
  }
  return fail(ctx, PB2_ENLOVERFLOW, "neighbour-list capacity did not converge");
}

extern "C" int pb2_nl_build(pb2_batch *b, void *stream) {
  if (!b) return PB2_EINVAL;
  CUDA_TRY(b->ctx, cudaSetDevice(b->ctx->device));
  return nl_build_all(b, (cudaStream_t)stream);
}

extern "C" int pb2_nl_check(pb2_batch *b, int32_t *rebuilt, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  if (rebuilt) *rebuilt = 0;
  if (!b->nl_built) {
    const int rc = nl_build_all(b, st);
    if (rc == PB2_OK && rebuilt) *rebuilt = b->n_sys;
    return rc;
  }
  CUDA_TRY(ctx, nl_launch_disp(nl_args(b), st));
  std::vector<int> d(b->n_sys);
  CUDA_TRY(ctx, cudaMemcpyAsync(d.data(), b->nl_max_disp2, d.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  int moved = 0;
  for (int s = 0; s < b->n_sys; ++s) {
    float v;
    std::memcpy(&v, &d[s], sizeof v);
    if ((double)v > b->sys_host[s].skin_half2) ++moved;
  }
  if (moved == 0) return PB2_OK;
  const int rc = nl_build_all(b, st);
  if (rc == PB2_OK && rebuilt) *rebuilt = moved;
  return rc;
}

extern "C" int pb2_nl_capacity(const pb2_batch *b, int32_t *capacity) {
  if (!b || !capacity) return PB2_EINVAL;
  *capacity = b->nl_built ? b->nl_capacity : 0;
  return PB2_OK;
}

extern "C" int pb2_nl_get(pb2_batch *b, int32_t *neighbors, void *stream) {
  if (!b || !neighbors) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (!b->nl_built) return fail(ctx, PB2_EINVAL, "no neighbour list built yet");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t cap = (size_t)b->nl_capacity;
  std::vector<int> rows((size_t)b->n_total * cap);
  CUDA_TRY(ctx, cudaMemcpyAsync(rows.data(), b->nl_rows, rows.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  // rows and neighbour indices in the caller's atom order (local indices;
  // the sentinel, the system's atom count, stays)
  for (int s = 0; s < b->n_sys; ++s) {
    const int off = b->off[s], n = b->nat[s];
    for (int l = 0; l < n; ++l) {
      const int g = off + l;
      const int *src = &rows[(size_t)g * cap];
      int32_t *dst = neighbors + (size_t)b->user_host[g] * cap;
      for (size_t k = 0; k < cap; ++k) dst[k] = src[k] >= n ? src[k] : b->user_host[off + src[k]] - off;
    }
  }
  return PB2_OK;
}
