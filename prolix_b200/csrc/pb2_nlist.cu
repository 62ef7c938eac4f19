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
// Everything runs on the device, all systems of the batch at once, as a
// fixed sequence of launches that needs no host decision:
//   0. (check) each atom's displacement since the last build against
//      skin/2 sets the rebuild flag and its system's moved flag;
//   1. per system, a cell grid over the current block bounding boxes, cell
//      edge reach/2 (searched two cells out), widened where the system
//      would need more cells than its budget (2 per atom, at least 64);
//   2. each atom's cell and the counts per cell;
//   3. per system, an exclusive scan of its cells' counts;
//   4. atoms scattered to their cells; 5. each cell sorted by atom index
//      (list order is deterministic);
//   6. one thread block per cell: the cell's atoms test, from shared memory,
//      the atoms of the surrounding cells, each thread writing its atom's
//      row; rows beyond the capacity only count (the largest count and an
//      overflow bit are recorded for the host's next visit);
//   7. the positions become the new displacement reference; the last block
//      clears the flag.
// Each kernel returns at once while the flag is clear, so a check that
// finds nothing to do costs one launch per kernel and no host round trip.
// The HBM traffic is dominated by step 6's row writes (4 B per entry).
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
constexpr int kRowsThreads = 128;   // threads per cell block of the row pass

__device__ __forceinline__ bool nl_dirty(const NlArgs &a) { return *(volatile int32_t *)&a.ctl[NL_DIRTY] != 0; }

// 0. displacement since the last build (FP64 state) against skin/2
__global__ void nl_disp_kernel(const NlArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int s = a.atom_sys[i];
    const double dx = a.x[i] - a.xref[i], dy = a.y[i] - a.xref[a.n_total + i],
                 dz = a.z[i] - a.xref[2 * (size_t)a.n_total + i];
    if (dx * dx + dy * dy + dz * dz > a.sys[s].skin_half2) {
      a.sys_moved[s] = 1;
      a.ctl[NL_DIRTY] = 1;
    }
  }
}

// 1. per-system grid, one warp per system; also clears the system's cells
__global__ void nl_grid_kernel(const NlArgs a) {
  if (!nl_dirty(a)) return;
  const int lane = threadIdx.x & 31;
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int s = w; s < a.n_sys; s += nw) {
    const SysInfo &S = a.sys[s];
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (int k = lane; k < S.nblk; k += 32) {
      const float4 l = a.bbox[2 * (S.blk_base + k)], h = a.bbox[2 * (S.blk_base + k) + 1];
      lo[0] = fminf(lo[0], l.x); lo[1] = fminf(lo[1], l.y); lo[2] = fminf(lo[2], l.z);
      hi[0] = fmaxf(hi[0], h.x); hi[1] = fmaxf(hi[1], h.y); hi[2] = fmaxf(hi[2], h.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = fminf(lo[c], __shfl_xor_sync(kFull, lo[c], o));
        hi[c] = fmaxf(hi[c], __shfl_xor_sync(kFull, hi[c], o));
      }
    const int budget = a.cell_budget[s];
    // edge reach/2; widened until the grid fits the budget
    double edge = 0.5 * (double)a.reach;
    int n[3];
    for (int it = 0; it < 64; ++it) {
      long long cells = 1;
      for (int c = 0; c < 3; ++c) {
        n[c] = max(1, (int)ceil(((double)hi[c] - (double)lo[c]) / edge + 1e-6));
        cells *= n[c];
      }
      if (cells <= budget) break;
      edge *= fmax(1.01, cbrt((double)cells / budget));
    }
    if (lane == 0) {
      NlGrid g;
      g.x0 = lo[0]; g.y0 = lo[1]; g.z0 = lo[2];
      g.inv_cell = (float)(1.0 / edge);
      g.nx = n[0]; g.ny = n[1]; g.nz = n[2];
      g.stencil = (int)ceil((double)a.reach / edge - 1e-9);
      a.grid[s] = g;
    }
    const int base = a.cell_base[s];
    for (int c = lane; c < budget; c += 32) {
      a.cell_count[base + c] = 0;
      a.cell_cursor[base + c] = 0;
    }
  }
}

// 2. cell of each atom (clamped into the grid) and the counts
__global__ void nl_assign_kernel(const NlArgs a) {
  if (!nl_dirty(a)) return;
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
    const int c = a.cell_base[s] + (cz * g.ny + cy) * g.nx + cx;
    a.atom_cell[i] = c;
    atomicAdd(&a.cell_count[c], 1);
  }
}

// 3. exclusive scan of a system's cell counts, one block per system; cells
// past the grid (unused budget) start at the system's end
__global__ void nl_scan_kernel(const NlArgs a) {
  if (!nl_dirty(a)) return;
  __shared__ int buf[1024];
  __shared__ int carry;
  for (int s = blockIdx.x; s < a.n_sys; s += gridDim.x) {
    const SysInfo &S = a.sys[s];
    const NlGrid g = a.grid[s];
    const int base = a.cell_base[s], budget = a.cell_budget[s];
    const int used = g.nx * g.ny * g.nz;
    if (threadIdx.x == 0) carry = S.off;
    __syncthreads();
    for (int c0 = 0; c0 < used; c0 += 1024) {
      const int c = c0 + threadIdx.x;
      const int v = c < used ? a.cell_count[base + c] : 0;
      buf[threadIdx.x] = v;
      __syncthreads();
      for (int o = 1; o < 1024; o <<= 1) {
        const int t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
        __syncthreads();
        buf[threadIdx.x] += t;
        __syncthreads();
      }
      if (c < used) a.cell_start[base + c] = carry + buf[threadIdx.x] - v;
      __syncthreads();
      if (threadIdx.x == 1023) carry += buf[1023];
      __syncthreads();
    }
    for (int c = used + threadIdx.x; c <= budget; c += blockDim.x) a.cell_start[base + c] = S.off + S.n;
    __syncthreads();
  }
}

// 4. scatter atoms to their cells
__global__ void nl_scatter_kernel(const NlArgs a) {
  if (!nl_dirty(a)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    const int c = a.atom_cell[i];
    const int slot = atomicAdd(&a.cell_cursor[c], 1);
    a.cell_atoms[a.cell_start[c] + slot] = i;
  }
}

// 5. one block per cell: bitonic sort of the cell's atom indices in shared memory
__global__ void nl_sort_kernel(const NlArgs a) {
  if (!nl_dirty(a)) return;
  __shared__ int v[kMaxCellSort];
  for (int c = blockIdx.x; c < a.n_cells; c += gridDim.x) {
    const int start = a.cell_start[c];
    const int cnt = a.cell_count[c];
    if (cnt <= 1) continue;
    if (cnt > kMaxCellSort) {
      if (threadIdx.x == 0) atomicOr(&a.ctl[NL_CELLFULL], 1);
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

// 6. rows: one block per cell, one thread per atom of the cell (in chunks);
// the surrounding cells' atoms pass through shared memory in a fixed order
__global__ void __launch_bounds__(kRowsThreads) nl_rows_kernel(const NlArgs a) {
  if (!nl_dirty(a)) return;
  __shared__ float4 sp[kRowsThreads];
  __shared__ int sj[kRowsThreads];
  for (int c = blockIdx.x; c < a.n_cells; c += gridDim.x) {
    const int ci0 = a.cell_start[c], nci = a.cell_count[c];
    if (nci == 0) continue;  // block-uniform
    const int s = a.cell_sys[c];
    const SysInfo &S = a.sys[s];
    const NlGrid g = a.grid[s];
    const int lc = c - a.cell_base[s];
    const int cx = lc % g.nx, cy = (lc / g.nx) % g.ny, cz = lc / (g.nx * g.ny);
    const float reach2 = a.reach * a.reach;
    const int R = g.stencil;
    for (int i0 = 0; i0 < nci; i0 += kRowsThreads) {
      const int k = i0 + threadIdx.x;
      const bool has_i = k < nci;
      const int i = has_i ? a.cell_atoms[ci0 + k] : -1;
      const float4 p = has_i ? a.posq[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      int *row = has_i ? a.rows + (size_t)i * a.capacity : nullptr;
      int count = 0;
      for (int dz = -R; dz <= R; ++dz) {
        const int z = cz + dz;
        if (z < 0 || z >= g.nz) continue;
        for (int dy = -R; dy <= R; ++dy) {
          const int y = cy + dy;
          if (y < 0 || y >= g.ny) continue;
          for (int dx = -R; dx <= R; ++dx) {
            const int x = cx + dx;
            if (x < 0 || x >= g.nx) continue;
            const int nc = a.cell_base[s] + (z * g.ny + y) * g.nx + x;
            const int st = a.cell_start[nc], cnt = a.cell_count[nc];
            for (int b = 0; b < cnt; b += kRowsThreads) {
              __syncthreads();  // the previous chunk has been read
              const int m = min(kRowsThreads, cnt - b);
              if ((int)threadIdx.x < m) {
                const int j = a.cell_atoms[st + b + threadIdx.x];
                sj[threadIdx.x] = j;
                sp[threadIdx.x] = a.posq[j];
              }
              __syncthreads();
              if (has_i) {
                for (int t = 0; t < m; ++t) {
                  const float4 q = sp[t];
                  const float ex = p.x - q.x, ey = p.y - q.y, ez = p.z - q.z;
                  const int j = sj[t];
                  if (fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < reach2 && j != i) {
                    if (count < a.capacity) row[count] = j - S.off;
                    ++count;
                  }
                }
              }
            }
          }
        }
      }
      if (has_i) {
        for (int t = count; t < a.capacity; ++t) row[t] = S.n;  // sentinel
        a.counts[i] = count;
        if (count > a.capacity) {
          atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NLOVERFLOW);
        }
        atomicMax(&a.ctl[NL_MAXCOUNT], count);
      }
    }
  }
}

// 7. new displacement reference; the last block clears the rebuild flag
__global__ void nl_ref_kernel(const NlArgs a) {
  if (!nl_dirty(a)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_total; i += gridDim.x * blockDim.x) {
    a.xref[i] = a.x[i];
    a.xref[a.n_total + i] = a.y[i];
    a.xref[2 * (size_t)a.n_total + i] = a.z[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.ctl[NL_DONE], 1) == (int)gridDim.x - 1) {
      a.ctl[NL_DONE] = 0;
      a.ctl[NL_DIRTY] = 0;
      __threadfence();
    }
  }
}

static int grid_for(int n, int per) { return std::max(1, std::min((n + per - 1) / per, 65535)); }

cudaError_t nl_launch_build(const NlArgs &a, cudaStream_t st) {
  nl_grid_kernel<<<grid_for(a.n_sys, 8), 256, 0, st>>>(a);
  nl_assign_kernel<<<grid_for(a.n_total, 256), 256, 0, st>>>(a);
  nl_scan_kernel<<<std::min(a.n_sys, 65535), 1024, 0, st>>>(a);
  nl_scatter_kernel<<<grid_for(a.n_total, 256), 256, 0, st>>>(a);
  nl_sort_kernel<<<grid_for(a.n_cells, 1), 256, 0, st>>>(a);
  nl_rows_kernel<<<grid_for(a.n_cells, 1), kRowsThreads, 0, st>>>(a);
  nl_ref_kernel<<<grid_for(a.n_total, 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t nl_launch_disp(const NlArgs &a, cudaStream_t st) {
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
  a.sys = b->sys;
  a.atom_sys = b->atom_sys;
  a.bbox = b->bbox;
  a.grid = b->nl_grid;
  a.cell_base = b->nl_cell_base;
  a.cell_budget = b->nl_cell_budget;
  a.cell_sys = b->nl_cell_sys;
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
  a.sys_moved = b->nl_sys_moved;
  a.ctl = b->nl_ctl;
  a.capacity = b->nl_capacity;
  a.n_total = b->n_total;
  a.n_cells = b->nl_cells;
  a.n_sys = b->n_sys;
  a.status = b->status;
  a.reach = (float)nl_reach(b);
  return a;
}

// Device arrays of the list, allocated once: per-system cell budgets of
// max(64, 2 n) cells, the cell arrays over all budgets, the control words.
static int nl_alloc(pb2_batch *b) {
  pb2_ctx *ctx = b->ctx;
  if (b->nl_grid) return PB2_OK;
  std::vector<int32_t> base(b->n_sys), budget(b->n_sys), cell_sys;
  long long cells = 0;
  for (int s = 0; s < b->n_sys; ++s) {
    base[s] = (int32_t)cells;
    budget[s] = std::max(64, 2 * b->sys_host[s].n);
    cells += budget[s];
    if (cells > INT32_MAX / 2) return fail(ctx, PB2_EINVAL, "neighbour-list cell budget too large");
    cell_sys.insert(cell_sys.end(), budget[s], s);
  }
  Dev &D = b->nl;
  b->nl_cells = (int)cells;
  b->nl_grid = D.alloc<NlGrid>(b->n_sys);
  b->nl_cell_base = D.alloc<int32_t>(b->n_sys);
  b->nl_cell_budget = D.alloc<int32_t>(b->n_sys);
  b->nl_cell_sys = D.alloc<int32_t>(cells);
  b->nl_cell_count = D.alloc<int>(cells);
  b->nl_cell_start = D.alloc<int>(cells + 1);
  b->nl_cell_cursor = D.alloc<int>(cells);
  b->nl_atom_cell = D.alloc<int>(b->n_total);
  b->nl_cell_atoms = D.alloc<int>(b->n_total);
  b->nl_counts = D.alloc<int>(b->n_total);
  b->nl_xref = D.alloc<double>(3 * (size_t)b->n_total);
  b->nl_sys_moved = D.alloc<int32_t>(b->n_sys);
  b->nl_ctl = D.alloc<int32_t>(NL_WORDS);
  for (void *p : D.ptrs)
    if (!p) return fail(ctx, PB2_ENOMEM, "neighbour-list allocation failed");
  CUDA_TRY(ctx, cudaMemcpy(b->nl_cell_base, base.data(), base.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  CUDA_TRY(ctx, cudaMemcpy(b->nl_cell_budget, budget.data(), budget.size() * sizeof(int32_t),
                           cudaMemcpyHostToDevice));
  CUDA_TRY(ctx, cudaMemcpy(b->nl_cell_sys, cell_sys.data(), cell_sys.size() * sizeof(int32_t),
                           cudaMemcpyHostToDevice));
  CUDA_TRY(ctx, cudaMemset(b->nl_ctl, 0, NL_WORDS * sizeof(int32_t)));
  CUDA_TRY(ctx, cudaMemset(b->nl_sys_moved, 0, b->n_sys * sizeof(int32_t)));
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

// Current positions as the float32 pair-kernel layout and block boxes (the
// grid kernel reads the boxes).
static int nl_prepare(pb2_batch *b, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  CUDA_TRY(ctx, launch_posq(int_args_for_nl(b), st));
  CUDA_TRY(ctx, launch_bbox(b->sys, b->blk_sys, b->posq, b->bbox, b->n_blocks, st));
  return PB2_OK;
}

// Enqueue a build of every system (no host wait), timed with events.
static int nl_enqueue_build(pb2_batch *b, cudaStream_t st, bool force) {
  pb2_ctx *ctx = b->ctx;
  if (force) CUDA_TRY(ctx, cudaMemsetAsync(b->nl_ctl + NL_DIRTY, 1, 1, st));  // any nonzero byte
  CUDA_TRY(ctx, cudaMemsetAsync(b->nl_ctl + NL_MAXCOUNT, 0, sizeof(int32_t), st));
  CUDA_TRY(ctx, cudaEventRecord(b->nl_ev[0], st));
  CUDA_TRY(ctx, nl_launch_build(nl_args(b), st));
  CUDA_TRY(ctx, cudaEventRecord(b->nl_ev[1], st));
  b->nl_timed = true;
  return PB2_OK;
}

// Host visit: the largest row length of the last build; grow the rows (and
// rebuild) when they were too short, unless the capacity is fixed.
static int nl_settle(pb2_batch *b, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  int32_t ctl[NL_WORDS];
  CUDA_TRY(ctx, cudaMemcpyAsync(ctl, b->nl_ctl, sizeof ctl, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (ctl[NL_CELLFULL]) return fail(ctx, PB2_ENLOVERFLOW, "a neighbour-list cell holds more than 4096 atoms");
  const int maxc = ctl[NL_MAXCOUNT];
  if (maxc <= b->nl_capacity) return PB2_OK;
  const int fixed = b->params.nl_capacity;
  if (fixed > 0) {
    char buf[160];
    snprintf(buf, sizeof buf, "neighbour-list capacity %d exceeded (an atom has %d neighbours)", fixed, maxc);
    return fail(ctx, PB2_ENLOVERFLOW, buf);
  }
  int rc = nl_alloc_rows(b, ((maxc + maxc / 4 + 8 + 31) / 32) * 32);
  if (rc) return rc;
  // the overflow pass set the status bit; the rebuild supersedes it
  CUDA_TRY(ctx, cudaMemsetAsync(b->status, 0, b->n_sys * sizeof(uint32_t), st));
  if ((rc = nl_prepare(b, st)) || (rc = nl_enqueue_build(b, st, true))) return rc;
  CUDA_TRY(ctx, cudaMemcpyAsync(ctl, b->nl_ctl, sizeof ctl, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (ctl[NL_MAXCOUNT] > b->nl_capacity) return fail(ctx, PB2_ENLOVERFLOW, "neighbour-list capacity did not settle");
  return PB2_OK;
}

static int nl_build_all(pb2_batch *b, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  if (!(b->params.cutoff > 0.0 || b->params.gb_cutoff > 0.0))
    return fail(ctx, PB2_EINVAL, "a neighbour list needs cutoff > 0 (or gb_cutoff > 0)");
  int rc = nl_alloc(b);
  if (rc) return rc;
  if (!b->nl_rows && (rc = nl_alloc_rows(b, std::max(b->params.nl_capacity, 0)))) return rc;
  if ((rc = nl_prepare(b, st)) || (rc = nl_enqueue_build(b, st, true))) return rc;
  if ((rc = nl_settle(b, st))) return rc;
  b->nl_built = true;
  return PB2_OK;
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
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (rebuilt) *rebuilt = 0;
  if (!b->nl_built) {
    const int rc = nl_build_all(b, st);
    if (rc == PB2_OK && rebuilt) *rebuilt = b->n_sys;
    return rc;
  }
  int rc;
  CUDA_TRY(ctx, cudaMemsetAsync(b->nl_sys_moved, 0, b->n_sys * sizeof(int32_t), st));
  if ((rc = nl_prepare(b, st))) return rc;
  CUDA_TRY(ctx, nl_launch_disp(nl_args(b), st));
  if ((rc = nl_enqueue_build(b, st, false))) return rc;  // runs only if the check set the flag
  if (!rebuilt) return PB2_OK;                             // asynchronous: overflow seen at the next visit
  std::vector<int32_t> moved(b->n_sys);
  CUDA_TRY(ctx, cudaMemcpyAsync(moved.data(), b->nl_sys_moved, moved.size() * sizeof(int32_t),
                                cudaMemcpyDeviceToHost, st));
  if ((rc = nl_settle(b, st))) return rc;
  int n = 0;
  for (int v : moved) n += v != 0;
  *rebuilt = n;
  return PB2_OK;
}

extern "C" int pb2_nl_capacity(pb2_batch *b, int32_t *capacity) {
  if (!b || !capacity) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  *capacity = 0;
  if (!b->nl_built) return PB2_OK;
  // a host visit: a build an asynchronous check queued may have outgrown the
  // rows; grow them now, before the caller sizes its buffer
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  int rc = nl_settle(b, nullptr);
  if (rc) return rc;
  *capacity = b->nl_capacity;
  return PB2_OK;
}

extern "C" int pb2_nl_last_build_ms(pb2_batch *b, double *ms) {
  if (!b || !ms) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (!b->nl_timed) return fail(ctx, PB2_EINVAL, "no neighbour-list build yet");
  CUDA_TRY(ctx, cudaEventSynchronize(b->nl_ev[1]));
  float t = 0.f;
  CUDA_TRY(ctx, cudaEventElapsedTime(&t, b->nl_ev[0], b->nl_ev[1]));
  *ms = t;
  return PB2_OK;
}

extern "C" int pb2_nl_get(pb2_batch *b, int32_t *neighbors, void *stream) {
  if (!b || !neighbors) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (!b->nl_built) return fail(ctx, PB2_EINVAL, "no neighbour list built yet");
  cudaStream_t st = (cudaStream_t)stream;
  // the caller's buffer has the capacity pb2_nl_capacity reported; a build
  // queued since then that needs more rows is reported, not written
  int32_t maxc = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&maxc, b->nl_ctl + NL_MAXCOUNT, sizeof maxc, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (maxc > b->nl_capacity)
    return fail(ctx, PB2_ENLOVERFLOW, "the neighbour list outgrew its capacity: call pb2_nl_capacity "
                                      "(which grows it) and pass a buffer of that width");
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
