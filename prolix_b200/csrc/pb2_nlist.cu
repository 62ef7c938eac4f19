// Neighbour lists in jax_md's layout, built on the GPU.
//
// Reference: jax_md partition.neighbor_list as prolix uses it
// (physics/neighbor_list.py:155-172; batched_simulate.py:1429-1464), the
// host cell list of physics/cell_list.py:102-242, and the skin rule of
// batched_simulate.py:1600-1622 (rebuild when an atom moved more than
// skin/2 since the last build).  Output: per atom, the local indices of all
// atoms within cutoff + skin (both (i, j) and (j, i) present), padded with
// the sentinel n_atoms of its system; capacity K per atom.
//
// The spatial cells are the batch's own 32-atom blocks: each system's atoms
// are stored in a recursive-bisection order, so a block is a compact
// cluster, and its bounding box is already computed for the pair kernels.
// A cell grid is not built: the block boxes play its part, a box test
// standing in for the cell stencil.  One warp per four rows: the blocks of
// the system whose boxes come within cutoff + skin of one of its atoms are
// walked in index order, their atoms tested 32 at a time (lane =
// candidate).  Rows are therefore in stored-atom order, the same every
// build, whichever warp built them.
// A row longer than the capacity only counts (the largest count and an
// overflow bit are recorded for the host's next visit).
//
// Everything runs on the device as a fixed sequence of launches that needs
// no host decision:
//   0. (check) each atom's displacement since the last build against
//      skin/2 sets the rebuild flag and its system's moved flag;
//   1. the rows; 2. the positions become the new displacement reference,
//      and the last block clears the flag and the rows' unit counter.
// Each kernel returns at once while the flag is clear.  The HBM traffic is
// the row writes (4 B per slot).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pb2_common.cuh"
#include "pb2_internal.h"
#include "pb2_kernels.cuh"

namespace pb2 {

constexpr int kRowsWarps = 8;  // warps per thread block of the row pass (4 rows each)

__device__ __forceinline__ bool nl_dirty(const NlArgs &a) { return *(volatile int32_t *)&a.ctl[NL_DIRTY] != 0; }

__device__ __forceinline__ float nl_box_dist2(const float4 *bbox, int a, int b) {
  const float4 alo = bbox[2 * a], ahi = bbox[2 * a + 1];
  const float4 blo = bbox[2 * b], bhi = bbox[2 * b + 1];
  const float dx = fmaxf(0.f, fmaxf(alo.x - bhi.x, blo.x - ahi.x));
  const float dy = fmaxf(0.f, fmaxf(alo.y - bhi.y, blo.y - ahi.y));
  const float dz = fmaxf(0.f, fmaxf(alo.z - bhi.z, blo.z - ahi.z));
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

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

// 1. rows: a warp unit is four rows of a 32-atom block.  The warp tests the
// boxes of its system's blocks, 32 at a time (lane = block), against its
// four atoms, and walks the blocks within reach one at a time, lane =
// candidate atom: one position load serves the four rows, and each row's
// hits are compacted by a ballot and stored as one contiguous run
// (coalesced), so rows come out in j order.  The warps of one resident wave
// take units from a counter until none is left.
// A unit is 2 NH rows: four (NH = 2) in general, two (NH = 1) when a
// build has so few blocks that four-row units would leave most resident
// warps idle (each unit's blocks are walked in sequence, so more, shorter
// units finish sooner there).

// One j-block's 32 candidates (lane = candidate lj; nq = minus its
// position, duplicated) against the warp's rows l0 .. l0 + 2 NH - 1, whose
// positions are held in pairs (rows 0, 1 and 2, 3) so that the distances
// run as packed f32x2 arithmetic (per component the same roundings as the
// scalar fmaf chain).  Each row's hits are compacted by a ballot and stored
// as one contiguous run.  DIAG: the block holds the rows' own atoms.
template <int NH>
struct NlRows {
  float2 x[NH], y[NH], z[NH];
};

// row: the row's first slot; cap: its capacity.
__device__ __forceinline__ void nl_hit_row(bool hit, int lj, int *row, int cap, unsigned below, int &cnt) {
  const unsigned m = __ballot_sync(kFull, hit);
  const int t = cnt + __popc(m & below);
  if (hit && t < cap) row[t] = lj;
  cnt += __popc(m);
}

template <bool DIAG, int NH>
__device__ __forceinline__ void nl_rows_block(const NlRows<NH> &P, float4 q, int lj, int l0, float reach2,
                                              int *const *row, int cap, unsigned below, int *cnt) {
  const float2 nqx = make_float2(-q.x, -q.x), nqy = make_float2(-q.y, -q.y), nqz = make_float2(-q.z, -q.z);
#pragma unroll
  for (int h = 0; h < NH; ++h) {
    const float2 ex = __fadd2_rn(P.x[h], nqx), ey = __fadd2_rn(P.y[h], nqy), ez = __fadd2_rn(P.z[h], nqz);
    const float2 d2 = __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, __fmul2_rn(ez, ez)));
    const int r0 = 2 * h, r1 = 2 * h + 1;
    bool hit0 = d2.x < reach2, hit1 = d2.y < reach2;
    if (DIAG) {
      hit0 = hit0 && lj != l0 + r0;
      hit1 = hit1 && lj != l0 + r1;
    }
    nl_hit_row(hit0, lj, row[r0], cap, below, cnt[r0]);
    nl_hit_row(hit1, lj, row[r1], cap, below, cnt[r1]);
  }
}

// The rows of one warp unit: 2 NH rows of a 32-atom block against every
// block of its system, culled by box (lane = block, 32 at a time), then the
// near blocks' atoms, lane = candidate.
template <int NH>
__device__ __forceinline__ void nl_rows_unit(const NlArgs &a, int ib, int w, int lane, unsigned below, int cap,
                                             float reach2) {
  constexpr int kRowsPerWarp = 2 * NH;
  const int s = a.blk_sys[ib];
  // the system's fields in registers: the row stores could alias them
  const int off = a.sys[s].off, n = a.sys[s].n, nblk = a.sys[s].nblk, blk_base = a.sys[s].blk_base;
  const int l0 = (ib - blk_base) * 32 + w * kRowsPerWarp;  // the unit's first row, local index
  if (l0 >= n) return;  // past the system's last atom: no rows
  int cnt[kRowsPerWarp];
  int *row[kRowsPerWarp];  // each row's first slot
  NlRows<NH> P;
#pragma unroll
  for (int h = 0; h < NH; ++h) {
    float4 u = a.posq[off + min(l0 + 2 * h, n - 1)], v = a.posq[off + min(l0 + 2 * h + 1, n - 1)];
    if (l0 + 2 * h >= n) u.x = -1e30f;  // no row: never within reach of an atom
    if (l0 + 2 * h + 1 >= n) v.x = -1e30f;
    P.x[h] = make_float2(u.x, v.x);
    P.y[h] = make_float2(u.y, v.y);
    P.z[h] = make_float2(u.z, v.z);
    cnt[2 * h] = cnt[2 * h + 1] = 0;
  }
#pragma unroll
  for (int r = 0; r < kRowsPerWarp; ++r) row[r] = a.rows + (size_t)(off + min(l0 + r, n - 1)) * cap;
  const int own = ib - blk_base;
  for (int c0 = 0; c0 < nblk; c0 += 32) {
    // the blocks within reach of one of the unit's atoms (the margin keeps
    // the test conservative under rounding).  A block whose every atom is
    // within reach of all the unit's rows (its box's farthest corner is,
    // by the same rounded operations as the atom test, so each atom's
    // computed distance is no larger) is stored without its distances: the
    // same slots in the same order.
    bool near = false, inside = false;
    if (c0 + lane < nblk) {
      const int jb = c0 + lane;
      const float4 lo = a.bbox[2 * (blk_base + jb)], hi = a.bbox[2 * (blk_base + jb) + 1];
      inside = jb != own && jb * 32 + 32 <= n;
#pragma unroll
      for (int r = 0; r < kRowsPerWarp; ++r) {
        const float px = r & 1 ? P.x[r >> 1].y : P.x[r >> 1].x;
        const float py = r & 1 ? P.y[r >> 1].y : P.y[r >> 1].x;
        const float pz = r & 1 ? P.z[r >> 1].y : P.z[r >> 1].x;
        const float dx = fmaxf(0.f, fmaxf(lo.x - px, px - hi.x));
        const float dy = fmaxf(0.f, fmaxf(lo.y - py, py - hi.y));
        const float dz = fmaxf(0.f, fmaxf(lo.z - pz, pz - hi.z));
        near |= fmaf(dx, dx, fmaf(dy, dy, dz * dz)) < reach2 * 1.0001f;
        const float fx = fmaxf(fabsf(px - lo.x), fabsf(hi.x - px));
        const float fy = fmaxf(fabsf(py - lo.y), fabsf(hi.y - py));
        const float fz = fmaxf(fabsf(pz - lo.z), fabsf(hi.z - pz));
        inside = inside && fmaf(fx, fx, fmaf(fy, fy, fz * fz)) < reach2;
      }
    }
    const unsigned in_m = __ballot_sync(kFull, inside);
    for (unsigned blocks = __ballot_sync(kFull, near); blocks != 0u; blocks &= blocks - 1u) {
      const int k = __ffs(blocks) - 1;
      const int jb = c0 + k;
      const int lj = jb * 32 + lane;
      if ((in_m >> k) & 1u) {
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r) {
          const int t = cnt[r] + lane;
          if (t < cap) row[r][t] = lj;
          cnt[r] += 32;
        }
        continue;
      }
      float4 q = a.posq[off + min(lj, n - 1)];
      if (lj >= n) q.x = 1e30f;  // no atom: never within reach of a row
      if (jb == own) nl_rows_block<true, NH>(P, q, lj, l0, reach2, row, cap, below, cnt);  // skips i = j
      else nl_rows_block<false, NH>(P, q, lj, l0, reach2, row, cap, below, cnt);
    }
  }
#pragma unroll
  for (int r = 0; r < kRowsPerWarp; ++r) {
    const int li = l0 + r;
    if (li >= n) break;
    const int i = off + li;
    // sentinels; with rows of a multiple of 4 slots (each row 16-byte
    // aligned) as 16-byte stores after at most 3 single slots
    int *rp = row[r];
    if ((cap & 3) == 0 && (reinterpret_cast<uintptr_t>(a.rows) & 15) == 0) {
      const int ta = min(cap, (cnt[r] + 3) & ~3);
      if (cnt[r] + lane < ta) rp[cnt[r] + lane] = n;
      const int4 s4 = make_int4(n, n, n, n);
      for (int t = ta + 4 * lane; t < cap; t += 128) *reinterpret_cast<int4 *>(rp + t) = s4;
    } else {
      for (int t = cnt[r] + lane; t < cap; t += 32) rp[t] = n;
    }
    if (lane == 0) {
      a.counts[i] = cnt[r];
      if (cnt[r] > cap) atomicOr(&a.status[s], (uint32_t)PB2_STATUS_NLOVERFLOW);
      atomicMax(&a.ctl[NL_MAXCOUNT], cnt[r]);
    }
  }
}

// Each warp takes units (2 NH rows of a 32-atom block) from a counter in
// ctl[NL_NEXT] until none is left, so that the blocks' uneven costs (a
// globule's core against its surface) spread over every SM; the reference
// kernel resets the counter after the build.
template <int NH>
__global__ void __launch_bounds__(32 * kRowsWarps) nl_rows_kernel(const NlArgs a) {
  constexpr int kRowsPerWarp = 2 * NH;
  if (!nl_dirty(a)) return;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int cap = a.capacity;
  const float reach2 = a.reach2;
  const int n_units = a.n_blocks * (32 / kRowsPerWarp);
  for (;;) {
    int u = 0;
    if (lane == 0) u = atomicAdd(&a.ctl[NL_NEXT], 1);
    u = __shfl_sync(kFull, u, 0);
    if (u >= n_units) break;
    nl_rows_unit<NH>(a, u / (32 / kRowsPerWarp), u % (32 / kRowsPerWarp), lane, below, cap, reach2);
  }
}

// 2. new displacement reference; the last block clears the rebuild flag
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
      a.ctl[NL_NEXT] = 0;
      a.ctl[NL_DIRTY] = 0;
      __threadfence();
    }
  }
}

static int grid_for(int n, int per) { return std::max(1, std::min((n + per - 1) / per, 65535)); }

// Resident thread blocks of the rows kernel (2 NH rows per unit) on the
// current device: one wave, whose warps take their units from the counter.
// The first query for a device comes from the list's allocation, outside
// any stream capture.
template <int NH>
static int nl_rows_resident() {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  int g = cached[dev].load(std::memory_order_relaxed);
  if (g == 0) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, nl_rows_kernel<NH>, 32 * kRowsWarps, 0);
    g = std::max(1, sms * std::max(per, 1));
    cached[dev].store(g, std::memory_order_relaxed);
  }
  return g;
}

static void nl_rows_warm() {
  nl_rows_resident<1>();
  nl_rows_resident<2>();
}

cudaError_t nl_launch_build(const NlArgs &a, cudaStream_t st) {
  // two-row units when even they fit in one wave of resident warps
  const long long units2 = 16LL * a.n_blocks;
  if (units2 <= (long long)nl_rows_resident<1>() * kRowsWarps) {
    const int grid = (int)std::max(1LL, std::min((units2 + kRowsWarps - 1) / kRowsWarps,
                                                  (long long)nl_rows_resident<1>()));
    nl_rows_kernel<1><<<grid, 32 * kRowsWarps, 0, st>>>(a);
  } else {
    nl_rows_kernel<2><<<std::max(1, std::min(a.n_blocks, nl_rows_resident<2>())), 32 * kRowsWarps, 0, st>>>(a);
  }
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
  a.blk_sys = b->blk_sys;
  a.bbox = b->bbox;
  a.posq = b->posq;
  a.x = b->x; a.y = b->y; a.z = b->z;
  a.xref = b->nl_xref;
  a.rows = b->nl_rows;
  a.counts = b->nl_counts;
  a.sys_moved = b->nl_sys_moved;
  a.ctl = b->nl_ctl;
  a.capacity = b->nl_capacity;
  a.n_total = b->n_total;
  a.n_blocks = b->n_blocks;
  a.n_sys = b->n_sys;
  a.status = b->status;
  const float reach = (float)nl_reach(b);
  a.reach2 = reach * reach;
  return a;
}

// Device arrays of the list, allocated once: counts, reference positions,
// moved flags, control words (the rows follow the capacity).
static int nl_alloc(pb2_batch *b) {
  pb2_ctx *ctx = b->ctx;
  if (b->nl_ctl) return PB2_OK;
  Dev &D = b->nl;
  b->nl_counts = D.alloc<int>(b->n_total);
  b->nl_xref = D.alloc<double>(3 * (size_t)b->n_total);
  b->nl_sys_moved = D.alloc<int32_t>(b->n_sys);
  b->nl_ctl = D.alloc<int32_t>(NL_WORDS);
  for (void *p : D.ptrs)
    if (!p) return fail(ctx, PB2_ENOMEM, "neighbour-list allocation failed");
  CUDA_TRY(ctx, cudaMemset(b->nl_ctl, 0, NL_WORDS * sizeof(int32_t)));
  CUDA_TRY(ctx, cudaMemset(b->nl_sys_moved, 0, b->n_sys * sizeof(int32_t)));
  nl_rows_warm();  // the device's occupancy, queried outside any capture
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
