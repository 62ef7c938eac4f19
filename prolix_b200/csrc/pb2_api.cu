// C ABI of prolix_b200: context and batch management, force evaluation,
// Langevin runs (captured as CUDA graphs), state access.
//
// Data layout in HBM (batch order = systems concatenated, atoms in input
// order within a system):
//   FP64 SoA state x, y, z, px, py, pz; int64 fixed-point forces fx, fy, fz;
//   float4 posq (x, y, z relative to the system origin, charge) and
//   float4 par (sigma/2, sqrt(eps), rho~, scaled radius) for the pair
//   kernels; float4 born (B, 1/B, dB/dI); int64 descreening and dE/dB sums;
//   per-system SysInfo records, keys (two buffers), step counters, status.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "pb2_common.cuh"
#include "pb2_kernels.cuh"
#include "pb2_obc_series.cuh"


#include "pb2_internal.h"

using namespace pb2;

int pb2::set_error(pb2_ctx *ctx, int code, const char *msg) { return fail(ctx, code, msg); }

extern "C" int pb2_abi_version(void) { return PB2_ABI_VERSION; }

extern "C" int pb2_ctx_create(int device, pb2_ctx **out) {
  if (!out) return PB2_EINVAL;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) return PB2_ENODEV;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PB2_ENODEV;
  if (prop.major != 10) return PB2_ENODEV;  // built for sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return PB2_ENODEV;
  auto *c = new (std::nothrow) pb2_ctx;
  if (!c) return PB2_ENOMEM;
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  // keep memory freed by dropped batches in this process's pool (the
  // attribute belongs to this process's context and ends with it)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  *out = c;
  return PB2_OK;
}

extern "C" int pb2_ctx_destroy(pb2_ctx *ctx) {
  delete ctx;
  return PB2_OK;
}

extern "C" const char *pb2_last_error(const pb2_ctx *ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

// ------------------------------------------------------------ batch build

static PairArgs pair_args(pb2_batch *b) {
  PairArgs a;
  a.sys = b->sys;
  a.items = b->items2;
  a.n_items = b->n_items2;
  a.item_count = b->item_count;
  a.terms = b->params.terms;
  a.excl_ent = b->excl_ent;
  a.excl_rows = b->excl_rows;
  a.posq = b->posq;
  a.par = b->par;
  a.born = b->born;
  a.bbox = b->bbox;
  a.cut = b->cut ? 1 : 0;
  a.sched = b->sched;
  a.born_acc = b->born_acc;
  a.dedb_acc = b->dedb_acc;
  a.fx = b->fx;
  a.fy = b->fy;
  a.fz = b->fz;
  a.energy = b->energy;
  a.pl_ctl = b->pl_on ? b->pl_ctl : nullptr;
  a.pl_items0 = b->pl_items[0];
  a.pl_items1 = b->pl_items[1];
  a.pl_jlist = b->pl_jlist;
  a.bonded = b->bonded;
  a.n_bonded_chunks = 0;
  a.sys_items = nullptr;
  a.sys_done = b->sys_done;
  a.fin = FinalizeArgs{};
  a.pl_sys_items0 = b->pl_sys_items[0];
  a.pl_sys_items1 = b->pl_sys_items[1];
  return a;
}

static PlArgs pl_args(pb2_batch *b) {
  PlArgs a;
  a.sys = b->sys;
  a.rows = b->pl_rows;
  a.n_rows = b->n_pl_rows;
  a.bbox = b->bbox;
  a.posq = b->posq;
  a.ref = b->pl_ref;
  a.jlist = b->pl_jlist;
  a.items0 = b->pl_items[0];
  a.items1 = b->pl_items[1];
  a.sys_items0 = b->pl_sys_items[0];
  a.sys_items1 = b->pl_sys_items[1];
  a.n_sys = b->n_sys;
  a.ctl = b->pl_ctl;
  a.reach2 = b->pl_reach2;
  a.seg = b->params.tile_segment;
  a.retired = b->retired;
  return a;
}

IntArgs int_args_for_nl(pb2_batch *b);

static IntArgs int_args(pb2_batch *b, int parity, int finish_prev) {
  IntArgs a;
  a.sys = b->sys;
  a.atom_sys = b->atom_sys;
  a.user = b->user;
  a.x = b->x; a.y = b->y; a.z = b->z;
  a.px = b->px; a.py = b->py; a.pz = b->pz;
  a.fx = b->fx; a.fy = b->fy; a.fz = b->fz;
  a.mass = b->mass;
  a.sigma = b->sigma;
  a.charge = b->charge;
  a.posq = b->posq;
  a.keys = b->keys;
  a.splits = b->key_splits;
  a.steps = b->steps;
  a.status = b->status;
  a.n_total = b->n_total;
  a.n_sys = b->n_sys;
  a.parity = parity;
  a.finish_prev = finish_prev;
  a.partitionable = b->params.partitionable_keys;
  a.vlimit = b->guard[0];
  a.max_dx = b->guard[1];
  a.force_cap = b->guard[2];
  a.guard_end = b->guard_end;
  a.warn_flags = b->warn_flags;
  a.warn_counts = b->warn_counts;
  a.blk_sys = b->blk_sys;
  a.bbox = b->bbox;
  a.n_blocks = b->n_blocks;
  a.pl_ref = b->pl_on ? b->pl_ref : nullptr;
  a.pl_ctl = b->pl_on ? b->pl_ctl : nullptr;
  a.retired = b->retired;
  a.blk_info = b->blk_info;
  return a;
}

// The force accumulators no longer hold a step's closing force (the state
// was set or moved outside a Langevin step): the next step applies them as
// they are, without the force cap.
static int forces_not_from_step(pb2_batch *b, cudaStream_t st) {
  CUDA_TRY(b->ctx, cudaMemsetAsync(b->guard_end, 0, sizeof(int32_t), st));
  return PB2_OK;
}

IntArgs int_args_for_nl(pb2_batch *b) { return int_args(b, b->key_parity, 0); }

// Tile work items: for each system and i-block, its tiles (iblk, jb >= iblk)
// cut into segments of `seg` tiles; sorted by tile count, largest first
// (the kernels hand them out dynamically).
// Spatial order of one system's atoms: recursive bisection of the input
// positions along the longest side of their bounding box, cut at a multiple
// of 32 atoms near the middle, so that every 32-atom block is a compact
// cluster (smaller block boxes: more tile pairs in the far field and beyond
// cutoffs).  Ties go by input index, so the order depends on the positions
// alone.  ord[l] = input index of the atom stored at l.  Non-finite
// positions keep the input order.
static void spatial_order(const double *pos, int n, std::vector<int> &ord) {
  ord.resize(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int i = 0; i < 3 * n; ++i)
    if (!std::isfinite(pos[i])) return;
  struct At {
    double c[3];
    int i;
  };
  std::vector<At> at(n);  // positions travel with their indices (contiguous)
  for (int i = 0; i < n; ++i) at[i] = At{{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]}, i};
  std::vector<std::pair<int, int>> todo{{0, n}};
  while (!todo.empty()) {
    const auto [a, e] = todo.back();
    todo.pop_back();
    if (e - a <= 32) continue;
    double lo[3] = {at[a].c[0], at[a].c[1], at[a].c[2]};
    double hi[3] = {lo[0], lo[1], lo[2]};
    for (int k = a; k < e; ++k)
      for (int c = 0; c < 3; ++c) {
        lo[c] = std::min(lo[c], at[k].c[c]);
        hi[c] = std::max(hi[c], at[k].c[c]);
      }
    int ax = 0;
    for (int c = 1; c < 3; ++c)
      if (hi[c] - lo[c] > hi[ax] - lo[ax]) ax = c;
    const int half = (e - a) / 2;
    const int m = a + std::max(32, std::min((half + 16) / 32 * 32, (e - a - 1) / 32 * 32));
    // partition only: the atoms below the cut come first (a strict total
    // order, so the result is the same on every run)
    std::nth_element(at.begin() + a, at.begin() + m, at.begin() + e, [ax](const At &p, const At &q) {
      return p.c[ax] < q.c[ax] || (p.c[ax] == q.c[ax] && p.i < q.i);
    });
    todo.push_back({a, m});
    todo.push_back({m, e});
  }
  for (int l = 0; l < n; ++l) ord[l] = at[l].i;
  // within each block, input order
  for (int a = 0; a < n; a += 32) std::sort(ord.begin() + a, ord.begin() + std::min(n, a + 32));
}

static std::vector<TileItem> build_items(const std::vector<SysInfo> &sinfo, int seg) {
  std::vector<TileItem> items;
  for (int s = 0; s < (int)sinfo.size(); ++s) {
    const int nblk = sinfo[s].nblk;
    for (int ib = 0; ib < nblk; ++ib)
      for (int j0 = ib; j0 < nblk; j0 += seg) items.push_back(TileItem{s, ib, j0, std::min(j0 + seg, nblk)});
  }
  std::stable_sort(items.begin(), items.end(), [](const TileItem &p, const TileItem &q) {
    return (p.jb1 - p.jb0) > (q.jb1 - q.jb0);
  });
  return items;
}

// Work items of the two-i-block force kernel: even i-blocks ib (with ib + 1)
// against j-blocks [j0, j1), j0 >= ib.
static std::vector<TileItem> build_items2(const std::vector<SysInfo> &sinfo, int seg) {
  std::vector<TileItem> items;
  for (int s = 0; s < (int)sinfo.size(); ++s) {
    const int nblk = sinfo[s].nblk;
    for (int ib = 0; ib < nblk; ib += 2)
      for (int j0 = ib; j0 < nblk; j0 += seg) items.push_back(TileItem{s, ib, j0, std::min(j0 + seg, nblk)});
  }
  std::stable_sort(items.begin(), items.end(), [](const TileItem &p, const TileItem &q) {
    return (p.jb1 - p.jb0) > (q.jb1 - q.jb0);
  });
  return items;
}

// Work items of the four-block force kernel: i-blocks ib, ib % 4 == 0 (with
// ib + 1 .. ib + 3), against j-blocks [j0, j1), j0 >= ib; sorted by cost.
static std::vector<TileItem> build_items4(const std::vector<SysInfo> &sinfo, int seg) {
  std::vector<TileItem> items;
  for (int s = 0; s < (int)sinfo.size(); ++s) {
    const int nblk = sinfo[s].nblk;
    for (int ib = 0; ib < nblk; ib += 4)
      for (int j0 = ib; j0 < nblk; j0 += seg) items.push_back(TileItem{s, ib, j0, std::min(j0 + seg, nblk)});
  }
  std::stable_sort(items.begin(), items.end(), [](const TileItem &p, const TileItem &q) {
    return (p.jb1 - p.jb0) > (q.jb1 - q.jb0);
  });
  return items;
}

static void set_force4_grid(pb2_batch *b) {
  const int cap = force4_occupancy(b->cut, b->shape4) * b->ctx->sm_count;
  int t = 0, m = 0;
  force4_shape(b->shape4, &t, &m);
  const int w = t / 32;
  b->grid4 = std::max(1, std::min(cap, (b->n_items4 + w - 1) / w));
}

// Grid of pair pass p for its block shape: one resident wave (warps take
// items dynamically), no more warps than items.
static void set_pair_grid(pb2_batch *b, int p) {
  const int cap = tile_kernel_occupancy(p, b->cut, b->shape[p]) * b->ctx->sm_count;
  const int w = tile_kernel_warps(p, b->shape[p]);
  b->grid_pair[p] = std::max(1, std::min(cap, (b->n_items2 + w - 1) / w));
}

// (Re)build the pair kernels' two-i-block work list and their grids (one
// resident wave each; warps take items dynamically).  The kernels read the
// live list: the full one without the items of retired systems.
static int setup_items2(pb2_batch *b, int seg) {
  pb2_ctx *ctx = b->ctx;
  std::vector<TileItem> items = build_items2(b->sys_host, seg);
  b->dev.release(b->items2);
  b->dev.release(b->items2_all);
  b->items2 = b->dev.alloc<TileItem>(std::max<size_t>(items.size(), 1));
  b->items2_all = b->dev.alloc<TileItem>(std::max<size_t>(items.size(), 1));
  if (!b->items2 || !b->items2_all) return fail(ctx, PB2_ENOMEM, "work-item allocation failed");
  if (!items.empty())
    CUDA_TRY(ctx, cudaMemcpy(b->items2_all, items.data(), items.size() * sizeof(TileItem), cudaMemcpyHostToDevice));
  b->n_items2 = (int)items.size();
  if (!b->retired) {
    b->retired = b->dev.alloc<int8_t>(b->n_sys);
    b->item_count = b->dev.alloc<int32_t>(1);
    if (!b->retired || !b->item_count) return fail(ctx, PB2_ENOMEM, "work-item allocation failed");
    CUDA_TRY(ctx, cudaMemset(b->retired, 0, b->n_sys));
    b->retired_host.assign(b->n_sys, 0);
  }
  CUDA_TRY(ctx, launch_retire(-1, b->retired, b->items2_all, b->n_items2, b->items2, b->item_count, nullptr, nullptr));
  {
    std::vector<TileItem> items4 = build_items4(b->sys_host, seg);
    b->dev.release(b->items4);
    b->dev.release(b->items4_all);
    b->items4 = b->dev.alloc<TileItem>(std::max<size_t>(items4.size(), 1));
    b->items4_all = b->dev.alloc<TileItem>(std::max<size_t>(items4.size(), 1));
    if (!b->item_count4) b->item_count4 = b->dev.alloc<int32_t>(1);
    if (!b->items4 || !b->items4_all || !b->item_count4) return fail(ctx, PB2_ENOMEM, "work-item allocation failed");
    if (!items4.empty())
      CUDA_TRY(ctx, cudaMemcpy(b->items4_all, items4.data(), items4.size() * sizeof(TileItem), cudaMemcpyHostToDevice));
    b->n_items4 = (int)items4.size();
    CUDA_TRY(ctx, launch_retire(-1, b->retired, b->items4_all, b->n_items4, b->items4, b->item_count4, nullptr, nullptr));
  }
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  std::vector<int32_t> per_sys(b->n_sys, 0);
  for (const TileItem &t : items) ++per_sys[t.sys];
  if (!b->sys_items) {
    b->sys_items = b->dev.alloc<int32_t>(b->n_sys);
    b->sys_done = b->dev.alloc<int32_t>(b->n_sys);
    b->sys_fin = b->dev.alloc<int32_t>(b->n_sys);
    if (!b->sys_items || !b->sys_done || !b->sys_fin) return fail(ctx, PB2_ENOMEM, "work-item allocation failed");
    CUDA_TRY(ctx, cudaMemset(b->sys_done, 0, b->n_sys * sizeof(int32_t)));
    CUDA_TRY(ctx, cudaMemset(b->sys_fin, 0, b->n_sys * sizeof(int32_t)));
  }
  CUDA_TRY(ctx, cudaMemcpy(b->sys_items, per_sys.data(), per_sys.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  b->sys_items_host = per_sys;
  for (int p = 0; p < 3; ++p) set_pair_grid(b, p);
  set_force4_grid(b);
  return PB2_OK;
}

// The pair list of a cutoff run (pb2_pairlist.cu): rows (one per pair of
// i-blocks), room for every j-block of each row, two item buffers sized for
// the segment, and the control words, with the rebuild flag set so that the
// first force evaluation builds it.
static int setup_pair_list(pb2_batch *b, int seg) {
  pb2_ctx *ctx = b->ctx;
  if (!b->pl_on) return PB2_OK;
  std::vector<PlRow> rows;
  size_t jcap = 0, icap = 0;
  for (int s = 0; s < b->n_sys; ++s) {
    const int nblk = b->sys_host[s].nblk;
    for (int ib = 0; ib < nblk; ib += 2) {
      rows.push_back(PlRow{s, ib, (int32_t)jcap, 0});
      jcap += (size_t)(nblk - ib);
      icap += (size_t)((nblk - ib + seg - 1) / seg);
    }
  }
  if (jcap > (size_t)INT32_MAX) return fail(ctx, PB2_EINVAL, "pair list too large");
  Dev &D = b->dev;
  if (!b->pl_rows) {
    b->pl_rows = D.alloc<PlRow>(rows.size());
    b->pl_jlist = D.alloc<int32_t>(std::max<size_t>(jcap, 1));
    b->pl_ctl = D.alloc<int32_t>(PL_WORDS);
    b->pl_ref = D.alloc<float4>(b->n_total);
    b->pl_sys_items[0] = D.alloc<int32_t>(b->n_sys);
    b->pl_sys_items[1] = D.alloc<int32_t>(b->n_sys);
    if (!b->pl_rows || !b->pl_jlist || !b->pl_ctl || !b->pl_ref || !b->pl_sys_items[0] ||
        !b->pl_sys_items[1])
      return fail(ctx, PB2_ENOMEM, "pair-list allocation failed");
    CUDA_TRY(ctx, cudaMemcpy(b->pl_rows, rows.data(), rows.size() * sizeof(PlRow), cudaMemcpyHostToDevice));
    b->n_pl_rows = (int)rows.size();
  }
  if (icap > b->pl_item_cap) {
    for (auto &p : b->pl_items) {
      D.release(p);
      p = D.alloc<TileItem>(icap);
      if (!p) return fail(ctx, PB2_ENOMEM, "pair-list item allocation failed");
    }
    b->pl_item_cap = icap;
  }
  const int32_t ctl[PL_WORDS] = {1, 0, 0, 0, 0, 0, 0, 0};  // dirty: rebuild at the next evaluation
  CUDA_TRY(ctx, cudaMemcpy(b->pl_ctl, ctl, sizeof ctl, cudaMemcpyHostToDevice));
  for (auto p : b->pl_sys_items) CUDA_TRY(ctx, cudaMemset(p, 0, b->n_sys * sizeof(int32_t)));
  b->grid_pl = std::max(1, std::min(8 * ctx->sm_count, (b->n_pl_rows + 7) / 8));
  return PB2_OK;
}

static int validate(pb2_ctx *ctx, const pb2_system_desc &d, int s) {
  char buf[256];
  auto bad = [&](const char *what) {
    snprintf(buf, sizeof buf, "system %d: %s", s, what);
    return fail(ctx, PB2_EINVAL, buf);
  };
  if (d.n_atoms <= 0) return bad("n_atoms must be > 0");
  if (!d.positions || !d.charges || !d.sigmas || !d.epsilons || !d.radii || !d.scaled_radii ||
      !d.masses)
    return bad("per-atom arrays must not be NULL");
  const int n = d.n_atoms;
  for (int i = 0; i < n; ++i) {
    if (!(d.masses[i] > 0.0)) return bad("masses must be > 0");
    if (!(d.radii[i] > 0.0)) return bad("radii must be > 0");
  }
  auto check_idx = [&](const int32_t *idx, int64_t count, const char *what) -> bool {
    for (int64_t k = 0; k < count; ++k)
      if (idx[k] < 0 || idx[k] >= n) {
        snprintf(buf, sizeof buf, "system %d: %s index %d out of range", s, what, idx[k]);
        return false;
      }
    return true;
  };
  if (d.n_bonds < 0 || d.n_angles < 0 || d.n_torsions < 0 || d.n_cmap < 0 || d.n_excl < 0 ||
      d.n_exceptions < 0 || d.n_impropers < 0 || d.n_urey_bradley < 0)
    return bad("negative term count");
  if (d.n_impropers && (!d.impropers || !d.improper_params || d.n_improper_terms <= 0 ||
                        (d.improper_form != 0 && d.improper_form != 1)))
    return bad("improper arrays missing or improper_form not 0 (periodic) / 1 (harmonic)");
  if (d.n_urey_bradley && (!d.urey_bradley_bonds || !d.urey_bradley_params))
    return bad("Urey-Bradley arrays missing");
  if (d.n_bonds && (!d.bonds || !d.bond_params)) return bad("bond arrays missing");
  if (d.n_angles && (!d.angles || !d.angle_params)) return bad("angle arrays missing");
  if (d.n_torsions && (!d.torsions || !d.torsion_params || d.n_torsion_terms <= 0))
    return bad("torsion arrays missing");
  if (d.n_cmap && (!d.cmap_rows || !d.cmap_map || !d.cmap_coeffs || d.n_cmap_maps <= 0 ||
                   d.cmap_grid <= 0))
    return bad("cmap arrays missing");
  if (d.n_excl && (!d.excl_pairs || !d.excl_kind)) return bad("exclusion arrays missing");
  if (d.n_exceptions && (!d.exception_pairs || !d.exception_params)) return bad("exception arrays missing");
  if (!check_idx(d.bonds, 2LL * d.n_bonds, "bond") ||
      !check_idx(d.angles, 3LL * d.n_angles, "angle") ||
      !check_idx(d.torsions, 4LL * d.n_torsions, "torsion") ||
      !check_idx(d.cmap_rows, 5LL * d.n_cmap, "cmap") ||
      !check_idx(d.excl_pairs, 2LL * d.n_excl, "exclusion") ||
      !check_idx(d.exception_pairs, 2LL * d.n_exceptions, "exception") ||
      !check_idx(d.impropers, 4LL * d.n_impropers, "improper") ||
      !check_idx(d.urey_bradley_bonds, 2LL * d.n_urey_bradley, "Urey-Bradley"))
    return fail(ctx, PB2_EINVAL, buf);
  for (int k = 0; k < d.n_cmap; ++k)
    if (d.cmap_map[k] < 0 || d.cmap_map[k] >= d.n_cmap_maps) return bad("cmap map index out of range");
  for (int k = 0; k < d.n_excl; ++k) {
    if (d.excl_pairs[2 * k] >= d.excl_pairs[2 * k + 1]) return bad("exclusion pairs need i < j");
    if (d.excl_kind[k] != 0 && d.excl_kind[k] != 1) return bad("exclusion kind must be 0 or 1");
  }
  if (!(d.dt > 0.0) || !(d.kT >= 0.0) || !(d.gamma >= 0.0)) return bad("dt > 0, kT >= 0, gamma >= 0");
  if (!(d.eps_in > 0.0) || !(d.eps_out > 0.0)) return bad("dielectrics must be > 0");
  return PB2_OK;
}

template <class T>
static int upload(pb2_ctx *ctx, T *dst, const std::vector<T> &src) {
  if (src.empty()) return PB2_OK;
  CUDA_TRY(ctx, cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return PB2_OK;
}

extern "C" int pb2_batch_create(pb2_ctx *ctx, int32_t n_systems, const pb2_system_desc *systems,
                                const pb2_run_params *params, pb2_batch **out) {
  if (!ctx || !out || !systems || !params || n_systems <= 0) return fail(ctx, PB2_EINVAL, "bad arguments");
  *out = nullptr;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  for (int s = 0; s < n_systems; ++s) {
    int rc = validate(ctx, systems[s], s);
    if (rc) return rc;
  }
  std::unique_ptr<pb2_batch> b(new (std::nothrow) pb2_batch);
  if (!b) return fail(ctx, PB2_ENOMEM, "host allocation");
  b->ctx = ctx;
  b->params = *params;
  if (b->params.tile_segment <= 0) {
    // default work-item length: the longest (8, 4, 2 or 1 j-blocks) that
    // still gives every resident warp of the force pass a few items, so a
    // small batch spreads over the whole GPU
    const long long want = 4LL * ctx->sm_count * 16;
    int seg = 1;
    for (int cand : {8, 4, 2}) {
      long long items = 0;
      for (int s = 0; s < n_systems; ++s) {
        const int nb = (systems[s].n_atoms + 31) / 32;
        for (int ib = 0; ib < nb; ib += 2) items += (nb - ib + cand - 1) / cand;
      }
      if (items >= want) {
        seg = cand;
        break;
      }
    }
    b->params.tile_segment = seg;
  }
  if (b->params.graph_chunk <= 0) b->params.graph_chunk = 50;
  b->n_sys = n_systems;
  const bool cutoff_mode = params->cutoff > 0.0;
  const double gb_cut = params->gb_cutoff < 0.0 ? (cutoff_mode ? params->cutoff : 0.0) : params->gb_cutoff;
  const bool gb_cut_mode = gb_cut > 0.0;
  const double born_cut = params->born_cutoff > 0.0 ? params->born_cutoff : gb_cut;
  const bool born_mode = born_cut > 0.0;  // Born radii from a cutoff: its clamps apply

  // --- stored atom order of each system (spatial unless asked to keep the
  // input order), computed for all systems at once on the host's cores
  std::vector<std::vector<int>> orders(n_systems);
  {
    auto work = [&](int s) {
      std::vector<int> &ord = orders[s];
      const int n = systems[s].n_atoms;
      if (params->keep_atom_order) {
        ord.resize(n);
        for (int i = 0; i < n; ++i) ord[i] = i;
      } else {
        spatial_order(systems[s].positions, n, ord);
      }
    };
    const int n_threads =
        std::max(1, std::min<int>(n_systems, std::min(16u, std::max(1u, std::thread::hardware_concurrency()))));
    std::atomic<int> next{0};
    auto worker = [&]() {
      for (int s; (s = next.fetch_add(1)) < n_systems;) work(s);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < n_threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
  }

  // --- per-atom host arrays
  int64_t total = 0;
  int blocks_total = 0;
  for (int s = 0; s < n_systems; ++s) {
    b->off.push_back((int)total);
    b->nat.push_back(systems[s].n_atoms);
    total += systems[s].n_atoms;
    blocks_total += (systems[s].n_atoms + 31) / 32;
  }
  if (total > (1LL << 30)) return fail(ctx, PB2_EINVAL, "too many atoms");
  const int N = (int)total;
  b->n_total = N;
  std::vector<double> hx(N), hy(N), hz(N), hm(N), hsig(N), hq(N), hrad(N);
  std::vector<float4> hposq(N), hpar(N);
  std::vector<double> hhs(N), hse(N), hro(N), hsr(N);
  std::vector<int32_t> hsys(N);
  b->user_host.resize(N);
  b->dev_host.resize(N);
  std::vector<std::vector<int>> inv_all(n_systems);  // per system: input index -> stored index
  std::vector<SysInfo> sinfo(n_systems);
  std::vector<uint32_t> hkeys(4 * (size_t)n_systems, 0u);
  std::vector<int2> hent((size_t)blocks_total * kExclPerBlock, make_int2(-1, -1));
  std::vector<int32_t> hblk_sys(blocks_total);
  std::vector<int4> hblk_info(blocks_total);
  std::vector<ExclRow> hrows;
  std::vector<TileItem> hitems;
  int blk_base = 0;
  for (int s = 0; s < n_systems; ++s) {
    const pb2_system_desc &d = systems[s];
    const int n = d.n_atoms, o = b->off[s];
    SysInfo &S = sinfo[s];
    memset(&S, 0, sizeof S);
    S.n = n;
    S.off = o;
    S.nblk = (n + 31) / 32;
    S.blk_base = blk_base;
    const double pref = -0.5 * d.k_gb * (1.0 / d.eps_in - 1.0 / d.eps_out);
    S.pref = (float)pref;
    S.pref_d = pref;
    S.kcoul = (float)d.k_coulomb;
    S.kcoul_d = d.k_coulomb;
    S.lj14 = (float)d.lj14_scale;
    S.coul14 = (float)d.coul14_scale;
    S.cutoff2 = cutoff_mode ? (float)(params->cutoff * params->cutoff) : 0.f;
    S.gb_cutoff2 = gb_cut_mode ? (float)(gb_cut * gb_cut) : 0.f;
    S.born_cut2 = born_mode ? (float)(born_cut * born_cut) : 0.f;
    S.clamp = born_mode ? 1 : 0;
    b->gamma_host.push_back(d.gamma);
    S.dt = d.dt;
    S.half_dt = 0.5 * d.dt;
    S.c1 = std::exp(-d.gamma * d.dt);
    S.c2 = std::sqrt(1.0 - S.c1 * S.c1);
    S.kT = d.kT;
    S.skin_half2 = 0.25 * params->skin * params->skin;
    double cx = 0, cy = 0, cz = 0;
    for (int i = 0; i < n; ++i) {
      cx += d.positions[3 * i];
      cy += d.positions[3 * i + 1];
      cz += d.positions[3 * i + 2];
    }
    S.ox = std::round(cx / n);
    S.oy = std::round(cy / n);
    S.oz = std::round(cz / n);
    if (d.use_origin) {
      S.ox = d.origin[0];
      S.oy = d.origin[1];
      S.oz = d.origin[2];
    }
    // the stored atom order computed above, or the input order when that
    // one gives an i-block exclusion partners in more j-blocks than the
    // exclusion table holds
    std::vector<int> ord;
    std::vector<int> &inv = inv_all[s];
    inv.resize(n);
    const size_t rows_before = hrows.size();
    int2 *ent_sys = &hent[(size_t)blk_base * kExclPerBlock];
    auto build_excl = [&]() -> int {  // -1: fits; else the i-block that overflows
      for (size_t e = 0; e < (size_t)S.nblk * kExclPerBlock; ++e) ent_sys[e] = make_int2(-1, -1);
      hrows.resize(rows_before);
      for (int k = 0; k < d.n_excl; ++k) {
        const int p = inv[d.excl_pairs[2 * k]], q = inv[d.excl_pairs[2 * k + 1]];
        const int i = std::min(p, q), j = std::max(p, q);
        const int ib = i >> 5, jb = j >> 5;
        int2 *ent = ent_sys + (size_t)ib * kExclPerBlock;
        int slot = -1;
        for (int e = 0; e < kExclPerBlock; ++e) {
          if (ent[e].x == jb) { slot = e; break; }
          if (ent[e].x < 0) {
            ent[e] = make_int2(jb, (int)hrows.size());
            hrows.resize(hrows.size() + 32, ExclRow{0u, 0u});
            slot = e;
            break;
          }
        }
        if (slot < 0) return ib;
        ExclRow &row = hrows[ent[slot].y + (i & 31)];
        if (d.excl_kind[k] == 0) row.excl |= 1u << (j & 31);
        else row.s14 |= 1u << (j & 31);
      }
      return -1;
    };
    ord.swap(orders[s]);
    for (int l = 0; l < n; ++l) inv[ord[l]] = l;
    int over = build_excl();
    if (over >= 0 && !params->keep_atom_order) {
      for (int l = 0; l < n; ++l) ord[l] = inv[l] = l;
      over = build_excl();
    }
    if (over >= 0) {
      char buf[200];
      snprintf(buf, sizeof buf,
               "system %d: atoms %d..%d have exclusion partners in more than %d 32-atom blocks",
               s, over * 32, over * 32 + 31, kExclPerBlock);
      return fail(ctx, PB2_EINVAL, buf);
    }
    for (int l = 0; l < n; ++l) {
      const int i = ord[l];
      const int g = o + l;
      b->user_host[g] = o + i;
      b->dev_host[o + i] = g;
      hx[g] = d.positions[3 * i];
      hy[g] = d.positions[3 * i + 1];
      hz[g] = d.positions[3 * i + 2];
      hm[g] = d.masses[i];
      hsig[g] = S.c2 * std::sqrt(d.masses[i] * d.kT);
      hq[g] = d.charges[i];
      hrad[g] = d.radii[i];
      hsys[g] = s;
      hposq[g] = make_float4((float)(hx[g] - S.ox), (float)(hy[g] - S.oy), (float)(hz[g] - S.oz),
                             (float)d.charges[i]);
      double ro = d.radii[i] - kDielOffset;
      if (born_mode) ro = std::max(std::max(d.radii[i], 1e-6) - kDielOffset, 1e-4);
      hhs[g] = 0.5 * std::max(d.sigmas[i], 1e-6);
      hse[g] = std::sqrt(std::max(d.epsilons[i], 0.0));
      hro[g] = ro;
      hsr[g] = d.scaled_radii[i];
      // float copy for the pair kernels: sqrt(24 eps), so eps_ij * 24 is one product
      hpar[g] = make_float4((float)hhs[g], (float)(hse[g] * std::sqrt(24.0)), (float)ro, (float)hsr[g]);
    }
    {  // far-field tiles: every pair has r - s >= rho~ and (s/r)^2 <= u_K
      float smax = 0.f, romax = 0.f;
      for (int i = 0; i < n; ++i) {
        smax = std::max(smax, hpar[o + i].w);
        romax = std::max(romax, hpar[o + i].z);
      }
      auto bound2 = [&](double u) {
        const double r = 1.001 * std::max((double)smax / std::sqrt(u), (double)smax + (double)romax);
        return (float)(r * r);
      };
      S.far2 = bound2(kValueTierU[3]);
      for (int t = 0; t < 3; ++t) {
        S.tier2[0][t] = bound2(kValueTierU[t]);
        S.tier2[1][t] = bound2(kDerivTierU[t]);
      }
      S.ro_max = romax;
    }
    for (int bk = 0; bk < S.nblk; ++bk) {
      hblk_sys[blk_base + bk] = s;
      hblk_info[blk_base + bk] = make_int4(s, S.off + 32 * bk, std::min(32, S.n - 32 * bk), 0);
    }
    hkeys[2 * (size_t)s] = d.key[0];
    hkeys[2 * (size_t)s + 1] = d.key[1];
    blk_base += S.nblk;
  }
  hitems = build_items(sinfo, b->params.tile_segment);
  b->n_items = (int)hitems.size();
  b->sys_host = sinfo;

  // --- bonded tables (global atom indices)
  std::vector<int2> bidx, uidx;  // bonds, Urey-Bradley springs
  std::vector<double2> bpar, upar;
  std::vector<int4> aidx;
  std::vector<double2> apar;
  std::vector<int4> tidx;
  std::vector<double4> tpar;
  std::vector<int32_t> cidx;
  std::vector<double> ccoef;
  std::vector<int32_t> cgrid;
  std::vector<int64_t> cmoff;
  std::vector<int2> eidx;
  std::vector<double4> epar;
  for (int s = 0; s < n_systems; ++s) {
    const pb2_system_desc &d = systems[s];
    const int o = b->off[s];
    const std::vector<int> &inv = inv_all[s];
    auto at = [&](int32_t i) { return o + inv[i]; };  // stored batch index of input atom i
    for (int k = 0; k < d.n_bonds; ++k) {
      bidx.push_back(make_int2(at(d.bonds[2 * k]), at(d.bonds[2 * k + 1])));
      bpar.push_back(make_double2(d.bond_params[2 * k], d.bond_params[2 * k + 1]));
    }
    for (int k = 0; k < d.n_angles; ++k) {
      aidx.push_back(make_int4(at(d.angles[3 * k]), at(d.angles[3 * k + 1]), at(d.angles[3 * k + 2]), 0));
      apar.push_back(make_double2(d.angle_params[2 * k], d.angle_params[2 * k + 1]));
    }
    for (int k = 0; k < d.n_torsions; ++k)
      for (int t = 0; t < d.n_torsion_terms; ++t) {
        const double *p = d.torsion_params + ((size_t)k * d.n_torsion_terms + t) * 3;
        tidx.push_back(make_int4(at(d.torsions[4 * k]), at(d.torsions[4 * k + 1]),
                                 at(d.torsions[4 * k + 2]), at(d.torsions[4 * k + 3])));
        tpar.push_back(make_double4(p[0], p[1], p[2], kTorsProper));
      }
    for (int k = 0; k < d.n_impropers; ++k)
      for (int t = 0; t < d.n_improper_terms; ++t) {
        tidx.push_back(make_int4(at(d.impropers[4 * k]), at(d.impropers[4 * k + 1]),
                                 at(d.impropers[4 * k + 2]), at(d.impropers[4 * k + 3])));
        if (d.improper_form == 1) {
          const double *p = d.improper_params + ((size_t)k * d.n_improper_terms + t) * 2;
          tpar.push_back(make_double4(p[0], p[1], 0.0, kTorsHarmonic));
        } else {
          const double *p = d.improper_params + ((size_t)k * d.n_improper_terms + t) * 3;
          tpar.push_back(make_double4(p[0], p[1], p[2], kTorsImproper));
        }
      }
    for (int k = 0; k < d.n_urey_bradley; ++k) {
      uidx.push_back(make_int2(at(d.urey_bradley_bonds[2 * k]), at(d.urey_bradley_bonds[2 * k + 1])));
      upar.push_back(make_double2(d.urey_bradley_params[2 * k], d.urey_bradley_params[2 * k + 1]));
    }
    const int map_base = (int)cgrid.size();
    const size_t per_map = (size_t)d.cmap_grid * d.cmap_grid * 16;
    for (int m = 0; m < d.n_cmap_maps && d.n_cmap > 0; ++m) {
      cgrid.push_back(d.cmap_grid);
      cmoff.push_back((int64_t)ccoef.size());
      ccoef.insert(ccoef.end(), d.cmap_coeffs + m * per_map, d.cmap_coeffs + (m + 1) * per_map);
    }
    for (int k = 0; k < d.n_cmap; ++k) {
      for (int c = 0; c < 5; ++c) cidx.push_back(at(d.cmap_rows[5 * k + c]));
      cidx.push_back(map_base + d.cmap_map[k]);
    }
    for (int k = 0; k < d.n_exceptions; ++k) {
      const double *p = d.exception_params + 3 * (size_t)k;
      eidx.push_back(make_int2(at(d.exception_pairs[2 * k]), at(d.exception_pairs[2 * k + 1])));
      epar.push_back(make_double4(d.k_coulomb * p[0], p[1], p[2], 0.0));
    }
  }

  // terms in order of their (central) atom: with atoms in spatial order, the
  // threads of a warp then read and update nearby atoms
  auto by_atom = [N](auto &idx, auto &par, auto key) {  // stable counting sort by key in [0, N)
    std::vector<int> start(N + 1, 0);
    for (const auto &t : idx) ++start[key(t) + 1];
    for (int a = 0; a < N; ++a) start[a + 1] += start[a];
    auto idx2 = idx;
    auto par2 = par;
    for (size_t k = 0; k < idx.size(); ++k) {
      const int dst = start[key(idx[k])]++;
      idx2[dst] = idx[k];
      par2[dst] = par[k];
    }
    idx.swap(idx2);
    par.swap(par2);
  };
  by_atom(bidx, bpar, [](const int2 &t) { return std::min(t.x, t.y); });
  by_atom(uidx, upar, [](const int2 &t) { return std::min(t.x, t.y); });
  const int n_bond_plain = (int)bidx.size();  // Urey-Bradley springs follow the bonds
  bidx.insert(bidx.end(), uidx.begin(), uidx.end());
  bpar.insert(bpar.end(), upar.begin(), upar.end());
  by_atom(aidx, apar, [](const int4 &t) { return t.y; });
  by_atom(tidx, tpar, [](const int4 &t) { return std::min(t.y, t.z); });
  by_atom(eidx, epar, [](const int2 &t) { return std::min(t.x, t.y); });

  // --- device allocation
  Dev &D = b->dev;
  b->sys = D.alloc<SysInfo>(n_systems);
  b->atom_sys = D.alloc<int32_t>(N);
  b->x = D.alloc<double>(N); b->y = D.alloc<double>(N); b->z = D.alloc<double>(N);
  b->px = D.alloc<double>(N); b->py = D.alloc<double>(N); b->pz = D.alloc<double>(N);
  b->fx = D.alloc<long long>(N); b->fy = D.alloc<long long>(N); b->fz = D.alloc<long long>(N);
  b->mass = D.alloc<double>(N);
  b->sigma = D.alloc<double>(N);
  b->charge = D.alloc<double>(N);
  b->radius = D.alloc<double>(N);
  b->posq = D.alloc<float4>(N);
  b->par = D.alloc<float4>(N);
  b->born = D.alloc<float4>(N);
  b->bbox = D.alloc<float4>(2 * (size_t)blocks_total);
  b->sched = D.alloc<int32_t>(8);
  b->blk_sys = D.alloc<int32_t>(blocks_total);
  b->blk_info = D.alloc<int4>(blocks_total);
  b->n_blocks = blocks_total;
  b->cut = cutoff_mode || gb_cut_mode || born_mode;
  {
    // the pair list needs a finite reach for every pair term in use
    const uint32_t t = params->terms;
    const bool direct = (t & (PB2_USE_LJ | PB2_USE_COULOMB)) != 0, gbt = (t & PB2_USE_GB) != 0;
    double reach = 0.0;
    bool finite = b->cut && params->skin >= 0.0 && params->pair_list >= 0;
    if (direct) {
      finite = finite && cutoff_mode;
      reach = std::max(reach, params->cutoff);
    }
    if (gbt) {
      finite = finite && gb_cut_mode;
      reach = std::max(reach, std::max(gb_cut, born_cut));
    }
    b->pl_on = finite && (direct || gbt);
    b->pl_reach2 = (float)((reach + params->skin) * (reach + params->skin));
  }
  b->q64 = D.alloc<double>(N);
  b->hs64 = D.alloc<double>(N);
  b->se64 = D.alloc<double>(N);
  b->ro64 = D.alloc<double>(N);
  b->sr64 = D.alloc<double>(N);
  b->born64 = D.alloc<double>(N);
  b->stage = D.alloc<double>(9 * (size_t)N);  // x, p, F rows of a host round trip
  b->user = D.alloc<int32_t>(N);
  b->devidx = D.alloc<int32_t>(N);
  b->born_acc = D.alloc<long long>(N);
  b->dedb_acc = D.alloc<long long>(N);
  b->energy = D.alloc<long long>((size_t)n_systems * PB2_NTERMS);
  b->keys = D.alloc<uint32_t>(4 * (size_t)n_systems);
  b->key_splits = D.alloc<uint32_t>(8 * (size_t)n_systems);
  b->steps = D.alloc<long long>(n_systems);
  b->status = D.alloc<uint32_t>(n_systems);
  b->guard_end = D.alloc<int32_t>(1);
  b->warn_flags = D.alloc<uint32_t>(2 * (size_t)n_systems);
  b->warn_counts = D.alloc<int32_t>((size_t)n_systems * kWarnTypes);
  b->items = D.alloc<TileItem>(hitems.size());
  b->excl_ent = D.alloc<int2>(hent.size());
  b->excl_rows = D.alloc<ExclRow>(hrows.size());
  BondedArgs &B = b->bonded;
  B.n_bond = (int)bidx.size();
  B.n_bond_plain = n_bond_plain;
  B.n_angle = (int)aidx.size();
  B.n_tors = (int)tidx.size();
  B.n_cmap = (int)(cidx.size() / 6);
  B.n_exc = (int)eidx.size();
  int2 *d_eidx = D.alloc<int2>(eidx.size());
  double4 *d_epar = D.alloc<double4>(epar.size());
  int2 *d_bidx = D.alloc<int2>(bidx.size());
  double2 *d_bpar = D.alloc<double2>(bpar.size());
  int4 *d_aidx = D.alloc<int4>(aidx.size());
  double2 *d_apar = D.alloc<double2>(apar.size());
  int4 *d_tidx = D.alloc<int4>(tidx.size());
  double4 *d_tpar = D.alloc<double4>(tpar.size());
  int32_t *d_cidx = D.alloc<int32_t>(cidx.size());
  double *d_ccoef = D.alloc<double>(ccoef.size());
  int32_t *d_cgrid = D.alloc<int32_t>(cgrid.size());
  int64_t *d_cmoff = D.alloc<int64_t>(cmoff.size());
  for (void *p : D.ptrs)
    if (!p) return fail(ctx, PB2_ENOMEM, "device allocation failed");
  if (!d_cmoff || !d_cgrid || !d_ccoef || !d_cidx || !b->excl_rows)
    return fail(ctx, PB2_ENOMEM, "device allocation failed");

  int rc;
  if ((rc = upload(ctx, b->sys, sinfo)) || (rc = upload(ctx, b->atom_sys, hsys)) ||
      (rc = upload(ctx, b->x, hx)) || (rc = upload(ctx, b->y, hy)) || (rc = upload(ctx, b->z, hz)) ||
      (rc = upload(ctx, b->mass, hm)) || (rc = upload(ctx, b->sigma, hsig)) ||
      (rc = upload(ctx, b->charge, hq)) || (rc = upload(ctx, b->radius, hrad)) ||
      (rc = upload(ctx, b->posq, hposq)) || (rc = upload(ctx, b->par, hpar)) ||
      (rc = upload(ctx, b->q64, hq)) || (rc = upload(ctx, b->hs64, hhs)) ||
      (rc = upload(ctx, b->se64, hse)) || (rc = upload(ctx, b->ro64, hro)) ||
      (rc = upload(ctx, b->sr64, hsr)) || (rc = upload(ctx, b->user, b->user_host)) ||
      (rc = upload(ctx, b->devidx, b->dev_host)) ||
      (rc = upload(ctx, b->keys, hkeys)) || (rc = upload(ctx, b->blk_sys, hblk_sys)) ||
      (rc = upload(ctx, b->blk_info, hblk_info)) || (rc = upload(ctx, b->items, hitems)) ||
      (rc = upload(ctx, b->excl_ent, hent)) || (rc = upload(ctx, b->excl_rows, hrows)) ||
      (rc = upload(ctx, d_bidx, bidx)) || (rc = upload(ctx, d_bpar, bpar)) ||
      (rc = upload(ctx, d_aidx, aidx)) || (rc = upload(ctx, d_apar, apar)) ||
      (rc = upload(ctx, d_tidx, tidx)) || (rc = upload(ctx, d_tpar, tpar)) ||
      (rc = upload(ctx, d_cidx, cidx)) || (rc = upload(ctx, d_ccoef, ccoef)) ||
      (rc = upload(ctx, d_cgrid, cgrid)) || (rc = upload(ctx, d_cmoff, cmoff)) ||
      (rc = upload(ctx, d_eidx, eidx)) || (rc = upload(ctx, d_epar, epar)))
    return rc;
  warm_step_launch(b->n_blocks);
  CUDA_TRY(ctx, launch_key_splits(int_args(b.get(), 0, 0), nullptr));
  CUDA_TRY(ctx, cudaMemset(b->px, 0, N * sizeof(double)));
  CUDA_TRY(ctx, cudaMemset(b->py, 0, N * sizeof(double)));
  CUDA_TRY(ctx, cudaMemset(b->pz, 0, N * sizeof(double)));
  CUDA_TRY(ctx, cudaMemset(b->fx, 0, N * sizeof(long long)));
  CUDA_TRY(ctx, cudaMemset(b->fy, 0, N * sizeof(long long)));
  CUDA_TRY(ctx, cudaMemset(b->fz, 0, N * sizeof(long long)));
  CUDA_TRY(ctx, cudaMemset(b->born_acc, 0, N * sizeof(long long)));
  CUDA_TRY(ctx, cudaMemset(b->dedb_acc, 0, N * sizeof(long long)));
  CUDA_TRY(ctx, cudaMemset(b->born, 0, N * sizeof(float4)));
  CUDA_TRY(ctx, cudaMemset(b->steps, 0, n_systems * sizeof(long long)));
  CUDA_TRY(ctx, cudaMemset(b->sched, 0, 8 * sizeof(int32_t)));
  CUDA_TRY(ctx, cudaMemset(b->status, 0, n_systems * sizeof(uint32_t)));
  CUDA_TRY(ctx, cudaMemset(b->guard_end, 0, sizeof(int32_t)));
  CUDA_TRY(ctx, cudaMemset(b->warn_flags, 0, 2 * (size_t)n_systems * sizeof(uint32_t)));
  CUDA_TRY(ctx, cudaMemset(b->warn_counts, 0, (size_t)n_systems * kWarnTypes * sizeof(int32_t)));
  B.atom_sys = b->atom_sys;
  B.x = b->x; B.y = b->y; B.z = b->z;
  B.fx = b->fx; B.fy = b->fy; B.fz = b->fz;
  B.energy = b->energy;
  B.terms = params->terms;
  B.bond_idx = d_bidx; B.bond_par = d_bpar;
  B.angle_idx = d_aidx; B.angle_par = d_apar;
  B.tors_idx = d_tidx; B.tors_par = d_tpar;
  B.cmap_idx = d_cidx; B.cmap_coeff = d_ccoef; B.cmap_grid = d_cgrid; B.cmap_map_off = d_cmoff;
  B.exc_idx = d_eidx; B.exc_par = d_epar;
  if (!(params->terms & PB2_USE_BONDED)) B.n_bond = B.n_angle = B.n_tors = 0;
  if (!(params->terms & PB2_USE_CMAP)) B.n_cmap = 0;
  if (!(params->terms & (PB2_USE_LJ | PB2_USE_COULOMB))) B.n_exc = 0;

  b->grid_bonded = 8 * ctx->sm_count;
  if ((rc = setup_items2(b.get(), b->params.tile_segment))) return rc;
  if ((rc = setup_pair_list(b.get(), b->params.tile_segment))) return rc;
  {
    b->fuse = PB2_FUSE_BONDED;  // the autotuner may change this
  }
  CUDA_TRY(ctx, cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
  CUDA_TRY(ctx, cudaEventCreate(&b->ev[0]));
  CUDA_TRY(ctx, cudaEventCreate(&b->ev[1]));
  for (auto &e : b->ev_io) CUDA_TRY(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto &e : b->nl_ev) CUDA_TRY(ctx, cudaEventCreate(&e));
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  *out = b.release();
  return PB2_OK;
}

extern "C" int pb2_batch_destroy(pb2_batch *b) {
  if (!b) return PB2_OK;
  cudaSetDevice(b->ctx->device);
  cudaDeviceSynchronize();
  delete b;
  return PB2_OK;
}

extern "C" int pb2_batch_info(const pb2_batch *b, int32_t *n_systems, int64_t *n_atoms_total) {
  if (!b) return PB2_EINVAL;
  if (n_systems) *n_systems = b->n_sys;
  if (n_atoms_total) *n_atoms_total = b->n_total;
  return PB2_OK;
}

// ------------------------------------------------------------ force evaluation

// In profiling mode, time one launch with CUDA events (eager runs only).
struct Timer {
  pb2_batch *b;
  cudaStream_t st;
  template <class F>
  cudaError_t operator()(int slot, F &&launch) {
    if (!b->profiling) return launch();
    cudaEventRecord(b->ev[0], st);
    const cudaError_t e = launch();
    cudaEventRecord(b->ev[1], st);
    cudaEventSynchronize(b->ev[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
    b->timings[slot] += ms;
    return e;
  }
};

// Force kernels on the current posq; force accumulators must be zero (or
// hold contributions to keep) and born_acc zero.  bonded_energy: also
// accumulate the (FP64) bonded energies.  boxes_ready: the step kernel just
// wrote the block boxes (and ran the pair list's displacement test).
static cudaError_t enqueue_forces(pb2_batch *b, cudaStream_t st, bool bonded_energy,
                                  bool boxes_ready = false) {
  cudaError_t e;
  Timer tm{b, st};
  PairArgs pa = pair_args(b);
  const bool gb = (b->params.terms & PB2_USE_GB) != 0;
  if (!boxes_ready && (e = tm(kTimBbox, [&] {
         return launch_bbox(b->sys, b->blk_sys, b->posq, b->bbox, b->n_blocks, st,
                            b->pl_on ? b->pl_ref : nullptr, b->pl_on ? b->pl_ctl : nullptr);
       })) != cudaSuccess)
    return e;
  if (b->pl_on && (e = tm(kTimBbox, [&] { return launch_pl_update(pl_args(b), b->grid_pl, st); })) != cudaSuccess)
    return e;
  if (gb) {
    FinalizeArgs fa;
    fa.sys = b->sys;
    fa.atom_sys = b->atom_sys;
    fa.radius = b->radius;
    fa.charge = b->charge;
    fa.born_acc = b->born_acc;
    fa.born = b->born;
    fa.dedb_acc = b->dedb_acc;
    fa.energy = b->energy;
    fa.born64 = nullptr;
    fa.n_total = b->n_total;
    fa.energy_mode = 0;
    fa.blk_sys = b->blk_sys;
    fa.n_blocks = b->n_blocks;
    fa.sys_fin = b->sys_fin;
    fa.retired = b->retired;
    fa.status = b->status;
    // the descreening pass finalizes each block once its system's items are
    // summed (profiling keeps the separate launch, to time it)
    const bool fuse_finalize = !b->profiling && (b->fuse & PB2_FUSE_FINALIZE);
    PairArgs pb = pa;
    pb.sched = b->sched + 2 * PASS_BORN;
    if (fuse_finalize) {
      pb.sys_items = b->sys_items;
      pb.fin = fa;
    }
    if ((e = tm(kTimBorn, [&] { return launch_tiles(PASS_BORN, pb, b->grid_pair[PASS_BORN], b->shape[PASS_BORN], st); })) != cudaSuccess)
      return e;
    if (!fuse_finalize &&
        (e = tm(kTimFinalize, [&] { return launch_born_finalize(fa, st); })) != cudaSuccess)
      return e;
  }
  pa.sched = b->sched + 2 * PASS_FORCE;
  if (b->force_blocks == 4 && !b->pl_on) {
    PairArgs p4 = pa;
    p4.items = b->items4;
    p4.n_items = b->n_items4;
    p4.item_count = b->item_count4;
    if ((e = tm(kTimForce, [&] { return launch_force4(p4, b->grid4, b->shape4, st); })) != cudaSuccess) return e;
  } else if ((e = tm(kTimForce, [&] {
                return launch_tiles(PASS_FORCE, pa, b->grid_pair[PASS_FORCE], b->shape[PASS_FORCE], st);
              })) != cudaSuccess) {
    return e;
  }
  pa.sched = b->sched + 2 * PASS_CHAIN;
  BondedArgs ba = b->bonded;
  ba.energy_mode = bonded_energy ? 1 : 0;
  const int n_bonded = ba.n_bond + ba.n_angle + ba.n_tors + ba.n_cmap + ba.n_exc;
  // the bonded terms ride along as the chain pass's tail work, except when
  // their energies are wanted or there is no chain pass
  const bool fuse_bonded = gb && !bonded_energy && !b->profiling && (b->fuse & PB2_FUSE_BONDED);
  if (fuse_bonded) {
    pa.bonded = ba;
    pa.n_bonded_chunks = (n_bonded + kBondedChunk - 1) / kBondedChunk;
  }
  if (gb)
    if ((e = tm(kTimChain, [&] { return launch_tiles(PASS_CHAIN, pa, b->grid_pair[PASS_CHAIN], b->shape[PASS_CHAIN], st); })) != cudaSuccess)
      return e;
  if (fuse_bonded) return cudaSuccess;
  return tm(kTimBonded, [&] { return launch_bonded(ba, b->grid_bonded, st); });
}

// FP64 pair energies (GB polar incl. self, ACE, Coulomb, LJ) into b->energy.
static cudaError_t enqueue_energy64(pb2_batch *b, cudaStream_t st) {
  cudaError_t e;
  Energy64Args ea;
  ea.sys = b->sys;
  ea.items = b->items;
  ea.n_items = b->n_items;
  ea.terms = b->params.terms;
  ea.excl_ent = b->excl_ent;
  ea.excl_rows = b->excl_rows;
  ea.x = b->x; ea.y = b->y; ea.z = b->z;
  ea.q = b->q64; ea.hs = b->hs64; ea.se = b->se64; ea.ro = b->ro64; ea.sr = b->sr64;
  ea.born64 = b->born64;
  ea.born_acc = b->born_acc;
  ea.energy = b->energy;
  const int grid = b->grid_pair[PASS_FORCE];
  if (b->params.terms & PB2_USE_GB) {
    if ((e = cudaMemsetAsync(b->born_acc, 0, (size_t)b->n_total * sizeof(long long), st)) != cudaSuccess) return e;
    if ((e = launch_energy64(0, ea, grid, st)) != cudaSuccess) return e;
    FinalizeArgs fa;
    fa.sys = b->sys;
    fa.atom_sys = b->atom_sys;
    fa.radius = b->radius;
    fa.charge = b->charge;
    fa.born_acc = b->born_acc;
    fa.born = b->born;
    fa.dedb_acc = b->dedb_acc;
    fa.energy = b->energy;
    fa.born64 = b->born64;
    fa.n_total = b->n_total;
    fa.energy_mode = 1;
    if ((e = launch_born_finalize(fa, st)) != cudaSuccess) return e;
  }
  return launch_energy64(1, ea, grid, st);
}

static int fresh_forces(pb2_batch *b, cudaStream_t st, bool energy) {
  pb2_ctx *ctx = b->ctx;
  const size_t nb = (size_t)b->n_total * sizeof(long long);
  CUDA_TRY(ctx, cudaMemsetAsync(b->fx, 0, nb, st));
  CUDA_TRY(ctx, cudaMemsetAsync(b->fy, 0, nb, st));
  CUDA_TRY(ctx, cudaMemsetAsync(b->fz, 0, nb, st));
  if (energy)
    CUDA_TRY(ctx, cudaMemsetAsync(b->energy, 0, (size_t)b->n_sys * PB2_NTERMS * sizeof(long long), st));
  CUDA_TRY(ctx, launch_posq(int_args(b, b->key_parity, 0), st));
  CUDA_TRY(ctx, enqueue_forces(b, st, energy));
  if (energy) CUDA_TRY(ctx, enqueue_energy64(b, st));
  b->forces_valid = true;
  return PB2_OK;
}

static int copy_forces(pb2_batch *b, double *forces, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  const int N = b->n_total;
  CUDA_TRY(ctx, launch_fix_to_rows(b->fx, b->fy, b->fz, b->user, b->stage, N, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(forces, b->stage, 3 * (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

// Device-pointer variant: no host copy, no allocation, no synchronisation
// (usable from an XLA custom call or under stream capture).
extern "C" int pb2_energy_forces_device(pb2_batch *b, const double *positions, double *energies,
                                        double *forces, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t N = b->n_total;
  if (positions) {
    CUDA_TRY(ctx, cudaMemcpyAsync(b->stage, positions, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(ctx, launch_rows_to_soa(b->stage, b->user, b->x, b->y, b->z, b->n_total, st));
  }
  int rc = fresh_forces(b, st, energies != nullptr);
  if (rc) return rc;
  if (energies) CUDA_TRY(ctx, launch_energies_to_double(b->energy, energies, b->n_sys, st));
  if (forces) CUDA_TRY(ctx, launch_fix_to_rows(b->fx, b->fy, b->fz, b->user, forces, b->n_total, st));
  return PB2_OK;
}

extern "C" int pb2_energy_forces(pb2_batch *b, double *energies, double *forces, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  int rc = fresh_forces(b, st, energies != nullptr);
  if (rc) return rc;
  if (energies) {
    std::vector<long long> he((size_t)b->n_sys * PB2_NTERMS);
    CUDA_TRY(ctx, cudaMemcpyAsync(he.data(), b->energy, he.size() * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    for (int s = 0; s < b->n_sys; ++s) {
      double tot = 0.0;
      for (int t = 0; t < PB2_TERM_TOTAL; ++t) {
        const double v = (double)he[(size_t)s * PB2_NTERMS + t] * kEnergyInv;
        energies[(size_t)s * PB2_NTERMS + t] = v;
        tot += v;
      }
      energies[(size_t)s * PB2_NTERMS + PB2_TERM_TOTAL] = tot;
    }
  }
  if (forces) return copy_forces(b, forces, st);
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_born_radii(pb2_batch *b, double *out, void *stream) {
  if (!b || !out) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  if (!(b->params.terms & PB2_USE_GB)) return fail(ctx, PB2_EINVAL, "GB term disabled");
  int rc = fresh_forces(b, st, false);
  if (rc) return rc;
  std::vector<float4> hb(b->n_total);
  CUDA_TRY(ctx, cudaMemcpyAsync(hb.data(), b->born, hb.size() * sizeof(float4), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  for (int g = 0; g < b->n_total; ++g) out[b->user_host[g]] = (double)hb[g].x;
  return PB2_OK;
}

// Row-major (n, 3) host arrays move through the device staging buffer in one
// copy each; the (de)interleave runs on the device.  The staging buffer is
// reused by the next transfer on the same stream, so each helper finishes
// its copy before returning.
static int upload_soa3(pb2_batch *b, const double *aos, double *dx, double *dy, double *dz, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  const int N = b->n_total;
  CUDA_TRY(ctx, cudaMemcpyAsync(b->stage, aos, 3 * (size_t)N * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, launch_rows_to_soa(b->stage, b->user, dx, dy, dz, N, st));
  return PB2_OK;
}

static int download_soa3(pb2_batch *b, double *aos, const double *dx, const double *dy, const double *dz,
                         cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  const int N = b->n_total;
  CUDA_TRY(ctx, launch_soa_to_rows(dx, dy, dz, b->user, b->stage, N, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(aos, b->stage, 3 * (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_set_positions(pb2_batch *b, const double *positions, void *stream) {
  if (!b || !positions) return PB2_EINVAL;
  b->forces_valid = false;
  int rc = upload_soa3(b, positions, b->x, b->y, b->z, (cudaStream_t)stream);
  if (rc || (rc = forces_not_from_step(b, (cudaStream_t)stream))) return rc;
  CUDA_TRY(b->ctx, cudaStreamSynchronize((cudaStream_t)stream));
  return PB2_OK;
}

// ------------------------------------------------------------ Langevin

static int run_eager(pb2_batch *b, int n_steps, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  Timer tm{b, st};
  for (int t = 0; t < n_steps; ++t) {
    const IntArgs ia = int_args(b, b->key_parity, t > 0);
    CUDA_TRY(ctx, tm(kTimStep, [&] { return launch_step(ia, st); }));
    CUDA_TRY(ctx, enqueue_forces(b, st, false, true));
    b->key_parity ^= 1;
  }
  const IntArgs fa = int_args(b, b->key_parity, 0);
  CUDA_TRY(ctx, tm(kTimStep, [&] { return launch_finish(fa, st); }));
  return PB2_OK;
}

static int get_graph(pb2_batch *b, int chunk, int parity, cudaGraphExec_t *out) {
  pb2_ctx *ctx = b->ctx;
  auto key = std::make_pair(chunk, parity);
  auto it = b->graphs.find(key);
  if (it != b->graphs.end()) {
    *out = it->second;
    return PB2_OK;
  }
  cudaStream_t cs = b->cap_stream;
  CUDA_TRY(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  int p = parity;
  for (int t = 0; t < chunk && err == cudaSuccess; ++t) {
    err = launch_step(int_args(b, p, t > 0), cs);
    if (err == cudaSuccess) err = enqueue_forces(b, cs, false, true);
    p ^= 1;
  }
  if (err == cudaSuccess) err = launch_finish(int_args(b, p, 0), cs);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(cs, &g);
  if (err != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(ctx, PB2_ECUDA, std::string("graph capture failed: ") +
                                    cudaGetErrorString(err != cudaSuccess ? err : e2));
  }
  cudaGraphExec_t ex = nullptr;
  cudaError_t e3 = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) return fail(ctx, PB2_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e3));
  b->graphs[key] = ex;
  *out = ex;
  return PB2_OK;
}

extern "C" int pb2_langevin_init(pb2_batch *b, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, launch_init(int_args(b, b->key_parity, 0), st));
  b->key_parity ^= 1;
  int rc = fresh_forces(b, st, false);
  if (rc || (rc = forces_not_from_step(b, st))) return rc;
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_set_langevin_params(pb2_batch *b, const double *dt, const double *kT,
                                       const double *gamma, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  const int S = b->n_sys;
  for (int s = 0; s < S; ++s)
    if ((dt && !(dt[s] > 0.0)) || (kT && !(kT[s] >= 0.0)) || (gamma && !(gamma[s] >= 0.0)))
      return fail(ctx, PB2_EINVAL, "dt > 0, kT >= 0, gamma >= 0");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  // steps already queued, on any stream of the device, finish with the old
  // values: the per-system constants are overwritten in place
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  for (int s = 0; s < S; ++s) {
    SysInfo &I = b->sys_host[s];
    if (dt) I.dt = dt[s];
    if (kT) I.kT = kT[s];
    if (gamma) b->gamma_host[s] = gamma[s];
    I.half_dt = 0.5 * I.dt;
    I.c1 = std::exp(-b->gamma_host[s] * I.dt);
    I.c2 = std::sqrt(1.0 - I.c1 * I.c1);
  }
  CUDA_TRY(ctx, cudaMemcpyAsync(b->sys, b->sys_host.data(), S * sizeof(SysInfo), cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, launch_noise_scale(b->sys, b->atom_sys, b->mass, b->sigma, b->n_total, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_langevin_center_momentum(pb2_batch *b, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, launch_center(int_args(b, b->key_parity, 0), st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_langevin_run(pb2_batch *b, int32_t n_steps, void *stream) {
  if (!b || n_steps < 0) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (n_steps == 0) return PB2_OK;
  if (!b->forces_valid) {
    int rc = fresh_forces(b, st, false);
    if (rc) return rc;
  }
  if (b->profiling) {
    for (double &t : b->timings) t = 0.0;
    cudaEvent_t a0, a1;
    cudaEventCreate(&a0);
    cudaEventCreate(&a1);
    cudaEventRecord(a0, st);
    int rc = run_eager(b, n_steps, st);
    cudaEventRecord(a1, st);
    cudaEventSynchronize(a1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a0, a1);
    b->timings[kTimAll] = ms;
    cudaEventDestroy(a0);
    cudaEventDestroy(a1);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return PB2_OK;
  }
  const int chunk = b->params.graph_chunk;
  int done = 0;
  while (done < n_steps) {
    const int c = std::min(chunk, n_steps - done);
    cudaGraphExec_t ex;
    int rc = get_graph(b, c, b->key_parity, &ex);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaGraphLaunch(ex, st));
    b->key_parity ^= (c & 1);
    done += c;
  }
  return PB2_OK;
}

extern "C" int pb2_get_state(pb2_batch *b, double *x, double *p, double *f, uint32_t *keys,
                             int64_t *steps, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (x && (rc = download_soa3(b, x, b->x, b->y, b->z, st))) return rc;
  if (p && (rc = download_soa3(b, p, b->px, b->py, b->pz, st))) return rc;
  if (f && (rc = copy_forces(b, f, st))) return rc;
  if (keys) {
    CUDA_TRY(ctx, cudaMemcpyAsync(keys, b->keys + (size_t)b->key_parity * b->n_sys * 2,
                                  (size_t)b->n_sys * 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  }
  if (steps) {
    std::vector<long long> h(b->n_sys);
    CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), b->steps, h.size() * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    for (int s = 0; s < b->n_sys; ++s) steps[s] = h[s];
  }
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_set_state(pb2_batch *b, const double *x, const double *p, const uint32_t *keys,
                             void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (x && (rc = upload_soa3(b, x, b->x, b->y, b->z, st))) return rc;
  if (p && (rc = upload_soa3(b, p, b->px, b->py, b->pz, st))) return rc;
  if (keys) {
    CUDA_TRY(ctx, cudaMemcpyAsync(b->keys + (size_t)b->key_parity * b->n_sys * 2, keys,
                                  (size_t)b->n_sys * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, launch_key_splits(int_args(b, b->key_parity, 0), st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
  }
  if (x) {  // forces must follow the positions
    rc = fresh_forces(b, st, false);
    if (rc || (rc = forces_not_from_step(b, st))) return rc;
  }
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_set_full_state(pb2_batch *b, const double *x, const double *p, const double *f,
                                  const uint32_t *keys, void *stream) {
  if (!b || !x || !p || !f) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  int rc;
  if ((rc = upload_soa3(b, x, b->x, b->y, b->z, st))) return rc;
  if ((rc = upload_soa3(b, p, b->px, b->py, b->pz, st))) return rc;
  CUDA_TRY(ctx, cudaMemcpyAsync(b->stage, f, 3 * (size_t)b->n_total * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, launch_rows_to_fix(b->stage, b->user, b->fx, b->fy, b->fz, b->n_total, st));
  if (keys) {
    CUDA_TRY(ctx, cudaMemcpyAsync(b->keys + (size_t)b->key_parity * b->n_sys * 2, keys,
                                  (size_t)b->n_sys * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, launch_key_splits(int_args(b, b->key_parity, 0), st));
  }
  CUDA_TRY(ctx, launch_posq(int_args(b, b->key_parity, 0), st));
  b->forces_valid = true;
  if ((rc = forces_not_from_step(b, st))) return rc;
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}


// The functional step on caller-held state: copies in on copy_in, steps on
// stream, copies out on copy_out.  kind_in / kind_out are the directions of
// the copies (host arrays, or the caller's device arrays).
static int run_caller_state(pb2_batch *b, double *x, double *p, double *f, int32_t n_steps,
                            void *stream, void *copy_in, void *copy_out, cudaMemcpyKind kind_in,
                            cudaMemcpyKind kind_out) {
  if (!b || !x || !p || !f || n_steps < 0) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream, ci = (cudaStream_t)copy_in, co = (cudaStream_t)copy_out;
  const int N = b->n_total;
  const size_t rows = 3 * (size_t)N, bytes = rows * sizeof(double);
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  // in: the previous round trip's copies out of the staging buffer are done;
  // the three copies back to back, then one conversion
  CUDA_TRY(ctx, cudaStreamWaitEvent(ci, b->ev_io[2], 0));
  CUDA_TRY(ctx, cudaMemcpyAsync(b->stage, x, bytes, kind_in, ci));
  CUDA_TRY(ctx, cudaMemcpyAsync(b->stage + rows, p, bytes, kind_in, ci));
  CUDA_TRY(ctx, cudaMemcpyAsync(b->stage + 2 * rows, f, bytes, kind_in, ci));
  CUDA_TRY(ctx, cudaEventRecord(b->ev_io[0], ci));
  CUDA_TRY(ctx, cudaStreamWaitEvent(st, b->ev_io[0], 0));
  CUDA_TRY(ctx, launch_state_from_rows(b->stage, b->user, b->x, b->y, b->z, b->px, b->py, b->pz, b->fx, b->fy, b->fz,
                                       N, st));
  CUDA_TRY(ctx, launch_posq(int_args(b, b->key_parity, 0), st));
  b->forces_valid = true;
  int rc = pb2_langevin_run(b, n_steps, stream);
  if (rc) return rc;
  // out: one conversion, then the three copies
  CUDA_TRY(ctx, launch_state_to_rows(b->x, b->y, b->z, b->px, b->py, b->pz, b->fx, b->fy, b->fz, b->user,
                                     b->stage, N, st));
  CUDA_TRY(ctx, cudaEventRecord(b->ev_io[1], st));
  CUDA_TRY(ctx, cudaStreamWaitEvent(co, b->ev_io[1], 0));
  CUDA_TRY(ctx, cudaMemcpyAsync(x, b->stage, bytes, kind_out, co));
  CUDA_TRY(ctx, cudaMemcpyAsync(p, b->stage + rows, bytes, kind_out, co));
  CUDA_TRY(ctx, cudaMemcpyAsync(f, b->stage + 2 * rows, bytes, kind_out, co));
  CUDA_TRY(ctx, cudaEventRecord(b->ev_io[2], co));
  return PB2_OK;
}

extern "C" int pb2_langevin_run_host(pb2_batch *b, double *x, double *p, double *f, int32_t n_steps,
                                     void *stream, void *copy_in, void *copy_out) {
  return run_caller_state(b, x, p, f, n_steps, stream, copy_in, copy_out, cudaMemcpyHostToDevice,
                          cudaMemcpyDeviceToHost);
}

extern "C" int pb2_langevin_run_device(pb2_batch *b, double *x, double *p, double *f, int32_t n_steps,
                                       void *stream) {
  return run_caller_state(b, x, p, f, n_steps, stream, stream, stream, cudaMemcpyDeviceToDevice,
                          cudaMemcpyDeviceToDevice);
}

// ------------------------------------------------------------ minimisation

static MinArgs min_args(pb2_batch *b) {
  MinArgs a;
  a.sys = b->sys;
  a.atom_sys = b->atom_sys;
  a.x = b->x; a.y = b->y; a.z = b->z;
  a.px = b->px; a.py = b->py; a.pz = b->pz;
  a.fx = b->fx; a.fy = b->fy; a.fz = b->fz;
  a.mass = b->mass;
  a.charge = b->charge;
  a.posq = b->posq;
  a.x0 = b->m_x0;
  a.sel = b->m_sel;
  a.ft = b->m_ft; a.xb = b->m_xb; a.best = b->m_best;
  a.sys_dt = b->m_sys;
  a.sys_alpha = b->m_sys + b->n_sys;
  a.sys_best = b->m_sys + 2 * (size_t)b->n_sys;
  a.sys_npos = b->m_npos;
  a.status = b->status;
  a.par = b->m_par;
  a.n_total = b->n_total;
  a.n_sys = b->n_sys;
  return a;
}

extern "C" int pb2_min_setup(pb2_batch *b, const uint8_t *heavy, const uint8_t *backbone) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const size_t N = b->n_total;
  if (!b->m_x0) {
    Dev &D = b->mdev;
    b->m_x0 = D.alloc<double>(3 * N);
    b->m_ft = D.alloc<double>(3 * N);
    b->m_xb = D.alloc<double>(3 * N);
    b->m_best = D.alloc<double>(3 * N);
    b->m_par = D.alloc<double>(kMinNPar);
    b->m_sys = D.alloc<double>(4 * (size_t)b->n_sys);
    b->m_npos = D.alloc<int32_t>(b->n_sys);
    b->m_sel = D.alloc<uint8_t>(N);
    if (!b->m_x0 || !b->m_ft || !b->m_xb || !b->m_best || !b->m_par || !b->m_sys || !b->m_npos || !b->m_sel)
      return fail(ctx, PB2_ENOMEM, "minimiser allocation failed");
  }
  // selections: heavy atoms default to mass > 1.1 amu (prolix simulate.py:596),
  // backbone to the heavy atoms
  std::vector<double> hm(N);
  CUDA_TRY(ctx, cudaMemcpy(hm.data(), b->mass, N * sizeof(double), cudaMemcpyDeviceToHost));
  std::vector<uint8_t> sel(N);
  for (size_t g = 0; g < N; ++g) {  // heavy, backbone: caller's atom order
    const int32_t u = b->user_host[g];
    const bool h = heavy ? heavy[u] != 0 : hm[g] > 1.1;
    const bool bb = backbone ? backbone[u] != 0 : h;
    sel[g] = (uint8_t)((h ? 1 : 0) | (bb ? 2 : 0));
  }
  CUDA_TRY(ctx, cudaMemcpy(b->m_sel, sel.data(), N, cudaMemcpyHostToDevice));
  CUDA_TRY(ctx, cudaMemcpy(b->m_x0, b->x, N * sizeof(double), cudaMemcpyDeviceToDevice));
  CUDA_TRY(ctx, cudaMemcpy(b->m_x0 + N, b->y, N * sizeof(double), cudaMemcpyDeviceToDevice));
  CUDA_TRY(ctx, cudaMemcpy(b->m_x0 + 2 * N, b->z, N * sizeof(double), cudaMemcpyDeviceToDevice));
  b->min_ready = true;
  return PB2_OK;
}

// mode 0: steepest descent steps; mode 1: FIRE iterations
static int min_graph(pb2_batch *b, int mode, int chunk, cudaGraphExec_t *out) {
  pb2_ctx *ctx = b->ctx;
  auto key = std::make_pair(mode, chunk);
  auto it = b->min_graphs.find(key);
  if (it != b->min_graphs.end()) {
    *out = it->second;
    return PB2_OK;
  }
  const MinArgs ma = min_args(b);
  cudaStream_t cs = b->cap_stream;
  CUDA_TRY(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  for (int t = 0; t < chunk && err == cudaSuccess; ++t) {
    if (mode == 0) {
      err = launch_min(kMinOpSd, ma, nullptr, cs);
      if (err == cudaSuccess) err = enqueue_forces(b, cs, false);
    } else {
      err = launch_min(kMinOpFireBegin, ma, nullptr, cs);
      if (err == cudaSuccess) err = launch_min(kMinOpFireDrift, ma, nullptr, cs);
      if (err == cudaSuccess) err = enqueue_forces(b, cs, false);
      if (err == cudaSuccess) err = launch_min(kMinOpFireMix, ma, nullptr, cs);
    }
  }
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(cs, &g);
  if (err != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(ctx, PB2_ECUDA, std::string("graph capture failed: ") +
                                    cudaGetErrorString(err != cudaSuccess ? err : e2));
  }
  cudaGraphExec_t ex = nullptr;
  cudaError_t e3 = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) return fail(ctx, PB2_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e3));
  b->min_graphs[key] = ex;
  *out = ex;
  return PB2_OK;
}

static int min_run(pb2_batch *b, int mode, int n, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  int done = 0;
  while (done < n) {
    const int c = std::min(b->params.graph_chunk, n - done);
    cudaGraphExec_t ex;
    int rc = min_graph(b, mode, c, &ex);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaGraphLaunch(ex, st));
    done += c;
  }
  return PB2_OK;
}

static int min_begin(pb2_batch *b, int32_t n_steps, double k, int32_t kind, cudaStream_t st) {
  pb2_ctx *ctx = b->ctx;
  if (!b->min_ready) return fail(ctx, PB2_EINVAL, "call pb2_min_setup first");
  if (n_steps < 0 || kind < 0 || kind > 2 || !(k >= 0.0)) return fail(ctx, PB2_EINVAL, "bad minimiser arguments");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  b->m_par_host[kMinK] = k;
  b->m_par_host[kMinKind] = kind;
  CUDA_TRY(ctx, cudaMemcpyAsync(b->m_par, b->m_par_host, kMinNPar * sizeof(double), cudaMemcpyHostToDevice, st));
  if (!b->forces_valid) {
    int rc = fresh_forces(b, st, false);
    if (rc) return rc;
  }
  return PB2_OK;
}

extern "C" int pb2_min_sd(pb2_batch *b, int32_t n_steps, double k, int32_t kind, double dt, double max_dx,
                          void *stream) {
  if (!b) return PB2_EINVAL;
  if (!(dt > 0.0) || !(max_dx > 0.0)) return fail(b->ctx, PB2_EINVAL, "dt and max_dx must be > 0");
  b->m_par_host[kMinSdDt] = dt;
  b->m_par_host[kMinMaxDx] = max_dx;
  b->m_par_host[kMinForceCap] = 0.0;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = min_begin(b, n_steps, k, kind, st);
  if (rc) return rc;
  if ((rc = min_run(b, 0, n_steps, st))) return rc;
  CUDA_TRY(b->ctx, launch_min(kMinOpRollback, min_args(b), nullptr, st));
  b->forces_valid = false;  // a rolled-back system moved
  if ((rc = forces_not_from_step(b, st))) return rc;
  CUDA_TRY(b->ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_min_fire(pb2_batch *b, int32_t n_steps, double k, int32_t kind, double dt_start,
                            double dt_max, double max_disp, double force_cap, int32_t flags, void *stream) {
  if (!b) return PB2_EINVAL;
  if (!(dt_start > 0.0) || !(dt_max > 0.0) || !(max_disp >= 0.0) || !(force_cap >= 0.0))
    return fail(b->ctx, PB2_EINVAL, "dt_start, dt_max must be > 0; max_disp, force_cap >= 0");
  b->m_par_host[kMinDtStart] = dt_start;
  b->m_par_host[kMinDtMax] = dt_max;
  b->m_par_host[kMinMaxDisp] = max_disp;
  b->m_par_host[kMinForceCap] = force_cap;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = min_begin(b, n_steps, k, kind, st);
  if (rc) return rc;
  const MinArgs ma = min_args(b);
  CUDA_TRY(b->ctx, launch_min(kMinOpFireInit, ma, nullptr, st));
  if ((rc = min_run(b, 1, n_steps, st))) return rc;
  if (flags & PB2_FIRE_KEEP_BEST) CUDA_TRY(b->ctx, launch_min(kMinOpTakeBest, ma, nullptr, st));
  CUDA_TRY(b->ctx, launch_min(kMinOpRollback, ma, nullptr, st));
  b->forces_valid = false;
  if ((rc = forces_not_from_step(b, st))) return rc;
  CUDA_TRY(b->ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}


static LbfgsArgs lbfgs_args(pb2_batch *b, double tol, double max_step) {
  LbfgsArgs a;
  a.m = min_args(b);
  a.energy = b->lb_energy;
  a.g = b->lb_g; a.d = b->lb_d; a.x0 = b->lb_x0;
  a.hs = b->lb_hs; a.hy = b->lb_hy; a.rho = b->lb_rho;
  a.e0 = b->lb_sys; a.gd = b->lb_sys + b->n_sys; a.t = b->lb_sys + 2 * (size_t)b->n_sys;
  a.count = b->lb_int; a.head = b->lb_int + b->n_sys; a.flags = b->lb_int + 2 * (size_t)b->n_sys;
  a.hist = b->lb_hist;
  a.tol = tol;
  a.max_step = max_step;
  return a;
}

// Forces and FP64 energies at the current positions into lb_energy.
static int lbfgs_eval(pb2_batch *b, cudaStream_t st) {
  int rc = fresh_forces(b, st, true);
  if (rc) return rc;
  CUDA_TRY(b->ctx, launch_energies_to_double(b->energy, b->lb_energy, b->n_sys, st));
  return PB2_OK;
}

extern "C" int pb2_min_lbfgs(pb2_batch *b, int32_t n_iter, double tol, double max_step, int32_t hist,
                             int32_t max_trials, int32_t *converged, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (!b->min_ready) return fail(ctx, PB2_EINVAL, "call pb2_min_setup first");
  if (n_iter < 0 || hist < 1 || hist > kLbfgsMaxHist || !(max_step > 0.0) || !(tol >= 0.0) || max_trials < 1)
    return fail(ctx, PB2_EINVAL, "bad L-BFGS arguments");
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const size_t N3 = 3 * (size_t)b->n_total, S = b->n_sys;
  if (b->lb_hist != hist) {
    Dev &D = b->mdev;
    for (void *p : {(void *)b->lb_g, (void *)b->lb_d, (void *)b->lb_x0, (void *)b->lb_hs, (void *)b->lb_hy,
                    (void *)b->lb_rho, (void *)b->lb_sys, (void *)b->lb_energy, (void *)b->lb_int})
      if (p) D.release(p);
    b->lb_g = D.alloc<double>(N3);
    b->lb_d = D.alloc<double>(N3);
    b->lb_x0 = D.alloc<double>(N3);
    b->lb_hs = D.alloc<double>(hist * N3);
    b->lb_hy = D.alloc<double>(hist * N3);
    b->lb_rho = D.alloc<double>(hist * S);
    b->lb_sys = D.alloc<double>(3 * S);
    b->lb_energy = D.alloc<double>(S * PB2_NTERMS);
    b->lb_int = D.alloc<int32_t>(3 * S);
    if (!b->lb_g || !b->lb_d || !b->lb_x0 || !b->lb_hs || !b->lb_hy || !b->lb_rho || !b->lb_sys ||
        !b->lb_energy || !b->lb_int) {
      b->lb_hist = 0;
      return fail(ctx, PB2_ENOMEM, "L-BFGS allocation failed");
    }
    b->lb_hist = hist;
  }
  const LbfgsArgs la = lbfgs_args(b, tol, max_step);
  int rc = lbfgs_eval(b, st);
  if (rc) return rc;
  CUDA_TRY(ctx, launch_lbfgs(kLbfgsOpBegin, la, 0, st));
  std::vector<int32_t> flags(S);
  for (int it = 0; it < n_iter; ++it) {
    CUDA_TRY(ctx, launch_lbfgs(kLbfgsOpDirection, la, 0, st));
    for (int trial = 0; trial < max_trials; ++trial) {
      CUDA_TRY(ctx, launch_lbfgs(kLbfgsOpTrial, la, 0, st));
      if ((rc = lbfgs_eval(b, st))) return rc;
      CUDA_TRY(ctx, launch_lbfgs(kLbfgsOpCheck, la, trial == max_trials - 1, st));
      CUDA_TRY(ctx, cudaMemcpyAsync(flags.data(), la.flags, S * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      CUDA_TRY(ctx, cudaStreamSynchronize(st));
      bool searching = false;
      for (int32_t f : flags) searching |= !(f & (kLbfgsAccepted | kLbfgsDone));
      if (!searching) break;
    }
    bool all_done = true;
    for (int32_t f : flags) all_done &= (f & kLbfgsDone) != 0;
    if (all_done) break;
  }
  if (converged)
    for (size_t s = 0; s < S; ++s) converged[s] = (flags[s] & kLbfgsDone) ? 1 : 0;
  b->forces_valid = true;  // the last evaluation is at the final positions
  if (int rc2 = forces_not_from_step(b, st)) return rc2;
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_min_rms(pb2_batch *b, double *rms, void *stream) {
  if (!b || !rms) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (!b->min_ready) return fail(ctx, PB2_EINVAL, "call pb2_min_setup first");
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (!b->forces_valid) {
    int rc = fresh_forces(b, st, false);
    if (rc) return rc;
  }
  double *out = b->m_sys + 3 * (size_t)b->n_sys;
  CUDA_TRY(ctx, launch_min(kMinOpRms, min_args(b), out, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(rms, out, b->n_sys * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}


// Exchange the dynamical state of whole systems: slot s takes x, p and F of
// slot perm[s].  Keys, step counters and per-system constants (kT, dt)
// stay with their slots.  The systems swapped must have the same atom count.
extern "C" int pb2_permute_systems(pb2_batch *b, const int32_t *perm, void *stream) {
  if (!b || !perm) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<char> seen(b->n_sys, 0);
  for (int s = 0; s < b->n_sys; ++s) {
    const int t = perm[s];
    if (t < 0 || t >= b->n_sys || seen[t]) return fail(ctx, PB2_EINVAL, "perm is not a permutation");
    seen[t] = 1;
    if (b->nat[t] != b->nat[s]) return fail(ctx, PB2_EINVAL, "permuted systems differ in atom count");
  }
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (!b->d_perm) {
    b->d_perm = b->dev.alloc<int32_t>(b->n_sys);
    if (!b->d_perm) return fail(ctx, PB2_ENOMEM, "permutation buffer allocation failed");
  }
  CUDA_TRY(ctx, cudaMemcpyAsync(b->d_perm, perm, b->n_sys * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  const size_t N = b->n_total;
  void *groups[3][3] = {{b->x, b->y, b->z}, {b->px, b->py, b->pz}, {b->fx, b->fy, b->fz}};
  for (auto &g : groups) {
    for (int c = 0; c < 3; ++c)
      CUDA_TRY(ctx, launch_gather_systems(b->sys, b->atom_sys, b->d_perm, b->user, b->devidx, g[c], b->stage + c * N,
                                            b->n_total, st));
    for (int c = 0; c < 3; ++c)
      CUDA_TRY(ctx, cudaMemcpyAsync(g[c], b->stage + c * N, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  CUDA_TRY(ctx, launch_posq(int_args(b, b->key_parity, 0), st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}


// ------------------------------------------------------------ trajectories

extern "C" int pb2_traj_setup(pb2_batch *b, int32_t capacity) {
  if (!b || capacity <= 0) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const size_t f = 3 * (size_t)b->n_total;
  if (capacity != b->traj_cap) {
    if (b->traj_pos) {
      b->tdev.release(b->traj_pos);
      b->tdev.release(b->traj_vel);
      b->tdev.release(b->traj_steps);
    }
    b->traj_pos = b->tdev.alloc<float>((size_t)capacity * f);
    b->traj_vel = b->tdev.alloc<float>((size_t)capacity * f);
    b->traj_steps = b->tdev.alloc<long long>((size_t)capacity * b->n_sys);
    if (!b->traj_pos || !b->traj_vel || !b->traj_steps) {
      b->traj_cap = 0;
      return fail(ctx, PB2_ENOMEM, "trajectory ring allocation failed");
    }
    b->traj_cap = capacity;
  }
  return PB2_OK;
}

extern "C" int pb2_traj_snapshot(pb2_batch *b, int32_t slot, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (slot < 0 || slot >= b->traj_cap) return fail(ctx, PB2_EINVAL, "trajectory slot out of range");
  const size_t f = 3 * (size_t)b->n_total;
  CUDA_TRY(ctx, launch_snapshot(b->x, b->y, b->z, b->px, b->py, b->pz, b->mass, b->steps, b->user,
                                b->traj_pos + slot * f, b->traj_vel + slot * f,
                                b->traj_steps + (size_t)slot * b->n_sys, b->n_total, b->n_sys,
                                (cudaStream_t)stream));
  return PB2_OK;
}

extern "C" int pb2_traj_fetch(pb2_batch *b, int32_t first, int32_t count, float *positions, float *velocities,
                              int64_t *steps, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (first < 0 || count < 0 || first + count > b->traj_cap)
    return fail(ctx, PB2_EINVAL, "trajectory slots out of range");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t f = 3 * (size_t)b->n_total;
  if (positions)
    CUDA_TRY(ctx, cudaMemcpyAsync(positions, b->traj_pos + first * f, count * f * sizeof(float),
                                  cudaMemcpyDeviceToHost, st));
  if (velocities)
    CUDA_TRY(ctx, cudaMemcpyAsync(velocities, b->traj_vel + first * f, count * f * sizeof(float),
                                  cudaMemcpyDeviceToHost, st));
  if (steps)
    CUDA_TRY(ctx, cudaMemcpyAsync(steps, b->traj_steps + (size_t)first * b->n_sys,
                                  (size_t)count * b->n_sys * sizeof(long long), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_get_status(pb2_batch *b, uint32_t *status, int clear, void *stream) {
  if (!b || !status) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(ctx, cudaMemcpyAsync(status, b->status, b->n_sys * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (clear) CUDA_TRY(ctx, cudaMemsetAsync(b->status, 0, b->n_sys * sizeof(uint32_t), st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return PB2_OK;
}

extern "C" int pb2_set_safeguards(pb2_batch *b, double vlimit, double max_dx, double force_cap) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (!std::isfinite(vlimit) || !std::isfinite(max_dx) || !std::isfinite(force_cap))
    return fail(ctx, PB2_EINVAL, "safeguard limits must be finite");
  const double g[3] = {vlimit > 0.0 ? vlimit : 0.0, max_dx > 0.0 ? max_dx : 0.0,
                       force_cap > 0.0 ? force_cap : 0.0};
  if (g[0] == b->guard[0] && g[1] == b->guard[1] && g[2] == b->guard[2]) return PB2_OK;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  for (int k = 0; k < 3; ++k) b->guard[k] = g[k];
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);  // they captured the old limits
  b->graphs.clear();
  return PB2_OK;
}

extern "C" int pb2_get_safeguards(const pb2_batch *b, double *vlimit, double *max_dx, double *force_cap) {
  if (!b) return PB2_EINVAL;
  if (vlimit) *vlimit = b->guard[0];
  if (max_dx) *max_dx = b->guard[1];
  if (force_cap) *force_cap = b->guard[2];
  return PB2_OK;
}

extern "C" int pb2_get_warn_counts(pb2_batch *b, int32_t *counts, int reset, void *stream) {
  if (!b || !counts) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t S = (size_t)b->n_sys;
  std::vector<uint32_t> flags(2 * S);
  CUDA_TRY(ctx, cudaMemcpyAsync(counts, b->warn_counts, S * kWarnTypes * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(flags.data(), b->warn_flags, 2 * S * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  if (reset) {
    CUDA_TRY(ctx, cudaMemsetAsync(b->warn_counts, 0, S * kWarnTypes * sizeof(int32_t), st));
    CUDA_TRY(ctx, cudaMemsetAsync(b->warn_flags, 0, 2 * S * sizeof(uint32_t), st));
  }
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  // caps recorded by the last launch and not yet folded into the counts
  for (size_t h = 0; h < 2; ++h)
    for (size_t s = 0; s < S; ++s)
      for (int k = 0; k < kWarnTypes; ++k)
        if (flags[h * S + s] & (1u << k)) counts[s * kWarnTypes + k] += 1;
  return PB2_OK;
}

extern "C" int pb2_set_tile_segment(pb2_batch *b, int32_t segment) {
  if (!b || segment <= 0) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (segment == b->params.tile_segment) return PB2_OK;
  std::vector<TileItem> items = build_items(b->sys_host, segment);
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  b->dev.release(b->items);
  b->items = b->dev.alloc<TileItem>(items.size());
  if (!b->items) return fail(ctx, PB2_ENOMEM, "work-item allocation failed");
  CUDA_TRY(ctx, cudaMemcpy(b->items, items.data(), items.size() * sizeof(TileItem), cudaMemcpyHostToDevice));
  b->n_items = (int)items.size();
  b->params.tile_segment = segment;
  if (int rc = setup_items2(b, segment)) return rc;
  if (int rc = setup_pair_list(b, segment)) return rc;
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);  // they captured the old list
  b->graphs.clear();
  for (auto &kv : b->min_graphs) cudaGraphExecDestroy(kv.second);
  b->min_graphs.clear();
  return PB2_OK;
}

extern "C" int pb2_retire_system(pb2_batch *b, int32_t sys, void *stream) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (sys < 0 || sys >= b->n_sys) return fail(ctx, PB2_EINVAL, "system index out of range");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (b->retired_host[sys]) return PB2_OK;
  b->retired_host[sys] = 1;
  CUDA_TRY(ctx, launch_retire(sys, b->retired, b->items2_all, b->n_items2, b->items2, b->item_count,
                              b->pl_on ? b->pl_ctl : nullptr, (cudaStream_t)stream));
  CUDA_TRY(ctx, launch_retire(-1, b->retired, b->items4_all, b->n_items4, b->items4, b->item_count4, nullptr,
                              (cudaStream_t)stream));
  return PB2_OK;
}

extern "C" int pb2_test_hold_system(pb2_batch *b, int32_t sys, int32_t hold) {
  if (!b) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  if (sys < 0 || sys >= b->n_sys || hold < 0) return fail(ctx, PB2_EINVAL, "bad system or hold");
  if (b->pl_on) return fail(ctx, PB2_EINVAL, "the pair list writes its own item counts");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  const int32_t v = b->sys_items_host[sys] + hold;
  CUDA_TRY(ctx, cudaMemcpy(b->sys_items + sys, &v, sizeof v, cudaMemcpyHostToDevice));
  return PB2_OK;
}

extern "C" int pb2_get_tile_segment(const pb2_batch *b, int32_t *segment) {
  if (!b || !segment) return PB2_EINVAL;
  *segment = b->params.tile_segment;
  return PB2_OK;
}

static void any_shape(int pass, int k, int *t, int *m) {
  if (pass == 3) force4_shape(k, t, m);
  else tile_shape(pass, k, t, m);
}

extern "C" int pb2_block_shapes(int32_t pass, int32_t *threads, int32_t *min_blocks, int32_t capacity) {
  if (pass < 0 || pass > 3) return PB2_EINVAL;
  for (int k = 0; k < kShapesPerPass && k < capacity; ++k) {
    int t = 0, m = 0;
    any_shape(pass, k, &t, &m);
    if (threads) threads[k] = t;
    if (min_blocks) min_blocks[k] = m;
  }
  return kShapesPerPass;
}

extern "C" int pb2_set_block_shape(pb2_batch *b, int32_t pass, int32_t threads, int32_t min_blocks) {
  if (!b || pass < 0 || pass > 3) return PB2_EINVAL;
  pb2_ctx *ctx = b->ctx;
  int found = -1;
  for (int k = 0; k < kShapesPerPass; ++k) {
    int t = 0, m = 0;
    any_shape(pass, k, &t, &m);
    if (t == threads && m == min_blocks) found = k;
  }
  if (found < 0) return fail(ctx, PB2_EINVAL, "block shape not compiled for this pass (see pb2_block_shapes)");
  if (found == (pass == 3 ? b->shape4 : b->shape[pass])) return PB2_OK;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  if (pass == 3) {
    b->shape4 = found;
    set_force4_grid(b);
  } else {
    b->shape[pass] = found;
    set_pair_grid(b, pass);
  }
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);  // they captured the old kernel
  b->graphs.clear();
  for (auto &kv : b->min_graphs) cudaGraphExecDestroy(kv.second);
  b->min_graphs.clear();
  return PB2_OK;
}

extern "C" int pb2_get_block_shape(const pb2_batch *b, int32_t pass, int32_t *threads, int32_t *min_blocks) {
  if (!b || pass < 0 || pass > 3 || !threads || !min_blocks) return PB2_EINVAL;
  int t = 0, m = 0;
  any_shape(pass, pass == 3 ? b->shape4 : b->shape[pass], &t, &m);
  *threads = t;
  *min_blocks = m;
  return PB2_OK;
}

extern "C" int pb2_set_force_blocks(pb2_batch *b, int32_t blocks) {
  if (!b || (blocks != 2 && blocks != 4)) return PB2_EINVAL;
  if (blocks == b->force_blocks) return PB2_OK;
  CUDA_TRY(b->ctx, cudaSetDevice(b->ctx->device));
  CUDA_TRY(b->ctx, cudaDeviceSynchronize());
  b->force_blocks = blocks;
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);  // they captured the other kernel
  b->graphs.clear();
  for (auto &kv : b->min_graphs) cudaGraphExecDestroy(kv.second);
  b->min_graphs.clear();
  return PB2_OK;
}

extern "C" int pb2_get_force_blocks(const pb2_batch *b, int32_t *blocks) {
  if (!b || !blocks) return PB2_EINVAL;
  *blocks = b->force_blocks;
  return PB2_OK;
}

extern "C" int pb2_set_fusion(pb2_batch *b, int32_t flags) {
  if (!b || (flags & ~(PB2_FUSE_BONDED | PB2_FUSE_FINALIZE))) return PB2_EINVAL;
  if (flags == b->fuse) return PB2_OK;
  CUDA_TRY(b->ctx, cudaSetDevice(b->ctx->device));
  CUDA_TRY(b->ctx, cudaDeviceSynchronize());
  b->fuse = flags;
  for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);  // they captured the old schedule
  b->graphs.clear();
  for (auto &kv : b->min_graphs) cudaGraphExecDestroy(kv.second);
  b->min_graphs.clear();
  return PB2_OK;
}

extern "C" int pb2_get_fusion(const pb2_batch *b, int32_t *flags) {
  if (!b || !flags) return PB2_EINVAL;
  *flags = b->fuse;
  return PB2_OK;
}

extern "C" int pb2_set_profiling(pb2_batch *b, int enable) {
  if (!b) return PB2_EINVAL;
  b->profiling = enable != 0;
  return PB2_OK;
}

extern "C" int pb2_last_timings(pb2_batch *b, double *out_ms) {
  if (!b || !out_ms) return PB2_EINVAL;
  for (int k = 0; k < kTimSlots; ++k) out_ms[k] = b->timings[k];
  return PB2_OK;
}

// Neighbour-list entry points: the list is built in pb2_nlist.cu.
