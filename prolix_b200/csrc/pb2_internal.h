// Host-side definitions shared by the C ABI translation units: the context
// and batch records and the error helpers.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "pb2_common.cuh"
#include "pb2_kernels.cuh"

using namespace pb2;


struct pb2_ctx {
  int device = 0;
  int sm_count = 148;
  std::string err;
};

// slots of pb2_last_timings
constexpr int kTimBorn = 0, kTimFinalize = 1, kTimForce = 2, kTimChain = 3, kTimBonded = 4,
              kTimStep = 5, kTimBbox = 6, kTimAll = 7, kTimSlots = 8;

// Device allocations owned by a batch, freed with it.
// Device allocations of one batch.  They come from the device's stream-ordered
// memory pool (which pb2_ctx_create sets to keep freed memory), so building
// and dropping batches -- what a serving loop does all the time -- reuses
// memory instead of calling the driver's allocator and its implicit device
// synchronisation.  Allocation completes before alloc() returns; frees are
// ordered on the default stream after the owner has synchronised the device.
struct Dev {
  std::vector<void *> ptrs;
  ~Dev() {
    for (void *p : ptrs)
      if (p) cudaFreeAsync(p, 0);
  }
  template <class T>
  T *alloc(size_t n) {
    void *p = nullptr;
    if (n == 0) n = 1;
    if (cudaMallocAsync(&p, n * sizeof(T), 0) != cudaSuccess) return nullptr;
    if (cudaStreamSynchronize(0) != cudaSuccess) {
      cudaFreeAsync(p, 0);
      return nullptr;
    }
    ptrs.push_back(p);
    return static_cast<T *>(p);
  }
  void release(void *p) {  // rare (rebuilds): wait for every user of p first
    for (auto &q : ptrs)
      if (q == p) {
        cudaDeviceSynchronize();
        cudaFreeAsync(q, 0);
        q = nullptr;
      }
  }
};

struct pb2_batch {
  pb2_ctx *ctx = nullptr;
  pb2_run_params params{};
  int n_sys = 0;
  int n_total = 0;
  std::vector<int> off, nat;
  std::vector<SysInfo> sys_host;
  Dev dev;
  SysInfo *sys = nullptr;
  int32_t *atom_sys = nullptr;
  double *x = nullptr, *y = nullptr, *z = nullptr, *px = nullptr, *py = nullptr, *pz = nullptr;
  long long *fx = nullptr, *fy = nullptr, *fz = nullptr;
  double *mass = nullptr, *sigma = nullptr, *charge = nullptr, *radius = nullptr;
  float4 *posq = nullptr, *par = nullptr, *born = nullptr, *bbox = nullptr;
  int32_t *blk_sys = nullptr;
  int32_t *sched = nullptr;  // per pass: (next item, finished warps)
  int n_blocks = 0;
  double *q64 = nullptr, *hs64 = nullptr, *se64 = nullptr, *ro64 = nullptr, *sr64 = nullptr;
  double *born64 = nullptr;
  double *stage = nullptr;  // 3 x (n_total, 3) row-major staging for host transfers
  // atom order: the batch stores atom g where the caller's arrays hold atom
  // user[g] (both batch-wide indices; systems keep their ranges)
  int32_t *user = nullptr, *devidx = nullptr;  // device copies: g -> user, user -> g
  std::vector<int32_t> user_host, dev_host;
  int32_t *d_perm = nullptr;  // system permutation (replica exchange)
  // trajectory ring: capacity frames of float32 (n, 3) positions and
  // velocities, and the step counters of every system
  Dev tdev;
  int traj_cap = 0;
  float *traj_pos = nullptr, *traj_vel = nullptr;
  long long *traj_steps = nullptr;
  long long *born_acc = nullptr, *dedb_acc = nullptr, *energy = nullptr;
  uint32_t *keys = nullptr, *status = nullptr;
  uint32_t *key_splits = nullptr;  // (2, n_sys, 4): split of each key buffer entry
  long long *steps = nullptr;
  // safeguards of the batched Langevin step (vlimit, max_dx, force_cap; <= 0
  // off), the closing-force flag and the per-system cap counters
  double guard[3] = {0.0, 0.0, 0.0};
  std::vector<double> gamma_host;  // per-system friction (1/tau); c1, c2 derive from it
  int32_t *guard_end = nullptr;
  uint32_t *warn_flags = nullptr;
  int32_t *warn_counts = nullptr;
  TileItem *items = nullptr;   // (i-block, j-range) items of the FP64 energy kernels
  int n_items = 0;
  TileItem *items2 = nullptr;  // pair kernels: the live items (those of systems not retired)
  TileItem *items2_all = nullptr;  // every system's items over pairs of i-blocks
  int n_items2 = 0;                // items in items2_all
  int32_t *item_count = nullptr;   // items in items2 (device)
  // the four-block force kernel's items (i-blocks ib % 4 == 0): all, live, counts
  TileItem *items4_all = nullptr, *items4 = nullptr;
  int n_items4 = 0;
  int32_t *item_count4 = nullptr;
  int force_blocks = 2;  // i-blocks per warp of the force pass (2 or 4; 4 only without a pair list)
  int shape4 = 0, grid4 = 1;
  int8_t *retired = nullptr;       // per system: 1 = retired (pb2_retire_system)
  std::vector<int8_t> retired_host;
  int32_t *sys_items = nullptr;  // items2 per system (the descreening pass's completion count)
  std::vector<int32_t> sys_items_host;
  int32_t *sys_done = nullptr;   // items of each system completed in the current pass
  int4 *blk_info = nullptr;      // per 32-atom block: system, first atom, atoms
  int32_t *sys_fin = nullptr;    // finalize chunks of each system completed in the current pass
  int2 *excl_ent = nullptr;
  ExclRow *excl_rows = nullptr;
  BondedArgs bonded{};
  int key_parity = 0;
  bool forces_valid = false;
  bool cut = false;  // any cutoff active  // force accumulators hold F(x) of the current state
  int grid_pair[3] = {1, 1, 1};
  int shape[3] = {0, 0, 0};  // block shape of each pair pass (index into the compiled shapes)
  int fuse = PB2_FUSE_BONDED;  // PB2_FUSE_* bits: work folded into the pair passes
  int grid_bonded = 1;
  cudaStream_t cap_stream = nullptr;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  bool profiling = false;
  double timings[kTimSlots] = {0, 0, 0, 0, 0, 0, 0, 0};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  // host round trips on separate copy streams: copies in done, steps done,
  // copies out done
  cudaEvent_t ev_io[3] = {nullptr, nullptr, nullptr};
  // minimiser state (allocated by pb2_min_setup)
  Dev mdev;
  bool min_ready = false;
  double *m_x0 = nullptr, *m_ft = nullptr, *m_xb = nullptr, *m_best = nullptr, *m_par = nullptr;
  double *m_sys = nullptr;  // dt, alpha, best rms, rms: (4, n_sys)
  int32_t *m_npos = nullptr;
  uint8_t *m_sel = nullptr;
  std::map<std::pair<int, int>, cudaGraphExec_t> min_graphs;  // (mode, chunk)
  // L-BFGS polish state (allocated on first use)
  int lb_hist = 0;
  double *lb_g = nullptr, *lb_d = nullptr, *lb_x0 = nullptr, *lb_hs = nullptr, *lb_hy = nullptr;
  double *lb_rho = nullptr, *lb_sys = nullptr, *lb_energy = nullptr;  // lb_sys: e0, gd, t
  int32_t *lb_int = nullptr;  // count, head, flags
  double m_par_host[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // kMinNPar stage parameters
  // pair list of the cutoff runs (pb2_pairlist.cu): rows, j-block lists,
  // two item buffers and the control words; on when every pair term of the
  // batch has a cutoff
  bool pl_on = false;
  float pl_reach2 = 0.f;
  PlRow *pl_rows = nullptr;
  int n_pl_rows = 0;
  int32_t *pl_jlist = nullptr;
  TileItem *pl_items[2] = {nullptr, nullptr};
  int32_t *pl_sys_items[2] = {nullptr, nullptr};
  size_t pl_item_cap = 0;
  int32_t *pl_ctl = nullptr;
  float4 *pl_ref = nullptr;
  int grid_pl = 1;
  // neighbour list (allocated on first build)
  Dev nl;
  bool nl_built = false;
  int nl_capacity = 0;
  int *nl_rows = nullptr, *nl_counts = nullptr;
  int32_t *nl_sys_moved = nullptr, *nl_ctl = nullptr;
  double *nl_xref = nullptr;
  cudaEvent_t nl_ev[2] = {nullptr, nullptr};  // around the last build's launches
  bool nl_timed = false;

  ~pb2_batch() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    for (auto &kv : min_graphs) cudaGraphExecDestroy(kv.second);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
    for (auto &e : ev_io)
      if (e) cudaEventDestroy(e);
    for (auto &e : nl_ev)
      if (e) cudaEventDestroy(e);
  }
};

static inline int fail(pb2_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return code;
}


IntArgs int_args_for_nl(pb2_batch *b);

#define CUDA_TRY(ctx, expr)                                                                  \
  do {                                                                                       \
    cudaError_t e_ = (expr);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail((ctx), PB2_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));     \
  } while (0)

