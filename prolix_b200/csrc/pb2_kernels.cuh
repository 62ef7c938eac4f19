// Argument records and launchers of the device kernels (shared by the
// kernel translation units and the C ABI).
#pragma once

#include "pb2_common.cuh"

namespace pb2 {

// Record a message as the context's last error (ctx may be NULL); returns code.
int set_error(pb2_ctx *ctx, int code, const char *msg);

// torsion-list entry kinds (BondedArgs::tors_par .w)
constexpr double kTorsProper = 0.0, kTorsImproper = 1.0, kTorsHarmonic = 2.0;
struct BondedArgs {
  const int32_t *atom_sys;
  const double *x, *y, *z;
  long long *fx, *fy, *fz;
  long long *energy;
  int32_t energy_mode;
  uint32_t terms;
  int32_t n_bond;        // bonds [0, n_bond_plain), then Urey-Bradley springs
  int32_t n_bond_plain;
  const int2 *bond_idx;
  const double2 *bond_par;
  int32_t n_angle;
  const int4 *angle_idx;
  const double2 *angle_par;
  int32_t n_tors;
  const int4 *tors_idx;
  const double4 *tors_par;  // .w: kTorsProper (n, phase, k), kTorsImproper (n, phase, k),
                            // kTorsHarmonic (k, phi0)
  int32_t n_cmap;
  const int32_t *cmap_idx;
  const double *cmap_coeff;
  const int32_t *cmap_grid;
  const int64_t *cmap_map_off;
  int32_t n_exc;
  const int2 *exc_idx;
  const double4 *exc_par;  // (k_coulomb * charge product, sigma, epsilon, 0)
};
enum { PASS_BORN = 0, PASS_FORCE = 1, PASS_CHAIN = 2 };
struct FinalizeArgs {
  const SysInfo *sys;
  const int32_t *atom_sys;
  const double *radius;
  const double *charge;
  long long *born_acc;
  float4 *born;
  long long *dedb_acc;
  long long *energy;
  double *born64;   // NULL, or FP64 Born radii out
  int32_t n_total;
  int32_t energy_mode;
  // finalize as the descreening pass's tail chunks (one per 32-atom block)
  const int32_t *blk_sys;
  int32_t n_blocks;
  int32_t *sys_fin;        // per system: chunks finished in this launch
  const int8_t *retired;   // per system: retired systems are skipped
  uint32_t *status;
};
struct PairArgs {
  const SysInfo *sys;
  const TileItem *items;
  int32_t n_items;
  const int32_t *item_count;  // non-NULL: the item count, in device memory (overrides n_items)
  uint32_t terms;
  const int2 *excl_ent;
  const ExclRow *excl_rows;
  const float4 *posq;
  const float4 *par;
  const float4 *born;
  const float4 *bbox;       // per global block: (lo, hi) of the float32 positions
  long long *born_acc;
  long long *dedb_acc;
  long long *fx, *fy, *fz;
  long long *energy;
  int32_t cut;              // any cutoff active
  int32_t *sched;           // (next item, finished warps) of this pass; zero between launches
  // pair list (cutoff runs; NULL otherwise): items come from pl_items[pl_ctl[1]],
  // pl_ctl[2 + pl_ctl[1]] of them, and an item's tiles t in [jb0, jb1) are
  // the j-blocks pl_jlist[t]
  const int32_t *pl_ctl;
  const TileItem *pl_items0, *pl_items1;
  const int32_t *pl_jlist;
  // chain pass: after its tiles, the warps take the bonded terms in chunks
  // of kBondedChunk (0 chunks: the bonded kernel runs on its own)
  BondedArgs bonded;
  int32_t n_bonded_chunks;
  // descreening pass: with sys_items set, the warps count each system's
  // completed items in sys_done, and after the items come fin.n_blocks
  // finalize chunks, each waiting until its system's count reaches
  // sys_items[s]; the system's last chunk resets both counters
  const int32_t *sys_items;
  int32_t *sys_done;
  FinalizeArgs fin;
  const int32_t *pl_sys_items0, *pl_sys_items1;  // per-system item counts of the pair list's buffers
};
constexpr int kBondedChunk = 32;  // one term per lane: small systems get no long FP64 tail
// Pair-list control words (PlArgs::ctl)
enum { PL_DIRTY = 0, PL_CUR = 1, PL_COUNT0 = 2, PL_COUNT1 = 3, PL_NEW = 4, PL_DONE = 5, PL_WORDS = 8 };
struct PlArgs {
  const SysInfo *sys;
  const PlRow *rows;
  int32_t n_rows;
  const float4 *bbox;
  const float4 *posq;
  float4 *ref;           // positions at the last build (displacement reference)
  int32_t *jlist;
  TileItem *items0, *items1;
  int32_t *sys_items0, *sys_items1;  // per-system item counts of each buffer
  int32_t n_sys;
  int32_t *ctl;
  float reach2;          // (largest pair-term cutoff + skin)^2
  int32_t seg;           // tiles per work item
  const int8_t *retired; // per system: 1 = retired (its rows list nothing)
};

struct Energy64Args {
  const SysInfo *sys;
  const TileItem *items;
  int32_t n_items;
  uint32_t terms;
  const int2 *excl_ent;
  const ExclRow *excl_rows;
  const double *x, *y, *z;
  const double *q, *hs, *se, *ro, *sr;  // charge, sigma/2, sqrt(eps), rho~, scaled radius
  const double *born64;
  long long *born_acc;
  long long *energy;
};

// Neighbour-list control words (NlArgs::ctl)
enum { NL_DIRTY = 0, NL_MAXCOUNT = 1, NL_DONE = 2, NL_NEXT = 3, NL_WORDS = 4 };
struct NlArgs {
  const SysInfo *sys;
  const int32_t *atom_sys;
  const int32_t *blk_sys;      // per global 32-atom block: its system
  const float4 *bbox;          // current block boxes
  const float4 *posq;
  const double *x, *y, *z;
  double *xref;                // positions at the last build, SoA (3, n_total)
  int *rows, *counts;
  int32_t *sys_moved;          // per system: moved more than skin / 2 (the last check)
  int32_t *ctl;                // NL_* words; the build kernels run only while ctl[NL_DIRTY] != 0
  int32_t capacity, n_total, n_blocks, n_sys;
  uint32_t *status;
  float reach2;                // (cutoff + skin)^2
};
// The build (every kernel returns at once unless ctl[NL_DIRTY] is set; the
// last one clears it) and the half-skin test that sets it.
cudaError_t nl_launch_build(const NlArgs &a, cudaStream_t st);
cudaError_t nl_launch_disp(const NlArgs &a, cudaStream_t st);
struct IntArgs {
  const SysInfo *sys;
  const int32_t *atom_sys;
  const int32_t *user;  // batch atom -> the caller's batch-wide index (noise streams follow it)
  double *x, *y, *z;
  double *px, *py, *pz;
  long long *fx, *fy, *fz;
  const double *mass;
  const double *sigma;
  const double *charge;
  float4 *posq;
  uint32_t *keys;
  // (2, n_sys, 4): for the key in keys[parity][s], its split (next key,
  // subkey), kept ahead by the thread of each system's first atom, so that
  // a step's atoms read their subkey instead of each deriving it
  uint32_t *splits;
  long long *steps;
  uint32_t *status;
  int32_t n_total;
  int32_t n_sys;
  int32_t parity;
  int32_t finish_prev;
  int32_t partitionable;
  // Safeguards of prolix's batched Langevin step (batched_simulate.py:263-356);
  // each <= 0 is off, all off is the plain BAOAB step.
  double vlimit;     // |p/m| limit after the opening half kick
  double max_dx;     // per-step displacement limit (A)
  double force_cap;  // |F| limit of a step's closing force
  int32_t *guard_end;     // 1: the force accumulators hold a step's closing force
  uint32_t *warn_flags;   // (2, n_sys) caps that fired, by key parity; kWarnBit*
  int32_t *warn_counts;   // (n_sys, 4) in prolix's warn order (typing.py:559-563)
  // the step kernels also write the block bounding boxes of the new
  // positions (one warp per 32-atom block) and, with a pair list, raise its
  // rebuild flag when an atom moved more than skin/2 from pl_ref
  const int32_t *blk_sys;
  float4 *bbox;
  int32_t n_blocks;
  const float4 *pl_ref;
  int32_t *pl_ctl;
  const int8_t *retired;  // per system: 1 = retired, never stepped again
  const int4 *blk_info;   // per 32-atom block: system, first atom, atoms (the plain step)
};
// warn_counts columns (prolix typing.py:559-563) and their warn_flags bits
enum { kWarnVlimit = 0, kWarnForceCap = 1, kWarnConstr = 2, kWarnDxCap = 3, kWarnTypes = 4 };
// Minimiser (pb2_minimize.cu).  Stage parameters live in device memory
// (par[kMin*]) so that captured graphs serve every stage.
enum { kMinK = 0, kMinKind, kMinSdDt, kMinMaxDx, kMinDtStart, kMinDtMax, kMinMaxDisp, kMinForceCap, kMinNPar };
enum { kMinOpSd = 0, kMinOpRollback, kMinOpFireInit, kMinOpFireBegin, kMinOpFireDrift, kMinOpFireMix,
       kMinOpTakeBest, kMinOpRms };
// FIRE constants (Bitzek et al. 2006; jax_md fire_descent defaults)
constexpr int kFireNmin = 5;
constexpr double kFireFinc = 1.1, kFireFdec = 0.5, kFireAlphaStart = 0.1, kFireFalpha = 0.99;
struct MinArgs {
  const SysInfo *sys;
  const int32_t *atom_sys;
  double *x, *y, *z, *px, *py, *pz;
  long long *fx, *fy, *fz;
  const double *mass, *charge;
  float4 *posq;
  const double *x0;    // restraint reference, (3, n_total)
  const uint8_t *sel;  // bit 0: heavy atom, bit 1: backbone atom
  double *ft, *xb, *best;  // state force, positions before the step, best positions: (3, n_total)
  double *sys_dt, *sys_alpha, *sys_best;
  int32_t *sys_npos;
  uint32_t *status;
  const double *par;
  int32_t n_total, n_sys;
};
cudaError_t launch_min(int op, const MinArgs &a, double *out, cudaStream_t st);
// L-BFGS polish (pb2_minimize.cu)
constexpr int kLbfgsMaxHist = 16;
enum { kLbfgsAccepted = 1, kLbfgsDone = 2 };
enum { kLbfgsOpBegin = 0, kLbfgsOpDirection, kLbfgsOpTrial, kLbfgsOpCheck };
struct LbfgsArgs {
  MinArgs m;
  const double *energy;  // (n_sys, PB2_NTERMS) FP64 energies of the current positions
  double *g, *d, *x0;    // gradient, direction, base positions: (3, n_total)
  double *hs, *hy;       // history: (hist, 3, n_total)
  double *rho;           // (hist, n_sys)
  double *e0, *gd, *t;   // per system
  int32_t *count, *head, *flags;
  int32_t hist;
  double tol, max_step;
};
cudaError_t launch_lbfgs(int op, const LbfgsArgs &a, int last_trial, cudaStream_t st);
// Block shapes of the pair kernels: kShapesPerPass compiled per pass;
// tile_shape gives (threads, min blocks per SM) of one (-1: no such shape).
constexpr int kShapesPerPass = 3;
int tile_shape(int pass, int shape, int *threads, int *min_blocks);
cudaError_t launch_tiles(int pass, const PairArgs &a, int grid, int shape, cudaStream_t st);
cudaError_t launch_energy64(int pass, const Energy64Args &a, int grid, cudaStream_t st);
cudaError_t launch_born_finalize(const FinalizeArgs &a, cudaStream_t st);
int tile_kernel_occupancy(int pass, bool cut, int shape);
int tile_kernel_warps(int pass, int shape);  // warps per block of a pair pass
// Bounding boxes of every 32-atom block.  With pl_ref / pl_ctl set, also
// flags the pair list for a rebuild (pl_ctl[PL_DIRTY]) when an atom moved
// more than half the skin since the list was built.
cudaError_t launch_bbox(const SysInfo *sys, const int32_t *blk_sys, const float4 *posq, float4 *bbox,
                        int n_blocks, cudaStream_t st, const float4 *pl_ref = nullptr,
                        int32_t *pl_ctl = nullptr);
// Rebuild the pair list when flagged (one launch; returns at once when clean).
cudaError_t launch_pl_update(const PlArgs &a, int grid, cudaStream_t st);
// The live work list: items of all[0, n_all) whose system is not retired,
// in their order, into live and *count (one thread block).  With sys >= 0,
// that system is retired first (and a pair list, if any, is marked for a
// rebuild without it).
// The force pass with four i-blocks per warp (items with iblk % 4 == 0);
// the same sums as launch_tiles(PASS_FORCE) bit for bit.
cudaError_t launch_force4(const PairArgs &a, int grid, int shape, cudaStream_t st);
int force4_occupancy(bool cut, int shape);
int force4_shape(int shape, int *threads, int *min_blocks);
cudaError_t launch_retire(int32_t sys, int8_t *retired, const TileItem *all, int n_all, TileItem *live,
                          int32_t *count, int32_t *pl_ctl, cudaStream_t st);
cudaError_t launch_bonded(const BondedArgs &a, int grid_cap, cudaStream_t st);
cudaError_t launch_step(const IntArgs &a, cudaStream_t st);
// The plain step kernel's grid for this device, queried once outside any capture.
void warm_step_launch(int n_blocks);
// Refresh splits[parity] from keys[parity] (after keys came from the host).
cudaError_t launch_key_splits(const IntArgs &a, cudaStream_t st);
cudaError_t launch_finish(const IntArgs &a, cudaStream_t st);
cudaError_t launch_center(const IntArgs &a, cudaStream_t st);
cudaError_t launch_noise_scale(const SysInfo *sys, const int32_t *atom_sys, const double *mass,
                               double *sigma, int n, cudaStream_t st);
cudaError_t launch_init(const IntArgs &a, cudaStream_t st);
cudaError_t launch_posq(const IntArgs &a, cudaStream_t st);
// Host transfers: `user` maps each batch atom to its row in the caller's
// (n, 3) arrays.
cudaError_t launch_rows_to_soa(const double *rows, const int32_t *user, double *x, double *y, double *z, int n,
                               cudaStream_t st);
cudaError_t launch_soa_to_rows(const double *x, const double *y, const double *z, const int32_t *user,
                               double *rows, int n, cudaStream_t st);
cudaError_t launch_fix_to_rows(const long long *fx, const long long *fy, const long long *fz, const int32_t *user,
                               double *rows, int n, cudaStream_t st);
cudaError_t launch_rows_to_fix(const double *rows, const int32_t *user, long long *fx, long long *fy,
                               long long *fz, int n, cudaStream_t st);
cudaError_t launch_state_from_rows(const double *rows, const int32_t *user, double *x, double *y, double *z,
                                   double *px, double *py, double *pz, long long *fx, long long *fy,
                                   long long *fz, int n, cudaStream_t st);
cudaError_t launch_state_to_rows(const double *x, const double *y, const double *z, const double *px,
                                 const double *py, const double *pz, const long long *fx, const long long *fy,
                                 const long long *fz, const int32_t *user, double *rows, int n, cudaStream_t st);
cudaError_t launch_energies_to_double(const long long *e, double *out, int n_sys, cudaStream_t st);
cudaError_t launch_snapshot(const double *x, const double *y, const double *z, const double *px,
                            const double *py, const double *pz, const double *mass, const long long *steps,
                            const int32_t *user, float *pos, float *vel, long long *frame_steps, int n, int n_sys,
                            cudaStream_t st);
cudaError_t launch_gather_systems(const SysInfo *sys, const int32_t *atom_sys, const int32_t *perm,
                                  const int32_t *user, const int32_t *devidx, const void *src, void *dst, int n,
                                  cudaStream_t st);

}  // namespace pb2
