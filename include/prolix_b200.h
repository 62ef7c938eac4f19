/*
 * prolix_b200 C ABI: a B200 (sm_100a) implementation of prolix's
 * implicit-solvent (OBC2 GBSA) energy/force function and its BAOAB Langevin
 * integrator, batched over many systems of uneven size.
 *
 * Conventions
 *  - Every entry point returns an int status: PB2_OK (0) or a negative
 *    PB2_E* code; pb2_last_error() describes the most recent failure of the
 *    context.  No C++ exception crosses this boundary.
 *  - Units are AKMA, as in prolix (src/prolix/simulate.py:52-57, 770-772):
 *    A, kcal/mol, e, amu, time in tau = 48.88821291839 fs.
 *  - Host arrays are read only during the call.  Device state is owned by
 *    the batch handle.  All GPU work is issued on the stream passed in
 *    (NULL = the legacy default stream); calls that return host data
 *    synchronise that stream.
 *  - A context is used by one host thread at a time.
 *
 * Reference interfaces replaced (paths within maraxen/prolix):
 *  - make_energy_fn(..., implicit_solvent=True)   src/prolix/physics/system.py:29-271
 *  - -jax.grad of that energy / single_padded_force src/prolix/batched_energy.py:730-850
 *  - nvt_langevin / langevin_with_constraints init_fn, apply_fn
 *                                                  src/prolix/physics/settle.py:1637-1746
 *  - batched BAOAB step over many systems          src/prolix/batched_simulate.py:218-382
 *  - neighbour list allocate/update, skin rebuild  src/prolix/physics/neighbor_list.py:155-172,
 *                                                  src/prolix/batched_simulate.py:1524-1640
 * The reference has no compiled FFI of its own; these functions are what a
 * jax.ffi custom-call registration (or the ctypes binding in
 * prolix_b200/_lib.py) binds.
 */
#ifndef PROLIX_B200_H
#define PROLIX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PB2_ABI_VERSION 3

/* status codes */
#define PB2_OK 0
#define PB2_EINVAL (-1)      /* bad argument */
#define PB2_ENOMEM (-2)      /* device or host allocation failed */
#define PB2_ECUDA (-3)       /* a CUDA runtime call failed */
#define PB2_ENLOVERFLOW (-4) /* neighbour-list capacity exceeded (rebuild with more) */
#define PB2_ENONFINITE (-5)  /* a non-finite force or position was produced */
#define PB2_ETIMEOUT (-6)    /* a bounded device-side wait ran out */
#define PB2_ENODEV (-7)      /* no usable sm_100 device */

/* energy term slots (per system), in this order */
#define PB2_TERM_BOND 0
#define PB2_TERM_ANGLE 1
#define PB2_TERM_DIHEDRAL 2
#define PB2_TERM_CMAP 3
#define PB2_TERM_LJ 4
#define PB2_TERM_COULOMB 5
#define PB2_TERM_GB 6
#define PB2_TERM_NONPOLAR 7
#define PB2_TERM_EXCEPTION 8 /* explicit 1-4 exception pairs (prolix bonded.py:186-230) */
#define PB2_TERM_IMPROPER 9  /* impropers, periodic or harmonic (system.py:63-88) */
#define PB2_TERM_UREY_BRADLEY 10 /* Urey-Bradley 1-3 springs (system.py:93-95) */
#define PB2_TERM_TOTAL 11
#define PB2_NTERMS 12

/* term-enable bits (pb2_run_params.terms) */
#define PB2_USE_BONDED 0x1u    /* bonds, angles, torsions, impropers, Urey-Bradley */
#define PB2_USE_CMAP 0x2u
#define PB2_USE_LJ 0x4u
#define PB2_USE_COULOMB 0x8u
#define PB2_USE_GB 0x10u       /* OBC2 Born radii + GB polar + ACE nonpolar */
#define PB2_USE_ALL 0x1Fu

/* per-system status bits (pb2_get_status) */
#define PB2_STATUS_NONFINITE 0x1u
#define PB2_STATUS_NLOVERFLOW 0x2u
#define PB2_STATUS_FORCE_RANGE 0x4u /* |F| beyond the fixed-point range */
/* a bounded device-side wait gave up; that evaluation's results for the
 * system are invalid (never expected: the waits are for work already in
 * flight on the same launch) */
#define PB2_STATUS_WAIT_TIMEOUT 0x8u

/* One system, host arrays.  Atom indices are local to the system. */
typedef struct pb2_system_desc {
  int32_t n_atoms;
  const double *positions;    /* (n, 3) */
  const double *charges;      /* (n) e */
  const double *sigmas;       /* (n) A, LJ sigma */
  const double *epsilons;     /* (n) kcal/mol */
  const double *radii;        /* (n) A, GB intrinsic radius rho */
  const double *scaled_radii; /* (n) A, rho * OBC scale factor */
  const double *masses;       /* (n) amu */

  int32_t n_bonds;
  const int32_t *bonds;       /* (n_bonds, 2) */
  const double *bond_params;  /* (n_bonds, 2) = (r0, k), E = k/2 (r - r0)^2 */
  int32_t n_angles;
  const int32_t *angles;      /* (n_angles, 3) */
  const double *angle_params; /* (n_angles, 2) = (theta0, k) */
  int32_t n_torsions;
  int32_t n_torsion_terms;    /* T terms per torsion */
  const int32_t *torsions;    /* (n_torsions, 4) */
  const double *torsion_params; /* (n_torsions, T, 3) = (n, phase, k) */

  int32_t n_cmap;
  const int32_t *cmap_rows;   /* (n_cmap, 5): phi = atoms 0-3, psi = atoms 1-4 */
  const int32_t *cmap_map;    /* (n_cmap) map index */
  int32_t n_cmap_maps;
  int32_t cmap_grid;          /* G, grid points per angle */
  const double *cmap_coeffs;  /* (n_cmap_maps, G, G, 16) bicubic patch coefficients,
                                 c[a*4+b] multiplies u^a v^b, u along phi */

  int32_t n_excl;
  const int32_t *excl_pairs;  /* (n_excl, 2), i < j */
  const int32_t *excl_kind;   /* (n_excl): 0 = excluded (1-2, 1-3), 1 = 1-4 scaled */

  double lj14_scale;          /* LJ scale of 1-4 pairs (prolix: 0.5) */
  double coul14_scale;        /* Coulomb scale of 1-4 pairs (prolix: 0.83333333) */
  double eps_in, eps_out;     /* solute / solvent dielectric */
  double k_gb;                /* Coulomb constant in the GB prefactor */
  double k_coulomb;           /* Coulomb constant of the direct term (332.0637) */
  uint32_t key[2];            /* threefry key of this system's noise stream */

  double dt;                  /* tau */
  double kT;                  /* kcal/mol */
  double gamma;               /* 1/tau */
  int32_t use_origin;         /* 1: take origin below; 0: the rounded centroid of positions */
  double origin[3];           /* A; float32 pair coordinates are taken relative to it, so a
                                 system moved between batches keeps bit-identical forces */

  /* Explicit 1-4 exception pairs (prolix ExclusionSpec.exception_*,
   * physics/neighbor_list.py:44-50; energy bonded.py:186-230): per pair,
   * d = sqrt(r^2 + 1e-12), E = 4 eps ((sigma/d)^12 - (sigma/d)^6) + k_coulomb qq / d,
   * parameters already scaled.  The LJ part follows PB2_USE_LJ, the Coulomb
   * part PB2_USE_COULOMB.  As in ExclusionSpec.from_protein, these pairs
   * should also be listed as excluded (kind 0) so that the main LJ/Coulomb
   * terms skip them; GB keeps every pair. */
  int32_t n_exceptions;
  const int32_t *exception_pairs;  /* (n_exceptions, 2) */
  const double *exception_params;  /* (n_exceptions, 3) = (charge product, sigma, epsilon) */

  /* Impropers (prolix make_energy_fn, system.py:63-88; bonded.py:110-185).
   * improper_form 0, periodic: params (n_impropers, T, 3) = (n, phase, k),
   *   E = sum k (1 + cos(n phi - phase)), the torsion formula;
   * improper_form 1, harmonic: params (n_impropers, T, 2) = (k, phi0),
   *   E = sum k d^2 with d = ((phi - phi0 + pi) mod 2 pi) - pi (no 1/2).
   * phi is the dihedral of atoms 0-1-2-3 of a row, as for torsions. */
  int32_t n_impropers;
  int32_t n_improper_terms;   /* T */
  int32_t improper_form;      /* 0 periodic, 1 harmonic */
  const int32_t *impropers;   /* (n_impropers, 4) */
  const double *improper_params;

  /* Urey-Bradley springs between 1-3 atoms (system.py:93-95): E = k/2 (r - r0)^2. */
  int32_t n_urey_bradley;
  const int32_t *urey_bradley_bonds;   /* (n_urey_bradley, 2) */
  const double *urey_bradley_params;   /* (n_urey_bradley, 2) = (r0, k) */
} pb2_system_desc;

/* Batch-wide settings. */
typedef struct pb2_run_params {
  uint32_t terms;       /* PB2_USE_* bits */
  double cutoff;        /* A; LJ and Coulomb; <= 0: all pairs */
  double skin;          /* A; neighbour-list skin (rebuild when any atom moved > skin/2) */
  int32_t nl_capacity;  /* per-atom neighbour capacity; 0 = automatic */
  int32_t tile_segment; /* tiles per work item; 0 = autotuned/default */
  int32_t graph_chunk;  /* steps per captured CUDA graph; 0 = 50 */
  int32_t partitionable_keys; /* 1: jax_threefry_partitionable layout (JAX default) */
  double gb_cutoff;     /* A; GB pairs and descreening: < 0 same as cutoff, 0 all pairs.
                           prolix's make_energy_fn keeps GB all-pairs while LJ/Coulomb
                           use the cutoff (system.py:196-216); with a GB cutoff the
                           neighbour-list clamps of generalized_born.py:300-337 apply */
  double born_cutoff;   /* A; > 0: descreening sums and their chain rule only (the NL-Born +
                           dense-GB split, generalized_born.py:706-817); the GB pair terms keep
                           gb_cutoff.  <= 0: the descreening uses gb_cutoff too */
  int32_t keep_atom_order; /* 0: the batch stores each system's atoms in a spatial order
                              (compact 32-atom blocks, which the pair kernels' bounding-box
                              tests favour); 1: in input order.  Either way every array
                              crossing this interface is in input order. */
  int32_t pair_list;    /* 0: automatic: when every pair term in use has a cutoff, the pair
                           kernels work from a skin-buffered list of 32-atom block pairs
                           within cutoff + skin, rebuilt on the device when an atom has
                           moved more than skin/2 since the last build (jax_md's
                           dr_threshold rule, batched_simulate.py:1600-1622); -1: off (every
                           block pair, culled by bounding boxes at each step) */
} pb2_run_params;

typedef struct pb2_ctx pb2_ctx;
typedef struct pb2_batch pb2_batch;

int pb2_abi_version(void);

/* Context: binds one CUDA device. */
int pb2_ctx_create(int device, pb2_ctx **out);
int pb2_ctx_destroy(pb2_ctx *ctx);
const char *pb2_last_error(const pb2_ctx *ctx);

/*
 * Upload n_systems systems as one ragged batch (atoms of all systems
 * concatenated, each system's tiles its own).  Replaces building
 * PhysicsSystem/PaddedSystem pytrees (prolix typing.py:248-420,
 * padding.py:21-26) and ExclusionSpec tables (physics/neighbor_list.py:25-303).
 */
int pb2_batch_create(pb2_ctx *ctx, int32_t n_systems, const pb2_system_desc *systems,
                     const pb2_run_params *params, pb2_batch **out);
int pb2_batch_destroy(pb2_batch *batch);
int pb2_batch_info(const pb2_batch *batch, int32_t *n_systems, int64_t *n_atoms_total);

/*
 * Energies and forces at the batch's current positions.  energies: NULL or
 * (n_systems, PB2_NTERMS); forces: NULL or (n_atoms_total, 3), atoms in
 * batch order.  Replaces total_energy / decomposed dict (system.py:229-270)
 * and -jax.grad(total_energy).
 */
int pb2_energy_forces(pb2_batch *batch, double *energies, double *forces, void *stream);

/* Born radii (n_atoms_total) at the current positions (system.py:204-216). */
int pb2_born_radii(pb2_batch *batch, double *born, void *stream);

/* The same with DEVICE pointers on the batch's device: positions (may be
 * NULL: keep the current ones), energies (n_systems, PB2_NTERMS) and forces
 * (n_atoms_total, 3), row-major FP64, either may be NULL.  Asynchronous on
 * `stream`; allocates and synchronises nothing, so an XLA FFI handler (the
 * binding a prolix maintainer adds for make_energy_fn, system.py:29-271)
 * or a captured CUDA graph can call it. */
int pb2_energy_forces_device(pb2_batch *batch, const double *positions, double *energies,
                             double *forces, void *stream);

/* Overwrite positions (n_atoms_total, 3). */
int pb2_set_positions(pb2_batch *batch, const double *positions, void *stream);

/*
 * BAOAB state.  pb2_langevin_init replaces init_fn (settle.py:1676-1696):
 * (key, sub) = split(key); p = sqrt(m kT) normal(sub); F = force(x).
 * pb2_langevin_run replaces n_steps calls of apply_fn (settle.py:1698-1744)
 * for every system of the batch; steps are issued as CUDA graphs of
 * graph_chunk steps.
 */
int pb2_langevin_init(pb2_batch *batch, void *stream);
int pb2_langevin_run(pb2_batch *batch, int32_t n_steps, void *stream);

/* Subtract each system's mean momentum, as jax_md's nvt_langevin init_fn
 * does with center_velocity (prolix applies it over real atoms only,
 * physics/settle.py:1121-1142); systems of one atom are left alone.  Call
 * after pb2_langevin_init for jax_md's init; prolix's own BAOAB init
 * (settle.py:1676-1696) does not center. */
int pb2_langevin_center_momentum(pb2_batch *batch, void *stream);

/* New Langevin parameters for the following steps, per system (n_systems
 * each; NULL keeps that parameter): dt (tau), kT (kcal/mol), gamma (1/tau).
 * Replaces apply_fn's per-call dt / kT overrides (settle.py:1698-1700).
 * c1 = exp(-gamma dt), c2 = sqrt(1 - c1^2) and the per-atom noise amplitude
 * c2 sqrt(m kT) are recomputed exactly as at batch creation, so a batch
 * created with these values steps bit for bit the same.  Captured graphs
 * stay valid (they read the parameters from device memory).  The call
 * first waits for all work queued on the device, on every stream, so steps
 * issued before it run with the old values. */
int pb2_set_langevin_params(pb2_batch *batch, const double *dt, const double *kT, const double *gamma,
                            void *stream);

/* Read or write the integrator state; any pointer may be NULL.
 * x, p, f: (n_atoms_total, 3); keys: (n_systems, 2); steps: (n_systems). */
int pb2_get_state(pb2_batch *batch, double *x, double *p, double *f, uint32_t *keys,
                  int64_t *steps, void *stream);
int pb2_set_state(pb2_batch *batch, const double *x, const double *p, const uint32_t *keys,
                  void *stream);

/* Restore the whole BAOAB state (the fields of prolix's NVTLangevinState,
 * typing.py:611-618: positions, momentum, force, rng) without evaluating
 * forces: f must be the forces at x, as pb2_get_state returned them (the
 * round trip is exact).  x, p, f required; keys may be NULL.  Transfers run
 * at full PCIe speed when the host buffers are page-locked. */
int pb2_set_full_state(pb2_batch *batch, const double *x, const double *p, const double *f,
                       const uint32_t *keys, void *stream);

/* n_steps BAOAB steps on a state the caller keeps in host memory: the
 * functional form of apply_fn (settle.py:1698-1744, state in, new state
 * out).  x, p, f ((n_atoms_total, 3), f the forces at x as pb2_get_state
 * returned them) are copied to the device on `copy_in`, stepped on
 * `stream`, and copied back into the same arrays on `copy_out`; the rng
 * keys and step counters stay on the device.  Pass `stream` three times to
 * use one stream.  Nothing waits: the arrays hold the new state once
 * `copy_out` has finished (cudaStreamSynchronize), and must not be touched
 * before.  With page-locked arrays the copies are asynchronous: batches
 * stepped on their own streams but sharing one copy_in and one copy_out
 * stream move their states one after another at full PCIe speed while
 * other batches compute. */
int pb2_langevin_run_host(pb2_batch *batch, double *x, double *p, double *f, int32_t n_steps,
                          void *stream, void *copy_in, void *copy_out);

/* The same functional apply_fn (settle.py:1698-1744) on DEVICE arrays of the
 * batch's device: x, p, f ((n_atoms_total, 3) FP64 row-major, f the forces
 * at x) are read, n_steps steps run, and the new state is written back into
 * them, all on `stream` without waiting.  This is what a jax.ffi handler
 * binds (XLA owns the buffers).  Steps run as CUDA graphs of up to
 * graph_chunk steps, captured the first time each chunk length is needed:
 * make a first call with the same n_steps outside any stream capture. */
int pb2_langevin_run_device(pb2_batch *batch, double *x, double *p, double *f, int32_t n_steps,
                            void *stream);

/*
 * Batched energy minimisation (replaces prolix batched_simulate.py:682-960,
 * `batched_minimize`, whose SD and FIRE stages run per system under vmap).
 * pb2_min_setup stores the current positions as the restraint reference and
 * the per-atom selections (heavy / backbone; NULL: heavy = mass > 1.1 amu,
 * backbone = heavy).  Each call then runs one stage on every system:
 *   pb2_min_sd   : restrained steepest descent, dr = F dt capped at max_dx
 *                  per atom (batched_simulate.py:748-791);
 *   pb2_min_fire : FIRE from zero momentum (jax_md fire_descent, called at
 *                  :818-878) with a per-atom displacement cap max_disp
 *                  (0: none) and, for the first half kick, a per-atom force
 *                  cap force_cap (0: none; prolix simulate.py:613-638);
 *                  with PB2_FIRE_KEEP_BEST in flags the state ends at the
 *                  positions of the lowest force RMS seen, else at the last;
 * with restraint E = k/2 sum |r - r0|^2 on kind 0 all atoms, 1 heavy atoms,
 * 2 backbone atoms.  A system that turns non-finite returns to r0 and gets
 * PB2_STATUS_NONFINITE.  FIRE uses the momentum arrays: call
 * pb2_langevin_init before dynamics.  pb2_min_rms: per-system RMS over atoms
 * of the unrestrained force (the convergence gate, :944-951).
 */
int pb2_min_setup(pb2_batch *batch, const uint8_t *heavy, const uint8_t *backbone);
int pb2_min_sd(pb2_batch *batch, int32_t n_steps, double k, int32_t kind, double dt, double max_dx,
               void *stream);
#define PB2_FIRE_KEEP_BEST 1
int pb2_min_fire(pb2_batch *batch, int32_t n_steps, double k, int32_t kind, double dt_start,
                 double dt_max, double max_disp, double force_cap, int32_t flags, void *stream);
int pb2_min_rms(pb2_batch *batch, double *rms, void *stream);

/* L-BFGS polish of every system (the reference's jaxopt stage,
 * batched_simulate.py:885-936): history `hist` (<= 16), backtracking line
 * search from t = min(1, max_step) by 0.8 over at most max_trials energy
 * evaluations (Armijo 1e-4, curvature 0.9), stopping a system when its
 * gradient norm falls below tol; converged (may be NULL) receives 1 per
 * system that did.  Uses the unrestrained energy. */
int pb2_min_lbfgs(pb2_batch *batch, int32_t n_iter, double tol, double max_step, int32_t hist,
                  int32_t max_trials, int32_t *converged, void *stream);

/* Replica exchange (replaces the state shuffle of prolix
 * pt/replica_exchange.py:197-228): slot s takes the positions, momenta and
 * forces of slot perm[s]; keys, step counters, kT and dt stay with the
 * slots.  perm must be a permutation of 0..n_systems-1 pairing systems of
 * equal atom count. */
int pb2_permute_systems(pb2_batch *batch, const int32_t *perm, void *stream);

/*
 * Trajectory frames (the state prolix's TrajectoryWriter stores,
 * simulate.py:146-203, typing.py:652-707): a device ring of `capacity`
 * frames of float32 positions and velocities (n_atoms_total, 3) plus every
 * system's step counter.  pb2_traj_snapshot copies the current state into a
 * slot asynchronously on `stream` (no host synchronisation; capturable);
 * pb2_traj_fetch copies `count` slots from `first` to host buffers
 * (frames in slot order, each (n_atoms_total, 3); steps (count, n_systems))
 * and returns when they have arrived.  Any pointer may be NULL.
 */
int pb2_traj_setup(pb2_batch *batch, int32_t capacity);
int pb2_traj_snapshot(pb2_batch *batch, int32_t slot, void *stream);
int pb2_traj_fetch(pb2_batch *batch, int32_t first, int32_t count, float *positions, float *velocities,
                   int64_t *steps, void *stream);

/* Per-system status bits (PB2_STATUS_*) accumulated since the last clear. */
int pb2_get_status(pb2_batch *batch, uint32_t *status, int clear, void *stream);

/*
 * Safeguards of prolix's batched Langevin step (make_langevin_step,
 * batched_simulate.py:218-382; its production values are vlimit 20,
 * max_dx 0.5 A, force_cap 1e4 kcal/mol/A).  Each limit <= 0 is off; all off
 * (the default) is the plain BAOAB step of pb2_langevin_run.  With limits set
 * a step is
 *   p += dt/2 F;  where |p/m| > vlimit: p *= min(1, vlimit / (|p/m| + 1e-30));
 *   x_old = x;  A;  O;  A;
 *   s = min(1, max_dx / |x - x_old|);  x = x_old + (x - x_old) s;
 *   where |x - x_old| > max_dx: p *= s;
 *   F = force(x);  F *= min(1, force_cap / |F|);  p += dt/2 F
 * with |v| = sqrt(v.v + 1e-30) (1e-12 for F).  The capped closing force also
 * opens the next step (the reference keeps it as the state's force); a force
 * that no step produced (after pb2_langevin_init, pb2_set_positions,
 * pb2_set_state, pb2_set_full_state or minimisation) opens the next step as
 * it is.  pb2_get_state and pb2_langevin_run_host hand out the uncapped
 * force; a host round trip that passes it back unchanged continues the run
 * exactly.  Setting new limits drops captured graphs.
 */
int pb2_set_safeguards(pb2_batch *batch, double vlimit, double max_dx, double force_cap);
int pb2_get_safeguards(const pb2_batch *batch, double *vlimit, double *max_dx, double *force_cap);

/* Per-system counts (n_systems, 4) of the steps in which each safeguard
 * fired, in prolix's warn_counts order (typing.py:559-563): vlimit, force
 * cap, constraint violation (always 0: no constraints), displacement cap.
 * The force-cap column is the reference's cap_count.  reset != 0 zeroes the
 * counts after reading them. */
int pb2_get_warn_counts(pb2_batch *batch, int32_t *counts, int reset, void *stream);

/*
 * Neighbour list (cutoff > 0 only), built on the device with the batch's
 * spatially sorted 32-atom blocks as the cells (block bounding boxes in place
 * of a cell stencil), in jax_md partition.neighbor_list's layout
 * (physics/neighbor_list.py:155-172; batched_simulate.py:1429-1464).  pb2_nl_build rebuilds unconditionally
 * and returns when the capacity is known (the first build sizes it, as
 * jax_md's allocate does).  pb2_nl_check compares each atom's displacement
 * since the last build against skin/2 (batched_simulate.py:1600-1622) and
 * rebuilds when any exceeds it, all decided on the device; with rebuilt
 * non-NULL it waits and *rebuilt receives how many systems had moved that
 * far, with rebuilt NULL it only enqueues (a list that outgrew its capacity
 * is flagged with PB2_STATUS_NLOVERFLOW and grown at the next pb2_nl_check
 * with rebuilt, pb2_nl_build or pb2_nl_capacity).  pb2_nl_capacity waits
 * for the device and reports the row width after any such growth.
 * pb2_nl_get copies the per-atom list in jax_md layout into a buffer of that
 * width: (n_atoms_total, capacity) int32 local indices, both (i, j) and
 * (j, i) present, padded with the sentinel n_atoms of the atom's system; it
 * returns PB2_ENLOVERFLOW, writing nothing, when a build queued after the
 * capacity query needs wider rows.  pb2_nl_last_build_ms: device time of the last
 * build's launches (CUDA events; diagnostic, no reference counterpart).
 */
int pb2_nl_build(pb2_batch *batch, void *stream);
int pb2_nl_check(pb2_batch *batch, int32_t *rebuilt, void *stream);
int pb2_nl_capacity(pb2_batch *batch, int32_t *capacity);
int pb2_nl_get(pb2_batch *batch, int32_t *neighbors, void *stream);
int pb2_nl_last_build_ms(pb2_batch *batch, double *ms);

/* Device time of the last pb2_langevin_run with profiling enabled (eager
 * launches, CUDA events around each kernel), milliseconds summed over the
 * run: out[0] descreening pass, out[1] Born finalize, out[2] force pass,
 * out[3] chain pass, out[4] bonded, out[5] integrator, out[6] bounding boxes,
 * out[7] whole run. */
/* Tiles per work item of the pair kernels (the autotuned knob).  Setting it
 * rebuilds the work list and drops captured graphs.  No reference
 * counterpart (prolix's tile sizes are fixed, physics/tiling.py:29-50). */
int pb2_set_tile_segment(pb2_batch *batch, int32_t segment);
int pb2_get_tile_segment(const pb2_batch *batch, int32_t *segment);

/* Retire system `sys` of the batch, in stream order on `stream`: no later
 * step, closing half kick or pair evaluation of the batch touches it, so its
 * positions, momenta and key stay as the last step left them, and the pair
 * kernels' live work list drops its items (an ordered on-device compaction;
 * with a pair list, a rebuild without it).  It then costs only its memory;
 * the other systems' results are bit-identical with or without it.  Its
 * forces, energies and Born radii are undefined from then on.  Irreversible;
 * retiring a retired system does nothing.  For continuous batching, where
 * prolix has no counterpart (its batches run to the end,
 * batched_simulate.py:1125-1163). */
int pb2_retire_system(pb2_batch *batch, int32_t sys, void *stream);

/* Test hook for the bounded device waits: raises the number of descreening
 * items the fused Born finalize of system `sys` waits for by `hold` (0
 * restores it), so that its wait runs out (about a second) and the system
 * is flagged with PB2_STATUS_WAIT_TIMEOUT while the other systems' results
 * stay exact.  Not for a batch with a pair list.  Waits for the device. */
int pb2_test_hold_system(pb2_batch *batch, int32_t sys, int32_t hold);

/* Block shape of a pair pass (pass 0 descreening, 1 force, 2 chain rule,
 * 3 the force pass's four-block kernel): threads per block and the resident
 * blocks per SM its registers are sized for.  Each pass is compiled for a
 * few shapes: pb2_block_shapes fills up to capacity of them and returns how
 * many there are; pb2_set_block_shape picks one (PB2_EINVAL if not
 * compiled) and drops captured graphs.  The autotuner's other knob; no
 * reference counterpart. */
int pb2_block_shapes(int32_t pass, int32_t *threads, int32_t *min_blocks, int32_t capacity);
int pb2_set_block_shape(pb2_batch *batch, int32_t pass, int32_t threads, int32_t min_blocks);
int pb2_get_block_shape(const pb2_batch *batch, int32_t pass, int32_t *threads, int32_t *min_blocks);

/* I-blocks per warp of the force pass: 2, or 4 (two packed pairs of
 * i-blocks share every j atom's loads; used without a pair list, where the
 * list's rows are pairs of i-blocks).  Both give the same forces and dE/dB
 * bit for bit; setting it drops captured graphs.  No reference
 * counterpart. */
int pb2_set_force_blocks(pb2_batch *batch, int32_t blocks);
int pb2_get_force_blocks(const pb2_batch *batch, int32_t *blocks);

/* Which per-step work rides inside the pair passes instead of a launch of
 * its own (an MD step is then four launches: step, descreening, force,
 * chain rule; a cutoff run with a pair list adds the list's update):
 * PB2_FUSE_BONDED, the bonded terms as the chain pass's tail work, 32 terms
 * per chunk; PB2_FUSE_FINALIZE, the Born radii as the descreening pass's
 * tail work, one chunk per 32-atom block, each started once its system's
 * pair items have all been summed (a bounded wait on work already in
 * flight; PB2_STATUS_WAIT_TIMEOUT if it ever gives up).  Default:
 * PB2_FUSE_BONDED (five launches per step); the autotuner times the
 * alternatives.  Results are bit-identical either way.
 * No reference counterpart. */
#define PB2_FUSE_BONDED 0x1
#define PB2_FUSE_FINALIZE 0x2
int pb2_set_fusion(pb2_batch *batch, int32_t flags);
int pb2_get_fusion(const pb2_batch *batch, int32_t *flags);

int pb2_set_profiling(pb2_batch *batch, int enable);
int pb2_last_timings(pb2_batch *batch, double *out_ms);

/* Measured FP32 FMA throughput of the context's GPU (TFLOP/s), the roofline
 * denominator of the pair kernels.  Diagnostic: no reference counterpart. */
int pb2_fp32_peak(pb2_ctx *ctx, double *tflops);
/* Checks the integrator's FP64 division (a precomputed reciprocal and two
 * Markstein corrections) bit for bit against the correctly rounded division
 * on n seeded operand pairs (masses 0.5-512, momenta of any sign and
 * exponents -40..40, plus structured cases).  mismatches: pairs whose bits
 * differ; example (may be NULL): the first such (p, m).  Diagnostic, no
 * reference counterpart. */
int pb2_diag_div_check(pb2_ctx *ctx, long long n, unsigned long long seed, long long *mismatches,
                       double *example);

/*
 * Born radii of one system with no device allocation (no counterpart in the
 * reference: prolix allocates through JAX).  For callers that cannot call
 * cudaMalloc -- an XLA custom-call handler, which may use only the buffers
 * the runtime hands it; code running while a stream is captured into a CUDA
 * graph; hosts that give the library a fixed memory pool.  The caller
 * passes device buffers: positions (n, 3), radii (n), scaled_radii (n) and
 * born (n) out, all FP64.  cutoff <= 0 sums all pairs.  The descreening
 * scratch is a static 256 KiB device array shared by every call, so n_atoms
 * is limited to PB2_NOALLOC_MAX_ATOMS; calls that overlap on the GPU race on
 * it and must be serialised.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) with that device current: make it before any
 * stream capture (after a cudaDeviceReset the next call looks it up again).
 * The buffers must be device memory of the current device, which must be
 * the context's device when ctx is given (PB2_EINVAL otherwise).  ctx may
 * be NULL (errors are then not recorded).
 */
#define PB2_NOALLOC_MAX_ATOMS 32768
int pb2_born_radii_noalloc(pb2_ctx *ctx, int32_t n_atoms, const double *positions,
                           const double *radii, const double *scaled_radii, double cutoff,
                           double *born, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PROLIX_B200_H */
