/*
 * pystarc_b200 -- C ABI of the B200-native batched rigid-body Brownian-dynamics engine.
 *
 * Every entry point returns an int status (BD_OK = 0, negative on error) and
 * never exits or aborts; bd_last_error() gives the message.  One handle is used
 * by one host thread at a time; handles are independent.  `stream` arguments are
 * cudaStream_t values (NULL = the legacy default stream).  Array arguments are
 * plain pointers; which side (device or host) each pointer lives on is stated
 * per function.  Units are the reference's: Angstrom, ps, kBT, e.
 *
 * Reference interfaces replaced (paths inside anandojha/PySTARC):
 *   GPUBatchForceEngine.__init__ / _upload_grids   pystarc/forces/gpu_batch_engine.py:139-287
 *   GPUBatchForceEngine.__call__                  pystarc/forces/gpu_batch_engine.py:531-605
 *   GPUBatchSimulator.__init__                    pystarc/simulation/gpu_batch_simulator.py:159-318
 *   GPUBatchSimulator.run (step loop)             pystarc/simulation/gpu_batch_simulator.py:462-1594
 */
#ifndef PYSTARC_B200_H
#define PYSTARC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct BdHandle BdHandle;

enum {
  BD_OK = 0,
  BD_ERR_ARG = -1,      /* invalid argument or unsupported size */
  BD_ERR_CUDA = -2,     /* CUDA runtime error */
  BD_ERR_OOM = -3,      /* device allocation failed */
  BD_ERR_NAN = -4,      /* non-finite input or result */
  BD_ERR_STALL = -5,    /* watchdog: a bounded device loop gave up */
  BD_ERR_STATE = -6     /* call out of order (e.g. run before configure) */
};

enum { BD_GRID_ELEC = 0, BD_GRID_BORN = 1, BD_GRID_LIG_BORN = 2 };
enum { BD_PREC_FP64 = 0, BD_PREC_MIXED = 1 };         /* force/torque/mobility arithmetic */
enum { BD_TORQUE_ZERO = 0, BD_TORQUE_CENTROID = 1 };  /* zero = reference GPU path */

/* Far-field and Born parameters (gpu_batch_engine.py:139-175). */
typedef struct {
  double receptor_charge; /* Q_rec, e */
  double debye_length;    /* A */
  double sdie;            /* solvent dielectric of the far-field */
  double alpha;           /* Born desolvation alpha */
  int use_multipole;      /* 1: dipole + quadrupole terms (MultipoleExpansion) */
  double dipole[3];
  double quadrupole[9];   /* row-major, 1/2 sum q (3 r r - r^2 I) */
  double four_pi_eps;     /* 4 pi sdie eps0 of the multipole terms */
} BdForceParams;

/* Stepper parameters (GPUBatchSimulator.run, gpu_batch_simulator.py:462-1254). */
typedef struct {
  int64_t n_traj;
  uint64_t seed;
  double r_start, r_escape;  /* b-sphere, escape sphere */
  double return_prob;        /* host-computed (Romberg), applied at r_escape */
  int32_t max_steps;         /* per-trajectory cap; reached -> max-steps outcome */
  double max_dt, min_core_dt;
  int32_t use_hi, overlap;
  double D_t, D_r;           /* relative translational / rotational diffusion */
  double q_rec_total, q_lig_total, adt_debye;  /* adaptive-dt force criterion */
  double r_hydro_rec, r_hydro_lig;
  int32_t precision, torque_mode;
  int32_t slots;             /* live-slot capacity; 0 = automatic */
  int64_t id_offset;         /* global id of local trajectory 0 (keys the noise; shards across GPUs) */
  int32_t stats;             /* 1: collect the per-step statistics read by bd_sim_stats */
  double min_core_rxn_dt;    /* state-machine mode: floor of the reaction-surface dt refinement
                              * (params.minimum_core_reaction_dt, gpu_batch_simulator.py:636) */
  int32_t save_interval;     /* with stats: record a path and an energy row of every running trajectory
                              * whose step index is a multiple of this (output_cfg.save_interval, 10) */
  int64_t trace_capacity;    /* with stats: rows kept on the device for bd_sim_traces (0: no traces) */
  int32_t hi_mode;           /* with use_hi: BD_HI_REFERENCE_GPU or BD_HI_ZUK */
  double hi_kT_eta;          /* BD_HI_ZUK: kBT/eta = sqrt(D_t1 6 pi a1 D_t2 6 pi a2), A^3/ps
                              * (hydrodynamics/rotne_prager.py:121-122) */
} BdSimParams;

/* Relative translational diffusion D(r) of the stepper when use_hi is set.
 * BD_HI_REFERENCE_GPU: the reference GPU stepper's line-of-centres formula
 *   D = Df ainv - 2 Df (2/r - (4/3) a2/r^3) / (8 pi), Df = 1/0.243, clamped at 1e-6
 *   (gpu_batch_simulator.py:741-751, :1074-1084).
 * BD_HI_ZUK: the Rotne-Prager-Yamakawa coupling of MobilityTensor.relative_translational_diffusion,
 *   D = D_t - (2/3) tr M12(r), M12 by the three regimes of Zuk et al. (2014): far field, partial
 *   overlap, one sphere inside the other; clamped at 1e-12 (hydrodynamics/rotne_prager.py:67-124,
 *   :177-200). */
enum { BD_HI_REFERENCE_GPU = 0, BD_HI_ZUK = 1 };

/* Host arrays filled by bd_sim_stats (NULL members are skipped).  Per trajectory
 * (n_traj entries, x3 / x4 for poses): start pose, closest approach |c| with its
 * step and pose, accumulated time, reaction pose and step, bridge flag.  Histograms
 * as the reference's (gpu_batch_simulator.py:577-620, :1255-1317): radial 200 bins on
 * [0, 1.2 r_escape], angular 36 x 72 (theta, phi), milestone crossings of 11 shells
 * from r_start to r_escape (out and in), radial transition matrix 50 x 50, pair
 * contact counts at the force-evaluation pose; plus the bin edges used. */
typedef struct {
  double *start_pos, *start_q, *min_dist, *near_miss_pos, *near_miss_q, *total_time, *encounter_pos, *encounter_q;
  int32_t *step_at_min, *encounter_step;
  int8_t* bridge;
  uint64_t *radial, *angular, *milestone_out, *milestone_in, *transition, *contact;
  double *radial_edges, *transition_edges, *milestone_radii;
} BdStatsOut;

/* Counter indices of bd_sim_counters(). */
enum {
  BD_CTR_STARTED = 0, BD_CTR_REACTED, BD_CTR_ESCAPED, BD_CTR_MAXSTEPS, BD_CTR_STEPS, BD_CTR_RETURNS,
  BD_CTR_OVERLAP, BD_CTR_BRIDGE, BD_CTR_GRID_EVALS, BD_CTR_REV_EVALS, BD_CTR_FF_EVALS, BD_CTR_NONFINITE,
  BD_CTR_NUM = 12
};

/* Library version string. */
const char* bd_version(void);

/* Create a handle bound to CUDA device `device`.  Replaces the engine's device setup. */
int bd_create(int device, BdHandle** out);
int bd_destroy(BdHandle* h);
/* Copy the last error message of `h` (or of the last failed bd_create when h is NULL). */
int bd_last_error(const BdHandle* h, char* buf, int len);

/* Ligand atoms in the body frame (about the centroid), host arrays: xyz (n*3), charges (n).
 * Replaces GPUBatchSimulator._mol2_pos0 / _charges (gpu_batch_simulator.py:171-176). */
int bd_set_ligand(BdHandle* h, int n, const double* body_xyz, const double* charges);
/* Receptor atoms (receptor at the origin), host arrays.  Replaces the engine's
 * rec_positions / rec_charges and the stepper's overlap table (gpu_batch_engine.py:207-217,
 * gpu_batch_simulator.py:771-781). */
int bd_set_receptor(BdHandle* h, int n, const double* xyz, const double* charges);
/* State-machine reactions (gpu_batch_simulator.py:216-319): reaction p is reaction pair p of
 * bd_set_reactions (one pair per reaction) and fires only while the trajectory is in state
 * state_before[p]; it then moves to state_after[p], and the trajectory has reacted when that
 * state is terminal (terminal[k] != 0: no reaction leaves state k).  States are 0..n_states-1,
 * 0 the first state; -1 stands for an unlabelled state and is looked up in `terminal` from the
 * end, as the reference's arrays index.  The lowest-numbered reaction that can fire wins, in the
 * discrete test (:818-854) and in the Brownian bridge (:1185-1234); near a reachable reaction
 * surface dt is refined (:1005-1060).  n_pairs = 0 returns to the flattened-pairs mode. */
int bd_set_reaction_states(BdHandle* h, int n_pairs, const int32_t* state_before, const int32_t* state_after,
                           int n_states, const uint8_t* terminal);
/* WCA contact forces (the repulsive part of Lennard-Jones) between every ligand and receptor
 * atom, from their radii: sigma = r_lig + r_rec, force eps (12 (sigma/r)^12 - 6 (sigma/r)^6) / r^2
 * along the pair for r < 1.122462 sigma, only for poses whose centroid is within `activation`
 * of the origin.  Radii follow the order of bd_set_ligand / bd_set_receptor (all atoms, charged
 * or not); activation < 0 selects 2.5 (max r_rec + max r_lig).  n_rec = 0 turns the term off.
 * Replaces GPUBatchForceEngine's rec_radii / lig_radii / use_lj and _wca_forces_gpu
 * (gpu_batch_engine.py:233-246, :474-529, :600-602); eps is the reference's 0.17 kBT. */
int bd_set_contact(BdHandle* h, int n_rec, const double* rec_radii, int n_lig, const double* lig_radii, double eps,
                   double activation);
/* Add a FP32 grid (host array, C order, z fastest).  kind = BD_GRID_*.  Grids are sorted
 * finest-first and dropped as the reference does (gpu_batch_engine.py:179-211, :248-287). */
int bd_add_grid(BdHandle* h, int kind, const float* data, int nx, int ny, int nz, const double* origin,
                const double* spacing);
int bd_clear_grids(BdHandle* h);
int bd_set_force_params(BdHandle* h, const BdForceParams* p);
/* Flattened reaction pairs (gpu_batch_simulator.py:186-215, :643-660): receptor atom
 * positions (n*3), ligand atom body positions (n*3), cutoffs, bridge D_eff per pair,
 * n_needed (already resolved: -1 handled by the caller).  Host arrays. */
int bd_set_reactions(BdHandle* h, int n_pairs, const double* rec_xyz, const double* lig_body_xyz,
                     const double* cutoffs, const double* d_eff, int n_needed);

/* Net force, torque and energy for n poses.  DEVICE arrays: centroids (n*3), rotations
 * (n*4 quaternions w,x,y,z or n*9 row-major matrices), outputs F (n*3), T (n*3), E (n).
 * Same result as GPUBatchForceEngine.__call__ (gpu_batch_engine.py:531-605) with the
 * ligand placed as R b + c; torque_mode BD_TORQUE_ZERO reproduces its zero torque. */
int bd_eval_forces(BdHandle* h, int64_t n, const double* centroids, const double* rotations, int rot_is_matrix,
                   double* F, double* T, double* E, int precision, int torque_mode, void* stream);
/* Same with explicit lab-frame ligand atom positions (n * n_lig * 3), rotation matrices
 * (n*9) and centroids (n*3): the reference __call__ argument list.  DEVICE arrays. */
int bd_eval_forces_atoms(BdHandle* h, int64_t n, const double* lig_positions, const double* R,
                         const double* centroids, double* F, double* T, double* E, int precision, int torque_mode,
                         void* stream);
/* The stepper's overlap test for n centroids: out[i] = 1 when some receptor atom lies within
 * 1.5 A of centroid i (gpu_batch_simulator.py:770-781, 1102-1128), else 0.  DEVICE arrays
 * centroids (n*3) and out (n); uses the occupancy grid when the layout has it. */
int bd_eval_overlap(BdHandle* h, int64_t n, const double* centroids, int8_t* out, void* stream);

/* Stepper.  configure allocates the live-slot pool and per-trajectory outputs; reset
 * starts the first `slots` trajectories; run enqueues n_launch launches of
 * steps_per_launch BD steps each (refill from the pending pool inside, compaction
 * between launches).  run is asynchronous on `stream`. */
int bd_sim_configure(BdHandle* h, const BdSimParams* p);
int bd_sim_reset(BdHandle* h, void* stream);
int bd_sim_run(BdHandle* h, int n_launch, int steps_per_launch, void* stream);
/* Synchronise `stream` and copy the BD_CTR_NUM counters to a host array. */
int bd_sim_counters(BdHandle* h, uint64_t* out, int n, void* stream);
/* Host copies of the per-trajectory outcome (0 running/unstarted, 1 reacted, 2 escaped,
 * 3 max-steps, 5 non-finite pose), step counts and return counts (n_traj each). */
int bd_sim_outcomes(BdHandle* h, int8_t* status, int32_t* steps, int32_t* returns);
/* Path and energy traces (gpu_batch_simulator.py:1319-1340): every step whose index s is a
 * multiple of save_interval adds, per running trajectory, a path row [traj_id, s, x, y, z, q0, q1,
 * q2] (pose after the step) and an energy row [traj_id, s, fx, fy, fz, dt] (force of the step).
 * Rows land in device order; up to `cap` of them are copied to path (cap x 8) and energy (cap x 6)
 * host arrays (either may be NULL).  n_rows receives the rows copied, n_dropped the rows that did
 * not fit the trace_capacity of the configuration. */
int bd_sim_traces(BdHandle* h, double* path, double* energy, int64_t cap, int64_t* n_rows, int64_t* n_dropped);
/* No counterpart in the reference: D(r) of the configured stepper (its HI mode and
 * precision, BdSimParams) at n centroid distances r.  Host arrays; for parity tests. */
int bd_sim_hi_diffusion(BdHandle* h, int n, const double* r, double* D);
/* Per-step statistics (BdSimParams.stats = 1) to host arrays.  Replaces the host-side
 * statistics loops of GPUBatchSimulator.run (gpu_batch_simulator.py:1255-1317). */
int bd_sim_stats(BdHandle* h, const BdStatsOut* out);
/* Live-slot count after the last compaction (synchronises the handle's work). */
int bd_sim_live(BdHandle* h, int32_t* n_live);
/* Checkpoint: host copies of the live slots (cap entries each; c: 3*cap, q: 4*cap, SoA)
 * plus counters and outcomes are enough to resume exactly (bd_sim_restore). */
int bd_sim_capacity(BdHandle* h, int32_t* cap);
/* State-machine mode: the per-reaction fire counts since bd_sim_reset, by the discrete test
 * (discrete[n]) and by the Brownian bridge (bridge[n]); replaces the reference's
 * _sm_rxn_fire_counts_discrete / _bridge (gpu_batch_simulator.py:531-541). */
int bd_sim_reaction_fires(BdHandle* h, uint64_t* discrete, uint64_t* bridge, int n);
/* State-machine state of each live slot (cap entries, slot order of bd_sim_snapshot), read
 * after bd_sim_snapshot and written after bd_sim_restore. */
int bd_sim_get_states(BdHandle* h, int8_t* state);
int bd_sim_set_states(BdHandle* h, const int8_t* state);
int bd_sim_snapshot(BdHandle* h, double* c, double* q, int32_t* traj, int32_t* steps, int32_t* rets,
                    int8_t* status, int32_t* n_live, uint64_t* counters);
int bd_sim_restore(BdHandle* h, const double* c, const double* q, const int32_t* traj, const int32_t* steps,
                   const int32_t* rets, const int8_t* status, int32_t n_live, const uint64_t* counters,
                   const int8_t* out_status, const int32_t* out_steps, const int32_t* out_returns);

/* Launch shape: lanes per trajectory (1, 4, 8, 16 or 32: the lanes of a group share one
 * trajectory's whole step) or BD_GROUP_WARP (each lane owns one trajectory's step logic and
 * the warp sweeps each trajectory's atoms together; BD_GROUP_WARP_CAPPED is the same with
 * registers capped at 128 per thread), or BD_GROUP_SPLIT (each BD step as three kernels: the
 * ligand-atom forces, Born direction 2 in a kernel capped at 64 registers, then the rest of the
 * step; the same trajectories as BD_GROUP_WARP), and threads per block (multiple of 32, <= 256).
 * Set by the autotuner; 0 keeps the current value. */
enum { BD_GROUP_WARP = 64, BD_GROUP_WARP_CAPPED = 65, BD_GROUP_SPLIT = 66 };
int bd_set_launch(BdHandle* h, int group, int block_threads);
int bd_get_launch(BdHandle* h, int* group, int* block_threads, int* grid_blocks);

/* Device data layout (bit flags, default BD_LAYOUT_DEFAULT; applied when the device system
 * is next built, i.e. at the next configure or force evaluation):
 * BD_LAYOUT_STAGE_RECEPTOR: the stepper kernels copy an FP32 receptor table of at most
 *   BD_STAGE_MAX_BYTES (atoms + chunk spheres) into each block's shared memory for the
 *   sweeps' distance pre-tests; every accept/reject is still decided in FP64.
 * BD_LAYOUT_WINDOWS_1: each single-channel grid (ligand Born grid, unpaired receptor grids)
 *   gets a float4 copy whose entry n holds nodes n..n+3 of node n's z row, so one force
 *   stencil is 8 vector loads instead of 20 scalar ones (4x the grid's memory).
 * BD_LAYOUT_WINDOWS_2: the interleaved elec+Born grid gets a float4 copy whose entry n holds
 *   both channels of nodes n and n+1: 12 loads per stencil instead of 20 (2x its memory).
 * BD_LAYOUT_CUBES_1: the ligand Born grid gets a copy whose entry n holds the 2x2x2 block of
 *   nodes at node n (32 bytes, one sector; 8x the grid's memory, made only up to
 *   BD_CUBE_MAX_BYTES), so a reverse-Born stencil is three 32-byte loads and one 16-byte load.
 * BD_LAYOUT_OVERLAP_GRID: an occupancy grid of 0.5 A cells over the receptor (one 32-bit word
 *   per cell: no atom within 1.5 A of the cell, every point within 1.5 A of an atom, or a
 *   short list of atoms to test), so the overlap test of a centroid is one load and a few
 *   distances in one lane instead of a warp's sweep of the receptor chunks (made only up to
 *   BD_OVERLAP_MAX_CELLS cells).
 * BD_LAYOUT_XY_1 (with BD_LAYOUT_CUBES_1): the ligand Born grid also gets, per node, four
 *   32-byte records holding the extra x plane and extra y row of a stencil for each cell half
 *   (16x the grid's memory, made only up to BD_XY_MAX_BYTES), so a reverse-Born stencil is three
 *   32-byte loads.
 * BD_LAYOUT_ZTEX_1 (with BD_LAYOUT_CUBES_1): the stencil's extra z nodes come from 16-byte
 *   records read through the texture path instead of a third 32-byte global load (2x the
 *   grid's memory in float4 records).
 * BD_LAYOUT_XYTEX_1 (with BD_LAYOUT_XY_1): the xy records are read through the texture path as
 *   two 16-byte fetches instead of one 32-byte global load.
 * BD_LAYOUT_PTEX_2: the interleaved elec+Born grid gets a float2 texture view, and a forward
 *   stencil reads its eight extra nodes through the texture path (its twelve centre-row nodes
 *   stay global loads).
 * The same values enter the same arithmetic in every layout: results are identical. */
enum {
  BD_LAYOUT_STAGE_RECEPTOR = 1,
  BD_LAYOUT_WINDOWS_1 = 2,
  BD_LAYOUT_WINDOWS_2 = 4,
  BD_LAYOUT_CUBES_1 = 8,
  BD_LAYOUT_OVERLAP_GRID = 16,
  BD_LAYOUT_XY_1 = 32,
  BD_LAYOUT_ZTEX_1 = 64,
  BD_LAYOUT_XYTEX_1 = 128,
  BD_LAYOUT_PTEX_2 = 256
};
#define BD_CUBE_MAX_BYTES (48ll * 1024 * 1024)
#define BD_OVERLAP_MAX_CELLS (32ll * 1024 * 1024)
#define BD_XY_MAX_BYTES (64ll * 1024 * 1024)
#define BD_LAYOUT_DEFAULT \
  (BD_LAYOUT_WINDOWS_1 | BD_LAYOUT_CUBES_1 | BD_LAYOUT_OVERLAP_GRID | BD_LAYOUT_XY_1 | BD_LAYOUT_ZTEX_1)
#define BD_STAGE_MAX_BYTES (64 * 1024)
int bd_set_layout(BdHandle* h, int flags);
int bd_get_layout(BdHandle* h, int* flags);

/* No counterpart in the reference.  Runs p->n_traj trajectories to completion (or for
 * max_launches launches of steps_per_launch steps) on the handle's system WITHOUT
 * allocating device memory, for callers that cannot call cudaMalloc at that point: an
 * application whose allocator already holds the GPU's memory, or a process under a
 * device-memory quota.  The live-slot
 * pool, live counts and counters use a fixed file-scope device array of 9.2 MB, enough for
 * BD_NOALLOC_MAX_SLOTS live slots; p->slots above that is rejected with BD_ERR_ARG
 * (0 = use the maximum).  Outputs are DEVICE arrays the caller owns: out_status,
 * out_steps, out_returns (p->n_traj each, as bd_sim_outcomes) and counters (BD_CTR_NUM).
 * The system must already be on the device (its upload allocates): call bd_sim_configure
 * or an evaluation once before.  The first call on a device looks up the array's device
 * address; make that first call before any stream capture.  Every call shares the array
 * and clears the parts it uses; calls that overlap on the GPU race.  The launch shape is
 * chosen from p (as bd_sim_configure would), not from an earlier configuration.  A handle
 * with a surrogate installed (bd_sim_set_surrogate) is rejected with BD_ERR_STATE.  The
 * per-reaction fire counts of state-machine runs are not returned (bd_sim_reaction_fires
 * reads the regular stepper's counters).  Synchronous: it copies a few words between host
 * and device and waits on `stream`. */
enum { BD_NOALLOC_MAX_SLOTS = 65536 };
int bd_sim_run_noalloc(BdHandle* h, const BdSimParams* p, int8_t* out_status, int32_t* out_steps,
                       int32_t* out_returns, uint64_t* counters, int steps_per_launch, int max_launches,
                       void* stream);

/* ---- Force terms of the evaluation entry points ------------------------------------------
 * No reference counterpart: bit flags choosing which terms bd_eval_forces(_atoms) sum.
 * BD_TERM_GRID: electrostatic and Born direction-1 grid forces on the ligand atoms;
 * BD_TERM_FARFIELD: the Yukawa multipole far-field of atoms outside every electrostatic grid;
 * BD_TERM_REV_BORN: Born direction 2 (ligand Born grid at the receptor atoms);
 * BD_TERM_CONTACT: WCA contact forces (bd_set_contact).  Default: all.
 * The surrogate is trained on the terms it replaces (BdSurrogateParams.terms).  The stepper
 * always sums every term (or the surrogate's share, see bd_sim_set_surrogate). */
enum { BD_TERM_GRID = 1, BD_TERM_FARFIELD = 2, BD_TERM_REV_BORN = 4, BD_TERM_CONTACT = 8, BD_TERM_ALL = 15 };
int bd_set_terms(BdHandle* h, int terms);

/* ---- Surrogate MLP ensemble -------------------------------------------------------------------
 * No reference counterpart: the engine's learned part.  Every member maps in_dim inputs
 * through n_hidden SiLU layers of width `hidden` to out_dim outputs.  BF16 weights and
 * activations, FP32 accumulation on the tensor cores, FP32 biases, master weights and Adam
 * moments.  A parameter vector (FP32, per member) holds, layer by layer, W (out x in,
 * row-major) and then b (out).  Device arrays unless stated; streams follow CUDA (NULL =
 * legacy default stream).  Errors: bd_mlp_last_error. */
typedef struct BdMlp BdMlp;
typedef struct {
  int32_t n_members; /* 1..8 */
  int32_t in_dim;    /* 1..32 */
  int32_t hidden;    /* 128, 256, 384 or 512 */
  int32_t n_hidden;  /* 1..8 */
  int32_t out_dim;   /* 1..32 */
  int32_t reserved;
  uint64_t seed; /* weight initialisation: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) */
} BdMlpDesc;
int bd_mlp_create(int device, const BdMlpDesc* d, BdMlp** out);
int bd_mlp_destroy(BdMlp* m);
int bd_mlp_last_error(const BdMlp* m, char* buf, int len);
int bd_mlp_n_params(const BdMlp* m, int64_t* n);
/* HOST arrays of bd_mlp_n_params floats; set also clears the member's Adam state. */
int bd_mlp_get_params(BdMlp* m, int member, float* params);
int bd_mlp_set_params(BdMlp* m, int member, const float* params);
/* Y (n x out_dim) = member(X (n x in_dim)). */
int bd_mlp_forward(BdMlp* m, int member, int64_t n, const float* X, float* Y, void* stream);
/* Mean squared error over rows and outputs against T (n x out_dim) into *loss (device float,
 * may be NULL) and its gradient into grad (device, parameter layout, may be NULL).
 * n is a positive multiple of 32. */
int bd_mlp_grad(BdMlp* m, int member, int n, const float* X, const float* T, float* grad, float* loss, void* stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected) of one member on a batch. */
int bd_mlp_train_step(BdMlp* m, int member, int n, const float* X, const float* T, float lr, float* loss,
                      void* stream);
/* Inference kernels of bd_mlp_forward / bd_mlp_ensemble and of the surrogate stepper:
 * 1 (default) = tcgen05 MMAs with TMEM accumulators, one CTA per 128 rows running every layer
 * (hidden <= 256, in_dim <= 32, out_dim <= 32; other shapes use 0); 0 = the mma.sync GEMM chain
 * the training kernels use.  Both give the same values up to FP32 summation order. */
int bd_mlp_set_inference(BdMlp* m, int mode);
/* No reference counterpart.  GEMMs of training (forward, weight and activation gradients) and of
 * the GEMM-chain inference: 1 (default) on tcgen05 with TMEM accumulators, 0 on mma.sync.  Both
 * accumulate BF16 products in FP32 with the same fused epilogues. */
int bd_mlp_set_gemm(BdMlp* m, int mode);
/* `steps` Adam steps of one member on random batches (rows drawn with replacement by a
 * counter-based hash of seed, member and step) of device-resident data X (n_data x in_dim),
 * T (n_data x out_dim).  The step is captured once as a CUDA graph and replayed; loss_trace
 * (device, `steps` floats, may be NULL) receives each step's batch loss. */
int bd_mlp_train(BdMlp* m, int member, int64_t n_data, const float* X, const float* T, int batch, int steps,
                 float lr, uint64_t seed, float* loss_trace, void* stream);
/* All members on n rows: mean (n x out_dim) and spread (n x out_dim, RMS deviation of the
 * members from the mean; may be NULL). */
int bd_mlp_ensemble(BdMlp* m, int64_t n, const float* X, float* mean, float* spread, void* stream);

/* Stepper with the surrogate (no reference counterpart).  While set, each BD step of
 * bd_sim_run runs as three phases: every exact force term outside the trust region
 * r_min <= |c| <= r_max and the terms the surrogate does not replace inside it; the ensemble on
 * the trusted poses' features (c / r_scale, |c| / r_scale, q with w >= 0, five Gaussian radial
 * basis values exp(-((|c| - rbf_centre[k]) / rbf_width)^2 / 2)); then the surrogate's share of
 * the force and torque (mean output x out_scale x envelope) where the members agree (spread of
 * the force <= threshold x max(|force|, force_floor x envelope)), the exact kernels for that
 * share elsewhere, and the rest of the step.  `terms` are the BD_TERM_* flags the surrogate
 * replaces: a non-empty subset of BD_TERM_GRID | BD_TERM_FARFIELD | BD_TERM_REV_BORN (0 means
 * BD_TERM_FARFIELD | BD_TERM_REV_BORN); contact forces are always exact.  envelope(|c|) = exp of env_log interpolated linearly over 32 evenly spaced radii
 * from env_r0 to env_r1 (clamped outside), or 1 when env_r1 <= env_r0.  The
 * ensemble needs 13 inputs and 6 outputs (force, torque).  m = NULL returns to the fused
 * exact stepper.  The ensemble must not be used by other calls while the stepper runs, and
 * per-step statistics are not collected in this mode. */
typedef struct {
  double r_scale;
  double rbf_centre[5];
  double rbf_width;
  double out_scale[6];
  double r_min, r_max;
  double threshold;
  double force_floor;
  double env_r0, env_r1;
  double env_log[32];
  int32_t terms;
  int32_t reserved;
} BdSurrogateParams;
int bd_sim_set_surrogate(BdHandle* h, BdMlp* m, const BdSurrogateParams* p);
/* Trusted-pose evaluations and exact fallbacks since configure: out[0], out[1]. */
int bd_sim_surrogate_counters(BdHandle* h, uint64_t* out);

/* ---- Heterogeneous batch -----------------------------------------------------------------
 * No reference counterpart (the reference runs one system per process).  Trajectories of n
 * configured handles (each with its own grids, atoms, reactions and BdSimParams; the same
 * precision and torque mode) share one slot pool and one persistent launch; a slot holds the
 * trajectory's index in the concatenation of the systems' ranges.  Outcomes land in each
 * handle's own arrays (read them with bd_sim_outcomes); the counters are summed over the
 * systems.  The handles must stay configured and unchanged while the batch exists.  Noise keys
 * are each handle's (seed, id_offset + local id, step), so a trajectory runs exactly as it
 * would in its handle's own stepper. */
typedef struct BdMulti BdMulti;
int bd_multi_create(BdHandle* const* handles, int n, BdMulti** out);
int bd_multi_destroy(BdMulti* m);
int bd_multi_last_error(const BdMulti* m, char* buf, int len);
int bd_multi_reset(BdMulti* m, void* stream);
int bd_multi_run(BdMulti* m, int n_launch, int steps_per_launch, void* stream);
int bd_multi_counters(BdMulti* m, uint64_t* out, int n, void* stream);
int bd_multi_live(BdMulti* m, int32_t* n_live);

#ifdef __cplusplus
}
#endif

#endif /* PYSTARC_B200_H */
