/*
 * galaxy_b200.h -- C ABI of libgalaxy_b200.so, a B200 (sm_100a) implementation of
 * galaxy's LBVH Barnes-Hut gravity step.
 *
 * Every entry point is plain C: pointers, sizes and status codes, no C++ or torch
 * types. Every call returns GX_OK (0) or a negative GX_ERR_* code and never aborts
 * the process; the text of the last error of a handle is gx_last_error(handle)
 * (gx_last_error(NULL) for failures that happen before a handle exists).
 *
 * Host arrays are owned by the caller and borrowed for the duration of a call.
 * Positions, velocities and accelerations use the reference's DVec3 layout: 3
 * consecutive f64 per particle (x, y, z), particle-major. Device memory is owned
 * by the handle, grows lazily with N and is released by gx_destroy. A handle is
 * used by one host thread at a time (the reference's `&mut self`).
 *
 * Reference interfaces (paths relative to the reference project root) replaced by
 * these entry points are cited beside each declaration.
 */
#ifndef GALAXY_B200_H
#define GALAXY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------- */
#define GX_OK 0
#define GX_ERR_INVALID_ARG -1   /* bad pointer, size or parameter */
#define GX_ERR_CUDA -2          /* a CUDA runtime call failed (text in gx_last_error) */
#define GX_ERR_NO_DEVICE -3     /* no CUDA device or not an sm_100 part */
#define GX_ERR_BUDGET -4        /* device-memory budget would be exceeded */
#define GX_ERR_STATE -5         /* call out of order (e.g. step before upload) */
#define GX_ERR_DEVICE_CHECK -6  /* a kernel's bounded wait or bounds check tripped */
#define GX_ERR_NOT_FOUND -7     /* unknown system / request id */
#define GX_ERR_CAPACITY -8      /* a fixed-size table is full */
#define GX_ERR_CANCELLED -9     /* the request was cancelled (gx_server_cancel) */

/* ---- options --------------------------------------------------------------- */
#define GX_PREC_F32 0  /* FP32 interactions with Kahan-compensated accumulation (default) */
#define GX_PREC_F64 1  /* FP64 walk in the reference's exact operation order */

#define GX_MULTIPOLE_MONO 0  /* monopole nodes, the reference's approximation (default) */
#define GX_MULTIPOLE_QUAD 1  /* monopole + traceless quadrupole per node */

#define GX_FLAG_NO_KAHAN 1u     /* plain FP32 accumulation in the F32 walk */
#define GX_FLAG_STATS 2u        /* count interactions/openings per call (slower) */
#define GX_FLAG_STAGE_TIMES 4u  /* time each stage with CUDA events (eager launches) */
#define GX_FLAG_MORTON63 8u     /* 63-bit Morton keys (21 bits per axis) instead of the reference's
                                   30-bit keys: the refinement the reference defers
                                   (solvers/src/lbvh.rs:29-32) for dense cores and heavy tails;
                                   changes the tree, so it is not a reference-parity mode */

typedef struct gx_options {
  uint32_t struct_size;    /* sizeof(gx_options); 0 means "all defaults" */
  uint32_t precision;      /* GX_PREC_* */
  uint32_t multipole;      /* GX_MULTIPOLE_* */
  uint32_t flags;          /* GX_FLAG_* */
  int32_t device;          /* CUDA ordinal, -1 = current device */
  uint32_t walk_block;     /* threads per block of the tree walk: 0 = default (128), else a
                              multiple of 32 up to 128 */
  uint32_t walk_ctas_per_sm; /* >0: persistent work-stealing walk with this many CTAs per SM;
                                0: tuned default (one warp per item for a single system) */
  uint32_t walk_group;     /* targets per warp of the FP32 walk: 8, 16 or 32; 0 = the tuning
                              table's entry for the system's N, else a rule of N. It changes
                              the order in which the walk sums its terms (never which terms),
                              so FP32 results can differ in their last bits between groups */
  uint32_t radix_bits;     /* digit width of the radix sort of 30-bit keys: 8 (4 passes) or 10
                              (3 passes); 0 = the tuning table's entry, else 8. The sort is
                              exact: the width never changes a result. 63-bit keys use 8 */
} gx_options;

typedef struct gx_handle gx_handle;

/* Per-call statistics of the most recent force evaluation. */
typedef struct gx_stats {
  uint64_t n;              /* particles */
  uint64_t leaf_interactions;
  uint64_t far_interactions;
  uint64_t nodes_opened;
  uint64_t f64_rechecks;   /* opening decisions re-evaluated in FP64 (guard band) */
  uint64_t warp_node_visits;
  float ms_bbox_morton;    /* stage times of the last call, CUDA events */
  float ms_sort;
  float ms_build;
  float ms_walk;
  float ms_total;
  float ms_sph;            /* gas density + hydro + scatter (gas mode), CUDA events */
  float ms_sph_density;    /* the density part of ms_sph (grids, seeds, root-find) */
} gx_stats;

/* ---- lifecycle ------------------------------------------------------------- */
/* GpuLbvhFused::new / GpuResidentLeapfrog::new / Lbvh::new(g, softening, theta):
 * gpu/src/gpu_lbvh_fused.rs:50, gpu/src/gpu_resident.rs:1292, solvers/src/lbvh.rs:653 */
int gx_create(double g, double softening, double theta, const gx_options* opt, gx_handle** out);
void gx_destroy(gx_handle* h);
const char* gx_last_error(const gx_handle* h);
int gx_device_info(int device, char* name_out, size_t name_len, int* sm_count, int* cc_major, int* cc_minor,
                   size_t* total_mem);
/* Wait until all work on the device has finished (every stream, every handle). A timing
 * helper with no counterpart in the reference. */
int gx_device_synchronize(int device);
/* Failure-detection self-test (no counterpart in the reference): one warp waits, through
 * the same bounded wait as the radix sort's look-back, for a status word nothing ever
 * sets, re-reading it `spins` times. The wait runs out, the kernel raises its error word
 * and returns: the call gives GX_ERR_DEVICE_CHECK with the word in *err_word_out (bit 0:
 * a wait ran out), and the device stays usable. Nothing faults or hangs. */
int gx_selftest_bounded_wait(int device, uint32_t spins, uint32_t* err_word_out);

/* ---- ForceSolver (core/src/traits.rs:27, :95) ------------------------------- */
/* ForceSolver::accelerations -- gpu/src/gpu_lbvh_fused.rs:58-134, solvers/src/lbvh.rs:663-676.
 * acc_out[3n] receives the acceleration of each particle (x G). n == 0 is a no-op,
 * n == 1 yields zero, as in the reference. */
int gx_accelerations(gx_handle* h, size_t n, const double* pos, const double* mass, double* acc_out);
/* Same on device pointers (pos[3n], mass[n], acc_out[3n] f64 in device memory),
 * enqueued on the handle's stream; no host synchronisation. */
int gx_accelerations_device(gx_handle* h, size_t n, const double* d_pos, const double* d_mass, double* d_acc);
/* ForceSolver::accelerations_active (core/src/traits.rs:52-54) and gravity_active_cached
 * (:89-91; Lbvh keeps both defaults: the accelerations of a fresh full pass). For every i in
 * active[0 .. n_active), acc_out[3i .. 3i+2] receives the acceleration gx_accelerations gives
 * particle i (FP64 walk: bit for bit; FP32: within the walk's rounding). The tree is built
 * from all n particles and walked for the active ones only; acc_out entries of inactive
 * particles are left as they are. Indices >= n are GX_ERR_INVALID_ARG; repeats are allowed. */
int gx_accelerations_active(gx_handle* h, size_t n, const double* pos, const double* mass, size_t n_active,
                            const uint32_t* active, double* acc_out);
/* The stale-tree active walk of TreeGravity (solvers/src/barnes_hut.rs:647-711: its
 * rebuild_gravity_cache and gravity_active_cached) over this LBVH, for individual time
 * steps. gx_rebuild_gravity_cache builds the tree of (pos, mass) and keeps it: topology,
 * internal-node aggregates and thresholds, and which leaves are massless.
 * gx_gravity_active_cached then walks that tree for the active targets at the CURRENT
 * positions: targets and leaf sources take pos / mass given here, internal nodes keep the
 * cached aggregates (the reference's "only far cell COMs are stale"). With unchanged
 * positions the result equals gx_accelerations_active. Any other force call or step on
 * the handle replaces the cached tree (GX_ERR_STATE until the next rebuild); n must equal
 * the cached n. */
int gx_rebuild_gravity_cache(gx_handle* h, size_t n, const double* pos, const double* mass);
int gx_gravity_active_cached(gx_handle* h, size_t n, const double* pos, const double* mass, size_t n_active,
                             const uint32_t* active, double* acc_out);
/* ForceSolver::potential_energy -- gpu/src/gpu_lbvh_fused.rs:140-146 delegating to
 * solvers/src/potential.rs:51-58: the exact O(N^2) softened potential, here an FP64
 * GPU reduction. */
int gx_potential_energy(gx_handle* h, size_t n, const double* pos, const double* mass, double* out);
/* FP64 direct summation (solvers/src/direct_sum.rs:25-45 semantics, unpaired) for the
 * listed targets: the force oracle for large systems. targets == NULL means all. */
int gx_direct_sum_f64(gx_handle* h, size_t n, const double* pos, const double* mass, size_t n_targets,
                      const uint32_t* targets, double* acc_out);

/* ---- resident leapfrog (gpu/src/gpu_resident.rs:1685-1960) ------------------- */
/* GpuResidentLeapfrog::upload: copies state to the device and primes a(x0); resets time. */
int gx_upload(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass);
/* GpuResidentLeapfrog::step / step_many: KDK steps of dt, kept on the device. */
int gx_step(gx_handle* h, double dt);
int gx_step_many(gx_handle* h, double dt, uint64_t steps);
/* Enqueue steps without waiting for them (for pipelined callers and CUDA-graph replay). */
int gx_step_many_async(gx_handle* h, double dt, uint64_t steps);
int gx_synchronize(gx_handle* h);
/* GpuResidentLeapfrog::snapshot: pos_out/vel_out[3n] f64 (either may be NULL). */
int gx_snapshot(gx_handle* h, double* pos_out, double* vel_out);
/* The resident accelerations a(x_n) of the current state, acc_out[3n]. */
int gx_resident_accelerations(gx_handle* h, double* acc_out);
int gx_time(const gx_handle* h, double* t_out);                 /* gpu_resident.rs:1947 */
int gx_len(const gx_handle* h, size_t* n_out);                  /* gpu_resident.rs:1960 */
int gx_launches(const gx_handle* h, uint64_t* submits_out);     /* gpu_resident.rs:1955 */
/* Energy and momentum diagnostics of the resident state (core/src/diagnostics.rs:8-68),
 * FP64 on the device. out[8] = {kinetic, potential, px, py, pz, lx, ly, lz}; the O(N^2)
 * potential is skipped (reported as 0) when with_potential == 0. */
int gx_diagnostics(gx_handle* h, int with_potential, double* out);

int gx_get_stats(const gx_handle* h, gx_stats* out);

/* Enqueue `steps` resident steps and return their device time in milliseconds
 * (CUDA events on the handle's stream around the steps). */
int gx_step_many_timed(gx_handle* h, double dt, uint64_t steps, float* ms_out);

/* ---- SPH on the gas subset (solvers/src/sph, gpu/src/gpu_resident.rs:1393-1660) ----
 * Species: kind[i] == 1 is gas (core/src/state.rs:17-22 Species::Gas), 0 collisionless.
 * Gravity acts on every particle; density, smoothing lengths and the hydro force on the
 * gas rows only, as GravitySph (solvers/src/sph/gravity_sph.rs:172-207). The SPH stages
 * run in FP64 in the reference's per-pair operation order; neighbour sums are reduced
 * across a warp, so results agree with the reference to rounding (the CFL bound, a
 * max/min, agrees bit for bit given the same h). */
#define GX_EOS_ISOTHERMAL 0 /* P = c_s^2 rho */
#define GX_EOS_ADIABATIC 1  /* P = (gamma - 1) rho u, c_s = sqrt(gamma (gamma - 1) u) */

/* HydroParams (forces.rs:64-87) + DensityConfig (density.rs:33-51). */
typedef struct gx_sph_params {
  double n_ngb;      /* target kernel-weighted neighbour count (48) */
  double h_tol_rel;  /* bisection tolerance on h (1e-3) */
  int eos;           /* GX_EOS_* (resident gas mode: isothermal only) */
  int warm_start;    /* seed each h bracket from the previous evaluation's h (GravitySph) */
  double c_s;        /* isothermal sound speed (1.0) */
  double gamma;      /* adiabatic index */
  double alpha;      /* Monaghan viscosity, linear (1.0) */
  double beta;       /* Monaghan viscosity, quadratic (2.0) */
  double visc_eps2;  /* mu denominator regulariser (0.01) */
} gx_sph_params;

/* The reference defaults (n_ngb 48, tol 1e-3, isothermal c_s 1, alpha 1, beta 2,
 * eps2 0.01, warm start on). */
void gx_sph_default_params(gx_sph_params* out);
/* GpuResidentLeapfrog::new_with_sph: put the handle in gas mode (params == NULL leaves
 * it). Takes effect at the next gx_upload_species / force call. */
int gx_sph_enable(gx_handle* h, const gx_sph_params* params);
/* GpuResidentLeapfrog::upload of a State with species: kind[n] (NULL: no gas) and the
 * internal energy u[n] (NULL: zero). Builds the gas map (ascending global index) and
 * primes a(x0) = gravity(all) + hydro(gas). */
int gx_upload_species(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                      const uint8_t* kind, const double* u);
int gx_gas_count(const gx_handle* h, size_t* n_gas_out);
/* snapshot_gas_density (gpu_resident.rs:1566): gas map, rho and h of the last force
 * evaluation, in ascending gas index order (any pointer may be NULL). */
int gx_snapshot_gas_density(gx_handle* h, uint32_t* gas_idx_out, double* rho_out, double* h_out);
/* snapshot_gas_accel (gpu_resident.rs:1593): the hydro acceleration alone (before the
 * scatter-add), acc_out[3 n_gas]; dudt_out[n_gas] (nullable) its du/dt partner. */
int gx_snapshot_gas_accel(gx_handle* h, double* acc_out, double* dudt_out);
/* snapshot_accel (gpu_resident.rs:1655): the full acceleration of every particle. */
int gx_snapshot_accel(gx_handle* h, double* acc_out);
/* min_stable_dt (gpu_resident.rs:1614; cfl.rs:49-125): min over gas of c_cfl h_i / v_sig,i
 * reduced on the device, at the current velocities and the last evaluation's h;
 * +inf without gas. snapshot_gas_dt (:1632): the per-gas vector, dt_out[n_gas]. */
int gx_min_stable_dt(gx_handle* h, double c_cfl, double* out);
int gx_snapshot_gas_dt(gx_handle* h, double c_cfl, double* dt_out);

/* Host-state SPH (the resident state is replaced, as by gx_accelerations). */
/* GravitySph::accelerations: gravity on all n, hydro added to the gas rows; h is
 * warm-started across calls while the gas count is unchanged (params.warm_start). */
int gx_sph_accelerations(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                         const uint8_t* kind, const double* u, double* acc_out);
/* GravitySph::accel_and_dudt (gravity_sph.rs:209-245; core/src/traits.rs:37-40): the same
 * accelerations and, in dudt_out[n], the gas rows' du/dt (PdV work + viscous heating,
 * forces.rs:160-172); 0 on collisionless rows. */
int gx_sph_accel_and_dudt(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                          const uint8_t* kind, const double* u, double* acc_out, double* dudt_out);
/* GravitySph::accelerations_active (gravity_sph.rs:247-286, the fresh-gravity path): gravity
 * of all n into acc_out (as gx_sph_accelerations), then density and hydro for the active
 * gas particles only (active[n_active], global indices; non-gas entries are ignored),
 * their hydro added to their rows. The handle keeps the reference's persistent (rho, h)
 * scratch of the gas: h shared with gx_sph_accelerations (its warm start), rho the active
 * path's own; inactive neighbours are read from it (the reference's bounded staleness).
 * While either scratch is unset for this gas count, every gas particle is refreshed. */
int gx_sph_accelerations_active(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                                const uint8_t* kind, const double* u, size_t n_active, const uint32_t* active,
                                double* acc_out);
/* GravitySph::accel_and_dudt_active (gravity_sph.rs:288-319; core/src/traits.rs:63-71):
 * gx_sph_accelerations_active plus dudt_out[n]: zero on every row, then the du/dt of the
 * refreshed gas rows (the active gas, or all gas when the scratch was refreshed). */
int gx_sph_accel_and_dudt_active(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                                 const uint8_t* kind, const double* u, size_t n_active, const uint32_t* active,
                                 double* acc_out, double* dudt_out);
/* The three diagnostics below are &self in the reference: each runs its own cold-start
 * density solve but leaves the warm-start h and the active path's scratch as they were.
 * GravitySph::sf_fields (gravity_sph.rs:353-382): rho_out[n] and div_out[n] (velocity
 * divergence, divergence.rs:34-72) of the gas rows from a cold-start density solve;
 * collisionless rows 0. */
int gx_sph_sf_fields(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                     const uint8_t* kind, double* rho_out, double* div_out);
/* GravitySph::max_stable_dt_per_particle / max_stable_dt (gravity_sph.rs:364-380;
 * cfl.rs:49-185): after a cold-start density solve of the gas, dt_out[n] (nullable) gets
 * c_cfl h_i / v_sig,i on gas rows and +inf elsewhere; *min_out (nullable) its minimum
 * (+inf without gas). The reference's trait methods use c_cfl = 1. */
int gx_sph_max_stable_dt(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                         const uint8_t* kind, const double* u, double c_cfl, double* dt_out, double* min_out);
/* GravitySph::coupled_pairs (cfl.rs:195-228): the gas pairs the force couples, 0 < r <
 * 2 max(h_a, h_b) after a cold-start density solve, as (global a, global b), a < b, in
 * ascending order; up to cap pairs are written to pairs_out[2 cap], *count_out = all. */
int gx_sph_coupled_pairs(gx_handle* h, size_t n, const double* pos, const double* mass, const uint8_t* kind,
                         uint64_t* pairs_out, size_t cap, size_t* count_out);
/* density_adaptive (density.rs:86-96) over n gas particles: rho_out[n], h_out[n];
 * h_init[n] (nullable) seeds the brackets. */
int gx_sph_density(gx_handle* h, size_t n, const double* pos, const double* mass, const double* h_init,
                   double* rho_out, double* h_out);
/* hydro_accel_and_dudt (forces.rs:160-172) with caller rho / h (u nullable). */
int gx_sph_hydro(gx_handle* h, size_t n, const double* pos, const double* vel, const double* mass,
                 const double* rho, const double* hsml, const double* u, double* acc_out, double* dudt_out);
/* The per-particle CFL bound (cfl.rs:134-185 body) with caller h; *min_out (nullable)
 * its minimum. */
int gx_sph_cfl(gx_handle* h, size_t n, const double* pos, const double* vel, const double* hsml, const double* u,
               double c_cfl, double* dt_out, double* min_out);

/* ---- autotuning of the walk launch and the sort (no counterpart in the reference) --
 * The walk's block size, its scheduling (one warp per item over a grid, or a persistent
 * kernel with CTAs per SM stealing items) and, for a single system, its warp grouping
 * (targets per warp) are picked per N bucket (floor(log2 N)) by timing candidates on a
 * resident state: force evaluations only, so the resident state is untouched. A handle
 * whose options fix walk_group is tuned at that grouping only. For 30-bit
 * keys the radix sort's digit width (8 bits, 4 passes; 10 bits, 3 passes) is then picked
 * by timing the sort stage of each. Block size, scheduling and digit width never change a
 * result; the grouping changes the FP32 walk's summation order only. The winner is
 * recorded in a process-wide table keyed by (device, precision, multipole, Morton key
 * width, single system or batch, N bucket); handles and batches created with
 * walk_block == 0 and walk_ctas_per_sm == 0 use the table's entry for their N, and every
 * system (alone or in a batch) created with walk_group == 0 takes the single-system
 * entry's grouping for its own N, so a system's result in a batch equals its result
 * alone. */
typedef struct gx_tuning {
  uint32_t walk_block;       /* threads per block of the walk */
  uint32_t walk_ctas_per_sm; /* 0 = grid of one warp per item; > 0 persistent CTAs per SM */
  uint32_t walk_group;       /* targets per warp (single-system entries; 0 in batch entries) */
  uint32_t radix_bits;       /* digit width of the sort (8 or 10; 8 with 63-bit keys) */
  float ms;                  /* median device time of one force evaluation with it */
  float sort_ms;             /* median device time of the sort stage with radix_bits */
} gx_tuning;
#define GX_TUNE_MAX_CANDIDATES 24
/* Time every candidate `repeats` times (median) on the handle's resident state; best
 * (and, if non-NULL, tried[GX_TUNE_MAX_CANDIDATES] with *n_tried) receive the results. */
int gx_autotune(gx_handle* h, uint32_t repeats, gx_tuning* best, gx_tuning* tried, uint32_t* n_tried);
/* The table's entry for n particles under these options (batched != 0: a batch of n
 * particles in total); GX_ERR_STATE when nothing has been tuned for that bucket. */
int gx_tuning_lookup(int device, size_t n, const gx_options* opt, int batched, gx_tuning* out);

/* LeapfrogKdk::step (core/src/integrator.rs:38-78) on HOST arrays with this handle as
 * the ForceSolver: half kicks and drift on the host in f64 (the reference's operations,
 * on all host threads), accelerations as gx_accelerations (upload of pos and mass,
 * download of acc; positions are sent in chunks as soon as they are drifted). acc[3n]
 * is the integrator's cached acceleration and *primed its `primed` flag. */
int gx_kdk_step_host(gx_handle* h, size_t n, double* pos, double* vel, const double* mass, double* acc,
                     int* primed, double dt);

/* Page-locked host memory (for host buffers whose copies should run at full PCIe/C2C speed). */
int gx_host_alloc(size_t bytes, void** out);
void gx_host_free(void* p);

/* ---- stage entry points for parity tests ------------------------------------- */
/* reference_morton (solvers/src/lbvh.rs:105-129): lanes_out[3n] (may be NULL),
 * codes_out[n], bounds_out[5] = {bmin.x, bmin.y, bmin.z, size, scale} (may be NULL). */
int gx_stage_morton(gx_handle* h, size_t n, const double* pos, uint32_t* lanes_out, uint32_t* codes_out,
                    double* bounds_out);
/* reference_sort (solvers/src/lbvh.rs:143-147): stable permutation by (code, index). */
int gx_stage_sort(gx_handle* h, size_t n, const uint32_t* codes, uint32_t* order_out, uint32_t* sorted_codes_out);
/* reference_karras + reference_aggregate (solvers/src/lbvh.rs:276-348) from sorted
 * codes and the sorted leaf payload. left/right[n-1], parent[2n-1] (unified index:
 * leaves [0,n), internal node i at n+i); aabb_min/aabb_max/com[3(2n-1)], mass[2n-1]
 * f64. quad_out[6(2n-1)] (may be NULL) = traceless quadrupole about each node's com. */
int gx_stage_build(gx_handle* h, size_t n, const uint32_t* sorted_codes, const double* sorted_pos,
                   const double* sorted_mass, uint32_t* left, uint32_t* right, uint32_t* parent, double* aabb_min,
                   double* aabb_max, double* com, double* mass, double* quad_out);

/* ---- sort without device allocation ------------------------------------------- */
/* No counterpart in the reference. For callers that may not allocate device memory
 * (an application that owns every device buffer through its own pool, a real-time
 * loop that must not allocate after start-up, a plugin host that hands over buffers
 * but no allocation rights): the stable (code, index) radix sort of gx_stage_sort on
 * caller-owned DEVICE buffers -- d_codes[n] in, d_sorted_codes[n] and d_order[n] out,
 * the order starting from the identity -- with all working memory in one static
 * device array of the library (about 9 MiB per GPU, held until the process exits).
 * n may not exceed GX_NOALLOC_MAX_KEYS (GX_ERR_CAPACITY otherwise). Enqueued on
 * `stream` (a cudaStream_t; NULL = default stream) and waited for before returning.
 * Calls no cudaMalloc/cudaFree. The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress) and should come before any stream capture;
 * that address is kept for the life of the device's primary context (no calls after a
 * cudaDeviceReset). All calls share the array: calls overlapping on one GPU race and
 * must be serialised by the caller. Errors: gx_last_error(NULL). */
#define GX_NOALLOC_MAX_KEYS (1u << 20)
int gx_sort_noalloc(const uint32_t* d_codes, uint32_t* d_sorted_codes, uint32_t* d_order, size_t n, void* stream);

/* ---- batched systems (one launch per stage over many independent systems) ----- */
typedef struct gx_batch gx_batch;

typedef struct gx_batch_stats {
  uint64_t systems;
  uint64_t particles;
  uint64_t steps;           /* batched steps taken */
  uint64_t bytes_in_use;    /* device bytes held by the batch */
  uint64_t budget_bytes;
  float ms_last_step;
} gx_batch_stats;

/* budget_bytes: device-memory ceiling for system state and scratch (0 = no limit). */
int gx_batch_create(size_t budget_bytes, const gx_options* opt, gx_batch** out);
void gx_batch_destroy(gx_batch* b);
const char* gx_batch_last_error(const gx_batch* b);
/* Add one system (copies its state, primes a(x0)); GX_ERR_BUDGET when over budget. */
int gx_system_add(gx_batch* b, size_t n, const double* pos, const double* vel, const double* mass, double g,
                  double softening, double theta, double dt, uint64_t* id_out);
int gx_system_remove(gx_batch* b, uint64_t id);
/* Bytes a system of n particles would add to the batch. */
int gx_system_bytes(const gx_batch* b, size_t n, size_t* bytes_out);
/* Advance every live system by `steps` KDK steps of its own dt. */
int gx_batch_step(gx_batch* b, uint64_t steps);
int gx_system_snapshot(gx_batch* b, uint64_t id, double* pos_out, double* vel_out, double* time_out);
int gx_system_len(const gx_batch* b, uint64_t id, size_t* n_out);
int gx_batch_stats_get(const gx_batch* b, gx_batch_stats* out);
/* Capture one batched step as a CUDA graph and replay it (1) or launch eagerly (0). */
int gx_batch_set_graph(gx_batch* b, int enable);
/* gx_autotune for a batch: persistent walk candidates timed on the live systems. */
int gx_batch_autotune(gx_batch* b, uint32_t repeats, gx_tuning* best, gx_tuning* tried, uint32_t* n_tried);

/* ---- continuous-batching server ----------------------------------------------- */
/* A stepping thread admits submitted systems in arrival order as the device budget
 * allows (between batched steps, so new requests join systems in flight), keeps every
 * admitted system resident, advances all live systems together one KDK step per
 * iteration and retires each after its steps. A result is bit-identical to running
 * the same system alone. (No counterpart in the reference, which runs one scenario
 * per process: xtask/src/simulate.rs.) */
typedef struct gx_server gx_server;

#define GX_REQ_QUEUED 0
#define GX_REQ_RUNNING 1
#define GX_REQ_DONE 2
#define GX_REQ_REJECTED 3
#define GX_REQ_CANCELLED 4

typedef struct gx_server_stats {
  uint64_t steps;            /* batched steps taken */
  uint64_t particle_steps;   /* sum over steps of live particles */
  uint64_t completed;
  uint64_t queued;
  uint64_t live;
  uint64_t max_live;
  uint64_t bytes_in_use;
  double busy_s;             /* host time spent in batched steps */
  double wall_s;             /* since creation */
  double step_ms_p50;        /* device time per batched step (CUDA events) */
  double step_ms_p99;
  double step_ms_mean;
  double particle_steps_per_s_device;
  double queue_s_p50;        /* submit -> admission delay */
  double queue_s_p99;
} gx_server_stats;

int gx_server_create(size_t budget_bytes, const gx_options* opt, gx_server** out);
void gx_server_destroy(gx_server* s);
const char* gx_server_last_error(const gx_server* s);
/* Copy a scenario in and queue it; thread-safe. */
int gx_server_submit(gx_server* s, size_t n, const double* pos, const double* vel, const double* mass, double g,
                     double softening, double theta, double dt, uint64_t steps, uint64_t* rid_out);
int gx_server_status(gx_server* s, uint64_t rid, int* status_out, uint64_t* steps_done);
/* Block until the request is done (GX_OK) or rejected; GX_ERR_STATE on timeout. */
int gx_server_wait(gx_server* s, uint64_t rid, double timeout_s);
/* Final state of a finished request (pos/vel [3n], time). */
int gx_server_result(gx_server* s, uint64_t rid, double* pos_out, double* vel_out, double* time_out);
int gx_server_release(gx_server* s, uint64_t rid);
int gx_server_stats_get(gx_server* s, gx_server_stats* out);
/* Cancel a request: a queued one leaves the queue, a running one leaves the batch at the
 * next step boundary (the other systems are unaffected); gx_server_wait then returns
 * GX_ERR_CANCELLED. GX_ERR_STATE if it has already finished. */
int gx_server_cancel(gx_server* s, uint64_t rid);
/* Append one JSON line per batched step to `path` (NULL: stop): step, device ms, systems
 * stepped ("live"), their particles, queued requests, completed requests, device bytes in use. */
int gx_server_set_metrics_log(gx_server* s, const char* path);

/* ---- GLXYSNAP v4 snapshots (io/src/snapshot.rs:1-60 layout, :130-199 to_writer) ---
 * Files readable by the reference's io::snapshot::read_file: header (time, step, scale
 * factor 1, softening, n, rng seed, config hash, units, code version) and the SoA
 * columns pos, vel (f64), mass (f32), then the columns the gravity path does not evolve
 * at the reference State's defaults: id = index, progenitor 0, kind collisionless,
 * u = 0, formation time -inf. */
int gx_glxysnap_write(const char* path, double time, uint64_t step, double softening, uint64_t rng_seed,
                      uint64_t config_hash, const char* units, size_t n, const double* pos, const double* vel,
                      const double* mass);

/* Snapshot emission for a served scenario (the reference's snapshot cadence,
 * sim/src/lib.rs:110-170, without a host round trip in the step loop): every `every`
 * steps and after the last one, the system's state is staged on the device (velocities
 * with the owed closing half kick, as gx_server_result), copied on a side stream while
 * the batch steps on, and written by a server thread to
 * "<path_prefix>.<step, 8 digits>.glxysnap". gx_server_wait returns once the request's
 * files are written. */
typedef struct gx_snap_opts {
  uint32_t struct_size;     /* sizeof(gx_snap_opts) */
  uint64_t every;           /* steps between snapshots; 0 = none */
  const char* path_prefix;  /* copied at submit */
  uint64_t rng_seed;        /* header fields */
  uint64_t config_hash;
  const char* units;        /* NULL: "nbody-G1" */
} gx_snap_opts;
int gx_server_submit_snapshots(gx_server* s, size_t n, const double* pos, const double* vel, const double* mass,
                               double g, double softening, double theta, double dt, uint64_t steps,
                               const gx_snap_opts* snap, uint64_t* rid_out);
/* Snapshots written so far for a request; GX_ERR_STATE (text in gx_server_last_error)
 * if one could not be written. */
int gx_server_snapshots_written(gx_server* s, uint64_t rid, uint64_t* written_out);

/* ---- seeded initial conditions (the reference's ic/ crate as input generator) -- */
/* Plummer::sample (ic/src/plummer.rs:94-140): G, total mass M, scale radius a; seed. */
int gx_ic_plummer(size_t n, uint64_t seed, double g, double total_mass, double scale_radius, double* pos,
                  double* vel, double* mass);
/* Composite disk galaxy pair on a parabolic orbit: halo (60% of particles), exponential
 * disk (35%), Hernquist bulge (5%) per galaxy; mass_ratio m2/m1; pericentre in units
 * of the disk scale length; inclinations in degrees. n_total particles. */
int gx_ic_collision(size_t n_total, uint64_t seed, double mass_ratio, double pericentre, double incl1_deg,
                    double incl2_deg, double* pos, double* vel, double* mass);
/* A single disk + halo galaxy (no bulge) of n particles, total mass 1. */
int gx_ic_disk_galaxy(size_t n, uint64_t seed, double* pos, double* vel, double* mass);

#ifdef __cplusplus
}
#endif

#endif /* GALAXY_B200_H */
