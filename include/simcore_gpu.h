/* simcore_gpu.h -- C ABI of the B200 Brownian-dynamics filament step.
 *
 * Drop-in replacement for the two halves of simcore's filament timestep:
 *   - InteractionManager::Interact's pair path (reference
 *     src/interaction_manager.cpp:63-95; declared at
 *     include/simcore/interaction_manager.hpp:72): cell-list rebuild on the
 *     accumulated-displacement rule, segment-segment minimum distance, WCA
 *     forces and torques, scatter onto bond force/torque accumulators;
 *   - FilamentSpecies::UpdatePositions -> Filament::UpdatePosition(bool
 *     midstep) (src/filament_species.cpp:59-85, src/filament.cpp:394-428;
 *     declared at include/simcore/species_base.hpp:29 and
 *     include/simcore/filament.hpp:109): bond-to-site forces, bending and
 *     metric forces, random-force projection, tension solve, midpoint
 *     position update, bond renormalisation.
 * sc_step() runs whole Simulation::RunSimulation steps
 * (src/simulation.cpp:37-62) back to back on the GPU.
 *
 * Conventions: plain C types only; every vector is 3 doubles (z = 0 in 2D);
 * sites and bonds are numbered filament by filament in the order given to
 * sc_add_filaments.  Host arrays are caller owned and copied.  No call
 * exits, throws or aborts: every entry point returns an sc_status, and
 * sc_last_error() describes the last failure of a context.  A context is
 * not thread safe; several contexts may live in one process (there is no
 * static state, unlike the reference's CellList and MinimumDistance). */
#ifndef SIMCORE_GPU_H
#define SIMCORE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SC_OK = 0,
  SC_ERR_INVALID_ARG = 1,   /* bad descriptor, sizes or call order */
  SC_ERR_OOM = 2,           /* device allocation failed */
  SC_ERR_NAN = 3,           /* NaN/Inf in forces or positions */
  SC_ERR_LIST_OVERFLOW = 4, /* pair list larger than its capacity */
  SC_ERR_TIMEOUT = 5,       /* a bounded device wait gave up */
  SC_ERR_CUDA = 6,          /* CUDA runtime error (see sc_last_error) */
  SC_ERR_UNPHYSICAL = 7,    /* accumulated displacement > 10000, as the
                               reference's "Unphysical result"
                               (include/simcore/species.hpp:114-118) */
  SC_ERR_INSERTION = 8,     /* random insertion could not place a filament */
  SC_ERR_NO_DEVICE = 9      /* no usable CUDA device */
} sc_status;

typedef enum {
  /* Every stage in FP64 with the reference's operation order and no FMA
   * contraction: bit-identical to the reference's CPU code. */
  SC_PREC_FP64 = 0,
  /* Pair geometry and WCA forces in FP32 (Kahan-compensated per-bond sums);
   * bending, tension solves and positions stay FP64. */
  SC_PREC_MIXED = 1
} sc_precision;

typedef struct {
  int n_dim;                  /* 2 or 3; every dimension periodic */
  double system_radius;       /* R: box side 2R (system_radius) */
  double delta;               /* delta: one step advances delta/2 */
  double wca_eps;             /* wca_eps */
  double wca_sig;             /* wca_sig; cutoff 2^(1/6) wca_sig */
  double f_cutoff;            /* f_cutoff: cap on |WCA force| */
  int stoch_flag;             /* thermal noise on/off */
  int interaction_flag;       /* pair forces on/off */
  int like_like_interactions; /* 0: filaments do not interact */
  uint32_t seed;              /* Philox key word 0 of the noise streams */
  int precision;              /* sc_precision */
  int device;                 /* CUDA device ordinal */
} sc_system_desc;

typedef struct {
  double length;              /* filament length */
  double persistence_length;  /* bending stiffness in kT units */
  double diameter;
  double min_bond_length;     /* bonds: floor(length/(1.5*min_bond_length)) */
  double friction_ratio;      /* gamma_perp / gamma_par */
} sc_filament_params;

typedef struct {
  int64_t i_step;             /* steps (i_steps) taken */
  int64_t n_rebuilds;         /* rebuild passes (any system) since loading */
  int64_t n_pairs;            /* current candidate pairs */
  int64_t pair_capacity;
  int64_t n_filaments, n_sites, n_bonds;
  int32_t n_cells_1d;
  double cell_length;         /* of system 0 */
  double dr_update;           /* rebuild threshold 0.25 * cell_length^2 (system 0) */
  int64_t kernel_launches;    /* kernels launched by this context */
  int32_t n_replicas;         /* independent systems in the context */
  int64_t n_list_regrowths;   /* pair lists grown after a rebuild outgrew them */
} sc_counters;

typedef struct sc_ctx sc_ctx;

/* Context life cycle.  sc_create = Simulation::InitSimulation's space and
 * interaction set-up (src/simulation.cpp:139-173). */
sc_status sc_create(const sc_system_desc *desc, sc_ctx **out);
sc_status sc_destroy(sc_ctx *ctx);
const char *sc_last_error(const sc_ctx *ctx);

/* Loads all filaments at once (FilamentSpecies with its members in place,
 * src/simulation.cpp:261-405 minus the random insertion): n filaments with
 * their parameters and site positions (n_sites_total x 3 doubles, each
 * filament's sites tail to head).  Builds the initial pair list as the
 * forced update that ends the reference's insertion does.  A filament has at
 * most 511 bonds (the reference's max_length of 500 at min_bond_length
 * 0.666 gives 500). */
sc_status sc_add_filaments(sc_ctx *ctx, int n, const sc_filament_params *p,
                           const double *site_xyz, int64_t n_sites_total);

/* Number of bonds the reference gives a filament (src/filament.cpp:142-147). */
int sc_filament_n_bonds(const sc_filament_params *p);

/* Batched independent systems (replicas) in one context, instead of
 * sc_add_filaments: system r is a periodic box of radius system_radius[r]
 * whose noise key is seed[r] (the desc's radius and seed are not used), with
 * the next n_filaments[r] of the n filaments (parameters p, sites site_xyz,
 * systems back to back).  Every system behaves exactly as a context of its
 * own would: its own cell grid, pair list and rebuilds, decided by its own
 * displacements; every stage of a step runs for all systems in one launch.
 * Pair lists are kept in per-system segments with room for half again their
 * initial length; a list that outgrows its segment is SC_ERR_LIST_OVERFLOW. */
sc_status sc_add_replicas(sc_ctx *ctx, int n_replicas, const double *system_radius,
                          const uint32_t *seed, const int32_t *n_filaments, int n,
                          const sc_filament_params *p, const double *site_xyz,
                          int64_t n_sites_total);
/* Checkpoint of the whole simulation state: positions, previous positions,
 * projected noise, displacement trackers, renormalisation state, each
 * system's pair list with its stored pair forces and per-bond entries,
 * crosslink contributions and the step, midstep and noise counters.  With
 * buf NULL only *size (the bytes needed) is set.  sc_restore loads one into a
 * context holding the same systems (same filaments loaded); the restored
 * context continues bit for bit as the checkpointed one would
 * (the reference's checkpoint cadence, Simulation n_checkpoint). */
sc_status sc_checkpoint(sc_ctx *ctx, void *buf, size_t cap, size_t *size);
sc_status sc_restore(sc_ctx *ctx, const void *buf, size_t size);
/* Noise key (Philox key word 0) of system `replica`, or of every system for
 * -1; the draws continue from the current noise counter. */
sc_status sc_set_noise_key(sc_ctx *ctx, int replica, uint32_t seed);
/* Reference-format output: the filament species' spec and posit files
 * (<run_name>_filament_<species_name>.spec / .posit; with several systems
 * <run_name>_rNNN_... per system), with the reference's headers (n_steps,
 * cadence, delta) and frames (spec: per filament diameter, length, bond
 * length, site count, site positions, bending stiffness, polymerisation
 * state; posit: average position, its scaled image, average orientation,
 * diameter, length).  A cadence of 0 skips that file.  sc_output_write
 * writes the frames due at the current step (i_step % cadence == 0), as
 * OutputManager::WriteOutputs does after every step: the state is
 * snapshotted on the device, copied on a separate stream while the run
 * continues, and written to the file at the next call or at close. */
sc_status sc_output_open(sc_ctx *ctx, const char *run_name, const char *species_name,
                         int n_steps, int n_posit, int n_spec);
sc_status sc_output_write(sc_ctx *ctx);
sc_status sc_output_close(sc_ctx *ctx);
/* Filament analyses on the device, per system.  sc_analysis_sample adds one
 * sample of FilamentSpecies::RunMse2eAnalysis (|head - tail|^2 and its square
 * over the filaments) and RunThetaAnalysis (per joint index i, the histogram
 * of cos(theta_i) = u_i . u_{i+1} in n_bins bins, bin = floor((1 + cos)
 * (n_bins / 2)) clamped to the range; src/filament_species.cpp:569-610).
 * sc_analysis_results gives, per system, the mean-square end-to-end distance
 * and its standard error as FinalizeMse2eAnalysis computes them, the sample
 * count, the joint count per filament of the histograms (max_joints) and the
 * histograms (n_replicas x max_joints x n_bins).  sc_global_order gives the
 * polar order vector (3) and nematic order tensor (9) per system
 * (RunGlobalOrderAnalysis with Filament::GetPolarOrder/GetNematicOrder).
 * Bond orientations are the current ones. */
sc_status sc_analysis_sample(sc_ctx *ctx, int n_bins);
sc_status sc_analysis_results(sc_ctx *ctx, double *mse2e, double *mse2e_err, int64_t *n_samples,
                              int32_t *max_joints, int64_t *theta_hist);
sc_status sc_global_order(sc_ctx *ctx, double *polar, double *nematic);
/* Centre-of-mass diffusion on the device, per system: the reference's
 * diffusion analysis (SpherocylinderSpecies::InitDiffusionAnalysis,
 * DiffusionAnalysis, CalculateMSD, CalculateVCF, FinalizeDiffusionAnalysis,
 * src/spherocylinder_species.cpp:30-134) applied to the filaments' average
 * positions and orientations (Filament::UpdateAvgPosition, src/filament.cpp:
 * 953-968).  sc_diffusion_init(ctx, interval) takes the current averages as
 * time origins and clears the sums; every sc_diffusion_sample adds window
 * point t (0 .. interval-1) of the mean square displacement <|r - r0|^2>
 * and the orientation correlation <u . u0> over each system's filaments,
 * each weighted by the inverse of its variance over the filaments, and
 * after the last point of a window takes new origins.  sc_diffusion_results
 * gives per system and window point (n_replicas x interval) the weighted
 * means and their errors, as FinalizeDiffusionAnalysis computes them.  The
 * sums over filaments run in a fixed order other than the reference's
 * serial one (agreement to rounding). */
sc_status sc_diffusion_init(sc_ctx *ctx, int interval);
sc_status sc_diffusion_sample(sc_ctx *ctx);
sc_status sc_diffusion_results(sc_ctx *ctx, double *msd, double *msd_err, double *vcf,
                               double *vcf_err);
/* Thermo (InteractionManager::CalculatePressure, src/interaction_manager.cpp:
 * 500-517, 535-559, called by Simulation::Statistics every n_thermo steps).
 * sc_set_thermo(ctx, n) makes every step add its pairs' virial -dr x F (each
 * pair's values from its last evaluation, like its force) to a per-system
 * sum, and every step with i_step % n == 0 record the pressure tensor
 * n_bonds/V I + sum/(V n) and the pressure (its trace / n_dim) and reset the
 * sum; the sums start when it is called (call it before the first step for
 * the reference's values) and run inside captured runs too.  n = 0 stops
 * them.  The sums are summed in a fixed order other than the reference's
 * serial one (agreement to rounding; the same bits on every run).
 * sc_thermo_open writes <run_name>.thermo (<run_name>_rNNN.thermo per
 * system) as OutputManager::InitThermo/WriteThermo do: header n_steps,
 * n_thermo, delta, n_dim; per record unit cell (9), pressure tensor (9),
 * pressure, volume.  sc_get_thermo returns and removes up to max_records
 * records: i_step (per record), tensor (9 per record and system, n_dim x
 * n_dim packed), pressure and volume (per record and system); any pointer
 * but n_records may be NULL.  sc_get_potential_energy gives every
 * filament's potential energy of the last pair stage (Object::
 * GetPotentialEnergy: its bonds' pair potentials), with thermo on. */
sc_status sc_set_thermo(sc_ctx *ctx, int n_thermo);
sc_status sc_thermo_open(sc_ctx *ctx, const char *run_name, int n_steps);
sc_status sc_get_thermo(sc_ctx *ctx, int max_records, int *n_records, int64_t *i_step,
                        double *tensor, double *pressure, double *volume);
sc_status sc_get_potential_energy(sc_ctx *ctx, double *pote);
/* Mixed precision only: nearly parallel pairs side by side (FP32
 * |u1 x u2|^2 between 0 and the threshold, 1e-5 by default; the centres'
 * separation along u1 within the two half-lengths plus 0.25; a stored force
 * or a perpendicular separation within 1.5 cutoffs) are evaluated from the
 * FP64 sites, as the FP64 path evaluates them, by the pair kernel's thread
 * that meets them.  FP32 orientations cannot resolve the closest points of
 * such pairs: their torques (and forces) could be off by far more than
 * 1e-5.  On by default; sc_set_exact_near_parallel(ctx, 0) evaluates them in
 * FP32 like every other pair; sc_set_near_parallel_threshold sets the
 * threshold on |u1 x u2|^2 (0 to 1).  No counterpart in the reference, whose
 * pair stage is FP64 throughout. */
sc_status sc_set_exact_near_parallel(sc_ctx *ctx, int on);
sc_status sc_set_near_parallel_threshold(sc_ctx *ctx, double s2);
/* Fast mixed precision only, with the option above switched off (the fused
 * evaluation is FP32 throughout) and without thermo: sc_step
 * and sc_step_graph evaluate each bond's pairs inside the integrator and
 * launch no pair stage.  The results are bit-identical to the separate pair
 * stage, and sc_get_bond_forces still returns the last step's evaluation.
 * Off by default: every bond walks its own pairs one after another, and on
 * workload B the fused integrator (58.5 us) is slower than the pair stage
 * and the integrator together (54.9 us).  No counterpart in the
 * reference. */
sc_status sc_set_fused_pairs(sc_ctx *ctx, int on);
/* Per-system rebuild counts and current pair counts (n_replicas entries
 * each; either pointer may be NULL). */
sc_status sc_get_replica_counters(sc_ctx *ctx, int64_t *n_rebuilds, int64_t *n_pairs);

/* Static doubly-bound crosslinks: n harmonic tethers between sites site_a[k]
 * and site_b[k] (global site indices), force k_spring (|dr| - rest_length)
 * along the minimum-image separation of the two anchors, k_spring_compress
 * instead when compressed and k_spring_compress >= 0 (Crosslink::
 * CalculateTetherForces, src/crosslink.cpp:247-275).  An anchor on site j
 * sits at the tail of bond j; on a filament's last site, at the head of the
 * last bond.  Forces and torques go to the anchors' bonds
 * (Anchor::ApplyAnchorForces, src/anchor.cpp:132-146), recomputed on even
 * steps and re-applied unchanged on odd steps (CrosslinkSpecies::
 * UpdatePositions, src/crosslink_species.cpp:218-238).  Active only with
 * interaction_flag on, as the reference's Interact returns early otherwise.
 * Once, after sc_add_filaments and before the first step. */
sc_status sc_add_crosslinks(sc_ctx *ctx, int n, const int32_t *site_a,
                            const int32_t *site_b, double k_spring,
                            double k_spring_compress, double rest_length);
/* Tether force of every link from its last recomputation (n x 3; anchor 0
 * receives +F, anchor 1 -F). */
sc_status sc_get_crosslink_forces(sc_ctx *ctx, double *f);

/* InteractionManager::Interact for the next step: rebuild check, pair
 * forces and torques into the device bond accumulators. */
sc_status sc_interact(sc_ctx *ctx);
/* FilamentSpecies::UpdatePositions: one integrator (half) step of every
 * filament from the bond accumulators; toggles the midstep flag. */
sc_status sc_update_positions(sc_ctx *ctx);
/* n reference steps (Simulation::RunSimulation bodies), each a pair-force
 * kernel and an integrator kernel.  Bit-identical to n x (sc_interact +
 * sc_update_positions). */
sc_status sc_step(sc_ctx *ctx, int n);
/* Same as sc_step, replaying a captured CUDA graph of n steps. */
sc_status sc_step_graph(sc_ctx *ctx, int n);
/* Waits for the context's stream and reports any deferred device error. */
sc_status sc_synchronize(sc_ctx *ctx);

/* Host copies of state (caller-sized arrays). */
sc_status sc_get_sites(sc_ctx *ctx, double *xyz);            /* N_s x 3 */
sc_status sc_set_sites(sc_ctx *ctx, const double *xyz);      /* N_s x 3 */
sc_status sc_get_prev_sites(sc_ctx *ctx, double *xyz);       /* N_s x 3 */
sc_status sc_get_random_forces(sc_ctx *ctx, double *f);      /* N_s x 3 */
sc_status sc_get_bond_forces(sc_ctx *ctx, double *f, double *t); /* N_b x 3 */
sc_status sc_get_bond_geometry(sc_ctx *ctx, double *pos, double *spos,
                               double *u, double *len);
/* Integrator variant of the mixed-precision step: 1 (default) uses FMA
 * contraction, one reciprocal per shared denominator and rsqrt
 * normalisation; 0 runs the exact FP64 integrator of SC_PREC_FP64.  No
 * effect in SC_PREC_FP64, which is always exact. */
sc_status sc_set_fast_integrator(sc_ctx *ctx, int on);
/* Integrator layout, a tuning knob (every layout gives the same results):
 * filaments of at most warp_max_sites sites (<= 32) run on the
 * warp-synchronous kernel, one warp per group of whole filaments; longer
 * ones on the block kernel, block_sites sites per block (a multiple of 32 up
 * to 512, at least the longest such filament; 0 picks 128, 256 or 512).
 * warp_max_sites 0 puts every filament on the block kernel. */
sc_status sc_set_integrator_layout(sc_ctx *ctx, int warp_max_sites, int block_sites);
/* Autotuner for the layout above: times every candidate on the context's
 * own state (saved and restored, so the simulation is unchanged), applies
 * the fastest and reports it.  With cache_path (may be NULL) the choice is
 * read from, or appended to, that text file under a key of device, precision,
 * filament count and site range, so a later context of the same shape skips
 * the timing. */
sc_status sc_autotune(sc_ctx *ctx, const char *cache_path, int *warp_max_sites,
                      int *block_sites);
/* Site forces and tensions of the last integrator step; recorded only while
 * capture is on (sc_set_capture(ctx, 1)), since they are not state. */
sc_status sc_set_capture(sc_ctx *ctx, int on);
sc_status sc_get_site_forces(sc_ctx *ctx, double *f);        /* N_s x 3 */
sc_status sc_get_tensions(sc_ctx *ctx, double *t);           /* N_b */
sc_status sc_get_filament_state(sc_ctx *ctx, int *normalize_switch,
                                int *n_normalize);           /* N_f each */
/* Accumulated squared displacement per site since the last rebuild
 * (Object::dr_tot_).  The GPU adds a full step's contribution in that step
 * itself; the reference adds it at the following step's rebuild check, so
 * the two agree after every odd number of steps. */
sc_status sc_get_dr_tot(sc_ctx *ctx, double *dr);            /* N_s */
/* Current pair list as (obj1, obj2) global bond ids, in the reference's
 * list order; *n_pairs receives the count, at most cap pairs written. */
sc_status sc_get_pairs(sc_ctx *ctx, int32_t *pairs, int64_t cap,
                       int64_t *n_pairs);
/* Cell (x, y, z) of every bond from its current scaled position
 * (CellList::FindCellCoords, src/cell_list.cpp:139-157). */
sc_status sc_get_bond_cells(sc_ctx *ctx, int32_t *xyz);
sc_status sc_get_counters(sc_ctx *ctx, sc_counters *out);
/* The cudaStream_t all work of the context is issued on. */
void *sc_get_stream(sc_ctx *ctx);
/* Per-launch CUDA-event timing of the pair-force and integrator kernels
 * launched by host-driven calls (sc_step, sc_interact, sc_update_positions);
 * the total and the number of timed launches since timing was (re)switched
 * on. */
sc_status sc_set_kernel_timing(sc_ctx *ctx, int on);
sc_status sc_get_kernel_timing(sc_ctx *ctx, double *total_ms, int64_t *launches);
/* Device time (CUDA events on the context's stream) of the graph launch of
 * the last sc_step_graph call, in ms. */
sc_status sc_get_graph_time(sc_ctx *ctx, double *ms);

/* Pair forces for callers that cannot allocate device memory.
 *
 * No counterpart in the reference.  Some callers cannot call cudaMalloc:
 * an application whose device memory belongs to its own pool or caching
 * allocator, which must not be grown or fragmented behind its back, or one
 * that runs under a fixed device-memory budget reserved at start-up (a
 * solver embedded in a larger code, a real-time controller).  This
 * entry point computes, for a configuration in the caller's device buffers,
 * the bond forces and torques that the first Interact after a pair-list
 * rebuild produces (fresh pairs, FP64, bit-identical to sc_interact on a
 * context just loaded with the same sites), without allocating anything: its
 * scratch is a fixed array inside the library (SC_NOALLOC_SCRATCH_BYTES,
 * held by every GPU that loads the library until the process exits).
 *
 *   species         min_bond_length and diameter (they set the cell size)
 *   d_site_offsets  device, n_filaments + 1 int32 site offsets (first 0)
 *   d_site_xyz      device, n_sites x 3 doubles (z = 0 in 2D)
 *   d_bond_force    device, n_bonds x 3 doubles (output)
 *   d_bond_torque   device, n_bonds x 3 doubles (output)
 *   stream          cudaStream_t the work is issued on (0: legacy stream)
 *
 * Limits: at most SC_NOALLOC_MAX_BONDS bonds and filaments, a cell grid of
 * at most SC_NOALLOC_MAX_CELLS cells (at most 50 cells a side in 3D, 362 in
 * 2D, with the cell length of the species), at most SC_NOALLOC_MAX_PAIRS
 * candidate pairs; larger inputs, or a radius that is not finite, return
 * SC_ERR_INVALID_ARG (sizes, cells) or SC_ERR_LIST_OVERFLOW (pairs).  Site
 * offsets that do not rise from 0 by at least 2 sites a filament return
 * SC_ERR_INVALID_ARG (checked on the device, where they are; nothing is
 * written outside the scratch).  The call reads the last site offset back
 * and synchronises the stream, so it must be made outside stream capture.
 * The first call on a device (and the first after a cudaDeviceReset, which
 * makes a new context) looks up the scratch address with
 * cudaGetSymbolAddress.  All calls on a device share the scratch and leave
 * their data in it; calls whose GPU work overlaps race and must be
 * serialised by the caller. */
#define SC_NOALLOC_MAX_BONDS 8192
#define SC_NOALLOC_MAX_CELLS 131072
#define SC_NOALLOC_MAX_PAIRS 32768
#define SC_NOALLOC_SCRATCH_BYTES 8882432 /* 8.5 MiB per GPU */
sc_status sc_pair_forces_noalloc(const sc_system_desc *desc,
                                 const sc_filament_params *species, int n_filaments,
                                 const int32_t *d_site_offsets, const double *d_site_xyz,
                                 double *d_bond_force, double *d_bond_torque,
                                 void *stream);

/* Seeded random insertion with overlap rejection on the host (the
 * distributions of Mesh::InitRandomBond and Filament::InsertFilament,
 * src/mesh.cpp:244-258, src/filament.cpp:225-249,350-383, rejection of
 * InteractionManager::CheckOverlap, src/interaction_manager.cpp:561-571).
 * insertion_type follows the filament species' insertion_type
 * (Filament::InsertFirstBond, src/filament.cpp:192-222): SC_INSERT_RANDOM
 * draws an isotropic first bond and later bonds from the bending
 * distribution; SC_INSERT_RANDOM_NEMATIC / _POLAR place straight filaments
 * along -+z / +z (y in 2D).  Writes sum(n_bonds[i] + 1) x 3 doubles. */
enum { SC_INSERT_RANDOM = 0, SC_INSERT_RANDOM_NEMATIC = 1, SC_INSERT_RANDOM_POLAR = 2 };
int sc_insert_filaments(int n_dim, double system_radius, uint64_t seed,
                        int n_fil, const int *n_bonds, const double *length,
                        const double *persistence_length, double diameter,
                        int insertion_type, int max_attempts, double *site_xyz);
/* The same insertion with the overlap tests on GPU `device`: the result is
 * sc_insert_filaments' for the same arguments, bit for bit.  Candidates of
 * the next filaments are drawn on the host at the stream positions they
 * take if every earlier one succeeds; the GPU tests each candidate bond
 * against the accepted bonds and the earlier candidates of the batch, and
 * the candidates before the first one that overlaps are accepted.  No
 * counterpart beyond the reference's insertion (src/simulation.cpp:261-405),
 * which runs serially. */
int sc_insert_filaments_gpu(int device, int n_dim, double system_radius, uint64_t seed,
                            int n_fil, const int *n_bonds, const double *length,
                            const double *persistence_length, double diameter,
                            int insertion_type, int max_attempts, double *site_xyz);

#ifdef __cplusplus
}
#endif
#endif
