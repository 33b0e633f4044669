/*
 * pmc_coag_gpu.h -- C ABI of the B200 coagulation library (libpmc_coag_gpu.so).
 *
 * This is the drop-in boundary for PartMC's particle-resolved coagulation
 * step.  The reference calls
 *     mc_coag(coag_kernel_type, env_state, aero_data, aero_state, del_t,
 *             tot_n_samp, tot_n_coag)                (src/coagulation.F90:43-59)
 * from run_part_timestep (src/run_part.F90:917-931).  A Fortran module with
 * bind(c) interfaces maps that call onto
 * pmc_coag_gpu_step(); the particle state lives on the GPU between calls and
 * is synchronised with aero_state_t only when another process needs it.
 *
 * Conventions
 *  - Every function returns a status code (PMC_OK = 0), following the int
 *    status pattern of the reference's C RNG wrapper (src/rand_gsl.c:80-152,
 *    checked by rand_check_gsl in src/rand.F90:38-58).  The reference instead
 *    stops the program (die_msg / assert, src/util.F90:103-143).
 *  - Species volumes are passed as the reference stores them: n_spec values
 *    per particle, particle-major (Fortran vol(n_spec) per particle), i.e.
 *    vol[i * n_spec + s].
 *  - Groups and classes are 1-based, as in aero_particle_t (aero_particle.F90:34-36).
 *  - Weights are n_group x n_class arrays, entry (g, c) at (g-1) + n_group*(c-1),
 *    the layout of aero_weight_array_t%weight (aero_weight_array.F90:35-39).
 *  - No entry point takes ownership of caller memory.  All pointers are host
 *    pointers unless a name says _dev.
 */
#ifndef PMC_COAG_GPU_H
#define PMC_COAG_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PMC_OK 0
#define PMC_ERR_INVALID_ARG 1
#define PMC_ERR_OUT_OF_GRID 2     /* die_msg(765620746 / 134572570), coagulation.F90:561-565 */
#define PMC_ERR_CAPACITY 3        /* particle capacity or bin limit exceeded */
#define PMC_ERR_CUDA 4            /* a CUDA runtime call failed */
#define PMC_ERR_TIMEOUT 5         /* a bounded device loop ran out of iterations */
#define PMC_ERR_RNG_EXHAUSTED 6   /* replay stream shorter than the draws needed */
#define PMC_ERR_ASSERT 7          /* a reference assert() condition failed */
#define PMC_ERR_NO_DEVICE 8

/* kernel types, coag_kernel.F90:29-45 */
#define PMC_KERNEL_SEDI 1
#define PMC_KERNEL_ADDITIVE 2
#define PMC_KERNEL_CONSTANT 3
#define PMC_KERNEL_BROWN 4
#define PMC_KERNEL_ZERO 5
#define PMC_KERNEL_BROWN_FREE 6  /* coag_kernel_brown_free.F90, with the context's fractal parameters */
#define PMC_KERNEL_BROWN_CONT 7  /* coag_kernel_brown_cont.F90, with the context's fractal parameters */

/* aerosol mode types, aero_mode.F90:31-37 */
#define PMC_AERO_MODE_LOG_NORMAL 1
#define PMC_AERO_MODE_EXP 2
#define PMC_AERO_MODE_MONO 3
#define PMC_AERO_MODE_SAMPLED 4

/* weight types, aero_weight.F90:24-30 */
#define PMC_WEIGHT_NONE 1
#define PMC_WEIGHT_POWER 2
#define PMC_WEIGHT_MFA 3

/* execution modes */
#define PMC_MODE_FP64 0   /* parallel pair tests in FP64 */
#define PMC_MODE_MIXED 1  /* FP32 kernel evaluation and accept test; FP64 k_max, merges, sums */
#define PMC_MODE_REPLAY 2 /* one device thread runs the reference's sequential order on a given uniform stream */

typedef struct pmc_coag_gpu_ctx pmc_coag_gpu_ctx;

/* Create a context holding one particle population.  Replaces the state
 * set-up the reference does with aero_data_t (density, aero_data.F90), the
 * weight array (aero_state_set_weight, aero_state.F90:184-235) and the RNG
 * seed (pmc_srand, rand.F90:66-113).  i_water is the 1-based water species
 * (0 if none), used only when merging frozen particles. */
int pmc_coag_gpu_init(int n_spec, const double *density, int i_water,
                      int n_group, int n_class, const int *w_type,
                      const double *w_mag, const double *w_exp, uint64_t seed,
                      pmc_coag_gpu_ctx **ctx);

/* Create a context holding n_pop independent populations that share species,
 * weights' shape and kernel, and advance together (batched mode). */
int pmc_coag_gpu_init_batch(int n_pop, int n_spec, const double *density,
                            int i_water, int n_group, int n_class,
                            const int *w_type, const double *w_mag,
                            const double *w_exp, const uint64_t *seeds,
                            pmc_coag_gpu_ctx **ctx);

int pmc_coag_gpu_destroy(pmc_coag_gpu_ctx *ctx);

/* Replace the whole particle list of population `pop` (0-based; 0 for a
 * one-population context).  Equivalent to filling aero_state%apa and
 * clearing aero_state%valid_sort (aero_state.F90:69-84).  Optional arrays may
 * be NULL: group/cls default to 1, id to consecutive values from the
 * context's next id, n_primary to 1.  Components default to one component
 * with source 1 and create time 0 (aero_particle_set_component,
 * aero_particle.F90:186-200). */
int pmc_coag_gpu_upload(pmc_coag_gpu_ctx *ctx, int pop, int n_part,
                        const double *vol, const int *group, const int *cls,
                        const int64_t *id, const int *n_primary);

/* Components of the uploaded particles: n_comp[i] <= 20, comp_source and
 * comp_create_time are 20 entries per particle (aero_particle_t%component,
 * aero_particle.F90:54). */
int pmc_coag_gpu_upload_components(pmc_coag_gpu_ctx *ctx, int pop, int n_part,
                                   const int *n_comp, const int *comp_source,
                                   const double *comp_create_time);

/* The mc_coag drop-in (coagulation.F90:43-96): advance the population(s) by
 * one coagulation step of length del_t.  tot_n_samp / tot_n_coag receive the
 * reference's counters (summed over populations in a batched context). */
int pmc_coag_gpu_step(pmc_coag_gpu_ctx *ctx, int kernel_type, double temp,
                      double pressure, double additive_coeff, double del_t,
                      int *tot_n_samp, int *tot_n_coag);

/* Batched form: temp[pop], pressure[pop] per population, n_steps steps, the
 * counters summed over populations and steps. */
int pmc_coag_gpu_step_batch(pmc_coag_gpu_ctx *ctx, int kernel_type,
                            const double *temp, const double *pressure,
                            double additive_coeff, double del_t, int n_steps,
                            int64_t *tot_n_samp, int64_t *tot_n_coag);

/* Number of particles of population `pop` (aero_state_n_part). */
int pmc_coag_gpu_n_part(pmc_coag_gpu_ctx *ctx, int pop, int *n_part);

/* Copy population `pop` back to the host (aero_state%apa).  Arrays sized for
 * max_part particles; any pointer may be NULL. */
int pmc_coag_gpu_download(pmc_coag_gpu_ctx *ctx, int pop, int max_part,
                          double *vol, int *group, int *cls, int64_t *id,
                          int *n_primary, int *n_part);
int pmc_coag_gpu_download_components(pmc_coag_gpu_ctx *ctx, int pop,
                                     int max_part, int *n_comp,
                                     int *comp_source,
                                     double *comp_create_time);

/* Keep a host copy of population `pop` current, slot by slot.  The host
 * arrays have room for `cap` slots (vol: cap x n_spec, particle-major; the
 * others: cap entries); alive[] marks the live slots, and the live slots in
 * increasing order are the particles, in the order pmc_coag_gpu_download
 * returns them.  Only slots written since the previous call are copied (and
 * scattered into the arrays by the library).  Every slot is copied when *full
 * is nonzero on entry (new or regrown host arrays), and on the first call
 * after an upload or after the library compacted its slots; *full is 1 on
 * return when that happened.  *n_slots: slots in use (PMC_ERR_CAPACITY,
 * nothing copied, if above cap); *n_changed: slots copied.  This serves the reference's ownership of aero_state
 * (aero_state.F90:69-84: the host reads the particle list after mc_coag)
 * without moving the unchanged particles across the bus every step. */
int pmc_coag_gpu_sync_host(pmc_coag_gpu_ctx *ctx, int pop, int cap,
                           double *vol, int *group, int *cls, int64_t *id,
                           int *n_primary, uint8_t *alive, int *n_slots,
                           int *n_changed, int *full);

/* Particle shape of aero_data (fractal_t, fractal.F90:59-66), as
 * spec_file_read_fractal sets it from the spec file's do_fractal, frac_dim,
 * prime_radius and vol_fill_factor (fractal.F90:550-593).  Every radius
 * then follows fractal_vol2rad / fractal_rad2vol (bins, weights, k_max
 * bounds), the Brownian and sedimentation kernels use the mobility radius
 * of fractal_vol_to_mobility_rad (fractal.F90:315-362), and the free
 * molecular and continuum kernels the number of monomers.  d_f = 3 and f = 1
 * are spherical particles (the default, fractal_set_spherical).  Returns
 * PMC_ERR_INVALID_ARG for d_f outside (0, 3] (the reference stops for
 * d_f > 3) or a non-positive R0 or f.  The next step re-sorts every
 * population and recomputes its k_max bounds. */
int pmc_coag_gpu_set_fractal(pmc_coag_gpu_ctx *ctx, double frac_dim,
                             double prime_radius, double vol_fill_factor);

/* New weight magnitudes/exponents, e.g. after aero_state_rebalance doubles or
 * halves a group (aero_state.F90:1722-1852).  Invalidates the sort. */
int pmc_coag_gpu_set_weight(pmc_coag_gpu_ctx *ctx, const int *w_type,
                            const double *w_mag, const double *w_exp);

/* Weights of one population of a batched context (same shape as the
 * context's weights); each population keeps its own magnitudes, as separate
 * aero_state_t instances do. */
int pmc_coag_gpu_set_weight_pop(pmc_coag_gpu_ctx *ctx, int pop,
                                const int *w_type, const double *w_mag,
                                const double *w_exp);

/* aero_state_rebalance (aero_state.F90:1797-1852) for population `pop`,
 * called by run_part after every step (run_part.F90:982).  While a weight
 * (group, class) holds fewer than n_part_ideal/2 particles, and at least
 * one, it is doubled (aero_state_double, :1722-1746: every member copied
 * with a new ID, the weight magnitude halved); while it holds more than
 * 2*n_part_ideal it is halved (aero_state_halve, :1749-1783: each member
 * removed with probability 1/2, the magnitude doubled).  n_part_ideal is
 * n_group x n_class (aero_state%n_part_ideal).  The population then has
 * weights of its own (read them back with pmc_coag_gpu_get_weight). */
int pmc_coag_gpu_rebalance(pmc_coag_gpu_ctx *ctx, int pop,
                           const double *n_part_ideal, int allow_doubling,
                           int allow_halving);

/* Autotuning of the step's launch shapes (no counterpart in the reference).
 * Five launch sites have a threads-per-block choice: the pair tests, the
 * merge decisions and claim resolution, the walks, the chains, and the
 * apply.  pmc_coag_gpu_autotune(ctx, 1) makes the context's next steps
 * (ordinary pmc_coag_gpu_step / _step_batch calls) a coordinate search over
 * those choices: each site in turn tries its PMC_TUNE_CANDIDATES shapes for
 * PMC_TUNE_REPS steps each and keeps the best before moving on.  A shape's
 * score is the device time of the site's launches (CUDA events on the
 * library's stream) per million pair tests of its steps; during the search
 * the later rounds run from the host loop instead of the CUDA graph, so
 * that each launch can be timed.  The search takes PMC_TUNE_SITES *
 * PMC_TUNE_CANDIDATES * PMC_TUNE_REPS steps.  The particles do not depend
 * on the shapes or on the loop, so these steps are the caller's own.
 * pmc_coag_gpu_tune_state reports whether the search is still running, the
 * shapes in use (threads[PMC_TUNE_SITES]) and the scores
 * (ms[site * PMC_TUNE_CANDIDATES + candidate], 0 where not yet measured);
 * either pointer may be NULL.  pmc_coag_gpu_set_tune sets shapes
 * found earlier (each must be one of the site's candidates: 64, 128 or 256
 * threads, 32, 64 or 128 for the chains) and stops a search. */
#define PMC_TUNE_SITES 5
#define PMC_TUNE_CANDIDATES 3
#define PMC_TUNE_REPS 3
int pmc_coag_gpu_autotune(pmc_coag_gpu_ctx *ctx, int enable);
int pmc_coag_gpu_tune_state(pmc_coag_gpu_ctx *ctx, int *tuning, int *threads,
                            float *ms);
int pmc_coag_gpu_set_tune(pmc_coag_gpu_ctx *ctx, const int *threads);

/* aero_state_add_aero_dist_sample (aero_state.F90:758-831) on the device:
 * add a Poisson sample of a distribution of n_mode modes to population
 * `pop`, with the given sample proportion, characteristic factor and
 * creation time.  For every weight group and then every mode, in the
 * reference's order, the mode's expected number of computational particles
 * is sample_prop * aero_mode_number (aero_mode.F90:495-546) under the weight
 * of (group, class); the class is the mode's source when the context has
 * more than one class, else 1 (aero_state_weight_class_for_source,
 * aero_state.F90:263-282).  With n_part_ideal (n_group x n_class, the
 * layout of the weights; NULL skips this) the weight is first prepared as
 * aero_state_prepare_weight_for_add does (:704-752): if the members of
 * (group, class) plus the expected new ones fall outside [ideal/2, 2 ideal],
 * the weight is scaled to bring them to ideal, halving (a uniform random
 * subset removed, recorded as AERO_INFO_HALVED) or doubling (each member
 * copied to prob_round(1/ratio) particles) the members as
 * aero_state_scale_weight does (:1859-1922) when allow_halving /
 * allow_doubling permit it or the group is empty.  Each particle's radius
 * comes from aero_mode_sample_radius (aero_mode.F90:550-630; log-normal
 * draws truncated at min(1 / (characteristic_factor * mean), 0.32)), its
 * volume from the context's particle shape (aero_data_rad2vol), its species
 * volumes from aero_mode_sample_vols (:633-665); it gets a new ID, one
 * component (source, create_time) and one primary particle.
 * Mode arrays, one entry per mode: mode_type (PMC_AERO_MODE_*),
 * char_radius (m), log10_std (log10 of the geometric standard deviation;
 * log-normal modes, may be NULL otherwise), num_conc (m^-3), vol_frac and
 * vol_frac_std (n_mode x n_spec, mode-major; vol_frac_std may be NULL for
 * all zero), source (1-based; NULL: mode m has source m + 1, one source per
 * named mode as aero_mode_read assigns them).  Sampled modes: n_sample[m]
 * intervals, their n_sample[m] + 1 radius edges (m) concatenated over the
 * sampled modes in sample_radius, their number concentrations (m^-3)
 * concatenated in sample_num_conc; n_sample may be NULL when no mode is
 * sampled.  n_part_add (may be NULL) receives the number of particles
 * added.  Exponential modes need flat weights (die_msg(822252601) in the
 * reference).  The draws come from the population's counter-based stream,
 * keyed by its seed, its step count and the call. */
int pmc_coag_gpu_add_dist_sample(pmc_coag_gpu_ctx *ctx, int pop, int n_mode,
                                 const int *mode_type,
                                 const double *char_radius,
                                 const double *log10_std,
                                 const double *num_conc,
                                 const double *vol_frac,
                                 const double *vol_frac_std,
                                 const int *source, const int *n_sample,
                                 const double *sample_radius,
                                 const double *sample_num_conc,
                                 double sample_prop,
                                 double characteristic_factor,
                                 double create_time,
                                 const double *n_part_ideal,
                                 int allow_doubling, int allow_halving,
                                 int64_t *n_part_add);

/* Size distributions of population `pop` without a download: the
 * reference's aero_state diameter histograms (extract_aero_size.F90:132-138,
 * bin_grid_histogram_1d, bin_grid.F90:225-248) on a log grid of n_bin
 * diameter bins from d_min to d_max (m).  Each particle counts with its
 * number concentration, divided by the bin's log width: num_dist[b] in
 * m^-3 per unit ln(D); mass_dist (may be NULL) [b * n_spec + s] in kg m^-3
 * per unit ln(D), per species (their sum is the mass distribution).
 * Particles outside the grid are not counted.  n_bin * (1 + n_spec) <= 12288.
 * The per-bin sums are accumulated in an order that varies from call to
 * call (differences at the level of rounding). */
int pmc_coag_gpu_size_dist(pmc_coag_gpu_ctx *ctx, int pop, int n_bin,
                           double d_min, double d_max, double *num_dist,
                           double *mass_dist);

/* The weight magnitudes population `pop` uses now (n_group x n_class),
 * aero_weight_array_t%weight(:,:)%magnitude (aero_weight_array.F90:35-39). */
int pmc_coag_gpu_get_weight(pmc_coag_gpu_ctx *ctx, int pop, double *w_mag);

/* The ID counter (next_id, aero_particle.F90:72, new_id :157-165). */
int pmc_coag_gpu_set_next_id(pmc_coag_gpu_ctx *ctx, int pop, int64_t next_id);
int pmc_coag_gpu_get_next_id(pmc_coag_gpu_ctx *ctx, int pop, int64_t *next_id);

/* PMC_MODE_FP64 (default), PMC_MODE_MIXED or PMC_MODE_REPLAY. */
int pmc_coag_gpu_set_mode(pmc_coag_gpu_ctx *ctx, int mode);

/* Run the later rounds of a step (every round after the first: retried
 * events, walks of the particles the step made, chains) as one CUDA graph
 * whose loop condition is set on the device (enable = 1, the default), or
 * from a host loop (enable = 0).  Both give the same particles, bit for bit.
 * Rounds with per-particle (accelerated) redo operations use the host loop.
 * No counterpart in the reference (an execution choice). */
int pmc_coag_gpu_set_graphs(pmc_coag_gpu_ctx *ctx, int enable);

/* New seed for population `pop`, with its step counter back at zero
 * (pmc_srand, rand.F90:66-113, for one population): its random streams then
 * depend only on the seed and the steps taken since, not on when the
 * population entered a batched context.  A server that reuses a population
 * slot for a new job calls this when it uploads the job. */
int pmc_coag_gpu_set_seed(pmc_coag_gpu_ctx *ctx, int pop, uint64_t seed);

/* Replay stream: uniforms in [0, 1) consumed in the reference's order
 * (pmc_random, rand.F90:138-167).  Copied to the device. */
int pmc_coag_gpu_replay_set(pmc_coag_gpu_ctx *ctx, const double *u, int64_t n);
/* Same, read from a file of little-endian float64 values. */
int pmc_coag_gpu_replay_open(pmc_coag_gpu_ctx *ctx, const char *path);
/* Uniforms consumed so far from the replay stream. */
int pmc_coag_gpu_replay_used(pmc_coag_gpu_ctx *ctx, int64_t *n_used);

/* Counters of the last step: kernel-bound violations (warn_assert_msg
 * 532446093, coagulation.F90:749-751), events that lost a claim (each is
 * retried or dropped in the next round), rounds. */
int pmc_coag_gpu_stats(pmc_coag_gpu_ctx *ctx, int64_t *kmax_violations,
                       int64_t *redraws, int64_t *rounds);

/* Removal records (aero_state%aero_info_array, aero_info.F90:48-56), the
 * output run_part writes when record_removals is set (run_part.F90:745,
 * 995-1001).  After pmc_coag_gpu_set_record_removals(ctx, 1) every
 * population logs each particle it removes, on the device: coagulation
 * removals whose ID is lost (coagulate, coagulation.F90:928-985; other_id =
 * the ID of the particle the coagulation made, or 0), the sources a
 * per-particle coagulation removes (coagulation.F90:447-453; other_id = the
 * target's ID), weight removals (aero_state_dup_particle,
 * aero_state.F90:502-513) and halving removals (aero_state_halve,
 * aero_state.F90:1753-1785).  pmc_coag_gpu_removals copies population
 * pop's records into id/action/other_id (action: 2 coagulation, 3 halved, 4
 * weight) and clears them, as run_part does after an output
 * (aero_info_array_zero).  *n gets the record count; if it exceeds max_n the
 * call returns PMC_ERR_CAPACITY and copies and clears nothing.  Records come
 * in removal order in replay mode and in no particular order otherwise. */
int pmc_coag_gpu_set_record_removals(pmc_coag_gpu_ctx *ctx, int enable);
int pmc_coag_gpu_removals(pmc_coag_gpu_ctx *ctx, int pop, int64_t max_n,
                          int64_t *id, int *action, int64_t *other_id,
                          int64_t *n);

/* Pair tests that MIXED mode decided in FP64, summed over the populations
 * since they were uploaded.  A test's FP32 acceptance probability is used
 * only where the uniform lies farther from it than a margin (2^-12) that
 * bounds the FP32 rounding error; the other tests (near the uniform, or near
 * or above k_max) are decided from the FP64 records, so every decision, and
 * the count of k > k_max warnings, is the FP64 mode's.  No counterpart in the
 * reference, which evaluates in FP64 only. */
int pmc_coag_gpu_exact_tests(pmc_coag_gpu_ctx *ctx, int64_t *n);

/* Conflicts of the last step, summed over its rounds: accepted per-set
 * events and how many lost a claim, per-particle target operations and how
 * many lost a claim (each loser is retried, dropped or redone in a later
 * round).  No counterpart in the reference, which applies events one at a
 * time. */
int pmc_coag_gpu_conflicts(pmc_coag_gpu_ctx *ctx, int64_t *events,
                           int64_t *event_losers, int64_t *target_ops,
                           int64_t *target_op_losers);

/* ---- measurement ---- */

/* Time, with CUDA events on the library's own stream, every launch of the
 * pair-test kernel (which = 0; units = samples tested), of the sort scatter
 * and record build (1; units = slots), of the sort histogram (2; units =
 * slots) and whole steps (3).  enable = 0 turns timing off; either call
 * clears the totals.  No counterpart in the reference. */
int pmc_coag_gpu_profile(pmc_coag_gpu_ctx *ctx, int enable);
int pmc_coag_gpu_profile_read(pmc_coag_gpu_ctx *ctx, int which,
                              double *total_ms, int64_t *launches,
                              int64_t *units);
/* Kernel launches issued by this library since it was loaded. */
int pmc_coag_gpu_launch_count(int64_t *n);

/* ---- inspection entry points used by the parity tests ---- */

/* Sort population `pop` (aero_state_sort, aero_state.F90:3291-3307) and
 * return the bin grid edges (n_bin+1, radius in m), the per-(bin, class)
 * counts (n_bin x n_class, bin fastest) and each particle's 1-based bin in
 * upload order.  Any output may be NULL. */
int pmc_coag_gpu_sort(pmc_coag_gpu_ctx *ctx, int pop, int *n_bin,
                      double *edges, int max_bin, int *counts, int *bins);

/* k_max table of the current grid (est_k_minmax_binned_unweighted,
 * coag_kernel.F90:253-280), n_bin x n_bin column-major. */
int pmc_coag_gpu_kmax_table(pmc_coag_gpu_ctx *ctx, int kernel_type,
                            double temp, double pressure,
                            double additive_coeff, double *kmax, int max_bin);

/* Weighted kernel (num_conc_weighted_kernel, coag_kernel.F90:175-209)
 * evaluated on the device for n_pairs particle pairs given by species
 * volumes (particle-major) and 1-based classes, in FP64 (mode FP64) or FP32
 * (mode MIXED).  c_ij is the destination class of each pair. */
int pmc_coag_gpu_eval_kernel(pmc_coag_gpu_ctx *ctx, int kernel_type,
                             double temp, double pressure,
                             double additive_coeff, int n_pairs,
                             const double *vol1, const int *c1,
                             const double *vol2, const int *c2,
                             const int *c_ij, double *k_out);

/* Size-bin sort that allocates nothing.  No counterpart in the reference:
 * it exists for callers that cannot allocate device memory on the call path,
 * such as a host model whose device memory is all handed out up front by its
 * own allocator.
 *
 * Same result as the sort inside a context (aero_sorted_sort_particles on a
 * log grid of n_bin bins from edge_min to edge_max, bin_grid.F90:143-167):
 *   bin_dev[i]        1-based bin of particle i (0 below the grid, n_bin+1 above)
 *   cell_count_dev    n_bin x n_class entries, bin fastest
 *   cell_start_dev    n_bin*n_class + 1 exclusive offsets into list_dev
 *   list_dev          0-based particle numbers grouped by (bin, class), in
 *                     increasing particle order inside each group; only the
 *                     first cell_start_dev[n_bin*n_class] entries are
 *                     written, since particles off the grid (bin 0 or
 *                     n_bin+1) or with a class outside 1..n_class are in no
 *                     group
 * from vtot_dev[i] (total particle volume, m^3) and 1-based cls_dev[i].
 * All pointers are caller-owned device buffers; work is queued on `stream`
 * (a cudaStream_t, NULL for the legacy default stream) and the call returns
 * without waiting for it.
 *
 * Limits: n_part <= 2,097,152 and n_bin * n_class <= 1024 (n_bin <= 256);
 * larger sizes return PMC_ERR_CAPACITY.  The scratch is one 4 MiB static
 * device array per GPU, held until the process exits and shared by every
 * call: calls whose work overlaps on the GPU (different streams, or other
 * threads) race on it and must be serialised by the caller.  The first call
 * on each device looks up that array's address (a runtime call, made once
 * per device). */
int pmc_coag_gpu_bin_sort_noalloc(int n_part, const double *vtot_dev,
                                  const int *cls_dev, int n_bin, int n_class,
                                  double edge_min, double edge_max,
                                  int *bin_dev, int *cell_count_dev,
                                  int *cell_start_dev, int *list_dev,
                                  void *stream);

/* Human-readable name of a status code. */
const char *pmc_coag_gpu_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif
