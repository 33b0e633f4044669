/*
 * pmc_oracle.h -- CPU oracle for PartMC's particle-resolved coagulation step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a sequential FP64 restatement, in plain
 * C, of the reference's mc_coag (src/coagulation.F90:43-985) and everything it
 * calls.  It is the checker for the CUDA library in partmc_b200/: only the
 * tests, the smoke check and the CPU-baseline leg of bench.py may load it.
 * Nothing in the product links it.
 *
 * Pinning: the reference is Fortran and no Fortran compiler exists where this
 * was written, so the oracle cannot be compared with the reference binary
 * draw by draw.  It is pinned instead by the reference's own known-answer
 * tests: the additive-kernel run against the exact solution
 * (test/additive, rel-tol 0.05 number / 0.2 mass), the constant kernel against
 * its exact solution, the Poisson and binomial samplers against their pmfs
 * (test/rand), and by hand-checkable kernel values.  Bit-exact replay against a
 * dump of the reference's own uniform draws is supported (see
 * orc_set_replay) but such a dump is not available here, so draw-level
 * parity with the reference binary is unpinned.
 *
 * Conventions: every index that the reference keeps 1-based (bins, particle
 * numbers, entries of the inverse maps, groups, classes) is stored 1-based
 * here too, and arrays are addressed with [x - 1].  Species volumes of
 * particle i are vol[(i - 1) * n_spec + s], the layout of the reference's
 * vol(n_spec) per particle.
 */
#ifndef PMC_ORACLE_H
#define PMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* kernel type codes, src/coag_kernel.F90:29-45 */
enum {
  ORC_KERNEL_SEDI = 1,
  ORC_KERNEL_ADDITIVE = 2,
  ORC_KERNEL_CONSTANT = 3,
  ORC_KERNEL_BROWN = 4,
  ORC_KERNEL_ZERO = 5,
  ORC_KERNEL_BROWN_FREE = 6,
  ORC_KERNEL_BROWN_CONT = 7
};

/* removal actions, src/aero_info.F90:19-28 */
enum {
  ORC_INFO_NONE = 0,
  ORC_INFO_DILUTION = 1,
  ORC_INFO_COAG = 2,
  ORC_INFO_HALVED = 3,
  ORC_INFO_WEIGHT = 4
};

/* weight type codes, src/aero_weight.F90:24-30 */
enum { ORC_WEIGHT_NONE = 1, ORC_WEIGHT_POWER = 2, ORC_WEIGHT_MFA = 3 };

/* status codes (the reference stops the program instead) */
enum {
  ORC_OK = 0,
  ORC_ERR_ARG = 1,
  ORC_ERR_OUT_OF_GRID = 2, /* die_msg 765620746 / 134572570 */
  ORC_ERR_ASSERT = 3,      /* a reference assert() that would have stopped */
  ORC_ERR_RNG_EXHAUSTED = 4,
  ORC_ERR_NOMEM = 5
};

#define ORC_MAX_COMPONENT 20 /* MAX_AERO_COMPONENT_SIZE, aero_particle.F90:22 */

typedef struct orc_state orc_state;

/* Particle record used to move particles in and out (one per particle). */
typedef struct {
  int32_t weight_group; /* 1-based */
  int32_t weight_class; /* 1-based */
  int64_t id;
  int32_t n_primary_parts;
  int32_t n_comp;
  int32_t comp_source[ORC_MAX_COMPONENT];
  double comp_create_time[ORC_MAX_COMPONENT];
  double least_create_time;
  double greatest_create_time;
  int32_t water_hyst_leg;
  int32_t frozen;
  double imf_temperature;
  double den_ice;
  double ice_shape_phi;
} orc_particle_meta;

/* weights: w_type/w_mag/w_exp are n_group x n_class, entry (g, c) at
 * (g - 1) + n_group * (c - 1), like the reference's weight(n_group, n_class). */
orc_state *orc_create(int n_spec, const double *density, int i_water,
                      int n_group, int n_class, const int *w_type,
                      const double *w_mag, const double *w_exp);
void orc_destroy(orc_state *st);
int orc_set_weight(orc_state *st, const int *w_type, const double *w_mag,
                   const double *w_exp);

/* Uniform source.  seed: internal xoshiro256** stream.  replay: a fixed
 * array of uniforms consumed in order.  dump: record every uniform drawn. */
void orc_set_seed(orc_state *st, uint64_t seed);
int orc_set_replay(orc_state *st, const double *u, int64_t n);
int orc_enable_dump(orc_state *st, int64_t capacity);
int64_t orc_dump_count(const orc_state *st);
int64_t orc_dump_copy(const orc_state *st, double *out, int64_t max_n);
int64_t orc_uniforms_used(const orc_state *st);
double orc_random(orc_state *st);

void orc_set_next_id(orc_state *st, int64_t next_id);
int64_t orc_get_next_id(const orc_state *st);

/* Append particles (aero_state_add_particle without sort). vol is n_spec x n
 * col-major (species fastest). */
int orc_add_particles(orc_state *st, int n, const double *vol,
                      const orc_particle_meta *meta);
int orc_n_part(const orc_state *st);
int orc_get_particles(const orc_state *st, double *vol, orc_particle_meta *meta);

/* mc_coag, src/coagulation.F90:43-96.  Returns a status code. */
int orc_mc_coag(orc_state *st, int kernel_type, double temp, double pressure,
                double additive_coeff, double del_t, int *tot_n_samp,
                int *tot_n_coag);
/* count of k/k_max > 1 warnings (warn_assert_msg 532446093 / 383983415) */
int64_t orc_kmax_warnings(const orc_state *st);
/* target particles the per-particle path has handled since creation */
int64_t orc_pp_targets(const orc_state *st);

/* aero_state_sort: (re)make the bin grid and the inverse maps. */
int orc_sort(orc_state *st);
/* Bin grid and sorted counts after the last sort. */
int orc_n_bin(const orc_state *st);
int orc_bin_edges(const orc_state *st, double *edges /* n_bin+1 */);
int orc_bin_counts(const orc_state *st, int *counts /* n_bin x n_class */);
/* forward bin of every particle (1-based), after a sort */
int orc_particle_bins(const orc_state *st, int *bins);
/* Consistency check of the rmap2 structures (aero_sorted_check). */
int orc_check(const orc_state *st);
/* k_max table (n_bin x n_bin, column-major like the reference) */
int orc_kmax_table(orc_state *st, int kernel_type, double temp,
                   double pressure, double additive_coeff, double *kmin,
                   double *kmax);

/* Keep removal records (aero_state%aero_info_array) from now on.  Records
 * are appended in the reference's order of removals: coagulation removals
 * whose ID is lost (coagulation.F90:928-985, other_id = the coagulated
 * particle's ID or 0), per-particle source removals (:447-453, other_id =
 * the target's ID), weight removals of aero_state_dup_particle and halving
 * removals of aero_state_halve. */
void orc_set_record_removals(orc_state *st, int on);
/* Copy the records out (id, action, other_id) and clear them, as run_part
 * does after an output (aero_info_array_zero); returns the count, or minus
 * the count (nothing copied) if it exceeds max_n. */
int64_t orc_removals(orc_state *st, int64_t max_n, int64_t *id, int *action,
                     int64_t *other_id);

/* Particle shape of aero_data (fractal_t, fractal.F90:59-66); d_f = 3 and
 * f = 1 are spherical particles, the default.  Invalidates the sort and the
 * k_max bounds.  ORC_ERR_ARG for d_f outside (0, 3] or R0, f <= 0. */
int orc_set_fractal(orc_state *st, double frac_dim, double prime_radius,
                    double vol_fill_factor);

/* ----- pure functions, for unit tests ----- */
/* fractal_vol2rad of volume v; *mobility (if not NULL) gets
 * fractal_vol_to_mobility_rad at temp, pressure (NAN if the Newton loop
 * does not converge) */
double orc_fractal_radius(double v, double frac_dim, double prime_radius,
                          double vol_fill_factor, double temp, double pressure,
                          double *mobility);
/* orc_kernel_value for particles of the given fractal shape */
double orc_kernel_value_fractal(int kernel_type, double v1, double d1,
                                double v2, double d2, double temp,
                                double pressure, double additive_coeff,
                                double frac_dim, double prime_radius,
                                double vol_fill_factor);
double orc_vol2rad(double v);
double orc_rad2vol(double r);
/* unweighted kernel between particles of total volume v and density d */
double orc_kernel_value(int kernel_type, double v1, double d1, double v2,
                        double d2, double temp, double pressure,
                        double additive_coeff);
void orc_kernel_minmax(orc_state *st, int kernel_type, double v1, double v2,
                       double temp, double pressure, double additive_coeff,
                       double *kmin, double *kmax);
/* num_conc_weighted_kernel for two particles given by species volumes */
double orc_weighted_kernel(orc_state *st, int kernel_type, const double *vol1,
                           int class1, const double *vol2, int class2,
                           int ij_class, double temp, double pressure,
                           double additive_coeff);
double orc_num_conc_at_radius(const orc_state *st, int i_class, double r);
int orc_bin_find(int n_bin, double e_min, double e_max, double r);
void orc_bin_grid_make(int n_bin, double rmin, double rmax, double *edges,
                       double *centers);
int orc_coag_dest_class(const orc_state *st, const double *edges,
                        const double *centers, int b1, int b2, int c1, int c2);
double orc_max_num_conc_factor(const orc_state *st, const double *edges,
                               int b1, int b2, int c1, int c2, int cc);
double orc_student_t_95(int n_sample);

/* samplers on the state's uniform stream */
int orc_rand_poisson(orc_state *st, double mean);
int orc_rand_binomial(orc_state *st, int n, double p);
double orc_rand_normal(orc_state *st, double mean, double stddev);
int orc_rand_int(orc_state *st, int n);
int orc_prob_round(orc_state *st, double val);

/* aero_state_rebalance (aero_state.F90:1722-1852): double or halve each
 * (group, class) towards n_part_ideal[(g-1) + n_group*(c-1)]; the weight
 * magnitudes change accordingly (read them back with orc_get_weight). */
int orc_rebalance(orc_state *st, const double *n_part_ideal, int allow_doubling,
                  int allow_halving);
int orc_get_weight(const orc_state *st, double *w_mag);

/* One step of the reference's sectional coagulation solver (coad,
 * run_sect.F90:283-359, Bott's exponential flux method), 0-based: g[n_bin]
 * mass distribution (updated in place), e[n_bin] bin masses (mg),
 * c[i*n_bin+j] Courant numbers, ima[i*n_bin+j] the bin that i + j goes to
 * (-1: none), ck[i*n_bin+j] the smoothed kernel times del_t and bin width. */
void orc_sect_coad(int n_bin, const double *c, const int *ima, double *g, const double *e, const double *ck);

/* histograms of n draws (k = 0..k_max) */
void orc_poisson_hist(orc_state *st, double mean, int64_t n, int k_max,
                      int64_t *counts);
void orc_binomial_hist(orc_state *st, int nn, double p, int64_t n, int k_max,
                       int64_t *counts);

/* Run many independent populations on host threads (CPU baseline). Each
 * population p has its own state; returns total samples and coagulations. */
int orc_step_many(orc_state **states, int n_states, int n_threads,
                  int kernel_type, const double *temp, const double *pressure,
                  double additive_coeff, double del_t, int n_steps,
                  int64_t *tot_n_samp, int64_t *tot_n_coag);

#ifdef __cplusplus
}
#endif

#endif
