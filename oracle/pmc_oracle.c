/*
 * pmc_oracle.c -- sequential FP64 restatement of PartMC's mc_coag.
 *
 * TEST INFRASTRUCTURE ONLY (see pmc_oracle.h).  Each function names the
 * reference routine (path:line inside the PartMC source tree) whose behaviour
 * it restates.  Arithmetic is written in the reference's evaluation order so
 * that results agree to the last bit where the same libm is used; build with
 * -ffp-contract=off so no fused multiply-add changes a rounding.
 */
#include "pmc_oracle.h"

#include <math.h>
#include <pthread.h>
#include <setjmp.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------- */
/* physical constants, src/constants.F90:31-61                             */

static const double C_PI = 3.14159265358979323846;
static const double C_BOLTZMANN = 1.3806505e-23;
static const double C_AVOGADRO = 6.02214179e23;
static const double C_UNIV_GAS = 8.314472;
static const double C_AIR_MOLEC_WEIGHT = 2.89644e-2;
static const double C_WATER_DENSITY = 1e3;

/* aero_sorted.F90:69-73 */
static const double SORTED_BINS_PER_DECADE = 10.0;
static const double SORTED_BIN_OVER_FACTOR = 10.0;
static const double SORTED_BIN_SAFETY_FACTOR = 3.0;

/* coagulation.F90:30-36 */
static const double COAG_ACCEL_N_EVENT = 1.0;
static const double COAG_ACCEL_MAX_CV = 0.1;
static const double MAX_ALLOWABLE_GROWTH_FACTOR = 1.5;

/* ---------------------------------------------------------------------- */
/* growable integer list with the reference's swap-last removal            */
/* (integer_varray.F90:131-171); values are stored as given (1-based).     */

typedef struct {
  int n, cap;
  int *e;
} ivec;

/* rmap2 = forward maps, inverse lists per (range1, range2), and the index of
 * each domain element inside its inverse list (integer_rmap2.F90:53-62). */
typedef struct {
  ivec fwd1, fwd2, index;
  int n_r1, n_r2;
  ivec *inv;
} rmap2;

/* fractal_t, fractal.F90:59-66: volume fractal dimension, primary radius
 * (m), volume filling factor; sph: fractal_is_spherical (d_f = 3, f = 1) */
typedef struct {
  double frac_dim, prime_radius, vol_fill_factor;
  int sph;
} orc_fractal;

struct orc_state {
  orc_fractal frac; /* particle shape of aero_data (spherical by default) */
  int n_spec;
  double *density;
  int i_water; /* 1-based, 0 if none */
  int n_group, n_class;
  int *w_type;
  double *w_mag, *w_exp;

  int n_part, cap;
  double *vol;
  orc_particle_meta *meta;

  int valid_sort;
  int n_bin;
  double *edges, *centers;
  rmap2 size_class, group_class;
  int kbounds_valid;
  double *kmin, *kmax;

  uint64_t rs[4];
  const double *replay;
  int64_t replay_n, replay_pos;
  int use_replay;
  double *dump;
  int64_t dump_n, dump_cap;
  int dump_on;
  int64_t used;

  int64_t next_id;
  int64_t kmax_warn;
  /* aero_info_array (aero_info_array.F90): removal records, kept when on */
  int rec_removals;
  int64_t rm_n, rm_cap;
  int64_t *rm_id, *rm_other;
  int *rm_action;
  int64_t pp_targets; /* targets handled by the per-particle path (a counter for tests) */

  jmp_buf *fail;
  int fail_code;
};

static void orc_fail(orc_state *st, int code) {
  st->fail_code = code;
  if (st->fail) longjmp(*st->fail, 1);
  abort();
}

static void ivec_push(orc_state *st, ivec *v, int x) {
  if (v->n == v->cap) {
    int nc = v->cap ? 2 * v->cap : 8;
    int *ne = (int *)realloc(v->e, sizeof(int) * nc);
    if (!ne) orc_fail(st, ORC_ERR_NOMEM);
    v->e = ne;
    v->cap = nc;
  }
  v->e[v->n++] = x;
}

/* integer_varray_remove_entry, integer_varray.F90:151-171 (1-based idx) */
static void ivec_remove_entry(orc_state *st, ivec *v, int idx) {
  if (idx < 1 || idx > v->n) orc_fail(st, ORC_ERR_ASSERT);
  if (idx < v->n) v->e[idx - 1] = v->e[v->n - 1];
  v->e[v->n - 1] = 0;
  v->n--;
}

static void rmap2_free(rmap2 *m) {
  free(m->fwd1.e);
  free(m->fwd2.e);
  free(m->index.e);
  if (m->inv) {
    for (int i = 0; i < m->n_r1 * m->n_r2; i++) free(m->inv[i].e);
    free(m->inv);
  }
  memset(m, 0, sizeof(*m));
}

/* integer_rmap2_set_ranges (intent(out): everything is reset),
 * integer_rmap2.F90:69-84 */
static void rmap2_set_ranges(orc_state *st, rmap2 *m, int n1, int n2) {
  rmap2_free(m);
  m->n_r1 = n1;
  m->n_r2 = n2;
  if (n1 * n2 > 0) {
    m->inv = (ivec *)calloc((size_t)n1 * n2, sizeof(ivec));
    if (!m->inv) orc_fail(st, ORC_ERR_NOMEM);
  }
}

static ivec *rmap2_cell(rmap2 *m, int j1, int j2) {
  return &m->inv[(j1 - 1) + m->n_r1 * (j2 - 1)];
}

/* integer_rmap2_zero, integer_rmap2.F90:89-101 */
static void rmap2_zero(rmap2 *m) {
  m->fwd1.n = m->fwd2.n = m->index.n = 0;
  for (int i = 0; i < m->n_r1 * m->n_r2; i++) m->inv[i].n = 0;
}

/* integer_rmap2_append, integer_rmap2.F90:107-130 */
static void rmap2_append(orc_state *st, rmap2 *m, int j1, int j2) {
  if (j1 < 1 || j1 > m->n_r1 || j2 < 1 || j2 > m->n_r2)
    orc_fail(st, ORC_ERR_ASSERT);
  ivec_push(st, &m->fwd1, j1);
  ivec_push(st, &m->fwd2, j2);
  ivec *c = rmap2_cell(m, j1, j2);
  ivec_push(st, c, m->fwd1.n);
  ivec_push(st, &m->index, c->n);
}

/* integer_rmap2_change, integer_rmap2.F90:135-184.  Keeps the reference's
 * early return that tests only the first range (line 160). */
static void rmap2_change(orc_state *st, rmap2 *m, int i, int j1, int j2) {
  if (i < 1 || i > m->fwd1.n) orc_fail(st, ORC_ERR_ASSERT);
  if (j1 < 1 || j1 > m->n_r1 || j2 < 1 || j2 > m->n_r2)
    orc_fail(st, ORC_ERR_ASSERT);
  int old1 = m->fwd1.e[i - 1];
  int old2 = m->fwd2.e[i - 1];
  if (old1 == j1) return;
  int idx_old = m->index.e[i - 1];
  ivec *c_old = rmap2_cell(m, old1, old2);
  ivec_remove_entry(st, c_old, idx_old);
  if (idx_old <= c_old->n) {
    int shifted = c_old->e[idx_old - 1];
    m->index.e[shifted - 1] = idx_old;
  }
  m->fwd1.e[i - 1] = j1;
  m->fwd2.e[i - 1] = j2;
  ivec *c_new = rmap2_cell(m, j1, j2);
  ivec_push(st, c_new, i);
  m->index.e[i - 1] = c_new->n;
}

/* integer_rmap2_remove, integer_rmap2.F90:190-243 */
static void rmap2_remove(orc_state *st, rmap2 *m, int i) {
  if (i < 1 || i > m->fwd1.n) orc_fail(st, ORC_ERR_ASSERT);
  int old1 = m->fwd1.e[i - 1];
  int old2 = m->fwd2.e[i - 1];
  int idx_old = m->index.e[i - 1];
  int shifted = m->fwd1.n;
  if (shifted != i) {
    int f1 = m->fwd1.e[shifted - 1];
    int f2 = m->fwd2.e[shifted - 1];
    int fi = m->index.e[shifted - 1];
    rmap2_cell(m, f1, f2)->e[fi - 1] = i;
  }
  ivec_remove_entry(st, &m->fwd1, i);
  ivec_remove_entry(st, &m->fwd2, i);
  ivec_remove_entry(st, &m->index, i);
  ivec *c_old = rmap2_cell(m, old1, old2);
  int idx_fix = c_old->n;
  int dom_fix = c_old->e[idx_fix - 1];
  ivec_remove_entry(st, c_old, idx_old);
  if (idx_fix != idx_old) m->index.e[dom_fix - 1] = idx_old;
}

/* ---------------------------------------------------------------------- */
/* uniform source                                                          */

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* splitmix64 seeding of xoshiro256** (Blackman & Vigna, 2018) */
void orc_set_seed(orc_state *st, uint64_t seed) {
  uint64_t z = seed;
  for (int i = 0; i < 4; i++) {
    z += 0x9e3779b97f4a7c15ULL;
    uint64_t x = z;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    st->rs[i] = x ^ (x >> 31);
  }
  st->use_replay = 0;
}

static uint64_t xoshiro_next(uint64_t *s) {
  uint64_t out = rotl64(s[1] * 5, 7) * 9;
  uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return out;
}

int orc_set_replay(orc_state *st, const double *u, int64_t n) {
  st->replay = u;
  st->replay_n = n;
  st->replay_pos = 0;
  st->use_replay = 1;
  return ORC_OK;
}

int orc_enable_dump(orc_state *st, int64_t capacity) {
  free(st->dump);
  st->dump = NULL;
  st->dump_n = 0;
  st->dump_cap = 0;
  st->dump_on = capacity > 0;
  if (capacity > 0) {
    st->dump = (double *)malloc(sizeof(double) * capacity);
    if (!st->dump) return ORC_ERR_NOMEM;
    st->dump_cap = capacity;
  }
  return ORC_OK;
}

int64_t orc_dump_count(const orc_state *st) { return st->dump_n; }

int64_t orc_dump_copy(const orc_state *st, double *out, int64_t max_n) {
  int64_t n = st->dump_n < max_n ? st->dump_n : max_n;
  memcpy(out, st->dump, sizeof(double) * n);
  return n;
}

int64_t orc_uniforms_used(const orc_state *st) { return st->used; }

/* pmc_random, rand.F90:138-167: a uniform in [0, 1). */
double orc_random(orc_state *st) {
  double u;
  if (st->use_replay) {
    if (st->replay_pos >= st->replay_n) orc_fail(st, ORC_ERR_RNG_EXHAUSTED);
    u = st->replay[st->replay_pos++];
  } else {
    u = (double)(xoshiro_next(st->rs) >> 11) * 0x1.0p-53;
  }
  if (st->dump_on) {
    if (st->dump_n == st->dump_cap) {
      int64_t nc = 2 * st->dump_cap;
      double *nd = (double *)realloc(st->dump, sizeof(double) * nc);
      if (!nd) orc_fail(st, ORC_ERR_NOMEM);
      st->dump = nd;
      st->dump_cap = nc;
    }
    st->dump[st->dump_n++] = u;
  }
  st->used++;
  return u;
}

/* pmc_rand_int, rand.F90:172-207: mod(int(u*n), n) + 1 */
int orc_rand_int(orc_state *st, int n) {
  if (n < 1) orc_fail(st, ORC_ERR_ASSERT);
  double u = orc_random(st);
  int k = (int)(u * (double)n);
  return k % n + 1;
}

/* prob_round, rand.F90:214-227 */
int orc_prob_round(orc_state *st, double val) {
  double c = ceil(val);
  if (orc_random(st) < c - val) return (int)floor(val);
  return (int)c;
}

/* rand_normal without threshold (Box-Muller), rand.F90:410-487 */
double orc_rand_normal(orc_state *st, double mean, double stddev) {
  double u1 = orc_random(st);
  double u2 = orc_random(st);
  double r = sqrt(-2.0 * log(u1));
  double theta = 2.0 * C_PI * u2;
  double z0 = r * cos(theta);
  return stddev * z0 + mean;
}

/* Fortran nint: round half away from zero */
static int f_nint(double x) { return (int)lround(x); }

/* rand_poisson (non-GSL branch), rand.F90:252-305 */
int orc_rand_poisson(orc_state *st, double mean) {
  if (!(mean >= 0.0)) orc_fail(st, ORC_ERR_ASSERT);
  if (mean <= 10.0) {
    double L = exp(-mean);
    int k = 0;
    double p = 1.0;
    for (;;) {
      k++;
      p = p * orc_random(st);
      if (p < L) break;
    }
    return k - 1;
  }
  int k = f_nint(orc_rand_normal(st, mean, sqrt(mean)));
  return k > 0 ? k : 0;
}

/* rand_binomial (non-GSL branch), rand.F90:319-404 */
int orc_rand_binomial(orc_state *st, int n, double p) {
  if (n < 0 || !(p >= 0.0) || !(p <= 1.0)) orc_fail(st, ORC_ERR_ASSERT);
  double np = (double)n * p;
  double nomp = (double)n * (1.0 - p);
  if (np >= 10.0 && nomp >= 10.0) {
    int k = f_nint(orc_rand_normal(st, np, sqrt(np * (1.0 - p))));
    if (k < 0) k = 0;
    if (k > n) k = n;
    return k;
  } else if (p < 1e-15) {
    return 0;
  } else if (np < 1e-200) {
    return 0;
  } else if (nomp < 1e-200) {
    return n;
  }
  double q = p <= 0.5 ? p : 1.0 - p;
  int k = 0, sum = 0;
  for (;;) {
    double g_real = log(orc_random(st)) / log(1.0 - q);
    if (g_real > (double)(n - sum)) break;
    int g = (int)ceil(g_real);
    sum += g;
    if (sum > n) break;
    k++;
  }
  return p <= 0.5 ? k : n - k;
}

/* sample_without_replacement, rand.F90:515-542; sample[] gets 1-based
 * indices in increasing order. */
static void sample_wo_replacement(orc_state *st, int size, int pop,
                                  int *sample) {
  int t = 0, m = 0;
  while (m < size) {
    double r = orc_random(st);
    if ((double)(pop - t) * r >= (double)(size - m)) {
      t++;
    } else {
      t++;
      m++;
      sample[m - 1] = t;
    }
  }
}

/* sample_cts_pdf, rand.F90:550-576 (accept-reject) */
static int sample_cts_pdf(orc_state *st, const double *pdf, int n) {
  double pmax = pdf[0], pmin = pdf[0];
  for (int i = 1; i < n; i++) {
    if (pdf[i] > pmax) pmax = pdf[i];
    if (pdf[i] < pmin) pmin = pdf[i];
  }
  if (pmin < 0.0 || pmax <= 0.0) orc_fail(st, ORC_ERR_ASSERT);
  for (;;) {
    int k = orc_rand_int(st, n);
    if (orc_random(st) < pdf[k - 1] / pmax) return k;
  }
}

/* ---------------------------------------------------------------------- */
/* util / geometry                                                         */

/* __powidf2-style integer power by squaring, the code gfortran emits for
 * x**i with a variable integer i (used by fall_g, coag_kernel_sedi.F90:150) */
static double powi(double x, int m) {
  unsigned n = m < 0 ? (unsigned)(-m) : (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

/* sphere_vol2rad, util.F90:240-247 */
double orc_vol2rad(double v) { return pow(3.0 * v / 4.0 / C_PI, 1.0 / 3.0); }

/* sphere_rad2vol, util.F90:264-271 */
double orc_rad2vol(double r) { return 4.0 * C_PI * (r * r * r) / 3.0; }

/* fractal_set_spherical, fractal.F90:73-82 */
static const orc_fractal SPHERE = {3.0, 1e-8, 1.0, 1};

/* fractal_vol_to_num_of_monomers, fractal.F90:90-100 */
static double num_of_monomers(const orc_fractal *fr, double v) {
  double x = orc_vol2rad(v) / fr->prime_radius;
  return x * x * x;
}

/* fractal_vol2rad, fractal.F90:106-121 */
static double frac_vol2rad(const orc_fractal *fr, double v) {
  if (fr->sph) return orc_vol2rad(v);
  return fr->prime_radius *
         pow(num_of_monomers(fr, v) * fr->vol_fill_factor, 1.0 / fr->frac_dim);
}

/* fractal_rad2vol, fractal.F90:142-157 */
static double frac_rad2vol(const orc_fractal *fr, double r) {
  if (fr->sph) return orc_rad2vol(r);
  return orc_rad2vol(fr->prime_radius) * pow(r / fr->prime_radius, fr->frac_dim) /
         fr->vol_fill_factor;
}

/* air_mean_free_path, util.F90:289-312 */
static double air_mean_free_path(double temp, double pressure) {
  double rhoair = (pressure * C_AIR_MOLEC_WEIGHT) / (C_UNIV_GAS * temp);
  double viscosd =
      (1.8325e-5 * (296.16 + 120.0) / (temp + 120.0)) * pow(temp / 296.16, 1.5);
  double viscosk = viscosd / rhoair;
  double gasspeed =
      sqrt(8.0 * C_BOLTZMANN * temp * C_AVOGADRO / (C_PI * C_AIR_MOLEC_WEIGHT));
  return 2.0 * viscosk / gasspeed;
}

/* fractal_vol_to_mobility_rad, fractal.F90:315-362, with its helpers:
 * surface fractal dimension (:177-191), accessible surface (:199-216),
 * Kirkwood-Riseman ratio (:223-231), continuum mobility radius (:239-249),
 * effective radius (:257-268) and slip correction (:276-291); constants
 * fractal.F90:43-53.  Newton's method from the continuum mobility radius,
 * relative step 1e-14, at most 10 steps; *ok is cleared where the reference
 * asserts (728724732). */
static double mobility_rad(const orc_fractal *fr, double v, double temp,
                           double pressure, int *ok) {
  if (fr->sph) return frac_vol2rad(fr, v);
  const double A = 1.142, Q = 0.588, B = 0.999, SF = 1.0, SE = 0.86;
  double df = fr->frac_dim;
  double ds = df <= 2.0 ? 3.0 : 6.0 / df;
  double n = num_of_monomers(fr, v);
  double s_acc = 4.0 * C_PI * (fr->prime_radius * fr->prime_radius) *
                 pow(n, ds / 3.0) *
                 ((ds - 2.0) * pow(SF / n, 1.0 - SE) - ds + 3.0);
  double kr = -0.06483 * (df * df) + 0.6353 * df - 0.4898;
  double rmec = kr * frac_vol2rad(fr, v);
  double reff = s_acc / 4.0 / C_PI / rmec;
  double fp = air_mean_free_path(temp, pressure);
  double c_reff = 1.0 + A * fp / reff + Q * fp / reff * exp(-B * reff / fp);
  double a1 = c_reff, a2 = -rmec, a3 = -rmec * Q * fp, a4 = -B / fp;
  double a5 = -rmec * A * fp;
  double x = rmec;
  int step;
  for (step = 1; step <= 10; step++) {
    double f = a1 * (x * x) + a2 * x + a3 * exp(a4 * x) + a5;
    double dfx = 2.0 * a1 * x + a2 + a3 * a4 * exp(a4 * x);
    x = x - f / dfx;
    if (fabs(f / dfx) / (fabs(x + f / dfx) + fabs(x)) < 1e-14) break;
  }
  if (!(step < 10)) *ok = 0;
  return x;
}

/* interp_linear_disc, util.F90:663-683 */
static double interp_linear_disc(double x1, double xn, int n, int i) {
  if (x1 == xn) return x1;
  double a = (double)(i - 1) / (double)(n - 1);
  return (1.0 - a) * x1 + a * xn;
}

/* fast_pow, util.F90:1978-2003 */
static double fast_pow(double b, double e) {
  if (e == 0.0) return 1.0;
  if (e == 1.0) return b;
  if (e == 2.0) return b * b;
  if (e == 3.0) return b * b * b;
  if (e == -1.0) return 1.0 / b;
  if (e == -2.0) return 1.0 / (b * b);
  if (e == -3.0) return 1.0 / (b * b * b);
  return pow(b, e);
}

/* student_t_95_coeff, stats.F90:510-536: 97.5% quantiles of Student's t for
 * 1..15 degrees of freedom, then the A/nu bound beyond that. */
double orc_student_t_95(int n_sample) {
  static const double limit = 1.959963984540054;
  static const double tq[15] = {
      12.7062047364, 4.30265272991, 3.18244630528, 2.7764451052,
      2.57058183661, 2.44691184879, 2.36462425101, 2.30600413503,
      2.26215716274, 2.22813885196, 2.20098516008, 2.17881282966,
      2.16036865646, 2.14478668792, 2.13144954556};
  int dof = n_sample - 1;
  if (dof <= 15) return tq[dof - 1];
  if (dof <= 20) return (2.11990529922 - limit) * 16.0 / (double)dof + limit;
  return (2.07961384473 - limit) * 21.0 / (double)dof + limit;
}

/* linspace, util.F90:460-487 */
static void linspace(double a, double b, int n, double *out) {
  for (int i = 2; i <= n - 1; i++) {
    double t = (double)(i - 1) / (double)(n - 1);
    out[i - 1] = (1.0 - t) * a + t * b;
  }
  if (n > 0) {
    out[0] = a;
    out[n - 1] = b;
  }
}

/* logspace, util.F90:492-518 */
static void logspace(double a, double b, int n, double *out) {
  if (n == 0) return;
  linspace(log(a), log(b), n, out);
  for (int i = 0; i < n; i++) out[i] = exp(out[i]);
  out[0] = a;
  out[n - 1] = b;
}

/* bin_grid_make (log type), bin_grid.F90:83-134 */
void orc_bin_grid_make(int n_bin, double rmin, double rmax, double *edges,
                       double *centers) {
  if (n_bin == 0) return;
  logspace(rmin, rmax, n_bin + 1, edges);
  double c1 = exp(interp_linear_disc(log(rmin), log(rmax), 2 * n_bin + 1, 2));
  double c2 =
      exp(interp_linear_disc(log(rmin), log(rmax), 2 * n_bin + 1, 2 * n_bin));
  logspace(c1, c2, n_bin, centers);
}

/* bin_grid_find -> logspace_find -> linspace_find, bin_grid.F90:143-167,
 * util.F90:532-579.  Returns 0..n_bin+1. */
int orc_bin_find(int n_bin, double e_min, double e_max, double r) {
  if (n_bin <= 0) return -1;
  double lo = log(e_min), hi = log(e_max), x = log(r);
  int n = n_bin + 1;
  if (x == hi) return n - 1;
  int i = (int)floor((x - lo) / (hi - lo) * (double)(n - 1)) + 1;
  if (i > n) i = n;
  if (i < 0) i = 0;
  return i;
}

/* ---------------------------------------------------------------------- */
/* weights                                                                 */

static double weight_nc_at_radius(const orc_state *st, int g, int c, double r) {
  int k = (g - 1) + st->n_group * (c - 1);
  int t = st->w_type[k];
  if (t == ORC_WEIGHT_NONE) return st->w_mag[k];
  return st->w_mag[k] * fast_pow(r, st->w_exp[k]);
}

/* aero_weight_array_num_conc_at_radius, aero_weight_array.F90:232-252 */
double orc_num_conc_at_radius(const orc_state *st, int c, double r) {
  double inv_sum = 0.0;
  for (int g = 1; g <= st->n_group; g++)
    inv_sum = inv_sum + 1.0 / weight_nc_at_radius(st, g, c, r);
  return 1.0 / inv_sum;
}

/* aero_weight_array_check_monotonicity, aero_weight_array.F90:304-332 */
static void weight_monotonicity(const orc_state *st, int *inc, int *dec) {
  *inc = 1;
  *dec = 1;
  for (int k = 0; k < st->n_group * st->n_class; k++) {
    if (st->w_type[k] == ORC_WEIGHT_POWER) {
      if (st->w_exp[k] < 0.0) *inc = 0;
      if (st->w_exp[k] > 0.0) *dec = 0;
    }
    if (st->w_type[k] == ORC_WEIGHT_MFA) *inc = 0;
  }
}

/* aero_weight_array_minmax_num_conc, aero_weight_array.F90:338-368 */
static void weight_minmax_nc(orc_state *st, int c, double r1, double r2,
                             double *mn, double *mx) {
  int inc, dec;
  weight_monotonicity(st, &inc, &dec);
  if (!(inc || dec)) orc_fail(st, ORC_ERR_ASSERT);
  double n1 = orc_num_conc_at_radius(st, c, r1);
  double n2 = orc_num_conc_at_radius(st, c, r2);
  *mn = n1 < n2 ? n1 : n2;
  *mx = n1 > n2 ? n1 : n2;
}

/* aero_weight_array_rand_group, aero_weight_array.F90:374-393 */
static int weight_rand_group(orc_state *st, int c, double r) {
  double pdf[64];
  if (st->n_group > 64) orc_fail(st, ORC_ERR_ASSERT);
  for (int g = 1; g <= st->n_group; g++)
    pdf[g - 1] = 1.0 / weight_nc_at_radius(st, g, c, r);
  return sample_cts_pdf(st, pdf, st->n_group);
}

/* ---------------------------------------------------------------------- */
/* particles                                                               */

static double *pvol(orc_state *st, int i) {
  return st->vol + (size_t)(i - 1) * st->n_spec;
}

static double vol_sum(const double *v, int n) {
  double s = 0.0;
  for (int k = 0; k < n; k++) s = s + v[k];
  return s;
}

static double part_volume(orc_state *st, int i) {
  return vol_sum(pvol(st, i), st->n_spec);
}

static double part_radius(orc_state *st, int i) {
  return frac_vol2rad(&st->frac, part_volume(st, i));
}

/* aero_particle_density = mass / volume, aero_particle.F90:491-501 */
static double vol_density(const orc_state *st, const double *v) {
  double m = 0.0;
  for (int k = 0; k < st->n_spec; k++) m = m + v[k] * st->density[k];
  return m / vol_sum(v, st->n_spec);
}

static void ensure_cap(orc_state *st, int n) {
  if (n <= st->cap) return;
  int nc = st->cap ? st->cap : 16;
  while (nc < n) nc *= 2;
  double *nv = (double *)realloc(st->vol, sizeof(double) * (size_t)nc * st->n_spec);
  if (!nv) orc_fail(st, ORC_ERR_NOMEM);
  st->vol = nv;
  orc_particle_meta *nm =
      (orc_particle_meta *)realloc(st->meta, sizeof(orc_particle_meta) * nc);
  if (!nm) orc_fail(st, ORC_ERR_NOMEM);
  st->meta = nm;
  st->cap = nc;
}

/* A particle held outside the array (accumulators, copies). */
typedef struct {
  double vol[64];
  orc_particle_meta m;
} tpart;

static void tpart_from(orc_state *st, tpart *t, int i) {
  memcpy(t->vol, pvol(st, i), sizeof(double) * st->n_spec);
  t->m = st->meta[i - 1];
}

/* aero_particle_zero, aero_particle.F90:118-152 */
static void tpart_zero(orc_state *st, tpart *t) {
  memset(t->vol, 0, sizeof(double) * st->n_spec);
  memset(&t->m, 0, sizeof(t->m));
  t->m.den_ice = NAN;
  t->m.ice_shape_phi = NAN;
}

/* aero_particle_coagulate, aero_particle.F90:917-1033.  out may alias a or
 * b: all inputs are read before anything is written. */
static void particle_coagulate(orc_state *st, const double *va,
                               const orc_particle_meta *a, const double *vb,
                               const orc_particle_meta *b, double *vout,
                               orc_particle_meta *out) {
  int ns = st->n_spec;
  orc_particle_meta r;
  memset(&r, 0, sizeof(r));
  double ice1 = 0.0, ice2 = 0.0;
  if (st->i_water > 0) {
    ice1 = va[st->i_water - 1];
    ice2 = vb[st->i_water - 1];
  }
  r.weight_group = 0;
  r.weight_class = 0;
  r.water_hyst_leg = (a->water_hyst_leg == 1 && b->water_hyst_leg == 1) ? 1 : 0;
  r.id = 0;
  int n1 = a->n_comp, n2 = b->n_comp;
  if (a->n_primary_parts < n1 || b->n_primary_parts < n2)
    orc_fail(st, ORC_ERR_ASSERT);
  if (n1 + n2 > ORC_MAX_COMPONENT) {
    int n1_new = orc_prob_round(
        st, (double)a->n_primary_parts /
                (double)(a->n_primary_parts + b->n_primary_parts) *
                (double)ORC_MAX_COMPONENT);
    /* The reference can ask for more components than a particle has (when
     * n_primary_parts > n_components) and then reads past its component
     * array; both counts are clamped here instead. */
    if (n1_new > n1) n1_new = n1;
    int n2_new = ORC_MAX_COMPONENT - n1_new;
    if (n2_new > n2) n2_new = n2;
    int sample[ORC_MAX_COMPONENT];
    sample_wo_replacement(st, n1_new, n1, sample);
    for (int i = 0; i < n1_new; i++) {
      r.comp_source[i] = a->comp_source[sample[i] - 1];
      r.comp_create_time[i] = a->comp_create_time[sample[i] - 1];
    }
    sample_wo_replacement(st, n2_new, n2, sample);
    for (int i = 0; i < n2_new; i++) {
      r.comp_source[n1_new + i] = b->comp_source[sample[i] - 1];
      r.comp_create_time[n1_new + i] = b->comp_create_time[sample[i] - 1];
    }
    r.n_comp = n1_new + n2_new;
  } else {
    for (int i = 0; i < n1; i++) {
      r.comp_source[i] = a->comp_source[i];
      r.comp_create_time[i] = a->comp_create_time[i];
    }
    for (int i = 0; i < n2; i++) {
      r.comp_source[n1 + i] = b->comp_source[i];
      r.comp_create_time[n1 + i] = b->comp_create_time[i];
    }
    r.n_comp = n1 + n2;
  }
  r.least_create_time = a->least_create_time < b->least_create_time
                            ? a->least_create_time
                            : b->least_create_time;
  r.greatest_create_time = a->greatest_create_time > b->greatest_create_time
                               ? a->greatest_create_time
                               : b->greatest_create_time;
  r.frozen = a->frozen || b->frozen;
  r.imf_temperature = a->imf_temperature > b->imf_temperature
                          ? a->imf_temperature
                          : b->imf_temperature;
  if (r.frozen) {
    if (a->frozen && b->frozen) {
      ice1 = ice1 * C_WATER_DENSITY / a->den_ice;
      ice2 = ice2 * C_WATER_DENSITY / b->den_ice;
      r.den_ice = (a->den_ice * ice1 + b->den_ice * ice2) / (ice1 + ice2);
    } else if (a->frozen) {
      r.den_ice = a->den_ice;
    } else {
      r.den_ice = b->den_ice;
    }
    r.ice_shape_phi = 1.0;
  } else {
    r.den_ice = NAN;
    r.ice_shape_phi = a->ice_shape_phi; /* unchanged by the reference */
  }
  r.n_primary_parts = a->n_primary_parts + b->n_primary_parts;
  for (int k = 0; k < ns; k++) vout[k] = va[k] + vb[k];
  *out = r;
}

/* ---------------------------------------------------------------------- */
/* coagulation kernels                                                     */

/* kernel_brown_helper, coag_kernel_brown.F90:111-197: geometric radii in
 * the sum, mobility radii (fractal_vol_to_mobility_rad) in the diffusion
 * terms */
static double brown_helper(const orc_fractal *fr, double vol_i, double den_i,
                           double vol_j, double den_j, double temp,
                           double pressure, int *ok) {
  double rhoair = (pressure * C_AIR_MOLEC_WEIGHT) / (C_UNIV_GAS * temp);
  double viscosd =
      1.8325e-05 * (416.16 / (temp + 120.0)) * pow(temp / 296.16, 1.5);
  double viscosk = viscosd / rhoair;
  double gasspeed = sqrt((8.0 * C_BOLTZMANN * temp * C_AVOGADRO) /
                         (C_PI * C_AIR_MOLEC_WEIGHT));
  double gasfreepath = 2.0 * viscosk / gasspeed;

  double rad_i = frac_vol2rad(fr, vol_i);
  double rme_i = mobility_rad(fr, vol_i, temp, pressure, ok);
  double knud = gasfreepath / rme_i;
  double cunning = 1.0 + knud * (1.249 + 0.42 * exp(-0.87 / knud));
  double diffus_i =
      (C_BOLTZMANN * temp * cunning) / (6.0 * C_PI * rme_i * viscosd);
  double speedsq_i = 8.0 * C_BOLTZMANN * temp / (C_PI * den_i * vol_i);
  double freepath = 8.0 * diffus_i / (C_PI * sqrt(speedsq_i));
  double t = 2.0 * rme_i + freepath;
  double tmp1 = t * t * t;
  double tmp2 = pow(4.0 * rme_i * rme_i + freepath * freepath, 1.5);
  double d = (tmp1 - tmp2) / (6.0 * rme_i * freepath) - 2.0 * rme_i;
  double deltasq_i = d * d;

  double rad_j = frac_vol2rad(fr, vol_j);
  double rme_j = mobility_rad(fr, vol_j, temp, pressure, ok);
  knud = gasfreepath / rme_j;
  cunning = 1.0 + knud * (1.249 + 0.42 * exp(-0.87 / knud));
  double diffus_j =
      (C_BOLTZMANN * temp * cunning) / (6.0 * C_PI * rme_j * viscosd);
  double speedsq_j = 8.0 * C_BOLTZMANN * temp / (C_PI * den_j * vol_j);
  freepath = 8.0 * diffus_j / (C_PI * sqrt(speedsq_j));
  t = 2.0 * rme_j + freepath;
  tmp1 = t * t * t;
  tmp2 = pow(4.0 * rme_j * rme_j + freepath * freepath, 1.5);
  d = (tmp1 - tmp2) / (6.0 * rme_j * freepath) - 2.0 * rme_j;
  double deltasq_j = d * d;

  double rad_sum = rad_i + rad_j;
  double diffus_sum = diffus_i + diffus_j;
  tmp1 = rad_sum / (rad_sum + sqrt(deltasq_i + deltasq_j));
  tmp2 = 4.0 * diffus_sum / (rad_sum * sqrt(speedsq_i + speedsq_j));
  return 4.0 * C_PI * rad_sum * diffus_sum / (tmp1 + tmp2);
}

/* fall_g, coag_kernel_sedi.F90:110-172 (terminal velocity, Beard 1976 as
 * coded by Bott) */
static double fall_g(double r) {
  static const double b[7] = {-0.318657e1,  0.992696,     -0.153193e-2,
                              -0.987059e-3, -0.578878e-3, 0.855176e-4,
                              -0.327815e-5};
  static const double c[6] = {-0.500015e1, 0.523778e1,  -0.204914e1,
                              0.475294,    -0.542819e-1, 0.238449e-2};
  double eta = 1.818e-4, xlamb = 6.62e-6, rhow = 1.0, rhoa = 1.225e-3;
  double grav = 980.665, cunh = 1.257 * xlamb, t0 = 273.15;
  double sigma = 76.1 - 0.155 * (293.15 - t0);
  double stok = 2.0 * grav * (rhow - rhoa) / (9.0 * eta);
  double stb = 32.0 * rhoa * (rhow - rhoa) * grav / (3.0 * eta * eta);
  double eta4 = (eta * eta) * (eta * eta);
  double phy = sigma * sigma * sigma * rhoa * rhoa /
               (eta4 * grav * (rhow - rhoa));
  double py = pow(phy, 1.0 / 6.0);
  double rr = r * 1e2;
  double w = 0.0;
  if (rr <= 1e-3) {
    w = stok * (rr * rr + cunh * rr);
  } else if (rr > 1e-3 && rr <= 5.35e-2) {
    double x = log(stb * rr * rr * rr);
    double y = 0.0;
    for (int i = 1; i <= 7; i++) y = y + b[i - 1] * powi(x, i - 1);
    double xrey = (1.0 + cunh / rr) * exp(y);
    w = xrey * eta / (2.0 * rhoa * rr);
  } else if (rr > 5.35e-2) {
    double bond = grav * (rhow - rhoa) * (rr * rr) / sigma;
    if (rr > 0.35) bond = grav * (rhow - rhoa) * (0.35 * 0.35) / sigma;
    double x = log(16.0 * bond * py / 3.0);
    double y = 0.0;
    for (int i = 1; i <= 6; i++) y = y + c[i - 1] * powi(x, i - 1);
    double xrey = py * exp(y);
    w = xrey * eta / (2.0 * rhoa * rr);
    if (rr > 0.35) w = xrey * eta / (2.0 * rhoa * 0.35);
  }
  return w / 100.0;
}

/* Hall (1980) collision efficiencies as tabulated in Bott's coad1d: row k is
 * collector radius R0[k] (um), column q is radius ratio RAT[q]. */
static const double HALL_R0[15] = {6.0,  8.0,  10.0, 15.0,  20.0,
                                   25.0, 30.0, 40.0, 50.0,  60.0,
                                   70.0, 100.0, 150.0, 200.0, 300.0};
static const double HALL_RAT[21] = {0.0,  0.05, 0.1,  0.15, 0.2,  0.25, 0.3,
                                    0.35, 0.4,  0.45, 0.5,  0.55, 0.6,  0.65,
                                    0.7,  0.75, 0.8,  0.85, 0.9,  0.95, 1.0};
/* HALL_EC[q][k]: ratio column q (0..20), collector row k (0..14) */
static const double HALL_EC[21][15] = {
    {0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001,
     0.001, 0.001, 0.001, 0.001, 0.001},
    {0.003, 0.003, 0.003, 0.004, 0.005, 0.005, 0.005, 0.010, 0.100, 0.050,
     0.200, 0.500, 0.770, 0.870, 0.970},
    {0.007, 0.007, 0.007, 0.008, 0.009, 0.010, 0.010, 0.070, 0.400, 0.430,
     0.580, 0.790, 0.930, 0.960, 1.000},
    {0.009, 0.009, 0.009, 0.012, 0.015, 0.010, 0.020, 0.280, 0.600, 0.640,
     0.750, 0.910, 0.970, 0.980, 1.000},
    {0.014, 0.014, 0.014, 0.015, 0.016, 0.030, 0.060, 0.500, 0.700, 0.770,
     0.840, 0.950, 0.970, 1.000, 1.000},
    {0.017, 0.017, 0.017, 0.020, 0.022, 0.060, 0.100, 0.620, 0.780, 0.840,
     0.880, 0.950, 1.000, 1.000, 1.000},
    {0.030, 0.030, 0.024, 0.022, 0.032, 0.062, 0.200, 0.680, 0.830, 0.870,
     0.900, 0.950, 1.000, 1.000, 1.000},
    {0.025, 0.025, 0.025, 0.036, 0.043, 0.130, 0.270, 0.740, 0.860, 0.890,
     0.920, 1.000, 1.000, 1.000, 1.000},
    {0.027, 0.027, 0.027, 0.040, 0.052, 0.200, 0.400, 0.780, 0.880, 0.900,
     0.940, 1.000, 1.000, 1.000, 1.000},
    {0.030, 0.030, 0.030, 0.047, 0.064, 0.250, 0.500, 0.800, 0.900, 0.910,
     0.950, 1.000, 1.000, 1.000, 1.000},
    {0.040, 0.040, 0.033, 0.037, 0.068, 0.240, 0.550, 0.800, 0.900, 0.910,
     0.950, 1.000, 1.000, 1.000, 1.000},
    {0.035, 0.035, 0.035, 0.055, 0.079, 0.290, 0.580, 0.800, 0.900, 0.910,
     0.950, 1.000, 1.000, 1.000, 1.000},
    {0.037, 0.037, 0.037, 0.062, 0.082, 0.290, 0.590, 0.780, 0.900, 0.910,
     0.950, 1.000, 1.000, 1.000, 1.000},
    {0.037, 0.037, 0.037, 0.060, 0.080, 0.290, 0.580, 0.770, 0.890, 0.910,
     0.950, 1.000, 1.000, 1.000, 1.000},
    {0.037, 0.037, 0.037, 0.041, 0.075, 0.250, 0.540, 0.760, 0.880, 0.920,
     0.950, 1.000, 1.000, 1.000, 1.000},
    {0.037, 0.037, 0.037, 0.052, 0.067, 0.250, 0.510, 0.770, 0.880, 0.930,
     0.970, 1.000, 1.000, 1.000, 1.000},
    {0.037, 0.037, 0.037, 0.047, 0.057, 0.250, 0.490, 0.770, 0.890, 0.950,
     1.000, 1.000, 1.000, 1.000, 1.000},
    {0.036, 0.036, 0.036, 0.042, 0.048, 0.230, 0.470, 0.780, 0.920, 1.000,
     1.020, 1.020, 1.020, 1.020, 1.020},
    {0.040, 0.040, 0.035, 0.033, 0.040, 0.112, 0.450, 0.790, 1.010, 1.030,
     1.040, 1.040, 1.040, 1.040, 1.040},
    {0.033, 0.033, 0.033, 0.033, 0.033, 0.119, 0.470, 0.950, 1.300, 1.700,
     2.300, 2.300, 2.300, 2.300, 2.300},
    {0.027, 0.027, 0.027, 0.027, 0.027, 0.125, 0.520, 1.400, 2.300, 3.000,
     4.000, 4.000, 4.000, 4.000, 4.000}};

/* effic, coag_kernel_sedi.F90:180-285 (bilinear interpolation).  Returns a
 * negative value where the reference stops with pmc_stop(99). */
static double effic(double r1, double r2) {
  double rs = r1 * 1e6 < r2 * 1e6 ? r1 * 1e6 : r2 * 1e6;
  double rb = r1 * 1e6 > r2 * 1e6 ? r1 * 1e6 : r2 * 1e6;
  double rq = rs / rb;
  int ir = 1;
  for (int k = 1; k <= 15; k++)
    if (rb > HALL_R0[k - 1]) ir = k + 1;
  int iq = 1;
  for (int k = 1; k <= 21; k++)
    if (rq > HALL_RAT[k - 1]) iq = k + 1;
  double ec, p, q;
#define EC(i, j) HALL_EC[(j)-1][(i)-1]
  if (iq < 2 || iq > 21) return -1.0; /* rq outside (0, 1]: reference reads
                                          outside its table here */
  if (ir < 16) {
    if (ir >= 2) {
      p = (rb - HALL_R0[ir - 2]) / (HALL_R0[ir - 1] - HALL_R0[ir - 2]);
      q = (rq - HALL_RAT[iq - 2]) / (HALL_RAT[iq - 1] - HALL_RAT[iq - 2]);
      ec = (1.0 - p) * (1.0 - q) * EC(ir - 1, iq - 1) +
           p * (1.0 - q) * EC(ir, iq - 1) + q * (1.0 - p) * EC(ir - 1, iq) +
           p * q * EC(ir, iq);
    } else {
      q = (rq - HALL_RAT[iq - 2]) / (HALL_RAT[iq - 1] - HALL_RAT[iq - 2]);
      ec = (1.0 - q) * EC(1, iq - 1) + q * EC(1, iq);
    }
  } else {
    q = (rq - HALL_RAT[iq - 2]) / (HALL_RAT[iq - 1] - HALL_RAT[iq - 2]);
    double ek = (1.0 - q) * EC(15, iq - 1) + q * EC(15, iq);
    ec = ek < 1.0 ? ek : 1.0;
  }
#undef EC
  if (ec < 1e-20) return -1.0;
  return ec;
}

/* kernel_sedi_helper, coag_kernel_sedi.F90:79-105 */
static double sedi_helper(orc_state *st, const orc_fractal *fr, double v1,
                          double v2, double temp, double pressure) {
  int ok = 1;
  double r1 = frac_vol2rad(fr, v1);
  double r2 = frac_vol2rad(fr, v2);
  double w1 = fall_g(mobility_rad(fr, v1, temp, pressure, &ok));
  double w2 = fall_g(mobility_rad(fr, v2, temp, pressure, &ok));
  double ec = effic(r1, r2);
  if (ec < 0.0 || !ok) {
    if (st) orc_fail(st, ORC_ERR_ASSERT);
    return NAN;
  }
  double rs = r1 + r2;
  return ec * C_PI * (rs * rs) * fabs(w1 - w2);
}

static const double BETA_0 = 0.25 / (60.0 * 2e8); /* coag_kernel_constant.F90:22 */

static const double AIR_DYN_VISC = 1.78e-5; /* constants.F90:65 */

/* kernel_brown_free_helper, coag_kernel_brown_free.F90:118-147 (free
 * molecular regime) */
static double brown_free_helper(const orc_fractal *fr, double v1, double d1,
                                double v2, double d2, double temp) {
  double rho = (v1 / (v1 + v2)) * d1 + (v2 / (v1 + v2)) * d2;
  double ni = num_of_monomers(fr, v1), nj = num_of_monomers(fr, v2);
  double nif = pow(ni, 1.0 / fr->frac_dim), njf = pow(nj, 1.0 / fr->frac_dim);
  double s = nif + njf;
  return sqrt(6.0 * C_BOLTZMANN * temp * fr->prime_radius / rho *
              (1.0 / ni + 1.0 / nj)) * (s * s);
}

/* kernel_brown_cont_helper, coag_kernel_brown_cont.F90:115-144 (continuum
 * regime) */
static double brown_cont_helper(const orc_fractal *fr, double v1, double v2,
                                double temp) {
  double nif = pow(num_of_monomers(fr, v1), 1.0 / fr->frac_dim);
  double njf = pow(num_of_monomers(fr, v2), 1.0 / fr->frac_dim);
  return 2.0 * C_BOLTZMANN * temp / 3.0 / AIR_DYN_VISC *
         (1.0 / nif + 1.0 / njf) * (nif + njf);
}

static double kernel_value_fr(const orc_fractal *fr, int kt, double v1,
                              double d1, double v2, double d2, double temp,
                              double pressure, double coeff) {
  int ok = 1;
  double k = NAN;
  switch (kt) {
    case ORC_KERNEL_SEDI: return sedi_helper(NULL, fr, v1, v2, temp, pressure);
    case ORC_KERNEL_ADDITIVE: return coeff * (v1 + v2);
    case ORC_KERNEL_CONSTANT: return BETA_0;
    case ORC_KERNEL_BROWN:
      k = brown_helper(fr, v1, d1, v2, d2, temp, pressure, &ok);
      return ok ? k : NAN;
    case ORC_KERNEL_ZERO: return 0.0;
    case ORC_KERNEL_BROWN_FREE: return brown_free_helper(fr, v1, d1, v2, d2, temp);
    case ORC_KERNEL_BROWN_CONT: return brown_cont_helper(fr, v1, v2, temp);
  }
  return k;
}

double orc_kernel_value(int kt, double v1, double d1, double v2, double d2,
                        double temp, double pressure, double coeff) {
  return kernel_value_fr(&SPHERE, kt, v1, d1, v2, d2, temp, pressure, coeff);
}

double orc_kernel_value_fractal(int kt, double v1, double d1, double v2,
                                double d2, double temp, double pressure,
                                double coeff, double frac_dim,
                                double prime_radius, double vol_fill_factor) {
  orc_fractal fr = {frac_dim, prime_radius, vol_fill_factor,
                    frac_dim == 3.0 && vol_fill_factor == 1.0};
  return kernel_value_fr(&fr, kt, v1, d1, v2, d2, temp, pressure, coeff);
}

double orc_fractal_radius(double v, double frac_dim, double prime_radius,
                          double vol_fill_factor, double temp, double pressure,
                          double *mobility) {
  orc_fractal fr = {frac_dim, prime_radius, vol_fill_factor,
                    frac_dim == 3.0 && vol_fill_factor == 1.0};
  int ok = 1;
  if (mobility) *mobility = mobility_rad(&fr, v, temp, pressure, &ok);
  if (!ok && mobility) *mobility = NAN;
  return frac_vol2rad(&fr, v);
}

int orc_set_fractal(orc_state *st, double frac_dim, double prime_radius,
                    double vol_fill_factor) {
  if (!(frac_dim > 0.0 && frac_dim <= 3.0) || !(prime_radius > 0.0) ||
      !(vol_fill_factor > 0.0))
    return ORC_ERR_ARG;
  st->frac.frac_dim = frac_dim;
  st->frac.prime_radius = prime_radius;
  st->frac.vol_fill_factor = vol_fill_factor;
  st->frac.sph = frac_dim == 3.0 && vol_fill_factor == 1.0;
  st->valid_sort = 0; /* radii, bins and bounds all change */
  st->kbounds_valid = 0;
  return ORC_OK;
}

/* kernel dispatch on two particles, coag_kernel.F90:83-125 */
static double kernel_particles(orc_state *st, int kt, const double *va,
                               const double *vb, double temp, double pressure,
                               double coeff) {
  double v1 = vol_sum(va, st->n_spec), v2 = vol_sum(vb, st->n_spec);
  const orc_fractal *fr = &st->frac;
  int ok = 1;
  double k;
  switch (kt) {
    case ORC_KERNEL_SEDI: return sedi_helper(st, fr, v1, v2, temp, pressure);
    case ORC_KERNEL_ADDITIVE: return coeff * (v1 + v2);
    case ORC_KERNEL_CONSTANT: return BETA_0;
    case ORC_KERNEL_BROWN:
      k = brown_helper(fr, v1, vol_density(st, va), v2, vol_density(st, vb),
                       temp, pressure, &ok);
      if (!ok) orc_fail(st, ORC_ERR_ASSERT);
      return k;
    case ORC_KERNEL_ZERO: return 0.0;
    case ORC_KERNEL_BROWN_FREE:
      return brown_free_helper(fr, v1, vol_density(st, va), v2,
                               vol_density(st, vb), temp);
    case ORC_KERNEL_BROWN_CONT: return brown_cont_helper(fr, v1, v2, temp);
  }
  orc_fail(st, ORC_ERR_ARG);
  return 0.0;
}

/* kernel_minmax, coag_kernel.F90:130-169, with kernel_brown_minmax
 * (coag_kernel_brown.F90:58-101) sampling 3x3 densities */
void orc_kernel_minmax(orc_state *st, int kt, double v1, double v2,
                       double temp, double pressure, double coeff,
                       double *kmin, double *kmax) {
  switch (kt) {
    case ORC_KERNEL_SEDI:
      *kmin = *kmax = sedi_helper(st, &st->frac, v1, v2, temp, pressure);
      return;
    case ORC_KERNEL_ADDITIVE:
      *kmin = *kmax = coeff * (v1 + v2);
      return;
    case ORC_KERNEL_CONSTANT:
      *kmin = *kmax = BETA_0;
      return;
    case ORC_KERNEL_ZERO:
      *kmin = *kmax = 0.0;
      return;
    case ORC_KERNEL_BROWN:
    case ORC_KERNEL_BROWN_FREE:
    case ORC_KERNEL_BROWN_CONT: {
      /* kernel_brown*_minmax: 3x3 density samples */
      double dmin = st->density[0], dmax = st->density[0];
      for (int k = 1; k < st->n_spec; k++) {
        if (st->density[k] < dmin) dmin = st->density[k];
        if (st->density[k] > dmax) dmax = st->density[k];
      }
      int first = 1, ok = 1;
      const orc_fractal *fr = &st->frac;
      for (int i = 1; i <= 3; i++)
        for (int j = 1; j <= 3; j++) {
          double d1 = interp_linear_disc(dmin, dmax, 3, i);
          double d2 = interp_linear_disc(dmin, dmax, 3, j);
          double k = kt == ORC_KERNEL_BROWN
                         ? brown_helper(fr, v1, d1, v2, d2, temp, pressure, &ok)
                         : kt == ORC_KERNEL_BROWN_FREE
                               ? brown_free_helper(fr, v1, d1, v2, d2, temp)
                               : brown_cont_helper(fr, v1, v2, temp);
          if (!ok) orc_fail(st, ORC_ERR_ASSERT);
          if (first) {
            first = 0;
            *kmin = k;
            *kmax = k;
          } else {
            if (k < *kmin) *kmin = k;
            if (k > *kmax) *kmax = k;
          }
        }
      return;
    }
  }
  orc_fail(st, ORC_ERR_ARG);
}

/* coag_num_conc_factor, coag_kernel.F90:346-377 */
static double num_conc_factor(const orc_state *st, double ri, double rj,
                              int ci, int cj, int cij) {
  const orc_fractal *fr = &st->frac;
  double rij = frac_vol2rad(fr, frac_rad2vol(fr, ri) + frac_rad2vol(fr, rj));
  double nci = orc_num_conc_at_radius(st, ci, ri);
  double ncj = orc_num_conc_at_radius(st, cj, rj);
  double ncij = orc_num_conc_at_radius(st, cij, rij);
  double mn = nci;
  if (ncj < mn) mn = ncj;
  if (ncij < mn) mn = ncij;
  return nci * ncj / mn;
}

/* num_conc_weighted_kernel, coag_kernel.F90:175-209 */
static double weighted_kernel(orc_state *st, int kt, const double *va,
                              const double *vb, int ci, int cj, int cij,
                              double temp, double pressure, double coeff) {
  double k = kernel_particles(st, kt, va, vb, temp, pressure, coeff);
  double ri = frac_vol2rad(&st->frac, vol_sum(va, st->n_spec));
  double rj = frac_vol2rad(&st->frac, vol_sum(vb, st->n_spec));
  return k * num_conc_factor(st, ri, rj, ci, cj, cij);
}

double orc_weighted_kernel(orc_state *st, int kt, const double *vol1, int c1,
                           const double *vol2, int c2, int cij, double temp,
                           double pressure, double coeff) {
  return weighted_kernel(st, kt, vol1, vol2, c1, c2, cij, temp, pressure,
                         coeff);
}

/* coag_dest_class, coag_kernel.F90:382-416 -- uses centers(i_bin) for both
 * radii, as the reference does at lines 402-403. */
int orc_coag_dest_class(const orc_state *st, const double *edges,
                        const double *centers, int b1, int b2, int c1,
                        int c2) {
  (void)edges;
  (void)b2;
  double ri = centers[b1 - 1];
  double rj = centers[b1 - 1];
  const orc_fractal *fr = &st->frac;
  double rij = frac_vol2rad(fr, frac_rad2vol(fr, ri) + frac_rad2vol(fr, rj));
  double nci = orc_num_conc_at_radius(st, c1, rij);
  double ncj = orc_num_conc_at_radius(st, c2, rij);
  return nci < ncj ? c1 : c2;
}

/* max_coag_num_conc_factor, coag_kernel.F90:422-465 (5x5 radius samples) */
double orc_max_num_conc_factor(const orc_state *st, const double *edges,
                               int b1, int b2, int c1, int c2, int cc) {
  double i0 = edges[b1 - 1], i1 = edges[b1];
  double j0 = edges[b2 - 1], j1 = edges[b2];
  double fmax = 0.0;
  for (int a = 1; a <= 5; a++)
    for (int b = 1; b <= 5; b++) {
      double ri = interp_linear_disc(i0, i1, 5, a);
      double rj = interp_linear_disc(j0, j1, 5, b);
      double f = num_conc_factor(st, ri, rj, c1, c2, cc);
      if (f > fmax) fmax = f;
    }
  return fmax;
}

/* est_k_minmax_for_bin_unweighted, coag_kernel.F90:286-341 */
static void kminmax_for_bin(orc_state *st, int kt, const double *edges,
                            int b1, int b2, double temp, double pressure,
                            double coeff, double *kmin, double *kmax) {
  double v1lo = frac_rad2vol(&st->frac, edges[b1 - 1]);
  double v1hi = frac_rad2vol(&st->frac, edges[b1]);
  double v2lo = frac_rad2vol(&st->frac, edges[b2 - 1]);
  double v2hi = frac_rad2vol(&st->frac, edges[b2]);
  for (int i = 1; i <= 3; i++)
    for (int j = 1; j <= 3; j++) {
      double v1 = interp_linear_disc(v1lo, v1hi, 3, i);
      double v2 = interp_linear_disc(v2lo, v2hi, 3, j);
      double a, b;
      orc_kernel_minmax(st, kt, v1, v2, temp, pressure, coeff, &a, &b);
      if (i == 1 && j == 1) {
        *kmin = a;
        *kmax = b;
      } else {
        if (a < *kmin) *kmin = a;
        if (b > *kmax) *kmax = b;
      }
    }
  *kmax = *kmax * 2.0;
}

/* ---------------------------------------------------------------------- */
/* sorted state                                                            */

/* aero_sorted_set_bin_grid, aero_sorted.F90:116-148 */
static void sorted_set_grid(orc_state *st, int n_bin, double rmin,
                            double rmax) {
  free(st->edges);
  free(st->centers);
  free(st->kmin);
  free(st->kmax);
  st->edges = st->centers = st->kmin = st->kmax = NULL;
  st->n_bin = n_bin;
  if (n_bin > 0) {
    st->edges = (double *)malloc(sizeof(double) * (n_bin + 1));
    st->centers = (double *)malloc(sizeof(double) * n_bin);
    st->kmin = (double *)malloc(sizeof(double) * n_bin * n_bin);
    st->kmax = (double *)malloc(sizeof(double) * n_bin * n_bin);
    if (!st->edges || !st->centers || !st->kmin || !st->kmax)
      orc_fail(st, ORC_ERR_NOMEM);
    orc_bin_grid_make(n_bin, rmin, rmax, st->edges, st->centers);
  }
  rmap2_set_ranges(st, &st->size_class, n_bin, st->n_class);
  rmap2_set_ranges(st, &st->group_class, st->n_group, st->n_class);
  st->kbounds_valid = 0;
}

static int particle_in_bin(orc_state *st, int i) {
  if (st->n_bin <= 0) return -1;
  return orc_bin_find(st->n_bin, st->edges[0], st->edges[st->n_bin],
                      part_radius(st, i));
}

/* aero_sorted_sort_particles, aero_sorted.F90:185-209 */
static void sorted_sort_particles(orc_state *st) {
  rmap2_zero(&st->size_class);
  rmap2_zero(&st->group_class);
  for (int i = 1; i <= st->n_part; i++) {
    int b = particle_in_bin(st, i);
    rmap2_append(st, &st->size_class, b, st->meta[i - 1].weight_class);
    rmap2_append(st, &st->group_class, st->meta[i - 1].weight_group,
                 st->meta[i - 1].weight_class);
  }
}

/* aero_sorted_remake_if_needed without bin_grid / all_procs_same arguments,
 * aero_sorted.F90:214-373 */
static void sorted_remake_if_needed(orc_state *st, int valid_sort) {
  double rmin = 0.0, rmax = 0.0;
  if (valid_sort) {
    int bmin = 0, bmax = 0;
    for (int b = 1; b <= st->n_bin; b++) {
      int s = 0;
      for (int c = 1; c <= st->n_class; c++)
        s += rmap2_cell(&st->size_class, b, c)->n;
      if (s > 0) {
        if (bmin == 0) bmin = b;
        bmax = b;
      }
    }
    if (bmin == 0) {
      if (st->n_bin > 0) {
        rmin = st->edges[st->n_bin];
        rmax = st->edges[0];
      }
    } else {
      rmin = st->edges[bmin - 1];
      rmax = st->edges[bmax];
    }
  } else {
    for (int i = 1; i <= st->n_part; i++) {
      double r = part_radius(st, i);
      if (i == 1) {
        rmin = r;
        rmax = r;
      } else {
        if (r < rmin) rmin = r;
        if (r > rmax) rmax = r;
      }
    }
  }
  if (rmax == 0.0) {
    if (valid_sort) return;
    sorted_set_grid(st, 0, 0.0, 0.0);
    return;
  }
  int need = 0;
  if (st->n_bin < 1) {
    need = 1;
  } else {
    double gmin = st->edges[0], gmax = st->edges[st->n_bin];
    if (rmin / gmin < SORTED_BIN_SAFETY_FACTOR ||
        gmax / rmax < SORTED_BIN_SAFETY_FACTOR)
      need = 1;
  }
  if (need) {
    double gmin = rmin / SORTED_BIN_OVER_FACTOR;
    double gmax = rmax * SORTED_BIN_OVER_FACTOR;
    int n_bin =
        (int)ceil((log10(gmax) - log10(gmin)) * SORTED_BINS_PER_DECADE);
    sorted_set_grid(st, n_bin, gmin, gmax);
    sorted_sort_particles(st);
  } else if (!valid_sort) {
    sorted_sort_particles(st);
  }
}

/* aero_state_sort, aero_state.F90:3291-3307 */
static void state_sort(orc_state *st) {
  sorted_remake_if_needed(st, st->valid_sort);
  st->valid_sort = 1;
}

/* aero_particle_array_remove_particle (swap-last),
 * aero_particle_array.F90:178-198 */
static void array_remove(orc_state *st, int i) {
  if (i < 1 || i > st->n_part) orc_fail(st, ORC_ERR_ASSERT);
  if (i < st->n_part) {
    memcpy(pvol(st, i), pvol(st, st->n_part), sizeof(double) * st->n_spec);
    st->meta[i - 1] = st->meta[st->n_part - 1];
  }
  st->n_part--;
}

static void array_add(orc_state *st, const double *v,
                      const orc_particle_meta *m) {
  ensure_cap(st, st->n_part + 1);
  st->n_part++;
  memcpy(pvol(st, st->n_part), v, sizeof(double) * st->n_spec);
  st->meta[st->n_part - 1] = *m;
}

/* aero_info_array_add_aero_info (aero_info_array.F90): one aero_info
 * (aero_info.F90:48-56) of a removed particle, when records are kept */
static void log_removal(orc_state *st, int64_t id, int action, int64_t other_id) {
  if (!st->rec_removals) return;
  if (st->rm_n == st->rm_cap) {
    int64_t cap = st->rm_cap ? 2 * st->rm_cap : 1024;
    int64_t *a = (int64_t *)realloc(st->rm_id, sizeof(int64_t) * cap);
    if (a) st->rm_id = a;
    int64_t *b = (int64_t *)realloc(st->rm_other, sizeof(int64_t) * cap);
    if (b) st->rm_other = b;
    int *c = (int *)realloc(st->rm_action, sizeof(int) * cap);
    if (c) st->rm_action = c;
    if (!a || !b || !c) orc_fail(st, ORC_ERR_NOMEM);
    st->rm_cap = cap;
  }
  st->rm_id[st->rm_n] = id;
  st->rm_action[st->rm_n] = action;
  st->rm_other[st->rm_n] = other_id;
  st->rm_n++;
}

/* aero_state_remove_particle(_no_info / _with_info), aero_state.F90:382-446;
 * the callers log the removal first where the reference records it */
static void state_remove(orc_state *st, int i) {
  if (st->valid_sort) {
    array_remove(st, i);
    rmap2_remove(st, &st->size_class, i);
    rmap2_remove(st, &st->group_class, i);
  } else {
    array_remove(st, i);
  }
}

/* aero_state_add_particle -> aero_sorted_add_particle,
 * aero_state.F90:365-377, aero_sorted.F90:397-449.  allow_resort: -1 absent,
 * 0 false, 1 true. */
static void state_add(orc_state *st, const double *v,
                      const orc_particle_meta *m, int allow_resort) {
  if (!st->valid_sort) {
    array_add(st, v, m);
    return;
  }
  int b = -1;
  if (st->n_bin > 0)
    b = orc_bin_find(st->n_bin, st->edges[0], st->edges[st->n_bin],
                     frac_vol2rad(&st->frac, vol_sum(v, st->n_spec)));
  if (m->weight_group < 1 || m->weight_group > st->n_group ||
      m->weight_class < 1 || m->weight_class > st->n_class)
    orc_fail(st, ORC_ERR_ASSERT);
  array_add(st, v, m);
  if (b < 1 || b > st->n_bin) {
    if (allow_resort == 0) orc_fail(st, ORC_ERR_OUT_OF_GRID);
    sorted_remake_if_needed(st, 0);
  } else {
    rmap2_append(st, &st->size_class, b, m->weight_class);
    rmap2_append(st, &st->group_class, m->weight_group, m->weight_class);
  }
}

static void new_id(orc_state *st, orc_particle_meta *m) {
  m->id = st->next_id; /* (next_id - 1) * 1 + 0 + 1 on one process */
  st->next_id++;
}

/* aero_state_dup_particle, aero_state.F90:488-539 (random_weight_group) */
static void state_dup(orc_state *st, int i, double n_mean, int rand_group) {
  int n_copies = orc_prob_round(st, n_mean);
  if (n_copies == 0) {
    log_removal(st, st->meta[i - 1].id, ORC_INFO_WEIGHT, 0);
    state_remove(st, i);
  } else if (n_copies > 1) {
    for (int d = 1; d <= n_copies - 1; d++) {
      tpart c;
      tpart_from(st, &c, i);
      new_id(st, &c.m);
      if (rand_group) {
        int g = weight_rand_group(st, st->meta[i - 1].weight_class,
                                  part_radius(st, i));
        c.m.weight_group = g;
      }
      state_add(st, c.vol, &c.m, -1);
    }
  }
}

static int cell_n(orc_state *st, int b, int c) {
  return rmap2_cell(&st->size_class, b, c)->n;
}

static int cell_entry(orc_state *st, int b, int c, int k) {
  return rmap2_cell(&st->size_class, b, c)->e[k - 1];
}

/* ---------------------------------------------------------------------- */
/* mc_coag and its parts, coagulation.F90                                  */

typedef struct {
  int kt;
  double temp, pressure, coeff, del_t;
} coag_env;

/* coagulate_weighting, coagulation.F90:810-922 */
static void coagulate_weighting(orc_state *st, int p1, int p2, int c1, int c2,
                                int cc, tpart *ptc, int *remove_1,
                                int *remove_2, int *create_new,
                                int *id_1_lost, int *id_2_lost) {
  orc_particle_meta *m1 = &st->meta[p1 - 1], *m2 = &st->meta[p2 - 1];
  if (m1->id == m2->id) orc_fail(st, ORC_ERR_ASSERT);
  double r1 = part_radius(st, p1);
  double r2 = part_radius(st, p2);
  double rc = frac_vol2rad(&st->frac, frac_rad2vol(&st->frac, r1) +
                                         frac_rad2vol(&st->frac, r2));
  double nc1 = orc_num_conc_at_radius(st, c1, r1);
  double nc2 = orc_num_conc_at_radius(st, c2, r2);
  double ncc = orc_num_conc_at_radius(st, cc, rc);
  int new_group = weight_rand_group(st, cc, rc);
  double mn = nc1;
  if (nc2 < mn) mn = nc2;
  if (ncc < mn) mn = ncc;
  double pr1 = mn / nc1, pr2 = mn / nc2, pcn = mn / ncc;
  *remove_1 = orc_random(st) < pr1;
  *remove_2 = orc_random(st) < pr2;
  *create_new = orc_random(st) < pcn;
  if (*create_new) {
    *id_1_lost = 0;
    *id_2_lost = 0;
    if (*remove_1 && *remove_2) {
      if (part_volume(st, p1) > part_volume(st, p2))
        *id_2_lost = 1;
      else
        *id_1_lost = 1;
    }
  } else {
    *id_1_lost = *remove_1;
    *id_2_lost = *remove_2;
  }
  if (*create_new) {
    particle_coagulate(st, pvol(st, p1), m1, pvol(st, p2), m2, ptc->vol,
                       &ptc->m);
    ptc->m.weight_group = new_group;
    ptc->m.weight_class = cc;
    if (*remove_1 && !*id_1_lost) {
      ptc->m.id = m1->id;
    } else if (*remove_2 && !*id_2_lost) {
      ptc->m.id = m2->id;
    } else {
      new_id(st, &ptc->m);
    }
  }
}

/* coagulate, coagulation.F90:928-985 */
static void coagulate(orc_state *st, int p1, int p2, int c1, int c2, int cc) {
  tpart ptc;
  int rm1, rm2, cn, l1, l2;
  coagulate_weighting(st, p1, p2, c1, c2, cc, &ptc, &rm1, &rm2, &cn, &l1, &l2);
  /* aero_info_1/2 (coagulation.F90:900-920), recorded when the id is lost */
  int64_t id1 = st->meta[p1 - 1].id, id2 = st->meta[p2 - 1].id;
  int64_t other = cn ? ptc.m.id : 0;
  if (p2 > p1) {
    if (rm2) {
      if (l2) log_removal(st, id2, ORC_INFO_COAG, other);
      state_remove(st, p2);
    }
    if (rm1) {
      if (l1) log_removal(st, id1, ORC_INFO_COAG, other);
      state_remove(st, p1);
    }
  } else {
    if (rm1) {
      if (l1) log_removal(st, id1, ORC_INFO_COAG, other);
      state_remove(st, p1);
    }
    if (rm2) {
      if (l2) log_removal(st, id2, ORC_INFO_COAG, other);
      state_remove(st, p2);
    }
  }
  if (cn) state_add(st, ptc.vol, &ptc.m, 0);
}

/* find_rand_pair, coagulation.F90:766-803 */
static void find_rand_pair(orc_state *st, int b1, int b2, int c1, int c2,
                           int *i1, int *i2) {
  int n1 = cell_n(st, b1, c1), n2 = cell_n(st, b2, c2);
  if (n1 < 1) orc_fail(st, ORC_ERR_ASSERT);
  *i1 = orc_rand_int(st, n1);
  if (b1 == b2 && c1 == c2) {
    if (n2 < 2) orc_fail(st, ORC_ERR_ASSERT);
    *i2 = orc_rand_int(st, n2 - 1);
    if (*i2 == *i1) *i2 = n2;
  } else {
    if (n2 < 1) orc_fail(st, ORC_ERR_ASSERT);
    *i2 = orc_rand_int(st, n2);
  }
}

/* maybe_coag_pair, coagulation.F90:712-759 */
static int maybe_coag_pair(orc_state *st, const coag_env *env, int b1, int b2,
                           int c1, int c2, int cc, double accept_factor) {
  int i1, i2;
  find_rand_pair(st, b1, b2, c1, c2, &i1, &i2);
  int p1 = cell_entry(st, b1, c1, i1);
  int p2 = cell_entry(st, b2, c2, i2);
  double k = weighted_kernel(st, env->kt, pvol(st, p1), pvol(st, p2), c1, c2,
                             cc, env->temp, env->pressure, env->coeff);
  double p = k * accept_factor;
  if (!(p <= 1.0)) st->kmax_warn++;
  if (orc_random(st) < p) {
    coagulate(st, p1, p2, c1, c2, cc);
    return 1;
  }
  return 0;
}

/* compute_n_samp, coagulation.F90:648-702 */
static void compute_n_samp(orc_state *st, int ni, int nj, int same_bin,
                           double k_max, double del_t, int *n_samp,
                           double *accept_factor) {
  double n_possible;
  if (same_bin)
    n_possible = (double)ni * ((double)nj - 1.0) / 2.0;
  else
    n_possible = (double)ni * (double)nj;
  double r_samp = k_max * del_t;
  double mean = r_samp * n_possible;
  *n_samp = orc_rand_poisson(st, mean);
  *accept_factor = 1.0 / k_max;
}

/* per_set_coag, coagulation.F90:587-643 */
static void per_set_coag(orc_state *st, const coag_env *env, double k_max,
                         int b1, int b2, int c1, int c2, int cc,
                         int *tot_n_samp, int *tot_n_coag) {
  int n1 = cell_n(st, b1, c1), n2 = cell_n(st, b2, c2);
  int n_samp;
  double af;
  compute_n_samp(st, n1, n2, b1 == b2 && c1 == c2, k_max, env->del_t, &n_samp,
                 &af);
  *tot_n_samp += n_samp;
  for (int s = 1; s <= n_samp; s++) {
    n1 = cell_n(st, b1, c1);
    n2 = cell_n(st, b2, c2);
    if ((n1 < 2 && b1 == b2 && c1 == c2) || n1 < 1 || n2 < 1) break;
    if (maybe_coag_pair(st, env, b1, b2, c1, c2, cc, af)) (*tot_n_coag)++;
  }
}

/* determine_target_and_source, coagulation.F90:247-307 */
static int determine_target_and_source(orc_state *st, int b1, int b2, int c1,
                                       int c2, int cc, int *bt, int *bs,
                                       int *ct, int *cs) {
  int inc, dec;
  weight_monotonicity(st, &inc, &dec);
  if (!dec) return 0;
  double n1min, n1max, n2min, n2max;
  weight_minmax_nc(st, c1, st->edges[b1 - 1], st->edges[b1], &n1min, &n1max);
  weight_minmax_nc(st, c2, st->edges[b2 - 1], st->edges[b2], &n2min, &n2max);
  int ok = 0;
  if (n1max < n2min && cc == c1) {
    *bt = b1;
    *bs = b2;
    *ct = c1;
    *cs = c2;
    ok = 1;
  }
  if (n2max < n1min && cc == c2) {
    *bt = b2;
    *bs = b1;
    *ct = c2;
    *cs = c1;
    ok = 1;
  }
  return ok;
}

/* sample_source_particle, coagulation.F90:333-517.  target is a copy of the
 * target particle; src receives the averaged source particle. */
static void sample_source_particle(orc_state *st, const coag_env *env, int bs,
                                   int cs, const tpart *target,
                                   double n_samp_mean, double accept_factor,
                                   int *n_samp_out, int *n_coag_out,
                                   tpart *src) {
  int ns = st->n_spec;
  *n_samp_out = 0;
  *n_coag_out = 0;
  if (cell_n(st, bs, cs) == 0) return;
  double nc_target = orc_num_conc_at_radius(
      st, target->m.weight_class, frac_vol2rad(&st->frac, vol_sum(target->vol, ns)));
  int ct = target->m.weight_class;
  double nc_src_min = orc_num_conc_at_radius(st, cs, st->edges[bs - 1]);
  double prm_max = nc_target / nc_src_min;
  if (!(prm_max <= 1.0)) orc_fail(st, ORC_ERR_ASSERT);
  int n_remove = orc_rand_poisson(st, prm_max * n_samp_mean);
  int n_extra = orc_rand_poisson(st, (1.0 - prm_max) * n_samp_mean);
  int n_total = n_remove + n_extra;
  int n_avg = 0, n_samp = 0;
  double prob_coag_tot = 0.0;
  double vol_sq[64], vol_cv[64];
  for (int k = 0; k < ns; k++) {
    vol_sq[k] = 0.0;
    vol_cv[k] = 0.0;
  }
  tpart_zero(st, src);
  for (int i_samp = 1; i_samp <= n_total; i_samp++) {
    if (cell_n(st, bs, cs) == 0) break;
    if (n_samp > n_remove && n_avg >= 2) {
      double cv_max = 0.0;
      int found = 0;
      for (int k = 0; k < ns; k++) {
        double mean = src->vol[k] / (double)n_avg;
        if (mean > 0.0)
          vol_cv[k] = sqrt(vol_sq[k] / (double)n_avg - mean * mean) / mean;
      }
      /* maxval ignoring NaN entries; NaN if every entry is NaN */
      for (int k = 0; k < ns; k++) {
        if (isnan(vol_cv[k])) continue;
        if (!found || vol_cv[k] > cv_max) cv_max = vol_cv[k];
        found = 1;
      }
      if (!found) cv_max = NAN;
      double conf = cv_max / sqrt((double)n_avg) * orc_student_t_95(n_avg);
      if (conf < COAG_ACCEL_MAX_CV) break;
    }
    n_samp++;
    int ie = orc_rand_int(st, cell_n(st, bs, cs));
    int ip = cell_entry(st, bs, cs, ie);
    double k = weighted_kernel(st, env->kt, pvol(st, ip), target->vol, cs, ct,
                               ct, env->temp, env->pressure, env->coeff);
    double pc = k * accept_factor;
    prob_coag_tot = prob_coag_tot + pc;
    if (orc_random(st) < pc) {
      n_avg++;
      particle_coagulate(st, src->vol, &src->m, pvol(st, ip), &st->meta[ip - 1],
                         src->vol, &src->m);
      double *vi = pvol(st, ip);
      for (int q = 0; q < ns; q++) vol_sq[q] = vol_sq[q] + vi[q] * vi[q];
      if (i_samp <= n_remove) {
        double nc_i = orc_num_conc_at_radius(st, st->meta[ip - 1].weight_class,
                                             part_radius(st, ip));
        double pri = nc_target / nc_i;
        if (orc_random(st) < pri / prm_max) {
          /* coagulation.F90:447-453 */
          log_removal(st, st->meta[ip - 1].id, ORC_INFO_COAG, target->m.id);
          state_remove(st, ip);
        }
      }
    }
  }
  *n_samp_out = n_samp;
  if (n_avg == 0) return;
  double pc_mean = prob_coag_tot / (double)n_samp;
  if (!(pc_mean <= 1.0)) st->kmax_warn++;
  int n_coag = orc_rand_binomial(st, n_total, pc_mean);
  *n_coag_out = n_coag;
  for (int q = 0; q < ns; q++)
    src->vol[q] = src->vol[q] * ((double)n_coag / (double)n_avg);
  src->m.n_primary_parts = orc_prob_round(
      st, (double)src->m.n_primary_parts * ((double)n_coag / (double)n_avg));
  int n_comp = src->m.n_comp;
  int n_new = src->m.n_primary_parts < ORC_MAX_COMPONENT
                  ? src->m.n_primary_parts
                  : ORC_MAX_COMPONENT;
  int sample[ORC_MAX_COMPONENT];
  if (n_new < n_comp) {
    orc_particle_meta m = src->m;
    sample_wo_replacement(st, n_new, n_comp, sample);
    for (int i = 0; i < n_new; i++) {
      m.comp_source[i] = src->m.comp_source[sample[i] - 1];
      m.comp_create_time[i] = src->m.comp_create_time[sample[i] - 1];
    }
    m.n_comp = n_new;
    src->m = m;
  } else if (n_comp < ORC_MAX_COMPONENT) {
    orc_particle_meta m = src->m;
    int i_comp = 1;
    if (n_comp == 0 && n_new > 0) orc_fail(st, ORC_ERR_ASSERT); /* the
        reference loops forever here */
    while (i_comp <= n_new) {
      if (i_comp + n_comp <= n_new) {
        for (int i = 1; i <= n_comp; i++) {
          m.comp_source[i_comp + i - 2] = src->m.comp_source[i - 1];
          m.comp_create_time[i_comp + i - 2] = src->m.comp_create_time[i - 1];
        }
        i_comp += n_comp;
      } else {
        int size = n_new - i_comp + 1;
        sample_wo_replacement(st, size, n_comp, sample);
        for (int i = 1; i <= size; i++) {
          m.comp_source[i_comp + i - 2] = src->m.comp_source[sample[i - 1] - 1];
          m.comp_create_time[i_comp + i - 2] =
              src->m.comp_create_time[sample[i - 1] - 1];
        }
        i_comp = n_new + 1;
      }
    }
    m.n_comp = n_new;
    src->m = m;
  }
  if (src->m.n_primary_parts < src->m.n_comp) orc_fail(st, ORC_ERR_ASSERT);
}

/* coag_target_with_source, coagulation.F90:522-582 */
static void coag_target_with_source(orc_state *st, int bt, int ct, int entry,
                                    const tpart *src, int cc) {
  int ns = st->n_spec;
  int tp = cell_entry(st, bt, ct, entry);
  int64_t tid = st->meta[tp - 1].id;
  double old_nc = orc_num_conc_at_radius(st, st->meta[tp - 1].weight_class,
                                         part_radius(st, tp));
  particle_coagulate(st, pvol(st, tp), &st->meta[tp - 1], src->vol, &src->m,
                     pvol(st, tp), &st->meta[tp - 1]);
  st->meta[tp - 1].id = tid;
  int g = weight_rand_group(st, cc, part_radius(st, tp));
  st->meta[tp - 1].weight_group = g;
  st->meta[tp - 1].weight_class = cc;
  int nb = particle_in_bin(st, tp);
  if (nb < 1 || nb > st->n_bin) orc_fail(st, ORC_ERR_OUT_OF_GRID);
  rmap2_change(st, &st->size_class, tp, nb, cc);
  rmap2_change(st, &st->group_class, tp, g, cc);
  double new_nc = orc_num_conc_at_radius(st, st->meta[tp - 1].weight_class,
                                         part_radius(st, tp));
  state_dup(st, tp, old_nc / new_nc, 1);
  if (st->meta[tp - 1].id != tid) orc_fail(st, ORC_ERR_ASSERT);
  (void)ns;
}

/* try_per_particle_coag, coagulation.F90:150-241 */
static int try_per_particle_coag(orc_state *st, const coag_env *env,
                                 double k_max, int b1, int b2, int c1, int c2,
                                 int cc, int *tot_n_samp, int *tot_n_coag) {
  int bt, bs, ct, cs;
  if (!determine_target_and_source(st, b1, b2, c1, c2, cc, &bt, &bs, &ct, &cs))
    return 0;
  /* compute_n_source, coagulation.F90:311-328 */
  double nspt = k_max * env->del_t * (double)cell_n(st, bs, cs);
  double af = 1.0 / k_max;
  if (nspt < COAG_ACCEL_N_EVENT) return 0;
  double min_tv = frac_rad2vol(&st->frac, st->edges[bt - 1]);
  double max_sv = frac_rad2vol(&st->frac, st->edges[bs]);
  double max_new = min_tv + max_sv * nspt;
  if (max_new / min_tv > MAX_ALLOWABLE_GROWTH_FACTOR) return 0;
  for (int e = cell_n(st, bt, ct); e >= 1; e--) {
    int tp = cell_entry(st, bt, ct, e);
    tpart target, src;
    tpart_from(st, &target, tp);
    int n_samp, n_coag;
    st->pp_targets++;
    sample_source_particle(st, env, bs, cs, &target, nspt, af, &n_samp,
                           &n_coag, &src);
    if (n_coag > 0) coag_target_with_source(st, bt, ct, e, &src, cc);
    *tot_n_samp += n_samp;
    *tot_n_coag += n_coag;
  }
  return 1;
}

/* mc_coag_for_bin, coagulation.F90:101-145 */
static void mc_coag_for_bin(orc_state *st, const coag_env *env, int b1, int b2,
                            int c1, int c2, int *tot_n_samp, int *tot_n_coag) {
  int cc = orc_coag_dest_class(st, st->edges, st->centers, b1, b2, c1, c2);
  double f_max = orc_max_num_conc_factor(st, st->edges, b1, b2, c1, c2, cc);
  double k_max = st->kmax[(b1 - 1) + st->n_bin * (b2 - 1)] * f_max;
  if (try_per_particle_coag(st, env, k_max, b1, b2, c1, c2, cc, tot_n_samp,
                            tot_n_coag))
    return;
  per_set_coag(st, env, k_max, b1, b2, c1, c2, cc, tot_n_samp, tot_n_coag);
}

static void compute_kbounds(orc_state *st, int kt, double temp,
                            double pressure, double coeff) {
  for (int i = 1; i <= st->n_bin; i++)
    for (int j = 1; j <= st->n_bin; j++)
      kminmax_for_bin(st, kt, st->edges, i, j, temp, pressure, coeff,
                      &st->kmin[(i - 1) + st->n_bin * (j - 1)],
                      &st->kmax[(i - 1) + st->n_bin * (j - 1)]);
}

int orc_mc_coag(orc_state *st, int kt, double temp, double pressure,
                double coeff, double del_t, int *tot_n_samp, int *tot_n_coag) {
  jmp_buf jb;
  *tot_n_samp = 0;
  *tot_n_coag = 0;
  if (kt < ORC_KERNEL_SEDI || kt > ORC_KERNEL_BROWN_CONT) return ORC_ERR_ARG;
  st->fail = &jb;
  st->fail_code = ORC_OK;
  if (setjmp(jb)) {
    st->fail = NULL;
    return st->fail_code;
  }
  coag_env env = {kt, temp, pressure, coeff, del_t};
  state_sort(st);
  if (!st->kbounds_valid) {
    compute_kbounds(st, kt, temp, pressure, coeff);
    st->kbounds_valid = 1;
  }
  for (int c1 = 1; c1 <= st->n_class; c1++)
    for (int c2 = 1; c2 <= c1; c2++)
      for (int b1 = 1; b1 <= st->n_bin; b1++) {
        if (cell_n(st, b1, c1) == 0) continue;
        int b2s = (c1 == c2) ? b1 : 1;
        for (int b2 = b2s; b2 <= st->n_bin; b2++) {
          if (cell_n(st, b2, c2) == 0) continue;
          mc_coag_for_bin(st, &env, b1, b2, c1, c2, tot_n_samp, tot_n_coag);
        }
      }
  st->fail = NULL;
  return ORC_OK;
}

int64_t orc_kmax_warnings(const orc_state *st) { return st->kmax_warn; }
int64_t orc_pp_targets(const orc_state *st) { return st->pp_targets; }

/* ---------------------------------------------------------------------- */
/* creation / IO                                                           */

orc_state *orc_create(int n_spec, const double *density, int i_water,
                      int n_group, int n_class, const int *w_type,
                      const double *w_mag, const double *w_exp) {
  if (n_spec < 1 || n_spec > 64 || n_group < 1 || n_group > 64 || n_class < 1)
    return NULL;
  orc_state *st = (orc_state *)calloc(1, sizeof(orc_state));
  if (!st) return NULL;
  st->frac = SPHERE;
  st->n_spec = n_spec;
  st->density = (double *)malloc(sizeof(double) * n_spec);
  memcpy(st->density, density, sizeof(double) * n_spec);
  st->i_water = i_water;
  st->n_group = n_group;
  st->n_class = n_class;
  st->w_type = (int *)malloc(sizeof(int) * n_group * n_class);
  st->w_mag = (double *)malloc(sizeof(double) * n_group * n_class);
  st->w_exp = (double *)malloc(sizeof(double) * n_group * n_class);
  orc_set_weight(st, w_type, w_mag, w_exp);
  st->next_id = 1;
  orc_set_seed(st, 1);
  return st;
}

int orc_set_weight(orc_state *st, const int *w_type, const double *w_mag,
                   const double *w_exp) {
  int n = st->n_group * st->n_class;
  memcpy(st->w_type, w_type, sizeof(int) * n);
  memcpy(st->w_mag, w_mag, sizeof(double) * n);
  memcpy(st->w_exp, w_exp, sizeof(double) * n);
  return ORC_OK;
}

void orc_destroy(orc_state *st) {
  if (!st) return;
  free(st->density);
  free(st->w_type);
  free(st->w_mag);
  free(st->w_exp);
  free(st->vol);
  free(st->meta);
  free(st->edges);
  free(st->centers);
  free(st->kmin);
  free(st->kmax);
  rmap2_free(&st->size_class);
  rmap2_free(&st->group_class);
  free(st->dump);
  free(st->rm_id);
  free(st->rm_other);
  free(st->rm_action);
  free(st);
}

void orc_set_record_removals(orc_state *st, int on) { st->rec_removals = on != 0; }

int64_t orc_removals(orc_state *st, int64_t max_n, int64_t *id, int *action,
                     int64_t *other_id) {
  int64_t n = st->rm_n;
  if (n > max_n) return -n;
  for (int64_t k = 0; k < n; k++) {
    id[k] = st->rm_id[k];
    action[k] = st->rm_action[k];
    other_id[k] = st->rm_other[k];
  }
  st->rm_n = 0;
  return n;
}

void orc_set_next_id(orc_state *st, int64_t id) { st->next_id = id; }
int64_t orc_get_next_id(const orc_state *st) { return st->next_id; }

int orc_add_particles(orc_state *st, int n, const double *vol,
                      const orc_particle_meta *meta) {
  jmp_buf jb;
  st->fail = &jb;
  if (setjmp(jb)) {
    st->fail = NULL;
    return st->fail_code;
  }
  for (int i = 0; i < n; i++) {
    if (meta[i].n_comp < 0 || meta[i].n_comp > ORC_MAX_COMPONENT)
      orc_fail(st, ORC_ERR_ARG);
    state_add(st, vol + (size_t)i * st->n_spec, &meta[i], -1);
  }
  st->fail = NULL;
  return ORC_OK;
}

int orc_n_part(const orc_state *st) { return st->n_part; }

int orc_get_particles(const orc_state *st, double *vol,
                      orc_particle_meta *meta) {
  if (vol) memcpy(vol, st->vol, sizeof(double) * (size_t)st->n_part * st->n_spec);
  if (meta) memcpy(meta, st->meta, sizeof(orc_particle_meta) * st->n_part);
  return st->n_part;
}

int orc_sort(orc_state *st) {
  jmp_buf jb;
  st->fail = &jb;
  if (setjmp(jb)) {
    st->fail = NULL;
    return st->fail_code;
  }
  state_sort(st);
  st->fail = NULL;
  return ORC_OK;
}

int orc_n_bin(const orc_state *st) { return st->n_bin; }

int orc_bin_edges(const orc_state *st, double *edges) {
  if (st->n_bin > 0) memcpy(edges, st->edges, sizeof(double) * (st->n_bin + 1));
  return st->n_bin;
}

int orc_bin_counts(const orc_state *st, int *counts) {
  for (int c = 1; c <= st->n_class; c++)
    for (int b = 1; b <= st->n_bin; b++)
      counts[(b - 1) + st->n_bin * (c - 1)] =
          st->size_class.inv[(b - 1) + st->size_class.n_r1 * (c - 1)].n;
  return st->n_bin;
}

int orc_particle_bins(const orc_state *st, int *bins) {
  if (!st->valid_sort) return ORC_ERR_ARG;
  memcpy(bins, st->size_class.fwd1.e, sizeof(int) * st->n_part);
  return ORC_OK;
}

/* aero_sorted_check + integer_rmap2_check, aero_sorted.F90:499-560,
 * integer_rmap2.F90:248-... */
int orc_check(const orc_state *st) {
  if (!st->valid_sort) return ORC_OK;
  const rmap2 *maps[2] = {&st->size_class, &st->group_class};
  for (int w = 0; w < 2; w++) {
    const rmap2 *m = maps[w];
    if (m->fwd1.n != st->n_part || m->fwd2.n != st->n_part ||
        m->index.n != st->n_part)
      return 10 + w;
    for (int i = 1; i <= st->n_part; i++) {
      int j1 = m->fwd1.e[i - 1], j2 = m->fwd2.e[i - 1], k = m->index.e[i - 1];
      if (j1 < 1 || j1 > m->n_r1 || j2 < 1 || j2 > m->n_r2) return 20 + w;
      const ivec *c = &m->inv[(j1 - 1) + m->n_r1 * (j2 - 1)];
      if (k < 1 || k > c->n || c->e[k - 1] != i) return 30 + w;
    }
    int tot = 0;
    for (int q = 0; q < m->n_r1 * m->n_r2; q++) tot += m->inv[q].n;
    if (tot != st->n_part) return 40 + w;
  }
  for (int i = 1; i <= st->n_part; i++) {
    int b = orc_bin_find(st->n_bin, st->edges[0], st->edges[st->n_bin],
                         frac_vol2rad(&st->frac,
                                      vol_sum(st->vol + (size_t)(i - 1) * st->n_spec,
                                              st->n_spec)));
    if (b != st->size_class.fwd1.e[i - 1]) return 50;
    if (st->meta[i - 1].weight_group != st->group_class.fwd1.e[i - 1] ||
        st->meta[i - 1].weight_class != st->group_class.fwd2.e[i - 1])
      return 51;
  }
  return ORC_OK;
}

int orc_kmax_table(orc_state *st, int kt, double temp, double pressure,
                   double coeff, double *kmin, double *kmax) {
  jmp_buf jb;
  st->fail = &jb;
  if (setjmp(jb)) {
    st->fail = NULL;
    return st->fail_code;
  }
  compute_kbounds(st, kt, temp, pressure, coeff);
  st->kbounds_valid = 1;
  memcpy(kmin, st->kmin, sizeof(double) * st->n_bin * st->n_bin);
  memcpy(kmax, st->kmax, sizeof(double) * st->n_bin * st->n_bin);
  st->fail = NULL;
  return ORC_OK;
}

/* ---------------------------------------------------------------------- */
/* many populations on host threads                                        */

typedef struct {
  orc_state **states;
  int n_states;
  int next;
  pthread_mutex_t mu;
  int kt;
  const double *temp, *pressure;
  double coeff, del_t;
  int n_steps;
  int64_t samp, coag;
  int err;
} many_job;

static void *many_worker(void *arg) {
  many_job *j = (many_job *)arg;
  int64_t ls = 0, lc = 0;
  int err = 0;
  for (;;) {
    pthread_mutex_lock(&j->mu);
    int p = j->next++;
    pthread_mutex_unlock(&j->mu);
    if (p >= j->n_states) break;
    for (int s = 0; s < j->n_steps; s++) {
      int a, b;
      int rc = orc_mc_coag(j->states[p], j->kt, j->temp[p], j->pressure[p],
                           j->coeff, j->del_t, &a, &b);
      if (rc) {
        err = rc;
        break;
      }
      ls += a;
      lc += b;
    }
  }
  pthread_mutex_lock(&j->mu);
  j->samp += ls;
  j->coag += lc;
  if (err) j->err = err;
  pthread_mutex_unlock(&j->mu);
  return NULL;
}

int orc_step_many(orc_state **states, int n_states, int n_threads, int kt,
                  const double *temp, const double *pressure, double coeff,
                  double del_t, int n_steps, int64_t *tot_n_samp,
                  int64_t *tot_n_coag) {
  many_job j;
  memset(&j, 0, sizeof(j));
  j.states = states;
  j.n_states = n_states;
  pthread_mutex_init(&j.mu, NULL);
  j.kt = kt;
  j.temp = temp;
  j.pressure = pressure;
  j.coeff = coeff;
  j.del_t = del_t;
  j.n_steps = n_steps;
  if (n_threads < 1) n_threads = 1;
  pthread_t th[256];
  if (n_threads > 256) n_threads = 256;
  for (int t = 0; t < n_threads; t++) pthread_create(&th[t], NULL, many_worker, &j);
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  pthread_mutex_destroy(&j.mu);
  *tot_n_samp = j.samp;
  *tot_n_coag = j.coag;
  return j.err;
}

/* ---------------------------------------------------------------------- */
/* sampler histograms for the test/rand checks (test_poisson_sample.F90,  */
/* test_binomial_sample.F90): counts[k] for k = 0..k_max                  */

void orc_poisson_hist(orc_state *st, double mean, int64_t n, int k_max,
                      int64_t *counts) {
  for (int k = 0; k <= k_max; k++) counts[k] = 0;
  for (int64_t i = 0; i < n; i++) {
    int k = orc_rand_poisson(st, mean);
    if (k <= k_max) counts[k]++;
  }
}

void orc_binomial_hist(orc_state *st, int nn, double p, int64_t n, int k_max,
                       int64_t *counts) {
  for (int k = 0; k <= k_max; k++) counts[k] = 0;
  for (int64_t i = 0; i < n; i++) {
    int k = orc_rand_binomial(st, nn, p);
    if (k <= k_max) counts[k]++;
  }
}

/* ---------------------------------------------------------------------- */
/* aero_state_rebalance with aero_state_double / aero_state_halve,        */
/* aero_state.F90:1722-1852 (one process)                                 */

static int count_group_class(const orc_state *st, int g, int c) {
  int n = 0;
  for (int i = 0; i < st->n_part; i++)
    if (st->meta[i].weight_group == g && st->meta[i].weight_class == c) n++;
  return n;
}

static void state_double(orc_state *st, int g, int c) {
  int n = st->n_part;
  for (int i = 1; i <= n; i++) {
    if (st->meta[i - 1].weight_group == g && st->meta[i - 1].weight_class == c) {
      tpart t;
      tpart_from(st, &t, i);
      new_id(st, &t.m);
      state_add(st, t.vol, &t.m, -1);
    }
  }
  st->valid_sort = 0;
  st->w_mag[(g - 1) + st->n_group * (c - 1)] *= 0.5;
}

static void state_halve(orc_state *st, int g, int c) {
  for (int i = st->n_part; i >= 1; i--) {
    if (st->meta[i - 1].weight_group == g && st->meta[i - 1].weight_class == c) {
      if (orc_random(st) < 0.5) {
        log_removal(st, st->meta[i - 1].id, ORC_INFO_HALVED, 0);
        state_remove(st, i);
      }
    }
  }
  st->w_mag[(g - 1) + st->n_group * (c - 1)] *= 2.0;
}

int orc_rebalance(orc_state *st, const double *n_part_ideal, int allow_doubling,
                  int allow_halving) {
  jmp_buf jb;
  st->fail = &jb;
  if (setjmp(jb)) {
    st->fail = NULL;
    return st->fail_code;
  }
  if (allow_doubling)
    for (int g = 1; g <= st->n_group; g++)
      for (int c = 1; c <= st->n_class; c++) {
        double ideal = n_part_ideal[(g - 1) + st->n_group * (c - 1)];
        int n = count_group_class(st, g, c);
        while ((double)n < ideal / 2.0 && n > 0) {
          state_double(st, g, c);
          n = count_group_class(st, g, c);
        }
      }
  if (allow_halving)
    for (int g = 1; g <= st->n_group; g++)
      for (int c = 1; c <= st->n_class; c++) {
        double ideal = n_part_ideal[(g - 1) + st->n_group * (c - 1)];
        while ((double)count_group_class(st, g, c) > ideal * 2.0)
          state_halve(st, g, c);
      }
  st->fail = NULL;
  return ORC_OK;
}

int orc_get_weight(const orc_state *st, double *w_mag) {
  memcpy(w_mag, st->w_mag, sizeof(double) * st->n_group * st->n_class);
  return ORC_OK;
}

/* coad, run_sect.F90:283-359: the loss and gain of one time step over every
 * bin pair (i <= j) inside the occupied range, in the reference's order. */
void orc_sect_coad(int n_bin, const double *c, const int *ima, double *g, const double *e, const double *ck) {
  const double gmin = 1e-60;
  int i0, i1;
  /* the Fortran loops leave i0 = n_bin and i1 = 0 when nothing is found */
  for (i0 = 0; i0 < n_bin - 1; i0++)
    if (g[i0] > gmin) break;
  for (i1 = n_bin - 2; i1 >= 0; i1--)
    if (g[i1] > gmin) break;
  for (int i = i0; i <= i1; i++)
    for (int j = i; j <= i1; j++) {
      int k = ima[i * n_bin + j];
      double x0 = ck[i * n_bin + j] * g[i] * g[j];
      double t = g[i] * e[j];
      x0 = x0 < t ? x0 : t;
      if (j != k) {
        t = g[j] * e[i];
        x0 = x0 < t ? x0 : t;
      }
      double gsi = x0 / e[j], gsj = x0 / e[i], gsk = gsi + gsj;
      g[i] = g[i] - gsi;
      g[j] = g[j] - gsj;
      if (k >= 0) {
        int kp = k + 1;
        double gk = g[k] + gsk;
        if (gk > gmin) {
          double x1 = log(g[kp] / gk + 1e-60);
          double flux = gsk / x1 * (exp(0.5 * x1) - exp(x1 * (0.5 - c[i * n_bin + j])));
          flux = flux < gk ? flux : gk;
          g[k] = gk - flux;
          g[kp] = g[kp] + flux;
        }
      }
    }
}
