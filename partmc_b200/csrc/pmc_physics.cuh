// pmc_physics.cuh -- device/host physics of PartMC's coagulation step.
//
// Every function states the reference routine (path:line in the PartMC
// source tree) whose arithmetic it follows.  The FP64 forms keep the
// reference's evaluation order; the per-particle terms of the Brownian and
// sedimentation kernels are split from the pair terms so that a pair test
// reads two precomputed particle records instead of recomputing both
// particles (the pair formula is unchanged).
#pragma once

#include <cstdint>
#include <cmath>

#ifndef PMC_HD
#define PMC_HD __host__ __device__ __forceinline__
#endif

namespace pmc {

// src/constants.F90:31-61
constexpr double kPi = 3.14159265358979323846;
constexpr double kBoltzmann = 1.3806505e-23;
constexpr double kAvogadro = 6.02214179e23;
constexpr double kUnivGas = 8.314472;
constexpr double kAirMolecWeight = 2.89644e-2;
constexpr double kWaterDensity = 1e3;

// coag_kernel.F90:29-45
enum KernelType : int {
  kKernelSedi = 1,
  kKernelAdditive = 2,
  kKernelConstant = 3,
  kKernelBrown = 4,
  kKernelZero = 5,
  kKernelBrownFree = 6,  // coag_kernel_brown_free.F90 (free molecular regime)
  kKernelBrownCont = 7   // coag_kernel_brown_cont.F90 (continuum regime)
};
constexpr double kAirDynVisc = 1.78e-5;  // constants.F90:65
// aero_weight.F90:24-30
enum WeightType : int { kWeightNone = 1, kWeightPower = 2, kWeightMfa = 3 };

constexpr double kBeta0 = 0.25 / (60.0 * 2e8);  // coag_kernel_constant.F90:22
constexpr int kMaxComponent = 20;               // aero_particle.F90:22
constexpr int kMaxSpec = 64;
constexpr int kMaxGroup = 4;
constexpr int kMaxClass = 4;
constexpr int kMaxBin = 256;

// sphere_vol2rad, util.F90:240-247
PMC_HD double vol2rad(double v) { return pow(3.0 * v / 4.0 / kPi, 1.0 / 3.0); }
// sphere_rad2vol, util.F90:264-271
PMC_HD double rad2vol(double r) { return 4.0 * kPi * (r * r * r) / 3.0; }
PMC_HD float vol2rad(float v) { return cbrtf(v * (float)(3.0 / (4.0 * kPi))); }
PMC_HD float rad2vol(float r) { return (float)(4.0 * kPi / 3.0) * (r * r * r); }

// fractal_t (fractal.F90:59-66, after Naumann 2003): volume fractal
// dimension, primary-particle radius (m) and volume filling factor.  With
// d_f = 3 and f = 1 (fractal_is_spherical) every conversion is the sphere's.
struct Fractal {
  double frac_dim, prime_radius, vol_fill_factor;
  int spherical;
};
// fractal_set_spherical, fractal.F90:73-82
PMC_HD Fractal fractal_spherical() { return Fractal{3.0, 1e-8, 1.0, 1}; }
PMC_HD Fractal make_fractal(double frac_dim, double prime_radius, double vol_fill_factor) {
  return Fractal{frac_dim, prime_radius, vol_fill_factor, (frac_dim == 3.0 && vol_fill_factor == 1.0) ? 1 : 0};
}

// fractal_vol_to_num_of_monomers, fractal.F90:90-100: (r_sphere(v) / R0)^3
PMC_HD double num_of_monomers(const Fractal& F, double v) {
  double x = vol2rad(v) / F.prime_radius;
  return x * x * x;
}
// fractal_vol2rad, fractal.F90:106-121: R0 (N f)^(1/d_f)
PMC_HD double vol2rad(const Fractal& F, double v) {
  if (F.spherical) return vol2rad(v);
  return F.prime_radius * pow(num_of_monomers(F, v) * F.vol_fill_factor, 1.0 / F.frac_dim);
}
PMC_HD float vol2rad(const Fractal& F, float v) {
  if (F.spherical) return vol2rad(v);
  float x = vol2rad(v) / (float)F.prime_radius;
  return (float)F.prime_radius * powf(x * x * x * (float)F.vol_fill_factor, (float)(1.0 / F.frac_dim));
}
// fractal_rad2vol, fractal.F90:142-157: V(R0) (r / R0)^d_f / f
PMC_HD double rad2vol(const Fractal& F, double r) {
  if (F.spherical) return rad2vol(r);
  return rad2vol(F.prime_radius) * pow(r / F.prime_radius, F.frac_dim) / F.vol_fill_factor;
}
PMC_HD float rad2vol(const Fractal& F, float r) {
  if (F.spherical) return rad2vol(r);
  return (float)(rad2vol(F.prime_radius) / F.vol_fill_factor) * powf(r / (float)F.prime_radius, (float)F.frac_dim);
}

// air_mean_free_path, util.F90:289-312
PMC_HD double air_mean_free_path(double temp, double pressure) {
  double rhoair = (pressure * kAirMolecWeight) / (kUnivGas * temp);
  double viscosd = (1.8325e-5 * (296.16 + 120.0) / (temp + 120.0)) * pow(temp / 296.16, 1.5);
  double viscosk = viscosd / rhoair;
  double gasspeed = sqrt(8.0 * kBoltzmann * temp * kAvogadro / (kPi * kAirMolecWeight));
  return 2.0 * viscosk / gasspeed;
}

// slip-correction and accessible-surface constants, fractal.F90:43-53
constexpr double kFracASlip = 1.142, kFracQSlip = 0.588, kFracBSlip = 0.999;
constexpr double kFracScaleFactorSAcc = 1.0, kFracScaleExponentSAcc = 0.86;

// fractal_surface_frac_dim, fractal.F90:177-191 (d_f above 3 is rejected
// when the parameters are set)
PMC_HD double surface_frac_dim(const Fractal& F) { return F.frac_dim <= 2.0 ? 3.0 : 6.0 / F.frac_dim; }
// fractal_vol_to_accessible_surface, fractal.F90:199-216 (Naumann eq. 26)
PMC_HD double accessible_surface(const Fractal& F, double v) {
  double ds = surface_frac_dim(F);
  double n = num_of_monomers(F, v);
  return 4.0 * kPi * (F.prime_radius * F.prime_radius) * pow(n, ds / 3.0) *
         ((ds - 2.0) * pow(kFracScaleFactorSAcc / n, 1.0 - kFracScaleExponentSAcc) - ds + 3.0);
}
// fractal_kirkwood_riseman, fractal.F90:223-231 (Naumann eq. 21)
PMC_HD double kirkwood_riseman(const Fractal& F) {
  return -0.06483 * (F.frac_dim * F.frac_dim) + 0.6353 * F.frac_dim - 0.4898;
}
// fractal_vol_to_mobility_rad_in_continuum, fractal.F90:239-249
PMC_HD double mobility_rad_in_continuum(const Fractal& F, double v) { return kirkwood_riseman(F) * vol2rad(F, v); }
// fractal_vol_to_effective_rad, fractal.F90:257-268 (Naumann eq. 28)
PMC_HD double effective_rad(const Fractal& F, double v) {
  return accessible_surface(F, v) / 4.0 / kPi / mobility_rad_in_continuum(F, v);
}
// fractal_slip_correct, fractal.F90:276-291, with the mean free path fp
PMC_HD double slip_correct(double r_eff, double fp) {
  return 1.0 + kFracASlip * fp / r_eff + kFracQSlip * fp / r_eff * exp(-kFracBSlip * r_eff / fp);
}

// fractal_vol_to_mobility_rad, fractal.F90:315-362: the mobility-equivalent
// radius x solves C(R_eff) x^2 - R_mec x - R_mec Q fp exp(-B x / fp)
// - R_mec A fp = 0 (Naumann eq. 30), by Newton's method from x = R_mec with
// the reference's relative step tolerance 1e-14 and at most 10 steps.  fp is
// air_mean_free_path(temp, pressure).  *ok is cleared where the reference
// stops (no convergence before the 10th step, assert 728724732).
PMC_HD double mobility_rad(const Fractal& F, double v, double fp, bool* ok) {
  if (F.spherical) return vol2rad(F, v);
  double rmec = mobility_rad_in_continuum(F, v);
  double c_reff = slip_correct(effective_rad(F, v), fp);
  double a1 = c_reff, a2 = -rmec, a3 = -rmec * kFracQSlip * fp, a4 = -kFracBSlip / fp;
  double a5 = -rmec * kFracASlip * fp;
  double x = rmec;
  int step;
  for (step = 1; step <= 10; step++) {
    double e = exp(a4 * x);
    double f = a1 * (x * x) + a2 * x + a3 * e + a5;
    double df = 2.0 * a1 * x + a2 + a3 * a4 * e;
    x = x - f / df;
    if (fabs(f / df) / (fabs(x + f / df) + fabs(x)) < 1e-14) break;
  }
  if (!(step < 10)) *ok = false;
  return x;
}

// interp_linear_disc, util.F90:663-683
PMC_HD double interp_linear_disc(double x1, double xn, int n, int i) {
  if (x1 == xn) return x1;
  double a = (double)(i - 1) / (double)(n - 1);
  return (1.0 - a) * x1 + a * xn;
}

// fast_pow, util.F90:1978-2003
template <class T>
PMC_HD T fast_pow(T b, T e) {
  if (e == T(0)) return T(1);
  if (e == T(1)) return b;
  if (e == T(2)) return b * b;
  if (e == T(3)) return b * b * b;
  if (e == T(-1)) return T(1) / b;
  if (e == T(-2)) return T(1) / (b * b);
  if (e == T(-3)) return T(1) / (b * b * b);
  return pow(b, e);
}

// integer power by squaring (the code gfortran emits for x**i with a
// variable integer exponent, as in coag_kernel_sedi.F90:150,162)
PMC_HD double powi(double x, int m) {
  unsigned n = m < 0 ? (unsigned)(-m) : (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

// Weights of one population: n_group x n_class, entry (g, c) 0-based at
// g + kMaxGroup * c.
struct Weights {
  int n_group, n_class;
  int type[kMaxGroup * kMaxClass];
  double mag[kMaxGroup * kMaxClass];
  double expo[kMaxGroup * kMaxClass];
};

// aero_weight_num_conc_at_radius, aero_weight.F90:127-146 (g, c 0-based)
template <class T>
PMC_HD T weight_nc(const Weights& w, int g, int c, T r) {
  int k = g + kMaxGroup * c;
  if (w.type[k] == kWeightNone) return (T)w.mag[k];
  return (T)w.mag[k] * fast_pow<T>(r, (T)w.expo[k]);
}

// aero_weight_array_num_conc_at_radius (harmonic combination over groups),
// aero_weight_array.F90:232-252 (c 0-based)
template <class T>
PMC_HD T num_conc_at_radius(const Weights& w, int c, T r) {
  T inv_sum = T(0);
  for (int g = 0; g < w.n_group; g++) inv_sum = inv_sum + T(1) / weight_nc<T>(w, g, c, r);
  return T(1) / inv_sum;
}

// aero_weight_array_check_monotonicity, aero_weight_array.F90:304-332
PMC_HD void weight_monotonicity(const Weights& w, bool* inc, bool* dec) {
  *inc = true;
  *dec = true;
  for (int c = 0; c < w.n_class; c++)
    for (int g = 0; g < w.n_group; g++) {
      int k = g + kMaxGroup * c;
      if (w.type[k] == kWeightPower) {
        if (w.expo[k] < 0.0) *inc = false;
        if (w.expo[k] > 0.0) *dec = false;
      }
      if (w.type[k] == kWeightMfa) *inc = false;
    }
}

PMC_HD bool weights_flat(const Weights& w) {
  for (int c = 0; c < w.n_class; c++)
    for (int g = 0; g < w.n_group; g++)
      if (w.type[g + kMaxGroup * c] != kWeightNone) return false;
  return true;
}

// Air properties of kernel_brown_helper that depend only on the
// environment, coag_kernel_brown.F90:143-151.
// The particle shape (fractal_t) travels with the environment because every
// kernel's per-particle terms need it; fp is util.F90's air mean free path
// for the fractal mobility radius.
struct BrownEnv {
  double temp, viscosd, gasfreepath;
  Fractal frac;
  double fp;
};

PMC_HD BrownEnv brown_env(double temp, double pressure, const Fractal& frac) {
  BrownEnv e;
  double rhoair = (pressure * kAirMolecWeight) / (kUnivGas * temp);
  e.viscosd = 1.8325e-05 * (416.16 / (temp + 120.0)) * pow(temp / 296.16, 1.5);
  double viscosk = e.viscosd / rhoair;
  double gasspeed = sqrt((8.0 * kBoltzmann * temp * kAvogadro) / (kPi * kAirMolecWeight));
  e.gasfreepath = 2.0 * viscosk / gasspeed;
  e.temp = temp;
  e.frac = frac;
  e.fp = air_mean_free_path(temp, pressure);
  return e;
}

// The per-particle half of kernel_brown_helper, coag_kernel_brown.F90:163-189:
// geometric radius and, for the diffusion terms, the mobility radius.
// *ok is cleared if the fractal mobility radius does not converge.
struct BrownPart {
  double rad, diffus, speedsq, deltasq;
};

PMC_HD BrownPart brown_part(const BrownEnv& e, double vol, double den, bool* ok) {
  BrownPart p;
  double temp = e.temp;
  p.rad = vol2rad(e.frac, vol);
  double rme = mobility_rad(e.frac, vol, e.fp, ok);
  double knud = e.gasfreepath / rme;
  double cunning = 1.0 + knud * (1.249 + 0.42 * exp(-0.87 / knud));
  p.diffus = (kBoltzmann * temp * cunning) / (6.0 * kPi * rme * e.viscosd);
  p.speedsq = 8.0 * kBoltzmann * temp / (kPi * den * vol);
  double freepath = 8.0 * p.diffus / (kPi * sqrt(p.speedsq));
  double t = 2.0 * rme + freepath;
  double tmp1 = t * t * t;
  double tmp2 = pow(4.0 * rme * rme + freepath * freepath, 1.5);
  double d = (tmp1 - tmp2) / (6.0 * rme * freepath) - 2.0 * rme;
  p.deltasq = d * d;
  return p;
}

// The pair half of kernel_brown_helper, coag_kernel_brown.F90:191-195.
template <class T>
PMC_HD T brown_pair(T rad_i, T diffus_i, T speedsq_i, T deltasq_i, T rad_j, T diffus_j,
                    T speedsq_j, T deltasq_j) {
  T rad_sum = rad_i + rad_j;
  T diffus_sum = diffus_i + diffus_j;
  T tmp1 = rad_sum / (rad_sum + sqrt(deltasq_i + deltasq_j));
  T tmp2 = T(4) * diffus_sum / (rad_sum * sqrt(speedsq_i + speedsq_j));
  return T(4.0 * kPi) * rad_sum * diffus_sum / (tmp1 + tmp2);
}

// Full FP64 form in the reference's order, for k-bound tables and checks.
PMC_HD double brown_kernel(const BrownEnv& e, double vi, double di, double vj, double dj, bool* ok) {
  BrownPart a = brown_part(e, vi, di, ok);
  BrownPart b = brown_part(e, vj, dj, ok);
  double rad_sum = a.rad + b.rad;
  double diffus_sum = a.diffus + b.diffus;
  double tmp1 = rad_sum / (rad_sum + sqrt(a.deltasq + b.deltasq));
  double tmp2 = 4.0 * diffus_sum / (rad_sum * sqrt(a.speedsq + b.speedsq));
  return 4.0 * kPi * rad_sum * diffus_sum / (tmp1 + tmp2);
}

// fall_g, coag_kernel_sedi.F90:110-172 (terminal velocity, m/s; r in m)
PMC_HD double fall_g(double r) {
  const double b[7] = {-0.318657e1,  0.992696,     -0.153193e-2, -0.987059e-3,
                       -0.578878e-3, 0.855176e-4, -0.327815e-5};
  const double c[6] = {-0.500015e1, 0.523778e1, -0.204914e1, 0.475294, -0.542819e-1, 0.238449e-2};
  double eta = 1.818e-4, xlamb = 6.62e-6, rhow = 1.0, rhoa = 1.225e-3;
  double grav = 980.665, cunh = 1.257 * xlamb, t0 = 273.15;
  double sigma = 76.1 - 0.155 * (293.15 - t0);
  double stok = 2.0 * grav * (rhow - rhoa) / (9.0 * eta);
  double stb = 32.0 * rhoa * (rhow - rhoa) * grav / (3.0 * eta * eta);
  double eta4 = (eta * eta) * (eta * eta);
  double phy = sigma * sigma * sigma * rhoa * rhoa / (eta4 * grav * (rhow - rhoa));
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

// Hall (1980) collision efficiencies as tabulated in Bott's coad1d and in
// coag_kernel_sedi.F90:194-245: collector radii (um), radius ratios, and the
// efficiency for ratio column q, collector row k.
struct HallTable {
  double r0[15];
  double rat[21];
  double ec[21][15];
};

#define PMC_HALL_INIT { \
    {6.0, 8.0, 10.0, 15.0, 20.0, 25.0, 30.0, 40.0, 50.0, 60.0, 70.0, 100.0, 150.0, 200.0, 300.0}, \
    {0.0, 0.05, 0.1, 0.15, 0.2, 0.25, 0.3, 0.35, 0.4, 0.45, 0.5, \
     0.55, 0.6, 0.65, 0.7, 0.75, 0.8, 0.85, 0.9, 0.95, 1.0}, \
    {{0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, 0.001, \
      0.001, 0.001}, \
     {0.003, 0.003, 0.003, 0.004, 0.005, 0.005, 0.005, 0.010, 0.100, 0.050, 0.200, 0.500, 0.770, \
      0.870, 0.970}, \
     {0.007, 0.007, 0.007, 0.008, 0.009, 0.010, 0.010, 0.070, 0.400, 0.430, 0.580, 0.790, 0.930, \
      0.960, 1.000}, \
     {0.009, 0.009, 0.009, 0.012, 0.015, 0.010, 0.020, 0.280, 0.600, 0.640, 0.750, 0.910, 0.970, \
      0.980, 1.000}, \
     {0.014, 0.014, 0.014, 0.015, 0.016, 0.030, 0.060, 0.500, 0.700, 0.770, 0.840, 0.950, 0.970, \
      1.000, 1.000}, \
     {0.017, 0.017, 0.017, 0.020, 0.022, 0.060, 0.100, 0.620, 0.780, 0.840, 0.880, 0.950, 1.000, \
      1.000, 1.000}, \
     {0.030, 0.030, 0.024, 0.022, 0.032, 0.062, 0.200, 0.680, 0.830, 0.870, 0.900, 0.950, 1.000, \
      1.000, 1.000}, \
     {0.025, 0.025, 0.025, 0.036, 0.043, 0.130, 0.270, 0.740, 0.860, 0.890, 0.920, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.027, 0.027, 0.027, 0.040, 0.052, 0.200, 0.400, 0.780, 0.880, 0.900, 0.940, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.030, 0.030, 0.030, 0.047, 0.064, 0.250, 0.500, 0.800, 0.900, 0.910, 0.950, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.040, 0.040, 0.033, 0.037, 0.068, 0.240, 0.550, 0.800, 0.900, 0.910, 0.950, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.035, 0.035, 0.035, 0.055, 0.079, 0.290, 0.580, 0.800, 0.900, 0.910, 0.950, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.037, 0.037, 0.037, 0.062, 0.082, 0.290, 0.590, 0.780, 0.900, 0.910, 0.950, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.037, 0.037, 0.037, 0.060, 0.080, 0.290, 0.580, 0.770, 0.890, 0.910, 0.950, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.037, 0.037, 0.037, 0.041, 0.075, 0.250, 0.540, 0.760, 0.880, 0.920, 0.950, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.037, 0.037, 0.037, 0.052, 0.067, 0.250, 0.510, 0.770, 0.880, 0.930, 0.970, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.037, 0.037, 0.037, 0.047, 0.057, 0.250, 0.490, 0.770, 0.890, 0.950, 1.000, 1.000, 1.000, \
      1.000, 1.000}, \
     {0.036, 0.036, 0.036, 0.042, 0.048, 0.230, 0.470, 0.780, 0.920, 1.000, 1.020, 1.020, 1.020, \
      1.020, 1.020}, \
     {0.040, 0.040, 0.035, 0.033, 0.040, 0.112, 0.450, 0.790, 1.010, 1.030, 1.040, 1.040, 1.040, \
      1.040, 1.040}, \
     {0.033, 0.033, 0.033, 0.033, 0.033, 0.119, 0.470, 0.950, 1.300, 1.700, 2.300, 2.300, 2.300, \
      2.300, 2.300}, \
     {0.027, 0.027, 0.027, 0.027, 0.027, 0.125, 0.520, 1.400, 2.300, 3.000, 4.000, 4.000, 4.000, \
      4.000, 4.000}}}

#ifdef __CUDACC__
__device__ __constant__ HallTable kHallDev = PMC_HALL_INIT;
#endif
static const HallTable kHallHost = PMC_HALL_INIT;

PMC_HD const HallTable& hall() {
#if defined(__CUDA_ARCH__)
  return kHallDev;
#else
  return kHallHost;
#endif
}

// effic, coag_kernel_sedi.F90:180-285.  Returns a negative value where the
// reference stops (pmc_stop(99)) or would index outside its table.
template <class T>
PMC_HD T effic(T r1, T r2) {
  const HallTable& H = hall();
  T rs = r1 * T(1e6) < r2 * T(1e6) ? r1 * T(1e6) : r2 * T(1e6);
  T rb = r1 * T(1e6) > r2 * T(1e6) ? r1 * T(1e6) : r2 * T(1e6);
  T rq = rs / rb;
  int ir = 1;
  for (int k = 1; k <= 15; k++)
    if (rb > (T)H.r0[k - 1]) ir = k + 1;
  int iq = 1;
  for (int k = 1; k <= 21; k++)
    if (rq > (T)H.rat[k - 1]) iq = k + 1;
  if (iq < 2 || iq > 21) return T(-1);
  auto E = [&](int i, int j) { return (T)H.ec[j - 1][i - 1]; };
  T ec;
  if (ir < 16) {
    if (ir >= 2) {
      T p = (rb - (T)H.r0[ir - 2]) / ((T)H.r0[ir - 1] - (T)H.r0[ir - 2]);
      T q = (rq - (T)H.rat[iq - 2]) / ((T)H.rat[iq - 1] - (T)H.rat[iq - 2]);
      ec = (T(1) - p) * (T(1) - q) * E(ir - 1, iq - 1) + p * (T(1) - q) * E(ir, iq - 1) +
           q * (T(1) - p) * E(ir - 1, iq) + p * q * E(ir, iq);
    } else {
      T q = (rq - (T)H.rat[iq - 2]) / ((T)H.rat[iq - 1] - (T)H.rat[iq - 2]);
      ec = (T(1) - q) * E(1, iq - 1) + q * E(1, iq);
    }
  } else {
    T q = (rq - (T)H.rat[iq - 2]) / ((T)H.rat[iq - 1] - (T)H.rat[iq - 2]);
    T ek = (T(1) - q) * E(15, iq - 1) + q * E(15, iq);
    ec = ek < T(1) ? ek : T(1);
  }
  if (ec < T(1e-20)) return T(-1);
  return ec;
}

// kernel_sedi_helper pair formula, coag_kernel_sedi.F90:96-103, with the
// terminal velocities precomputed per particle.
template <class T>
PMC_HD T sedi_pair(T r1, T w1, T r2, T w2) {
  T ec = effic<T>(r1, r2);
  if (ec < T(0)) return T(-1);
  T rs = r1 + r2;
  return ec * T(kPi) * (rs * rs) * fabs(w1 - w2);
}

// kernel_sedi_helper, coag_kernel_sedi.F90:96-103: the collision
// efficiency from the geometric radii, the fall speeds from the mobility radii
PMC_HD double sedi_kernel(const BrownEnv& e, double v1, double v2, bool* ok) {
  double r1 = vol2rad(e.frac, v1), r2 = vol2rad(e.frac, v2);
  return sedi_pair<double>(r1, fall_g(mobility_rad(e.frac, v1, e.fp, ok)), r2,
                           fall_g(mobility_rad(e.frac, v2, e.fp, ok)));
}

// kernel_brown_free_helper (coag_kernel_brown_free.F90:118-147): free
// molecular regime, d1/d2 particle densities
PMC_HD double brown_free_kernel(const BrownEnv& e, double v1, double d1, double v2, double d2) {
  const Fractal& F = e.frac;
  double rho = (v1 / (v1 + v2)) * d1 + (v2 / (v1 + v2)) * d2;
  double ni = num_of_monomers(F, v1), nj = num_of_monomers(F, v2);
  double nif = pow(ni, 1.0 / F.frac_dim), njf = pow(nj, 1.0 / F.frac_dim);
  double s = nif + njf;
  return sqrt(6.0 * kBoltzmann * e.temp * F.prime_radius / rho * (1.0 / ni + 1.0 / nj)) * (s * s);
}

// kernel_brown_cont_helper (coag_kernel_brown_cont.F90:115-144): continuum
// regime
PMC_HD double brown_cont_kernel(const BrownEnv& e, double v1, double v2) {
  const Fractal& F = e.frac;
  double nif = pow(num_of_monomers(F, v1), 1.0 / F.frac_dim);
  double njf = pow(num_of_monomers(F, v2), 1.0 / F.frac_dim);
  return 2.0 * kBoltzmann * e.temp / 3.0 / kAirDynVisc * (1.0 / nif + 1.0 / njf) * (nif + njf);
}

// kernel_minmax, coag_kernel.F90:130-169 (Brownian: 3x3 density samples,
// coag_kernel_brown.F90:58-101).  Returns false for a sedimentation error.
PMC_HD bool kernel_minmax(int kt, double v1, double v2, const BrownEnv& be, double coeff,
                          double dmin, double dmax, double* kmin, double* kmax) {
  switch (kt) {
    case kKernelSedi: {
      bool ok = true;
      double k = sedi_kernel(be, v1, v2, &ok);
      *kmin = *kmax = k;
      return k >= 0.0 && ok;
    }
    case kKernelAdditive: *kmin = *kmax = coeff * (v1 + v2); return true;
    case kKernelConstant: *kmin = *kmax = kBeta0; return true;
    case kKernelZero: *kmin = *kmax = 0.0; return true;
    case kKernelBrown:
    case kKernelBrownFree:
    case kKernelBrownCont: {
      // kernel_brown*_minmax: 3x3 density samples
      bool first = true, ok = true;
      for (int i = 1; i <= 3; i++)
        for (int j = 1; j <= 3; j++) {
          double d1 = interp_linear_disc(dmin, dmax, 3, i);
          double d2 = interp_linear_disc(dmin, dmax, 3, j);
          double k = kt == kKernelBrown ? brown_kernel(be, v1, d1, v2, d2, &ok)
                     : kt == kKernelBrownFree ? brown_free_kernel(be, v1, d1, v2, d2)
                                              : brown_cont_kernel(be, v1, v2);
          if (first) {
            first = false;
            *kmin = *kmax = k;
          } else {
            if (k < *kmin) *kmin = k;
            if (k > *kmax) *kmax = k;
          }
        }
      return ok;
    }
  }
  return false;
}

// est_k_minmax_for_bin_unweighted, coag_kernel.F90:286-341 (edges 0-based:
// bin b spans edges[b]..edges[b+1])
PMC_HD bool kminmax_for_bin(int kt, const double* edges, int b1, int b2, const BrownEnv& be,
                            double coeff, double dmin, double dmax, double* kmin,
                            double* kmax) {
  double v1lo = rad2vol(be.frac, edges[b1]), v1hi = rad2vol(be.frac, edges[b1 + 1]);
  double v2lo = rad2vol(be.frac, edges[b2]), v2hi = rad2vol(be.frac, edges[b2 + 1]);
  bool ok = true;
  for (int i = 1; i <= 3; i++)
    for (int j = 1; j <= 3; j++) {
      double v1 = interp_linear_disc(v1lo, v1hi, 3, i);
      double v2 = interp_linear_disc(v2lo, v2hi, 3, j);
      double a, b;
      ok = kernel_minmax(kt, v1, v2, be, coeff, dmin, dmax, &a, &b) && ok;
      if (i == 1 && j == 1) {
        *kmin = a;
        *kmax = b;
      } else {
        if (a < *kmin) *kmin = a;
        if (b > *kmax) *kmax = b;
      }
    }
  *kmax = *kmax * 2.0;
  return ok;
}

// coag_num_conc_factor, coag_kernel.F90:346-377 (classes 0-based)
PMC_HD double num_conc_factor(const Weights& w, const Fractal& F, double ri, double rj, int ci, int cj, int cij) {
  double rij = vol2rad(F, rad2vol(F, ri) + rad2vol(F, rj));
  double nci = num_conc_at_radius<double>(w, ci, ri);
  double ncj = num_conc_at_radius<double>(w, cj, rj);
  double ncij = num_conc_at_radius<double>(w, cij, rij);
  double mn = nci;
  if (ncj < mn) mn = ncj;
  if (ncij < mn) mn = ncij;
  return nci * ncj / mn;
}

// coag_dest_class, coag_kernel.F90:382-416, including the reference's use of
// centers(i_bin) for both radii (lines 402-403).  Bins/classes 0-based.
PMC_HD int coag_dest_class(const Weights& w, const Fractal& F, const double* centers, int b1, int b2, int c1,
                           int c2) {
  double ri = centers[b1];
  double rj = centers[b1];
  double rij = vol2rad(F, rad2vol(F, ri) + rad2vol(F, rj));
  double nci = num_conc_at_radius<double>(w, c1, rij);
  double ncj = num_conc_at_radius<double>(w, c2, rij);
  (void)b2;
  return nci < ncj ? c1 : c2;
}

// max_coag_num_conc_factor, coag_kernel.F90:422-465 (5x5 radius samples)
PMC_HD double max_num_conc_factor(const Weights& w, const Fractal& F, const double* edges, int b1, int b2, int c1,
                                  int c2, int cc) {
  double i0 = edges[b1], i1 = edges[b1 + 1], j0 = edges[b2], j1 = edges[b2 + 1];
  double fmax = 0.0;
  for (int a = 1; a <= 5; a++)
    for (int b = 1; b <= 5; b++) {
      double ri = interp_linear_disc(i0, i1, 5, a);
      double rj = interp_linear_disc(j0, j1, 5, b);
      double f = num_conc_factor(w, F, ri, rj, c1, c2, cc);
      if (f > fmax) fmax = f;
    }
  return fmax;
}

// bin_grid_find for a log grid, bin_grid.F90:143-167 -> util.F90:532-579.
// Returns 1..n_bin inside the grid, 0 below, n_bin+1 above (1-based like
// the reference).
PMC_HD int bin_find(int n_bin, double log_lo, double log_hi, double r) {
  if (n_bin <= 0) return -1;
  double x = log(r);
  int n = n_bin + 1;
  if (x == log_hi) return n - 1;
  double f = floor((x - log_lo) / (log_hi - log_lo) * (double)(n - 1));
  int i;
  if (!(f > -1e9)) i = 0;          // -inf or NaN
  else if (f > 1e9) i = n;
  else i = (int)f + 1;
  if (i > n) i = n;
  if (i < 0) i = 0;
  return i;
}

// student_t_95_coeff, stats.F90:510-536
PMC_HD double student_t_95(int n_sample) {
  const double limit = 1.959963984540054;
  const double tq[15] = {12.7062047364, 4.30265272991, 3.18244630528, 2.7764451052,
                         2.57058183661, 2.44691184879, 2.36462425101, 2.30600413503,
                         2.26215716274, 2.22813885196, 2.20098516008, 2.17881282966,
                         2.16036865646, 2.14478668792, 2.13144954556};
  int dof = n_sample - 1;
  if (dof <= 15) return tq[dof - 1];
  if (dof <= 20) return (2.11990529922 - limit) * 16.0 / (double)dof + limit;
  return (2.07961384473 - limit) * 21.0 / (double)dof + limit;
}

// ------------------------------------------------------------------------
// Counter-based Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11).  Every
// random decision of the parallel path is a pure function of
// (population seed, step, round, stream, index), so results do not depend
// on launch shape or thread scheduling.
struct U4 {
  uint32_t x, y, z, w;
};

PMC_HD U4 philox4x32_10(U4 ctr, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)M0 * ctr.x;
    uint64_t p1 = (uint64_t)M1 * ctr.z;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    U4 n;
    n.x = hi1 ^ ctr.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ ctr.w ^ k1;
    n.w = lo0;
    ctr = n;
    k0 += W0;
    k1 += W1;
  }
  return ctr;
}

// uniform in (0, 1) with 53 random bits
PMC_HD double u53(uint32_t a, uint32_t b) {
  uint64_t x = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
  return ((double)x + 0.5) * 0x1.0p-53;
}
// uniform in (0, 1) with 32 random bits
PMC_HD double u32d(uint32_t a) { return ((double)a + 0.5) * 0x1.0p-32; }

// A stream of uniforms for one decision site: counter (site, index).
struct Rng {
  uint32_t k0, k1;     // key: population seed
  uint32_t c0, c1, c2;  // counter words fixed for this stream
  uint32_t n;           // next index
  U4 buf;
  int have;
  PMC_HD Rng(uint64_t seed, uint32_t a, uint32_t b, uint32_t c)
      : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), c0(a), c1(b), c2(c), n(0), have(0) {}
  PMC_HD double next() {
    if (have == 0) {
      buf = philox4x32_10(U4{c0, c1, c2, n++}, k0, k1);
      have = 2;
      return u53(buf.x, buf.y);
    }
    have = 0;
    return u53(buf.z, buf.w);
  }
  // uniforms drawn so far, and the state after exactly u draws
  PMC_HD uint32_t used() const { return 2 * n - (have ? 1u : 0u); }
  PMC_HD void seek(uint32_t u) {
    n = (u + 1) / 2;
    if (u & 1u) {
      buf = philox4x32_10(U4{c0, c1, c2, n - 1}, k0, k1);
      have = 2;
    } else {
      have = 0;
    }
  }
};

// Samplers with the reference's methods (rand.F90), drawing from an Rng.
// pmc_rand_int, rand.F90:172-207 (returns 1..n)
template <class R>
PMC_HD int rand_int(R& g, int n) {
  int k = (int)(g.next() * (double)n);
  return k % n + 1;
}
// prob_round, rand.F90:214-227
template <class R>
PMC_HD int prob_round(R& g, double val) {
  double c = ceil(val);
  if (g.next() < c - val) return (int)floor(val);
  return (int)c;
}
// rand_normal (Box-Muller), rand.F90:410-487
template <class R>
PMC_HD double rand_normal(R& g, double mean, double stddev) {
  double u1 = g.next();
  double u2 = g.next();
  double r = sqrt(-2.0 * log(u1));
  double theta = 2.0 * kPi * u2;
  return stddev * (r * cos(theta)) + mean;
}
PMC_HD int f_nint(double x) { return (int)llround(x); }
// rand_poisson, rand.F90:252-305 (Knuth below mean 10, normal above).  A
// negative result means the Knuth loop passed max_iter draws.
template <class R>
PMC_HD int rand_poisson(R& g, double mean, int max_iter = 1 << 20) {
  if (!(mean >= 0.0)) return -1;
  if (mean <= 10.0) {
    double L = exp(-mean);
    int k = 0;
    double p = 1.0;
    for (;;) {
      k++;
      p = p * g.next();
      if (p < L) break;
      if (k > max_iter) return -1;
    }
    return k - 1;
  }
  double x = rand_normal(g, mean, sqrt(mean));
  if (x > 2.0e9) return -1;
  int k = f_nint(x);
  return k > 0 ? k : 0;
}
// rand_binomial, rand.F90:319-404 (normal approximation or Devroye's first
// waiting-time method)
template <class R>
PMC_HD int rand_binomial(R& g, int n, double p) {
  double np = (double)n * p;
  double nomp = (double)n * (1.0 - p);
  if (np >= 10.0 && nomp >= 10.0) {
    int k = f_nint(rand_normal(g, np, sqrt(np * (1.0 - p))));
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
    double gr = log(g.next()) / log(1.0 - q);
    if (gr > (double)(n - sum)) break;
    int gi = (int)ceil(gr);
    sum += gi;
    if (sum > n) break;
    k++;
  }
  return p <= 0.5 ? k : n - k;
}
// sample_without_replacement, rand.F90:515-542 (1-based, increasing)
template <class R>
PMC_HD void sample_wo_replacement(R& g, int size, int pop, int* sample) {
  int t = 0, m = 0;
  while (m < size) {
    double r = g.next();
    if ((double)(pop - t) * r >= (double)(size - m)) {
      t++;
    } else {
      t++;
      m++;
      sample[m - 1] = t;
    }
  }
}
// sample_cts_pdf, rand.F90:550-576 (returns 1..n); 0 if max_iter exceeded
template <class R>
PMC_HD int sample_cts_pdf(R& g, const double* pdf, int n, int max_iter = 1 << 16) {
  double pmax = pdf[0];
  for (int i = 1; i < n; i++)
    if (pdf[i] > pmax) pmax = pdf[i];
  for (int it = 0; it < max_iter; it++) {
    int k = rand_int(g, n);
    if (g.next() < pdf[k - 1] / pmax) return k;
  }
  return 0;
}
// aero_weight_array_rand_group, aero_weight_array.F90:374-393 (c 0-based,
// returns a 1-based group, 0 on failure)
template <class R>
PMC_HD int rand_group(R& g, const Weights& w, int c, double r) {
  double pdf[kMaxGroup];
  for (int i = 0; i < w.n_group; i++) pdf[i] = 1.0 / weight_nc<double>(w, i, c, r);
  return sample_cts_pdf(g, pdf, w.n_group);
}

}  // namespace pmc
