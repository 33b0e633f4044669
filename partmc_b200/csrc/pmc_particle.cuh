// pmc_particle.cuh -- one particle's metadata and aero_particle_coagulate
// on the device (header-only; shared by the parallel and replay paths).
#pragma once

#include "pmc_physics.cuh"
#include "pmc_state.cuh"

namespace pmc {

// Metadata of one particle (the non-volume fields of aero_particle_t,
// aero_particle.F90:30-69, without optical properties).
struct PMeta {
  int grp, cls;
  long long id;
  int nprim, ncomp;
  int csrc[kMaxComponent];
  double ctime[kMaxComponent];
  double lct, gct, imf, den_ice, phi;
  int hyst, frozen;
};

__device__ __forceinline__ void load_meta(const PopDev& P, int i, PMeta& m) {
  m.grp = P.grp[i];
  m.cls = P.cls[i];
  m.id = P.id[i];
  m.nprim = P.nprim[i];
  m.ncomp = P.ncomp[i];
  for (int k = 0; k < m.ncomp; k++) {
    m.csrc[k] = P.csrc[(size_t)k * P.cap + i];
    m.ctime[k] = P.ctime[(size_t)k * P.cap + i];
  }
  m.lct = P.lct[i];
  m.gct = P.gct[i];
  m.imf = P.imf[i];
  m.den_ice = P.den_ice[i];
  m.phi = P.phi[i];
  m.hyst = P.hyst[i];
  m.frozen = P.frozen[i];
}

__device__ __forceinline__ void store_particle(const PopDev& P, int i, const double* v,
                                               const PMeta& m) {
  double vt = 0.0, ms = 0.0;
  for (int s = 0; s < P.n_spec; s++) {
    P.vol[(size_t)s * P.cap + i] = v[s];
    vt = vt + v[s];
  }
  for (int s = 0; s < P.n_spec; s++) ms = ms + v[s] * P.density[s];
  P.vtot[i] = vt;
  P.mass[i] = ms;
  P.grp[i] = m.grp;
  P.cls[i] = m.cls;
  P.id[i] = m.id;
  P.nprim[i] = m.nprim;
  P.ncomp[i] = m.ncomp;
  for (int k = 0; k < m.ncomp; k++) {
    P.csrc[(size_t)k * P.cap + i] = m.csrc[k];
    P.ctime[(size_t)k * P.cap + i] = m.ctime[k];
  }
  P.lct[i] = m.lct;
  P.gct[i] = m.gct;
  P.imf[i] = m.imf;
  P.den_ice[i] = m.den_ice;
  P.phi[i] = m.phi;
  P.hyst[i] = m.hyst;
  P.frozen[i] = m.frozen;
  P.alive[i] = 1;
}

__device__ __forceinline__ void zero_meta(PMeta& m) {
  m.grp = m.cls = 0;
  m.id = 0;
  m.nprim = m.ncomp = 0;
  m.lct = m.gct = m.imf = 0.0;
  m.den_ice = __longlong_as_double(0x7ff8000000000000LL);
  m.phi = m.den_ice;
  m.hyst = m.frozen = 0;
}

// aero_particle_coagulate, aero_particle.F90:917-1033 (metadata part; the
// caller adds the volumes).  out may alias a: inputs are read first.
template <class R>
__device__ __forceinline__ void coag_meta(R& g, const PMeta& a, double ice_a, const PMeta& b, double ice_b,
                          PMeta& out) {
  PMeta r;
  r.grp = 0;
  r.cls = 0;
  r.hyst = (a.hyst == 1 && b.hyst == 1) ? 1 : 0;
  r.id = 0;
  int n1 = a.ncomp, n2 = b.ncomp;
  if (n1 + n2 > kMaxComponent) {
    int n1_new = prob_round(g, (double)a.nprim / (double)(a.nprim + b.nprim) * (double)kMaxComponent);
    if (n1_new > n1) n1_new = n1;  // cannot sample more than exist
    int n2_new = kMaxComponent - n1_new;
    if (n2_new > n2) n2_new = n2;
    int sample[kMaxComponent];
    sample_wo_replacement(g, n1_new, n1, sample);
    for (int i = 0; i < n1_new; i++) {
      r.csrc[i] = a.csrc[sample[i] - 1];
      r.ctime[i] = a.ctime[sample[i] - 1];
    }
    sample_wo_replacement(g, n2_new, n2, sample);
    for (int i = 0; i < n2_new; i++) {
      r.csrc[n1_new + i] = b.csrc[sample[i] - 1];
      r.ctime[n1_new + i] = b.ctime[sample[i] - 1];
    }
    r.ncomp = n1_new + n2_new;
  } else {
    for (int i = 0; i < n1; i++) {
      r.csrc[i] = a.csrc[i];
      r.ctime[i] = a.ctime[i];
    }
    for (int i = 0; i < n2; i++) {
      r.csrc[n1 + i] = b.csrc[i];
      r.ctime[n1 + i] = b.ctime[i];
    }
    r.ncomp = n1 + n2;
  }
  r.lct = a.lct < b.lct ? a.lct : b.lct;
  r.gct = a.gct > b.gct ? a.gct : b.gct;
  r.frozen = (a.frozen || b.frozen) ? 1 : 0;
  r.imf = a.imf > b.imf ? a.imf : b.imf;
  if (r.frozen) {
    if (a.frozen && b.frozen) {
      double i1 = ice_a * kWaterDensity / a.den_ice;
      double i2 = ice_b * kWaterDensity / b.den_ice;
      r.den_ice = (a.den_ice * i1 + b.den_ice * i2) / (i1 + i2);
    } else if (a.frozen) {
      r.den_ice = a.den_ice;
    } else {
      r.den_ice = b.den_ice;
    }
    r.phi = 1.0;
  } else {
    r.den_ice = __longlong_as_double(0x7ff8000000000000LL);
    r.phi = a.phi;
  }
  r.nprim = a.nprim + b.nprim;
  out = r;
}

}  // namespace pmc
