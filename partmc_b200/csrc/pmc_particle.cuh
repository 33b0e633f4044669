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
    m.csrc[k] = P.csrc[comp_at(i, k)];
    m.ctime[k] = P.ctime[comp_at(i, k)];
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
    P.vol[vol_at(P, i, s)] = v[s];
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
    P.csrc[comp_at(i, k)] = m.csrc[k];
    P.ctime[comp_at(i, k)] = m.ctime[k];
  }
  P.lct[i] = m.lct;
  P.gct[i] = m.gct;
  P.imf[i] = m.imf;
  P.den_ice[i] = m.den_ice;
  P.phi[i] = m.phi;
  P.hyst[i] = m.hyst;
  P.frozen[i] = m.frozen;
  P.alive[i] = 1;
  P.changed[i] = 1;
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

// The scalar fields of a particle (PMeta without the component lists).
struct PScal {
  int grp, cls;
  long long id;
  int nprim, ncomp;
  double lct, gct, imf, den_ice, phi;
  int hyst, frozen;
};

__device__ __forceinline__ void load_scal(const PopDev& P, int i, PScal& m) {
  m.grp = P.grp[i];
  m.cls = P.cls[i];
  m.id = P.id[i];
  m.nprim = P.nprim[i];
  m.ncomp = P.ncomp[i];
  m.lct = P.lct[i];
  m.gct = P.gct[i];
  m.imf = P.imf[i];
  m.den_ice = P.den_ice[i];
  m.phi = P.phi[i];
  m.hyst = P.hyst[i];
  m.frozen = P.frozen[i];
}

// The non-component fields of aero_particle_coagulate (aero_particle.F90:
// 917-1033): the caller sets id, weight group and class.  r may alias a.
template <class M>
__device__ __forceinline__ void coag_scalars(const M& a, double ice_a, const M& b, double ice_b, M& r) {
  int hyst = (a.hyst == 1 && b.hyst == 1) ? 1 : 0;
  double lct = a.lct < b.lct ? a.lct : b.lct;
  double gct = a.gct > b.gct ? a.gct : b.gct;
  int frozen = (a.frozen || b.frozen) ? 1 : 0;
  double imf = a.imf > b.imf ? a.imf : b.imf;
  double den_ice, phi;
  if (frozen) {
    if (a.frozen && b.frozen) {
      double i1 = ice_a * kWaterDensity / a.den_ice;
      double i2 = ice_b * kWaterDensity / b.den_ice;
      den_ice = (a.den_ice * i1 + b.den_ice * i2) / (i1 + i2);
    } else if (a.frozen) {
      den_ice = a.den_ice;
    } else {
      den_ice = b.den_ice;
    }
    phi = 1.0;
  } else {
    den_ice = __longlong_as_double(0x7ff8000000000000LL);
    phi = a.phi;
  }
  int nprim = a.nprim + b.nprim;
  r.hyst = hyst;
  r.lct = lct;
  r.gct = gct;
  r.frozen = frozen;
  r.imf = imf;
  r.den_ice = den_ice;
  r.phi = phi;
  r.nprim = nprim;
}

// Component selection of aero_particle_coagulate: the first n1_new output
// components come from a, the next n2_new from b.  Without overflow they are
// all of a's then all of b's; with more than kMaxComponent in total,
// prob_round picks a's share (by primary-particle counts) and each share is
// sampled without replacement (aero_particle.F90:944-975).  sa/sb receive the
// 1-based source indices.
template <class R>
__device__ __forceinline__ void coag_components(R& g, int n1, int nprim1, int n2, int nprim2, int* n1_new,
                                                int* n2_new, int* sa, int* sb) {
  if (n1 + n2 > kMaxComponent) {
    int a_new = prob_round(g, (double)nprim1 / (double)(nprim1 + nprim2) * (double)kMaxComponent);
    if (a_new > n1) a_new = n1;  // cannot sample more than exist
    int b_new = kMaxComponent - a_new;
    if (b_new > n2) b_new = n2;
    sample_wo_replacement(g, a_new, n1, sa);
    sample_wo_replacement(g, b_new, n2, sb);
    *n1_new = a_new;
    *n2_new = b_new;
  } else {
    for (int i = 0; i < n1; i++) sa[i] = i + 1;
    for (int i = 0; i < n2; i++) sb[i] = i + 1;
    *n1_new = n1;
    *n2_new = n2;
  }
}

// aero_particle_coagulate, aero_particle.F90:917-1033 (metadata part; the
// caller adds the volumes).  out may alias a: inputs are read first.
template <class R>
__device__ __forceinline__ void coag_meta(R& g, const PMeta& a, double ice_a, const PMeta& b, double ice_b,
                          PMeta& out) {
  PMeta r;
  r.grp = 0;
  r.cls = 0;
  r.id = 0;
  int sa[kMaxComponent], sb[kMaxComponent], n1_new, n2_new;
  coag_components(g, a.ncomp, a.nprim, b.ncomp, b.nprim, &n1_new, &n2_new, sa, sb);
  for (int i = 0; i < n1_new; i++) {
    r.csrc[i] = a.csrc[sa[i] - 1];
    r.ctime[i] = a.ctime[sa[i] - 1];
  }
  for (int i = 0; i < n2_new; i++) {
    r.csrc[n1_new + i] = b.csrc[sb[i] - 1];
    r.ctime[n1_new + i] = b.ctime[sb[i] - 1];
  }
  r.ncomp = n1_new + n2_new;
  coag_scalars(a, ice_a, b, ice_b, r);
  out = r;
}

}  // namespace pmc
