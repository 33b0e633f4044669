// pmc_sample.cuh -- the initial-condition sampler on the device:
// aero_state_add_aero_dist_sample (aero_state.F90:758-831) with the mode
// samplers of aero_mode.F90 (aero_mode_sample_radius :550-630,
// aero_mode_sample_vols :633-665) and the weight preparation it calls
// (aero_state_prepare_weight_for_add :704-752, aero_state_scale_weight
// :1859-1922).
//
// The host walks the (group, mode) batches in the reference's order, draws
// each batch's Poisson count and every whole-batch decision from one
// counter-based stream, and launches one kernel per batch that writes the
// batch's particles straight into new slots: one thread per particle, each
// with its own Philox stream keyed by (population seed, step, call, index),
// so the particles do not depend on launch shape.  Nothing crosses to the
// host but the counts.
#pragma once

#include "pmc_kernels.cuh"
#include "pmc_merge.cuh"

namespace pmc {

constexpr uint32_t kStreamSample = 8;  // initial-condition draws, keyed by the call and an index
// sub-streams of a call (bits 4-7 of the second counter word)
enum : uint32_t { kSubParticle = 0, kSubHost = 1, kSubSelect = 2, kSubDup = 3 };
constexpr int kMaxSampleLoops = 1000000;  // AERO_MODE_MAX_SAMPLE_LOOPS, aero_mode.F90:643
constexpr int kMaxNormalTries = 4096;     // truncated normal redraws before the sampler gives up

enum : int { kModeLogNormal = 1, kModeExp = 2, kModeMono = 3, kModeSampled = 4 };  // aero_mode.F90:31-37

PMC_HD uint32_t sample_ctr(uint32_t call, uint32_t sub) { return (call << 8) | (sub << 4) | kStreamSample; }

// One (group, mode) batch of aero_state_add_aero_dist_sample.  The host
// computes every per-batch constant in FP64 exactly as the reference does
// (x_mean_prime, the size factor, the weighted interval concentrations).
struct SampleBatch {
  int n;             // particles in the batch (the Poisson draw)
  int type;          // mode type
  int group, cls;    // 1-based weight group and class of the new particles
  int w_type;        // weight of (group, class)
  double w_mag, w_expo;
  double x_mean;     // x_mean_prime (log10 m), log-normal modes
  double log10_std;  // log10 of the geometric standard deviation
  double threshold;  // prob_threshold of rand_normal: the size factor
  double char_radius;
  double char_vol;   // aero_data_rad2vol(char_radius), exponential modes
  int n_sample;      // sampled modes: intervals
  const double* sample_radius;  // [n_sample + 1] (device)
  const double* wnc;            // [n_sample] weighted number concentration per interval (device)
  const double* vol_frac;       // [n_spec] (device)
  const double* vol_frac_std;   // [n_spec] (device)
  int any_std;                  // some vol_frac_std is non-zero
  int source;                   // component source (aero_mode%source)
  double create_time;
};

// rand_normal with a prob_threshold (rand.F90:410-487, Box-Muller branch):
// redraw while 1 - |erf(z0 / 2.0**.5)| < threshold.  The reference divides
// by 2.0**.5 evaluated in default (single) precision, 1.41421353816986...;
// the same constant is used here.  ok is cleared after kMaxNormalTries
// redraws.
template <class R>
__device__ double rand_normal_trunc(R& g, double mean, double stddev, double threshold, bool* ok) {
  const double kSqrt2Single = (double)1.41421356f;
  for (int t = 0; t < kMaxNormalTries; t++) {
    double u1 = g.next();
    double u2 = g.next();
    double r = sqrt(-2.0 * log(u1));
    double z0 = r * cos(2.0 * kPi * u2);
    if (1.0 - fabs(erf(z0 / kSqrt2Single)) >= threshold) return stddev * z0 + mean;
  }
  *ok = false;
  return mean;
}

// aero_mode_sample_radius (aero_mode.F90:550-630) for one particle
template <class R>
__device__ double sample_radius(R& g, const SampleBatch& B, const Fractal& F, bool* ok) {
  if (B.type == kModeLogNormal) {
    double x = rand_normal_trunc(g, B.x_mean, B.log10_std, B.threshold, ok);
    return pow(10.0, x);
  }
  if (B.type == kModeSampled) {
    int i = sample_cts_pdf(g, B.wnc, B.n_sample);  // 1-based, 0 on failure
    if (i == 0) {
      *ok = false;
      return B.sample_radius[0];
    }
    double r0 = B.sample_radius[i - 1], r1 = B.sample_radius[i];
    if (B.w_type == kWeightNone || B.w_expo == 0.0) {
      double x0 = log(r0), x1 = log(r1);
      double u = g.next();
      return exp((1.0 - u) * x0 + u * x1);
    }
    // interpolate linearly in 1 / num_conc and invert the weight
    // (aero_weight_num_conc_at_radius / _radius_at_num_conc,
    // aero_weight.F90:127-190)
    double inv0 = 1.0 / (B.w_mag * fast_pow<double>(r0, B.w_expo));
    double inv1 = 1.0 / (B.w_mag * fast_pow<double>(r1, B.w_expo));
    double u = g.next();
    double inv = (1.0 - u) * inv0 + u * inv1;
    return exp(log((1.0 / inv) / B.w_mag) / B.w_expo);
  }
  if (B.type == kModeExp) return vol2rad(F, -B.char_vol * log(g.next()));
  return B.char_radius;  // mono-disperse
}

// Every field of slot i copied to slot d with a new ID: aero_state_double
// and aero_state_dup_particle copies (aero_state.F90:488-539, :1722-1746);
// caches included, claims cleared.
__device__ __forceinline__ void copy_particle(const PopDev& P, int i, int d, long long id) {
  for (int s = 0; s < P.n_spec; s++) P.vol[vol_at(P, d, s)] = P.vol[vol_at(P, i, s)];
  P.vtot[d] = P.vtot[i];
  P.mass[d] = P.mass[i];
  P.rad[d] = P.rad[i];
  P.grp[d] = P.grp[i];
  P.cls[d] = P.cls[i];
  P.id[d] = id;
  P.nprim[d] = P.nprim[i];
  P.ncomp[d] = P.ncomp[i];
  for (int k = 0; k < P.ncomp[i]; k++) {
    P.csrc[comp_at(d, k)] = P.csrc[comp_at(i, k)];
    P.ctime[comp_at(d, k)] = P.ctime[comp_at(i, k)];
  }
  P.lct[d] = P.lct[i];
  P.gct[d] = P.gct[i];
  P.imf[d] = P.imf[i];
  P.den_ice[d] = P.den_ice[i];
  P.phi[d] = P.phi[i];
  P.hyst[d] = P.hyst[i];
  P.frozen[d] = P.frozen[i];
  P.cell[d] = P.cell[i];
  P.recd[d] = P.recd[i];
  P.recf[d] = P.recf[i];
  P.claim[d] = ~0ULL;
  P.rclaim[d] = ~0ULL;
  P.touched[d] = ~0u;
  P.alive[d] = 1;
  P.changed[d] = 1;
}

// The particles of one batch: particle j of the batch goes to slot slot0 + j
// with ID id0 + j (aero_particle_new_id in the reference's order), its
// radius from the mode, its species volumes from aero_mode_sample_vols
// (normal perturbations of the volume fractions projected back onto sum 1
// along the fractions, redrawn while any is negative, then scaled to the
// particle's volume), one component (source, create time) and one primary
// particle (aero_state.F90:811-826).  The slot's species array is the
// scratch space of the accept-reject loop.
__global__ void k_sample_batch(PopDev P, SampleBatch B, int slot0, long long id0, uint32_t call, uint32_t idx0) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < B.n; j += gridDim.x * blockDim.x) {
    int d = slot0 + j;
    if (d >= P.cap) {
      cap_fail(P.ctr, kCapSampleSlot);
      continue;
    }
    Rng g(P.seed, P.step, sample_ctr(call, kSubParticle), idx0 + (uint32_t)j);
    bool ok = true;
    double radius = sample_radius(g, B, P.benv.frac, &ok);
    double total_vol = rad2vol(P.benv.frac, radius);
    double* v = P.vol + vol_at(P, d, 0);
    bool placed = false;
    for (int loop = 0; loop < (B.any_std ? kMaxSampleLoops : 1); loop++) {
      double sum = 0.0;
      for (int s = 0; s < P.n_spec; s++) {
        double f = B.vol_frac[s], sd = B.vol_frac_std[s];
        // rand_normal(f, 0) is f whatever the draw: no draw is needed
        double x = sd > 0.0 ? rand_normal(g, f, sd) : f;
        v[s] = x;
        sum = sum + x;
      }
      double offset = 1.0 - sum;
      double vmin = 0.0;
      for (int s = 0; s < P.n_spec; s++) {
        v[s] = v[s] + offset * B.vol_frac[s];
        vmin = s == 0 ? v[s] : fmin(vmin, v[s]);
      }
      if (vmin >= 0.0) {
        placed = true;
        break;
      }
    }
    if (!placed || !ok) {
      // die_msg(549015143) in the reference: a bounded loop ran out
      set_status(P.ctr, kErrTimeout);
      for (int s = 0; s < P.n_spec; s++) v[s] = 0.0;
    }
    double vs = 0.0;
    for (int s = 0; s < P.n_spec; s++) vs = vs + v[s];
    double vt = 0.0, ms = 0.0;
    for (int s = 0; s < P.n_spec; s++) {
      v[s] = placed ? v[s] / vs * total_vol : 0.0;
      vt = vt + v[s];
    }
    for (int s = 0; s < P.n_spec; s++) ms = ms + v[s] * P.density[s];
    P.vtot[d] = vt;
    P.mass[d] = ms;
    P.grp[d] = B.group;
    P.cls[d] = B.cls;
    P.id[d] = id0 + j;
    P.nprim[d] = 1;
    P.ncomp[d] = 1;
    P.csrc[comp_at(d, 0)] = B.source;
    P.ctime[comp_at(d, 0)] = B.create_time;
    P.lct[d] = B.create_time;  // aero_particle_set_create_time, aero_particle.F90:169-180
    P.gct[d] = B.create_time;
    P.imf[d] = 0.0;
    P.den_ice[d] = __longlong_as_double(0x7ff8000000000000LL);
    P.phi[d] = __longlong_as_double(0x7ff8000000000000LL);
    P.hyst[d] = 0;
    P.frozen[d] = 0;
    P.cell[d] = -1;  // placed by the next sort
    P.claim[d] = ~0ULL;
    P.rclaim[d] = ~0ULL;
    P.touched[d] = ~0u;
    P.alive[d] = 1;
    P.changed[d] = 1;
  }
}

// ---------------------------------------------------------------------------
// aero_state_scale_weight, halving branch (aero_state.F90:1890-1909): remove
// n_remove members of (g, c) chosen uniformly without replacement.  Every
// member gets a 64-bit key from its own stream; the members with the
// n_remove smallest keys form a uniform random subset.  The threshold key is
// found by a radix select over four 16-bit digits: per digit, a histogram of
// the candidates that share the digits chosen so far, then one block finds
// the digit at which the running count reaches the number still to remove.
// Members whose key equals the final threshold (64-bit ties, probability
// about n^2 / 2^65) are removed in arrival order up to the count.
struct SelectState {
  unsigned long long prefix, mask;
  long long need;  // members still to remove among the candidates
  long long ties;  // tickets handed out to members at the threshold
  int hist[1 << 16];
};

__device__ __forceinline__ unsigned long long select_key(const PopDev& P, uint32_t call, int i) {
  U4 r = philox4x32_10(U4{P.step, sample_ctr(call, kSubSelect), (uint32_t)i, 0u}, (uint32_t)P.seed,
                       (uint32_t)(P.seed >> 32));
  return ((unsigned long long)r.x << 32) | r.y;
}

__global__ void k_select_hist(PopDev P, int g, int c, uint32_t call, SelectState* S, int shift) {
  int n = P.ctr->n_slots;
  unsigned long long prefix = S->prefix, mask = S->mask;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!(P.alive[i] && P.grp[i] == g && P.cls[i] == c)) continue;
    unsigned long long k = select_key(P, call, i);
    if ((k & mask) != prefix) continue;
    atomicAdd(&S->hist[(k >> shift) & 0xffffu], 1);
  }
}

// one block of 1024 threads: thread t owns bins [64 t, 64 t + 64)
__global__ void __launch_bounds__(1024) k_select_pick(SelectState* S, int shift) {
  __shared__ long long part[1024];
  __shared__ int found;
  int t = threadIdx.x;
  long long own = 0;
  for (int b = 0; b < 64; b++) own += S->hist[t * 64 + b];
  part[t] = own;
  if (t == 0) found = -1;
  __syncthreads();
  // inclusive scan of the per-thread totals (Hillis-Steele)
  for (int o = 1; o < 1024; o <<= 1) {
    long long v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  long long need = S->need;
  long long before = t > 0 ? part[t - 1] : 0;
  if (before < need && need <= part[t]) found = t;
  __syncthreads();
  if (t == found) {
    long long run = before;
    for (int b = 0; b < 64; b++) {
      long long h = S->hist[t * 64 + b];
      if (run + h >= need) {
        unsigned long long d = (unsigned long long)(t * 64 + b);
        S->prefix |= d << shift;
        S->mask |= 0xffffULL << shift;
        S->need = need - run;
        break;
      }
      run += h;
    }
  }
  __syncthreads();
  for (int b = 0; b < 64; b++) S->hist[t * 64 + b] = 0;
}

__global__ void k_select_remove(PopDev P, int g, int c, uint32_t call, SelectState* S) {
  int n = P.ctr->n_slots;
  unsigned long long thr = S->prefix;
  long long at_thr = S->need;
  int removed = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!(P.alive[i] && P.grp[i] == g && P.cls[i] == c)) continue;
    unsigned long long k = select_key(P, call, i);
    bool rm = k < thr;
    if (k == thr) rm = atomicAdd((unsigned long long*)&S->ties, 1ULL) < (unsigned long long)at_thr;
    if (!rm) continue;
    log_removal(P, P.id[i], kInfoHalved, 0);  // aero_state.F90:1900-1908
    kill_slot(P, i);
    removed++;
  }
  if (removed) add_ll(&P.ctr->n_live, -(long long)removed);
}

// aero_state_scale_weight, doubling branch (aero_state.F90:1910-1920): each
// member of (g, c) ends as prob_round(n_mean) particles
// (aero_state_dup_particle): n_copies[i] = that number minus one copies.
__global__ void k_dup_count(PopDev P, int n, int g, int c, double n_mean, uint32_t call, int* n_copies) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int k = 0;
    if (P.alive[i] && P.grp[i] == g && P.cls[i] == c) {
      Rng r(P.seed, P.step, sample_ctr(call, kSubDup), (uint32_t)i);
      k = prob_round(r, n_mean) - 1;
      if (k < 0) k = 0;  // n_mean >= 1 here: a member is never removed
    }
    n_copies[i] = k;
  }
}

// the copies of slot i go to slots n + off[i] ... with IDs id0 + off[i] ...
__global__ void k_dup_write(PopDev P, int n, const int* n_copies, const long long* off, long long id0) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int k = n_copies[i];
    for (int j = 0; j < k; j++) {
      long long o = off[i] + j;
      int d = n + (int)o;
      if (d >= P.cap) {
        cap_fail(P.ctr, kCapDupSlot);
        break;
      }
      copy_particle(P, i, d, id0 + o);
    }
  }
}

}  // namespace pmc
