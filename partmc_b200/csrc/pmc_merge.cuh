// pmc_merge.cuh -- applying accepted coagulation events on the device.
//
// Per-set events: coagulate_weighting + coagulate (coagulation.F90:810-985).
// Per-particle (accelerated) path: sample_source_particle +
// coag_target_with_source (coagulation.F90:333-582), one thread per target.
// Every write to a particle slot is guarded by the slot's claim word: an
// event or target operation is applied only if it holds the lowest priority
// on every slot it writes or removes; otherwise it is redone in the next
// round against the re-sorted state.
#pragma once

#include "pmc_kernels.cuh"
#include "pmc_particle.cuh"

namespace pmc {

__device__ __forceinline__ void kill_slot(const PopDev& P, int i) {
  P.alive[i] = 0;
  P.changed[i] = 1;
  P.cell[i] = -1;
}

// Decisions of coagulate_weighting (coagulation.F90:855-892).
struct MergeDecision {
  bool rm1, rm2, create, lost1, lost2;
  int new_group;  // 1-based
};

template <class R>
__device__ MergeDecision merge_decide(const PopDev& P, R& g, int s1, int s2, int c1, int c2, int cc) {
  MergeDecision d;
  double r1 = P.rad[s1], r2 = P.rad[s2];
  double rc = vol2rad(rad2vol(r1) + rad2vol(r2));
  double nc1 = num_conc_at_radius<double>(P.w, c1, r1);
  double nc2 = num_conc_at_radius<double>(P.w, c2, r2);
  double ncc = num_conc_at_radius<double>(P.w, cc, rc);
  d.new_group = rand_group(g, P.w, cc, rc);
  double mn = nc1;
  if (nc2 < mn) mn = nc2;
  if (ncc < mn) mn = ncc;
  d.rm1 = g.next() < mn / nc1;
  d.rm2 = g.next() < mn / nc2;
  d.create = g.next() < mn / ncc;
  if (d.create) {
    d.lost1 = d.lost2 = false;
    if (d.rm1 && d.rm2) {
      if (P.vtot[s1] > P.vtot[s2]) d.lost2 = true;
      else d.lost1 = true;
    }
  } else {
    d.lost1 = d.rm1;
    d.lost2 = d.rm2;
  }
  return d;
}

// A merge decision and the number of uniforms its stream had used, in one
// word: bits 0-4 rm1, rm2, create, lost1, lost2; bits 5-7 the new weight
// group; bits 8-31 the uniforms used.
__device__ __forceinline__ uint32_t pack_decision(const MergeDecision& m, uint32_t used) {
  return (m.rm1 ? 1u : 0u) | (m.rm2 ? 2u : 0u) | (m.create ? 4u : 0u) | (m.lost1 ? 8u : 0u) |
         (m.lost2 ? 16u : 0u) | ((uint32_t)(m.new_group & 7) << 5) | (used << 8);
}
__device__ __forceinline__ MergeDecision unpack_decision(uint32_t x, uint32_t* used) {
  MergeDecision m;
  m.rm1 = x & 1u;
  m.rm2 = x & 2u;
  m.create = x & 4u;
  m.lost1 = x & 8u;
  m.lost2 = x & 16u;
  m.new_group = (int)((x >> 5) & 7u);
  *used = x >> 8;
  return m;
}

// Resolve accepted per-set samples: winner test, slot/id needs.  Event e
// has sample index ev_w[e], slots ev[e] and global pair ev_gp[e] (in sample
// order, compacted from the pair tests).
__global__ void k_resolve_set(const PopDev* pops, const int* gpair_pop, const int* gpair_local,
                              const long long* work_off, const long long* prio_off,
                              const long long* n_events, const long long* ev_w, const int2* ev,
                              const int* ev_gp, int* pair_losers, int* need_slot, int* need_id,
                              uint8_t* win, uint32_t* dec, long long* n_losers) {
  long long E = *n_events;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
       e += (long long)gridDim.x * blockDim.x) {
    long long w = ev_w[e];
    int gp = ev_gp[e];
    const PopDev& P = pops[gpair_pop[gp]];
    int p = gpair_local[gp];
    long long s = w - work_off[gp];
    unsigned prio = (unsigned)(prio_off[gp] + s);
    int2 sl = ev[e];
    if (sl.x < 0 || sl.x >= P.cap || sl.y < 0 || sl.y >= P.cap) {
      bad_index(P.ctr, kBadEventSlot, sl.x < 0 || sl.x >= P.cap ? sl.x : sl.y);
      win[e] = 0;
      need_slot[e] = 0;
      need_id[e] = 0;
      continue;
    }
    unsigned long long key = claim_key(P, prio);
    bool winner = P.claim[sl.x] == key && P.claim[sl.y] == key;
    win[e] = winner ? 1 : 0;
    need_slot[e] = 0;
    need_id[e] = 0;
    if (!winner) {
      atomicAdd(&pair_losers[gp], 1);
      add_ll(n_losers, 1);
      continue;
    }
    PairDesc d = P.pair_desc[p];
    const PairState& S = P.pair[p];
    Rng g = make_rng(P, kStreamMerge, (uint32_t)p, (uint32_t)s);
    MergeDecision m = merge_decide(P, g, sl.x, sl.y, d.c1, d.c2, S.cc);
    if (m.new_group == 0) set_status(P.ctr, kErrTimeout);
    dec[e] = pack_decision(m, g.used());
    if (m.create) {
      need_slot[e] = (!m.rm1 && !m.rm2) ? 1 : 0;
      bool keep1 = m.rm1 && !m.lost1, keep2 = m.rm2 && !m.lost2;
      need_id[e] = (!keep1 && !keep2) ? 1 : 0;
    }
  }
}

// destination slot of a winning event that creates a particle (-1: none)
__device__ __forceinline__ int event_dest(const MergeDecision& m, int s1, int s2, int slot_base,
                                          long long slot_rank) {
  if (!m.create) return -1;
  if (m.rm1) return s1;
  if (m.rm2) return s2;
  return slot_base + (int)slot_rank;
}

// Apply winning per-set events (coagulate, coagulation.F90:928-985), part 1:
// the per-particle vectors.  One warp per event: lane q adds species q of the
// two sources (particle-major, so each source is a few cache lines) and lane
// k places component k; the random component selection is computed by every
// lane alike from the stream position k_resolve_set stored.  The summed
// volume and mass go to the destination's caches for part 2; the water
// volumes of the sources, which part 2 needs after the destination may have
// been overwritten, go to ice[e].
__global__ void __launch_bounds__(256) k_apply_move(const PopDev* pops, const int* gpair_pop,
                                                    const int* gpair_local, const long long* work_off,
                                                    const long long* n_events, const long long* ev_w,
                                                    const int2* ev, const int* ev_gp, const uint8_t* win,
                                                    const uint32_t* dec, const long long* slot_rank,
                                                    const int* slot_base, double2* ice) {
  constexpr unsigned kFull = 0xffffffffu;
  long long E = *n_events;
  int lane = threadIdx.x & 31;
  long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  long long n_warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long e = warp; e < E; e += n_warps) {
    if (!win[e]) continue;  // the same e for the whole warp
    uint32_t used;
    MergeDecision m = unpack_decision(dec[e], &used);
    if (!m.create) continue;
    int gp = ev_gp[e];
    int pop = gpair_pop[gp];
    const PopDev& P = pops[pop];
    int2 sl = ev[e];
    int s1 = sl.x, s2 = sl.y;
    int dest = event_dest(m, s1, s2, slot_base[pop], m.rm1 || m.rm2 ? 0 : slot_rank[e]);
    if (dest < 0 || dest >= P.cap) continue;  // reported by part 2
    // every read of the two sources comes before the first write to dest
    int na = P.ncomp[s1], nb = P.ncomp[s2];
    if (P.i_water > 0 && lane == 0)
      ice[e] = make_double2(P.vol[vol_at(P, s1, P.i_water - 1)], P.vol[vol_at(P, s2, P.i_water - 1)]);
    int ca = 0, cb = 0;
    double ta = 0.0, tb = 0.0;
    if (lane < na && lane < kMaxComponent) {
      ca = P.csrc[comp_at(s1, lane)];
      ta = P.ctime[comp_at(s1, lane)];
    }
    if (lane < nb && lane < kMaxComponent) {
      cb = P.csrc[comp_at(s2, lane)];
      tb = P.ctime[comp_at(s2, lane)];
    }
    const int ns = P.n_spec;
    double v_lo = 0.0, v_hi = 0.0;  // species lane and lane + 32
    if (lane < ns) v_lo = P.vol[vol_at(P, s1, lane)] + P.vol[vol_at(P, s2, lane)];
    if (lane + 32 < ns) v_hi = P.vol[vol_at(P, s1, lane + 32)] + P.vol[vol_at(P, s2, lane + 32)];
    int n1_new = na, n2_new = nb;
    int k_src = lane < na ? lane : lane - na;
    bool from_a = lane < na;
    if (na + nb > kMaxComponent) {
      int np1 = P.nprim[s1], np2 = P.nprim[s2];
      Rng g = make_rng(P, kStreamMerge, (uint32_t)gpair_local[gp], (uint32_t)(ev_w[e] - work_off[gp]));
      g.seek(used);
      int sa[kMaxComponent], sb[kMaxComponent];
      coag_components(g, na, np1, nb, np2, &n1_new, &n2_new, sa, sb);
      from_a = lane < n1_new;
      k_src = 0;
      if (from_a) k_src = sa[lane] - 1;
      else if (lane - n1_new < n2_new) k_src = sb[lane - n1_new] - 1;
    }
    k_src &= 31;
    int xa = __shfl_sync(kFull, ca, k_src), xb = __shfl_sync(kFull, cb, k_src);
    double ya = __shfl_sync(kFull, ta, k_src), yb = __shfl_sync(kFull, tb, k_src);
    // totals in the reference's order (species 1..n)
    double vt = 0.0, ms = 0.0;
    for (int q = 0; q < ns && q < 64; q++) {
      double v = __shfl_sync(kFull, q < 32 ? v_lo : v_hi, q & 31);
      vt = vt + v;
      ms = ms + v * P.density[q];
    }
    __syncwarp();
    if (lane < ns) P.vol[vol_at(P, dest, lane)] = v_lo;
    if (lane + 32 < ns) P.vol[vol_at(P, dest, lane + 32)] = v_hi;
    int n_out = n1_new + n2_new;
    if (lane < n_out) {
      P.csrc[comp_at(dest, lane)] = from_a ? xa : xb;
      P.ctime[comp_at(dest, lane)] = from_a ? ya : yb;
    }
    if (lane == 0) {
      P.vtot[dest] = vt;
      P.mass[dest] = ms;
      P.ncomp[dest] = n_out;
    }
  }
}

// particle fields that coag_scalars reads (component lists excluded)
__device__ __forceinline__ void load_scalars(const PopDev& P, int i, PMeta& m) {
  m.id = P.id[i];
  m.nprim = P.nprim[i];
  m.lct = P.lct[i];
  m.gct = P.gct[i];
  m.imf = P.imf[i];
  m.den_ice = P.den_ice[i];
  m.phi = P.phi[i];
  m.hyst = P.hyst[i];
  m.frozen = P.frozen[i];
}

// Part 2, one thread per event: removals, the scalar fields of the
// coagulated particle, its radius, bin and pair-test record.
__global__ void k_apply_set(const PopDev* pops, const int* gpair_pop, const int* gpair_local,
                            const long long* n_events, const int2* ev, const int* ev_gp, const uint8_t* win,
                            const uint32_t* dec, const long long* slot_rank, const long long* id_rank,
                            const int* slot_base, const long long* id_base, const double2* ice) {
  long long E = *n_events;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
       e += (long long)gridDim.x * blockDim.x) {
    if (!win[e]) continue;
    int gp = ev_gp[e];
    int pop = gpair_pop[gp];
    const PopDev& P = pops[pop];
    int p = gpair_local[gp];
    int2 sl = ev[e];
    int s1 = sl.x, s2 = sl.y;
    uint32_t used;
    MergeDecision m = unpack_decision(dec[e], &used);
    add_ll(&P.ctr->tot_coag, (long long)(1LL));
    if (!m.create) {
      if (m.rm1) kill_slot(P, s1);
      if (m.rm2) kill_slot(P, s2);
      int dlive = -(int)m.rm1 - (int)m.rm2;
      if (dlive) add_ll(&P.ctr->n_live, (long long)dlive);
      continue;
    }
    int dest = event_dest(m, s1, s2, slot_base[pop], m.rm1 || m.rm2 ? 0 : slot_rank[e]);
    if (dest >= P.cap) {
      set_status(P.ctr, kErrCapacity);
      continue;
    }
    if (dest < 0) {
      bad_index(P.ctr, kBadDest, dest);
      continue;
    }
    PMeta a, b, c;
    load_scalars(P, s1, a);
    load_scalars(P, s2, b);
    double2 wi = P.i_water > 0 ? ice[e] : make_double2(0.0, 0.0);
    coag_scalars(a, wi.x, b, wi.y, c);
    P.grp[dest] = m.new_group;
    P.cls[dest] = P.pair[p].cc + 1;
    if (m.rm1 && !m.lost1) P.id[dest] = a.id;
    else if (m.rm2 && !m.lost2) P.id[dest] = b.id;
    else P.id[dest] = id_base[pop] + id_rank[e];
    P.nprim[dest] = c.nprim;
    P.lct[dest] = c.lct;
    P.gct[dest] = c.gct;
    P.imf[dest] = c.imf;
    P.den_ice[dest] = c.den_ice;
    P.phi[dest] = c.phi;
    P.hyst[dest] = c.hyst;
    P.frozen[dest] = c.frozen;
    P.alive[dest] = 1;
    P.changed[dest] = 1;
    // the coagulated particle must lie on the grid (aero_state_add_particle
    // with allow_resort=.false., aero_sorted.F90:427-440)
    int nbin = refresh_slot(P, dest);
    if (nbin < 1 || nbin > P.grid->n_bin) set_status(P.ctr, kErrOutOfGrid);
    if (m.rm1 && dest != s1) kill_slot(P, s1);
    if (m.rm2 && dest != s2) kill_slot(P, s2);
    int dlive = 1 - (int)m.rm1 - (int)m.rm2;
    if (dlive) add_ll(&P.ctr->n_live, (long long)dlive);
  }
}

// ---------------------------------------------------------------------------
// Per-particle (accelerated) path, phase 1: run sample_source_particle and
// the target update of coag_target_with_source for one target, store the
// result, and claim the target and every removed source.
constexpr int kMaxRemove = 64;  // removals stored per target operation
constexpr int kMaxCopies = 8;   // dup copies per target operation

struct PPResult {
  int target, p;        // target slot, pair (local)
  int n_samp, n_coag;   // counted into tot_n_samp / tot_n_coag when the operation is applied
  int merged;           // n_coag > 0
  int n_copies;         // prob_round(old_nc / new_nc); 0 removes the target
  int n_rm;
  int copy_group[kMaxCopies];
  int rm[kMaxRemove];
  PMeta meta;           // new target metadata
};

template <int KT>
__device__ double pp_kernel(const PopDev& P, const RecD& qs, const RecD& qt, int cs, int ct) {
  const double* a = (const double*)&qs;
  const double* b = (const double*)&qt;
  return pair_kernel<KT, double, false>(P, a, b, cs, ct, ct, 0.0, P.coeff);
}

template <int KT>
__global__ void k_pp_ops(const PopDev* pops, const int* op_pop, const int* op_pair,
                         const int* op_slot, const int* op_k, const unsigned* op_prio,
                         const long long* n_ops, PPResult* res, double* res_vol) {
  long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    const PopDev& P = pops[op_pop[q]];
    int p = op_pair[q], t = op_slot[q];
    unsigned prio = op_prio[q];
    PPResult& R = res[q];
    R.target = t;
    R.p = p;
    R.n_samp = 0;
    R.n_coag = 0;
    R.merged = 0;
    R.n_copies = 1;
    R.n_rm = 0;
    if (!P.alive[t]) continue;
    const PairState& S = P.pair[p];
    const GridDev& G = *P.grid;
    int nb = G.n_bin;
    int cs = S.cs, ct = S.ct;
    int src_cell = S.bs + nb * cs;
    int n_src = P.cell_count[src_cell];
    int src_start = P.cell_start[src_cell];
    if (n_src == 0) continue;
    RecD qt = P.recd[t];
    double nc_target = qt.nc;
    double nc_src_min = num_conc_at_radius<double>(P.w, cs, G.edges[S.bs]);
    double prm_max = nc_target / nc_src_min;
    if (!(prm_max <= 1.0)) {
      set_status(P.ctr, kErrAssert);
      continue;
    }
    Rng g = make_rng(P, kStreamPart, (uint32_t)p, (uint32_t)op_k[q]);
    int n_remove = rand_poisson(g, prm_max * S.nspt);
    int n_extra = rand_poisson(g, (1.0 - prm_max) * S.nspt);
    if (n_remove < 0 || n_extra < 0) {
      set_status(P.ctr, kErrTimeout);
      continue;
    }
    int n_total = n_remove + n_extra;
    int ns = P.n_spec;
    double* acc = res_vol + (size_t)q * ns;  // accumulated source volumes
    double vol_sq[kMaxSpec], vol_cv[kMaxSpec];
    for (int k = 0; k < ns; k++) {
      acc[k] = 0.0;
      vol_sq[k] = 0.0;
      vol_cv[k] = 0.0;
    }
    PMeta src;
    zero_meta(src);
    int n_avg = 0, n_samp = 0;
    double pc_tot = 0.0;
    for (int i_samp = 1; i_samp <= n_total; i_samp++) {
      if (n_samp > n_remove && n_avg >= 2) {
        double cv_max = 0.0;
        bool found = false;
        for (int k = 0; k < ns; k++) {
          double mean = acc[k] / (double)n_avg;
          if (mean > 0.0) vol_cv[k] = sqrt(vol_sq[k] / (double)n_avg - mean * mean) / mean;
        }
        for (int k = 0; k < ns; k++) {
          if (isnan(vol_cv[k])) continue;
          if (!found || vol_cv[k] > cv_max) cv_max = vol_cv[k];
          found = true;
        }
        if (!found) cv_max = __longlong_as_double(0x7ff8000000000000LL);
        double conf = cv_max / sqrt((double)n_avg) * student_t_95(n_avg);
        if (conf < 0.1) break;
      }
      n_samp++;
      int ie = rand_int(g, n_src);
      int e = src_start + ie - 1;
      int si = P.list[e];
      RecD qs = P.recd[si];
      double k = pp_kernel<KT>(P, qs, qt, cs, ct);
      double pc = k * S.inv_k_max;
      pc_tot = pc_tot + pc;
      if (g.next() < pc) {
        n_avg++;
        PMeta sm;
        load_meta(P, si, sm);
        double ice_a = 0.0, ice_b = 0.0;
        if (P.i_water > 0) {
          ice_a = acc[P.i_water - 1];
          ice_b = P.vol[vol_at(P, si, P.i_water - 1)];
        }
        coag_meta(g, src, ice_a, sm, ice_b, src);
        for (int k2 = 0; k2 < ns; k2++) {
          double vi = P.vol[vol_at(P, si, k2)];
          acc[k2] = acc[k2] + vi;
          vol_sq[k2] = vol_sq[k2] + vi * vi;
        }
        if (i_samp <= n_remove) {
          double pri = nc_target / qs.nc;
          if (g.next() < pri / prm_max) {
            bool dup = false;
            for (int z = 0; z < R.n_rm; z++) dup = dup || (R.rm[z] == si);
            if (!dup) {
              if (R.n_rm < kMaxRemove) {
                R.rm[R.n_rm++] = si;
                atomicMin(&P.claim[si], claim_key(P, prio));
              } else {
                set_status(P.ctr, kErrCapacity);
              }
            }
          }
        }
      }
    }
    R.n_samp = n_samp;
    if (n_avg == 0) continue;
    double pc_mean = pc_tot / (double)n_samp;
    if (!(pc_mean <= 1.0)) add_ll(&P.ctr->kmax_warn, (long long)(1LL));
    int n_coag = rand_binomial(g, n_total, pc_mean);
    double scale = (double)n_coag / (double)n_avg;
    for (int k = 0; k < ns; k++) acc[k] = acc[k] * scale;
    src.nprim = prob_round(g, (double)src.nprim * scale);
    {
      int n_comp = src.ncomp;
      int n_new = src.nprim < kMaxComponent ? src.nprim : kMaxComponent;
      int sample[kMaxComponent];
      if (n_new < n_comp) {
        PMeta m = src;
        sample_wo_replacement(g, n_new, n_comp, sample);
        for (int i = 0; i < n_new; i++) {
          m.csrc[i] = src.csrc[sample[i] - 1];
          m.ctime[i] = src.ctime[sample[i] - 1];
        }
        m.ncomp = n_new;
        src = m;
      } else if (n_comp < kMaxComponent && n_comp > 0) {
        PMeta m = src;
        int i_comp = 1;
        while (i_comp <= n_new) {
          if (i_comp + n_comp <= n_new) {
            for (int i = 1; i <= n_comp; i++) {
              m.csrc[i_comp + i - 2] = src.csrc[i - 1];
              m.ctime[i_comp + i - 2] = src.ctime[i - 1];
            }
            i_comp += n_comp;
          } else {
            int size = n_new - i_comp + 1;
            sample_wo_replacement(g, size, n_comp, sample);
            for (int i = 1; i <= size; i++) {
              m.csrc[i_comp + i - 2] = src.csrc[sample[i - 1] - 1];
              m.ctime[i_comp + i - 2] = src.ctime[sample[i - 1] - 1];
            }
            i_comp = n_new + 1;
          }
        }
        m.ncomp = n_new;
        src = m;
      }
    }
    R.n_coag = n_coag;
    if (n_coag == 0) continue;
    // coag_target_with_source (coagulation.F90:522-582): new target
    PMeta tm;
    load_meta(P, t, tm);
    double ice_t = 0.0;
    if (P.i_water > 0) ice_t = P.vol[vol_at(P, t, P.i_water - 1)];
    double ice_s = P.i_water > 0 ? acc[P.i_water - 1] : 0.0;
    long long tid = tm.id;
    double old_nc = nc_target;
    PMeta nm;
    coag_meta(g, tm, ice_t, src, ice_s, nm);
    nm.id = tid;
    double vt = 0.0;
    for (int k = 0; k < ns; k++) {
      acc[k] = P.vol[vol_at(P, t, k)] + acc[k];  // now the new target volumes
      vt = vt + acc[k];
    }
    double rnew = vol2rad(vt);
    int cc = S.cc;
    nm.grp = rand_group(g, P.w, cc, rnew);
    nm.cls = cc + 1;
    int b = bin_find(nb, G.log_lo, G.log_hi, rnew);
    if (b < 1 || b > nb) set_status(P.ctr, kErrOutOfGrid);
    double new_nc = num_conc_at_radius<double>(P.w, cc, rnew);
    int n_copies = prob_round(g, old_nc / new_nc);
    if (n_copies > kMaxCopies) {
      set_status(P.ctr, kErrCapacity);
      n_copies = kMaxCopies;
    }
    for (int z = 1; z < n_copies; z++) R.copy_group[z] = rand_group(g, P.w, cc, rnew);
    R.merged = 1;
    R.n_copies = n_copies;
    R.meta = nm;
    atomicMin(&P.claim[t], claim_key(P, prio));
  }
}

// phase 2a: winners and allocation needs of the target operations
__global__ void k_pp_resolve(const PopDev* pops, const int* op_pop, const unsigned* op_prio,
                             const long long* n_ops, const PPResult* res, uint8_t* win,
                             int* need_slot, int* need_id, int* lost) {
  long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    const PopDev& P = pops[op_pop[q]];
    const PPResult& R = res[q];
    unsigned prio = op_prio[q];
    bool ok = true;
    if (R.merged) ok = ok && P.claim[R.target] == claim_key(P, prio);
    for (int z = 0; z < R.n_rm; z++) ok = ok && P.claim[R.rm[z]] == claim_key(P, prio);
    win[q] = ok ? 1 : 0;
    lost[q] = ok ? 0 : 1;
    int extra = (ok && R.merged && R.n_copies > 1) ? R.n_copies - 1 : 0;
    need_slot[q] = extra;
    need_id[q] = extra;
  }
}

// phase 2b: apply the winning target operations
__global__ void k_pp_apply(const PopDev* pops, const int* op_pop, const long long* n_ops,
                           const PPResult* res, const double* res_vol, const uint8_t* win,
                           const long long* slot_rank, const long long* id_rank,
                           const int* slot_base, const long long* id_base) {
  long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    if (!win[q]) continue;
    int pop = op_pop[q];
    const PopDev& P = pops[pop];
    const PPResult& R = res[q];
    // an operation that lost a claim is redone from scratch, so only applied
    // operations count their samples and coagulations
    if (R.n_samp) add_ll(&P.ctr->tot_samp, (long long)R.n_samp);
    if (R.n_coag) add_ll(&P.ctr->tot_coag, (long long)R.n_coag);
    int dlive = 0;
    for (int z = 0; z < R.n_rm; z++) {
      kill_slot(P, R.rm[z]);
      dlive--;
    }
    if (R.merged) {
      const double* v = res_vol + (size_t)q * P.n_spec;
      int t = R.target;
      if (R.n_copies == 0) {
        kill_slot(P, t);
        dlive--;
      } else {
        store_particle(P, t, v, R.meta);
        refresh_slot(P, t);
        for (int z = 1; z < R.n_copies; z++) {
          int dest = slot_base[pop] + (int)slot_rank[q] + (z - 1);
          if (dest >= P.cap) {
            set_status(P.ctr, kErrCapacity);
            break;
          }
          PMeta cm = R.meta;
          cm.grp = R.copy_group[z];
          cm.id = id_base[pop] + id_rank[q] + (z - 1);
          store_particle(P, dest, v, cm);
          refresh_slot(P, dest);
          dlive++;
        }
      }
    }
    if (dlive) add_ll(&P.ctr->n_live, (long long)(dlive));
  }
}

}  // namespace pmc
