// pmc_merge.cuh -- applying accepted coagulation events on the device.
//
// Per-set events: coagulate_weighting + coagulate (coagulation.F90:810-985).
// Per-particle (accelerated) path: sample_source_particle +
// coag_target_with_source (coagulation.F90:333-582), one thread per target.
// Every write to a particle slot is guarded by the slot's claim word: an
// event or target operation is applied only if it holds the lowest priority
// on every slot it writes or removes; otherwise it is retried (or dropped,
// k_items) in the next round.
#pragma once

#include "pmc_kernels.cuh"
#include "pmc_particle.cuh"

namespace pmc {

// Chains (see the walks below): the events of one walk that absorbs its
// partners one after another, in chunks of kChainChunk entries; entry
// kChainChunk - 1 of a chunk's y holds the index of the next chunk (-1: none)
constexpr int kChainChunk = 32;
constexpr int kChainMaxLen = 1 << 16;  // events of one chain in one round
// q of an entry: the pair, and kChainRemoves if the merge removes the partner
constexpr int kChainPairMask = (1 << 20) - 1;
constexpr int kChainRemoves = 1 << 30;

struct ChainPool {
  int* y;          // [n_chunks * kChainChunk] partner slot; the last entry of a chunk links the next chunk
  int* q;          // pair (local), with kChainRemoves if the merge removes the partner
  float* pos;      // position in the pair's test sequence
  long long* ctr;  // chunks handed out in this round (device)
  long long n_chunks;
};

struct ChainWriter {
  int head = -1, chunk = -1, fill = 0, len = 0;
  __device__ bool append(const ChainPool& C, int y, int q, float pos) {
    if (chunk < 0 || fill == kChainChunk - 1) {
      long long nc = (long long)atomicAdd((unsigned long long*)C.ctr, 1ULL);
      if (nc >= C.n_chunks) return false;
      if (chunk >= 0) C.y[(size_t)chunk * kChainChunk + kChainChunk - 1] = (int)nc;
      else head = (int)nc;
      chunk = (int)nc;
      fill = 0;
      C.y[(size_t)chunk * kChainChunk + kChainChunk - 1] = -1;
    }
    size_t i = (size_t)chunk * kChainChunk + fill;
    C.y[i] = y;
    C.q[i] = q;
    C.pos[i] = pos;
    fill++;
    len++;
    return true;
  }
};

struct ChainReader {
  int chunk, k = 0;
  __device__ explicit ChainReader(int head) : chunk(head) {}
  // index of the next entry, -1 past the end of the links
  __device__ long long next(const ChainPool& C) {
    if (chunk < 0 || (long long)chunk >= C.n_chunks) return -1;
    size_t i = (size_t)chunk * kChainChunk + k;
    if (++k == kChainChunk - 1) {
      chunk = C.y[(size_t)chunk * kChainChunk + kChainChunk - 1];
      k = 0;
    }
    return (long long)i;
  }
};

__device__ __forceinline__ void kill_slot(const PopDev& P, int i) {
  P.alive[i] = 0;
  P.changed[i] = 1;
  P.cell[i] = -1;
}

// Resolve the events of a round: winner test, slot/id needs.  Event e has
// key ev_key[e], slots ev[e], global pair ev_gp[e] and merge decision dec[e]
// (drawn when the event was formed); the events are ordered by population.
// A winning chain (ev_len[e] > 0) gets win 2 and the number of its events
// whose claims hold (ev_app[e]).
__global__ void k_resolve_set(const PopDev* pops, const int* gpair_pop, const long long* n_events,
                              const unsigned long long* ev_key, const int2* ev, const int* ev_gp, int* need_slot,
                              int* need_id, uint8_t* win, const uint32_t* dec, long long* n_losers, const int* ev_len,
                              const int* ev_head, int* ev_app, ChainPool pool) {
  long long E = *n_events;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
       e += (long long)gridDim.x * blockDim.x) {
    int gp = ev_gp[e];
    const PopDev& P = pops[gpair_pop[gp]];
    unsigned long long key = ev_key[e];
    int p = (int)key_pair(key);
    int2 sl = ev[e];
    win[e] = 0;
    need_slot[e] = 0;
    need_id[e] = 0;
    if (sl.x < 0 || sl.x >= P.cap || sl.y < 0 || sl.y >= P.cap || p >= P.n_pairs) {
      bad_index(P.ctr, kBadEventSlot, sl.x < 0 || sl.x >= P.cap ? sl.x : sl.y);
      continue;
    }
    uint32_t used;
    MergeDecision m = unpack_decision(dec[e], &used);
    unsigned long long ck = claim_key(P, key);
    bool winner = holds_slot(P, sl.x, ck, m.rm1) && holds_slot(P, sl.y, ck, m.rm2);
    if (!winner) {
      add_ll(n_losers, 1);
      continue;
    }
    int len = ev_len[e];
    if (len > 0) {
      // a chain: its events apply as far as each partner's claim holds (the
      // walking particle's is the first event's)
      ChainReader rd(ev_head[e]);
      uint32_t x = key_idx(key);
      int app = 0;
      for (int i = 0; i < len; i++) {
        long long ix = rd.next(pool);
        if (ix < 0) break;
        int y = pool.y[ix], qw = pool.q[ix];
        int q = qw & kChainPairMask;
        if (y < 0 || y >= P.cap || q < 0 || q >= P.n_pairs) break;
        if (!holds_slot(P, y, claim_key(P, make_key((uint32_t)q, 1u, x)), (qw & kChainRemoves) != 0)) break;
        app++;
      }
      ev_app[e] = app;
      win[e] = 2;
      continue;
    }
    win[e] = 1;
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
                                                    const long long* n_events, const unsigned long long* ev_key,
                                                    const int2* ev, const int* ev_gp, const uint8_t* win,
                                                    const uint32_t* dec, const long long* slot_rank,
                                                    const int* slot_base, double2* ice) {
  constexpr unsigned kFull = 0xffffffffu;
  long long E = *n_events;
  int lane = threadIdx.x & 31;
  long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  long long n_warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long e = warp; e < E; e += n_warps) {
    if (win[e] != 1) continue;  // the same e for the whole warp; chains apply in k_apply_chain
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
      Rng g = merge_rng(P, ev_key[e]);
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
// coagulated particle, its radius, bin and pair-test record.  Every slot an
// event removes or rewrites is stamped with the round's claim generation,
// and dest[e] gets the slot of the particle the event made (-1 if none).
__global__ void k_apply_set(const PopDev* pops, const int* gpair_pop, const long long* n_events,
                            const unsigned long long* ev_key, const int2* ev, const int* ev_gp,
                            const uint8_t* win, const uint32_t* dec, const long long* slot_rank,
                            const long long* id_rank, const int* slot_base, const long long* id_base,
                            const double2* ice, int* dest_out) {
  long long E = *n_events;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
       e += (long long)gridDim.x * blockDim.x) {
    dest_out[e] = -1;
    if (win[e] != 1) continue;
    int gp = ev_gp[e];
    int pop = gpair_pop[gp];
    const PopDev& P = pops[pop];
    int p = (int)key_pair(ev_key[e]);
    int2 sl = ev[e];
    int s1 = sl.x, s2 = sl.y;
    uint32_t gen = *P.gen_p;
    uint32_t used;
    MergeDecision m = unpack_decision(dec[e], &used);
    add_ll(&P.ctr->tot_coag, (long long)(1LL));
    if (m.rm1) P.touched[s1] = gen;
    if (m.rm2) P.touched[s2] = gen;
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
    P.touched[dest] = gen;
    int nbin = refresh_slot(P, dest);
    if (nbin < 1 || nbin > P.grid->n_bin) set_status(P.ctr, kErrOutOfGrid);
    else dest_out[e] = dest;
    if (m.rm1 && dest != s1) kill_slot(P, s1);
    if (m.rm2 && dest != s2) kill_slot(P, s2);
    int dlive = 1 - (int)m.rm1 - (int)m.rm2;
    if (dlive) add_ll(&P.ctr->n_live, (long long)dlive);
  }
}

// ---------------------------------------------------------------------------
// Walks.  In the sequential loop a particle that an event creates (or
// changes) at pair p0 takes part in the rest of the step: every later pair
// that contains its cell draws its samples with the particle among the
// cell's members, so it is tested against each member of the pair's other
// cell at rate k_max * del_t (the pair's samples, n1 * n2 * k_max * del_t in
// mean, fall on each of the n1 * n2 possible pairs alike; for one cell with
// itself n (n - 1) / 2 pairs and n - 1 partners).  A walk draws those tests
// as one Poisson process along the pairs that follow p0 in loop order, the
// rest of p0 itself from position pos0 (the fraction of p0's test sequence
// already done).
//
// Partners come from the cell lists of the sort at the round's start, so a
// walk meets every particle that earlier rounds of the step made.  A listed
// slot that is dead, has left the cell since, is the walking particle itself
// or was absorbed earlier in its chain is no member now, and a test that
// falls on it is dropped.  Particles that other walks of the same round
// change are met with the values they had at the round's start.  Pairs on
// the per-particle path are not walked.
//
// Chains.  A walk's accepted test whose merge decision (coagulate_weighting,
// drawn from the stream the event's apply uses) replaces the walking particle
// by the coagulated one is an absorb: the walk goes on at once with the
// coagulated particle's values (volumes summed as the apply sums them,
// radius, record, cell), as the sequential loop would test it next.  Each
// absorbed partner is claimed with its own key; the events are recorded in
// a chain (ChainPool) and applied, as far as their claims hold, by one
// thread in order (k_apply_chain).  A runaway collector that absorbs
// thousands of droplets in one step (the sedimentation kernel) takes one
// round, not one round per droplet.  The chain stops before an accepted
// test that is not an absorb; the walk resumes there in the next round.

// cell of a particle of radius r and class cls (1-based); -1 off the grid
__device__ __forceinline__ int cell_of(const PopDev& P, double r, int cls) {
  const GridDev& G = *P.grid;
  int b = bin_find(G.n_bin, G.log_lo, G.log_hi, r);
  if (b < 1 || b > G.n_bin || cls < 1 || cls > P.n_class) return -1;
  return (b - 1) + G.n_bin * (cls - 1);
}

// the walk's first accepted test, and its chain
struct WalkOut {
  bool found = false;
  int q = 0, y = 0;  // pair and partner of the first event
  float pos = 0.f;
  bool first_cell1 = true;  // the walking particle is in the pair's first cell
  int chain_len = 0;        // events in the chain (0: the first event alone)
  int chain_head = -1;
  bool done = false;        // the walk ran to the end after its last event
  uint32_t dec = 0;         // merge decision of the first event
  bool cont = false;        // the first event is an absorb: k_chain carries the walk on
  uint32_t g_used = 0;      // uniforms the walk's stream had used at the first event
};

// true if this round's claim on slot y is the chain of walker x
__device__ __forceinline__ bool claimed_by_walk(const PopDev& P, int y, int x) {
  unsigned long long w = P.claim[y];
  return (w >> 53) == (unsigned long long)(~*P.gen_p & kGenLimit) && ((w >> 32) & 1ULL) &&
         (uint32_t)w == (uint32_t)x;
}

// The rest of a chain after its first absorb (kept out of line: the chain's
// state, the coagulated particle's volumes and record, stays out of the
// walk's registers).  Continues the Poisson process of g along the pairs of
// the coagulated particle's cell from (q, pos); returns the walk's end state.
template <int KT, class T, bool FLAT>
__device__ void walk_chain(const PopDev& P, const ChainPool& pool, int x, int y1, int q, double pos,
                                        int cls, Rng& g, ChainWriter& cw, WalkOut* out, long long* n_tests_io) {
  const int nb = P.grid->n_bin;
  double vcur[kMaxSpec];
  double vt, r;
  RecD rec;
  RecF recf;
  long long n_tests = *n_tests_io, n_iter = 0;
  int y = y1;
  int C = -1, p0 = q;
  float pos0 = (float)pos;
  for (int s = 0; s < P.n_spec; s++) vcur[s] = P.vol[vol_at(P, x, s)];
  bool stop = false;
  for (;;) {
    // absorb y: the coagulated particle's volumes, radius, class, record
    double s_v = 0.0, s_m = 0.0;
    for (int s = 0; s < P.n_spec; s++) vcur[s] = vcur[s] + P.vol[vol_at(P, y, s)];
    for (int s = 0; s < P.n_spec; s++) s_v = s_v + vcur[s];
    for (int s = 0; s < P.n_spec; s++) s_m = s_m + vcur[s] * P.density[s];
    vt = s_v;
    r = vol2rad(vt);
    rec = make_rec_v(P, r, vt, s_m, cls);
    recf = to_f32(rec);
    C = cell_of(P, r, cls);
    if (C < 0 || cw.len >= kChainMaxLen) break;  // off the grid (reported by the apply) or long enough
    // the next accepted test of the coagulated particle
    bool found = false, moved = true;
    while (moved && !stop && !found) {
      moved = false;
      int lo = P.cp_off[C], end = P.cp_off[C + 1];
      const double* cum = P.cp_cum + (P.cp_off[C] + C) - lo;
      {
        int hi = end;
        while (lo < hi) {
          int mid = (lo + hi) >> 1;
          if (P.cp_list[mid] < p0) lo = mid + 1;
          else hi = mid;
        }
      }
      double at = cum[lo];
      if (lo < end && P.cp_list[lo] == p0) at += (cum[lo + 1] - cum[lo]) * (double)pos0;
      const double at_end = cum[end];
      int j = lo;
      for (;;) {
        at += -log(g.next());
        if (!(at < at_end)) {
          out->done = true;  // every later pair of the cell was walked
          stop = true;
          break;
        }
        if (++n_iter > (1LL << 26)) {
          set_status(P.ctr, kErrTimeout);
          stop = true;
          break;
        }
        {
          int a = j, b = end - 1;
          while (a < b) {
            int mid = (a + b + 1) >> 1;
            if (cum[mid] <= at) a = mid;
            else b = mid - 1;
          }
          j = a;
        }
        int qq = P.cp_list[j];
        double lam = cum[j + 1] - cum[j];
        if (!(lam > 0.0)) continue;
        double pp = (at - cum[j]) / lam;
        const PairState& S = P.pair[qq];
        PairDesc d = P.pair_desc[qq];
        int cell1 = d.b1 + nb * d.c1, cell2 = d.b2 + nb * d.c2;
        int O = cell1 == C ? cell2 : cell1;
        int n_o = P.cell_count[O];
        int o_start = P.cell_start[O];
        if (n_o < 1) continue;
        if (o_start < 0 || (long long)o_start + n_o > P.cap) {
          bad_index(P.ctr, kBadPairCells, qq);
          stop = true;
          break;
        }
        int i = (int)(g.next() * (double)n_o);
        if (i >= n_o) i = n_o - 1;
        int yy = P.list[o_start + i];
        if (yy < 0 || yy >= P.cap) {
          bad_index(P.ctr, kBadTestSlot, yy);
          continue;
        }
        if (yy == x || !P.alive[yy] || P.cell[yy] != O) continue;
        if (claimed_by_walk(P, yy, x)) continue;  // absorbed earlier in this chain
        n_tests++;
        bool first = cell1 == C;
        T k;
        if constexpr (sizeof(T) == 8) {
          const double* qw = (const double*)&rec;
          const double* qy = (const double*)&P.recd[yy];
          k = (T)pair_kernel<KT, double, FLAT>(P, first ? qw : qy, first ? qy : qw, d.c1, d.c2, S.cc, S.fflat,
                                               P.coeff);
        } else {
          const float* qw = (const float*)&recf;
          const float* qy = (const float*)&P.recf[yy];
          k = (T)pair_kernel<KT, float, FLAT>(P, first ? qw : qy, first ? qy : qw, d.c1, d.c2, S.cc,
                                              (float)S.fflat, (float)P.coeff);
        }
        T prob = k * (T)S.inv_k_max;
        if (!(prob <= T(1))) add_ll(&P.ctr->kmax_warn, 1LL);
        if (!((T)g.next() < prob)) continue;
        // the chain ends before an event that is no absorb, or when the pool
        // is full; the walk resumes there in the next round
        unsigned long long key = make_key((uint32_t)qq, 1u, (uint32_t)x);
        Rng gm = make_rng(P, kStreamChain, (uint32_t)(cw.len + 1), (uint32_t)x);
        double ry = P.rad[yy], vty = P.vtot[yy];
        MergeDecision m = first ? merge_decide_v(P, gm, r, vt, ry, vty, d.c1, d.c2, S.cc)
                                : merge_decide_v(P, gm, ry, vty, r, vt, d.c1, d.c2, S.cc);
        bool rm_x = first ? m.rm1 : m.rm2, rm_y = first ? m.rm2 : m.rm1;
        if (!(m.create && rm_x && m.new_group != 0) ||
            !cw.append(pool, yy, qq | (rm_y ? kChainRemoves : 0), (float)pp)) {
          stop = true;
          break;
        }
        claim_slot(P, yy, claim_key(P, key), rm_y);
        y = yy;
        cls = S.cc + 1;
        p0 = qq;
        pos0 = (float)pp;
        found = true;
        break;
      }
    }
    if (stop || !found) break;
  }
  *n_tests_io = n_tests;
}

template <int KT, class T, bool FLAT>
__device__ void walk(const PopDev& P, const ChainPool& pool, int x, int p0, float pos0, WalkOut* out) {
  if (x < 0 || x >= P.cap || !P.alive[x]) return;
  const int C = P.cell[x];
  if (C < 0 || C >= P.n_cells) return;
  const int nb = P.grid->n_bin;
  Rng g = make_rng(P, kStreamWalk, 0u, (uint32_t)x);
  long long n_tests = 0, n_iter = 0;
  // the pairs of cell C from (p0, pos0) on, as one stretch of expected
  // tests: cum[j] over the cell's pairs (cp_cum)
  int lo = P.cp_off[C], end = P.cp_off[C + 1];
  const double* cum = P.cp_cum + (P.cp_off[C] + C) - lo;  // cum[j], j = lo..end
  {
    int hi = end;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (P.cp_list[mid] < p0) lo = mid + 1;
      else hi = mid;
    }
  }
  double at = cum[lo];
  if (lo < end && P.cp_list[lo] == p0) at += (cum[lo + 1] - cum[lo]) * (double)pos0;
  const double at_end = cum[end];
  int j = lo;
  for (;;) {
    at += -log(g.next());
    if (!(at < at_end)) {
      out->done = true;  // no test left in the cell's later pairs
      break;
    }
    if (++n_iter > (1LL << 26)) {  // far past any mean the step can ask for
      set_status(P.ctr, kErrTimeout);
      break;
    }
    {
      // the pair whose stretch holds at: cum[j] <= at < cum[j + 1]
      int a = j, b = end - 1;
      while (a < b) {
        int mid = (a + b + 1) >> 1;
        if (cum[mid] <= at) a = mid;
        else b = mid - 1;
      }
      j = a;
    }
    int q = P.cp_list[j];
    double lam = cum[j + 1] - cum[j];
    if (!(lam > 0.0)) continue;
    double pos = (at - cum[j]) / lam;
    const PairState& S = P.pair[q];
    PairDesc d = P.pair_desc[q];
    int cell1 = d.b1 + nb * d.c1, cell2 = d.b2 + nb * d.c2;
    int O = cell1 == C ? cell2 : cell1;
    int n_o = P.cell_count[O];
    int o_start = P.cell_start[O];
    if (n_o < 1) continue;
    if (o_start < 0 || (long long)o_start + n_o > P.cap) {
      bad_index(P.ctr, kBadPairCells, q);
      break;
    }
    int i = (int)(g.next() * (double)n_o);
    if (i >= n_o) i = n_o - 1;
    int y = P.list[o_start + i];
    if (y < 0 || y >= P.cap) {
      bad_index(P.ctr, kBadTestSlot, y);
      continue;
    }
    if (y == x || !P.alive[y] || P.cell[y] != O) continue;
    n_tests++;
    bool first = cell1 == C;
    T k;
    if constexpr (sizeof(T) == 8) {
      const double* qw = (const double*)&P.recd[x];
      const double* qy = (const double*)&P.recd[y];
      k = (T)pair_kernel<KT, double, FLAT>(P, first ? qw : qy, first ? qy : qw, d.c1, d.c2, S.cc, S.fflat, P.coeff);
    } else {
      const float* qw = (const float*)&P.recf[x];
      const float* qy = (const float*)&P.recf[y];
      k = (T)pair_kernel<KT, float, FLAT>(P, first ? qw : qy, first ? qy : qw, d.c1, d.c2, S.cc, (float)S.fflat,
                                          (float)P.coeff);
    }
    T prob = k * (T)S.inv_k_max;
    if (!(prob <= T(1))) add_ll(&P.ctr->kmax_warn, 1LL);
    if (!((T)g.next() < prob)) continue;
    // the first accepted test: an event of the next step of the round,
    // claimed by its merge decision; an absorb (the walking particle is
    // replaced by the coagulated one) continues as a chain
    unsigned long long key = make_key((uint32_t)q, 1u, (uint32_t)x);
    unsigned long long ck = claim_key(P, key);
    Rng gm = merge_rng(P, key);
    double rx = P.rad[x], vtx = P.vtot[x], ry = P.rad[y], vty = P.vtot[y];
    MergeDecision m = first ? merge_decide_v(P, gm, rx, vtx, ry, vty, d.c1, d.c2, S.cc)
                            : merge_decide_v(P, gm, ry, vty, rx, vtx, d.c1, d.c2, S.cc);
    bool rm_x = first ? m.rm1 : m.rm2, rm_y = first ? m.rm2 : m.rm1;
    out->found = true;
    out->q = q;
    out->y = y;
    out->pos = (float)pos;
    out->first_cell1 = first;
    out->dec = pack_decision(m, gm.used());
    if (m.new_group == 0) set_status(P.ctr, kErrTimeout);
    claim_slot(P, x, ck, rm_x);
    claim_slot(P, y, ck, rm_y);
    out->cont = m.create && rm_x && m.new_group != 0;
    out->g_used = g.used();
    break;
  }
  if (n_tests) {
    add_ll(&P.ctr->tot_samp, n_tests);
    add_ll(&P.ctr->walk_tests, n_tests);
  }
}

// The work of a later round, one thread per event e of the round before:
//   - a winner that created or changed a particle (dest[e] >= 0): that
//     particle walks from the event's pair and position (for a chain, its
//     last applied event's);
//   - a loser: consumed = removed or rewritten in the round before
//     (touched), or dead.  A sample (kind 0) is retried with its key if
//     neither particle was consumed, else dropped.  A walk's test (kind 1,
//     a chain's first event): dropped if the walking particle was consumed,
//     the walk resumed after the test if only the partner was, else retried
//     alone.
// Output per e: flag, and key, slots, global pair and position of the new
// event (for a chain its first event) with the chain's length and head; the
// new event holds claims on its slots.
template <int KT, class T, bool FLAT>
__global__ void __launch_bounds__(256) k_items(const PopDev* pops, const int* gpair_pop, const int* gpair_local,
                                               const long long* pop_pair_base, int n_gpairs, const long long* n_items,
                                               const uint8_t* win, const int* dest,
                                               const unsigned long long* ev_key, const int2* ev_c,
                                               const int* gp_c, const float* ev_pos, const uint32_t* dec,
                                               ChainPool pool, uint8_t* it_flag, unsigned long long* it_key,
                                               int2* it_c, int* it_gp, float* it_pos, int* it_len, int* it_head,
                                               uint8_t* it_done, uint32_t* it_dec, uint32_t* it_gused) {
  long long n = *n_items;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    it_flag[e] = 0;
    int gp = gp_c[e];
    if (gp < 0 || gp >= n_gpairs) {
      bad_index(pops[0].ctr, kBadEventSlot, gp);
      continue;
    }
    int pop = gpair_pop[gp];
    const PopDev& P = pops[pop];
    int walker = -1, p0 = 0;
    float pos0 = ev_pos[e];
    unsigned long long key = ev_key[e];
    int2 sl = ev_c[e];
    if (win[e]) {
      walker = dest[e];
      p0 = gpair_local[gp];
      if (walker < 0) continue;
    } else {
      if (sl.x < 0 || sl.x >= P.cap || sl.y < 0 || sl.y >= P.cap) {
        bad_index(P.ctr, kBadEventSlot, sl.x < 0 || sl.x >= P.cap ? sl.x : sl.y);
        continue;
      }
      uint32_t gen_prev = *P.gen_p - 1u;
      bool c1 = P.touched[sl.x] == gen_prev || !P.alive[sl.x];
      bool c2 = P.touched[sl.y] == gen_prev || !P.alive[sl.y];
      if (key_kind(key) == 0u) {
        if (c1 || c2) continue;
      } else {
        int x = (int)key_idx(key);
        bool cx = x == sl.x ? c1 : c2, cy = x == sl.x ? c2 : c1;
        if (cx) continue;
        if (cy) {
          walker = x;
          p0 = (int)key_pair(key);
        }
      }
    }
    int len = 0, head = -1;
    bool done = false;
    uint32_t dc = dec[e];
    if (walker >= 0) {
      WalkOut w;
      walk<KT, T, FLAT>(P, pool, walker, p0, pos0, &w);
      if (!w.found) continue;
      key = make_key((uint32_t)w.q, 1u, (uint32_t)walker);
      sl = w.first_cell1 ? make_int2(walker, w.y) : make_int2(w.y, walker);
      gp = (int)(pop_pair_base[pop] + w.q);
      pos0 = w.pos;
      len = w.cont ? -1 : 0;  // -1: k_chain carries the walk on
      done = w.done;
      dc = w.dec;
      it_gused[e] = w.g_used;
    } else {
      // a retry keeps its merge decision and claims by it
      uint32_t used;
      MergeDecision m = unpack_decision(dc, &used);
      unsigned long long ck = claim_key(P, key);
      claim_slot(P, sl.x, ck, m.rm1);
      claim_slot(P, sl.y, ck, m.rm2);
    }
    it_flag[e] = 1;
    it_key[e] = key;
    it_c[e] = sl;
    it_gp[e] = gp;
    it_pos[e] = pos0;
    it_len[e] = len;
    it_head[e] = head;
    it_done[e] = done ? 1 : 0;
    it_dec[e] = dc;
  }
}

// Chains, after k_items: an item whose first event is an absorb (it_len -1)
// carries its walk on from that event with the coagulated particle
// (walk_chain), from the stream position the walk had reached.  The chain's
// events go to the pool, the first one included; the item gets the chain's
// length and head, or length 0 (the first event alone) if the pool is full.
template <int KT, class T, bool FLAT>
__global__ void __launch_bounds__(128) k_chain(const PopDev* pops, const int* gpair_pop, const long long* n_items,
                                               const uint8_t* it_flag, const unsigned long long* it_key,
                                               const int2* it_c, const int* it_gp, const float* it_pos,
                                               const uint32_t* it_dec, const uint32_t* it_gused, ChainPool pool,
                                               int* it_len, int* it_head, uint8_t* it_done) {
  long long n = *n_items;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    if (!it_flag[e] || it_len[e] != -1) continue;
    const PopDev& P = pops[gpair_pop[it_gp[e]]];
    unsigned long long key = it_key[e];
    int x = (int)key_idx(key), q = (int)key_pair(key);
    int2 sl = it_c[e];
    bool first = sl.x == x;
    int y = first ? sl.y : sl.x;
    uint32_t used;
    MergeDecision m = unpack_decision(it_dec[e], &used);
    bool rm_y = first ? m.rm2 : m.rm1;
    it_len[e] = 0;
    if (x < 0 || x >= P.cap || y < 0 || y >= P.cap || q >= P.n_pairs) continue;
    ChainWriter cw;
    if (!cw.append(pool, y, q | (rm_y ? kChainRemoves : 0), it_pos[e])) continue;
    Rng g = make_rng(P, kStreamWalk, 0u, (uint32_t)x);
    g.seek(it_gused[e]);
    WalkOut out;
    long long n_tests = 0;
    walk_chain<KT, T, FLAT>(P, pool, x, y, q, (double)it_pos[e], P.pair[q].cc + 1, g, cw, &out, &n_tests);
    it_len[e] = cw.len;
    it_head[e] = cw.head;
    it_done[e] = out.done ? 1 : 0;
    if (n_tests) {
      add_ll(&P.ctr->tot_samp, n_tests);
      add_ll(&P.ctr->walk_tests, n_tests);
    }
  }
}

// Apply the winning chains (win[e] == 2), one warp per chain: the first
// ev_app[e] events in order, each a coagulate (coagulation.F90:928-985) of
// the walking particle with the next partner, with the merge decision
// recomputed from the values and the stream the walk used.  Lanes hold the
// particle's species (lane, lane + 32) and components (lane); every lane
// draws the same merge decision and component selection; sums run in the
// walk's order (per species over the events, then over the species), so the
// decisions are the walk's.  The coagulated particle stays in the walking
// particle's slot; partners that a decision removes are killed.  dest[e],
// gp_c[e] and ev_pos[e] are set to where the particle walks on (dest -1 if
// its walk ran to the end).
__global__ void __launch_bounds__(256) k_apply_chain(const PopDev* pops, const int* gpair_pop,
                                                     const long long* pop_pair_base, const long long* n_events,
                                                     const unsigned long long* ev_key, const uint8_t* win,
                                                     const int* ev_len, const int* ev_app, const int* ev_head,
                                                     const uint8_t* ev_done, ChainPool pool, int* gp_c, float* ev_pos,
                                                     int* dest_out) {
  constexpr unsigned kFull = 0xffffffffu;
  long long E = *n_events;
  const int lane = threadIdx.x & 31;
  long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  long long n_warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long e = warp; e < E; e += n_warps) {
    if (win[e] != 2) continue;  // the same e for the whole warp
    int pop = gpair_pop[gp_c[e]];
    const PopDev& P = pops[pop];
    unsigned long long key1 = ev_key[e];
    int x = (int)key_idx(key1);
    int app = ev_app[e];
    if (x < 0 || x >= P.cap) {
      if (lane == 0) bad_index(P.ctr, kBadEventSlot, x);
      continue;
    }
    const int nb = P.grid->n_bin, ns = P.n_spec;
    uint32_t gen = *P.gen_p;
    // the walking particle, spread over the lanes
    double v_lo = lane < ns ? P.vol[vol_at(P, x, lane)] : 0.0;
    double v_hi = lane + 32 < ns ? P.vol[vol_at(P, x, lane + 32)] : 0.0;
    PScal cur;
    load_scal(P, x, cur);
    int cc_ = 0;
    double ct_ = 0.0;
    if (lane < cur.ncomp && lane < kMaxComponent) {
      cc_ = P.csrc[comp_at(x, lane)];
      ct_ = P.ctime[comp_at(x, lane)];
    }
    double r = P.rad[x], vt = P.vtot[x];
    int C = P.cell[x];
    ChainReader rd(ev_head[e]);
    int done_ev = 0, last_q = -1, dlive = 0;
    float last_pos = 0.f;
    for (int i = 0; i < app; i++) {
      long long ix = rd.next(pool);
      int y = ix < 0 ? -1 : pool.y[ix];
      int q = ix < 0 ? -1 : (pool.q[ix] & kChainPairMask);
      if (ix < 0 || y < 0 || y >= P.cap || q >= P.n_pairs) {
        if (lane == 0) bad_index(P.ctr, kBadEventSlot, y);
        break;
      }
      PairDesc d = P.pair_desc[q];
      const PairState& S = P.pair[q];
      bool first = C == d.b1 + nb * d.c1;
      Rng g = i == 0 ? merge_rng(P, key1) : make_rng(P, kStreamChain, (uint32_t)(i + 1), (uint32_t)x);
      double ry = P.rad[y], vty = P.vtot[y];
      MergeDecision m = first ? merge_decide_v(P, g, r, vt, ry, vty, d.c1, d.c2, S.cc)
                              : merge_decide_v(P, g, ry, vty, r, vt, d.c1, d.c2, S.cc);
      bool rm_x = first ? m.rm1 : m.rm2, rm_y = first ? m.rm2 : m.rm1;
      bool lost_x = first ? m.lost1 : m.lost2, lost_y = first ? m.lost2 : m.lost1;
      if (!(m.create && rm_x && m.new_group != 0) || (lost_x && !(rm_y && !lost_y))) {
        if (lane == 0) set_status(P.ctr, kErrAssert);  // the walk decided an absorb here
        break;
      }
      // the partner
      PScal ys;
      load_scal(P, y, ys);
      double y_lo = lane < ns ? P.vol[vol_at(P, y, lane)] : 0.0;
      double y_hi = lane + 32 < ns ? P.vol[vol_at(P, y, lane + 32)] : 0.0;
      int yc = 0;
      double yt = 0.0;
      if (lane < ys.ncomp && lane < kMaxComponent) {
        yc = P.csrc[comp_at(y, lane)];
        yt = P.ctime[comp_at(y, lane)];
      }
      double ice_x = 0.0, ice_y = 0.0;
      if (P.i_water > 0) {
        int w = P.i_water - 1;
        ice_x = __shfl_sync(kFull, w < 32 ? v_lo : v_hi, w & 31);
        ice_y = __shfl_sync(kFull, w < 32 ? y_lo : y_hi, w & 31);
      }
      // components of aero_particle_coagulate with a = particle 1, b = particle 2
      const PScal& A = first ? cur : ys;
      const PScal& B = first ? ys : cur;
      int ca = first ? cc_ : yc, cb = first ? yc : cc_;
      double ta = first ? ct_ : yt, tb = first ? yt : ct_;
      int na = A.ncomp, nbc = B.ncomp;
      int n1_new = na, n2_new = nbc;
      bool from_a = lane < na;
      int k_src = from_a ? lane : lane - na;
      if (na + nbc > kMaxComponent) {
        int sa[kMaxComponent], sb[kMaxComponent];
        coag_components(g, na, A.nprim, nbc, B.nprim, &n1_new, &n2_new, sa, sb);
        from_a = lane < n1_new;
        k_src = 0;
        if (from_a) k_src = sa[lane] - 1;
        else if (lane - n1_new < n2_new) k_src = sb[lane - n1_new] - 1;
      }
      k_src &= 31;
      int xa = __shfl_sync(kFull, ca, k_src), xb = __shfl_sync(kFull, cb, k_src);
      double za = __shfl_sync(kFull, ta, k_src), zb = __shfl_sync(kFull, tb, k_src);
      int n_out = n1_new + n2_new;
      PScal nm;
      coag_scalars(A, first ? ice_x : ice_y, B, first ? ice_y : ice_x, nm);
      nm.ncomp = n_out;
      nm.id = !lost_x ? cur.id : ys.id;
      nm.grp = m.new_group;
      nm.cls = S.cc + 1;
      cc_ = lane < n_out ? (from_a ? xa : xb) : 0;
      ct_ = lane < n_out ? (from_a ? za : zb) : 0.0;
      // volumes: per species over the events, then the total over the species
      v_lo = v_lo + y_lo;
      v_hi = v_hi + y_hi;
      double s_v = 0.0;
      for (int s = 0; s < ns; s++) s_v = s_v + __shfl_sync(kFull, s < 32 ? v_lo : v_hi, s & 31);
      vt = s_v;
      r = vol2rad(vt);
      C = cell_of(P, r, nm.cls);
      if (rm_y) {
        if (lane == 0) {
          kill_slot(P, y);
          P.touched[y] = gen;
        }
        dlive--;
      }
      cur = nm;
      done_ev++;
      last_q = q;
      last_pos = pool.pos[ix];
    }
    if (done_ev == 0) continue;
    // the coagulated particle in the walking particle's slot
    __syncwarp();
    if (lane < ns) P.vol[vol_at(P, x, lane)] = v_lo;
    if (lane + 32 < ns) P.vol[vol_at(P, x, lane + 32)] = v_hi;
    if (lane < cur.ncomp && lane < kMaxComponent) {
      P.csrc[comp_at(x, lane)] = cc_;
      P.ctime[comp_at(x, lane)] = ct_;
    }
    double ms = 0.0;
    for (int s = 0; s < ns; s++)
      ms = ms + __shfl_sync(kFull, s < 32 ? v_lo : v_hi, s & 31) * P.density[s];
    if (lane == 0) {
      P.vtot[x] = vt;
      P.mass[x] = ms;
      P.grp[x] = cur.grp;
      P.cls[x] = cur.cls;
      P.id[x] = cur.id;
      P.nprim[x] = cur.nprim;
      P.ncomp[x] = cur.ncomp;
      P.lct[x] = cur.lct;
      P.gct[x] = cur.gct;
      P.imf[x] = cur.imf;
      P.den_ice[x] = cur.den_ice;
      P.phi[x] = cur.phi;
      P.hyst[x] = cur.hyst;
      P.frozen[x] = cur.frozen;
      P.alive[x] = 1;
      P.changed[x] = 1;
      P.touched[x] = gen;
      int nbin = refresh_slot(P, x);
      bool on_grid = nbin >= 1 && nbin <= nb;
      if (!on_grid) set_status(P.ctr, kErrOutOfGrid);
      add_ll(&P.ctr->tot_coag, (long long)done_ev);
      if (dlive) add_ll(&P.ctr->n_live, (long long)dlive);
      bool walk_done = ev_done[e] && done_ev == ev_len[e];
      dest_out[e] = (walk_done || !on_grid) ? -1 : x;
      gp_c[e] = (int)(pop_pair_base[pop] + last_q);
      ev_pos[e] = last_pos;
    }
  }
}

// Walk rates after a round's sort: for every cell, the running sum over its
// pairs (loop order) of k_max * del_t * members of the pair's other cell;
// pairs on the per-particle path add nothing.  One block per cell, its
// threads over the cell's pairs, a block-wide scan in a fixed order.
__global__ void __launch_bounds__(128) k_walk_rates(const PopDev* pops) {
  const PopDev& P = pops[blockIdx.y];
  int c = blockIdx.x;
  if (c >= P.n_cells || P.n_pairs == 0) return;
  const int nb = P.grid->n_bin;
  const int lo = P.cp_off[c], hi = P.cp_off[c + 1];
  double* cum = P.cp_cum + lo + c;
  __shared__ double wsum[4];
  __shared__ double carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0.0;
  __syncthreads();
  for (int base = lo; base < hi; base += blockDim.x) {
    int j = base + threadIdx.x;
    double lam = 0.0;
    if (j < hi) {
      int q = P.cp_list[j];
      const PairState& S = P.pair[q];
      if (S.path != kPathParticle) {
        PairDesc d = P.pair_desc[q];
        int cell1 = d.b1 + nb * d.c1, cell2 = d.b2 + nb * d.c2;
        int O = cell1 == c ? cell2 : cell1;
        double l = S.k_max * P.del_t * (double)P.cell_count[O];
        if (l > 0.0) lam = l;
      }
    }
    double x = lam;  // inclusive scan within the warp
    for (int o = 1; o < 32; o <<= 1) {
      double y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    double before = carry;
    for (int w = 0; w < wid; w++) before += wsum[w];
    if (j < hi) cum[j - lo] = before + x - lam;
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[0] + wsum[1] + wsum[2] + wsum[3];
    __syncthreads();
  }
  if (threadIdx.x == 0) cum[hi - lo] = carry;
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
                         const int* op_slot, const int* op_k, const unsigned long long* op_key,
                         const long long* n_ops, PPResult* res, double* res_vol) {
  long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    const PopDev& P = pops[op_pop[q]];
    int p = op_pair[q], t = op_slot[q];
    unsigned long long prio = op_key[q];
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
__global__ void k_pp_resolve(const PopDev* pops, const int* op_pop, const unsigned long long* op_key,
                             const long long* n_ops, const PPResult* res, uint8_t* win,
                             int* need_slot, int* need_id, int* lost) {
  long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    const PopDev& P = pops[op_pop[q]];
    const PPResult& R = res[q];
    unsigned long long prio = op_key[q];
    bool ok = true;
    if (R.merged) ok = ok && holds_slot(P, R.target, claim_key(P, prio), true);
    for (int z = 0; z < R.n_rm; z++) ok = ok && holds_slot(P, R.rm[z], claim_key(P, prio), true);
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
    uint32_t gen = *P.gen_p;
    int dlive = 0;
    for (int z = 0; z < R.n_rm; z++) {
      kill_slot(P, R.rm[z]);
      P.touched[R.rm[z]] = gen;
      dlive--;
    }
    if (R.merged) {
      const double* v = res_vol + (size_t)q * P.n_spec;
      int t = R.target;
      P.touched[t] = gen;
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
          P.touched[dest] = gen;
          dlive++;
        }
      }
    }
    if (dlive) add_ll(&P.ctr->n_live, (long long)(dlive));
  }
}

}  // namespace pmc
