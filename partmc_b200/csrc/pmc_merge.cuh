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
      long long nc = (long long)inc_warp((unsigned long long*)C.ctr);
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

// A chain stops at an accepted test that is no absorb (or that the pool has
// no room for).  That test has happened: dropping it and walking on afresh
// in the next round would redraw its merge decision until an absorb came up,
// which favours absorbs whenever the weights make some decisions keep the
// walking particle (with flat weights every decision absorbs).  So the
// stopping test is carried to the next round as a pending event with its
// decision: its partner, pair (and whether the walker is in the pair's first
// cell), decision and position, packed as {y, q | first << 30, decision,
// position bits}; y = -1 for none.  An event whose dest_out is kPendingTerm
// hands that test to the next round (k_items) instead of a walk.
constexpr int kPendingTerm = -2;
// The same holds for a chain cut short where a partner's claim failed: the
// claim's kind (write or read) follows the event's decision, so the cut
// depends on it, and walking on afresh would redraw that decision.  The
// first event not applied is pending for the next round (kPendingChain),
// its decision recomputed there from the chain's stream (event index in
// the decision word) and the particles' values, which give the decision
// the walk made whenever the partner is unchanged.
constexpr int kPendingChain = -3;
constexpr int kTermFirst = 1 << 30;
__device__ __forceinline__ int4 no_term() { return make_int4(-1, 0, 0, 0); }

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
                              const int* ev_head, int* ev_app, ChainPool pool, int* chain_list, long long* n_chain) {
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
      add_ll_warp(n_losers, 1);
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
      chain_list[inc_warp((unsigned long long*)n_chain)] = (int)e;
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
// the per-particle vectors, one thread per event.  The species of the two
// sources (particle-major, each source a few cache lines) are added in blocks
// of kMoveBlock: a block's loads are all issued before its sums are stored,
// and the destination (which may be a source) is written species by species
// after that species was read.  The components are gathered into local
// arrays before any is written, in the order of the random selection
// (computed from the stream position the test stored).  The summed volume and
// mass go to the destination's caches for part 2; the water volumes of the
// sources, which part 2 needs after the destination may have been
// overwritten, go to ice[e].
constexpr int kMoveBlock = 8;

__global__ void __launch_bounds__(256) k_apply_move(const PopDev* pops, const int* gpair_pop,
                                                    const long long* n_events, const unsigned long long* ev_key,
                                                    const int2* ev, const int* ev_gp, const uint8_t* win,
                                                    const uint32_t* dec, const long long* slot_rank,
                                                    const int* slot_base, double2* ice) {
  long long E = *n_events;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
       e += (long long)gridDim.x * blockDim.x) {
    if (win[e] != 1) continue;  // chains apply in k_apply_chain
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
    const int ns = P.n_spec;
    const double* v1 = P.vol + vol_at(P, s1, 0);
    const double* v2 = P.vol + vol_at(P, s2, 0);
    double* vd = P.vol + vol_at(P, dest, 0);
    if (P.i_water > 0) ice[e] = make_double2(v1[P.i_water - 1], v2[P.i_water - 1]);
    // components: every source entry is read before the first write
    int na = P.ncomp[s1], nb = P.ncomp[s2];
    na = na < kMaxComponent ? na : kMaxComponent;
    nb = nb < kMaxComponent ? nb : kMaxComponent;
    int ca[kMaxComponent], cb[kMaxComponent];
    double ta[kMaxComponent], tb[kMaxComponent];
    for (int k = 0; k < na; k++) {
      ca[k] = P.csrc[comp_at(s1, k)];
      ta[k] = P.ctime[comp_at(s1, k)];
    }
    for (int k = 0; k < nb; k++) {
      cb[k] = P.csrc[comp_at(s2, k)];
      tb[k] = P.ctime[comp_at(s2, k)];
    }
    // totals in the reference's order (species 1..n)
    double vt = 0.0, ms = 0.0;
    for (int s0 = 0; s0 < ns; s0 += kMoveBlock) {
      double x1[kMoveBlock], x2[kMoveBlock];
#pragma unroll
      for (int j = 0; j < kMoveBlock; j++) {
        x1[j] = s0 + j < ns ? v1[s0 + j] : 0.0;
        x2[j] = s0 + j < ns ? v2[s0 + j] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < kMoveBlock; j++) {
        if (s0 + j < ns) {
          double v = x1[j] + x2[j];
          vt = vt + v;
          ms = ms + v * P.density[s0 + j];
          vd[s0 + j] = v;
        }
      }
    }
    int n1_new = na, n2_new = nb;
    if (na + nb > kMaxComponent) {
      int sa[kMaxComponent], sb[kMaxComponent];
      Rng g = merge_rng(P, ev_key[e]);
      g.seek(used);
      coag_components(g, na, P.nprim[s1], nb, P.nprim[s2], &n1_new, &n2_new, sa, sb);
      for (int k = 0; k < n1_new; k++) {
        P.csrc[comp_at(dest, k)] = ca[sa[k] - 1];
        P.ctime[comp_at(dest, k)] = ta[sa[k] - 1];
      }
      for (int k = 0; k < n2_new; k++) {
        P.csrc[comp_at(dest, n1_new + k)] = cb[sb[k] - 1];
        P.ctime[comp_at(dest, n1_new + k)] = tb[sb[k] - 1];
      }
    } else {
      for (int k = 0; k < na; k++) {
        P.csrc[comp_at(dest, k)] = ca[k];
        P.ctime[comp_at(dest, k)] = ta[k];
      }
      for (int k = 0; k < nb; k++) {
        P.csrc[comp_at(dest, na + k)] = cb[k];
        P.ctime[comp_at(dest, na + k)] = tb[k];
      }
    }
    P.vtot[dest] = vt;
    P.mass[dest] = ms;
    P.ncomp[dest] = n1_new + n2_new;
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
                            const double2* ice, const uint8_t* ev_done, int* dest_out, unsigned long long* ev_key_w,
                            int2* ev_w, int* gp_w, float* pos_w, uint32_t* dec_w, const int4* ev_term,
                            const long long* pop_pair_base) {
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
    add_ll_warp(&P.ctr->tot_coag, 1);
    if (m.rm1) P.touched[s1] = gen;
    if (m.rm2) P.touched[s2] = gen;
    if (!m.create) {
      // coagulate (coagulation.F90:928-985) records a removal whose ID is lost
      if (m.rm1 && m.lost1) log_removal(P, P.id[s1], kInfoCoag, 0);
      if (m.rm2 && m.lost2) log_removal(P, P.id[s2], kInfoCoag, 0);
      if (m.rm1) kill_slot(P, s1);
      if (m.rm2) kill_slot(P, s2);
      int dlive = -(int)m.rm1 - (int)m.rm2;
      if (dlive) add_ll_warp(&P.ctr->n_live, dlive);
      continue;
    }
    int dest = event_dest(m, s1, s2, slot_base[pop], m.rm1 || m.rm2 ? 0 : slot_rank[e]);
    if (dest >= P.cap) {
      cap_fail(P.ctr, kCapEventDest);
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
    long long new_id;
    if (m.rm1 && !m.lost1) new_id = a.id;
    else if (m.rm2 && !m.lost2) new_id = b.id;
    else new_id = id_base[pop] + id_rank[e];
    P.id[dest] = new_id;
    if (m.rm1 && m.lost1) log_removal(P, a.id, kInfoCoag, new_id);
    if (m.rm2 && m.lost2) log_removal(P, b.id, kInfoCoag, new_id);
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
    if (nbin < 1 || nbin > P.grid->n_bin) {
      set_status(P.ctr, kErrOutOfGrid);
    } else if (ev_term[e].x >= 0) {
      // a one-event chain that stopped at a pending test: the coagulated
      // particle (in slot dest) meets that test in the next round
      const int4 t = ev_term[e];
      const int tq = t.y & (kTermFirst - 1);
      const bool tfirst = (t.y & kTermFirst) != 0;
      ev_key_w[e] = make_key((uint32_t)tq, 1u, (uint32_t)dest);
      ev_w[e] = tfirst ? make_int2(dest, t.x) : make_int2(t.x, dest);
      gp_w[e] = (int)(pop_pair_base[pop] + tq);
      pos_w[e] = __int_as_float(t.w);
      dec_w[e] = (uint32_t)t.z;
      dest_out[e] = kPendingTerm;
    } else if (!(key_kind(ev_key[e]) == 1u && ev_done[e])) {
      dest_out[e] = dest;  // a walk that ran to its end stops
    }
    if (m.rm1 && dest != s1) kill_slot(P, s1);
    if (m.rm2 && dest != s2) kill_slot(P, s2);
    int dlive = 1 - (int)m.rm1 - (int)m.rm2;
    if (dlive) add_ll_warp(&P.ctr->n_live, dlive);
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
  bool done = false;        // the walk ran to the end after its last event
  uint32_t dec = 0;         // merge decision of the first event
  bool cont = false;        // the first event is an absorb: k_chain carries the walk on
  uint32_t g_used = 0;      // index of the walk's next test after the first event
  bool stop = false;        // the walk reached a per-particle pair (q) whose target cell is its cell
};

// true if this round's claim on slot y is the chain of walker x
__device__ __forceinline__ bool claimed_by_walk(const PopDev& P, int y, int x) {
  unsigned long long w = P.claim[y];
  return (w >> 53) == (unsigned long long)(~*P.gen_p & kGenLimit) && ((w >> 32) & 1ULL) &&
         (uint32_t)w == (uint32_t)x;
}

// The uniforms of a walk's test t: one Philox block keyed by the population,
// counted by (step, round, walk stream, walking slot, t).  x, y: the gap to
// the test (u53 -> exponential); z: the partner; w: the accept draw.  Every
// test takes one block whether or not its partner is a member, so a test's
// draws depend on its index alone.
__device__ __forceinline__ U4 walk_draws(const PopDev& P, int x, uint32_t t) {
  return philox4x32_10(U4{P.step, ((*P.round_p & 0xffu) << 4) | kStreamWalk, (uint32_t)x, t}, (uint32_t)P.seed,
                       (uint32_t)(P.seed >> 32));
}

// A walk's place in the stretch of its cell C: the entries lo..end of the
// cell's pair list, cum[j] (indexable by list entry j) the expected tests
// before entry j, at the running position, j the entry that holds it.
struct Stretch {
  const double* cum;
  const int* tab;
  int C, end, j;
  double at, total;
  int stop;  // the stop (cp_nstop) that ends the stretch, or -1: it runs to the cell's last pair
};

// the stretch of cell C from (pair p0, position pos0 in it) on.  The first
// entry of the cell's pair list whose pair is p0 or later: the cell's coarse
// row (every 16th entry, read as int4) counts the coarse entries before p0,
// then the at most 15 entries after the last of them are counted.
__device__ __forceinline__ void walk_stretch(const PopDev& P, int C, int p0, float pos0, Stretch* s) {
  int lo = P.cp_off[C], end = P.cp_off[C + 1];
  const double* cum = P.cp_cum + (lo + C) - lo;
  const int4* cz = reinterpret_cast<const int4*>(P.cp_coarse + (size_t)C * P.n_coarse);
  int k = 0;
#pragma unroll 4
  for (int b = 0; b < P.n_coarse / 4; b++) {
    const int4 v = cz[b];
    k += (v.x < p0) + (v.y < p0) + (v.z < p0) + (v.w < p0);
  }
  int a = k == 0 ? lo : lo + 16 * (k - 1) + 1;
  const int hi = min(lo + 16 * k, end);
  int cnt = 0;
#pragma unroll
  for (int t = 0; t < 15; t++)
    if (a + t < hi) cnt += P.cp_list[a + t] < p0;
  a += cnt;
  double at = cum[a];
  if (a < end && P.cp_list[a] == p0) at += (cum[a + 1] - cum[a]) * (double)pos0;
  // the stretch ends at the first stop after the start; a walk that starts
  // at the end of a pair (its target operation there is done) looks past it
  const int sa = (a < end && P.cp_list[a] == p0 && pos0 >= 1.0f) ? a + 1 : a;
  const int stop = (P.walk_stops && sa < end) ? P.cp_nstop[sa] : end;
  s->cum = cum;
  s->tab = P.cp_tab + (size_t)C * kWalkTab;
  s->C = C;
  s->stop = stop < end ? stop : -1;
  if (stop < end) end = stop;
  s->end = end;
  s->j = a < end ? a : (end > P.cp_off[C] ? end - 1 : end);
  s->at = at;
  s->total = cum[end];
}

// the entry j >= s.j with cum[j] <= at < cum[j + 1] (at < total): the
// cell's bucket table gives a start at or before it, a short scan forward
// usually ends there, a binary search covers the rest
__device__ __forceinline__ int walk_pair(const Stretch& s, double at) {
  const double* cum = s.cum;
  int b = (int)(at / s.total * (double)kWalkTab);
  b = b < 0 ? 0 : (b >= kWalkTab ? kWalkTab - 1 : b);
  int hi = s.end - 1;
  int j = s.tab[b];
  j = j < s.j ? s.j : (j > hi ? hi : j);
  int a, z;
  if (cum[j] > at) {  // rounding put the bucket past at
    a = s.j;
    z = j - 1 < s.j ? s.j : j - 1;
  } else {
    for (int k = 0; k < 4 && j < hi; k++) {
      if (cum[j + 1] > at) return j;
      j++;
    }
    a = j;
    z = hi;
  }
  while (a < z) {
    int mid = (a + z + 1) >> 1;
    if (cum[mid] <= at) a = mid;
    else z = mid - 1;
  }
  return a;
}

// Partner draws of a chain's test t after the first: the walk stream's
// block (x, t + r * 2^26) for the r-th redraw (t stays below 2^26).
constexpr uint32_t kChainRedraws = 64;
__device__ __forceinline__ uint32_t walk_redraw(const PopDev& P, int x, uint32_t t, uint32_t r) {
  return walk_draws(P, x, t | (r << 26)).x;
}

// One walk test t of particle x (records qxd/qxf) at running position at of
// its stretch, in entry j: the partner drawn from the other cell's members
// and the accept test.  The pair's fields and the partner slot are loaded
// together, then the partner's state.  In a chain, a partner that the chain
// has absorbed already is drawn again: the reference draws a pair's samples
// from the members left when each sample runs, after the earlier samples'
// merges, and exits the pair when a cell is empty (per_set_coag,
// coagulation.F90:628-638); a test whose kChainRedraws draws all land on
// absorbed members counts as that exit.  Returns 0 for no test (no member,
// itself, a dead or moved member, the exit), 1 for a rejected test, 2 for an
// accepted one, -1 for a failed bounds check.
template <int KT, class T, bool FLAT>
__device__ __forceinline__ int walk_test(const PopDev& P, int x, const Stretch& s, int j, double at, uint32_t t,
                                         uint32_t pick, uint32_t accu, const RecD& qxd, const RecF& qxf, bool chain,
                                         int* y_out, float* pos_out, int* q_out, bool* first_out, double* ry_out,
                                         double* vty_out) {
  const double c0 = s.cum[j], c1 = s.cum[j + 1];
  const int4 ent = P.cp_ent[j];
  double lam = c1 - c0;
  int n_o = ent.w, o_start = ent.z;
  if (!(lam > 0.0) || n_o < 1) return 0;
  if (o_start < 0 || (long long)o_start + n_o > P.cap || ent.x < 0 || ent.x >= P.n_pairs) {
    bad_index(P.ctr, kBadPairCells, ent.x);
    return -1;
  }
  const int q = ent.x, O = ent.y & ((1 << 30) - 1);
  const bool first = (ent.y >> 30) & 1;
  int i = (int)(u32d(pick) * (double)n_o);
  if (i >= n_o) i = n_o - 1;
  int y = P.list[o_start + i];
  if (chain) {
    for (uint32_t r = 1; y >= 0 && y < P.cap && claimed_by_walk(P, y, x); r++) {
      if (r >= kChainRedraws) return 0;
      i = (int)(u32d(walk_redraw(P, x, t, r)) * (double)n_o);
      if (i >= n_o) i = n_o - 1;
      y = P.list[o_start + i];
    }
  }
  const PairDesc d = P.pair_desc[q];
  const PairState& S = P.pair[q];
  const double inv_k_max = S.inv_k_max, fflat = S.fflat;
  const int cc = S.cc;
  if (y < 0 || y >= P.cap) {
    bad_index(P.ctr, kBadTestSlot, y);
    return -1;
  }
  const uint8_t alive = P.alive[y];
  const int cell_y = P.cell[y];
  const double ry = P.rad[y], vty = P.vtot[y];  // for the merge decision if the test accepts
  if (y == x || !alive || cell_y != O) return 0;
  const double u = u32d(accu);
  bool acc;
  if constexpr (sizeof(T) == 8) {
    const RecD qy = P.recd[y];
    acc = accept_f64_rec<KT, FLAT>(P, first ? qxd : qy, first ? qy : qxd, d, cc, fflat, inv_k_max, u);
  } else {
    const RecF qy = P.recf[y];
    const float* qw = (const float*)&qxf;
    const float* py = (const float*)&qy;
    const float pf = pair_kernel<KT, float, FLAT>(P, first ? qw : py, first ? py : qw, d.c1, d.c2, cc,
                                                  (float)fflat, (float)P.coeff) *
                     (float)inv_k_max;
    if (f32_decides(pf, u)) {
      acc = u < (double)pf;
    } else {  // decided in FP64 (see f32_decides)
      const RecD qy = P.recd[y];
      acc = accept_f64_rec<KT, FLAT>(P, first ? qxd : qy, first ? qy : qxd, d, cc, fflat, inv_k_max, u);
      add_ll(&P.ctr->exact_tests, 1LL);
    }
  }
  *y_out = y;
  *pos_out = (float)((at - c0) / lam);
  *q_out = q;
  *first_out = first;
  *ry_out = ry;
  *vty_out = vty;
  return acc ? 2 : 1;
}

// The next accepted test of walker x from s on, drawing tests t_next,
// t_next + 1, ...: returns 1 with the test's entry in s.j and position in
// s.at, 0 if the walk ran to the end of the stretch, -1 on a failed check or
// the test limit.  n_tests counts the tests with a partner.
template <int KT, class T, bool FLAT>
__device__ __forceinline__ int walk_next(const PopDev& P, int x, Stretch& s, uint32_t& t_next, const RecD& qxd,
                                         const RecF& qxf, bool chain, long long* n_tests, int* y, float* pos,
                                         int* q, bool* first, double* ry, double* vty) {
  for (;;) {
    const uint32_t t = t_next++;
    U4 u = walk_draws(P, x, t);
    double at = s.at - log(u53(u.x, u.y));
    if (!(at < s.total)) {
      s.at = at;
      if (s.stop >= 0) {  // a per-particle pair that takes the particle as a target
        *q = P.cp_list[s.stop];
        return 3;
      }
      return 0;  // no test left in the cell's later pairs
    }
    if (t >= (1u << 26)) {  // far past any mean the step can ask for
      set_status(P.ctr, kErrTimeout);
      return -1;
    }
    int j = walk_pair(s, at);
    s.j = j;
    s.at = at;
    int r = walk_test<KT, T, FLAT>(P, x, s, j, at, t, u.z, u.w, qxd, qxf, chain, y, pos, q, first, ry, vty);
    if (r < 0) return -1;
    if (r == 0) continue;
    (*n_tests)++;
    if (r == 2) return 1;
  }
}

// The first event of walker x from (p0, pos0): the first accepted test,
// claimed by its merge decision; an absorb (the walking particle is replaced
// by the coagulated one) is carried on as a chain by k_chain from the next
// test on.
template <int KT, class T, bool FLAT>
__device__ void walk(const PopDev& P, int x, int p0, float pos0, WalkOut* out) {
  if (x < 0 || x >= P.cap || !P.alive[x]) return;
  const int C = P.cell[x];
  if (C < 0 || C >= P.n_cells) return;
  Stretch s;
  walk_stretch(P, C, p0, pos0, &s);
  const RecD qxd = P.recd[x];
  const RecF qxf = P.recf[x];
  long long n_tests = 0;
  uint32_t t_next = 0;
  int y, q;
  float pos;
  bool first;
  double ry, vty;
  int r = walk_next<KT, T, FLAT>(P, x, s, t_next, qxd, qxf, false, &n_tests, &y, &pos, &q, &first, &ry, &vty);
  if (r == 0) out->done = true;
  if (r == 3) {
    out->stop = true;
    out->q = q;
  }
  if (r == 1) {
    const PairDesc d = P.pair_desc[q];
    const PairState& S = P.pair[q];
    unsigned long long key = make_key((uint32_t)q, 1u, (uint32_t)x);
    unsigned long long ck = claim_key(P, key);
    Rng gm = merge_rng(P, key);
    double rx = P.rad[x], vtx = P.vtot[x];
    MergeDecision m = first ? merge_decide_v(P, gm, rx, vtx, ry, vty, d.c1, d.c2, S.cc)
                            : merge_decide_v(P, gm, ry, vty, rx, vtx, d.c1, d.c2, S.cc);
    bool rm_x = first ? m.rm1 : m.rm2, rm_y = first ? m.rm2 : m.rm1;
    out->found = true;
    out->q = q;
    out->y = y;
    out->pos = pos;
    out->first_cell1 = first;
    out->dec = pack_decision(m, gm.used());
    if (m.new_group == 0) set_status(P.ctr, kErrTimeout);
    claim_slot(P, x, ck, rm_x);
    claim_slot(P, y, ck, rm_y);
    out->cont = m.create && rm_x && m.new_group != 0;
    out->g_used = t_next;
  }
  if (n_tests) {
    add_ll_warp(&P.ctr->tot_samp, (int)n_tests);
    add_ll_warp(&P.ctr->walk_tests, (int)n_tests);
  }
}

// A chain's event i again, for the pending event of a chain cut short: the
// decision the walk made, from the chain's stream and the particles' values
// (0xffffffff for a bad pair index)
__device__ __noinline__ uint32_t chain_event_decision(const PopDev& P, unsigned long long key, int2 sl, int x, int y,
                                                      uint32_t i) {
  const int q = (int)key_pair(key);
  if (q >= P.n_pairs) {
    bad_index(P.ctr, kBadEventSlot, q);
    return 0xffffffffu;
  }
  const PairDesc d = P.pair_desc[q];
  const PairState& S = P.pair[q];
  Rng g = make_rng(P, kStreamChain, i + 1u, (uint32_t)x);
  MergeDecision m = sl.x == x ? merge_decide_v(P, g, P.rad[x], P.vtot[x], P.rad[y], P.vtot[y], d.c1, d.c2, S.cc)
                              : merge_decide_v(P, g, P.rad[y], P.vtot[y], P.rad[x], P.vtot[x], d.c1, d.c2, S.cc);
  if (m.new_group == 0) set_status(P.ctr, kErrTimeout);
  return pack_decision(m, g.used());
}

// A target operation for particle x at per-particle pair q (its walk reached
// the pair with x in the pair's target cell), at place k of the round's
// operations: after the redone ones, at the item's own index, so that the
// list's order does not depend on scheduling (the places of items without
// one hold population -1 and are dropped when the list is grouped).  It runs
// in this round; its key puts it after the pair's own operations.
__device__ __noinline__ void add_target_op(const PopDev& P, int pop, int q, int x, int* op_pop, int* op_pair,
                                              int* op_slot, int* op_k, unsigned long long* op_key, long long k,
                                              long long op_cap) {
  if (k >= op_cap) {
    cap_fail(P.ctr, kCapTargetOps);
    return;
  }
  op_pop[k] = pop;
  op_pair[k] = q;
  op_slot[k] = x;
  op_k[k] = 0x40000000 | x;  // its own stream: round-0 operations count from 0, redos add 1 << 24
  op_key[k] = make_key((uint32_t)q, 1u, (uint32_t)x);
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
                                               const long long* n_items_ev, const int* ppw_slot, const int* ppw_gp,
                                               int* op_pop, int* op_pair, int* op_slot, int* op_k,
                                               unsigned long long* op_key, long long* n_ops, long long op_cap,
                                               const uint8_t* win, const int* dest,
                                               const unsigned long long* ev_key, const int2* ev_c,
                                               const int* gp_c, const float* ev_pos, const uint32_t* dec,
                                               uint8_t* it_flag, unsigned long long* it_key,
                                               int2* it_c, int* it_gp, float* it_pos, int* it_len, int* it_head,
                                               uint8_t* it_done, uint32_t* it_dec, uint32_t* it_gused, int4* it_term) {
  long long n = *n_items, n_ev = *n_items_ev;
  const long long op_base = op_cap > 0 ? *n_ops : 0;  // the redone operations come first
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    it_flag[e] = 0;
    it_term[e] = no_term();
    if (op_cap > 0 && op_base + e < op_cap) op_pop[op_base + e] = -1;
    int gp, walker = -1, p0 = 0;
    float pos0 = 1.0f;
    unsigned long long key = 0;
    int2 sl = make_int2(-1, -1);
    uint32_t dc = 0;
    if (e >= n_ev) {
      // a particle that a target operation of the round before made or
      // changed walks from the end of that operation's pair
      gp = ppw_gp[e - n_ev];
      if (gp < 0 || gp >= n_gpairs) {
        bad_index(pops[0].ctr, kBadEventSlot, gp);
        continue;
      }
      walker = ppw_slot[e - n_ev];
      p0 = gpair_local[gp];
    } else {
      gp = gp_c[e];
      if (gp < 0 || gp >= n_gpairs) {
        bad_index(pops[0].ctr, kBadEventSlot, gp);
        continue;
      }
      const PopDev& P = pops[gpair_pop[gp]];
      uint32_t pend_dec = 0xffffffffu;  // a pending chain event's recomputed decision
      pos0 = ev_pos[e];
      key = ev_key[e];
      sl = ev_c[e];
      if (win[e] && (dest[e] == kPendingTerm || dest[e] == kPendingChain)) {
        // the test where the previous round's chain stopped, with its
        // decision: the walker was rewritten by its own chain, so only its
        // death counts; a partner consumed in that round is no member now,
        // and the walk goes on after the test
        if (sl.x < 0 || sl.x >= P.cap || sl.y < 0 || sl.y >= P.cap) {
          bad_index(P.ctr, kBadEventSlot, sl.x < 0 || sl.x >= P.cap ? sl.x : sl.y);
          continue;
        }
        const int x = (int)key_idx(key), y = x == sl.x ? sl.y : sl.x;
        if (!P.alive[x]) continue;
        if (P.touched[y] == *P.gen_p - 1u || !P.alive[y]) {
          walker = x;
          p0 = (int)key_pair(key);
        } else if (dest[e] == kPendingChain) {
          pend_dec = chain_event_decision(P, key, sl, x, y, dec[e]);
          if (pend_dec == 0xffffffffu) continue;
        }
      } else if (win[e]) {
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
      dc = pend_dec != 0xffffffffu ? pend_dec : dec[e];
    }
    const int pop = gpair_pop[gp];
    const PopDev& P = pops[pop];
    int len = 0, head = -1;
    bool done = false;
    if (walker >= 0) {
      WalkOut w;
      walk<KT, T, FLAT>(P, walker, p0, pos0, &w);
      if (w.stop) add_target_op(P, pop, w.q, walker, op_pop, op_pair, op_slot, op_k, op_key, op_base + e, op_cap);
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
// carries its walk on from that event with the coagulated particle, one
// thread per chain, drawing the walk's tests on from where k_items stopped.
// The coagulated particle's volumes are summed per species over the events,
// then over the species, as k_apply_chain sums them, so its decisions are
// the apply's.  While the particle stays in the cell it walked, the walk goes
// on in place; a new cell's stretch starts at the event's pair and position.
// The next accepted test is the next event: an absorb extends the chain, any
// other decision ends the chain before it (the walk resumes there in the
// next round).  The chain's events go to the pool, the first one included;
// the item gets the chain's length and head, or length 0 (the first event
// alone) if the pool is full.
template <int KT, class T, bool FLAT>
__global__ void __launch_bounds__(128) k_chain(const PopDev* pops, const int* gpair_pop, const long long* n_items,
                                               const uint8_t* it_flag, const unsigned long long* it_key,
                                               const int2* it_c, const int* it_gp, const float* it_pos,
                                               const uint32_t* it_dec, const uint32_t* it_gused, ChainPool pool,
                                               int* it_len, int* it_head, uint8_t* it_done, int4* it_term) {
  long long n = *n_items;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    if (!it_flag[e] || it_len[e] != -1) continue;
    const PopDev& P = pops[gpair_pop[it_gp[e]]];
    unsigned long long key = it_key[e];
    const int x = (int)key_idx(key);
    int q = (int)key_pair(key);
    int2 sl = it_c[e];
    int y = sl.x == x ? sl.y : sl.x;
    uint32_t used;
    MergeDecision m1 = unpack_decision(it_dec[e], &used);
    bool rm_y1 = sl.x == x ? m1.rm2 : m1.rm1;
    it_len[e] = 0;
    if (x < 0 || x >= P.cap || y < 0 || y >= P.cap || q >= P.n_pairs) continue;
    ChainWriter cw;
    float pos = it_pos[e];
    if (!cw.append(pool, y, q | (rm_y1 ? kChainRemoves : 0), pos)) continue;
    uint32_t t_next = it_gused[e];
    long long n_tests = 0;
    bool done = false;
    const int ns = P.n_spec;
    double vcur[kMaxSpec];
    for (int sp = 0; sp < ns; sp++) vcur[sp] = P.vol[vol_at(P, x, sp)];
    int cls = P.pair[q].cc + 1;
    Stretch s;
    s.C = -1;
    for (;;) {
      // absorb y: the coagulated particle's volumes, radius, class, record
      for (int sp = 0; sp < ns; sp++) vcur[sp] = vcur[sp] + P.vol[vol_at(P, y, sp)];
      double s_v = 0.0, s_m = 0.0;
      for (int sp = 0; sp < ns; sp++) s_v = s_v + vcur[sp];
      for (int sp = 0; sp < ns; sp++) s_m = s_m + vcur[sp] * P.density[sp];
      const double vt = s_v, r = vol2rad(P.benv.frac, vt);
      const RecD qxd = make_rec_v(P, r, vt, s_m, cls);
      const RecF qxf = to_f32(qxd);
      const int C = cell_of(P, r, cls);
      if (C < 0 || cw.len >= kChainMaxLen) break;  // off the grid (reported by the apply) or long enough
      if (C != s.C) walk_stretch(P, C, q, pos, &s);
      int yy, qq;
      bool first;
      double ry, vty;
      int rw = walk_next<KT, T, FLAT>(P, x, s, t_next, qxd, qxf, true, &n_tests, &yy, &pos, &qq, &first, &ry,
                                      &vty);
      if (rw == 0) done = true;  // every later pair of the cell was walked
      if (rw != 1) break;
      const PairDesc d = P.pair_desc[qq];
      const PairState& S = P.pair[qq];
      unsigned long long k2 = make_key((uint32_t)qq, 1u, (uint32_t)x);
      Rng gm = make_rng(P, kStreamChain, (uint32_t)(cw.len + 1), (uint32_t)x);
      MergeDecision m = first ? merge_decide_v(P, gm, r, vt, ry, vty, d.c1, d.c2, S.cc)
                              : merge_decide_v(P, gm, ry, vty, r, vt, d.c1, d.c2, S.cc);
      bool rm_x = first ? m.rm1 : m.rm2, rm_y = first ? m.rm2 : m.rm1;
      // the chain ends before an event that is no absorb, or when the pool
      // is full; that event is pending for the next round (kPendingTerm)
      if (!(m.create && rm_x && m.new_group != 0) || !cw.append(pool, yy, qq | (rm_y ? kChainRemoves : 0), pos)) {
        if (m.new_group == 0) set_status(P.ctr, kErrTimeout);
        it_term[e] = make_int4(yy, qq | (first ? kTermFirst : 0), (int)pack_decision(m, gm.used()), __float_as_int(pos));
        break;
      }
      claim_slot(P, yy, claim_key(P, k2), rm_y);
      y = yy;
      q = qq;
      cls = S.cc + 1;
    }
    // a chain that ended at its first event is that event alone
    it_len[e] = cw.len > 1 ? cw.len : 0;
    it_head[e] = cw.head;
    it_done[e] = done ? 1 : 0;
    if (n_tests) {
      add_ll_warp(&P.ctr->tot_samp, (int)n_tests);
      add_ll_warp(&P.ctr->walk_tests, (int)n_tests);
    }
  }
}

// Apply the winning chains (win[e] == 2), one warp per chain: the first
// ev_app[e] events in order, each a coagulate (coagulation.F90:928-985) of
// the walking particle with the next partner, with the merge decision
// recomputed from the values and the stream the walk used.  One warp per
// chain of the round's list (chain_list, filled by k_resolve_set); a chain's entries
// are taken a pool chunk at a time (kBatch events):
//   1. lane k loads event k's partner (slot, pair, radius, scalar fields,
//      species volumes) into shared memory;
//   2. lane s runs species s's sum over the events (the walking particle's
//      volume plus the partners' in order), keeping the sum after each event;
//   3. lane k totals event k's sums over the species (the walk's order, so
//      the values and decisions are the walk's), takes the radius and cell,
//      and draws event k's merge decision from the particle before event k;
//   4. the events' scalar fields and components are merged in order (lanes
//      hold components), and removed partners are killed.
// The coagulated particle stays in the walking particle's slot.  dest[e],
// gp_c[e] and ev_pos[e] are set to where the particle walks on (dest -1 if
// its walk ran to the end).
struct ChainStage {
  int y, q, cell1, cc;
  int c1, c2;
  float pos;
  int pad;
  double ry, vty, ice_y;
  PScal s;
};
constexpr int kApplyBatch = kChainChunk - 1;

__global__ void __launch_bounds__(32) k_apply_chain(const PopDev* pops, const int* gpair_pop,
                                                    const long long* pop_pair_base, const int* chain_list,
                                                    const long long* n_chain, const unsigned long long* ev_key,
                                                    const int* ev_len, const int* ev_app, const int* ev_head,
                                                    const uint8_t* ev_done, ChainPool pool, int* gp_c, float* ev_pos,
                                                    int* dest_out, unsigned long long* ev_key_w, int2* ev_w,
                                                    uint32_t* dec_w, const int4* ev_term) {
  constexpr unsigned kFull = 0xffffffffu;
  constexpr int kBatch = kApplyBatch;
  __shared__ ChainStage stage[kBatch];
  __shared__ double pre[kBatch * kMaxSpec];  // [event][species]
  const long long n_ch = *n_chain;
  const int lane = threadIdx.x;
  for (long long ci = blockIdx.x; ci < n_ch; ci += gridDim.x) {
    {
      const long long e = chain_list[ci];
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
      const int w_ice = P.i_water - 1;  // -1: no water species
      uint32_t gen = *P.gen_p;
      // the walking particle: species (lane, lane + 32), scalars, components (lane)
      double v_lo = lane < ns ? P.vol[vol_at(P, x, lane)] : 0.0;
      double v_hi = lane + 32 < ns ? P.vol[vol_at(P, x, lane + 32)] : 0.0;
      double ice_cur = w_ice >= 0 ? P.vol[vol_at(P, x, w_ice)] : 0.0;
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
      int chunk = ev_head[e];
      int done_ev = 0, last_q = -1, dlive = 0;
      float last_pos = 0.f;
      bool stop = false;
      for (int base = 0; base < app && !stop; base += kBatch) {
        const int nbatch = app - base < kBatch ? app - base : kBatch;
        // 1. the chunk's partners, one lane each
        const bool chunk_ok = chunk >= 0 && (long long)chunk < pool.n_chunks;  // the same on every lane
        bool bad = !chunk_ok;
        if (chunk_ok && lane < nbatch) {
          size_t ix = (size_t)chunk * kChainChunk + lane;
          int y = pool.y[ix];
          int q = pool.q[ix] & kChainPairMask;
          bad = y < 0 || y >= P.cap || q >= P.n_pairs;
          if (!bad) {
            ChainStage& st = stage[lane];
            const PairDesc d = P.pair_desc[q];
            st.y = y;
            st.q = q;
            st.cell1 = d.b1 + nb * d.c1;
            st.c1 = d.c1;
            st.c2 = d.c2;
            st.cc = P.pair[q].cc;
            st.pos = pool.pos[ix];
            st.ry = P.rad[y];
            st.vty = P.vtot[y];
            st.ice_y = w_ice >= 0 ? P.vol[vol_at(P, y, w_ice)] : 0.0;
            load_scal(P, y, st.s);
            for (int sp = 0; sp < ns; sp++) pre[lane * kMaxSpec + sp] = P.vol[vol_at(P, y, sp)];
          }
        }
        // entries past the first bad one are not applied
        const unsigned bad_mask = __ballot_sync(kFull, bad && lane < nbatch);
        const int n_ok = bad_mask ? __ffs(bad_mask) - 1 : nbatch;
        if (chunk_ok) chunk = pool.y[(size_t)chunk * kChainChunk + kChainChunk - 1];
        __syncwarp();
        // 2. per species, the sums after each event
        const double v_lo0 = v_lo, v_hi0 = v_hi;
        for (int k = 0; k < n_ok; k++) {
          if (lane < ns) {
            v_lo = v_lo + pre[k * kMaxSpec + lane];
            pre[k * kMaxSpec + lane] = v_lo;
          }
          if (lane + 32 < ns) {
            v_hi = v_hi + pre[k * kMaxSpec + lane + 32];
            pre[k * kMaxSpec + lane + 32] = v_hi;
          }
        }
        __syncwarp();
        // 3. per event: total, radius, cell, merge decision
        double vt_k = 0.0, r_k = 0.0;
        int C_k = -1;
        if (lane < n_ok) {
          double s_v = 0.0;
          for (int sp = 0; sp < ns; sp++) s_v = s_v + pre[lane * kMaxSpec + sp];
          vt_k = s_v;
          r_k = vol2rad(P.benv.frac, vt_k);
          C_k = cell_of(P, r_k, stage[lane].cc + 1);
        }
        double r_b = __shfl_up_sync(kFull, r_k, 1), vt_b = __shfl_up_sync(kFull, vt_k, 1);
        int C_b = __shfl_up_sync(kFull, C_k, 1);
        if (lane == 0) {
          r_b = r;
          vt_b = vt;
          C_b = C;
        }
        bool ok = true, first_k = false, rm_y_k = false, lost_x_k = false, lost_y_k = false;
        int group_k = 0;
        uint32_t used_k = 0;
        if (lane < n_ok) {
          const ChainStage& st = stage[lane];
          first_k = C_b == st.cell1;
          const int i = base + lane;
          Rng g = i == 0 ? merge_rng(P, key1) : make_rng(P, kStreamChain, (uint32_t)(i + 1), (uint32_t)x);
          MergeDecision m = first_k ? merge_decide_v(P, g, r_b, vt_b, st.ry, st.vty, st.c1, st.c2, st.cc)
                                    : merge_decide_v(P, g, st.ry, st.vty, r_b, vt_b, st.c1, st.c2, st.cc);
          bool rm_x = first_k ? m.rm1 : m.rm2;
          rm_y_k = first_k ? m.rm2 : m.rm1;
          lost_x_k = first_k ? m.lost1 : m.lost2;
          bool lost_y = first_k ? m.lost2 : m.lost1;
          lost_y_k = rm_y_k && lost_y;
          ok = m.create && rm_x && m.new_group != 0 && !(lost_x_k && !(rm_y_k && !lost_y));
          group_k = m.new_group;
          used_k = g.used();
        }
        const unsigned bad_dec = __ballot_sync(kFull, lane < n_ok && !ok);
        const int n_app = bad_dec ? __ffs(bad_dec) - 1 : n_ok;
        if (bad_dec) {
          if (lane == 0) set_status(P.ctr, kErrAssert);  // the walk decided an absorb here
          stop = true;
        }
        // 4. scalar fields and components, in order
        int yc = 0;
        double yt = 0.0;
        if (n_app > 0 && lane < stage[0].s.ncomp && lane < kMaxComponent) {
          yc = P.csrc[comp_at(stage[0].y, lane)];
          yt = P.ctime[comp_at(stage[0].y, lane)];
        }
        for (int k = 0; k < n_app; k++) {
          const ChainStage& st = stage[k];
          // the next partner's components, loaded ahead
          int yc_n = 0;
          double yt_n = 0.0;
          if (k + 1 < n_app && lane < stage[k + 1].s.ncomp && lane < kMaxComponent) {
            yc_n = P.csrc[comp_at(stage[k + 1].y, lane)];
            yt_n = P.ctime[comp_at(stage[k + 1].y, lane)];
          }
          const bool first = __shfl_sync(kFull, first_k ? 1 : 0, k) != 0;
          const bool rm_y = __shfl_sync(kFull, rm_y_k ? 1 : 0, k) != 0;
          const bool lost_x = __shfl_sync(kFull, lost_x_k ? 1 : 0, k) != 0;
          const bool lost_y = __shfl_sync(kFull, lost_y_k ? 1 : 0, k) != 0;
          const int new_group = __shfl_sync(kFull, group_k, k);
          const uint32_t used = __shfl_sync(kFull, used_k, k);
          const PScal ys = st.s;
          const double ice_x = k == 0 ? ice_cur : (w_ice >= 0 ? pre[(k - 1) * kMaxSpec + w_ice] : 0.0);
          const double ice_y = st.ice_y;
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
            const int i = base + k;
            Rng g = i == 0 ? merge_rng(P, key1) : make_rng(P, kStreamChain, (uint32_t)(i + 1), (uint32_t)x);
            g.seek(used);
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
          // the removals of this event whose ID is lost (coagulate,
          // coagulation.F90:928-985): the walking particle's is always removed
          if (lane == 0) {
            if (lost_x) log_removal(P, cur.id, kInfoCoag, nm.id);
            if (lost_y) log_removal(P, ys.id, kInfoCoag, nm.id);
          }
          nm.grp = new_group;
          nm.cls = st.cc + 1;
          cc_ = lane < n_out ? (from_a ? xa : xb) : 0;
          ct_ = lane < n_out ? (from_a ? za : zb) : 0.0;
          if (rm_y) {
            if (lane == 0) {
              kill_slot(P, st.y);
              P.touched[st.y] = gen;
            }
            dlive--;
          }
          cur = nm;
          done_ev++;
          last_q = st.q;
          last_pos = st.pos;
          yc = yc_n;
          yt = yt_n;
        }
        // the particle after the batch's last applied event
        if (n_app > 0) {
          r = __shfl_sync(kFull, r_k, n_app - 1);
          vt = __shfl_sync(kFull, vt_k, n_app - 1);
          C = __shfl_sync(kFull, C_k, n_app - 1);
          v_lo = lane < ns ? pre[(n_app - 1) * kMaxSpec + lane] : 0.0;
          v_hi = lane + 32 < ns ? pre[(n_app - 1) * kMaxSpec + lane + 32] : 0.0;
          if (w_ice >= 0) ice_cur = pre[(n_app - 1) * kMaxSpec + w_ice];
        } else {
          v_lo = v_lo0;
          v_hi = v_hi0;
        }
        if (n_ok < nbatch && !stop) {
          if (lane == 0) bad_index(P.ctr, kBadEventSlot, -1);
          stop = true;
        }
        __syncwarp();  // the stage is read before the next chunk overwrites it
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
      const int4 t = ev_term[e];
      if (on_grid && done_ev == ev_len[e] && t.x >= 0) {
        // every event applied: the test where the chain stopped is pending
        const int tq = t.y & (kTermFirst - 1);
        const bool tfirst = (t.y & kTermFirst) != 0;
        ev_key_w[e] = make_key((uint32_t)tq, 1u, (uint32_t)x);
        ev_w[e] = tfirst ? make_int2(x, t.x) : make_int2(t.x, x);
        gp_c[e] = (int)(pop_pair_base[pop] + tq);
        ev_pos[e] = __int_as_float(t.w);
        dec_w[e] = (uint32_t)t.z;
        dest_out[e] = kPendingTerm;
      } else if (on_grid && !stop && done_ev < ev_len[e]) {
        // cut short where a partner's claim failed: that event is pending
        ChainReader rd(ev_head[e]);
        long long ix = -1;
        for (int i = 0; i <= done_ev; i++) ix = rd.next(pool);
        const int y = ix >= 0 ? pool.y[ix] : -1;
        const int q = ix >= 0 ? (pool.q[ix] & kChainPairMask) : -1;
        if (y >= 0 && y < P.cap && q >= 0 && q < P.n_pairs) {
          const PairDesc d = P.pair_desc[q];
          const bool first = C == d.b1 + nb * d.c1;
          ev_key_w[e] = make_key((uint32_t)q, 1u, (uint32_t)x);
          ev_w[e] = first ? make_int2(x, y) : make_int2(y, x);
          gp_c[e] = (int)(pop_pair_base[pop] + q);
          ev_pos[e] = pool.pos[ix];
          dec_w[e] = (uint32_t)done_ev;
          dest_out[e] = kPendingChain;
        } else {
          bad_index(P.ctr, kBadEventSlot, y);
          dest_out[e] = -1;
        }
      } else {
        // off the grid, or stopped by an error: no walk on
        dest_out[e] = (walk_done || !on_grid || stop) ? -1 : x;
        gp_c[e] = (int)(pop_pair_base[pop] + last_q);
        ev_pos[e] = last_pos;
      }
    }
    }
  }
}

// Walk rates after a round's sort: for every cell, the running sum over its
// pairs (loop order) of k_max * del_t * members of the pair's other cell;
// pairs on the per-particle path add nothing.  One block per cell, its
// threads over the cell's pairs, a block-wide scan in a fixed order.
// P.walk_stops: 1 when the population's round 0 has target operations (the
// step's later rounds then run from the host and take the operations that
// walks stop for); with 0, its per-particle pairs (whose target cells were
// all empty at the step's start) are walked at the per-set rate like any
// pair.
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
  const int stops = P.walk_stops;
  if (threadIdx.x == 0) carry = 0.0;
  __syncthreads();
  for (int base = lo; base < hi; base += blockDim.x) {
    int j = base + threadIdx.x;
    double lam = 0.0;
    if (j < hi) {
      int q = P.cp_list[j];
      const PairState& S = P.pair[q];
      PairDesc d = P.pair_desc[q];
      int cell1 = d.b1 + nb * d.c1, cell2 = d.b2 + nb * d.c2;
      int O = cell1 == c ? cell2 : cell1;
      int n_o = P.cell_count[O];
      P.cp_ent[j] = make_int4(q, O | (cell1 == c ? (1 << 30) : 0), P.cell_start[O], n_o);
      // per-set pairs, and per-particle pairs seen from their source cell: a
      // particle that arrives in the cell meets the other cell's members at
      // the per-set rate.  Seen from its target cell a per-particle pair is a
      // stop (no rate, cp_nstop): a particle that arrives there is one of
      // its targets, and its walk ends at the pair in a target operation
      if (!(stops && S.path == kPathParticle && c == S.bt + nb * S.ct)) {
        double l = S.k_max * P.del_t * (double)n_o;
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
  const double total = carry;
  if (threadIdx.x == 0) cum[hi - lo] = total;
  if (threadIdx.x == 0 && stops) {
    // per entry, the first stop at or after it (hi: none)
    int nxt = hi;
    for (int j = hi - 1; j >= lo; j--) {
      const PairState& S = P.pair[P.cp_list[j]];
      if (stops && S.path == kPathParticle && c == S.bt + nb * S.ct) nxt = j;
      P.cp_nstop[j] = nxt;
    }
  }
  // the bucket table: the last entry whose stretch starts at or before each
  // bucket's start (cum is visible to the block after the barrier above)
  if (threadIdx.x < kWalkTab) {
    double target = total * (double)threadIdx.x / (double)kWalkTab;
    int a = 0, b = hi - lo - 1;
    while (a < b) {
      int mid = (a + b + 1) >> 1;
      if (cum[mid] <= target) a = mid;
      else b = mid - 1;
    }
    P.cp_tab[c * kWalkTab + threadIdx.x] = lo + a;
  }
}

// ---------------------------------------------------------------------------
// Per-particle (accelerated) path, phase 1: run sample_source_particle and
// the target update of coag_target_with_source for one target, store the
// result, and claim the target and every removed source.
constexpr int kMaxCopies = 8;  // dup copies per target operation (the growth limit keeps them at 2 or less)

struct PPResult {
  int target, p;        // target slot, pair (local)
  int n_samp, n_coag;   // counted into tot_n_samp / tot_n_coag when the operation is applied
  int merged;           // n_coag > 0
  int n_copies;         // prob_round(old_nc / new_nc); 0 removes the target
  int n_rm;             // sources it removes: rm_pool[rm_off .. rm_off + n_rm)
  int nofit;            // its removals did not fit the pool (the host sizes it to fit): it loses
  int copy_group[kMaxCopies];
  long long rm_off;
  PMeta meta;           // new target metadata
};

template <int KT>
__device__ double pp_kernel(const PopDev& P, const RecD& qs, const RecD& qt, int cs, int ct) {
  const double* a = (const double*)&qs;
  const double* b = (const double*)&qt;
  return pair_kernel<KT, double, false>(P, a, b, cs, ct, ct, 0.0, P.coeff);
}

// The first draws of a target operation: the number of removal samples,
// which bounds the sources it can remove (sample_source_particle,
// coagulation.F90:397).  k_pp_count stores that bound per operation;
// its scan places every operation's removals in one pool, so an operation
// can remove any number of sources.  Returns -1 for an operation that
// draws nothing (void, dead target, empty source cell).
__device__ __forceinline__ int pp_remove_bound(const PopDev& P, int p, int t, int k, Rng* g_out, int* n_extra,
                                               double* prm_out) {
  if (t < 0 || t >= P.cap || !P.alive[t]) return -1;
  const PairState& S = P.pair[p];
  const GridDev& G = *P.grid;
  int nb = G.n_bin;
  int src_cell = S.bs + nb * S.cs;
  if (P.cell_count[src_cell] == 0) return -1;
  double nc_target = P.recd[t].nc;
  double nc_src_min = num_conc_at_radius<double>(P.w, S.cs, G.edges[S.bs]);
  double prm_max = nc_target / nc_src_min;
  if (!(prm_max <= 1.0)) return -2;
  Rng g = make_rng(P, kStreamPart, (uint32_t)p, (uint32_t)k);
  int n_remove = rand_poisson(g, prm_max * S.nspt);
  *n_extra = rand_poisson(g, (1.0 - prm_max) * S.nspt);
  *g_out = g;
  *prm_out = prm_max;
  return n_remove;
}

__global__ void k_pp_count(const PopDev* pops, const int* op_pop, const int* op_pair, const int* op_slot,
                           const int* op_k, const long long* n_ops, int* rm_n) {
  long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    const PopDev& P = pops[op_pop[q]];
    Rng g(0, 0, 0, 0);
    int n_extra = 0;
    double prm = 0.0;
    int n = pp_remove_bound(P, op_pair[q], op_slot[q], op_k[q], &g, &n_extra, &prm);
    rm_n[q] = n > 0 ? n : 0;
  }
}

template <int KT>
__global__ void k_pp_ops(const PopDev* pops, const int* op_pop, const int* op_pair,
                         const int* op_slot, const int* op_k, const unsigned long long* op_key,
                         const long long* n_ops, PPResult* res, double* res_vol, const long long* rm_off,
                         int* rm_pool, long long rm_cap) {
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
    R.nofit = 0;
    R.rm_off = rm_off[q];
    if (t < 0 || t >= P.cap || !P.alive[t]) continue;  // t = -1: a redo voided by k_build_redo
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
    if (R.rm_off + n_remove > rm_cap) {
      R.nofit = 1;  // no draws, no claims; the host sized the pool from the round's total, so a guard only
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
      // a source this operation removed already has left the bin in the
      // reference, whose later samples draw from the sources left
      // (coagulation.F90:428-430): draw again
      for (int r = 0; r < 64 && R.n_rm > 0 && P.claim[si] == claim_key(P, prio); r++) {
        ie = rand_int(g, n_src);
        e = src_start + ie - 1;
        si = P.list[e];
      }
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
            for (int z = 0; z < R.n_rm; z++) dup = dup || (rm_pool[R.rm_off + z] == si);
            if (!dup) {
              if (R.n_rm < n_remove) {  // at most one per removal sample: the pool holds n_remove
                rm_pool[R.rm_off + R.n_rm++] = si;
                atomicMin(&P.claim[si], claim_key(P, prio));
              } else {
                cap_fail(P.ctr, kCapRemovals);
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
    double rnew = vol2rad(P.benv.frac, vt);
    int cc = S.cc;
    nm.grp = rand_group(g, P.w, cc, rnew);
    nm.cls = cc + 1;
    int b = bin_find(nb, G.log_lo, G.log_hi, rnew);
    if (b < 1 || b > nb) set_status(P.ctr, kErrOutOfGrid);
    double new_nc = num_conc_at_radius<double>(P.w, cc, rnew);
    int n_copies = prob_round(g, old_nc / new_nc);
    if (n_copies > kMaxCopies) {
      cap_fail(P.ctr, kCapCopies);
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
                             const long long* n_ops, const PPResult* res, const int* rm_pool, uint8_t* win,
                             int* need_slot, int* need_id, int* lost) {
  long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    const PopDev& P = pops[op_pop[q]];
    const PPResult& R = res[q];
    unsigned long long prio = op_key[q];
    bool ok = !R.nofit;
    if (R.merged) ok = ok && holds_slot(P, R.target, claim_key(P, prio), true);
    for (int z = 0; z < R.n_rm; z++) ok = ok && holds_slot(P, rm_pool[R.rm_off + z], claim_key(P, prio), true);
    win[q] = ok ? 1 : 0;
    lost[q] = ok ? 0 : 1;
    int extra = (ok && R.merged && R.n_copies > 1) ? R.n_copies - 1 : 0;
    need_slot[q] = extra;
    need_id[q] = extra;
  }
}

// phase 2b: apply the winning target operations
// walker places of the round's operations, compacted in order
__global__ void k_walkers_span(const long long* n_ops, long long* n_places) { *n_places = *n_ops * kMaxCopies; }

__global__ void k_compact_walkers(const long long* n_places, const uint8_t* flag, const long long* off,
                                  const int* wk_slot, const int* wk_gp, int* ppw_slot, int* ppw_gp) {
  const long long n = *n_places;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (flag[i]) {
      ppw_slot[off[i]] = wk_slot[i];
      ppw_gp[off[i]] = wk_gp[i];
    }
}

__global__ void k_pp_apply(const PopDev* pops, const int* op_pop, const long long* n_ops,
                           const PPResult* res, const double* res_vol, const int* rm_pool, const uint8_t* win,
                           const long long* slot_rank, const long long* id_rank,
                           const int* slot_base, const long long* id_base, const long long* pop_pair_base,
                           const int* op_k, int* wk_slot, int* wk_gp, uint8_t* wk_flag) {
  // the walkers an operation makes (its target, then its copies) go to the
  // operation's own kMaxCopies places, compacted afterwards in operation
  // order, so that the next round's items do not depend on scheduling
  long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    for (int z = 0; z < kMaxCopies; z++) wk_flag[q * kMaxCopies + z] = 0;
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
      // sample_source_particle records each source it removes with the
      // target's ID (coagulation.F90:447-453)
      const int sz = rm_pool[R.rm_off + z];
      log_removal(P, P.id[sz], kInfoCoag, P.id[R.target]);
      kill_slot(P, sz);
      P.touched[sz] = gen;
      dlive--;
    }
    if (R.merged) {
      const double* v = res_vol + (size_t)q * P.n_spec;
      int t = R.target;
      P.touched[t] = gen;
      if (R.n_copies == 0) {
        log_removal(P, P.id[t], kInfoWeight, 0);  // aero_state_dup_particle (aero_state.F90:502-513)
        kill_slot(P, t);
        dlive--;
      } else {
        // the changed target and its copies take part in the rest of the
        // step: they walk from the end of this pair in the next round
        const int wgp = (int)(pop_pair_base[pop] + R.p);
        auto add_walker = [&](int slot, int z) {
          const long long k = q * kMaxCopies + z;
          wk_slot[k] = slot;
          wk_gp[k] = wgp;
          wk_flag[k] = 1;
        };
        store_particle(P, t, v, R.meta);
        refresh_slot(P, t);
        add_walker(t, 0);
        for (int z = 1; z < R.n_copies; z++) {
          int dest = slot_base[pop] + (int)slot_rank[q] + (z - 1);
          if (dest >= P.cap) {
            cap_fail(P.ctr, kCapCopySlot);
            break;
          }
          PMeta cm = R.meta;
          cm.grp = R.copy_group[z];
          cm.id = id_base[pop] + id_rank[q] + (z - 1);
          store_particle(P, dest, v, cm);
          refresh_slot(P, dest);
          P.touched[dest] = gen;
          add_walker(dest, z);
          dlive++;
        }
      }
    } else if ((op_k[q] & 0x40000000) && R.target >= 0 && R.target < P.cap && P.alive[R.target] &&
               P.touched[R.target] != gen) {
      // a walk that stopped here for this operation, which changed nothing,
      // goes on from the end of the pair: the reference's target stays in
      // its bin for the step's later pairs.  A target that an event of this
      // round rewrote walks on from that event instead (one walker per
      // particle: two would draw the same tests and make the same event)
      const long long k = q * kMaxCopies;
      wk_slot[k] = R.target;
      wk_gp[k] = (int)(pop_pair_base[pop] + R.p);
      wk_flag[k] = 1;
    }
    if (dlive) add_ll(&P.ctr->n_live, (long long)(dlive));
  }
}

}  // namespace pmc
