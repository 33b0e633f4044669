// pmc_coag.cu -- host orchestration and C ABI of the B200 coagulation step.
//
// The C ABI (include/pmc_coag_gpu.h) is the drop-in for mc_coag
// (coagulation.F90:43-96).  A context owns one or more particle
// populations resident in HBM; a step runs the rounds described in
// pmc_kernels.cuh over all populations at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <type_traits>

#include "../../include/pmc_coag_gpu.h"
#include "pmc_kernels.cuh"
#include "pmc_merge.cuh"
#include "pmc_replay.cuh"
#include "pmc_sample.cuh"

using namespace pmc;

namespace {

inline void note_launch();

// ---------------------------------------------------------------------------
// exclusive scan of n values into out[0..n] (out[n] = total): one
// single-pass launch with decoupled look-back, for up to kScanMaxJobs arrays
// of the same element type at once (blockIdx.y selects the array)
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kScanMaxJobs = 4;
constexpr int kScanSpinLimit = 1 << 20;  // bounded wait on a predecessor tile

// the element count is n, or *nd when nd is given (a count that only the
// device knows; n is then its upper bound)
__device__ __forceinline__ long long scan_n(long long n, const long long* nd) {
  if (!nd) return n;
  long long m = *nd;
  return m < n ? m : n;
}

__device__ long long block_excl_scan_ll(long long v, long long* total) {
  __shared__ long long ws[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  if (wid == 0) {
    long long s = lane < nw ? ws[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    ws[lane] = s;
  }
  __syncthreads();
  long long pre = (wid > 0 ? ws[wid - 1] : 0) + x - v;
  if (total) *total = ws[nw - 1];
  __syncthreads();
  return pre;
}

struct ScanJob {
  const void* in;
  long long* out;
  long long n_max;
  const long long* nd;
  long long* total_out;  // optional second copy of the total at a fixed address
};
struct ScanJobs {
  ScanJob j[kScanMaxJobs];
};

// tile status word: flag (2 bits: 1 aggregate, 2 inclusive prefix) | value
// (62 bits); 0 = not published.  The last block of a launch to finish
// clears the launch's words, so the array is all zero between launches and
// a launch can be replayed (CUDA graphs) without host bookkeeping.
__device__ __forceinline__ unsigned long long scan_word(unsigned flag, long long v) {
  return ((unsigned long long)flag << 62) | ((unsigned long long)v & ((1ULL << 62) - 1));
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_lb(ScanJobs jobs, unsigned long long* status,
                                                          int status_stride, unsigned* tile_ctr,
                                                          unsigned* done_ctr, unsigned long long* err) {
  const ScanJob J = jobs.j[blockIdx.y];
  __shared__ unsigned tile_sh;
  __shared__ long long carry_sh;
  unsigned long long* st = status + (size_t)blockIdx.y * status_stride;
  if (threadIdx.x == 0) {
    // tiles in the order blocks start, so a tile only waits on running blocks
    unsigned t = atomicAdd(&tile_ctr[blockIdx.y], 1u);
    if (t == gridDim.x - 1) tile_ctr[blockIdx.y] = 0;  // the last claimant re-arms the counter
    tile_sh = t;
  }
  __syncthreads();
  long long tile = tile_sh;
  long long n = scan_n(J.n_max, J.nd);
  long long nb = (n + kScanTile - 1) / kScanTile;
  if (n <= 0) {
    if (tile == 0 && threadIdx.x == 0) {
      J.out[0] = 0;
      if (J.total_out) *J.total_out = 0;
    }
  } else if (tile < nb) {
    const T* in = (const T*)J.in;
    long long base = tile * kScanTile + (long long)threadIdx.x * kScanItems;
    long long v[kScanItems];
    long long s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      long long i = base + k;
      v[k] = i < n ? (long long)in[i] : 0;
      s += v[k];
    }
    long long agg;
    long long pre = block_excl_scan_ll(s, &agg);
    if (threadIdx.x == 0) {
      long long excl = 0;
      if (tile == 0) {
        atomicExch(&st[0], scan_word(2u, agg));
      } else {
        atomicExch(&st[tile], scan_word(1u, agg));
        long long look = tile - 1;
        int spins = 0;
        while (look >= 0) {
          unsigned long long w = *(volatile unsigned long long*)&st[look];
          unsigned flag = (unsigned)(w >> 62);
          if (flag == 0) {
            if (++spins > kScanSpinLimit) {
              atomicAdd(err, 1ULL);
              break;
            }
            __nanosleep(32);
            continue;
          }
          excl += (long long)(w & ((1ULL << 62) - 1));
          if (flag == 2u) break;
          look--;
        }
        atomicExch(&st[tile], scan_word(2u, excl + agg));
      }
      carry_sh = excl;
    }
    __syncthreads();
    long long off = carry_sh + pre;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      long long i = base + k;
      if (i < n) J.out[i] = off;
      off += v[k];
    }
    if (tile == nb - 1 && threadIdx.x == 0) {
      J.out[n] = carry_sh + agg;
      if (J.total_out) *J.total_out = carry_sh + agg;
    }
  }
  // the last block of this job to finish clears the job's status words
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned d = atomicAdd(&done_ctr[blockIdx.y], 1u);
    if (d == gridDim.x - 1) {
      for (unsigned k = 0; k < gridDim.x; k++) st[k] = 0ULL;
      done_ctr[blockIdx.y] = 0;
      __threadfence();
    }
  }
}

// ---------------------------------------------------------------------------
// small helper kernels


// accepted samples of round 0 in sample order: event e gets its key (pair,
// sample), its two slots, its global pair and its position in the pair's
// test sequence ((s + 1) / n_samp: the part of the pair done after it)
__global__ void k_compact_flags(const uint8_t* flag, const long long* off, const long long* n_samples,
                                const int2* ev, const int* ev_gp, const int* gpair_local, const long long* work_off,
                                unsigned long long* ev_key, int2* ev_c, int* gp_c, float* ev_pos, int* ev_len,
                                int4* ev_term) {
  long long n = *n_samples;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (flag[i]) {
      long long e = off[i];
      int gp = ev_gp[i];
      long long s = i - work_off[gp], ns = work_off[gp + 1] - work_off[gp];
      ev_key[e] = make_key((uint32_t)gpair_local[gp], 0u, (uint32_t)s);
      ev_c[e] = ev[i];
      gp_c[e] = gp;
      ev_pos[e] = (float)((double)(s + 1) / (double)ns);
      ev_len[e] = 0;
      ev_term[e] = no_term();
    }
}

// the events a later round's items made, in item order
__global__ void k_compact_items(const uint8_t* it_flag, const long long* off, const long long* n_items,
                                const unsigned long long* it_key, const int2* it_c, const int* it_gp,
                                const float* it_pos, const int* it_len, const int* it_head, const uint8_t* it_done,
                                const uint32_t* it_dec, const int4* it_term, unsigned long long* ev_key, int2* ev_c,
                                int* gp_c, float* ev_pos, int* ev_len, int* ev_head, uint8_t* ev_done, uint32_t* dec,
                                int4* ev_term, const long long* grouped) {
  long long n = *n_items;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (it_flag[i]) {
      long long e = grouped ? grouped[i] : off[i];
      if (e < 0) continue;
      ev_key[e] = it_key[i];
      ev_c[e] = it_c[i];
      gp_c[e] = it_gp[i];
      ev_pos[e] = it_pos[i];
      ev_len[e] = it_len[i];
      ev_head[e] = it_head[i];
      ev_done[e] = it_done[i];
      dec[e] = it_dec[i];
      ev_term[e] = it_term[i];
    }
}

// target operations of round 0, in the reference's backwards target order
// (coagulation.F90:220-237)
__global__ void k_build_ops(const PopDev* pops, const int* gpair_pop, const int* gpair_local,
                            const long long* pp_off, int n_gpairs, int* op_pop, int* op_pair, int* op_slot,
                            int* op_k, unsigned long long* op_key) {
  int gp = blockIdx.x;
  if (gp >= n_gpairs) return;
  long long n = pp_off[gp + 1] - pp_off[gp];
  if (n == 0) return;
  int pop = gpair_pop[gp];
  const PopDev& P = pops[pop];
  int p = gpair_local[gp];
  const PairState& S = P.pair[p];
  int tcell = S.bt + P.grid->n_bin * S.ct;
  int start = P.cell_start[tcell];
  for (long long k = threadIdx.x; k < n; k += blockDim.x) {
    long long q = pp_off[gp] + k;
    op_pop[q] = pop;
    op_pair[q] = p;
    op_slot[q] = P.list[start + (int)(n - 1 - k)];
    op_k[q] = (int)k;
    op_key[q] = make_key((uint32_t)p, 0u, (uint32_t)k);
  }
}

// redo list of lost target operations (order of q kept); a redo keeps its
// place in the loop order (its key)
__global__ void k_build_redo(const PopDev* pops, const int* op_pop, const int* op_pair, const int* op_slot,
                             const int* op_k, const unsigned long long* op_key, const int* lost,
                             const long long* lost_off, const long long* n_ops, int* r_pop, int* r_pair, int* r_slot,
                             int* r_k, unsigned long long* r_key) {
  const long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q;
       q += (long long)gridDim.x * blockDim.x) {
    if (!lost[q]) continue;
    long long j = lost_off[q];
    const PopDev& P = pops[op_pop[q]];
    const int t = op_slot[q];
    r_pop[j] = op_pop[q];
    r_pair[j] = op_pair[q];
    // a target that an earlier operation or event of the round consumed
    // (removed or rewrote) walks on from there instead: its redo is void
    const bool consumed = t < 0 || t >= P.cap || !P.alive[t] || P.touched[t] == *P.gen_p;
    r_slot[j] = consumed ? -1 : t;
    r_k[j] = op_k[q] + (1 << 24);  // fresh random stream for the redo
    r_key[j] = op_key[q];
  }
}

// first event of population k (events are ordered by population)
__device__ long long first_event_of(int k, long long E, const int* ev_gp, const int* gpair_pop) {
  long long lo = 0, hi = E;
  while (lo < hi) {
    long long mid = (lo + hi) >> 1;
    if (gpair_pop[ev_gp[mid]] < k) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Per-population bases of the allocations of one round.  Events and target
// operations are ordered by population, so a global exclusive rank minus the
// count of earlier populations is the rank inside the population.  Per-set
// counts come from the rank scans at the population boundaries (and are
// stored in per_pop for the host); per-particle counts were summed into
// per_pop by k_count_per_pop.  The slot and ID counters of each population
// advance here by the round's allocations: the apply kernels read only the
// bases.  One block; populations in tiles of blockDim.x.
__global__ void k_alloc_bases(const PopDev* pops, int n_pop, const long long* n_events, const int* ev_gp,
                              const int* gpair_pop, int has_set, const long long* rank_slot_set,
                              const long long* rank_id_set, int* per_pop, int* set_slot_base,
                              long long* set_id_base, int* pp_slot_base, long long* pp_id_base) {
  long long carry[4] = {0, 0, 0, 0};
  long long E = has_set ? *n_events : 0;
  for (int base = 0; base < n_pop; base += blockDim.x) {
    int k = base + threadIdx.x;
    long long cnt[4] = {0, 0, 0, 0};
    if (k < n_pop) {
      if (E > 0) {
        long long e_lo = n_pop == 1 ? 0 : first_event_of(k, E, ev_gp, gpair_pop);
        long long e_hi = n_pop == 1 ? E : first_event_of(k + 1, E, ev_gp, gpair_pop);
        cnt[0] = rank_slot_set[e_hi] - rank_slot_set[e_lo];
        cnt[1] = rank_id_set[e_hi] - rank_id_set[e_lo];
      }
      per_pop[k] = (int)cnt[0];
      per_pop[n_pop + k] = (int)cnt[1];
      cnt[2] = per_pop[2 * n_pop + k];
      cnt[3] = per_pop[3 * n_pop + k];
    }
    long long pre[4], tot[4];
    for (int j = 0; j < 4; j++) pre[j] = block_excl_scan_ll(cnt[j], &tot[j]);
    if (k < n_pop) {
      PopCtr* c = pops[k].ctr;
      long long cs = carry[0] + pre[0], ci = carry[1] + pre[1], ps = carry[2] + pre[2], pi = carry[3] + pre[3];
      set_slot_base[k] = c->n_slots - (int)cs;
      set_id_base[k] = c->next_id - ci;
      pp_slot_base[k] = c->n_slots + (int)cnt[0] - (int)ps;
      pp_id_base[k] = c->next_id + cnt[1] - pi;
      c->n_slots += (int)(cnt[0] + cnt[2]);
      c->next_id += cnt[1] + cnt[3];
    }
    for (int j = 0; j < 4; j++) carry[j] += tot[j];
  }
}

// need[q] of target operation q summed per population (op_pop[q])
__global__ void k_count_per_pop(const int* need, const long long* n_items, const int* item_pop_of,
                                int* per_pop) {
  long long n = *n_items;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    if (!need[e]) continue;
    atomicAdd(&per_pop[item_pop_of[e]], need[e]);
  }
}

// particle upload: the caller's arrays were copied straight into slots
// 0..n-1 (same particle-major layout); fill the caches and the fields the
// caller did not give
__global__ void k_upload(PopDev P, int n, int have_grp, int have_cls, int have_id, int have_nprim,
                         long long id0, int* bad, unsigned long long* max_id) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    // the caller's groups and classes are checked here, on the device
    if (have_grp && (P.grp[i] < 1 || P.grp[i] > P.n_group)) atomicOr(bad, 1);
    if (have_cls && (P.cls[i] < 1 || P.cls[i] > P.n_class)) atomicOr(bad, 2);
    if (have_id && P.id[i] >= 0) atomicMax(max_id, (unsigned long long)P.id[i]);
    P.changed[i] = 0;
    double vt = 0.0, ms = 0.0;
    for (int s = 0; s < P.n_spec; s++) vt = vt + P.vol[vol_at(P, i, s)];
    for (int s = 0; s < P.n_spec; s++) ms = ms + P.vol[vol_at(P, i, s)] * P.density[s];
    P.vtot[i] = vt;
    P.mass[i] = ms;
    if (!have_grp) P.grp[i] = 1;
    if (!have_cls) P.cls[i] = 1;
    if (!have_id) P.id[i] = id0 + i;
    if (!have_nprim) P.nprim[i] = 1;
    P.ncomp[i] = 1;
    P.csrc[comp_at(i, 0)] = 1;
    P.ctime[comp_at(i, 0)] = 0.0;
    P.lct[i] = 0.0;
    P.gct[i] = 0.0;
    P.imf[i] = 0.0;
    P.den_ice[i] = __longlong_as_double(0x7ff8000000000000LL);
    P.phi[i] = __longlong_as_double(0x7ff8000000000000LL);
    P.hyst[i] = 0;
    P.frozen[i] = 0;
    P.alive[i] = 1;
    P.cell[i] = -1;  // set by the first refresh after the grid decision
  }
}

__global__ void k_download(PopDev P, const long long* live_off, int n_slots, double* vol_pm,
                           int* grp, int* cls, long long* id, int* nprim, int* ncomp, int* csrc,
                           double* ctime) {
  // only the fields asked for (non-null outputs) are gathered
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_slots; i += gridDim.x * blockDim.x) {
    if (!P.alive[i]) continue;
    long long j = live_off[i];
    if (vol_pm)
      for (int s = 0; s < P.n_spec; s++) vol_pm[j * P.n_spec + s] = P.vol[vol_at(P, i, s)];
    if (grp) grp[j] = P.grp[i];
    if (cls) cls[j] = P.cls[i];
    if (id) id[j] = P.id[i];
    if (nprim) nprim[j] = P.nprim[i];
    if (ncomp) ncomp[j] = P.ncomp[i];
    if (csrc)
      for (int k = 0; k < kMaxComponent; k++)
        csrc[j * kMaxComponent + k] = k < P.ncomp[i] ? P.csrc[comp_at(i, k)] : 0;
    if (ctime)
      for (int k = 0; k < kMaxComponent; k++)
        ctime[j * kMaxComponent + k] = k < P.ncomp[i] ? P.ctime[comp_at(i, k)] : 0.0;
  }
}

// Changed slots of [lo, hi) packed for the host copy, one record of
// rec_bytes = kSyncHead + 8 n_spec bytes rounded up to a multiple of 16:
// {slot, alive, group, class, n_primary, 0, id (8 bytes)} then the species
// volumes.  Each warp takes 32 slots and reserves places for its changed
// ones with one atomic; it assembles their records in shared memory (one
// lane per species for the volumes) and writes them out as consecutive
// 16-byte words, so that a write into host memory goes over the bus in full
// lines.  Record order is arbitrary (the host scatters by slot).  Clears the
// changed flags.
constexpr int kSyncHead = 32;
__global__ void k_pack_changed(PopDev P, int lo, int hi, unsigned long long* count, unsigned char* out,
                               int rec_bytes) {
  extern __shared__ int4 pack_stage[];  // [warps of the block][32 records]
  const int lane = threadIdx.x & 31;
  unsigned char* my = (unsigned char*)pack_stage + (size_t)(threadIdx.x >> 5) * 32 * rec_bytes;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int base = lo + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < hi; base += warps * 32) {
    const int i = base + lane;
    const bool ch = i < hi && P.changed[i];
    const unsigned m = __ballot_sync(0xffffffffu, ch);
    if (!m) continue;
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(count, (unsigned long long)__popc(m));
    b = __shfl_sync(0xffffffffu, b, 0);
    if (ch) {
      unsigned char* r = my + (size_t)__popc(m & ((1u << lane) - 1u)) * rec_bytes;
      const int a = P.alive[i];
      *(int4*)r = make_int4(i, a, a ? P.grp[i] : 0, a ? P.cls[i] : 0);
      *(int2*)(r + 16) = make_int2(a ? P.nprim[i] : 0, 0);
      *(long long*)(r + 24) = a ? P.id[i] : 0;
      P.changed[i] = 0;
    }
    for (unsigned mm = m; mm; mm &= mm - 1) {
      const int src = __ffs(mm) - 1;
      const int si = base + src;
      if (!P.alive[si]) continue;
      double* v = (double*)(my + (size_t)__popc(m & ((1u << src) - 1u)) * rec_bytes + kSyncHead);
      for (int sp = lane; sp < P.n_spec; sp += 32) v[sp] = P.vol[vol_at(P, si, sp)];
    }
    __syncwarp();
    const int n16 = __popc(m) * (rec_bytes / 16);
    int4* d = (int4*)(out + (size_t)b * rec_bytes);
    const int4* sm = (const int4*)my;
    for (int k = lane; k < n16; k += 32) d[k] = sm[k];
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// aero_state_rebalance (aero_state.F90:1722-1852) on the device

// live particles per (group, class): counts[(g-1) + n_group*(c-1)]
__global__ void k_count_group_class(PopDev P, int* counts) {
  int n = P.ctr->n_slots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!P.alive[i]) continue;
    int g = P.grp[i], c = P.cls[i];
    if (g >= 1 && g <= P.n_group && c >= 1 && c <= P.n_class) atomicAdd(&counts[(g - 1) + P.n_group * (c - 1)], 1);
  }
}

// members of (g, c) among slots 0..n-1
__global__ void k_flag_group_class(PopDev P, int n, int g, int c, uint8_t* flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flag[i] = (P.alive[i] && P.grp[i] == g && P.cls[i] == c) ? 1 : 0;
}

// aero_state_double: member j (in slot order) is copied to slot n + j with
// ID id0 + j (aero_particle_new_id); every field is copied, caches included
__global__ void k_double(PopDev P, int n, const uint8_t* flag, const long long* off, long long id0) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    int d = n + (int)off[i];
    if (d >= P.cap) {
      cap_fail(P.ctr, kCapDupSlot);
      continue;
    }
    copy_particle(P, i, d, id0 + off[i]);
  }
}

// aero_state_halve: each member removed with probability 1/2; the draw of
// slot i is keyed by the population's seed and step, the rebalance call and i
__global__ void k_halve(PopDev P, int g, int c, uint32_t call) {
  int n = P.ctr->n_slots;
  int removed = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!(P.alive[i] && P.grp[i] == g && P.cls[i] == c)) continue;
    U4 r = philox4x32_10(U4{P.step, (call << 4) | kStreamHalve, (uint32_t)i, 0u}, (uint32_t)P.seed,
                         (uint32_t)(P.seed >> 32));
    if (u53(r.x, r.y) < 0.5) {
      log_removal(P, P.id[i], kInfoHalved, 0);  // aero_state_halve records it (aero_state.F90:1768-1781)
      kill_slot(P, i);
      removed++;
    }
  }
  if (removed) add_ll(&P.ctr->n_live, -(long long)removed);
}

// ---------------------------------------------------------------------------
// size distributions (extract_aero_size.F90:132-138 with
// bin_grid_histogram_1d, bin_grid.F90:225-248): diameters on a log grid of
// n_bin bins from d_min to d_max, each particle weighted by its number
// concentration (aero_state_num_concs), per unit log diameter.  out holds
// n_bin number values, then n_bin x n_spec species masses (kg m^-3).
// Per-block partial sums in shared memory, then one atomic per bin and block.
__global__ void k_size_dist(PopDev P, int n_bin, double log_lo, double log_hi, double inv_width, double* out) {
  extern __shared__ double hs[];  // [n_bin * (1 + n_spec)]
  int nv = n_bin * (1 + P.n_spec);
  for (int k = threadIdx.x; k < nv; k += blockDim.x) hs[k] = 0.0;
  __syncthreads();
  int n = P.ctr->n_slots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!P.alive[i]) continue;
    double r = vol2rad(P.benv.frac, P.vtot[i]);  // aero_particle_radius (fractal_vol2rad)
    int b = bin_find(n_bin, log_lo, log_hi, 2.0 * r);
    if (b < 1 || b > n_bin) continue;
    double nc = num_conc_at_radius<double>(P.w, P.cls[i] - 1, r) * inv_width;
    atomicAdd(&hs[b - 1], nc);
    for (int s = 0; s < P.n_spec; s++)
      atomicAdd(&hs[n_bin + (b - 1) * P.n_spec + s], nc * P.vol[vol_at(P, i, s)] * P.density[s]);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nv; k += blockDim.x)
    if (hs[k] != 0.0) atomicAdd(&out[k], hs[k]);
}

// move live slots of src into dst compactly (relayout)
__global__ void k_relayout(PopDev S, PopDev D, const long long* live_off, int n_slots,
                           int compact) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_slots; i += gridDim.x * blockDim.x) {
    if (compact && !S.alive[i]) continue;
    int j = compact ? (int)live_off[i] : i;
    for (int s = 0; s < S.n_spec; s++) D.vol[vol_at(D, j, s)] = S.vol[vol_at(S, i, s)];
    D.vtot[j] = S.vtot[i];
    D.mass[j] = S.mass[i];
    D.rad[j] = S.rad[i];
    D.grp[j] = S.grp[i];
    D.cls[j] = S.cls[i];
    D.id[j] = S.id[i];
    D.nprim[j] = S.nprim[i];
    D.ncomp[j] = S.ncomp[i];
    for (int k = 0; k < S.ncomp[i]; k++) {
      D.csrc[comp_at(j, k)] = S.csrc[comp_at(i, k)];
      D.ctime[comp_at(j, k)] = S.ctime[comp_at(i, k)];
    }
    D.lct[j] = S.lct[i];
    D.gct[j] = S.gct[i];
    D.imf[j] = S.imf[i];
    D.den_ice[j] = S.den_ice[i];
    D.phi[j] = S.phi[i];
    D.hyst[j] = S.hyst[i];
    D.frozen[j] = S.frozen[i];
    D.alive[j] = S.alive[i];
    D.changed[j] = S.changed[i];
    D.cell[j] = S.cell[i];
    D.claim[j] = S.claim[i];
    D.rclaim[j] = S.rclaim[i];
    D.touched[j] = S.touched[i];
    D.recd[j] = S.recd[i];
    D.recf[j] = S.recf[i];
  }
  // growth keeps slot numbers, so the current cell list (positions below
  // n_slots) stays valid and is carried over; compaction renumbers slots
  // and the next sort rebuilds the list
  if (!compact)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_slots; i += gridDim.x * blockDim.x)
      D.list[i] = S.list[i];
}

__global__ void k_eval_kernel(PopDev P, int n, const double* v1, const int* c1, const double* v2,
                              const int* c2, const int* cij, double* out, int precision) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // records of the two particles, built as the sort pass builds them
  double vt1 = 0.0, vt2 = 0.0, m1 = 0.0, m2 = 0.0;
  for (int s = 0; s < P.n_spec; s++) {
    vt1 = vt1 + v1[(size_t)i * P.n_spec + s];
    vt2 = vt2 + v2[(size_t)i * P.n_spec + s];
  }
  for (int s = 0; s < P.n_spec; s++) {
    m1 = m1 + v1[(size_t)i * P.n_spec + s] * P.density[s];
    m2 = m2 + v2[(size_t)i * P.n_spec + s] * P.density[s];
  }
  RecD q[2];
  double vt[2] = {vt1, vt2}, ms[2] = {m1, m2};
  int cl[2] = {c1[i] - 1, c2[i] - 1};
  for (int k = 0; k < 2; k++) q[k] = make_rec_v(P, vol2rad(P.benv.frac, vt[k]), vt[k], ms[k], cl[k] + 1);
  int cc = cij[i] - 1;
  double k;
  if (precision == 0) {
    const double* a = (const double*)&q[0];
    const double* b = (const double*)&q[1];
    switch (P.kernel_type) {
      case kKernelAdditive: k = pair_kernel<kKernelAdditive, double, false>(P, a, b, cl[0], cl[1], cc, 0.0, P.coeff); break;
      case kKernelConstant: k = pair_kernel<kKernelConstant, double, false>(P, a, b, cl[0], cl[1], cc, 0.0, P.coeff); break;
      case kKernelBrown: k = pair_kernel<kKernelBrown, double, false>(P, a, b, cl[0], cl[1], cc, 0.0, P.coeff); break;
      case kKernelSedi: k = pair_kernel<kKernelSedi, double, false>(P, a, b, cl[0], cl[1], cc, 0.0, P.coeff); break;
      case kKernelBrownFree: k = pair_kernel<kKernelBrownFree, double, false>(P, a, b, cl[0], cl[1], cc, 0.0, P.coeff); break;
      case kKernelBrownCont: k = pair_kernel<kKernelBrownCont, double, false>(P, a, b, cl[0], cl[1], cc, 0.0, P.coeff); break;
      default: k = 0.0;
    }
  } else {
    float a[6], b[6];
    const double* qa = (const double*)&q[0];
    const double* qb = (const double*)&q[1];
    for (int j = 0; j < 6; j++) {
      a[j] = (float)qa[j];
      b[j] = (float)qb[j];
    }
    float kf;
    switch (P.kernel_type) {
      case kKernelAdditive: kf = pair_kernel<kKernelAdditive, float, false>(P, a, b, cl[0], cl[1], cc, 0.f, (float)P.coeff); break;
      case kKernelConstant: kf = pair_kernel<kKernelConstant, float, false>(P, a, b, cl[0], cl[1], cc, 0.f, (float)P.coeff); break;
      case kKernelBrown: kf = pair_kernel<kKernelBrown, float, false>(P, a, b, cl[0], cl[1], cc, 0.f, (float)P.coeff); break;
      case kKernelSedi: kf = pair_kernel<kKernelSedi, float, false>(P, a, b, cl[0], cl[1], cc, 0.f, (float)P.coeff); break;
      case kKernelBrownFree: kf = pair_kernel<kKernelBrownFree, float, false>(P, a, b, cl[0], cl[1], cc, 0.f, (float)P.coeff); break;
      case kKernelBrownCont: kf = pair_kernel<kKernelBrownCont, float, false>(P, a, b, cl[0], cl[1], cc, 0.f, (float)P.coeff); break;
      default: kf = 0.f;
    }
    k = kf;
  }
  out[i] = k;
}

// ---------------------------------------------------------------------------
// host side

#define CK(x)                                                          \
  do {                                                                 \
    cudaError_t e_ = (x);                                              \
    if (e_ != cudaSuccess) {                                           \
      snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", #x, \
               cudaGetErrorString(e_), __FILE__, __LINE__);            \
      throw Fail(PMC_ERR_CUDA);                                        \
    }                                                                  \
  } while (0)

char g_last_error[512];
char g_last_assert[256];  // site and index of the last failed device bounds check
char g_last_capacity[256];  // which limit the last PMC_ERR_CAPACITY hit
[[noreturn]] void cap_throw(const char* why);
// kernel launches issued by this library (for the benchmark's launch count)
long long g_launches = 0;
inline void note_launch() { ++g_launches; }

struct Fail {
  int code;
  explicit Fail(int c) : code(c) {}
};

void cap_throw(const char* why) {
  cudaGetLastError();  // a failed allocation leaves an error behind
  snprintf(g_last_capacity, sizeof(g_last_capacity), "capacity exceeded: %s", why);
  throw Fail(PMC_ERR_CAPACITY);
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void reserve(size_t m) {
    if (m <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    // geometric growth: sizes that creep up step by step (slot counts,
    // sample counts) reallocate rarely
    size_t want = std::max<size_t>(std::max<size_t>(m, n + n / 2), 1024);
    n = 0;
    if (cudaMalloc(&p, want * sizeof(T)) != cudaSuccess) {
      p = nullptr;
      cap_throw("device memory: an allocation failed");
    }
    n = want;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// page-locked host staging (cudaHostAlloc), grown on demand
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void reserve(size_t b) {
    if (b <= bytes) return;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    size_t want = std::max<size_t>(b + b / 4, 1 << 20);
    if (cudaHostAlloc(&p, want, cudaHostAllocDefault) != cudaSuccess) {
      p = nullptr;
      cap_throw("page-locked host memory: an allocation failed");
    }
    bytes = want;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
  }
};

// page-locked host memory that the device writes directly (mapped into the
// device's address space), grown on demand
struct MappedBuf {
  void* p = nullptr;    // host address
  void* dev = nullptr;  // device address of the same memory
  size_t bytes = 0;
  void reserve(size_t b) {
    if (b <= bytes) return;
    release();
    size_t want = std::max<size_t>(b + b / 4, 1 << 20);
    if (cudaHostAlloc(&p, want, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&dev, p, 0) != cudaSuccess) {
      cudaGetLastError();
      release();
      cap_throw("mapped host memory: an allocation failed");
    }
    bytes = want;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = dev = nullptr;
    bytes = 0;
  }
};

// Persistent host workers for the scatter of pmc_coag_gpu_sync_host: run(n,
// f) calls f(q, n) for q = 0..n-1 on n threads (the caller's among them) and
// returns when all are done.
class HostPool {
 public:
  ~HostPool() {
    {
      std::lock_guard<std::mutex> l(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  void run(int n, const std::function<void(int, int)>& f) {
    if (n <= 1) {
      f(0, 1);
      return;
    }
    while ((int)th_.size() < n - 1) {
      int q = (int)th_.size() + 1;
      th_.emplace_back([this, q] { loop(q); });
    }
    {
      std::lock_guard<std::mutex> l(mu_);
      job_ = &f;
      n_ = n;
      left_ = n - 1;
      gen_++;
    }
    cv_.notify_all();
    f(0, n);
    std::unique_lock<std::mutex> l(mu_);
    done_.wait(l, [this] { return left_ == 0; });
    job_ = nullptr;
  }

 private:
  void loop(int q) {
    unsigned long long seen = 0;
    for (;;) {
      const std::function<void(int, int)>* f;
      int n;
      {
        std::unique_lock<std::mutex> l(mu_);
        cv_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        f = job_;
        n = n_;
      }
      if (q < n) (*f)(q, n);
      std::lock_guard<std::mutex> l(mu_);
      if (q < n && --left_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int, int)>* job_ = nullptr;
  int n_ = 0, left_ = 0;
  unsigned long long gen_ = 0;
  bool stop_ = false;
};

struct PopHost {
  PopDev h{};
  bool valid_sort = false;
  int n_bin = 0;
  std::vector<double> edges, centers;
  std::vector<PairDesc> pair_desc;
  // owned allocations (freed on relayout / destroy)
  std::vector<void*> slot_allocs;
  std::vector<void*> sort_allocs;
  std::vector<void*> fixed_allocs;
  uint64_t seed = 1;
  uint32_t step = 0;
  int kmax_kt = 0;  // kernel type of the current k_max table
  bool own_w = false;  // weights set for this population alone
  // host copy kept slot by slot (pmc_coag_gpu_sync_host): refreshed in full
  // after an upload or a compaction, else by the slots written since
  bool mirror_full = true;
  int mirror_slots = 0;
  uint32_t rebalance_calls = 0;  // halving draws: one stream per call
  uint32_t sample_calls = 0;     // initial-condition samples: one stream per call
  Weights w{};
  int chunk_hist_cap = 0;
  // per-slot radius/bin/record caches are valid for this grid, kernel,
  // environment and weights
  bool caches_valid = false;
  int key_kt = 0, key_wver = -1;
  int wver = 0;  // bumped when this population's weights change
  double key_temp = 0, key_press = 0, key_coeff = 0;
  long long rm_count = 0;  // removal records on the device at the last counter read
};

// Launch shapes of the step that the autotuner chooses: threads per block
// at five launch sites.  Every kernel there walks its work with a
// grid-stride loop and keeps no per-block state, every draw is keyed by
// index and every counter is a sum, so the particles do not depend on these
// shapes, and tuning runs on the caller's own steps.
enum TuneSite : int { kTuneTest, kTuneResolve, kTuneItems, kTuneChain, kTuneApply, kTuneSites };
constexpr int kTuneCands = 3;
// candidates per site (within each kernel's __launch_bounds__)
constexpr int kTuneCand[kTuneSites][kTuneCands] = {
    {64, 128, 256},  // k_test: one pair test per thread
    {64, 128, 256},  // k_decide and k_resolve_set: one event per thread
    {64, 128, 256},  // k_items: one walk per thread
    {32, 64, 128},   // k_chain: one chain per thread
    {64, 128, 256},  // k_apply_move and k_apply_set: one event per thread
};
constexpr int kTuneReps = 3;  // steps per candidate
struct Tune {
  int threads[kTuneSites] = {256, 256, 256, 128, 256};
};
// Coordinate search, one site at a time.  While it runs the later rounds
// are launched from the host loop (the same particles as the graph), so
// that every launch of the site being searched can be bracketed by CUDA
// events.  A candidate's score is the device time of the site's launches
// over its kTuneReps steps divided by those steps' pair tests: the site's
// cost per unit of work, which does not drift with the state as the whole
// step's time does.  The site keeps its best candidate before the next site
// is searched.
struct Tuner {
  bool on = false;
  int site = 0, cand = 0, rep = 0, best = 0;
  float best_ms = 0.f;           // best score (ms per million pair tests)
  double cand_ms = 0.0;          // the candidate's site time so far (ms)
  long long cand_tests = 0;      // and its steps' pair tests
  float site_ms[kTuneSites][kTuneCands] = {};
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;  // this step's launches of the site
  std::vector<cudaEvent_t> spare;
};

struct Ctx {
  int n_pop = 1, n_spec = 1, n_group = 1, n_class = 1, i_water = 0;
  std::vector<double> density;
  Weights w{};
  int wver = 0;  // bumped on every weight change
  int mode = PMC_MODE_FP64;
  std::vector<PopHost> pops;
  PopDev* d_pops = nullptr;
  PopCtr* d_ctrs = nullptr;  // one counter block per population
  uint32_t* d_round = nullptr;  // [round of the current step, claim generation], read by the kernels
  uint32_t claim_gen = 0;
  bool dirty = true;            // host PopDev copies changed since the last push
  std::vector<PopCtr> h_ctrs;
  cudaStream_t stream = nullptr;
  int max_rounds = 200;  // below 256: the round is 8 bits of the random streams' counters
  int n_sm = 148;        // multiprocessors of the device
  // later rounds as a CUDA graph
  bool use_graph = true;
  cudaStream_t cap_stream = nullptr;  // capture stream
  cudaGraph_t rg_graph = nullptr;
  cudaGraphExec_t rg_exec = nullptr;
  std::vector<long long> rg_key;
  std::vector<long long> rg_seen;  // the key of the previous step's later rounds
  long long rg_nodes = 0, rg_builds = 0;
  DevBuf<long long> graph_stats;
  Tune tune;
  Tuner tuner;
  // removal pool of the round's target operations
  DevBuf<int> pp_rm_n, pp_rm_pool;
  // a batched round's lists grouped by population (group_by_pop)
  DevBuf<int> grp_hist, item_pop, g_pop, g_pair, g_slot, g_k;
  DevBuf<long long> grp_off, grp_dest;
  // walkers of the round's operations, one place per operation and copy
  DevBuf<int> wk_slot, wk_gp;
  DevBuf<uint8_t> wk_flag;
  DevBuf<long long> wk_off;
  DevBuf<unsigned long long> g_key;
  DevBuf<long long> pp_rm_off, pp_rm_tot;
  // initial-condition sampler: staging of the modes, copy counts, radix select
  DevBuf<double> sample_buf;
  DevBuf<int> dup_n;
  DevBuf<unsigned char> select_buf;
  size_t sort_smem = 0;  // dynamic shared memory the sort grid was sized for
  int sort_blocks = 0;   // co-resident sort blocks at that size
  // per-round buffers
  DevBuf<int> gpair_pop, gpair_local;
  DevBuf<long long> pop_pair_base;
  DevBuf<long long> nwork_set, nwork_pp, work_off, pp_off;
  DevBuf<uint8_t> flag, win_set, win_pp;
  DevBuf<uint32_t> dec_set;  // merge decision of each event (drawn when the event is formed)
  DevBuf<int> ev_gp, gp_c;   // global pair of each accepted sample / event
  DevBuf<int2> ev_c;         // slots of each event
  DevBuf<unsigned long long> ev_key;  // key of each event (make_key)
  DevBuf<float> ev_pos;      // position of each event in its pair's test sequence
  DevBuf<int> ev_dest;       // slot of the particle each event made (-1: none)
  DevBuf<int> ev_len, ev_head, ev_app;  // chains: events, first chunk, events applied
  DevBuf<uint8_t> ev_done;   // chains: the walk ran to the end
  DevBuf<int> chain_list;    // the round's winning chains (round_dev[4] of them)
  DevBuf<double2> ice_set;   // water volumes of the sources of each event
  DevBuf<int2> ev;
  DevBuf<long long> flag_off;
  // a later round's items (one per event of the round before) and what they made
  DevBuf<uint8_t> it_flag, it_done;
  DevBuf<unsigned long long> it_key;
  DevBuf<int2> it_c;
  DevBuf<int> it_gp, it_len, it_head;
  DevBuf<float> it_pos;
  DevBuf<uint32_t> it_dec, it_gused;
  DevBuf<int4> it_term, ev_term;  // pending tests where chains stopped (kPendingTerm)
  // walkers made by target operations (slot, global pair), read by the next
  // round's k_items; their count is round_dev[5]
  DevBuf<int> ppw_slot, ppw_gp;      // written by this round's k_pp_apply
  DevBuf<int> ppw_slot_in, ppw_gp_in;  // read by this round's k_items (the round before's)
  long long ppw_cap = 0;
  long long op_cap = 0;   // room in the target-operation arrays this round
  bool pp_step = false;   // the step has target operations (per-particle path)
  DevBuf<long long> it_off;
  // chain events of a round (ChainPool), in chunks
  DevBuf<int> ch_y, ch_q;
  DevBuf<float> ch_pos;
  long long ch_chunks = 0;
  DevBuf<int> need_slot_set, need_id_set, need_slot_pp, need_id_pp, lost_pp;
  DevBuf<long long> rank_slot_set, rank_id_set, rank_slot_pp, rank_id_pp, lost_off;
  DevBuf<int> op_pop, op_pair, op_slot, op_k, r_pop, r_pair, r_slot, r_k;
  DevBuf<unsigned long long> op_key, r_key;
  DevBuf<PPResult> pp_res;
  DevBuf<double> pp_vol;
  DevBuf<int> per_pop_i;  // 4 x n_pop counters
  DevBuf<int> slot_base_set, slot_base_pp;
  DevBuf<long long> id_base_set, id_base_pp;
  DevBuf<unsigned long long> scan_status;  // look-back tile words
  size_t scan_status_n = 0;                // words cleared so far
  DevBuf<unsigned> scan_ctr;               // per-job tile and finished-block counters (re-armed by the kernel)
  DevBuf<unsigned long long> scan_err;     // look-backs that gave up
  DevBuf<long long> n_dev;  // device scalars
  // staging for upload / download (shared by all populations; every call
  // synchronises before it returns)
  DevBuf<double> st_d;
  DevBuf<int> st_i;
  DevBuf<long long> st_l;
  PinnedBuf pin;  // host staging of the changed slots
  MappedBuf map;  // packed changed slots, written by the device into host memory
  cudaEvent_t sync_ev[4] = {nullptr, nullptr, nullptr, nullptr};  // chunks of a host sync
  DevBuf<unsigned long long> st_cnt;        // their count
  std::unique_ptr<HostPool> pool;           // scatter workers
  long long h_total = 0;
  // stats of the last step
  long long last_redraws = 0, last_rounds = 0, last_kmax_warn = 0, exact_tests = 0;
  long long last_set_losers = 0, last_pp_lost = 0, last_events = 0, last_ops = 0;
  // optional per-kernel timing with CUDA events on the library's stream:
  // 0 pair tests, 1 sorts (k_sort_all), 2 later-round graph launches,
  // 3 whole steps
  bool prof = false;
  struct ProfPair {
    int id;
    long long units;
    cudaEvent_t e0, e1;
  };
  std::vector<ProfPair> prof_pending;
  std::vector<cudaEvent_t> prof_free;
  // host copy of each population's slot count, kept current after every
  // round so the sort can size itself without reading the device
  std::vector<int> n_slots_host;
  // device scalars of a round: [0] events that lost a claim, [1] events,
  // [2] items (the events of the round before), [3] chain chunks handed out,
  // [4] winning chains of the round
  DevBuf<long long> round_dev;
  std::vector<long long> base_cached;  // pair-list layout last uploaded
  double prof_ms[4] = {0, 0, 0, 0};
  long long prof_launch[4] = {0, 0, 0, 0}, prof_units[4] = {0, 0, 0, 0};
  // replay
  DevBuf<double> replay_u;
  long long replay_n = 0, replay_used = 0;
  ReplayBuffers replay;
  // particle shape of aero_data (fractal_t); spherical unless set
  Fractal frac = fractal_spherical();
};

void free_list(std::vector<void*>& v) {
  for (void* p : v) cudaFree(p);
  v.clear();
}

template <class T>
T* dalloc(std::vector<void*>& owner, size_t n) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess)
    cap_throw("device memory: an allocation failed");
  owner.push_back(p);
  return (T*)p;
}

int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

// Times the launches issued inside its scope when profiling is on: a pair
// of CUDA events on the library's stream, read back only when the totals
// are asked for, so timing adds no synchronisation to the step.
struct ProfScope {
  Ctx& c;
  int id;
  long long units;
  cudaEvent_t e0 = nullptr;
  ProfScope(Ctx& c_, int id_, long long units_) : c(c_), id(id_), units(units_) {
    if (!c.prof) return;
    e0 = prof_event(c);
    cudaEventRecord(e0, c.stream);
  }
  ~ProfScope() {
    if (!c.prof || !e0) return;
    cudaEvent_t e1 = prof_event(c);
    cudaEventRecord(e1, c.stream);
    c.prof_pending.push_back({id, units, e0, e1});
  }
  static cudaEvent_t prof_event(Ctx& c) {
    if (!c.prof_free.empty()) {
      cudaEvent_t e = c.prof_free.back();
      c.prof_free.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
};

// fold the recorded event pairs into the per-kernel totals
void prof_collect(Ctx& c) {
  if (c.prof_pending.empty()) return;
  cudaStreamSynchronize(c.stream);
  for (auto& p : c.prof_pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.e0, p.e1);
    c.prof_ms[p.id] += ms;
    c.prof_launch[p.id] += 1;
    c.prof_units[p.id] += p.units;
    c.prof_free.push_back(p.e0);
    c.prof_free.push_back(p.e1);
  }
  c.prof_pending.clear();
}

// exclusive scans of in[0..n) into out[0..n] (out[n] = total), up to
// kScanMaxJobs arrays of one element type in one launch.  With nd, a job's
// count is *nd (device memory) and n only bounds it.
template <class T>
struct ScanArg {
  const T* in;
  long long n;
  const long long* nd;
  long long* out;
  long long* total_out = nullptr;
};

template <class T>
void scan_multi(Ctx& c, std::initializer_list<ScanArg<T>> args, cudaStream_t st = nullptr) {
  if (!st) st = c.stream;
  ScanJobs jobs{};
  int k = 0;
  long long nb = 1;
  for (const auto& a : args) {
    jobs.j[k].in = a.in;
    jobs.j[k].out = a.out;
    jobs.j[k].n_max = a.n;
    jobs.j[k].nd = a.nd;
    jobs.j[k].total_out = a.total_out;
    nb = std::max(nb, (a.n + kScanTile - 1) / kScanTile);
    k++;
  }
  if (k == 0) return;
  if (nb > (1LL << 30)) cap_throw("scan longer than its tile limit");
  c.scan_status.reserve((size_t)kScanMaxJobs * nb);
  if (c.scan_status.n > c.scan_status_n) {  // fresh memory: clear it once
    CK(cudaMemsetAsync(c.scan_status.p, 0, sizeof(unsigned long long) * c.scan_status.n, st));
    c.scan_status_n = c.scan_status.n;
  }
  dim3 g((unsigned)nb, (unsigned)k);
  k_scan_lb<T><<<g, kScanThreads, 0, st>>>(jobs, c.scan_status.p, (int)nb, c.scan_ctr.p, c.scan_ctr.p + kScanMaxJobs,
                                           c.scan_err.p);
  note_launch();
}

template <class T>
void scan_dev(Ctx& c, const T* in, long long n, const long long* nd, long long* out) {
  scan_multi<T>(c, {ScanArg<T>{in, n, nd, out}});
}

// a look-back that gave up is reported as a timed-out step
void check_scan_err(Ctx& c) {
  unsigned long long e = 0;
  CK(cudaMemcpyAsync(&e, c.scan_err.p, sizeof(e), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  if (e) {
    CK(cudaMemsetAsync(c.scan_err.p, 0, sizeof(e), c.stream));
    throw Fail(PMC_ERR_TIMEOUT);
  }
}

template <class T>
long long scan(Ctx& c, const T* in, long long n, long long* out, bool read_total) {
  scan_dev(c, in, n, (const long long*)nullptr, out);
  if (!read_total) return -1;
  long long t = 0;
  CK(cudaMemcpyAsync(&t, out + n, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  check_scan_err(c);
  return t;
}

void push_pops(Ctx& c) {
  std::vector<PopDev> v(c.n_pop);
  for (int k = 0; k < c.n_pop; k++) {
    v[k] = c.pops[k].h;
    v[k].round_p = c.d_round;
    v[k].gen_p = c.d_round + 1;
  }
  CK(cudaMemcpyAsync(c.d_pops, v.data(), sizeof(PopDev) * c.n_pop, cudaMemcpyHostToDevice, c.stream));
  c.dirty = false;
}

// counters of every population in one copy
std::vector<PopCtr>& read_ctrs(Ctx& c) {
  c.h_ctrs.resize(c.n_pop);
  CK(cudaMemcpyAsync(c.h_ctrs.data(), c.d_ctrs, sizeof(PopCtr) * c.n_pop, cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  return c.h_ctrs;
}

void write_ctrs(Ctx& c) {
  CK(cudaMemcpyAsync(c.d_ctrs, c.h_ctrs.data(), sizeof(PopCtr) * c.n_pop, cudaMemcpyHostToDevice, c.stream));
  CK(cudaStreamSynchronize(c.stream));
}

PopCtr read_ctr(Ctx& c, int k) { return read_ctrs(c)[k]; }

void write_ctr(Ctx& c, int k, const PopCtr& r) {
  CK(cudaMemcpyAsync(c.d_ctrs + k, &r, sizeof(PopCtr), cudaMemcpyHostToDevice, c.stream));
  CK(cudaStreamSynchronize(c.stream));
}

// allocate the slot arrays of a population with capacity cap
void alloc_slots(Ctx& c, PopHost& ph, int cap) {
  PopDev& h = ph.h;
  std::vector<void*>& o = ph.slot_allocs;
  h.cap = cap;
  h.vol = dalloc<double>(o, (size_t)cap * c.n_spec);
  h.vtot = dalloc<double>(o, cap);
  h.mass = dalloc<double>(o, cap);
  h.rad = dalloc<double>(o, cap);
  h.grp = dalloc<int>(o, cap);
  h.cls = dalloc<int>(o, cap);
  h.id = dalloc<long long>(o, cap);
  h.nprim = dalloc<int>(o, cap);
  h.ncomp = dalloc<int>(o, cap);
  h.csrc = dalloc<int>(o, (size_t)cap * kMaxComponent);
  h.ctime = dalloc<double>(o, (size_t)cap * kMaxComponent);
  h.lct = dalloc<double>(o, cap);
  h.gct = dalloc<double>(o, cap);
  h.imf = dalloc<double>(o, cap);
  h.den_ice = dalloc<double>(o, cap);
  h.phi = dalloc<double>(o, cap);
  h.hyst = dalloc<int>(o, cap);
  h.frozen = dalloc<int>(o, cap);
  h.alive = dalloc<uint8_t>(o, cap);
  h.changed = dalloc<uint8_t>(o, cap);
  h.cell = dalloc<int>(o, cap);
  h.list = dalloc<int>(o, cap);
  h.recd = dalloc<RecD>(o, cap);
  h.recf = dalloc<RecF>(o, cap);
  h.claim = dalloc<unsigned long long>(o, cap);
  h.rclaim = dalloc<unsigned long long>(o, cap);
  h.touched = dalloc<uint32_t>(o, cap);
  CK(cudaMemsetAsync(h.alive, 0, cap, c.stream));
  CK(cudaMemsetAsync(h.changed, 0, cap, c.stream));
  CK(cudaMemsetAsync(h.claim, 0xff, sizeof(unsigned long long) * cap, c.stream));  // no claim
  CK(cudaMemsetAsync(h.rclaim, 0xff, sizeof(unsigned long long) * cap, c.stream));
  CK(cudaMemsetAsync(h.touched, 0xff, sizeof(uint32_t) * cap, c.stream));        // no generation
  c.dirty = true;
}

// sort structures that depend on the grid and the slot count
void alloc_sort(Ctx& c, PopHost& ph) {
  PopDev& h = ph.h;
  free_list(ph.sort_allocs);
  std::vector<void*>& o = ph.sort_allocs;
  int nb = std::max(ph.n_bin, 1);
  h.n_cells = nb * c.n_class;
  ph.chunk_hist_cap = 0;  // reallocated by the sort when needed
  h.chunk_hist = nullptr;
  h.chunk_hist_len = 0;
  h.cell_count = dalloc<int>(o, h.n_cells);
  h.cell_start = dalloc<int>(o, h.n_cells + 1);
  h.kmax_tab = dalloc<double>(o, (size_t)nb * nb);
  // pairs in the reference's loop order (coagulation.F90:74-94)
  ph.pair_desc.clear();
  for (int c1 = 0; c1 < c.n_class; c1++)
    for (int c2 = 0; c2 <= c1; c2++)
      for (int b1 = 0; b1 < ph.n_bin; b1++)
        for (int b2 = (c1 == c2 ? b1 : 0); b2 < ph.n_bin; b2++) {
          PairDesc d;
          d.b1 = (int16_t)b1;
          d.b2 = (int16_t)b2;
          d.c1 = (int8_t)c1;
          d.c2 = (int8_t)c2;
          d.pad0 = d.pad1 = 0;
          ph.pair_desc.push_back(d);
        }
  h.n_pairs = (int)ph.pair_desc.size();
  if (h.n_pairs >= (1 << 20)) cap_throw("more than 2^20 bin pairs");  // pair numbers in keys and random streams
  // the pairs of each cell in loop order, for walks
  {
    std::vector<int> off(h.n_cells + 1, 0), list;
    for (const PairDesc& d : ph.pair_desc) {
      off[d.b1 + nb * d.c1 + 1]++;
      if (d.b2 + nb * d.c2 != d.b1 + nb * d.c1) off[d.b2 + nb * d.c2 + 1]++;
    }
    for (int k = 0; k < h.n_cells; k++) off[k + 1] += off[k];
    list.assign(std::max(off[h.n_cells], 1), 0);
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int p = 0; p < h.n_pairs; p++) {
      const PairDesc& d = ph.pair_desc[p];
      int a = d.b1 + nb * d.c1, b = d.b2 + nb * d.c2;
      list[fill[a]++] = p;
      if (b != a) list[fill[b]++] = p;
    }
    int max_len = 1;
    for (int k = 0; k < h.n_cells; k++) max_len = std::max(max_len, off[k + 1] - off[k]);
    const int n_coarse = ((max_len + 15) / 16 + 3) / 4 * 4;
    std::vector<int> coarse((size_t)h.n_cells * n_coarse, INT_MAX);
    for (int k = 0; k < h.n_cells; k++)
      for (int j = off[k], i = 0; j < off[k + 1]; j += 16, i++) coarse[(size_t)k * n_coarse + i] = list[j];
    int* d_coarse = dalloc<int>(o, coarse.size());
    CK(cudaMemcpyAsync(d_coarse, coarse.data(), sizeof(int) * coarse.size(), cudaMemcpyHostToDevice, c.stream));
    h.cp_coarse = d_coarse;
    h.n_coarse = n_coarse;
    int* d_off = dalloc<int>(o, off.size());
    int* d_list = dalloc<int>(o, list.size());
    h.cp_cum = dalloc<double>(o, (size_t)off[h.n_cells] + h.n_cells);
    h.cp_ent = dalloc<int4>(o, std::max(off[h.n_cells], 1));
    h.cp_nstop = dalloc<int>(o, std::max(off[h.n_cells], 1));
    h.cp_tab = dalloc<int>(o, (size_t)h.n_cells * kWalkTab);
    CK(cudaMemcpyAsync(d_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(d_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));  // the host vectors go out of scope
    h.cp_off = d_off;
    h.cp_list = d_list;
  }
  PairDesc* pd = dalloc<PairDesc>(o, std::max<size_t>(ph.pair_desc.size(), 1));
  if (!ph.pair_desc.empty())
    CK(cudaMemcpyAsync(pd, ph.pair_desc.data(), sizeof(PairDesc) * ph.pair_desc.size(),
                       cudaMemcpyHostToDevice, c.stream));
  h.pair_desc = pd;
  h.pair = dalloc<PairState>(o, std::max<size_t>(ph.pair_desc.size(), 1));
  h.kmax_valid = 0;
  h.pair_setup_valid = 0;
  c.dirty = true;
}

// bin_grid_make (log) on the host, with glibc's log/exp like the reference
void make_grid(Ctx& c, PopHost& ph, int n_bin, double rmin, double rmax) {
  ph.n_bin = n_bin;
  ph.edges.assign(n_bin + 1, 0.0);
  ph.centers.assign(std::max(n_bin, 1), 0.0);
  if (n_bin > 0) {
    auto linspace = [](double a, double b, int n, double* out) {
      for (int i = 2; i <= n - 1; i++) {
        double t = (double)(i - 1) / (double)(n - 1);
        out[i - 1] = (1.0 - t) * a + t * b;
      }
      if (n > 0) {
        out[0] = a;
        out[n - 1] = b;
      }
    };
    auto logspace = [&](double a, double b, int n, double* out) {
      if (n == 0) return;
      linspace(log(a), log(b), n, out);
      for (int i = 0; i < n; i++) out[i] = exp(out[i]);
      out[0] = a;
      out[n - 1] = b;
    };
    logspace(rmin, rmax, n_bin + 1, ph.edges.data());
    double c1 = exp(interp_linear_disc(log(rmin), log(rmax), 2 * n_bin + 1, 2));
    double c2 = exp(interp_linear_disc(log(rmin), log(rmax), 2 * n_bin + 1, 2 * n_bin));
    logspace(c1, c2, n_bin, ph.centers.data());
  }
  GridDev g{};
  g.n_bin = n_bin;
  if (n_bin > 0) {
    g.log_lo = log(ph.edges[0]);
    g.log_hi = log(ph.edges[n_bin]);
    for (int i = 0; i <= n_bin; i++) g.edges[i] = ph.edges[i];
    for (int i = 0; i < n_bin; i++) g.centers[i] = ph.centers[i];
  }
  CK(cudaMemcpyAsync(ph.h.grid, &g, sizeof(GridDev), cudaMemcpyHostToDevice, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  alloc_sort(c, ph);
}

void set_params(Ctx& c, PopHost& ph) {
  PopDev& h = ph.h;
  h.n_spec = c.n_spec;
  h.n_group = c.n_group;
  h.n_class = c.n_class;
  h.i_water = c.i_water;
  h.w = ph.own_w ? ph.w : c.w;
  h.flat = weights_flat(h.w);
  bool inc, dec;
  weight_monotonicity(h.w, &inc, &dec);
  h.mono_dec = dec;
  h.dmin = *std::min_element(c.density.begin(), c.density.end());
  h.dmax = *std::max_element(c.density.begin(), c.density.end());
  h.seed = ph.seed;
  h.pair_setup_valid = 0;  // the per-pair weight factors depend on the weights
  // radii follow the particle shape from the first sort on, before any step
  // sets the environment
  h.benv.frac = c.frac;
  c.dirty = true;
}

void init_pop(Ctx& c, PopHost& ph, int cap) {
  std::vector<void*>& o = ph.fixed_allocs;
  ph.h.ctr = c.d_ctrs + (&ph - c.pops.data());
  ph.h.grid = dalloc<GridDev>(o, 1);
  double* dens = dalloc<double>(o, c.n_spec);
  CK(cudaMemcpy(dens, c.density.data(), sizeof(double) * c.n_spec, cudaMemcpyHostToDevice));
  ph.h.density = dens;
  set_params(c, ph);
  alloc_slots(c, ph, cap);
  PopCtr z{};
  ph.rm_count = 0;  // the population's removal records start empty
  z.next_id = 1;
  z.bmin = 1 << 30;
  z.bmax = -1;
  write_ctr(c, (int)(&ph - c.pops.data()), z);
  ph.n_bin = 0;
  GridDev g{};
  CK(cudaMemcpyAsync(ph.h.grid, &g, sizeof(GridDev), cudaMemcpyHostToDevice, c.stream));
  alloc_sort(c, ph);
}

// grow (compact = false, slot numbers kept) or compact (slot order kept)
void relayout(Ctx& c, int k, int new_cap, bool compact) {
  PopHost& ph = c.pops[k];
  PopCtr r = read_ctr(c, k);
  PopDev old = ph.h;
  std::vector<void*> old_allocs;
  old_allocs.swap(ph.slot_allocs);
  alloc_slots(c, ph, new_cap);
  DevBuf<long long> off;
  off.reserve((size_t)r.n_slots + 1);
  long long n_live = r.n_slots;
  if (compact) n_live = scan(c, old.alive, r.n_slots, off.p, true);
  if (r.n_slots > 0)
    k_relayout<<<grid_for(r.n_slots, 256), 256, 0, c.stream>>>(old, ph.h, off.p, r.n_slots,
                                                               compact ? 1 : 0); note_launch();
  CK(cudaStreamSynchronize(c.stream));
  off.release();
  free_list(old_allocs);
  if (compact) {
    r.n_slots = (int)n_live;
    ph.mirror_full = true;  // slots renumbered
  }
  write_ctr(c, k, r);
  push_pops(c);
  CK(cudaStreamSynchronize(c.stream));
}

// ---------------------------------------------------------------------------
// sort, with the grid decision of aero_sorted_remake_if_needed
// (aero_sorted.F90:214-373)

__global__ void k_radius_minmax_masked(const PopDev* pops, const uint8_t* on) {
  if (!on[blockIdx.y]) return;
  const PopDev& P = pops[blockIdx.y];
  int n = P.ctr->n_slots;
  // positive doubles order like their bit patterns: reduce the bits in the
  // block, then one atomic per block
  unsigned long long lo = ~0ULL, hi = 0ULL;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!P.alive[i]) continue;
    unsigned long long b = (unsigned long long)__double_as_longlong(vol2rad(P.benv.frac, P.vtot[i]));
    lo = b < lo ? b : lo;
    hi = b > hi ? b : hi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long l2 = __shfl_down_sync(0xffffffffu, lo, o);
    unsigned long long h2 = __shfl_down_sync(0xffffffffu, hi, o);
    lo = l2 < lo ? l2 : lo;
    hi = h2 > hi ? h2 : hi;
  }
  __shared__ unsigned long long slo[32], shi[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    slo[wid] = lo;
    shi[wid] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
      lo = slo[k] < lo ? slo[k] : lo;
      hi = shi[k] > hi ? shi[k] : hi;
    }
    if (hi > 0ULL) {
      atomicMin(&P.ctr->rmin_bits, lo);
      atomicMax(&P.ctr->rmax_bits, hi);
    }
  }
}


// chunk counts from the host's copy of the slot counts
// chunk histograms for the current slot counts plus extra slots per
// population (the growth a device-driven loop may add before the host looks)
void prepare_chunks(Ctx& c, long long extra = 0) {
  for (int k = 0; k < c.n_pop; k++) {
    PopHost& ph = c.pops[k];
    ph.h.n_chunks = (int)((c.n_slots_host[k] + extra + kChunk - 1) / kChunk);
    int need = std::max(ph.h.n_chunks, 1) * ph.h.n_cells;
    if (need > ph.chunk_hist_cap) {
      int want = std::max(need * 2, 1024);  // headroom: slots grow inside a step
      ph.h.chunk_hist = dalloc<int>(ph.sort_allocs, want);
      ph.h.chunk_hist_len = want;
      ph.chunk_hist_cap = want;
      c.dirty = true;
    }
  }
}

// one cooperative launch of k_sort_all on a persistent grid of co-resident
// blocks, for chunk and cell counts up to max_chunks and max_cells
// co-resident blocks of the sort for max_cells cells (its shared memory)
size_t size_sort(Ctx& c, int max_cells) {
  size_t smem = sizeof(int) * (kSortWarps + 1) * (size_t)max_cells;
  if (smem != c.sort_smem) {
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sort_all, kSortThreads, smem));
    if (per_sm < 1) cap_throw("the sort does not fit one block per multiprocessor");
    c.sort_blocks = per_sm * c.n_sm;
    c.sort_smem = smem;
  }
  return smem;
}

void launch_sort(Ctx& c, cudaStream_t st, int max_chunks, int max_cells) {
  size_t smem = size_sort(c, max_cells);
  long long items = (long long)c.n_pop * max_chunks;
  int blocks = (int)std::min<long long>(c.sort_blocks, std::max<long long>(items, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(kSortThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const PopDev* pops = c.d_pops;
  CK(cudaLaunchKernelEx(&cfg, k_sort_all, pops, c.n_pop, max_chunks, max_cells));
  note_launch();
}

int max_cells_of(const Ctx& c) {
  int m = 1;
  for (int k = 0; k < c.n_pop; k++) m = std::max(m, c.pops[k].h.n_cells);
  return m;
}

// the full sort of every population with its current grid
void run_sort(Ctx& c) {
  prepare_chunks(c);
  if (c.dirty) push_pops(c);
  int max_chunks = 1;
  long long units = 0;
  for (int k = 0; k < c.n_pop; k++) {
    max_chunks = std::max(max_chunks, c.pops[k].h.n_chunks);
    units += (long long)c.n_slots_host[k];
  }
  ProfScope ps(c, 1, units);
  launch_sort(c, c.stream, max_chunks, max_cells_of(c));
}

bool caches_current(const Ctx& c, const PopHost& ph) {
  return ph.caches_valid && ph.key_kt == ph.h.kernel_type && ph.key_temp == ph.h.temp &&
         ph.key_press == ph.h.pressure && ph.key_coeff == ph.h.coeff && ph.key_wver == ph.wver;
}

// recompute radius, bin and records of every live slot of the marked
// populations (after a grid, environment, kernel or weight change)
void refresh_caches(Ctx& c, const std::vector<uint8_t>& on) {
  bool any = false;
  for (int k = 0; k < c.n_pop; k++) any = any || on[k];
  if (!any) return;  // no read-back (a stream sync) in the common case
  int max_slots = 1;
  std::vector<PopCtr>& r = read_ctrs(c);
  for (int k = 0; k < c.n_pop; k++)
    if (on[k]) max_slots = std::max(max_slots, r[k].n_slots);
  push_pops(c);
  DevBuf<uint8_t> don;
  don.reserve(c.n_pop);
  CK(cudaMemcpyAsync(don.p, on.data(), c.n_pop, cudaMemcpyHostToDevice, c.stream));
  dim3 g(grid_for(max_slots, 256), c.n_pop);
  k_refresh_all<<<g, 256, 0, c.stream>>>(c.d_pops, don.p);
  note_launch();
  CK(cudaStreamSynchronize(c.stream));
  don.release();
  for (int k = 0; k < c.n_pop; k++)
    if (on[k]) {
      PopHost& ph = c.pops[k];
      ph.caches_valid = true;
      ph.key_kt = ph.h.kernel_type;
      ph.key_temp = ph.h.temp;
      ph.key_press = ph.h.pressure;
      ph.key_coeff = ph.h.coeff;
      ph.key_wver = ph.wver;
    }
}

// aero_state_sort: grid decision (remake_if_needed) then the sort itself
void sort_pops(Ctx& c, bool decide_grid) {
  bool hist_current = false;
  if (decide_grid) {
    std::vector<PopCtr>& r0 = read_ctrs(c);
    c.n_slots_host.resize(c.n_pop);
    for (int k = 0; k < c.n_pop; k++) c.n_slots_host[k] = r0[k].n_slots;
    // radius range of populations without a valid sort
    std::vector<uint8_t> on(c.n_pop, 0), fresh(c.n_pop, 0);
    bool any = false;
    std::vector<PopCtr>& r = r0;
    int max_slots = 1;
    for (int k = 0; k < c.n_pop; k++) {
      if (!c.pops[k].valid_sort) {
        on[k] = 1;
        any = true;
        r[k].rmin_bits = 0x7ff0000000000000ULL;
        r[k].rmax_bits = 0;
        max_slots = std::max(max_slots, r[k].n_slots);
      } else if (!caches_current(c, c.pops[k])) {
        fresh[k] = 1;  // current grid, stale caches
      }
    }
    if (any) {
      write_ctrs(c);
      DevBuf<uint8_t> don;
      don.reserve(c.n_pop);
      CK(cudaMemcpyAsync(don.p, on.data(), c.n_pop, cudaMemcpyHostToDevice, c.stream));
      dim3 g(grid_for(max_slots, 256), c.n_pop);
      k_radius_minmax_masked<<<g, 256, 0, c.stream>>>(c.d_pops, don.p);
      note_launch();
      CK(cudaStreamSynchronize(c.stream));
      don.release();
    }
    refresh_caches(c, fresh);
    // sort with the current grid; the occupied bin range decides whether the
    // grid is kept
    run_sort(c);
    hist_current = true;
    std::vector<PopCtr>& q = read_ctrs(c);
    std::vector<uint8_t> regrid(c.n_pop, 0);
    for (int k = 0; k < c.n_pop; k++) {
      PopHost& ph = c.pops[k];
      double rmin = 0.0, rmax = 0.0;
      if (!ph.valid_sort) {
        if (q[k].n_live > 0) {
          memcpy(&rmin, &q[k].rmin_bits, 8);
          memcpy(&rmax, &q[k].rmax_bits, 8);
        }
      } else if (q[k].bmax < 0) {
        if (ph.n_bin > 0) {
          rmin = ph.edges[ph.n_bin];
          rmax = ph.edges[0];
        }
      } else {
        rmin = ph.edges[q[k].bmin];
        rmax = ph.edges[q[k].bmax + 1];
      }
      bool need = false;
      if (rmax == 0.0) {
        if (!ph.valid_sort && ph.n_bin != 0) make_grid(c, ph, 0, 0.0, 0.0);
      } else if (ph.n_bin < 1) {
        need = true;
      } else {
        double gmin = ph.edges[0], gmax = ph.edges[ph.n_bin];
        if (rmin / gmin < 3.0 || gmax / rmax < 3.0) need = true;
      }
      if (need) {
        double gmin = rmin / 10.0, gmax = rmax * 10.0;
        int n_bin = (int)ceil((log10(gmax) - log10(gmin)) * 10.0);
        if (n_bin > kMaxBin) cap_throw("more than 256 bins");
        make_grid(c, ph, n_bin, gmin, gmax);
      }
      // a new grid or a population without a valid sort: all bins change
      if (need || !ph.valid_sort) {
        regrid[k] = 1;
        ph.caches_valid = false;
        hist_current = false;
      }
      ph.valid_sort = true;
    }
    refresh_caches(c, regrid);
  }
  if (!hist_current) run_sort(c);
}

// ---------------------------------------------------------------------------
// one step over all populations

// call f(std::integral_constant<int, KT>, T{}) with the kernel type kt and the
// pair-test arithmetic of the mode (FP32 in MIXED, else FP64)
template <class F>
void with_kt(const Ctx& c, int kt, F&& f) {
  bool f32 = c.mode == PMC_MODE_MIXED;
  auto go = [&](auto ktc) {
    if (f32) f(ktc, float{});
    else f(ktc, double{});
  };
  switch (kt) {
    case kKernelAdditive: go(std::integral_constant<int, kKernelAdditive>{}); break;
    case kKernelConstant: go(std::integral_constant<int, kKernelConstant>{}); break;
    case kKernelBrown: go(std::integral_constant<int, kKernelBrown>{}); break;
    case kKernelSedi: go(std::integral_constant<int, kKernelSedi>{}); break;
    case kKernelBrownFree: go(std::integral_constant<int, kKernelBrownFree>{}); break;
    case kKernelBrownCont: go(std::integral_constant<int, kKernelBrownCont>{}); break;
    default: f(std::integral_constant<int, kKernelZero>{}, double{});
  }
}

// Brackets the launches of one tunable site with CUDA events while the
// autotuner searches that site; otherwise does nothing.
struct TuneScope {
  Ctx& c;
  cudaEvent_t e0 = nullptr;
  cudaStream_t st;
  static cudaEvent_t event(Ctx& c) {
    if (!c.tuner.spare.empty()) {
      cudaEvent_t e = c.tuner.spare.back();
      c.tuner.spare.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    CK(cudaEventCreate(&e));
    return e;
  }
  TuneScope(Ctx& c_, int site, cudaStream_t st_) : c(c_), st(st_) {
    if (!c.tuner.on || c.tuner.site != site) return;
    e0 = event(c);
    CK(cudaEventRecord(e0, st));
  }
  ~TuneScope() {
    if (!e0) return;
    cudaEvent_t e1 = event(c);
    cudaEventRecord(e1, st);
    c.tuner.pending.push_back({e0, e1});
  }
};

void launch_test_kt(Ctx& c, int kt, bool flat, int n_gpairs, long long W, cudaStream_t st) {
  TuneScope ts(c, kTuneTest, st);
  // sized from the round's sample count, at most 8 x 256 threads per SM
  const int tb = c.tune.threads[kTuneTest];
  int blocks = (int)std::min<long long>((long long)c.n_sm * 8 * 256 / tb, std::max<long long>(1, (W + tb - 1) / tb));
  with_kt(c, kt, [&](auto ktc, auto tt) {
    constexpr int KT = decltype(ktc)::value;
    using T = decltype(tt);
    if (flat)
      k_test<KT, T, true><<<blocks, tb, 0, st>>>(c.d_pops, c.gpair_pop.p, c.gpair_local.p, c.work_off.p, n_gpairs,
                                                 c.work_off.p + n_gpairs, c.flag.p, c.ev.p, c.ev_gp.p);
    else
      k_test<KT, T, false><<<blocks, tb, 0, st>>>(c.d_pops, c.gpair_pop.p, c.gpair_local.p, c.work_off.p, n_gpairs,
                                                  c.work_off.p + n_gpairs, c.flag.p, c.ev.p, c.ev_gp.p);
  });
  note_launch();
}

ChainPool chain_pool(Ctx& c) {
  ChainPool pool;
  pool.y = c.ch_y.p;
  pool.q = c.ch_q.p;
  pool.pos = c.ch_pos.p;
  pool.ctr = c.round_dev.p + 3;
  pool.n_chunks = c.ch_chunks;
  return pool;
}

// a later round's items: the events of the round before, n_items =
// round_dev[2] on the device, W bounds it
void launch_items_kt(Ctx& c, int kt, bool flat, int n_gpairs, long long W, cudaStream_t st) {
  const int ti = c.tune.threads[kTuneItems], tc = c.tune.threads[kTuneChain];
  int blocks = grid_for(W, ti);
  const long long* n_items = c.round_dev.p + 2;
  ChainPool pool = chain_pool(c);
  with_kt(c, kt, [&](auto ktc, auto tt) {
    constexpr int KT = decltype(ktc)::value;
    using T = decltype(tt);
    auto k = flat ? k_items<KT, T, true> : k_items<KT, T, false>;
    {
      TuneScope ts_items(c, kTuneItems, st);
      k<<<blocks, ti, 0, st>>>(c.d_pops, c.gpair_pop.p, c.gpair_local.p, c.pop_pair_base.p, n_gpairs, n_items,
                                c.round_dev.p + 6, c.ppw_slot_in.p, c.ppw_gp_in.p, c.op_pop.p, c.op_pair.p,
                                c.op_slot.p, c.op_k.p, c.op_key.p, c.n_dev.p, c.op_cap,
                                c.win_set.p, c.ev_dest.p, c.ev_key.p, c.ev_c.p, c.gp_c.p, c.ev_pos.p, c.dec_set.p,
                                c.it_flag.p, c.it_key.p, c.it_c.p, c.it_gp.p, c.it_pos.p, c.it_len.p, c.it_head.p,
                                c.it_done.p, c.it_dec.p, c.it_gused.p, c.it_term.p);
    }
    auto kc = flat ? k_chain<KT, T, true> : k_chain<KT, T, false>;
    {
      TuneScope ts_chain(c, kTuneChain, st);
      kc<<<grid_for(W, tc), tc, 0, st>>>(c.d_pops, c.gpair_pop.p, n_items, c.it_flag.p, c.it_key.p, c.it_c.p,
                                           c.it_gp.p, c.it_pos.p, c.it_dec.p, c.it_gused.p, pool, c.it_len.p,
                                           c.it_head.p, c.it_done.p, c.it_term.p);
    }
  });
  note_launch();
  note_launch();
}

__global__ void k_ops_span(long long* n_ops, long long n_redo, const long long* n_items) {
  n_ops[0] = n_redo + *n_items;
}

// Stable grouping by population of a batched context's per-round lists.
// Slot and ID ranks come from one scan over a list, and the per-population
// bases of k_alloc_bases assume that each population's entries lie together
// and in population order.  Round 0's samples and target operations are
// built that way; later rounds add entries from every population at the end
// (the walkers of target operations, and the target operations that walks
// add).  Entry i with population pop_of[i] >= 0 (negative: not kept) goes to
// dest[i]: all of population 0 first, then 1, ..., each in list order.
// Tiles of kGrpTile entries: per tile and population a count (hist, laid
// out population-major so that one scan gives every (population, tile) its
// start), then each entry's rank within its tile.
constexpr int kGrpTile = 256;

__global__ void __launch_bounds__(kGrpTile) k_grp_hist(const long long* n, const int* pop_of, int n_pop, int n_tiles,
                                                       int* hist, PopCtr* ctr0) {
  const long long N = *n;
  const long long i = blockIdx.x * (long long)kGrpTile + threadIdx.x;
  if (i >= N) return;
  const int p = pop_of[i];
  if (p < 0) return;
  if (p >= n_pop || blockIdx.x >= (unsigned)n_tiles) {
    bad_index(ctr0, kBadEventSlot, p);
    return;
  }
  atomicAdd(&hist[(size_t)p * n_tiles + blockIdx.x], 1);
}

__global__ void __launch_bounds__(kGrpTile) k_grp_rank(const long long* n, const int* pop_of, int n_tiles,
                                                       const long long* off, long long* dest) {
  __shared__ int wpop[kGrpTile / 32][32], wcnt[kGrpTile / 32][32];
  const long long N = *n;
  const long long i = blockIdx.x * (long long)kGrpTile + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int p = i < N ? pop_of[i] : -1;
  const unsigned same = __match_any_sync(0xffffffffu, p);
  const int rank = __popc(same & ((1u << lane) - 1u));
  // one entry per distinct population of the warp: its count there
  wpop[w][lane] = -1;
  wcnt[w][lane] = 0;
  __syncthreads();
  // the lowest lane of each group writes at its own lane index
  if (rank == 0) {
    wpop[w][lane] = p;
    wcnt[w][lane] = __popc(same);
  }
  __syncthreads();
  if (p < 0) {
    if (i < N) dest[i] = -1;  // not kept
    return;
  }
  int before = 0;
  for (int v = 0; v < w; v++)
    for (int l = 0; l < 32; l++)
      if (wpop[v][l] == p) before += wcnt[v][l];
  dest[i] = off[(size_t)p * n_tiles + blockIdx.x] + before + rank;
}

__global__ void k_scatter_ops(const long long* n_ops, const long long* dest, const int* pop, const int* pair,
                              const int* slot, const int* k, const unsigned long long* key, int* pop_o, int* pair_o,
                              int* slot_o, int* k_o, unsigned long long* key_o) {
  const long long Q = *n_ops;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Q; q += (long long)gridDim.x * blockDim.x) {
    const long long d = dest[q];
    if (d < 0) continue;  // a place without an operation: dropped
    pop_o[d] = pop[q];
    pair_o[d] = pair[q];
    slot_o[d] = slot[q];
    k_o[d] = k[q];
    key_o[d] = key[q];
  }
}

// the population of each kept item of a later round (-1 for an item that
// made no event)
__global__ void k_item_pops(const long long* n_items, const uint8_t* it_flag, const int* it_gp, const int* gpair_pop,
                            int n_gpairs, int* pop_of) {
  const long long n = *n_items;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int gp = it_gp[i];
    pop_of[i] = (it_flag[i] && gp >= 0 && gp < n_gpairs) ? gpair_pop[gp] : -1;
  }
}

// dest for the entries of a list of at most bound entries (count *n on the
// device), grouped by population (k_grp_hist, k_grp_rank)
void group_by_pop(Ctx& c, const long long* n, long long bound, const int* pop_of, long long* dest, cudaStream_t st) {
  const int n_tiles = (int)std::max<long long>(1, (bound + kGrpTile - 1) / kGrpTile);
  const long long nh = (long long)n_tiles * c.n_pop;
  c.grp_hist.reserve((size_t)nh);
  c.grp_off.reserve((size_t)nh + 1);
  CK(cudaMemsetAsync(c.grp_hist.p, 0, sizeof(int) * (size_t)nh, st));
  k_grp_hist<<<n_tiles, kGrpTile, 0, st>>>(n, pop_of, c.n_pop, n_tiles, c.grp_hist.p, c.d_ctrs);
  note_launch();
  scan_multi<int>(c, {ScanArg<int>{c.grp_hist.p, nh, nullptr, c.grp_off.p}}, st);
  k_grp_rank<<<n_tiles, kGrpTile, 0, st>>>(n, pop_of, n_tiles, c.grp_off.p, dest);
  note_launch();
}

// The round's target operations (at most Q, counted on the device): the
// bound on each one's removals, scanned into its place in the removal pool,
// then the operations themselves.  An operation whose place runs past the
// pool loses, as one that lost a claim does, and is redone in the next
// round; the host reads the round's total with its other counts and grows
// the pool before that round.
void launch_pp(Ctx& c, int kt, long long Q, bool grouped) {
  int blocks = grid_for(Q, 128);
  if (!grouped) {
    // a later round's list: the redone operations, then one place per item
    // (population -1 where the item made none); grouping also drops those
    c.grp_dest.reserve((size_t)Q + 1);
    c.g_pop.reserve(Q); c.g_pair.reserve(Q); c.g_slot.reserve(Q); c.g_k.reserve(Q); c.g_key.reserve(Q);
    group_by_pop(c, c.n_dev.p + 0, Q, c.op_pop.p, c.grp_dest.p, c.stream);
    k_scatter_ops<<<grid_for(Q, 256), 256, 0, c.stream>>>(c.n_dev.p + 0, c.grp_dest.p, c.op_pop.p, c.op_pair.p,
                                                          c.op_slot.p, c.op_k.p, c.op_key.p, c.g_pop.p, c.g_pair.p,
                                                          c.g_slot.p, c.g_k.p, c.g_key.p);
    note_launch();
    // the operations kept: the scan's total
    const long long nh = (long long)std::max<long long>(1, (Q + kGrpTile - 1) / kGrpTile) * c.n_pop;
    CK(cudaMemcpyAsync(c.n_dev.p, c.grp_off.p + nh, sizeof(long long), cudaMemcpyDeviceToDevice, c.stream));
    std::swap(c.op_pop, c.g_pop); std::swap(c.op_pair, c.g_pair); std::swap(c.op_slot, c.g_slot);
    std::swap(c.op_k, c.g_k); std::swap(c.op_key, c.g_key);
  }
  c.pp_rm_n.reserve((size_t)Q + 1);
  c.pp_rm_off.reserve((size_t)Q + 2);
  c.pp_rm_tot.reserve(1);
  k_pp_count<<<blocks, 128, 0, c.stream>>>(c.d_pops, c.op_pop.p, c.op_pair.p, c.op_slot.p, c.op_k.p,
                                           c.n_dev.p + 0, c.pp_rm_n.p);
  note_launch();
  scan_multi<int>(c, {ScanArg<int>{c.pp_rm_n.p, Q, c.n_dev.p + 0, c.pp_rm_off.p, c.pp_rm_tot.p}});
  // every operation's removals fit the pool: one that did not would lose
  // and draw anew a round later, so the pool's size (in a batch, the other
  // populations' removals) would decide the particles.  One read-back; the
  // steps that have target operations run their rounds from the host.
  {
    long long rm_tot = 0;
    unsigned long long scan_err = 0;
    CK(cudaMemcpyAsync(&rm_tot, c.pp_rm_tot.p, sizeof(rm_tot), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(&scan_err, c.scan_err.p, sizeof(scan_err), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (scan_err) {
      CK(cudaMemsetAsync(c.scan_err.p, 0, sizeof(scan_err), c.stream));
      throw Fail(PMC_ERR_TIMEOUT);
    }
    if (rm_tot < 0 || rm_tot >= (1LL << 31)) cap_throw("more than 2^31 removals in one round");
    if (rm_tot + 1 > (long long)c.pp_rm_pool.n) c.pp_rm_pool.reserve((size_t)(rm_tot + rm_tot / 2 + 1024));
  }
  with_kt(c, kt, [&](auto ktc, auto) {
    constexpr int KT = decltype(ktc)::value;
    k_pp_ops<KT><<<blocks, 128, 0, c.stream>>>(c.d_pops, c.op_pop.p, c.op_pair.p, c.op_slot.p, c.op_k.p,
                                               c.op_key.p, c.n_dev.p + 0, c.pp_res.p, c.pp_vol.p, c.pp_rm_off.p,
                                               c.pp_rm_pool.p, (long long)c.pp_rm_pool.n);
  });
  note_launch();
}

void set_n_dev(Ctx& c, long long v) {
  CK(cudaMemcpyAsync(c.n_dev.p, &v, sizeof(long long), cudaMemcpyHostToDevice, c.stream));
}

// One mc_coag call in replay mode: the grid decision of
// aero_sorted_remake_if_needed on the host (glibc log/exp, as the reference),
// then one device thread runs the reference's loop on the persisted inverse
// maps.  One population only.
int replay_step_host(Ctx& c, long long* s_out, long long* k_out) {
  if (c.n_pop != 1) return PMC_ERR_INVALID_ARG;
  PopHost& ph = c.pops[0];
  ReplayBuffers& rb = c.replay;
  PopCtr r = read_ctr(c, 0);
  if (r.n_live != r.n_slots) {
    relayout(c, 0, ph.h.cap, true);  // dense slots, order kept
    r = read_ctr(c, 0);
    rb.valid = false;
  }
  if (ph.h.cap < 2 * r.n_slots + 1024) {
    relayout(c, 0, 2 * r.n_slots + 1024, false);
    rb.valid = false;
  }
  // radius range: from the inverse maps while they are valid, else from the
  // particles (aero_sorted.F90:263-306)
  double rmin = 0.0, rmax = 0.0;
  if (!rb.valid || ph.n_bin < 1) {
    r.rmin_bits = 0x7ff0000000000000ULL;
    r.rmax_bits = 0;
    write_ctr(c, 0, r);
    push_pops(c);
    DevBuf<uint8_t> on;
    on.reserve(1);
    uint8_t one = 1;
    CK(cudaMemcpyAsync(on.p, &one, 1, cudaMemcpyHostToDevice, c.stream));
    dim3 g(grid_for(std::max(r.n_slots, 1), 256), 1);
    k_radius_minmax_masked<<<g, 256, 0, c.stream>>>(c.d_pops, on.p);
    note_launch();
    PopCtr q = read_ctr(c, 0);
    on.release();
    if (q.n_live > 0) {
      memcpy(&rmin, &q.rmin_bits, 8);
      memcpy(&rmax, &q.rmax_bits, 8);
    }
  } else {
    std::vector<int> cnt(ph.n_bin * c.n_class);
    DevBuf<int> d;
    d.reserve(cnt.size());
    replay_cell_counts(rb.dev, d.p, c.stream);
    note_launch();
    CK(cudaMemcpyAsync(cnt.data(), d.p, sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    d.release();
    int bmin = 0, bmax = 0;
    for (int b = 1; b <= ph.n_bin; b++) {
      int s = 0;
      for (int cl = 0; cl < c.n_class; cl++) s += cnt[(b - 1) + ph.n_bin * cl];
      if (s > 0) {
        if (bmin == 0) bmin = b;
        bmax = b;
      }
    }
    if (bmin == 0) {
      rmin = ph.edges[ph.n_bin];
      rmax = ph.edges[0];
    } else {
      rmin = ph.edges[bmin - 1];
      rmax = ph.edges[bmax];
    }
  }
  bool rebuild = !rb.valid;
  if (rmax == 0.0) {
    if (!rb.valid) make_grid(c, ph, 0, 0.0, 0.0);
  } else {
    bool need = ph.n_bin < 1;
    if (!need) {
      double gmin = ph.edges[0], gmax = ph.edges[ph.n_bin];
      need = rmin / gmin < 3.0 || gmax / rmax < 3.0;
    }
    if (need) {
      double gmin = rmin / 10.0, gmax = rmax * 10.0;
      int n_bin = (int)ceil((log10(gmax) - log10(gmin)) * 10.0);
      if (n_bin > kMaxBin) return PMC_ERR_CAPACITY;
      make_grid(c, ph, n_bin, gmin, gmax);
      rebuild = true;
    }
  }
  ph.valid_sort = true;
  int nb = std::max(ph.n_bin, 1);
  if (!replay_reserve(rb, ph.h.cap, nb * c.n_class, c.n_group * c.n_class, nb, c.n_class, c.n_group))
    return PMC_ERR_CAPACITY;
  if (rb.n_cells != nb * c.n_class || !rb.valid) rebuild = true;
  push_pops(c);
  if (!ph.h.kmax_valid && ph.n_bin > 0) {
    dim3 g((ph.n_bin * ph.n_bin + 255) / 256, 1);
    k_kmax_table<<<g, 256, 0, c.stream>>>(c.d_pops);
    note_launch();
    ph.h.kmax_valid = 1;
    push_pops(c);
  }
  long long hv[4] = {c.replay_used, 0, 0, r.next_id};
  CK(cudaMemcpyAsync(rb.dev.used, hv, sizeof(long long) * 4, cudaMemcpyHostToDevice, c.stream));
  int hi[2] = {0, r.n_slots};
  CK(cudaMemcpyAsync(rb.dev.status, hi, sizeof(int) * 2, cudaMemcpyHostToDevice, c.stream));
  ReplayDev rd = rb.dev;
  rd.u = c.replay_u.p;
  rd.n_u = c.replay_n;
  rd.rebuild = rebuild ? 1 : 0;
  size_t stack = 0;
  cudaDeviceGetLimit(&stack, cudaLimitStackSize);
  if (stack < 16384) CK(cudaDeviceSetLimit(cudaLimitStackSize, 16384));
  replay_launch(c.d_pops, 0, rd, c.stream);
  note_launch();
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(hv, rb.dev.used, sizeof(long long) * 4, cudaMemcpyDeviceToHost, c.stream));
  CK(cudaMemcpyAsync(hi, rb.dev.status, sizeof(int) * 2, cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  c.replay_used = hv[0];
  *s_out = hv[1];
  *k_out = hv[2];
  r = read_ctr(c, 0);
  r.n_slots = r.n_live = hi[1];
  r.next_id = hv[3];
  r.tot_samp = hv[1];
  r.tot_coag = hv[2];
  write_ctr(c, 0, r);
  rb.valid = hi[0] == 0;
  ph.caches_valid = false;  // the replay rewrote slots without the caches
  static const int map[] = {PMC_OK, PMC_ERR_INVALID_ARG, PMC_ERR_OUT_OF_GRID, PMC_ERR_CAPACITY,
                            PMC_ERR_CUDA, PMC_ERR_TIMEOUT, PMC_ERR_RNG_EXHAUSTED, PMC_ERR_ASSERT};
  return (hi[0] >= 0 && hi[0] <= 7) ? map[hi[0]] : PMC_ERR_ASSERT;
}

__global__ void k_step_reset(PopCtr* ctrs, int n_pop) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_pop) return;
  ctrs[k].tot_samp = ctrs[k].tot_coag = ctrs[k].kmax_warn = ctrs[k].redraws = ctrs[k].walk_tests = 0;
  ctrs[k].status = 0;
  ctrs[k].bad_site = 0;
  ctrs[k].bad_index = 0;
  ctrs[k].cap_site = 0;
}

__global__ void k_fill_claims(const PopDev* pops) {
  const PopDev& P = pops[blockIdx.y];
  int n = P.ctr->n_slots;
  if (n > P.cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) bad_index(P.ctr, kBadSlotCount, n);
    n = P.cap;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    P.claim[i] = ~0ULL;
    P.rclaim[i] = ~0ULL;
    P.touched[i] = ~0u;
  }
}

// per-population work of a round: samples and target operations
__global__ void k_pop_work(const long long* pop_pair_base, int n_pop, const long long* work_off,
                           const long long* pp_off, long long* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_pop) return;
  long long a = pop_pair_base[k], b = pop_pair_base[k + 1];
  out[2 * k] = work_off[b] - work_off[a];
  out[2 * k + 1] = pp_off[b] - pp_off[a];
}

// ---------------------------------------------------------------------------
// Later rounds.  After round 0 every kernel of a round reads its counts from
// the device, and round 0's events bound every later round's items and
// events (each event yields at most one item of the next round, each item at
// most one event or chain).  So the later rounds run as the body of a
// conditional WHILE node of one CUDA graph: k_round_begin advances the round
// and the claim generation and makes the last round's events this round's
// items; the sort brings the cell lists to the round's start, so walks meet
// the particles earlier rounds made; k_round_end adds up the step's
// statistics and sets the loop condition: events in this round, fewer than
// max_rounds rounds, and room in every population for the next round's new
// slots, in the slot arrays and in the sort's chunks.  Without room the
// graph stops and the host loop, which can grow both, carries on.  Rounds
// with per-particle redo operations run from the host loop.

__global__ void k_round_begin(uint32_t* d_round, long long* round_dev, int* per_pop, int n_per_pop) {
  if (blockIdx.x != 0) return;
  if (threadIdx.x == 0) {
    d_round[0] += 1u;
    d_round[1] += 1u;
    // this round's items: the events of the round before, then the walkers
    // its target operations made
    round_dev[6] = round_dev[1];
    round_dev[7] = round_dev[5];
    round_dev[2] = round_dev[1] + round_dev[5];
    round_dev[0] = 0;
    round_dev[1] = 0;
    round_dev[3] = 0;
    round_dev[4] = 0;
    round_dev[5] = 0;
    round_dev[8] = 0;
  }
  for (int k = threadIdx.x; k < n_per_pop; k += blockDim.x) per_pop[k] = 0;
}

// stats: [0] events that lost a claim, [1] events, [2] rounds, [3] 1 if the
// graph stopped for lack of slots with events left
__global__ void k_round_end(const long long* round_dev, long long* stats, const uint32_t* d_round, int max_rounds,
                            const PopDev* pops, PopCtr* ctrs, int n_pop, long long sort_slots,
                            cudaGraphConditionalHandle cond) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  long long E = round_dev[1];
  stats[0] += round_dev[0];
  stats[1] += E;
  stats[2] += 1;
  bool room = true;
  for (int k = 0; k < n_pop; k++) {
    long long need = (long long)ctrs[k].n_slots + E;
    if (need > (long long)pops[k].cap || need > sort_slots) room = false;
  }
  bool more = E > 0 && room && (int)d_round[0] + 1 < max_rounds;
  if (E > 0 && room && !more)
    for (int k = 0; k < n_pop; k++)
      if (ctrs[k].status == 0) ctrs[k].status = kErrTimeout;
  if (E > 0 && !room) stats[3] = 1;
  cudaGraphSetConditional(cond, more ? 1u : 0u);
}

// Resolve and apply the events of a round (E at round_dev[1], at most W) and,
// with Q > 0 (host loop only), its Q target operations.
void resolve_apply(Ctx& c, cudaStream_t st, long long W, long long Q) {
  long long* Ed = c.round_dev.p + 1;
  ChainPool pool = chain_pool(c);
  if (W > 0) {
    const int tr = c.tune.threads[kTuneResolve];
    {
      TuneScope ts(c, kTuneResolve, st);
      k_resolve_set<<<grid_for(W, tr), tr, 0, st>>>(c.d_pops, c.gpair_pop.p, Ed, c.ev_key.p, c.ev_c.p, c.gp_c.p,
                                                      c.need_slot_set.p, c.need_id_set.p, c.win_set.p, c.dec_set.p,
                                                      c.round_dev.p, c.ev_len.p, c.ev_head.p, c.ev_app.p, pool,
                                                      c.chain_list.p, c.round_dev.p + 4);
    }
    note_launch();
    scan_multi<int>(c, {{c.need_slot_set.p, W, Ed, c.rank_slot_set.p}, {c.need_id_set.p, W, Ed, c.rank_id_set.p}},
                    st);
  }
  // Q bounds the round's target operations; their count is n_dev[0] (the
  // redone ones, then those that walks appended)
  if (Q > 0) {
    k_pp_resolve<<<grid_for(Q, 256), 256, 0, st>>>(c.d_pops, c.op_pop.p, c.op_key.p, c.n_dev.p, c.pp_res.p,
                                                   c.pp_rm_pool.p, c.win_pp.p, c.need_slot_pp.p, c.need_id_pp.p, c.lost_pp.p);
    note_launch();
    scan_multi<int>(c, {{c.need_slot_pp.p, Q, c.n_dev.p, c.rank_slot_pp.p}, {c.need_id_pp.p, Q, c.n_dev.p, c.rank_id_pp.p}},
                    st);
    k_count_per_pop<<<grid_for(Q, 256), 256, 0, st>>>(c.need_slot_pp.p, c.n_dev.p, c.op_pop.p,
                                                      c.per_pop_i.p + 2 * c.n_pop);
    note_launch();
    k_count_per_pop<<<grid_for(Q, 256), 256, 0, st>>>(c.need_id_pp.p, c.n_dev.p, c.op_pop.p,
                                                      c.per_pop_i.p + 3 * c.n_pop);
    note_launch();
  }
  k_alloc_bases<<<1, 256, 0, st>>>(c.d_pops, c.n_pop, Ed, c.gp_c.p, c.gpair_pop.p, W > 0 ? 1 : 0, c.rank_slot_set.p,
                                   c.rank_id_set.p, c.per_pop_i.p, c.slot_base_set.p, c.id_base_set.p,
                                   c.slot_base_pp.p, c.id_base_pp.p);
  note_launch();
  if (W > 0) {
    // part 1, one thread per event: species and components
    const int ta = c.tune.threads[kTuneApply];
    {
      TuneScope ts(c, kTuneApply, st);
      k_apply_move<<<grid_for(W, ta), ta, 0, st>>>(c.d_pops, c.gpair_pop.p, Ed, c.ev_key.p, c.ev_c.p, c.gp_c.p,
                                                          c.win_set.p, c.dec_set.p, c.rank_slot_set.p,
                                                          c.slot_base_set.p, c.ice_set.p);
      note_launch();
      // part 2, one thread per event: removals, scalar fields, caches
      k_apply_set<<<grid_for(W, ta), ta, 0, st>>>(c.d_pops, c.gpair_pop.p, Ed, c.ev_key.p, c.ev_c.p, c.gp_c.p,
                                                    c.win_set.p, c.dec_set.p, c.rank_slot_set.p, c.rank_id_set.p,
                                                    c.slot_base_set.p, c.id_base_set.p, c.ice_set.p, c.ev_done.p,
                                                    c.ev_dest.p, c.ev_key.p, c.ev_c.p, c.gp_c.p, c.ev_pos.p, c.dec_set.p,
                                                    c.ev_term.p, c.pop_pair_base.p);
      note_launch();
    }
    // chains, one warp each
    k_apply_chain<<<grid_for(W, 32), 32, 0, st>>>(c.d_pops, c.gpair_pop.p, c.pop_pair_base.p, c.chain_list.p,
                                                    c.round_dev.p + 4, c.ev_key.p, c.ev_len.p, c.ev_app.p,
                                                    c.ev_head.p, c.ev_done.p, pool, c.gp_c.p, c.ev_pos.p,
                                                    c.ev_dest.p, c.ev_key.p, c.ev_c.p, c.dec_set.p, c.ev_term.p);
    note_launch();
  }
  if (Q > 0) {
    const size_t nw = (size_t)Q * kMaxCopies;
    c.wk_slot.reserve(nw); c.wk_gp.reserve(nw); c.wk_flag.reserve(nw); c.wk_off.reserve(nw + 1);
    k_pp_apply<<<grid_for(Q, 256), 256, 0, st>>>(c.d_pops, c.op_pop.p, c.n_dev.p, c.pp_res.p, c.pp_vol.p,
                                                 c.pp_rm_pool.p, c.win_pp.p, c.rank_slot_pp.p, c.rank_id_pp.p,
                                                 c.slot_base_pp.p, c.id_base_pp.p, c.pop_pair_base.p, c.op_k.p,
                                                 c.wk_slot.p, c.wk_gp.p, c.wk_flag.p);
    note_launch();
    k_walkers_span<<<1, 1, 0, st>>>(c.n_dev.p, c.round_dev.p + 9);
    note_launch();
    scan_multi<uint8_t>(c, {ScanArg<uint8_t>{c.wk_flag.p, (long long)nw, c.round_dev.p + 9, c.wk_off.p,
                                             c.round_dev.p + 5}}, st);
    k_compact_walkers<<<grid_for((long long)nw, 256), 256, 0, st>>>(c.round_dev.p + 9, c.wk_flag.p, c.wk_off.p,
                                                                    c.wk_slot.p, c.wk_gp.p, c.ppw_slot.p, c.ppw_gp.p);
    note_launch();
    scan_multi<int>(c, {ScanArg<int>{c.lost_pp.p, Q, c.n_dev.p, c.lost_off.p, c.round_dev.p + 8}}, st);
  }
}

struct RoundBounds {
  int kt;
  bool flat;
  int n_gpairs;
  long long W;     // items and events of a round, at most
  int max_chunks;  // sort chunks per population, at most
  int max_cells;
};

// The kernels of one later round on stream st, after k_round_begin: the
// sort, items, their events in item order, then resolve and apply.  With
// Q > 0 (host loop only) the round's per-particle redo operations claim
// alongside.
// Qn: the round's redone target operations (host loop only); with
// per-particle pairs in the step, walks append more (at most one per item),
// so the operations are bounded by Qb = Qn + W and counted on the device.
void enqueue_round_body(Ctx& c, cudaStream_t st, const RoundBounds& b, long long Qn) {
  long long W = b.W;
  const long long Q = c.pp_step ? Qn + W : Qn;
  launch_sort(c, st, b.max_chunks, b.max_cells);
  {
    dim3 g(b.max_cells, c.n_pop);
    k_walk_rates<<<g, 128, 0, st>>>(c.d_pops);
    note_launch();
  }
  if (Q > 0) set_n_dev(c, Qn);
  launch_items_kt(c, b.kt, b.flat, b.n_gpairs, W, st);
  if (Q > 0) {
    k_ops_span<<<1, 1, 0, st>>>(c.n_dev.p, Qn, c.round_dev.p + 2);  // redone ones + one place per item
    note_launch();
    launch_pp(c, b.kt, Q, false);
  }
  const long long* Id = c.round_dev.p + 2;
  long long* Ed = c.round_dev.p + 1;
  scan_multi<uint8_t>(c, {ScanArg<uint8_t>{c.it_flag.p, W, Id, c.it_off.p, Ed}}, st);
  // a batched step with target operations: the walkers they made join the
  // items after the events, from every population, so the events are
  // grouped by population for the allocation (group_by_pop)
  const long long* grouped = nullptr;
  if (c.pp_step && c.n_pop > 1) {
    c.item_pop.reserve((size_t)W + 1);
    c.grp_dest.reserve((size_t)W + 1);
    k_item_pops<<<grid_for(W, 256), 256, 0, st>>>(Id, c.it_flag.p, c.it_gp.p, c.gpair_pop.p, b.n_gpairs,
                                                  c.item_pop.p);
    note_launch();
    group_by_pop(c, Id, W, c.item_pop.p, c.grp_dest.p, st);
    grouped = c.grp_dest.p;
  }
  k_compact_items<<<grid_for(W, 256), 256, 0, st>>>(c.it_flag.p, c.it_off.p, Id, c.it_key.p, c.it_c.p, c.it_gp.p,
                                                    c.it_pos.p, c.it_len.p, c.it_head.p, c.it_done.p, c.it_dec.p,
                                                    c.it_term.p, c.ev_key.p, c.ev_c.p, c.gp_c.p, c.ev_pos.p,
                                                    c.ev_len.p, c.ev_head.p, c.ev_done.p, c.dec_set.p, c.ev_term.p,
                                                    grouped);
  note_launch();
  resolve_apply(c, st, W, Q);
}

// everything the captured launches depend on: sizes and device addresses
std::vector<long long> round_graph_key(const Ctx& c, const RoundBounds& b) {
  return {c.n_pop, b.kt, b.flat, b.n_gpairs, b.W, b.max_chunks, b.max_cells, c.sort_blocks, (long long)c.sort_smem,
          c.max_rounds, c.mode, c.ch_chunks, c.tune.threads[kTuneItems], c.tune.threads[kTuneChain],
          c.tune.threads[kTuneResolve], c.tune.threads[kTuneApply],
          (long long)c.d_pops, (long long)c.d_round, (long long)c.d_ctrs, (long long)c.round_dev.p,
          (long long)c.per_pop_i.p, (long long)c.pop_pair_base.p, (long long)c.gpair_pop.p,
          (long long)c.gpair_local.p, (long long)c.ev_key.p, (long long)c.ev_c.p, (long long)c.gp_c.p,
          (long long)c.ev_pos.p, (long long)c.ev_dest.p, (long long)c.ev_len.p, (long long)c.ev_head.p,
          (long long)c.ev_app.p, (long long)c.ev_done.p, (long long)c.chain_list.p, (long long)c.it_flag.p, (long long)c.it_key.p,
          (long long)c.it_c.p, (long long)c.it_gp.p, (long long)c.it_pos.p, (long long)c.it_len.p,
          (long long)c.it_head.p, (long long)c.it_done.p, (long long)c.it_dec.p, (long long)c.it_gused.p, (long long)c.it_off.p,
          (long long)c.it_term.p, (long long)c.ev_term.p, (long long)c.ppw_slot.p, (long long)c.ppw_gp.p,
          (long long)c.ch_y.p,
          (long long)c.ch_q.p, (long long)c.ch_pos.p, (long long)c.need_slot_set.p, (long long)c.need_id_set.p,
          (long long)c.win_set.p, (long long)c.dec_set.p, (long long)c.rank_slot_set.p, (long long)c.rank_id_set.p,
          (long long)c.slot_base_set.p, (long long)c.id_base_set.p, (long long)c.slot_base_pp.p,
          (long long)c.id_base_pp.p, (long long)c.ice_set.p, (long long)c.scan_status.p, (long long)c.scan_ctr.p,
          (long long)c.scan_err.p, (long long)c.graph_stats.p};
}

void free_redraw_graph(Ctx& c) {
  if (c.rg_exec) cudaGraphExecDestroy(c.rg_exec);
  if (c.rg_graph) cudaGraphDestroy(c.rg_graph);
  c.rg_exec = nullptr;
  c.rg_graph = nullptr;
  c.rg_key.clear();
}

// the item and event bound of the later rounds' graph for round-0 events
// e0: a power of two, at least 4096, so that it holds from step to step
long long graph_bound(long long e0) {
  long long w = 4096;
  while (w < e0) w *= 2;
  return w;
}

// Event arrays, sized in round 0 for graph_bound(samples), which bounds the
// events of every later round.  Some of them (key, slots, pair, position,
// win, destination) carry a round's events into the next one (k_items reads
// them), so nothing may reallocate them while a step runs.  The chain pool
// gets one chunk per possible chain start and 4096 more for long chains.
void reserve_events(Ctx& c, long long W) {
  size_t w = (size_t)graph_bound(W);
  c.ev_key.reserve(w + 1); c.ev_c.reserve(w + 1); c.gp_c.reserve(w + 1); c.ev_pos.reserve(w + 1);
  c.ev_dest.reserve(w + 1); c.win_set.reserve(w + 1); c.dec_set.reserve(w + 1);
  c.ev_len.reserve(w + 1); c.ev_head.reserve(w + 1); c.ev_app.reserve(w + 1); c.ev_done.reserve(w + 1);
  c.ev_term.reserve(w + 1);
  c.chain_list.reserve(w + 1);
  c.need_slot_set.reserve(w + 1); c.need_id_set.reserve(w + 1); c.ice_set.reserve(w + 1);
  c.rank_slot_set.reserve(w + 2); c.rank_id_set.reserve(w + 2);
  size_t chunks = w + 4096;
  c.ch_y.reserve(chunks * kChainChunk);
  c.ch_q.reserve(chunks * kChainChunk);
  c.ch_pos.reserve(chunks * kChainChunk);
  c.ch_chunks = (long long)(std::min(std::min(c.ch_y.n, c.ch_q.n), c.ch_pos.n) / kChainChunk);
}

bool events_fit(const Ctx& c, long long W) {
  size_t w = (size_t)W;
  return c.ev_key.n >= w + 1 && c.ev_c.n >= w + 1 && c.gp_c.n >= w + 1 && c.ev_pos.n >= w + 1 &&
         c.ev_dest.n >= w + 1 && c.win_set.n >= w + 1 && c.dec_set.n >= w + 1 && c.ev_len.n >= w + 1 &&
         c.ev_head.n >= w + 1 && c.ev_app.n >= w + 1 && c.ev_done.n >= w + 1 && c.chain_list.n >= w + 1 &&
         c.ev_term.n >= w + 1 &&
         c.need_slot_set.n >= w + 1 &&
         c.need_id_set.n >= w + 1 && c.ice_set.n >= w + 1 && c.rank_slot_set.n >= w + 2 &&
         c.rank_id_set.n >= w + 2;
}

// the item buffers of a later round, sized for W items (they hold nothing
// from one round to the next)
void reserve_round(Ctx& c, long long W) {
  size_t w = (size_t)std::max<long long>(W, 1);
  c.it_flag.reserve(w + 1); c.it_key.reserve(w + 1); c.it_c.reserve(w + 1); c.it_gp.reserve(w + 1);
  c.it_pos.reserve(w + 1); c.it_len.reserve(w + 1); c.it_head.reserve(w + 1); c.it_done.reserve(w + 1);
  c.it_dec.reserve(w + 1); c.it_gused.reserve(w + 1); c.it_term.reserve(w + 1);
  c.it_off.reserve(w + 2);
}

struct GraphRun {
  long long rounds = -1;  // -1: the caller runs the rounds from the host loop
  long long losers = 0, events = 0;
  bool stopped_for_room = false;
};

// Run the later rounds of this step as the graph (captured again when a
// bound or an address changed and the change held for two steps in a row).
// e0: the events of the round before.
GraphRun run_round_graph(Ctx& c, int kt, bool flat, int n_gpairs, long long e0) {
  GraphRun out;
  RoundBounds b;
  b.kt = kt;
  b.flat = flat;
  b.n_gpairs = n_gpairs;
  // rounded up so that the graph survives ordinary step-to-step changes
  b.W = graph_bound(e0);
  // the event arrays hold the last round's events: they must already be
  // large enough (reserve_events), never reallocated here
  if (!events_fit(c, b.W)) return out;
  // the sort's chunks cover the slots of several rounds' growth; the graph
  // stops before they would not
  long long slots = 0, min_slots = -1;
  for (int k = 0; k < c.n_pop; k++) {
    slots = std::max<long long>(slots, c.n_slots_host[k]);
    min_slots = min_slots < 0 ? c.n_slots_host[k] : std::min<long long>(min_slots, c.n_slots_host[k]);
  }
  b.max_chunks = (int)((slots + 4 * b.W + kChunk - 1) / kChunk);
  b.max_chunks = (b.max_chunks + 15) / 16 * 16;
  b.max_cells = max_cells_of(c);
  prepare_chunks(c, (long long)b.max_chunks * kChunk - min_slots);
  size_sort(c, b.max_cells);
  // every other buffer at its final size before the addresses are taken
  reserve_round(c, b.W);
  c.graph_stats.reserve(4);
  {
    long long nb = (b.W + kScanTile - 1) / kScanTile;
    c.scan_status.reserve((size_t)kScanMaxJobs * nb);
    if (c.scan_status.n > c.scan_status_n) {
      CK(cudaMemsetAsync(c.scan_status.p, 0, sizeof(unsigned long long) * c.scan_status.n, c.stream));
      c.scan_status_n = c.scan_status.n;
    }
  }
  if (c.dirty) push_pops(c);
  std::vector<long long> key = round_graph_key(c, b);
  if (key != c.rg_key && key != c.rg_seen) {
    // bounds or addresses new since the last step: capturing pays only when
    // they hold, so this step's later rounds run from the host loop
    c.rg_seen = key;
    return out;
  }
  if (key != c.rg_key) {
    free_redraw_graph(c);
    CK(cudaGraphCreate(&c.rg_graph, 0));
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, c.rg_graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, c.rg_graph, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    bool prof = c.prof;
    c.prof = false;  // no event records inside the body
    long long n0 = g_launches;
    CK(cudaStreamBeginCaptureToGraph(c.cap_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    try {
      k_round_begin<<<1, 128, 0, c.cap_stream>>>(c.d_round, c.round_dev.p, c.per_pop_i.p, 4 * c.n_pop);
      note_launch();
      enqueue_round_body(c, c.cap_stream, b, 0);
      k_round_end<<<1, 32, 0, c.cap_stream>>>(c.round_dev.p, c.graph_stats.p, c.d_round, c.max_rounds, c.d_pops,
                                              c.d_ctrs, c.n_pop, (long long)b.max_chunks * kChunk, cond);
      note_launch();
    } catch (...) {
      cudaGraph_t dummy;
      cudaStreamEndCapture(c.cap_stream, &dummy);
      c.prof = prof;
      free_redraw_graph(c);
      throw;
    }
    cudaGraph_t captured = nullptr;
    CK(cudaStreamEndCapture(c.cap_stream, &captured));
    c.prof = prof;
    c.rg_nodes = g_launches - n0;
    g_launches = n0;  // counted when they run
    CK(cudaGraphInstantiate(&c.rg_exec, c.rg_graph, 0));
    c.rg_key = key;
    c.rg_builds++;
  }
  CK(cudaMemsetAsync(c.graph_stats.p, 0, sizeof(long long) * 4, c.stream));
  {
    ProfScope ps(c, 2, 1);
    CK(cudaGraphLaunch(c.rg_exec, c.stream));
  }
  long long st[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(st, c.graph_stats.p, sizeof(st), cudaMemcpyDeviceToHost, c.stream));
  unsigned long long scan_err = 0;
  CK(cudaMemcpyAsync(&scan_err, c.scan_err.p, sizeof(scan_err), cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  if (scan_err) {
    CK(cudaMemsetAsync(c.scan_err.p, 0, sizeof(scan_err), c.stream));
    throw Fail(PMC_ERR_TIMEOUT);
  }
  g_launches += c.rg_nodes * st[2];
  c.claim_gen += (uint32_t)st[2];
  out.rounds = st[2];
  out.losers = st[0];
  out.events = st[1];
  out.stopped_for_room = st[3] != 0;
  return out;
}

// capacity for a round that may add `slots` new slots to every population
void ensure_room(Ctx& c, long long slots) {
  for (int k = 0; k < c.n_pop; k++) {
    long long need = (long long)c.n_slots_host[k] + slots;
    if (need > c.pops[k].h.cap) {
      int nc = (int)std::min<long long>(std::max<long long>(need * 3 / 2, 1024), (1LL << 31) - 1);
      relayout(c, k, nc, false);  // slot numbers kept
    }
  }
}

void step_parallel(Ctx& c, int kt) {
  k_step_reset<<<(c.n_pop + 127) / 128, 128, 0, c.stream>>>(c.d_ctrs, c.n_pop);
  note_launch();
  push_pops(c);
  sort_pops(c, true);
  // global pair list, uploaded when its layout changes
  std::vector<long long> base(c.n_pop + 1, 0);
  for (int k = 0; k < c.n_pop; k++) base[k + 1] = base[k] + c.pops[k].h.n_pairs;
  int n_gpairs = (int)base[c.n_pop];
  size_t ng = (size_t)n_gpairs + 1;
  if (base != c.base_cached) {
    std::vector<int> gp_pop(std::max(n_gpairs, 1)), gp_loc(std::max(n_gpairs, 1));
    for (int k = 0; k < c.n_pop; k++)
      for (int p = 0; p < c.pops[k].h.n_pairs; p++) {
        gp_pop[base[k] + p] = k;
        gp_loc[base[k] + p] = p;
      }
    c.gpair_pop.reserve(gp_pop.size());
    c.gpair_local.reserve(gp_loc.size());
    c.pop_pair_base.reserve(base.size());
    CK(cudaMemcpyAsync(c.gpair_pop.p, gp_pop.data(), sizeof(int) * gp_pop.size(), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.gpair_local.p, gp_loc.data(), sizeof(int) * gp_loc.size(), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.pop_pair_base.p, base.data(), sizeof(long long) * base.size(), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.base_cached = base;
  }
  c.nwork_set.reserve(ng);
  c.nwork_pp.reserve(ng);
  c.work_off.reserve(ng);
  c.pp_off.reserve(ng);
  c.per_pop_i.reserve(4 * (size_t)c.n_pop);
  c.slot_base_set.reserve(c.n_pop);
  c.slot_base_pp.reserve(c.n_pop);
  c.id_base_set.reserve(c.n_pop);
  c.id_base_pp.reserve(c.n_pop);
  c.n_dev.reserve(4 + 2 * (size_t)c.n_pop);
  // round_dev: [0] losers, [1] events, [2] items, [3] chain chunks, [4] chains,
  // [5] walkers of target operations, [6] items that are events, [7] items
  // that are such walkers, [8] target operations that lost a claim
  c.round_dev.reserve(10);
  int max_pairs = 1, nb_max = 1, max_cap = 1;
  for (int k = 0; k < c.n_pop; k++) {
    max_pairs = std::max(max_pairs, c.pops[k].h.n_pairs);
    nb_max = std::max(nb_max, c.pops[k].n_bin);
    max_cap = std::max(max_cap, c.pops[k].h.cap);
  }
  bool flat = true;
  for (int k = 0; k < c.n_pop; k++) flat = flat && c.pops[k].h.flat;
  c.last_set_losers = c.last_pp_lost = c.last_events = c.last_ops = 0;
  std::vector<long long> hw(3 + 2 * (size_t)c.n_pop);
  std::vector<int> per_pop(4 * (size_t)c.n_pop);

  // ---- round 0: every pair's samples and target operations
  {
    // a new claim generation for every round; they restart (with every
    // claim and touched word cleared) before a step could run out of them
    c.claim_gen++;
    bool wrapped = false;
    if (c.claim_gen + (uint32_t)c.max_rounds + 2u >= kGenLimit) {
      c.claim_gen = 1;
      wrapped = true;
    }
    uint32_t rg[2] = {0u, c.claim_gen};  // staged before the call returns
    CK(cudaMemcpyAsync(c.d_round, rg, sizeof(rg), cudaMemcpyHostToDevice, c.stream));
    if (c.dirty) push_pops(c);
    if (wrapped) {
      dim3 g(grid_for(max_cap, 256), c.n_pop);
      k_fill_claims<<<g, 256, 0, c.stream>>>(c.d_pops);
      note_launch();
    }
  }
  bool need_kmax = false, need_setup = false;
  for (int k = 0; k < c.n_pop; k++) {
    need_kmax = need_kmax || !c.pops[k].h.kmax_valid;
    need_setup = need_setup || !c.pops[k].h.pair_setup_valid;
  }
  if (need_kmax) {
    dim3 g((nb_max * nb_max + 255) / 256, c.n_pop);
    k_kmax_table<<<g, 256, 0, c.stream>>>(c.d_pops);
    note_launch();
  }
  if (need_setup) {
    dim3 g((unsigned)(((long long)max_pairs * 32 + 255) / 256), c.n_pop);
    k_pair_setup<<<g, 256, 0, c.stream>>>(c.d_pops);
    note_launch();
  }
  {
    dim3 gp((max_pairs + 127) / 128, c.n_pop);
    k_pairs<<<gp, 128, 0, c.stream>>>(c.d_pops, c.pop_pair_base.p, c.nwork_set.p, c.nwork_pp.p, 1);
    note_launch();
  }
  // the device copies learn this with the next push
  for (int k = 0; k < c.n_pop; k++) {
    c.pops[k].h.kmax_valid = 1;
    c.pops[k].h.pair_setup_valid = 1;
  }
  c.dirty = true;
  scan_multi<long long>(c, {{c.nwork_set.p, n_gpairs, nullptr, c.work_off.p},
                            {c.nwork_pp.p, n_gpairs, nullptr, c.pp_off.p}});
  long long W, Q;
  {
    long long* popw = c.n_dev.p + 4;
    if (c.n_pop > 1) {
      k_pop_work<<<(c.n_pop + 127) / 128, 128, 0, c.stream>>>(c.pop_pair_base.p, c.n_pop, c.work_off.p, c.pp_off.p,
                                                              popw);
      note_launch();
    }
    // one read-back: totals and per-population work
    CK(cudaMemcpyAsync(&hw[0], c.work_off.p + n_gpairs, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(&hw[1], c.pp_off.p + n_gpairs, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    if (c.n_pop > 1)
      CK(cudaMemcpyAsync(&hw[3], popw, sizeof(long long) * 2 * c.n_pop, cudaMemcpyDeviceToHost, c.stream));
    unsigned long long pair_scan_err = 0;
    CK(cudaMemcpyAsync(&pair_scan_err, c.scan_err.p, sizeof(pair_scan_err), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (pair_scan_err) {
      CK(cudaMemsetAsync(c.scan_err.p, 0, sizeof(pair_scan_err), c.stream));
      throw Fail(PMC_ERR_TIMEOUT);
    }
    W = hw[0];
    Q = hw[1];
    if (c.n_pop == 1) {
      hw[3] = W;
      hw[4] = Q;
    }
    // a step with target operations runs its later rounds from the host,
    // where walks that reach a per-particle pair's target cell stop for one;
    // a population's walks stop when it has target operations of its own,
    // so it steps the same alone and in a batch
    c.pp_step = Q > 0;
    for (int k = 0; k < c.n_pop; k++) {
      const int stops = hw[3 + 2 * k + 1] > 0 ? 1 : 0;
      if (c.pops[k].h.walk_stops != stops) {
        c.pops[k].h.walk_stops = stops;
        c.dirty = true;
      }
    }
    // sample numbers fit in a key's 31 bits below the walk flag of the merge stream
    if (W + Q + 1 >= 0x7fffffffLL) cap_throw("more than 2^31 samples in one step");
  }
  // capacity for the worst case of this round: every sample creates a
  // particle and every target operation makes kMaxCopies - 1 copies
  for (int k = 0; k < c.n_pop; k++) {
    long long need = (long long)c.n_slots_host[k] + hw[3 + 2 * k] + (kMaxCopies - 1) * hw[3 + 2 * k + 1];
    if (need > c.pops[k].h.cap) {
      int nc = (int)std::min<long long>(std::max<long long>(need * 3 / 2, 1024), (1LL << 31) - 1);
      relayout(c, k, nc, false);  // slot numbers kept
    }
  }
  {
    size_t w = (size_t)W;
    c.flag.reserve(w + 1); c.ev.reserve(w + 1); c.flag_off.reserve(w + 2); c.ev_gp.reserve(w + 1);
    // the walkers that target operations make (the target and its copies)
    // join a later round's items and events
    reserve_events(c, W + kMaxCopies * Q);
    c.ppw_cap = kMaxCopies * (Q + 1);
    c.ppw_slot.reserve((size_t)c.ppw_cap);
    c.ppw_gp.reserve((size_t)c.ppw_cap);
    c.op_cap = Q;
    c.need_slot_pp.reserve(Q + 1); c.need_id_pp.reserve(Q + 1); c.win_pp.reserve(Q + 1); c.lost_pp.reserve(Q + 1);
    c.lost_off.reserve(Q + 2); c.rank_slot_pp.reserve(Q + 2); c.rank_id_pp.reserve(Q + 2);
  }
  if (c.dirty) push_pops(c);
  CK(cudaMemsetAsync(c.round_dev.p, 0, sizeof(long long) * 10, c.stream));
  CK(cudaMemsetAsync(c.per_pop_i.p, 0, sizeof(int) * 4 * c.n_pop, c.stream));
  if (W > 0) {
    ProfScope ps(c, 0, W);
    launch_test_kt(c, kt, flat, n_gpairs, W, c.stream);
  }
  if (Q > 0) {
    c.op_pop.reserve(Q); c.op_pair.reserve(Q); c.op_slot.reserve(Q); c.op_k.reserve(Q); c.op_key.reserve(Q);
    k_build_ops<<<n_gpairs, 128, 0, c.stream>>>(c.d_pops, c.gpair_pop.p, c.gpair_local.p, c.pp_off.p, n_gpairs,
                                                c.op_pop.p, c.op_pair.p, c.op_slot.p, c.op_k.p, c.op_key.p);
    note_launch();
    c.pp_res.reserve(Q);
    c.pp_vol.reserve((size_t)Q * c.n_spec);
    set_n_dev(c, Q);
    launch_pp(c, kt, Q, true);  // built in population order
  }
  // accepted samples in sample order; the sample count is work_off[n_gpairs]
  // and the event count E goes to round_dev[1], both on the device
  if (W > 0) {
    const long long* Wd = c.work_off.p + n_gpairs;
    scan_multi<uint8_t>(c, {ScanArg<uint8_t>{c.flag.p, W, Wd, c.flag_off.p, c.round_dev.p + 1}});
    k_compact_flags<<<grid_for(W, 256), 256, 0, c.stream>>>(c.flag.p, c.flag_off.p, Wd, c.ev.p, c.ev_gp.p,
                                                           c.gpair_local.p, c.work_off.p, c.ev_key.p, c.ev_c.p,
                                                           c.gp_c.p, c.ev_pos.p, c.ev_len.p, c.ev_term.p);
    note_launch();
    const int td = c.tune.threads[kTuneResolve];
    TuneScope ts(c, kTuneResolve, c.stream);
    k_decide<<<grid_for(W, td), td, 0, c.stream>>>(c.d_pops, c.gpair_pop.p, c.round_dev.p + 1, c.ev_key.p, c.ev_c.p,
                                                   c.gp_c.p, c.dec_set.p);
    note_launch();
  }
  resolve_apply(c, c.stream, W, Q);

  // ---- later rounds: retries, walks and per-particle redo operations
  long long redraws = 0, E = 0, pp_lost = 0;
  long long last_qb = Q;  // bound of the last round's target operations (0: it had none)
  int round = 0;
  bool graph_tried = false;
  for (;;) {
    // one read-back at the end of each host round
    long long losers = 0, ppw = 0;
    CK(cudaMemcpyAsync(&losers, c.round_dev.p, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(&E, c.round_dev.p + 1, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(&ppw, c.round_dev.p + 5, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    long long Qr = 0;
    pp_lost = 0;
    if (last_qb > 0) {
      CK(cudaMemcpyAsync(&pp_lost, c.round_dev.p + 8, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
      CK(cudaMemcpyAsync(&Qr, c.n_dev.p, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
    }
    CK(cudaMemcpyAsync(per_pop.data(), c.per_pop_i.p, sizeof(int) * 4 * c.n_pop, cudaMemcpyDeviceToHost, c.stream));
    unsigned long long scan_err = 0;
    CK(cudaMemcpyAsync(&scan_err, c.scan_err.p, sizeof(scan_err), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (scan_err) {
      CK(cudaMemsetAsync(c.scan_err.p, 0, sizeof(scan_err), c.stream));
      throw Fail(PMC_ERR_TIMEOUT);
    }
    for (int k = 0; k < c.n_pop; k++) c.n_slots_host[k] += per_pop[0 * c.n_pop + k] + per_pop[2 * c.n_pop + k];
    redraws += losers + pp_lost;
    c.last_set_losers += losers;
    c.last_pp_lost += pp_lost;
    c.last_events += E;
    c.last_ops += Qr;
    round++;
    if (E == 0 && pp_lost == 0 && ppw == 0) break;
    if (round >= c.max_rounds) {
      std::vector<PopCtr>& r = read_ctrs(c);
      for (int k = 0; k < c.n_pop; k++)
        if (r[k].status == 0) r[k].status = PMC_ERR_TIMEOUT;
      write_ctrs(c);
      break;
    }
    // this round's target operations: the redone ones, and with per-particle
    // pairs in the step at most one more per item (a walk that stops there)
    const long long Qb = pp_lost + (c.pp_step ? E + ppw : 0);
    // room for this round's new slots: at most one per item, and
    // kMaxCopies - 1 per target operation
    ensure_room(c, E + ppw + (kMaxCopies - 1) * Qb);
    // a round's items (events and walkers) each make at most one event
    if (!events_fit(c, E + ppw)) cap_throw("a round's events past the event arrays");
    if (!graph_tried && c.use_graph && !c.tuner.on && !c.pp_step && pp_lost == 0 && ppw == 0) {
      graph_tried = true;
      GraphRun g = run_round_graph(c, kt, flat, n_gpairs, E);
      if (g.rounds >= 0) {
        redraws += g.losers;
        c.last_set_losers += g.losers;
        c.last_events += g.events;
        round += (int)g.rounds;
        if (!g.stopped_for_room) break;
        // out of room inside the graph: the host loop grows the slot arrays
        // and carries on from the device's counts
        std::vector<PopCtr>& r = read_ctrs(c);
        for (int k = 0; k < c.n_pop; k++) c.n_slots_host[k] = r[k].n_slots;
        CK(cudaMemcpyAsync(&E, c.round_dev.p + 1, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        if (round >= c.max_rounds) {
          for (int k = 0; k < c.n_pop; k++)
            if (r[k].status == 0) r[k].status = PMC_ERR_TIMEOUT;
          write_ctrs(c);
          break;
        }
        ensure_room(c, E);
      }
    }
    // one host-driven round
    reserve_round(c, E + ppw);
    long long Qn = pp_lost;
    if (Qn > 0) {
      c.r_pop.reserve(Qb); c.r_pair.reserve(Qb); c.r_slot.reserve(Qb); c.r_k.reserve(Qb); c.r_key.reserve(Qb);
      k_build_redo<<<grid_for(last_qb, 256), 256, 0, c.stream>>>(c.d_pops, c.op_pop.p, c.op_pair.p, c.op_slot.p,
                                                                 c.op_k.p, c.op_key.p, c.lost_pp.p, c.lost_off.p,
                                                                 c.n_dev.p, c.r_pop.p, c.r_pair.p, c.r_slot.p,
                                                                 c.r_k.p, c.r_key.p);
      note_launch();
      std::swap(c.op_pop, c.r_pop); std::swap(c.op_pair, c.r_pair); std::swap(c.op_slot, c.r_slot);
      std::swap(c.op_k, c.r_k); std::swap(c.op_key, c.r_key);
    } else if (Qb > 0) {
      c.op_pop.reserve(Qb); c.op_pair.reserve(Qb); c.op_slot.reserve(Qb); c.op_k.reserve(Qb); c.op_key.reserve(Qb);
    }
    if (Qb > 0) {
      c.pp_res.reserve(Qb);
      c.pp_vol.reserve((size_t)Qb * c.n_spec);
      c.need_slot_pp.reserve(Qb + 1); c.need_id_pp.reserve(Qb + 1); c.win_pp.reserve(Qb + 1);
      c.lost_pp.reserve(Qb + 1); c.lost_off.reserve(Qb + 2); c.rank_slot_pp.reserve(Qb + 2);
      c.rank_id_pp.reserve(Qb + 2);
    }
    c.op_cap = Qb;
    // the walkers the last round's operations made are this round's to read;
    // this round's operations write theirs into the other pair of arrays
    std::swap(c.ppw_slot, c.ppw_slot_in);
    std::swap(c.ppw_gp, c.ppw_gp_in);
    c.ppw_cap = kMaxCopies * (Qb + 1);
    c.ppw_slot.reserve((size_t)c.ppw_cap);
    c.ppw_gp.reserve((size_t)c.ppw_cap);
    // the round's sort covers the current slots exactly
    prepare_chunks(c);
    int mc = 1;
    for (int k = 0; k < c.n_pop; k++) mc = std::max(mc, c.pops[k].h.n_chunks);
    if (c.dirty) push_pops(c);
    RoundBounds b{kt, flat, n_gpairs, E + ppw, mc, max_cells_of(c)};
    k_round_begin<<<1, 128, 0, c.stream>>>(c.d_round, c.round_dev.p, c.per_pop_i.p, 4 * c.n_pop);
    note_launch();
    c.claim_gen++;  // as k_round_begin on the device
    enqueue_round_body(c, c.stream, b, Qn);
    last_qb = Qb;
  }
  c.last_redraws = redraws;
  c.last_rounds = round;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI

struct pmc_coag_gpu_ctx {
  Ctx c;
};

extern "C" {

const char* pmc_coag_gpu_status_string(int s) {
  switch (s) {
    case PMC_OK: return "ok";
    case PMC_ERR_INVALID_ARG: return "invalid argument";
    case PMC_ERR_OUT_OF_GRID: return "particle outside of bin_grid: try reducing the timestep del_t";
    case PMC_ERR_CAPACITY: return g_last_capacity[0] ? g_last_capacity : "capacity exceeded";
    case PMC_ERR_CUDA: return g_last_error[0] ? g_last_error : "CUDA error";
    case PMC_ERR_TIMEOUT: return "bounded device loop ran out of iterations";
    case PMC_ERR_RNG_EXHAUSTED: return "replay stream exhausted";
    case PMC_ERR_ASSERT: return g_last_assert[0] ? g_last_assert : "reference assertion failed";
    case PMC_ERR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

#define GUARD_BEGIN try {
#define GUARD_END                 \
  }                               \
  catch (Fail & f) {              \
    return f.code;                \
  }                               \
  catch (...) {                   \
    return PMC_ERR_CAPACITY;      \
  }

static int do_init(int n_pop, int n_spec, const double* density, int i_water, int n_group, int n_class,
                   const int* w_type, const double* w_mag, const double* w_exp, const uint64_t* seeds,
                   pmc_coag_gpu_ctx** out) {
  if (!out || n_pop < 1 || n_spec < 1 || n_spec > kMaxSpec || n_group < 1 || n_group > kMaxGroup ||
      n_class < 1 || n_class > kMaxClass || !density || !w_type || !w_mag || !w_exp)
    return PMC_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return PMC_ERR_NO_DEVICE;
  std::unique_ptr<pmc_coag_gpu_ctx> x(new pmc_coag_gpu_ctx());
  Ctx& c = x->c;
  GUARD_BEGIN
  c.n_pop = n_pop;
  c.n_spec = n_spec;
  c.n_group = n_group;
  c.n_class = n_class;
  c.i_water = i_water;
  c.density.assign(density, density + n_spec);
  memset(&c.w, 0, sizeof(c.w));
  c.w.n_group = n_group;
  c.w.n_class = n_class;
  for (int cl = 0; cl < n_class; cl++)
    for (int g = 0; g < n_group; g++) {
      int src = g + n_group * cl;
      int dst = g + kMaxGroup * cl;
      if (w_type[src] < 1 || w_type[src] > 3) return PMC_ERR_INVALID_ARG;
      c.w.type[dst] = w_type[src];
      c.w.mag[dst] = w_mag[src];
      c.w.expo[dst] = w_exp[src];
    }
  CK(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c.cap_stream, cudaStreamNonBlocking));
  {
    int dev = 0, n_sm = 0, coop = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) throw Fail(PMC_ERR_NO_DEVICE);  // the sort needs cooperative launches
    c.n_sm = n_sm;
  }
  c.pops.resize(n_pop);
  CK(cudaMalloc(&c.d_pops, sizeof(PopDev) * n_pop));
  CK(cudaMalloc(&c.d_ctrs, sizeof(PopCtr) * n_pop));
  CK(cudaMalloc(&c.d_round, 2 * sizeof(uint32_t)));  // round of the step, claim generation
  CK(cudaMemset(c.d_round, 0, 2 * sizeof(uint32_t)));
  c.scan_ctr.reserve(2 * kScanMaxJobs);  // tile counters, then finished-block counters
  CK(cudaMemset(c.scan_ctr.p, 0, sizeof(unsigned) * c.scan_ctr.n));
  c.scan_err.reserve(1);
  CK(cudaMemset(c.scan_err.p, 0, sizeof(unsigned long long) * c.scan_err.n));
  CK(cudaMemset(c.d_ctrs, 0, sizeof(PopCtr) * n_pop));
  for (int k = 0; k < n_pop; k++) {
    c.pops[k].seed = seeds ? seeds[k] : (uint64_t)(k + 1);
    init_pop(c, c.pops[k], 1024);
  }
  push_pops(c);
  CK(cudaStreamSynchronize(c.stream));
  *out = x.release();
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_init(int n_spec, const double* density, int i_water, int n_group, int n_class,
                      const int* w_type, const double* w_mag, const double* w_exp, uint64_t seed,
                      pmc_coag_gpu_ctx** ctx) {
  return do_init(1, n_spec, density, i_water, n_group, n_class, w_type, w_mag, w_exp, &seed, ctx);
}

int pmc_coag_gpu_init_batch(int n_pop, int n_spec, const double* density, int i_water, int n_group,
                            int n_class, const int* w_type, const double* w_mag, const double* w_exp,
                            const uint64_t* seeds, pmc_coag_gpu_ctx** ctx) {
  return do_init(n_pop, n_spec, density, i_water, n_group, n_class, w_type, w_mag, w_exp, seeds, ctx);
}

int pmc_coag_gpu_destroy(pmc_coag_gpu_ctx* x) {
  if (!x) return PMC_OK;
  Ctx& c = x->c;
  cudaStreamSynchronize(c.stream);
  for (auto& ph : c.pops) {
    free_list(ph.slot_allocs);
    free_list(ph.sort_allocs);
    free_list(ph.fixed_allocs);
    if (ph.h.rm_log) cudaFree(ph.h.rm_log);
  }
  cudaFree(c.d_pops);
  cudaFree(c.d_ctrs);
  cudaFree(c.d_round);
  DevBuf<int>* bi[] = {&c.gpair_pop, &c.gpair_local, &c.need_slot_set, &c.need_id_set, &c.need_slot_pp,
                       &c.need_id_pp, &c.lost_pp, &c.op_pop, &c.op_pair, &c.op_slot, &c.op_k, &c.r_pop,
                       &c.r_pair, &c.r_slot, &c.r_k, &c.per_pop_i, &c.slot_base_set, &c.slot_base_pp,
                       &c.ev_dest, &c.ev_len, &c.ev_head, &c.ev_app, &c.it_gp, &c.it_len, &c.it_head,
                       &c.ch_y, &c.ch_q};
  for (auto* b : bi) b->release();
  DevBuf<long long>* bl[] = {&c.pop_pair_base, &c.nwork_set, &c.nwork_pp, &c.work_off, &c.pp_off, &c.flag_off,
                             &c.rank_slot_set, &c.rank_id_set, &c.rank_slot_pp, &c.rank_id_pp, &c.lost_off,
                             &c.id_base_set, &c.id_base_pp, &c.n_dev, &c.it_off};
  for (auto* b : bl) b->release();
  DevBuf<unsigned long long>* bk[] = {&c.ev_key, &c.it_key, &c.op_key, &c.r_key};
  for (auto* b : bk) b->release();
  c.ev_pos.release();
  c.it_pos.release();
  c.it_dec.release();
  c.it_gused.release();
  c.it_term.release();
  c.ev_term.release();
  c.ch_pos.release();
  c.it_flag.release();
  c.it_done.release();
  c.ev_done.release();
  c.chain_list.release();
  c.it_c.release();
  c.flag.release();
  c.win_set.release();
  c.dec_set.release();
  c.ev_gp.release();
  c.gp_c.release();
  c.ev_c.release();
  c.ice_set.release();
  c.scan_status.release();
  c.scan_ctr.release();
  c.scan_err.release();
  c.win_pp.release();
  c.ev.release();
  c.pp_res.release();
  c.pp_vol.release();
  c.replay_u.release();
  c.st_d.release();
  c.st_i.release();
  c.st_l.release();
  c.st_cnt.release();
  c.pin.release();
  c.map.release();
  for (auto& ev : c.sync_ev)
    if (ev) cudaEventDestroy(ev);
  replay_free(c.replay);
  free_redraw_graph(c);
  c.graph_stats.release();
  c.sample_buf.release();
  c.pp_rm_n.release();
  for (auto* b : {&c.grp_hist, &c.item_pop, &c.g_pop, &c.g_pair, &c.g_slot, &c.g_k}) b->release();
  c.grp_off.release();
  c.grp_dest.release();
  c.wk_slot.release();
  c.wk_gp.release();
  c.wk_flag.release();
  c.wk_off.release();
  c.g_key.release();
  c.pp_rm_pool.release();
  c.pp_rm_off.release();
  c.pp_rm_tot.release();
  c.dup_n.release();
  c.select_buf.release();
  for (auto& pr : c.tuner.pending) {
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  for (auto e : c.tuner.spare) cudaEventDestroy(e);
  cudaStreamDestroy(c.cap_stream);
  cudaStreamDestroy(c.stream);
  delete x;
  return PMC_OK;
}

int pmc_coag_gpu_upload(pmc_coag_gpu_ctx* x, int pop, int n_part, const double* vol, const int* group,
                        const int* cls, const int64_t* id, const int* n_primary) {
  if (!x || pop < 0 || pop >= x->c.n_pop || n_part < 0 || (n_part > 0 && !vol)) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  PopHost& ph = c.pops[pop];
  int cap = std::max(1024, n_part + n_part / 2 + 64);
  if (cap > ph.h.cap || cap < ph.h.cap / 4) {
    free_list(ph.slot_allocs);
    alloc_slots(c, ph, cap);
  }
  PopCtr r = read_ctr(c, pop);
  CK(cudaMemsetAsync(ph.h.alive, 0, ph.h.cap, c.stream));
  CK(cudaMemsetAsync(ph.h.changed, 0, ph.h.cap, c.stream));
  ph.mirror_full = true;  // a host copy kept slot by slot must be refreshed in full
  if (n_part > 0) {
    size_t n = (size_t)n_part;
    CK(cudaMemcpyAsync(ph.h.vol, vol, sizeof(double) * n * c.n_spec, cudaMemcpyHostToDevice, c.stream));
    if (group) CK(cudaMemcpyAsync(ph.h.grp, group, sizeof(int) * n, cudaMemcpyHostToDevice, c.stream));
    if (cls) CK(cudaMemcpyAsync(ph.h.cls, cls, sizeof(int) * n, cudaMemcpyHostToDevice, c.stream));
    if (id) CK(cudaMemcpyAsync(ph.h.id, id, sizeof(long long) * n, cudaMemcpyHostToDevice, c.stream));
    if (n_primary) CK(cudaMemcpyAsync(ph.h.nprim, n_primary, sizeof(int) * n, cudaMemcpyHostToDevice, c.stream));
    long long id0 = r.next_id;
    c.st_l.reserve(2);
    CK(cudaMemsetAsync(c.st_l.p, 0, 2 * sizeof(long long), c.stream));
    int* bad = (int*)c.st_l.p;
    unsigned long long* max_id = (unsigned long long*)(c.st_l.p + 1);
    k_upload<<<grid_for(n_part, 256), 256, 0, c.stream>>>(ph.h, n_part, group != nullptr, cls != nullptr,
                                                          id != nullptr, n_primary != nullptr, id0, bad, max_id);
    note_launch();
    long long chk[2] = {0, 0};
    CK(cudaMemcpyAsync(chk, c.st_l.p, sizeof(chk), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if ((int)chk[0] != 0) {
      // invalid groups or classes: the population is left empty
      CK(cudaMemsetAsync(ph.h.alive, 0, ph.h.cap, c.stream));
      r.n_slots = r.n_live = 0;
      write_ctr(c, pop, r);
      ph.valid_sort = false;
      ph.caches_valid = false;
      c.replay.valid = false;
      return PMC_ERR_INVALID_ARG;
    }
    if (id) r.next_id = std::max<long long>(r.next_id, chk[1] + 1);
    else r.next_id = id0 + n_part;
  }
  r.n_slots = n_part;
  r.n_live = n_part;
  write_ctr(c, pop, r);
  ph.valid_sort = false;
  ph.caches_valid = false;
  c.replay.valid = false;
  ph.n_bin = 0;
  {
    GridDev g{};
    CK(cudaMemcpyAsync(ph.h.grid, &g, sizeof(GridDev), cudaMemcpyHostToDevice, c.stream));
  }
  alloc_sort(c, ph);
  push_pops(c);
  CK(cudaStreamSynchronize(c.stream));
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_upload_components(pmc_coag_gpu_ctx* x, int pop, int n_part, const int* n_comp,
                                   const int* comp_source, const double* comp_create_time) {
  if (!x || pop < 0 || pop >= x->c.n_pop || !n_comp || !comp_source || !comp_create_time)
    return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  PopHost& ph = c.pops[pop];
  PopCtr r = read_ctr(c, pop);
  if (n_part != r.n_slots) return PMC_ERR_INVALID_ARG;
  // the slot arrays hold components particle-major, as the caller passes them
  std::vector<double> lct(n_part), gct(n_part);
  for (int i = 0; i < n_part; i++) {
    if (n_comp[i] < 0 || n_comp[i] > kMaxComponent) return PMC_ERR_INVALID_ARG;
    double lo = 0.0, hi = 0.0;
    for (int k = 0; k < n_comp[i]; k++) {
      double t = comp_create_time[comp_at(i, k)];
      if (k == 0 || t < lo) lo = t;
      if (k == 0 || t > hi) hi = t;
    }
    lct[i] = lo;
    gct[i] = hi;
  }
  size_t nc = (size_t)n_part * kMaxComponent;
  CK(cudaMemcpyAsync(ph.h.ncomp, n_comp, sizeof(int) * n_part, cudaMemcpyHostToDevice, c.stream));
  CK(cudaMemcpyAsync(ph.h.csrc, comp_source, sizeof(int) * nc, cudaMemcpyHostToDevice, c.stream));
  CK(cudaMemcpyAsync(ph.h.ctime, comp_create_time, sizeof(double) * nc, cudaMemcpyHostToDevice, c.stream));
  CK(cudaMemcpyAsync(ph.h.lct, lct.data(), sizeof(double) * n_part, cudaMemcpyHostToDevice, c.stream));
  CK(cudaMemcpyAsync(ph.h.gct, gct.data(), sizeof(double) * n_part, cudaMemcpyHostToDevice, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  return PMC_OK;
  GUARD_END
}

// Removal logs that record: room for the records kept so far plus the most
// one step or rebalance can add (each removal frees a slot, and a step ends
// with at most cap slots; twice that allows for slot growth within the
// step).  Grows a log by copying its records into a larger buffer.
void reserve_removal_logs(Ctx& c) {
  for (auto& ph : c.pops) {
    if (!ph.h.rm_on) continue;
    long long need = ph.rm_count + 2LL * ph.h.cap + 1024;
    if (ph.h.rm_cap >= need) continue;
    long long cap = std::max(need, ph.h.rm_cap + ph.h.rm_cap / 2);
    RemovalRec* p = nullptr;
    if (cudaMalloc(&p, sizeof(RemovalRec) * (size_t)cap) != cudaSuccess) {
      cudaGetLastError();
      throw Fail(PMC_ERR_CAPACITY);
    }
    if (ph.h.rm_log) {
      long long keep = std::min(ph.rm_count, ph.h.rm_cap);
      if (keep > 0)
        CK(cudaMemcpyAsync(p, ph.h.rm_log, sizeof(RemovalRec) * (size_t)keep, cudaMemcpyDeviceToDevice, c.stream));
      CK(cudaStreamSynchronize(c.stream));
      cudaFree(ph.h.rm_log);
    }
    ph.h.rm_log = p;
    ph.h.rm_cap = cap;
    c.dirty = true;
  }
}

static int finish_step(Ctx& c, long long* samp, long long* coag) {
  long long s = 0, k = 0, warn = 0, exact = 0;
  int status = 0;
  // one read-back (a stream sync) for every population; a compaction below
  // changes only its own population's counters
  const std::vector<PopCtr> all = read_ctrs(c);
  for (int p = 0; p < c.n_pop; p++) {
    const PopCtr& r = all[p];
    s += r.tot_samp;
    k += r.tot_coag;
    warn += r.kmax_warn;
    exact += r.exact_tests;
    c.pops[p].rm_count = r.n_removed;
    if (c.pops[p].h.rm_on && r.n_removed > c.pops[p].h.rm_cap) {
      snprintf(g_last_assert, sizeof(g_last_assert), "removal log of population %d overflowed", p);
      if (!status) status = PMC_ERR_CAPACITY;
    }
    if (r.status && !status) status = r.status;
    if (r.status == kErrCapacity && r.cap_site) {
      static const char* site[] = {"", "an event's new particle past the slot arrays",
                                   "the round's target-operation list is full",
                                   "a target operation's removals past its share of the pool",
                                   "more dup copies than one target operation holds",
                                   "a target operation's copy past the slot arrays",
                                   "the walker list of target operations is full",
                                   "a sampled particle past the slot arrays",
                                   "a doubled or dup copy past the slot arrays"};
      snprintf(g_last_capacity, sizeof(g_last_capacity), "capacity exceeded: %s (population %d)",
               r.cap_site < 9 ? site[r.cap_site] : "?", p);
    }
    if (r.bad_site) {
      static const char* site[] = {"", "pair test: list position", "pair test: slot", "event: slot",
                                   "sort scatter: list position", "sort: chunk histogram size",
                                   "pair set-up: cell range", "slot count above capacity",
                                   "event: destination slot"};
      snprintf(g_last_assert, sizeof(g_last_assert),
               "device bounds check failed (%s, population %d, index %lld)",
               r.bad_site < 9 ? site[r.bad_site] : "?", p, r.bad_index);
      status = PMC_ERR_ASSERT;
      continue;  // no compaction of a population in this state
    }
    // compact when more than half of the used slots are dead
    if (r.n_slots > 4096 && r.n_live < r.n_slots / 2) relayout(c, p, c.pops[p].h.cap, true);
  }
  c.last_kmax_warn = warn;
  c.exact_tests = exact;
  *samp = s;
  *coag = k;
  return status;
}

// the autotuner around one step: the candidate's shape before it; after it
// (finish_step has synchronised the stream) the device time of the site's
// launches and the step's pair tests
static void tune_before(Ctx& c) {
  Tuner& t = c.tuner;
  c.tune.threads[t.site] = kTuneCand[t.site][t.cand];
}

static void tune_after(Ctx& c, long long tests) {
  Tuner& t = c.tuner;
  for (auto& pr : t.pending) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
    t.cand_ms += ms;
    t.spare.push_back(pr.first);
    t.spare.push_back(pr.second);
  }
  t.pending.clear();
  t.cand_tests += tests;
  if (++t.rep < kTuneReps) return;
  const float score = (float)(t.cand_ms / (double)std::max(t.cand_tests, 1LL) * 1e6);
  t.site_ms[t.site][t.cand] = score;
  if (t.cand == 0 || score < t.best_ms) {
    t.best_ms = score;
    t.best = t.cand;
  }
  t.rep = 0;
  t.cand_ms = 0.0;
  t.cand_tests = 0;
  if (++t.cand < kTuneCands) return;
  c.tune.threads[t.site] = kTuneCand[t.site][t.best];
  t.cand = 0;
  if (++t.site < kTuneSites) return;
  t.on = false;
}

int pmc_coag_gpu_autotune(pmc_coag_gpu_ctx* x, int enable) {
  if (!x) return PMC_ERR_INVALID_ARG;
  Tuner& t = x->c.tuner;
  t.on = enable != 0;
  t.site = t.cand = t.rep = t.best = 0;
  t.best_ms = 0.f;
  t.cand_ms = 0.0;
  t.cand_tests = 0;
  for (auto& pr : t.pending) {
    t.spare.push_back(pr.first);
    t.spare.push_back(pr.second);
  }
  t.pending.clear();
  return PMC_OK;
}

int pmc_coag_gpu_tune_state(pmc_coag_gpu_ctx* x, int* tuning, int* threads, float* ms) {
  if (!x) return PMC_ERR_INVALID_ARG;
  const Ctx& c = x->c;
  if (tuning) *tuning = c.tuner.on ? 1 : 0;
  if (threads)
    for (int k = 0; k < kTuneSites; k++) threads[k] = c.tune.threads[k];
  if (ms)
    for (int k = 0; k < kTuneSites; k++)
      for (int j = 0; j < kTuneCands; j++) ms[k * kTuneCands + j] = c.tuner.site_ms[k][j];
  return PMC_OK;
}

int pmc_coag_gpu_set_tune(pmc_coag_gpu_ctx* x, const int* threads) {
  if (!x || !threads) return PMC_ERR_INVALID_ARG;
  for (int k = 0; k < kTuneSites; k++) {
    bool ok = false;
    for (int j = 0; j < kTuneCands; j++) ok = ok || threads[k] == kTuneCand[k][j];
    if (!ok) return PMC_ERR_INVALID_ARG;
  }
  for (int k = 0; k < kTuneSites; k++) x->c.tune.threads[k] = threads[k];
  x->c.tuner.on = false;
  return PMC_OK;
}

int pmc_coag_gpu_step_batch(pmc_coag_gpu_ctx* x, int kernel_type, const double* temp,
                            const double* pressure, double additive_coeff, double del_t, int n_steps,
                            int64_t* tot_n_samp, int64_t* tot_n_coag) {
  if (!x || kernel_type < 1 || kernel_type > 7 || !temp || !pressure || n_steps < 0)
    return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  long long S = 0, K = 0;
  for (int st = 0; st < n_steps; st++) {
    for (int k = 0; k < c.n_pop; k++) {
      PopHost& ph = c.pops[k];
      ph.h.kernel_type = kernel_type;
      ph.h.temp = temp[k];
      ph.h.pressure = pressure[k];
      ph.h.coeff = additive_coeff;
      ph.h.del_t = del_t;
      ph.h.benv = brown_env(temp[k], pressure[k], c.frac);
      ph.h.step = ++ph.step;
      // the reference keeps its bounds until the grid changes
      // (coag_kernel_bounds_valid, aero_sorted.F90:55); a new kernel type
      // would make them meaningless, so that case recomputes them
      if (ph.kmax_kt != kernel_type) {
        ph.h.kmax_valid = 0;
        ph.kmax_kt = kernel_type;
      }
    }
    reserve_removal_logs(c);
    push_pops(c);
    long long s = 0, k = 0;
    int status;
    if (c.mode == PMC_MODE_REPLAY) {
      status = replay_step_host(c, &s, &k);
    } else {
      ProfScope ps(c, 3, 1);
      c.replay.valid = false;  // the parallel step reorders and rewrites slots
      if (c.tuner.on) tune_before(c);
      step_parallel(c, kernel_type);
      status = finish_step(c, &s, &k);
      if (c.tuner.on && status == 0) tune_after(c, s);
    }
    S += s;
    K += k;
    if (status) {
      if (tot_n_samp) *tot_n_samp = S;
      if (tot_n_coag) *tot_n_coag = K;
      return status;
    }
  }
  if (tot_n_samp) *tot_n_samp = S;
  if (tot_n_coag) *tot_n_coag = K;
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_step(pmc_coag_gpu_ctx* x, int kernel_type, double temp, double pressure,
                      double additive_coeff, double del_t, int* tot_n_samp, int* tot_n_coag) {
  if (!x) return PMC_ERR_INVALID_ARG;
  std::vector<double> t(x->c.n_pop, temp), p(x->c.n_pop, pressure);
  int64_t s = 0, k = 0;
  int rc = pmc_coag_gpu_step_batch(x, kernel_type, t.data(), p.data(), additive_coeff, del_t, 1, &s, &k);
  if (tot_n_samp) *tot_n_samp = (int)s;
  if (tot_n_coag) *tot_n_coag = (int)k;
  return rc;
}

int pmc_coag_gpu_n_part(pmc_coag_gpu_ctx* x, int pop, int* n_part) {
  if (!x || pop < 0 || pop >= x->c.n_pop || !n_part) return PMC_ERR_INVALID_ARG;
  GUARD_BEGIN
  PopCtr r = read_ctr(x->c, pop);
  *n_part = r.n_live;
  return PMC_OK;
  GUARD_END
}

static int do_download(Ctx& c, int pop, int max_part, double* vol, int* group, int* cls, int64_t* id,
                       int* n_primary, int* n_comp, int* comp_source, double* comp_time, int* n_part) {
  PopHost& ph = c.pops[pop];
  PopCtr r = read_ctr(c, pop);
  if (n_part) *n_part = r.n_live;
  if (r.n_live > max_part) return PMC_ERR_CAPACITY;
  size_t ns = (size_t)r.n_slots + 1;
  size_t n = std::max(r.n_live, 1);
  c.st_l.reserve(ns + n);
  long long* off = c.st_l.p;
  long long nl = scan(c, ph.h.alive, r.n_slots, off, true);
  if (nl != r.n_live) return PMC_ERR_ASSERT;
  if (nl > 0 && nl == r.n_slots && !comp_source && !comp_time) {
    // no dead slots: the slot arrays already hold the particles in order,
    // in the caller's particle-major layout
    if (vol) CK(cudaMemcpyAsync(vol, ph.h.vol, sizeof(double) * nl * c.n_spec, cudaMemcpyDeviceToHost, c.stream));
    if (group) CK(cudaMemcpyAsync(group, ph.h.grp, sizeof(int) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (cls) CK(cudaMemcpyAsync(cls, ph.h.cls, sizeof(int) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (id) CK(cudaMemcpyAsync(id, ph.h.id, sizeof(long long) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (n_primary) CK(cudaMemcpyAsync(n_primary, ph.h.nprim, sizeof(int) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (n_comp) CK(cudaMemcpyAsync(n_comp, ph.h.ncomp, sizeof(int) * nl, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return PMC_OK;
  }
  c.st_d.reserve(n * (c.n_spec + kMaxComponent));
  c.st_i.reserve(n * (4 + kMaxComponent));
  long long* di = c.st_l.p + ns;
  double* dv = c.st_d.p;
  double* dct = c.st_d.p + n * c.n_spec;
  int* dg = c.st_i.p;
  int* dc = dg + n;
  int* dn = dc + n;
  int* dnc = dn + n;
  int* dcs = dnc + n;
  if (r.n_slots > 0)
    k_download<<<grid_for(r.n_slots, 256), 256, 0, c.stream>>>(
        ph.h, off, r.n_slots, vol ? dv : nullptr, group ? dg : nullptr, cls ? dc : nullptr, id ? di : nullptr,
        n_primary ? dn : nullptr, n_comp ? dnc : nullptr, comp_source ? dcs : nullptr,
        comp_time ? dct : nullptr);
  note_launch();
  if (nl > 0) {
    if (vol) CK(cudaMemcpyAsync(vol, dv, sizeof(double) * nl * c.n_spec, cudaMemcpyDeviceToHost, c.stream));
    if (group) CK(cudaMemcpyAsync(group, dg, sizeof(int) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (cls) CK(cudaMemcpyAsync(cls, dc, sizeof(int) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (id) CK(cudaMemcpyAsync(id, di, sizeof(long long) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (n_primary) CK(cudaMemcpyAsync(n_primary, dn, sizeof(int) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (n_comp) CK(cudaMemcpyAsync(n_comp, dnc, sizeof(int) * nl, cudaMemcpyDeviceToHost, c.stream));
    if (comp_source) CK(cudaMemcpyAsync(comp_source, dcs, sizeof(int) * nl * kMaxComponent, cudaMemcpyDeviceToHost, c.stream));
    if (comp_time) CK(cudaMemcpyAsync(comp_time, dct, sizeof(double) * nl * kMaxComponent, cudaMemcpyDeviceToHost, c.stream));
  }
  CK(cudaStreamSynchronize(c.stream));
  return PMC_OK;
}

// particles of population k per (group, class)
static std::vector<int> count_group_class(Ctx& c, int k) {
  PopHost& ph = c.pops[k];
  int ngc = c.n_group * c.n_class;
  c.st_i.reserve(ngc);
  CK(cudaMemsetAsync(c.st_i.p, 0, sizeof(int) * ngc, c.stream));
  PopCtr r = read_ctr(c, k);
  if (r.n_slots > 0) {
    k_count_group_class<<<grid_for(r.n_slots, 256), 256, 0, c.stream>>>(ph.h, c.st_i.p);
    note_launch();
  }
  std::vector<int> n(ngc);
  CK(cudaMemcpyAsync(n.data(), c.st_i.p, sizeof(int) * ngc, cudaMemcpyDeviceToHost, c.stream));
  CK(cudaStreamSynchronize(c.stream));
  return n;
}

// scale the weight magnitude of (g, c) of population k (aero_weight_scale);
// the population takes weights of its own
static void scale_weight(Ctx& c, int k, int g, int cl, double f) {
  PopHost& ph = c.pops[k];
  if (!ph.own_w) {
    ph.w = c.w;
    ph.own_w = true;
  }
  ph.w.mag[(g - 1) + kMaxGroup * (cl - 1)] *= f;
  ph.wver++;
  set_params(c, ph);
}

int pmc_coag_gpu_rebalance(pmc_coag_gpu_ctx* x, int pop, const double* n_part_ideal, int allow_doubling,
                           int allow_halving) {
  if (!x || pop < 0 || pop >= x->c.n_pop || !n_part_ideal) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  PopHost& ph = c.pops[pop];
  bool changed = false;
  if (allow_doubling)
    for (int g = 1; g <= c.n_group; g++)
      for (int cl = 1; cl <= c.n_class; cl++) {
        int idx = (g - 1) + c.n_group * (cl - 1);
        double ideal = n_part_ideal[idx];
        for (int it = 0; it < 64; it++) {
          int cnt = count_group_class(c, pop)[idx];
          if (!((double)cnt < ideal / 2.0 && cnt > 0)) break;
          PopCtr r = read_ctr(c, pop);
          long long need = (long long)r.n_slots + cnt;
          if (need > ph.h.cap)
            relayout(c, pop, (int)std::min<long long>(need * 3 / 2 + 1024, (1LL << 31) - 1), false);
          r = read_ctr(c, pop);
          size_t n = (size_t)r.n_slots;
          c.st_l.reserve(n + 1);
          c.flag.reserve(n + 1);
          if (c.dirty) push_pops(c);
          k_flag_group_class<<<grid_for(n, 256), 256, 0, c.stream>>>(ph.h, r.n_slots, g, cl, c.flag.p);
          note_launch();
          long long members = scan(c, c.flag.p, (long long)n, c.st_l.p, true);
          k_double<<<grid_for(n, 256), 256, 0, c.stream>>>(ph.h, r.n_slots, c.flag.p, c.st_l.p, r.next_id);
          note_launch();
          r.n_slots += (int)members;
          r.n_live += (int)members;
          r.next_id += members;
          write_ctr(c, pop, r);
          scale_weight(c, pop, g, cl, 0.5);
          changed = true;
        }
      }
  if (allow_halving) reserve_removal_logs(c);  // halving records its removals
  if (allow_halving)
    for (int g = 1; g <= c.n_group; g++)
      for (int cl = 1; cl <= c.n_class; cl++) {
        int idx = (g - 1) + c.n_group * (cl - 1);
        double ideal = n_part_ideal[idx];
        for (int it = 0; it < 64; it++) {
          int cnt = count_group_class(c, pop)[idx];
          if (!((double)cnt > ideal * 2.0)) break;
          push_pops(c);
          PopCtr r = read_ctr(c, pop);
          k_halve<<<grid_for(r.n_slots, 256), 256, 0, c.stream>>>(ph.h, g, cl, ph.rebalance_calls++);
          note_launch();
          scale_weight(c, pop, g, cl, 2.0);
          changed = true;
        }
      }
  if (changed) {
    ph.valid_sort = false;  // aero_state_double clears valid_sort; halving removed particles
    c.replay.valid = false;
    push_pops(c);
    CK(cudaStreamSynchronize(c.stream));
    PopCtr r = read_ctr(c, pop);
    ph.rm_count = r.n_removed;
    if (r.status) return r.status;
    if (ph.h.rm_on && r.n_removed > ph.h.rm_cap) return PMC_ERR_CAPACITY;
  }
  return PMC_OK;
  GUARD_END
}

// ---------------------------------------------------------------------------
// aero_state_add_aero_dist_sample (aero_state.F90:758-831) on the device

// One mode of the caller's distribution (aero_mode_t, aero_mode.F90:40-66)
struct HostMode {
  int type = 0;
  double char_radius = 0, log10_std = 0, num_conc = 0;
  int source = 1;
  int n_sample = 0;
  const double* sample_radius = nullptr;  // [n_sample + 1] (host)
  const double* sample_nc = nullptr;      // [n_sample] (host)
  long long r_off = 0;                    // offset of sample_radius in the device copy
};

// aero_mode_weighted_sampled_num_conc (aero_mode.F90:457-491).  Under a
// power weight of exponent 0 the reference's expression is 0/0; its limit,
// the unweighted concentration, is used.
static void weighted_sampled_num_conc(const HostMode& m, int w_type, double expo, std::vector<double>& out) {
  out.resize(m.n_sample);
  for (int i = 0; i < m.n_sample; i++) {
    if (w_type == kWeightNone || expo == 0.0) {
      out[i] = m.sample_nc[i];
      continue;
    }
    double x0 = log(m.sample_radius[i]), x1 = log(m.sample_radius[i + 1]);
    out[i] = m.sample_nc[i] / expo * (exp(-expo * x0) - exp(-expo * x1)) / (x1 - x0);
  }
}

// log10 of the weighted mode's median radius, x_mean_prime
// (aero_mode.F90:510-513, :574-577)
static double x_mean_prime(const HostMode& m, int w_type, double expo) {
  double x = log10(m.char_radius);
  if (w_type == kWeightNone) return x;
  return x - expo * (m.log10_std * m.log10_std) * log(10.0);
}

// aero_mode_number (aero_mode.F90:495-546): the mean number of computational
// particles per unit sample proportion under weight (w_type, mag, expo);
// wnc receives a sampled mode's weighted interval concentrations
static double mode_number(const HostMode& m, int w_type, double mag, double expo, std::vector<double>& wnc) {
  switch (m.type) {
    case kModeLogNormal: {
      if (w_type == kWeightNone) return m.num_conc / mag;
      double x = log10(m.char_radius), xp = x_mean_prime(m, w_type, expo);
      return m.num_conc / mag * exp((xp * xp - x * x) / (2.0 * (m.log10_std * m.log10_std)));
    }
    case kModeExp:
      if (w_type != kWeightNone) throw Fail(PMC_ERR_INVALID_ARG);  // die_msg(822252601)
      return m.num_conc / mag;
    case kModeMono:
      return m.num_conc / (w_type == kWeightNone ? mag : mag * fast_pow<double>(m.char_radius, expo));
    case kModeSampled: {
      weighted_sampled_num_conc(m, w_type, expo, wnc);
      double s = 0.0;
      for (double v : wnc) s = s + v;
      return s / mag;
    }
  }
  throw Fail(PMC_ERR_INVALID_ARG);
}

// aero_state_scale_weight (aero_state.F90:1859-1922) for (g, cl) of
// population k holding n members: returns the members after the call
static long long scale_weight_members(Ctx& c, int k, int g, int cl, long long n, double ratio, bool allow_doubling,
                                      bool allow_halving, Rng& hr, uint32_t call) {
  PopHost& ph = c.pops[k];
  if (ratio > 1.0 && (allow_halving || n == 0)) {
    scale_weight(c, k, g, cl, ratio);
    long long n_remove = prob_round(hr, (double)n * (1.0 - 1.0 / ratio));
    if (n_remove <= 0) return n;
    reserve_removal_logs(c);  // the removals are recorded (AERO_INFO_HALVED)
    if (c.dirty) push_pops(c);
    c.select_buf.reserve(sizeof(SelectState));
    SelectState* S = (SelectState*)c.select_buf.p;
    CK(cudaMemsetAsync(S, 0, sizeof(SelectState), c.stream));
    CK(cudaMemcpyAsync(&S->need, &n_remove, sizeof(long long), cudaMemcpyHostToDevice, c.stream));
    PopCtr r = read_ctr(c, k);
    int grid = grid_for(r.n_slots, 256);
    for (int shift = 48; shift >= 0; shift -= 16) {
      k_select_hist<<<grid, 256, 0, c.stream>>>(ph.h, g, cl, call, S, shift);
      note_launch();
      k_select_pick<<<1, 1024, 0, c.stream>>>(S, shift);
      note_launch();
    }
    k_select_remove<<<grid, 256, 0, c.stream>>>(ph.h, g, cl, call, S);
    note_launch();
    // the records kept so far, for a later growth of the log
    ph.rm_count = read_ctr(c, k).n_removed;
    return n - n_remove;
  }
  if (ratio < 1.0 && (allow_doubling || n == 0)) {
    scale_weight(c, k, g, cl, ratio);
    if (n == 0) return 0;
    if (c.dirty) push_pops(c);
    PopCtr r = read_ctr(c, k);
    size_t ns = (size_t)r.n_slots;
    c.dup_n.reserve(ns + 1);
    c.st_l.reserve(ns + 1);
    k_dup_count<<<grid_for(ns, 256), 256, 0, c.stream>>>(ph.h, r.n_slots, g, cl, 1.0 / ratio, call, c.dup_n.p);
    note_launch();
    long long copies = scan(c, c.dup_n.p, (long long)ns, c.st_l.p, true);
    if (copies > 0) {
      long long need = (long long)r.n_slots + copies;
      if (need > (1LL << 31) - 1) throw Fail(PMC_ERR_CAPACITY);
      if (need > ph.h.cap) {
        relayout(c, k, (int)std::min<long long>(need * 3 / 2 + 1024, (1LL << 31) - 1), false);
        push_pops(c);
      }
      k_dup_write<<<grid_for(ns, 256), 256, 0, c.stream>>>(ph.h, r.n_slots, c.dup_n.p, c.st_l.p, r.next_id);
      note_launch();
      r.n_slots += (int)copies;
      r.n_live += (int)copies;
      r.next_id += copies;
      write_ctr(c, k, r);
    }
    return n + copies;
  }
  return n;
}

int pmc_coag_gpu_add_dist_sample(pmc_coag_gpu_ctx* x, int pop, int n_mode, const int* mode_type,
                                 const double* char_radius, const double* log10_std, const double* num_conc,
                                 const double* vol_frac, const double* vol_frac_std, const int* source,
                                 const int* n_sample, const double* sample_radius, const double* sample_num_conc,
                                 double sample_prop, double characteristic_factor, double create_time,
                                 const double* n_part_ideal, int allow_doubling, int allow_halving,
                                 int64_t* n_part_add) {
  if (n_part_add) *n_part_add = 0;
  if (!x || pop < 0 || pop >= x->c.n_pop || n_mode < 0) return PMC_ERR_INVALID_ARG;
  if (n_mode > 0 && (!mode_type || !char_radius || !num_conc || !vol_frac)) return PMC_ERR_INVALID_ARG;
  if (!(sample_prop >= 0.0) || !(characteristic_factor > 0.0)) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  // the modes, checked as aero_mode_read and the samplers check them
  std::vector<HostMode> modes(n_mode);
  long long r_tot = 0, nc_tot = 0;
  for (int m = 0; m < n_mode; m++) {
    HostMode& h = modes[m];
    h.type = mode_type[m];
    h.char_radius = char_radius[m];
    h.log10_std = log10_std ? log10_std[m] : 0.0;
    h.num_conc = num_conc[m];
    h.source = source ? source[m] : m + 1;
    if (h.type < kModeLogNormal || h.type > kModeSampled || !(h.num_conc >= 0.0) || h.source < 1)
      return PMC_ERR_INVALID_ARG;
    if (c.n_class > 1 && h.source > c.n_class) return PMC_ERR_INVALID_ARG;  // assert(765048788)
    if (h.type == kModeLogNormal && (!log10_std || !(h.log10_std > 0.0) || !(h.char_radius > 0.0)))
      return PMC_ERR_INVALID_ARG;
    if ((h.type == kModeExp || h.type == kModeMono) && !(h.char_radius > 0.0)) return PMC_ERR_INVALID_ARG;
    if (h.type == kModeSampled) {
      if (!n_sample || !sample_radius || !sample_num_conc || n_sample[m] < 1) return PMC_ERR_INVALID_ARG;
      h.n_sample = n_sample[m];
      h.sample_radius = sample_radius + r_tot;
      h.sample_nc = sample_num_conc + nc_tot;
      h.r_off = r_tot;
      for (int i = 0; i <= h.n_sample; i++)
        if (!(h.sample_radius[i] > 0.0) || (i > 0 && !(h.sample_radius[i] > h.sample_radius[i - 1])))
          return PMC_ERR_INVALID_ARG;
      for (int i = 0; i < h.n_sample; i++)
        if (!(h.sample_nc[i] >= 0.0)) return PMC_ERR_INVALID_ARG;
      r_tot += h.n_sample + 1;
      nc_tot += h.n_sample;
    }
    for (int s = 0; s < c.n_spec; s++) {
      double f = vol_frac[m * c.n_spec + s], sd = vol_frac_std ? vol_frac_std[m * c.n_spec + s] : 0.0;
      if (!(f >= 0.0) || !(sd >= 0.0)) return PMC_ERR_INVALID_ARG;
    }
  }
  GUARD_BEGIN
  PopHost& ph = c.pops[pop];
  const uint32_t call = ph.sample_calls++;
  Rng hr(ph.seed, ph.step, sample_ctr(call, kSubHost), 0u);
  // device copies: fractions and their deviations per mode, the sampled
  // modes' radius edges, one weighted-concentration array per batch
  const int ns = c.n_spec;
  size_t n_vf = (size_t)n_mode * ns;
  std::vector<double> hbuf(2 * n_vf + (size_t)r_tot + (size_t)nc_tot * c.n_group + 1, 0.0);
  for (size_t i = 0; i < n_vf; i++) {
    hbuf[i] = vol_frac[i];
    hbuf[n_vf + i] = vol_frac_std ? vol_frac_std[i] : 0.0;
  }
  if (r_tot) std::memcpy(&hbuf[2 * n_vf], sample_radius, sizeof(double) * (size_t)r_tot);
  c.sample_buf.reserve(hbuf.size());
  double* d_vf = c.sample_buf.p;
  double* d_sr = d_vf + 2 * n_vf;
  double* d_wnc = d_sr + r_tot;
  std::vector<int> cnt = count_group_class(c, pop);
  {
    // room for the whole call at once: the batches' expected counts, with
    // the weight preparation run on expected values, plus a margin of 8
    // standard deviations (a larger draw grows the slots below)
    Weights w = ph.own_w ? ph.w : c.w;
    std::vector<double> est(cnt.begin(), cnt.end());
    double slots = 0.0, var = 0.0;
    std::vector<double> tmp;
    for (int g = 1; g <= c.n_group; g++)
      for (int m = 0; m < n_mode; m++) {
        int cl = c.n_class > 1 ? modes[m].source : 1;
        int kc = (g - 1) + c.n_group * (cl - 1), kw = (g - 1) + kMaxGroup * (cl - 1);
        double n_avg = sample_prop * mode_number(modes[m], w.type[kw], w.mag[kw], w.expo[kw], tmp);
        if (n_part_ideal) {
          double n_new = est[kc] + n_avg, ideal = n_part_ideal[kc];
          if (n_new != 0.0 && (n_new < ideal / 2.0 || n_new > ideal * 2.0)) {
            double ratio = n_new / ideal;
            bool halve = ratio > 1.0 && (allow_halving || est[kc] == 0.0);
            bool dbl = ratio < 1.0 && (allow_doubling || est[kc] == 0.0);
            if (halve || dbl) {
              if (dbl) slots += est[kc] * (1.0 / ratio - 1.0);
              est[kc] /= ratio;
              w.mag[kw] *= ratio;
            }
          }
        }
        if (n_avg == 0.0) continue;
        n_avg = sample_prop * mode_number(modes[m], w.type[kw], w.mag[kw], w.expo[kw], tmp);
        est[kc] += n_avg;
        slots += n_avg;
        var += n_avg;
      }
    PopCtr r = read_ctr(c, pop);
    double need = (double)r.n_slots + slots + 8.0 * std::sqrt(var) + 1024.0;
    if (need > (double)ph.h.cap && need < (double)((1LL << 31) - 1)) relayout(c, pop, (int)need, false);
  }
  long long wnc_used = 0, added = 0;
  uint32_t idx = 0;
  std::vector<double> wnc;
  for (int g = 1; g <= c.n_group; g++)
    for (int m = 0; m < n_mode; m++) {
      const HostMode& h = modes[m];
      int cl = c.n_class > 1 ? h.source : 1;  // aero_state_weight_class_for_source, aero_state.F90:263-282
      int kc = (g - 1) + c.n_group * (cl - 1);
      int kw = (g - 1) + kMaxGroup * (cl - 1);
      const Weights& W0 = ph.own_w ? ph.w : c.w;
      double n_avg = sample_prop * mode_number(h, W0.type[kw], W0.mag[kw], W0.expo[kw], wnc);
      if (n_part_ideal) {
        // aero_state_prepare_weight_for_add (aero_state.F90:704-752)
        double n_new = (double)cnt[kc] + n_avg;
        double ideal = n_part_ideal[kc];
        if (n_new != 0.0 && (n_new < ideal / 2.0 || n_new > ideal * 2.0))
          cnt[kc] = (int)scale_weight_members(c, pop, g, cl, cnt[kc], n_new / ideal, allow_doubling != 0,
                                              allow_halving != 0, hr, call);
      }
      if (n_avg == 0.0) continue;
      const Weights& W = ph.own_w ? ph.w : c.w;
      int wt = W.type[kw];
      double mag = W.mag[kw], expo = W.expo[kw];
      n_avg = sample_prop * mode_number(h, wt, mag, expo, wnc);
      int n = rand_poisson(hr, n_avg);
      if (n < 0) throw Fail(PMC_ERR_CAPACITY);
      double size_factor = std::min(1.0 / (characteristic_factor * n_avg), 0.32);
      added += n;
      if (n == 0) continue;
      PopCtr r = read_ctr(c, pop);
      long long need = (long long)r.n_slots + n;
      if (need > (1LL << 31) - 1) throw Fail(PMC_ERR_CAPACITY);
      if (need > ph.h.cap) relayout(c, pop, (int)std::min<long long>(need * 3 / 2 + 1024, (1LL << 31) - 1), false);
      SampleBatch B{};
      B.n = n;
      B.type = h.type;
      B.group = g;
      B.cls = cl;
      B.w_type = wt;
      B.w_mag = mag;
      B.w_expo = expo;
      B.log10_std = h.log10_std;
      B.x_mean = h.type == kModeLogNormal ? x_mean_prime(h, wt, expo) : 0.0;
      B.threshold = size_factor;
      B.char_radius = h.char_radius;
      B.char_vol = rad2vol(c.frac, h.char_radius);
      B.n_sample = h.n_sample;
      B.sample_radius = d_sr + h.r_off;
      if (h.type == kModeSampled) {
        std::memcpy(&hbuf[2 * n_vf + r_tot + wnc_used], wnc.data(), sizeof(double) * wnc.size());
        B.wnc = d_wnc + wnc_used;
        wnc_used += (long long)wnc.size();
      }
      B.vol_frac = d_vf + (size_t)m * ns;
      B.vol_frac_std = d_vf + n_vf + (size_t)m * ns;
      B.any_std = 0;
      for (int s = 0; s < ns; s++)
        if (hbuf[n_vf + (size_t)m * ns + s] > 0.0) B.any_std = 1;
      B.source = h.source;
      B.create_time = create_time;
      // the whole staging array is copied before every batch: it is small,
      // and the batch's weighted concentrations were just written into it
      CK(cudaMemcpyAsync(c.sample_buf.p, hbuf.data(), sizeof(double) * hbuf.size(), cudaMemcpyHostToDevice,
                         c.stream));
      if (c.dirty) push_pops(c);
      k_sample_batch<<<grid_for(n, 256), 256, 0, c.stream>>>(ph.h, B, r.n_slots, r.next_id, call, idx);
      note_launch();
      idx += (uint32_t)n;
      r.n_slots += n;
      r.n_live += n;
      r.next_id += n;
      write_ctr(c, pop, r);
      cnt[kc] += n;
    }
  ph.valid_sort = false;
  ph.caches_valid = false;
  c.replay.valid = false;
  push_pops(c);
  CK(cudaStreamSynchronize(c.stream));
  PopCtr r = read_ctr(c, pop);
  ph.rm_count = r.n_removed;
  if (n_part_add) *n_part_add = added;
  if (r.status) return r.status;
  if (ph.h.rm_on && r.n_removed > ph.h.rm_cap) return PMC_ERR_CAPACITY;
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_size_dist(pmc_coag_gpu_ctx* x, int pop, int n_bin, double d_min, double d_max, double* num_dist,
                           double* mass_dist) {
  if (!x || pop < 0 || pop >= x->c.n_pop || n_bin < 1 || !(d_min > 0.0) || !(d_max > d_min) || !num_dist)
    return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  size_t nv = (size_t)n_bin * (1 + c.n_spec);
  if (nv * sizeof(double) > 96 * 1024) return PMC_ERR_CAPACITY;  // the per-block histogram lives in shared memory
  GUARD_BEGIN
  PopHost& ph = c.pops[pop];
  c.st_d.reserve(nv);
  CK(cudaMemsetAsync(c.st_d.p, 0, sizeof(double) * nv, c.stream));
  PopCtr r = read_ctr(c, pop);
  if (r.n_slots > 0) {
    size_t smem = sizeof(double) * nv;
    if (smem > 48 * 1024)
      CK(cudaFuncSetAttribute(k_size_dist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_size_dist<<<std::min(grid_for(r.n_slots, 256), 148 * 4), 256, smem, c.stream>>>(
        ph.h, n_bin, log(d_min), log(d_max), (double)n_bin / (log(d_max) - log(d_min)), c.st_d.p);
    note_launch();
  }
  CK(cudaMemcpyAsync(num_dist, c.st_d.p, sizeof(double) * n_bin, cudaMemcpyDeviceToHost, c.stream));
  if (mass_dist)
    CK(cudaMemcpyAsync(mass_dist, c.st_d.p + n_bin, sizeof(double) * n_bin * c.n_spec, cudaMemcpyDeviceToHost,
                       c.stream));
  CK(cudaStreamSynchronize(c.stream));
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_get_weight(pmc_coag_gpu_ctx* x, int pop, double* w_mag) {
  if (!x || pop < 0 || pop >= x->c.n_pop || !w_mag) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  const Weights& w = c.pops[pop].own_w ? c.pops[pop].w : c.w;
  for (int cl = 0; cl < c.n_class; cl++)
    for (int g = 0; g < c.n_group; g++) w_mag[g + c.n_group * cl] = w.mag[g + kMaxGroup * cl];
  return PMC_OK;
}

int pmc_coag_gpu_sync_host(pmc_coag_gpu_ctx* x, int pop, int cap, double* vol, int* group, int* cls,
                           int64_t* id, int* n_primary, uint8_t* alive, int* n_slots, int* n_changed, int* full) {
  if (!x || pop < 0 || pop >= x->c.n_pop || cap < 0 || !vol || !group || !cls || !id || !n_primary || !alive)
    return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  PopHost& ph = c.pops[pop];
  PopCtr r = read_ctr(c, pop);
  if (n_slots) *n_slots = r.n_slots;
  if (r.n_slots > cap) return PMC_ERR_CAPACITY;
  int ns = c.n_spec;
  if (full && *full) ph.mirror_full = true;  // the caller asks for every slot (new arrays)
  if (ph.mirror_full) {
    // every slot: the slot arrays already have the host layout
    size_t n = (size_t)r.n_slots;
    if (n > 0) {
      CK(cudaMemcpyAsync(vol, ph.h.vol, sizeof(double) * n * ns, cudaMemcpyDeviceToHost, c.stream));
      CK(cudaMemcpyAsync(group, ph.h.grp, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
      CK(cudaMemcpyAsync(cls, ph.h.cls, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
      CK(cudaMemcpyAsync(id, ph.h.id, sizeof(long long) * n, cudaMemcpyDeviceToHost, c.stream));
      CK(cudaMemcpyAsync(n_primary, ph.h.nprim, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
      CK(cudaMemcpyAsync(alive, ph.h.alive, n, cudaMemcpyDeviceToHost, c.stream));
    }
    CK(cudaMemsetAsync(ph.h.changed, 0, ph.h.cap, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if ((size_t)cap > n) memset(alive + n, 0, (size_t)cap - n);
    ph.mirror_full = false;
    ph.mirror_slots = r.n_slots;
    if (n_changed) *n_changed = r.n_slots;
    if (full) *full = 1;
    return PMC_OK;
  }
  int range = std::max(ph.mirror_slots, r.n_slots);
  if (range > ph.h.cap) range = ph.h.cap;
  long long total = 0;
  if (range > 0) {
    // pack the changed slots into records that the device writes straight
    // into page-locked host memory (room for every slot of the range), so
    // the records cross the bus while the kernel runs.  The range goes in
    // up to four chunks: after each, a copy of the running record count and
    // an event, so the host scatters one chunk's records while the device
    // packs the next
    const int rec = (kSyncHead + 8 * ns + 15) & ~15;  // keeps every record's header 16-byte aligned
    c.map.reserve((size_t)range * rec);
    c.st_cnt.reserve(1);
    c.pin.reserve(64);
    for (auto& ev : c.sync_ev)
      if (!ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    const int n_chunk = range >= (1 << 18) ? 4 : 1;
    const int wpb = std::max(1, std::min(4, (int)(48 * 1024 / (32 * rec))));  // warps per block
    const size_t smem = (size_t)wpb * 32 * rec;
    unsigned long long* h_cnt = (unsigned long long*)c.pin.p;
    const unsigned char* h_rec = (const unsigned char*)c.map.p;
    CK(cudaMemsetAsync(c.st_cnt.p, 0, sizeof(unsigned long long), c.stream));
    for (int k = 0; k < n_chunk; k++) {
      const int lo = (int)((long long)range * k / n_chunk), hi = (int)((long long)range * (k + 1) / n_chunk);
      k_pack_changed<<<grid_for(hi - lo, 32 * wpb), 32 * wpb, smem, c.stream>>>(ph.h, lo, hi, c.st_cnt.p,
                                                                                (unsigned char*)c.map.dev, rec);
      note_launch();
      CK(cudaMemcpyAsync(h_cnt + k, c.st_cnt.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.stream));
      CK(cudaEventRecord(c.sync_ev[k], c.stream));
    }
    // scatter each chunk's records into the caller's slot-indexed arrays
    long long j0 = 0;
    const int n_thr = (int)std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
    if (!c.pool) c.pool.reset(new HostPool());
    for (int k = 0; k < n_chunk; k++) {
      CK(cudaEventSynchronize(c.sync_ev[k]));
      const long long j1 = (long long)h_cnt[k];
      const long long nk = j1 - j0;
      const std::function<void(int, int)> work = [&](int q, int nq) {
        const long long a1 = j0 + nk * (q + 1) / nq;
        for (long long j = j0 + nk * q / nq; j < a1; j++) {
          const unsigned char* e = h_rec + (size_t)j * rec;
          const int* hd = (const int*)e;
          const int sl = hd[0];
          alive[sl] = (uint8_t)hd[1];
          if (!hd[1]) continue;
          group[sl] = hd[2];
          cls[sl] = hd[3];
          n_primary[sl] = hd[4];
          memcpy(&id[sl], e + 24, sizeof(long long));
          memcpy(vol + (size_t)sl * ns, e + kSyncHead, sizeof(double) * ns);
        }
      };
      c.pool->run(nk > 4096 ? n_thr : 1, work);
      j0 = j1;
    }
    total = j0;
  }
  ph.mirror_slots = r.n_slots;
  if (n_changed) *n_changed = (int)total;
  if (full) *full = 0;
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_download(pmc_coag_gpu_ctx* x, int pop, int max_part, double* vol, int* group, int* cls,
                          int64_t* id, int* n_primary, int* n_part) {
  if (!x || pop < 0 || pop >= x->c.n_pop) return PMC_ERR_INVALID_ARG;
  GUARD_BEGIN
  return do_download(x->c, pop, max_part, vol, group, cls, id, n_primary, nullptr, nullptr, nullptr, n_part);
  GUARD_END
}

int pmc_coag_gpu_download_components(pmc_coag_gpu_ctx* x, int pop, int max_part, int* n_comp,
                                     int* comp_source, double* comp_create_time) {
  if (!x || pop < 0 || pop >= x->c.n_pop) return PMC_ERR_INVALID_ARG;
  GUARD_BEGIN
  return do_download(x->c, pop, max_part, nullptr, nullptr, nullptr, nullptr, nullptr, n_comp,
                     comp_source, comp_create_time, nullptr);
  GUARD_END
}

int pmc_coag_gpu_set_weight(pmc_coag_gpu_ctx* x, const int* w_type, const double* w_mag,
                            const double* w_exp) {
  if (!x || !w_type || !w_mag || !w_exp) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  for (int cl = 0; cl < c.n_class; cl++)
    for (int g = 0; g < c.n_group; g++) {
      int src = g + c.n_group * cl, dst = g + kMaxGroup * cl;
      if (w_type[src] < 1 || w_type[src] > 3) return PMC_ERR_INVALID_ARG;
      c.w.type[dst] = w_type[src];
      c.w.mag[dst] = w_mag[src];
      c.w.expo[dst] = w_exp[src];
    }
  c.wver++;
  for (auto& ph : c.pops) {
    if (!ph.own_w) ph.wver++;  // populations with weights of their own keep them
    set_params(c, ph);
    ph.valid_sort = false;  // aero_state_set_weight clears valid_sort
  }
  c.replay.valid = false;
  push_pops(c);
  CK(cudaStreamSynchronize(c.stream));
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_set_fractal(pmc_coag_gpu_ctx* x, double frac_dim, double prime_radius, double vol_fill_factor) {
  // spec_file_read_fractal stops for d_f > 3 (fractal.F90:587); d_f, R0 and
  // f also divide or take roots, so each must be positive
  if (!x || !(frac_dim > 0.0 && frac_dim <= 3.0) || !(prime_radius > 0.0) || !(vol_fill_factor > 0.0))
    return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  c.frac = make_fractal(frac_dim, prime_radius, vol_fill_factor);
  // radii, records, grid and k_max bounds all follow the particle shape
  for (auto& ph : c.pops) {
    ph.h.benv = brown_env(ph.h.temp > 0.0 ? ph.h.temp : 288.0, ph.h.pressure > 0.0 ? ph.h.pressure : 1e5, c.frac);
    ph.wver++;
    ph.valid_sort = false;
    ph.h.kmax_valid = 0;
    ph.h.pair_setup_valid = 0;
  }
  c.replay.valid = false;
  c.dirty = true;
  push_pops(c);
  CK(cudaStreamSynchronize(c.stream));
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_set_weight_pop(pmc_coag_gpu_ctx* x, int pop, const int* w_type, const double* w_mag,
                                const double* w_exp) {
  if (!x || pop < 0 || pop >= x->c.n_pop || !w_type || !w_mag || !w_exp) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  PopHost& ph = c.pops[pop];
  Weights w = c.w;
  for (int cl = 0; cl < c.n_class; cl++)
    for (int g = 0; g < c.n_group; g++) {
      int src = g + c.n_group * cl, dst = g + kMaxGroup * cl;
      if (w_type[src] < 1 || w_type[src] > 3) return PMC_ERR_INVALID_ARG;
      w.type[dst] = w_type[src];
      w.mag[dst] = w_mag[src];
      w.expo[dst] = w_exp[src];
    }
  ph.w = w;
  ph.own_w = true;
  ph.wver++;  // only this population's caches go stale
  set_params(c, ph);
  ph.valid_sort = false;
  c.replay.valid = false;
  push_pops(c);
  CK(cudaStreamSynchronize(c.stream));
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_set_next_id(pmc_coag_gpu_ctx* x, int pop, int64_t next_id) {
  if (!x || pop < 0 || pop >= x->c.n_pop) return PMC_ERR_INVALID_ARG;
  GUARD_BEGIN
  PopCtr r = read_ctr(x->c, pop);
  r.next_id = next_id;
  write_ctr(x->c, pop, r);
  CK(cudaStreamSynchronize(x->c.stream));
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_get_next_id(pmc_coag_gpu_ctx* x, int pop, int64_t* next_id) {
  if (!x || pop < 0 || pop >= x->c.n_pop || !next_id) return PMC_ERR_INVALID_ARG;
  GUARD_BEGIN
  *next_id = read_ctr(x->c, pop).next_id;
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_set_seed(pmc_coag_gpu_ctx* x, int pop, uint64_t seed) {
  if (!x || pop < 0 || pop >= x->c.n_pop) return PMC_ERR_INVALID_ARG;
  PopHost& ph = x->c.pops[pop];
  ph.seed = seed;
  ph.h.seed = seed;
  ph.step = 0;  // the population's streams start again at step 1
  x->c.dirty = true;
  return PMC_OK;
}

int pmc_coag_gpu_set_graphs(pmc_coag_gpu_ctx* x, int enable) {
  if (!x || (enable != 0 && enable != 1)) return PMC_ERR_INVALID_ARG;
  x->c.use_graph = enable == 1;
  return PMC_OK;
}

int pmc_coag_gpu_set_mode(pmc_coag_gpu_ctx* x, int mode) {
  if (!x || mode < PMC_MODE_FP64 || mode > PMC_MODE_REPLAY) return PMC_ERR_INVALID_ARG;
  x->c.mode = mode;
  for (auto& ph : x->c.pops) ph.valid_sort = ph.valid_sort && mode != PMC_MODE_REPLAY;
  return PMC_OK;
}

int pmc_coag_gpu_replay_set(pmc_coag_gpu_ctx* x, const double* u, int64_t n) {
  if (!x || (n > 0 && !u) || n < 0) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  c.replay_u.reserve((size_t)std::max<int64_t>(n, 1));
  if (n > 0) CK(cudaMemcpy(c.replay_u.p, u, sizeof(double) * n, cudaMemcpyHostToDevice));
  c.replay_n = n;
  c.replay_used = 0;
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_replay_open(pmc_coag_gpu_ctx* x, const char* path) {
  if (!x || !path) return PMC_ERR_INVALID_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return PMC_ERR_INVALID_ARG;
  std::vector<double> u;
  double buf[4096];
  size_t m;
  while ((m = fread(buf, sizeof(double), 4096, f)) > 0) u.insert(u.end(), buf, buf + m);
  fclose(f);
  return pmc_coag_gpu_replay_set(x, u.data(), (int64_t)u.size());
}

int pmc_coag_gpu_replay_used(pmc_coag_gpu_ctx* x, int64_t* n_used) {
  if (!x || !n_used) return PMC_ERR_INVALID_ARG;
  *n_used = x->c.replay_used;
  return PMC_OK;
}

int pmc_coag_gpu_stats(pmc_coag_gpu_ctx* x, int64_t* kmax_violations, int64_t* redraws, int64_t* rounds) {
  if (!x) return PMC_ERR_INVALID_ARG;
  if (kmax_violations) *kmax_violations = x->c.last_kmax_warn;
  if (redraws) *redraws = x->c.last_redraws;
  if (rounds) *rounds = x->c.last_rounds;
  return PMC_OK;
}

int pmc_coag_gpu_exact_tests(pmc_coag_gpu_ctx* x, int64_t* n) {
  if (!x || !n) return PMC_ERR_INVALID_ARG;
  *n = x->c.exact_tests;
  return PMC_OK;
}

int pmc_coag_gpu_set_record_removals(pmc_coag_gpu_ctx* x, int enable) {
  if (!x) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  for (auto& ph : c.pops) ph.h.rm_on = enable ? 1 : 0;
  reserve_removal_logs(c);
  push_pops(c);
  CK(cudaStreamSynchronize(c.stream));
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_removals(pmc_coag_gpu_ctx* x, int pop, int64_t max_n, int64_t* id, int* action,
                          int64_t* other_id, int64_t* n) {
  if (!x || pop < 0 || pop >= x->c.n_pop || max_n < 0 || !n || (max_n > 0 && (!id || !action || !other_id)))
    return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  PopHost& ph = c.pops[pop];
  PopCtr r = read_ctr(c, pop);
  *n = r.n_removed;
  ph.rm_count = r.n_removed;
  if (r.n_removed > ph.h.rm_cap && ph.h.rm_on) return PMC_ERR_CAPACITY;  // records were dropped
  if (r.n_removed > max_n) return PMC_ERR_CAPACITY;                     // nothing copied or cleared
  if (r.n_removed > 0) {
    std::vector<RemovalRec> h((size_t)r.n_removed);
    CK(cudaMemcpyAsync(h.data(), ph.h.rm_log, sizeof(RemovalRec) * h.size(), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    for (size_t k = 0; k < h.size(); k++) {
      id[k] = h[k].id;
      action[k] = h[k].action;
      other_id[k] = h[k].other_id;
    }
  }
  r.n_removed = 0;
  write_ctr(c, pop, r);
  ph.rm_count = 0;
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_profile(pmc_coag_gpu_ctx* x, int enable) {
  if (!x) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  prof_collect(c);
  c.prof = enable != 0;
  for (int i = 0; i < 4; i++) {
    c.prof_ms[i] = 0.0;
    c.prof_launch[i] = c.prof_units[i] = 0;
  }
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_profile_read(pmc_coag_gpu_ctx* x, int which, double* total_ms, int64_t* launches,
                              int64_t* units) {
  if (!x || which < 0 || which > 3) return PMC_ERR_INVALID_ARG;
  prof_collect(x->c);
  if (total_ms) *total_ms = x->c.prof_ms[which];
  if (launches) *launches = x->c.prof_launch[which];
  if (units) *units = x->c.prof_units[which];
  return PMC_OK;
}

int pmc_coag_gpu_launch_count(int64_t* n) {
  if (!n) return PMC_ERR_INVALID_ARG;
  *n = g_launches;
  return PMC_OK;
}

int pmc_coag_gpu_conflicts(pmc_coag_gpu_ctx* x, int64_t* events, int64_t* event_losers,
                           int64_t* target_ops, int64_t* target_op_losers) {
  if (!x) return PMC_ERR_INVALID_ARG;
  if (events) *events = x->c.last_events;
  if (event_losers) *event_losers = x->c.last_set_losers;
  if (target_ops) *target_ops = x->c.last_ops;
  if (target_op_losers) *target_op_losers = x->c.last_pp_lost;
  return PMC_OK;
}

int pmc_coag_gpu_sort(pmc_coag_gpu_ctx* x, int pop, int* n_bin, double* edges, int max_bin, int* counts,
                      int* bins) {
  if (!x || pop < 0 || pop >= x->c.n_pop) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  sort_pops(c, true);
  CK(cudaStreamSynchronize(c.stream));
  PopHost& ph = c.pops[pop];
  if (n_bin) *n_bin = ph.n_bin;
  if (ph.n_bin > max_bin) return PMC_ERR_CAPACITY;
  if (edges && ph.n_bin > 0) memcpy(edges, ph.edges.data(), sizeof(double) * (ph.n_bin + 1));
  if (counts && ph.n_bin > 0)
    CK(cudaMemcpy(counts, ph.h.cell_count, sizeof(int) * ph.n_bin * c.n_class, cudaMemcpyDeviceToHost));
  if (bins) {
    PopCtr r = read_ctr(c, pop);
    std::vector<int> b(std::max(r.n_slots, 1));
    std::vector<uint8_t> a(std::max(r.n_slots, 1));
    if (r.n_slots > 0) {
      CK(cudaMemcpy(b.data(), ph.h.cell, sizeof(int) * r.n_slots, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(a.data(), ph.h.alive, r.n_slots, cudaMemcpyDeviceToHost));
    }
    int j = 0;
    for (int i = 0; i < r.n_slots; i++)
      if (a[i]) bins[j++] = (b[i] >= 0 && ph.n_bin > 0) ? b[i] % ph.n_bin + 1 : 0;
  }
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_kmax_table(pmc_coag_gpu_ctx* x, int kernel_type, double temp, double pressure,
                            double additive_coeff, double* kmax, int max_bin) {
  if (!x || !kmax) return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  PopHost& ph = c.pops[0];
  if (ph.n_bin > max_bin) return PMC_ERR_CAPACITY;
  ph.h.kernel_type = kernel_type;
  ph.h.temp = temp;
  ph.h.pressure = pressure;
  ph.h.coeff = additive_coeff;
  ph.h.benv = brown_env(temp, pressure, c.frac);
  ph.h.kmax_valid = 0;
  push_pops(c);
  int nb = std::max(ph.n_bin, 1);
  dim3 g((nb * nb + 255) / 256, c.n_pop);
  k_kmax_table<<<g, 256, 0, c.stream>>>(c.d_pops); note_launch();
  CK(cudaStreamSynchronize(c.stream));
  CK(cudaGetLastError());
  if (ph.n_bin > 0) CK(cudaMemcpy(kmax, ph.h.kmax_tab, sizeof(double) * ph.n_bin * ph.n_bin, cudaMemcpyDeviceToHost));
  ph.h.kmax_valid = 1;
  push_pops(c);
  return PMC_OK;
  GUARD_END
}

int pmc_coag_gpu_eval_kernel(pmc_coag_gpu_ctx* x, int kernel_type, double temp, double pressure,
                             double additive_coeff, int n_pairs, const double* vol1, const int* c1,
                             const double* vol2, const int* c2, const int* c_ij, double* k_out) {
  if (!x || n_pairs < 0 || (n_pairs > 0 && (!vol1 || !vol2 || !c1 || !c2 || !c_ij || !k_out)))
    return PMC_ERR_INVALID_ARG;
  Ctx& c = x->c;
  GUARD_BEGIN
  if (n_pairs == 0) return PMC_OK;
  PopDev P = c.pops[0].h;
  P.kernel_type = kernel_type;
  P.temp = temp;
  P.pressure = pressure;
  P.coeff = additive_coeff;
  P.benv = brown_env(temp, pressure, c.frac);
  std::vector<void*> tmp;
  size_t nv = (size_t)n_pairs * c.n_spec;
  double* d1 = dalloc<double>(tmp, nv);
  double* d2 = dalloc<double>(tmp, nv);
  int* e1 = dalloc<int>(tmp, n_pairs);
  int* e2 = dalloc<int>(tmp, n_pairs);
  int* e3 = dalloc<int>(tmp, n_pairs);
  double* out = dalloc<double>(tmp, n_pairs);
  CK(cudaMemcpy(d1, vol1, sizeof(double) * nv, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d2, vol2, sizeof(double) * nv, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e1, c1, sizeof(int) * n_pairs, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e2, c2, sizeof(int) * n_pairs, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e3, c_ij, sizeof(int) * n_pairs, cudaMemcpyHostToDevice));
  k_eval_kernel<<<(n_pairs + 127) / 128, 128, 0, c.stream>>>(P, n_pairs, d1, e1, d2, e2, e3, out,
                                                             c.mode == PMC_MODE_MIXED ? 1 : 0); note_launch();
  CK(cudaStreamSynchronize(c.stream));
  CK(cudaGetLastError());
  CK(cudaMemcpy(k_out, out, sizeof(double) * n_pairs, cudaMemcpyDeviceToHost));
  free_list(tmp);
  return PMC_OK;
  GUARD_END
}

}  // extern "C"
