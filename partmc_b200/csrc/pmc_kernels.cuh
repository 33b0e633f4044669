// pmc_kernels.cuh -- kernels of the parallel coagulation step.
//
// One step of mc_coag (coagulation.F90:43-96) runs as rounds.  Round 0:
//   sort      stable counting sort of live slots into (bin, class) cells,
//             with each particle's pair-test record written in cell order
//             (aero_state_sort / aero_sorted_sort_particles,
//             aero_sorted.F90:185-373);
//   k bounds  the n_bin x n_bin k_max table when the grid changed
//             (est_k_minmax_binned_unweighted, coag_kernel.F90:253-280);
//   pairs     one thread per bin pair: destination class, f_max, k_max,
//             path choice and the Poisson number of samples
//             (mc_coag_for_bin / compute_n_samp, coagulation.F90:101-145,
//             648-702);
//   tests     one thread per sample: random pair, weighted kernel, accept
//             (maybe_coag_pair / find_rand_pair, coagulation.F90:712-803);
//             an accepted sample claims both particles with atomicMin of its
//             priority (its position in the reference's loop order);
//   resolve   an accepted sample that holds both claims is applied
//             (coagulate / coagulate_weighting, coagulation.F90:810-985).
// Later rounds (k_items, one thread per event of the round before) carry on
// the sequential loop's order:
//   - an event that lost a claim is retried unchanged if neither of its
//     particles was consumed, and dropped if one was: in the sequential loop
//     a test never meets a particle that an earlier event removed, so the
//     step-start samples that would have are thinned away;
//   - a particle that an event created or changed walks the pairs after the
//     event's pair that contain its cell, with Poisson tests against members
//     of the other cell at rate k_max * del_t per member, as the later pairs'
//     samples of the sequential loop would test it; its accepted tests are
//     the next events (a chain of them when each absorbs the partner).
// The step ends when a round has no events.
#pragma once

#include <cuda_runtime.h>

#include "pmc_physics.cuh"
#include <cooperative_groups.h>

#include "pmc_state.cuh"

namespace pmc {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kChunk = 2048;  // slots per sort block
constexpr int kWarpSlots = kChunk / kSortWarps;

enum Stream : uint32_t {
  kStreamPair = 1,
  kStreamTest = 2,
  kStreamMerge = 3,
  kStreamPart = 4,
  kStreamHalve = 5,  // aero_state_halve draws, keyed by the rebalance call and the slot
  kStreamWalk = 6,   // a walk's tests, keyed by the round and the walking slot
  kStreamChain = 7,  // merge of a chain's event i >= 2, keyed by i, the round and the walking slot
};

__device__ __forceinline__ void set_status(PopCtr* c, int code) { atomicCAS(&c->status, 0, code); }

// a capacity limit hit on the device: the status and the first site
__device__ __forceinline__ void cap_fail(PopCtr* c, int site) {
  atomicCAS(&c->cap_site, 0, site);
  set_status(c, kErrCapacity);
}

// a failed bounds check: record the first site and index, flag the step
__device__ __noinline__ void bad_index(PopCtr* c, int site, long long idx) {
  if (atomicCAS(&c->bad_site, 0, site) == 0) c->bad_index = idx;
  set_status(c, kErrAssert);
}

// the chunk histogram of the current slot count fits its allocation
__device__ __forceinline__ bool chunk_hist_fits(const PopDev& P, int n_chunks) {
  if ((long long)n_chunks * P.n_cells <= (long long)P.chunk_hist_len) return true;
  bad_index(P.ctr, kBadChunkHist, (long long)n_chunks * P.n_cells);
  return false;
}

__device__ __forceinline__ void add_ll(long long* p, long long v) {
  atomicAdd((unsigned long long*)p, (unsigned long long)v);
}
__device__ __forceinline__ void add_ll(int* p, long long v) { atomicAdd(p, (int)v); }


// add_ll for counters that many threads of a launch bump: the converged
// lanes that add to the same counter sum their values (|v| small) and one of
// them adds the sum, so a warp makes one atomic per counter instead of 32
__device__ __forceinline__ void add_ll_warp(long long* p, int v) {
  const unsigned peers = __match_any_sync(__activemask(), (unsigned long long)p);
  const int sum = (int)__reduce_add_sync(peers, (unsigned)v);
  if ((int)(threadIdx.x & 31) == __ffs(peers) - 1 && sum != 0)
    atomicAdd((unsigned long long*)p, (unsigned long long)(long long)sum);
}
// atomicAdd(p, 1) with the old value, one atomic for the converged lanes
// that bump the same counter: each gets the old value plus its rank
__device__ __forceinline__ unsigned long long inc_warp(unsigned long long* p) {
  const unsigned peers = __match_any_sync(__activemask(), (unsigned long long)p);
  const int lane = (int)(threadIdx.x & 31), leader = __ffs(peers) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(p, (unsigned long long)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + (unsigned long long)__popc(peers & ((1u << lane) - 1u));
}
__device__ __forceinline__ void add_ll_warp(int* p, int v) {
  const unsigned peers = __match_any_sync(__activemask(), (unsigned long long)p);
  const int sum = (int)__reduce_add_sync(peers, (unsigned)v);
  if ((int)(threadIdx.x & 31) == __ffs(peers) - 1 && sum != 0) atomicAdd(p, sum);
}

// sort chunks covering the population's slots (the slot count lives on the
// device and grows inside a step)
__device__ __forceinline__ int n_chunks_of(const PopDev& P) {
  return (P.ctr->n_slots + kChunk - 1) / kChunk;
}

__device__ __forceinline__ Rng make_rng(const PopDev& P, uint32_t stream, uint32_t p, uint32_t s) {
  return Rng(P.seed, P.step, (p << 12) | ((*P.round_p & 0xffu) << 4) | stream, s);
}

// ---------------------------------------------------------------------------
// block-wide exclusive scan of one int per thread (blockDim <= 1024)
__device__ int block_excl_scan(int v, int* total) {
  __shared__ int ws[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  if (wid == 0) {
    int s = lane < nw ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    ws[lane] = s;
  }
  __syncthreads();
  int pre = (wid > 0 ? ws[wid - 1] : 0) + x - v;
  if (total) *total = ws[nw - 1];
  __syncthreads();
  return pre;
}

// pair-test record of a particle of radius r, total volume v, mass m and
// class cls (1-based) (see RecD)
__device__ __forceinline__ RecD make_rec_v(const PopDev& P, double r, double v, double m, int cls) {
  RecD q;
  const Fractal& F = P.benv.frac;
  bool ok = true;
  q.r = r;
  q.rv = rad2vol(F, r);
  q.nc = num_conc_at_radius<double>(P.w, cls - 1, r);
  q.a = q.b = q.c = 0.0;
  switch (P.kernel_type) {
    case kKernelAdditive: q.a = v; break;
    case kKernelBrown: {
      BrownPart bp = brown_part(P.benv, v, m / v, &ok);
      q.a = bp.diffus;
      q.b = bp.speedsq;
      q.c = bp.deltasq;
      break;
    }
    case kKernelSedi: q.a = fall_g(mobility_rad(F, v, P.benv.fp, &ok)); break;
    case kKernelBrownFree: {
      q.a = v;
      q.b = m / v;
      q.c = pow(num_of_monomers(F, v), 1.0 / F.frac_dim);
      break;
    }
    case kKernelBrownCont: q.a = pow(num_of_monomers(F, v), 1.0 / F.frac_dim); break;
    default: break;
  }
  if (!ok) set_status(P.ctr, kErrAssert);  // the fractal Newton loop did not converge
  return q;
}

// pair-test record of slot i
__device__ __forceinline__ RecD make_rec(const PopDev& P, int i) {
  return make_rec_v(P, P.rad[i], P.vtot[i], P.mass[i], P.cls[i]);
}

__device__ __forceinline__ RecF to_f32(const RecD& q) {
  RecF f;
  f.r = (float)q.r;
  f.rv = (float)q.rv;
  f.nc = (float)q.nc;
  f.a = (float)q.a;
  f.b = (float)q.b;
  f.c = (float)q.c;
  f.pad0 = f.pad1 = 0.f;
  return f;
}

// radius, bin (aero_sorted_particle_in_bin, aero_sorted.F90:378-391) and
// pair-test records of live slot i; returns the 1-based bin (0 or n_bin+1
// off the grid, which leaves the slot unsorted)
__device__ __forceinline__ int refresh_slot(const PopDev& P, int i) {
  const GridDev& G = *P.grid;
  double r = vol2rad(P.benv.frac, P.vtot[i]);
  P.rad[i] = r;
  int b = bin_find(G.n_bin, G.log_lo, G.log_hi, r);
  int cl = P.cls[i] - 1;
  P.cell[i] = (b >= 1 && b <= G.n_bin && cl >= 0 && cl < P.n_class) ? (b - 1) + G.n_bin * cl : -1;
  RecD q = make_rec(P, i);
  P.recd[i] = q;
  P.recf[i] = to_f32(q);
  return b;
}

__global__ void k_refresh_all(const PopDev* pops, const uint8_t* on) {
  if (!on[blockIdx.y]) return;
  const PopDev& P = pops[blockIdx.y];
  int n = P.ctr->n_slots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (P.alive[i]) refresh_slot(P, i);
    else P.cell[i] = -1;
  }
}

// ---------------------------------------------------------------------------
// aero_sorted's bin lists rebuilt as one deterministic, stable counting sort
// of the slots by cell (slot order within each cell), for every population in
// one cooperative launch.  The grid is persistent (co-resident blocks looping
// over work items); two grid-wide barriers separate three phases:
//   1. per chunk of kChunk slots: the cell keys go to registers (thread
//      (w, lane) holds slots w * kWarpSlots + j * 32 + lane, j < kKeysPerThread)
//      and a warp-aggregated histogram to chunk_hist, cell-major
//      (chunk_hist[cell * n_chunks + chunk]); the occupied bin range is reset
//   2. per cell (one warp): exclusive scan of its chunk column in place and
//      the cell total; the occupied bin range
//   3. per chunk: the cell starts (a block scan of the totals; the chunk-0
//      block of each population stores them), then the scatter, ranking the
//      slots of one cell inside a 32-slot tile with __match_any_sync.  A block
//      reuses the keys it loaded in phase 1 for the same chunk.
constexpr int kKeysPerThread = kWarpSlots / 32;

__device__ __forceinline__ void sort_load_keys(const PopDev& P, int chunk, int n, int nc, int w, int lane,
                                               int* keys) {
#pragma unroll
  for (int j = 0; j < kKeysPerThread; j++) {
    int i = chunk * kChunk + w * kWarpSlots + j * 32 + lane;
    int key = i < n ? P.cell[i] : -1;
    keys[j] = key < nc ? key : -1;
  }
}

__global__ void __launch_bounds__(kSortThreads) k_sort_all(const PopDev* pops, int n_pop, int max_chunks,
                                                           int max_cells) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ int sm[];  // [kSortWarps][max_cells] counters, then [max_cells] cell starts
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long n_chunk_items = (long long)n_pop * max_chunks;
  int keys[kKeysPerThread];
  long long kept = -1;  // chunk item whose keys are in registers
  // phase 1
  if (blockIdx.x == 0)
    for (int k = threadIdx.x; k < n_pop; k += blockDim.x) {
      pops[k].ctr->bmin = 1 << 30;
      pops[k].ctr->bmax = -1;
    }
  for (long long item = blockIdx.x; item < n_chunk_items; item += gridDim.x) {
    const PopDev& P = pops[item / max_chunks];
    int chunk = (int)(item % max_chunks);
    int n_chunks = n_chunks_of(P);
    if (chunk >= n_chunks || !chunk_hist_fits(P, n_chunks)) continue;  // the same for the whole block
    int nc = P.n_cells;
    sort_load_keys(P, chunk, P.ctr->n_slots, nc, w, lane, keys);
    kept = item;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) sm[c] = 0;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kKeysPerThread; j++) {
      unsigned peers = __match_any_sync(0xffffffffu, keys[j]);
      if (keys[j] >= 0 && lane == __ffs(peers) - 1) atomicAdd(&sm[keys[j]], __popc(peers));
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += blockDim.x) P.chunk_hist[(size_t)c * n_chunks + chunk] = sm[c];
    __syncthreads();
  }
  grid.sync();
  // phase 2
  const long long warp_id = (long long)blockIdx.x * kSortWarps + w;
  const long long n_warps = (long long)gridDim.x * kSortWarps;
  for (long long item = warp_id; item < (long long)n_pop * max_cells; item += n_warps) {
    const PopDev& P = pops[item / max_cells];
    int c = (int)(item % max_cells);
    if (c >= P.n_cells) continue;
    int n_chunks = n_chunks_of(P);
    int run = 0;
    if (n_chunks > 0 && chunk_hist_fits(P, n_chunks)) {
      int* col = P.chunk_hist + (size_t)c * n_chunks;
      for (int base = 0; base < n_chunks; base += 128) {
        int h[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          int k = base + u * 32 + lane;
          h[u] = k < n_chunks ? col[k] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          int x = h[u];
          for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
          }
          int k = base + u * 32 + lane;
          if (k < n_chunks) col[k] = run + x - h[u];
          run += __shfl_sync(0xffffffffu, x, 31);
        }
      }
    }
    if (lane == 0) {
      P.cell_count[c] = run;
      if (run > 0 && P.grid->n_bin > 0) {
        int b = c % P.grid->n_bin;
        atomicMin(&P.ctr->bmin, b);
        atomicMax(&P.ctr->bmax, b);
      }
    }
  }
  grid.sync();
  // phase 3
  int* starts = sm + kSortWarps * max_cells;
  for (long long item = blockIdx.x; item < n_chunk_items; item += gridDim.x) {
    const PopDev& P = pops[item / max_chunks];
    int chunk = (int)(item % max_chunks);
    int n_chunks = n_chunks_of(P);
    int nc = P.n_cells;
    if (chunk == 0 && n_chunks == 0) {  // an empty population still gets its (zero) cell starts
      for (int c = threadIdx.x; c <= nc; c += blockDim.x) P.cell_start[c] = 0;
      continue;
    }
    if (chunk >= n_chunks || !chunk_hist_fits(P, n_chunks)) continue;
    int n = P.ctr->n_slots;
    if (item != kept) {
      sort_load_keys(P, chunk, n, nc, w, lane, keys);
      kept = item;
    }
    // cell starts
    int carry = 0;
    for (int base = 0; base < nc; base += blockDim.x) {
      int c = base + threadIdx.x;
      int v = c < nc ? P.cell_count[c] : 0;
      int tot;
      int pre = block_excl_scan(v, &tot);
      if (c < nc) starts[c] = carry + pre;
      carry += tot;
    }
    if (chunk == 0) {
      for (int c = threadIdx.x; c < nc; c += blockDim.x) P.cell_start[c] = starts[c];
      if (threadIdx.x == 0) P.cell_start[nc] = carry;
    }
    for (int k = threadIdx.x; k < kSortWarps * nc; k += blockDim.x) sm[k] = 0;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kKeysPerThread; j++) {
      unsigned peers = __match_any_sync(0xffffffffu, keys[j]);
      if (keys[j] >= 0 && lane == __ffs(peers) - 1) sm[w * nc + keys[j]] += __popc(peers);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
      int run = starts[c] + P.chunk_hist[(size_t)c * n_chunks + chunk];
      for (int q = 0; q < kSortWarps; q++) {
        int x = sm[q * nc + c];
        sm[q * nc + c] = run;
        run += x;
      }
    }
    __syncthreads();
    unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kKeysPerThread; j++) {
      int key = keys[j];
      int i = chunk * kChunk + w * kWarpSlots + j * 32 + lane;
      unsigned peers = __match_any_sync(0xffffffffu, key);
      int leader = __ffs(peers) - 1;
      int pos = 0;
      if (key >= 0) pos = sm[w * nc + key] + __popc(peers & lt);
      __syncwarp();
      if (key >= 0 && lane == leader) sm[w * nc + key] += __popc(peers);
      __syncwarp();
      if (key >= 0) {
        if (pos >= 0 && pos < P.cap) P.list[pos] = i;
        else bad_index(P.ctr, kBadScatterPos, pos);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// k_max table, est_k_minmax_binned_unweighted (coag_kernel.F90:253-280)
__global__ void k_kmax_table(const PopDev* pops) {
  const PopDev& P = pops[blockIdx.y];
  if (P.kmax_valid) return;
  int nb = P.grid->n_bin;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb * nb) return;
  int b1 = t % nb, b2 = t / nb;
  double kmin, kmax;
  bool ok = kminmax_for_bin(P.kernel_type, P.grid->edges, b1, b2, P.benv, P.coeff, P.dmin, P.dmax,
                            &kmin, &kmax);
  if (!ok) set_status(P.ctr, kErrAssert);
  P.kmax_tab[b1 + nb * b2] = kmax;
}

// ---------------------------------------------------------------------------
// Grid- and weight-dependent fields of every bin pair: the destination class
// (coag_dest_class, coag_kernel.F90:382-416), max_coag_num_conc_factor
// (coag_kernel.F90:422-465), the flat-weight factor, and the weight
// conditions of try_per_particle_coag (coagulation.F90:191-217).  One warp
// per pair; lane (a-1)*5 + (b-1) takes radius sample (a, b) of the 5x5 grid.
__global__ void k_pair_setup(const PopDev* pops) {
  const PopDev& P = pops[blockIdx.y];
  if (P.pair_setup_valid) return;
  int lane = threadIdx.x & 31;
  int p = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (p >= P.n_pairs) return;  // the whole warp
  PairDesc d = P.pair_desc[p];
  int b1 = d.b1, b2 = d.b2, c1 = d.c1, c2 = d.c2;
  const GridDev& G = *P.grid;
  const Fractal& F = P.benv.frac;
  int cc = coag_dest_class(P.w, F, G.centers, b1, b2, c1, c2);
  double f = 0.0;
  if (lane < 25) {
    double ri = interp_linear_disc(G.edges[b1], G.edges[b1 + 1], 5, lane / 5 + 1);
    double rj = interp_linear_disc(G.edges[b2], G.edges[b2 + 1], 5, lane % 5 + 1);
    f = num_conc_factor(P.w, F, ri, rj, c1, c2, cc);
  }
  // the factors are positive: the maximum does not depend on the order
  for (int o = 16; o > 0; o >>= 1) {
    double g = __shfl_xor_sync(0xffffffffu, f, o);
    if (g > f) f = g;
  }
  if (lane != 0) return;
  PairState& S = P.pair[p];
  S.cc = cc;
  S.f_max = f;
  S.fflat = P.flat ? num_conc_factor(P.w, F, G.centers[b1], G.centers[b2], c1, c2, cc) : 1.0;
  S.pp_ok = 0;
  if (P.mono_dec) {
    double n1min, n1max, n2min, n2max;
    {
      double a = num_conc_at_radius<double>(P.w, c1, G.edges[b1]);
      double b = num_conc_at_radius<double>(P.w, c1, G.edges[b1 + 1]);
      n1min = a < b ? a : b;
      n1max = a > b ? a : b;
      a = num_conc_at_radius<double>(P.w, c2, G.edges[b2]);
      b = num_conc_at_radius<double>(P.w, c2, G.edges[b2 + 1]);
      n2min = a < b ? a : b;
      n2max = a > b ? a : b;
    }
    int ok = 0, bt = 0, bs = 0, ct = 0, cs = 0;
    if (n1max < n2min && cc == c1) {
      bt = b1; bs = b2; ct = c1; cs = c2; ok = 1;
    }
    if (n2max < n1min && cc == c2) {
      bt = b2; bs = b1; ct = c2; cs = c1; ok = 1;
    }
    S.pp_ok = ok;
    S.bt = bt; S.bs = bs; S.ct = ct; S.cs = cs;
    S.pp_min_tv = rad2vol(F, G.edges[bt]);
    S.pp_max_sv = rad2vol(F, G.edges[bs + 1]);
  }
}

// ---------------------------------------------------------------------------
// pair set-up for round 0: mc_coag_for_bin, try_per_particle_coag's
// eligibility tests and compute_n_samp (coagulation.F90:101-241, 648-702).
// nwork_set[gp] = samples of a per-set pair; nwork_pp[gp] = targets of a
// per-particle pair.  k_max is set for every pair, empty ones included:
// walks test particles that arrive in a pair's cells during the step.
__global__ void k_pairs(const PopDev* pops, const long long* pop_pair_base, long long* nwork_set,
                        long long* nwork_pp, int use_particle_path) {
  const PopDev& P = pops[blockIdx.y];
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.n_pairs) return;
  long long gp = pop_pair_base[blockIdx.y] + p;
  PairDesc d = P.pair_desc[p];
  int nb = P.grid->n_bin;
  int b1 = d.b1, b2 = d.b2, c1 = d.c1, c2 = d.c2;
  int cell1 = b1 + nb * c1, cell2 = b2 + nb * c2;
  PairState& S = P.pair[p];
  int n1 = P.cell_count[cell1], n2 = P.cell_count[cell2];
  S.n1 = n1;
  S.n2 = n2;
  S.start1 = P.cell_start[cell1];
  S.start2 = P.cell_start[cell2];
  if (S.start1 < 0 || (long long)S.start1 + n1 > P.cap || S.start2 < 0 || (long long)S.start2 + n2 > P.cap) {
    bad_index(P.ctr, kBadPairCells, p);
    S.n1 = S.n2 = n1 = n2 = 0;
  }
  bool same = (b1 == b2) && (c1 == c2);
  double k_max = P.kmax_tab[b1 + nb * b2] * S.f_max;
  S.k_max = k_max;
  S.inv_k_max = 1.0 / k_max;
  // try_per_particle_coag eligibility (coagulation.F90:191-217): the weight
  // conditions were settled by k_pair_setup; the cell-count ones are here.
  // A pair whose target cell is empty now but whose source cell is not is
  // marked too: particles that reach the target cell during the step are
  // its targets when the pair's turn comes (walks stop there).
  if (use_particle_path && P.mono_dec && S.pp_ok) {
    int ns = P.cell_count[S.bs + nb * S.cs];
    double nspt = k_max * P.del_t * (double)ns;
    double max_new = S.pp_min_tv + S.pp_max_sv * nspt;
    if (ns > 0 && nspt >= 1.0 && !(max_new / S.pp_min_tv > 1.5)) {
      S.path = kPathParticle;
      S.nspt = nspt;
      int nt = P.cell_count[S.bt + nb * S.ct];
      nwork_set[gp] = 0;
      nwork_pp[gp] = nt;
      return;
    }
  }
  if (n1 == 0 || n2 == 0) {
    S.path = kPathSkip;
    nwork_set[gp] = nwork_pp[gp] = 0;
    return;
  }
  // per_set_coag / compute_n_samp
  double n_possible = same ? (double)n1 * ((double)n2 - 1.0) / 2.0 : (double)n1 * (double)n2;
  double mean = k_max * P.del_t * n_possible;
  Rng g = make_rng(P, kStreamPair, (uint32_t)p, 0);
  int ns = rand_poisson(g, mean);
  if (ns < 0) {
    set_status(P.ctr, kErrTimeout);
    ns = 0;
  }
  S.path = kPathSet;
  add_ll(&P.ctr->tot_samp, (long long)((long long)ns));
  if ((same && n1 < 2) || n1 < 1 || n2 < 1) ns = 0;
  nwork_set[gp] = ns;
  nwork_pp[gp] = 0;
}

// ---------------------------------------------------------------------------
// weighted kernel of a pair of records (num_conc_weighted_kernel,
// coag_kernel.F90:175-209)
template <int KT, class T, bool FLAT>
__device__ __forceinline__ T pair_kernel(const PopDev& P, const T* q1, const T* q2, int c1, int c2,
                                         int cc, T fflat, T coeff) {
  // q = {r, rv, nc, a, b, c}
  T k;
  if (KT == kKernelAdditive) {
    k = coeff * (q1[3] + q2[3]);
  } else if (KT == kKernelConstant) {
    k = (T)kBeta0;
  } else if (KT == kKernelBrown) {
    k = brown_pair<T>(q1[0], q1[3], q1[4], q1[5], q2[0], q2[3], q2[4], q2[5]);
  } else if (KT == kKernelSedi) {
    k = sedi_pair<T>(q1[0], q1[3], q2[0], q2[3]);
  } else if (KT == kKernelBrownFree) {
    // q = {r, rv, nc, volume, density, N^(1/d_f)}; 1/N = V(R0) / volume
    T v1 = q1[3], v2 = q2[3];
    T rho = (v1 / (v1 + v2)) * q1[4] + (v2 / (v1 + v2)) * q2[4];
    const T v0 = T(rad2vol(P.benv.frac.prime_radius));
    T s = q1[5] + q2[5];
    if constexpr (sizeof(T) == 8) {
      k = sqrt(T(6.0 * kBoltzmann * P.benv.temp * P.benv.frac.prime_radius) / rho * (v0 / v1 + v0 / v2)) * (s * s);
    } else {
      // the same product with the constant's square root taken apart: 6 k T R0
      // is about 1e-28, and divided by rho and multiplied by 1/N of a large
      // cluster it would fall below FP32's normal range
      k = T(sqrt(6.0 * kBoltzmann * P.benv.temp * P.benv.frac.prime_radius)) * sqrt((v0 / v1 + v0 / v2) / rho) *
          (s * s);
    }
  } else if (KT == kKernelBrownCont) {
    // q = {r, rv, nc, N^(1/d_f), -, -}
    k = T(2.0 * kBoltzmann * P.benv.temp / 3.0 / kAirDynVisc) * (T(1) / q1[3] + T(1) / q2[3]) * (q1[3] + q2[3]);
  } else {
    k = T(0);
  }
  if (FLAT) return k * fflat;
  T rij = vol2rad(P.benv.frac, q1[1] + q2[1]);
  T ncij = num_conc_at_radius<T>(P.w, cc, rij);
  T nci = q1[2], ncj = q2[2];
  T mn = nci;
  if (ncj < mn) mn = ncj;
  if (ncij < mn) mn = ncij;
  return k * (nci * ncj / mn);
}

// FP32 acceptance with an exact FP64 fallback.  The FP32 probability pf =
// k32 / k_max of a pair test differs from the FP64 one by less than
// kAcceptMargin (the rounding-error bound of the FP32 kernel and weight
// evaluation is below 2^-17 of k_max for every kernel; the margin leaves a
// factor 32).  So when the uniform u lies farther than the margin from pf,
// and pf is below 1 - margin, u < pf is the FP64 decision u < p64; otherwise
// (about 2 * 2^-12 of the tests, and every test near or above k_max) the
// test is decided in FP64 from the FP64 records.  The decisions, and the
// k > k_max warnings, are those of the FP64 mode for the same draws.
constexpr float kAcceptMargin = 1.0f / 4096.0f;
__device__ __forceinline__ bool f32_decides(float pf, double u) {
  return pf < 1.0f - kAcceptMargin && fabs((double)pf - u) > (double)kAcceptMargin;
}

// u < k / k_max in FP64 from the slots' FP64 records, for the pair p's
// orientation (first cell's particle first); counts k > k_max as the
// reference's warn_assert_msg does (coagulation.F90:749-751)
template <int KT, bool FLAT>
__device__ __forceinline__ bool accept_f64_rec(const PopDev& P, const RecD& a, const RecD& b, const PairDesc& d,
                                               int cc, double fflat, double inv_k_max, double u) {
  const double k = pair_kernel<KT, double, FLAT>(P, (const double*)&a, (const double*)&b, d.c1, d.c2, cc, fflat,
                                                 P.coeff);
  const double prob = k * inv_k_max;
  if (!(prob <= 1.0)) add_ll(&P.ctr->kmax_warn, 1LL);
  return u < prob;
}
template <int KT, bool FLAT>
__device__ __forceinline__ bool accept_f64(const PopDev& P, int s1, int s2, const PairDesc& d, const PairState& S,
                                           double u) {
  return accept_f64_rec<KT, FLAT>(P, P.recd[s1], P.recd[s2], d, S.cc, S.fflat, S.inv_k_max, u);
}

__device__ __forceinline__ int find_pair(const long long* off, int n, long long w) {
  // largest gp with off[gp] <= w (off is an exclusive scan, off[n] = total)
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (off[mid] <= w) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Decisions of coagulate_weighting (coagulation.F90:855-892).
struct MergeDecision {
  bool rm1, rm2, create, lost1, lost2;
  int new_group;  // 1-based
};

// particle 1 (radius r1, total volume vt1) from the pair's first cell,
// particle 2 from its second
template <class R>
__device__ MergeDecision merge_decide_v(const PopDev& P, R& g, double r1, double vt1, double r2, double vt2, int c1,
                                        int c2, int cc) {
  MergeDecision d;
  const Fractal& F = P.benv.frac;
  double rc = vol2rad(F, rad2vol(F, r1) + rad2vol(F, r2));
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
      if (vt1 > vt2) d.lost2 = true;
      else d.lost1 = true;
    }
  } else {
    d.lost1 = d.rm1;
    d.lost2 = d.rm2;
  }
  return d;
}

template <class R>
__device__ MergeDecision merge_decide(const PopDev& P, R& g, int s1, int s2, int c1, int c2, int cc) {
  return merge_decide_v(P, g, P.rad[s1], P.vtot[s1], P.rad[s2], P.vtot[s2], c1, c2, cc);
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

// random stream of an event's merge: the pair and the sample for the pair's
// own samples, the pair and the walking slot for a walk's test
__device__ __forceinline__ Rng merge_rng(const PopDev& P, unsigned long long key) {
  uint32_t idx = key_idx(key);
  if (key_kind(key)) idx |= 0x80000000u;
  return make_rng(P, kStreamMerge, key_pair(key), idx);
}

// Per-set pair tests (maybe_coag_pair, coagulation.F90:712-759).  One thread
// per sample w of the flattened (population, pair, sample) space; an
// accepted sample records its slots and global pair.  Its merge decision is
// drawn after the compaction (k_decide), so the FP64 decisions run in full
// warps instead of in the few accepting lanes of each warp of tests.
template <int KT, class T, bool FLAT>
__global__ void __launch_bounds__(256) k_test(const PopDev* pops, const int* gpair_pop,
                                              const int* gpair_local, const long long* work_off,
                                              int n_gpairs, const long long* total, uint8_t* flag,
                                              int2* ev, int* ev_gp) {
  long long W = *total;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < W;
       w += (long long)gridDim.x * blockDim.x) {
    int gp = find_pair(work_off, n_gpairs, w);
    const PopDev& P = pops[gpair_pop[gp]];
    int p = gpair_local[gp];
    long long s = w - work_off[gp];
    const PairState& S = P.pair[p];
    PairDesc d = P.pair_desc[p];
    U4 rnd = philox4x32_10(U4{P.step, (uint32_t)(p << 12) | ((*P.round_p & 0xffu) << 4) | kStreamTest,
                              (uint32_t)s, 0u},
                           (uint32_t)P.seed, (uint32_t)(P.seed >> 32));
    // find_rand_pair (coagulation.F90:766-803), 0-based entries
    int n1 = S.n1, n2 = S.n2;
    int i1 = (int)(u32d(rnd.x) * (double)n1);
    if (i1 >= n1) i1 = n1 - 1;
    int i2;
    bool same = (d.b1 == d.b2) && (d.c1 == d.c2);
    if (same) {
      i2 = (int)(u32d(rnd.y) * (double)(n2 - 1));
      if (i2 >= n2 - 1) i2 = n2 - 2;
      if (i2 == i1) i2 = n2 - 1;
    } else {
      i2 = (int)(u32d(rnd.y) * (double)n2);
      if (i2 >= n2) i2 = n2 - 1;
    }
    int e1 = S.start1 + i1, e2 = S.start2 + i2;
    if (e1 < 0 || e1 >= P.cap || e2 < 0 || e2 >= P.cap) {
      bad_index(P.ctr, kBadTestPos, e1 < 0 || e1 >= P.cap ? e1 : e2);
      flag[w] = 0;
      continue;
    }
    int s1 = P.list[e1], s2 = P.list[e2];
    if (s1 < 0 || s1 >= P.cap || s2 < 0 || s2 >= P.cap) {
      bad_index(P.ctr, kBadTestSlot, s1 < 0 || s1 >= P.cap ? s1 : s2);
      flag[w] = 0;
      continue;
    }
    const double u = u53(rnd.z, rnd.w);
    bool acc;
    if constexpr (sizeof(T) == 8) {
      acc = accept_f64<KT, FLAT>(P, s1, s2, d, S, u);
    } else {
      const float* q1 = (const float*)&P.recf[s1];
      const float* q2 = (const float*)&P.recf[s2];
      const float pf = pair_kernel<KT, float, FLAT>(P, q1, q2, d.c1, d.c2, S.cc, (float)S.fflat, (float)P.coeff) *
                       (float)S.inv_k_max;
      if (f32_decides(pf, u)) {
        acc = u < (double)pf;
      } else {
        acc = accept_f64<KT, FLAT>(P, s1, s2, d, S, u);
        add_ll(&P.ctr->exact_tests, 1LL);
      }
    }
    flag[w] = acc ? 1 : 0;
    if (acc) {
      ev[w] = make_int2(s1, s2);
      ev_gp[w] = gp;
    }
  }
}

// Round 0's merge decisions, one thread per accepted sample in sample order
// (after the compaction): the decision (coagulate_weighting,
// coagulation.F90:810-922) from the sample's own stream (merge_rng of its
// key), stored in dec[e], and the claims on its two slots by it: a write
// claim on a slot the merge removes or rewrites, a read claim on one it
// keeps.
__global__ void __launch_bounds__(256) k_decide(const PopDev* pops, const int* gpair_pop,
                                                const long long* n_events, const unsigned long long* ev_key,
                                                const int2* ev_c, const int* gp_c, uint32_t* dec) {
  long long E = *n_events;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < E;
       e += (long long)gridDim.x * blockDim.x) {
    const PopDev& P = pops[gpair_pop[gp_c[e]]];
    const unsigned long long key = ev_key[e];
    const int p = (int)key_pair(key);
    const int2 sl = ev_c[e];
    const PairState& S = P.pair[p];
    const PairDesc d = P.pair_desc[p];
    const unsigned long long ck = claim_key(P, key);
    Rng gm = merge_rng(P, key);
    MergeDecision m = merge_decide(P, gm, sl.x, sl.y, d.c1, d.c2, S.cc);
    if (m.new_group == 0) set_status(P.ctr, kErrTimeout);
    dec[e] = pack_decision(m, gm.used());
    claim_slot(P, sl.x, ck, m.rm1);
    claim_slot(P, sl.y, ck, m.rm2);
  }
}

}  // namespace pmc
