// pmc_state.cuh -- device-resident layout of particle populations.
//
// A population is the GPU form of aero_state_t (aero_state.F90:69-84):
//  - particle slots, one array per field; the per-particle vectors are
//    particle-major (species s of slot i at vol[i * n_spec + s], component k
//    at csrc/ctime[i * kMaxComponent + k]) because the step only ever reads
//    or writes whole particles: a warp moves one particle's 20 species in one
//    or two cache lines.  Per-slot caches vtot = sum(vol) and
//    mass = sum(vol*density) are recomputed in the reference's summation
//    order on every change;
//  - the aero_sorted_t equivalent (aero_sorted.F90:47-66): bin grid, one
//    list of slot numbers per (bin, class) cell in CSR form, and a
//    bin-ordered array of pair-test records;
//  - the k_max table per bin pair (coag_kernel_max) and per-pair state.
#pragma once

#include <cstdint>

#include "pmc_physics.cuh"

namespace pmc {

// Status codes shared with the C ABI.
enum : int {
  kOk = 0,
  kErrArg = 1,
  kErrOutOfGrid = 2,
  kErrCapacity = 3,
  kErrCuda = 4,
  kErrTimeout = 5,
  kErrRng = 6,
  kErrAssert = 7,
};

// Pair-test record of one particle, stored in cell order so that a test
// reads two records.  r: radius; rv: rad2vol(r) (for the coagulated radius
// of coag_num_conc_factor); nc: number concentration of the particle's class
// at r; a/b/c: per-particle kernel terms (additive: total volume; Brownian:
// diffusivity, squared thermal speed, delta^2; sedimentation: terminal
// velocity).
struct __align__(16) RecD {
  double r, rv, nc, a, b, c;
};
struct __align__(32) RecF {
  float r, rv, nc, a, b, c, pad0, pad1;
};

struct PopDev;

// aero_info_t (aero_info.F90:48-56): the ID of a removed particle, the
// action (aero_info.F90:19-28: kInfoCoag, kInfoHalved, kInfoWeight) and the
// ID of the particle the coagulation produced (the target's ID for a
// per-particle coagulation, 0 if none)
struct RemovalRec {
  long long id, other_id;
  int action, pad;
};
enum : int { kInfoCoag = 2, kInfoHalved = 3, kInfoWeight = 4 };

// index of species s of slot i, and of component k of slot i
#define PMC_VOL_AT(n_spec, i, s) ((size_t)(i) * (size_t)(n_spec) + (size_t)(s))
__host__ __device__ __forceinline__ size_t comp_at(long long i, int k) {
  return (size_t)i * kMaxComponent + (size_t)k;
}

struct GridDev {
  int n_bin;
  double log_lo, log_hi;  // log(edges[0]), log(edges[n_bin])
  double edges[kMaxBin + 1];
  double centers[kMaxBin];
};

// (b1, c1, b2, c2) of pair p, in the reference's loop order
// (coagulation.F90:74-94).  0-based.
struct PairDesc {
  int16_t b1, b2;
  int8_t c1, c2, pad0, pad1;
};

enum PairPath : int { kPathSkip = 0, kPathSet = 1, kPathParticle = 2 };

struct PairState {
  // set per step
  double k_max;      // coag_kernel_max(b1,b2) * f_max (FP32 mode: inflated)
  double inv_k_max;  // accept_factor = 1 / k_max
  double nspt;       // n_source_per_target (per-particle path)
  int path;
  int n1, n2;        // cell sizes at round start
  int start1, start2;
  // set when the grid or the weights change (k_pair_setup)
  double f_max;      // max_coag_num_conc_factor
  double fflat;      // constant weight factor when every weight is flat
  double pp_min_tv, pp_max_sv;  // rad2vol of the target bin's lower and the source bin's upper edge
  int cc;            // destination class (0-based)
  int pp_ok;         // the weights make the per-particle path possible
  int bt, bs, ct, cs;  // per-particle path target/source cells (0-based)
};

// Per-population counters and scalars that kernels update.
struct PopCtr {
  int n_slots;       // slots in use (high-water mark)
  int n_live;
  long long next_id;
  long long tot_samp, tot_coag;
  long long kmax_warn;
  long long redraws;
  int status;        // first error code seen
  int out_of_grid;   // unused (kept for the layout of the counter block)
  int bmin, bmax;    // occupied bin range after a sort (-1 if empty)
  unsigned long long rmin_bits, rmax_bits;  // radius range (positive doubles)
  int new_slots, new_ids;  // allocations in the current apply phase
  int losers;
  int n_events;
  long long rng_used;      // replay: uniforms consumed
  int bad_site;            // first failed bounds check (kBad*), 0 if none
  long long bad_index;     // the index that failed it
  long long walk_tests;    // pair tests made by walks in the current step
  long long exact_tests;   // FP32 pair tests decided in FP64 (f32_decides), since the context was made
  long long n_removed;     // removal records appended since the host last read them
  int cap_site;            // first capacity limit a kernel hit (kCap*), 0 if none
  int cap_pad;
};

// sites of the device capacity limits (PopCtr::cap_site)
enum : int {
  kCapNone = 0,
  kCapEventDest = 1,   // an event's new particle past the slot arrays
  kCapTargetOps = 2,   // the round's target-operation list is full
  kCapRemovals = 3,    // a target operation's removals past its share of the pool
  kCapCopies = 4,      // more dup copies than one target operation holds
  kCapCopySlot = 5,    // a target operation's copy past the slot arrays
  kCapWalkers = 6,     // the walker list of target operations is full
  kCapSampleSlot = 7,  // a sampled particle past the slot arrays
  kCapDupSlot = 8,     // a doubled or dup copy past the slot arrays
};

// sites of the device bounds checks (PopCtr::bad_site)
enum : int {
  kBadNone = 0,
  kBadTestPos = 1,     // pair test: cell-list position outside the list
  kBadTestSlot = 2,    // pair test: slot number outside the slots
  kBadEventSlot = 3,   // accepted event names a slot outside the slots
  kBadScatterPos = 4,  // sort scatter: list position outside the list
  kBadChunkHist = 5,   // sort: chunk histogram larger than its allocation
  kBadPairCells = 6,   // pair set-up: a cell runs past the list
  kBadSlotCount = 7,   // slot count above the capacity
  kBadDest = 8,        // event destination slot outside the slots
};

// One population as the kernels see it (kept in device memory).
struct PopDev {
  int cap, n_spec, n_group, n_class, i_water;
  int n_cells;  // n_bin * n_class
  int n_chunks; // sort chunks covering n_slots
  int n_pairs;
  uint64_t seed;
  uint32_t step;
  const uint32_t* round_p;  // the current round of the step (one device word for all populations)
  const uint32_t* gen_p;    // rounds since the context was made (claim generation)
  int kernel_type;
  double temp, pressure, coeff, del_t;
  BrownEnv benv;
  double dmin, dmax;  // min/max species density
  Weights w;
  bool flat;
  bool mono_dec;

  // slots
  double* vol;
  double* vtot;
  double* mass;
  double* rad;
  int* grp;  // 1-based
  int* cls;  // 1-based
  long long* id;
  int* nprim;
  int* ncomp;
  int* csrc;      // [kMaxComponent][cap]
  double* ctime;  // [kMaxComponent][cap]
  double* lct;
  double* gct;
  double* imf;
  double* den_ice;
  double* phi;
  int* hyst;
  int* frozen;
  uint8_t* alive;
  uint8_t* changed;  // slot written since the host copy was last brought up to date
  // sort key of each slot: the (bin, class) cell bin + n_bin * class
  // (0-based) of a live particle on the grid, -1 for a dead slot or a
  // particle off the grid
  int* cell;

  const double* density;  // [n_spec]

  // sort
  GridDev* grid;
  int* chunk_hist;  // [n_chunks][n_cells]
  int chunk_hist_len;  // ints allocated at chunk_hist
  int* cell_count;  // [n_cells]
  int* cell_start;  // [n_cells + 1]
  int* list;        // [cap] slot numbers in cell order
  RecD* recd;       // [cap] pair-test record of each slot (FP64)
  RecF* recf;       // [cap] the same in FP32

  double* kmax_tab;  // [n_bin * n_bin], (b1, b2) at b1 + n_bin * b2
  int kmax_valid;
  int pair_setup_valid;  // the grid/weight-dependent fields of pair[] are current

  const PairDesc* pair_desc;  // [n_pairs]
  PairState* pair;            // [n_pairs]
  // pairs that contain each cell, in loop order (CSR): the pairs of cell c
  // are cp_list[cp_off[c] .. cp_off[c + 1])
  const int* cp_off;   // [n_cells + 1]
  const int* cp_list;  // [cp_off[n_cells]]
  // walk rates, brought up to date after each later round's sort: the
  // segment of cell c, cp_cum[cp_off[c] + c + j] for j = 0..len, holds the
  // expected walk tests (k_max * del_t * members of the other cell) of the
  // cell's first j pairs
  double* cp_cum;      // [cp_off[n_cells] + n_cells]
  // with the rates, per entry j of the lists: {pair, other cell (bit 30 set
  // if this cell is the pair's first), the other cell's start and members}
  int4* cp_ent;        // [cp_off[n_cells]]
  // per entry j of a cell's list, the first entry at or after j whose pair is
  // on the per-particle path with this cell as its target cell (a walk stops
  // there for a target operation); the cell's end if none
  int* cp_nstop;       // [cp_off[n_cells]], valid when walk_stops
  int walk_stops;      // round 0 gave this population target operations: walks stop at per-particle pairs
  // per cell, kWalkTab buckets of its stretch of tests: entry b is the last
  // j of the cell with cp_cum[j] <= b / kWalkTab of the cell's total
  int* cp_tab;         // [n_cells * kWalkTab]
  // every 16th pair of each cell's list, padded with INT_MAX to n_coarse (a
  // multiple of 4) per cell: the first level of the search for a pair
  const int* cp_coarse;  // [n_cells * n_coarse]
  int n_coarse;

  // [cap] lowest claim key (claim_key) of the current round's events that
  // remove or rewrite the slot, and of those that only read it; a key from
  // any earlier round is larger and is replaced by the first claim of this
  // round, so no per-round reset is needed.  An event that writes a slot
  // wins it if it holds the write claim and no earlier event reads it; an
  // event that reads a slot wins it if no earlier event writes it.
  unsigned long long* claim;
  unsigned long long* rclaim;
  // [cap] claim generation of the round that last removed or rewrote the
  // slot: an event that lost a claim in round r is retried in round r + 1
  // only if neither of its particles was consumed in round r
  uint32_t* touched;

  PopCtr* ctr;

  // removal log (aero_state%aero_info_array) when rm_on: records
  // [0, ctr->n_removed), at most rm_cap kept (the host sizes it before
  // every step for the most removals a step can make)
  RemovalRec* rm_log;
  long long rm_cap;
  int rm_on;
};

__host__ __device__ __forceinline__ size_t vol_at(const PopDev& P, long long i, int s) {
  return PMC_VOL_AT(P.n_spec, i, s);
}

// Event priorities follow the reference's order of tests within one step:
// the pair p in loop order first, then the test.  kind 0 is test idx of the
// pair's own samples (round 0; a per-particle pair's target operation idx);
// kind 1 is a walk's test in pair p made by the particle in slot idx, placed
// after the pair's own samples.  p < 2^20, idx < 2^32: 53 bits.
__host__ __device__ __forceinline__ unsigned long long make_key(uint32_t p, uint32_t kind, uint32_t idx) {
  return ((unsigned long long)p << 33) | ((unsigned long long)kind << 32) | (unsigned long long)idx;
}
__host__ __device__ __forceinline__ uint32_t key_pair(unsigned long long k) { return (uint32_t)(k >> 33); }
__host__ __device__ __forceinline__ uint32_t key_kind(unsigned long long k) { return (uint32_t)(k >> 32) & 1u; }
__host__ __device__ __forceinline__ uint32_t key_idx(unsigned long long k) { return (uint32_t)k; }

// claim generations live in the top 11 bits of a claim word; the host
// restarts them (clearing every claim and touched word) before they run out
constexpr uint32_t kGenLimit = 2047;
constexpr int kWalkTab = 64;  // buckets of a cell's walk stretch (cp_tab)

#ifdef __CUDACC__
// claim word of an event key in the current round: a later generation gives
// a smaller word, so the first claim of a round replaces any older one
__device__ __forceinline__ unsigned long long claim_key(const PopDev& P, unsigned long long key) {
  return ((unsigned long long)(~*P.gen_p & kGenLimit) << 53) | key;
}

// an event's claim on slot s: a write claim if it removes or rewrites s,
// else a read claim; and whether it holds s after every claim of the round
__device__ __forceinline__ void claim_slot(const PopDev& P, int s, unsigned long long ck, bool write) {
  atomicMin(write ? &P.claim[s] : &P.rclaim[s], ck);
}
__device__ __forceinline__ bool holds_slot(const PopDev& P, int s, unsigned long long ck, bool write) {
  return write ? (P.claim[s] == ck && P.rclaim[s] > ck) : P.claim[s] > ck;
}

// aero_state_remove_particle_with_info (aero_state.F90:408-422): append
// the removal's aero_info to the population's log when records are kept.
// Records past the log's capacity are counted but dropped (the host reports
// that as PMC_ERR_CAPACITY).
__device__ __forceinline__ void log_removal(const PopDev& P, long long id, int action, long long other_id) {
  if (!P.rm_on) return;
  const unsigned long long k = atomicAdd((unsigned long long*)&P.ctr->n_removed, 1ULL);
  if ((long long)k < P.rm_cap) {
    RemovalRec r;
    r.id = id;
    r.other_id = other_id;
    r.action = action;
    r.pad = 0;
    P.rm_log[k] = r;
  }
}
#endif

}  // namespace pmc
