// pmc_replay.cuh -- sequential replay of the reference's mc_coag order on
// the device.
//
// One device thread runs mc_coag (coagulation.F90:43-96) exactly as the
// reference orders it -- bin-pair loop, per-set and per-particle paths,
// swap-last removals -- consuming a given stream of uniforms in the order
// pmc_random is called (rand.F90:138-167).  The inverse maps of
// aero_sorted_t (integer_rmap2, integer_rmap2.F90:53-243) live in device
// memory and persist between calls, as the reference's sort does while
// valid_sort holds.  Particle slots are kept dense: slot i holds the
// reference's particle i + 1.
#pragma once

#include <cuda_runtime.h>

#include "pmc_state.cuh"

namespace pmc {

// integer_rmap2_t on the device: values stored 1-based as in the reference.
struct RMapDev {
  int n_r1, n_r2;
  int cap;      // domain capacity = particle capacity
  int* fwd1;    // [cap]
  int* fwd2;    // [cap]
  int* index;   // [cap]
  int* inv_n;   // [n_r1 * n_r2]
  int* inv;     // [n_r1 * n_r2][cap]
  int* n;       // domain size (one int)
};

struct ReplayDev {
  RMapDev size_class, group_class;
  const double* u;   // uniform stream
  long long n_u;
  long long* used;   // uniforms consumed (persists across calls)
  int* status;
  long long* tot;    // [2]: samples, coagulations of this call
  int* n_part;       // particle count (in/out)
  long long* next_id;
  int rebuild;       // sort_particles before the loop (after a regrid / upload)
};

// host-side owner of the replay buffers of one population
struct ReplayBuffers {
  void* mem = nullptr;
  size_t bytes = 0;
  int cap = 0, n_cells = 0, n_gc = 0;
  bool valid = false;  // inverse maps match the particles (the reference's valid_sort)
  ReplayDev dev{};
};

// allocate (or keep) buffers for capacity cap and grids of n_cells size
// cells and n_gc group cells; returns false on allocation failure
bool replay_reserve(ReplayBuffers& rb, int cap, int n_cells, int n_gc, int n_bin, int n_class,
                    int n_group);
void replay_free(ReplayBuffers& rb);
// launch the single-thread replay of one mc_coag call on population `pop`
void replay_launch(const PopDev* d_pops, int pop, const ReplayDev& rd, cudaStream_t stream);
// per-(bin, class) entry counts of the size_class inverse map
void replay_cell_counts(const ReplayDev& rd, int* d_counts, cudaStream_t stream);

}  // namespace pmc
