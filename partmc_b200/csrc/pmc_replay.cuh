// pmc_replay.cuh -- sequential replay of the reference's mc_coag order on
// the device (declarations; implementation in pmc_replay.cu).
#pragma once

#include <cuda_runtime.h>

#include "pmc_state.cuh"

namespace pmc {

// device buffers of the replay mode (the inverse maps of integer_rmap2)
struct ReplayBuffers {
  void* mem = nullptr;
  size_t bytes = 0;
};

int replay_step(int n_pop, PopDev* d_pops, cudaStream_t stream, ReplayBuffers& rb,
                const double* u, long long n_u, long long* used, int kernel_type,
                long long* tot_samp, long long* tot_coag);
void replay_free(ReplayBuffers& rb);

}  // namespace pmc
