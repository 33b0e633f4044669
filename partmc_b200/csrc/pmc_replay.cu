// pmc_replay.cu -- placeholder until the replay kernel lands.
#include "pmc_replay.cuh"
namespace pmc {
int replay_step(int, PopDev*, cudaStream_t, ReplayBuffers&, const double*, long long, long long*,
                int, long long*, long long*) {
  return 1;
}
void replay_free(ReplayBuffers& rb) {
  if (rb.mem) cudaFree(rb.mem);
  rb.mem = nullptr;
  rb.bytes = 0;
}
}  // namespace pmc
