// pmc_noalloc.cu -- the size-bin sort with its scratch in a static device
// array, for callers that cannot allocate device memory.
//
// pmc_coag_gpu_bin_sort_noalloc() runs the same three passes as the sort
// inside a context (bin + per-chunk histogram, scan, stable scatter) on
// caller-owned device buffers.  Its only scratch, the per-chunk cell
// histogram, lives in the file-scope array below instead of coming from
// cudaMalloc, so the call allocates nothing: for a host program whose device
// memory is all handed out up front by another allocator.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/pmc_coag_gpu.h"
#include "pmc_physics.cuh"

namespace pmc {
namespace {

constexpr int kNaChunk = 2048;                 // particles per block
constexpr int kNaThreads = 256;
constexpr int kNaWarps = kNaThreads / 32;
constexpr int kNaWarpSlots = kNaChunk / kNaWarps;
constexpr int kNaMaxCells = 1024;               // n_bin * n_class
constexpr int kNaMaxPart = 1 << 21;             // 2,097,152 particles
constexpr int kNaMaxChunks = kNaMaxPart / kNaChunk;
constexpr size_t kNaScratchInts = (size_t)kNaMaxChunks * kNaMaxCells;  // 4 MiB

// Per-chunk cell histogram, then per-chunk cell offsets.  Shared by every
// call on the device; each call writes every entry it reads.
static __device__ __align__(256) int g_bin_sort_scratch[kNaScratchInts];

__global__ void k_na_hist(int n, const double* vtot, const int* cls, int n_bin, int n_class, int n_cells,
                          double log_lo, double log_hi, int* bin, int* scratch) {
  extern __shared__ int h[];
  for (int c = threadIdx.x; c < n_cells; c += blockDim.x) h[c] = 0;
  __syncthreads();
  int base = blockIdx.x * kNaChunk;
  for (int k = threadIdx.x; k < kNaChunk; k += blockDim.x) {
    int i = base + k;
    if (i >= n) break;
    int b = bin_find(n_bin, log_lo, log_hi, vol2rad(vtot[i]));
    bin[i] = b;
    if (b >= 1 && b <= n_bin && cls[i] >= 1 && cls[i] <= n_class)
      atomicAdd(&h[(b - 1) + n_bin * (cls[i] - 1)], 1);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < n_cells; c += blockDim.x) scratch[(size_t)blockIdx.x * n_cells + c] = h[c];
}

// one block: cell totals, starts and per-chunk offsets (one thread per cell)
__global__ void k_na_scan(int n_chunks, int n_cells, int* scratch, int* cell_count, int* cell_start) {
  __shared__ int ws[32];
  int c = threadIdx.x;
  int tot = 0;
  if (c < n_cells)
    for (int k = 0; k < n_chunks; k++) tot += scratch[(size_t)k * n_cells + c];
  // block exclusive scan of tot
  int lane = c & 31, wid = c >> 5;
  int x = tot;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int s = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    ws[lane] = s;
  }
  __syncthreads();
  int start = (wid > 0 ? ws[wid - 1] : 0) + x - tot;
  if (c < n_cells) {
    cell_count[c] = tot;
    cell_start[c] = start;
    int run = start;
    for (int k = 0; k < n_chunks; k++) {
      int v = scratch[(size_t)k * n_cells + c];
      scratch[(size_t)k * n_cells + c] = run;
      run += v;
    }
  }
  if (c == 0) cell_start[n_cells] = ws[(blockDim.x >> 5) - 1];
}

// stable scatter: particle order kept inside each cell
__global__ void k_na_scatter(int n, const int* cls, const int* bin, int n_bin, int n_class, int n_cells,
                             const int* scratch, int* list) {
  extern __shared__ int wc[];  // [kNaWarps][n_cells]
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < kNaWarps * n_cells; k += blockDim.x) wc[k] = 0;
  __syncthreads();
  int base = blockIdx.x * kNaChunk + w * kNaWarpSlots;
  for (int t = 0; t < kNaWarpSlots; t += 32) {
    int i = base + t + lane;
    int key = -1;
    if (i < n && bin[i] >= 1 && bin[i] <= n_bin && cls[i] >= 1 && cls[i] <= n_class)
      key = (bin[i] - 1) + n_bin * (cls[i] - 1);
    unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key >= 0 && lane == __ffs(peers) - 1) wc[w * n_cells + key] += __popc(peers);
  }
  __syncthreads();
  const int* off = scratch + (size_t)blockIdx.x * n_cells;
  for (int c = threadIdx.x; c < n_cells; c += blockDim.x) {
    int run = off[c];
    for (int q = 0; q < kNaWarps; q++) {
      int v = wc[q * n_cells + c];
      wc[q * n_cells + c] = run;
      run += v;
    }
  }
  __syncthreads();
  unsigned lt = (1u << lane) - 1u;
  for (int t = 0; t < kNaWarpSlots; t += 32) {
    int i = base + t + lane;
    int key = -1;
    if (i < n && bin[i] >= 1 && bin[i] <= n_bin && cls[i] >= 1 && cls[i] <= n_class)
      key = (bin[i] - 1) + n_bin * (cls[i] - 1);
    unsigned peers = __match_any_sync(0xffffffffu, key);
    int pos = key >= 0 ? wc[w * n_cells + key] + __popc(peers & lt) : 0;
    __syncwarp();
    if (key >= 0 && lane == __ffs(peers) - 1) wc[w * n_cells + key] += __popc(peers);
    __syncwarp();
    if (key >= 0) list[pos] = i;
  }
}

// device address of the static scratch, looked up once per device
constexpr int kMaxDevices = 64;
int* g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mu;

int scratch_for_current_device(int** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PMC_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return PMC_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    // host code may not use g_bin_sort_scratch as a device address; ask the
    // runtime for the address on this device
    if (cudaGetSymbolAddress(&p, g_bin_sort_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return PMC_ERR_CUDA;
    }
    g_scratch_addr[dev] = (int*)p;
  }
  *out = g_scratch_addr[dev];
  return PMC_OK;
}

}  // namespace
}  // namespace pmc

extern "C" int pmc_coag_gpu_bin_sort_noalloc(int n_part, const double* vtot_dev, const int* cls_dev,
                                             int n_bin, int n_class, double edge_min, double edge_max,
                                             int* bin_dev, int* cell_count_dev, int* cell_start_dev,
                                             int* list_dev, void* stream) {
  using namespace pmc;
  if (n_part < 0 || n_bin < 1 || n_class < 1 || !(edge_min > 0.0) || !(edge_max > edge_min))
    return PMC_ERR_INVALID_ARG;
  if (n_part > 0 && (!vtot_dev || !cls_dev || !bin_dev || !list_dev)) return PMC_ERR_INVALID_ARG;
  if (!cell_count_dev || !cell_start_dev) return PMC_ERR_INVALID_ARG;
  if (n_part > kNaMaxPart || (long long)n_bin * n_class > kNaMaxCells || n_bin > kMaxBin)
    return PMC_ERR_CAPACITY;
  int* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != PMC_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  int n_cells = n_bin * n_class;
  int n_chunks = n_part > 0 ? (n_part + kNaChunk - 1) / kNaChunk : 0;
  // the same host logarithms the context's sort uses for its grid
  double log_lo = log(edge_min), log_hi = log(edge_max);
  if (n_chunks > 0)
    k_na_hist<<<n_chunks, kNaThreads, sizeof(int) * n_cells, s>>>(n_part, vtot_dev, cls_dev, n_bin, n_class, n_cells,
                                                                   log_lo, log_hi, bin_dev, scratch);
  k_na_scan<<<1, 1024, 0, s>>>(n_chunks, n_cells, scratch, cell_count_dev, cell_start_dev);
  if (n_chunks > 0)
    k_na_scatter<<<n_chunks, kNaThreads, sizeof(int) * kNaWarps * n_cells, s>>>(
        n_part, cls_dev, bin_dev, n_bin, n_class, n_cells, scratch, list_dev);
  if (cudaGetLastError() != cudaSuccess) return PMC_ERR_CUDA;
  return PMC_OK;
}
