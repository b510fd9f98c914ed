// Measured ceiling of scattered float32 atomic additions on this GPU (no counterpart in the
// reference).  The additive spike delivery does one `red.global.add.f32` per synaptic event
// at a target index that the synapse table gives (brian2cuda's effect kernels do the same
// with atomicAdd, brian2cuda/templates/synapses.cu:117-162), so its throughput is bounded
// by how many such additions the L2 slices accept, not by DRAM bandwidth.  This probe
// measures that bound on the device it runs on, for a target array of the size of a
// population's synaptic variables, in two forms:
//   - the index of every event loaded from an index array in HBM (4 B per event, the way
//     the delivery reads its synapses' targets), then the addition;
//   - the index computed in registers (a hash of the event number): atomics alone.
// The indices are uniform over the targets, like the targets of random connectivity.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "kernels_common.cuh"

namespace b2b {
namespace {

__device__ __forceinline__ uint32_t mix32(uint64_t x) {
  // SplitMix64's finaliser (Steele, Lea, Flood, OOPSLA 2014), folded to 32 bits.
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (uint32_t)x;
}

__device__ __forceinline__ uint32_t target_of(uint64_t e, uint32_t n_targets) {
  return (uint32_t)(((uint64_t)mix32(e) * n_targets) >> 32);
}

__global__ void probe_fill_kernel(int32_t* __restrict__ idx, int64_t n, uint32_t n_targets) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
    idx[e] = (int32_t)target_of((uint64_t)e, n_targets);
}

// Four events per thread and round, their index loads issued before the additions (the
// delivery kernel keeps four loads in flight per lane the same way).
__global__ void probe_scatter_loaded_kernel(const int32_t* __restrict__ idx, int64_t n,
                                            float* __restrict__ target, float w) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; e + 3 * stride < n; e += 4 * stride) {
    int32_t t[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) t[u] = __ldcs(idx + e + u * stride);
#pragma unroll
    for (int u = 0; u < 4; ++u) atomicAdd(target + t[u], w);
  }
  for (; e < n; e += stride) atomicAdd(target + __ldcs(idx + e), w);
}

__global__ void probe_scatter_hashed_kernel(int64_t n, uint32_t n_targets,
                                            float* __restrict__ target, float w) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
    atomicAdd(target + target_of((uint64_t)e, n_targets), w);
}

}  // namespace
}  // namespace b2b

using namespace b2b;

extern "C" b2b_status b2b_atomic_rate(int32_t device, void* stream, int64_t n_targets,
                                      int64_t n_events, int32_t reps, double* loaded_per_s,
                                      double* hashed_per_s) {
  if (n_targets <= 0 || n_targets > (1ll << 31) - 1 || n_events <= 0 || reps <= 0 ||
      !loaded_per_s || !hashed_per_s)
    return B2B_ERR_INVALID_ARG;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return B2B_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return B2B_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float* target = nullptr;
  int32_t* idx = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  b2b_status st = B2B_OK;
  cudaError_t e = cudaMalloc(&target, sizeof(float) * (size_t)n_targets);
  if (e == cudaSuccess) e = cudaMalloc(&idx, sizeof(int32_t) * (size_t)n_events);
  if (e != cudaSuccess) st = B2B_ERR_OOM;
  if (st == B2B_OK) {
    int sms = kNumSMs;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const unsigned grid = (unsigned)(8 * sms);
    e = cudaMemsetAsync(target, 0, sizeof(float) * (size_t)n_targets, s);
    if (e == cudaSuccess) {
      probe_fill_kernel<<<grid, 256, 0, s>>>(idx, n_events, (uint32_t)n_targets);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float best[2] = {1e30f, 1e30f};
    for (int form = 0; form < 2 && e == cudaSuccess; ++form) {
      for (int r = 0; r < reps + 1 && e == cudaSuccess; ++r) {   // the first is a warm-up
        e = cudaEventRecord(e0, s);
        if (e != cudaSuccess) break;
        if (form == 0)
          probe_scatter_loaded_kernel<<<grid, 256, 0, s>>>(idx, n_events, target, 1e-9f);
        else
          probe_scatter_hashed_kernel<<<grid, 256, 0, s>>>(n_events, (uint32_t)n_targets,
                                                           target, 1e-9f);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && r > 0) best[form] = std::min(best[form], ms);
      }
    }
    if (e == cudaSuccess) {
      *loaded_per_s = (double)n_events / (best[0] * 1e-3);
      *hashed_per_s = (double)n_events / (best[1] * 1e-3);
    } else {
      st = B2B_ERR_CUDA;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (target) cudaFree(target);
  if (idx) cudaFree(idx);
  cudaSetDevice(prev);
  return st;
}
