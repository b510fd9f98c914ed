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
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "kernels_common.cuh"

namespace b2b {
namespace {
namespace cg = cooperative_groups;

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

// The same additions into the distributed shared memory of a cluster of kProbeCluster CTAs:
// the target array is split into kProbeCluster slices, one per CTA's shared memory, and an
// event adds into the slice of whichever CTA holds its target (a remote shared-memory atomic
// for all but 1/kProbeCluster of them).  Every cluster takes an equal share of the events; the
// slices are zeroed first and the cluster synchronises before and after, as an accumulating
// delivery would.
constexpr int kProbeCluster = 8;
__global__ void __cluster_dims__(kProbeCluster, 1, 1)
probe_dsmem_kernel(int64_t n, uint32_t n_targets, float w) {
  extern __shared__ float s_slice[];
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t slice = (n_targets + kProbeCluster - 1) / kProbeCluster;
  for (uint32_t i = threadIdx.x; i < slice; i += blockDim.x) s_slice[i] = 0.f;
  cluster.sync();
  const int64_t clusters = gridDim.x / kProbeCluster;
  const int64_t cid = blockIdx.x / kProbeCluster;
  const int64_t per = (n + clusters - 1) / clusters;
  const int64_t lo = cid * per, hi = lo + per < n ? lo + per : n;
  const int64_t stride = (int64_t)kProbeCluster * blockDim.x;
  for (int64_t e = lo + (int64_t)cluster.block_rank() * blockDim.x + threadIdx.x; e < hi;
       e += stride) {
    const uint32_t t = target_of((uint64_t)e, n_targets);
    float* dst = cluster.map_shared_rank(s_slice, t / slice);
    atomicAdd(dst + t % slice, w);
  }
  cluster.sync();
}

}  // namespace
}  // namespace b2b

using namespace b2b;

extern "C" b2b_status b2b_atomic_rate(int32_t device, void* stream, int64_t n_targets,
                                      int64_t n_events, int32_t reps, double* loaded_per_s,
                                      double* hashed_per_s, double* dsmem_per_s) {
  if (n_targets <= 0 || n_targets > (1ll << 31) - 1 || n_events <= 0 || reps <= 0 ||
      !loaded_per_s || !hashed_per_s || !dsmem_per_s)
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
    // the distributed-shared-memory form: a slice of the targets per CTA of a cluster, as
    // many clusters as are resident together (0 when a slice exceeds the shared memory)
    const size_t slice_bytes =
        sizeof(float) * (size_t)((n_targets + kProbeCluster - 1) / kProbeCluster);
    int clusters = 0;
    const int dsmem_block = 512;
    if (e == cudaSuccess && slice_bytes <= 200 * 1024) {
      e = cudaFuncSetAttribute(probe_dsmem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)slice_bytes);
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(kProbeCluster * 64);
      cfg.blockDim = dim3(dsmem_block);
      cfg.dynamicSmemBytes = slice_bytes;
      cudaLaunchAttribute attr;
      attr.id = cudaLaunchAttributeClusterDimension;
      attr.val.clusterDim.x = kProbeCluster;
      attr.val.clusterDim.y = 1;
      attr.val.clusterDim.z = 1;
      cfg.attrs = &attr;
      cfg.numAttrs = 1;
      if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&clusters, probe_dsmem_kernel, &cfg);
    }
    float best[3] = {1e30f, 1e30f, 1e30f};
    for (int form = 0; form < 3 && e == cudaSuccess; ++form) {
      if (form == 2 && clusters <= 0) break;
      for (int r = 0; r < reps + 1 && e == cudaSuccess; ++r) {   // the first is a warm-up
        e = cudaEventRecord(e0, s);
        if (e != cudaSuccess) break;
        if (form == 0)
          probe_scatter_loaded_kernel<<<grid, 256, 0, s>>>(idx, n_events, target, 1e-9f);
        else if (form == 1)
          probe_scatter_hashed_kernel<<<grid, 256, 0, s>>>(n_events, (uint32_t)n_targets,
                                                           target, 1e-9f);
        else
          probe_dsmem_kernel<<<(unsigned)(kProbeCluster * clusters), dsmem_block, slice_bytes,
                               s>>>(n_events, (uint32_t)n_targets, 1e-9f);
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
      *dsmem_per_s = clusters > 0 ? (double)n_events / (best[2] * 1e-3) : 0.0;
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
