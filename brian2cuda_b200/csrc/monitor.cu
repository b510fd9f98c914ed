// State and population-rate monitors: one launch per step for all state monitors (at the
// start of the step) and one for all rate monitors (at its end), present only when the net
// has such monitors.
//
// Reference: the StateMonitor code object writes, one thread per recorded index, the
// variable into a per-index thrust vector resized on the host before every run
// (brian2cuda/templates/statemonitor.cu:8-101); the PopulationRateMonitor runs a one-thread
// kernel that scans the whole spikespace every step (templates/ratemonitor.cu:40-100).
// Here the records go to preallocated device buffers, record-major (one row of all recorded
// indices per record, coalesced writes), with the record count kept on the device, so the
// monitors run inside the replayed step graphs; the spike count comes from the spike-history
// ring slot of the step (its count, or a CTA-wide count over the slot for a group that is
// part of a population).
#include "kernels_common.cuh"

namespace b2b {

namespace {

__global__ void __launch_bounds__(kBlock)
statemon_kernel(const StateMonDev* __restrict__ mons, const int64_t* __restrict__ clock, int k,
                int32_t* status) {
  const StateMonDev& M = mons[blockIdx.y];
  const int64_t ts = clock[0] + k;
  if (ts % M.every != 0) return;  // the same for every CTA of this monitor
  // the count changes only after every CTA of this monitor has taken its ticket below
  const unsigned long long r = __ldcg(M.cnt);
  const bool full = r >= (unsigned long long)M.cap;
  if (!full) {
    const int64_t row = (int64_t)r * M.n_idx;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < M.n_idx;
         q += (int64_t)gridDim.x * blockDim.x) {
      const int64_t i = M.idx[q];
      if (M.es == 8)
        reinterpret_cast<uint64_t*>(M.buf)[row + q] = reinterpret_cast<const uint64_t*>(M.src)[i];
      else if (M.es == 4)
        reinterpret_cast<uint32_t*>(M.buf)[row + q] = reinterpret_cast<const uint32_t*>(M.src)[i];
      else
        M.buf[row + q] = M.src[i];
    }
  } else if (blockIdx.x == 0 && threadIdx.x == 0) {
    set_status(status, B2B_ERR_QUEUE_OVERFLOW);
  }
  // the last CTA of this monitor to finish the record advances the count
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(M.ticket, 1u);
    if (done == gridDim.x - 1) {
      *M.ticket = 0u;
      if (!full) {
        M.steps[r] = ts;
        __threadfence();
        atomicAdd(M.cnt, 1ull);
      }
    }
  }
}

__global__ void __launch_bounds__(kBlock)
ratemon_kernel(const RateMonDev* __restrict__ mons, const int64_t* __restrict__ clock, int k,
               int32_t* status) {
  const RateMonDev& M = mons[blockIdx.x];
  const int64_t ts = clock[0] + k;
  const int slot = ring_slot(ts, M.ring_len);
  const int nspk = M.ring_cnt[slot];
  int c = 0;
  if (M.whole) {
    c = nspk;
  } else {
    const int32_t* spk = M.ring_idx + (int64_t)slot * M.ring_n;
    int mine = 0;
    for (int i = threadIdx.x; i < nspk; i += blockDim.x) {
      const int32_t j = spk[i];
      mine += (j >= M.lo && j < M.hi) ? 1 : 0;
    }
    __shared__ int s_sum;
    if (threadIdx.x == 0) s_sum = 0;
    __syncthreads();
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_sum, mine);
    __syncthreads();
    c = s_sum;
  }
  if (threadIdx.x == 0) {
    const unsigned long long r = *M.cnt;
    if (r < (unsigned long long)M.cap) {
      M.buf[r] = c;
      M.steps[r] = ts;
      *M.cnt = r + 1;
    } else {
      set_status(status, B2B_ERR_QUEUE_OVERFLOW);
    }
  }
}

}  // namespace

cudaError_t launch_statemon(const StateMonDev* d_mons, int n_mons, int64_t max_idx,
                            const int64_t* clock, int k, int32_t* status, cudaStream_t s) {
  if (n_mons <= 0) return cudaSuccess;
  int64_t gx = (max_idx + kBlock - 1) / kBlock;
  if (gx < 1) gx = 1;
  if (gx > 2 * kNumSMs) gx = 2 * kNumSMs;
  statemon_kernel<<<dim3((unsigned)gx, (unsigned)n_mons), kBlock, 0, s>>>(d_mons, clock, k,
                                                                         status);
  return cudaGetLastError();
}

cudaError_t launch_ratemon(const RateMonDev* d_mons, int n_mons, const int64_t* clock, int k,
                           int32_t* status, cudaStream_t s) {
  if (n_mons <= 0) return cudaSuccess;
  ratemon_kernel<<<(unsigned)n_mons, kBlock, 0, s>>>(d_mons, clock, k, status);
  return cudaGetLastError();
}

}  // namespace b2b
