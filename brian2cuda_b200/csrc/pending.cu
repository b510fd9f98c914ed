// The step as two concurrent launches, for networks whose every synaptic delay is at least
// one step: the delivery into a double-buffered input, and the fold at the end of a chunk.
//
// The per-step path (neuron.cu then propagate.cu) runs the neuron update and the spike
// delivery of a step as two dependent launches, because Brian2's schedule applies the
// synaptic effects of step t after the update of step t.  When every delay is >= 1 step the
// delivery of step t only reads spikes of steps t - d <= t - 1, so its one dependence on the
// update of step t is the target variable itself.  Double-buffering that input removes it:
//
//   delivery of step t:  the bundles due at step t are added into acc[t & 1] (this file);
//   update of step t:    the per-step neuron kernel (neuron.cu), which adds in the input
//                        that arrived during step t-1, acc[(t-1) & 1], and clears it.
//
// The library launches the two side by side, the delivery on a second stream: the delivery
// of step t waits for the update of step t-1, the update of step t for the update and the
// delivery of step t-1 (api.cu, enqueue_steps).  The update of step t+1 sees exactly the
// value Brian2's schedule produces (state after step t's update plus every effect of step t's
// synapses slot).  A fold kernel at the end of every chunk of steps adds the pending input
// into the target variables, so between chunks the state is the ordinary one.
#include "pending_body.cuh"

namespace b2b {

namespace {

// Bundles due at step clock+k (spikes of steps ts - d, d >= 1) added into acc[ts & 1].
template <typename R, bool WARP_PREFIX, int GROUP>
__global__ void __launch_bounds__(kPendingBlock)
deliver_pending_kernel(const __grid_constant__ PendingDev F, const int64_t* __restrict__ clock,
                       int k) {
  extern __shared__ int s_pref[];  // F.nd_max + 1 ints when !WARP_PREFIX
  deliver_pending_body<R, WARP_PREFIX, GROUP>(F, clock, k, blockIdx.x, gridDim.x, s_pref);
}

// Adds the input delivered in step clock+k_last into the target variables and zeroes it.
template <typename R>
__global__ void fold_pending_kernel(const __grid_constant__ PendingDev F,
                                    const int64_t* __restrict__ clock, int k_last) {
  const int last = (int)((clock[0] + k_last) & 1);
  const int64_t n = F.pop.n;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int v = B2B_VAR_GE; v <= B2B_VAR_GI; ++v) {
    if (!F.acc[v]) continue;
    R* X = static_cast<R*>(F.pop.var[v]);
    R* A = static_cast<R*>(F.acc[v]) + (int64_t)last * n;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
      X[q] += A[q];
      A[q] = (R)0;
    }
  }
}

template <typename R, bool WP>
cudaError_t launch_pending_r(const PendingDev& F, dim3 g, size_t smem, const int64_t* clock,
                             int k, cudaStream_t s) {
  if (F.group == 16)
    deliver_pending_kernel<R, WP, 16><<<g, kPendingBlock, smem, s>>>(F, clock, k);
  else if (F.group == 4)
    deliver_pending_kernel<R, WP, 4><<<g, kPendingBlock, smem, s>>>(F, clock, k);
  else if (F.group == 2)
    deliver_pending_kernel<R, WP, 2><<<g, kPendingBlock, smem, s>>>(F, clock, k);
  else
    deliver_pending_kernel<R, WP, 8><<<g, kPendingBlock, smem, s>>>(F, clock, k);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pending_delivery(const PendingDev& F, int dtype, int grid,
                                    const int64_t* clock, int k, cudaStream_t s) {
  const bool wp = F.nd_max <= kWarpPrefixMaxDelays;
  const size_t smem = wp ? 0 : sizeof(int) * (size_t)(F.nd_max + 1);
  const dim3 g((unsigned)grid);
  if (dtype == B2B_F32)
    return wp ? launch_pending_r<float, true>(F, g, smem, clock, k, s)
              : launch_pending_r<float, false>(F, g, smem, clock, k, s);
  return wp ? launch_pending_r<double, true>(F, g, smem, clock, k, s)
            : launch_pending_r<double, false>(F, g, smem, clock, k, s);
}

cudaError_t launch_fold_pending(const PendingDev& F, int dtype, const int64_t* clock, int k_last,
                                cudaStream_t s) {
  const int64_t n = F.pop.n;
  int64_t blocks = (n + kPendingBlock - 1) / kPendingBlock;
  if (blocks > 4 * kNumSMs) blocks = 4 * kNumSMs;
  const dim3 g((unsigned)blocks);
  if (dtype == B2B_F32) fold_pending_kernel<float><<<g, kPendingBlock, 0, s>>>(F, clock, k_last);
  else fold_pending_kernel<double><<<g, kPendingBlock, 0, s>>>(F, clock, k_last);
  return cudaGetLastError();
}

}  // namespace b2b
