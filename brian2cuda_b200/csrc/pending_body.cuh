// The delivery half of the step forms whose every synaptic delay is at least one step
// (pending.cu: its own launch beside the update; neuron.cu: the CTAs after the update's in
// the one-launch step): the bundles due at step clock+k are added into the pending input
// acc[ts & 1] instead of the target variables.
#pragma once
#include "delivery.cuh"

namespace b2b {
namespace {

constexpr int kPendingBlock = 256;
constexpr int kPendingUnroll = 4;   // rounds of a bundle whose loads a lane issues together

// The work of CTA `blk` of `nblk` delivering CTAs (blockDim.x threads each).
template <typename R, bool WARP_PREFIX, int GROUP>
__device__ __forceinline__ void deliver_pending_body(const PendingDev& F,
                                                     const int64_t* __restrict__ clock, int k,
                                                     int64_t blk, int64_t nblk, int* s_pref) {
  const int64_t ts = clock[0] + k;
  const int64_t warp0 = (blk * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (nblk * blockDim.x) >> 5;
  const int64_t row = (int64_t)(ts & 1) * F.pop.n;
  const int glane = (threadIdx.x & 31) % GROUP;
  for (int p = 0; p < F.n_proj; ++p) {
    const ProjDev& J = F.proj[p];
    const R* W = static_cast<const R*>(J.w);
    MemberCache<R> mc;
    for_each_due_item<WARP_PREFIX, GROUP>(J, ts, warp0, nwarps, s_pref,
                                          [&](int64_t b0, int64_t b1, int64_t len, int32_t pre) {
      member_lookup<R>(J, pre, mc);
      // the loads of kPendingUnroll rounds first, then their atomics
      for (int64_t off = 0; off < len; off += kPendingUnroll * GROUP) {
        int32_t post[kPendingUnroll];
        R w[kPendingUnroll];
        bool v[kPendingUnroll];
#pragma unroll
        for (int u = 0; u < kPendingUnroll; ++u) {
          const int64_t s = b0 + off + u * GROUP + glane;
          v[u] = s < b1;
          post[u] = v[u] ? __ldg(J.post + s) : 0;
          w[u] = v[u] && W ? __ldg(W + s) : mc.w;
        }
#pragma unroll
        for (int u = 0; u < kPendingUnroll; ++u)
          if (v[u]) atomicAdd(mc.target + row + post[u], w[u]);
      }
    });
  }
}

}  // namespace
}  // namespace b2b
