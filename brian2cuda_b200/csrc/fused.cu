// The step as two concurrent launches, for networks whose every synaptic delay is at least
// one step.
//
// The per-step path (neuron.cu then propagate.cu) runs the neuron update and the spike
// delivery of a step as two dependent launches, because Brian2's schedule applies the
// synaptic effects of step t after the update of step t.  When every delay is >= 1 step the
// delivery of step t only reads spikes of steps t - d <= t - 1, so its one dependence on the
// update of step t is the target variable itself.  Double-buffering that input removes it:
//
//   delivery of step t:  the bundles due at step t are added into acc[t & 1];
//   update of step t:    one neuron per thread, reading the input that arrived during step
//                        t-1 from acc[(t-1) & 1] (and zeroing it), spikes compacted into
//                        ring slot t.
//
// fused_step_kernel takes either role by CTA (CTAs below deliver_ctas deliver, the rest
// update), so one launch can hold both halves; the library launches it twice per step, once
// per role, the delivery on a second stream: the delivery of step t waits for the update of
// step t-1, the update of step t for the update and the delivery of step t-1, and the two
// launches of a step run side by side (api.cu, enqueue_steps).  The update of step t+1 sees
// exactly the value Brian2's schedule produces (state after step t's update plus every
// effect of step t's synapses slot).  A fold kernel at the end of every chunk of steps adds
// the pending accumulator into the target variables, so between chunks the state is the
// ordinary one.
#include "delivery.cuh"
#include "neuron_math.cuh"

namespace b2b {

namespace {

constexpr int kFusedBlock = 256;

// Appends this warp's spikes (flag per lane, neuron q) to ring slot `slot` and the monitor.
__device__ __forceinline__ void warp_emit(const PopDev& P, bool spk, int32_t q, int64_t ts,
                                          int slot, int32_t* status) {
  const unsigned ballot = __ballot_sync(kFull, spk);
  if (!ballot) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(ballot) - 1;
  const int cnt = __popc(ballot);
  int base = 0;
  unsigned long long mbase = 0;
  if (lane == leader) {
    base = atomicAdd(&P.ring_cnt[slot], cnt);
    if (P.mon_cnt) mbase = atomicAdd(P.mon_cnt, (unsigned long long)cnt);
  }
  base = __shfl_sync(kFull, base, leader);
  mbase = __shfl_sync(kFull, mbase, leader);
  if (spk) {
    const int r = __popc(ballot & ((1u << lane) - 1u));
    P.ring_idx[(int64_t)slot * P.n + base + r] = q;
    if (P.mon_cnt) {
      if (mbase + r < (unsigned long long)P.mon_cap) {
        P.mon_idx[mbase + r] = q;
        P.mon_step[mbase + r] = ts;
      } else {
        set_status(status, B2B_ERR_QUEUE_OVERFLOW);
      }
    }
  }
}

// Neuron q of step ts: fold the pending input, integrate, threshold, reset.
template <typename R, int KIND>
__device__ __forceinline__ bool update_neuron(const FusedDev& F, int64_t q, double t, double dt,
                                              double inv_dt, int prev) {
  const PopDev& P = F.pop;
  const int gidx = P.vec_group ? P.vec_group[q >> 2] : 0;
  R* V = static_cast<R*>(P.var[B2B_VAR_V]);
  R* GE = static_cast<R*>(P.var[B2B_VAR_GE]);
  R* GI = static_cast<R*>(P.var[B2B_VAR_GI]);
  R ge = GE[q], gi = GI[q];
  if (F.acc[B2B_VAR_GE]) {
    R* a = static_cast<R*>(F.acc[B2B_VAR_GE]) + (int64_t)prev * P.n + q;
    ge += *a;
    *a = (R)0;
  }
  if (F.acc[B2B_VAR_GI]) {
    R* a = static_cast<R*>(F.acc[B2B_VAR_GI]) + (int64_t)prev * P.n + q;
    gi += *a;
    *a = (R)0;
  }
  R* LS = static_cast<R*>(P.var[B2B_VAR_LASTSPIKE]);
  uint8_t* NR = static_cast<uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY]);
  bool spk = false;
  if constexpr (KIND == KIND_HH) {
    const HhRun<R> g = hh_run(static_cast<const HhDev*>(P.params)[gidx], R());  // no reloads
    const bool refr = g.ref_steps >= 0;
    bool nr = true;
    if (refr) nr = timestep_of(t - (double)LS[q], dt, inv_dt) >= g.ref_steps;
    R* M = static_cast<R*>(P.var[B2B_VAR_M]);
    R* H = static_cast<R*>(P.var[B2B_VAR_H]);
    R* N = static_cast<R*>(P.var[B2B_VAR_N]);
    R m = M[q], h = H[q], n = N[q];
    const R vn = hh_advance<R>(g, V[q], m, h, n, ge, gi, (R)dt);
    if ((q - g.offset) < g.n && vn > (R)g.Vthr && nr) {
      nr = false;
      spk = true;
      if (refr) LS[q] = (R)t;
    }
    V[q] = vn;
    M[q] = m;
    H[q] = h;
    N[q] = n;
    if (refr) NR[q] = nr ? 1 : 0;
  } else {
    const LifDev g = static_cast<const LifDev*>(P.params)[gidx];  // by value: no reloads
    const bool refr = g.ref_steps >= 0;
    bool nr = true;
    if (refr) nr = timestep_of(t - (double)LS[q], dt, inv_dt) >= g.ref_steps;
    R vn = lif_advance<R>(g, V[q], ge, gi, nr);
    if (g.has_threshold && (q - g.offset) < g.n && vn > (R)g.Vt && nr) {
      nr = false;
      spk = true;
      if (refr) LS[q] = (R)t;
      if (g.has_reset) vn = (R)g.Vr;
    }
    V[q] = vn;
    if (refr) NR[q] = nr ? 1 : 0;
  }
  GE[q] = ge;
  GI[q] = gi;
  return spk;
}

constexpr int kFusedUnroll = 4;   // rounds of a bundle whose loads a lane issues together

template <typename R, int KIND, bool WARP_PREFIX, int GROUP>
__global__ void __launch_bounds__(kFusedBlock)
fused_step_kernel(const __grid_constant__ FusedDev F, const int64_t* __restrict__ clock, int k,
                  double dt, int32_t* status) {
  extern __shared__ int s_pref[];  // F.nd_max + 1 ints when !WARP_PREFIX
  const PopDev& P = F.pop;
  const int64_t ts = clock[0] + k;
  if ((int)blockIdx.x >= F.deliver_ctas) {
    // ---- neuron half: one neuron per thread (scheduled after the delivery CTAs)
    const int slot = ring_slot(ts, P.ring_len);
    const int64_t nb = (int64_t)blockIdx.x - F.deliver_ctas;
    const int64_t q = nb * blockDim.x + threadIdx.x;
    if (q < P.n) {  // P.n is a multiple of 32: whole warps take this branch
      const bool spk = update_neuron<R, KIND>(F, q, (double)ts * dt, dt, 1.0 / dt,
                                              (int)((ts & 1) ^ 1));
      warp_emit(P, spk, (int32_t)q, ts, slot, status);
    }
    if (nb == 0 && threadIdx.x == 0) P.ring_cnt[ring_slot(ts + 1, P.ring_len)] = 0;
    return;
  }
  // ---- delivery half: bundles due at step ts (spikes of steps ts - d, d >= 1) into acc[ts & 1]
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)F.deliver_ctas * blockDim.x) >> 5;
  const int par = (int)(ts & 1);
  const int glane = (threadIdx.x & 31) % GROUP;
  for (int p = 0; p < F.n_proj; ++p) {
    const ProjDev& J = F.proj[p];
    const R* W = static_cast<const R*>(J.w);
    MemberCache<R> mc;
    for_each_due_item<WARP_PREFIX, GROUP>(J, ts, warp0, nwarps, s_pref,
                                          [&](int64_t b0, int64_t b1, int64_t len, int32_t pre) {
      member_lookup<R>(J, pre, mc);
      // the loads of kFusedUnroll rounds first, then their atomics
      for (int64_t off = 0; off < len; off += kFusedUnroll * GROUP) {
        int32_t post[kFusedUnroll];
        R w[kFusedUnroll];
        bool v[kFusedUnroll];
#pragma unroll
        for (int u = 0; u < kFusedUnroll; ++u) {
          const int64_t s = b0 + off + u * GROUP + glane;
          v[u] = s < b1;
          post[u] = v[u] ? __ldg(J.post + s) : 0;
          w[u] = v[u] && W ? __ldg(W + s) : mc.w;
        }
#pragma unroll
        for (int u = 0; u < kFusedUnroll; ++u)
          if (v[u]) atomicAdd(mc.target + (int64_t)par * P.n + post[u], w[u]);
      }
    });
  }
}

// Adds the input delivered in step clock+k_last into the target variables and zeroes it.
template <typename R>
__global__ void fused_fold_kernel(const __grid_constant__ FusedDev F,
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

}  // namespace

size_t fused_smem(const FusedDev& F) {
  return F.nd_max <= kWarpPrefixMaxDelays ? 0 : sizeof(int) * (size_t)(F.nd_max + 1);
}

int fused_block() { return kFusedBlock; }

int fused_resident_ctas(int kind, int dtype, const FusedDev& F, int sms) {
  const size_t smem = fused_smem(F);
  const bool wp = F.nd_max <= kWarpPrefixMaxDelays;
  int occ = 0;
#define B2B_OCC(R, KD, WP) \
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fused_step_kernel<R, KD, WP, 8>, kFusedBlock, smem)
  if (kind == KIND_HH) {
    if (dtype == B2B_F32) { if (wp) B2B_OCC(float, KIND_HH, true); else B2B_OCC(float, KIND_HH, false); }
    else { if (wp) B2B_OCC(double, KIND_HH, true); else B2B_OCC(double, KIND_HH, false); }
  } else {
    if (dtype == B2B_F32) { if (wp) B2B_OCC(float, KIND_LIF, true); else B2B_OCC(float, KIND_LIF, false); }
    else { if (wp) B2B_OCC(double, KIND_LIF, true); else B2B_OCC(double, KIND_LIF, false); }
  }
#undef B2B_OCC
  return occ * sms;
}

cudaError_t launch_fused_step(const FusedDev& F, int kind, int dtype, int grid,
                              const int64_t* clock, int k, double dt, int32_t* status,
                              cudaStream_t s) {
  const size_t smem = fused_smem(F);
  const dim3 g(grid);
  const bool wp = F.nd_max <= kWarpPrefixMaxDelays;
#define B2B_FS(R, KD, WP)                                                                    \
  (F.group == 16 ? (fused_step_kernel<R, KD, WP, 16><<<g, kFusedBlock, smem, s>>>(F, clock, k, dt, \
                                                                              status), 0)   \
   : F.group == 4 ? (fused_step_kernel<R, KD, WP, 4><<<g, kFusedBlock, smem, s>>>(F, clock, k, dt, \
                                                                              status), 0)   \
   : (fused_step_kernel<R, KD, WP, 8><<<g, kFusedBlock, smem, s>>>(F, clock, k, dt, status), 0), \
   cudaGetLastError())
  if (kind == KIND_HH) {
    if (dtype == B2B_F32) return wp ? B2B_FS(float, KIND_HH, true) : B2B_FS(float, KIND_HH, false);
    return wp ? B2B_FS(double, KIND_HH, true) : B2B_FS(double, KIND_HH, false);
  }
  if (dtype == B2B_F32) return wp ? B2B_FS(float, KIND_LIF, true) : B2B_FS(float, KIND_LIF, false);
  return wp ? B2B_FS(double, KIND_LIF, true) : B2B_FS(double, KIND_LIF, false);
#undef B2B_FS
}

cudaError_t launch_fused_fold(const FusedDev& F, int dtype, const int64_t* clock, int k_last,
                              cudaStream_t s) {
  const int64_t n = F.pop.n;
  int64_t blocks = (n + kFusedBlock - 1) / kFusedBlock;
  if (blocks > 4 * kNumSMs) blocks = 4 * kNumSMs;
  const dim3 g((unsigned)blocks);
  const dim3 b(kFusedBlock);
  if (dtype == B2B_F32) fused_fold_kernel<float><<<g, b, 0, s>>>(F, clock, k_last);
  else fused_fold_kernel<double><<<g, b, 0, s>>>(F, clock, k_last);
  return cudaGetLastError();
}

}  // namespace b2b
