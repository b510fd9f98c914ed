// Kernel template of generated neuron models (b2b_group_model).
//
// The device plugin turns a model that no hand-written kernel integrates into a struct of
// device functions — the integration step of its equations, its threshold condition and its
// reset statements, written out by brian2cuda_b200/codegen.py — and compiles it with this
// header into a shared object.  The kernel around them is the same fused pass as the
// hand-written neuron kernels (neuron.cu): one or four neurons per thread, refractoriness from
// lastspike, update, threshold, reset (unless a synapse writes a variable the reset writes:
// then a second launch resets the step's spiking neurons after the synaptic delivery, as
// Brian2's schedule orders them), and the CTA's spikes compacted into the population's slot of
// the spike-history ring with one atomic per CTA.  It replaces brian2cuda's per-code-object
// stateupdater, thresholder and resetter kernels (templates/common_group.cu:108-160,
// threshold.cu:19-45, reset.cu:3-27) for such models.
//
// The model struct M provides
//   static constexpr int NV, NN, NU;         state variables, normal and uniform draws
//   static constexpr unsigned RESET_MASK;    variables the reset writes
//   static constexpr bool HAS_THRESHOLD;
//   template <typename R> __device__ static void update(R (&x)[NV], double t, double dt,
//       bool not_refractory, const R* normal, const R* uniform, int64_t stride);
//   template <typename R> __device__ static bool threshold(const R (&x)[NV]);
//   template <typename R> __device__ static void reset(R (&x)[NV]);
// where draw d of the neuron's step is normal[d * stride] / uniform[d * stride].
#pragma once
#include "neuron_common.cuh"
#include "neuron_math.cuh"

namespace b2b {
namespace model {

template <typename R>
__device__ __forceinline__ R exprel(R z) {
  // (e^z - 1)/z with its limit 1 at z = 0 (Brian2's exprel, cuda_generator.py:858-867)
  return fabs(z) < (R)1e-16 ? (R)1 : expm1(z) / z;
}

template <typename R>
__device__ __forceinline__ R clip(R v, R lo, R hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

// A thread owns E consecutive neurons (E = 4 for populations large enough to fill the GPU
// that way: every state array and draw row read with one 128-bit access per thread, 8 B
// of index arithmetic and one compaction per four neurons); the arithmetic of each neuron is
// the same for every E.
template <class M, typename R, int E>
__global__ void __launch_bounds__(kBlock)
model_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k, double dt,
                  int32_t* status) {
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const double inv_dt = 1.0 / dt;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned fl = 0;
  if (q < P.n / E) {
    const ModelGroupDev g = static_cast<const ModelGroupDev*>(P.params)[0];
    const bool refr = g.ref_steps >= 0;
    Pack<R, E> X[M::NV];
#pragma unroll
    for (int v = 0; v < M::NV; ++v) X[v] = load_pack<R, E>(P.var[v], q);
    Pack<R, E> LS;
    if (refr) LS = load_pack<R, E>(P.var[B2B_VAR_LASTSPIKE], q);
    // this step's draws of the E neurons: draw d of neuron E q + e at D[d].x[e]
    constexpr int ND = M::NN + M::NU > 0 ? M::NN + M::NU : 1;
    Pack<R, E> D[ND];
#pragma unroll
    for (int d = 0; d < M::NN; ++d)
      D[d] = load_pack<R, E>(static_cast<const R*>(P.rng_normal) +
                                 ((int64_t)k * M::NN + d) * P.n, q);
#pragma unroll
    for (int d = 0; d < M::NU; ++d)
      D[M::NN + d] = load_pack<R, E>(static_cast<const R*>(P.rng) +
                                         ((int64_t)k * M::NU + d) * P.n, q);
    uint32_t NRout = 0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      R x[M::NV];
#pragma unroll
      for (int v = 0; v < M::NV; ++v) x[v] = X[v].x[e];
      bool nr = true;
      if (refr) nr = past_refractory(t - (double)LS.x[e], dt, inv_dt, g.ref_steps);
      R dn[ND], du[ND];
#pragma unroll
      for (int d = 0; d < M::NN; ++d) dn[d] = D[d].x[e];
#pragma unroll
      for (int d = 0; d < M::NU; ++d) du[d] = D[M::NN + d].x[e];
      M::template update<R>(x, t, dt, nr, dn, du, 1);
      const bool valid = E * q + e - g.offset < g.n;
      if (M::HAS_THRESHOLD && valid && nr && M::template threshold<R>(x)) {
        fl |= 1u << e;
        nr = false;
        if (refr) LS.x[e] = (R)t;
        if (!P.late_reset) M::template reset<R>(x);
      }
#pragma unroll
      for (int v = 0; v < M::NV; ++v) X[v].x[e] = x[v];
      NRout |= (nr ? 1u : 0u) << (8 * e);
    }
#pragma unroll
    for (int v = 0; v < M::NV; ++v) store_pack<R, E>(P.var[v], q, X[v]);
    if (refr) {
      if (fl) store_pack<R, E>(P.var[B2B_VAR_LASTSPIKE], q, LS);   // changes only on a spike
      store_flags<E>(P.var[B2B_VAR_NOT_REFRACTORY], q, NRout);
    }
  }
  emit_spikes<E>(P, q, fl, ts, slot, status);
  clear_next_slot(P, ts);
}

// The reset of the step's spiking neurons, after the synaptic delivery.
template <class M, typename R>
__global__ void model_late_reset_kernel(PopDev P, const int64_t* __restrict__ clock, int k) {
  const int64_t ts = clock[0] + k;
  const int slot = ring_slot(ts, P.ring_len);
  const int cnt = P.ring_cnt[slot];
  const int32_t* idx = P.ring_idx + (int64_t)slot * P.n;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < cnt; r += gridDim.x * blockDim.x) {
    const int32_t i = idx[r];
    R x[M::NV];
#pragma unroll
    for (int v = 0; v < M::NV; ++v) x[v] = static_cast<const R*>(P.var[v])[i];
    M::template reset<R>(x);
#pragma unroll
    for (int v = 0; v < M::NV; ++v)
      if (M::RESET_MASK & (1u << v)) static_cast<R*>(P.var[v])[i] = x[v];
  }
}

template <class M>
int32_t launch(const void* pop, const int64_t* clock, int32_t k, double dt, int32_t* status,
               void* stream, int32_t dtype, int32_t phase) {
  const PopDev& P = *static_cast<const PopDev*>(pop);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (phase == 0) {
    // four neurons per thread once that still gives every SM several CTAs' worth of warps
    const bool wide = P.n / 4 >= (int64_t)kNumSMs * 4 * kBlock;
    const unsigned grid = (unsigned)((P.n / (wide ? 4 : 1) + kBlock - 1) / kBlock);
    if (dtype == B2B_F32) {
      if (wide) model_step_kernel<M, float, 4><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
      else model_step_kernel<M, float, 1><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
    } else {
      if (wide) model_step_kernel<M, double, 4><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
      else model_step_kernel<M, double, 1><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
    }
  } else {
    const unsigned grid = 2 * kNumSMs;
    if (dtype == B2B_F32)
      model_late_reset_kernel<M, float><<<grid, kBlock, 0, s>>>(P, clock, k);
    else
      model_late_reset_kernel<M, double><<<grid, kBlock, 0, s>>>(P, clock, k);
  }
  return (int32_t)cudaGetLastError();
}

}  // namespace model
}  // namespace b2b

// The two entry points of a generated model's shared object (include/b2b.h).
#define B2B_MODEL_EXPORT(M)                                                                \
  extern "C" __attribute__((visibility("default"))) int32_t b2b_model_info_v1(             \
      b2b_model_info* info) {                                                              \
    info->abi = B2B_MODEL_ABI;                                                             \
    info->n_vars = M::NV;                                                                  \
    info->n_normal = M::NN;                                                                \
    info->n_uniform = M::NU;                                                               \
    info->reset_mask = (int32_t)M::RESET_MASK;                                             \
    info->has_threshold = M::HAS_THRESHOLD ? 1 : 0;                                        \
    return 0;                                                                              \
  }                                                                                        \
  extern "C" __attribute__((visibility("default"))) int32_t b2b_model_launch_v1(           \
      const void* pop, const int64_t* clock, int32_t k, double dt, int32_t* status,        \
      void* stream, int32_t dtype, int32_t phase) {                                        \
    return b2b::model::launch<M>(pop, clock, k, dt, status, stream, dtype, phase);         \
  }
