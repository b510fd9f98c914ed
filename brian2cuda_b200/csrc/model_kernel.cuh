// Kernel template of generated neuron models (b2b_group_model).
//
// The device plugin turns a model that no hand-written kernel integrates into a struct of
// device functions — the integration step of its equations, its threshold condition and its
// reset statements, written out by brian2cuda_b200/codegen.py — and compiles it with this
// header into a shared object.  The kernel around them is the same fused pass as the
// hand-written neuron kernels (neuron.cu): one thread per neuron, refractoriness from
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

template <class M, typename R>
__global__ void __launch_bounds__(kBlock)
model_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k, double dt,
                  int32_t* status) {
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const double inv_dt = 1.0 / dt;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned fl = 0;
  if (q < P.n) {
    const ModelGroupDev g = static_cast<const ModelGroupDev*>(P.params)[0];
    const bool refr = g.ref_steps >= 0;
    R x[M::NV];
#pragma unroll
    for (int v = 0; v < M::NV; ++v) x[v] = static_cast<const R*>(P.var[v])[q];
    R ls = (R)0;
    bool nr = true;
    if (refr) {
      ls = static_cast<const R*>(P.var[B2B_VAR_LASTSPIKE])[q];
      nr = timestep_of(t - (double)ls, dt, inv_dt) >= g.ref_steps;
    }
    const R* nrm = M::NN ? static_cast<const R*>(P.rng_normal) + (int64_t)k * M::NN * P.n + q
                         : nullptr;
    const R* uni = M::NU ? static_cast<const R*>(P.rng) + (int64_t)k * M::NU * P.n + q
                         : nullptr;
    M::template update<R>(x, t, dt, nr, nrm, uni, P.n);
    const bool valid = q - g.offset < g.n;
    if (M::HAS_THRESHOLD && valid && nr && M::template threshold<R>(x)) {
      fl = 1;
      nr = false;
      if (refr) ls = (R)t;
      if (!P.late_reset) M::template reset<R>(x);
    }
#pragma unroll
    for (int v = 0; v < M::NV; ++v) static_cast<R*>(P.var[v])[q] = x[v];
    if (refr) {
      if (fl) static_cast<R*>(P.var[B2B_VAR_LASTSPIKE])[q] = ls;
      static_cast<uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY])[q] = nr ? 1 : 0;
    }
  }
  emit_spikes<1>(P, q, fl, ts, slot, status);
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
    const unsigned grid = (unsigned)((P.n + kBlock - 1) / kBlock);
    if (dtype == B2B_F32)
      model_step_kernel<M, float><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
    else
      model_step_kernel<M, double><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
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
