// Fused per-neuron kernels: state update + refractoriness + threshold + reset + spikespace
// compaction, one launch per population and step.
//
// The reference runs these as separate code objects, each a separate launch over all N
// neurons: `_run_kernel_<group>_stateupdater` (brian2cuda/templates/common_group.cu:108-160),
// an eventspace reset kernel (templates/threshold.cu:50-75), the thresholder that appends
// spikes with one global atomicAdd per spike (threshold.cu:19-45), and the resetter over
// the spiking indices (templates/reset.cu:3-27).  Here one thread owns four consecutive
// neurons and loads each state array with one 128-bit access (two for float64); the CTA
// compacts its spikes with warp shuffles and a shared-memory scan and reserves its output
// range with a single atomicAdd on the step's slot of the spike-history ring.
//
// The reset is applied in the same pass when no synaptic effect of the population writes a
// variable the reset writes; otherwise `late_reset` defers it to a kernel that runs after
// the synaptic delivery, preserving Brian2's schedule (groups, thresholds, synapses,
// resets).
#include "kernels_common.cuh"

namespace b2b {

namespace {

// Brian2's `timestep(t, dt)` (brian2cuda/cuda_generator.py:997-1006).
__device__ __forceinline__ int64_t timestep_of(double t, double dt) {
  return (int64_t)((t + 1e-3 * dt) / dt);
}

template <typename R>
struct Quad {
  R x[4];
};

template <typename R>
__device__ __forceinline__ Quad<R> load4(const void* base, int64_t q) {
  Quad<R> r;
  if constexpr (sizeof(R) == 4) {
    float4 a = reinterpret_cast<const float4*>(base)[q];
    r.x[0] = a.x; r.x[1] = a.y; r.x[2] = a.z; r.x[3] = a.w;
  } else {
    const double2* p = reinterpret_cast<const double2*>(base) + 2 * q;
    double2 a = p[0], b = p[1];
    r.x[0] = a.x; r.x[1] = a.y; r.x[2] = b.x; r.x[3] = b.y;
  }
  return r;
}

template <typename R>
__device__ __forceinline__ void store4(void* base, int64_t q, const Quad<R>& r) {
  if constexpr (sizeof(R) == 4) {
    reinterpret_cast<float4*>(base)[q] = make_float4(r.x[0], r.x[1], r.x[2], r.x[3]);
  } else {
    double2* p = reinterpret_cast<double2*>(base) + 2 * q;
    p[0] = make_double2(r.x[0], r.x[1]);
    p[1] = make_double2(r.x[2], r.x[3]);
  }
}

// Writes the spikes flagged in `fl` (bit e = neuron 4q+e) into the ring slot and the spike
// monitor.  Every thread of the CTA must call this (it synchronises the block).
__device__ __forceinline__ void emit_spikes(const PopDev& P, int64_t q, unsigned fl,
                                            int64_t ts, int slot, int32_t* status) {
  __shared__ int s_warp[33];
  __shared__ int s_base;
  __shared__ unsigned long long s_mbase;
  int total;
  const int c = __popc(fl);
  const int excl = block_exclusive_scan(c, s_warp, &total);
  if (threadIdx.x == 0 && total > 0) {
    s_base = atomicAdd(&P.ring_cnt[slot], total);
    if (P.mon_cnt) s_mbase = atomicAdd(P.mon_cnt, (unsigned long long)total);
  }
  __syncthreads();
  if (total == 0 || c == 0) return;
  int32_t* out = P.ring_idx + (int64_t)slot * P.n;
  int pos = s_base + excl;
  unsigned long long mpos = P.mon_cnt ? s_mbase + excl : 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    if (fl & (1u << e)) {
      const int32_t idx = (int32_t)(4 * q + e);
      out[pos++] = idx;
      if (P.mon_cnt) {
        if (mpos < (unsigned long long)P.mon_cap) {
          P.mon_idx[mpos] = idx;
          P.mon_step[mpos] = ts;
        } else {
          set_status(status, B2B_ERR_QUEUE_OVERFLOW);
        }
        ++mpos;
      }
    }
  }
}

__device__ __forceinline__ void clear_next_slot(const PopDev& P, int64_t ts) {
  if (blockIdx.x == 0 && threadIdx.x == 0) P.ring_cnt[ring_slot(ts + 1, P.ring_len)] = 0;
}

// ---- LIF, exact integration ------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kBlock)
lif_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k, double dt,
                int32_t* status) {
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t nvec = P.n >> 2;
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned fl = 0;
  if (q < nvec) {
    const LifDev* prm = static_cast<const LifDev*>(P.params);
    const LifDev g = prm[P.vec_group ? P.vec_group[q] : 0];
    const R A = (R)g.A, Be = (R)g.Be, Bi = (R)g.Bi, De = (R)g.De, Di = (R)g.Di;
    const R El = (R)g.El, Vt = (R)g.Vt, Vr = (R)g.Vr;
    const bool refr = g.ref_steps >= 0;
    Quad<R> V = load4<R>(P.var[B2B_VAR_V], q);
    Quad<R> GE = load4<R>(P.var[B2B_VAR_GE], q);
    Quad<R> GI = load4<R>(P.var[B2B_VAR_GI], q);
    Quad<R> LS;
    if (refr) LS = load4<R>(P.var[B2B_VAR_LASTSPIKE], q);
    uint32_t NRout = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const R v = V.x[e], ge = GE.x[e], gi = GI.x[e];
      bool nr = true;
      if (refr) nr = timestep_of(t - (double)LS.x[e], dt) >= g.ref_steps;
      R vn = dfma(Bi, gi, dfma(Be, ge, dfma(A, v - El, El)));
      if (g.unless_refractory && !nr) vn = v;
      GE.x[e] = De * ge;
      GI.x[e] = Di * gi;
      const bool valid = (4 * q + e - g.offset) < g.n;
      if (g.has_threshold && valid && vn > Vt && nr) {
        nr = false;
        if (refr) LS.x[e] = (R)t;
        if (g.has_reset && !P.late_reset) vn = Vr;
        fl |= 1u << e;
      }
      V.x[e] = vn;
      NRout |= (nr ? 1u : 0u) << (8 * e);
    }
    store4<R>(P.var[B2B_VAR_V], q, V);
    store4<R>(P.var[B2B_VAR_GE], q, GE);
    store4<R>(P.var[B2B_VAR_GI], q, GI);
    if (refr) {
      store4<R>(P.var[B2B_VAR_LASTSPIKE], q, LS);
      reinterpret_cast<uint32_t*>(P.var[B2B_VAR_NOT_REFRACTORY])[q] = NRout;
    }
  }
  emit_spikes(P, q, fl, ts, slot, status);
  clear_next_slot(P, ts);
}

// ---- Hodgkin-Huxley (COBAHH), exponential Euler ----------------------------------------
// Rate functions of examples/cobahh.py:169-180 in SI units; every right-hand side is
// evaluated with the values at the start of the step, and each variable x with
// dx/dt = A x + B advances as x' = -B/A + (x + B/A) exp(A dt).
template <typename R>
__device__ __forceinline__ R expeuler(R x, R A, R B, R dt) {
  const R BA = B / A;
  return -BA + (BA + x) * dexp(A * dt);
}

template <typename R>
__global__ void __launch_bounds__(kBlock)
hh_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k, double dt,
               int32_t* status) {
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t nvec = P.n >> 2;
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned fl = 0;
  if (q < nvec) {
    const HhDev* prm = static_cast<const HhDev*>(P.params);
    const HhDev g = prm[P.vec_group ? P.vec_group[q] : 0];
    const R Cm = (R)g.Cm, gl = (R)g.gl, El = (R)g.El, EK = (R)g.EK, ENa = (R)g.ENa;
    const R gNa = (R)g.gNa, gK = (R)g.gK, VT = (R)g.VT, Ee = (R)g.Ee, Ei = (R)g.Ei;
    const R De = (R)g.De, Di = (R)g.Di, Vthr = (R)g.Vthr, dtR = (R)dt;
    const bool refr = g.ref_steps >= 0;
    Quad<R> V = load4<R>(P.var[B2B_VAR_V], q);
    Quad<R> M = load4<R>(P.var[B2B_VAR_M], q);
    Quad<R> H = load4<R>(P.var[B2B_VAR_H], q);
    Quad<R> N = load4<R>(P.var[B2B_VAR_N], q);
    Quad<R> GE = load4<R>(P.var[B2B_VAR_GE], q);
    Quad<R> GI = load4<R>(P.var[B2B_VAR_GI], q);
    Quad<R> LS;
    if (refr) LS = load4<R>(P.var[B2B_VAR_LASTSPIKE], q);
    uint32_t NRout = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const R v = V.x[e], m = M.x[e], h = H.x[e], n = N.x[e], ge = GE.x[e], gi = GI.x[e];
      bool nr = true;
      if (refr) nr = timestep_of(t - (double)LS.x[e], dt) >= g.ref_steps;
      const R xm = (R)13e-3 - v + VT;
      const R am = (R)0.32e6 * xm / (dexp(xm / (R)4e-3) - (R)1);
      const R ym = v - VT - (R)40e-3;
      const R bm = (R)0.28e6 * ym / (dexp(ym / (R)5e-3) - (R)1);
      const R ah = (R)128 * dexp(((R)17e-3 - v + VT) / (R)18e-3);
      const R bh = (R)4000 / ((R)1 + dexp(((R)40e-3 - v + VT) / (R)5e-3));
      const R xn = (R)15e-3 - v + VT;
      const R an = (R)0.032e6 * xn / (dexp(xn / (R)5e-3) - (R)1);
      const R bn = (R)500 * dexp(((R)10e-3 - v + VT) / (R)40e-3);
      const R gna = gNa * (m * m * m) * h;
      const R gk = gK * (n * n * n * n);
      const R Av = -(gl + ge + gi + gna + gk) / Cm;
      const R Bv = (gl * El + ge * Ee + gi * Ei + gna * ENa + gk * EK) / Cm;
      const R vn = expeuler(v, Av, Bv, dtR);
      M.x[e] = expeuler(m, -(am + bm), am, dtR);
      H.x[e] = expeuler(h, -(ah + bh), ah, dtR);
      N.x[e] = expeuler(n, -(an + bn), an, dtR);
      GE.x[e] = De * ge;
      GI.x[e] = Di * gi;
      const bool valid = (4 * q + e - g.offset) < g.n;
      if (valid && vn > Vthr && nr) {
        nr = false;
        if (refr) LS.x[e] = (R)t;
        fl |= 1u << e;
      }
      V.x[e] = vn;
      NRout |= (nr ? 1u : 0u) << (8 * e);
    }
    store4<R>(P.var[B2B_VAR_V], q, V);
    store4<R>(P.var[B2B_VAR_M], q, M);
    store4<R>(P.var[B2B_VAR_H], q, H);
    store4<R>(P.var[B2B_VAR_N], q, N);
    store4<R>(P.var[B2B_VAR_GE], q, GE);
    store4<R>(P.var[B2B_VAR_GI], q, GI);
    if (refr) {
      store4<R>(P.var[B2B_VAR_LASTSPIKE], q, LS);
      reinterpret_cast<uint32_t*>(P.var[B2B_VAR_NOT_REFRACTORY])[q] = NRout;
    }
  }
  emit_spikes(P, q, fl, ts, slot, status);
  clear_next_slot(P, ts);
}

// ---- PoissonGroup: spike when u < rate*dt, u read in place from the bulk buffer ---------
template <typename R>
__global__ void __launch_bounds__(kBlock)
poisson_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k, int32_t* status) {
  const int64_t ts = clock[0] + k;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t nvec = P.n >> 2;
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned fl = 0;
  if (q < nvec) {
    const PoissonDev* prm = static_cast<const PoissonDev*>(P.params);
    const PoissonDev g = prm[P.vec_group ? P.vec_group[q] : 0];
    const R thr = (R)g.p_spike;
    const R* row = static_cast<const R*>(P.rng) + (int64_t)k * P.n;
    Quad<R> U = load4<R>(row, q);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const bool valid = (4 * q + e - g.offset) < g.n;
      if (valid && U.x[e] < thr) fl |= 1u << e;
    }
  }
  emit_spikes(P, q, fl, ts, slot, status);
  clear_next_slot(P, ts);
}

// ---- SpikeGeneratorGroup: entries sorted by step, one CTA ---------------------------------
__device__ __forceinline__ int64_t lower_bound_i64(const int64_t* a, int64_t n, int64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void spikegen_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k,
                                     int32_t* status) {
  const int64_t ts = clock[0] + k;
  const int slot = ring_slot(ts, P.ring_len);
  __shared__ int64_t s_lo, s_hi;
  __shared__ unsigned long long s_mbase;
  if (threadIdx.x == 0) {
    s_lo = lower_bound_i64(P.sg_step, P.sg_n, ts);
    s_hi = lower_bound_i64(P.sg_step, P.sg_n, ts + 1);
    const int cnt = (int)(s_hi - s_lo);
    P.ring_cnt[slot] = cnt;
    P.ring_cnt[ring_slot(ts + 1, P.ring_len)] = 0;
    if (P.mon_cnt) s_mbase = atomicAdd(P.mon_cnt, (unsigned long long)cnt);
  }
  __syncthreads();
  const int64_t cnt = s_hi - s_lo;
  int32_t* out = P.ring_idx + (int64_t)slot * P.n;
  for (int64_t r = threadIdx.x; r < cnt; r += blockDim.x) {
    const int32_t idx = P.sg_idx[s_lo + r];
    out[r] = idx;
    if (P.mon_cnt) {
      const unsigned long long mp = s_mbase + (unsigned long long)r;
      if (mp < (unsigned long long)P.mon_cap) {
        P.mon_idx[mp] = idx;
        P.mon_step[mp] = ts;
      } else {
        set_status(status, B2B_ERR_QUEUE_OVERFLOW);
      }
    }
  }
}

// ---- reset after synaptic delivery (Brian2's 'resets' slot) -------------------------------
template <typename R>
__global__ void lif_late_reset_kernel(PopDev P, const int64_t* __restrict__ clock, int k) {
  const int64_t ts = clock[0] + k;
  const int slot = ring_slot(ts, P.ring_len);
  const int cnt = P.ring_cnt[slot];
  const int32_t* idx = P.ring_idx + (int64_t)slot * P.n;
  const LifDev* prm = static_cast<const LifDev*>(P.params);
  R* V = static_cast<R*>(P.var[B2B_VAR_V]);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < cnt; r += gridDim.x * blockDim.x) {
    const int32_t i = idx[r];
    const LifDev& g = prm[P.vec_group ? P.vec_group[i >> 2] : 0];
    if (g.has_reset) V[i] = (R)g.Vr;
  }
}

}  // namespace

cudaError_t launch_pop_step(const Pop& pop, const int64_t* clock, int k, double dt,
                            int32_t* status, cudaStream_t s) {
  const PopDev& P = pop.dev;
  const int64_t nvec = P.n >> 2;
  const unsigned grid = (unsigned)((nvec + kBlock - 1) / kBlock);
  switch (pop.kind) {
    case KIND_LIF:
      if (pop.dtype == B2B_F32) lif_step_kernel<float><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
      else lif_step_kernel<double><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
      break;
    case KIND_HH:
      if (pop.dtype == B2B_F32) hh_step_kernel<float><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
      else hh_step_kernel<double><<<grid, kBlock, 0, s>>>(P, clock, k, dt, status);
      break;
    case KIND_POISSON:
      if (pop.dtype == B2B_F32) poisson_step_kernel<float><<<grid, kBlock, 0, s>>>(P, clock, k, status);
      else poisson_step_kernel<double><<<grid, kBlock, 0, s>>>(P, clock, k, status);
      break;
    case KIND_SPIKEGEN:
      spikegen_step_kernel<<<1, kBlock, 0, s>>>(P, clock, k, status);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_pop_late_reset(const Pop& pop, const int64_t* clock, int k, cudaStream_t s) {
  if (pop.kind != KIND_LIF) return cudaSuccess;
  const unsigned grid = 2 * kNumSMs;
  if (pop.dtype == B2B_F32) lif_late_reset_kernel<float><<<grid, kBlock, 0, s>>>(pop.dev, clock, k);
  else lif_late_reset_kernel<double><<<grid, kBlock, 0, s>>>(pop.dev, clock, k);
  return cudaGetLastError();
}

namespace {
__global__ void tick_kernel(int64_t* clock, int steps) { clock[0] += steps; }
}  // namespace

cudaError_t launch_tick(int64_t* clock, int steps, cudaStream_t s) {
  tick_kernel<<<1, 1, 0, s>>>(clock, steps);
  return cudaGetLastError();
}

}  // namespace b2b
