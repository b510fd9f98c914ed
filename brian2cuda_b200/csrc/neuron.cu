// Fused per-neuron kernels: state update + refractoriness + threshold + reset + spikespace
// compaction, one launch per population and step.
//
// The reference runs these as separate code objects, each a separate launch over all N
// neurons: `_run_kernel_<group>_stateupdater` (brian2cuda/templates/common_group.cu:108-160),
// an eventspace reset kernel (templates/threshold.cu:50-75), the thresholder that appends
// spikes with one global atomicAdd per spike (threshold.cu:19-45), and the resetter over
// the spiking indices (templates/reset.cu:3-27).  Here a thread owns E consecutive neurons:
// E = 4 for large populations (each state array read with one 128-bit access, two for
// float64), E = 1 when the population is too small to fill the GPU that way.  The CTA
// compacts its spikes with warp shuffles and a shared-memory scan and reserves its output
// range with a single atomicAdd on the step's slot of the spike-history ring (the streaming
// kernel, which compacts once per pack iteration, does this per warp instead).
//
// The reset is applied in the same pass when no synaptic effect of the population writes a
// variable the reset writes; otherwise `late_reset` defers it to a kernel that runs after
// the synaptic delivery, preserving Brian2's schedule (groups, thresholds, synapses,
// resets).
#include <algorithm>

#include "neuron_common.cuh"
#include "pending_body.cuh"

namespace b2b {

namespace {
// Adds the input delivered during the previous step (fold buffer of variable v, parity
// (ts-1) & 1) into pack X and returns the pack's address in the buffer, to be cleared after
// the update's stores; no-op when the population has no fold buffer for v.
template <typename R, int E>
__device__ __forceinline__ R* fold_in(const PopDev& P, int v, int64_t ts, int64_t q,
                                      Pack<R, E>& X) {
  if (!P.fold[v]) return nullptr;
  R* a = static_cast<R*>(P.fold[v]) + (int64_t)((ts & 1) ^ 1) * P.n;
  const Pack<R, E> A = load_pack<R, E>(a, q);
#pragma unroll
  for (int e = 0; e < E; ++e) X.x[e] += A.x[e];
  return a;
}

template <typename R, int E>
__device__ __forceinline__ void fold_clear(R* a, int64_t q) {
  if (!a) return;
  Pack<R, E> z;
#pragma unroll
  for (int e = 0; e < E; ++e) z.x[e] = (R)0;
  store_pack<R, E>(a, q, z);
}

// ---- LIF, exact integration ------------------------------------------------------------
// INPUTS: the population has TimedArray or PoissonInput inputs (compiled out otherwise).
// The work of CTA `blk` of the update (blockDim.x threads, E neurons each).
template <typename R, int E, bool INPUTS>
__device__ __forceinline__ void lif_step_body(const PopDev& P, const int64_t* __restrict__ clock,
                                              int k, double dt, int32_t* status, int64_t blk) {
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const double inv_dt = 1.0 / dt;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t nthr = P.n / E;
  const int64_t q = blk * blockDim.x + threadIdx.x;
  unsigned fl = 0;
  if (q < nthr) {
    const LifDev* prm = static_cast<const LifDev*>(P.params);
    const int grp = group_of<E>(P, q);
    const LifDev g = prm[grp];
    const GroupInputs* gin = INPUTS ? P.inputs + grp : nullptr;
    const bool after_reset = INPUTS && gin->pin.after_reset;
    const R Vt = (R)g.Vt, Vr = (R)g.Vr;
    const bool refr = g.ref_steps >= 0;
    Pack<R, E> V = load_pack<R, E>(P.var[B2B_VAR_V], q);
    Pack<R, E> GE = load_pack<R, E>(P.var[B2B_VAR_GE], q);
    Pack<R, E> GI = load_pack<R, E>(P.var[B2B_VAR_GI], q);
    Pack<R, E> LS;
    if (refr) LS = load_pack<R, E>(P.var[B2B_VAR_LASTSPIKE], q);
    R* fge = fold_in<R, E>(P, B2B_VAR_GE, ts, q, GE);
    R* fgi = fold_in<R, E>(P, B2B_VAR_GI, ts, q, GI);
    uint32_t NRout = 0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      R ge = GE.x[e], gi = GI.x[e];
      bool nr = true;
      if (refr) nr = past_refractory(t - (double)LS.x[e], dt, inv_dt, g.ref_steps);
      R vn = lif_advance<R>(g, V.x[e], ge, gi, nr,
                            INPUTS ? timed_input<R>(gin->ta, ts, E * q + e - g.offset) : R(0));
      GE.x[e] = ge;
      GI.x[e] = gi;
      const int64_t local = E * q + e - g.offset;
      const bool valid = local < g.n;
      bool reset_now = false;
      if (g.has_threshold && valid && vn > Vt && nr) {
        nr = false;
        if (refr) LS.x[e] = (R)t;
        reset_now = g.has_reset && !P.late_reset;
        fl |= 1u << e;
      }
      // PoissonInputs act in the synapses slot: after the threshold, and before the reset
      // unless the schedule resets first
      if (reset_now && after_reset) vn = Vr;
      if (INPUTS && gin->pin.count && valid)
        add_poisson_inputs<R>(gin->pin, ts, local, vn, GE.x[e], GI.x[e]);
      if (reset_now && !after_reset) vn = Vr;
      V.x[e] = vn;
      NRout |= (nr ? 1u : 0u) << (8 * e);
    }
    store_pack<R, E>(P.var[B2B_VAR_V], q, V);
    store_pack<R, E>(P.var[B2B_VAR_GE], q, GE);
    store_pack<R, E>(P.var[B2B_VAR_GI], q, GI);
    if (refr) {
      if (fl) store_pack<R, E>(P.var[B2B_VAR_LASTSPIKE], q, LS);   // changes only on a spike
      store_flags<E>(P.var[B2B_VAR_NOT_REFRACTORY], q, NRout);
    }
    fold_clear<R, E>(fge, q);
    fold_clear<R, E>(fgi, q);
  }
  emit_spikes<E>(P, q, fl, ts, slot, status);
  clear_next_slot(P, ts, blk);
}

template <typename R, int E, bool INPUTS>
__global__ void __launch_bounds__(kBlock)
lif_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k, double dt,
                int32_t* status) {
  lif_step_body<R, E, INPUTS>(P, clock, k, dt, status, blockIdx.x);
}

// ---- Hodgkin-Huxley (COBAHH), exponential Euler (hh_advance) ------------------------
template <typename R, int E, bool INPUTS>
__device__ __forceinline__ void hh_step_body(const PopDev& P, const int64_t* __restrict__ clock,
                                             int k, double dt, int32_t* status, int64_t blk) {
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const double inv_dt = 1.0 / dt;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t nthr = P.n / E;
  const int64_t q = blk * blockDim.x + threadIdx.x;
  unsigned fl = 0;
  if (q < nthr) {
    const HhDev* prm = static_cast<const HhDev*>(P.params);
    const int grp = group_of<E>(P, q);
    const HhRun<R> g = hh_run(prm[grp], R());
    const GroupInputs* gin = INPUTS ? P.inputs + grp : nullptr;
    const R Vthr = (R)g.Vthr, dtR = (R)dt;
    const bool refr = g.ref_steps >= 0;
    Pack<R, E> V = load_pack<R, E>(P.var[B2B_VAR_V], q);
    Pack<R, E> M = load_pack<R, E>(P.var[B2B_VAR_M], q);
    Pack<R, E> H = load_pack<R, E>(P.var[B2B_VAR_H], q);
    Pack<R, E> N = load_pack<R, E>(P.var[B2B_VAR_N], q);
    Pack<R, E> GE = load_pack<R, E>(P.var[B2B_VAR_GE], q);
    Pack<R, E> GI = load_pack<R, E>(P.var[B2B_VAR_GI], q);
    Pack<R, E> LS;
    if (refr) LS = load_pack<R, E>(P.var[B2B_VAR_LASTSPIKE], q);
    R* fge = fold_in<R, E>(P, B2B_VAR_GE, ts, q, GE);
    R* fgi = fold_in<R, E>(P, B2B_VAR_GI, ts, q, GI);
    uint32_t NRout = 0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      bool nr = true;
      if (refr) nr = past_refractory(t - (double)LS.x[e], dt, inv_dt, g.ref_steps);
      const int64_t local = E * q + e - g.offset;
      R vn = hh_advance<R>(g, V.x[e], M.x[e], H.x[e], N.x[e], GE.x[e], GI.x[e], dtR,
                           INPUTS ? timed_input<R>(gin->ta, ts, local) : R(0));
      const bool valid = local < g.n;
      if (valid && vn > Vthr && nr) {
        nr = false;
        if (refr) LS.x[e] = (R)t;
        fl |= 1u << e;
      }
      if (INPUTS && gin->pin.count && valid)
        add_poisson_inputs<R>(gin->pin, ts, local, vn, GE.x[e], GI.x[e]);
      V.x[e] = vn;
      NRout |= (nr ? 1u : 0u) << (8 * e);
    }
    store_pack<R, E>(P.var[B2B_VAR_V], q, V);
    store_pack<R, E>(P.var[B2B_VAR_M], q, M);
    store_pack<R, E>(P.var[B2B_VAR_H], q, H);
    store_pack<R, E>(P.var[B2B_VAR_N], q, N);
    store_pack<R, E>(P.var[B2B_VAR_GE], q, GE);
    store_pack<R, E>(P.var[B2B_VAR_GI], q, GI);
    if (refr) {
      if (fl) store_pack<R, E>(P.var[B2B_VAR_LASTSPIKE], q, LS);   // changes only on a spike
      store_flags<E>(P.var[B2B_VAR_NOT_REFRACTORY], q, NRout);
    }
    fold_clear<R, E>(fge, q);
    fold_clear<R, E>(fgi, q);
  }
  emit_spikes<E>(P, q, fl, ts, slot, status);
  clear_next_slot(P, ts, blk);
}

template <typename R, int E, bool INPUTS>
__global__ void __launch_bounds__(kBlock)
hh_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k, double dt,
               int32_t* status) {
  hh_step_body<R, E, INPUTS>(P, clock, k, dt, status, blockIdx.x);
}

// ---- one launch per step (nets of the two-launch form, pending.cu) --------------------
// The update of step t and the delivery of step t into the pending input are independent
// (pending.cu); here they are one grid: CTAs [0, n_upd) do the per-step update (one neuron
// per thread, folding in the input pending from step t-1), the CTAs after them deliver the
// bundles due at step t into acc[t & 1].  Consecutive steps are consecutive launches on one
// stream, so one launch boundary orders step t+1 after both halves of step t, where the two
// concurrent launches need a boundary each and dependencies across two streams.
template <typename R, int KIND, int E, int GROUP>
__global__ void __launch_bounds__(kBlock, E == 1 ? (sizeof(R) == 4 ? 5 : 4) : 3)
one_launch_step_kernel(const __grid_constant__ PopDev U, const __grid_constant__ PendingDev F,
                       const int64_t* __restrict__ clock, int k, double dt, int32_t* status,
                       int n_upd) {
  // chained launches (programmatic dependent launch): wait for the previous step's grid to
  // complete and its memory to be visible, then let the next step's grid be scheduled, so its
  // CTAs are resident by the time this one ends; without that launch attribute both are no-ops
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;");
  if ((int)blockIdx.x < n_upd) {
    if constexpr (KIND == KIND_HH)
      hh_step_body<R, E, false>(U, clock, k, dt, status, blockIdx.x);
    else
      lif_step_body<R, E, false>(U, clock, k, dt, status, blockIdx.x);
  } else {
    deliver_pending_body<R, true, GROUP>(F, clock, k, (int64_t)blockIdx.x - n_upd,
                                         (int64_t)gridDim.x - n_upd, nullptr);
  }
}

template <typename R, int KIND, int E, int GROUP>
cudaError_t launch_one_g(const PopDev& U, const PendingDev& F, unsigned grid, int block,
                         bool chained, const int64_t* clock, int k, double dt, int32_t* status,
                         int n_upd, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = chained ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, one_launch_step_kernel<R, KIND, E, GROUP>, U, F, clock, k,
                            dt, status, n_upd);
}

template <typename R, int KIND, int E>
cudaError_t launch_one_r(const PopDev& U, const PendingDev& F, unsigned grid, int block,
                         bool chained, const int64_t* clock, int k, double dt, int32_t* status,
                         int n_upd, cudaStream_t s) {
  if (F.group == 16)
    return launch_one_g<R, KIND, E, 16>(U, F, grid, block, chained, clock, k, dt, status, n_upd, s);
  if (F.group == 4)
    return launch_one_g<R, KIND, E, 4>(U, F, grid, block, chained, clock, k, dt, status, n_upd, s);
  if (F.group == 2)
    return launch_one_g<R, KIND, E, 2>(U, F, grid, block, chained, clock, k, dt, status, n_upd, s);
  return launch_one_g<R, KIND, E, 8>(U, F, grid, block, chained, clock, k, dt, status, n_upd, s);
}

template <int KIND, int E>
cudaError_t launch_one_k(const PopDev& U, const PendingDev& F, bool f32, unsigned grid,
                         int block, bool chained, const int64_t* clock, int k, double dt,
                         int32_t* status, int n_upd, cudaStream_t s) {
  return f32 ? launch_one_r<float, KIND, E>(U, F, grid, block, chained, clock, k, dt, status,
                                            n_upd, s)
             : launch_one_r<double, KIND, E>(U, F, grid, block, chained, clock, k, dt, status,
                                             n_upd, s);
}

// Large HH populations: a persistent grid (resident CTAs only) walks the population in
// strides, and every thread loads the state of its next four neurons before it updates the
// current four, so the loads of one pack overlap the arithmetic of the previous one.  The
// per-neuron arithmetic is hh_step_kernel's.
template <typename R>
struct HhPack {
  Pack<R, 4> V, M, H, N, GE, GI, LS;
  int grp;
};

// lastspike is loaded whatever the group's refractoriness (every HH population holds it):
// deciding on the group's flag first would make the prefetch wait for the group id and the
// group's constants, two dependent loads, when a population holds many groups.
template <typename R>
__device__ __forceinline__ void hh_pack_load(const PopDev& P, int64_t q, HhPack<R>& s) {
  s.grp = group_of<4>(P, q);
  s.V = load_pack<R, 4>(P.var[B2B_VAR_V], q);
  s.M = load_pack<R, 4>(P.var[B2B_VAR_M], q);
  s.H = load_pack<R, 4>(P.var[B2B_VAR_H], q);
  s.N = load_pack<R, 4>(P.var[B2B_VAR_N], q);
  s.GE = load_pack<R, 4>(P.var[B2B_VAR_GE], q);
  s.GI = load_pack<R, 4>(P.var[B2B_VAR_GI], q);
  s.LS = load_pack<R, 4>(P.var[B2B_VAR_LASTSPIKE], q);
}

template <typename R, bool INPUTS>
__global__ void __launch_bounds__(kBlock, 2)
hh_stream_kernel(PopDev P, const int64_t* __restrict__ clock, int k, double dt,
                 int32_t* status) {
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const double inv_dt = 1.0 / dt;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t nthr = P.n / 4;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t iters = (nthr + stride - 1) / stride;   // the same for every thread
  const HhDev* prm = static_cast<const HhDev*>(P.params);
  const R dtR = (R)dt;
  int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  HhPack<R> cur;
  if (q < nthr) hh_pack_load<R>(P, q, cur);
  for (int64_t it = 0; it < iters; ++it, q += stride) {
    HhPack<R> nxt;
    if (q + stride < nthr) hh_pack_load<R>(P, q + stride, nxt);
    unsigned fl = 0;
    if (q < nthr) {
      const HhRun<R> g = hh_run(prm[cur.grp], R());
      const GroupInputs* gin = INPUTS ? P.inputs + cur.grp : nullptr;
      const bool refr = g.ref_steps >= 0;
      R* fge = fold_in<R, 4>(P, B2B_VAR_GE, ts, q, cur.GE);
      R* fgi = fold_in<R, 4>(P, B2B_VAR_GI, ts, q, cur.GI);
      uint32_t NRout = 0;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        bool nr = true;
        if (refr) nr = past_refractory(t - (double)cur.LS.x[e], dt, inv_dt, g.ref_steps);
        const int64_t local = 4 * q + e - g.offset;
        R vn = hh_advance<R>(g, cur.V.x[e], cur.M.x[e], cur.H.x[e], cur.N.x[e],
                             cur.GE.x[e], cur.GI.x[e], dtR,
                             INPUTS ? timed_input<R>(gin->ta, ts, local) : R(0));
        const bool valid = local < g.n;
        if (valid && vn > (R)g.Vthr && nr) {
          nr = false;
          if (refr) cur.LS.x[e] = (R)t;
          fl |= 1u << e;
        }
        if (INPUTS && gin->pin.count && valid)
          add_poisson_inputs<R>(gin->pin, ts, local, vn, cur.GE.x[e], cur.GI.x[e]);
        cur.V.x[e] = vn;
        NRout |= (nr ? 1u : 0u) << (8 * e);
      }
      store_pack<R, 4>(P.var[B2B_VAR_V], q, cur.V);
      store_pack<R, 4>(P.var[B2B_VAR_M], q, cur.M);
      store_pack<R, 4>(P.var[B2B_VAR_H], q, cur.H);
      store_pack<R, 4>(P.var[B2B_VAR_N], q, cur.N);
      store_pack<R, 4>(P.var[B2B_VAR_GE], q, cur.GE);
      store_pack<R, 4>(P.var[B2B_VAR_GI], q, cur.GI);
      if (refr) {
        if (fl) store_pack<R, 4>(P.var[B2B_VAR_LASTSPIKE], q, cur.LS);   // changes on a spike
        store_flags<4>(P.var[B2B_VAR_NOT_REFRACTORY], q, NRout);
      }
      fold_clear<R, 4>(fge, q);
      fold_clear<R, 4>(fgi, q);
    }
    emit_spikes_warp<4>(P, q, fl, ts, slot, status);
    cur = nxt;
  }
  clear_next_slot(P, ts);
}

// ---- PoissonGroup: spike when u < rate*dt, u read in place from the bulk buffer ---------
template <typename R, int E, bool INPUTS>
__global__ void __launch_bounds__(kBlock)
poisson_step_kernel(PopDev P, const int64_t* __restrict__ clock, int k, double dt,
                    int32_t* status) {
  const int64_t ts = clock[0] + k;
  const int slot = ring_slot(ts, P.ring_len);
  const int64_t nthr = P.n / E;
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned fl = 0;
  if (q < nthr) {
    const PoissonDev* prm = static_cast<const PoissonDev*>(P.params);
    const int grp = group_of<E>(P, q);
    const PoissonDev g = prm[grp];
    const GroupInputs* gin = INPUTS ? P.inputs + grp : nullptr;
    const R thr = (R)g.p_spike;
    const R* row = static_cast<const R*>(P.rng) + (int64_t)k * P.n;
    Pack<R, E> U = load_pack<R, E>(row, q);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int64_t local = E * q + e - g.offset;
      const bool valid = local < g.n;
      // a TimedArray gives the rate in Hz (PoissonGroup(rates='ta(t)')): u < rate dt
      const R th = INPUTS && gin->ta.val
                       ? (R)((double)timed_input<R>(gin->ta, ts, local) * dt) : thr;
      if (valid && U.x[e] < th) fl |= 1u << e;
    }
  }
  emit_spikes<E>(P, q, fl, ts, slot, status);
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
    // with a period, step ts emits the entries of bin ts mod period
    // (brian2cuda/templates/spikegenerator.cu:42-49)
    const int64_t bin = P.sg_period > 0 ? ts % P.sg_period : ts;
    s_lo = lower_bound_i64(P.sg_step, P.sg_n, bin);
    s_hi = lower_bound_i64(P.sg_step, P.sg_n, bin + 1);
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

// Four neurons per thread once that still gives every SM several CTAs' worth of warps.
bool wide(int64_t n) { return n / 4 >= (int64_t)kNumSMs * 4 * kBlock; }

template <int E, bool IN>
cudaError_t launch_e(const Pop& pop, const PopDev& P, const int64_t* clock, int k, double dt,
                     int32_t* status, cudaStream_t s) {
  const int block = pop.tune_block > 0 ? pop.tune_block : kBlock;   // <= kBlock
  const unsigned grid = (unsigned)((P.n / E + block - 1) / block);
  const bool f32 = pop.dtype == B2B_F32;
  switch (pop.kind) {
    case KIND_LIF:
      if (f32) lif_step_kernel<float, E, IN><<<grid, block, 0, s>>>(P, clock, k, dt, status);
      else lif_step_kernel<double, E, IN><<<grid, block, 0, s>>>(P, clock, k, dt, status);
      break;
    case KIND_HH:
      if (E == 4 && f32) {
        // resident CTAs only (2 per SM of 256 threads by the launch bounds); float64 keeps
        // one pack per thread (two packs of doubles do not fit the register budget)
        const unsigned g2 = std::min<unsigned>(grid, 2 * kNumSMs * (kBlock / block));
        hh_stream_kernel<float, IN><<<g2, block, 0, s>>>(P, clock, k, dt, status);
      } else if (f32) {
        hh_step_kernel<float, E, IN><<<grid, block, 0, s>>>(P, clock, k, dt, status);
      } else {
        hh_step_kernel<double, E, IN><<<grid, block, 0, s>>>(P, clock, k, dt, status);
      }
      break;
    case KIND_POISSON:
      if (f32) poisson_step_kernel<float, E, IN><<<grid, block, 0, s>>>(P, clock, k, dt, status);
      else poisson_step_kernel<double, E, IN><<<grid, block, 0, s>>>(P, clock, k, dt, status);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pop_step(const Pop& pop, const int64_t* clock, int k, double dt,
                            int32_t* status, cudaStream_t s) {
  return launch_pop_step_dev(pop, pop.dev, clock, k, dt, status, s);
}

cudaError_t launch_pop_step_dev(const Pop& pop, const PopDev& dev, const int64_t* clock, int k,
                                double dt, int32_t* status, cudaStream_t s) {
  if (pop.kind == KIND_HH && pop.surr_img) return launch_hh_surrogate(pop, clock, k, dt, status, s);
  if (pop.kind == KIND_MODEL)   // the generated model's own kernel, from its shared object
    return (cudaError_t)pop.model_launch(&dev, clock, k, dt, status, s, pop.dtype, 0);
  if (pop.kind == KIND_SPIKEGEN) {
    spikegen_step_kernel<<<1, kBlock, 0, s>>>(pop.dev, clock, k, status);
    return cudaGetLastError();
  }
  // neurons per thread: the autotuner's choice (1, 2 or 4), else 4 for wide populations
  const int e = pop.tune_e > 0 ? pop.tune_e : (wide(pop.dev.n) ? 4 : 1);
  if (pop.inputs) {
    if (e == 4) return launch_e<4, true>(pop, dev, clock, k, dt, status, s);
    if (e == 2) return launch_e<2, true>(pop, dev, clock, k, dt, status, s);
    return launch_e<1, true>(pop, dev, clock, k, dt, status, s);
  }
  if (e == 4) return launch_e<4, false>(pop, dev, clock, k, dt, status, s);
  if (e == 2) return launch_e<2, false>(pop, dev, clock, k, dt, status, s);
  return launch_e<1, false>(pop, dev, clock, k, dt, status, s);
}

bool one_launch_supported(const Pop& pop, const PendingDev& F) {
  return (pop.kind == KIND_LIF || pop.kind == KIND_HH) && !pop.inputs && !pop.surr_img &&
         F.nd_max <= kWarpPrefixMaxDelays;
}

cudaError_t launch_one_launch_step(const Pop& pop, const PopDev& U, const PendingDev& F,
                                   int deliver_ctas, bool chained, const int64_t* clock, int k,
                                   double dt, int32_t* status, cudaStream_t s) {
  if (!one_launch_supported(pop, F) || deliver_ctas < 1) return cudaErrorInvalidValue;
  // the update half takes the population's tuned shape (neurons per thread 1 or 2, 128 or
  // 256 threads per CTA); the delivery half the same threads per CTA, deliver_ctas counted
  // in CTAs of kBlock threads
  const int e = pop.tune_e == 2 || pop.tune_e == 4 ? 2 : 1;
  const int block = pop.tune_block > 0 ? pop.tune_block : kBlock;
  const int n_upd = (int)((U.n / e + block - 1) / block);
  const unsigned grid = (unsigned)(n_upd + (int64_t)deliver_ctas * kBlock / block);
  const bool f32 = pop.dtype == B2B_F32;
  if (pop.kind == KIND_HH)
    return e == 2 ? launch_one_k<KIND_HH, 2>(U, F, f32, grid, block, chained, clock, k, dt,
                                             status, n_upd, s)
                  : launch_one_k<KIND_HH, 1>(U, F, f32, grid, block, chained, clock, k, dt,
                                             status, n_upd, s);
  return e == 2 ? launch_one_k<KIND_LIF, 2>(U, F, f32, grid, block, chained, clock, k, dt,
                                            status, n_upd, s)
                : launch_one_k<KIND_LIF, 1>(U, F, f32, grid, block, chained, clock, k, dt,
                                            status, n_upd, s);
}

cudaError_t launch_pop_late_reset(const Pop& pop, const int64_t* clock, int k, cudaStream_t s) {
  if (pop.kind == KIND_MODEL)
    return (cudaError_t)pop.model_launch(&pop.dev, clock, k, 0.0, nullptr, s, pop.dtype, 1);
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
