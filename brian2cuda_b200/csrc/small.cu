// Small networks: every step of a chunk inside one CTA, with the neuron state in shared
// memory.
//
// A network of a few thousand neurons (the CUBA example: 4000 LIF neurons, about two spikes
// per step) leaves the per-step path launch-bound: each step is a neuron launch and a delivery
// launch of a few microseconds, nearly all of it launch and synchronisation latency (the
// reference is bound the same way at a larger scale: one launch per code object per step,
// brian2cuda/templates/network.cu:65-115).  When the net is one LIF or HH population of at
// most 4096 neurons whose synapses are all additive and target it, and the caller opts in
// (B2B_NET_SMALL), one CTA of 1024 threads runs a whole chunk of steps: it loads the state into shared memory once, then per step
// updates four neurons per thread, compacts the spikes with a block scan into the same
// spike-history ring and monitor the per-step kernels write, delivers the due bundles
// (every warp of the CTA, 32 synapses per warp and item) with atomic additions into the
// shared-memory targets,
// applies a deferred reset if the schedule needs one, and writes the state back at the end.
// Block barriers separate the phases, so Brian2's order within a step (groups, thresholds,
// synapses, resets) is kept, delays of zero steps included.  Measured on B200 against the
// per-step kernels: CUBA-type LIF nets of 500 / 1000 / 2000 neurons 3.8 / 4.4 / 5.8 us per
// step against 4.9 / 5.5 / 6.6 us; at 4000 neurons, or with many delays (COBAHH with delays
// of 1-50 steps), one SM's issue rate loses to the whole GPU, so the path is opt-in.
#include <cooperative_groups.h>

#include <algorithm>

#include "delivery.cuh"
#include "neuron_common.cuh"

namespace b2b {

namespace {

constexpr int kSmallThreads = 1024;
// the pull form keeps these in shared memory (larger nets use the push form)
constexpr int kPullMaxGroups = 16;
constexpr int kPullMaxMembers = 16;

// Shared-memory image of the population: one array per real-valued variable of the kind,
// then the not_refractory flags, then the delivery prefix of the block path.
struct SmallLayout {
  int nvars;              // real-valued variables held
  int var[kMaxVars];      // their B2B_VAR_* ids
};

__host__ __device__ inline SmallLayout small_layout(int kind) {
  SmallLayout L{};
  const int lif[] = {B2B_VAR_V, B2B_VAR_GE, B2B_VAR_GI, B2B_VAR_LASTSPIKE};
  const int hh[] = {B2B_VAR_V, B2B_VAR_GE, B2B_VAR_GI, B2B_VAR_M, B2B_VAR_H, B2B_VAR_N,
                    B2B_VAR_LASTSPIKE};
  if (kind == KIND_LIF) {
    L.nvars = 4;
    for (int i = 0; i < 4; ++i) L.var[i] = lif[i];
  } else {
    L.nvars = 7;
    for (int i = 0; i < 7; ++i) L.var[i] = hh[i];
  }
  return L;
}

// Delivery of the bundles of projection J due at step ts by every warp of the CTA: a work
// item is 32 synapses of one due bundle (one synapse per lane), items go to the warps in
// turn, so the few bundles of a small network's step are spread over the whole CTA rather
// than walked by one warp while the others wait at the next barrier.
template <typename R, bool WP>
__device__ __forceinline__ void small_deliver(const ProjDev& J, int64_t ts, int* s_pref) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  DuePrefix wp{};
  int nspk;
  if constexpr (WP) {
    wp = due_prefix_warp(J.src_ring_cnt, J.src_ring_len, ts, J.dmin, J.nd, J.src_lo,
                         J.src_hi);
    nspk = wp.total;
  } else {
    nspk = due_prefix_block(J.src_ring_cnt, J.src_ring_len, ts, J.dmin, J.nd, J.src_lo,
                            J.src_hi, s_pref);
  }
  const int sub = J.chunks * (kChunk / 32);
  const int64_t items = (int64_t)nspk * sub;
  const int base = ring_slot(ts, J.src_ring_len);
  const R* W = static_cast<const R*>(J.w);
  MemberCache<R> mc;
  for (int64_t it = warp; it < items; it += nwarps) {   // warp-uniform
    const int sp = (int)(it / sub);
    const int ch = (int)(it - (int64_t)sp * sub);
    int kk;
    int di;
    if constexpr (WP) di = find_delay_warp(wp, sp, &kk);
    else di = find_delay_block(s_pref, J.nd, sp, &kk);
    const int slot = ring_back(base, J.dmin + di, J.src_ring_len);
    const int32_t pre = J.src_ring_idx[(int64_t)slot * J.src_n + kk];
    const int64_t key = (int64_t)pre * J.nd + di;
    const int64_t s = J.off[key] + (int64_t)ch * 32 + lane;
    if (s < J.off[key + 1]) {
      const int32_t post = __ldg(J.post + s);
      member_lookup<R>(J, pre, mc);
      const R w = W ? __ldg(W + s) : mc.w;
      atomicAdd(mc.target + post, w);
    }
  }
}

template <typename R, int KIND>
__global__ void __launch_bounds__(kSmallThreads, 1)
small_net_kernel(const __grid_constant__ SmallDev D, const int64_t* __restrict__ clock,
                 int steps, double dt, int32_t* status) {
  extern __shared__ __align__(16) uint8_t smem[];
  const PopDev& P = D.pop;
  const SmallLayout L = small_layout(KIND);
  const int64_t n = P.n;   // padded population size, <= 4 * kSmallThreads
  // column c of the image holds variable L.var[c]; v, ge, gi are columns 0-2 for both kinds,
  // lastspike the last one, m, h, n columns 3-5 of HH
  R* const base = reinterpret_cast<R*>(smem);
  constexpr int kLS = KIND == KIND_LIF ? 3 : 6;
  R* const sV = base;
  R* const sGE = base + n;
  R* const sGI = base + 2 * n;
  R* const sLS = base + kLS * n;
  R* const sM = base + 3 * n;   // HH only
  R* const sH = base + 4 * n;
  R* const sN = base + 5 * n;
  uint8_t* snr = smem + sizeof(R) * L.nvars * n;
  int* s_pref = reinterpret_cast<int*>(smem + ((sizeof(R) * L.nvars * n + n + 15) & ~15));
  // the spike-history ring's counts, and its indices when they fit, mirrored in shared memory
  // (every write goes to both; delivery reads the mirror)
  int32_t* s_ring_cnt = s_pref + D.nd_max + 2;
  int32_t* s_ring = D.ring_in_smem ? s_ring_cnt + ((P.ring_len + 3) & ~3) : nullptr;
  __shared__ int s_warp[33];
  __shared__ unsigned long long s_mbase, s_mon;
  const int tid = threadIdx.x;
  const int64_t ts0 = clock[0];

  // state -> shared memory
  for (int i = 0; i < L.nvars; ++i) {
    const R* g = static_cast<const R*>(P.var[L.var[i]]);
    for (int64_t q = tid; q < n; q += blockDim.x) base[i * n + q] = g[q];
  }
  {
    const uint8_t* g = static_cast<const uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY]);
    for (int64_t q = tid; q < n; q += blockDim.x) snr[q] = g[q];
  }
  for (int r = tid; r < P.ring_len; r += blockDim.x) s_ring_cnt[r] = P.ring_cnt[r];
  if (s_ring)
    for (int64_t r = tid; r < (int64_t)P.ring_len * n; r += blockDim.x) s_ring[r] = P.ring_idx[r];
  if (tid == 0) s_mon = P.mon_cnt ? *P.mon_cnt : 0ull;
  // the delivery targets of every projection are the shared-memory arrays, and its source
  // ring the shared-memory mirror
  __shared__ ProjDev J[kMaxProjBatch];
  if (tid < D.n_proj) {
    J[tid] = D.proj[tid];
    for (int v = 0; v < 3; ++v) J[tid].targets[v] = base + v * n;   // v, ge, gi
    J[tid].target = base + D.proj_target[tid] * n;
    J[tid].src_ring_cnt = s_ring_cnt;
    if (s_ring) J[tid].src_ring_idx = s_ring;
  }
  __syncthreads();

  const double inv_dt = 1.0 / dt;
  for (int k = 0; k < steps; ++k) {
    const int64_t ts = ts0 + k;
    const double t = (double)ts * dt;
    const int slot = ring_slot(ts, P.ring_len);
    // ---- groups and thresholds: neurons 4*tid .. 4*tid + 3
    unsigned fl = 0;
    const int64_t q4 = (int64_t)tid;
    if (4 * q4 < n) {
      const int gidx = P.vec_group ? P.vec_group[q4] : 0;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t i = 4 * q4 + e;
        R v = sV[i], ge = sGE[i], gi = sGI[i];
        R ls = sLS[i];
        bool nr = true;
        if constexpr (KIND == KIND_LIF) {
          const LifDev& g = static_cast<const LifDev*>(P.params)[gidx];
          const bool refr = g.ref_steps >= 0;
          if (refr) nr = past_refractory(t - (double)ls, dt, inv_dt, g.ref_steps);
          R vn = lif_advance<R>(
              g, v, ge, gi, nr,
              P.inputs ? timed_input<R>(P.inputs[gidx].ta, ts, i - g.offset) : R(0));
          if (g.has_threshold && (i - g.offset) < g.n && vn > (R)g.Vt && nr) {
            nr = false;
            if (refr) ls = (R)t;
            if (g.has_reset && !P.late_reset) vn = (R)g.Vr;
            fl |= 1u << e;
          }
          v = vn;
          if (refr) {
            sLS[i] = ls;
            snr[i] = nr ? 1 : 0;
          }
        } else {
          const HhRun<R> g = hh_run(static_cast<const HhDev*>(P.params)[gidx], R());
          const bool refr = g.ref_steps >= 0;
          if (refr) nr = past_refractory(t - (double)ls, dt, inv_dt, g.ref_steps);
          R m = sM[i], h = sH[i], nn = sN[i];
          const R vn = hh_advance<R>(g, v, m, h, nn, ge, gi, (R)dt,
                                     P.inputs ? timed_input<R>(P.inputs[gidx].ta, ts,
                                                               i - g.offset)
                                              : R(0));
          if ((i - g.offset) < g.n && vn > (R)g.Vthr && nr) {
            nr = false;
            if (refr) ls = (R)t;
            fl |= 1u << e;
          }
          v = vn;
          sM[i] = m;
          sH[i] = h;
          sN[i] = nn;
          if (refr) {
            sLS[i] = ls;
            snr[i] = nr ? 1 : 0;
          }
        }
        sV[i] = v;
        sGE[i] = ge;
        sGI[i] = gi;
      }
    }
    // ---- compaction into ring slot ts (ascending neuron order) and the monitor
    int total;
    const int c = __popc(fl);
    const int excl = block_exclusive_scan(c, s_warp, &total);
    if (tid == 0) {
      const int next = ring_slot(ts + 1, P.ring_len);
      P.ring_cnt[slot] = total;
      P.ring_cnt[next] = 0;
      s_ring_cnt[slot] = total;
      s_ring_cnt[next] = 0;
      s_mbase = s_mon;     // this kernel is the monitor's only writer while it runs
      s_mon += (unsigned long long)total;
    }
    if (c) {
      int pos = excl;
      int32_t* out = P.ring_idx + (int64_t)slot * P.n;
      int32_t* sout = s_ring ? s_ring + (int64_t)slot * n : nullptr;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (!(fl & (1u << e))) continue;
        out[pos] = (int32_t)(4 * q4 + e);
        if (sout) sout[pos] = (int32_t)(4 * q4 + e);
        ++pos;
      }
    }
    __syncthreads();
    if (c && P.mon_cnt) {
      unsigned long long mpos = s_mbase + (unsigned long long)excl;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (!(fl & (1u << e))) continue;
        if (mpos < (unsigned long long)P.mon_cap) {
          P.mon_idx[mpos] = (int32_t)(4 * q4 + e);
          P.mon_step[mpos] = ts;
        } else {
          set_status(status, B2B_ERR_QUEUE_OVERFLOW);
        }
        ++mpos;
      }
    }
    // ---- synapses: bundles due at step ts, effects into the shared-memory targets
    for (int p = 0; p < D.n_proj; ++p) {
      if (D.warp_prefix) small_deliver<R, true>(J[p], ts, s_pref);
      else small_deliver<R, false>(J[p], ts, s_pref);
      __syncthreads();
    }
    // ---- resets deferred after the synapses (a synapse writes the reset variable)
    if constexpr (KIND == KIND_LIF) {
      if (P.late_reset) {
        const int32_t* idx = s_ring ? s_ring + (int64_t)slot * n : P.ring_idx + (int64_t)slot * P.n;
        for (int r = tid; r < total; r += blockDim.x) {
          const int32_t i = idx[r];
          const LifDev& g = static_cast<const LifDev*>(P.params)[P.vec_group ? P.vec_group[i >> 2] : 0];
          if (g.has_reset) sV[i] = (R)g.Vr;
        }
        __syncthreads();
      }
    }
  }
  // shared memory -> state
  for (int i = 0; i < L.nvars; ++i) {
    R* g = static_cast<R*>(P.var[L.var[i]]);
    for (int64_t q = tid; q < n; q += blockDim.x) g[q] = base[i * n + q];
  }
  {
    uint8_t* g = static_cast<uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY]);
    for (int64_t q = tid; q < n; q += blockDim.x) g[q] = snr[q];
  }
  if (tid == 0 && P.mon_cnt) *P.mon_cnt = s_mon;
}

// Shared-memory copies of what the cluster kernels' step loops read repeatedly (the cluster
// barrier's acquire empties the L1 cache every step): the groups' parameters (at most
// kPullMaxGroups) and the group id of every four neurons of the slice [lo, lo + mine).
template <int KIND>
__device__ __forceinline__ void load_slice_constants(const PopDev& P, int64_t lo, int64_t mine,
                                                     unsigned char* s_prm, int32_t* s_vg) {
  const size_t psz = KIND == KIND_LIF ? sizeof(LifDev) : sizeof(HhDev);
  const unsigned char* gp = static_cast<const unsigned char*>(P.params);
  for (size_t b = threadIdx.x; b < psz * (size_t)P.n_groups; b += blockDim.x) s_prm[b] = gp[b];
  for (int64_t q = threadIdx.x; q < (mine + 3) / 4; q += blockDim.x)
    s_vg[q] = P.vec_group ? P.vec_group[(lo >> 2) + q] : 0;
}

// Update and threshold of this thread's E neurons of the slice (local E tid .. E tid + E - 1,
// population index lo + local) held in shared memory at base (variable c of the layout at
// base + c S, flags at snr), each variable of the E read and written as one vector.  Returns
// the spike bits (bit e: neuron E tid + e).  The cluster kernels give every neuron of a slice
// its own thread (E = 1), so that a step's update is one neuron's chain long: at four neurons
// per thread CUBA 4000 took 4.20 against 3.37 µs per step.
template <typename R, int KIND, int E>
__device__ __forceinline__ unsigned slice_update(R* base, uint8_t* snr, int64_t S,
                                                 const unsigned char* s_prm,
                                                 const int32_t* s_vg, const PopDev& P,
                                                 int64_t lo, int64_t ts, double t, double dt,
                                                 double inv_dt) {
  constexpr int kLS = KIND == KIND_LIF ? 3 : 6;
  R* const sV = base;
  R* const sGE = base + S;
  R* const sGI = base + 2 * S;
  R* const sLS = base + kLS * S;
  R* const sM = base + 3 * S;   // HH only
  R* const sH = base + 4 * S;
  R* const sN = base + 5 * S;
  const int tid = threadIdx.x;
  const int64_t j0 = E * (int64_t)tid;
  unsigned fl = 0;
  const int gidx = s_vg[j0 >> 2];
  Pack<R, E> V = load_pack<R, E>(sV, tid), GE = load_pack<R, E>(sGE, tid);
  Pack<R, E> GI = load_pack<R, E>(sGI, tid), LS = load_pack<R, E>(sLS, tid);
  uint32_t NR = 0;
  if constexpr (KIND == KIND_LIF) {
    const LifDev& g = reinterpret_cast<const LifDev*>(s_prm)[gidx];
    const bool refr = g.ref_steps >= 0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int64_t i = lo + j0 + e;
      bool nr = true;
      if (refr) nr = past_refractory(t - (double)LS.x[e], dt, inv_dt, g.ref_steps);
      R vn = lif_advance<R>(
          g, V.x[e], GE.x[e], GI.x[e], nr,
          P.inputs ? timed_input<R>(P.inputs[gidx].ta, ts, i - g.offset) : R(0));
      if (g.has_threshold && (i - g.offset) < g.n && vn > (R)g.Vt && nr) {
        nr = false;
        if (refr) LS.x[e] = (R)t;
        if (g.has_reset && !P.late_reset) vn = (R)g.Vr;
        fl |= 1u << e;
      }
      V.x[e] = vn;
      NR |= (nr ? 1u : 0u) << (8 * e);
    }
    if (refr) {
      store_pack<R, E>(sLS, tid, LS);
      store_flags<E>(snr, tid, NR);
    }
  } else {
    const HhRun<R> g = hh_run(reinterpret_cast<const HhDev*>(s_prm)[gidx], R());
    const bool refr = g.ref_steps >= 0;
    Pack<R, E> M = load_pack<R, E>(sM, tid), H = load_pack<R, E>(sH, tid);
    Pack<R, E> NN = load_pack<R, E>(sN, tid);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int64_t i = lo + j0 + e;
      bool nr = true;
      if (refr) nr = past_refractory(t - (double)LS.x[e], dt, inv_dt, g.ref_steps);
      const R vn = hh_advance<R>(g, V.x[e], M.x[e], H.x[e], NN.x[e], GE.x[e], GI.x[e],
                                 (R)dt,
                                 P.inputs ? timed_input<R>(P.inputs[gidx].ta, ts,
                                                           i - g.offset)
                                          : R(0));
      if ((i - g.offset) < g.n && vn > (R)g.Vthr && nr) {
        nr = false;
        if (refr) LS.x[e] = (R)t;
        fl |= 1u << e;
      }
      V.x[e] = vn;
      NR |= (nr ? 1u : 0u) << (8 * e);
    }
    store_pack<R, E>(sM, tid, M);
    store_pack<R, E>(sH, tid, H);
    store_pack<R, E>(sN, tid, NN);
    if (refr) {
      store_pack<R, E>(sLS, tid, LS);
      store_flags<E>(snr, tid, NR);
    }
  }
  store_pack<R, E>(sV, tid, V);
  store_pack<R, E>(sGE, tid, GE);
  store_pack<R, E>(sGI, tid, GI);
  return fl;
}

// ---- the same, spread over one thread-block cluster ------------------------------------
// The one-CTA form is bound by one SM's issue rate once a step has a few thousand neurons;
// here the CTAs of one cluster (up to 16 SMs) share the chunk: CTA r keeps neurons
// [r S, (r+1) S) in its shared memory, and cluster barriers (hardware, no spinning) take the
// place of the block barriers between the phases of a step:
//   update and threshold of the CTA's slice, compaction of its spikes in shared memory;
//   barrier; each CTA reads every CTA's spike count from distributed shared memory, writes its
//   spikes at its offset into the step's slot of the spike-history ring in global memory (in
//   ascending neuron order, as the per-step kernels' compaction leaves them per CTA);
//   barrier (the ring slot is complete and visible to the cluster);
//   delivery of the due bundles by every warp of the cluster, each effect an atomic addition
//   into the shared memory of the CTA that owns the target neuron;
//   barrier (every effect has landed); a deferred reset by each CTA for its own neurons.
// Requires every projection to have at most 64 delays (the per-warp prefix).
namespace cg = cooperative_groups;

template <typename R>
__device__ __forceinline__ void cluster_deliver(const cg::cluster_group& cl, const ProjDev& J,
                                                int64_t ts, int64_t S, int64_t wid,
                                                int64_t nw) {
  const int lane = threadIdx.x & 31;
  const DuePrefix wp = due_prefix_warp(J.src_ring_cnt, J.src_ring_len, ts, J.dmin, J.nd,
                                       J.src_lo, J.src_hi);
  const int sub = J.chunks * (kChunk / 32);
  const int64_t items = (int64_t)wp.total * sub;
  const int base = ring_slot(ts, J.src_ring_len);
  const R* W = static_cast<const R*>(J.w);
  MemberCache<R> mc;
  for (int64_t it = wid; it < items; it += nw) {   // warp-uniform
    const int sp = (int)(it / sub);
    const int ch = (int)(it - (int64_t)sp * sub);
    int kk;
    const int di = find_delay_warp(wp, sp, &kk);
    const int slot = ring_back(base, J.dmin + di, J.src_ring_len);
    const int32_t pre = J.src_ring_idx[(int64_t)slot * J.src_n + kk];
    const int64_t key = (int64_t)pre * J.nd + di;
    const int64_t s = J.off[key] + (int64_t)ch * 32 + lane;
    if (s < J.off[key + 1]) {
      const int32_t post = __ldg(J.post + s);
      member_lookup<R>(J, pre, mc);
      const R w = W ? __ldg(W + s) : mc.w;
      const unsigned owner = (unsigned)(post / S);
      R* dst = cl.map_shared_rank(mc.target, owner) + (post - (int64_t)owner * S);
      atomicAdd(dst, w);
    }
  }
}

template <typename R, int KIND>
__global__ void __launch_bounds__(kSmallThreads, 1)
small_cluster_kernel(const __grid_constant__ SmallDev D, const int64_t* __restrict__ clock,
                     int steps, double dt, int32_t* status, int64_t S) {
  extern __shared__ __align__(16) uint8_t smem[];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int C = (int)cl.num_blocks();
  const PopDev& P = D.pop;
  const SmallLayout L = small_layout(KIND);
  const int64_t n = P.n;
  const int64_t lo = (int64_t)rank * S;
  const int64_t mine = lo < n ? (n - lo < S ? n - lo : S) : 0;   // neurons of this CTA
  R* const base = reinterpret_cast<R*>(smem);   // the slice's variables, as in slice_update
  R* const sV = base;
  uint8_t* snr = smem + sizeof(R) * L.nvars * S;
  int32_t* s_ring_cnt = reinterpret_cast<int32_t*>(smem + ((sizeof(R) * L.nvars * S + S + 15) & ~15));
  int32_t* s_vg = s_ring_cnt + ((P.ring_len + 3) & ~3);   // group of each 4 neurons of the slice
  __shared__ int s_warp[33];
  __shared__ int s_cnt, s_off, s_tot;
  __shared__ unsigned long long s_mon;
  __shared__ __align__(16) unsigned char s_prm[kPullMaxGroups * sizeof(HhDev)];
  const int tid = threadIdx.x;
  const int64_t ts0 = clock[0];
  load_slice_constants<KIND>(P, lo, mine, s_prm, s_vg);

  for (int i = 0; i < L.nvars; ++i) {
    const R* g = static_cast<const R*>(P.var[L.var[i]]);
    for (int64_t q = tid; q < mine; q += blockDim.x) base[i * S + q] = g[lo + q];
  }
  {
    const uint8_t* g = static_cast<const uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY]);
    for (int64_t q = tid; q < mine; q += blockDim.x) snr[q] = g[lo + q];
  }
  for (int r = tid; r < P.ring_len; r += blockDim.x) s_ring_cnt[r] = P.ring_cnt[r];
  if (tid == 0) s_mon = P.mon_cnt ? *P.mon_cnt : 0ull;
  // delivery targets: this CTA's shared-memory arrays (the same offsets in every CTA of the
  // cluster, mapped to the owner's at each effect); source ring: the global ring, counts
  // from the shared-memory mirror
  __shared__ ProjDev J[kMaxProjBatch];
  if (tid < D.n_proj) {
    J[tid] = D.proj[tid];
    for (int v = 0; v < 3; ++v) J[tid].targets[v] = base + v * S;   // v, ge, gi
    J[tid].target = base + D.proj_target[tid] * S;
    J[tid].src_ring_cnt = s_ring_cnt;
  }
  __syncthreads();
  const int64_t nwarps = blockDim.x >> 5;
  const int64_t wid = (int64_t)rank * nwarps + (tid >> 5);
  const int64_t nw = (int64_t)C * nwarps;

  const double inv_dt = 1.0 / dt;
  for (int k = 0; k < steps; ++k) {
    const int64_t ts = ts0 + k;
    const double t = (double)ts * dt;
    const int slot = ring_slot(ts, P.ring_len);
    // ---- groups and thresholds: local neuron tid
    const int64_t j0 = tid;
    const unsigned fl =
        j0 < mine ? slice_update<R, KIND, 1>(base, snr, S, s_prm, s_vg, P, lo, ts, t, dt, inv_dt)
                  : 0u;
    // ---- compaction: this CTA's count, then its offset among the cluster's CTAs
    int total;
    const int c = __popc(fl);
    const int excl = block_exclusive_scan(c, s_warp, &total);
    if (tid == 0) s_cnt = total;
    cl.sync();
    if (tid == 0) {
      int off = 0, tot = 0;
      for (int q = 0; q < C; ++q) {
        const int cq = *cl.map_shared_rank(&s_cnt, (unsigned)q);
        if (q < rank) off += cq;
        tot += cq;
      }
      s_off = off;
      s_tot = tot;
      const int next = ring_slot(ts + 1, P.ring_len);
      s_ring_cnt[slot] = tot;
      s_ring_cnt[next] = 0;
      if (rank == 0) {
        P.ring_cnt[slot] = tot;
        P.ring_cnt[next] = 0;
      }
    }
    __syncthreads();
    if (c) {
      int pos = s_off + excl;
      int32_t* out = P.ring_idx + (int64_t)slot * P.n;
      unsigned long long mpos = s_mon + (unsigned long long)(s_off + excl);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (!(fl & (1u << e))) continue;
        const int32_t idx = (int32_t)(lo + j0 + e);
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
    cl.sync();   // the ring slot is complete, and every CTA has read the counts
    if (tid == 0) s_mon += (unsigned long long)s_tot;
    // ---- synapses: every warp of the cluster, effects into the owners' shared memory
    for (int p = 0; p < D.n_proj; ++p) cluster_deliver<R>(cl, J[p], ts, S, wid, nw);
    cl.sync();   // every effect has landed
    // ---- resets deferred after the synapses, each CTA for its own neurons
    if constexpr (KIND == KIND_LIF) {
      if (P.late_reset) {
        const int32_t* idx = P.ring_idx + (int64_t)slot * P.n;
        const int tot = s_tot;
        for (int r = tid; r < tot; r += blockDim.x) {
          const int32_t i = idx[r];
          if (i < lo || i >= lo + mine) continue;
          const LifDev& g = reinterpret_cast<const LifDev*>(s_prm)[s_vg[(i - lo) >> 2]];
          if (g.has_reset) sV[i - lo] = (R)g.Vr;
        }
      }
    }
    __syncthreads();
  }
  for (int i = 0; i < L.nvars; ++i) {
    R* g = static_cast<R*>(P.var[L.var[i]]);
    for (int64_t q = tid; q < mine; q += blockDim.x) g[lo + q] = base[i * S + q];
  }
  {
    uint8_t* g = static_cast<uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY]);
    for (int64_t q = tid; q < mine; q += blockDim.x) g[lo + q] = snr[q];
  }
  if (tid == 0 && rank == 0 && P.mon_cnt) *P.mon_cnt = s_mon;
}

// ---- the cluster form with the effects gathered per slice -----------------------------
// For a net whose synapses have no delays and no weights of their own (the CUBA example), a
// step needs one cluster barrier: CTA r keeps, beside its slice of the state, the synapses
// into its slice grouped by presynaptic neuron (offsets and slice-local targets, loaded into
// shared memory at launch):
//   update and threshold of the slice; compaction of its spikes into a local list (double
//   buffered by step parity);
//   barrier;
//   every CTA copies all CTAs' lists (distributed shared memory) into one list of the step's
//   spikes, in rank order, and writes its own spikes at their offset into the global ring and
//   monitor (the per-step kernels' record of the step);
//   each spike's synapses into the slice add that Synapses object's weight to their target
//   variable in shared memory (a warp per spike; the synapses slot), then the deferred reset.
// No global memory is read inside the step loop.  The group parameters, group ids and member
// tables are copied to shared memory first as well: the cluster barrier's acquire empties
// the L1 cache every step.  A final barrier keeps every CTA's lists alive until all CTAs
// have read them.
template <typename R, int KIND>
__global__ void __launch_bounds__(kSmallThreads, 1)
small_pull_kernel(const __grid_constant__ SmallDev D, const int64_t* __restrict__ clock,
                  int steps, double dt, int32_t* status, int64_t S) {
  extern __shared__ __align__(16) uint8_t smem[];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int C = (int)cl.num_blocks();
  const PopDev& P = D.pop;
  const SmallLayout L = small_layout(KIND);
  const int64_t n = P.n;
  const int64_t lo = (int64_t)rank * S;
  const int64_t mine = lo < n ? (n - lo < S ? n - lo : S) : 0;
  R* const base = reinterpret_cast<R*>(smem);   // the slice's variables, as in slice_update
  R* const sV = base;
  uint8_t* snr = smem + sizeof(R) * L.nvars * S;
  int32_t* lists = reinterpret_cast<int32_t*>(smem + ((sizeof(R) * L.nvars * S + S + 15) & ~15));
  int32_t* all = lists + 2 * S;                 // lists: [2][S]; the step's spikes, [n]
  int32_t* s_vg = all + n;                      // group of each 4 neurons of the slice
  int32_t* s_off = s_vg + (S + 3) / 4;          // [n_proj][n + 1] synapses into the slice by pre
  uint16_t* s_tgt = reinterpret_cast<uint16_t*>(s_off + (int64_t)D.n_proj * (n + 1));
  __shared__ int32_t s_tstart[kMaxProjBatch + 1];   // each projection's targets in s_tgt
  __shared__ int s_warp[33];
  __shared__ int s_cnt[2];
  __shared__ int s_pre[17];                     // counts of the ranks before each rank
  __shared__ unsigned long long s_mon;
  // The cluster barrier's acquire empties the L1 cache every step, so whatever the step loop
  // reads repeatedly lives in shared memory: the groups' parameters, the slice's group ids and
  // the projections' member tables (Synapses object of a presynaptic range: target variable
  // and weight).
  __shared__ __align__(16) unsigned char s_prm[kPullMaxGroups * sizeof(HhDev)];
  __shared__ int64_t s_mhi[kMaxProjBatch][kPullMaxMembers];
  __shared__ int32_t s_mvar[kMaxProjBatch][kPullMaxMembers];
  __shared__ double s_mw[kMaxProjBatch][kPullMaxMembers];
  __shared__ int32_t s_nmem[kMaxProjBatch];
  const int tid = threadIdx.x;
  const int64_t ts0 = clock[0];
  {
    load_slice_constants<KIND>(P, lo, mine, s_prm, s_vg);
    if (tid == 0) {
      int32_t acc = 0;
      for (int p = 0; p < D.n_proj; ++p) {
        s_tstart[p] = acc;
        acc += (int32_t)(D.pull_base[p * (C + 1) + rank + 1] - D.pull_base[p * (C + 1) + rank]);
      }
      s_tstart[D.n_proj] = acc;
    }
    __syncthreads();
    for (int p = 0; p < D.n_proj; ++p) {
      const int32_t* goff = D.pull_off + ((int64_t)p * C + rank) * (n + 1);
      for (int64_t x = tid; x <= n; x += blockDim.x) s_off[p * (n + 1) + x] = goff[x];
      const uint16_t* gtgt = D.pull_tgt + D.pull_base[p * (C + 1) + rank];
      for (int64_t x = tid; x < s_tstart[p + 1] - s_tstart[p]; x += blockDim.x)
        s_tgt[s_tstart[p] + x] = gtgt[x];
    }
    for (int x = tid; x < D.n_proj * kPullMaxMembers; x += blockDim.x) {
      const int p = x / kPullMaxMembers, m = x - p * kPullMaxMembers;
      const ProjDev& J = D.proj[p];
      if (m == 0) s_nmem[p] = J.n_mem;
      if (m < J.n_mem) {
        s_mhi[p][m] = J.n_mem == 1 ? INT64_MAX : J.mem_hi[m];
        s_mvar[p][m] = J.n_mem == 1 ? D.proj_target[p] : (int32_t)J.mem_var[m];
        s_mw[p][m] = J.mem_w ? J.mem_w[m] : J.w_scalar;
      }
    }
  }

  for (int i = 0; i < L.nvars; ++i) {
    const R* g = static_cast<const R*>(P.var[L.var[i]]);
    for (int64_t q = tid; q < mine; q += blockDim.x) base[i * S + q] = g[lo + q];
  }
  {
    const uint8_t* g = static_cast<const uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY]);
    for (int64_t q = tid; q < mine; q += blockDim.x) snr[q] = g[lo + q];
  }
  if (tid == 0) s_mon = P.mon_cnt ? *P.mon_cnt : 0ull;
  __syncthreads();

  const double inv_dt = 1.0 / dt;
  for (int k = 0; k < steps; ++k) {
    const int64_t ts = ts0 + k;
    const double t = (double)ts * dt;
    const int slot = ring_slot(ts, P.ring_len);
    const int par = k & 1;
    int32_t* mylist = lists + par * S;
    // ---- groups and thresholds: local neuron tid
    const int64_t j0 = tid;
    const unsigned fl =
        j0 < mine ? slice_update<R, KIND, 1>(base, snr, S, s_prm, s_vg, P, lo, ts, t, dt, inv_dt)
                  : 0u;
    // ---- this CTA's spikes into its local list (ascending neuron order)
    // (most CTAs of most steps have no spike: one barrier decides that for the CTA)
    int total = 0, excl = 0;
    const int c = __popc(fl);
    if (__syncthreads_or(fl != 0)) excl = block_exclusive_scan(c, s_warp, &total);
    if (c) {
      int pos = excl;
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (fl & (1u << e)) mylist[pos++] = (int32_t)(lo + j0 + e);
    }
    if (tid == 0) s_cnt[par] = total;
    cl.sync();
    // ---- every CTA's spikes of the step, in rank order
    if (tid < 32) {   // warp 0: one rank's count per lane, then their prefix
      const int cq = tid < C ? *cl.map_shared_rank(&s_cnt[par], (unsigned)tid) : 0;
      const int incl = warp_incl_scan(cq);
      if (tid < C) s_pre[tid] = incl - cq;
      if (tid == 31) s_pre[C] = incl;
    }
    __syncthreads();
    const int tot = s_pre[C];
    for (int x = tid; x < tot; x += blockDim.x) {
      int q = 0;
      while (q + 1 < C && s_pre[q + 1] <= x) ++q;
      all[x] = *cl.map_shared_rank(lists + par * S + (x - s_pre[q]), (unsigned)q);
    }
    // the per-step kernels' record of the step: global ring slot and monitor
    {
      const int off = s_pre[rank];
      int32_t* out = P.ring_idx + (int64_t)slot * P.n;
      for (int x = tid; x < total; x += blockDim.x) {
        const int32_t idx = mylist[x];
        out[off + x] = idx;
        if (P.mon_cnt) {
          const unsigned long long mpos = s_mon + (unsigned long long)(off + x);
          if (mpos < (unsigned long long)P.mon_cap) {
            P.mon_idx[mpos] = idx;
            P.mon_step[mpos] = ts;
          } else {
            set_status(status, B2B_ERR_QUEUE_OVERFLOW);
          }
        }
      }
      if (tid == 0 && rank == 0) {
        P.ring_cnt[slot] = tot;
        P.ring_cnt[ring_slot(ts + 1, P.ring_len)] = 0;
      }
    }
    __syncthreads();
    if (tid == 0) s_mon += (unsigned long long)tot;
    // ---- synapses slot: a warp per spike and projection, its synapses into this slice
    {
      const int lane = tid & 31;
      const int nw = (int)(blockDim.x >> 5);
      for (int p = 0; p < D.n_proj; ++p) {
        const int32_t* o = s_off + p * (n + 1);
        const uint16_t* tg = s_tgt + s_tstart[p];
        for (int x = tid >> 5; x < tot; x += nw) {
          const int32_t pre = all[x];
          if (o[pre] == o[pre + 1]) continue;
          int m = 0, mh = s_nmem[p] - 1;            // the member whose range holds pre
          while (m < mh) {
            const int mid = (m + mh) >> 1;
            if (pre < s_mhi[p][mid]) mh = mid; else m = mid + 1;
          }
          R* T = base + s_mvar[p][m] * S;           // v, ge, gi: columns 0-2
          const R wgt = (R)s_mw[p][m];
          for (int32_t s = o[pre] + lane; s < o[pre + 1]; s += 32) atomicAdd(T + tg[s], wgt);
        }
      }
    }
    __syncthreads();
    // ---- resets deferred after the synapses, for this CTA's spiking neurons
    if constexpr (KIND == KIND_LIF) {
      if (P.late_reset) {
        for (int x = tid; x < total; x += blockDim.x) {
          const int32_t i = mylist[x];
          const LifDev& g = reinterpret_cast<const LifDev*>(s_prm)[s_vg[(i - lo) >> 2]];
          if (g.has_reset) sV[i - lo] = (R)g.Vr;
        }
      }
    }
    __syncthreads();
  }
  cl.sync();   // every CTA is done reading the others' lists
  for (int i = 0; i < L.nvars; ++i) {
    R* g = static_cast<R*>(P.var[L.var[i]]);
    for (int64_t q = tid; q < mine; q += blockDim.x) g[lo + q] = base[i * S + q];
  }
  {
    uint8_t* g = static_cast<uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY]);
    for (int64_t q = tid; q < mine; q += blockDim.x) g[lo + q] = snr[q];
  }
  if (tid == 0 && rank == 0 && P.mon_cnt) *P.mon_cnt = s_mon;
}

}  // namespace

size_t small_smem(const SmallDev& D, int kind, int dtype) {
  const SmallLayout L = small_layout(kind);
  const size_t rs = dtype == B2B_F32 ? 4 : 8;
  const size_t base = (rs * L.nvars * (size_t)D.pop.n + (size_t)D.pop.n + 15) & ~(size_t)15;
  size_t bytes = base + sizeof(int) * (size_t)(D.nd_max + 2) +
                 sizeof(int) * (size_t)((D.pop.ring_len + 3) & ~3);
  if (D.ring_in_smem) bytes += sizeof(int32_t) * (size_t)D.pop.ring_len * (size_t)D.pop.n;
  return bytes;
}

// Shared memory of one CTA of the cluster form: its slice of the state and flags, then the
// ring counts (push form) or the slice's bit rows, two local spike lists and the step's list
// (pull form).
size_t small_cluster_smem(const SmallDev& D, int kind, int dtype) {
  const SmallLayout L = small_layout(kind);
  const size_t rs = dtype == B2B_F32 ? 4 : 8;
  const size_t S = (size_t)D.slice;
  const size_t state = (rs * L.nvars * S + S + 15) & ~(size_t)15;
  if (D.pull)
    return state +
           sizeof(int32_t) * (2 * S + (size_t)D.pop.n + (S + 3) / 4 +
                              (size_t)D.n_proj * (D.pop.n + 1)) +
           sizeof(uint16_t) * (size_t)D.pull_max_tgt;
  return state + sizeof(int32_t) * ((size_t)((D.pop.ring_len + 3) & ~3) + (S + 3) / 4);
}

namespace {
bool pull_members_fit(const SmallDev& D) {
  for (int p = 0; p < D.n_proj; ++p)
    if (D.proj[p].n_mem > kPullMaxMembers) return false;
  return true;
}

template <typename R, int K>
cudaError_t launch_cluster_rk(const SmallDev& D, const int64_t* clock, int steps, double dt,
                              int32_t* status, cudaStream_t s, size_t smem, bool probe) {
  auto kern = D.pull ? small_pull_kernel<R, K> : small_cluster_kernel<R, K>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e == cudaSuccess && D.cluster > 8)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  // a thread per neuron of the slice, at least 256 (the delivery's warps)
  const int threads = (int)std::max<int64_t>(256, ((D.slice + 31) / 32) * 32);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)D.cluster);
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)D.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (probe) {
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, (const void*)kern, &cfg);
    return e != cudaSuccess ? e : (clusters >= 1 ? cudaSuccess : cudaErrorInvalidConfiguration);
  }
  return cudaLaunchKernelEx(&cfg, kern, D, clock, steps, dt, status, (int64_t)D.slice);
}

cudaError_t launch_cluster(const SmallDev& D, int kind, int dtype, const int64_t* clock,
                           int steps, double dt, int32_t* status, cudaStream_t s, bool probe) {
  if (D.cluster < 2 || D.cluster > 16 || D.slice < 4 || D.slice % 4 || !D.warp_prefix ||
      D.slice > kSmallThreads || D.pop.n_groups > kPullMaxGroups ||
      (D.pull && (!D.pull_off || !pull_members_fit(D))))
    return cudaErrorInvalidValue;
  const size_t smem = small_cluster_smem(D, kind, dtype);
  if (kind == KIND_LIF && dtype == B2B_F32)
    return launch_cluster_rk<float, KIND_LIF>(D, clock, steps, dt, status, s, smem, probe);
  if (kind == KIND_LIF)
    return launch_cluster_rk<double, KIND_LIF>(D, clock, steps, dt, status, s, smem, probe);
  if (dtype == B2B_F32)
    return launch_cluster_rk<float, KIND_HH>(D, clock, steps, dt, status, s, smem, probe);
  return launch_cluster_rk<double, KIND_HH>(D, clock, steps, dt, status, s, smem, probe);
}
}  // namespace

bool small_cluster_possible(const SmallDev& D, int kind, int dtype) {
  const bool ok =
      launch_cluster(D, kind, dtype, nullptr, 0, 0.0, nullptr, nullptr, true) == cudaSuccess;
  // a refused attribute or occupancy query leaves its (non-sticky) error as the last error,
  // which the next launch check would report as its own
  if (!ok) cudaGetLastError();
  return ok;
}

cudaError_t launch_small(const SmallDev& D, int kind, int dtype, const int64_t* clock,
                         int steps, double dt, int32_t* status, cudaStream_t s) {
  if (D.cluster > 1)
    return launch_cluster(D, kind, dtype, clock, steps, dt, status, s, false);
  const size_t smem = small_smem(D, kind, dtype);
  cudaError_t e = cudaSuccess;
#define B2B_SMALL(R, K)                                                                       \
  do {                                                                                        \
    e = cudaFuncSetAttribute(small_net_kernel<R, K>,                                          \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);         \
    if (e == cudaSuccess)                                                                     \
      small_net_kernel<R, K><<<1, kSmallThreads, smem, s>>>(D, clock, steps, dt, status);     \
  } while (0)
  if (kind == KIND_LIF && dtype == B2B_F32) B2B_SMALL(float, KIND_LIF);
  else if (kind == KIND_LIF) B2B_SMALL(double, KIND_LIF);
  else if (dtype == B2B_F32) B2B_SMALL(float, KIND_HH);
  else B2B_SMALL(double, KIND_HH);
#undef B2B_SMALL
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace b2b
