// Spike propagation: delivery of due synapse bundles from the spike-history ring, with the
// on_pre / on_post effects (additive, and event-driven STDP with its traces) applied in the
// same pass.
//
// Reference: the per-step push of (pre, post-block, delay) bundle ids into CudaSpikeQueue
// slots `(current_offset + delay) % num_queues` under per-post-block spin locks with
// device-malloc growth (brian2cuda/brianlib/spikequeue.h:432-511, templates/
// synapses_push_spikes.cu:1056-1131), then the effect kernel over the current slot
// (templates/synapses.cu:12-164) with `_brian_atomicAdd` (cuda_generator.py:33-157).
//
// Here nothing is pushed.  Each population keeps the compacted spikes of its last
// `ring_len` steps (written by the neuron kernel).  A bundle (pre, d) is due at step ts
// exactly when pre spiked at step ts - d, so the delivery kernels enumerate, for every delay
// d of the projection, the spikes of ring slot ts - d and walk the synapse range of bundle
// (pre, d) in the (pre, delay)-sorted synapse arrays (delivery.cuh).  This is the same set of
// bundles the reference's queue holds in slot `current_offset` after its push, without the
// push kernel, the host sync on the spike count, the locks or the device heap.
#include <cooperative_groups.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "delivery.cuh"

namespace cg = cooperative_groups;

namespace b2b {

namespace {

constexpr int kDeliverBlock = 256;
constexpr int kAddUnroll = 4;

// Sum of `v` over the lanes whose key equals this lane's key; valid in every lane.
template <typename R>
__device__ __forceinline__ R peer_sum(unsigned peers, R v) {
  R acc = 0;
#pragma unroll 1
  for (int src = 0; src < 32; ++src) {
    const R x = __shfl_sync(kFull, v, src);
    if ((peers >> src) & 1u) acc += x;
  }
  return acc;
}

// T[post] += w for one synapse per lane; AGG sums lanes hitting the same element first.  The
// lanes of a warp may write different target arrays (the members of a projection that merges
// several Synapses objects), so lanes are matched on the element's address.
template <typename R, bool AGG>
__device__ __forceinline__ void add_to_target(R* T, int32_t post, R w, bool valid) {
  if constexpr (AGG) {
    const unsigned peers =
        __match_any_sync(kFull, valid ? (unsigned long long)(T + post) : 0ull);
    const R sum = peer_sum<R>(peers, valid ? w : (R)0);
    if (valid && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(T + post, sum);
  } else {
    if (valid) atomicAdd(T + post, w);
  }
}

// Several additive projections in one launch: blockIdx.y picks the projection.
struct ProjBatch {
  ProjDev p[kMaxProjBatch];
  int n;
};

// ---- on_pre: target[post] += w -------------------------------------------------------------
template <typename R, bool HAS_W, bool AGG, bool WARP_PREFIX, int GROUP>
__global__ void __launch_bounds__(kDeliverBlock)
deliver_add_batch_kernel(const __grid_constant__ ProjBatch B, const int64_t* __restrict__ clock,
                         int k) {
  extern __shared__ int s_pref[];
  const ProjDev& P = B.p[blockIdx.y];
  const int64_t ts = clock[0] + k;
  const R* __restrict__ W = static_cast<const R*>(P.w);
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int glane = (threadIdx.x & 31) % GROUP;
  MemberCache<R> mc;
  for_each_due_item<WARP_PREFIX, GROUP>(P, ts, warp0, nwarps, s_pref,
                                        [&](int64_t b0, int64_t b1, int64_t len, int32_t pre) {
    member_lookup<R>(P, pre, mc);
    // kAddUnroll rounds of the bundle per pass: their loads are all issued before the first
    // atomic, so each lane keeps several independent loads in flight
    for (int64_t off = 0; off < len; off += kAddUnroll * GROUP) {
      int32_t post[kAddUnroll];
      R w[kAddUnroll];
      bool v[kAddUnroll];
#pragma unroll
      for (int u = 0; u < kAddUnroll; ++u) {
        const int64_t s = b0 + off + u * GROUP + glane;
        v[u] = s < b1;
        post[u] = v[u] ? __ldg(P.post + s) : 0;
        w[u] = mc.w;
        if constexpr (HAS_W) w[u] = v[u] ? __ldg(W + s) : (R)0;
      }
#pragma unroll
      for (int u = 0; u < kAddUnroll; ++u)
        if (off + u * GROUP < len)  // warp-uniform
          add_to_target<R, AGG>(mc.target, post[u], w[u], v[u]);
    }
  });
}

// ---- on_pre of event-driven additive STDP (examples/stdp.py:125-186) ----------------------
// Traces decay lazily from lastupdate to t (Brian2's event-driven update); in float32 the
// elapsed time is rounded to float first, as brian2cuda does (brian2cuda/device.py:1034-1039).
// A synapse's four variables are one interleaved record (one 16-byte access in float32).
template <typename R>
struct __align__(4 * sizeof(R)) SynRec {
  R w, apre, apost, lu;
};

template <typename R, bool AGG, bool WARP_PREFIX>
__global__ void __launch_bounds__(kDeliverBlock)
deliver_stdp_pre_kernel(ProjDev P, const int64_t* __restrict__ clock, int k, double dt) {
  extern __shared__ int s_pref[];
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  SynRec<R>* __restrict__ S = static_cast<SynRec<R>*>(P.syn4);
  R* __restrict__ T = static_cast<R*>(P.target);
  const R taupre = (R)P.taupre, taupost = (R)P.taupost, dApre = (R)P.dApre;
  const R wmin = (R)P.wmin, wmax = (R)P.wmax;
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for_each_due_item<WARP_PREFIX, 32>(P, ts, warp0, nwarps, s_pref,
                                     [&](int64_t b0, int64_t b1, int64_t len, int32_t) {
    // the item's (at most kChunk) synapses, kChunk/32 per lane: every load of the lane is
    // issued before the first record is updated (distinct records: no ordering between them)
    static_assert(kChunk % 32 == 0, "an item is whole rounds of the warp");
    constexpr int kPer = kChunk / 32;
    SynRec<R> r[kPer];
    int64_t at[kPer];
    int32_t post[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int64_t s = b0 + lane + 32 * u;
      const bool ok = s < b1;
      post[u] = ok ? __ldg(P.post + s) : 0;
      at[u] = ok ? (P.rec_of ? (int64_t)__ldg(P.rec_of + s) : s) : -1;
      if (ok) r[u] = S[at[u]];
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      R w = 0;
      if (at[u] >= 0) {
        w = r[u].w;
        const R tau = (R)(t - (double)r[u].lu);
        R apre = r[u].apre * dexp(-tau / taupre);
        const R apost = r[u].apost * dexp(-tau / taupost);
        apre = apre + dApre;
        r[u].w = dclip(w + apost, wmin, wmax);
        r[u].apre = apre;
        r[u].apost = apost;
        r[u].lu = (R)t;
        S[at[u]] = r[u];
      }
      if (P.pre_adds_weight && 32 * u < len)  // warp-uniform
        add_to_target<R, AGG>(T, post[u], w, at[u] >= 0);
    }
  });
}

// ---- on_post of event-driven additive STDP -------------------------------------------------
// Every synapse of each neuron of the target population that spiked this step, reached
// through the transposed (post-sorted) index.
template <typename R>
__global__ void __launch_bounds__(kDeliverBlock)
deliver_stdp_post_kernel(ProjDev P, const int64_t* __restrict__ clock, int k, double dt) {
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const int slot = ring_slot(ts, P.post_ring_len);
  const int nspk = P.post_ring_cnt[slot];
  const int32_t* spikes = P.post_ring_idx + (int64_t)slot * P.post_src_n;
  SynRec<R>* __restrict__ S = static_cast<SynRec<R>*>(P.syn4);
  const R taupre = (R)P.taupre, taupost = (R)P.taupost, dApost = (R)P.dApost;
  const R wmin = (R)P.wmin, wmax = (R)P.wmax;
  const int lane = threadIdx.x & 31;
  const int64_t items = (int64_t)nspk * P.post_chunks;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t it = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); it < items;
       it += warps) {
    const int sp = (int)(it / P.post_chunks);
    const int ch = (int)(it - (int64_t)sp * P.post_chunks);
    const int32_t j = spikes[sp];
    const int64_t b0 = P.post_off[j] + (int64_t)ch * kChunk;
    int64_t b1 = P.post_off[j + 1];
    if (b1 > b0 + kChunk) b1 = b0 + kChunk;
    // the lane's (up to) kChunk/32 records of the item, all loaded before any is updated so
    // that their loads are in flight together (distinct records: no ordering between them)
    static_assert(kChunk % 32 == 0, "an item is whole rounds of the warp");
    constexpr int kPer = kChunk / 32;
    SynRec<R> q[kPer];
    int64_t at[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int64_t r = b0 + lane + 32 * u;
      // post-grouped records: record r itself (contiguous); otherwise its synapse's record
      at[u] = r < b1 ? (P.rec_of ? r : (int64_t)P.post_syn[r]) : -1;
      if (at[u] >= 0) q[u] = S[at[u]];
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      if (at[u] < 0) continue;
      const R tau = (R)(t - (double)q[u].lu);
      const R apre = q[u].apre * dexp(-tau / taupre);
      R apost = q[u].apost * dexp(-tau / taupost);
      apost = apost + dApost;
      q[u].w = dclip(q[u].w + apre, wmin, wmax);
      q[u].apre = apre;
      q[u].apost = apost;
      q[u].lu = (R)t;
      S[at[u]] = q[u];
    }
  }
}

unsigned deliver_grid(const Proj& pr) {
  const int64_t want = (pr.dev.src_n * (int64_t)pr.dev.chunks) / 64 + 1;
  const int64_t cap = 4 * kNumSMs;
  return (unsigned)(want < cap ? want : cap);
}

template <typename R, bool HAS_W, bool AGG, int GROUP>
void launch_add_g(const ProjBatch& B, dim3 g, bool warp_prefix, size_t smem,
                  const int64_t* clock, int k, cudaStream_t s) {
  if (warp_prefix)
    deliver_add_batch_kernel<R, HAS_W, AGG, true, GROUP><<<g, kDeliverBlock, 0, s>>>(B, clock, k);
  else
    deliver_add_batch_kernel<R, HAS_W, AGG, false, GROUP><<<g, kDeliverBlock, smem, s>>>(B, clock,
                                                                                         k);
}

// Lanes per work item: 8 (four items in flight per warp, the default), 2, 4, 16 or 32.
template <typename R, bool HAS_W, bool AGG>
void launch_add(const ProjBatch& B, dim3 g, bool warp_prefix, size_t smem, const int64_t* clock,
                int k, cudaStream_t s, int group) {
  if (group == 32) launch_add_g<R, HAS_W, AGG, 32>(B, g, warp_prefix, smem, clock, k, s);
  else if (group == 16) launch_add_g<R, HAS_W, AGG, 16>(B, g, warp_prefix, smem, clock, k, s);
  else if (group == 4) launch_add_g<R, HAS_W, AGG, 4>(B, g, warp_prefix, smem, clock, k, s);
  else if (group == 2) launch_add_g<R, HAS_W, AGG, 2>(B, g, warp_prefix, smem, clock, k, s);
  else launch_add_g<R, HAS_W, AGG, 8>(B, g, warp_prefix, smem, clock, k, s);
}

template <typename R>
void launch_add_r(const ProjBatch& B, dim3 g, bool hw, bool ag, bool wp, size_t smem,
                  const int64_t* clock, int k, cudaStream_t s, int group) {
  if (hw) {
    if (ag) launch_add<R, true, true>(B, g, wp, smem, clock, k, s, group);
    else launch_add<R, true, false>(B, g, wp, smem, clock, k, s, group);
  } else {
    if (ag) launch_add<R, false, true>(B, g, wp, smem, clock, k, s, group);
    else launch_add<R, false, false>(B, g, wp, smem, clock, k, s, group);
  }
}

// ---- on_pre accumulated in the distributed shared memory of thread-block clusters -------
// One L2 atomic per event bounds the scattered delivery at high event rates.  Here every
// cluster of kClusterCtas CTAs holds a private copy of the target variables the batch adds
// into (slots of the padded target population laid end to end, one slice per CTA's shared
// memory), adds its share of the events there (remote shared-memory atomics within the
// cluster), and after a cluster barrier adds its non-zero partial sums to the targets with
// one vector atomic per four elements.  The sums are regrouped (partial sums per cluster),
// so results equal the scattered form's up to rounding.  float32 only.
constexpr int kClusterCtas = 8;

struct ClusterAcc {
  float* slot_ptr[3];            // target array of each slot
  int32_t slot_of_var[3];        // slot of variable v (v, ge, gi), -1 if none
  int32_t n_slots;
  int32_t slice;                 // floats per CTA (a multiple of 4)
  int64_t n;                     // padded target population size (a multiple of 128)
};

template <bool HAS_W, bool WARP_PREFIX, int GROUP>
__global__ void __launch_bounds__(kDeliverBlock)
deliver_cluster_kernel(const __grid_constant__ ProjBatch B,
                       const __grid_constant__ ClusterAcc A, const int64_t* __restrict__ clock,
                       int k, int pref_ints) {
  extern __shared__ __align__(16) float s_dyn[];
  int* s_pref = reinterpret_cast<int*>(s_dyn);
  float* s_acc = s_dyn + pref_ints;          // pref_ints is a multiple of 4
  cg::cluster_group cl = cg::this_cluster();
  const unsigned rank = cl.block_rank();
  for (int i = 4 * threadIdx.x; i < A.slice; i += 4 * blockDim.x)
    *reinterpret_cast<float4*>(s_acc + i) = make_float4(0.f, 0.f, 0.f, 0.f);
  cl.sync();
  const ProjDev& P = B.p[blockIdx.y];
  const int64_t ts = clock[0] + k;
  const float* __restrict__ W = static_cast<const float*>(P.w);
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int glane = (threadIdx.x & 31) % GROUP;
  MemberCache<float> mc;
  for_each_due_item<WARP_PREFIX, GROUP>(P, ts, warp0, nwarps, s_pref,
                                        [&](int64_t b0, int64_t b1, int64_t len, int32_t pre) {
    member_lookup<float>(P, pre, mc);
    const int v = mc.target == P.targets[0] ? 0 : (mc.target == P.targets[1] ? 1 : 2);
    const int64_t base = (int64_t)A.slot_of_var[v] * A.n;
    for (int64_t off = 0; off < len; off += kAddUnroll * GROUP) {
      int32_t post[kAddUnroll];
      float w[kAddUnroll];
      bool ok[kAddUnroll];
#pragma unroll
      for (int u = 0; u < kAddUnroll; ++u) {
        const int64_t s = b0 + off + u * GROUP + glane;
        ok[u] = s < b1;
        post[u] = ok[u] ? __ldg(P.post + s) : 0;
        w[u] = mc.w;
        if constexpr (HAS_W) w[u] = ok[u] ? __ldg(W + s) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < kAddUnroll; ++u) {
        if (!ok[u]) continue;
        const int64_t flat = base + post[u];
        const unsigned r = (unsigned)(flat / A.slice);
        float* dst = cl.map_shared_rank(s_acc, r);
        atomicAdd(dst + (flat - (int64_t)r * A.slice), w[u]);
      }
    }
  });
  cl.sync();
  // this CTA's slice of the cluster's partial sums into the targets
  const int64_t lo = (int64_t)rank * A.slice;
  const int64_t total = (int64_t)A.n_slots * A.n;
  for (int i = 4 * threadIdx.x; i < A.slice; i += 4 * blockDim.x) {
    const int64_t flat = lo + i;
    if (flat >= total) break;
    const float4 x = *reinterpret_cast<const float4*>(s_acc + i);
    if (x.x == 0.f && x.y == 0.f && x.z == 0.f && x.w == 0.f) continue;
    const int slot = (int)(flat / A.n);
    atomicAdd(reinterpret_cast<float4*>(A.slot_ptr[slot] + (flat - (int64_t)slot * A.n)), x);
  }
}

// Whether a batch can accumulate in clusters, and its accumulator layout (slice <= 200 KB).
bool cluster_layout(const Proj* const* prs, int n, ClusterAcc* A) {
  if (prs[0]->dtype != B2B_F32) return false;
  uint8_t mask = 0;
  for (int i = 0; i < n; ++i) {
    if (prs[i]->dst_pop != prs[0]->dst_pop || prs[i]->dev.aggregate) return false;
    mask |= prs[i]->var_mask;
  }
  *A = ClusterAcc{};
  A->n = 0;
  int ns = 0;
  for (int v = 0; v < 3; ++v) {
    A->slot_of_var[v] = -1;
    if (mask & (1u << v)) {
      A->slot_of_var[v] = ns;
      A->slot_ptr[ns] = static_cast<float*>(prs[0]->dev.targets[v]);
      ++ns;
    }
  }
  if (mask & ~7u || ns == 0) return false;
  A->n_slots = ns;
  A->n = prs[0]->dst_n;                     // every projection targets the same population
  const int64_t total = (int64_t)ns * A->n;
  A->slice = (int32_t)(((total + 4 * kClusterCtas - 1) / (4 * kClusterCtas)) * 4);
  return (int64_t)A->slice * 4 <= 200 * 1024;
}

// Clusters of the cluster kernel that are resident together for `smem` bytes per CTA
// (queried once per shared-memory size).
unsigned resident_clusters(const void* kern, size_t smem) {
  static std::mutex mu;
  static std::vector<std::pair<size_t, int>> cache;
  std::lock_guard<std::mutex> lock(mu);
  for (auto& c : cache)
    if (c.first == smem) return (unsigned)c.second;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kClusterCtas * 64);
  cfg.blockDim = dim3(kDeliverBlock);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = kClusterCtas;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess) {
    clusters = 0;
    cudaGetLastError();   // the refusal's error must not be reported by the next launch
  }
  cache.emplace_back(smem, clusters);
  return (unsigned)clusters;
}

template <bool HAS_W, int GROUP>
cudaError_t launch_cluster_g(const ProjBatch& B, const ClusterAcc& A, unsigned clusters,
                             bool wp, int pref_ints, size_t smem, const int64_t* clock, int k,
                             cudaStream_t s, int n) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kClusterCtas * clusters, (unsigned)n);
  cfg.blockDim = dim3(kDeliverBlock);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = kClusterCtas;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  if (wp) {
    auto kern = deliver_cluster_kernel<HAS_W, true, GROUP>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return cudaLaunchKernelEx(&cfg, kern, B, A, clock, k, pref_ints);
  }
  auto kern = deliver_cluster_kernel<HAS_W, false, GROUP>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaLaunchKernelEx(&cfg, kern, B, A, clock, k, pref_ints);
}

template <typename R>
void launch_stdp_pre(const ProjDev& P, unsigned grid, bool ag, bool wp, size_t smem,
                     const int64_t* clock, int k, double dt, cudaStream_t s) {
  if (wp) {
    if (ag) deliver_stdp_pre_kernel<R, true, true><<<grid, kDeliverBlock, 0, s>>>(P, clock, k, dt);
    else deliver_stdp_pre_kernel<R, false, true><<<grid, kDeliverBlock, 0, s>>>(P, clock, k, dt);
  } else {
    if (ag) deliver_stdp_pre_kernel<R, true, false><<<grid, kDeliverBlock, smem, s>>>(P, clock, k, dt);
    else deliver_stdp_pre_kernel<R, false, false><<<grid, kDeliverBlock, smem, s>>>(P, clock, k, dt);
  }
}

}  // namespace

cudaError_t launch_proj_add_batch(const Proj* const* prs, int n, const int64_t* clock, int k,
                                  cudaStream_t s, const AddTune* tune) {
  if (n <= 0 || n > kMaxProjBatch) return cudaErrorInvalidValue;
  ProjBatch B{};
  B.n = n;
  unsigned grid = 1;
  int nd = 1;
  for (int i = 0; i < n; ++i) {
    B.p[i] = prs[i]->dev;
    grid = std::max(grid, deliver_grid(*prs[i]));
    nd = std::max(nd, (int)prs[i]->dev.nd);
  }
  const bool wp = nd <= kWarpPrefixMaxDelays;
  const size_t smem = sizeof(int) * (size_t)(nd + 1);
  const int group = tune && tune->group > 0 ? tune->group : 8;
  ClusterAcc A;
  if (tune && tune->cluster && cluster_layout(prs, n, &A)) {
    const int pref_ints = ((nd + 1 + 3) / 4) * 4;
    const size_t csmem = sizeof(float) * ((size_t)pref_ints + A.slice);
    const unsigned clusters =
        resident_clusters((const void*)deliver_cluster_kernel<false, true, 8>, csmem);
    if (clusters > 0) {
      const bool hw = prs[0]->dev.w != nullptr;
      switch (group) {
        case 4:
          return hw ? launch_cluster_g<true, 4>(B, A, clusters, wp, pref_ints, csmem, clock, k, s, n)
                    : launch_cluster_g<false, 4>(B, A, clusters, wp, pref_ints, csmem, clock, k, s, n);
        case 16:
          return hw ? launch_cluster_g<true, 16>(B, A, clusters, wp, pref_ints, csmem, clock, k, s, n)
                    : launch_cluster_g<false, 16>(B, A, clusters, wp, pref_ints, csmem, clock, k, s, n);
        case 32:
          return hw ? launch_cluster_g<true, 32>(B, A, clusters, wp, pref_ints, csmem, clock, k, s, n)
                    : launch_cluster_g<false, 32>(B, A, clusters, wp, pref_ints, csmem, clock, k, s, n);
        default:
          return hw ? launch_cluster_g<true, 8>(B, A, clusters, wp, pref_ints, csmem, clock, k, s, n)
                    : launch_cluster_g<false, 8>(B, A, clusters, wp, pref_ints, csmem, clock, k, s, n);
      }
    }
  }
  if (tune && tune->grid > 0) grid = (unsigned)tune->grid;
  const dim3 g(grid, (unsigned)n);
  const bool hw = prs[0]->dev.w != nullptr;
  const bool ag = prs[0]->dev.aggregate != 0;
  if (prs[0]->dtype == B2B_F32) launch_add_r<float>(B, g, hw, ag, wp, smem, clock, k, s, group);
  else launch_add_r<double>(B, g, hw, ag, wp, smem, clock, k, s, group);
  return cudaGetLastError();
}

bool add_batch_cluster_capable(const Proj* const* prs, int n) {
  ClusterAcc A;
  return n > 0 && n <= kMaxProjBatch && cluster_layout(prs, n, &A);
}

cudaError_t launch_proj_pre(const Proj& pr, const int64_t* clock, int k, double dt,
                            int32_t* status, cudaStream_t s) {
  (void)status;
  if (pr.effect == B2B_EFFECT_ADD) {
    const Proj* one = &pr;
    return launch_proj_add_batch(&one, 1, clock, k, s);
  }
  if (pr.effect != B2B_EFFECT_STDP) return cudaErrorInvalidValue;
  const ProjDev& P = pr.dev;
  const unsigned grid = deliver_grid(pr);
  const bool wp = P.nd <= kWarpPrefixMaxDelays;
  const size_t smem = sizeof(int) * (size_t)(P.nd + 1);
  const bool ag = P.aggregate != 0;
  if (pr.dtype == B2B_F32) launch_stdp_pre<float>(P, grid, ag, wp, smem, clock, k, dt, s);
  else launch_stdp_pre<double>(P, grid, ag, wp, smem, clock, k, dt, s);
  return cudaGetLastError();
}

cudaError_t launch_proj_post(const Proj& pr, const int64_t* clock, int k, double dt,
                             int32_t* status, cudaStream_t s) {
  (void)status;
  if (pr.effect != B2B_EFFECT_STDP) return cudaSuccess;
  const ProjDev& P = pr.dev;
  int64_t want = (P.post_src_n * (int64_t)P.post_chunks) / 8 + 1;
  const unsigned grid = (unsigned)(want < 2 * kNumSMs ? want : 2 * kNumSMs);
  if (pr.dtype == B2B_F32)
    deliver_stdp_post_kernel<float><<<grid, kDeliverBlock, 0, s>>>(P, clock, k, dt);
  else
    deliver_stdp_post_kernel<double><<<grid, kDeliverBlock, 0, s>>>(P, clock, k, dt);
  return cudaGetLastError();
}

}  // namespace b2b
