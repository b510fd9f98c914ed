// Enumeration of the synapse bundles due at a step, shared by every delivery kernel.
//
// A bundle (pre, d) is due at step ts when pre spiked at step ts - d.  The due work of a
// projection is therefore the spikes of ring slots ts - dmin .. ts - dmin - nd + 1, each
// split into `chunks` work items of up to kChunk synapses.  An item is located by a prefix
// sum over the per-delay spike counts.  With nd <= 64 every warp computes that prefix in two
// registers per lane (two coalesced loads and a warp scan) and finds an item's delay with two
// ballots, so no shared memory or block barrier is involved; larger delay ranges use a
// per-CTA prefix in shared memory.
#pragma once
#include "kernels_common.cuh"

namespace b2b {

constexpr int kWarpPrefixMaxDelays = 64;

// Slot of step (ts - d) given ts's slot, for 0 <= d < ring_len.
__device__ __forceinline__ int ring_back(int base, int d, int ring_len) {
  const int s = base - d;
  return s < 0 ? s + ring_len : s;
}

__device__ __forceinline__ int warp_incl_scan(int x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Per-warp inclusive prefix of the due spike counts of up to 64 delays: lane l holds the
// prefix through delay index l (incl0) and through 32 + l (incl1).
struct DuePrefix {
  int incl0, incl1, total;
};

// Whether the spikes of source step ts - d are delivered: the step exists (>= 0) and lies
// in the projection's source window [lo, hi) (a projection whose delays changed between runs
// delivers the spikes sent before the change through its old bundles, and the later ones
// through its new bundles).
__device__ __forceinline__ bool in_window(int64_t ts, int d, int64_t lo, int64_t hi) {
  const int64_t s = ts - d;
  return s >= 0 && s >= lo && s < hi;
}

__device__ __forceinline__ DuePrefix due_prefix_warp(const int32_t* __restrict__ ring_cnt,
                                                     int ring_len, int64_t ts, int dmin, int nd,
                                                     int64_t lo, int64_t hi) {
  const int lane = threadIdx.x & 31;
  const int base = ring_slot(ts, ring_len);
  int c0 = 0, c1 = 0;
  if (lane < nd && in_window(ts, dmin + lane, lo, hi))
    c0 = ring_cnt[ring_back(base, dmin + lane, ring_len)];
  if (32 + lane < nd && in_window(ts, dmin + 32 + lane, lo, hi))
    c1 = ring_cnt[ring_back(base, dmin + 32 + lane, ring_len)];
  DuePrefix p;
  p.incl0 = warp_incl_scan(c0);
  const int t0 = __shfl_sync(kFull, p.incl0, 31);
  p.incl1 = warp_incl_scan(c1) + t0;
  p.total = __shfl_sync(kFull, p.incl1, 31);
  return p;
}

// Delay index of due spike number sp (0 <= sp < total) and its rank within its slot.
__device__ __forceinline__ int find_delay_warp(const DuePrefix& p, int sp, int* rank) {
  const int di = __popc(__ballot_sync(kFull, p.incl0 <= sp)) +
                 __popc(__ballot_sync(kFull, p.incl1 <= sp));
  const int src = (di - 1) & 31;
  const int v0 = __shfl_sync(kFull, p.incl0, src);
  const int v1 = __shfl_sync(kFull, p.incl1, src);
  const int excl = di == 0 ? 0 : (di - 1 < 32 ? v0 : v1);
  *rank = sp - excl;
  return di;
}

// The same for every lane's own sp at once (lanes may ask for different spikes): the count
// of delay indices whose inclusive prefix is <= sp, found by binary lifting over the 64
// prefix values spread over the warp (lane l holds indices l and 32 + l), 14 shuffles.  Every
// lane of the warp must call this.
__device__ __forceinline__ int find_delay_lane(const DuePrefix& p, int sp, int* rank) {
  int di = 0;
#pragma unroll
  for (int b = 32; b >= 1; b >>= 1) {
    const int probe = di + b - 1;              // is the prefix through index probe <= sp?
    const int a0 = __shfl_sync(kFull, p.incl0, probe & 31);
    const int a1 = __shfl_sync(kFull, p.incl1, probe & 31);
    if ((probe < 32 ? a0 : a1) <= sp) di += b;
  }
  const int src = (di - 1) & 31;
  const int v0 = __shfl_sync(kFull, p.incl0, src);
  const int v1 = __shfl_sync(kFull, p.incl1, src);
  const int excl = di == 0 ? 0 : (di - 1 < 32 ? v0 : v1);
  *rank = sp - excl;
  return di;
}

// Per-CTA prefix in shared memory (any nd): s_pref[0] = 0, s_pref[i] = counts of delay
// indices < i.  Every thread of the CTA must call this.
__device__ __forceinline__ int due_prefix_block(const int32_t* __restrict__ ring_cnt,
                                                int ring_len, int64_t ts, int dmin, int nd,
                                                int64_t lo, int64_t hi, int* s_pref) {
  const int base = ring_slot(ts, ring_len);
  for (int di = threadIdx.x; di < nd; di += blockDim.x)
    s_pref[di + 1] = in_window(ts, dmin + di, lo, hi)
                         ? ring_cnt[ring_back(base, dmin + di, ring_len)] : 0;
  if (threadIdx.x == 0) s_pref[0] = 0;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int carry = 0;
    for (int b0 = 1; b0 <= nd; b0 += 32) {
      const int i = b0 + lane;
      int x = warp_incl_scan(i <= nd ? s_pref[i] : 0);
      if (i <= nd) s_pref[i] = x + carry;
      carry += __shfl_sync(kFull, x, 31);
    }
  }
  __syncthreads();
  return s_pref[nd];
}

__device__ __forceinline__ int find_delay_block(const int* s_pref, int nd, int sp, int* rank) {
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s_pref[mid] <= sp) lo = mid; else hi = mid - 1;
  }
  *rank = sp - s_pref[lo];
  return lo;
}

// Calls item(b0, b1, len, pre) for every work item of projection J due at step ts: the
// synapse positions [b0, b1) of one chunk of the bundle of presynaptic neuron pre (b1 == b0
// for a lane group without an item).  Work items go to warps warp0, warp0 + nwarps, ...;
// inside a warp, groups of GROUP lanes take one item each, so 32/GROUP items' dependent loads
// (spike index, bundle offsets, synapse data) are in flight together.  All 32 lanes of a warp
// call item together; len, the longest b1 - b0 of the warp's groups, is the same in every
// lane.  WARP_PREFIX requires J.nd <= 64; otherwise every thread of the CTA must call this
// (block prefix in s_pref, J.nd + 1 ints).
template <bool WARP_PREFIX, int GROUP = 32, class Item>
__device__ __forceinline__ void for_each_due_item(const ProjDev& J, int64_t ts, int64_t warp0,
                                                  int64_t nwarps, int* s_pref, Item item) {
  static_assert(GROUP == 32 || GROUP == 16 || GROUP == 8 || GROUP == 4 || GROUP == 2,
                "group size");
  constexpr int G = 32 / GROUP;  // items per warp per round
  const int lane = threadIdx.x & 31;
  const int grp = lane / GROUP;
  DuePrefix wp{};
  int nspk;
  if constexpr (WARP_PREFIX) {
    wp = due_prefix_warp(J.src_ring_cnt, J.src_ring_len, ts, J.dmin, J.nd, J.src_lo,
                         J.src_hi);
    nspk = wp.total;
  } else {
    nspk = due_prefix_block(J.src_ring_cnt, J.src_ring_len, ts, J.dmin, J.nd, J.src_lo,
                            J.src_hi, s_pref);
  }
  const int64_t items = (int64_t)nspk * J.chunks;
  const int base = ring_slot(ts, J.src_ring_len);
  for (int64_t r0 = warp0 * G; r0 < items; r0 += nwarps * G) {
    const int64_t it = r0 + grp;
    const bool have = it < items;
    const int sp = have ? (int)(it / J.chunks) : 0;
    const int ch = have ? (int)(it - (int64_t)sp * J.chunks) : 0;
    int kk = 0, di = 0;
    if constexpr (WARP_PREFIX && G >= 4) {
      di = find_delay_lane(wp, sp, &kk);     // one search for all groups of the warp
    } else if constexpr (WARP_PREFIX) {
#pragma unroll
      for (int g = 0; g < G; ++g) {
        int r;
        const int d = find_delay_warp(wp, __shfl_sync(kFull, sp, g * GROUP), &r);
        if (grp == g) { di = d; kk = r; }
      }
    } else {
      di = find_delay_block(s_pref, J.nd, sp, &kk);
    }
    int64_t b0 = 0, b1 = 0;
    int32_t pre = 0;
    if (have) {
      const int slot = ring_back(base, J.dmin + di, J.src_ring_len);
      pre = J.src_ring_idx[(int64_t)slot * J.src_n + kk];
      const int64_t key = (int64_t)pre * J.nd + di;
      b0 = J.off[key] + (int64_t)ch * kChunk;
      b1 = J.off[key + 1];
      if (b1 > b0 + kChunk) b1 = b0 + kChunk;
    }
    // rounds until the longest bundle of this warp's groups is done (warp-uniform)
    int64_t len = b1 - b0;
#pragma unroll
    for (int o = 16; o >= GROUP; o >>= 1) len = max(len, __shfl_xor_sync(kFull, len, o));
    item(b0, b1, len, pre);
  }
}

// Calls body(s, valid, pre) for every synapse position s of every bundle of projection J
// due at step ts, GROUP lanes to a work item (for_each_due_item); all 32 lanes of a warp call
// body together, valid marking real synapses.
template <bool WARP_PREFIX, int GROUP = 32, class Body>
__device__ __forceinline__ void for_each_due(const ProjDev& J, int64_t ts, int64_t warp0,
                                             int64_t nwarps, int* s_pref, Body body) {
  const int glane = (threadIdx.x & 31) % GROUP;
  for_each_due_item<WARP_PREFIX, GROUP>(J, ts, warp0, nwarps, s_pref,
                                        [&](int64_t b0, int64_t b1, int64_t len, int32_t pre) {
    for (int64_t off = 0; off < len; off += GROUP) {
      const int64_t s = b0 + off + glane;
      body(s, s < b1, pre);
    }
  });
}

// Member of presynaptic neuron pre in a projection of several Synapses objects (binary
// search over the members' upper bounds).
__device__ __forceinline__ int member_of(const ProjDev& J, int32_t pre) {
  int lo = 0, hi = J.n_mem - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (pre < J.mem_hi[mid]) hi = mid; else lo = mid + 1;
  }
  return lo;
}

// Target array and scalar weight of presynaptic neuron pre.  A lane keeps its last lookup:
// the synapses a lane visits for one work item share their pre.
template <typename R>
struct MemberCache {
  int32_t pre = -1;
  R* target = nullptr;
  R w = 0;
};

template <typename R>
__device__ __forceinline__ void member_lookup(const ProjDev& J, int32_t pre, MemberCache<R>& c) {
  if (pre == c.pre) return;
  c.pre = pre;
  if (J.n_mem <= 1) {
    c.target = static_cast<R*>(J.target);
    c.w = (R)J.w_scalar;
    return;
  }
  const int m = member_of(J, pre);
  c.target = static_cast<R*>(J.targets[J.mem_var[m]]);
  c.w = J.mem_w ? (R)J.mem_w[m] : (R)J.w_scalar;
}

}  // namespace b2b
