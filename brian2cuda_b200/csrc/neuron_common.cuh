// Per-neuron kernel helpers shared by the per-step neuron kernels (neuron.cu) and the
// tensor-core gating-surrogate step (surrogate.cu): vectorised state access, group lookup
// and spike compaction into the spike-history ring.
#pragma once
#include "neuron_math.cuh"

namespace b2b {
namespace {

template <typename R, int E>
struct Pack {
  R x[E];
};

// Loads/stores the E values of thread q from one state array (vectorised for E = 2, 4).
template <typename R, int E>
__device__ __forceinline__ Pack<R, E> load_pack(const void* base, int64_t q) {
  static_assert(E == 1 || E == 2 || E == 4, "neurons per thread");
  Pack<R, E> r;
  if constexpr (E == 1) {
    r.x[0] = static_cast<const R*>(base)[q];
  } else if constexpr (E == 2 && sizeof(R) == 4) {
    float2 a = reinterpret_cast<const float2*>(base)[q];
    r.x[0] = a.x; r.x[1] = a.y;
  } else if constexpr (E == 2) {
    double2 a = reinterpret_cast<const double2*>(base)[q];
    r.x[0] = a.x; r.x[1] = a.y;
  } else if constexpr (sizeof(R) == 4) {
    float4 a = reinterpret_cast<const float4*>(base)[q];
    r.x[0] = a.x; r.x[1] = a.y; r.x[2] = a.z; r.x[3] = a.w;
  } else {
    const double2* p = reinterpret_cast<const double2*>(base) + 2 * q;
    double2 a = p[0], b = p[1];
    r.x[0] = a.x; r.x[1] = a.y; r.x[2] = b.x; r.x[3] = b.y;
  }
  return r;
}

template <typename R, int E>
__device__ __forceinline__ void store_pack(void* base, int64_t q, const Pack<R, E>& r) {
  if constexpr (E == 1) {
    static_cast<R*>(base)[q] = r.x[0];
  } else if constexpr (E == 2 && sizeof(R) == 4) {
    reinterpret_cast<float2*>(base)[q] = make_float2(r.x[0], r.x[1]);
  } else if constexpr (E == 2) {
    reinterpret_cast<double2*>(base)[q] = make_double2(r.x[0], r.x[1]);
  } else if constexpr (sizeof(R) == 4) {
    reinterpret_cast<float4*>(base)[q] = make_float4(r.x[0], r.x[1], r.x[2], r.x[3]);
  } else {
    double2* p = reinterpret_cast<double2*>(base) + 2 * q;
    p[0] = make_double2(r.x[0], r.x[1]);
    p[1] = make_double2(r.x[2], r.x[3]);
  }
}

template <int E>
__device__ __forceinline__ void store_flags(void* base, int64_t q, uint32_t packed) {
  if constexpr (E == 1) static_cast<uint8_t*>(base)[q] = (uint8_t)packed;
  else if constexpr (E == 2) reinterpret_cast<uint16_t*>(base)[q] = (uint16_t)packed;
  else reinterpret_cast<uint32_t*>(base)[q] = packed;
}

// Group-parameter index of thread q (the table holds one entry per 4 neurons).
template <int E>
__device__ __forceinline__ int group_of(const PopDev& P, int64_t q) {
  if (!P.vec_group) return 0;
  return P.vec_group[E == 4 ? q : (E == 2 ? (q >> 1) : (q >> 2))];
}

// Writes the spikes flagged in `fl` (bit e = neuron E*q+e) into the ring slot and the spike
// monitor.  Every thread of the CTA must call this (it synchronises the block).
template <int E>
__device__ __forceinline__ void emit_spikes(const PopDev& P, int64_t q, unsigned fl,
                                            int64_t ts, int slot, int32_t* status) {
  __shared__ int s_warp[33];
  __shared__ int s_base;
  __shared__ unsigned long long s_mbase;
  // most CTAs of most steps have no spike: one barrier decides that for the whole CTA
  if (!__syncthreads_or(fl != 0)) return;
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
  for (int e = 0; e < E; ++e) {
    if (fl & (1u << e)) {
      const int32_t idx = (int32_t)(E * q + e);
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

// emit_spikes for kernels that call it in a loop (hh_stream_kernel): every lane of a warp
// must call this, which synchronises the warp, not the block, so the warps of a CTA are not
// held in step once per iteration.  A warp with spikes reserves its range in the slot (and
// the monitor) with one atomicAdd from its last lane after a warp-wide scan of the counts;
// a warp without spikes returns after one ballot.  The order of spikes within a slot is
// arbitrary (the monitor is read sorted, and delivery sums commute).  One-shot kernels keep
// the block form: at 1e5 neurons a burst step reaches ~3000 warps with spikes, whose
// atomics on the one slot counter would serialise where ~400 CTAs' do not.
template <int E>
__device__ __forceinline__ void emit_spikes_warp(const PopDev& P, int64_t q, unsigned fl,
                                            int64_t ts, int slot, int32_t* status) {
  constexpr unsigned kAll = 0xffffffffu;
  if (!__ballot_sync(kAll, fl != 0)) return;
  const int lane = threadIdx.x & 31;
  const int c = __popc(fl);
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kAll, incl, o);
    if (lane >= o) incl += t;
  }
  const int total = __shfl_sync(kAll, incl, 31);
  int base = 0;
  unsigned long long mbase = 0;
  if (lane == 31) {
    base = atomicAdd(&P.ring_cnt[slot], total);
    if (P.mon_cnt) mbase = atomicAdd(P.mon_cnt, (unsigned long long)total);
  }
  base = __shfl_sync(kAll, base, 31);
  mbase = __shfl_sync(kAll, mbase, 31);
  if (c == 0) return;
  int32_t* out = P.ring_idx + (int64_t)slot * P.n;
  int pos = base + incl - c;
  unsigned long long mpos = P.mon_cnt ? mbase + (unsigned long long)(incl - c) : 0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    if (fl & (1u << e)) {
      const int32_t idx = (int32_t)(E * q + e);
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
// The same from CTA `blk` of the update when the update's CTAs are not the whole grid.
__device__ __forceinline__ void clear_next_slot(const PopDev& P, int64_t ts, int64_t blk) {
  if (blk == 0 && threadIdx.x == 0) P.ring_cnt[ring_slot(ts + 1, P.ring_len)] = 0;
}

}  // namespace
}  // namespace b2b
