#include <algorithm>
// Connectivity build on the GPU (the role of `_before_run_<pathway>_push_spikes`,
// brian2cuda/templates/synapses_push_spikes.cu:171-993, which buckets synapses by (pre,
// post-block), sorts each bucket by delay on the host and copies every bundle with its own
// cudaMemcpy).  Here a stable radix sort keyed by (pre, delay) puts each bundle's synapses
// contiguously, a histogram + exclusive scan gives the bundle offsets, and a scatter writes
// the target indices and weights in bundle order.  Also: Philox-based random connectivity
// (connect(p=...)) and the post-sorted index used by on_post pathways.
#include <cub/cub.cuh>

#include "b2b_build.h"
#include "kernels_common.cuh"
#include "philox.cuh"

namespace b2b {

namespace {

template <typename T>
cudaError_t dmalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

__global__ void keys_kernel(const int32_t* __restrict__ i, const int32_t* __restrict__ d,
                            int64_t n, int32_t pre_lo, int32_t nd, int32_t dmin, int64_t key_base,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                            unsigned long long* __restrict__ counts) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t key = (uint32_t)(i[s] - pre_lo) * (uint32_t)nd + (uint32_t)(d[s] - dmin);
    keys[s] = key;
    vals[s] = (uint32_t)s;
    atomicAdd(&counts[key_base + key], 1ull);
  }
}

template <typename R>
__global__ void scatter_kernel(const uint32_t* __restrict__ vals_sorted, int64_t n,
                               const int64_t* __restrict__ off, int64_t key_base,
                               const int32_t* __restrict__ j, int64_t dst_offset,
                               const R* __restrict__ w_in, int32_t* __restrict__ post,
                               R* __restrict__ w_out, int64_t* __restrict__ inv) {
  const int64_t base = off[key_base];
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t v = vals_sorted[r];
    const int64_t pos = base + r;
    post[pos] = (int32_t)(j[v] + dst_offset);
    if (w_in) w_out[pos] = w_in[v];
    if (inv) inv[v] = pos;
  }
}

template <typename R>
__global__ void fill_kernel(R* a, int64_t n, R v) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x)
    a[r] = v;
}

unsigned grid_for(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g > 8 * kNumSMs) g = 8 * kNumSMs;
  if (g < 1) g = 1;
  return (unsigned)g;
}

int bits_for(uint64_t max_key) {
  int b = 1;
  while (b < 32 && (max_key >> b) != 0) ++b;
  return b;
}

// ---- random connectivity: one warp per presynaptic row ------------------------------------
__global__ void random_count_kernel(int64_t pre_lo, int64_t n_pre, int64_t n_post, uint64_t thr,
                                    uint64_t seed, int64_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t nq = (n_post + 3) >> 2;
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n_pre;
       i += warps) {
    int64_t c = 0;
    for (int64_t jq = lane; jq < nq; jq += 32) {
      unsigned b = connect_bits(seed, (uint32_t)(pre_lo + i), (uint32_t)jq, thr);
      const int64_t valid = n_post - 4 * jq;
      if (valid < 4) b &= (1u << valid) - 1u;
      c += __popc(b);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
    if (lane == 0) counts[i] = c;
  }
}

__global__ void random_fill_kernel(int64_t pre_lo, int64_t n_pre, int64_t n_post, uint64_t thr,
                                   uint64_t seed, int32_t dmin, int32_t nd,
                                   const int64_t* __restrict__ row_off,
                                   int32_t* __restrict__ oi, int32_t* __restrict__ oj,
                                   int32_t* __restrict__ od) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t nq = (n_post + 3) >> 2;
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n_pre;
       i += warps) {
    int64_t pos = row_off[i];
    for (int64_t q0 = 0; q0 < nq; q0 += 32) {
      const int64_t jq = q0 + lane;
      unsigned b = 0;
      if (jq < nq) {
        b = connect_bits(seed, (uint32_t)(pre_lo + i), (uint32_t)jq, thr);
        const int64_t valid = n_post - 4 * jq;
        if (valid < 4) b &= (1u << valid) - 1u;
      }
      const int c = __popc(b);
      int x = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
      }
      int64_t p = pos + (x - c);
      for (int e = 0; e < 4; ++e) {
        if (b & (1u << e)) {
          const uint32_t jj = (uint32_t)(4 * jq + e);
          oi[p] = (int32_t)(pre_lo + i);
          oj[p] = (int32_t)jj;
          od[p] = connect_delay(seed, (uint32_t)(pre_lo + i), jj, dmin, nd);
          ++p;
        }
      }
      pos += __shfl_sync(kFull, x, 31);
    }
  }
}

__global__ void post_keys_kernel(const int32_t* __restrict__ post, int64_t n,
                                 int64_t dst_lo, uint32_t* __restrict__ keys,
                                 uint32_t* __restrict__ vals,
                                 unsigned long long* __restrict__ counts) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t key = (uint32_t)(post[s] - dst_lo);
    keys[s] = key;
    vals[s] = (uint32_t)s;
    atomicAdd(&counts[key], 1ull);
  }
}

// Synapse variable gather in input order.  var: B2B_SYN_*.
template <typename R>
__global__ void gather_kernel(int var, int64_t n, int64_t pos_base, const int64_t* __restrict__ inv,
                              const int64_t* __restrict__ off, int64_t key_lo, int64_t key_hi,
                              int32_t nd, int32_t dmin, int64_t src_offset,
                              const int32_t* __restrict__ post, int64_t dst_offset,
                              const R* __restrict__ arr, int64_t stride,
                              const int32_t* __restrict__ rec, double w_scalar, void* out) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pos = inv ? inv[q] : pos_base + q;
    if (var == B2B_SYN_J) {
      static_cast<int32_t*>(out)[q] = (int32_t)(post[pos] - dst_offset);
    } else if (var == B2B_SYN_I || var == B2B_SYN_DELAY) {
      // largest key in [key_lo, key_hi) with off[key] <= pos
      int64_t lo = key_lo, hi = key_hi - 1;
      while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= pos) lo = mid; else hi = mid - 1;
      }
      const int32_t val = var == B2B_SYN_I ? (int32_t)(lo / nd - src_offset)
                                           : (int32_t)(lo % nd + dmin);
      static_cast<int32_t*>(out)[q] = val;
    } else {
      static_cast<R*>(out)[q] = arr ? arr[(rec ? (int64_t)rec[pos] : pos) * stride] : (R)w_scalar;
    }
  }
}

}  // namespace

cudaError_t member_keys(const int32_t* d_i, const int32_t* d_d, int64_t n, int32_t pre_lo,
                        int32_t nd, int32_t dmin, int64_t key_base, uint32_t* d_keys,
                        uint32_t* d_vals, int64_t* d_counts, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  keys_kernel<<<grid_for(n), 256, 0, s>>>(d_i, d_d, n, pre_lo, nd, dmin, key_base, d_keys, d_vals,
                                          reinterpret_cast<unsigned long long*>(d_counts));
  return cudaGetLastError();
}

cudaError_t counts_to_offsets(int64_t* d_counts, int64_t nkeys, int64_t* max_count,
                              cudaStream_t s) {
  // d_counts has nkeys + 1 entries; afterwards d_counts[k] = first position of key k.
  cudaError_t e;
  int64_t* d_max = nullptr;
  if ((e = dmalloc(&d_max, 1)) != cudaSuccess) return e;
  size_t bytes = 0, bytes2 = 0;
  cub::DeviceReduce::Max(nullptr, bytes, d_counts, d_max, (int)nkeys, s);
  cub::DeviceScan::ExclusiveSum(nullptr, bytes2, d_counts, d_counts, (int)(nkeys + 1), s);
  if (bytes2 > bytes) bytes = bytes2;
  void* tmp = nullptr;
  if ((e = cudaMalloc(&tmp, bytes)) != cudaSuccess) { cudaFree(d_max); return e; }
  cub::DeviceReduce::Max(tmp, bytes, d_counts, d_max, (int)nkeys, s);
  cub::DeviceScan::ExclusiveSum(tmp, bytes, d_counts, d_counts, (int)(nkeys + 1), s);
  e = cudaMemcpyAsync(max_count, d_max, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(tmp);
  cudaFree(d_max);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e;
}

cudaError_t member_sort_scatter(uint32_t* d_keys, uint32_t* d_vals, int64_t n,
                                uint64_t max_key, const int64_t* d_off, int64_t key_base,
                                const int32_t* d_j, int64_t dst_offset, const void* d_w,
                                int dtype, int32_t* d_post, void* d_wout, int64_t* d_inv,
                                cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  cudaError_t e;
  uint32_t *k2 = nullptr, *v2 = nullptr;
  if ((e = dmalloc(&k2, n)) != cudaSuccess) return e;
  if ((e = dmalloc(&v2, n)) != cudaSuccess) { cudaFree(k2); return e; }
  const int end_bit = bits_for(max_key);
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, d_keys, k2, d_vals, v2, (int)n, 0, end_bit, s);
  void* tmp = nullptr;
  e = cudaMalloc(&tmp, bytes);
  if (e == cudaSuccess) {
    cub::DeviceRadixSort::SortPairs(tmp, bytes, d_keys, k2, d_vals, v2, (int)n, 0, end_bit, s);
    if (dtype == B2B_F32)
      scatter_kernel<float><<<grid_for(n), 256, 0, s>>>(v2, n, d_off, key_base, d_j, dst_offset,
                                                        static_cast<const float*>(d_w), d_post,
                                                        static_cast<float*>(d_wout), d_inv);
    else
      scatter_kernel<double><<<grid_for(n), 256, 0, s>>>(v2, n, d_off, key_base, d_j, dst_offset,
                                                         static_cast<const double*>(d_w), d_post,
                                                         static_cast<double*>(d_wout), d_inv);
    e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaFree(tmp);
  }
  cudaFree(k2);
  cudaFree(v2);
  return e;
}

namespace {
// STDP records between synapse order and post-grouped order (record r of the post-grouped
// order is synapse post_syn[r]).
template <typename R>
__global__ void permute_records_kernel(const R* __restrict__ in, R* __restrict__ out,
                                       const int32_t* __restrict__ post_syn, int64_t n,
                                       bool to_post) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = post_syn[r];
    const R* src = in + 4 * (to_post ? s : r);
    R* dst = out + 4 * (to_post ? r : s);
    for (int c = 0; c < 4; ++c) dst[c] = src[c];
  }
}

__global__ void rec_of_kernel(const int32_t* __restrict__ post_syn, int64_t n,
                              int32_t* __restrict__ rec_of) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x)
    rec_of[post_syn[r]] = (int32_t)r;
}
}  // namespace

cudaError_t permute_stdp_records(const void* d_in, void* d_out, const int32_t* d_post_syn,
                                 int64_t n, int dtype, bool to_post, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (dtype == B2B_F32)
    permute_records_kernel<float><<<grid_for(n), 256, 0, s>>>(
        static_cast<const float*>(d_in), static_cast<float*>(d_out), d_post_syn, n, to_post);
  else
    permute_records_kernel<double><<<grid_for(n), 256, 0, s>>>(
        static_cast<const double*>(d_in), static_cast<double*>(d_out), d_post_syn, n, to_post);
  return cudaGetLastError();
}

cudaError_t build_rec_of(const int32_t* d_post_syn, int64_t n, int32_t* d_rec_of,
                         cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  rec_of_kernel<<<grid_for(n), 256, 0, s>>>(d_post_syn, n, d_rec_of);
  return cudaGetLastError();
}

cudaError_t fill_value(void* d, int dtype, int64_t n, double v, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (dtype == B2B_F32) fill_kernel<float><<<grid_for(n), 256, 0, s>>>((float*)d, n, (float)v);
  else fill_kernel<double><<<grid_for(n), 256, 0, s>>>((double*)d, n, v);
  return cudaGetLastError();
}

cudaError_t generate_random_ijd(int64_t pre_lo, int64_t pre_hi, int64_t n_post, double p,
                                int32_t dmin, int32_t dmax, uint64_t seed, int32_t** d_i,
                                int32_t** d_j, int32_t** d_d, int64_t* n_syn, cudaStream_t s) {
  const int64_t n_pre = pre_hi - pre_lo;
  cudaError_t e;
  const uint64_t thr = connect_threshold(p);
  const int32_t nd = dmax - dmin + 1;
  int64_t* row = nullptr;
  if ((e = dmalloc(&row, n_pre + 1)) != cudaSuccess) return e;
  cudaMemsetAsync(row, 0, sizeof(int64_t) * (n_pre + 1), s);
  unsigned grid = (unsigned)((n_pre + 7) / 8);
  if (grid > 16 * kNumSMs) grid = 16 * kNumSMs;
  if (grid < 1) grid = 1;
  random_count_kernel<<<grid, 256, 0, s>>>(pre_lo, n_pre, n_post, thr, seed, row);
  if ((e = cudaGetLastError()) != cudaSuccess) { cudaFree(row); return e; }
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, row, row, (int)(n_pre + 1), s);
  void* tmp = nullptr;
  if ((e = cudaMalloc(&tmp, bytes)) != cudaSuccess) { cudaFree(row); return e; }
  cub::DeviceScan::ExclusiveSum(tmp, bytes, row, row, (int)(n_pre + 1), s);
  int64_t total = 0;
  cudaMemcpyAsync(&total, row + n_pre, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  cudaFree(tmp);
  if (e != cudaSuccess) { cudaFree(row); return e; }
  int32_t *oi = nullptr, *oj = nullptr, *od = nullptr;
  if ((e = dmalloc(&oi, total)) != cudaSuccess) { cudaFree(row); return e; }
  if ((e = dmalloc(&oj, total)) != cudaSuccess) { cudaFree(row); cudaFree(oi); return e; }
  if ((e = dmalloc(&od, total)) != cudaSuccess) {
    cudaFree(row); cudaFree(oi); cudaFree(oj); return e;
  }
  random_fill_kernel<<<grid, 256, 0, s>>>(pre_lo, n_pre, n_post, thr, seed, dmin, nd, row, oi, oj, od);
  e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFree(row);
  if (e != cudaSuccess) { cudaFree(oi); cudaFree(oj); cudaFree(od); return e; }
  *d_i = oi; *d_j = oj; *d_d = od; *n_syn = total;
  return cudaSuccess;
}

cudaError_t build_post_index(const int32_t* d_post, int64_t n_syn, int64_t dst_lo,
                             int64_t n_dst, int64_t* d_post_off, int32_t* d_post_syn,
                             int64_t* max_count, cudaStream_t s) {
  cudaError_t e;
  cudaMemsetAsync(d_post_off, 0, sizeof(int64_t) * (n_dst + 1), s);
  if (n_syn == 0) { *max_count = 0; return cudaStreamSynchronize(s); }
  uint32_t *k1 = nullptr, *v1 = nullptr, *k2 = nullptr;
  if ((e = dmalloc(&k1, n_syn)) != cudaSuccess) return e;
  if ((e = dmalloc(&v1, n_syn)) != cudaSuccess) { cudaFree(k1); return e; }
  if ((e = dmalloc(&k2, n_syn)) != cudaSuccess) { cudaFree(k1); cudaFree(v1); return e; }
  post_keys_kernel<<<grid_for(n_syn), 256, 0, s>>>(d_post, n_syn, dst_lo, k1, v1,
                                                   reinterpret_cast<unsigned long long*>(d_post_off));
  size_t bytes = 0;
  const int end_bit = bits_for((uint64_t)n_dst);
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, k1, k2, v1,
                                  reinterpret_cast<uint32_t*>(d_post_syn), (int)n_syn, 0, end_bit, s);
  void* tmp = nullptr;
  e = cudaMalloc(&tmp, bytes);
  if (e == cudaSuccess) {
    cub::DeviceRadixSort::SortPairs(tmp, bytes, k1, k2, v1,
                                    reinterpret_cast<uint32_t*>(d_post_syn), (int)n_syn, 0,
                                    end_bit, s);
    e = cudaStreamSynchronize(s);
    cudaFree(tmp);
  }
  cudaFree(k1); cudaFree(v1); cudaFree(k2);
  if (e != cudaSuccess) return e;
  return counts_to_offsets(d_post_off, n_dst, max_count, s);
}

cudaError_t gather_syn_var(const Proj& pr, int var, const int64_t* d_inv, int64_t pos_base,
                           int64_t n, int64_t key_lo, int64_t key_hi, int64_t src_offset,
                           int64_t dst_offset, const void* d_arr, int64_t stride,
                           double w_scalar, void* d_out, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  // STDP record components are read through the record order
  const int32_t* rec = stride == 4 ? pr.dev.rec_of : nullptr;
  if (pr.dtype == B2B_F32)
    gather_kernel<float><<<grid_for(n), 256, 0, s>>>(var, n, pos_base, d_inv, pr.off, key_lo,
                                                     key_hi, pr.dmax - pr.dmin + 1, pr.dmin,
                                                     src_offset, pr.post, dst_offset,
                                                     static_cast<const float*>(d_arr),
                                                     stride, rec, w_scalar, d_out);
  else
    gather_kernel<double><<<grid_for(n), 256, 0, s>>>(var, n, pos_base, d_inv, pr.off, key_lo,
                                                      key_hi, pr.dmax - pr.dmin + 1, pr.dmin,
                                                      src_offset, pr.post, dst_offset,
                                                      static_cast<const double*>(d_arr),
                                                      stride, rec, w_scalar, d_out);
  return cudaGetLastError();
}

// Out-degree of neurons [first, first + n) of a projection's source population:
// off[(first + i + 1) * nd] - off[(first + i) * nd] (all delays of neuron first + i), added
// into out[i].
namespace {
__global__ void out_degree_kernel(const int64_t* __restrict__ off, int32_t nd, int64_t first,
                                  int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] += (int32_t)(off[(first + i + 1) * nd] - off[(first + i) * nd]);
}
}  // namespace

cudaError_t add_out_degree(const int64_t* d_off, int32_t nd, int64_t first, int64_t n,
                           int32_t* d_out, cudaStream_t s) {
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096));
  out_degree_kernel<<<(unsigned)blocks, 256, 0, s>>>(d_off, nd, first, n, d_out);
  return cudaGetLastError();
}

// STDP synapse records {w, 0, 0, 0} from the per-synapse initial weights.
namespace {
template <typename R>
__global__ void pack_stdp_kernel(const R* __restrict__ w, R* __restrict__ syn4, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    syn4[4 * i] = w[i];
    syn4[4 * i + 1] = (R)0;
    syn4[4 * i + 2] = (R)0;
    syn4[4 * i + 3] = (R)0;
  }
}
}  // namespace

cudaError_t pack_stdp(const void* d_w, void* d_syn4, int dtype, int64_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8192));
  if (dtype == B2B_F32)
    pack_stdp_kernel<float><<<g, 256, 0, s>>>(static_cast<const float*>(d_w),
                                              static_cast<float*>(d_syn4), n);
  else
    pack_stdp_kernel<double><<<g, 256, 0, s>>>(static_cast<const double*>(d_w),
                                               static_cast<double*>(d_syn4), n);
  return cudaGetLastError();
}

}  // namespace b2b
