// Connectivity generation into caller-provided device arrays, with no allocation.
//
// The same generator as b2b_synapses_random (Philox-4x32-10 counter-based connect(p) with
// uniform integer delays, philox.cuh), for callers that must not allocate device memory:
// applications whose device memory is owned by a pooling allocator (PyTorch's caching
// allocator, RMM) that a library's own cudaMalloc would bypass and fragment, and host loops
// with latency budgets that the implicit device-wide synchronisation of cudaMalloc/cudaFree
// would break.  Its only scratch — the per-row synapse counts and their prefix sum — lives
// in a file-scope __device__ array of B2B_STATIC_MAX_ROWS + 1 int64 entries (8 MiB), which
// every GPU that loads the library holds until exit.  All calls share that array, so calls
// that overlap on the GPU (different streams, or different host threads) race; each call
// writes every entry it reads before reading it.
//
// The device address of the array is looked up with cudaGetSymbolAddress once per device
// and CUDA context: the lookup is repeated when the device's current context is another
// one than at the last lookup (after cudaDeviceReset, or a primary context released and
// created again), so a cached address never outlives the context it belongs to.
#include <cuda_runtime.h>

#include <mutex>

#include "kernels_common.cuh"
#include "philox.cuh"

namespace b2b {
namespace {

constexpr int kMaxDevices = 64;

// Per-row synapse counts, then their exclusive prefix (entry `rows` = total).
__device__ __align__(256) int64_t g_row_scratch[B2B_STATIC_MAX_ROWS + 1];

std::mutex g_setup_mutex;
int64_t* g_scratch_addr[kMaxDevices] = {};
void* g_scratch_ctx[kMaxDevices] = {};

// cuCtxGetCurrent, fetched through the runtime so that the library needs no link against
// the driver library (the CPU-only test machines load it without a driver).
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn g_ctx_get_current = nullptr;

__global__ void static_count_kernel(int64_t pre_lo, int64_t rows, int64_t n_post, uint64_t thr,
                                    uint64_t seed, int64_t* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t nq = (n_post + 3) >> 2;
  if (blockIdx.x == 0 && threadIdx.x == 0) counts[rows] = 0;
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < rows;
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

// Exclusive scan of n entries in place with one CTA: each thread scans a contiguous chunk.
__global__ void static_scan_kernel(int64_t* __restrict__ a, int64_t n) {
  __shared__ int64_t s_tot[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const int64_t per = (n + T - 1) / T;
  const int64_t lo = t * per, hi = lo + per < n ? lo + per : n;
  int64_t sum = 0;
  for (int64_t i = lo; i < hi; ++i) sum += a[i];
  s_tot[t] = sum;
  __syncthreads();
  if (t == 0) {
    int64_t run = 0;
    for (int k = 0; k < T; ++k) {
      const int64_t x = s_tot[k];
      s_tot[k] = run;
      run += x;
    }
  }
  __syncthreads();
  int64_t run = s_tot[t];
  for (int64_t i = lo; i < hi; ++i) {
    const int64_t x = a[i];
    a[i] = run;
    run += x;
  }
}

__global__ void static_fill_kernel(int64_t pre_lo, int64_t rows, int64_t n_post, uint64_t thr,
                                   uint64_t seed, int32_t dmin, int32_t nd,
                                   const int64_t* __restrict__ row_off, int64_t capacity,
                                   int32_t* __restrict__ oi, int32_t* __restrict__ oj,
                                   int32_t* __restrict__ od) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t nq = (n_post + 3) >> 2;
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < rows;
       i += warps) {
    int64_t pos = row_off[i];
    if (pos >= capacity) continue;
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
        if (!(b & (1u << e))) continue;
        if (p < capacity) {
          const uint32_t jj = (uint32_t)(4 * jq + e);
          oi[p] = (int32_t)(pre_lo + i);
          oj[p] = (int32_t)jj;
          od[p] = connect_delay(seed, (uint32_t)(pre_lo + i), jj, dmin, nd);
        }
        ++p;
      }
      pos += __shfl_sync(kFull, x, 31);
    }
  }
}

// Device address of the scratch array on `device` (the current device, whose primary
// context cudaSetDevice has made current), looked up once per device and context.
cudaError_t scratch_for(int device, int64_t** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  cudaError_t e = cudaSuccess;
  if (!g_ctx_get_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
  }
  void* ctx = nullptr;
  if (g_ctx_get_current(&ctx) != 0 || !ctx) return cudaErrorDeviceUninitialized;
  if (!g_scratch_addr[device] || g_scratch_ctx[device] != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_row_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<int64_t*>(p);
    g_scratch_ctx[device] = ctx;
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

}  // namespace
}  // namespace b2b

using namespace b2b;

extern "C" b2b_status b2b_connect_random_static(int32_t device, void* stream, int32_t pre_lo,
                                                int32_t pre_hi, int32_t n_post, double p,
                                                int32_t dmin, int32_t dmax, uint64_t seed,
                                                int32_t* dev_i, int32_t* dev_j,
                                                int32_t* dev_delay, int64_t capacity,
                                                int64_t* n_syn) {
  if (!dev_i || !dev_j || !dev_delay || !n_syn || capacity < 0) return B2B_ERR_INVALID_ARG;
  if (device < 0 || device >= kMaxDevices) return B2B_ERR_INVALID_ARG;
  if (pre_lo < 0 || pre_hi <= pre_lo || n_post <= 0 || !(p >= 0 && p <= 1) || dmin < 0 ||
      dmax < dmin)
    return B2B_ERR_INVALID_ARG;
  if ((int64_t)pre_hi - pre_lo > B2B_STATIC_MAX_ROWS) return B2B_ERR_INVALID_ARG;
  // An error left pending by earlier work of the caller is reported as it is and not
  // consumed: a launch error of this call must not be confused with it.
  if (cudaPeekAtLastError() != cudaSuccess) return B2B_ERR_CUDA;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return B2B_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return B2B_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t rows = (int64_t)pre_hi - pre_lo;
  const uint64_t thr = connect_threshold(p);
  int64_t* row = nullptr;
  int64_t total = 0;
  cudaError_t e = scratch_for(device, &row);
  if (e == cudaSuccess) {
    int64_t grid = (rows + 7) / 8;
    if (grid > 16 * kNumSMs) grid = 16 * kNumSMs;
    static_count_kernel<<<(unsigned)grid, 256, 0, s>>>(pre_lo, rows, n_post, thr, seed, row);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    static_scan_kernel<<<1, 1024, 0, s>>>(row, rows + 1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    int64_t grid = (rows + 7) / 8;
    if (grid > 16 * kNumSMs) grid = 16 * kNumSMs;
    static_fill_kernel<<<(unsigned)grid, 256, 0, s>>>(pre_lo, rows, n_post, thr, seed, dmin,
                                                      dmax - dmin + 1, row, capacity, dev_i,
                                                      dev_j, dev_delay);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&total, row + rows, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaSetDevice(prev);
  if (e != cudaSuccess) return B2B_ERR_CUDA;
  *n_syn = total;
  return total > capacity ? B2B_ERR_QUEUE_OVERFLOW : B2B_OK;
}
