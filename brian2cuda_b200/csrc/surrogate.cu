// Gating surrogate for the COBAHH neuron: a 4 -> 64 -> 64 -> 3 multilayer perceptron that
// predicts the exponential-Euler step of the Hodgkin-Huxley gating variables (m, h, n) over
// one dt from (v, m, h, n), with BF16 weights and activations and FP32 accumulation on the
// sm_100a tensor cores (tcgen05.mma, accumulators in TMEM).  No counterpart in the
// reference: brian2cuda integrates the gates with the code Brian2 generates for
// `method='exponential_euler'` (examples/cobahh.py:159-180), which stays the fallback here
// and the judge of the surrogate's error.
//
// Network (per sample):
//   xh = ((v, m, h, n) - shift) * scale, xh[4] = 1 (carries the first bias), xh[5..15] = 0
//   h1 = tanh(W1 xh)            (64, bf16)      z in fp32, rounded to bf16, then tanh
//   h2 = tanh(W2 h1 + b2)       (64, bf16)
//   y  = W3 h2 + b3             (3, fp32)
//   (m, h, n)' = clip((m, h, n) + out_scale * y, 0, 1)
// Training minimises mean_s sum_o (y_o - (t_o - x_o)/out_scale_o)^2 with Adam on fp32 master
// weights; every product runs on the tensor cores (forward, backward and the weight
// gradients, the latter accumulated in TMEM across all tiles of a CTA).
//
// Tiles are 128 samples (one per thread of a 128-thread CTA, the MMA's M = 128 rows in
// TMEM lanes).  Operands in shared memory use the group-major layout of tc_sm100.cuh with
// R = 128 rows for activations and gradients; the weight images are packed once per update
// into global memory in the same layout and copied into each CTA's shared memory.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "b2b_internal.h"
#include "neuron_common.cuh"
#include "tc_sm100.cuh"

namespace b2b {
namespace {

using namespace tc;

constexpr int kHid = 64;
constexpr int kIn = 4;
constexpr int kOut = 3;
constexpr int kTile = 128;               // samples per tile = threads per CTA
constexpr uint32_t kWaitLimit = 1u << 20; // polls of an mbarrier before giving up

// Offsets of the fp32 master parameters (PyTorch nn.Linear order: weight [out][in], bias).
constexpr int kW1 = 0, kB1 = kW1 + kHid * kIn, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid,
              kW3 = kB2 + kHid, kB3 = kW3 + kOut * kHid, kNParams = kB3 + kOut;
static_assert(kNParams == B2B_MLP_NPARAMS, "parameter count");

// Packed device image.  The first part (the forward operands, biases, scaling) is what the
// inference kernels copy to shared memory; the transposed images follow for the backward.
struct MlpImage {
  uint16_t B1[kHid * 16];   // N = 64 x K = 16: W1 | b1 | 0
  uint16_t B2[kHid * kHid]; // N = 64 x K = 64
  uint16_t B3[16 * kHid];   // N = 16 x K = 64: W3 rows, zero rows 3..15
  float b2[kHid];
  float b3[16];
  float in_shift[4], in_scale[4], out_scale[4];
  uint16_t B3T[kHid * 16];  // N = 64 x K = 16: W3^T | 0
  uint16_t B2T[kHid * kHid];// N = 64 x K = 64: W2^T
};
constexpr uint32_t kFwdBytes = offsetof(MlpImage, B3T);
static_assert(kFwdBytes % 16 == 0 && sizeof(MlpImage) % 16 == 0, "16-byte copies");
static_assert(offsetof(MlpImage, B2) % 16 == 0 && offsetof(MlpImage, B3) % 16 == 0 &&
                  offsetof(MlpImage, b2) % 16 == 0 && offsetof(MlpImage, B2T) % 16 == 0,
              "operand alignment");

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<uint16_t*>(&h);
}

// Index (in uint16 elements) of (r, k) in a group-major operand with R rows.
__device__ __forceinline__ uint32_t gm_idx(uint32_t R, uint32_t r, uint32_t k) {
  return gm_offset(R, r, k) >> 1;
}

// Writes the bf16 operand images of the master parameters p (called by one whole CTA).
__device__ void pack_image(const float* __restrict__ p, const float* __restrict__ scaling,
                           MlpImage* __restrict__ img) {
  for (int t = threadIdx.x; t < kHid * 16; t += blockDim.x) {
    const int o = t / 16, k = t % 16;
    const float w = k < kIn ? p[kW1 + o * kIn + k] : (k == kIn ? p[kB1 + o] : 0.f);
    img->B1[gm_idx(kHid, o, k)] = bf16_bits(w);
  }
  for (int t = threadIdx.x; t < kHid * kHid; t += blockDim.x) {
    const int o = t / kHid, i = t % kHid;
    const uint16_t w = bf16_bits(p[kW2 + o * kHid + i]);
    img->B2[gm_idx(kHid, o, i)] = w;
    img->B2T[gm_idx(kHid, i, o)] = w;
  }
  for (int t = threadIdx.x; t < 16 * kHid; t += blockDim.x) {
    const int o = t / kHid, j = t % kHid;
    const uint16_t w = o < kOut ? bf16_bits(p[kW3 + o * kHid + j]) : (uint16_t)0;
    img->B3[gm_idx(16, o, j)] = w;
    img->B3T[gm_idx(kHid, j, o)] = w;
  }
  for (int t = threadIdx.x; t < kHid; t += blockDim.x) img->b2[t] = p[kB2 + t];
  for (int t = threadIdx.x; t < 16; t += blockDim.x) img->b3[t] = t < kOut ? p[kB3 + t] : 0.f;
  for (int t = threadIdx.x; t < 4; t += blockDim.x) {
    img->in_shift[t] = scaling[t];
    img->in_scale[t] = scaling[4 + t];
    img->out_scale[t] = t < kOut ? scaling[8 + t] : 0.f;
  }
}

__global__ void mlp_pack_kernel(const float* __restrict__ p, const float* __restrict__ scaling,
                                MlpImage* __restrict__ img) {
  pack_image(p, scaling, img);
}

// Copies `bytes` (multiple of 16) from global to shared memory with the whole CTA.
__device__ __forceinline__ void copy_to_smem(void* dst, const void* src, uint32_t bytes) {
  const int4* s = static_cast<const int4*>(src);
  int4* d = static_cast<int4*>(dst);
  for (uint32_t i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = s[i];
}

// Bounded wait on the CTA's MMA barrier; a CTA whose wait gave up records B2B_ERR_TIMEOUT.
// Returns the CTA-uniform outcome, so every thread leaves a tile loop together.
__device__ __forceinline__ bool wait_mma(uint64_t* bar, uint32_t& phase, int32_t* status) {
  const bool ok = mbar_wait(bar, phase, kWaitLimit);
  phase ^= 1u;
  const bool all_ok = !__syncthreads_or(!ok);
  if (!all_ok && threadIdx.x == 0) set_status(status, B2B_ERR_TIMEOUT);
  fence_after_sync();
  return all_ok;
}

// Makes this thread's shared-memory operand writes visible to the tensor core and orders its
// earlier TMEM loads before the MMAs that thread 0 issues next.
__device__ __forceinline__ void operands_ready() {
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
}

// Writes 64 bf16 values (32 packed pairs) as row r of a group-major R = 128 operand.
__device__ __forceinline__ void store_row64(uint8_t* base, int r, const uint32_t (&hp)[32]) {
#pragma unroll
  for (int g = 0; g < 8; ++g)
    *reinterpret_cast<uint4*>(base + gm_offset(kTile, r, 8 * g)) =
        make_uint4(hp[4 * g], hp[4 * g + 1], hp[4 * g + 2], hp[4 * g + 3]);
}

// Row r of a 16-wide operand: values v0..v3 in columns 0..3, c4 in column 4, zeros after.
__device__ __forceinline__ void store_row16(uint8_t* base, int r, float v0, float v1, float v2,
                                            float v3, float c4) {
  *reinterpret_cast<uint4*>(base + gm_offset(kTile, r, 0)) =
      make_uint4(pack_bf16x2(v0, v1), pack_bf16x2(v2, v3), pack_bf16x2(c4, 0.f), 0u);
  *reinterpret_cast<uint4*>(base + gm_offset(kTile, r, 8)) = make_uint4(0u, 0u, 0u, 0u);
}

// Loads 64 accumulator columns of this thread's row, adds bias (or nothing) and applies
// tanh in bf16: hp receives the 64 activations as packed bf16 pairs.
__device__ __forceinline__ void epilogue_tanh64(uint32_t taddr, const float* bias,
                                                uint32_t (&hp)[32]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    float v[16];
    tmem_ld16(taddr + 16 * c, v);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      float a = v[2 * i], b = v[2 * i + 1];
      if (bias) {
        a += bias[16 * c + 2 * i];
        b += bias[16 * c + 2 * i + 1];
      }
      hp[8 * c + i] = tanh_bf16x2(pack_bf16x2(a, b));
    }
  }
}

constexpr uint32_t kG = kTile * 16;      // bytes of one 8-column group of an R = 128 operand

// Shared memory of the inference kernels (one 128-sample tile at a time).
struct FwdSmem {
  alignas(128) uint8_t img[kFwdBytes];
  alignas(128) uint8_t X[2 * kG];        // inputs, K = 16
  alignas(128) uint8_t H[8 * kG];        // hidden activations, K = 64 (h1, then h2)
  uint64_t bar;
  uint32_t tmem;
};

__device__ __forceinline__ const MlpImage* image_of(const FwdSmem& S) {
  return reinterpret_cast<const MlpImage*>(S.img);
}

// Prologue of the inference kernels: weights to shared memory, barrier, 64 TMEM columns.
__device__ __forceinline__ void fwd_setup(FwdSmem& S, const MlpImage* img) {
  copy_to_smem(S.img, img, kFwdBytes);
  if (threadIdx.x == 0) {
    mbar_init(&S.bar, 1);
    fence_mbar_init();
  }
  if (threadIdx.x < 32) {
    tmem_alloc(&S.tmem, 64);
    tmem_relinquish();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
}

__device__ __forceinline__ void fwd_teardown(FwdSmem& S) {
  fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) {
    fence_after_sync();
    tmem_dealloc(S.tmem, 64);
  }
}

// Normalised network input of (v, m, h, n).
__device__ __forceinline__ void normalise(const MlpImage* I, float v, float m, float h, float n,
                                          float (&xh)[4]) {
  xh[0] = (v - I->in_shift[0]) * I->in_scale[0];
  xh[1] = (m - I->in_shift[1]) * I->in_scale[1];
  xh[2] = (h - I->in_shift[2]) * I->in_scale[2];
  xh[3] = (n - I->in_shift[3]) * I->in_scale[3];
}

// Forward pass of one tile; thread r supplies row r's input and receives its 3 outputs.
// Every thread of the CTA calls it.  Returns false (CTA-uniformly) if an MMA wait gave up.
__device__ bool mlp_tile_forward(FwdSmem& S, uint32_t& phase, const float (&xh)[4],
                                 float (&y)[3], int32_t* status) {
  const int r = threadIdx.x;
  const MlpImage* I = image_of(S);
  const uint32_t tmem = S.tmem;
  const uint32_t taddr = tmem + tmem_lane_base();
  const uint32_t id64 = idesc_bf16(128, 64, false, false);
  const uint32_t id16 = idesc_bf16(128, 16, false, false);
  const uint32_t sX = smem_u32(S.X), sH = smem_u32(S.H);
  const uint32_t sB1 = smem_u32(I->B1), sB2 = smem_u32(I->B2), sB3 = smem_u32(I->B3);

  store_row16(S.X, r, xh[0], xh[1], xh[2], xh[3], 1.f);
  operands_ready();
  if (r == 0) {
    fence_after_sync();
    mma_bf16(tmem, sdesc(sX, kG, 128), sdesc(sB1, kHid * 16, 128), id64, 0u);
    mma_commit(&S.bar);
  }
  if (!wait_mma(&S.bar, phase, status)) return false;
  uint32_t hp[32];
  epilogue_tanh64(taddr, nullptr, hp);
  store_row64(S.H, r, hp);
  operands_ready();
  if (r == 0) {
    fence_after_sync();
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      mma_bf16(tmem, sdesc(sH + kk * 2 * kG, kG, 128), sdesc(sB2 + kk * 2 * kHid * 16, kHid * 16, 128),
               id64, kk > 0);
    mma_commit(&S.bar);
  }
  if (!wait_mma(&S.bar, phase, status)) return false;
  epilogue_tanh64(taddr, I->b2, hp);
  store_row64(S.H, r, hp);
  operands_ready();
  if (r == 0) {
    fence_after_sync();
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      mma_bf16(tmem, sdesc(sH + kk * 2 * kG, kG, 128), sdesc(sB3 + kk * 2 * 16 * 16, 16 * 16, 128),
               id16, kk > 0);
    mma_commit(&S.bar);
  }
  if (!wait_mma(&S.bar, phase, status)) return false;
  float v[16];
  tmem_ld16(taddr, v);
  y[0] = v[0] + I->b3[0];
  y[1] = v[1] + I->b3[1];
  y[2] = v[2] + I->b3[2];
  fence_before_sync();
  return true;
}

// Network outputs (raw = 1) or predicted gating values (raw = 0) for n samples.
__global__ void __launch_bounds__(kTile)
mlp_forward_kernel(const MlpImage* __restrict__ img, const float4* __restrict__ x,
                   float* __restrict__ out, int64_t n, int raw, int32_t* status) {
  __shared__ FwdSmem S;
  fwd_setup(S, img);
  const MlpImage* I = image_of(S);
  uint32_t phase = 0;
  const int64_t ntiles = (n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t i = tile * kTile + threadIdx.x;
    const float4 s = i < n ? x[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    float xh[4], y[3];
    normalise(I, s.x, s.y, s.z, s.w, xh);
    if (!mlp_tile_forward(S, phase, xh, y, status)) break;
    if (i < n) {
      if (raw) {
        out[3 * i] = y[0]; out[3 * i + 1] = y[1]; out[3 * i + 2] = y[2];
      } else {
        out[3 * i] = dclip(s.y + I->out_scale[0] * y[0], 0.f, 1.f);
        out[3 * i + 1] = dclip(s.z + I->out_scale[1] * y[1], 0.f, 1.f);
        out[3 * i + 2] = dclip(s.w + I->out_scale[2] * y[2], 0.f, 1.f);
      }
    }
  }
  fwd_teardown(S);
}

// ---- COBAHH step with surrogate gating ---------------------------------------------------
// Device view of a population's surrogate (one per HH float32 population).
struct SurrDev {
  const MlpImage* img;
  unsigned long long* counters;   // [0] neuron-updates, [1] exact fallbacks
  float tol;                      // largest accepted |surrogate - exact| per gate
  float vmax_hat;                 // |normalised v| beyond which the input is out of range
  int32_t judge;                  // 1: compare every step with the exact update
  int32_t pad;
};

// hh_step_kernel (neuron.cu) with the gating step predicted by the MLP: one thread per
// neuron, 128-neuron tiles, persistent over the population.  The membrane update uses the
// gating state at the start of the step, as the exact kernel does.  A neuron is re-stepped
// exactly when its normalised v lies outside the training range or, with `judge`, when a
// predicted gate differs from the exact exponential-Euler value by more than `tol`.
__global__ void __launch_bounds__(kTile, 6)
hh_surrogate_step_kernel(PopDev P, SurrDev D, const int64_t* __restrict__ clock, int k,
                         double dt, int32_t* status) {
  __shared__ FwdSmem S;
  fwd_setup(S, D.img);
  const MlpImage* I = image_of(S);
  const int64_t ts = clock[0] + k;
  const double t = (double)ts * dt;
  const double inv_dt = 1.0 / dt;
  const int slot = ring_slot(ts, P.ring_len);
  const float dtR = (float)dt;
  const HhDev* prm = static_cast<const HhDev*>(P.params);
  float* Vv = static_cast<float*>(P.var[B2B_VAR_V]);
  float* Mv = static_cast<float*>(P.var[B2B_VAR_M]);
  float* Hv = static_cast<float*>(P.var[B2B_VAR_H]);
  float* Nv = static_cast<float*>(P.var[B2B_VAR_N]);
  float* GEv = static_cast<float*>(P.var[B2B_VAR_GE]);
  float* GIv = static_cast<float*>(P.var[B2B_VAR_GI]);
  float* LSv = static_cast<float*>(P.var[B2B_VAR_LASTSPIKE]);
  uint8_t* NRv = static_cast<uint8_t*>(P.var[B2B_VAR_NOT_REFRACTORY]);
  uint32_t phase = 0;
  unsigned long long n_upd = 0, n_fb = 0;
  const int64_t ntiles = P.n / kTile;   // populations are padded to a multiple of 128
  const int64_t tstride = (int64_t)gridDim.x * kTile;
  int64_t tile = blockIdx.x;
  float v = 0.f, m = 0.f, h = 0.f, n = 0.f, ge = 0.f, gi = 0.f, ls = 0.f;
  if (tile < ntiles) {
    const int64_t q = tile * kTile + threadIdx.x;
    v = Vv[q]; m = Mv[q]; h = Hv[q]; n = Nv[q]; ge = GEv[q]; gi = GIv[q]; ls = LSv[q];
  }
  for (; tile < ntiles; tile += gridDim.x) {
    const int64_t q = tile * kTile + threadIdx.x;
    float xh[4], y[3];
    normalise(I, v, m, h, n, xh);
    // the next tile's state loads are in flight during this tile's tensor-core chain
    float nv = 0.f, nm = 0.f, nh = 0.f, nn_ = 0.f, nge = 0.f, ngi = 0.f, nls = 0.f;
    if (tile + gridDim.x < ntiles) {
      const int64_t qn = q + tstride;
      nv = Vv[qn]; nm = Mv[qn]; nh = Hv[qn]; nn_ = Nv[qn]; nge = GEv[qn]; ngi = GIv[qn];
      nls = LSv[qn];
    }
    if (!mlp_tile_forward(S, phase, xh, y, status)) break;
    const HhRun<float> g = hh_run(prm[group_of<1>(P, q)], 0.f);
    const bool refr = g.ref_steps >= 0;
    float mn = dclip(m + I->out_scale[0] * y[0], 0.f, 1.f);
    float hn = dclip(h + I->out_scale[1] * y[1], 0.f, 1.f);
    float nn = dclip(n + I->out_scale[2] * y[2], 0.f, 1.f);
    bool exact = !(fabsf(xh[0]) <= D.vmax_hat);
    if (D.judge || exact) {
      float me = m, he = h, ne = n;
      hh_gating<float>((float)g.VT, v, me, he, ne, dtR);
      const float err = fmaxf(fabsf(mn - me), fmaxf(fabsf(hn - he), fabsf(nn - ne)));
      if (exact || !(err <= D.tol)) {
        exact = true;
        mn = me; hn = he; nn = ne;
      }
    }
    const bool valid = (q - g.offset) < g.n;
    const unsigned vb = __ballot_sync(kFull, valid), fb = __ballot_sync(kFull, valid && exact);
    if ((threadIdx.x & 31) == 0) {
      n_upd += __popc(vb);
      n_fb += __popc(fb);
    }
    bool nr = true;
    if (refr) nr = past_refractory(t - (double)ls, dt, inv_dt, g.ref_steps);
    const float vn = hh_membrane<float>(g, v, m, h, n, ge, gi, dtR);
    unsigned fl = 0;
    if (valid && vn > (float)g.Vthr && nr) {
      nr = false;
      ls = (float)t;
      fl = 1u;
    }
    Vv[q] = vn;
    Mv[q] = mn;
    Hv[q] = hn;
    Nv[q] = nn;
    GEv[q] = (float)g.De * ge;
    GIv[q] = (float)g.Di * gi;
    if (refr) {
      LSv[q] = ls;
      NRv[q] = nr ? 1 : 0;
    }
    emit_spikes<1>(P, q, fl, ts, slot, status);
    v = nv; m = nm; h = nh; n = nn_; ge = nge; gi = ngi; ls = nls;
  }
  clear_next_slot(P, ts);
  if ((threadIdx.x & 31) == 0 && D.counters) {
    atomicAdd(&D.counters[0], n_upd);
    atomicAdd(&D.counters[1], n_fb);
  }
  fwd_teardown(S);
}

// ---- training --------------------------------------------------------------------------
// Shared memory of the gradient kernel.  FS stacks the tile's features as 18 column groups
// (x: 0-1, h1: 2-9, h2: 10-17), GS the gradients (dz1: 0-7, dz2: 8-15, dy: 16-17), so that
// the weight-gradient products read contiguous 128-feature slices of them MN-major.
struct TrainSmem {
  alignas(128) MlpImage img;
  alignas(128) uint8_t FS[18 * kG];
  alignas(128) uint8_t GS[18 * kG];
  uint64_t bar;
  uint32_t tmem;
};
constexpr uint32_t kColS = 0, kColA = 64, kColB = 208, kTrainCols = 512;
constexpr int kNA = 144, kNB = 80;   // columns of the two weight-gradient accumulators

// Gradient of the mean loss over samples [mb_start, mb_start + mb_n) of the (permuted)
// dataset; adds into grad (fp32, parameter order) and the summed squared error into *loss.
// Sample s of the minibatch is dataset row (a * (mb_start + s) + c) mod n.
__global__ void __launch_bounds__(kTile)
mlp_grad_kernel(const MlpImage* __restrict__ img, const float4* __restrict__ x,
                const float* __restrict__ tgt, int64_t n, int64_t mb_start, int64_t mb_n,
                int64_t pa, int64_t pc, float inv_batch, float* __restrict__ grad,
                double* __restrict__ loss, int32_t* status) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
  copy_to_smem(&S.img, img, sizeof(MlpImage));
  if (threadIdx.x == 0) {
    mbar_init(&S.bar, 1);
    fence_mbar_init();
  }
  if (threadIdx.x < 32) {
    tmem_alloc(&S.tmem, kTrainCols);
    tmem_relinquish();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const MlpImage* I = &S.img;
  const int r = threadIdx.x;
  const uint32_t tmem = S.tmem;
  const uint32_t taddr = tmem + tmem_lane_base();
  const uint32_t sFS = smem_u32(S.FS), sGS = smem_u32(S.GS);
  const uint32_t id64 = idesc_bf16(128, 64, false, false);
  const uint32_t id16 = idesc_bf16(128, 16, false, false);
  const uint32_t idA = idesc_bf16(128, kNA, true, true);
  const uint32_t idB = idesc_bf16(128, kNB, true, true);
  uint32_t phase = 0;
  float sq = 0.f;
  bool ok = true;
  int tiles_done = 0;
  const int64_t ntiles = (mb_n + kTile - 1) / kTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t pos = tile * kTile + r;
    const bool valid = pos < mb_n;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    float t0 = 0.f, t1 = 0.f, t2 = 0.f;
    if (valid) {
      const int64_t row = (int64_t)(((unsigned long long)pa * (unsigned long long)(mb_start + pos) +
                                     (unsigned long long)pc) % (unsigned long long)n);
      s = x[row];
      t0 = tgt[3 * row]; t1 = tgt[3 * row + 1]; t2 = tgt[3 * row + 2];
    }
    float xh[4];
    normalise(I, s.x, s.y, s.z, s.w, xh);
    // forward
    store_row16(S.FS, r, xh[0], xh[1], xh[2], xh[3], 1.f);
    operands_ready();
    if (r == 0) {
      fence_after_sync();
      mma_bf16(tmem + kColS, sdesc(sFS, kG, 128), sdesc(smem_u32(I->B1), kHid * 16, 128), id64, 0u);
      mma_commit(&S.bar);
    }
    if (!(ok = wait_mma(&S.bar, phase, status))) break;
    uint32_t h1[32], h2[32];
    epilogue_tanh64(taddr + kColS, nullptr, h1);
    store_row64(S.FS + 2 * kG, r, h1);
    operands_ready();
    if (r == 0) {
      fence_after_sync();
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma_bf16(tmem + kColS, sdesc(sFS + (2 + 2 * kk) * kG, kG, 128),
                 sdesc(smem_u32(I->B2) + kk * 2 * kHid * 16, kHid * 16, 128), id64, kk > 0);
      mma_commit(&S.bar);
    }
    if (!(ok = wait_mma(&S.bar, phase, status))) break;
    epilogue_tanh64(taddr + kColS, I->b2, h2);
    store_row64(S.FS + 10 * kG, r, h2);
    operands_ready();
    if (r == 0) {
      fence_after_sync();
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma_bf16(tmem + kColS, sdesc(sFS + (10 + 2 * kk) * kG, kG, 128),
                 sdesc(smem_u32(I->B3) + kk * 2 * 16 * 16, 16 * 16, 128), id16, kk > 0);
      mma_commit(&S.bar);
    }
    if (!(ok = wait_mma(&S.bar, phase, status))) break;
    float v[16];
    tmem_ld16(taddr + kColS, v);
    // loss and output gradient
    float d0 = 0.f, d1 = 0.f, d2 = 0.f;
    if (valid) {
      const float e0 = v[0] + I->b3[0] - (t0 - s.y) / I->out_scale[0];
      const float e1 = v[1] + I->b3[1] - (t1 - s.z) / I->out_scale[1];
      const float e2 = v[2] + I->b3[2] - (t2 - s.w) / I->out_scale[2];
      sq += e0 * e0 + e1 * e1 + e2 * e2;
      d0 = 2.f * e0 * inv_batch; d1 = 2.f * e1 * inv_batch; d2 = 2.f * e2 * inv_batch;
    }
    store_row16(S.GS + 16 * kG, r, d0, d1, d2, 0.f, 0.f);
    operands_ready();
    if (r == 0) {
      fence_after_sync();
      mma_bf16(tmem + kColS, sdesc(sGS + 16 * kG, kG, 128), sdesc(smem_u32(I->B3T), kHid * 16, 128),
               id64, 0u);
      mma_commit(&S.bar);
    }
    if (!(ok = wait_mma(&S.bar, phase, status))) break;
    // dz2 = dh2 * (1 - h2^2), then dz1 = (dz2 W2) * (1 - h1^2)
    uint32_t gz[32];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      tmem_ld16(taddr + kColS + 16 * c, v);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const uint32_t hh = h2[8 * c + i];
        const float a = bf16_lo(hh), b = bf16_hi(hh);
        gz[8 * c + i] = pack_bf16x2(v[2 * i] * (1.f - a * a), v[2 * i + 1] * (1.f - b * b));
      }
    }
    store_row64(S.GS + 8 * kG, r, gz);
    operands_ready();
    if (r == 0) {
      fence_after_sync();
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mma_bf16(tmem + kColS, sdesc(sGS + (8 + 2 * kk) * kG, kG, 128),
                 sdesc(smem_u32(I->B2T) + kk * 2 * kHid * 16, kHid * 16, 128), id64, kk > 0);
      mma_commit(&S.bar);
    }
    if (!(ok = wait_mma(&S.bar, phase, status))) break;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      tmem_ld16(taddr + kColS + 16 * c, v);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const uint32_t hh = h1[8 * c + i];
        const float a = bf16_lo(hh), b = bf16_hi(hh);
        gz[8 * c + i] = pack_bf16x2(v[2 * i] * (1.f - a * a), v[2 * i + 1] * (1.f - b * b));
      }
    }
    store_row64(S.GS, r, gz);
    operands_ready();
    // weight gradients: A = features^T (MN-major), B = gradients (MN-major), K = samples
    if (r == 0) {
      fence_after_sync();
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) {
        const uint32_t acc = (tiles_done > 0 || kk > 0) ? 1u : 0u;
        mma_bf16(tmem + kColA, sdesc(sFS + kk * 256, 128, kG), sdesc(sGS + kk * 256, 128, kG),
                 idA, acc);
        mma_bf16(tmem + kColB, sdesc(sFS + 2 * kG + kk * 256, 128, kG),
                 sdesc(sGS + 8 * kG + kk * 256, 128, kG), idB, acc);
      }
      mma_commit(&S.bar);
    }
    if (!(ok = wait_mma(&S.bar, phase, status))) break;
    ++tiles_done;
  }
  // loss
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(kFull, sq, o);
  if ((r & 31) == 0 && sq != 0.f) atomicAdd(loss, (double)sq);
  if (ok && tiles_done > 0) {
    // rows 0..4 of the first accumulator: x features (4 inputs and the constant 1)
    if (r < 32) {
      for (int c = 0; c < kNA; c += 16) {
        float a[16];
        tmem_ld16(taddr + kColA + c, a);
        for (int i = 0; i < 16; ++i) {
          const int col = c + i;
          if (r < kIn) {
            if (col < kHid) atomicAdd(&grad[kW1 + col * kIn + r], a[i]);
          } else if (r == kIn) {
            if (col < kHid) atomicAdd(&grad[kB1 + col], a[i]);
            else if (col < 2 * kHid) atomicAdd(&grad[kB2 + col - kHid], a[i]);
            else if (col < 2 * kHid + kOut) atomicAdd(&grad[kB3 + col - 2 * kHid], a[i]);
          }
        }
      }
    }
    // second accumulator: rows 0..63 = h1 features x dz2 columns 0..63; rows 64..127 = h2
    // features x dy columns 64..66
    for (int c = 0; c < kNB; c += 16) {
      float b[16];
      tmem_ld16(taddr + kColB + c, b);
      for (int i = 0; i < 16; ++i) {
        const int col = c + i;
        if (r < kHid) {
          if (col < kHid) atomicAdd(&grad[kW2 + col * kHid + r], b[i]);
        } else if (col >= kHid && col < kHid + kOut) {
          atomicAdd(&grad[kW3 + (col - kHid) * kHid + (r - kHid)], b[i]);
        }
      }
    }
  }
  fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) {
    fence_after_sync();
    tmem_dealloc(tmem, kTrainCols);
  }
}

// One Adam step on the master parameters (gradient then cleared), followed by the repack
// of the bf16 images.  One CTA.
__global__ void mlp_adam_kernel(float* __restrict__ p, float* __restrict__ grad,
                                float* __restrict__ m1, float* __restrict__ m2,
                                const float* __restrict__ scaling, MlpImage* __restrict__ img,
                                float lr_t, float beta1, float beta2, float eps) {
  for (int i = threadIdx.x; i < kNParams; i += blockDim.x) {
    const float g = grad[i];
    const float a = beta1 * m1[i] + (1.f - beta1) * g;
    const float b = beta2 * m2[i] + (1.f - beta2) * g * g;
    m1[i] = a;
    m2[i] = b;
    p[i] -= lr_t * a / (sqrtf(b) + eps);
    grad[i] = 0.f;
  }
  __syncthreads();
  pack_image(p, scaling, img);
}

// ---- data ----------------------------------------------------------------------------------
// Exact exponential-Euler gating step of every sample (the training targets).
__global__ void hh_gating_exact_kernel(HhDev g, float dt, const float4* __restrict__ x,
                                       float* __restrict__ t, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float4 s = x[i];
    float m = s.y, h = s.z, nn = s.w;
    hh_gating<float>((float)g.VT, s.x, m, h, nn, dt);
    t[3 * i] = m;
    t[3 * i + 1] = h;
    t[3 * i + 2] = nn;
  }
}

// (v, m, h, n) rows of neurons [off, off + n) of a float32 HH population.
__global__ void hh_sample_kernel(PopDev P, int64_t off, int64_t n, float4* __restrict__ x) {
  const float* V = static_cast<const float*>(P.var[B2B_VAR_V]);
  const float* M = static_cast<const float*>(P.var[B2B_VAR_M]);
  const float* H = static_cast<const float*>(P.var[B2B_VAR_H]);
  const float* N = static_cast<const float*>(P.var[B2B_VAR_N]);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = make_float4(V[off + i], M[off + i], H[off + i], N[off + i]);
}

// Order-preserving map of floats to ints (for atomicMin/atomicMax).
__device__ __forceinline__ int ord_of(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__host__ __device__ inline float float_of_ord(int i) {
  const int b = i >= 0 ? i : i ^ 0x7FFFFFFF;
  float f;
  memcpy(&f, &b, sizeof f);
  return f;
}

// stats[0] = min v, [1] = max v, [2..4] = max |t_o - x_o| (as ordered ints).
__global__ void mlp_stats_kernel(const float4* __restrict__ x, const float* __restrict__ t,
                                 int64_t n, int* __restrict__ stats) {
  int vmin = 0x7FFFFFFF, vmax = (int)0x80000000, d0 = 0, d1 = 0, d2 = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float4 s = x[i];
    const int o = ord_of(s.x);
    vmin = min(vmin, o);
    vmax = max(vmax, o);
    d0 = max(d0, ord_of(fabsf(t[3 * i] - s.y)));
    d1 = max(d1, ord_of(fabsf(t[3 * i + 1] - s.z)));
    d2 = max(d2, ord_of(fabsf(t[3 * i + 2] - s.w)));
  }
  atomicMin(&stats[0], vmin);
  atomicMax(&stats[1], vmax);
  atomicMax(&stats[2], d0);
  atomicMax(&stats[3], d1);
  atomicMax(&stats[4], d2);
}

}  // namespace
}  // namespace b2b

// ---- host -----------------------------------------------------------------------------------
struct b2b_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  float* p = nullptr;         // master parameters
  float* g = nullptr;         // gradient accumulator
  float* m1 = nullptr;        // Adam moments
  float* m2 = nullptr;
  float* scaling = nullptr;   // in_shift[4], in_scale[4], out_scale[3], pad
  b2b::MlpImage* img = nullptr;
  double* loss = nullptr;
  int32_t* status = nullptr;
  int* stats = nullptr;
  int64_t adam_t = 0;
};

namespace b2b {

const void* mlp_image(const b2b_mlp* m) { return m->img; }
int mlp_device(const b2b_mlp* m) { return m->device; }

namespace {

#define MCU(call)                                   \
  do {                                              \
    if ((call) != cudaSuccess) return B2B_ERR_CUDA; \
  } while (0)

// Makes m's device current for the scope.
struct DeviceScope {
  int prev = -1;
  bool ok = false;
  explicit DeviceScope(int dev) {
    ok = cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int sm_count(int device) {
  int sms = kNumSMs;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return sms;
}

// Device status word of m: returns it and clears it.
b2b_status take_status(b2b_mlp* m) {
  int32_t st = 0;
  if (cudaMemcpyAsync(&st, m->status, sizeof st, cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
      cudaStreamSynchronize(m->stream) != cudaSuccess)
    return B2B_ERR_CUDA;
  if (st != 0 && cudaMemsetAsync(m->status, 0, sizeof(int32_t), m->stream) != cudaSuccess)
    return B2B_ERR_CUDA;
  return st;
}

cudaError_t repack(b2b_mlp* m) {
  mlp_pack_kernel<<<1, 256, 0, m->stream>>>(m->p, m->scaling, m->img);
  return cudaGetLastError();
}

int64_t gcd64(int64_t a, int64_t b) {
  while (b) {
    const int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// Resident CTAs per SM of a 128-thread inference kernel, from its registers and shared
// memory (carveout set to the largest shared-memory share) and its 64 TMEM columns (at most
// 8 per SM).  The runtime's occupancy query answers 1 for these kernels on this toolchain
// although 6 fit (the profiler's limits agree with this computation), so it is not used.
template <class K>
int inference_ctas_per_sm(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                       cudaSharedmemCarveoutMaxShared);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess || fa.numRegs <= 0) {
    cudaGetLastError();
    return 1;
  }
  const int regs = (fa.numRegs + 7) / 8 * 8;                      // allocation granule
  const int by_regs = 65536 / (regs * kTile);
  const int by_smem = (int)((228 * 1024) / (fa.sharedSizeBytes + 1024));  // +1 KB per CTA
  return std::max(1, std::min(std::min(by_regs, by_smem), 8));
}

int surrogate_ctas_per_sm() {
  static int cached = 0;
  if (cached == 0) cached = inference_ctas_per_sm(hh_surrogate_step_kernel);
  return cached;
}

int forward_ctas_per_sm() {
  static int cached = 0;
  if (cached == 0) cached = inference_ctas_per_sm(mlp_forward_kernel);
  return cached;
}

}  // namespace

cudaError_t launch_hh_surrogate(const Pop& pop, const int64_t* clock, int k, double dt,
                                int32_t* status, cudaStream_t s) {
  SurrDev D{};
  D.img = static_cast<const MlpImage*>(pop.surr_img);
  D.counters = pop.surr_cnt;
  D.tol = pop.surr_tol;
  D.vmax_hat = 1.0f;
  D.judge = pop.surr_judge;
  const int64_t ntiles = pop.dev.n / kTile;
  const int per_sm = pop.tune_ctas > 0 ? std::min(pop.tune_ctas, surrogate_ctas_per_sm())
                                       : surrogate_ctas_per_sm();
  const int64_t resident = (int64_t)per_sm * kNumSMs;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min(ntiles, resident));
  hh_surrogate_step_kernel<<<grid, kTile, 0, s>>>(pop.dev, D, clock, k, dt, status);
  return cudaGetLastError();
}

cudaError_t launch_hh_sample(const Pop& pop, int64_t off, int64_t n, float* dev_x,
                             cudaStream_t s) {
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8 * kNumSMs));
  hh_sample_kernel<<<(unsigned)blocks, 256, 0, s>>>(pop.dev, off, n,
                                                    reinterpret_cast<float4*>(dev_x));
  return cudaGetLastError();
}

}  // namespace b2b

using namespace b2b;

extern "C" {

b2b_status b2b_mlp_create(int32_t device, void* stream, uint64_t seed, b2b_mlp** out) {
  if (!out) return B2B_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return B2B_ERR_CUDA;
  DeviceScope ds(device);
  if (!ds.ok) return B2B_ERR_CUDA;
  b2b_mlp* m = new (std::nothrow) b2b_mlp;
  if (!m) return B2B_ERR_OOM;
  m->device = device;
  m->stream = static_cast<cudaStream_t>(stream);
  bool ok = true;
  if (!m->stream) {
    ok = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) == cudaSuccess;
    m->own_stream = ok;
  }
  ok = ok && cudaMalloc(&m->p, kNParams * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->g, kNParams * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->m1, kNParams * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->m2, kNParams * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->scaling, 12 * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->img, sizeof(MlpImage)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->loss, sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->status, sizeof(int32_t)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->stats, 8 * sizeof(int)) == cudaSuccess;
  if (!ok) {
    b2b_mlp_destroy(m);
    return B2B_ERR_OOM;
  }
  // Xavier-uniform weights from a seeded 64-bit LCG, zero biases
  std::vector<float> p(kNParams, 0.f);
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&st]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int fan_out, int fan_in) {
    const double a = std::sqrt(6.0 / (fan_in + fan_out));
    for (int i = 0; i < fan_out * fan_in; ++i) p[off + i] = (float)((2 * uni() - 1) * a);
  };
  fill(kW1, kHid, kIn);
  fill(kW2, kHid, kHid);
  fill(kW3, kOut, kHid);
  const float scaling[12] = {-0.065f, 0.5f, 0.5f, 0.5f, 20.f, 2.f, 2.f, 2.f, 0.1f, 0.1f, 0.1f, 0.f};
  ok = cudaMemcpyAsync(m->p, p.data(), kNParams * sizeof(float), cudaMemcpyHostToDevice,
                       m->stream) == cudaSuccess &&
       cudaMemcpyAsync(m->scaling, scaling, sizeof scaling, cudaMemcpyHostToDevice, m->stream) ==
           cudaSuccess &&
       cudaMemsetAsync(m->g, 0, kNParams * sizeof(float), m->stream) == cudaSuccess &&
       cudaMemsetAsync(m->m1, 0, kNParams * sizeof(float), m->stream) == cudaSuccess &&
       cudaMemsetAsync(m->m2, 0, kNParams * sizeof(float), m->stream) == cudaSuccess &&
       cudaMemsetAsync(m->status, 0, sizeof(int32_t), m->stream) == cudaSuccess &&
       repack(m) == cudaSuccess && cudaStreamSynchronize(m->stream) == cudaSuccess;
  if (!ok) {
    b2b_mlp_destroy(m);
    return B2B_ERR_CUDA;
  }
  *out = m;
  return B2B_OK;
}

b2b_status b2b_mlp_destroy(b2b_mlp* m) {
  if (!m) return B2B_ERR_INVALID_ARG;
  DeviceScope ds(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  for (void* a : {(void*)m->p, (void*)m->g, (void*)m->m1, (void*)m->m2, (void*)m->scaling,
                  (void*)m->img, (void*)m->loss, (void*)m->status, (void*)m->stats})
    if (a) cudaFree(a);
  if (m->own_stream && m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return B2B_OK;
}

b2b_status b2b_mlp_params_get(b2b_mlp* m, float* host, int64_t n) {
  if (!m || !host || n != kNParams) return B2B_ERR_INVALID_ARG;
  DeviceScope ds(m->device);
  MCU(cudaMemcpyAsync(host, m->p, kNParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  MCU(cudaStreamSynchronize(m->stream));
  return B2B_OK;
}

b2b_status b2b_mlp_params_set(b2b_mlp* m, const float* host, int64_t n) {
  if (!m || !host || n != kNParams) return B2B_ERR_INVALID_ARG;
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(host[i])) return B2B_ERR_INVALID_ARG;
  DeviceScope ds(m->device);
  MCU(cudaMemcpyAsync(m->p, host, kNParams * sizeof(float), cudaMemcpyHostToDevice, m->stream));
  MCU(cudaMemsetAsync(m->m1, 0, kNParams * sizeof(float), m->stream));
  MCU(cudaMemsetAsync(m->m2, 0, kNParams * sizeof(float), m->stream));
  m->adam_t = 0;
  MCU(repack(m));
  MCU(cudaStreamSynchronize(m->stream));
  return B2B_OK;
}

b2b_status b2b_mlp_scaling_get(b2b_mlp* m, float* host11) {
  if (!m || !host11) return B2B_ERR_INVALID_ARG;
  DeviceScope ds(m->device);
  MCU(cudaMemcpyAsync(host11, m->scaling, 11 * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  MCU(cudaStreamSynchronize(m->stream));
  return B2B_OK;
}

b2b_status b2b_mlp_scaling_set(b2b_mlp* m, const float* host11) {
  if (!m || !host11) return B2B_ERR_INVALID_ARG;
  for (int i = 0; i < 11; ++i)
    if (!std::isfinite(host11[i])) return B2B_ERR_INVALID_ARG;
  for (int i = 4; i < 11; ++i)
    if (!(host11[i] > 0)) return B2B_ERR_INVALID_ARG;
  DeviceScope ds(m->device);
  float s[12];
  std::memcpy(s, host11, 11 * sizeof(float));
  s[11] = 0.f;
  MCU(cudaMemcpyAsync(m->scaling, s, sizeof s, cudaMemcpyHostToDevice, m->stream));
  MCU(repack(m));
  MCU(cudaStreamSynchronize(m->stream));
  return B2B_OK;
}

b2b_status b2b_mlp_fit_scaling(b2b_mlp* m, const float* dev_x, const float* dev_t, int64_t n) {
  if (!m || !dev_x || !dev_t || n <= 0) return B2B_ERR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(dev_x) & 15) != 0) return B2B_ERR_INVALID_ARG;
  DeviceScope ds(m->device);
  const int init[5] = {0x7FFFFFFF, (int)0x80000000, 0, 0, 0};
  MCU(cudaMemcpyAsync(m->stats, init, sizeof init, cudaMemcpyHostToDevice, m->stream));
  mlp_stats_kernel<<<2 * sm_count(m->device), 256, 0, m->stream>>>(
      reinterpret_cast<const float4*>(dev_x), dev_t, n, m->stats);
  MCU(cudaGetLastError());
  int st[5];
  MCU(cudaMemcpyAsync(st, m->stats, sizeof st, cudaMemcpyDeviceToHost, m->stream));
  MCU(cudaStreamSynchronize(m->stream));
  const float vmin = float_of_ord(st[0]), vmax = float_of_ord(st[1]);
  if (!std::isfinite(vmin) || !std::isfinite(vmax)) return B2B_ERR_INVALID_ARG;
  const float half = std::max(0.5f * (vmax - vmin), 1e-6f);
  float s[11] = {0.5f * (vmin + vmax), 0.5f, 0.5f, 0.5f, 1.f / half, 2.f, 2.f, 2.f, 0, 0, 0};
  for (int o = 0; o < 3; ++o) s[8 + o] = std::max(float_of_ord(st[2 + o]), 1e-6f);
  return b2b_mlp_scaling_set(m, s);
}

b2b_status b2b_mlp_forward(b2b_mlp* m, const float* dev_x, float* dev_out, int64_t n,
                           int32_t raw) {
  if (!m || !dev_x || !dev_out || n < 0) return B2B_ERR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(dev_x) & 15) != 0) return B2B_ERR_INVALID_ARG;
  if (n == 0) return B2B_OK;
  DeviceScope ds(m->device);
  const int64_t ntiles = (n + kTile - 1) / kTile;
  const int64_t resident = (int64_t)forward_ctas_per_sm() * sm_count(m->device);
  const unsigned grid = (unsigned)std::min(ntiles, resident);
  mlp_forward_kernel<<<grid, kTile, 0, m->stream>>>(m->img, reinterpret_cast<const float4*>(dev_x),
                                                   dev_out, n, raw ? 1 : 0, m->status);
  MCU(cudaGetLastError());
  return take_status(m);
}

namespace {
b2b_status launch_grad(b2b_mlp* m, const float* dev_x, const float* dev_t, int64_t n,
                       int64_t mb_start, int64_t mb_n, int64_t pa, int64_t pc) {
  // more than half an SM's shared memory, so that one CTA (holding all 512 TMEM columns)
  // runs per SM and no CTA waits in tcgen05.alloc for another
  const size_t smem = std::max<size_t>(sizeof(TrainSmem), 120 * 1024);
  static bool attr[64] = {};
  if (m->device < 64 && !attr[m->device]) {
    MCU(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem));
    attr[m->device] = true;
  }
  const int64_t ntiles = (mb_n + kTile - 1) / kTile;
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, sm_count(m->device));
  mlp_grad_kernel<<<grid, kTile, smem, m->stream>>>(
      m->img, reinterpret_cast<const float4*>(dev_x), dev_t, n, mb_start, mb_n, pa, pc,
      1.0f / (float)mb_n, m->g, m->loss, m->status);
  MCU(cudaGetLastError());
  return B2B_OK;
}
}  // namespace

b2b_status b2b_mlp_grad(b2b_mlp* m, const float* dev_x, const float* dev_t, int64_t n,
                        float* host_grad, int64_t n_grad, double* loss) {
  if (!m || !dev_x || !dev_t || n <= 0 || !host_grad || n_grad != kNParams)
    return B2B_ERR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(dev_x) & 15) != 0) return B2B_ERR_INVALID_ARG;
  DeviceScope ds(m->device);
  MCU(cudaMemsetAsync(m->g, 0, kNParams * sizeof(float), m->stream));
  MCU(cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream));
  if (b2b_status st = launch_grad(m, dev_x, dev_t, n, 0, n, 1, 0)) return st;
  double l = 0;
  MCU(cudaMemcpyAsync(host_grad, m->g, kNParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  MCU(cudaMemcpyAsync(&l, m->loss, sizeof l, cudaMemcpyDeviceToHost, m->stream));
  MCU(cudaMemsetAsync(m->g, 0, kNParams * sizeof(float), m->stream));
  if (b2b_status st = take_status(m)) return st;
  if (loss) *loss = l / (double)n;
  return B2B_OK;
}

b2b_status b2b_mlp_train(b2b_mlp* m, const float* dev_x, const float* dev_t, int64_t n,
                         int32_t epochs, int32_t batch, double lr, double* loss_per_epoch) {
  if (!m || !dev_x || !dev_t || n <= 0 || epochs < 0 || batch < kTile || batch % kTile != 0 ||
      !(lr > 0))
    return B2B_ERR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(dev_x) & 15) != 0) return B2B_ERR_INVALID_ARG;
  DeviceScope ds(m->device);
  const double beta1 = 0.9, beta2 = 0.999, eps = 1e-8;
  const int64_t steps_per_epoch = (n + batch - 1) / batch;
  const int64_t total = steps_per_epoch * (int64_t)epochs;
  uint64_t rs = (uint64_t)n * 0x9E3779B97F4A7C15ull + (uint64_t)m->adam_t;
  auto rnd = [&rs]() {
    rs ^= rs << 13; rs ^= rs >> 7; rs ^= rs << 17;
    return rs;
  };
  MCU(cudaMemsetAsync(m->g, 0, kNParams * sizeof(float), m->stream));
  int64_t step = 0;
  for (int e = 0; e < epochs; ++e) {
    // sample order of this epoch: row = (pa * s + pc) mod n with gcd(pa, n) = 1
    int64_t pa = 1, pc = 0;
    if (n > 1) {
      do {
        pa = (int64_t)(rnd() % (uint64_t)n);
      } while (pa == 0 || gcd64(pa, n) != 1);
      pc = (int64_t)(rnd() % (uint64_t)n);
    }
    MCU(cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream));
    for (int64_t mb = 0; mb < n; mb += batch, ++step) {
      const int64_t mb_n = std::min<int64_t>(batch, n - mb);
      if (b2b_status st = launch_grad(m, dev_x, dev_t, n, mb, mb_n, pa, pc)) return st;
      ++m->adam_t;
      const double frac = total > 1 ? (double)step / (double)(total - 1) : 0.0;
      const double lr_s = lr * (0.02 + 0.98 * 0.5 * (1.0 + std::cos(3.141592653589793 * frac)));
      const double lr_t = lr_s * std::sqrt(1.0 - std::pow(beta2, (double)m->adam_t)) /
                          (1.0 - std::pow(beta1, (double)m->adam_t));
      mlp_adam_kernel<<<1, 1024, 0, m->stream>>>(m->p, m->g, m->m1, m->m2, m->scaling, m->img,
                                                 (float)lr_t, (float)beta1, (float)beta2,
                                                 (float)eps);
      MCU(cudaGetLastError());
    }
    double l = 0;
    MCU(cudaMemcpyAsync(&l, m->loss, sizeof l, cudaMemcpyDeviceToHost, m->stream));
    if (b2b_status st = take_status(m)) return st;
    if (loss_per_epoch) loss_per_epoch[e] = l / (double)n;
  }
  return take_status(m);
}

b2b_status b2b_hh_gating_exact(const b2b_hh_params* p, double dt, const float* dev_x,
                               float* dev_t, int64_t n, int32_t device, void* stream) {
  if (!p || !dev_x || !dev_t || n < 0 || !(dt > 0)) return B2B_ERR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(dev_x) & 15) != 0) return B2B_ERR_INVALID_ARG;
  if (n == 0) return B2B_OK;
  DeviceScope ds(device);
  if (!ds.ok) return B2B_ERR_CUDA;
  HhDev g{};
  g.VT = p->VT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 8 * sm_count(device));
  hh_gating_exact_kernel<<<(unsigned)blocks, 256, 0, s>>>(g, (float)dt,
                                                          reinterpret_cast<const float4*>(dev_x),
                                                          dev_t, n);
  MCU(cudaGetLastError());
  MCU(cudaStreamSynchronize(s));
  return B2B_OK;
}

}  // extern "C"

// ---- the bounded wait, made to run out ------------------------------------------------------
namespace b2b {
namespace {
// One CTA waits on an mbarrier with the kernels' own bounded wait (wait_mma, here with `polls`
// polls).  arrive = 0: nothing arrives and no MMA is in flight, so the wait gives up and the
// CTA records B2B_ERR_TIMEOUT and returns; arrive = 1: thread 0 arrives first, so the wait
// completes and the status stays B2B_OK.
__global__ void wait_selftest_kernel(uint32_t polls, int32_t arrive, int32_t* status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (arrive && threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&bar)) : "memory");
  }
  __syncthreads();
  const bool ok = mbar_wait(&bar, 0u, polls);
  const bool all_ok = !__syncthreads_or(!ok);
  if (!all_ok && threadIdx.x == 0) set_status(status, B2B_ERR_TIMEOUT);
}
}  // namespace
}  // namespace b2b

extern "C" b2b_status b2b_wait_selftest(int32_t device, void* stream, uint32_t polls,
                                        int32_t arrive, int32_t* device_status) {
  if (!device_status || polls == 0 || polls > (1u << 20)) return B2B_ERR_INVALID_ARG;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess)
    return B2B_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t* d = nullptr;
  int32_t h = -1;
  cudaError_t e = cudaMalloc(&d, sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, sizeof(int32_t), s);
  if (e == cudaSuccess) {
    b2b::wait_selftest_kernel<<<1, 128, 0, s>>>(polls, arrive, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (d) cudaFree(d);
  cudaSetDevice(prev);
  if (e != cudaSuccess) return B2B_ERR_CUDA;
  *device_status = h;
  return B2B_OK;
}
