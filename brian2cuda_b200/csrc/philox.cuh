// Philox-4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011), written from the paper's definition.  Used for
// connectivity generation so that the same (seed, i, j) always yields the same synapse, on
// the GPU and in the CPU oracle alike.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define B2B_HD __host__ __device__ __forceinline__
#else
#define B2B_HD inline
#endif

namespace b2b {

struct U32x4 {
  uint32_t x, y, z, w;
};

B2B_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

// Round multipliers and Weyl key increments from the paper (Table 2 / section 3.3).
B2B_HD U32x4 philox4x32_10(U32x4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, c.x, &hi0, &lo0);
    mulhilo32(M1, c.z, &hi1, &lo1);
    U32x4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Connection test for the pair block (i, 4*jq .. 4*jq+3): bit e set when pre i connects to
// post 4*jq+e.  thr = floor(p * 2^32) (p >= 1 connects every pair).
B2B_HD unsigned connect_bits(uint64_t seed, uint32_t i, uint32_t jq, uint64_t thr) {
  const U32x4 r = philox4x32_10(U32x4{jq, i, 0x5EEDu, 0u}, (uint32_t)seed,
                                (uint32_t)(seed >> 32));
  unsigned b = 0;
  b |= ((uint64_t)r.x < thr) ? 1u : 0u;
  b |= ((uint64_t)r.y < thr) ? 2u : 0u;
  b |= ((uint64_t)r.z < thr) ? 4u : 0u;
  b |= ((uint64_t)r.w < thr) ? 8u : 0u;
  return b;
}

// Delay of synapse (i, j), uniform on the integers [dmin, dmin + nd).
B2B_HD int32_t connect_delay(uint64_t seed, uint32_t i, uint32_t j, int32_t dmin, int32_t nd) {
  const U32x4 r = philox4x32_10(U32x4{j, i, 0xDE1Au, 1u}, (uint32_t)seed,
                                (uint32_t)(seed >> 32));
  return dmin + (int32_t)(((uint64_t)r.x * (uint64_t)(uint32_t)nd) >> 32);
}

B2B_HD uint64_t connect_threshold(double p) {
  if (p >= 1.0) return (uint64_t)1 << 32;
  if (p <= 0.0) return 0;
  return (uint64_t)(p * 4294967296.0);
}

}  // namespace b2b
