// ---------------------------------------------------------------------------
//  philox.cuh -- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
//  numbers: as easy as 1, 2, 3", SC 2011), the counter-based generator of the
//  variation operators and of the generation loop's selection draws.  A draw
//  is a pure function of (key, counter), so every stream is reproducible
//  element by element, on the host as on the device.
// ---------------------------------------------------------------------------
#pragma once
#include <stdint.h>

namespace sidon {
namespace rng {

struct U4 {
  uint32_t x, y, z, w;
};

// ten rounds of two 32x32 -> 64 multiplications on the counter, the key
// bumped by the Weyl constants between rounds
__host__ __device__ inline U4 philox(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    const U4 n = {(uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1,
                  (uint32_t)p0};
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// uniform in (0, 1): the top 24 bits plus one half, exactly representable
__host__ __device__ inline float u01(uint32_t w) {
  return ((float)(w >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// uniform in [0, 1) with 53 random bits: (27 bits of hi, 26 of lo) / 2^53,
// exact in fp64
__host__ __device__ inline double u53(uint32_t hi, uint32_t lo) {
  return ((double)(hi >> 5) * 67108864.0 + (double)(lo >> 6)) * (1.0 / 9007199254740992.0);
}

}  // namespace rng
}  // namespace sidon
