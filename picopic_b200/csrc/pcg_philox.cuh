// pcg_philox.cuh — counter-based Philox4x32-10 (Salmon et al., SC'11),
// used for beam injection so that a particle's random numbers depend only
// on (seed, species stream, step, index), never on thread scheduling.
#pragma once

#include <cstdint>

namespace pcg {

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                       uint32_t c3, uint32_t k0, uint32_t k1,
                                                       uint32_t out[4]) {
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Two uniforms in [0, 1) with 53 random bits each from one Philox block:
// counter (index, step lo, step hi, stream), key = seed.
__host__ __device__ __forceinline__ void philox_uniform2(uint64_t seed, uint32_t stream,
                                                         uint64_t step, uint32_t index,
                                                         double u[2]) {
  uint32_t o[4];
  philox4x32_10(index, (uint32_t)step, (uint32_t)(step >> 32), stream, (uint32_t)seed,
                (uint32_t)(seed >> 32), o);
  const double k26 = 67108864.0, k53 = 1.0 / 9007199254740992.0;
  u[0] = ((double)(o[0] >> 5) * k26 + (double)(o[1] >> 6)) * k53;
  u[1] = ((double)(o[2] >> 5) * k26 + (double)(o[3] >> 6)) * k53;
}

}  // namespace pcg
