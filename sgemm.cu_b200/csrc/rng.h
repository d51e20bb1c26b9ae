// rng.h — seeded counter-based generator shared by host and device code.
//
// value(seed, tag, i) depends only on its arguments, so any element of any
// matrix can be regenerated anywhere (device fill kernel, host oracle,
// sampled-row checks) without storing the matrix.  The mixing function is the
// SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014).  The reference draws inputs with
// rand() seeded by time(NULL) (test.cu:19, common/helper_matrix.h:19-23), which
// cannot be reproduced; this generator replaces it.
//
// The oracle carries an independent C restatement of the same function
// (oracle/oracle.c); the tests check both produce identical bits.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define SGB_HD __host__ __device__ __forceinline__
#else
#define SGB_HD static inline
#endif

SGB_HD uint64_t rng_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

SGB_HD uint64_t rng_key(uint64_t seed, uint32_t tag) {
    return rng_mix(seed ^ rng_mix(0xA0761D6478BD642Full + (uint64_t)tag));
}

// dist 0: uniform[-1, 1) on a 2^-23 grid; dist 1: uniform[0, 1) on a 2^-24
// grid; dist 2: random sign * 2^e * (1 + f), e uniform in [-10, 10],
// f uniform on the 23-bit mantissa grid.  All conversions are exact.
SGB_HD float rng_value(uint64_t key, uint64_t index, int dist) {
    const uint64_t b = rng_mix(key + index);
    if (dist == 0) {
        const int32_t u = (int32_t)(b >> 40) - (1 << 23);
        return (float)u * (1.0f / 8388608.0f);
    }
    if (dist == 1) {
        return (float)(uint32_t)(b >> 40) * (1.0f / 16777216.0f);
    }
    const uint32_t sign = (uint32_t)(b & 1u) << 31;
    const int32_t e = (int32_t)((b >> 1) % 21u) - 10;
    const uint32_t mant = (uint32_t)(b >> 41) & 0x7FFFFFu;
    const uint32_t bits = sign | ((uint32_t)(127 + e) << 23) | mant;
    union {
        uint32_t u;
        float f;
    } cvt;
    cvt.u = bits;
    return cvt.f;
}
