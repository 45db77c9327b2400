// Seeded synthetic inputs, identical on host and device (integer arithmetic
// only).  R-MAT with a/b/c/d = 0.57/0.19/0.19/0.05 and no noise: pair i draws
// one 32-bit uniform per level from a counter-based splitmix64 hash of
// (seed, i, level pair), so any thread or device regenerates any pair alone.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GV_HD __host__ __device__ __forceinline__
#else
#define GV_HD static inline
#endif

GV_HD uint64_t gv_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Thresholds of the quadrant draw: P(a), P(a+b), P(a+b+c) scaled by 2^32.
#define GV_RMAT_TA 2448131358u   /* 0.57 * 2^32 */
#define GV_RMAT_TAB 3264175145u  /* 0.76 * 2^32 */
#define GV_RMAT_TABC 4080218931u /* 0.95 * 2^32 */

GV_HD void gv_rmat_pair(uint64_t seed, uint64_t i, uint32_t scale, uint32_t *src, uint32_t *dst) {
    uint32_t u = 0, v = 0;
    const uint64_t key = gv_mix64(seed ^ 0x5DEECE66Dull) ^ (i * 0xD1B54A32D192ED03ull);
    for (uint32_t l = 0; l < scale; l += 2) {
        uint64_t h = gv_mix64(key + (uint64_t)(l >> 1) * 0x9E3779B97F4A7C15ull);
        for (uint32_t t = 0; t < 2 && l + t < scale; ++t) {
            uint32_t r = (uint32_t)(h >> (32 * t));
            uint32_t bu, bv;
            if (r < GV_RMAT_TA) { bu = 0; bv = 0; }
            else if (r < GV_RMAT_TAB) { bu = 0; bv = 1; }
            else if (r < GV_RMAT_TABC) { bu = 1; bv = 0; }
            else { bu = 1; bv = 1; }
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
    }
    *src = u;
    *dst = v;
}

// Uniform integer in [0, range) from a 64-bit hash (multiply-shift).
GV_HD uint32_t gv_uniform_u32(uint64_t h, uint32_t range) {
    return (uint32_t)(((h >> 32) * (uint64_t)range) >> 32);
}

// Uniform pair u != v over [0, n): u uniform, v uniform over the other n-1
// vertices; pair i depends only on (n, seed, i).
GV_HD void gv_uniform_pair(uint32_t n, uint64_t seed, uint64_t i, uint32_t *s, uint32_t *d) {
    const uint64_t h1 = gv_mix64(seed * 0x9E3779B97F4A7C15ull + 2 * i);
    const uint64_t h2 = gv_mix64(seed * 0x9E3779B97F4A7C15ull + 2 * i + 1);
    const uint32_t u = gv_uniform_u32(h1, n);
    uint32_t v = gv_uniform_u32(h2, n - 1);  // v in [0, n-1) then skip u
    if (v >= u) ++v;
    *s = u;
    *d = v;
}
