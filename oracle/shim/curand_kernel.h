/* Host-only stand-in for <curand_kernel.h>, used solely to compile the reference's headers
 * for the CPU (oracle/_ref). It defines the two names those headers use with a PCG32
 * generator of our own; no curand code or tables are involved. Integrator-level use of the
 * reference is not made through this header (the pinning entry points pass explicit
 * uniform variates). */
#pragma once
#include <stdint.h>

typedef struct curandStateShim {
    uint64_t state;
    uint64_t inc;
} curandState;

static inline float curand_uniform(curandState* s) {
    const uint64_t old = s->state;
    s->state = old * 6364136223846793005ULL + s->inc;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    const uint32_t r = (xs >> rot) | (xs << ((0u - rot) & 31u));
    return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f);
}

static inline void curand_init(unsigned long long seed, unsigned long long subsequence, unsigned long long offset,
                               curandState* s) {
    s->inc = (subsequence << 1) | 1ULL;
    s->state = seed + offset;
}
