// Device vector math and the per-path random number generator.
//
// Expressions follow the reference's Vec3/Frame formulas (include/core/vec3.h,
// include/frame.h:7-59) term for term; shading may contract into FMA. The intersection code
// in dev_trace.cuh uses the uncontracted IEEE forms instead (bit-compatible hit results).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

namespace pt {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kInvPiF = 0.318309886183790671538f;
constexpr float kTwoPiF = 6.28318530717958647692f;

struct V {
    float x, y, z;
};

__device__ __forceinline__ V mkv(float a, float b, float c) { return V{a, b, c}; }
__device__ __forceinline__ V mkv(float a) { return V{a, a, a}; }
__device__ __forceinline__ V mkv(float4 a) { return V{a.x, a.y, a.z}; }
__device__ __forceinline__ V operator+(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V operator-(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V operator-(V a) { return V{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V operator*(V a, V b) { return V{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V operator*(V a, float s) { return V{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V operator*(float s, V a) { return V{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V operator/(V a, float s) { return V{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V cross(V a, V b) {
    return V{a.y * b.z - a.z * b.y, -(a.x * b.z - a.z * b.x), a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(V a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ V normalized(V a) { return a / length(a); }
__device__ __forceinline__ bool is_zero(V a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
// Vec3::reflect (vec3.h:48-50): normal * (normal . v) * 2 - v
__device__ __forceinline__ V reflect(V v, V n) {
    const float d = dot(v, n);
    return V{n.x * d * 2.f - v.x, n.y * d * 2.f - v.y, n.z * d * 2.f - v.z};
}

// Frame from a (not necessarily unit) normal: coordinateSystem of include/frame.h:7-17.
struct Frame {
    V s, t, n;
};
__device__ __forceinline__ Frame make_frame(V a) {
    Frame f;
    f.n = a;
    if (fabsf(a.x) > fabsf(a.y)) {
        const float inv = 1.0f / sqrtf(a.x * a.x + a.z * a.z);
        f.t = V{a.z * inv, 0.0f, -a.x * inv};
    } else {
        const float inv = 1.0f / sqrtf(a.y * a.y + a.z * a.z);
        f.t = V{0.0f, a.z * inv, -a.y * inv};
    }
    f.s = cross(f.t, a);
    return f;
}
__device__ __forceinline__ V to_world(const Frame& f, V l) {
    return V{f.s.x * l.x + f.t.x * l.y + f.n.x * l.z, f.s.y * l.x + f.t.y * l.y + f.n.y * l.z,
             f.s.z * l.x + f.t.z * l.y + f.n.z * l.z};
}
__device__ __forceinline__ V to_local(const Frame& f, V w) {
    return V{f.s.x * w.x + f.s.y * w.y + f.s.z * w.z, f.t.x * w.x + f.t.y * w.y + f.t.z * w.z,
             f.n.x * w.x + f.n.y * w.y + f.n.z * w.z};
}

// ---------------------------------------------------------------------------------------
// PCG32 (O'Neill 2014, XSH-RR output), one stream per pixel (increment 2*pixel+1) and one
// starting state per (seed, sample index): a path's draws are a pure function of
// (seed, pixel, sample), independent of how paths are scheduled on the GPU.
// Uniform variates lie in (0, 1] like curand_uniform, whose range the reference relies on
// (include/math/distribution.h:26-36, include/lights/sampler.h:158-159).
// ---------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
constexpr uint64_t kPcgMult = 6364136223846793005ULL;

__host__ __device__ __forceinline__ uint32_t pcg_step(uint64_t& state, uint64_t inc) {
    const uint64_t old = state;
    state = old * kPcgMult + inc;
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}
__host__ __device__ __forceinline__ uint64_t pcg_inc(uint32_t pixel) { return ((uint64_t)pixel << 1) | 1ULL; }
// pcg32_srandom(initstate, initseq)
__host__ __device__ __forceinline__ uint64_t pcg_seed(uint64_t seed, uint64_t sample, uint32_t pixel) {
    const uint64_t inc = pcg_inc(pixel);
    uint64_t st = 0;
    pcg_step(st, inc);
    st += splitmix64(seed ^ splitmix64(sample));
    pcg_step(st, inc);
    return st;
}
__host__ __device__ __forceinline__ float pcg_uniform(uint64_t& state, uint64_t inc) {
    const uint32_t r = pcg_step(state, inc);
    return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f);
}

}  // namespace pt
