// Learned path guiding: input encoding, network parameter layout and the von Mises-Fisher
// mixture the network outputs. Not part of the reference (which has no guiding); the
// integrator combines the guide with BSDF sampling by one-sample MIS.
//
// Network: 80 inputs -> 64 -> 64 -> 64 (ReLU) -> 40 outputs.
//   inputs  : sin/cos(f_k p_a), f_k = pi r^k, r = 2^(5/11), k = 0..11 (pi .. 32 pi), for the
//             3 axes of the position normalised to [-1, 1] over the scene bounds (72),
//             shading normal (3), outgoing direction (3, world space), two zeros of padding
//   outputs : 8 lobes x (mu_raw.xyz, kappa_raw, logit)
//   lobe j  : mu = normalize(mu_raw), kappa = exp(clamp(kappa_raw, -4, 10)), weight = softmax(logit)
//   vMF pdf : kappa / (2 pi (1 - exp(-2 kappa))) exp(kappa (mu . w - 1))
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dev_math.cuh"

namespace pt {

constexpr int kGuideIn = 80;
constexpr int kGuideHidden = 64;
constexpr int kGuideOut = 40;
constexpr int kGuideLobes = 8;
constexpr int kGuideFreqs = 12;
// parameter offsets (row-major W[in][out], then bias[out]) in one contiguous array
constexpr int kGW1 = 0;
constexpr int kGB1 = kGW1 + kGuideIn * kGuideHidden;        // 5120
constexpr int kGW2 = kGB1 + kGuideHidden;                   // 5184
constexpr int kGB2 = kGW2 + kGuideHidden * kGuideHidden;    // 9280
constexpr int kGW3 = kGB2 + kGuideHidden;                   // 9344
constexpr int kGB3 = kGW3 + kGuideHidden * kGuideHidden;    // 13440
constexpr int kGW4 = kGB3 + kGuideHidden;                   // 13504
constexpr int kGB4 = kGW4 + kGuideHidden * kGuideOut;       // 16064
constexpr int kGuideParams = kGB4 + kGuideOut;              // 16104
constexpr float kKappaLogMin = -4.f, kKappaLogMax = 10.f;

// Scene bounds for the position encoding.
struct GuideFrame {
    float lo[3];
    float inv_ext[3];  // 2 / (hi - lo)
};

#ifndef PT_GUIDE_FREQ_RATIO
#define PT_GUIDE_FREQ_RATIO 1.37035f  // 2^(5/11): frequencies pi .. 32 pi
#endif

__host__ __device__ __forceinline__ void guide_encode(const GuideFrame& gf, const float p[3], const float n[3],
                                                      const float wo[3], float out[kGuideIn]) {
    int o = 0;
    for (int a = 0; a < 3; a++) {
        const float x = (p[a] - gf.lo[a]) * gf.inv_ext[a] - 1.f;
        float f = 3.14159265358979f;
        for (int k = 0; k < kGuideFreqs; k++) {
            float s, c;
#if defined(__CUDA_ARCH__)
            __sincosf(f * x, &s, &c);  // |f x| <= 32 pi: the hardware approximation suffices for features
#else
            s = sinf(f * x);
            c = cosf(f * x);
#endif
            out[o++] = s;
            out[o++] = c;
            f *= PT_GUIDE_FREQ_RATIO;
        }
    }
    for (int a = 0; a < 3; a++) out[o++] = n[a];
    for (int a = 0; a < 3; a++) out[o++] = wo[a];
    out[o++] = 0.f;
    out[o++] = 0.f;
}

// log of the vMF normaliser kappa / (2 pi (1 - exp(-2 kappa)))
__host__ __device__ __forceinline__ float vmf_log_norm(float kappa) {
    return logf(kappa) - 1.8378770664093453f /* log(2 pi) */ - log1pf(-expf(-2.f * kappa));
}

// Mixture as stored per queue slot for sampling and evaluation (40 floats): lobe j as the
// float4 (kappa_j mu_j, c_j) with c_j = log pi_j + log C(kappa_j) - kappa_j, then the 8
// cumulative lobe weights. The density is then sum_j exp(c_j + kappa_j mu_j . w): one
// exponential per lobe.
constexpr int kMixCdf = 4 * kGuideLobes;

#if defined(__CUDACC__)
// Raw network outputs -> stored mixture. The stored values define the distribution that is
// both sampled and evaluated, so hardware approximations of exp/log are exact enough here.
__device__ __forceinline__ void guide_activate(const float raw[kGuideOut], float mix[kGuideOut]) {
    float mx = -1e30f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) mx = fmaxf(mx, raw[5 * j + 4]);
    float sum = 0.f;
    float e[kGuideLobes];
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        e[j] = __expf(raw[5 * j + 4] - mx);
        sum += e[j];
    }
    const float inv_sum = 1.f / sum;
    float cdf = 0.f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        const float mxr = raw[5 * j], myr = raw[5 * j + 1], mzr = raw[5 * j + 2];
        const float il = rsqrtf(mxr * mxr + myr * myr + mzr * mzr + 1e-24f);
        const float lk = fminf(kKappaLogMax, fmaxf(kKappaLogMin, raw[5 * j + 3]));
        const float kappa = __expf(lk);
        const float pi = e[j] * inv_sum;
        mix[4 * j] = kappa * mxr * il;
        mix[4 * j + 1] = kappa * myr * il;
        mix[4 * j + 2] = kappa * mzr * il;
        // log pi + log kappa - log(2 pi) - log(1 - exp(-2 kappa)) - kappa
        mix[4 * j + 3] = __logf(pi) + lk - 1.8378770664093453f - __logf(1.f - __expf(-2.f * kappa)) - kappa;
        cdf += pi;
        mix[kMixCdf + j] = cdf;
    }
}

// Density of the stored mixture at unit direction w.
__device__ __forceinline__ float guide_pdf(const float* mix, V w) {
    const float4* l = reinterpret_cast<const float4*>(mix);
    float p = 0.f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        const float4 v = l[j];
        p += __expf(v.w + v.x * w.x + v.y * w.y + v.z * w.z);
    }
    return p;
}

// Sample the mixture: lobe by weight (u0), direction by the numerically stable vMF inverse
// (Jakob, "Numerically stable sampling of the von Mises-Fisher distribution on S^2", 2012).
__device__ __forceinline__ V guide_sample(const float* mix, float u0, float u1, float u2) {
    int j = kGuideLobes - 1;
#pragma unroll
    for (int k = kGuideLobes - 2; k >= 0; k--)
        if (u0 < mix[kMixCdf + k]) j = k;
    const float4 v = reinterpret_cast<const float4*>(mix)[j];
    const float kappa = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    const float u = fmaxf(u1, 1e-7f);
    const float wz = fminf(1.f, fmaxf(-1.f, 1.f + logf(u + (1.f - u) * expf(-2.f * kappa)) / kappa));
    const float r = sqrtf(fmaxf(0.f, 1.f - wz * wz));
    float s, c;
    sincosf(kTwoPiF * u2, &s, &c);
    const float ik = 1.f / kappa;
    const V mu = V{v.x * ik, v.y * ik, v.z * ik};
    // orthonormal frame around mu
    const Frame f = make_frame(mu);
    return to_world(f, V{r * c, r * s, wz});
}
#endif  // __CUDACC__

}  // namespace pt
