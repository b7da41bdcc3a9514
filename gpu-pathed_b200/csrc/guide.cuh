// Learned path guiding: input encoding, network parameter layout and the von Mises-Fisher
// mixture the network outputs. Not part of the reference (which has no guiding); the
// integrator combines the guide with BSDF sampling by one-sample MIS.
//
// Network: 80 inputs -> 64 -> 64 -> 64 (ReLU) -> 40 outputs.
//   inputs  : sin/cos(2^k pi p_a), k = 0..11, for the 3 axes of the position normalised to
//             [-1, 1] over the scene bounds (72), shading normal (3), outgoing direction
//             (3, world space), two zeros of padding
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

// Mixture as stored per queue slot: for each lobe mu.xyz, kappa, weight (40 floats).
struct GuideMixture {
    float v[kGuideOut];
};

// Scene bounds for the position encoding.
struct GuideFrame {
    float lo[3];
    float inv_ext[3];  // 2 / (hi - lo)
};

__host__ __device__ __forceinline__ void guide_encode(const GuideFrame& gf, const float p[3], const float n[3],
                                                      const float wo[3], float out[kGuideIn]) {
    int o = 0;
    for (int a = 0; a < 3; a++) {
        const float x = (p[a] - gf.lo[a]) * gf.inv_ext[a] - 1.f;
        float f = 3.14159265358979f;
        for (int k = 0; k < kGuideFreqs; k++) {
            float s, c;
#if defined(__CUDA_ARCH__)
            sincosf(f * x, &s, &c);
#else
            s = sinf(f * x);
            c = cosf(f * x);
#endif
            out[o++] = s;
            out[o++] = c;
            f *= 2.f;
        }
    }
    for (int a = 0; a < 3; a++) out[o++] = n[a];
    for (int a = 0; a < 3; a++) out[o++] = wo[a];
    out[o++] = 0.f;
    out[o++] = 0.f;
}

// Raw network outputs -> mixture parameters (mu normalised, kappa, softmax weight).
__host__ __device__ __forceinline__ void guide_activate(const float raw[kGuideOut], float mix[kGuideOut]) {
    float mx = -1e30f;
    for (int j = 0; j < kGuideLobes; j++) mx = fmaxf(mx, raw[5 * j + 4]);
    float sum = 0.f;
    float e[kGuideLobes];
    for (int j = 0; j < kGuideLobes; j++) {
        e[j] = expf(raw[5 * j + 4] - mx);
        sum += e[j];
    }
    for (int j = 0; j < kGuideLobes; j++) {
        const float mxr = raw[5 * j], myr = raw[5 * j + 1], mzr = raw[5 * j + 2];
        const float len = sqrtf(mxr * mxr + myr * myr + mzr * mzr) + 1e-12f;
        mix[5 * j] = mxr / len;
        mix[5 * j + 1] = myr / len;
        mix[5 * j + 2] = mzr / len;
        mix[5 * j + 3] = expf(fminf(kKappaLogMax, fmaxf(kKappaLogMin, raw[5 * j + 3])));
        mix[5 * j + 4] = e[j] / sum;
    }
}

// log of the vMF normaliser kappa / (2 pi (1 - exp(-2 kappa)))
__host__ __device__ __forceinline__ float vmf_log_norm(float kappa) {
    return logf(kappa) - 1.8378770664093453f /* log(2 pi) */ - log1pf(-expf(-2.f * kappa));
}

__device__ __forceinline__ float guide_pdf(const float* mix, V w) {
    float p = 0.f;
#pragma unroll
    for (int j = 0; j < kGuideLobes; j++) {
        const float k = mix[5 * j + 3];
        const float d = mix[5 * j] * w.x + mix[5 * j + 1] * w.y + mix[5 * j + 2] * w.z;
        p += mix[5 * j + 4] * expf(vmf_log_norm(k) + k * (d - 1.f));
    }
    return p;
}

// Sample the mixture: lobe by weight (u0), direction by the numerically stable vMF inverse
// (Jakob, "Numerically stable sampling of the von Mises-Fisher distribution on S^2", 2012).
__device__ __forceinline__ V guide_sample(const float* mix, float u0, float u1, float u2) {
    int j = kGuideLobes - 1;
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < kGuideLobes; k++) {
        acc += mix[5 * k + 4];
        if (u0 < acc) {
            j = k;
            break;
        }
    }
    const float kappa = mix[5 * j + 3];
    const float u = fmaxf(u1, 1e-7f);
    const float wz = fminf(1.f, fmaxf(-1.f, 1.f + logf(u + (1.f - u) * expf(-2.f * kappa)) / kappa));
    const float r = sqrtf(fmaxf(0.f, 1.f - wz * wz));
    float s, c;
    sincosf(kTwoPiF * u2, &s, &c);
    const V mu = V{mix[5 * j], mix[5 * j + 1], mix[5 * j + 2]};
    // orthonormal frame around mu
    const Frame f = make_frame(mu);
    return to_world(f, V{r * c, r * s, wz});
}

}  // namespace pt
