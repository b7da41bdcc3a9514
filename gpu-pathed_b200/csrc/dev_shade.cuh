// Shading: BSDFs, emitter sampling, environment light and camera rays (FP32).
//
// Each function restates the reference routine it cites, including its numerical
// conventions (unnormalised interpolated shading normals, the glass refraction helper's
// second eta swap, the microfacet alpha scaling by the incident cosine, pixel-centre
// environment directions). Constants the reference evaluates in double through M_PI are
// evaluated in single precision here.
#pragma once

#include <cuda_runtime.h>

#include "dev_math.cuh"
#include "pt_types.h"

namespace pt {

struct BsdfSample {
    V wi;      // local frame
    float pdf;
    V f;
    bool delta;
};

// ---- Lambertian (include/materials/lambertian.h:43-76) --------------------------------
__device__ __forceinline__ V lambert_f(const Material& m, V wo, V wi) {
    if (wo.z < 0.f || wi.z < 0.f) return mkv(0.f);
    return mkv(m.albedo[0], m.albedo[1], m.albedo[2]) / kPiF;
}
__device__ __forceinline__ float lambert_pdf(V wi) {  // core/sample.h:18-23
    if (wi.z < 0.f) return 0.f;
    return 1.f / (2.f * kPiF);
}
// Sample::uniformHemisphere (include/core/sample.h:7-16)
__device__ __forceinline__ BsdfSample lambert_sample(const Material& m, V wo, float xi1, float xi2) {
    const float z = xi1;
    const float r = sqrtf(fmaxf(0.f, 1.f - z * z));
    const float phi = kTwoPiF * xi2;
    float sp, cp;
    sincosf(phi, &sp, &cp);
    const V wi{r * cp, r * sp, z};
    return BsdfSample{wi, lambert_pdf(wi), lambert_f(m, wo, wi), false};
}

// ---- Mirror (include/materials/mirror.h:47-55) -----------------------------------------
__device__ __forceinline__ BsdfSample mirror_sample(V wo) {
    const V wi = reflect(wo, mkv(0.f, 0.f, 1.f));
    return BsdfSample{wi, 1.f, mkv(fmaxf(0.f, 1.f / wi.z)), true};
}

// ---- Optics (include/optics/fresnel.h:14-42, include/optics/snell.h:10-66) ---------------
__device__ __forceinline__ float fresnel_dielectric(float cos_i, float eta_i, float eta_t) {
    const float sin_t = (eta_i / eta_t) * sqrtf(fmaxf(0.f, 1.f - cos_i * cos_i));
    if (sin_t > 1.f) return 1.f;  // total internal reflection
    const float cos_t = sqrtf(fmaxf(0.f, 1.f - sin_t * sin_t));
    const float r_par = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
    const float r_perp = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
    return 0.5f * (r_par * r_par + r_perp * r_perp);
}
// Snell::refract with normal (0,0,1); swaps the normal and the etas itself when the incident
// direction is below the surface.
__device__ __forceinline__ V snell_refract(V wo, float eta_i, float eta_t) {
    V n = mkv(0.f, 0.f, 1.f);
    if (dot(wo, n) < 0.f) {
        n = n * -1.f;
        const float tmp = eta_i;
        eta_i = eta_t;
        eta_t = tmp;
    }
    const float d = dot(wo, n);
    const V perp_i = wo - V{n.x * d, n.y * d, n.z * d};
    const V perp_t = (-perp_i) * (eta_i / eta_t);
    const float l = length(perp_t);
    const float par_len = sqrtf(fmaxf(0.f, 1.f - l * l));
    const V par_t = n * -par_len;
    return normalized(par_t + perp_t);
}

// ---- Glass (include/materials/glass.h:44-109) ------------------------------------------
__device__ __forceinline__ BsdfSample glass_sample(const Material& m, V wo, float xi1) {
    float eta_i = 1.f, eta_t = m.ior;
    if (wo.z < 0.f) {
        const float tmp = eta_i;
        eta_i = eta_t;
        eta_t = tmp;
    }
    V wi = snell_refract(wo, eta_i, eta_t);
    const float F = fresnel_dielectric(fabsf(wo.z), eta_i, eta_t);
    if (xi1 < F) {
        wi = reflect(wo, mkv(0.f, 0.f, 1.f));
        const float c = fabsf(wi.z);
        return BsdfSample{wi, F, c == 0.f ? mkv(0.f) : mkv(F / c), true};
    }
    const float T = 1.f - F;
    const float c = fabsf(wi.z);
    const float r = eta_i / eta_t;
    const V thr = c == 0.f ? mkv(0.f) : mkv(T / c);
    return BsdfSample{wi, T, thr * (r * r), true};
}

// ---- Beckmann microfacet (include/materials/microfacet.h:19-164) ------------------------
__device__ __forceinline__ float mf_sample_alpha(float alpha, float abs_cos) {
    return (1.2f - 0.2f * sqrtf(abs_cos)) * alpha;
}
__device__ __forceinline__ float mf_D(float alpha, V wi, V wh) {
    const float a = mf_sample_alpha(alpha, fabsf(wi.z));
    const float a2 = a * a;
    const float cos2 = wh.z * wh.z;
    const float cos4 = cos2 * cos2;
    const float tan2 = (1.f - cos2) / cos2;
    if (isinf(tan2)) return 0.f;
    return expf(-tan2 / a2) / (kPiF * a2 * cos4);
}
__device__ __forceinline__ float mf_G1(float alpha, V v) {
    const float sin_t = sqrtf(fmaxf(0.f, 1.f - v.z * v.z));
    const float a = 1.f / (alpha * fabsf(sin_t / v.z));
    if (a >= 1.6f) return 1.f;
    return (3.535f * a + 2.181f * a * a) / (1.f + 2.276f * a + 2.577f * a * a);
}
__device__ __forceinline__ float sgn(float x) { return x < 0.f ? -1.f : 1.f; }
__device__ __forceinline__ float mf_G(float alpha, V wi, V wo, V wh) {
    if (sgn(dot(wo, wh)) != sgn(wo.z)) return 0.f;
    if (sgn(dot(wi, wh)) != sgn(wi.z)) return 0.f;
    return mf_G1(alpha, wi) * mf_G1(alpha, wo);
}
__device__ __forceinline__ V mf_f(float alpha, V wo, V wi) {
    if (wo.z < 0.f || wi.z < 0.f) return mkv(0.f);
    const float co = fabsf(wo.z), ci = fabsf(wi.z);
    const V wh = normalized(wo + wi);
    if (co == 0.f || ci == 0.f) return mkv(0.f);
    if (is_zero(wh)) return mkv(0.f);
    const float cinc = fminf(1.f, fmaxf(dot(wi, wh), 0.f));
    const float F = fresnel_dielectric(cinc, 1.f, 1.5f);  // fixed eta 1.5 (microfacet.h:111)
    const float D = mf_D(alpha, wi, wh);
    const float G = mf_G(alpha, wi, wo, wh);
    return mkv(D * G * F / (4.f * ci * co));
}
// kMetal: the same D and G with a per-channel Schlick Fresnel, F = F0 + (1 - F0)(1 - c)^5 at
// c = wi . wh, F0 the material's albedo (Schlick 1994).
__device__ __forceinline__ V mf_metal_f(const Material& m, V wo, V wi) {
    if (wo.z < 0.f || wi.z < 0.f) return mkv(0.f);
    const float co = fabsf(wo.z), ci = fabsf(wi.z);
    const V wh = normalized(wo + wi);
    if (co == 0.f || ci == 0.f) return mkv(0.f);
    if (is_zero(wh)) return mkv(0.f);
    const float cinc = fminf(1.f, fmaxf(dot(wi, wh), 0.f));
    const float q = 1.f - cinc, q2 = q * q, q5 = q2 * q2 * q;
    const float s = mf_D(m.alpha, wi, wh) * mf_G(m.alpha, wi, wo, wh) / (4.f * ci * co);
    return mkv((m.albedo[0] + (1.f - m.albedo[0]) * q5) * s, (m.albedo[1] + (1.f - m.albedo[1]) * q5) * s,
               (m.albedo[2] + (1.f - m.albedo[2]) * q5) * s);
}
__device__ __forceinline__ float mf_pdf(float alpha, V wo, V wi) {
    if (wo.z < 0.f || wi.z < 0.f) return 0.f;
    const V wh = normalized(wo + wi);
    return mf_D(alpha, wi, wh) * fabsf(wh.z) / (4.f * fabsf(dot(wo, wh)));
}
__device__ __forceinline__ BsdfSample mf_sample(float alpha, V wo, float xi1, float xi2) {
    const float phi = xi1 * kPiF * 2.f;
    const float a = mf_sample_alpha(alpha, fabsf(wo.z));
    const float a2 = a * a;
    const float st = -a2 * logf(1.f - xi2);
    const float theta = atanf(sqrtf(st));
    float sp, cp, sth, cth;
    sincosf(phi, &sp, &cp);
    sincosf(theta, &sth, &cth);
    const V wh{sth * cp, sth * sp, cth};
    const V wi = reflect(wo, wh);
    const float pdf = mf_D(alpha, wo, wh) * fabsf(wh.z) / (4.f * fabsf(dot(wi, wh)));
    return BsdfSample{wi, pdf, mf_f(alpha, wo, wi), false};
}

// ---- BSDF dispatch (include/materials/bsdf.h:19-115) -------------------------------------
__device__ __forceinline__ V bsdf_f(const Material& m, V wo, V wi) {
    switch (m.type) {
        case kLambertian: return lambert_f(m, wo, wi);
        case kMicrofacet: return mf_f(m.alpha, wo, wi);
        case kMetal: return mf_metal_f(m, wo, wi);
        default: return mkv(0.f);  // mirror, glass: f = 0
    }
}
__device__ __forceinline__ float bsdf_pdf(const Material& m, V wo, V wi) {
    switch (m.type) {
        case kLambertian: return lambert_pdf(wi);
        case kMicrofacet:
        case kMetal: return mf_pdf(m.alpha, wo, wi);
        default: return 0.f;
    }
}

// ---- Environment light (include/lights/environment_light.h:46-83,
//      include/math/distribution.h:197-375, include/math/spherical_coordinates.h:8-28) ------
__device__ __forceinline__ void to_spherical(V w, float& phi, float& theta) {
    phi = atan2f(w.z, w.x);
    if (phi < 0.f) phi += kTwoPiF;
    theta = acosf(fminf(1.f, fmaxf(w.y, -1.f)));
}
__device__ __forceinline__ V env_emit(const EnvDevice& e, V w) {
    if (!e.present) return mkv(0.f);
    float phi, theta;
    to_spherical(w, phi, theta);
    const int x = (int)floorf(phi / kTwoPiF * e.width);
    const int y = (int)floorf(theta / kPiF * e.height);
    // texel (x, y) as the reference addresses it (x == width runs into the next row);
    // clamped to the map so that theta == pi stays inside the buffer
    long long idx = (long long)y * e.width + x;
    const long long last = (long long)e.width * e.height - 1;
    idx = idx < 0 ? 0 : (idx > last ? last : idx);
    const float4 t = __ldg(reinterpret_cast<const float4*>(e.rgba) + idx);
    return mkv(t.x, t.y, t.z);
}
// Distribution::pmf (distribution.h:226-233)
__device__ __forceinline__ float cdf_pmf(const float* cdf, int i) {
    const float c = __ldg(cdf + i);
    return i == 0 ? c : c - __ldg(cdf + i - 1);
}
// Distribution::sample (distribution.h:197-224): first index with xi < cdf[i]; for xi == 1
// the first index whose cdf equals 1. Binary search over the monotone CDF.
__device__ __forceinline__ int cdf_sample(const float* cdf, int n, float xi) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (xi < __ldg(cdf + mid)) hi = mid; else lo = mid + 1;
    }
    if (lo < n) return lo;
    lo = 0;
    hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) >= 1.f) hi = mid; else lo = mid + 1;
    }
    return lo < n ? lo : n - 1;
}
__device__ __forceinline__ float env_pmf(const EnvDevice& e, int x, int y) {
    if (e.total_mass == 0.f) return 0.f;
    const float yp = cdf_pmf(e.marg_cdf, y);
    const float xp = __ldg(e.row_mass + y) == 0.f ? 0.f : cdf_pmf(e.cond_cdf + (size_t)y * e.width, x);
    return xp * yp;
}
// PhiThetaDistribution::pdf (distribution.h:354-375)
__device__ __forceinline__ float env_pdf_dir(const EnvDevice& e, V w) {
    float phi, theta;
    to_spherical(w, phi, theta);
    const float xc = phi / kTwoPiF, yc = theta / kPiF;
    const int xs = (int)fminf(floorf(xc * e.width), (float)(e.width - 1));
    const int ys = (int)fminf(floorf(yc * e.height), (float)(e.height - 1));
    const float pdf = env_pmf(e, xs, ys) * e.width * e.height;
    return pdf / (sinf(theta) * kPiF * kPiF * 2.f);
}
// PhiThetaDistribution::sample (distribution.h:335-352): pixel-centre direction, or a
// uniform point inside the texel when `continuous` is set.
__device__ __forceinline__ V env_sample_dir(const EnvDevice& e, float xi1, float xi2, float& pdf, float cx = 0.5f,
                                            float cy = 0.5f) {
    const int y = cdf_sample(e.marg_cdf, e.height, xi1);
    const int x = cdf_sample(e.cond_cdf + (size_t)y * e.width, e.width, xi2);
    const float phi = ((x + cx) / e.width) * kPiF * 2.f;
    const float theta = ((y + cy) / e.height) * kPiF;
    float sp, cp, st, ct;
    sincosf(phi, &sp, &cp);
    sincosf(theta, &st, &ct);
    const V wi{st * cp, ct, st * sp};
    pdf = env_pdf_dir(e, wi);
    return wi;
}

// ---- Emitters (include/lights/sampler.h:20-183, surface_sample.h, core/measure.h) -------
struct LightSample {
    V wi, normal;
    float distance, pdf;
    V emitted;
};

__device__ __forceinline__ float tri_area(V p0, V p1, V p2) {
    const V c = cross(p1 - p0, p2 - p0);
    return fabsf(length(c) / 2.f);
}

__device__ __forceinline__ LightSample sample_lights(const SceneDevice& sc, V p, float xi1, float xi2,
                                                     float xi3) {
    LightSample ls;
    const int n_choice = sc.num_lights + (sc.env.present ? 1 : 0);
    const int choice = (int)fminf((float)(n_choice - 1), (float)(int)floorf(xi1 * n_choice));
    const float choice_pdf = 1.f / n_choice;
    if (choice < sc.num_lights) {
        const LightRef lr = sc.lights[choice];
        V point, normal;
        float area_pdf;
        int mat;
        if (lr.type == kTriangle) {
            const V p0 = mkv(__ldg(sc.tri_p + 3 * lr.index + 0));
            const V p1 = mkv(__ldg(sc.tri_p + 3 * lr.index + 1));
            const V p2 = mkv(__ldg(sc.tri_p + 3 * lr.index + 2));
            const float sr = sqrtf(xi2);
            const float a = 1.f - sr;
            const float b = sr * (1.f - xi3);
            const float c = 1.f - a - b;
            point = p0 * a + p1 * b + p2 * c;
            normal = normalized(cross(p1 - p0, p2 - p0));
            area_pdf = 1.f / tri_area(p0, p1, p2);
            mat = __ldg(sc.tri_mat + lr.index);
        } else {
            const float4 s = __ldg(sc.sph + lr.index);
            const float z = xi2 * 2.f - 1.f;
            const float r = sqrtf(fmaxf(0.f, 1.f - z * z));
            float sp, cp;
            sincosf(kTwoPiF * xi3, &sp, &cp);
            const V local{r * cp, r * sp, z};
            point = local * s.w + mkv(s.x, s.y, s.z);
            normal = local;
            area_pdf = 1.f / (4.f * kPiF * s.w * s.w);
            mat = __ldg(sc.sph_mat + lr.index);
        }
        const V dir = point - p;
        const float dist = length(dir);
        // SurfaceSample::solidAnglePDF
        const V lwo = -normalized(dir);
        const float proj = fabsf(dot(normal, lwo));
        const float sa = proj == 0.f ? 0.f : area_pdf * (dist * dist) / proj;
        ls.wi = normalized(dir);
        ls.normal = normal;
        ls.distance = dist;
        ls.pdf = sa * choice_pdf;
        const Material& m = sc.mats[mat];
        ls.emitted = mkv(m.emit[0], m.emit[1], m.emit[2]);
        if (m.type != kLambertian) ls.emitted = mkv(0.f);
    } else {
        float pdf;
        const V w = env_sample_dir(sc.env, xi2, xi3, pdf);
        const V wi = normalized(w);
        ls.wi = wi;
        ls.normal = -wi;
        ls.distance = 1e16f;
        ls.pdf = pdf * choice_pdf;
        ls.emitted = env_emit(sc.env, w);
    }
    return ls;
}

// Sampler::pdfSceneLights (sampler.h:89-125) for an emitting hit seen from `ref`.
__device__ __forceinline__ float pdf_scene_light(const SceneDevice& sc, V ref, V point, V normal, int prim) {
    float area_pdf;
    if (prim >= 0) {
        const V p0 = mkv(__ldg(sc.tri_p + 3 * prim + 0));
        const V p1 = mkv(__ldg(sc.tri_p + 3 * prim + 1));
        const V p2 = mkv(__ldg(sc.tri_p + 3 * prim + 2));
        area_pdf = 1.f / tri_area(p0, p1, p2);
    } else {
        const float4 s = __ldg(sc.sph + ~prim);
        area_pdf = 1.f / (4.f * kPiF * s.w * s.w);
    }
    const V sd = ref - point;
    const V swo = normalized(sd);
    const float dist = length(sd);
    const float proj = fmaxf(0.f, dot(normal, swo));
    const float sa = area_pdf * (dist * dist) / proj;
    const int n_choice = sc.num_lights + (sc.env.present ? 1 : 0);
    return sa / n_choice;
}
// Sampler::pdfEnvironmentLight (sampler.h:127-140)
__device__ __forceinline__ float pdf_env_light(const SceneDevice& sc, V w) {
    if (!sc.env.present) return 0.f;
    return env_pdf_dir(sc.env, w) * (1.f / (sc.num_lights + 1));
}
// MIS::balanceWeight (include/math/mis.h:5-8)
__device__ __forceinline__ float balance(float p1, float p2) { return p1 / (p1 + p2); }

// ---- Camera (include/core/camera.h:40-61) -------------------------------------------------
__device__ __forceinline__ void camera_ray(const CameraParams& c, int row, int col, float xi1, float xi2, V& o,
                                           V& d) {
    // every operation rounded on its own, in the order written (no FMA contraction), so a
    // camera ray is bit-identical to the one the reference's arithmetic gives on the host
    const float xc = __fdiv_rn(__fadd_rn((float)col, xi1), (float)c.res_x);
    const float yc = __fdiv_rn(__fadd_rn((float)row, xi2), (float)c.res_y);
    const float y = __fsub_rn(__fmul_rn(yc, c.height), c.top);
    const float x = __fsub_rn(__fmul_rn(xc, c.width), c.right);
    const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), 1.f));
    const V dir = mkv(__fdiv_rn(x, len), __fdiv_rn(y, len), __fdiv_rn(-1.f, len));
    // Transform::apply: the origin (0, 0, 0) maps to the translation column
    o = mkv(c.m[0][3], c.m[1][3], c.m[2][3]);
    d = mkv(__fadd_rn(__fadd_rn(__fmul_rn(c.m[0][0], dir.x), __fmul_rn(c.m[0][1], dir.y)), __fmul_rn(c.m[0][2], dir.z)),
            __fadd_rn(__fadd_rn(__fmul_rn(c.m[1][0], dir.x), __fmul_rn(c.m[1][1], dir.y)), __fmul_rn(c.m[1][2], dir.z)),
            __fadd_rn(__fadd_rn(__fmul_rn(c.m[2][0], dir.x), __fmul_rn(c.m[2][1], dir.y)), __fmul_rn(c.m[2][2], dir.z)));
}

// ---- sRGB (include/core/color.h:7-28) ---------------------------------------------------
__device__ __forceinline__ float to_srgb(float v) {
    return v <= 0.0031308f ? v * 12.92f : 1.055f * powf(v, 1.f / 2.2f) - 0.055f;
}

}  // namespace pt
