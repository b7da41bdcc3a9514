// ORACLE - test infrastructure, not product code.
//
// Harness that links the reference's own sources, compiled for the host CPU, and exposes
// its intersection, BSDF, emitter-sampling, environment and camera routines through a C
// API, so that the oracle restatement (oracle/oracle.cpp) can be checked against the
// reference bit for bit. Built by oracle/Makefile into oracle/_ref/libref_cpu.so from the
// sources under the reference tree (src/world.cu, src/primitives/*.cu,
// src/materials/{lambertian,mirror}.cu, src/core/camera.cu, src/transform.cu,
// src/math/distribution.cu) with __device__/__host__ defined empty; nothing of the
// reference is copied into this repository.
//
// The reference's host-side distribution builders allocate "device" memory with cudaMalloc
// and fill it with cudaMemcpy (src/math/distribution.cu:41-49, :476-484). This harness
// defines those two runtime entry points over host memory, so the builders run unchanged on
// the CPU; the CUDA runtime library is not linked.
#include <cfloat>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include "core/camera.h"
#include "lights/environment_light.h"
#include "lights/sampler.h"
#include "materials/glass.h"
#include "materials/lambertian.h"
#include "materials/material_lookup.h"
#include "materials/microfacet.h"
#include "materials/mirror.h"
#include "math/distribution.h"
#include "world.h"

extern "C" {
cudaError_t cudaMalloc(void** p, size_t n) {
    *p = std::malloc(n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t n, cudaMemcpyKind) {
    std::memcpy(dst, src, n);
    return cudaSuccess;
}
cudaError_t cudaFree(void* p) {
    std::free(p);
    return cudaSuccess;
}
const char* cudaGetErrorString(cudaError_t) { return "host stand-in"; }
}

using namespace rays;

namespace {

struct RefScene {
    std::vector<Triangle> tris;
    std::vector<Sphere> sphs;
    std::vector<LightIndex> lights;
    std::vector<MaterialIndex> indices;
    std::vector<Lambertian> lambertians;
    std::vector<Mirror> mirrors;
    std::vector<Glass> glasses;
    std::vector<Microfacet> microfacets;
    std::vector<float> env_rgba;
    MaterialLookup lookup;
    EnvironmentLight env = EnvironmentLight::None();
    std::unique_ptr<World> world;
};

}  // namespace

extern "C" {

void* ref_scene_create(int ntri, const float* tri_p, const float* tri_n, const int* tri_mat, int nsph, const float* sph,
                       const int* sph_mat, int nmat, const int* mtype, const float* albedo, const float* emit,
                       const float* ior, const float* alpha, int env_w, int env_h, const float* env_rgba) {
    RefScene* s = new RefScene();
    for (int i = 0; i < ntri; i++) {
        const float* p = tri_p + (size_t)i * 9;
        const float* n = tri_n + (size_t)i * 9;
        s->tris.push_back(Triangle(Vec3(p[0], p[1], p[2]), Vec3(p[3], p[4], p[5]), Vec3(p[6], p[7], p[8]),
                                   Vec3(n[0], n[1], n[2]), Vec3(n[3], n[4], n[5]), Vec3(n[6], n[7], n[8]), tri_mat[i]));
    }
    for (int i = 0; i < nsph; i++) {
        const float* q = sph + (size_t)i * 4;
        s->sphs.push_back(Sphere(Vec3(q[0], q[1], q[2]), q[3], sph_mat[i]));
    }
    // MaterialLookup::copyMaterials (src/materials/material_lookup.cu:48-123)
    for (int i = 0; i < nmat; i++) {
        switch (mtype[i]) {
            case 0: {
                LambertianParams prm(Vec3(albedo[3 * i], albedo[3 * i + 1], albedo[3 * i + 2]),
                                     Vec3(emit[3 * i], emit[3 * i + 1], emit[3 * i + 2]));
                s->lambertians.push_back(Lambertian(prm));
                s->indices.push_back({MaterialType::Lambertian, s->lambertians.size() - 1});
                break;
            }
            case 1: {
                s->mirrors.push_back(Mirror());
                s->indices.push_back({MaterialType::Mirror, s->mirrors.size() - 1});
                break;
            }
            case 2: {
                GlassParams prm(ior[i]);
                s->glasses.push_back(Glass(prm));
                s->indices.push_back({MaterialType::Glass, s->glasses.size() - 1});
                break;
            }
            default: {
                MicrofacetParams prm(alpha[i]);
                s->microfacets.push_back(Microfacet(prm));
                s->indices.push_back({MaterialType::Microfacet, s->microfacets.size() - 1});
            }
        }
    }
    s->lookup.indices = s->indices.data();
    s->lookup.lambertians = s->lambertians.data();
    s->lookup.mirrors = s->mirrors.data();
    s->lookup.glasses = s->glasses.data();
    s->lookup.microfacets = s->microfacets.data();
    // emitter list (src/scene_data.cu:92-115)
    auto emits = [&](int m) {
        return mtype[m] == 0 && !Vec3(emit[3 * m], emit[3 * m + 1], emit[3 * m + 2]).isZero();
    };
    for (int i = 0; i < ntri; i++)
        if (emits(tri_mat[i])) s->lights.push_back({PrimitiveType::Triangle, i});
    for (int i = 0; i < nsph; i++)
        if (emits(sph_mat[i])) s->lights.push_back({PrimitiveType::Sphere, i});
    if (env_rgba && env_w > 0) {
        // EnvironmentLightParams::createEnvironmentLight without the file load
        // (src/lights/environment_light.cu:40-53)
        s->env_rgba.assign(env_rgba, env_rgba + (size_t)env_w * env_h * 4);
        std::vector<float> inten((size_t)env_w * env_h);
        for (int i = 0; i < env_w * env_h; i++)
            inten[i] = env_rgba[i * 4 + 0] + env_rgba[i * 4 + 1] + env_rgba[i * 4 + 2];
        PhiThetaDistributionBuilder b(inten.data(), env_w, env_h);
        s->env = EnvironmentLight(s->env_rgba.data(), b.buildPhiThetaDistribution(), env_w, env_h);
    }
    s->world.reset(new World(s->tris.data(), s->tris.size(), s->sphs.data(), s->sphs.size(), s->lights.data(),
                             s->lights.size(), &s->env, &s->lookup));
    return s;
}

void ref_scene_destroy(void* p) { delete static_cast<RefScene*>(p); }

// World::hit over n rays (src/world.cu:5-41)
void ref_trace(void* p, const float* o, const float* d, const float* tmin, const float* tmax, int n, int* prim_type,
               int* prim_id, int* mat_id, float* t) {
    RefScene* s = static_cast<RefScene*>(p);
    for (int i = 0; i < n; i++) {
        Ray r(Vec3(o[3 * i], o[3 * i + 1], o[3 * i + 2]), Vec3(d[3 * i], d[3 * i + 1], d[3 * i + 2]));
        HitRecord rec;
        if (s->world->hit(r, tmin[i], tmax[i], rec)) {
            prim_type[i] = rec.index.primitiveType == PrimitiveType::Triangle ? 0 : 1;
            prim_id[i] = rec.index.index;
            mat_id[i] = rec.materialID;
            t[i] = rec.t;
        } else {
            prim_type[i] = -1;
            prim_id[i] = -1;
            mat_id[i] = -1;
            t[i] = 0.f;
        }
    }
}

// BSDF sample with explicit variates. out: wi[3], pdf, f[3], delta
void ref_bsdf_sample(int type, const float* albedo, float ior, float alpha, const float* wo, float xi1, float xi2,
                     float* out) {
    const Vec3 w(wo[0], wo[1], wo[2]);
    BSDFSample b;
    switch (type) {
        case 0: b = Lambertian(Vec3(albedo[0], albedo[1], albedo[2])).sample(w, xi1, xi2); break;
        case 1: b = Mirror().sample(w); break;
        case 2: b = Glass(ior).sample(w, xi1); break;
        default: b = Microfacet(MicrofacetParams(alpha)).sample(w, xi1, xi2);
    }
    out[0] = b.wiLocal.x(); out[1] = b.wiLocal.y(); out[2] = b.wiLocal.z();
    out[3] = b.pdf;
    out[4] = b.f.x(); out[5] = b.f.y(); out[6] = b.f.z();
    out[7] = b.isDelta ? 1.f : 0.f;
}

// BSDF f and pdf. out: f[3], pdf
void ref_bsdf_eval(int type, const float* albedo, float ior, float alpha, const float* wo, const float* wi, float* out) {
    const Vec3 a(wo[0], wo[1], wo[2]), b(wi[0], wi[1], wi[2]);
    Vec3 f(0.f);
    float pdf = 0.f;
    switch (type) {
        case 0: { Lambertian l(Vec3(albedo[0], albedo[1], albedo[2])); f = l.f(a, b); pdf = l.pdf(a, b); break; }
        case 1: { Mirror m; f = m.f(a, b); pdf = m.pdf(a, b); break; }
        case 2: { Glass g(ior); f = g.f(a, b); pdf = g.pdf(a, b); break; }
        default: { const MicrofacetParams prm(alpha); Microfacet m(prm); f = m.f(a, b); pdf = m.pdf(a, b); }
    }
    out[0] = f.x(); out[1] = f.y(); out[2] = f.z();
    out[3] = pdf;
}

// Sampler::sampleDirectLights with explicit variates. out: wi[3], normal[3], distance, pdf, emitted[3]
void ref_light_sample(void* p, const float* pt, float x1, float x2, float x3, float* out) {
    RefScene* s = static_cast<RefScene*>(p);
    const Vec3 hp(pt[0], pt[1], pt[2]);
    const LightSample ls = Sampler::sampleDirectLights(hp, Frame(Vec3(0.f, 1.f, 0.f)), make_float3(x1, x2, x3),
                                                       s->lights.data(), (int)s->lights.size(), s->tris.data(),
                                                       s->sphs.data(), s->env, s->lookup);
    const float v[11] = {ls.wi.x(), ls.wi.y(), ls.wi.z(), ls.normal.x(), ls.normal.y(), ls.normal.z(),
                         ls.distance, ls.pdf, ls.emitted.x(), ls.emitted.y(), ls.emitted.z()};
    std::memcpy(out, v, sizeof(v));
}

// Camera::generateRay with explicit variates (include/core/camera.h:40-61). out: o[3], d[3]
void ref_camera_ray(const float* cam, int width, int height, int row, int col, float x1, float x2, float* out) {
    Camera c(Vec3(cam[0], cam[1], cam[2]), Vec3(cam[3], cam[4], cam[5]), Vec3(cam[6], cam[7], cam[8]), cam[9],
             Resolution{width, height}, cam[10] != 0.f);
    const Ray r = c.generateRay(row, col, make_float2(x1, x2));
    for (int k = 0; k < 3; k++) {
        out[k] = r.origin()[k];
        out[3 + k] = r.direction()[k];
    }
}

// The normals G-buffer's per-pixel value (g_buffer.cu:27-57) through the reference's own
// Camera::generateRay(row, col) and World::hit. out: width * height * 3, pixel = row * width + col.
void ref_normals(void* p, const float* cam, int width, int height, float* out) {
    RefScene* s = static_cast<RefScene*>(p);
    Camera c(Vec3(cam[0], cam[1], cam[2]), Vec3(cam[3], cam[4], cam[5]), Vec3(cam[6], cam[7], cam[8]), cam[9],
             Resolution{width, height}, cam[10] != 0.f);
    for (int row = 0; row < height; row++) {
        for (int col = 0; col < width; col++) {
            const Ray r = c.generateRay(row, col);
            HitRecord rec;
            const Vec3 v = s->world->hit(r, 0.f, FLT_MAX, rec) ? (rec.normal + 1.f) / 2.f : Vec3(0.f);
            for (int k = 0; k < 3; k++) out[3 * ((size_t)row * width + col) + k] = v[k];
        }
    }
}

// DistributionParams / Distribution (distribution.h:11-65, distribution.cu:19-55)
void ref_dist1d(const float* values, int n, const float* xis, int nxi, float* pmf_out, float* total_out, int* idx_out,
                float* spmf_out) {
    DistributionParams prm(std::vector<float>(values, values + n));
    const Distribution d = prm.createDistribution();
    for (int i = 0; i < n; i++) pmf_out[i] = d.pmf(i);
    *total_out = d.getTotalMass();
    for (int k = 0; k < nxi; k++) {
        float pm = 0.f;
        idx_out[k] = (int)d.sample(&pm, xis[k]);
        spmf_out[k] = pm;
    }
}

// Distribution2DBuilder / Distribution2D (distribution.h:80-131, distribution.cu:57-91)
void ref_dist2d(const float* values, int w, int h, const float* xis, int nxi, float* pmf_out, int* sx, int* sy,
                float* spmf) {
    Distribution2DBuilder b(values, w, h);
    const Distribution2D d = b.buildDistribution2D();
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) pmf_out[y * w + x] = d.pmf(x, y);
    for (int k = 0; k < nxi; k++) {
        float pm = 0.f;
        const Distribution2D::Sample smp = d.sample(&pm, make_float2(xis[2 * k], xis[2 * k + 1]));
        sx[k] = smp.x;
        sy[k] = smp.y;
        spmf[k] = pm;
    }
}

// PhiThetaDistribution pdfs (distribution.h:149-201)
void ref_phitheta_pdf(const float* values, int w, int h, const float* canon, int ncanon, float* pdf_canon,
                      const float* dirs, int ndirs, float* pdf_dir) {
    PhiThetaDistributionBuilder b(values, w, h);
    const PhiThetaDistribution d = b.buildPhiThetaDistribution();
    for (int k = 0; k < ncanon; k++) pdf_canon[k] = d.pdf(canon[2 * k], canon[2 * k + 1]);
    for (int k = 0; k < ndirs; k++) pdf_dir[k] = d.pdf(Vec3(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]));
}

// EnvironmentLight::sample + getEmit (environment_light.h:50-83). out: wi[3], pdf, emit[3]
void ref_env_sample(void* p, float x1, float x2, float* out) {
    RefScene* s = static_cast<RefScene*>(p);
    const EnvironmentLightSample smp = s->env.sample(Vec3(0.f), Frame(Vec3(0.f, 1.f, 0.f)), x1, x2);
    const Vec3 w = smp.occlusionRay.direction();
    const float v[7] = {w.x(), w.y(), w.z(), smp.pdf, smp.emitted.x(), smp.emitted.y(), smp.emitted.z()};
    std::memcpy(out, v, sizeof(v));
}

}  // extern "C"
