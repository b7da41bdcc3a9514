// extern "C" entry points of libpathed.so (declared in include/pathed.h).
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/pathed.h"
#include "assets.h"
#include "session.h"

struct pt_session {
    pt::Session impl;
    pt_session(int w, int h) : impl(w, h) {}
};

namespace {
thread_local std::string g_create_error;

template <class F>
int guarded(pt_session* s, F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return s ? s->impl.fail(PT_ERR_CUDA, "host allocation failed") : PT_ERR_CUDA;
    } catch (const std::exception& e) {
        return s ? s->impl.fail(PT_ERR_ARG, e.what()) : PT_ERR_ARG;
    }
}
// Material arrays of pt_scene_desc / pt_scene_request (absent arrays take defaults)
std::vector<pt::Material> materials_of(int n, const int* types, const float* albedo, const float* emit,
                                       const float* ior, const float* alpha) {
    std::vector<pt::Material> mats((size_t)n);
    for (int i = 0; i < n; i++) {
        pt::Material& m = mats[i];
        std::memset(&m, 0, sizeof(m));
        m.type = types[i];
        for (int k = 0; k < 3; k++) {
            m.albedo[k] = albedo ? albedo[3 * i + k] : 0.f;
            m.emit[k] = emit ? emit[3 * i + k] : 0.f;
        }
        m.ior = ior ? ior[i] : 1.f;
        m.alpha = alpha ? alpha[i] : 0.1f;
    }
    return mats;
}
}  // namespace

extern "C" {

const char* pt_version(void) { return "pathed-b200 0.1 (sm_100a)"; }

int pt_set_watertight(pt_session* s, int on) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.set_watertight(on); });
}

int pt_set_test_limits(pt_session* s, int stack_entries, int mma_polls) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.set_test_limits(stack_entries, mma_polls); });
}

int pt_measure_l2_read(int device, size_t bytes, int reps, int trials, double* gbs, double* ms) {
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = pt::measure_l2_read(bytes, reps, trials, gbs, ms);
    return e == cudaSuccess ? PT_OK : (e == cudaErrorInvalidValue ? PT_ERR_ARG : PT_ERR_CUDA);
}

int pt_create(int width, int height, pt_session** out) {
    if (!out) return PT_ERR_ARG;
    *out = nullptr;
    if (width <= 0 || height <= 0 || (long long)width * height > (1LL << 28)) {
        g_create_error = "resolution must be positive and at most 2^28 pixels";
        return PT_ERR_ARG;
    }
    try {
        *out = new pt_session(width, height);
    } catch (...) {
        g_create_error = "host allocation failed";
        return PT_ERR_CUDA;
    }
    return PT_OK;
}

int pt_destroy(pt_session* s) {
    delete s;
    return PT_OK;
}

const char* pt_last_error(const pt_session* s) {
    return s ? s->impl.error().c_str() : g_create_error.c_str();
}

int pt_set_device(pt_session* s, int device) {
    if (!s) return PT_ERR_ARG;
    return s->impl.set_device(device);
}

int pt_load_config(pt_session* s, int config, uint64_t seed) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.load_config(config, seed, -1); });
}

int pt_load_config_level(pt_session* s, int config, uint64_t seed, int level) {
    if (!s) return PT_ERR_ARG;
    if (level < 0 || level > 9) return s->impl.fail(PT_ERR_ARG, "icosphere level must be in [0, 9]");
    return guarded(s, [&] { return s->impl.load_config(config, seed, level); });
}

int pt_load_arrays(pt_session* s, const pt_scene_desc* d) {
    if (!s) return PT_ERR_ARG;
    if (!d) return s->impl.fail(PT_ERR_ARG, "null scene description");
    return guarded(s, [&]() -> int {
        pt::HostScene sc;
        if (d->num_triangles < 0 || d->num_spheres < 0 || d->num_materials <= 0)
            return s->impl.fail(PT_ERR_ARG, "negative counts or no materials");
        if (d->num_triangles > 0 && (!d->tri_vertices || !d->tri_materials))
            return s->impl.fail(PT_ERR_ARG, "triangle arrays missing");
        if (d->num_spheres > 0 && (!d->spheres || !d->sphere_materials))
            return s->impl.fail(PT_ERR_ARG, "sphere arrays missing");
        if (!d->material_types) return s->impl.fail(PT_ERR_ARG, "material types missing");
        const size_t nt = (size_t)d->num_triangles;
        sc.tri_p.assign(d->tri_vertices, d->tri_vertices + nt * 9);
        if (d->tri_normals) {
            sc.tri_n.assign(d->tri_normals, d->tri_normals + nt * 9);
        } else {
            sc.tri_n.resize(nt * 9);
            for (size_t i = 0; i < nt; i++) {
                const float* p = &sc.tri_p[i * 9];
                const float e1[3] = {p[3] - p[0], p[4] - p[1], p[5] - p[2]};
                const float e2[3] = {p[6] - p[0], p[7] - p[1], p[8] - p[2]};
                float n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                              e1[0] * e2[1] - e1[1] * e2[0]};
                const float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                for (int k = 0; k < 3; k++) n[k] = l > 0 ? n[k] / l : 0.f;
                for (int v = 0; v < 3; v++)
                    for (int k = 0; k < 3; k++) sc.tri_n[i * 9 + v * 3 + k] = n[k];
            }
        }
        sc.tri_mat.assign(d->tri_materials, d->tri_materials + nt);
        const size_t ns = (size_t)d->num_spheres;
        if (ns) {
            sc.sph.assign(d->spheres, d->spheres + ns * 4);
            sc.sph_mat.assign(d->sphere_materials, d->sphere_materials + ns);
        }
        sc.mats = materials_of(d->num_materials, d->material_types, d->material_albedo, d->material_emit,
                               d->material_ior, d->material_alpha);
        if (d->env_rgba) {
            if (d->env_width <= 0 || d->env_height <= 0)
                return s->impl.fail(PT_ERR_ARG, "environment map size must be positive");
            sc.env_w = d->env_width;
            sc.env_h = d->env_height;
            sc.env_rgba.assign(d->env_rgba, d->env_rgba + (size_t)d->env_width * d->env_height * 4);
        }
        sc.name = "arrays";
        return s->impl.load_scene(std::move(sc));
    });
}

int pt_load_request(pt_session* s, const pt_scene_request* r) {
    if (!s) return PT_ERR_ARG;
    if (!r) return s->impl.fail(PT_ERR_ARG, "null scene request");
    return guarded(s, [&]() -> int {
        if (r->num_files < 0 || r->num_spheres < 0 || r->num_materials <= 0 || !r->material_types)
            return s->impl.fail(PT_ERR_ARG, "negative counts or no materials");
        if ((r->num_files > 0 && !r->files) || (r->num_spheres > 0 && (!r->spheres || !r->sphere_materials)))
            return s->impl.fail(PT_ERR_ARG, "request arrays missing");
        if (!r->camera) return s->impl.fail(PT_ERR_ARG, "a camera is required");
        pt::SceneRequest q;
        for (int i = 0; i < r->num_files; i++) {
            if (!r->files[i].path) return s->impl.fail(PT_ERR_ARG, "mesh file without a path");
            q.files.push_back({r->files[i].path, r->files[i].format, r->files[i].default_material});
        }
        q.mats = materials_of(r->num_materials, r->material_types, r->material_albedo, r->material_emit,
                              r->material_ior, r->material_alpha);
        q.sph.assign(r->spheres, r->spheres + 4 * (size_t)r->num_spheres);
        q.sph_mat.assign(r->sphere_materials, r->sphere_materials + (size_t)r->num_spheres);
        if (r->env_exr) q.env_path = r->env_exr;
        pt::CameraSpec cam{};
        for (int k = 0; k < 3; k++) {
            cam.origin[k] = r->camera[k];
            cam.target[k] = r->camera[3 + k];
            cam.up[k] = r->camera[6 + k];
        }
        cam.vfov = r->camera[9];
        cam.flip = r->camera[10] != 0.f;
        return s->impl.load_request(q, cam);
    });
}

int pt_load_reference_scene(pt_session* s, int index, const char* scenes_dir) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.load_reference_scene(index, scenes_dir ? scenes_dir : ""); });
}

int pt_read_exr(const char* path, int* width, int* height, float* rgba, size_t n) {
    if (!path || !width || !height) {
        g_create_error = "pt_read_exr: null argument";
        return PT_ERR_ARG;
    }
    try {
        std::vector<float> img;
        std::string err;
        int w = 0, h = 0;
        if (!pt::read_exr(path, w, h, img, err)) {
            g_create_error = err;
            return PT_ERR_ARG;
        }
        *width = w;
        *height = h;
        if (rgba) {
            if (n < img.size()) {
                g_create_error = "pt_read_exr: destination holds fewer than width * height * 4 floats";
                return PT_ERR_ARG;
            }
            std::memcpy(rgba, img.data(), img.size() * sizeof(float));
        }
        return PT_OK;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return PT_ERR_ARG;
    }
}

int pt_save_exr(pt_session* s, const char* path) {
    if (!s) return PT_ERR_ARG;
    if (!path) return s->impl.fail(PT_ERR_ARG, "null path");
    return guarded(s, [&]() -> int {
        const int w = s->impl.width(), h = s->impl.height();
        std::vector<float> rgb((size_t)w * h * 3);
        const int r = s->impl.readback(rgb.data(), rgb.size(), false);
        if (r) return r;
        std::string err;
        if (!pt::write_exr(path, w, h, rgb.data(), err)) return s->impl.fail(PT_ERR_ARG, err);
        return PT_OK;
    });
}

int pt_write_exr(const char* path, int width, int height, const float* rgb) {
    if (!path || !rgb || width <= 0 || height <= 0) {
        g_create_error = "pt_write_exr: bad argument";
        return PT_ERR_ARG;
    }
    try {
        std::string err;
        if (!pt::write_exr(path, width, height, rgb, err)) {
            g_create_error = err;
            return PT_ERR_ARG;
        }
        return PT_OK;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return PT_ERR_ARG;
    }
}

int pt_scene_counts_get(const pt_session* s, pt_scene_counts* out) {
    if (!s || !out) return PT_ERR_ARG;
    return s->impl.counts(out);
}

int pt_export_scene(const pt_session* s, pt_scene_export* out) {
    if (!s || !out) return PT_ERR_ARG;
    return s->impl.export_scene(out);
}

int pt_set_bvh(pt_session* s, int width, int max_leaf) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.set_bvh(width, max_leaf); });
}

int pt_check_bvh(const pt_session* s) {
    if (!s) return PT_ERR_ARG;
    // a GPU-built tree is built (if still pending) and downloaded first: no visible state changes
    return const_cast<pt_session*>(s)->impl.check_bvh();
}

int pt_set_camera(pt_session* s, const float origin[3], const float target[3], const float up[3], float vfov,
                  int flip) {
    if (!s || !origin || !target || !up) return PT_ERR_ARG;
    pt::CameraSpec c;
    for (int k = 0; k < 3; k++) {
        c.origin[k] = origin[k];
        c.target[k] = target[k];
        c.up[k] = up[k];
    }
    c.vfov = vfov;
    c.flip = flip != 0;
    if (!(vfov > 0.f && vfov < 3.14159f)) return s->impl.fail(PT_ERR_ARG, "vertical field of view out of range");
    return s->impl.set_camera(c);
}

int pt_set_material(pt_session* s, int id, int type, const float albedo[3], const float emit[3], float ior,
                    float alpha) {
    if (!s) return PT_ERR_ARG;
    return s->impl.set_material(id, type, albedo, emit, ior, alpha);
}

int pt_set_max_depth(pt_session* s, int d) { return s ? s->impl.set_max_depth(d) : PT_ERR_ARG; }
int pt_set_nee(pt_session* s, int on) { return s ? s->impl.set_nee(on) : PT_ERR_ARG; }
int pt_set_seed(pt_session* s, uint64_t seed) {
    if (!s) return PT_ERR_ARG;
    s->impl.set_seed(seed);
    return PT_OK;
}
int pt_set_guiding(pt_session* s, int enabled) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.set_guiding(enabled); });
}
int pt_guide_reset(pt_session* s) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.guide_reset(); });
}
int pt_set_guide_options(pt_session* s, int steps_per_frame, int batch, float lr, int warmup_steps) {
    if (!s) return PT_ERR_ARG;
    return s->impl.set_guide_options(steps_per_frame, batch, lr, warmup_steps);
}
int pt_set_consistent_mis(pt_session* s, int enabled) {
    if (!s) return PT_ERR_ARG;
    return s->impl.set_consistent_mis(enabled);
}
int pt_guide_get_info(const pt_session* s, pt_guide_info* out) {
    if (!s || !out) return PT_ERR_ARG;
    return s->impl.guide_info(out);
}
int pt_guide_get_params(pt_session* s, float* out, int n) {
    if (!s || !out) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.guide_params(out, n, false); });
}
int pt_guide_set_params(pt_session* s, const float* in, int n) {
    if (!s || !in) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.guide_params(const_cast<float*>(in), n, true); });
}
int pt_guide_forward(pt_session* s, const float* x, int n, float* raw) {
    if (!s || (n > 0 && (!x || !raw))) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.guide_forward(x, n, raw); });
}
int pt_set_guide_fraction(pt_session* s, float fraction) {
    if (!s) return PT_ERR_ARG;
    return s->impl.set_guide_fraction(fraction);
}

int pt_set_guide_inference(pt_session* s, int tc) {
    if (!s) return PT_ERR_ARG;
    return s->impl.set_guide_inference(tc);
}
int pt_set_guide_training(pt_session* s, int tc) {
    if (!s) return PT_ERR_ARG;
    return s->impl.set_guide_training(tc);
}
int pt_guide_gradients(pt_session* s, const float* x, const float* wi, const float* w, int n, float* grad) {
    if (!s || !x || !wi || !w || !grad) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.guide_gradients(x, wi, w, n, grad); });
}
int pt_reset(pt_session* s) {
    if (!s) return PT_ERR_ARG;
    s->impl.reset();
    return PT_OK;
}
int pt_set_launch(pt_session* s, const pt_launch_config* c) {
    if (!s || !c) return PT_ERR_ARG;
    return s->impl.set_launch(c);
}
int pt_get_launch(const pt_session* s, pt_launch_config* c) {
    if (!s || !c) return PT_ERR_ARG;
    s->impl.get_launch(c);
    return PT_OK;
}

int pt_autotune(pt_session* s, int spp, const char* cache_path, pt_tune_result* out) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.autotune(spp, cache_path, out); });
}

int pt_render_async(pt_session* s, int spp) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.render_async(spp); });
}
int pt_poll(pt_session* s, int* done, float* ms) { return s ? s->impl.poll(done, ms) : PT_ERR_ARG; }
int pt_wait(pt_session* s, float* ms) { return s ? s->impl.wait(ms) : PT_ERR_ARG; }
int pt_get_spp(const pt_session* s, int* spp) {
    if (!s || !spp) return PT_ERR_ARG;
    *spp = s->impl.spp();
    return PT_OK;
}
int pt_get_stats(const pt_session* s, pt_stats* out) {
    if (!s || !out) return PT_ERR_ARG;
    return s->impl.stats(out);
}

int pt_set_profiling(pt_session* s, int stage_timing, int work_counters) {
    return s ? s->impl.set_profiling(stage_timing, work_counters) : PT_ERR_ARG;
}
int pt_get_profile(const pt_session* s, pt_profile* out) {
    if (!s || !out) return PT_ERR_ARG;
    return s->impl.profile(out);
}

int pt_readback(pt_session* s, float* rgb, size_t n) { return s ? s->impl.readback(rgb, n, false) : PT_ERR_ARG; }
int pt_readback_pass(pt_session* s, float* rgb, size_t n) { return s ? s->impl.readback(rgb, n, true) : PT_ERR_ARG; }
int pt_readback_async(pt_session* s, float* rgb, size_t n) {
    return s ? s->impl.readback_async(rgb, n) : PT_ERR_ARG;
}
int pt_readback_wait(pt_session* s) { return s ? s->impl.readback_wait() : PT_ERR_ARG; }
int pt_readback_rgba8(pt_session* s, uint8_t* rgba, size_t n) {
    return s ? s->impl.readback_rgba8(rgba, n) : PT_ERR_ARG;
}

int pt_hit_test(pt_session* s, int x, int y, int* material_id) {
    if (!s || !material_id) return PT_ERR_ARG;
    return s->impl.hit_test(x, y, material_id);
}

int pt_trace_rays(pt_session* s, const float* o, const float* d, const float* tmin, const float* tmax, int n,
                  int* prim_type, int* prim_id, int* mat_id, float* t, float* bary) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.trace_rays(o, d, tmin, tmax, n, prim_type, prim_id, mat_id, t, bary, false); });
}

int pt_trace_rays_device(pt_session* s, const float* o, const float* d, const float* tmin, const float* tmax, int n,
                         int* prim_type, int* prim_id, int* mat_id, float* t, float* bary) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.trace_rays(o, d, tmin, tmax, n, prim_type, prim_id, mat_id, t, bary, true); });
}

int pt_trace_rays_static(pt_session* s, const float* o, const float* d, const float* tmin, const float* tmax, int n,
                         int* prim_type, int* prim_id, int* mat_id, float* t, float* bary) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.trace_rays_static(o, d, tmin, tmax, n, prim_type, prim_id, mat_id, t, bary); });
}

int pt_occluded(pt_session* s, const float* o, const float* d, const float* tmin, const float* tmax, int n,
                int* occluded) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.occluded(o, d, tmin, tmax, n, occluded); });
}

int pt_set_bvh_builder(pt_session* s, int gpu) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.set_bvh_builder(gpu); });
}

int pt_set_bvh_nodes(pt_session* s, int quantized) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.set_bvh_nodes(quantized); });
}

int pt_set_renderer(pt_session* s, int kind) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.set_renderer(kind); });
}

int pt_batch_generate(unsigned long long seed, int n, pt_batch_scene* out) {
    if (n < 1 || n > pt::kMaxBatchScenes || !out) return PT_ERR_ARG;
    try {
        const std::vector<pt::BatchSpec> specs = pt::generate_batch_specs(seed, n);
        for (int i = 0; i < n; i++) {
            pt_batch_scene& o = out[i];
            std::memset(&o, 0, sizeof(o));
            o.config = specs[i].config;
            o.level = specs[i].level;
            o.seed = specs[i].seed;
            o.width = specs[i].width;
            o.height = specs[i].height;
            o.spp = specs[i].spp;
            o.max_depth = specs[i].max_depth;
            o.guided = specs[i].guided;
        }
    } catch (const std::exception&) {
        return PT_ERR_ARG;
    }
    return PT_OK;
}

int pt_load_batch(pt_session* s, const pt_batch_scene* scenes, int n) {
    if (!s) return PT_ERR_ARG;
    if (!scenes || n < 1) return s->impl.fail(PT_ERR_ARG, "empty batch");
    return guarded(s, [&] {
        std::vector<pt::BatchSpec> specs(n);
        for (int i = 0; i < n; i++) {
            specs[i].config = scenes[i].config;
            specs[i].level = scenes[i].level;
            specs[i].seed = scenes[i].seed;
            specs[i].width = scenes[i].width;
            specs[i].height = scenes[i].height;
            specs[i].spp = scenes[i].spp;
            specs[i].max_depth = scenes[i].max_depth;
            specs[i].guided = scenes[i].guided;
        }
        return s->impl.load_batch(specs);
    });
}

int pt_batch_get_info(const pt_session* s, int scene, pt_batch_info* out) {
    if (!s || !out) return PT_ERR_ARG;
    return s->impl.batch_info(scene, out);
}

int pt_batch_readback(pt_session* s, int scene, float* rgb, size_t n, int pass_only) {
    if (!s) return PT_ERR_ARG;
    return guarded(s, [&] { return s->impl.batch_readback(scene, rgb, n, pass_only != 0); });
}

}  // extern "C"
