// Batched frames (configuration 4): many scenes merged into one session so that every stage
// of the wavefront is one launch over the rays of all scenes.
//
// Merge: triangles, spheres, materials and emitters of the scenes are concatenated (ids
// offset per scene); each scene's BVH is built on its own and appended to one node / leaf
// entry array with its own root (append_bvh). Environments stay per scene. The device scene
// table (BatchScene) gives each path's scene its root, emitter range, environment, camera,
// resolution, spp, depth and guide network; queue entries carry the scene id.
#include <algorithm>
#include <cstring>
#include <future>

#include "session.h"

namespace pt {

void Session::clear_batch() {
    batch_.clear();
    batch_specs_.clear();
    batch_waves_.clear();
    d_batch_env_.clear();
    batch_pixels_ = batch_paths_ = 0;
    batch_max_depth_ = 0;
}

int Session::load_batch(const std::vector<BatchSpec>& specs) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    if (renderer_ != 0) return fail(PT_ERR_STATE, "batches render with the path tracer only");
    const int n = (int)specs.size();
    if (n < 1 || n > kMaxBatchScenes) return fail(PT_ERR_ARG, "a batch holds 1 to 64 scenes");
    long long paths = 0, pixels = 0;
    for (const BatchSpec& b : specs) {
        if (b.config < 0 || b.config > 3) return fail(PT_ERR_ARG, "batch scene configuration must be 0-3");
        if (b.width < 1 || b.height < 1 || b.width > 8192 || b.height > 8192)
            return fail(PT_ERR_ARG, "batch scene resolution out of range");
        if (b.spp < 1 || b.spp > 1024) return fail(PT_ERR_ARG, "batch scene spp must be 1-1024");
        if (b.max_depth < 0 || b.max_depth > kMaxDepthLimit) return fail(PT_ERR_ARG, "batch scene depth out of range");
        if (b.level > 9) return fail(PT_ERR_ARG, "batch scene icosphere level must be at most 9");
        pixels += (long long)b.width * b.height;
        paths += (long long)b.width * b.height * b.spp;
    }
    if (pixels > (1LL << 31) - 1) return fail(PT_ERR_ARG, "batch has too many pixels");
    // generate and build every scene (independent: in parallel)
    std::vector<HostScene> scenes(n);
    std::vector<BvhBuild> bvhs(n);
    std::vector<std::string> errs(n);
    std::vector<int> ok(n, 0);
    {
        std::vector<std::future<void>> jobs;
        for (int i = 0; i < n; i++) {
            jobs.push_back(std::async(std::launch::async, [&, i]() {
                if (!generate_config(specs[i].config, specs[i].seed, scenes[i], errs[i], specs[i].level)) return;
                finalize_materials(scenes[i]);
                if (!validate_scene(scenes[i], errs[i])) return;
                if (!build_bvh(scenes[i], bvh_width_, bvh_leaf_, bvhs[i], errs[i])) return;
                ok[i] = 1;
            }));
        }
        for (auto& j : jobs) j.get();
    }
    for (int i = 0; i < n; i++)
        if (!ok[i]) return fail(PT_ERR_SCENE, "batch scene " + std::to_string(i) + ": " + errs[i]);
    HostScene merged;
    BvhBuild mb;
    mb.width = bvh_width_;
    std::vector<LightRef> lights;
    std::vector<BatchHost> hosts(n);
    long long path_base = 0, pixel_base = 0, guided_base = 0;
    int max_depth = 0;
    for (int i = 0; i < n; i++) {
        HostScene& sc = scenes[i];
        BatchHost& h = hosts[i];
        const int tri_base = merged.num_tri(), sph_base = merged.num_sph(), mat_base = (int)merged.mats.size();
        merged.tri_p.insert(merged.tri_p.end(), sc.tri_p.begin(), sc.tri_p.end());
        merged.tri_n.insert(merged.tri_n.end(), sc.tri_n.begin(), sc.tri_n.end());
        for (int m : sc.tri_mat) merged.tri_mat.push_back(m + mat_base);
        merged.sph.insert(merged.sph.end(), sc.sph.begin(), sc.sph.end());
        for (int m : sc.sph_mat) merged.sph_mat.push_back(m + mat_base);
        merged.mats.insert(merged.mats.end(), sc.mats.begin(), sc.mats.end());
        h.spec = specs[i];
        h.camspec = sc.camera;
        h.root = append_bvh(bvhs[i], tri_base, sph_base, mb);
        h.num_tri = sc.num_tri();
        h.num_sph = sc.num_sph();
        h.light_first = (int)lights.size();
        for (LightRef l : build_light_list(sc)) {
            l.index += l.type == kTriangle ? tri_base : sph_base;
            lights.push_back(l);
        }
        h.num_lights = (int)lights.size() - h.light_first;
        if (sc.env_w > 0) {
            h.env_w = sc.env_w;
            h.env_h = sc.env_h;
            h.env_rgba = std::move(sc.env_rgba);
            build_env_cdf(h.env_rgba.data(), h.env_w, h.env_h, h.env_cdf);
        }
        h.gframe = guide_frame_of(sc);
        h.path_base = path_base;
        h.pixel_base = pixel_base;
        h.guided_base = guided_base;
        if (specs[i].guided) guided_base += (long long)specs[i].width * specs[i].height * specs[i].spp;
        path_base += (long long)specs[i].width * specs[i].height * specs[i].spp;
        pixel_base += (long long)specs[i].width * specs[i].height;
        max_depth = std::max(max_depth, specs[i].max_depth);
        sc = HostScene();  // release the scene's copy
        bvhs[i] = BvhBuild();
    }
    merged.camera = hosts[0].camspec;
    merged.res_x = specs[0].width;
    merged.res_y = specs[0].height;
    merged.default_spp = specs[0].spp;
    merged.default_depth = max_depth;
    merged.default_nee = true;
    merged.name = "batch-" + std::to_string(n);
    scene_ = std::move(merged);
    bvh_ = std::move(mb);
    lights_ = std::move(lights);
    env_cdf_ = EnvCdf();
    batch_ = std::move(hosts);
    batch_specs_ = specs;
    batch_pixels_ = pixels;
    batch_paths_ = paths;
    batch_max_depth_ = max_depth;
    batch_waves_.clear();
    d_batch_env_.clear();
    have_scene_ = true;
    scene_dirty_ = true;
    mats_dirty_ = true;
    update_material_classes();
    gframe_ = guide_frame_of(scene_);
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
    }
    graph_valid_ = false;
    reset();
    return PT_OK;
}

// Per-scene environments and the scene table (static fields; per-frame fields are rewritten
// before every frame).
int Session::upload_batch() {
    int r;
    const int n = (int)batch_.size();
    d_batch_env_.clear();
    for (int i = 0; i < n; i++) {
        d_batch_env_.emplace_back(new DevBuf[4]);
        const BatchHost& h = batch_[i];
        if (h.env_w > 0) {
            DevBuf* e = d_batch_env_.back().get();
            if ((r = check_cuda(upload(e[0], h.env_rgba, stream_), "upload environment"))) return r;
            if ((r = check_cuda(upload(e[1], h.env_cdf.marg, stream_), "upload environment CDF"))) return r;
            if ((r = check_cuda(upload(e[2], h.env_cdf.cond, stream_), "upload environment CDF"))) return r;
            if ((r = check_cuda(upload(e[3], h.env_cdf.row_mass, stream_), "upload environment CDF"))) return r;
        }
    }
    if (!h_batch_ && (r = check_cuda(cudaMallocHost((void**)&h_batch_, kMaxBatchScenes * sizeof(BatchScene)),
                                     "cudaMallocHost")))
        return r;
    std::vector<long long> pb(n + 1), xb(n + 1);
    for (int i = 0; i < n; i++) {
        const BatchHost& h = batch_[i];
        BatchScene& b = h_batch_[i];
        std::memset(&b, 0, sizeof(b));
        b.root = h.root;
        b.light_first = h.light_first;
        b.num_lights = h.num_lights;
        b.width = h.spec.width;
        b.height = h.spec.height;
        b.spp = h.spec.spp;
        b.max_depth = h.spec.max_depth;
        b.guide_net = -1;
        b.path_base = h.path_base;
        b.pixel_base = h.pixel_base;
        b.guided_base = h.guided_base;
        if (h.env_w > 0) {
            const DevBuf* e = d_batch_env_[i].get();
            b.env.rgba = e[0].as<float>();
            b.env.marg_cdf = e[1].as<float>();
            b.env.cond_cdf = e[2].as<float>();
            b.env.row_mass = e[3].as<float>();
            b.env.width = h.env_w;
            b.env.height = h.env_h;
            b.env.total_mass = h.env_cdf.total;
            b.env.present = 1;
        }
        b.gframe = h.gframe;
        std::string err;
        if (!make_camera(h.camspec, h.spec.width, h.spec.height, b.cam, err))
            return fail(PT_ERR_SCENE, "batch scene " + std::to_string(i) + ": " + err);
        b.seed = seed_;
        pb[i] = h.path_base;
        xb[i] = h.pixel_base;
    }
    pb[n] = batch_paths_;
    xb[n] = batch_pixels_;
    if ((r = check_cuda(d_batch_.alloc(kMaxBatchScenes * sizeof(BatchScene)), "batch scene table"))) return r;
    if ((r = check_cuda(upload(d_batch_path_base_, pb, stream_), "batch offsets"))) return r;
    if ((r = check_cuda(upload(d_batch_pixel_base_, xb, stream_), "batch offsets"))) return r;
    return check_cuda(cudaStreamSynchronize(stream_), "batch upload");
}

int Session::batch_readback(int scene, float* rgb, size_t n, bool pass) {
    if (!batch_mode()) return fail(PT_ERR_STATE, "no batch loaded");
    if (scene < 0 || scene >= (int)batch_.size()) return fail(PT_ERR_ARG, "batch scene index out of range");
    const BatchHost& h = batch_[scene];
    const size_t need = (size_t)h.spec.width * h.spec.height * 3;
    if (!rgb || n < need) return fail(PT_ERR_ARG, "buffer too small");
    int r;
    if (in_flight_ && (r = wait(nullptr))) return r;
    const DevBuf& src = pass ? d_pass_ : d_accum_;
    if (!src.p || frames_ == 0) {
        std::memset(rgb, 0, need * sizeof(float));
        return PT_OK;
    }
    return check_cuda(cudaMemcpy(rgb, src.as<float>() + h.pixel_base * 3, need * sizeof(float),
                                 cudaMemcpyDeviceToHost),
                      "batch readback");
}

int Session::batch_info(int scene, pt_batch_info* out) const {
    if (!batch_mode()) return PT_ERR_STATE;
    if (scene < 0 || scene >= (int)batch_.size() || !out) return PT_ERR_ARG;
    const BatchHost& h = batch_[scene];
    out->num_triangles = h.num_tri;
    out->num_spheres = h.num_sph;
    out->num_lights = h.num_lights;
    out->width = h.spec.width;
    out->height = h.spec.height;
    out->spp = h.spec.spp;
    out->max_depth = h.spec.max_depth;
    out->guided = h.spec.guided;
    out->spp_accumulated = h.total_spp;
    out->first_pixel = h.pixel_base;
    out->first_path = h.path_base;
    return PT_OK;
}

}  // namespace pt
