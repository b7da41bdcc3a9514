// Render session: owns the host scene, its BVH, every device buffer and the frame loop.
// The C ABI (capi.cpp) is a thin shell over this class.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/pathed.h"
#include "assets.h"
#include "bvh_build.h"
#include "bvh_gpu.h"
#include "devbuf.h"
#include "host_scene.h"
#include "host_util.h"
#include "wavefront.h"

namespace pt {

// Guide position-encoding frame from a scene's bounds.
GuideFrame guide_frame_of(const HostScene& s);

// Host state of one scene of a batch (configuration 4).
struct BatchHost {
    BatchSpec spec;
    CameraSpec camspec;
    int root = 0, light_first = 0, num_lights = 0;
    int num_tri = 0, num_sph = 0;
    long long path_base = 0, pixel_base = 0;
    long long guided_base = 0;  // paths of guided scenes before this one
    int env_w = 0, env_h = 0;
    std::vector<float> env_rgba;
    EnvCdf env_cdf;
    GuideFrame gframe{};
    int total_spp = 0;
};

// Allocate (grow) `b` and copy `v` into it on stream `st`.
template <class T>
cudaError_t upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
    cudaError_t e = b.alloc(v.size() * sizeof(T));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

class Session {
public:
    Session(int w, int h);
    ~Session();

    int width() const { return w_; }
    int height() const { return h_; }
    const std::string& error() const { return err_; }
    int fail(int code, const std::string& msg) {
        err_ = msg;
        return code;
    }

    int set_device(int dev);
    int load_config(int config, uint64_t seed, int level);
    int load_scene(HostScene&& s);
    // scene files (OBJ/MTL, PLY, EXR environment) with the given camera
    int load_request(const SceneRequest& r, const CameraSpec& cam);
    // the reference's built-in scene 0-3 from its scenes directory, with its camera and the
    // reference's defaults (max depth 3, NEE on)
    int load_reference_scene(int index, const std::string& scenes_dir);
    int set_bvh(int width, int max_leaf);
    int check_bvh();
    // 1: build the BVH on the GPU (Morton-order LBVH collapsed to the wide format) at the next
    // upload; 0: the host's binned-SAH builder (default)
    int set_bvh_builder(int gpu);
    // 1: traverse quantized nodes (widths 4 and 8; 64 / 96 B per node), 0: float nodes
    int set_bvh_nodes(int quantized);
    int check_quantized(const BvhBuild& b);
    int bvh_nodes_quantized() const { return bvh_quant_ && (bvh_.width == 4 || bvh_.width == 8) ? 1 : 0; }
    int counts(::pt_scene_counts* out) const;
    int export_scene(::pt_scene_export* out) const;

    int set_camera(const CameraSpec& c);
    int set_material(int id, int type, const float* albedo, const float* emit, float ior, float alpha);
    int set_max_depth(int d);
    int set_nee(int on);
    void set_seed(uint64_t s) { seed_ = s; reset(); }
    void reset() { reset_pending_ = true; }
    // PT_RENDERER_CUDA (path tracer) or PT_RENDERER_NORMALS (G-buffer: one pixel-centre ray
    // per pixel and frame); a change restarts accumulation, as RenderSession's switch does
    int set_renderer(int type);
    int renderer() const { return renderer_; }
    int set_launch(const ::pt_launch_config* c);
    void get_launch(::pt_launch_config* c) const;

    int render_async(int spp);
    int poll(int* done, float* ms);
    int wait(float* ms);
    int spp() const { return total_spp_; }
    int stats(::pt_stats* out) const;
    int set_profiling(int stage_timing, int work_counters);
    int profile(::pt_profile* out) const;

    int readback(float* rgb, size_t n, bool pass);
    int readback_async(float* rgb, size_t n);
    int readback_wait();
    int readback_rgba8(uint8_t* out, size_t n);
    int hit_test(int x, int y, int* mat);
    int trace_rays(const float* o, const float* d, const float* tmin, const float* tmax, int n, int* pt,
                   int* pid, int* mid, float* t, float* bary, bool device_ptrs);
    int occluded(const float* o, const float* d, const float* tmin, const float* tmax, int n, int* occ);
    // Allocation-free closest-hit queries (staging in a static device array); the scene must
    // already be resident on the device.
    int trace_rays_static(const float* o, const float* d, const float* tmin, const float* tmax, int n, int* pt,
                          int* pid, int* mid, float* t, float* bary);

    const HostScene& scene() const { return scene_; }
    const CameraSpec& camera_spec() const { return camspec_; }
    int max_depth() const { return max_depth_; }
    int nee() const { return nee_; }

private:
    int ensure_device();
    int upload_scene();
    int upload_materials();
    int ensure_frame_buffers(int spp);
    int check_cuda(cudaError_t e, const char* what);
    int finish_frame(float* ms);
    cudaError_t enqueue_frame_and_training(const FrameParams& p, StageMarks* marks);
    SceneDevice scene_view() const;

    int w_, h_;
    std::string err_;
    // host scene
    HostScene scene_;
    bool have_scene_ = false;
    BvhBuild bvh_;
    int bvh_width_ = 4, bvh_leaf_ = 4;
    EnvCdf env_cdf_;
    std::vector<LightRef> lights_;
    CameraSpec camspec_{};
    CameraParams cam_{};
    int max_depth_ = 3;  // include/scene.h:12
    int nee_ = 1;        // include/scene.h:28
    uint64_t seed_ = 0x5EEDULL;
    // device
    int device_ = -1;
    bool dev_ready_ = false;
    bool scene_dirty_ = true;
    bool mats_dirty_ = true;
    cudaStream_t stream_ = nullptr;
    // allocation-free queries (trace_rays_static): their own stream, so a query does not wait
    // behind a frame in flight on stream_ (the scene buffers it reads are written only by
    // uploads, which complete before the call that made them returns)
    cudaStream_t query_stream_ = nullptr;
    int num_sms_ = 0;
    size_t max_smem_ = 0;
    DevBuf d_qnodes_, d_qfail_;
    int bvh_quant_ = 0;
    DevBuf d_nodes_, d_prims_, d_tri_p_, d_tri_n_, d_tri_mat_, d_sph_, d_sph_mat_, d_mats_, d_lights_;
    DevBuf d_env_rgba_, d_env_marg_, d_env_cond_, d_env_row_;
    // frame state
    DevBuf d_pass_, d_accum_, d_rgba8_;
    DevBuf d_q_[2][6];
    DevBuf d_sq_[3];
    DevBuf d_L_, d_hitd_, d_sort_, d_counters_, d_stats_, d_scratch_;
    DevBuf d_rindex_, d_rhist_;  // ray sorting: slot order and bucket counts/cursors
    int queue_cap_ = 0;
    LaunchShape shape_;
    int wave_paths_ = 1 << 25;  // 32M paths in flight (about 7.4 GB of queues)
    int use_graph_ = 1;
    int total_spp_ = 0;
    bool reset_pending_ = true;
    bool in_flight_ = false;
    int inflight_spp_ = 0;
    cudaEvent_t ev_begin_ = nullptr, ev_end_ = nullptr;
    // side stream of the overlapped shadow stages, with a fork and a join event per depth
    cudaStream_t side_stream_ = nullptr;
    std::vector<cudaEvent_t> side_shaded_, side_shadowed_;
    std::vector<cudaStream_t> cls_streams_;
    std::vector<cudaEvent_t> cls_done_;
    cudaEvent_t cls_fork_ = nullptr;
    SideStream side_;
    // asynchronous readback: snapshot on stream_, device-to-host copy on copy_stream_
    cudaStream_t copy_stream_ = nullptr;
    cudaEvent_t rb_snap_ = nullptr, rb_done_ = nullptr;
    DevBuf d_rb_stage_;
    bool rb_pending_ = false;
    float last_ms_ = 0.f;
    int last_spp_ = 0;
    int frames_ = 0;
    FrameStats last_stats_{};
    FrameStats* h_stats_ = nullptr;  // pinned
    // profiling
    int stage_timing_ = 0;
    int work_counters_ = 0;
    int renderer_ = 0;
    std::vector<cudaEvent_t> mark_events_;
    std::vector<int> mark_stage_, mark_begin_;
    StageMarks marks_{};
    bool marks_active_ = false;
    float stage_ms_[kNumStages] = {};
    int stage_launches_[kNumStages] = {};
    int last_wave_paths_ = 0;
    size_t smem_configured_ = 48 * 1024;
    // per-frame constants (device) and their pinned staging copy
    DevBuf d_dyn_;
    FrameDyn* h_dyn_ = nullptr;
    // CUDA graph of one frame's launches, valid while the captured FrameParams are unchanged
    cudaGraphExec_t graph_exec_ = nullptr;
    FrameParams graph_params_{};
    bool graph_valid_ = false;
    int graph_captures_ = 0;
    // material sorting: 1 on, 0 off, -1 automatic (on when >= 3 material classes are present)
    int sort_mode_ = -1;
    int material_classes_ = 1;
    int class_mask_ = 1;  // material classes present (bit 0 miss, bit type + 1)
    void update_material_classes();

    // ---- learned path guiding ----
    bool guiding_ = false;
    int consistent_mis_ = 0;
    bool guide_alloc_ = false;
    DevBuf d_gw_, d_gwpack_, d_ggrad_, d_gm_, d_gv_, d_gwsum_, d_gmix_, d_grec_, d_grec_count_, d_gacc_, d_gring_,
        d_gring_count_;
    int guide_iters_ = 0;       // Adam steps taken
    int guide_warmup_ = 4;      // steps before the guide is used for sampling
    int guide_batch_ = 1 << 16;      // samples per Adam step
    int guide_steps_per_frame_ = 0;  // 0: automatic schedule
    float guide_lr_ = 3e-3f;
    uint64_t guide_seed_ = 0x9e11deULL;
    GuideFrame gframe_{};
    int ensure_guide();
    int bvh_gpu_ = 0;  // 0 host SAH, kGpuBvhLbvh, kGpuBvhPloc
    GpuBvhScratch gbvh_;
    int guide_nets_ = 1;
    int guide_ring_cap_ = 1 << 21;
    DevBuf d_gframes_;
    int wanted_guide_nets() const;
    // batch mode
    std::vector<BatchHost> batch_;
    std::vector<BatchSpec> batch_specs_;
    std::vector<WaveRange> batch_waves_;
    std::vector<std::unique_ptr<DevBuf[]>> d_batch_env_;  // per scene: rgba, marg, cond, row
    DevBuf d_batch_, d_batch_path_base_, d_batch_pixel_base_;
    BatchScene* h_batch_ = nullptr;  // pinned
    int batch_max_depth_ = 0;
    long long batch_pixels_ = 0, batch_paths_ = 0;
    void clear_batch();
    int upload_batch();
    int render_async_batch();
    int guide_init_weights();
    GuideDevice guide_view() const;

public:
    int graph_captures() const { return graph_captures_; }
    int autotune(int spp, const char* cache_path, ::pt_tune_result* out);
    int set_guiding(int on);
    int set_consistent_mis(int on) {
        consistent_mis_ = on ? 1 : 0;
        reset();
        return 0;
    }
    int guide_reset();
    int set_guide_options(int steps, int batch, float lr, int warmup) {
        if (batch > (1 << 21)) return fail(-1, "batch must be at most 2^21 samples");
        if (steps > 64) return fail(-1, "at most 64 Adam steps per frame");
        if (steps >= 0) guide_steps_per_frame_ = steps;
        if (batch > 0) guide_batch_ = batch;
        if (lr > 0.f) guide_lr_ = lr;
        if (warmup >= 0) guide_warmup_ = warmup;
        return 0;
    }
    int guide_info(::pt_guide_info* out) const;
    // guide inference on tcgen05 / TMEM (1) or on mma.sync (0)
    int set_guide_inference(int tc) {
        guide_infer_tc_ = tc != 0;
        return PT_OK;
    }
    bool guide_infer_tc_ = false;
    // guide training on tcgen05 / TMEM (1) or on mma.sync (0)
    int set_guide_training(int tc) {
        if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
        guide_train_tc_ = tc != 0;
        return PT_OK;
    }
    bool guide_train_tc_ = true;  // 64 us per 2^16-sample step against 95 us on mma.sync
    // probability of sampling the guide at a non-delta vertex (one-sample MIS), in (0, 1)
    int set_guide_fraction(float f) {
        if (!(f > 0.f && f < 1.f)) return fail(PT_ERR_ARG, "guide fraction must lie in (0, 1)");
        guide_frac_ = f;
        return PT_OK;
    }
    float guide_frac_ = 0.7f;

    // ---- batched frames (configuration 4): every scene rendered by one launch per stage ----
    int load_batch(const std::vector<BatchSpec>& specs);
    int batch_readback(int scene, float* rgb, size_t n, bool pass);
    int batch_info(int scene, ::pt_batch_info* out) const;
    bool batch_mode() const { return !batch_.empty(); }
    int num_batch_scenes() const { return (int)batch_.size(); }
    int guide_params(float* out, int n, bool set);
    int guide_forward(const float* x, int n, float* raw);
    int guide_gradients(const float* x, const float* wi, const float* w, int n, float* grad);
    int set_test_limits(int stack_entries, int mma_polls);
    int set_watertight(int on);

private:
    bool watertight_ = false;  // triangles take the watertight test (leaf entries hold vertices)
    // test hooks for the device-error paths (0: off): traversal stack entries per query, and
    // non-blocking polls of the first wait of each tensor-core inference layer
    int test_stack_cap_ = 0;
    int test_mma_polls_ = 0;
    int stack_entries() const {
        const int sd = bvh_.depth + 1;
        return test_stack_cap_ > 0 && test_stack_cap_ < sd ? test_stack_cap_ : sd;
    }
};

}  // namespace pt
