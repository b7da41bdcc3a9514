#include "session.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/pathed.h"

#ifndef PT_GUIDE_TRAIN_PATHS
#define PT_GUIDE_TRAIN_PATHS 524288
#endif
#ifndef PT_GUIDE_TRAIN_PATHS_BATCH
#define PT_GUIDE_TRAIN_PATHS_BATCH 4194304
#endif

namespace pt {

namespace {
constexpr int kMaxStackBytesDefault = 48 * 1024;

// pt_launch_config.speculate (1 both stages, 2 off, 3 closest hit, 4 shadow) <-> kSpeculate* bits
int speculate_bits(int code) {
    return code == 1 ? kSpeculateExtend | kSpeculateShadow : code == 3 ? kSpeculateExtend
                                                           : code == 4 ? kSpeculateShadow
                                                                       : 0;
}
int speculate_code(int bits) {
    return bits == (kSpeculateExtend | kSpeculateShadow) ? 1 : bits == kSpeculateExtend ? 3
                                                           : bits == kSpeculateShadow   ? 4
                                                                                        : 2;
}
}  // namespace

Session::Session(int w, int h) : w_(w), h_(h) {
    // Reference default camera of scene 0 (src/scene.cu:176-184).
    camspec_ = {{0.f, 1.f, 6.8f}, {0.f, 1.f, 0.f}, {0.f, 1.f, 0.f}, (float)(19.5f / 180.f * M_PI), false};
}

Session::~Session() {
    if (dev_ready_) {
        cudaSetDevice(device_);
        if (stream_) cudaStreamSynchronize(stream_);
        if (copy_stream_) {
            cudaStreamSynchronize(copy_stream_);
            cudaStreamDestroy(copy_stream_);
        }
        if (rb_snap_) cudaEventDestroy(rb_snap_);
        if (rb_done_) cudaEventDestroy(rb_done_);
        if (ev_begin_) cudaEventDestroy(ev_begin_);
        if (ev_end_) cudaEventDestroy(ev_end_);
        if (side_stream_) {
            cudaStreamSynchronize(side_stream_);
            cudaStreamDestroy(side_stream_);
        }
        for (cudaEvent_t e : side_shaded_)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : side_shadowed_)
            if (e) cudaEventDestroy(e);
        for (cudaStream_t c : cls_streams_)
            if (c) {
                cudaStreamSynchronize(c);
                cudaStreamDestroy(c);
            }
        for (cudaEvent_t e : cls_done_)
            if (e) cudaEventDestroy(e);
        if (cls_fork_) cudaEventDestroy(cls_fork_);
        for (cudaEvent_t e : mark_events_) cudaEventDestroy(e);
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (h_dyn_) cudaFreeHost(h_dyn_);
        if (h_batch_) cudaFreeHost(h_batch_);
        if (stream_) cudaStreamDestroy(stream_);
        if (query_stream_) {
            cudaStreamSynchronize(query_stream_);
            cudaStreamDestroy(query_stream_);
        }
        if (h_stats_) cudaFreeHost(h_stats_);
    }
}

int Session::check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PT_OK;
    cudaGetLastError();
    return fail(PT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int Session::set_device(int dev) {
    if (dev_ready_) return fail(PT_ERR_STATE, "device already selected for this session");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || dev < 0 || dev >= n) {
        cudaGetLastError();
        return fail(PT_ERR_ARG, "no CUDA device with index " + std::to_string(dev));
    }
    device_ = dev;
    return PT_OK;
}

int Session::ensure_device() {
    if (dev_ready_) return check_cuda(cudaSetDevice(device_), "cudaSetDevice");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(PT_ERR_CUDA, "no CUDA device available (the CUDA path has no CPU fallback)");
    }
    if (device_ < 0) {
        if (cudaGetDevice(&device_) != cudaSuccess) device_ = 0;
    }
    int r;
    if ((r = check_cuda(cudaSetDevice(device_), "cudaSetDevice"))) return r;
    cudaDeviceProp prop;
    if ((r = check_cuda(cudaGetDeviceProperties(&prop, device_), "cudaGetDeviceProperties"))) return r;
    num_sms_ = prop.multiProcessorCount;
    max_smem_ = prop.sharedMemPerBlockOptin;
    if ((r = check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate"))) return r;
    if ((r = check_cuda(cudaStreamCreateWithFlags(&query_stream_, cudaStreamNonBlocking), "cudaStreamCreate")))
        return r;
    if ((r = check_cuda(cudaEventCreate(&ev_begin_), "cudaEventCreate"))) return r;
    if ((r = check_cuda(cudaEventCreate(&ev_end_), "cudaEventCreate"))) return r;
    if ((r = check_cuda(cudaStreamCreateWithFlags(&side_stream_, cudaStreamNonBlocking), "cudaStreamCreate")))
        return r;
    side_shaded_.assign(kMaxDepthLimit, nullptr);
    side_shadowed_.assign(kMaxDepthLimit, nullptr);
    for (int d = 0; d < kMaxDepthLimit; d++) {
        if ((r = check_cuda(cudaEventCreateWithFlags(&side_shaded_[d], cudaEventDisableTiming), "cudaEventCreate")))
            return r;
        if ((r = check_cuda(cudaEventCreateWithFlags(&side_shadowed_[d], cudaEventDisableTiming), "cudaEventCreate")))
            return r;
    }
    cls_streams_.assign(kMaterialClasses, nullptr);
    cls_done_.assign(kMaterialClasses, nullptr);
    for (int c = 0; c < kMaterialClasses; c++) {
        if ((r = check_cuda(cudaStreamCreateWithFlags(&cls_streams_[c], cudaStreamNonBlocking), "cudaStreamCreate")))
            return r;
        if ((r = check_cuda(cudaEventCreateWithFlags(&cls_done_[c], cudaEventDisableTiming), "cudaEventCreate")))
            return r;
    }
    if ((r = check_cuda(cudaEventCreateWithFlags(&cls_fork_, cudaEventDisableTiming), "cudaEventCreate"))) return r;
    side_ = SideStream{side_stream_, side_shaded_.data(), side_shadowed_.data(), cls_streams_.data(), cls_fork_,
                       cls_done_.data()};
    if ((r = check_cuda(cudaMallocHost((void**)&h_stats_, sizeof(FrameStats)), "cudaMallocHost"))) return r;
    std::memset(h_stats_, 0, sizeof(FrameStats));
    if ((r = check_cuda(d_counters_.alloc(sizeof(WaveCounters)), "counters"))) return r;
    if ((r = check_cuda(d_stats_.alloc(sizeof(FrameStats)), "stats"))) return r;
    if ((r = check_cuda(d_dyn_.alloc(sizeof(FrameDyn)), "frame constants"))) return r;
    if ((r = check_cuda(cudaMallocHost((void**)&h_dyn_, sizeof(FrameDyn)), "cudaMallocHost"))) return r;
    dev_ready_ = true;
    return PT_OK;
}

void Session::update_material_classes() {
    bool seen[8] = {false};
    for (int m : scene_.tri_mat) seen[scene_.mats[m].type & 7] = true;
    for (int m : scene_.sph_mat) seen[scene_.mats[m].type & 7] = true;
    material_classes_ = 0;
    class_mask_ = 1;  // misses
    for (int t = 0; t < 8; t++)
        if (seen[t]) {
            material_classes_++;
            if (t + 1 < 8) class_mask_ |= 1 << (t + 1);
        }
}

int Session::load_config(int config, uint64_t seed, int level) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    HostScene s;
    std::string err;
    if (!generate_config(config, seed, s, err, level)) return fail(PT_ERR_ARG, err);
    const CameraSpec cam = s.camera;
    const int depth = s.default_depth;
    const int nee = s.default_nee ? 1 : 0;
    int r = load_scene(std::move(s));
    if (r) return r;
    camspec_ = cam;
    max_depth_ = depth;
    nee_ = nee;
    return PT_OK;
}

int Session::load_request(const SceneRequest& r, const CameraSpec& cam) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    HostScene s;
    std::string err;
    if (!build_request(r, s, err)) return fail(PT_ERR_SCENE, err);
    s.name = "request";
    const int rc = load_scene(std::move(s));
    if (rc) return rc;
    camspec_ = cam;
    return PT_OK;
}

int Session::load_reference_scene(int index, const std::string& scenes_dir) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    HostScene s;
    std::string err;
    if (index < 0 || index > 3) return fail(PT_ERR_ARG, "reference scene index must be 0-3");
    if (!reference_scene(index, scenes_dir, s, err)) return fail(PT_ERR_SCENE, err);
    const CameraSpec cam = s.camera;
    const int rc = load_scene(std::move(s));
    if (rc) return rc;
    camspec_ = cam;
    max_depth_ = scene_.default_depth;
    nee_ = scene_.default_nee ? 1 : 0;
    return PT_OK;
}

int Session::load_scene(HostScene&& s) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    std::string err;
    finalize_materials(s);
    if (!validate_scene(s, err)) return fail(PT_ERR_SCENE, err);
    BvhBuild b;
    b.width = bvh_width_;
    if (!bvh_gpu_ && !build_bvh(s, bvh_width_, bvh_leaf_, b, err)) return fail(PT_ERR_SCENE, err);
    if (bvh_gpu_ && s.num_tri() + s.num_sph() == 0) return fail(PT_ERR_SCENE, "scene has no primitives");
    scene_ = std::move(s);
    bvh_ = std::move(b);
    lights_ = build_light_list(scene_);
    env_cdf_ = EnvCdf();
    if (scene_.env_w > 0) build_env_cdf(scene_.env_rgba.data(), scene_.env_w, scene_.env_h, env_cdf_);
    have_scene_ = true;
    scene_dirty_ = true;
    mats_dirty_ = true;
    update_material_classes();
    gframe_ = guide_frame_of(scene_);
    clear_batch();
    reset();
    return PT_OK;
}

GuideFrame guide_frame_of(const HostScene& s) {
    // scene bounds for the guide's position encoding
    GuideFrame g{};
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (size_t i = 0; i < s.tri_p.size(); i += 3)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], s.tri_p[i + k]);
            hi[k] = std::max(hi[k], s.tri_p[i + k]);
        }
    for (int j = 0; j < s.num_sph(); j++)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], s.sph[4 * j + k] - s.sph[4 * j + 3]);
            hi[k] = std::max(hi[k], s.sph[4 * j + k] + s.sph[4 * j + 3]);
        }
    for (int k = 0; k < 3; k++) {
        const float ext = std::max(hi[k] - lo[k], 1e-6f);
        g.lo[k] = lo[k];
        g.inv_ext[k] = 2.f / ext;
    }
    return g;
}

GuideDevice Session::guide_view() const {
    GuideDevice g{};
    g.w = d_gw_.as<float>();
    g.wpack = d_gwpack_.as<uint32_t>();
    g.grad = d_ggrad_.as<float>();
    g.adam_m = d_gm_.as<float>();
    g.adam_v = d_gv_.as<float>();
    g.wsum = d_gwsum_.as<float>();
    g.step = reinterpret_cast<int*>(d_gwsum_.as<float>() + 3);
    g.num_sms = num_sms_;
    g.nets = guide_nets_;
    g.train_tc = guide_train_tc_ ? 1 : 0;
    g.frame = gframe_;
    g.frames = guide_nets_ > 1 || batch_mode() ? d_gframes_.as<GuideFrame>() : nullptr;
    return g;
}

// Networks a frame needs: one per guided scene of a batch, else one.
int Session::wanted_guide_nets() const {
    if (!batch_mode()) return 1;
    int n = 0;
    for (const BatchHost& b : batch_) n += b.spec.guided ? 1 : 0;
    return std::max(1, n);
}

int Session::guide_init_weights() {
    // He-normal initialisation from a seeded generator; zero biases; the output layer starts
    // small so that the first mixture is broad (kappa about 1) and evenly weighted. Network k
    // of a batch continues the generator of network k - 1.
    std::vector<float> w((size_t)kGuideParams * guide_nets_, 0.f);
    uint64_t s = guide_seed_;
    auto next = [&]() {
        s += 0x9E3779B97F4A7C15ULL;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return (double)((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    auto normal = [&]() {
        const double u1 = std::max(next(), 1e-300), u2 = next();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    auto fill = [&](int off, int fan_in, int count, double scale) {
        const double sd = std::sqrt(2.0 / fan_in) * scale;
        for (int i = 0; i < count; i++) w[off + i] = (float)(normal() * sd);
    };
    for (int net = 0; net < guide_nets_; net++) {
        const int base = net * kGuideParams;
        fill(base + kGW1, kGuideIn, kGuideIn * kGuideHidden, 1.0);
        fill(base + kGW2, kGuideHidden, kGuideHidden * kGuideHidden, 1.0);
        fill(base + kGW3, kGuideHidden, kGuideHidden * kGuideHidden, 1.0);
        fill(base + kGW4, kGuideHidden, kGuideHidden * kGuideOut, 0.1);
        for (int j = 0; j < kGuideLobes; j++) {  // mean directions spread by the bias
            const double z = 2.0 * next() - 1.0, ph = 6.283185307179586 * next(), r = std::sqrt(1 - z * z);
            w[base + kGB4 + 5 * j] = (float)(r * std::cos(ph));
            w[base + kGB4 + 5 * j + 1] = (float)(r * std::sin(ph));
            w[base + kGB4 + 5 * j + 2] = (float)z;
        }
    }
    const size_t pbytes = (size_t)kGuideParams * 4 * guide_nets_;
    int r;
    if ((r = check_cuda(cudaMemcpyAsync(d_gw_.p, w.data(), pbytes, cudaMemcpyHostToDevice, stream_), "guide weights")))
        return r;
    if ((r = check_cuda(cudaMemsetAsync(d_ggrad_.p, 0, pbytes, stream_), "guide"))) return r;
    if ((r = check_cuda(cudaMemsetAsync(d_gm_.p, 0, pbytes, stream_), "guide"))) return r;
    if ((r = check_cuda(cudaMemsetAsync(d_gv_.p, 0, pbytes, stream_), "guide"))) return r;
    if ((r = check_cuda(cudaMemsetAsync(d_gring_count_.p, 0, sizeof(int) * guide_nets_, stream_), "guide"))) return r;
    // weight sums, losses and step counters (4 words per network)
    if ((r = check_cuda(cudaMemsetAsync(d_gwsum_.p, 0, 16 * guide_nets_, stream_), "guide"))) return r;
    if (batch_mode()) {  // per-network position-encoding frames: the guided scenes' bounds
        std::vector<GuideFrame> frames;
        for (const BatchHost& b : batch_)
            if (b.spec.guided) frames.push_back(b.gframe);
        if (frames.empty()) frames.push_back(gframe_);
        if ((r = check_cuda(upload(d_gframes_, frames, stream_), "guide frames"))) return r;
    }
    if ((r = check_cuda(guide_pack(guide_view(), stream_), "guide pack"))) return r;
    guide_iters_ = 0;
    return check_cuda(cudaStreamSynchronize(stream_), "guide init");
}

int Session::ensure_guide() {
    int r;
    if ((r = ensure_device())) return r;
    const int nets = wanted_guide_nets();
    if (!guide_alloc_ || nets != guide_nets_) {
        guide_nets_ = nets;
        guide_ring_cap_ = nets > 1 ? 1 << 20 : 1 << 21;
        const size_t pbytes = (size_t)kGuideParams * 4 * nets;
        if ((r = check_cuda(d_gw_.alloc(pbytes), "guide"))) return r;
        if ((r = check_cuda(d_gwpack_.alloc((size_t)kGuidePackWords * 4 * nets), "guide"))) return r;
        if ((r = check_cuda(d_ggrad_.alloc(pbytes), "guide"))) return r;
        if ((r = check_cuda(d_gm_.alloc(pbytes), "guide"))) return r;
        if ((r = check_cuda(d_gv_.alloc(pbytes), "guide"))) return r;
        if ((r = check_cuda(d_gwsum_.alloc(16 * nets), "guide"))) return r;
        if ((r = check_cuda(d_grec_count_.alloc(16), "guide"))) return r;
        if ((r = check_cuda(configure_guide_infer(), "guide inference configuration"))) return r;
        if ((r = check_cuda(guide_configure(), "guide training configuration"))) return r;
        if ((r = check_cuda(d_gring_.alloc((size_t)guide_ring_cap_ * nets * sizeof(GuideSample)), "guide samples")))
            return r;
        if ((r = check_cuda(d_gring_count_.alloc(4 * nets), "guide"))) return r;
        guide_alloc_ = true;
        if ((r = guide_init_weights())) return r;
    }
    return PT_OK;
}

int Session::set_guiding(int on) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    if (on) {
        int r;
        if ((r = ensure_guide())) return r;
    }
    guiding_ = on != 0;
    reset();
    return PT_OK;
}

int Session::guide_reset() {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    int r;
    if ((r = ensure_guide())) return r;
    if ((r = guide_init_weights())) return r;
    reset();
    return PT_OK;
}

int Session::guide_info(pt_guide_info* out) const {
    std::memset(out, 0, sizeof(*out));
    out->enabled = guiding_ ? 1 : 0;
    out->mode = !guiding_ ? 0 : guide_iters_ >= guide_warmup_ ? 2 : 1;
    out->steps = guide_iters_;
    out->params = kGuideParams;
    if (guide_alloc_) {
        int c = 0;
        float ws[2] = {0.f, 0.f};
        cudaMemcpy(&c, d_gring_count_.p, sizeof(int), cudaMemcpyDeviceToHost);
        cudaMemcpy(ws, d_gwsum_.p, sizeof(ws), cudaMemcpyDeviceToHost);
        out->samples = (unsigned long long)(unsigned)c;
        out->loss = ws[1];
    }
    return PT_OK;
}

int Session::guide_params(float* out, int n, bool set) {
    if (n != kGuideParams) return fail(PT_ERR_ARG, "parameter count must be 16104");
    int r;
    if ((r = ensure_guide())) return r;
    if (in_flight_ && (r = wait(nullptr))) return r;
    if (set) {
        if ((r = check_cuda(cudaMemcpyAsync(d_gw_.p, out, n * 4, cudaMemcpyHostToDevice, stream_), "guide params")))
            return r;
        if ((r = check_cuda(guide_pack(guide_view(), stream_), "guide pack"))) return r;
    } else if ((r = check_cuda(cudaMemcpyAsync(out, d_gw_.p, n * 4, cudaMemcpyDeviceToHost, stream_), "guide params"))) {
        return r;
    }
    return check_cuda(cudaStreamSynchronize(stream_), "guide params");
}

int Session::set_watertight(int on) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    if ((on != 0) == watertight_) return PT_OK;
    watertight_ = on != 0;
    scene_dirty_ = true;     // leaf entries re-uploaded in the test's format
    reset_pending_ = true;   // another intersection test: a new image
    return PT_OK;
}

int Session::set_test_limits(int stack_entries, int mma_polls) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    if (stack_entries < 0 || mma_polls < 0) return fail(PT_ERR_ARG, "limits must be >= 0 (0: none)");
    test_stack_cap_ = stack_entries;
    test_mma_polls_ = mma_polls;
    return PT_OK;
}

int Session::guide_forward(const float* x, int n, float* raw) {
    if (n < 0) return fail(PT_ERR_ARG, "negative count");
    int r;
    if ((r = ensure_guide())) return r;
    if (in_flight_ && (r = wait(nullptr))) return r;
    if (n == 0) return PT_OK;
    if ((r = check_cuda(d_scratch_.alloc((size_t)n * (kGuideIn + kGuideOut) * 4 + 16), "scratch"))) return r;
    float* dx = d_scratch_.as<float>();
    float* dy = dx + (size_t)n * kGuideIn;
    int* derr = reinterpret_cast<int*>(dy + (size_t)n * kGuideOut);
    if ((r = check_cuda(cudaMemcpyAsync(dx, x, (size_t)n * kGuideIn * 4, cudaMemcpyHostToDevice, stream_), "copy")))
        return r;
    if ((r = check_cuda(cudaMemsetAsync(derr, 0, sizeof(int), stream_), "copy"))) return r;
    const cudaError_t e = guide_infer_tc_ ? guide_forward_features_tc(guide_view(), dx, n, dy, derr, stream_,
                                                                      test_mma_polls_)
                                          : guide_forward_features(guide_view(), dx, n, dy, stream_);
    if ((r = check_cuda(e, "guide forward"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(raw, dy, (size_t)n * kGuideOut * 4, cudaMemcpyDeviceToHost, stream_), "copy")))
        return r;
    int herr = 0;
    if ((r = check_cuda(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy"))) return r;
    if ((r = check_cuda(cudaStreamSynchronize(stream_), "guide forward"))) return r;
    if (herr) return fail(PT_ERR_DEVICE, "tensor-core inference: a wait for the MMA completion gave up");
    return PT_OK;
}

int Session::guide_gradients(const float* x, const float* wi, const float* w, int n, float* grad) {
    if (n <= 0) return fail(PT_ERR_ARG, "need at least one sample");
    int r;
    if ((r = ensure_guide())) return r;
    if (in_flight_ && (r = wait(nullptr))) return r;
    if ((r = check_cuda(d_scratch_.alloc((size_t)n * (kGuideIn + 4) * 4), "scratch"))) return r;
    float* dx = d_scratch_.as<float>();
    float* dwi = dx + (size_t)n * kGuideIn;
    float* dw = dwi + (size_t)n * 3;
    if ((r = check_cuda(cudaMemcpyAsync(dx, x, (size_t)n * kGuideIn * 4, cudaMemcpyHostToDevice, stream_), "copy")))
        return r;
    if ((r = check_cuda(cudaMemcpyAsync(dwi, wi, (size_t)n * 3 * 4, cudaMemcpyHostToDevice, stream_), "copy"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(dw, w, (size_t)n * 4, cudaMemcpyHostToDevice, stream_), "copy"))) return r;
    if ((r = check_cuda(guide_gradients_features(guide_view(), dx, dwi, dw, n, stream_), "guide gradients"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(grad, d_ggrad_.p, kGuideParams * 4, cudaMemcpyDeviceToHost, stream_), "copy")))
        return r;
    float sums[4] = {0.f, 0.f, 0.f, 0.f};
    if ((r = check_cuda(cudaMemcpyAsync(sums, d_gwsum_.p, sizeof(sums), cudaMemcpyDeviceToHost, stream_), "copy")))
        return r;
    if ((r = check_cuda(cudaMemsetAsync(d_ggrad_.p, 0, kGuideParams * 4, stream_), "guide"))) return r;
    if ((r = check_cuda(cudaStreamSynchronize(stream_), "guide gradients"))) return r;
    if (sums[2] != 0.f) return fail(PT_ERR_DEVICE, "tensor-core training: a wait for the MMA completion gave up");
    return PT_OK;
}

int Session::set_bvh(int width, int max_leaf) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    if (width != 2 && width != 4 && width != 8) return fail(PT_ERR_ARG, "BVH width must be 2, 4 or 8");
    if (max_leaf < 1 || max_leaf > kMaxLeafPrims) return fail(PT_ERR_ARG, "leaf size must be in [1, 16]");
    bvh_width_ = width;
    bvh_leaf_ = max_leaf;
    if (!have_scene_) return PT_OK;
    if (batch_mode()) {  // rebuild every scene of the batch with the new shape
        const std::vector<BatchSpec> specs = batch_specs_;
        return load_batch(specs);
    }
    if (bvh_gpu_) {  // rebuilt on the device at the next upload
        bvh_ = BvhBuild();
        bvh_.width = width;
        scene_dirty_ = true;
        return PT_OK;
    }
    BvhBuild b;
    std::string err;
    if (!build_bvh(scene_, bvh_width_, bvh_leaf_, b, err)) return fail(PT_ERR_SCENE, err);
    bvh_ = std::move(b);
    scene_dirty_ = true;
    return PT_OK;
}

int Session::set_bvh_builder(int gpu) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    if (gpu < 0 || gpu > 2) return fail(PT_ERR_ARG, "builder must be 0 (host SAH), 1 (GPU LBVH) or 2 (GPU PLOC)");
    const int g = gpu == 1 ? kGpuBvhLbvh : gpu == 2 ? kGpuBvhPloc : 0;
    if (g == bvh_gpu_) return PT_OK;
    bvh_gpu_ = g;
    if (have_scene_ && !batch_mode()) return set_bvh(bvh_width_, bvh_leaf_);  // rebuild with the new builder
    return PT_OK;
}

int Session::set_bvh_nodes(int quantized) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    const int q = quantized ? 1 : 0;
    if (q == bvh_quant_) return PT_OK;
    bvh_quant_ = q;
    if (have_scene_) scene_dirty_ = true;  // the next device call uploads the chosen node format
    reset();
    return PT_OK;
}

// The quantized node copy on the device against the float nodes (host copy `b`).
int Session::check_quantized(const BvhBuild& b) {
    if (!bvh_nodes_quantized()) return PT_OK;
    int r;
    if ((r = ensure_device())) return r;
    if (scene_dirty_ && (r = upload_scene())) return r;
    std::vector<uint8_t> q((size_t)b.num_nodes * qnode_bytes(b.width));
    if ((r = check_cuda(cudaMemcpy(q.data(), d_qnodes_.p, q.size(), cudaMemcpyDeviceToHost), "BVH download")))
        return r;
    std::string err;
    return pt::check_qnodes(b, q, err) ? PT_OK : fail(PT_ERR_SCENE, err);
}

int Session::check_bvh() {
    if (!have_scene_) return PT_ERR_STATE;
    std::string err;
    if (!bvh_gpu_ || batch_mode()) {
        if (!pt::check_bvh(scene_, bvh_, err)) return fail(PT_ERR_SCENE, err);
        return check_quantized(bvh_);
    }
    // GPU-built tree: build it if still pending, bring it to the host, run the same check
    int r;
    if ((r = ensure_device())) return r;
    if (scene_dirty_ && (r = upload_scene())) return r;
    BvhBuild h = bvh_;
    const size_t nb = (size_t)bvh_.num_nodes * (bvh_.width == 2 ? 64 : bvh_.width == 4 ? 128 : 256);
    const int ne = scene_.num_tri() + scene_.num_sph();
    h.nodes.resize(nb);
    h.prims.resize((size_t)ne * 12);
    if ((r = check_cuda(cudaMemcpy(h.nodes.data(), d_nodes_.p, nb, cudaMemcpyDeviceToHost), "BVH download"))) return r;
    if ((r = check_cuda(cudaMemcpy(h.prims.data(), d_prims_.p, h.prims.size() * 4, cudaMemcpyDeviceToHost),
                        "BVH download")))
        return r;
    h.prim_order.resize(ne);
    for (int e = 0; e < ne; e++) std::memcpy(&h.prim_order[e], &h.prims[(size_t)e * 12 + 3], 4);
    if (!pt::check_bvh(scene_, h, err)) return fail(PT_ERR_SCENE, err);
    return check_quantized(h);
}

int Session::counts(pt_scene_counts* out) const {
    if (!have_scene_) return PT_ERR_STATE;
    std::memset(out, 0, sizeof(*out));
    out->num_triangles = scene_.num_tri();
    out->num_spheres = scene_.num_sph();
    out->num_materials = (int)scene_.mats.size();
    out->num_lights = (int)lights_.size();
    out->env_width = scene_.env_w;
    out->env_height = scene_.env_h;
    out->bvh_width = bvh_.width;
    out->bvh_nodes = bvh_.num_nodes;
    out->bvh_depth = bvh_.depth;
    out->bvh_max_leaf = bvh_.max_leaf;
    out->res_x = scene_.res_x;
    out->res_y = scene_.res_y;
    out->default_spp = scene_.default_spp;
    out->default_depth = scene_.default_depth;
    out->default_nee = scene_.default_nee ? 1 : 0;
    out->bvh_build_ms = bvh_.build_ms;
    return PT_OK;
}

int Session::export_scene(pt_scene_export* o) const {
    if (!have_scene_ || batch_mode()) return PT_ERR_STATE;
    const HostScene& s = scene_;
    if (o->tri_vertices) std::memcpy(o->tri_vertices, s.tri_p.data(), s.tri_p.size() * 4);
    if (o->tri_normals) std::memcpy(o->tri_normals, s.tri_n.data(), s.tri_n.size() * 4);
    if (o->tri_materials) std::memcpy(o->tri_materials, s.tri_mat.data(), s.tri_mat.size() * 4);
    if (o->spheres) std::memcpy(o->spheres, s.sph.data(), s.sph.size() * 4);
    if (o->sphere_materials) std::memcpy(o->sphere_materials, s.sph_mat.data(), s.sph_mat.size() * 4);
    for (size_t i = 0; i < s.mats.size(); i++) {
        const Material& m = s.mats[i];
        if (o->material_types) o->material_types[i] = m.type;
        for (int k = 0; k < 3; k++) {
            if (o->material_albedo) o->material_albedo[3 * i + k] = m.albedo[k];
            if (o->material_emit) o->material_emit[3 * i + k] = m.emit[k];
        }
        if (o->material_ior) o->material_ior[i] = m.ior;
        if (o->material_alpha) o->material_alpha[i] = m.alpha;
    }
    for (size_t i = 0; i < lights_.size(); i++) {
        if (o->light_types) o->light_types[i] = lights_[i].type;
        if (o->light_indices) o->light_indices[i] = lights_[i].index;
    }
    if (o->env_rgba && !s.env_rgba.empty()) std::memcpy(o->env_rgba, s.env_rgba.data(), s.env_rgba.size() * 4);
    if (o->camera) {
        for (int k = 0; k < 3; k++) {
            o->camera[k] = camspec_.origin[k];
            o->camera[3 + k] = camspec_.target[k];
            o->camera[6 + k] = camspec_.up[k];
        }
        o->camera[9] = camspec_.vfov;
        o->camera[10] = camspec_.flip ? 1.f : 0.f;
    }
    return PT_OK;
}

int Session::set_camera(const CameraSpec& c) {
    if (batch_mode()) return fail(PT_ERR_STATE, "not available for a batch (one query per scene session)");
    CameraParams tmp;
    std::string err;
    if (!make_camera(c, w_, h_, tmp, err)) return fail(PT_ERR_ARG, err);
    camspec_ = c;
    reset();
    return PT_OK;
}

int Session::set_material(int id, int type, const float* albedo, const float* emit, float ior, float alpha) {
    if (!have_scene_) return fail(PT_ERR_STATE, "no scene loaded");
    if (batch_mode()) return fail(PT_ERR_STATE, "not available for a batch (one query per scene session)");
    if (id < 0 || id >= (int)scene_.mats.size()) return fail(PT_ERR_ARG, "material id out of range");
    if (type < kLambertian || type > kMetal || type == kMaterialNone) return fail(PT_ERR_ARG, "unknown material type");
    Material& m = scene_.mats[id];
    if (m.type != type) {
        // Scene::setMaterialType defaults (include/scene.h:36-61)
        Material n{};
        n.type = type;
        if (type == kGlass) n.ior = 1.4f;
        if (type == kMicrofacet || type == kMetal) n.alpha = 0.1f;
        if (type == kMetal) {  // copper's F0 until an albedo is given
            n.albedo[0] = 0.955f;
            n.albedo[1] = 0.638f;
            n.albedo[2] = 0.538f;
        }
        m = n;
    } else {
        // the type's own parameters only (MaterialParams setters, include/materials/params.h)
        if (type == kLambertian) {
            for (int k = 0; k < 3; k++) {
                if (albedo) m.albedo[k] = albedo[k];
                if (emit) m.emit[k] = emit[k];
            }
        } else if (type == kGlass) {
            m.ior = ior;
        } else if (type == kMicrofacet) {
            m.alpha = alpha;
        } else if (type == kMetal) {  // F0 in the albedo, and the roughness
            for (int k = 0; k < 3; k++)
                if (albedo) m.albedo[k] = albedo[k];
            m.alpha = alpha;
        }
    }
    finalize_materials(scene_);
    lights_ = build_light_list(scene_);
    update_material_classes();
    mats_dirty_ = true;
    reset();
    return PT_OK;
}

int Session::set_max_depth(int d) {
    if (d < 0 || d > kMaxDepthLimit) return fail(PT_ERR_ARG, "max depth must be in [0, 64]");
    max_depth_ = d;
    reset();
    return PT_OK;
}

int Session::set_renderer(int type) {
    if (type != PT_RENDERER_CUDA && type != PT_RENDERER_NORMALS)
        return fail(PT_ERR_ARG, "renderer must be PT_RENDERER_CUDA or PT_RENDERER_NORMALS (no OptiX backend)");
    const int kind = type == PT_RENDERER_NORMALS ? 1 : 0;
    if (kind == 1 && batch_mode()) return fail(PT_ERR_STATE, "the normals renderer takes a single scene");
    if (kind != renderer_) reset();
    renderer_ = kind;
    return PT_OK;
}

int Session::set_nee(int on) {
    nee_ = on ? 1 : 0;
    reset();
    return PT_OK;
}

int Session::set_launch(const pt_launch_config* c) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    auto ok_block = [](int b) { return b == 0 || (b >= 32 && b <= 1024 && b % 32 == 0); };
    if (!ok_block(c->block_extend) || !ok_block(c->block_shade) || !ok_block(c->block_shadow))
        return fail(PT_ERR_ARG, "block sizes must be multiples of 32 in [32, 1024]");
    if (c->block_shade > 512) return fail(PT_ERR_ARG, "the shade stage takes at most 512 threads per block");
    if (c->wave_paths < 0 || c->blocks_per_sm < 0 || c->blocks_per_sm > 64)
        return fail(PT_ERR_ARG, "invalid wave size or blocks per SM");
    if (c->sort_materials < 0 || c->sort_materials > 3 || c->use_graph < 0 || c->use_graph > 2 ||
        c->sort_rays < 0 || c->sort_rays > 2 || c->speculate < 0 || c->speculate > 4 || c->split_shade < 0 ||
        c->split_shade > 3 || c->overlap_shadow < 0 || c->overlap_shadow > 2 || c->shadow_order < 0 ||
        c->shadow_order > 2 || c->fuse_camera < 0 || c->fuse_camera > 2)
        return fail(PT_ERR_ARG, "invalid sort or graph mode");
    if (c->refill_idle < 0 || c->refill_idle > 32) return fail(PT_ERR_ARG, "refill_idle must be in [1, 32]");
    if (c->wave_paths) wave_paths_ = c->wave_paths;
    if (c->block_extend) shape_.block_extend = c->block_extend;
    if (c->block_shade) shape_.block_shade = c->block_shade;
    if (c->block_shadow) shape_.block_shadow = c->block_shadow;
    if (c->blocks_per_sm) shape_.blocks_per_sm = c->blocks_per_sm;
    if (c->sort_materials) sort_mode_ = c->sort_materials == 1 ? 1 : c->sort_materials == 2 ? 0 : -1;
    if (c->use_graph) use_graph_ = c->use_graph == 1 ? 1 : 0;
    if (c->sort_rays) shape_.sort_rays = c->sort_rays == 1 ? 1 : 0;
    if (c->refill_idle) shape_.refill_idle = c->refill_idle;
    if (c->speculate) shape_.speculate = speculate_bits(c->speculate);
    if (c->split_shade) shape_.shade_kernel = c->split_shade == 1 ? kShadeClasses : c->split_shade == 2 ? kShadeAll128 : kShadeAll80;
    if (c->overlap_shadow) shape_.overlap_shadow = c->overlap_shadow == 1 ? 1 : 0;
    if (c->shadow_order) shape_.shadow_near = c->shadow_order == 1 ? 1 : 0;
    if (c->fuse_camera) shape_.fuse_camera = c->fuse_camera == 1 ? 1 : 0;
    return PT_OK;
}

void Session::get_launch(pt_launch_config* c) const {
    c->wave_paths = wave_paths_;
    c->block_extend = shape_.block_extend;
    c->block_shade = shape_.block_shade;
    c->block_shadow = shape_.block_shadow;
    c->blocks_per_sm = shape_.blocks_per_sm;
    c->sort_materials = sort_mode_ == 1 ? 1 : sort_mode_ == 0 ? 2 : 3;
    c->use_graph = use_graph_ ? 1 : 2;
    c->sort_rays = shape_.sort_rays ? 1 : 2;
    c->refill_idle = shape_.refill_idle;
    c->speculate = speculate_code(shape_.speculate);
    c->split_shade = shape_.shade_kernel == kShadeClasses ? 1 : shape_.shade_kernel == kShadeAll128 ? 2 : 3;
    c->overlap_shadow = shape_.overlap_shadow ? 1 : 2;
    c->shadow_order = shape_.shadow_near ? 1 : 2;
    c->fuse_camera = shape_.fuse_camera ? 1 : 2;
}

int Session::upload_materials() {
    int r;
    if ((r = check_cuda(upload(d_mats_, scene_.mats, stream_), "upload materials"))) return r;
    if ((r = check_cuda(upload(d_lights_, lights_, stream_), "upload lights"))) return r;
    if ((r = check_cuda(cudaStreamSynchronize(stream_), "upload materials"))) return r;
    mats_dirty_ = false;
    return PT_OK;
}

int Session::upload_scene() {
    int r;
    const int nt = scene_.num_tri();
    std::vector<float> tp((size_t)nt * 12, 0.f), tn((size_t)nt * 12, 0.f);
    for (int i = 0; i < nt; i++)
        for (int v = 0; v < 3; v++)
            for (int k = 0; k < 3; k++) {
                tp[(size_t)i * 12 + v * 4 + k] = scene_.tri_p[(size_t)i * 9 + v * 3 + k];
                tn[(size_t)i * 12 + v * 4 + k] = scene_.tri_n[(size_t)i * 9 + v * 3 + k];
            }
    const bool gpu_tree = bvh_gpu_ != 0 && !batch_mode();
    if (!gpu_tree) {
        if ((r = check_cuda(upload(d_nodes_, bvh_.nodes, stream_), "upload BVH nodes"))) return r;
        if ((r = check_cuda(upload(d_prims_, bvh_.prims, stream_), "upload BVH primitives"))) return r;
    }
    if ((r = check_cuda(upload(d_tri_p_, tp, stream_), "upload triangles"))) return r;
    if ((r = check_cuda(upload(d_tri_n_, tn, stream_), "upload normals"))) return r;
    if ((r = check_cuda(upload(d_tri_mat_, scene_.tri_mat, stream_), "upload triangle materials"))) return r;
    if ((r = check_cuda(upload(d_sph_, scene_.sph, stream_), "upload spheres"))) return r;
    if ((r = check_cuda(upload(d_sph_mat_, scene_.sph_mat, stream_), "upload sphere materials"))) return r;
    if (scene_.env_w > 0) {
        if ((r = check_cuda(upload(d_env_rgba_, scene_.env_rgba, stream_), "upload environment"))) return r;
        if ((r = check_cuda(upload(d_env_marg_, env_cdf_.marg, stream_), "upload environment CDF"))) return r;
        if ((r = check_cuda(upload(d_env_cond_, env_cdf_.cond, stream_), "upload environment CDF"))) return r;
        if ((r = check_cuda(upload(d_env_row_, env_cdf_.row_mass, stream_), "upload environment CDF"))) return r;
    }
    if (gpu_tree) {  // the wide BVH built on the device from the uploaded primitives
        cudaEvent_t e0, e1;
        if ((r = check_cuda(cudaEventCreate(&e0), "cudaEventCreate"))) return r;
        if ((r = check_cuda(cudaEventCreate(&e1), "cudaEventCreate"))) return r;
        cudaEventRecord(e0, stream_);
        GpuBvhInfo info;
        const cudaError_t be = gpu_build_bvh(d_tri_p_.as<float4>(), nt, d_sph_.as<float4>(), scene_.num_sph(),
                                             bvh_width_, bvh_leaf_, gbvh_, d_nodes_, d_prims_, info, stream_, bvh_gpu_);
        cudaEventRecord(e1, stream_);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if ((r = check_cuda(be, "GPU BVH build"))) return r;
        bvh_ = BvhBuild();
        bvh_.width = info.width;
        bvh_.root = info.root;
        bvh_.num_nodes = info.num_nodes;
        bvh_.depth = info.depth;
        bvh_.max_leaf = info.max_leaf;
        bvh_.build_ms = ms;
    }
    if (watertight_) {  // triangle entries carry their vertices for the watertight test
        const int entries = gpu_tree ? nt + scene_.num_sph() : (int)(bvh_.prims.size() / 12);
        if ((r = check_cuda(prims_to_vertices(d_prims_.as<float4>(), entries, d_tri_p_.as<float4>(), stream_),
                            "watertight leaf entries")))
            return r;
    }
    if (bvh_nodes_quantized()) {  // the quantized copy the traversal reads instead
        if ((r = check_cuda(d_qnodes_.alloc((size_t)bvh_.num_nodes * qnode_bytes(bvh_.width)), "quantized BVH")))
            return r;
        if ((r = check_cuda(d_qfail_.alloc(sizeof(int)), "quantized BVH"))) return r;
        if ((r = check_cuda(cudaMemsetAsync(d_qfail_.p, 0, sizeof(int), stream_), "quantized BVH"))) return r;
        if ((r = check_cuda(quantize_bvh_nodes(d_nodes_.p, bvh_.num_nodes, bvh_.width, d_qnodes_.p,
                                               d_qfail_.as<int>(), stream_),
                            "BVH quantization")))
            return r;
    }
    // host vectors above must outlive the async copies
    if ((r = check_cuda(cudaStreamSynchronize(stream_), "scene upload"))) return r;
    if (bvh_nodes_quantized()) {
        int qf = 0;
        if ((r = check_cuda(cudaMemcpy(&qf, d_qfail_.p, sizeof(int), cudaMemcpyDeviceToHost), "BVH quantization")))
            return r;
        if (qf) return fail(PT_ERR_SCENE, "a BVH node could not be quantized conservatively");
    }
    if (batch_mode() && (r = upload_batch())) return r;
    scene_dirty_ = false;
    return upload_materials();
}

SceneDevice Session::scene_view() const {
    SceneDevice v{};
    // the watertight kernels read float nodes
    const bool qn = bvh_nodes_quantized() && !watertight_;
    v.nodes = qn ? d_qnodes_.as<float4>() : d_nodes_.as<float4>();
    v.node_q = qn;
    v.prims = d_prims_.as<float4>();
    v.tri_p = d_tri_p_.as<float4>();
    v.tri_n = d_tri_n_.as<float4>();
    v.tri_mat = d_tri_mat_.as<int>();
    v.sph = d_sph_.as<float4>();
    v.sph_mat = d_sph_mat_.as<int>();
    v.mats = d_mats_.as<Material>();
    v.lights = d_lights_.as<LightRef>();
    v.num_tri = scene_.num_tri();
    v.num_sph = scene_.num_sph();
    v.num_mat = (int)scene_.mats.size();
    v.num_lights = (int)lights_.size();
    v.bvh_width = bvh_.width;
    v.root = bvh_.root;
    v.watertight = watertight_ ? 1 : 0;
    if (scene_.env_w > 0) {
        v.env.rgba = d_env_rgba_.as<float>();
        v.env.marg_cdf = d_env_marg_.as<float>();
        v.env.cond_cdf = d_env_cond_.as<float>();
        v.env.row_mass = d_env_row_.as<float>();
        v.env.width = scene_.env_w;
        v.env.height = scene_.env_h;
        v.env.total_mass = env_cdf_.total;
        v.env.present = 1;
    }
    return v;
}

int Session::ensure_frame_buffers(int spp) {
    int r;
    const size_t np = batch_mode() ? (size_t)batch_pixels_ : (size_t)w_ * h_;
    if ((r = check_cuda(d_pass_.alloc(np * 3 * 4), "frame buffer"))) return r;
    if ((r = check_cuda(d_accum_.alloc(np * 3 * 4), "frame buffer"))) return r;
    if ((r = check_cuda(d_rgba8_.alloc(np * 4), "frame buffer"))) return r;
    const int wave_pixels = std::max(1, std::min((int)np, wave_paths_ / spp));
    size_t cap = (size_t)wave_pixels * spp;
    if (batch_mode()) {  // waves of whole pixels of the batch's global pixel order
        cap = (size_t)std::min<long long>(wave_paths_, batch_paths_);
        batch_waves_.clear();
        long long px = 0;
        for (const BatchHost& b : batch_) {
            const long long npx = (long long)b.spec.width * b.spec.height;
            for (long long q = 0; q < npx;) {
                if (batch_waves_.empty() || (long long)batch_waves_.back().npaths + b.spec.spp > (long long)cap) {
                    WaveRange w{};
                    w.first_pixel = (int)(b.pixel_base + q);
                    w.first_path = b.path_base + q * b.spec.spp;
                    batch_waves_.push_back(w);
                }
                WaveRange& w = batch_waves_.back();
                const long long room = ((long long)cap - w.npaths) / b.spec.spp;
                const long long take = std::min(room, npx - q);
                w.npix += (int)take;
                w.npaths += (int)(take * b.spec.spp);
                q += take;
            }
            px += npx;
        }
        // guided paths before a global path index (training paths are counted over them)
        auto guided_before = [&](long long x) {
            long long g = 0;
            for (const BatchHost& b : batch_) {
                if (!b.spec.guided) continue;
                const long long np = (long long)b.spec.width * b.spec.height * b.spec.spp;
                g += std::max(0LL, std::min(x - b.path_base, np));
            }
            return g;
        };
        for (WaveRange& w : batch_waves_) {
            w.guided_first = guided_before(w.first_path);
            w.guided_n = (int)(guided_before(w.first_path + w.npaths) - w.guided_first);
        }
    }
    const size_t f4 = cap * sizeof(float4);
    for (int k = 0; k < 2; k++) {
        for (int a = 0; a < 6; a++) {
            const size_t bytes = a == 3 ? cap * sizeof(uint2) : a == 5 ? cap * sizeof(int) : f4;
            if ((r = check_cuda(d_q_[k][a].alloc(bytes), "ray queue"))) return r;
        }
    }
    for (int a = 0; a < 3; a++)
        if ((r = check_cuda(d_sq_[a].alloc(f4), "shadow queue"))) return r;
    if ((r = check_cuda(d_L_.alloc(f4), "path radiance"))) return r;
    if ((r = check_cuda(d_hitd_.alloc(f4), "BSDF-direct hits"))) return r;
    if ((r = check_cuda(d_sort_.alloc(cap * sizeof(int)), "sort index"))) return r;
    if ((r = check_cuda(d_rindex_.alloc(cap * sizeof(int)), "ray-sort index"))) return r;
    if ((r = check_cuda(d_rhist_.alloc(2 * (kMaxDepthLimit + 1) * kRayBuckets * sizeof(int)), "ray-sort buckets")))
        return r;
    queue_cap_ = (int)cap;
    return PT_OK;
}

int Session::render_async(int spp) {
    if (!have_scene_) return fail(PT_ERR_STATE, "no scene loaded");
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is already in flight");
    const bool batch = batch_mode();
    if (batch) spp = 1;  // each scene of a batch renders its own spp
    const bool normals = renderer_ == 1;
    if (normals) spp = 1;  // GBuffer::renderAsync: one sample per frame (g_buffer.cu:97-116)
    if (spp < 1) return fail(PT_ERR_ARG, "spp must be >= 1");
    int r;
    if ((r = ensure_device())) return r;
    if (scene_dirty_ && (r = upload_scene())) return r;
    if (mats_dirty_ && (r = upload_materials())) return r;
    if ((r = ensure_frame_buffers(spp))) return r;
    std::string err;
    if (!batch && !make_camera(camspec_, w_, h_, cam_, err)) return fail(PT_ERR_ARG, err);
    const int stack_depth = bvh_.depth + 1;
    const int maxb = std::max(shape_.block_extend, shape_.block_shadow);
    const size_t smem = stack_bytes(stack_depth, maxb);
    if (smem > max_smem_) return fail(PT_ERR_SCENE, "BVH too deep for the traversal stack in shared memory");
    if (smem > smem_configured_) {
        if ((r = check_cuda(configure_traversal_smem(smem), "shared memory configuration"))) return r;
        smem_configured_ = smem;
    }
    if (reset_pending_) {  // PathTracer::renderAsync resets m_currentSamples (path_tracer.cu:306-309)
        total_spp_ = 0;
        for (BatchHost& b : batch_) b.total_spp = 0;
        reset_pending_ = false;
    }
    FrameParams p;
    std::memset(&p, 0, sizeof(p));  // padding too: the graph cache compares these bytes
    p.sc = scene_view();
    p.dyn = d_dyn_.as<FrameDyn>();
    for (int k = 0; k < 2; k++) {
        p.q[k].o = d_q_[k][0].as<float4>();
        p.q[k].d = d_q_[k][1].as<float4>();
        p.q[k].beta = d_q_[k][2].as<float4>();
        p.q[k].rng = d_q_[k][3].as<uint2>();
        p.q[k].hit = d_q_[k][4].as<float4>();
        p.q[k].hitd = d_hitd_.as<float4>();
        p.q[k].key = d_q_[k][5].as<int>();
    }
    p.sq.o = d_sq_[0].as<float4>();
    p.sq.d = d_sq_[1].as<float4>();
    p.sq.c = d_sq_[2].as<float4>();
    p.L = d_L_.as<float4>();
    p.sort_index = d_sort_.as<int>();
    p.ray_index = d_rindex_.as<int>();
    p.ray_hist = d_rhist_.as<int>();
    p.counters = d_counters_.as<WaveCounters>();
    p.stats = d_stats_.as<FrameStats>();
    p.pass_rgb = d_pass_.as<float>();
    p.accum_rgb = d_accum_.as<float>();
    p.rgba8 = d_rgba8_.as<uchar4>();
    p.width = w_;
    p.height = h_;
    p.spp = spp;
    p.max_depth = batch ? batch_max_depth_ : max_depth_;
    p.nee = nee_;
    p.wave_pixels = queue_cap_ / spp;
    if (batch) {
        p.width = p.height = 0;
        p.batch = d_batch_.as<BatchScene>();
        p.batch_path_base = d_batch_path_base_.as<long long>();
        p.batch_pixel_base = d_batch_pixel_base_.as<long long>();
        p.num_scenes = (int)batch_.size();
    }
    p.stack_depth = stack_entries();
    p.mma_test_polls = test_mma_polls_;
    p.num_sms = num_sms_;
    p.count_work = work_counters_;
    p.renderer = renderer_;
    p.shape = shape_;
    p.shape.sort_materials = sort_mode_ >= 0 ? sort_mode_ : (material_classes_ >= 2 ? 1 : 0);
    p.class_mask = class_mask_;
    p.gframe = gframe_;  // scene bounds: guide encoding and ray-sort cells
    last_wave_paths_ = p.wave_pixels * spp;
    p.consistent_mis = consistent_mis_ || guiding_;
    if (guiding_ && !normals) {
        if ((r = ensure_guide())) return r;
        const size_t mix_bytes = (size_t)queue_cap_ * kGuideOut * sizeof(float);
        if ((r = check_cuda(d_gmix_.alloc(mix_bytes), "guide mixtures"))) return r;
        // every gstride-th path of a wave records training data: about 2^19 training paths
        // per wave; in a batch, every gstride-th path of the wave's guided scenes, about 2^22
        long long train_pool = queue_cap_;
        int gstride = std::max(1, queue_cap_ / PT_GUIDE_TRAIN_PATHS);
        if (batch) {
            train_pool = 1;
            for (const WaveRange& w : batch_waves_) train_pool = std::max<long long>(train_pool, w.guided_n);
            gstride = (int)std::max<long long>(1, (train_pool + PT_GUIDE_TRAIN_PATHS_BATCH - 1) /
                                                      PT_GUIDE_TRAIN_PATHS_BATCH);
        }
        const size_t tpaths = (size_t)((train_pool + gstride - 1) / gstride);
        if ((r = check_cuda(d_gacc_.alloc(tpaths * (size_t)p.max_depth * 3 * sizeof(float)), "guide accumulators")))
            return r;
        // one record per scattering vertex of a training path
        const size_t rec_cap = tpaths * (size_t)std::max(1, p.max_depth - 1);
        if ((r = check_cuda(d_grec_.alloc(rec_cap * sizeof(GuideRecord)), "guide records"))) return r;
        p.guide_mode = guide_iters_ >= guide_warmup_ ? 2 : 1;
        p.guide_tc = guide_infer_tc_ ? 1 : 0;
        p.gfrac = guide_frac_;
        p.gwpack = d_gwpack_.as<uint32_t>();
        p.gmix = d_gmix_.as<float>();
        p.gframe = gframe_;
        p.grec = d_grec_.as<GuideRecord>();
        p.grec_count = d_grec_count_.as<int>();
        p.grec_cap = (int)rec_cap;
        p.gacc = d_gacc_.as<float>();
        p.gstride = gstride;
        p.gring = d_gring_.as<GuideSample>();
        p.gring_count = d_gring_count_.as<int>();
        p.gring_cap = guide_ring_cap_;
        p.gnets = guide_nets_;
        // Adam steps this frame: automatic schedule (many while the network is young) unless set
        p.gtrain_steps = guide_steps_per_frame_ > 0 ? guide_steps_per_frame_
                         : guide_iters_ < 512      ? 16
                         : guide_iters_ < 1024     ? 4
                                                   : 2;
        p.gtrain_batch = guide_batch_;
        p.gtrain_lr = guide_lr_;
    }
    // per-frame constants: one pinned copy ahead of the frame's launches
    h_dyn_->cam = cam_;
    h_dyn_->seed = seed_;
    h_dyn_->sample_base = (uint64_t)total_spp_;
    h_dyn_->prev_spp = total_spp_;
    if (batch) {
        int net = 0;
        for (size_t i = 0; i < batch_.size(); i++) {
            const bool g = guiding_ && batch_[i].spec.guided;
            h_batch_[i].guide_net = g ? net++ : -1;
            h_batch_[i].guide_mode = g ? p.guide_mode : 0;
            h_batch_[i].seed = seed_;
            h_batch_[i].sample_base = (uint64_t)batch_[i].total_spp;
            h_batch_[i].prev_spp = batch_[i].total_spp;
        }
    }
    StageMarks* mk = nullptr;
    marks_active_ = false;
    if (stage_timing_) {
        const int waves = batch ? (int)batch_waves_.size() : (w_ * h_ + p.wave_pixels - 1) / p.wave_pixels;
        const size_t need = (size_t)waves * (p.max_depth * 10 + 4) + 8;
        while (mark_events_.size() < need) {
            cudaEvent_t e;
            if ((r = check_cuda(cudaEventCreate(&e), "cudaEventCreate"))) return r;
            mark_events_.push_back(e);
        }
        mark_stage_.assign(mark_events_.size(), -1);
        mark_begin_.assign(mark_events_.size(), -1);
        marks_.events = mark_events_.data();
        marks_.stage = mark_stage_.data();
        marks_.begin = mark_begin_.data();
        marks_.capacity = (int)mark_events_.size();
        marks_.used = 0;
        mk = &marks_;
        marks_active_ = true;
    }
    if ((r = check_cuda(cudaMemsetAsync(d_stats_.p, 0, sizeof(FrameStats), stream_), "stats reset"))) return r;
    if ((r = check_cuda(cudaEventRecord(ev_begin_, stream_), "cudaEventRecord"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(d_dyn_.p, h_dyn_, sizeof(FrameDyn), cudaMemcpyHostToDevice, stream_),
                        "frame constants")))
        return r;
    if (batch && (r = check_cuda(cudaMemcpyAsync(d_batch_.p, h_batch_, batch_.size() * sizeof(BatchScene),
                                                 cudaMemcpyHostToDevice, stream_),
                                 "batch scene table")))
        return r;
    if (use_graph_ && !mk) {
        // replay the captured frame while every launch parameter is unchanged
        if (!graph_valid_ || std::memcmp(&graph_params_, &p, sizeof(p)) != 0) {
            if (graph_exec_) {
                cudaGraphExecDestroy(graph_exec_);
                graph_exec_ = nullptr;
            }
            graph_valid_ = false;
            cudaGraph_t g = nullptr;
            if ((r = check_cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "graph capture")))
                return r;
            const cudaError_t ce = enqueue_frame_and_training(p, nullptr);
            const cudaError_t ee = cudaStreamEndCapture(stream_, &g);
            if ((r = check_cuda(ce != cudaSuccess ? ce : ee, "graph capture"))) {
                if (g) cudaGraphDestroy(g);
                return r;
            }
            const cudaError_t ie = cudaGraphInstantiate(&graph_exec_, g, 0);
            cudaGraphDestroy(g);
            if ((r = check_cuda(ie, "graph instantiate"))) return r;
            graph_params_ = p;
            graph_valid_ = true;
            graph_captures_++;
        }
        if ((r = check_cuda(cudaGraphLaunch(graph_exec_, stream_), "graph launch"))) return r;
    } else if ((r = check_cuda(enqueue_frame_and_training(p, mk), "frame launch"))) {
        return r;
    }
    if (guiding_) guide_iters_ += p.gtrain_steps;
    if ((r = check_cuda(cudaMemcpyAsync(h_stats_, d_stats_.p, sizeof(FrameStats), cudaMemcpyDeviceToHost, stream_),
                        "stats readback")))
        return r;
    if ((r = check_cuda(cudaEventRecord(ev_end_, stream_), "cudaEventRecord"))) return r;
    in_flight_ = true;
    inflight_spp_ = spp;
    return PT_OK;
}

// The frame's launches, then (guiding) online training on the newest samples inside the
// frame's timed region.
cudaError_t Session::enqueue_frame_and_training(const FrameParams& p, StageMarks* marks) {
    cudaError_t e = p.num_scenes > 0
                        ? enqueue_batch_frame(p, batch_waves_.data(), (int)batch_waves_.size(), stream_, marks, &side_)
                        : enqueue_frame(p, stream_, marks, &side_);
    if (e != cudaSuccess || !p.guide_mode) return e;
    for (int k = 0; k < p.gtrain_steps; k++) {
        e = guide_train_step(guide_view(), p.gring, p.gring_cap, p.gring_count, p.gtrain_batch, p.gtrain_lr, stream_);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int Session::finish_frame(float* ms) {
    int r;
    float t = 0.f;
    if ((r = check_cuda(cudaEventElapsedTime(&t, ev_begin_, ev_end_), "cudaEventElapsedTime"))) return r;
    in_flight_ = false;
    last_ms_ = t;
    last_spp_ = inflight_spp_;
    total_spp_ += inflight_spp_;  // PathTracer::pollRender (path_tracer.cu:354)
    for (BatchHost& b : batch_) b.total_spp += b.spec.spp;
    frames_++;
    last_stats_ = *h_stats_;
    if (ms) *ms = t;
    if (marks_active_) {
        for (int k = 0; k < kNumStages; k++) {
            stage_ms_[k] = 0.f;
            stage_launches_[k] = 0;
        }
        for (int i = 1; i < marks_.used; i++) {
            const int st = marks_.stage[i], b = marks_.begin[i];
            if (st < 0 || b < 0) continue;
            float dt = 0.f;
            if ((r = check_cuda(cudaEventElapsedTime(&dt, marks_.events[b], marks_.events[i]), "stage timing")))
                return r;
            stage_ms_[st] += dt;
            stage_launches_[st]++;
        }
        marks_active_ = false;
    }
    if (last_stats_.error & 1) return fail(PT_ERR_DEVICE, "traversal stack overflow reported by a kernel");
    if (last_stats_.error & 2) return fail(PT_ERR_DEVICE, "tensor-core inference: a wait for the MMA completion gave up");
    return PT_OK;
}

int Session::poll(int* done, float* ms) {
    if (!in_flight_) {
        if (done) *done = 1;
        if (ms) *ms = last_ms_;
        return PT_OK;
    }
    cudaError_t e = cudaEventQuery(ev_end_);
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        if (done) *done = 0;
        return PT_OK;
    }
    if (e != cudaSuccess) {
        in_flight_ = false;
        return check_cuda(e, "frame execution");
    }
    if (done) *done = 1;
    return finish_frame(ms);
}

int Session::wait(float* ms) {
    if (!in_flight_) {
        if (ms) *ms = last_ms_;
        return PT_OK;
    }
    cudaError_t e = cudaEventSynchronize(ev_end_);
    if (e != cudaSuccess) {
        in_flight_ = false;
        return check_cuda(e, "frame execution");
    }
    return finish_frame(ms);
}

int Session::stats(pt_stats* out) const {
    std::memset(out, 0, sizeof(*out));
    out->rays_camera = last_stats_.rays_camera;
    out->rays_extend = last_stats_.rays_extend;
    out->rays_shadow = last_stats_.rays_shadow;
    out->last_frame_ms = last_ms_;
    out->last_frame_spp = last_spp_;
    out->total_spp = total_spp_;
    out->frames = frames_;
    return PT_OK;
}

namespace {
std::string tune_key(const HostScene& s, int classes, int w, int h, int spp, int depth, int nee) {
    return "t" + std::to_string(s.num_tri()) + "_s" + std::to_string(s.num_sph()) + "_c" + std::to_string(classes) +
           "_e" + std::to_string(s.env_w) + "_" + std::to_string(w) + "x" + std::to_string(h) + "_spp" +
           std::to_string(spp) + "_d" + std::to_string(depth) + "_n" + std::to_string(nee);
}
// A batch's key: its scene count and an FNV-1a hash over every scene's draw (configuration,
// seed, level, size, spp, depth, guided), so a different draw never reuses another's choice.
std::string batch_tune_key(const std::vector<BatchSpec>& specs, int nee) {
    uint64_t h = 1469598103934665603ULL;
    auto mix = [&](uint64_t v) {
        for (int k = 0; k < 8; k++) {
            h ^= (v >> (8 * k)) & 0xff;
            h *= 1099511628211ULL;
        }
    };
    for (const BatchSpec& b : specs) {
        mix((uint64_t)b.config);
        mix(b.seed);
        mix((uint64_t)(int64_t)b.level);
        mix((uint64_t)b.width);
        mix((uint64_t)b.height);
        mix((uint64_t)b.spp);
        mix((uint64_t)b.max_depth);
        mix((uint64_t)b.guided);
    }
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%016llx", (unsigned long long)h);
    return "batch" + std::to_string(specs.size()) + "_" + buf + "_n" + std::to_string(nee);
}
int json_int(const std::string& line, const char* field, int dflt) {
    const std::string k = std::string("\"") + field + "\": ";
    const size_t p = line.find(k);
    return p == std::string::npos ? dflt : std::atoi(line.c_str() + p + k.size());
}
double json_num(const std::string& line, const char* field, double dflt) {
    const std::string k = std::string("\"") + field + "\": ";
    const size_t p = line.find(k);
    return p == std::string::npos ? dflt : std::atof(line.c_str() + p + k.size());
}
}  // namespace

int Session::autotune(int spp, const char* cache_path, pt_tune_result* out) {
    if (!have_scene_) return fail(PT_ERR_STATE, "no scene loaded");
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    if (spp < 1) return fail(PT_ERR_ARG, "spp must be >= 1");
    pt_tune_result res;
    std::memset(&res, 0, sizeof(res));
    const bool batch = batch_mode();
    const std::string key =
        batch ? batch_tune_key(batch_specs_, nee_) : tune_key(scene_, material_classes_, w_, h_, spp, max_depth_, nee_);
    // paths of one frame: waves smaller than this split the frame
    const long long frame_paths = batch ? batch_paths_ : (long long)w_ * h_ * spp;
    struct Cand {
        int width, sort, bps, block, rays, spec, wave, split, leaf, builder, near, fuse;
    };
    auto apply = [&](const Cand& c) -> int {
        int r;
        if (c.width != bvh_width_ || c.leaf != bvh_leaf_ || c.builder != bvh_gpu_) {
            bvh_gpu_ = c.builder;
            if ((r = set_bvh(c.width, c.leaf))) return r;
        }
        sort_mode_ = c.sort;
        shape_.blocks_per_sm = c.bps;
        shape_.block_extend = shape_.block_shadow = c.block;
        shape_.sort_rays = c.rays;
        shape_.speculate = c.spec;
        wave_paths_ = c.wave;
        shape_.shade_kernel = c.split;
        shape_.shadow_near = c.near;
        shape_.fuse_camera = c.fuse;
        return PT_OK;
    };
    auto report = [&](const Cand& c) {
        res.bvh_width = c.width;
        res.sort_materials = c.sort == 1 ? 1 : 2;
        res.blocks_per_sm = c.bps;
        res.block = c.block;
        res.sort_rays = c.rays ? 1 : 2;
        res.speculate = speculate_code(c.spec);
        res.wave_paths = c.wave;
        res.split_shade = c.split == kShadeClasses ? 1 : c.split == kShadeAll128 ? 2 : 3;
        res.max_leaf = c.leaf;
        res.bvh_builder = c.builder == kGpuBvhPloc ? 2 : c.builder == kGpuBvhLbvh ? 1 : 0;
        res.shadow_order = c.near ? 1 : 2;
        res.fuse_camera = c.fuse ? 1 : 2;
    };
    if (cache_path) {
        FILE* f = std::fopen(cache_path, "r");
        if (f) {
            char buf[1024];
            const std::string want = "\"key\": \"" + key + "\"";
            while (std::fgets(buf, sizeof(buf), f)) {
                const std::string line(buf);
                if (line.find(want) == std::string::npos) continue;
                Cand c{json_int(line, "bvh_width", 4), json_int(line, "sort", 0), json_int(line, "blocks_per_sm", 16),
                       json_int(line, "block", 128), json_int(line, "sort_rays", 0), json_int(line, "speculate", 0),
                       json_int(line, "wave_paths", wave_paths_), json_int(line, "shade_kernel", kShadeClasses),
                       json_int(line, "max_leaf", bvh_leaf_), batch ? bvh_gpu_ : json_int(line, "builder", bvh_gpu_),
                       json_int(line, "shadow_near", shape_.shadow_near),
                       json_int(line, "fuse_camera", shape_.fuse_camera)};
                std::fclose(f);
                int r;
                if ((r = apply(c))) return r;
                report(c);
                res.best_ms = (float)json_num(line, "ms", 0.0);
                res.from_cache = 1;
                reset();
                if (out) *out = res;
                return PT_OK;
            }
            std::fclose(f);
        }
    }
    const int saved_timing = stage_timing_;
    stage_timing_ = 0;
    int trials = 0;
    auto measure = [&](const Cand& c, float& ms_out) -> int {
        int r;
        if ((r = apply(c))) return r;
        float best = 1e30f;
        for (int k = 0; k < 3; k++) {  // first frame warms up (and captures the graph)
            reset();
            if ((r = render_async(spp))) return r;
            float ms = 0.f;
            if ((r = wait(&ms))) return r;
            if (k > 0) best = std::min(best, ms);
        }
        trials += 2;
        ms_out = best;
        return PT_OK;
    };
    const int prims = scene_.num_tri() + scene_.num_sph();
    Cand best{bvh_width_, sort_mode_ >= 0 ? sort_mode_ : (material_classes_ >= 2 ? 1 : 0), shape_.blocks_per_sm,
              shape_.block_extend, shape_.sort_rays, shape_.speculate, wave_paths_, shape_.shade_kernel, bvh_leaf_,
              bvh_gpu_, shape_.shadow_near, shape_.fuse_camera};
    float best_ms;
    int r;
    if ((r = measure(best, best_ms))) return r;
    res.default_ms = best_ms;
    auto consider = [&](Cand c) -> int {
        float ms;
        int rr;
        if ((rr = measure(c, ms))) return rr;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
        return PT_OK;
    };
    // coordinate descent: BVH width, then material sorting, ray sorting, speculation, grid and
    // block size, then the wave size (the queues' capacity). A batch keeps its BVH width (a
    // change rebuilds every scene of the batch) and its queue order (no ray sorting).
    const int widths_small[3] = {2, 4, 8}, widths_large[2] = {4, 8};
    const int* widths = prims < 100000 ? widths_small : widths_large;
    const int nw = batch ? 0 : (prims < 100000 ? 3 : 2);
    const Cand start = best;
    for (int i = 0; i < nw; i++)
        if (widths[i] != start.width) {
            Cand c = best;
            c.width = widths[i];
            if ((r = consider(c))) return r;
        }
    if (!batch) {  // the tree's builder: the host's binned SAH or the device's PLOC clustering
        Cand c = best;
        c.builder = best.builder == kGpuBvhPloc ? 0 : kGpuBvhPloc;
        if ((r = consider(c))) return r;
    }
    if (!batch) {  // primitives per leaf (each a rebuild of the tree)
        const int start_leaf = best.leaf;
        for (int lf : {2, 4, 8, 16})
            if (lf != start_leaf) {
                Cand c = best;
                c.leaf = lf;
                if ((r = consider(c))) return r;
            }
    }
    if (material_classes_ >= 2) {
        Cand c = best;
        c.sort = best.sort ? 0 : 1;
        if ((r = consider(c))) return r;
    }
    if (!guiding_) {  // the plain shade stage: per-class kernels (sorted frames), one kernel at 128 or 80 registers
        const Cand base = best;
        for (int k : {kShadeAll128, kShadeClasses, kShadeAll80})
            if (k != base.split && (k != kShadeClasses || base.sort)) {
                Cand c = base;
                c.split = k;
                if ((r = consider(c))) return r;
            }
    }
    if (!batch && max_depth_ > 1) {
        Cand c = best;
        c.rays = best.rays ? 0 : 1;
        if ((r = consider(c))) return r;
    }
    {
        const Cand base = best;  // speculation per traversal stage: none, either, both
        for (int bits = 0; bits <= (kSpeculateExtend | kSpeculateShadow); bits++)
            if (bits != base.spec) {
                Cand c = base;
                c.spec = bits;
                if ((r = consider(c))) return r;
            }
    }
    if (nee_ && max_depth_ > 1) {  // the shadow stage's child order: nearest first or the node's order
        Cand c = best;
        c.near = best.near ? 0 : 1;
        if ((r = consider(c))) return r;
    }
    if (!guiding_) {  // camera rays computed where used (the 128-register shade kernel) or queued
        Cand c = best;
        c.fuse = best.fuse ? 0 : 1;
        if ((r = consider(c))) return r;
    }
    for (int bps : {8, 24}) {
        Cand c = best;
        c.bps = bps;
        if ((r = consider(c))) return r;
    }
    {
        Cand c = best;
        c.block = best.block == 128 ? 256 : 128;
        if ((r = consider(c))) return r;
    }
    {
        // a wave holds at most kMaxWavePaths paths; halving it only matters where it splits
        // the frame into more waves (shallower queues, shorter deep-depth tails)
        const int base_wave = best.wave;
        for (int wv : {kMaxWavePaths, kMaxWavePaths / 2, kMaxWavePaths / 4})
            if (wv != base_wave && (long long)wv < frame_paths) {
                Cand c = best;
                c.wave = wv;
                if ((r = consider(c))) return r;
            }
    }
    if ((r = apply(best))) return r;
    stage_timing_ = saved_timing;
    reset();
    report(best);
    res.best_ms = best_ms;
    res.trials = trials;
    if (cache_path) {
        FILE* f = std::fopen(cache_path, "a");
        if (f) {
            std::fprintf(f,
                         "{\"key\": \"%s\", \"bvh_width\": %d, \"sort\": %d, \"blocks_per_sm\": %d, \"block\": %d, "
                         "\"sort_rays\": %d, \"speculate\": %d, \"wave_paths\": %d, \"shade_kernel\": %d, "
                         "\"max_leaf\": %d, \"builder\": %d, \"shadow_near\": %d, \"fuse_camera\": %d, "
                         "\"ms\": %.4f, \"default_ms\": %.4f}\n",
                         key.c_str(), best.width, best.sort, best.bps, best.block, best.rays, best.spec, best.wave,
                         best.split, best.leaf, best.builder, best.near, best.fuse, best_ms, res.default_ms);
            std::fclose(f);
        }
    }
    if (out) *out = res;
    return PT_OK;
}

int Session::set_profiling(int stage_timing, int work_counters) {
    if (in_flight_) return fail(PT_ERR_STATE, "a frame is in flight");
    stage_timing_ = stage_timing ? 1 : 0;
    work_counters_ = work_counters ? 1 : 0;
    return PT_OK;
}

int Session::profile(pt_profile* out) const {
    std::memset(out, 0, sizeof(*out));
    for (int k = 0; k < kNumStages && k < PT_NUM_STAGES; k++) {
        out->stage_ms[k] = stage_ms_[k];
        out->stage_launches[k] = stage_launches_[k];
    }
    out->extend_nodes = last_stats_.extend_nodes;
    out->extend_prims = last_stats_.extend_prims;
    out->shadow_nodes = last_stats_.shadow_nodes;
    out->shadow_prims = last_stats_.shadow_prims;
    out->bvh_width = bvh_.width;
    out->node_bytes = bvh_nodes_quantized() ? qnode_bytes(bvh_.width) : bvh_.width == 2 ? 64 : bvh_.width == 4 ? 128 : 256;
    out->prim_bytes = 48;
    out->wave_paths = last_wave_paths_;
    out->graph_captures = graph_captures_;
    return PT_OK;
}

int Session::readback(float* rgb, size_t n, bool pass) {
    const size_t need = (size_t)w_ * h_ * 3;
    if (!rgb || n < need) return fail(PT_ERR_ARG, "readback buffer too small");
    if (!dev_ready_ || frames_ == 0) return fail(PT_ERR_STATE, "nothing rendered yet");
    int r;
    if ((r = wait(nullptr))) return r;
    DevBuf& src = pass ? d_pass_ : d_accum_;
    if ((r = check_cuda(cudaMemcpyAsync(rgb, src.p, need * 4, cudaMemcpyDeviceToHost, stream_), "readback"))) return r;
    return check_cuda(cudaStreamSynchronize(stream_), "readback");
}

int Session::readback_async(float* rgb, size_t n) {
    const size_t need = (size_t)w_ * h_ * 3;
    if (!rgb || n < need) return fail(PT_ERR_ARG, "readback buffer too small");
    if (!dev_ready_ || (frames_ == 0 && !in_flight_)) return fail(PT_ERR_STATE, "nothing rendered yet");
    int r;
    if ((r = readback_wait())) return r;  // the staging buffer holds one image at a time
    if (!copy_stream_) {
        if ((r = check_cuda(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking), "cudaStreamCreate")))
            return r;
        if ((r = check_cuda(cudaEventCreateWithFlags(&rb_snap_, cudaEventDisableTiming), "cudaEventCreate"))) return r;
        if ((r = check_cuda(cudaEventCreateWithFlags(&rb_done_, cudaEventDisableTiming), "cudaEventCreate"))) return r;
    }
    if ((r = check_cuda(d_rb_stage_.alloc(need * 4), "readback staging"))) return r;
    // snapshot behind the last enqueued frame (device to device), then copy out on the side
    if ((r = check_cuda(cudaMemcpyAsync(d_rb_stage_.p, d_accum_.p, need * 4, cudaMemcpyDeviceToDevice, stream_),
                        "readback snapshot")))
        return r;
    if ((r = check_cuda(cudaEventRecord(rb_snap_, stream_), "cudaEventRecord"))) return r;
    if ((r = check_cuda(cudaStreamWaitEvent(copy_stream_, rb_snap_, 0), "cudaStreamWaitEvent"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(rgb, d_rb_stage_.p, need * 4, cudaMemcpyDeviceToHost, copy_stream_),
                        "readback")))
        return r;
    if ((r = check_cuda(cudaEventRecord(rb_done_, copy_stream_), "cudaEventRecord"))) return r;
    rb_pending_ = true;
    return PT_OK;
}

int Session::readback_wait() {
    if (!rb_pending_) return PT_OK;
    rb_pending_ = false;
    return check_cuda(cudaEventSynchronize(rb_done_), "readback");
}

int Session::readback_rgba8(uint8_t* out, size_t n) {
    const size_t need = (size_t)w_ * h_ * 4;
    if (!out || n < need) return fail(PT_ERR_ARG, "readback buffer too small");
    if (!dev_ready_ || frames_ == 0) return fail(PT_ERR_STATE, "nothing rendered yet");
    int r;
    if ((r = wait(nullptr))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(out, d_rgba8_.p, need, cudaMemcpyDeviceToHost, stream_), "readback"))) return r;
    return check_cuda(cudaStreamSynchronize(stream_), "readback");
}

int Session::hit_test(int x, int y, int* mat) {
    if (!have_scene_) return fail(PT_ERR_STATE, "no scene loaded");
    if (batch_mode()) return fail(PT_ERR_STATE, "not available for a batch (one query per scene session)");
    if (x < 0 || y < 0 || x >= w_ || y >= h_) {
        // the reference's kernel matches no thread and reports no hit
        *mat = -1;
        return PT_OK;
    }
    int r;
    if ((r = ensure_device())) return r;
    if (in_flight_ && (r = wait(nullptr))) return r;
    if (scene_dirty_ && (r = upload_scene())) return r;
    if (mats_dirty_ && (r = upload_materials())) return r;
    std::string err;
    if (!make_camera(camspec_, w_, h_, cam_, err)) return fail(PT_ERR_ARG, err);
    if ((r = check_cuda(d_scratch_.alloc(64), "scratch"))) return r;
    int* dm = d_scratch_.as<int>();
    if ((r = check_cuda(cudaMemsetAsync(dm, 0, 8, stream_), "memset"))) return r;
    if ((r = check_cuda(enqueue_hit_test(scene_view(), cam_, bvh_.depth + 1, x, y, dm, dm + 1, stream_), "hit test")))
        return r;
    int res[2];
    if ((r = check_cuda(cudaMemcpyAsync(res, dm, 8, cudaMemcpyDeviceToHost, stream_), "hit test readback"))) return r;
    if ((r = check_cuda(cudaStreamSynchronize(stream_), "hit test"))) return r;
    if (res[1]) return fail(PT_ERR_DEVICE, "traversal stack overflow reported by a kernel");
    *mat = res[0];
    return PT_OK;
}

int Session::trace_rays(const float* o, const float* d, const float* tmin, const float* tmax, int n, int* pty,
                        int* pid, int* mid, float* t, float* bary, bool device_ptrs) {
    if (!have_scene_) return fail(PT_ERR_STATE, "no scene loaded");
    if (batch_mode()) return fail(PT_ERR_STATE, "not available for a batch (one query per scene session)");
    if (n < 0) return fail(PT_ERR_ARG, "negative ray count");
    if (n == 0) return PT_OK;
    if (!o || !d || !tmin || !tmax || !pty || !pid || !mid || !t) return fail(PT_ERR_ARG, "null array");
    int r;
    if ((r = ensure_device())) return r;
    if (in_flight_ && (r = wait(nullptr))) return r;
    if (scene_dirty_ && (r = upload_scene())) return r;
    if (mats_dirty_ && (r = upload_materials())) return r;
    const int sd = stack_entries();
    if (stack_bytes(sd, 128) > (size_t)kMaxStackBytesDefault)
        return fail(PT_ERR_SCENE, "BVH too deep for the traversal stack in shared memory");
    if (device_ptrs) {
        if ((r = check_cuda(d_scratch_.alloc(64), "scratch"))) return r;
        int* of = d_scratch_.as<int>();
        if ((r = check_cuda(cudaMemsetAsync(of, 0, 4, stream_), "memset"))) return r;
        if ((r = check_cuda(enqueue_trace_rays(scene_view(), sd, o, d, tmin, tmax, n, pty, pid, mid, t, bary, of, stream_),
                            "trace rays")))
            return r;
        int hof = 0;
        if ((r = check_cuda(cudaMemcpyAsync(&hof, of, 4, cudaMemcpyDeviceToHost, stream_), "readback"))) return r;
        if ((r = check_cuda(cudaStreamSynchronize(stream_), "trace rays"))) return r;
        if (hof) return fail(PT_ERR_DEVICE, "traversal stack overflow reported by a kernel");
        return PT_OK;
    }
    // inputs 3+3+1+1 floats, outputs 3 ints + t + 2 bary, plus the overflow flag
    const size_t N = (size_t)n;
    const size_t bytes = N * 4 * (8 + 6) + 256;
    if ((r = check_cuda(d_scratch_.alloc(bytes), "scratch"))) return r;
    char* base = d_scratch_.as<char>();
    float* dO = (float*)base;
    float* dD = dO + 3 * N;
    float* dTmin = dD + 3 * N;
    float* dTmax = dTmin + N;
    int* dPt = (int*)(dTmax + N);
    int* dPid = dPt + N;
    int* dMid = dPid + N;
    float* dT = (float*)(dMid + N);
    float* dB = dT + N;
    int* dOf = (int*)(dB + 2 * N);
    cudaStream_t st = stream_;
    if ((r = check_cuda(cudaMemcpyAsync(dO, o, 12 * N, cudaMemcpyHostToDevice, st), "copy rays"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(dD, d, 12 * N, cudaMemcpyHostToDevice, st), "copy rays"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(dTmin, tmin, 4 * N, cudaMemcpyHostToDevice, st), "copy rays"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(dTmax, tmax, 4 * N, cudaMemcpyHostToDevice, st), "copy rays"))) return r;
    if ((r = check_cuda(cudaMemsetAsync(dOf, 0, 4, st), "memset"))) return r;
    if ((r = check_cuda(enqueue_trace_rays(scene_view(), sd, dO, dD, dTmin, dTmax, n, dPt, dPid, dMid, dT,
                                           bary ? dB : nullptr, dOf, st),
                        "trace rays")))
        return r;
    if ((r = check_cuda(cudaMemcpyAsync(pty, dPt, 4 * N, cudaMemcpyDeviceToHost, st), "copy hits"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(pid, dPid, 4 * N, cudaMemcpyDeviceToHost, st), "copy hits"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(mid, dMid, 4 * N, cudaMemcpyDeviceToHost, st), "copy hits"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(t, dT, 4 * N, cudaMemcpyDeviceToHost, st), "copy hits"))) return r;
    if (bary && (r = check_cuda(cudaMemcpyAsync(bary, dB, 8 * N, cudaMemcpyDeviceToHost, st), "copy hits"))) return r;
    int hof = 0;
    if ((r = check_cuda(cudaMemcpyAsync(&hof, dOf, 4, cudaMemcpyDeviceToHost, st), "copy flag"))) return r;
    if ((r = check_cuda(cudaStreamSynchronize(st), "trace rays"))) return r;
    if (hof) return fail(PT_ERR_DEVICE, "traversal stack overflow reported by a kernel");
    return PT_OK;
}

int Session::trace_rays_static(const float* o, const float* d, const float* tmin, const float* tmax, int n, int* pty,
                               int* pid, int* mid, float* t, float* bary) {
    if (batch_mode()) return fail(PT_ERR_STATE, "not available for a batch (one query per scene session)");
    if (n < 0 || n > kStaticTraceMaxRays)
        return fail(PT_ERR_ARG, "ray count must be in [0, " + std::to_string(kStaticTraceMaxRays) + "]");
    if (n > 0 && (!o || !d || !tmin || !tmax || !pty || !pid || !mid || !t)) return fail(PT_ERR_ARG, "null array");
    // Nothing may be allocated here: device set-up and the scene upload must already be done.
    if (!have_scene_) return fail(PT_ERR_STATE, "no scene loaded");
    if (!dev_ready_ || scene_dirty_ || mats_dirty_)
        return fail(PT_ERR_STATE,
                    "scene not resident on the device; make one allocating device call (render, trace, hit "
                    "test) after loading or editing the scene");
    const int sd = bvh_.depth + 1;
    if (stack_bytes(sd, 128) > (size_t)kMaxStackBytesDefault)
        return fail(PT_ERR_SCENE, "BVH too deep for the traversal stack in shared memory");
    int r;
    if ((r = check_cuda(cudaSetDevice(device_), "cudaSetDevice"))) return r;
    int of = 0;
    // on the session's query stream: a frame in flight on the render stream keeps running
    if ((r = check_cuda(pt::trace_rays_static(scene_view(), sd, o, d, tmin, tmax, n, pty, pid, mid, t, bary, &of,
                                              query_stream_),
                        "static trace rays")))
        return r;
    if (of) return fail(PT_ERR_DEVICE, "traversal stack overflow reported by a kernel");
    return PT_OK;
}

int Session::occluded(const float* o, const float* d, const float* tmin, const float* tmax, int n, int* occ) {
    if (!have_scene_) return fail(PT_ERR_STATE, "no scene loaded");
    if (batch_mode()) return fail(PT_ERR_STATE, "not available for a batch (one query per scene session)");
    if (n < 0) return fail(PT_ERR_ARG, "negative ray count");
    if (n == 0) return PT_OK;
    if (!o || !d || !tmin || !tmax || !occ) return fail(PT_ERR_ARG, "null array");
    int r;
    if ((r = ensure_device())) return r;
    if (in_flight_ && (r = wait(nullptr))) return r;
    if (scene_dirty_ && (r = upload_scene())) return r;
    if (mats_dirty_ && (r = upload_materials())) return r;
    const int sd = stack_entries();
    const size_t N = (size_t)n;
    if ((r = check_cuda(d_scratch_.alloc(N * 4 * 9 + 256), "scratch"))) return r;
    float* dO = d_scratch_.as<float>();
    float* dD = dO + 3 * N;
    float* dTmin = dD + 3 * N;
    float* dTmax = dTmin + N;
    int* dOcc = (int*)(dTmax + N);
    int* dOf = dOcc + N;
    cudaStream_t st = stream_;
    if ((r = check_cuda(cudaMemcpyAsync(dO, o, 12 * N, cudaMemcpyHostToDevice, st), "copy rays"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(dD, d, 12 * N, cudaMemcpyHostToDevice, st), "copy rays"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(dTmin, tmin, 4 * N, cudaMemcpyHostToDevice, st), "copy rays"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(dTmax, tmax, 4 * N, cudaMemcpyHostToDevice, st), "copy rays"))) return r;
    if ((r = check_cuda(cudaMemsetAsync(dOf, 0, 4, st), "memset"))) return r;
    if ((r = check_cuda(enqueue_occluded(scene_view(), sd, dO, dD, dTmin, dTmax, n, dOcc, dOf, st), "occluded"))) return r;
    if ((r = check_cuda(cudaMemcpyAsync(occ, dOcc, 4 * N, cudaMemcpyDeviceToHost, st), "copy"))) return r;
    int hof = 0;
    if ((r = check_cuda(cudaMemcpyAsync(&hof, dOf, 4, cudaMemcpyDeviceToHost, st), "copy flag"))) return r;
    if ((r = check_cuda(cudaStreamSynchronize(st), "occluded"))) return r;
    if (hof) return fail(PT_ERR_DEVICE, "traversal stack overflow reported by a kernel");
    return PT_OK;
}

}  // namespace pt
