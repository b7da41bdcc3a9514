// Host-visible launch interface of the wavefront integrator kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "guide.h"
#include "pt_types.h"

namespace pt {

// Per-slot path state of a ray queue (structure of arrays, 16-byte elements).
struct PathQueue {
    float4* o;     // origin.xyz, wave-local path index (int bits)
    float4* d;     // direction.xyz, pdf of the BSDF sample that produced the ray
    float4* beta;  // throughput.xyz, flags (int bits): bit 0 = no MIS on the next emission
    uint2* rng;    // PCG32 state
    float4* hit;   // t, b1, b2, primitive (int bits); written by the extend stage. A negative t
                   // (-t) marks a continuation hit whose BSDF-direct ray stopped closer (hitd)
    float4* hitd;  // the BSDF-direct ray's hit where it lies closer than the continuation's tMin
                   // (written and read only for marked slots; one array shared by both queues)
    int* key;      // material-sort key of the hit (shade stage order), optional
};

struct ShadowQueue {
    float4* o;  // origin.xyz, tmax
    float4* d;  // direction.xyz, wave-local path index (int bits)
    float4* c;  // contribution (beta * f * cos * Le * w / pdf).xyz, unused
};

constexpr int kMaxDepthLimit = 64;

// Device counters of one wave (zeroed at wave start).
struct WaveCounters {
    int ray_count[kMaxDepthLimit + 1];     // rays in the queue consumed at depth d
    int shadow_count[kMaxDepthLimit + 1];  // shadow rays produced at depth d
    int work_extend[kMaxDepthLimit + 1];   // persistent work-fetch cursors
    int work_shade[kMaxDepthLimit + 1];
    int work_shadow[kMaxDepthLimit + 1];
    int work_class[kMaxDepthLimit + 1][8];  // fetch cursors of the per-class shade kernels
    int sort_count[kMaxDepthLimit + 1][8]; // per material class hit counts (sorted shading)
    int sort_fill[kMaxDepthLimit + 1][8];
};

// Frame-wide device statistics (not reset per wave).
struct FrameStats {
    unsigned long long rays_camera;
    unsigned long long rays_extend;   // closest-hit queries (camera + continuation)
    unsigned long long rays_shadow;   // any-hit queries
    unsigned long long extend_nodes;  // wide nodes loaded by closest-hit queries (work-count frames)
    unsigned long long extend_prims;  // leaf entries tested by closest-hit queries
    unsigned long long shadow_nodes;
    unsigned long long shadow_prims;
    int error;                        // bit 0: traversal stack overflow
    int pad;
};

// Stages of a frame, for per-stage device timing.
enum Stage : int {
    kStageCamera = 0,
    kStageExtend,
    kStageSort,
    kStageShade,
    kStageShadow,
    kStageAccum,
    kStageGuide,  // guide inference + training-sample collection
    kNumStages
};

// Host-side recorder of stage boundaries: an event is recorded after every launch.
struct StageMarks {
    cudaEvent_t* events = nullptr;  // pool
    int capacity = 0;
    int used = 0;
    int* stage = nullptr;           // stage of the launch that ends at events[i] (-1: no launch)
    int* begin = nullptr;           // the event on the same stream before that launch (-1: none)
};

struct LaunchShape {
    int block_extend = 128;
    int block_shade = 128;
    int block_shadow = 128;
    int blocks_per_sm = 16;   // persistent grid = SMs * blocks_per_sm
    int sort_materials = 1;   // material-sorted shading
    int sort_rays = 0;        // continuation rays extended in (origin cell, direction octant) order
    int refill_idle = 16;     // traversal stages: a warp fetches new rays once this many lanes are idle
    int speculate = 0;        // kSpeculate* bits: stages that park a lane's first leaf and descend on
    int shade_kernel = 1;     // plain frames' shade stage: kShadeAll128, kShadeClasses, kShadeAll80
    int overlap_shadow = 1;   // shadow stage of depth d on the side stream beside extend of d + 1
    int shadow_near = 0;      // shadow stage: a node's hit children visited nearest first (else in order)
    int fuse_camera = 1;      // depth-0 rays computed where used when the shade kernel allows (cam_fused)
};

// The side streams of a frame whose independent stages overlap (LaunchShape.overlap_shadow):
// the shadow stage of depth d beside the closest-hit stage of depth d + 1, with one fork and
// one join event per depth, and the per-class shade kernels of a depth side by side, each on
// its own stream between a fork and a join event.
struct SideStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t* shaded = nullptr;    // recorded on the main stream after the shade stage of depth d
    cudaEvent_t* shadowed = nullptr;  // recorded on the side stream after the shadow stage of depth d
    cudaStream_t* cls = nullptr;      // kMaterialClasses streams of the class shade kernels
    cudaEvent_t cls_fork = nullptr;   // recorded on the main stream before them
    cudaEvent_t* cls_done = nullptr;  // recorded on each class stream after its kernel
};

constexpr int kShadeAll128 = 0;  // one kernel for all materials, 128 registers
constexpr int kShadeClasses = 1; // material-sorted frames: one kernel per material class present
constexpr int kShadeAll80 = 2;   // one kernel for all materials, 80 registers

constexpr int kSpeculateExtend = 1;  // closest-hit stage
constexpr int kSpeculateShadow = 2;  // shadow (any-hit) stage

// Ray sorting ahead of the closest-hit stage (single-scene frames, depth >= 1): the key of a
// ray is its origin's cell in a 4x4x4 grid over the scene bounds and its direction octant.
constexpr int kRaySortBlock = 256;
constexpr int kRayBuckets = 512;  // 2 per thread of a ray-sort block
static_assert(kRayBuckets == 2 * kRaySortBlock, "ray-sort scan layout");

// Values that change from frame to frame live in device memory, so a captured CUDA graph
// of the frame's launches stays valid across frames; the host updates them with one copy
// before each launch.
struct FrameDyn {
    CameraParams cam;
    uint64_t seed;
    uint64_t sample_base;    // samples per pixel rendered before this frame (RNG offset)
    int prev_spp;            // samples accumulated before this frame
    int pad[3];
};

// Queue tag carried in the origin's w (and the shadow direction's w): the path's index within
// its wave in the low 25 bits, the scene of a batched frame above them. A wave therefore holds
// at most 2^25 paths.
constexpr int kTagPathBits = 25;
constexpr int kTagPathMask = (1 << kTagPathBits) - 1;
constexpr int kMaxWavePaths = 1 << kTagPathBits;
constexpr int kMaxBatchScenes = 64;

// One scene of a batched frame: its part of the concatenated geometry, its image and sampling
// parameters and its guide network. The host rewrites the per-frame fields (camera, seed,
// sample base, previous spp) before every frame.
struct BatchScene {
    int root;                // root node in the concatenated BVH
    int light_first;         // first emitter in the concatenated emitter list
    int num_lights;
    int width, height, spp, max_depth;
    int guide_net;           // network index, -1 without guiding
    int guide_mode;          // 0 off, 1 collect, 2 guided sampling
    int pad0;
    long long path_base;     // first path of this scene in the frame's global path order
    long long pixel_base;    // first pixel in the concatenated image buffers
    long long guided_base;   // paths of guided scenes (spec.guided) before this one, in path order
    EnvDevice env;
    GuideFrame gframe;
    CameraParams cam;
    uint64_t seed;
    uint64_t sample_base;    // samples per pixel rendered before this frame
    int prev_spp;
    int pad1[3];
};

// A wave of a frame: whole pixels [first_pixel, first_pixel + npix) of the global pixel order,
// whose paths are [first_path, first_path + npaths).
struct WaveRange {
    int first_pixel, npix;
    long long first_path;
    int npaths, pad;
    // training paths are counted over guided scenes only: the wave's first guided-path index
    // and how many guided paths it holds (a single scene: 0 and npaths)
    long long guided_first;
    int guided_n, pad2;
};

struct FrameParams {
    SceneDevice sc;
    const FrameDyn* dyn;     // device pointer
    PathQueue q[2];
    ShadowQueue sq;
    float4* L;               // wave-local path radiance
    int* sort_index;         // material-sorted slot order
    int* ray_index;          // ray-sorted slot order of the closest-hit stage (shape.sort_rays)
    int* ray_hist;           // per depth: kRayBuckets bucket counts, then kRayBuckets fill cursors
    WaveCounters* counters;
    FrameStats* stats;
    float* pass_rgb;         // W*H*3: this frame's per-pixel mean (passRadiances)
    float* accum_rgb;        // W*H*3: running mean across frames (radiances)
    uchar4* rgba8;           // W*H display buffer
    int width, height;
    int spp;                 // samples per pixel of this frame
    int max_depth;
    int nee;
    int wave_pixels;         // pixels per wave
    int stack_depth;         // traversal stack entries per thread
    int num_sms;
    int count_work;          // 1: traversal kernels count nodes and leaf entries (slower)
    int renderer;            // 0 path tracer, 1 normals (one pixel-centre ray per pixel, spp 1)
    LaunchShape shape;
    // ---- learned path guiding (guide.cuh) ----
    int guide_mode;          // 0 off, 1 collect training data only, 2 guided sampling + collect
    int cam_fused;           // set per wave: depth-0 rays computed where used, not queued (see k_wave_start)
    float gfrac;             // probability of sampling the guide at a non-delta vertex
    int consistent_mis;      // NEE weights use the BSDF's true sampling density (microfacet)
    int guide_tc;            // guide inference on tcgen05 / tensor memory (single-scene frames)
    int class_mask;          // material classes that can occur (bit 0 miss, bit type + 1); 0: one shade kernel
    int mma_test_polls;      // test hook: > 0 limits the first wait of each tcgen05 layer (tc_network)
    const uint32_t* gwpack;  // packed inference weights
    GuideFrame gframe;       // scene bounds for the position encoding
    float* gmix;             // per queue slot: mixture (40 floats)
    GuideRecord* grec;       // vertex records of training paths (this wave)
    int* grec_count;
    int grec_cap;
    float* gacc;             // per training path and depth: U, R, W luminance (3 floats)
    int gstride;             // paths whose wave index is a multiple of gstride are training paths
    GuideSample* gring;      // training-sample ring
    int* gring_count;
    int gring_cap;
    // training launched after the frame (captured with it): Adam steps, minibatch, rate
    int gtrain_steps;
    int gtrain_batch;
    float gtrain_lr;
    // ---- batched frames (num_scenes > 0): the scene table and its prefix offsets ----
    const BatchScene* batch;
    const long long* batch_path_base;   // num_scenes + 1 entries
    const long long* batch_pixel_base;  // num_scenes + 1 entries
    int num_scenes;
    int gnets;               // guide networks trained after the frame
};

// Enqueue one batched frame (p.num_scenes > 0): the given waves over the scenes' global path
// order, every stage one launch for all scenes of the wave.
cudaError_t enqueue_batch_frame(const FrameParams& p, const WaveRange* waves, int nwaves, cudaStream_t stream,
                                StageMarks* marks = nullptr, const SideStream* side = nullptr);

// Enqueue one frame (all waves) on `stream`. Grid sizes do not depend on queue lengths,
// so the sequence can be captured into a CUDA graph. With `marks`, an event is recorded
// after every launch (per-stage timing; not capturable). With `side` and
// p.shape.overlap_shadow (and no marks), each depth's shadow stage runs on the side stream.
cudaError_t enqueue_frame(const FrameParams& p, cudaStream_t stream, StageMarks* marks = nullptr,
                          const SideStream* side = nullptr);

// Raise the dynamic shared-memory limit of the traversal kernels to `bytes`.
cudaError_t configure_traversal_smem(size_t bytes);
// Opt the guide inference kernel into its dynamic shared memory (weights + 8 warps x 32 rows).
cudaError_t configure_guide_infer();

// Closest-hit queries for caller-provided rays (parity entry). Arrays are device pointers.
cudaError_t enqueue_trace_rays(const SceneDevice& sc, int stack_depth, const float* o, const float* d,
                               const float* tmin, const float* tmax, int n, int* prim_type, int* prim_id,
                               int* mat_id, float* t, float* bary, int* overflow, cudaStream_t stream);

// Any-hit queries for caller-provided rays: occluded[i] = 1 if something lies in [tmin, tmax].
cudaError_t enqueue_occluded(const SceneDevice& sc, int stack_depth, const float* o, const float* d,
                             const float* tmin, const float* tmax, int n, int* occluded, int* overflow,
                             cudaStream_t stream);

// One camera ray through the centre of pixel (x = col, y = row) (src/hit_test.cu:25-47).
cudaError_t enqueue_hit_test(const SceneDevice& sc, const CameraParams& cam, int stack_depth, int x, int y,
                             int* out_material, int* overflow, cudaStream_t stream);

// Closest-hit queries that allocate nothing: host rays in, host results out, staged through
// a file-scope __device__ array of kStaticTraceMaxRays entries (see wavefront.cu). The
// first call on a device looks the array's address up (cudaGetSymbolAddress) with that
// device current. Returns cudaErrorInvalidValue for n outside [0, kStaticTraceMaxRays].
constexpr int kStaticTraceMaxRays = 65536;
cudaError_t trace_rays_static(const SceneDevice& sc, int stack_depth, const float* o, const float* d,
                              const float* tmin, const float* tmax, int n, int* prim_type, int* prim_id,
                              int* mat_id, float* t, float* bary, int* overflow, cudaStream_t stream);

// Read bandwidth (GB/s, best of `trials` launches of `reps` passes) of an L2-resident buffer of
// `bytes` on the current device (probe.cu).
cudaError_t measure_l2_read(size_t bytes, int reps, int trials, double* gbs, double* ms);

// Size in bytes of the traversal stack per block for `threads` threads.
inline size_t stack_bytes(int stack_depth, int threads) { return (size_t)stack_depth * threads * sizeof(int2); }

}  // namespace pt
