/*
 * pathed.h - C ABI of the B200 path-tracing core (libpathed.so).
 *
 * This is the drop-in boundary for the reference's vanilla CUDA backend. Each entry point
 * names the reference interface it replaces (paths are inside chellmuth/gpu-pathed):
 *
 *   RenderSession          include/render_session.h:41-134, src/render_session.cu:55-136
 *   Renderer / PathTracer  include/renderers/renderer.h:14-35, src/renderers/path_tracer.cu:266-361
 *   SceneModel setters     include/scene_model.h:34-99, src/scene_model.cu:41-347
 *   hit test               src/hit_test.cu:49-82
 *   World::hit             src/world.cu:5-41 (parity entry pt_trace_rays)
 *
 * Conventions: every function returns PT_OK (0) or a negative PT_ERR_* code; on error
 * pt_last_error() holds a message. No function calls exit() or traps the device (the
 * reference exits through gpuAssert, include/macro_helper.h:10-19). Caller-owned host arrays
 * are copied; the session owns all device memory and frees it in pt_destroy. A session is
 * not thread-safe (one thread per session, like the reference's GUI thread).
 *
 * Device work runs on the session's own CUDA stream. Rendering is asynchronous:
 * pt_render_async enqueues one progressive frame, pt_poll reports completion.
 */
#ifndef PATHED_H
#define PATHED_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PT_OK 0
#define PT_ERR_ARG (-1)      /* invalid argument */
#define PT_ERR_STATE (-2)    /* call not valid in the current state (no scene, frame in flight) */
#define PT_ERR_CUDA (-3)     /* CUDA runtime error (no device, out of memory, launch failure) */
#define PT_ERR_SCENE (-4)    /* scene rejected (validation, BVH build) */
#define PT_ERR_DEVICE (-5)   /* a kernel reported an error flag (e.g. traversal stack overflow) */

/* Material types: same values as the reference enum (include/materials/types.h:5-11). */
#define PT_LAMBERTIAN 0
#define PT_MIRROR 1
#define PT_GLASS 2
#define PT_MICROFACET 3

/* Renderer types (include/scene_model.h:16-20) for pt_set_renderer. CUDA (the path tracer)
 * and NORMALS (the G-buffer) are built; there is no OptiX backend. */
#define PT_RENDERER_CUDA 0
#define PT_RENDERER_OPTIX 1
#define PT_RENDERER_NORMALS 2

typedef struct pt_session pt_session;

/* Scene arrays handed over by a caller (replaces SceneData, include/scene_data.h:19-41,
 * which the reference fills from OBJ/PLY parsers). Triangles keep the reference's record:
 * three vertices, three shading normals (interpolated, not renormalised), a material id.
 * tri_normals may be NULL: each vertex then takes the normalised geometric normal of its
 * triangle (cross(p1 - p0, p2 - p0)). env_rgba may be NULL (no environment light). */
typedef struct pt_scene_desc {
    int num_triangles;
    const float* tri_vertices;   /* 9 floats per triangle: p0, p1, p2 */
    const float* tri_normals;    /* 9 floats per triangle: n0, n1, n2, or NULL */
    const int* tri_materials;
    int num_spheres;
    const float* spheres;        /* 4 floats per sphere: cx, cy, cz, radius */
    const int* sphere_materials;
    int num_materials;
    const int* material_types;   /* PT_LAMBERTIAN .. PT_MICROFACET */
    const float* material_albedo;/* 3 per material (Lambertian) */
    const float* material_emit;  /* 3 per material (Lambertian emitters) */
    const float* material_ior;   /* 1 per material (glass) */
    const float* material_alpha; /* 1 per material (Beckmann microfacet) */
    int env_width, env_height;
    const float* env_rgba;       /* env_width * env_height * 4 floats, row 0 = +y, or NULL */
} pt_scene_desc;

/* Sizes of the loaded scene, for pt_export_scene. */
typedef struct pt_scene_counts {
    int num_triangles, num_spheres, num_materials, num_lights;
    int env_width, env_height;
    int bvh_width, bvh_nodes, bvh_depth, bvh_max_leaf;
    int res_x, res_y;          /* preferred resolution of a generated configuration */
    int default_spp, default_depth, default_nee;
    double bvh_build_ms;
} pt_scene_counts;

/* Caller-allocated destination for pt_export_scene (any pointer may be NULL). */
typedef struct pt_scene_export {
    float* tri_vertices;   /* 9 * num_triangles */
    float* tri_normals;    /* 9 * num_triangles */
    int* tri_materials;
    float* spheres;        /* 4 * num_spheres */
    int* sphere_materials;
    int* material_types;
    float* material_albedo;/* 3 * num_materials */
    float* material_emit;
    float* material_ior;
    float* material_alpha;
    int* light_types;      /* num_lights: 0 triangle, 1 sphere (include/lights/types.h:14-17) */
    int* light_indices;
    float* env_rgba;       /* env_width * env_height * 4 */
    float* camera;         /* 11 floats: origin[3], target[3], up[3], vfov (radians), flip */
} pt_scene_export;

/* Launch shape and queue sizing (the autotuner's knobs). Zero fields keep the current value. */
typedef struct pt_launch_config {
    int wave_paths;        /* paths in flight per wave (queue capacity) */
    int block_extend;      /* threads per block of the closest-hit stage */
    int block_shade;       /* at most 512; guided frames shade with their own 128-thread blocks */
    int block_shadow;
    int blocks_per_sm;     /* persistent grid = SMs * blocks_per_sm */
    int sort_materials;    /* 1: material-sorted shading, 2: off, 3: automatic (on when the
                              scene has 2 or more material types; default) (0 keeps current) */
    int use_graph;         /* 1: capture each frame's launches in a CUDA graph and replay it
                              while the launch parameters are unchanged (default), 2: off */
    int sort_rays;         /* 1: sort continuation rays by origin cell and direction octant
                              before the closest-hit stage (single-scene frames), 2: off
                              (default); images are the same either way */
    int refill_idle;       /* closest-hit and shadow stages: a warp takes new rays from its queue
                              once this many of its 32 lanes are idle (1-32; 32 = only when all
                              are; default 16) */
    int speculate;         /* speculative traversal (a lane parks its first leaf and keeps
                              descending while other lanes of its warp search for one):
                              1 closest-hit and shadow stages, 2 off (default), 3 closest-hit
                              stage only, 4 shadow stage only */
    int split_shade;       /* the shade stage of frames without guiding: 1 one kernel per material
                              class present, each compiled for its BSDF only (material-sorted
                              frames; default), 2 one kernel for all materials at 128 registers,
                              3 the same at 80 registers (more resident warps, some spills);
                              images are the same either way */
    int overlap_shadow;    /* 1: the shadow stage of depth d runs on a second stream beside the
                              closest-hit stage of depth d + 1, each filling the other's tail
                              (default; the shade stage of depth d + 1 waits for both), 2: one
                              stream; images are the same either way */
    int shadow_order;      /* shadow stage: 1 a node's hit children are visited nearest first, 2 in
                              the node's order (default); the same occlusion results either way */
    int fuse_camera;       /* 1 (default): in plain frames whose shade stage is the one kernel at 128
                              registers, the closest-hit and shade stages of depth 0 compute each
                              camera ray from its path index instead of reading it from a queue
                              that a camera stage wrote; 2: always queued; the same images */
} pt_launch_config;

/* Result of pt_autotune. */
typedef struct pt_tune_result {
    int bvh_width;          /* chosen BVH width (2, 4, 8) */
    int sort_materials;     /* 1 on, 2 off */
    int blocks_per_sm;
    int block;              /* threads per block of the traversal stages */
    int wave_paths;
    float best_ms;          /* frame time of the chosen configuration */
    float default_ms;       /* frame time of the configuration before tuning */
    int trials;             /* frames measured (0 when taken from the cache) */
    int from_cache;
    int sort_rays;          /* 1 on, 2 off */
    int speculate;          /* as pt_launch_config.speculate: 1 both stages, 2 off, 3 closest hit, 4 shadow */
    int split_shade;        /* as pt_launch_config.split_shade: 1 per-class kernels, 2 one kernel (128
                               registers), 3 one kernel (80 registers) */
    int max_leaf;           /* primitives per BVH leaf (2, 4, 8 or 16; as pt_set_bvh) */
    int bvh_builder;        /* as pt_set_bvh_builder: 0 host binned SAH, 2 GPU PLOC (single scenes) */
    int shadow_order;       /* as pt_launch_config.shadow_order: 1 nearest first, 2 the node's order */
    int fuse_camera;        /* as pt_launch_config.fuse_camera */
} pt_tune_result;

typedef struct pt_stats {
    unsigned long long rays_camera;   /* camera rays of the last frame */
    unsigned long long rays_extend;   /* closest-hit queries (camera + continuation) */
    unsigned long long rays_shadow;   /* any-hit queries */
    float last_frame_ms;              /* device time of the last completed frame */
    int last_frame_spp;
    int total_spp;
    int frames;
} pt_stats;

/* Per-stage device time of the last frame (replaces the reference's single begin/end event
 * pair and "CUDA Frame: X ms" print, path_tracer.cu:300-352). Stages: 0 camera, 1 extend
 * (closest hit), 2 material sort, 3 shade, 4 shadow (any hit), 5 accumulate, 6 guide
 * (inference and training-sample collection). Work counters are filled only for frames
 * rendered with work counting on. */
#define PT_NUM_STAGES 7
typedef struct pt_profile {
    float stage_ms[PT_NUM_STAGES];
    int stage_launches[PT_NUM_STAGES];
    unsigned long long extend_nodes;  /* wide BVH nodes loaded by closest-hit queries */
    unsigned long long extend_prims;  /* leaf entries (triangles/spheres) tested */
    unsigned long long shadow_nodes;
    unsigned long long shadow_prims;
    int bvh_width;
    int node_bytes;                   /* bytes per wide node */
    int prim_bytes;                   /* bytes per leaf entry */
    int wave_paths;                   /* paths per wave of the last frame */
    int graph_captures;               /* frame CUDA graphs captured by this session so far */
} pt_profile;

/* ---- session lifetime (RenderSession ctor, render_session.cu:55-117) ------------------ */
int pt_create(int width, int height, pt_session** out);
int pt_destroy(pt_session* s);
const char* pt_last_error(const pt_session* s);
/* Select the CUDA device for this session (default: current device). Call before any
 * device work. */
int pt_set_device(pt_session* s, int device);

/* ---- scene (SceneParameters::getSceneData/getCamera, src/scene.cu:14-216) -------------- */
/* Seeded procedural configuration: 0 Cornell box (36 triangles), 1 sixty-four spheres on a
 * plane with 4 sphere emitters, 2 displaced icosphere (1,310,720 triangles) under a
 * 2048x1024 environment map, 3 the same mesh in a closed room lit through a 0.05-wide slit.
 * Also sets the camera and the default depth/NEE. Host work only (scene generation, BVH
 * build); device upload is deferred to the first device call. */
int pt_load_config(pt_session* s, int config, uint64_t seed);
/* Same with an explicit icosphere level for configurations 2 and 3 (smaller test scenes). */
int pt_load_config_level(pt_session* s, int config, uint64_t seed, int icosphere_level);
int pt_load_arrays(pt_session* s, const pt_scene_desc* desc);

/* Mesh files of a scene request (ObjParser / PLYParser, src/parsers/). */
#define PT_MESH_OBJ 0 /* OBJ with an optional MTL library: faces "a b c d" (two triangles,
                         geometric normal), "v/t/n v/t/n v/t/n" and "v//n v//n v//n"; other face
                         forms are skipped, as by the reference's parser */
#define PT_MESH_PLY 1 /* binary little-endian PLY, float x y z, a vertex_indices list */
typedef struct pt_mesh_file {
    const char* path;
    int format;            /* PT_MESH_OBJ or PT_MESH_PLY */
    int default_material;  /* material of faces without MTL materials */
} pt_mesh_file;

/* SceneAdapter::ParseRequest (include/scene_data.h) plus the camera. Triangles of OBJ files
 * come first, then PLY files', in request order; an OBJ's MTL materials are appended as
 * Lambertians (Kd albedo, Ke emission) after the request's own materials, ordered by name. */
typedef struct pt_scene_request {
    int num_files;
    const pt_mesh_file* files;
    int num_materials;           /* material arrays as in pt_scene_desc */
    const int* material_types;
    const float* material_albedo;
    const float* material_emit;
    const float* material_ior;
    const float* material_alpha;
    int num_spheres;
    const float* spheres;        /* 4 floats per sphere: cx, cy, cz, radius */
    const int* sphere_materials;
    const char* env_exr;         /* OpenEXR environment map (EnvironmentLightParams), or NULL */
    const float* camera;         /* 11 floats: origin[3], target[3], up[3], vfov (radians), flip */
} pt_scene_request;

/* Replaces SceneAdapter::createSceneData (src/scene_data.cu:9-118) fed by the reference's
 * parsers: loads the request's files into the session. PT_ERR_SCENE with pt_last_error naming
 * the file and line for a file that cannot be read or parsed. */
int pt_load_request(pt_session* s, const pt_scene_request* request);

/* The reference's built-in scene `index` (SceneParameters::getSceneData / getCamera,
 * src/scene.cu:14-218; RenderSession loads index 0, render_session.cu:68-72): 0 Cornell box,
 * 1 glossy Cornell box with a mirror box and a glass ball, 2 plane under the 1-pixel test
 * environment, 3 the MIS plates under an HDR environment. `scenes_dir` is the reference's
 * scenes/ directory (its files are read from there); max depth 3 and NEE on, as Scene's
 * defaults (include/scene.h:17-29). */
int pt_load_reference_scene(pt_session* s, int index, const char* scenes_dir);

/* LoadEXR (the reference's environment-map reader, src/lights/environment_light.cu:20-31):
 * width x height RGBA floats, rows top first. Single-part scanline files with NONE, RLE,
 * ZIPS, ZIP or PIZ compression and HALF or FLOAT channels; R, G and B are required (A defaults
 * to 1), a single channel fills all four. rgba NULL returns only the size; otherwise n must be
 * at least width * height * 4. Errors are reported through pt_last_error(NULL). */
int pt_read_exr(const char* path, int* width, int* height, float* rgba, size_t n);

/* Image::save (src/io/image.cpp:9-78) of the accumulated radiance, as RenderSession::pollRender
 * writes out.exr at every power-of-two spp (include/render_session.h:87-101): an uncompressed
 * EXR of HALF channels B, G, R with the image's top row first. Waits for a frame in flight. */
int pt_save_exr(pt_session* s, const char* path);
/* The same file from caller radiances: rgb holds width * height * 3 floats, row 0 = the image
 * bottom (the layout of pt_readback). Errors through pt_last_error(NULL). */
int pt_write_exr(const char* path, int width, int height, const float* rgb);
int pt_scene_counts_get(const pt_session* s, pt_scene_counts* out);
int pt_export_scene(const pt_session* s, pt_scene_export* out);
/* Rebuild the BVH with a given width (2, 4, 8) and maximum leaf size (1..16). */
int pt_set_bvh(pt_session* s, int width, int max_leaf);
/* Host-side structural check of the BVH (containment, references); 0 if sound. */
int pt_check_bvh(const pt_session* s);

/* ---- scene model edits (SceneModel setters, src/scene_model.cu:41-347) ---------------- */
/* Camera (Camera ctor + lookAt, src/core/camera.cu:5-21, src/transform.cu:7-33). */
int pt_set_camera(pt_session* s, const float origin[3], const float target[3], const float up[3],
                  float vfov_radians, int flip_handedness);
/* Material edit of an existing id; changing the type resets the parameters to the
 * reference's defaults for that type (Scene::setMaterialType, include/scene.h:36-61). */
int pt_set_material(pt_session* s, int material_id, int type, const float albedo[3],
                    const float emit[3], float ior, float alpha);
int pt_set_max_depth(pt_session* s, int max_depth);  /* vertices per path (path_tracer.cu:165) */
int pt_set_nee(pt_session* s, int enabled);          /* calculateLiNEE vs calculateLiNaive */
int pt_set_seed(pt_session* s, uint64_t seed);
/* ---- learned path guiding (no counterpart in the reference) -----------------------------
 * A network (80 -> 64 -> 64 -> 64 -> 40, ReLU; 16,104 parameters, BF16 weights on the
 * tensor cores, FP32 master copy) maps a 12-frequency sin/cos encoding of the hit position,
 * the shading normal and the outgoing direction to an 8-lobe von Mises-Fisher mixture. It is
 * trained online (Adam, lr 3e-3, minibatches of 2^16 samples, several steps per frame) on
 * radiance samples the integrator produces, and combined with BSDF sampling by one-sample MIS
 * (guide fraction 0.7) so the estimator stays unbiased; MIS weights of emitter sampling then use
 * the mixture density. Before the first steps have been taken, paths are sampled from the
 * BSDF alone while training data is collected. */
int pt_set_guiding(pt_session* s, int enabled);
/* Re-initialise the guide network (seeded) and its optimiser state. */
int pt_guide_reset(pt_session* s);
/* Training schedule: Adam steps per frame (0, the default: automatic, 16 steps per frame for
 * the first 512 steps, 4 up to 1024, then 2), samples per step (default 2^16), learning rate
 * (default 3e-3), steps before the guide is used for sampling (default 4). Negative values
 * (zero for batch and lr) keep the current setting. */
int pt_set_guide_options(pt_session* s, int steps_per_frame, int batch, float lr, int warmup_steps);
/* MIS weights of emitter samples use the BSDF's own sampling density (the reference's
 * Microfacet::pdf evaluates alpha at the incident direction instead, microfacet.h:124-134,
 * which biases the combination slightly). On by itself when guiding is on. */
int pt_set_consistent_mis(pt_session* s, int enabled);
typedef struct pt_guide_info {
    int enabled;
    int mode;              /* 0 off, 1 collecting only, 2 guided sampling */
    int steps;             /* Adam steps taken */
    int params;            /* 16104 */
    unsigned long long samples;  /* training samples collected so far */
    float loss;            /* weighted mean of -log q(wi|x) over the last training batch */
} pt_guide_info;
int pt_guide_get_info(const pt_session* s, pt_guide_info* out);
/* Network parameters (FP32 master copy): W1[80][64], b1[64], W2[64][64], b2, W3[64][64], b3,
 * W4[64][40], b4[40], row-major, concatenated; n must be 16104. */
int pt_guide_get_params(pt_session* s, float* out, int n);
int pt_guide_set_params(pt_session* s, const float* in, int n);
/* Raw outputs (n x 40) of the inference kernel for n explicit input vectors (n x 80). */
int pt_guide_forward(pt_session* s, const float* x, int n, float* raw);
/* Guide inference on the 5th-generation tensor cores (tcgen05.mma, accumulators in tensor
 * memory; tc = 1) or on warp-level mma.sync (tc = 0, the default and the fallback). */
int pt_set_guide_inference(pt_session* s, int tc);
/* Guide training on the 5th-generation tensor cores (tc = 1, the default): forward,
 * backward-data and weight-gradient products as tcgen05.mma with the gradient accumulators in
 * tensor memory across all of a CTA's samples; or on warp-level mma.sync (tc = 0). Same loss,
 * weight cap and BF16 operands either way. */
int pt_set_guide_training(pt_session* s, int tc);
/* Probability (default 0.7) of drawing a non-delta vertex's direction from the guide instead
 * of the BSDF; the MIS density is (1 - f) p_bsdf + f p_guide, so the estimator is unbiased for
 * any f in (0, 1) (PT_ERR_ARG outside). */
int pt_set_guide_fraction(pt_session* s, float fraction);
/* Gradient (16104 floats) of -sum w_i log q(wi_i | x_i) / sum w_i computed by the training
 * kernel for n explicit samples (x: n x 80, wi: n x 3 unit vectors, w: n weights). */
int pt_guide_gradients(pt_session* s, const float* x, const float* wi, const float* w, int n, float* grad);
/* Restart progressive accumulation at the next frame (Renderer::reset). */
int pt_reset(pt_session* s);
int pt_set_launch(pt_session* s, const pt_launch_config* cfg);
int pt_get_launch(const pt_session* s, pt_launch_config* out);
/* Autotuner (no counterpart in the reference, whose only tuning is SppOptimizer's spp
 * budget, src/spp_optimizer.cpp:8-29): times frames of `spp` samples on the loaded scene over
 * BVH width, the tree's builder (host SAH or GPU PLOC; single scenes) and leaf size, material
 * sorting, the shade kernel, ray sorting, speculative traversal, the shadow stage's child
 * order, persistent-grid size, block size and wave size (coordinate descent), applies the
 * fastest and restarts accumulation. With cache_path, results are stored as one
 * JSON object per line keyed by scene size, material classes, resolution, spp, depth and
 * NEE, and a cached key is applied without measuring. */
int pt_autotune(pt_session* s, int spp, const char* cache_path, pt_tune_result* out);

/* ---- rendering (PathTracer::renderAsync/pollRender, path_tracer.cu:285-356) ----------- */
int pt_render_async(pt_session* s, int spp);
/* done = 1 when the frame in flight finished (its spp is then added to the running total);
 * ms = its device time. done = 1 with no frame in flight. */
int pt_poll(pt_session* s, int* done, float* ms);
/* Block until the frame in flight finishes (pt_poll until done). */
int pt_wait(pt_session* s, float* ms);
int pt_get_spp(const pt_session* s, int* spp);
int pt_get_stats(const pt_session* s, pt_stats* out);
/* stage_timing: record an event after every launch of the following frames; work_counters:
 * traversal kernels count nodes and leaf entries (slower; for roofline accounting). */
int pt_set_profiling(pt_session* s, int stage_timing, int work_counters);
int pt_get_profile(const pt_session* s, pt_profile* out);

/* ---- readback (Renderer::getRadianceBuffer, src/renderers/renderer.cpp:20-42) --------- */
/* Running-mean linear radiance, rows bottom-up like the reference (row 0 = image bottom),
 * 3 floats per pixel; n = number of floats of `rgb` (>= 3 * width * height). */
int pt_readback(pt_session* s, float* rgb, size_t n);
/* Same for the last frame's own mean (passRadiances). */
int pt_readback_pass(pt_session* s, float* rgb, size_t n);
/* sRGB-encoded, clamped RGBA8 display buffer (framebuffer.cu:35-40); n bytes >= 4*W*H. */
int pt_readback_rgba8(pt_session* s, uint8_t* rgba, size_t n);
/* Asynchronous pt_readback: the running mean as of the last enqueued frame is snapshotted
 * behind that frame, then copied into `rgb` on a separate copy stream, so the copy overlaps
 * the next frame. Returns at once; once the frame is done (pt_poll / pt_wait), the next
 * pt_render_async may start while the copy runs.
 * pt_readback_wait blocks until `rgb` holds the image (a no-op with none pending). `rgb`
 * should be page-locked for the copy to run asynchronously, and must stay valid until the
 * wait. A second pt_readback_async first waits for the pending copy. (The reference reads
 * its display buffer synchronously each frame, renderer.cpp:20-42.) */
int pt_readback_async(pt_session* s, float* rgb, size_t n);
int pt_readback_wait(pt_session* s);

/* ---- queries --------------------------------------------------------------------------- */
/* Material id under pixel (x = column, y = row) through its centre, -1 on a miss
 * (RenderSession::hitTest, src/hit_test.cu:25-82). */
int pt_hit_test(pt_session* s, int x, int y, int* material_id);
/* Closest hit of n caller rays against the loaded scene, host arrays (parity entry for
 * World::hit, src/world.cu:5-41). o, d: 3 floats per ray. Outputs per ray: prim_type (0
 * triangle, 1 sphere, -1 miss), prim_id, mat_id (-1 on a miss), t. bary (2 per ray) may be
 * NULL. */
int pt_trace_rays(pt_session* s, const float* o, const float* d, const float* tmin, const float* tmax,
                  int n, int* prim_type, int* prim_id, int* mat_id, float* t, float* bary);
/* Same with device pointers (no copies; arrays must be device memory of this device). */
int pt_trace_rays_device(pt_session* s, const float* o, const float* d, const float* tmin,
                         const float* tmax, int n, int* prim_type, int* prim_id, int* mat_id,
                         float* t, float* bary);
/* Allocation-free variant of pt_trace_rays. It has no counterpart in the reference.
 * For callers that cannot call cudaMalloc: cudaMalloc and cudaFree may synchronize the
 * device, so an interactive caller (picking under the cursor while a frame renders) would
 * stall on the frame in flight; and a host whose device memory is fully owned by its own
 * allocator (an engine, or a framework's caching allocator) has none to give. The call
 * stages rays and results through one file-scope __device__ array of
 * PT_STATIC_MAX_RAYS entries (about 3.7 MB, reserved on every GPU that loads the library
 * until the process exits) and allocates nothing; n above PT_STATIC_MAX_RAYS is rejected
 * with PT_ERR_ARG. The scene must already be on the device: after loading or editing it,
 * make one ordinary device call first (otherwise PT_ERR_STATE). The query runs on a stream
 * of the session's own, not the render stream, so a call made while a frame is in flight
 * returns without waiting for that frame. The first call on a device looks the array's
 * address up; make that first call before any stream capture. All calls share the array and
 * it keeps the last call's contents; calls whose work overlaps on the GPU (other sessions,
 * streams or host threads) race on it. */
#define PT_STATIC_MAX_RAYS 65536
int pt_trace_rays_static(pt_session* s, const float* o, const float* d, const float* tmin, const float* tmax,
                         int n, int* prim_type, int* prim_id, int* mat_id, float* t, float* bary);
/* Any-hit of n caller rays: occluded[i] = 1 when a primitive lies in [tmin, tmax]
 * (the shadow query of directSampleLights, path_tracer.cu:101-113). */
int pt_occluded(pt_session* s, const float* o, const float* d, const float* tmin, const float* tmax,
                int n, int* occluded);

/* ---- batched frames (configuration 4) -------------------------------------------------
 * No counterpart in the reference, which renders one scene per session. A session loaded
 * with pt_load_batch renders all its scenes in every frame: each stage of the wavefront
 * (camera, closest hit, shading, shadow rays, accumulation, guide inference) is one launch
 * over the rays of all scenes, whose queue entries carry their scene's id. Each scene keeps
 * its own resolution, spp per frame, depth, camera, emitters, environment and, when
 * `guided`, its own guide network. pt_render_async's spp argument is ignored (pass 0);
 * pt_get_spp reports frames rendered. Single-scene queries (pt_hit_test, pt_trace_rays*,
 * pt_set_camera, pt_set_material, pt_export_scene) are refused in batch mode. */
typedef struct pt_batch_scene {
    int config;            /* generated configuration 0-3 */
    int level;             /* icosphere level: configs 2-3 their mesh, configs 0-1 an added
                              mesh; -1 = configuration default (no added mesh) */
    unsigned long long seed;
    int width, height;
    int spp;               /* samples per pixel per frame */
    int max_depth;
    int guided;            /* 1: own guide network (needs pt_set_guiding(s, 1)) */
    int pad;
} pt_batch_scene;

typedef struct pt_batch_info {
    int num_triangles, num_spheres, num_lights;
    int width, height, spp, max_depth, guided;
    int spp_accumulated;   /* samples per pixel in the scene's running mean */
    long long first_pixel; /* offset of the scene's pixels in the batch's pixel order */
    long long first_path;  /* offset of the scene's paths in a frame's path order */
} pt_batch_info;

/* Configuration 4's seeded draw of n scenes from configurations 0-3: log-uniform triangle
 * counts 1k-2M (icosphere levels 3-8), square resolutions 256-1024, spp 4-64, depth 4-10,
 * about half guided. */
int pt_batch_generate(unsigned long long seed, int n, pt_batch_scene* out);
/* Generate every scene, build its BVH and merge them into the session (n <= 64). */
int pt_load_batch(pt_session* s, const pt_batch_scene* scenes, int n);
int pt_batch_get_info(const pt_session* s, int scene, pt_batch_info* out);
/* Running mean (pass_only = 0) or last frame's pass of one scene: width * height * 3 floats. */
int pt_batch_readback(pt_session* s, int scene, float* rgb, size_t n, int pass_only);

/* BVH construction on the GPU: primitive boxes, 63-bit Morton codes and a radix sort, then a
 * binary tree, either (gpu = 1) a Karras radix tree with bottom-up bounds, or (gpu = 2)
 * locally-ordered agglomerative clustering (PLOC: mutual nearest neighbours by union surface
 * area within 16 positions in Morton order, merged pass by pass), and a top-down collapse to
 * the same wide-node format, run when the scene is next uploaded (the first render or query
 * after a load or edit). gpu = 0 (default) selects the host's binned-SAH builder. Closest hits
 * are identical with any tree. No counterpart in the reference, whose CUDA backend scans
 * every primitive (src/world.cu:5-41). Batches always use the host builder. Other values:
 * PT_ERR_ARG. */
int pt_set_bvh_builder(pt_session* s, int gpu);

/* quantized = 1: traversal reads quantized copies of the wide nodes (widths 4 and 8: 64 and
 * 96 bytes against 128 and 256). Each node stores per axis an FP32 origin and a power-of-two
 * scale, and every child plane as an 8-bit multiple of the scale, rounded outward so that the
 * decoded box contains the float box; closest hits stay identical. quantized = 0 (default):
 * float nodes. Width 2 always uses float nodes. It trades the node memory (2.7x smaller for
 * width 8) for decode work: on a B200 it traced 16-28% slower on the generated
 * configurations, whose nodes mostly stay in L2. No counterpart in the reference. */
int pt_set_bvh_nodes(pt_session* s, int quantized);

/* Renderer of the session's frames: PT_RENDERER_CUDA, the path tracer (default), or
 * PT_RENDERER_NORMALS, the normals G-buffer (PT_ERR_ARG for PT_RENDERER_OPTIX).
 * Replaces RenderSession's renderer switch (src/render_session.cu:79-87) to a
 * GBuffer(BufferType::Normals) (src/renderers/g_buffer.cu:27-117): each frame traces one
 * pixel-centre camera ray per pixel (Camera::generateRay(row, col)) and writes the closest
 * hit's (normal + 1) / 2, black on a miss, as a 1-spp pass into the running mean, whatever
 * spp pt_render_async asks for. A change restarts accumulation. Single scenes only
 * (PT_ERR_STATE for a batch). */
int pt_set_renderer(pt_session* s, int kind);

/* on = 1: triangles take a watertight ray/triangle test (Woop, Benthin and Wald 2013) in every
 * query and frame, in place of Triangle::hit's arithmetic (src/primitives/triangle.cu:7-48),
 * which a ray through a shared edge or vertex can slip between. The leaf entries then hold the
 * triangles' own vertices (re-uploaded on the next device call) and accumulation restarts.
 * on = 0 (default): the reference's test, bit for bit. Spheres keep Sphere::hit's test. */
int pt_set_watertight(pt_session* s, int on);

/* Test hook for the device-error paths (no counterpart in the reference, whose gpuAssert exits
 * the process, include/macro_helper.h:10-19). stack_entries > 0 caps the traversal stack of
 * every query of the frames, pt_trace_rays and pt_occluded at that many entries (below the BVH
 * depth a query that needs more gives up); mma_polls > 0 limits the first wait of each
 * tensor-core inference layer (pt_set_guide_inference(1)) to that many non-blocking polls, so
 * it gives up while the layer's MMA runs (a bounded drain still waits for that MMA before the
 * kernel releases tensor memory). Either way the kernel sets its error flag and returns; the
 * call reports PT_ERR_DEVICE and the session stays usable. 0 and 0 (default) turn both off. */
int pt_set_test_limits(pt_session* s, int stack_entries, int mma_polls);

/* Measurement support (no counterpart in the reference): the read bandwidth, in GB/s, of a
 * buffer of `bytes` (a multiple of 16, at least 1 MiB) that stays in L2, on CUDA device
 * `device` (made the library's current device).
 * A full persistent grid reads it `reps` times per launch with 16-byte loads cached in L2
 * only; the best of `trials` launches timed with CUDA events is returned in *gbs, its
 * duration in *ms (either may be NULL). Allocates the buffer for the call and frees it. It is
 * the denominator of the closest-hit roofline on scenes whose nodes and leaf entries fit in
 * L2 (the 1.31M-triangle mesh: about 100 MB against a 126 MB L2). */
int pt_measure_l2_read(int device, size_t bytes, int reps, int trials, double* gbs, double* ms);

/* Library version string. */
const char* pt_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PATHED_H */
