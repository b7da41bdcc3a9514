// Plain-old-data layouts shared by the host runtime and the sm_100a kernels.
//
// Scene layout in HBM (device side, all 16-byte aligned, coalesced float4 loads):
//   * BVH nodes           : BvhNode<W> (W = 2, 4 or 8 children, SoA bounds inside a node)
//   * BVH primitive refs  : 3 x float4 per leaf entry, in leaf order
//       triangle: (p0.xyz, id)  (e1.xyz, 0)  (e2.xyz, 0)      id >= 0 is the triangle index
//       sphere  : (c.xyz, ~id)  (r, 0, 0, 0) (0, 0, 0, 0)     ~id < 0 encodes the sphere index
//   * triangle shading data in original (reference) order: p0,p1,p2 and n0,n1,n2 as float4
//   * materials, emitter list, equirect environment (RGBA FP32) + its marginal/conditional CDF
//
// The triangle/sphere records keep the reference's per-primitive semantics
// (include/primitives/triangle.h:93-96, include/primitives/sphere.h:106-108); e1/e2 are
// precomputed with the same single-precision subtractions Triangle::hit performs
// (src/primitives/triangle.cu:13-14), so the hit arithmetic is unchanged bit for bit.
#pragma once

#include <stdint.h>
#include <vector_types.h>

#if defined(__CUDACC__)
#define PT_HD __host__ __device__ __forceinline__
#else
#define PT_HD inline
#endif

namespace pt {

// Material types: same enumerators and values as the reference (include/materials/types.h:5-11),
// plus kMetal, which the reference lacks: its Beckmann microfacet with a Schlick Fresnel term of
// RGB reflectance F0 (the material's albedo) at normal incidence, for metals; the reference's
// Microfacet uses a dielectric Fresnel of fixed eta 1.5 (F0 = 0.04, microfacet.h:111).
enum MaterialType : int {
    kLambertian = 0,
    kMirror = 1,
    kGlass = 2,
    kMicrofacet = 3,
    kMaterialNone = 4,
    kMetal = 5,
};
// Material classes of sorted shading: miss, then one per type (type + 1)
constexpr int kMaterialClasses = kMetal + 2;

// Primitive types (include/primitives/types.h:5-8).
enum PrimType : int { kTriangle = 0, kSphere = 1 };

struct alignas(16) Material {
    float albedo[3];
    int type;
    float emit[3];
    float ior;
    float alpha;
    int emitting;  // 1 if emit != 0 and the type can emit (Lambertian only, world.h:161-174)
    float pad[2];
};
static_assert(sizeof(Material) == 48, "Material layout");

// Camera in the form generateRay needs (include/core/camera.h:40-61): the 3x4 cameraToWorld
// matrix of lookAt (src/transform.cu:7-33) plus the image-plane extents.
struct alignas(16) CameraParams {
    float m[3][4];
    float top;     // tan(vfov / 2)
    float height;  // 2 * top
    float width;   // height * aspect
    float right;   // width / 2
    int res_x, res_y;
    float vfov;
    int flip;
    float origin[3], target[3], up[3];
    float pad;
};

// Child encoding of a wide node: >= 0 internal node index; kEmptyChild = no child;
// otherwise a leaf: ~((first << 4) | (count - 1)), count in [1, 16].
constexpr int kEmptyChild = (int)0x80000000;
constexpr int kMaxLeafPrims = 16;

PT_HD int leaf_code(int first, int count) { return ~((first << 4) | (count - 1)); }
PT_HD bool child_is_leaf(int c) { return c < 0 && c != kEmptyChild; }
PT_HD int leaf_first(int c) { return (~c) >> 4; }
PT_HD int leaf_count(int c) { return ((~c) & 15) + 1; }

template <int W>
struct alignas(16) BvhNode {
    float lo_x[W], hi_x[W], lo_y[W], hi_y[W], lo_z[W], hi_z[W];
    int child[W];
    int pad[(W == 2) ? 2 : W];  // node size 64 / 128 / 256 B
};
static_assert(sizeof(BvhNode<2>) == 64, "BVH2 node");
static_assert(sizeof(BvhNode<4>) == 128, "BVH4 node");
static_assert(sizeof(BvhNode<8>) == 256, "BVH8 node");

// Quantized wide node (W = 4 or 8; 64 / 96 B against 128 / 256 B): per axis an origin (the
// smallest child lower bound, FP32) and a power-of-two scale (its biased FP32 exponent), the
// child planes as 8-bit multiples of the scale, the child codes unchanged. A plane decodes as
// fmaf(q, scale, origin), correctly rounded on host and device alike; the builder chooses q so
// that every decoded box contains the float child box it replaces (lower planes rounded down,
// upper planes up), so traversal still never culls a hit.
//   bytes 0-11 origin xyz, 12-14 exponents xyz, 16.. q[6][W] (lo_x, hi_x, lo_y, hi_y, lo_z,
//   hi_z), then child[W] at 16 + 6W
PT_HD constexpr int qnode_bytes(int w) { return w == 8 ? 96 : 64; }
PT_HD constexpr int qnode_child_offset(int w) { return 16 + 6 * w; }

// Environment light (include/lights/environment_light.h:26-99): RGBA texels, y-up lat-long,
// row 0 = theta 0 (+y). CDFs: marginal over rows (H floats) and one conditional per row
// (H x W floats), both clamped to 1.0 from the last non-zero entry (src/math/distribution.cu:37-42).
struct EnvDevice {
    const float* rgba;      // H * W * 4
    const float* marg_cdf;  // H
    const float* cond_cdf;  // H * W
    const float* row_mass;  // H   (row totals; 0 marks an empty row)
    int width, height;
    float total_mass;
    int present;  // EnvironmentLightType::Image
    int continuous;  // 0: pixel-centre directions (reference), 1: uniform within the texel
    int pad[3];
};

// Emitter list entry (include/lights/types.h:14-17): primitive type + index in original order.
struct LightRef {
    int type;
    int index;
};

// Everything a kernel needs to see of a loaded scene (passed by value as a kernel argument).
struct SceneDevice {
    const float4* nodes;       // BvhNode<W> array viewed as float4
    const float4* prims;       // 3 float4 per leaf entry
    const float4* tri_p;       // 3 float4 per triangle: p0, p1, p2 (original order)
    const float4* tri_n;       // 3 float4 per triangle: n0, n1, n2
    const int* tri_mat;        // per triangle material id
    const float4* sph;         // per sphere: center.xyz, radius
    const int* sph_mat;        // per sphere material id
    const Material* mats;
    const LightRef* lights;
    EnvDevice env;
    int num_tri, num_sph, num_mat, num_lights;
    int bvh_width;             // 2, 4 or 8
    int root;                  // root node index (always an internal node)
    int node_q;                // 1: `nodes` holds quantized nodes (widths 4 and 8)
    int watertight;            // 1: triangle leaf entries hold p0, p1, p2 and take the watertight test
};

// Ray-query kinds and their [tMin, tMax] conventions (src/renderers/path_tracer.cu):
//   camera rays tMin 0 (:154), continuation 1e-3 (:177), BSDF-direct 1e-4 (:51),
//   shadow [1e-4, distance - 2e-4] (:104-108).
constexpr float kCameraTMin = 0.0f;
constexpr float kBounceTMin = 1e-3f;
constexpr float kDirectTMin = 1e-4f;  // directSampleBSDF's trace of the sampled direction (:51)
constexpr float kShadowTMin = 1e-4f;

}  // namespace pt
