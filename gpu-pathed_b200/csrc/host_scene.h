// Host-side scene model: the arrays the reference's SceneData carries
// (include/scene_data.h:19-41), flattened to plain vectors, plus the camera and the
// render defaults of a configuration.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "pt_types.h"

namespace pt {

struct CameraSpec {
    float origin[3];
    float target[3];
    float up[3];
    float vfov;  // radians
    bool flip;   // lookAt handedness flip (src/transform.cu:27)
};

struct HostScene {
    // Triangles in reference order: p0,p1,p2 (9 floats), n0,n1,n2 (9 floats), material.
    std::vector<float> tri_p;
    std::vector<float> tri_n;
    std::vector<int> tri_mat;
    // Spheres: center xyz + radius, material.
    std::vector<float> sph;
    std::vector<int> sph_mat;
    std::vector<Material> mats;
    // Equirect environment map, RGBA FP32, row 0 = +y (theta = 0). Empty when absent.
    int env_w = 0, env_h = 0;
    std::vector<float> env_rgba;

    CameraSpec camera{};
    int default_spp = 1;
    int default_depth = 3;  // include/scene.h:12 (defaultMaxDepth)
    bool default_nee = true;
    int res_x = 0, res_y = 0;  // preferred resolution of a generated configuration
    std::string name;

    int num_tri() const { return (int)tri_mat.size(); }
    int num_sph() const { return (int)sph_mat.size(); }
};

// Emitter list in the reference's order: emitting triangles first, then emitting spheres
// (src/scene_data.cu:92-115). A primitive emits when its material is a Lambertian with a
// non-zero emit (scene_data.h:38-40 + world.h:161-174).
std::vector<LightRef> build_light_list(const HostScene& s);

// Recompute Material::emitting from type and emit.
void finalize_materials(HostScene& s);

// Seeded procedural configurations.
//   0: Cornell box, 36 triangles (2 emitters), 512x512, 16 spp, depth 5, NEE.
//   1: 64 spheres on a 2-triangle plane + 4 sphere emitters, 1024x1024, 64 spp, depth 8.
//   2: displaced level-8 icosphere (1,310,720 triangles), Beckmann alpha 0.3, 2048x1024
//      lognormal + 3-sun environment, 1920x1080, 32 spp, depth 6.
//   3: closed room (~2k triangles) with a 0.05-wide ceiling slit around the config-2 mesh,
//      lit by the config-2 environment through the slit, 1024x1024, depth 10.
// Returns false (and leaves `err`) for an unknown id. `icosphere_level` >= 0 sets the mesh
// level of configs 2 and 3 and adds a displaced icosphere of that level to configs 0 and 1
// (batched workloads); -1 keeps each configuration as described.
bool generate_config(int config, uint64_t seed, HostScene& out, std::string& err,
                     int icosphere_level = -1);

// One scene of a batched frame (configuration 4).
struct BatchSpec {
    int config = 0;          // generated configuration 0-3
    uint64_t seed = 0;
    int level = -1;          // icosphere level (configs 0-1: an added mesh; -1: none/default)
    int width = 256, height = 256, spp = 4, max_depth = 4;
    int guided = 0;          // own guide network
};

// Configuration 4's draw of n scenes from configurations 0-3 (seeded).
std::vector<BatchSpec> generate_batch_specs(uint64_t seed, int n);

// Environment map of configuration 2 (lognormal background + 3 Gaussian suns).
void generate_sun_env(uint64_t seed, int w, int h, std::vector<float>& rgba);

// Basic validation of a scene handed over by a caller: finite vertices, material ids in
// range, known material types. Returns false with a message on the first problem.
bool validate_scene(const HostScene& s, std::string& err);

}  // namespace pt
