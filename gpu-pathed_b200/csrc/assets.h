// Asset path: the reference's scene-file loaders, restated for the host runtime.
//
//   OBJ + MTL  src/parsers/obj_parser.cpp, src/parsers/mtl_parser.cpp
//   PLY        src/parsers/ply_parser.cpp (binary little-endian triangle meshes)
//   EXR        environment maps (src/lights/environment_light.cu:14-56 through the vendored
//              tinyexr LoadEXR): single-part scanline images, NONE / RLE / ZIPS / ZIP / PIZ
//              compression, HALF or FLOAT channels, returned as RGBA FP32 rows top first
//   scenes     SceneAdapter::createSceneData (src/scene_data.cu:9-118) and the reference's
//              built-in scenes 0-3 (src/scene.cu:14-172 with getCamera, :174-218)
//
// Parsed faces follow the reference exactly (accepted face forms, index rules, normals and
// material order), so a file gives the same triangle list, in the same order, as the
// reference's parsers. Where the reference would read out of bounds or abort (an index past
// the vertex list, a truncated file, an unsupported header) the loader returns an error.
#pragma once

#include <string>
#include <vector>

#include "host_scene.h"

namespace pt {

// Mtl (include/parsers/types.h:71-91): diffuse Kd and emitted Ke.
struct MeshMtl {
    float kd[3] = {0.f, 0.f, 0.f};
    float ke[3] = {0.f, 0.f, 0.f};
};

// Faces of one mesh file: per face p0,p1,p2 (9 floats) and n0,n1,n2 (9 floats). OBJ files
// also give their MTL materials (ordered by name, as the reference's std::map) and each
// face's index into them.
struct MeshFaces {
    std::vector<float> p, n;
    std::vector<int> mtl;
    std::vector<MeshMtl> mtls;
    int num_faces() const { return (int)(p.size() / 9); }
};

bool parse_obj(const std::string& path, MeshFaces& out, std::string& err);
bool parse_ply(const std::string& path, MeshFaces& out, std::string& err);

// LoadEXR: width x height RGBA FP32, row 0 = the data window's first scanline. R, G and B
// channels are required (A defaults to 1); a single-channel image is replicated into all four.
bool read_exr(const std::string& path, int& width, int& height, std::vector<float>& rgba, std::string& err);

// Image::save (src/io/image.cpp:9-78): an uncompressed scanline EXR of HALF channels B, G, R
// from `rgb` (3 floats per pixel, row 0 = the image bottom, written last). Halves round as
// the writer the reference vendors does: to nearest, ties away from zero, overflow to inf.
bool write_exr(const std::string& path, int width, int height, const float* rgb, std::string& err);

constexpr int kMeshObj = 0;
constexpr int kMeshPly = 1;

struct MeshFile {
    std::string path;
    int format = kMeshObj;
    int default_material = 0;  // faces without MTL materials take this id
};

// SceneAdapter::ParseRequest (include/scene_data.h): mesh files, materials, spheres and an
// optional EXR environment map.
struct SceneRequest {
    std::vector<MeshFile> files;
    std::vector<Material> mats;
    std::vector<float> sph;  // cx, cy, cz, r per sphere
    std::vector<int> sph_mat;
    std::string env_path;    // empty: no environment light
};

// createSceneData: OBJ files' triangles first (file order), then PLY files', each OBJ's MTL
// materials appended as Lambertians (Kd, Ke) after the request's materials. Emitter lists are
// derived later from the materials.
bool build_request(const SceneRequest& req, HostScene& out, std::string& err);

// The reference's built-in scene `index` (0 Cornell box, 1 glossy Cornell box with a mirror
// box and a glass ball, 2 plane under the 1-pixel test environment, 3 the Veach MIS plates
// under an HDR environment) with its camera, read from the reference's scenes directory.
bool reference_scene(int index, const std::string& scenes_dir, HostScene& out, std::string& err);

}  // namespace pt
