// ORACLE - test infrastructure, not product code.
//
// C entry points over the reference's own scene-file readers, compiled for the host from the
// reference sources in place (oracle/Makefile, target refassets): ObjParser + MtlParser
// (src/parsers/obj_parser.cpp, mtl_parser.cpp), PLYParser (src/parsers/ply_parser.cpp),
// Image::save (src/io/image.cpp, which instantiates the vendored tinyexr) and tinyexr's
// LoadEXR. Tests compare the product's loaders and writer with these, file by file.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "io/image.h"
#include "parsers/obj_parser.h"
#include "parsers/ply_parser.h"
#include "tinyexr.h"

using namespace rays;

namespace {
struct RefMesh {
    std::vector<float> p, n, mtls;
    std::vector<int> mtl;
};

void put(std::vector<float>& v, const Vertex& a) {
    v.push_back(a.x);
    v.push_back(a.y);
    v.push_back(a.z);
}

void add_faces(RefMesh* m, const std::vector<Face>& faces) {
    for (const Face& f : faces) {
        put(m->p, f.v0);
        put(m->p, f.v1);
        put(m->p, f.v2);
        put(m->n, f.n0);
        put(m->n, f.n1);
        put(m->n, f.n2);
    }
}
}  // namespace

extern "C" {

// ply = 0: ObjParser(path).parse(); ply = 1: PLYParser(path).parse()
void* ref_mesh_parse(const char* path, int ply) {
    RefMesh* m = new RefMesh();
    std::string name(path);
    if (ply) {
        PLYParser parser(name);
        const PLYResult r = parser.parse();
        add_faces(m, r.faces);
        m->mtl.assign(r.faces.size(), 0);
    } else {
        ObjParser parser(name);
        const ObjResult r = parser.parse();
        add_faces(m, r.faces);
        m->mtl = r.mtlIndices;
        for (const Mtl& t : r.mtls) {
            const float v[6] = {t.r, t.g, t.b, t.emitR, t.emitG, t.emitB};
            m->mtls.insert(m->mtls.end(), v, v + 6);
        }
    }
    return m;
}

int ref_mesh_faces(void* h) { return (int)static_cast<RefMesh*>(h)->mtl.size(); }
int ref_mesh_mtls(void* h) { return (int)static_cast<RefMesh*>(h)->mtls.size() / 6; }

// p, n: 9 floats per face; mtl: one index per face; mtls: Kd rgb + Ke rgb per material
void ref_mesh_copy(void* h, float* p, float* n, int* mtl, float* mtls) {
    const RefMesh* m = static_cast<RefMesh*>(h);
    std::memcpy(p, m->p.data(), m->p.size() * sizeof(float));
    std::memcpy(n, m->n.data(), m->n.size() * sizeof(float));
    std::memcpy(mtl, m->mtl.data(), m->mtl.size() * sizeof(int));
    if (!m->mtls.empty()) std::memcpy(mtls, m->mtls.data(), m->mtls.size() * sizeof(float));
}

void ref_mesh_free(void* h) { delete static_cast<RefMesh*>(h); }

// LoadEXR: returns the RGBA buffer (free with ref_exr_free) or NULL with *code set
float* ref_exr_load(const char* path, int* width, int* height, int* code) {
    float* data = nullptr;
    const char* err = nullptr;
    *code = LoadEXR(&data, width, height, path, &err);
    if (*code != TINYEXR_SUCCESS) {
        if (err) FreeEXRErrorMessage(err);
        return nullptr;
    }
    return data;
}

void ref_exr_free(float* p) { std::free(p); }

// Image::save(width, height, radiances, filename): rgb row 0 = image bottom
void ref_image_save(int width, int height, const float* rgb, const char* path) {
    const std::vector<float> r(rgb, rgb + (size_t)width * height * 3);
    Image::save(width, height, r, path);
}

}  // extern "C"
