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

// tinyexr's SaveEXRImageToFile with PIZ compression: nch channel planes of width x height
// FLOAT values (names from `names`, one char each), stored as pixel_type (1 HALF, 2 FLOAT).
// Used to write multi-level PIZ files for the product's reader; returns tinyexr's code.
int ref_exr_save_piz(int width, int height, int nch, const char* names, int pixel_type, const float* planes,
                     const char* path) {
    EXRHeader header;
    InitEXRHeader(&header);
    EXRImage image;
    InitEXRImage(&image);
    std::vector<const float*> ptrs((size_t)nch);
    for (int c = 0; c < nch; c++) ptrs[c] = planes + (size_t)c * width * height;
    image.num_channels = nch;
    image.images = reinterpret_cast<unsigned char**>(const_cast<float**>(ptrs.data()));
    image.width = width;
    image.height = height;
    std::vector<EXRChannelInfo> ch((size_t)nch);
    std::vector<int> in_types((size_t)nch, TINYEXR_PIXELTYPE_FLOAT), out_types((size_t)nch, pixel_type);
    for (int c = 0; c < nch; c++) {
        std::memset(&ch[c], 0, sizeof(EXRChannelInfo));
        ch[c].name[0] = names[c];
    }
    header.num_channels = nch;
    header.channels = ch.data();
    header.pixel_types = in_types.data();
    header.requested_pixel_types = out_types.data();
    header.compression_type = TINYEXR_COMPRESSIONTYPE_PIZ;
    const char* err = nullptr;
    const int code = SaveEXRImageToFile(&image, &header, path, &err);
    if (err) FreeEXRErrorMessage(err);
    return code;
}

// Image::save(width, height, radiances, filename): rgb row 0 = image bottom
void ref_image_save(int width, int height, const float* rgb, const char* path) {
    const std::vector<float> r(rgb, rgb + (size_t)width * height * 3);
    Image::save(width, height, r, path);
}

}  // extern "C"
