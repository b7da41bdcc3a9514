// Scene-file loaders (OBJ/MTL, PLY, EXR) and the reference's built-in scenes. Compiled with
// -ffp-contract=off: the geometric normals of OBJ quads and PLY faces round exactly as the
// reference's float expressions (include/parsers/types.h:35-55).
#include "assets.h"

#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

namespace pt {

namespace {

bool read_file(const std::string& path, std::string& data) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    data = ss.str();
    return true;
}

// std::getline over the whole file: lines split at '\n' (a '\r' stays in the line).
template <class F>
void for_each_line(const std::string& data, F&& fn) {
    size_t pos = 0;
    while (pos < data.size()) {
        size_t e = data.find('\n', pos);
        if (e == std::string::npos) e = data.size();
        if (!fn(data.substr(pos, e - pos))) return;
        pos = e + 1;
    }
}

// StringUtil::lTrim (src/parsers/string_util.cpp:24-34): drop leading spaces and tabs.
std::string ltrim(const std::string& s) {
    const size_t i = s.find_first_not_of(" \t");
    return i == std::string::npos ? std::string() : s.substr(i);
}

// StringUtil::tokenize (string_util.cpp:5-22): split at spaces and tabs.
std::vector<std::string> tokenize(const std::string& line) {
    std::vector<std::string> out;
    std::string rest = ltrim(line);
    while (!rest.empty()) {
        const size_t e = rest.find_first_of(" \t");
        if (e == std::string::npos) {
            out.push_back(rest);
            break;
        }
        out.push_back(rest.substr(0, e));
        rest = ltrim(rest.substr(e));
    }
    return out;
}

// std::stof: leading whitespace skipped, the longest float prefix converted; `used` is the
// number of characters consumed. False where std::stof would throw.
bool stof_prefix(const std::string& s, float& v, size_t& used) {
    const char* b = s.c_str();
    char* e = nullptr;
    errno = 0;
    v = std::strtof(b, &e);
    if (e == b || errno == ERANGE) return false;
    used = (size_t)(e - b);
    return true;
}

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

// (-?\d+) at s[i], converted as std::stoi does
bool int_token(const std::string& s, size_t& i, int& v) {
    const size_t b = i;
    if (i < s.size() && s[i] == '-') i++;
    const size_t d = i;
    while (i < s.size() && s[i] >= '0' && s[i] <= '9') i++;
    if (i == d) return false;
    long long x = 0;
    for (size_t k = d; k < i; k++) {
        x = x * 10 + (s[k] - '0');
        if (x > 2147483648LL) return false;
    }
    if (s[b] == '-') x = -x;
    if (x > 2147483647LL || x < -2147483648LL) return false;
    v = (int)x;
    return true;
}

bool literal(const std::string& s, size_t& i, const char* lit) {
    const size_t n = std::strlen(lit);
    if (s.compare(i, n, lit) != 0) return false;
    i += n;
    return true;
}

bool trailing_space_only(const std::string& s, size_t i) {
    while (i < s.size() && is_space(s[i])) i++;
    return i == s.size();
}

// "a b c d" (ObjParser::processDoubleFaceGeometryOnly's pattern, obj_parser.cpp:95-114)
bool match_quad(const std::string& s, int idx[4]) {
    size_t i = 0;
    for (int k = 0; k < 4; k++) {
        if (k > 0) {
            const size_t w = i;
            while (i < s.size() && is_space(s[i])) i++;
            if (i == w) return false;
        }
        if (!int_token(s, i, idx[k])) return false;
    }
    return trailing_space_only(s, i);
}

// "v/t/n v/t/n v/t/n" (processSingleFaceTriplets, :116-144) with sep "/" and three fields,
// or "v//n v//n v//n" (processSingleFaceVertexAndNormal, :146-170) with sep "//" and two
bool match_groups(const std::string& s, const char* sep, int fields, int idx[9]) {
    size_t i = 0;
    for (int g = 0; g < 3; g++) {
        if (g > 0 && !literal(s, i, " ")) return false;
        for (int f = 0; f < fields; f++) {
            if (f > 0 && !literal(s, i, sep)) return false;
            if (!int_token(s, i, idx[g * fields + f])) return false;
        }
    }
    return trailing_space_only(s, i);
}

struct Vtx {
    float x, y, z;
};

// Vertex::cross(...).normalized() (include/parsers/types.h:35-55), float arithmetic
Vtx face_normal(const Vtx& v0, const Vtx& v1, const Vtx& v2) {
    const float e1x = v1.x - v0.x, e1y = v1.y - v0.y, e1z = v1.z - v0.z;
    const float e2x = v2.x - v0.x, e2y = v2.y - v0.y, e2z = v2.z - v0.z;
    const float cx = e1y * e2z - e1z * e2y;
    const float cy = -(e1x * e2z - e1z * e2x);
    const float cz = e1x * e2y - e1y * e2x;
    const float len = std::sqrt(cx * cx + cy * cy + cz * cz);
    return Vtx{cx / len, cy / len, cz / len};
}

void push_face(MeshFaces& out, const Vtx& a, const Vtx& b, const Vtx& c, const Vtx& na, const Vtx& nb,
               const Vtx& nc, int mtl) {
    for (const Vtx* v : {&a, &b, &c}) out.p.insert(out.p.end(), {v->x, v->y, v->z});
    for (const Vtx* v : {&na, &nb, &nc}) out.n.insert(out.n.end(), {v->x, v->y, v->z});
    out.mtl.push_back(mtl);
}

// ObjParser::correctIndex (obj_parser.cpp:236-244): negative indices count back from the
// current end, positive ones are 1-based. False when the result is outside the list.
bool correct_index(int& idx, size_t count) {
    long long v = idx;
    v = v < 0 ? v + (long long)count : v - 1;
    if (v < 0 || v >= (long long)count) return false;
    idx = (int)v;
    return true;
}

// MtlParser (src/parsers/mtl_parser.cpp): materials keyed by name; a missing file gives none.
bool parse_mtl(const std::string& path, std::vector<MeshMtl>& mtls, std::map<std::string, int>& lookup,
               std::string& err) {
    mtls.clear();
    lookup.clear();
    std::string data;
    if (!read_file(path, data)) return true;  // an unreadable library leaves the materials empty
    std::map<std::string, MeshMtl> byname;
    std::string current;
    int lineno = 0;
    bool ok = true;
    for_each_line(data, [&](const std::string& line) {
        lineno++;
        const std::vector<std::string> tok = tokenize(line);
        if (tok.empty() || tok[0][0] == '#') return true;
        const std::string& cmd = tok[0];
        if (cmd == "newmtl") {
            if (tok.size() < 2) {
                err = path + ":" + std::to_string(lineno) + ": newmtl without a name";
                return ok = false;
            }
            current = tok[1];
            byname[current] = MeshMtl();
        } else if (cmd == "Kd" || cmd == "Ke") {
            float v[3];
            size_t used;
            if (tok.size() < 4 || !stof_prefix(tok[1], v[0], used) || !stof_prefix(tok[2], v[1], used) ||
                !stof_prefix(tok[3], v[2], used)) {
                err = path + ":" + std::to_string(lineno) + ": " + cmd + " needs three numbers";
                return ok = false;
            }
            MeshMtl& m = byname[current];
            float* dst = cmd == "Kd" ? m.kd : m.ke;
            for (int k = 0; k < 3; k++) dst[k] = v[k];
        }
        return true;  // Ka, Ks, Ni, Ns, illum and unknown commands are skipped
    });
    if (!ok) return false;
    int index = 0;
    for (const auto& kv : byname) {
        mtls.push_back(kv.second);
        lookup[kv.first] = index++;
    }
    return true;
}

// boost::filesystem::path(obj).parent_path() / name
std::string sibling_path(const std::string& file, const std::string& name) {
    const size_t slash = file.find_last_of('/');
    if (slash == std::string::npos) return name;
    return file.substr(0, slash) + "/" + name;
}

uint16_t rd16(const uint8_t* p) { return (uint16_t)(p[0] | (p[1] << 8)); }
uint32_t rd32(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }
uint64_t rd64(const uint8_t* p) { return (uint64_t)rd32(p) | ((uint64_t)rd32(p + 4) << 32); }

}  // namespace

bool parse_obj(const std::string& path, MeshFaces& out, std::string& err) {
    out = MeshFaces();
    std::string data;
    if (!read_file(path, data)) {
        err = "cannot read " + path;
        return false;
    }
    std::vector<Vtx> verts, normals;
    std::map<std::string, int> lookup;
    int current = 0;
    int lineno = 0;
    bool ok = true;
    auto fail = [&](const std::string& what) {
        err = path + ":" + std::to_string(lineno) + ": " + what;
        ok = false;
        return false;
    };
    auto three_floats = [&](std::string rest, Vtx& v) {
        float f[3];
        for (int k = 0; k < 3; k++) {
            size_t used = 0;
            if (!stof_prefix(rest, f[k], used)) return false;
            rest = rest.substr(used);
        }
        v = Vtx{f[0], f[1], f[2]};
        return true;
    };
    for_each_line(data, [&](const std::string& line) {
        lineno++;
        // ObjParser::parseLine (obj_parser.cpp:38-62)
        if (line.empty()) return true;
        const size_t sp = line.find_first_of(" \t");
        if (sp == std::string::npos) return true;
        const std::string cmd = line.substr(0, sp);
        if (!cmd.empty() && cmd[0] == '#') return true;
        const std::string rest = ltrim(line.substr(sp + 1));
        if (cmd == "v" || cmd == "vn") {
            Vtx v;
            if (!three_floats(rest, v)) return fail("expected three coordinates");
            (cmd == "v" ? verts : normals).push_back(v);
        } else if (cmd == "f") {
            int q[4], g[9];
            if (match_quad(rest, q)) {
                // two triangles (a, b, c) and (a, c, d) with the geometric normal
                const int tris[2][3] = {{q[0], q[1], q[2]}, {q[0], q[2], q[3]}};
                for (const auto& t : tris) {
                    int a = t[0], b = t[1], c = t[2];
                    if (!correct_index(a, verts.size()) || !correct_index(b, verts.size()) ||
                        !correct_index(c, verts.size()))
                        return fail("vertex index out of range");
                    const Vtx n = face_normal(verts[a], verts[b], verts[c]);
                    push_face(out, verts[a], verts[b], verts[c], n, n, n, current);
                }
            } else if (match_groups(rest, "/", 3, g) || match_groups(rest, "//", 2, g)) {
                const int fields = match_groups(rest, "/", 3, g) ? 3 : 2;
                int v[3], n[3];
                for (int k = 0; k < 3; k++) {
                    v[k] = g[k * fields];
                    n[k] = g[k * fields + fields - 1];  // texture coordinates are ignored
                    if (!correct_index(v[k], verts.size())) return fail("vertex index out of range");
                    if (!correct_index(n[k], normals.size())) return fail("normal index out of range");
                }
                push_face(out, verts[v[0]], verts[v[1]], verts[v[2]], normals[n[0]], normals[n[1]], normals[n[2]],
                          current);
            }
            // any other face form (a plain "a b c" triangle included) is skipped, as the
            // reference's three patterns do not match it
        } else if (cmd == "mtllib") {
            if (!parse_mtl(sibling_path(path, rest), out.mtls, lookup, err)) {
                ok = false;
                return false;
            }
        } else if (cmd == "usemtl") {
            const auto it = lookup.find(rest);
            current = it == lookup.end() ? 0 : it->second;  // std::map::operator[] default
        }
        return true;
    });
    return ok;
}

bool parse_ply(const std::string& path, MeshFaces& out, std::string& err) {
    out = MeshFaces();
    std::string data;
    if (!read_file(path, data)) {
        err = "cannot read " + path;
        return false;
    }
    // header lines up to end_header
    struct Prop {
        std::string name;
        int size = 0;       // scalar size, or the list's index size
        int count_size = 0; // > 0 for a list property
        bool is_float = false, is_double = false, is_signed = false;
    };
    struct Element {
        std::string name;
        long long count = 0;
        std::vector<Prop> props;
    };
    auto type_size = [](const std::string& t, bool& fl, bool& db, bool& sg) {
        fl = db = sg = false;
        if (t == "char" || t == "int8") { sg = true; return 1; }
        if (t == "uchar" || t == "uint8") return 1;
        if (t == "short" || t == "int16") { sg = true; return 2; }
        if (t == "ushort" || t == "uint16") return 2;
        if (t == "int" || t == "int32") { sg = true; return 4; }
        if (t == "uint" || t == "uint32") return 4;
        if (t == "float" || t == "float32") { fl = true; return 4; }
        if (t == "double" || t == "float64") { db = true; return 8; }
        return 0;
    };
    std::vector<Element> elems;
    size_t pos = 0;
    int lineno = 0;
    bool header_done = false;
    while (pos < data.size()) {
        size_t e = data.find('\n', pos);
        if (e == std::string::npos) break;
        std::string line = data.substr(pos, e - pos);
        pos = e + 1;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        lineno++;
        const std::vector<std::string> tok = tokenize(line);
        if (lineno == 1) {
            if (line != "ply") { err = path + ": not a PLY file"; return false; }
            continue;
        }
        if (tok.empty() || tok[0] == "comment" || tok[0] == "obj_info") continue;
        if (tok[0] == "format") {
            if (tok.size() < 2 || tok[1] != "binary_little_endian") {
                err = path + ": only binary_little_endian PLY files are supported";
                return false;
            }
        } else if (tok[0] == "element" && tok.size() >= 3) {
            Element el;
            el.name = tok[1];
            el.count = std::atoll(tok[2].c_str());
            if (el.count < 0) { err = path + ": negative element count"; return false; }
            elems.push_back(el);
        } else if (tok[0] == "property" && !elems.empty()) {
            Prop p;
            bool fl, db, sg;
            if (tok.size() >= 5 && tok[1] == "list") {
                p.count_size = type_size(tok[2], fl, db, sg);
                p.size = type_size(tok[3], fl, db, sg);
                p.is_signed = sg;
                p.name = tok[4];
                if (!p.count_size || !p.size || fl || db || p.count_size > 4) {
                    err = path + ": unsupported list property " + line;
                    return false;
                }
            } else if (tok.size() >= 3) {
                p.size = type_size(tok[1], fl, db, sg);
                p.is_float = fl;
                p.is_double = db;
                p.is_signed = sg;
                p.name = tok[2];
                if (!p.size) { err = path + ": unknown property type " + tok[1]; return false; }
            } else {
                err = path + ": malformed property line";
                return false;
            }
            elems.back().props.push_back(p);
        } else if (tok[0] == "end_header") {
            header_done = true;
            break;
        } else {
            err = path + ": unexpected header line " + line;
            return false;
        }
    }
    if (!header_done) { err = path + ": no end_header"; return false; }
    const uint8_t* d = (const uint8_t*)data.data();
    const size_t n = data.size();
    auto read_uint = [&](size_t at, int size) -> uint64_t {
        uint64_t v = 0;
        for (int k = 0; k < size; k++) v |= (uint64_t)d[at + k] << (8 * k);
        return v;
    };
    auto read_sint = [&](size_t at, int size) -> long long {
        const uint64_t u = read_uint(at, size);
        const int sh = 64 - 8 * size;
        return (long long)(u << sh) >> sh;
    };
    std::vector<Vtx> verts;
    bool have_vertices = false, have_faces = false;
    for (const Element& el : elems) {
        if (el.name == "vertex") {
            int ix = -1, iy = -1, iz = -1;
            for (int k = 0; k < (int)el.props.size(); k++) {
                const Prop& p = el.props[k];
                if (p.count_size) { err = path + ": list properties on vertices are not supported"; return false; }
                if (p.name == "x") ix = k;
                if (p.name == "y") iy = k;
                if (p.name == "z") iz = k;
            }
            if (ix < 0 || iy < 0 || iz < 0) { err = path + ": vertices need x, y and z"; return false; }
            for (int k : {ix, iy, iz})
                if (!el.props[k].is_float && !el.props[k].is_double) {
                    err = path + ": vertex coordinates must be float or double";
                    return false;
                }
            verts.reserve((size_t)el.count);
            for (long long i = 0; i < el.count; i++) {
                float c[3] = {0.f, 0.f, 0.f};
                for (int k = 0; k < (int)el.props.size(); k++) {
                    const Prop& p = el.props[k];
                    if (pos + p.size > n) { err = path + ": truncated vertex data"; return false; }
                    const int axis = k == ix ? 0 : k == iy ? 1 : k == iz ? 2 : -1;
                    if (axis >= 0) {
                        if (p.is_float) {
                            float f;
                            std::memcpy(&f, d + pos, 4);
                            c[axis] = f;
                        } else {
                            double f;
                            std::memcpy(&f, d + pos, 8);
                            c[axis] = (float)f;
                        }
                    }
                    pos += p.size;
                }
                verts.push_back(Vtx{c[0], c[1], c[2]});
            }
            have_vertices = true;
        } else if (el.name == "face") {
            if (!have_vertices) { err = path + ": faces before vertices"; return false; }
            int il = -1;
            for (int k = 0; k < (int)el.props.size(); k++)
                if (el.props[k].count_size && (el.props[k].name == "vertex_indices" || el.props[k].name == "vertex_index"))
                    il = k;
            if (il < 0) { err = path + ": faces need a vertex_indices list"; return false; }
            for (long long i = 0; i < el.count; i++) {
                for (int k = 0; k < (int)el.props.size(); k++) {
                    const Prop& p = el.props[k];
                    if (!p.count_size) {
                        if (pos + p.size > n) { err = path + ": truncated face data"; return false; }
                        pos += p.size;
                        continue;
                    }
                    if (pos + p.count_size > n) { err = path + ": truncated face data"; return false; }
                    const long long cnt = (long long)read_uint(pos, p.count_size);
                    pos += p.count_size;
                    if (pos + (size_t)cnt * p.size > n) { err = path + ": truncated face data"; return false; }
                    if (k != il) {
                        pos += (size_t)cnt * p.size;
                        continue;
                    }
                    if (cnt < 3) { err = path + ": face with fewer than three vertices"; return false; }
                    std::vector<long long> idx((size_t)cnt);
                    for (long long j = 0; j < cnt; j++) {
                        idx[j] = p.is_signed ? read_sint(pos, p.size) : (long long)read_uint(pos, p.size);
                        pos += p.size;
                        if (idx[j] < 0 || idx[j] >= (long long)verts.size()) {
                            err = path + ": vertex index out of range";
                            return false;
                        }
                    }
                    // triangles as PLYParser::parse (ply_parser.cpp:84-104); larger polygons
                    // as a fan around their first vertex
                    for (long long j = 1; j + 1 < cnt; j++) {
                        const Vtx& a = verts[idx[0]];
                        const Vtx& b = verts[idx[j]];
                        const Vtx& c = verts[idx[j + 1]];
                        const Vtx nn = face_normal(a, b, c);
                        push_face(out, a, b, c, nn, nn, nn, 0);
                    }
                }
            }
            have_faces = true;
        } else {
            // skip an element this loader does not use
            for (long long i = 0; i < el.count; i++)
                for (const Prop& p : el.props) {
                    if (!p.count_size) {
                        pos += p.size;
                    } else {
                        if (pos + p.count_size > n) { err = path + ": truncated data"; return false; }
                        const uint64_t cnt = read_uint(pos, p.count_size);
                        pos += p.count_size + (size_t)cnt * p.size;
                    }
                    if (pos > n) { err = path + ": truncated data"; return false; }
                }
        }
        if (have_faces) break;
    }
    if (!have_vertices) { err = path + ": no vertex element"; return false; }
    return true;
}

// ---- EXR -------------------------------------------------------------------------------
// OpenEXR file layout (magic, version, attribute header, chunk offset table, chunks) for
// single-part scanline images. Decompression per the OpenEXR format:
//   RLE   signed run lengths, then the byte predictor and the two-half interleave
//   ZIPS/ZIP  zlib streams of 1/16 scanlines, same predictor and interleave
//   PIZ   32 scanlines: bitmap + reverse LUT, Huffman-coded 16-bit words with a run-length
//         symbol, a 2-D Haar-like wavelet per channel half-word plane, LUT, re-interleave
namespace {

constexpr int kHufEncSize = (1 << 16) + 1;  // symbols 0..65535 plus the run-length symbol
constexpr int kShortZeroRun = 59;           // 6-bit values 59..62: 2..5 zero code lengths
constexpr int kLongZeroRun = 63;            // 63 + 8 bits: 6..261 zero code lengths
constexpr int kShortestLongRun = 2 + kLongZeroRun - kShortZeroRun;
constexpr int kMaxCodeLen = 58;

struct BitReader {
    const uint8_t* p;
    size_t nbytes;
    uint64_t bit = 0;  // bits consumed
    bool get(int n, uint64_t& v) {  // n <= 32, most significant bit first
        v = 0;
        for (int k = 0; k < n; k++) {
            const size_t byte = (size_t)(bit >> 3);
            if (byte >= nbytes) return false;
            v = (v << 1) | ((p[byte] >> (7 - (bit & 7))) & 1u);
            bit++;
        }
        return true;
    }
};

// Huffman decoding of PIZ data: code lengths from the packed table, canonical codes assigned
// longest-first (the codes of length l start at (start[l+1] + count[l+1]) / 2, start[58] = 0,
// in increasing symbol order within a length); symbol `rlc` is followed by an 8-bit repeat
// count of the previous word.
bool huf_decode(const uint8_t* in, size_t nin, uint16_t* out, size_t nout, std::string& err) {
    if (nin == 0) {
        if (nout != 0) { err = "PIZ: empty Huffman stream"; return false; }
        return true;
    }
    if (nin < 20) { err = "PIZ: Huffman header truncated"; return false; }
    const int im = (int)rd32(in), iM = (int)rd32(in + 4);
    const uint32_t nbits = rd32(in + 12);
    if (im < 0 || im >= kHufEncSize || iM < 0 || iM >= kHufEncSize || im > iM) {
        err = "PIZ: bad Huffman symbol range";
        return false;
    }
    std::vector<uint8_t> len(kHufEncSize, 0);
    BitReader tb{in + 20, nin - 20};
    for (int s = im; s <= iM;) {
        uint64_t l;
        if (!tb.get(6, l)) { err = "PIZ: Huffman table truncated"; return false; }
        if (l == (uint64_t)kLongZeroRun || l >= (uint64_t)kShortZeroRun) {
            uint64_t run;
            if (l == (uint64_t)kLongZeroRun) {
                if (!tb.get(8, run)) { err = "PIZ: Huffman table truncated"; return false; }
                run += kShortestLongRun;
            } else {
                run = l - kShortZeroRun + 2;
            }
            if ((uint64_t)s + run > (uint64_t)iM + 1) { err = "PIZ: Huffman table overrun"; return false; }
            s += (int)run;  // lengths stay zero
        } else {
            len[s++] = (uint8_t)l;
        }
    }
    const size_t table_bytes = (size_t)((tb.bit + 7) >> 3);
    const uint8_t* data = in + 20 + table_bytes;
    const size_t ndata = nin - 20 - table_bytes;
    if ((uint64_t)nbits > 8ull * ndata) { err = "PIZ: Huffman bit count exceeds the data"; return false; }
    // canonical code starts per length
    uint64_t count[kMaxCodeLen + 1] = {}, start[kMaxCodeLen + 2] = {};
    for (int s = 0; s < kHufEncSize; s++) count[len[s]]++;
    uint64_t c = 0;
    for (int l = kMaxCodeLen; l > 0; l--) {
        start[l] = c;
        c = (c + count[l]) >> 1;
    }
    // symbols of each length in increasing order
    std::vector<int> first(kMaxCodeLen + 2, 0);
    for (int l = 1; l <= kMaxCodeLen; l++) first[l + 1] = first[l] + (int)count[l];
    std::vector<int> sym(first[kMaxCodeLen + 1]);
    {
        std::vector<int> fill(first.begin(), first.end());
        for (int s = 0; s < kHufEncSize; s++)
            if (len[s]) sym[fill[len[s]]++] = s;
    }
    // fast path: a table over the next kLook bits resolves every code of up to kLook bits
    constexpr int kLook = 12;
    std::vector<int32_t> fast(1 << kLook, -1);  // (symbol << 6) | length
    for (int l = 1; l <= kLook; l++)
        for (uint64_t r = 0; r < count[l]; r++) {
            const uint64_t code = start[l] + r;
            const int s = sym[first[l] + (int)r];
            const uint64_t lo = code << (kLook - l), hi = (code + 1) << (kLook - l);
            for (uint64_t k = lo; k < hi && k < (1u << kLook); k++) fast[k] = (s << 6) | l;
        }
    const int rlc = iM;
    size_t o = 0;
    uint64_t bit = 0;
    auto peek = [&](int n) -> uint64_t {  // next n bits, zero padded past the end of the stream
        uint64_t v = 0;
        for (int k = 0; k < n; k++) {
            const uint64_t b = bit + k;
            const uint64_t x = b < nbits ? ((data[b >> 3] >> (7 - (b & 7))) & 1u) : 0u;
            v = (v << 1) | x;
        }
        return v;
    };
    while (bit < nbits) {
        int s = -1, l = 0;
        const int32_t f = fast[peek(kLook)];
        if (f >= 0 && bit + (f & 63) <= nbits) {
            s = f >> 6;
            l = f & 63;
        } else {
            uint64_t code = 0;
            for (l = 1; l <= kMaxCodeLen; l++) {
                if (bit + l > nbits) break;
                code = (code << 1) | ((data[(bit + l - 1) >> 3] >> (7 - ((bit + l - 1) & 7))) & 1u);
                if (count[l] && code >= start[l] && code - start[l] < count[l]) {
                    s = sym[first[l] + (int)(code - start[l])];
                    break;
                }
            }
            if (s < 0) { err = "PIZ: invalid Huffman code"; return false; }
        }
        bit += l;
        if (s == rlc) {
            if (bit + 8 > nbits) { err = "PIZ: run length truncated"; return false; }
            const uint64_t run = peek(8);
            bit += 8;
            if (o == 0 || o + run > nout) { err = "PIZ: bad run length"; return false; }
            const uint16_t prev = out[o - 1];
            for (uint64_t k = 0; k < run; k++) out[o++] = prev;
        } else {
            if (o >= nout) { err = "PIZ: too much Huffman data"; return false; }
            out[o++] = (uint16_t)s;
        }
    }
    if (o != nout) { err = "PIZ: not enough Huffman data"; return false; }
    return true;
}

// Inverse of PIZ's lossless 2-D Haar wavelet (OpenEXR file format, PIZ compression). A
// forward step maps a pair (a, b) to a low word l and a high word h, h = a - b. Two pair
// rules exist, and a block uses the first when every word value it holds is below 2^14:
//   exact:  l = floor((a + b) / 2), words as signed 16-bit integers; so a = l + ceil(h / 2);
//   modulo: words as unsigned 16-bit integers mod 2^16, with b = l - floor(h / 2) and
//           a = b + h - 2^15 (the forward rule's 2^15 offset keeps h in range).
struct PizPair {
    bool exact;
    void inverse(uint16_t& lo_then_a, uint16_t& hi_then_b) const {
        if (exact) {
            const int l = (int16_t)lo_then_a, h = (int16_t)hi_then_b;
            const int a = l + ((h + 1) >> 1);  // arithmetic shift: ceil(h / 2)
            lo_then_a = (uint16_t)a;
            hi_then_b = (uint16_t)(a - h);
        } else {
            const unsigned l = lo_then_a, h = hi_then_b;
            const unsigned b = (l - (h >> 1)) & 0xffffu;
            lo_then_a = (uint16_t)((b + h - 0x8000u) & 0xffffu);
            hi_then_b = (uint16_t)b;
        }
    }
};

// Inverse 2-D wavelet over an nx x ny plane of words at element stride sx, row stride sy.
// Level `step` pairs samples `step` apart. At each level, the samples on the step grid are
// first inverted in vertical pairs (rows 2j*step and (2j+1)*step, every column of the
// grid, the unpaired last column of an odd count included), then in horizontal pairs (every
// row of the grid, the unpaired last row included); an unpaired last row or column keeps its
// value in the other direction. Levels run from the coarsest step (half the largest power
// of two not above min(nx, ny)) down to 1.
void wav2_decode(uint16_t* plane, int nx, int sx, int ny, int sy, uint16_t max_word) {
    const PizPair pair{max_word < (1 << 14)};
    const int n = std::min(nx, ny);
    int top = 1;
    while (top * 2 <= n) top *= 2;
    auto at = [&](int x, int y) -> uint16_t& { return plane[(ptrdiff_t)y * sy + (ptrdiff_t)x * sx]; };
    for (int step = top / 2; step >= 1; step /= 2) {
        const int cols = nx / step, rows = ny / step;  // grid samples in each direction
        for (int j = 0; j + 1 < rows; j += 2)          // vertical pairs
            for (int i = 0; i < cols; i++) pair.inverse(at(i * step, j * step), at(i * step, (j + 1) * step));
        for (int j = 0; j < rows; j++)                 // horizontal pairs
            for (int i = 0; i + 1 < cols; i += 2) pair.inverse(at(i * step, j * step), at((i + 1) * step, j * step));
    }
}

// PIZ block -> raw scanline bytes (each line: channels in order, width words of 1 or 2 16-bit
// halves per pixel, little-endian)
bool piz_decode(const uint8_t* in, size_t nin, uint8_t* raw, size_t nraw, int width, int lines,
                const std::vector<int>& words_per_px, std::string& err) {
    const size_t nwords = nraw / 2;
    if (nin < 4) { err = "PIZ: block truncated"; return false; }
    const int mn = rd16(in), mxnz = rd16(in + 2);
    size_t p = 4;
    if (mxnz >= 8192) { err = "PIZ: bad bitmap range"; return false; }
    std::vector<uint8_t> bitmap(8192, 0);
    if (mn <= mxnz) {
        const size_t nb = (size_t)(mxnz - mn + 1);
        if (p + nb > nin) { err = "PIZ: bitmap truncated"; return false; }
        std::memcpy(bitmap.data() + mn, in + p, nb);
        p += nb;
    }
    // reverse LUT: the k-th word value present (0 always), maxValue = entries - 1
    std::vector<uint16_t> lut(65536, 0);
    int k = 0;
    for (int i = 0; i < 65536; i++)
        if (i == 0 || (bitmap[i >> 3] & (1 << (i & 7)))) lut[k++] = (uint16_t)i;
    const uint16_t maxv = (uint16_t)(k - 1);
    if (p + 4 > nin) { err = "PIZ: block truncated"; return false; }
    const uint32_t hl = rd32(in + p);
    p += 4;
    if ((size_t)hl > nin - p) { err = "PIZ: Huffman length exceeds the block"; return false; }
    std::vector<uint16_t> tmp(nwords);
    if (!huf_decode(in + p, hl, tmp.data(), nwords, err)) return false;
    // wavelet per channel plane and half-word
    size_t start = 0;
    std::vector<size_t> plane(words_per_px.size());
    for (size_t c = 0; c < words_per_px.size(); c++) {
        const int sz = words_per_px[c];
        plane[c] = start;
        for (int j = 0; j < sz; j++)
            wav2_decode(tmp.data() + start + j, width, sz, lines, width * sz, maxv);
        start += (size_t)width * lines * sz;
    }
    for (uint16_t& w : tmp) w = lut[w];
    // channel planes -> scanlines
    size_t o = 0;
    std::vector<size_t> cur(plane);
    for (int y = 0; y < lines; y++)
        for (size_t c = 0; c < words_per_px.size(); c++) {
            const size_t nw = (size_t)width * words_per_px[c];
            for (size_t i = 0; i < nw; i++) {
                const uint16_t w = tmp[cur[c] + i];
                raw[o++] = (uint8_t)(w & 0xff);
                raw[o++] = (uint8_t)(w >> 8);
            }
            cur[c] += nw;
        }
    return o == nraw;
}

// undo the byte predictor and the even/odd split of ZIP and RLE blocks
void unpredict(std::vector<uint8_t>& t, uint8_t* out) {
    for (size_t i = 1; i < t.size(); i++) t[i] = (uint8_t)(t[i - 1] + t[i] - 128);
    const size_t n = t.size(), half = (n + 1) / 2;
    for (size_t i = 0, a = 0, b = half; i < n;) {
        out[i++] = t[a++];
        if (i < n) out[i++] = t[b++];
    }
}

bool rle_decode(const uint8_t* in, size_t nin, std::vector<uint8_t>& out) {
    size_t i = 0, o = 0;
    while (i < nin) {
        const int c = (int8_t)in[i++];
        if (c < 0) {
            const size_t cnt = (size_t)(-c);
            if (i + cnt > nin || o + cnt > out.size()) return false;
            std::memcpy(out.data() + o, in + i, cnt);
            i += cnt;
            o += cnt;
        } else {
            const size_t cnt = (size_t)c + 1;
            if (i >= nin || o + cnt > out.size()) return false;
            std::memset(out.data() + o, in[i++], cnt);
            o += cnt;
        }
    }
    return o == out.size();
}

float half_to_float(uint16_t h) {
    const int s = h >> 15, e = (h >> 10) & 31, m = h & 1023;
    float v;
    if (e == 0) v = std::ldexp((float)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = std::ldexp((float)(m | 1024), e - 25);
    return s ? -v : v;
}

}  // namespace

bool read_exr(const std::string& path, int& width, int& height, std::vector<float>& rgba, std::string& err) {
    std::string file;
    if (!read_file(path, file)) {
        err = "cannot read " + path;
        return false;
    }
    const uint8_t* d = (const uint8_t*)file.data();
    const size_t n = file.size();
    if (n < 8 || rd32(d) != 20000630u) { err = path + ": not an OpenEXR file"; return false; }
    const uint32_t ver = rd32(d + 4);
    if ((ver & 0xff) != 2) { err = path + ": unsupported OpenEXR version"; return false; }
    if (ver & (0x200 | 0x800 | 0x1000)) {
        err = path + ": tiled, deep and multi-part OpenEXR files are not supported";
        return false;
    }
    struct Chan {
        std::string name;
        int type;
    };
    std::vector<Chan> chans;
    int compression = -1;
    int32_t box[4] = {0, 0, -1, -1};
    bool have_box = false;
    size_t p = 8;
    auto cstr = [&](std::string& s) {
        const void* z = std::memchr(d + p, 0, n - p);
        if (!z) return false;
        const size_t e = (const uint8_t*)z - d;
        s.assign((const char*)d + p, e - p);
        p = e + 1;
        return true;
    };
    while (true) {
        if (p >= n) { err = path + ": header truncated"; return false; }
        if (d[p] == 0) {
            p++;
            break;
        }
        std::string name, type;
        if (!cstr(name) || !cstr(type) || p + 4 > n) { err = path + ": header truncated"; return false; }
        const uint32_t size = rd32(d + p);
        p += 4;
        if (size > n - p) { err = path + ": header truncated"; return false; }
        const uint8_t* v = d + p;
        if (name == "channels" && type == "chlist") {
            size_t q = 0;
            while (q < size && v[q] != 0) {
                const void* z = std::memchr(v + q, 0, size - q);
                if (!z) { err = path + ": bad channel list"; return false; }
                const size_t e = (const uint8_t*)z - v;
                Chan ch;
                ch.name.assign((const char*)v + q, e - q);
                q = e + 1;
                if (q + 16 > size) { err = path + ": bad channel list"; return false; }
                ch.type = (int)rd32(v + q);
                const int xs = (int)rd32(v + q + 8), ys = (int)rd32(v + q + 12);
                q += 16;
                if (xs != 1 || ys != 1) { err = path + ": subsampled channels are not supported"; return false; }
                if (ch.type != 1 && ch.type != 2) {
                    err = path + ": channel " + ch.name + " is not HALF or FLOAT";
                    return false;
                }
                chans.push_back(ch);
            }
        } else if (name == "compression" && size >= 1) {
            compression = v[0];
        } else if (name == "dataWindow" && type == "box2i" && size >= 16) {
            for (int k = 0; k < 4; k++) box[k] = (int32_t)rd32(v + 4 * k);
            have_box = true;
        }
        p += size;
    }
    if (chans.empty() || !have_box) { err = path + ": missing channels or dataWindow"; return false; }
    const long long w = (long long)box[2] - box[0] + 1, h = (long long)box[3] - box[1] + 1;
    if (w <= 0 || h <= 0 || w > (1 << 16) || h > (1 << 16)) { err = path + ": bad data window"; return false; }
    int lpc;
    switch (compression) {
        case 0: case 1: case 2: lpc = 1; break;
        case 3: lpc = 16; break;
        case 4: lpc = 32; break;
        default:
            err = path + ": unsupported compression " + std::to_string(compression) +
                  " (NONE, RLE, ZIPS, ZIP and PIZ are read)";
            return false;
    }
    std::vector<int> words;  // 16-bit words per pixel of each channel
    size_t row_bytes = 0;
    for (const Chan& c : chans) {
        words.push_back(c.type == 1 ? 1 : 2);
        row_bytes += (size_t)w * 2 * words.back();
    }
    const long long nchunks = (h + lpc - 1) / lpc;
    if (p + 8 * (size_t)nchunks > n) { err = path + ": offset table truncated"; return false; }
    std::vector<std::vector<float>> planes(chans.size(), std::vector<float>((size_t)(w * h)));
    std::vector<uint8_t> raw, tmp;
    for (long long c = 0; c < nchunks; c++) {
        const uint64_t off = rd64(d + p + 8 * c);
        if (off + 8 > n) { err = path + ": chunk offset out of range"; return false; }
        const int32_t y = (int32_t)rd32(d + off);
        const uint32_t size = rd32(d + off + 4);
        if (size > n - off - 8) { err = path + ": chunk truncated"; return false; }
        if (y < box[1] || y > box[3]) { err = path + ": chunk y out of range"; return false; }
        const int lines = (int)std::min<long long>(lpc, (long long)box[3] - y + 1);
        const size_t nraw = (size_t)lines * row_bytes;
        const uint8_t* src = d + off + 8;
        raw.assign(nraw, 0);
        if (size >= nraw || compression == 0) {
            if (size != nraw) { err = path + ": bad uncompressed chunk size"; return false; }
            std::memcpy(raw.data(), src, nraw);
        } else if (compression == 1) {
            tmp.assign(nraw, 0);
            if (!rle_decode(src, size, tmp)) { err = path + ": corrupt RLE chunk"; return false; }
            unpredict(tmp, raw.data());
        } else if (compression == 2 || compression == 3) {
            tmp.assign(nraw, 0);
            uLongf dl = (uLongf)nraw;
            if (uncompress(tmp.data(), &dl, src, size) != Z_OK || dl != nraw) {
                err = path + ": corrupt ZIP chunk";
                return false;
            }
            unpredict(tmp, raw.data());
        } else {
            if (!piz_decode(src, size, raw.data(), nraw, (int)w, lines, words, err)) {
                err = path + ": " + err;
                return false;
            }
        }
        size_t q = 0;
        for (int l = 0; l < lines; l++) {
            const size_t row = (size_t)(y - box[1] + l) * (size_t)w;
            for (size_t ch = 0; ch < chans.size(); ch++) {
                float* dst = planes[ch].data() + row;
                if (words[ch] == 1) {
                    for (long long x = 0; x < w; x++, q += 2) dst[x] = half_to_float(rd16(raw.data() + q));
                } else {
                    for (long long x = 0; x < w; x++, q += 4) std::memcpy(&dst[x], raw.data() + q, 4);
                }
            }
        }
    }
    // LoadEXR's RGBA assembly
    const size_t np = (size_t)(w * h);
    rgba.assign(np * 4, 0.f);
    if (chans.size() == 1) {
        for (size_t i = 0; i < np; i++)
            for (int k = 0; k < 4; k++) rgba[4 * i + k] = planes[0][i];
    } else {
        int idx[4] = {-1, -1, -1, -1};
        const char* names[4] = {"R", "G", "B", "A"};
        for (size_t ch = 0; ch < chans.size(); ch++)
            for (int k = 0; k < 4; k++)
                if (chans[ch].name == names[k]) idx[k] = (int)ch;
        for (int k = 0; k < 3; k++)
            if (idx[k] < 0) {
                err = path + ": " + names[k] + " channel not found";
                return false;
            }
        for (size_t i = 0; i < np; i++) {
            for (int k = 0; k < 3; k++) rgba[4 * i + k] = planes[idx[k]][i];
            rgba[4 * i + 3] = idx[3] >= 0 ? planes[idx[3]][i] : 1.f;
        }
    }
    width = (int)w;
    height = (int)h;
    return true;
}

namespace {

// FP32 -> FP16: mantissa truncated to 10 bits, plus one when the first dropped bit is set;
// FP32 denormals become zero, exponents past the half range infinity, NaN a quiet NaN.
// This is the rounding rule of the conversion the reference's Image::save goes through:
// tinyexr's float_to_half_full (vendor/tinyexr.h:7164-7197, which takes it from the ISPC
// reference code). It is restated case for case because the snapshot files must be
// byte-identical to the reference's.
uint16_t half_of(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    const uint32_t sign = x >> 31, ex = (x >> 23) & 0xff, man = x & 0x7fffff;
    uint32_t o = 0;
    if (ex == 0) {
        o = 0;
    } else if (ex == 0xff) {
        o = (31u << 10) | (man ? 0x200u : 0u);
    } else {
        const int ne = (int)ex - 127 + 15;
        if (ne >= 31) {
            o = 31u << 10;
        } else if (ne <= 0) {
            if (14 - ne <= 24) {
                const uint32_t m = man | 0x800000u;
                o = m >> (14 - ne);
                if ((m >> (13 - ne)) & 1u) o++;
            }
        } else {
            o = ((uint32_t)ne << 10) | (man >> 13);
            if (man & 0x1000u) o++;
        }
    }
    return (uint16_t)((sign << 15) | o);
}

void put32(std::string& s, uint32_t v) {
    for (int k = 0; k < 4; k++) s.push_back((char)((v >> (8 * k)) & 0xff));
}

void attribute(std::string& s, const char* name, const char* type, const std::string& value) {
    s.append(name).push_back('\0');
    s.append(type).push_back('\0');
    put32(s, (uint32_t)value.size());
    s.append(value);
}

}  // namespace

bool write_exr(const std::string& path, int width, int height, const float* rgb, std::string& err) {
    if (width <= 0 || height <= 0 || !rgb) {
        err = "write_exr: empty image";
        return false;
    }
    std::string head;
    put32(head, 20000630u);
    put32(head, 2u);
    std::string chl;
    for (const char* c : {"B", "G", "R"}) {
        chl.append(c).push_back('\0');
        put32(chl, 1u);  // HALF
        put32(chl, 0u);  // pLinear + reserved
        put32(chl, 1u);
        put32(chl, 1u);
    }
    chl.push_back('\0');
    std::string box;
    for (uint32_t v : {0u, 0u, (uint32_t)(width - 1), (uint32_t)(height - 1)}) put32(box, v);
    // pixelAspectRatio 1; screenWindowWidth holds the image width, as the vendored writer does
    const float one = 1.f, fw = (float)width;
    uint32_t onebits, wbits;
    std::memcpy(&onebits, &one, 4);
    std::memcpy(&wbits, &fw, 4);
    std::string f1, v2, sww;
    put32(f1, onebits);
    put32(sww, wbits);
    put32(v2, 0u);
    put32(v2, 0u);
    attribute(head, "channels", "chlist", chl);
    attribute(head, "compression", "compression", std::string(1, '\0'));
    attribute(head, "dataWindow", "box2i", box);
    attribute(head, "displayWindow", "box2i", box);
    attribute(head, "lineOrder", "lineOrder", std::string(1, '\0'));
    attribute(head, "pixelAspectRatio", "float", f1);
    attribute(head, "screenWindowCenter", "v2f", v2);
    attribute(head, "screenWindowWidth", "float", sww);
    head.push_back('\0');
    const size_t row_bytes = (size_t)width * 2 * 3;
    const size_t chunk = 8 + row_bytes;
    std::string out = head;
    uint64_t off = head.size() + 8ull * height;
    for (int y = 0; y < height; y++, off += chunk) {
        put32(out, (uint32_t)(off & 0xffffffffu));
        put32(out, (uint32_t)(off >> 32));
    }
    std::string line(row_bytes, '\0');
    for (int y = 0; y < height; y++) {
        put32(out, (uint32_t)y);
        put32(out, (uint32_t)row_bytes);
        const int row = height - 1 - y;  // file row y holds image row height - 1 - y
        for (int c = 0; c < 3; c++) {      // B, G, R
            const int k = 2 - c;
            for (int x = 0; x < width; x++) {
                const uint16_t h = half_of(rgb[3 * ((size_t)row * width + x) + k]);
                line[((size_t)c * width + x) * 2] = (char)(h & 0xff);
                line[((size_t)c * width + x) * 2 + 1] = (char)(h >> 8);
            }
        }
        out += line;
    }
    std::ofstream f(path, std::ios::binary);
    if (!f || !f.write(out.data(), (std::streamsize)out.size())) {
        err = "cannot write " + path;
        return false;
    }
    return true;
}

// ---- scenes ----------------------------------------------------------------------------

bool build_request(const SceneRequest& req, HostScene& out, std::string& err) {
    out = HostScene();
    out.mats = req.mats;
    const int nreq = (int)req.mats.size();
    auto check_default = [&](const MeshFile& f) {
        if (f.default_material < 0 || f.default_material >= nreq) {
            err = f.path + ": default material " + std::to_string(f.default_material) + " is not in the request";
            return false;
        }
        return true;
    };
    auto append = [&](const MeshFaces& m, const std::vector<int>& mat) {
        out.tri_p.insert(out.tri_p.end(), m.p.begin(), m.p.end());
        const size_t n0 = out.tri_n.size();
        out.tri_n.insert(out.tri_n.end(), m.n.begin(), m.n.end());
        // A face with coincident or collinear corners gets the reference's 0/0 normal; it is
        // kept (triangle indices stay those of the reference) with a zero normal instead.
        for (size_t v = n0; v < out.tri_n.size(); v += 3)
            if (!std::isfinite(out.tri_n[v]) || !std::isfinite(out.tri_n[v + 1]) || !std::isfinite(out.tri_n[v + 2]))
                out.tri_n[v] = out.tri_n[v + 1] = out.tri_n[v + 2] = 0.f;
        out.tri_mat.insert(out.tri_mat.end(), mat.begin(), mat.end());
    };
    for (int pass = 0; pass < 2; pass++) {  // OBJ files first, then PLY files
        for (const MeshFile& f : req.files) {
            if ((pass == 0) != (f.format == kMeshObj)) continue;
            if (f.format != kMeshObj && f.format != kMeshPly) {
                err = f.path + ": unknown mesh format " + std::to_string(f.format);
                return false;
            }
            if (!check_default(f)) return false;
            MeshFaces m;
            if (!(f.format == kMeshObj ? parse_obj(f.path, m, err) : parse_ply(f.path, m, err))) return false;
            std::vector<int> mat(m.num_faces(), f.default_material);
            if (f.format == kMeshObj && !m.mtls.empty()) {
                // MTL materials become Lambertians after the ones already present
                const int offset = (int)out.mats.size();
                for (const MeshMtl& t : m.mtls) {
                    Material x{};
                    x.type = kLambertian;
                    for (int k = 0; k < 3; k++) {
                        x.albedo[k] = t.kd[k];
                        x.emit[k] = t.ke[k];
                    }
                    out.mats.push_back(x);
                }
                for (int i = 0; i < m.num_faces(); i++) mat[i] = offset + m.mtl[i];
            }
            append(m, mat);
        }
    }
    if (req.sph.size() != req.sph_mat.size() * 4) {
        err = "sphere arrays have inconsistent sizes";
        return false;
    }
    out.sph = req.sph;
    out.sph_mat = req.sph_mat;
    if (!req.env_path.empty() && !read_exr(req.env_path, out.env_w, out.env_h, out.env_rgba, err)) return false;
    return true;
}

namespace {

Material lambertian(float r, float g, float b, float er = 0.f, float eg = 0.f, float eb = 0.f) {
    Material m{};
    m.type = kLambertian;
    m.albedo[0] = r; m.albedo[1] = g; m.albedo[2] = b;
    m.emit[0] = er; m.emit[1] = eg; m.emit[2] = eb;
    return m;
}
Material of_type(int type, float ior = 0.f, float alpha = 0.f) {
    Material m{};
    m.type = type;
    m.ior = ior;
    m.alpha = alpha;
    return m;
}

}  // namespace

bool reference_scene(int index, const std::string& scenes_dir, HostScene& out, std::string& err) {
    const std::string root = scenes_dir.empty() ? std::string(".") : scenes_dir;
    auto at = [&](const char* rel) { return root + "/" + rel; };
    SceneRequest r;
    CameraSpec cam{};
    // SceneParameters::getCamera (src/scene.cu:174-218): vfov = degrees / 180 * M_PI in double
    auto set_cam = [&](float ox, float oy, float oz, float tx, float ty, float tz, float ux, float uy, float uz,
                       float deg, bool flip) {
        const float o[3] = {ox, oy, oz}, t[3] = {tx, ty, tz}, u[3] = {ux, uy, uz};
        for (int k = 0; k < 3; k++) {
            cam.origin[k] = o[k];
            cam.target[k] = t[k];
            cam.up[k] = u[k];
        }
        cam.vfov = (float)((double)(deg / 180.f) * M_PI);
        cam.flip = flip;
    };
    switch (index) {
        case 0:  // scene.cu:18-33
            r.mats = {lambertian(1.f, 0.f, 0.f)};
            r.files = {{at("cornell-box/CornellBox-Original.obj"), kMeshObj, 0}};
            set_cam(0.f, 1.f, 6.8f, 0.f, 1.f, 0.f, 0.f, 1.f, 0.f, 19.5f, false);
            out.name = "reference-cornell-box";
            break;
        case 1:  // scene.cu:34-72
            r.mats = {lambertian(1.f, 0.f, 0.f), of_type(kMirror), of_type(kGlass, 1.4f)};
            r.files = {{at("cornell-glossy/CornellBox-Glossy.obj"), kMeshObj, 0},
                       {at("cornell-glossy/box.obj"), kMeshObj, 1}};
            r.sph = {0.45f, 0.451f, -0.4f, 0.45f};
            r.sph_mat = {2};
            set_cam(0.f, 1.f, 6.8f, 0.f, 1.f, 0.f, 0.f, 1.f, 0.f, 19.5f, false);
            out.name = "reference-cornell-glossy";
            break;
        case 2:  // scene.cu:73-93
            r.mats = {lambertian(1.f, 1.f, 1.f)};
            r.files = {{at("tests/plane.obj"), kMeshObj, 0}};
            r.env_path = at("assets/1_pixel_test.exr");
            set_cam(0.f, 1.f, 6.8f, 0.f, 1.f, 0.f, 0.f, 1.f, 0.f, 19.5f, false);
            out.name = "reference-env-plane";
            break;
        case 3: {  // scene.cu:94-166, the Veach MIS scene
            r.mats = {lambertian(0.4f, 0.4f, 0.4f), of_type(kMicrofacet, 0.f, 0.005f),
                      of_type(kMicrofacet, 0.f, 0.02f), of_type(kMicrofacet, 0.f, 0.05f),
                      of_type(kMicrofacet, 0.f, 0.1f)};
            const char* plies[5] = {"mis/floor.ply", "mis/plate1.ply", "mis/plate2.ply", "mis/plate3.ply",
                                    "mis/plate4.ply"};
            for (int i = 0; i < 5; i++) r.files.push_back({at(plies[i]), kMeshPly, i});
            const float emit[5] = {800.f, 100.f, 901.803f, 11.1111f, 1.234567f};
            for (float e : emit) r.mats.push_back(lambertian(0.f, 0.f, 0.f, e, e, e));
            r.sph = {10.f, 10.f, 4.f, 0.5f, -1.25f, 0.f, 0.f, 0.1f, -3.75f, 0.f, 0.f, 0.03333f,
                     1.25f, 0.f, 0.f, 0.3f, 3.75f, 0.f, 0.f, 0.9f};
            r.sph_mat = {5, 6, 7, 8, 9};
            r.env_path = at("assets/20060807_wells6_hd.exr");
            set_cam(0.f, 2.f, 15.f, 0.f, 1.69521f, 14.0476f, 0.f, 0.952421f, -0.304787f, 28.0000262073138f, true);
            out.name = "reference-veach-mis";
            break;
        }
        default:
            err = "reference scene index must be 0-3";
            return false;
    }
    const std::string name = out.name;
    if (!build_request(r, out, err)) return false;
    out.name = name;
    out.camera = cam;
    out.default_depth = 3;  // include/scene.h:18 defaultMaxDepth
    out.default_nee = true;
    out.default_spp = 1;
    return true;
}

}  // namespace pt
