// Seeded procedural scene generators and scene bookkeeping (host side).
//
// The reference loads fixed OBJ/PLY presets (src/scene.cu:14-172); this runtime generates
// seeded synthetic configurations instead, with the reference's scene semantics kept:
// emitters are Lambertian materials with non-zero emit (include/scene_data.h:38-40), the
// emitter list lists triangles before spheres (src/scene_data.cu:92-115), and emission is
// front-face only, so every generated surface carries vertex normals on its visible side and
// a winding whose geometric normal agrees with them (light sampling uses the winding,
// include/primitives/triangle.h:66-86).
#include "host_scene.h"

#include <algorithm>
#include <cmath>
#include <unordered_map>

namespace pt {

namespace {

constexpr double kPi = 3.14159265358979323846;

// SplitMix64 (Steele, Lea, Flood 2014) as a seeded integer hash / generator.
inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

struct HostRng {
    uint64_t s;
    explicit HostRng(uint64_t seed) : s(splitmix64(seed)) {}
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ULL;
        return splitmix64(s);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * uniform(); }
    double normal() {  // Box-Muller
        double u1 = uniform();
        double u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
    }
};

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross3(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 norm3(V3 a) {
    double l = std::sqrt(dot3(a, a));
    return l > 0 ? a * (1.0 / l) : a;
}

Material lambert(float r, float g, float b, float er = 0, float eg = 0, float eb = 0) {
    Material m{};
    m.type = kLambertian;
    m.albedo[0] = r; m.albedo[1] = g; m.albedo[2] = b;
    m.emit[0] = er; m.emit[1] = eg; m.emit[2] = eb;
    m.ior = 0.f;
    m.alpha = 0.f;
    return m;
}
Material mirror() {
    Material m{};
    m.type = kMirror;
    return m;
}
Material glass(float ior) {
    Material m{};
    m.type = kGlass;
    m.ior = ior;
    return m;
}
Material microfacet(float alpha) {
    Material m{};
    m.type = kMicrofacet;
    m.alpha = alpha;
    return m;
}

void push_tri(HostScene& s, V3 a, V3 b, V3 c, V3 na, V3 nb, V3 nc, int mat) {
    const V3 p[3] = {a, b, c};
    const V3 n[3] = {na, nb, nc};
    for (int i = 0; i < 3; i++) {
        s.tri_p.push_back((float)p[i].x);
        s.tri_p.push_back((float)p[i].y);
        s.tri_p.push_back((float)p[i].z);
        s.tri_n.push_back((float)n[i].x);
        s.tri_n.push_back((float)n[i].y);
        s.tri_n.push_back((float)n[i].z);
    }
    s.tri_mat.push_back(mat);
}

// Flat triangle whose winding is made to agree with `normal`.
void push_flat_tri(HostScene& s, V3 a, V3 b, V3 c, V3 normal, int mat) {
    if (dot3(cross3(b - a, c - a), normal) < 0) std::swap(b, c);
    push_tri(s, a, b, c, normal, normal, normal, mat);
}

// Quad a-b-c-d (in order around the rim) split into (a,b,c) and (a,c,d).
void push_quad(HostScene& s, V3 a, V3 b, V3 c, V3 d, V3 normal, int mat) {
    push_flat_tri(s, a, b, c, normal, mat);
    push_flat_tri(s, a, c, d, normal, mat);
}

// Axis-aligned rectangle subdivided into nu x nv quads. `origin` + u*du + v*dv.
void push_grid(HostScene& s, V3 origin, V3 du, V3 dv, int nu, int nv, V3 normal, int mat) {
    for (int j = 0; j < nv; j++) {
        for (int i = 0; i < nu; i++) {
            V3 a = origin + du * ((double)i / nu) + dv * ((double)j / nv);
            V3 b = origin + du * ((double)(i + 1) / nu) + dv * ((double)j / nv);
            V3 c = origin + du * ((double)(i + 1) / nu) + dv * ((double)(j + 1) / nv);
            V3 d = origin + du * ((double)i / nu) + dv * ((double)(j + 1) / nv);
            push_quad(s, a, b, c, d, normal, mat);
        }
    }
}

// Box of half-extents (hx, hy, hz) rotated by `angle` about +y, base centre at `base`.
void push_box(HostScene& s, V3 base, double hx, double hy, double hz, double angle, int mat) {
    const double ca = std::cos(angle), sa = std::sin(angle);
    auto xf = [&](V3 p) {  // local (centre at origin) -> world
        V3 r{ca * p.x + sa * p.z, p.y, -sa * p.x + ca * p.z};
        return r + V3{base.x, base.y + hy, base.z};
    };
    auto xn = [&](V3 n) { return V3{ca * n.x + sa * n.z, n.y, -sa * n.x + ca * n.z}; };
    const V3 c[8] = {{-hx, -hy, -hz}, {hx, -hy, -hz}, {hx, hy, -hz}, {-hx, hy, -hz},
                     {-hx, -hy, hz},  {hx, -hy, hz},  {hx, hy, hz},  {-hx, hy, hz}};
    struct Face { int a, b, cc, d; V3 n; };
    const Face faces[6] = {
        {0, 1, 2, 3, {0, 0, -1}}, {4, 5, 6, 7, {0, 0, 1}}, {0, 3, 7, 4, {-1, 0, 0}},
        {1, 2, 6, 5, {1, 0, 0}},  {3, 2, 6, 7, {0, 1, 0}}, {0, 1, 5, 4, {0, -1, 0}},
    };
    for (const Face& f : faces) {
        push_quad(s, xf(c[f.a]), xf(c[f.b]), xf(c[f.cc]), xf(c[f.d]), xn(f.n), mat);
    }
}

// 3-D value noise: hashed lattice values in [-1, 1], smoothstep-trilinear interpolation.
double lattice(uint64_t seed, int64_t x, int64_t y, int64_t z) {
    uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)x * 0x8DA6B343ULL ^
                                              (uint64_t)y * 0xD8163841ULL ^
                                              (uint64_t)z * 0xCB1AB31FULL));
    return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}
double value_noise(uint64_t seed, V3 p) {
    const double fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
    const int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
    auto sm = [](double t) { return t * t * (3.0 - 2.0 * t); };
    const double tx = sm(p.x - fx), ty = sm(p.y - fy), tz = sm(p.z - fz);
    double acc = 0.0;
    for (int dz = 0; dz < 2; dz++)
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                const double w = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
                acc += w * lattice(seed, ix + dx, iy + dy, iz + dz);
            }
    return acc;
}
double fbm3(uint64_t seed, V3 p) {  // 3 octaves, normalised to [-1, 1]
    double a = 1.0, f = 2.0, sum = 0.0, norm = 0.0;
    for (int o = 0; o < 3; o++) {
        sum += a * value_noise(seed + (uint64_t)o * 1013, p * f);
        norm += a;
        a *= 0.5;
        f *= 2.0;
    }
    return sum / norm;
}

// Icosphere of subdivision `level` (20 * 4^level faces), radius 1, displaced radially by
// amplitude * fbm3, with area-weighted smooth vertex normals.
void push_displaced_icosphere(HostScene& s, int level, double radius, double amplitude,
                              uint64_t seed, V3 centre, int mat) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<V3> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0},
                         {0, -1, t}, {0, 1, t}, {0, -1, -t}, {0, 1, -t},
                         {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : v) p = norm3(p);
    std::vector<int> f = {0, 11, 5, 0, 5,  1, 0, 1, 7, 0, 7,  10, 0, 10, 11, 1, 5, 9, 5, 11,
                          4, 11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9,  4, 3,  4,  2, 3, 2, 6, 3,
                          6, 8,  3, 8,  9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8,  6, 7, 9, 8, 1};
    for (int l = 0; l < level; l++) {
        std::unordered_map<uint64_t, int> mid;
        mid.reserve(f.size() * 2);
        std::vector<int> nf;
        nf.reserve(f.size() * 4);
        auto midpoint = [&](int a, int b) {
            const uint64_t key = a < b ? ((uint64_t)a << 32) | (uint32_t)b
                                       : ((uint64_t)b << 32) | (uint32_t)a;
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            v.push_back(norm3((v[a] + v[b]) * 0.5));
            const int id = (int)v.size() - 1;
            mid.emplace(key, id);
            return id;
        };
        for (size_t i = 0; i < f.size(); i += 3) {
            const int a = f[i], b = f[i + 1], c = f[i + 2];
            const int ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            const int add[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
            nf.insert(nf.end(), add, add + 12);
        }
        f.swap(nf);
    }
    // displacement
    std::vector<V3> p(v.size());
    for (size_t i = 0; i < v.size(); i++) {
        const double d = radius * (1.0 + amplitude * fbm3(seed, v[i] * 1.5));
        p[i] = centre + v[i] * d;
    }
    std::vector<V3> n(v.size(), V3{0, 0, 0});
    for (size_t i = 0; i < f.size(); i += 3) {
        const V3 fn = cross3(p[f[i + 1]] - p[f[i]], p[f[i + 2]] - p[f[i]]);  // area-weighted
        for (int k = 0; k < 3; k++) n[f[i + k]] = n[f[i + k]] + fn;
    }
    for (auto& q : n) q = norm3(q);
    const size_t base = s.tri_mat.size();
    s.tri_p.reserve((base + f.size() / 3) * 9);
    s.tri_n.reserve((base + f.size() / 3) * 9);
    s.tri_mat.reserve(base + f.size() / 3);
    for (size_t i = 0; i < f.size(); i += 3) {
        push_tri(s, p[f[i]], p[f[i + 1]], p[f[i + 2]], n[f[i]], n[f[i + 1]], n[f[i + 2]], mat);
    }
}

void gen_cornell(uint64_t seed, HostScene& s) {
    HostRng rng(seed);
    s.mats = {lambert(0.73f, 0.73f, 0.73f), lambert(0.65f, 0.05f, 0.05f),
              lambert(0.12f, 0.45f, 0.15f), lambert(0.78f, 0.78f, 0.78f, 15.f, 15.f, 15.f)};
    const int white = 0, red = 1, green = 2, light = 3;
    // room x in [-1, 1], y in [0, 2], z in [-1, 1]; open at z = +1
    push_quad(s, {-1, 0, -1}, {1, 0, -1}, {1, 0, 1}, {-1, 0, 1}, {0, 1, 0}, white);    // floor
    push_quad(s, {-1, 2, -1}, {1, 2, -1}, {1, 2, 1}, {-1, 2, 1}, {0, -1, 0}, white);   // ceiling
    push_quad(s, {-1, 0, -1}, {1, 0, -1}, {1, 2, -1}, {-1, 2, -1}, {0, 0, 1}, white);  // back
    push_quad(s, {-1, 0, -1}, {-1, 2, -1}, {-1, 2, 1}, {-1, 0, 1}, {1, 0, 0}, red);    // left
    push_quad(s, {1, 0, -1}, {1, 2, -1}, {1, 2, 1}, {1, 0, 1}, {-1, 0, 0}, green);     // right
    const double a1 = -0.30 + 0.12 * rng.uniform(-1, 1);
    const double a2 = 0.30 + 0.12 * rng.uniform(-1, 1);
    push_box(s, {0.36, 0, 0.32}, 0.3, 0.3, 0.3, a1, white);      // short box, 12 tris
    push_box(s, {-0.34, 0, -0.30}, 0.3, 0.6, 0.3, a2, white);    // tall box, 12 tris
    // emitter quad 0.5 x 0.5 (area 0.25) just below the ceiling, facing down
    const double ly = 1.999;
    push_quad(s, {-0.25, ly, -0.25}, {0.25, ly, -0.25}, {0.25, ly, 0.25}, {-0.25, ly, 0.25},
              {0, -1, 0}, light);
    s.camera = {{0.f, 1.f, 3.75f}, {0.f, 1.f, 0.f}, {0.f, 1.f, 0.f},
                (float)(40.0 / 180.0 * kPi), false};
    s.res_x = s.res_y = 512;
    s.default_spp = 16;
    s.default_depth = 5;
    s.default_nee = true;
    s.name = "cornell-box-36tri-512x512";
}

void gen_spheres(uint64_t seed, HostScene& s) {
    HostRng rng(seed);
    s.mats.push_back(lambert(0.5f, 0.5f, 0.5f));  // ground
    push_quad(s, {-14, 0, -14}, {14, 0, -14}, {14, 0, 14}, {-14, 0, 14}, {0, 1, 0}, 0);
    // Poisson-disk dart throwing for 64 spheres resting on the plane.
    struct Ball { double x, z, r; };
    std::vector<Ball> balls;
    int attempts = 0;
    while (balls.size() < 64 && attempts < 200000) {
        attempts++;
        const double r = rng.uniform(0.2, 1.0);
        const double x = rng.uniform(-8.0, 8.0), z = rng.uniform(-8.0, 8.0);
        bool ok = true;
        for (const Ball& b : balls) {
            const double dx = b.x - x, dz = b.z - z;
            if (dx * dx + dz * dz < (b.r + r + 0.05) * (b.r + r + 0.05)) { ok = false; break; }
        }
        if (ok) balls.push_back({x, z, r});
    }
    // material split: 40% Beckmann, 20% mirror, 20% glass, 20% Lambert (26/13/13/12)
    std::vector<int> kinds(64);
    for (int i = 0; i < 64; i++) kinds[i] = i < 26 ? kMicrofacet : i < 39 ? kMirror : i < 52 ? kGlass : kLambertian;
    for (int i = 63; i > 0; i--) {
        const int j = (int)(rng.next() % (uint64_t)(i + 1));
        std::swap(kinds[i], kinds[j]);
    }
    for (size_t i = 0; i < balls.size(); i++) {
        Material m;
        switch (kinds[i]) {
            case kMicrofacet: m = microfacet((float)rng.uniform(0.05, 0.5)); break;
            case kMirror: m = mirror(); break;
            case kGlass: m = glass(1.5f); break;
            default: m = lambert((float)rng.uniform(0.2, 0.9), (float)rng.uniform(0.2, 0.9),
                                 (float)rng.uniform(0.2, 0.9));
        }
        s.mats.push_back(m);
        s.sph.insert(s.sph.end(), {(float)balls[i].x, (float)balls[i].r, (float)balls[i].z,
                                   (float)balls[i].r});
        s.sph_mat.push_back((int)s.mats.size() - 1);
    }
    // F0 0.04 or a metallic RGB: half the Beckmann spheres (drawn from their own stream, so
    // the rest of the draw is unchanged) become metals with the normal-incidence reflectance of
    // gold, silver, copper or aluminium (linear RGB, the values tabulated in Hoffman's
    // physically based shading notes, SIGGRAPH 2010); the others keep the reference's
    // dielectric Fresnel of eta 1.5
    static const float kMetalF0[4][3] = {
        {1.000f, 0.766f, 0.336f}, {0.972f, 0.960f, 0.915f}, {0.955f, 0.638f, 0.538f}, {0.913f, 0.922f, 0.924f}};
    HostRng mrng(seed ^ 0x3E7A11C0FFEEULL);
    for (size_t i = 1; i < s.mats.size(); i++) {
        Material& m = s.mats[i];
        if (m.type != kMicrofacet || mrng.uniform(0.0, 1.0) >= 0.5) continue;
        const float* f0 = kMetalF0[mrng.next() % 4];
        m.type = kMetal;
        for (int k = 0; k < 3; k++) m.albedo[k] = f0[k];
    }
    for (int i = 0; i < 4; i++) {  // 4 sphere emitters, radiance 5..50
        const float e = (float)rng.uniform(5.0, 50.0);
        s.mats.push_back(lambert(0.f, 0.f, 0.f, e, e, e));
        const double x = rng.uniform(-6, 6), z = rng.uniform(-6, 6), y = rng.uniform(6.5, 9.0);
        s.sph.insert(s.sph.end(), {(float)x, (float)y, (float)z, (float)rng.uniform(0.6, 1.0)});
        s.sph_mat.push_back((int)s.mats.size() - 1);
    }
    s.camera = {{0.f, 6.f, 17.f}, {0.f, 0.5f, 0.f}, {0.f, 1.f, 0.f}, (float)(40.0 / 180.0 * kPi), false};
    s.res_x = s.res_y = 1024;
    s.default_spp = 64;
    s.default_depth = 8;
    s.default_nee = true;
    s.name = "spheres-64-1024x1024";
}

}  // namespace

void generate_sun_env(uint64_t seed, int w, int h, std::vector<float>& rgba) {
    rgba.assign((size_t)w * h * 4, 0.f);
    HostRng rng(seed ^ 0xE5E5E5E5ULL);
    V3 suns[3];
    float sun_rgb[3][3];
    for (int k = 0; k < 3; k++) {
        const double phi = rng.uniform(0, 2 * kPi);
        const double cy = rng.uniform(0.25, 0.95);
        const double sy = std::sqrt(1 - cy * cy);
        suns[k] = {sy * std::cos(phi), cy, sy * std::sin(phi)};
        for (int c = 0; c < 3; c++) sun_rgb[k][c] = (float)rng.uniform(0.8, 1.0);
    }
    const double sigma = 0.5 / 180.0 * kPi;  // Gaussian angular radius 0.5 degrees
    const double peak = 1e4;
    for (int y = 0; y < h; y++) {
        const double theta = (y + 0.5) / h * kPi;
        for (int x = 0; x < w; x++) {
            const double phi = (x + 0.5) / w * 2 * kPi;
            // lognormal background, mu 0 sigma 1, one independent draw per texel
            const uint64_t hsh = splitmix64(seed * 0x100000001B3ULL + (uint64_t)y * w + x);
            HostRng tr(hsh);
            const float bg = (float)std::exp(tr.normal());
            float rgb[3] = {bg, bg, bg};
            const V3 d{std::sin(theta) * std::cos(phi), std::cos(theta), std::sin(theta) * std::sin(phi)};
            for (int k = 0; k < 3; k++) {
                const double c = std::min(1.0, std::max(-1.0, dot3(d, suns[k])));
                const double ang = std::acos(c);
                if (ang < 6 * sigma) {
                    const double g = peak * std::exp(-0.5 * (ang / sigma) * (ang / sigma));
                    for (int ch = 0; ch < 3; ch++) rgb[ch] += (float)(g * sun_rgb[k][ch]);
                }
            }
            float* t = &rgba[((size_t)y * w + x) * 4];
            t[0] = rgb[0]; t[1] = rgb[1]; t[2] = rgb[2]; t[3] = 1.f;
        }
    }
}

namespace {

void gen_env_mesh(uint64_t seed, HostScene& s, int level) {
    s.mats.push_back(microfacet(0.3f));
    push_displaced_icosphere(s, level, 1.0, 0.05, seed, {0, 0, 0}, 0);
    s.env_w = 2048;
    s.env_h = 1024;
    generate_sun_env(seed, s.env_w, s.env_h, s.env_rgba);
    s.camera = {{0.f, 0.45f, 3.1f}, {0.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, (float)(40.0 / 180.0 * kPi), false};
    s.res_x = 1920;
    s.res_y = 1080;
    s.default_spp = 32;
    s.default_depth = 6;
    s.default_nee = true;
    s.name = "icosphere-env-1920x1080";
}

void gen_slit_room(uint64_t seed, HostScene& s, int level) {
    // room walls first (Lambert 0.6), then the config-2 mesh (Beckmann alpha 0.3)
    s.mats.push_back(lambert(0.6f, 0.6f, 0.6f));
    s.mats.push_back(microfacet(0.3f));
    const int wall = 0;
    const double X = 2.5, Y0 = -1.2, Y1 = 2.8, Z = 2.5, slit = 0.05;
    const int n = 13;
    push_grid(s, {-X, Y0, -Z}, {2 * X, 0, 0}, {0, 0, 2 * Z}, n, n, {0, 1, 0}, wall);   // floor
    push_grid(s, {-X, Y0, -Z}, {2 * X, 0, 0}, {0, Y1 - Y0, 0}, n, n, {0, 0, 1}, wall);  // back
    push_grid(s, {-X, Y0, Z}, {2 * X, 0, 0}, {0, Y1 - Y0, 0}, n, n, {0, 0, -1}, wall);  // front
    push_grid(s, {-X, Y0, -Z}, {0, 0, 2 * Z}, {0, Y1 - Y0, 0}, n, n, {1, 0, 0}, wall);  // left
    push_grid(s, {X, Y0, -Z}, {0, 0, 2 * Z}, {0, Y1 - Y0, 0}, n, n, {-1, 0, 0}, wall);  // right
    // ceiling in two halves, leaving a slit of width 0.05 along x at z in [-0.025, 0.025]
    push_grid(s, {-X, Y1, -Z}, {2 * X, 0, 0}, {0, 0, Z - slit / 2}, n, n / 2, {0, -1, 0}, wall);
    push_grid(s, {-X, Y1, slit / 2}, {2 * X, 0, 0}, {0, 0, Z - slit / 2}, n, n / 2, {0, -1, 0}, wall);
    push_displaced_icosphere(s, level, 1.0, 0.05, seed, {0, 0, 0}, 1);
    s.env_w = 2048;
    s.env_h = 1024;
    generate_sun_env(seed, s.env_w, s.env_h, s.env_rgba);
    s.camera = {{0.3f, 0.9f, 2.3f}, {0.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, (float)(50.0 / 180.0 * kPi), false};
    s.res_x = s.res_y = 1024;
    s.default_spp = 16;
    s.default_depth = 10;
    s.default_nee = true;
    s.name = "slit-room-1024x1024";
}

}  // namespace

void finalize_materials(HostScene& s) {
    for (Material& m : s.mats) {
        const bool nz = m.emit[0] != 0.f || m.emit[1] != 0.f || m.emit[2] != 0.f;
        m.emitting = (m.type == kLambertian && nz) ? 1 : 0;
    }
}

std::vector<LightRef> build_light_list(const HostScene& s) {
    std::vector<LightRef> out;
    auto emits = [&](int mat) {
        const Material& m = s.mats[mat];
        return m.type == kLambertian && (m.emit[0] != 0.f || m.emit[1] != 0.f || m.emit[2] != 0.f);
    };
    for (int i = 0; i < s.num_tri(); i++)
        if (emits(s.tri_mat[i])) out.push_back({kTriangle, i});
    for (int i = 0; i < s.num_sph(); i++)
        if (emits(s.sph_mat[i])) out.push_back({kSphere, i});
    return out;
}

bool generate_config(int config, uint64_t seed, HostScene& out, std::string& err, int level) {
    out = HostScene();
    const uint64_t s = seed + (uint64_t)config;
    switch (config) {
        case 0:
            gen_cornell(s, out);
            // batched workloads: a displaced icosphere (Beckmann 0.3) floating in the box
            if (level >= 0) {
                out.mats.push_back(microfacet(0.3f));
                push_displaced_icosphere(out, level, 0.3, 0.05, s, {0.05, 1.15, 0.35}, (int)out.mats.size() - 1);
            }
            break;
        case 1:
            gen_spheres(s, out);
            if (level >= 0) {  // batched workloads: a displaced icosphere among the spheres
                out.mats.push_back(microfacet(0.3f));
                push_displaced_icosphere(out, level, 1.2, 0.05, s, {0.0, 2.5, 0.0}, (int)out.mats.size() - 1);
            }
            break;
        case 2: gen_env_mesh(s, out, level < 0 ? 8 : level); break;
        case 3: gen_slit_room(s, out, level < 0 ? 8 : level); break;
        default:
            err = "unknown configuration id " + std::to_string(config);
            return false;
    }
    finalize_materials(out);
    return true;
}

std::vector<BatchSpec> generate_batch_specs(uint64_t seed, int n) {
    // Configuration 4: scenes drawn from configurations 0-3 with log-uniform triangle counts
    // (1k-2M, realised as the nearest icosphere level 3-8: 1,280 to 1,310,720 mesh triangles),
    // square resolutions 256-1024 in steps of 64, spp 4-64 (powers of two), depth 4-10, and a
    // guide network for about half of them.
    HostRng rng(seed ^ 0xB47C4ULL);
    std::vector<BatchSpec> out;
    for (int i = 0; i < n; i++) {
        BatchSpec b;
        b.config = (int)(rng.uniform() * 4.0) & 3;
        b.seed = seed + 1000003ULL * (uint64_t)(i + 1);
        const double tris = std::exp(rng.uniform(std::log(1e3), std::log(2e6)));
        int level = (int)std::lround(std::log(tris / 20.0) / std::log(4.0));
        b.level = std::max(3, std::min(8, level));
        const int res = 256 + 64 * (int)(rng.uniform() * 13.0);
        b.width = b.height = std::min(1024, res);
        b.spp = 4 << (int)(rng.uniform() * 5.0);
        b.max_depth = 4 + (int)(rng.uniform() * 7.0);
        b.guided = rng.uniform() < 0.5 ? 1 : 0;
        out.push_back(b);
    }
    return out;
}

bool validate_scene(const HostScene& s, std::string& err) {
    const int nm = (int)s.mats.size();
    if (s.tri_p.size() != (size_t)s.num_tri() * 9 || s.tri_n.size() != (size_t)s.num_tri() * 9) {
        err = "triangle arrays have inconsistent sizes";
        return false;
    }
    if (s.sph.size() != (size_t)s.num_sph() * 4) {
        err = "sphere arrays have inconsistent sizes";
        return false;
    }
    for (const Material& m : s.mats) {
        if (m.type < kLambertian || m.type > kMetal || m.type == kMaterialNone) {
            err = "unknown material type " + std::to_string(m.type);
            return false;
        }
    }
    for (int i = 0; i < s.num_tri(); i++) {
        if (s.tri_mat[i] < 0 || s.tri_mat[i] >= nm) {
            err = "triangle " + std::to_string(i) + " has material id out of range";
            return false;
        }
        for (int k = 0; k < 9; k++) {
            if (!std::isfinite(s.tri_p[(size_t)i * 9 + k]) || !std::isfinite(s.tri_n[(size_t)i * 9 + k])) {
                err = "triangle " + std::to_string(i) + " has a non-finite vertex or normal";
                return false;
            }
        }
    }
    for (int i = 0; i < s.num_sph(); i++) {
        if (s.sph_mat[i] < 0 || s.sph_mat[i] >= nm) {
            err = "sphere " + std::to_string(i) + " has material id out of range";
            return false;
        }
        for (int k = 0; k < 4; k++) {
            if (!std::isfinite(s.sph[(size_t)i * 4 + k])) {
                err = "sphere " + std::to_string(i) + " is not finite";
                return false;
            }
        }
        if (!(s.sph[(size_t)i * 4 + 3] > 0.f)) {
            err = "sphere " + std::to_string(i) + " has a non-positive radius";
            return false;
        }
    }
    if (s.env_w < 0 || s.env_h < 0 || s.env_rgba.size() != (size_t)s.env_w * s.env_h * 4) {
        err = "environment map has inconsistent size";
        return false;
    }
    for (float v : s.env_rgba) {
        if (!std::isfinite(v) || v < 0.f) {
            err = "environment map has a negative or non-finite texel";
            return false;
        }
    }
    if (s.num_tri() + s.num_sph() == 0) {
        err = "scene has no primitives";
        return false;
    }
    return true;
}

}  // namespace pt
