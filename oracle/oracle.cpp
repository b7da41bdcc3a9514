// ORACLE - test infrastructure, not product code.
//
// CPU restatement of the reference's vanilla-CUDA path integrator (chellmuth/gpu-pathed),
// used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
// checker. Each routine cites the reference file:line it restates. Arithmetic follows the
// reference's types, including its promotions to double through M_PI; it is built with
// -ffp-contract=off so single-precision expressions round exactly as written.
//
// Pinned against: the reference's own distribution tests (test/test_distribution.cu), and
// the reference's intersection/BSDF/sampling/camera code compiled for the host from the
// reference sources (oracle/ref_cpu.cpp -> oracle/_ref/libref_cpu.so), compared bit for bit.
//
// Random numbers: PCG32, one stream per pixel and one starting state per (seed, sample
// index), the same scheme the CUDA path uses, so both consume identical variates per path.
// The reference itself uses curand XORWOW (not reproduced), so integrator-level agreement
// with the reference is statistical.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace oracle {

// Dynamic parallel loop over [0, n) on `threads` host threads (0: all hardware threads).
template <class F>
void parallel_for(int n, int threads, int chunk, F&& fn) {
    int t = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    t = std::min(t, std::max(1, (n + chunk - 1) / chunk));
    std::atomic<int> next{0};
    auto worker = [&](int tid) {
        for (;;) {
            const int b = next.fetch_add(chunk);
            if (b >= n) break;
            const int e = std::min(n, b + chunk);
            for (int i = b; i < e; i++) fn(i, tid);
        }
    };
    if (t == 1) { worker(0); return; }
    std::vector<std::thread> pool;
    for (int k = 0; k < t; k++) pool.emplace_back(worker, k);
    for (auto& th : pool) th.join();
}

// ---- Vec3 (include/core/vec3.h) ---------------------------------------------------------
struct Vec3 {
    float e[3];
    Vec3() : e{0, 0, 0} {}
    Vec3(float a, float b, float c) : e{a, b, c} {}
    explicit Vec3(float a) : e{a, a, a} {}
    float x() const { return e[0]; }
    float y() const { return e[1]; }
    float z() const { return e[2]; }
    Vec3 operator-() const { return Vec3(-e[0], -e[1], -e[2]); }
    Vec3 operator*(float t) const { return Vec3(t * e[0], t * e[1], t * e[2]); }
    Vec3 operator*(const Vec3& v) const { return Vec3(v.e[0] * e[0], v.e[1] * e[1], v.e[2] * e[2]); }
    Vec3 operator-(const Vec3& v) const { return Vec3(e[0] - v.e[0], e[1] - v.e[1], e[2] - v.e[2]); }
    Vec3& operator+=(const Vec3& v) {
        e[0] += v.e[0]; e[1] += v.e[1]; e[2] += v.e[2];
        return *this;
    }
    Vec3& operator*=(const Vec3& v) {
        e[0] *= v.e[0]; e[1] *= v.e[1]; e[2] *= v.e[2];
        return *this;
    }
    float length() const { return sqrtf(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]); }
    bool isZero() const { return e[0] == 0.f && e[1] == 0.f && e[2] == 0.f; }
    Vec3 dotv(const Vec3& v) const { return Vec3(e[0] * v.e[0] + e[1] * v.e[1] + e[2] * v.e[2]); }
    Vec3 reflect(const Vec3& n) const { return n * dotv(n) * 2.f - *this; }  // vec3.h:48-50
};
inline Vec3 cross(const Vec3& a, const Vec3& b) {
    return Vec3(a.e[1] * b.e[2] - a.e[2] * b.e[1], -(a.e[0] * b.e[2] - a.e[2] * b.e[0]),
                a.e[0] * b.e[1] - a.e[1] * b.e[0]);
}
inline float dot(const Vec3& a, const Vec3& b) { return a.e[0] * b.e[0] + a.e[1] * b.e[1] + a.e[2] * b.e[2]; }
inline float absDot(const Vec3& a, const Vec3& b) { return fabsf(dot(a, b)); }
inline Vec3 operator+(const Vec3& a, const Vec3& b) { return Vec3(a.e[0] + b.e[0], a.e[1] + b.e[1], a.e[2] + b.e[2]); }
inline Vec3 operator*(float t, const Vec3& v) { return Vec3(t * v.e[0], t * v.e[1], t * v.e[2]); }
inline Vec3 operator/(const Vec3& v, float t) { return Vec3(v.e[0] / t, v.e[1] / t, v.e[2] / t); }
inline Vec3 normalized(const Vec3& v) { return v / v.length(); }

struct Ray {
    Vec3 o, d;
    Vec3 at(float t) const { return o + t * d; }  // core/ray.h:18
};

// ---- Frame (include/frame.h:7-59) -------------------------------------------------------
struct Frame {
    Vec3 s, t, n;
    explicit Frame(const Vec3& a) : n(a) {
        if (fabsf(a.x()) > fabsf(a.y())) {
            float inv = 1.0f / sqrtf(a.x() * a.x() + a.z() * a.z());
            t = Vec3(a.z() * inv, 0.0f, -a.x() * inv);
        } else {
            float inv = 1.0f / sqrtf(a.y() * a.y() + a.z() * a.z());
            t = Vec3(0.0f, a.z() * inv, -a.y() * inv);
        }
        s = cross(t, a);
    }
    Vec3 toWorld(const Vec3& l) const {
        return Vec3(s.x() * l.x() + t.x() * l.y() + n.x() * l.z(), s.y() * l.x() + t.y() * l.y() + n.y() * l.z(),
                    s.z() * l.x() + t.z() * l.y() + n.z() * l.z());
    }
    Vec3 toLocal(const Vec3& w) const {
        return Vec3(s.x() * w.x() + s.y() * w.y() + s.z() * w.z(), t.x() * w.x() + t.y() * w.y() + t.z() * w.z(),
                    n.x() * w.x() + n.y() * w.y() + n.z() * w.z());
    }
};

// ---- PCG32 -------------------------------------------------------------------------------
inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
struct Rng {
    uint64_t state, inc;
    uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((0u - rot) & 31u));
    }
    float uniform() { return (float)((next() >> 8) + 1u) * (1.0f / 16777216.0f); }  // (0, 1]
    static Rng seeded(uint64_t seed, uint64_t sample, uint32_t pixel) {
        Rng r;
        r.inc = ((uint64_t)pixel << 1) | 1ULL;
        r.state = 0;
        r.next();
        r.state += splitmix64(seed ^ splitmix64(sample));
        r.next();
        return r;
    }
};

// ---- scene -------------------------------------------------------------------------------
enum { LAMBERTIAN = 0, MIRROR = 1, GLASS = 2, MICROFACET = 3, METAL = 5 };  // METAL: the CUDA path's metallic Beckmann
enum { TRIANGLE = 0, SPHERE = 1 };

struct Triangle { Vec3 p0, p1, p2, n0, n1, n2; int mat; };
struct Sphere { Vec3 c; float r; int mat; };
struct Material { int type; Vec3 albedo, emit; float ior, alpha; };

// Distribution (include/math/distribution.h:11-65, src/math/distribution.cu:19-55)
struct Distribution {
    std::vector<float> cmf;
    float totalMass = 0.f;
    // DistributionParams::createDistribution, FP32 as in the reference
    static Distribution build(const float* values, int n) {
        Distribution d;
        float total = 0.f;
        for (int i = 0; i < n; i++) total += values[i];
        d.totalMass = total;
        d.cmf.resize(n);
        int last = -1;
        for (int i = 0; i < n; i++) {
            const float mass = values[i] / total;
            if (mass > 0.f) last = i;
            d.cmf[i] = mass;
            if (i > 0) d.cmf[i] += d.cmf[i - 1];
        }
        if (total > 0.f)
            for (int i = last; i < n; i++) d.cmf[i] = 1.f;
        return d;
    }
    float pmf(int i) const {
        if (totalMass == 0.f) return 0.f;
        const float c = cmf[i];
        if (i == 0) return c;
        return c - cmf[i - 1];
    }
    // linear scan; -1 where the reference asserts
    int sample(float* pmfOut, float xi) const {
        for (size_t i = 0; i < cmf.size(); i++)
            if (xi < cmf[i]) { *pmfOut = pmf((int)i); return (int)i; }
        if (xi == 1.f)
            for (size_t i = 0; i < cmf.size(); i++)
                if (cmf[i] == 1.f) { *pmfOut = pmf((int)i); return (int)i; }
        *pmfOut = 0.f;
        return -1;
    }
};

// Distribution2D (distribution.h:80-131, distribution.cu:57-91)
struct Distribution2D {
    Distribution y;
    std::vector<Distribution> x;
    int w = 0, h = 0;
    static Distribution2D build(const float* data, int w, int h) {
        Distribution2D d;
        d.w = w;
        d.h = h;
        std::vector<float> rowSums(h);
        for (int r = 0; r < h; r++) {
            d.x.push_back(Distribution::build(data + (size_t)r * w, w));
            float t = 0.f;
            for (int c = 0; c < w; c++) t += data[(size_t)r * w + c];
            rowSums[r] = t;
        }
        d.y = Distribution::build(rowSums.data(), h);
        return d;
    }
    bool sample(float* pmfOut, float xi1, float xi2, int* sx, int* sy) const {
        float xp, yp;
        const int yy = y.sample(&yp, xi1);
        if (yy < 0) return false;
        const int xx = x[yy].sample(&xp, xi2);
        if (xx < 0) return false;
        *pmfOut = xp * yp;
        *sx = xx;
        *sy = yy;
        return true;
    }
    float pmf(int xi, int yi) const {
        if (y.totalMass == 0.f) return 0.f;
        return x[yi].pmf(xi) * y.pmf(yi);
    }
};

// spherical_coordinates.h:8-47
inline void cartesianToSpherical(const Vec3& c, float* phi, float* theta) {
    *phi = atan2f(c.z(), c.x());
    if (*phi < 0.f) *phi += 2 * M_PI;
    *theta = acosf(fminf(1.f, fmaxf(c.y(), -1.f)));
}
inline Vec3 sphericalToCartesian(float phi, float theta) {
    const float ct = cosf(theta), st = sinf(theta);
    return Vec3(st * cosf(phi), ct, st * sinf(phi));
}
inline Vec3 sphericalToCartesianZ(float phi, float theta) {
    const float ct = cosf(theta), st = sinf(theta);
    return Vec3(st * cosf(phi), st * sinf(phi), ct);
}

// PhiThetaDistribution (distribution.h:149-201) + EnvironmentLight (environment_light.h:26-99)
struct Env {
    bool present = false;
    int w = 0, h = 0;
    std::vector<float> rgba;
    Distribution2D dist;
    float pdfCanonical(float xc, float yc) const {
        const int xs = (int)fminf(floorf(xc * w), w - 1);
        const int ys = (int)fminf(floorf(yc * h), h - 1);
        const float pmf = dist.pmf(xs, ys);
        return pmf * w * h;
    }
    float pdf(const Vec3& wi) const {
        float phi, theta;
        cartesianToSpherical(wi, &phi, &theta);
        const float xc = phi / (M_PI * 2.f);
        const float yc = theta / M_PI;
        return pdfCanonical(xc, yc) / (sinf(theta) * M_PI * M_PI * 2.f);
    }
    Vec3 sample(float* pdfOut, float xi1, float xi2) const {
        float lp;
        int sx = 0, sy = 0;
        if (!dist.sample(&lp, xi1, xi2, &sx, &sy)) { *pdfOut = 0.f; return Vec3(0.f, 1.f, 0.f); }
        const float phiC = (sx + 0.5f) / w;
        const float thetaC = (sy + 0.5f) / h;
        const float phi = phiC * M_PI * 2.f;
        const float theta = thetaC * M_PI;
        const Vec3 wi = sphericalToCartesian(phi, theta);
        *pdfOut = pdf(wi);
        return wi;
    }
    Vec3 emit(const Vec3& wi) const {
        if (!present) return Vec3(0.f);
        float phi, theta;
        cartesianToSpherical(wi, &phi, &theta);
        const int x = (int)floorf(phi / (M_PI * 2.f) * w);
        const int y = (int)floorf(theta / M_PI * h);
        long long off = (long long)(4 * w) * y + 4 * x;
        const long long last = (long long)w * h * 4 - 4;
        off = off < 0 ? 0 : (off > last ? last : off);  // the reference reads past the map at theta = pi
        return Vec3(rgba[off], rgba[off + 1], rgba[off + 2]);
    }
};

struct LightIndex { int type, index; };

// Parity accelerator (not part of the reference): a binary BVH over the scene's triangles
// and spheres, used only where the linear scan is too slow for a parity run (the
// 1.31M-triangle meshes). It returns World::hit's own answer, because that answer is the
// minimum of a total order over the candidates that the per-primitive tests accept
// (src/world.cu:14-38): smaller t first; at equal t a triangle before a sphere, the higher
// triangle index first (triangle.cu:34 accepts t <= tNear, so a later equal one replaces the
// earlier), the lower sphere index first (sphere.cu:16,29 need t < tNear). Each candidate is
// tested with the query's own [tMin, tMax], exactly as the scan tests it. Boxes are built in
// double and padded by 1e-5 of the scene diagonal plus 1e-6 of the coordinate, and a subtree
// is skipped only when its box lies wholly beyond the best t found so far (with the same
// relative slack), so the traversal never skips a candidate that the float tests accept
// within that distance of its primitive.
struct AccelNode {
    double lo[3], hi[3];
    int first, count;  // count > 0: leaf over order[first, first + count); else children first, first + 1
};
struct Accel {
    std::vector<AccelNode> nodes;
    std::vector<int> order;  // >= 0 triangle index, < 0 ~sphere index
};

struct Scene {
    std::vector<Triangle> tris;
    std::vector<Sphere> sphs;
    std::vector<Material> mats;
    std::vector<LightIndex> lights;
    Env env;
    Accel accel;  // empty: World::hit's linear scan
    bool watertight = false;  // triangles take the watertight test (the CUDA path's opt-in)
};

struct HitRecord {
    float t;
    Vec3 point, normal, wo;
    int materialID;
    int primType, primIndex;
    bool isFront() const { return wo.z() >= 0.f; }
};

// Triangle::hit (src/primitives/triangle.cu:7-48)
inline bool triangleHit(const Triangle& tr, const Ray& ray, float tMin, float tMax, HitRecord& rec) {
    const Vec3 e1 = tr.p1 - tr.p0;
    const Vec3 e2 = tr.p2 - tr.p0;
    const Vec3 s1 = cross(ray.d, e2);
    const float divisor = dot(s1, e1);
    if (divisor == 0.f) return false;
    const float inverseDivisor = 1.f / divisor;
    const Vec3 s = ray.o - tr.p0;
    const float b1 = dot(s, s1) * inverseDivisor;
    if (b1 < 0.f || b1 > 1.f) return false;
    const Vec3 s2 = cross(s, e1);
    const float b2 = dot(ray.d, s2) * inverseDivisor;
    if (b2 < 0.f || (b1 + b2) > 1.f) return false;
    const float t = dot(e2, s2) * inverseDivisor;
    if (t < tMin || t > tMax) return false;
    const Vec3 hitPoint = tr.p0 * (1.f - b1 - b2) + (tr.p1 * b1) + (tr.p2 * b2);
    const Vec3 shadingNormal = (1.f - b1 - b2) * tr.n0 + b1 * tr.n1 + b2 * tr.n2;  // triangle.h:51-56
    const Frame frame(shadingNormal);
    rec.t = t;
    rec.point = hitPoint;
    rec.normal = shadingNormal;
    rec.wo = normalized(frame.toLocal(-ray.d));
    rec.materialID = tr.mat;
    return true;
}

// Watertight ray/triangle test (Woop, Benthin and Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1), 2013): the CUDA path's opt-in alternative to Triangle::hit, in the
// same steps and FP32 roundings (this file is built without contraction):
// kz = the largest |d| component (first of x, y, z on ties), kx, ky the next two cyclically,
// swapped when d[kz] < 0; sz = 1 / d[kz], sx = d[kx] sz, sy = d[ky] sz; vertices relative to
// the origin and sheared; edge functions U, V, W, each recomputed in FP64 when exactly zero;
// mixed signs or det = U + V + W = 0 miss; t = T / det in [tMin, tMax]; b1 = V / det,
// b2 = W / det. The hit record is Triangle::hit's from those barycentrics.
inline bool triangleHitWT(const Triangle& tr, const Ray& ray, float tMin, float tMax, HitRecord& rec) {
    const Vec3& d = ray.d;
    const float adx = fabsf(d.x()), ady = fabsf(d.y()), adz = fabsf(d.z());
    const int kz = adx >= ady ? (adx >= adz ? 0 : 2) : (ady >= adz ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    if (d.e[kz] < 0.f) std::swap(kx, ky);
    const float sz = 1.f / d.e[kz];
    const float sx = d.e[kx] * sz, sy = d.e[ky] * sz;
    const Vec3 A = tr.p0 - ray.o, B = tr.p1 - ray.o, C = tr.p2 - ray.o;
    const float ax = A.e[kx] - sx * A.e[kz], ay = A.e[ky] - sy * A.e[kz];
    const float bx = B.e[kx] - sx * B.e[kz], by = B.e[ky] - sy * B.e[kz];
    const float cx = C.e[kx] - sx * C.e[kz], cy = C.e[ky] - sy * C.e[kz];
    float U = cx * by - cy * bx;
    float V = ax * cy - ay * cx;
    float W = bx * ay - by * ax;
    if (U == 0.f || V == 0.f || W == 0.f) {
        U = (float)((double)cx * (double)by - (double)cy * (double)bx);
        V = (float)((double)ax * (double)cy - (double)ay * (double)cx);
        W = (float)((double)bx * (double)ay - (double)by * (double)ax);
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    const float det = U + V + W;
    if (det == 0.f) return false;
    const float T = U * (sz * A.e[kz]) + V * (sz * B.e[kz]) + W * (sz * C.e[kz]);
    const float inv = 1.f / det;
    const float t = T * inv;
    if (!(t >= tMin && t <= tMax)) return false;
    const float b1 = V * inv, b2 = W * inv;
    const Vec3 hitPoint = tr.p0 * (1.f - b1 - b2) + (tr.p1 * b1) + (tr.p2 * b2);
    const Vec3 shadingNormal = (1.f - b1 - b2) * tr.n0 + b1 * tr.n1 + b2 * tr.n2;
    const Frame frame(shadingNormal);
    rec.t = t;
    rec.point = hitPoint;
    rec.normal = shadingNormal;
    rec.wo = normalized(frame.toLocal(-ray.d));
    rec.materialID = tr.mat;
    return true;
}
inline bool triangleTest(const Scene& sc, const Triangle& tr, const Ray& ray, float tMin, float tMax, HitRecord& rec) {
    return sc.watertight ? triangleHitWT(tr, ray, tMin, tMax, rec) : triangleHit(tr, ray, tMin, tMax, rec);
}

// Sphere::hit (src/primitives/sphere.cu:7-43)
inline bool sphereHit(const Sphere& sp, const Ray& ray, float tMin, float tMax, HitRecord& rec) {
    const Vec3 oc = ray.o - sp.c;
    const float a = dot(ray.d, ray.d);
    const float b = dot(oc, ray.d);
    const float c = dot(oc, oc) - sp.r * sp.r;
    const float disc = b * b - a * c;
    if (disc > 0) {
        float temp = (-b - sqrtf(disc)) / a;
        for (int k = 0; k < 2; k++) {
            if (temp < tMax && temp > tMin) {
                const Vec3 point = ray.at(temp);
                const Vec3 normal = normalized((point - sp.c) / sp.r);
                const Frame f(normal);
                rec.t = temp;
                rec.point = point;
                rec.normal = normal;
                rec.wo = normalized(f.toLocal(-ray.d));
                rec.materialID = sp.mat;
                return true;
            }
            temp = (-b + sqrtf(disc)) / a;
        }
    }
    return false;
}

// The linear scan's preference between two accepted candidates (a: t ta, primitive code
// a; b likewise; code >= 0 triangle index, < 0 ~sphere index): true if the scan ends on a
// rather than b. Same class at equal t: the larger code wins (a later triangle, or an
// earlier sphere, whose ~index is larger).
inline bool scanPrefers(float ta, int a, float tb, int b) {
    if (ta != tb) return ta < tb;
    if ((a >= 0) != (b >= 0)) return a >= 0;
    return a > b;
}

void buildAccel(Scene& s) {
    const int nt = (int)s.tris.size(), ns = (int)s.sphs.size(), n = nt + ns;
    s.accel = Accel{};
    if (n == 0) return;
    std::vector<double> lo(3 * (size_t)n), hi(3 * (size_t)n), cen(3 * (size_t)n);
    double slo[3] = {INFINITY, INFINITY, INFINITY}, shi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; i++) {
        for (int a = 0; a < 3; a++) {
            double l, h;
            if (i < nt) {
                const Triangle& t = s.tris[i];
                l = std::min({(double)t.p0.e[a], (double)t.p1.e[a], (double)t.p2.e[a]});
                h = std::max({(double)t.p0.e[a], (double)t.p1.e[a], (double)t.p2.e[a]});
            } else {
                const Sphere& sp = s.sphs[i - nt];
                l = (double)sp.c.e[a] - std::fabs((double)sp.r);
                h = (double)sp.c.e[a] + std::fabs((double)sp.r);
            }
            lo[3 * (size_t)i + a] = l;
            hi[3 * (size_t)i + a] = h;
            cen[3 * (size_t)i + a] = 0.5 * (l + h);
            slo[a] = std::min(slo[a], l);
            shi[a] = std::max(shi[a], h);
        }
    }
    const double diag = std::sqrt((shi[0] - slo[0]) * (shi[0] - slo[0]) + (shi[1] - slo[1]) * (shi[1] - slo[1]) +
                                  (shi[2] - slo[2]) * (shi[2] - slo[2]));
    for (size_t k = 0; k < 3 * (size_t)n; k++) {
        const double pad = 1e-5 * diag + 1e-6 * std::max(std::fabs(lo[k]), std::fabs(hi[k])) + 1e-30;
        lo[k] -= pad;
        hi[k] += pad;
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    Accel& A = s.accel;
    A.nodes.reserve(2 * (size_t)n / 3 + 2);
    struct Job { int node, first, count; };
    std::vector<Job> jobs;
    A.nodes.push_back(AccelNode{});
    jobs.push_back({0, 0, n});
    while (!jobs.empty()) {
        const Job j = jobs.back();
        jobs.pop_back();
        AccelNode nd;
        double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int a = 0; a < 3; a++) { nd.lo[a] = INFINITY; nd.hi[a] = -INFINITY; }
        for (int k = j.first; k < j.first + j.count; k++) {
            const size_t p = (size_t)idx[k];
            for (int a = 0; a < 3; a++) {
                nd.lo[a] = std::min(nd.lo[a], lo[3 * p + a]);
                nd.hi[a] = std::max(nd.hi[a], hi[3 * p + a]);
                clo[a] = std::min(clo[a], cen[3 * p + a]);
                chi[a] = std::max(chi[a], cen[3 * p + a]);
            }
        }
        if (j.count <= 4) {
            nd.first = j.first;
            nd.count = j.count;
            A.nodes[j.node] = nd;
            continue;
        }
        int axis = 0;
        for (int a = 1; a < 3; a++) if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
        const int half = j.count / 2;
        std::nth_element(idx.begin() + j.first, idx.begin() + j.first + half, idx.begin() + j.first + j.count,
                         [&](int x, int y) { return cen[3 * (size_t)x + axis] < cen[3 * (size_t)y + axis]; });
        nd.first = (int)A.nodes.size();
        nd.count = 0;
        A.nodes[j.node] = nd;
        A.nodes.push_back(AccelNode{});
        A.nodes.push_back(AccelNode{});
        jobs.push_back({nd.first, j.first, half});
        jobs.push_back({nd.first + 1, j.first + half, j.count - half});
    }
    A.order.resize(n);
    for (int k = 0; k < n; k++) A.order[k] = idx[k] < nt ? idx[k] : ~(idx[k] - nt);
}

// Ray against a padded box over the parameter range [t0, t1] (double); entry parameter out.
inline bool accelSlab(const AccelNode& nd, const double o[3], const double d[3], double t0, double t1, double& entry) {
    for (int a = 0; a < 3; a++) {
        if (d[a] == 0.0) {
            if (o[a] < nd.lo[a] || o[a] > nd.hi[a]) return false;
            continue;
        }
        double ta = (nd.lo[a] - o[a]) / d[a], tb = (nd.hi[a] - o[a]) / d[a];
        if (ta > tb) std::swap(ta, tb);
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
        if (t0 > t1) return false;
    }
    entry = t0;
    return true;
}

// World::hit through the accelerator: the same result as the scan (see scanPrefers). With
// `any`, returns at the first accepted candidate (occlusion queries need only the flag).
bool accelHit(const Scene& sc, const Ray& ray, float tMin, float tMax, HitRecord& rec, bool any) {
    const Accel& A = sc.accel;
    const double o[3] = {ray.o.e[0], ray.o.e[1], ray.o.e[2]}, d[3] = {ray.d.e[0], ray.d.e[1], ray.d.e[2]};
    const double dl = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (!(dl > 0.0)) return false;
    // slack in ray-parameter units: the boxes' padding is already in space units
    const auto upper = [&](float t) { return (double)t * (1.0 + 1e-5) + 1e-9 / dl; };
    const double lower = (double)tMin - 1e-3 * (std::fabs((double)tMin) + 1.0 / dl);
    bool found = false;
    float bestT = tMax;
    int bestCode = 0;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const AccelNode& nd = A.nodes[stack[--sp]];
        double e;
        // re-tested at pop time: the best hit may have moved closer since the push
        if (!accelSlab(nd, o, d, lower, upper(bestT), e)) continue;
        if (nd.count > 0) {
            for (int k = nd.first; k < nd.first + nd.count; k++) {
                const int code = A.order[k];
                HitRecord tmp;
                const bool h = code >= 0 ? triangleTest(sc, sc.tris[code], ray, tMin, tMax, tmp)
                                         : sphereHit(sc.sphs[~code], ray, tMin, tMax, tmp);
                if (!h) continue;
                if (any) return true;
                if (!found || scanPrefers(tmp.t, code, bestT, bestCode)) {
                    found = true;
                    bestT = tmp.t;
                    bestCode = code;
                    rec = tmp;
                    rec.primType = code >= 0 ? TRIANGLE : SPHERE;
                    rec.primIndex = code >= 0 ? code : ~code;
                }
            }
            continue;
        }
        const double lim = upper(bestT);
        double ea, eb;
        const bool ha = accelSlab(A.nodes[nd.first], o, d, lower, lim, ea);
        const bool hb = accelSlab(A.nodes[nd.first + 1], o, d, lower, lim, eb);
        if (sp + 2 > 128) std::abort();  // a median-split tree is far shallower than this
        if (ha && hb) {  // nearer child on top
            stack[sp++] = ea <= eb ? nd.first + 1 : nd.first;
            stack[sp++] = ea <= eb ? nd.first : nd.first + 1;
        } else if (ha) {
            stack[sp++] = nd.first;
        } else if (hb) {
            stack[sp++] = nd.first + 1;
        }
    }
    return found;
}

// World::hit (src/world.cu:5-41): all triangles, then all spheres. Scenes with an accelerator
// answer through it (same result; `any` lets an occlusion query stop at its first hit).
inline bool worldHit(const Scene& sc, const Ray& ray, float tMin, float tMax, HitRecord& rec, bool any = false) {
    if (!sc.accel.nodes.empty()) return accelHit(sc, ray, tMin, tMax, rec, any);
    bool isHit = false;
    double tNear = tMax;
    const int nt = (int)sc.tris.size();
    for (int i = 0; i < nt; i++) {
        HitRecord tmp;
        if (triangleTest(sc, sc.tris[i], ray, tMin, (float)tNear, tmp)) {
            isHit = true;
            tNear = tmp.t;
            rec = tmp;
            rec.primType = TRIANGLE;
            rec.primIndex = i;
        }
    }
    const int ns = (int)sc.sphs.size();
    for (int i = 0; i < ns; i++) {
        HitRecord tmp;
        if (sphereHit(sc.sphs[i], ray, tMin, (float)tNear, tmp)) {
            isHit = true;
            tNear = tmp.t;
            rec = tmp;
            rec.primType = SPHERE;
            rec.primIndex = i;
        }
    }
    return isHit;
}

// ---- BSDFs ---------------------------------------------------------------------------------
struct BSDFSample { Vec3 wiLocal; float pdf; Vec3 f; bool isDelta; };

// core/sample.h
inline Vec3 uniformHemisphere(float xi1, float xi2) {
    const float z = xi1;
    const float r = sqrtf(fmaxf(0.f, 1.f - z * z));
    const float phi = 2 * M_PI * xi2;
    return Vec3(r * cosf(phi), r * sinf(phi), z);
}
inline float uniformHemispherePDF(const Vec3& v) {
    if (v.z() < 0.f) return 0.f;
    return 1.f / (2.f * M_PI);
}
inline Vec3 uniformSphere(float xi1, float xi2) {
    const float z = xi1 * 2.f - 1.f;
    const float r = sqrtf(fmaxf(0.f, 1.f - z * z));
    const float phi = 2 * M_PI * xi2;
    return Vec3(r * cosf(phi), r * sinf(phi), z);
}

// lambertian.h:43-76
inline Vec3 lambertF(const Material& m, const Vec3& wo, const Vec3& wi) {
    if (wo.z() < 0.f || wi.z() < 0.f) return Vec3(0.f);
    return m.albedo / M_PI;
}
inline BSDFSample lambertSample(const Material& m, const Vec3& wo, float xi1, float xi2) {
    const Vec3 wi = uniformHemisphere(xi1, xi2);
    return BSDFSample{wi, uniformHemispherePDF(wi), lambertF(m, wo, wi), false};
}
// mirror.h:47-55
inline BSDFSample mirrorSample(const Vec3& wo) {
    const Vec3 wi = wo.reflect(Vec3(0.f, 0.f, 1.f));
    return BSDFSample{wi, 1.f, Vec3(fmaxf(0.f, 1.f / wi.z())), true};
}
// optics/snell.h:10-66
inline float transmittedSinTheta(float cosI, float etaI, float etaT) {
    return (etaI / etaT) * sqrtf(fmaxf(0.f, 1.f - cosI * cosI));
}
inline bool snellRefract(const Vec3& inc, Vec3* out, Vec3 normal, float etaI, float etaT) {
    if (dot(inc, normal) < 0.f) {
        normal = normal * -1.f;
        std::swap(etaI, etaT);
    }
    const Vec3 wIPerp = inc - (normal * inc.dotv(normal));
    const Vec3 wTPerp = -wIPerp * (etaI / etaT);
    const float l2 = wTPerp.length() * wTPerp.length();
    const float wTParLen = sqrtf(fmaxf(0.f, 1.f - l2));
    const Vec3 wTPar = normal * -wTParLen;
    const float cosI = absDot(inc, normal);
    const float sin2I = fmaxf(0.f, 1.f - (cosI * cosI));
    const float eta2 = (etaI / etaT) * (etaI / etaT);
    const float sin2T = eta2 * sin2I;
    *out = normalized(wTPar + wTPerp);
    return !(sin2T >= 1.f);
}
// optics/fresnel.h:14-42
inline float dielectricReflectance(float cosI, float etaI, float etaT) {
    const float sinT = transmittedSinTheta(cosI, etaI, etaT);
    if (sinT > 1.f) return 1.f;
    const float cosT = sqrtf(fmaxf(0.f, 1.f - sinT * sinT));
    const float rPar = (etaT * cosI - etaI * cosT) / (etaT * cosI + etaI * cosT);
    const float rPerp = (etaI * cosI - etaT * cosT) / (etaI * cosI + etaT * cosT);
    return 0.5f * (rPar * rPar + rPerp * rPerp);
}
// glass.h:44-109
inline BSDFSample glassSample(const Material& m, const Vec3& wo, float xi1) {
    float etaI = 1.f, etaT = m.ior;
    if (wo.z() < 0.f) std::swap(etaI, etaT);
    Vec3 wi(0.f);
    snellRefract(wo, &wi, Vec3(0.f, 0.f, 1.f), etaI, etaT);
    const float F = dielectricReflectance(fabsf(wo.z()), etaI, etaT);
    if (xi1 < F) {
        wi = wo.reflect(Vec3(0.f, 0.f, 1.f));
        const float c = fabsf(wi.z());
        return BSDFSample{wi, F, c == 0.f ? Vec3(0.f) : Vec3(F / c), true};
    }
    const float T = 1.f - F;
    const float c = fabsf(wi.z());
    const Vec3 thr = c == 0.f ? Vec3(0.f) : Vec3(T / c);
    const float corr = (etaI / etaT) * (etaI / etaT);
    return BSDFSample{wi, T, thr * corr, true};
}
// microfacet.h:19-164
struct Beckmann {
    float alpha;
    float sampleAlpha(float absCos) const { return (1.2f - 0.2f * sqrtf(absCos)) * alpha; }
    float D(const Vec3& wi, const Vec3& wh) const {
        const float a = sampleAlpha(fabsf(wi.z()));
        const float a2 = a * a;
        const float cos2 = wh.z() * wh.z();
        const float cos4 = cos2 * cos2;
        const float tan2 = (1.f - cos2) / cos2;
        if (std::isinf(tan2)) return 0.f;
        const float num = expf(-tan2 / a2);
        const float den = M_PI * a2 * cos4;  // the double product is stored as float (microfacet.h:47-48)
        return num / den;
    }
    Vec3 sampleWh(const Vec3& wo, float xi1, float xi2) const {
        const float phi = xi1 * M_PI * 2.f;
        const float a = sampleAlpha(fabsf(wo.z()));
        const float a2 = a * a;
        const float st = (-a2 * logf(1 - xi2));
        const float theta = atanf(sqrtf(st));
        return sphericalToCartesianZ(phi, theta);
    }
    float pdf(const Vec3& wi, const Vec3& wh) const { return D(wi, wh) * fabsf(wh.z()); }
    float G1(const Vec3& v) const {
        const float sinT = sqrtf(fmaxf(0.f, 1.f - v.z() * v.z()));
        const float a = 1.f / (alpha * fabsf(sinT / v.z()));
        if (a >= 1.6f) return 1.f;
        return (3.535f * a + 2.181f * a * a) / (1.f + 2.276f * a + 2.577f * a * a);
    }
    static float sign(float x) { return x < 0.f ? -1.f : 1.f; }
    float G(const Vec3& wi, const Vec3& wo, const Vec3& wh) const {
        if (sign(dot(wo, wh)) != sign(wo.z())) return 0.f;
        if (sign(dot(wi, wh)) != sign(wi.z())) return 0.f;
        return G1(wi) * G1(wo);
    }
};
inline Vec3 microfacetF(const Material& m, const Vec3& wo, const Vec3& wi) {
    const Beckmann d{m.alpha};
    if (wo.z() < 0.f || wi.z() < 0.f) return Vec3(0.f);
    const float cO = fabsf(wo.z()), cI = fabsf(wi.z());
    const Vec3 wh = normalized(wo + wi);
    if (cO == 0.f || cI == 0.f) return Vec3(0.f);
    if (wh.isZero()) return Vec3(0.f);
    const float cInc = fminf(1.f, fmaxf(dot(wi, wh), 0.f));
    const float F = dielectricReflectance(cInc, 1.f, 1.5f);
    const float Dv = d.D(wi, wh);
    const float Gv = d.G(wi, wo, wh);
    return Vec3(1.f) * Dv * Gv * F / (4 * cI * cO);
}
// METAL (the CUDA path's metallic Beckmann, no counterpart in the reference): the same D and
// G with a Schlick Fresnel per channel, F = F0 + (1 - F0)(1 - c)^5 at c = wi . wh, F0 = albedo.
inline Vec3 metalF(const Material& m, const Vec3& wo, const Vec3& wi) {
    const Beckmann d{m.alpha};
    if (wo.z() < 0.f || wi.z() < 0.f) return Vec3(0.f);
    const float cO = fabsf(wo.z()), cI = fabsf(wi.z());
    const Vec3 wh = normalized(wo + wi);
    if (cO == 0.f || cI == 0.f) return Vec3(0.f);
    if (wh.isZero()) return Vec3(0.f);
    const float cInc = fminf(1.f, fmaxf(dot(wi, wh), 0.f));
    const float q = 1.f - cInc, q2 = q * q, q5 = q2 * q2 * q;
    const float s = d.D(wi, wh) * d.G(wi, wo, wh) / (4.f * cI * cO);
    return Vec3((m.albedo.x() + (1.f - m.albedo.x()) * q5) * s, (m.albedo.y() + (1.f - m.albedo.y()) * q5) * s,
                (m.albedo.z() + (1.f - m.albedo.z()) * q5) * s);
}
inline float microfacetPdf(const Material& m, const Vec3& wo, const Vec3& wi) {
    const Beckmann d{m.alpha};
    if (wo.z() < 0.f || wi.z() < 0.f) return 0.f;
    const Vec3 wh = normalized(wo + wi);
    return d.pdf(wi, wh) / (4.f * absDot(wo, wh));
}
inline BSDFSample microfacetSample(const Material& m, const Vec3& wo, float xi1, float xi2) {
    const Beckmann d{m.alpha};
    const Vec3 wh = d.sampleWh(wo, xi1, xi2);
    const Vec3 wi = wo.reflect(wh);
    const Vec3 f = m.type == METAL ? metalF(m, wo, wi) : microfacetF(m, wo, wi);
    return BSDFSample{wi, d.pdf(wo, wh) / (4.f * absDot(wi, wh)), f, false};
}

// bsdf.h:19-115
inline Vec3 bsdfF(const Material& m, const Vec3& wo, const Vec3& wi) {
    switch (m.type) {
        case LAMBERTIAN: return lambertF(m, wo, wi);
        case MICROFACET: return microfacetF(m, wo, wi);
        case METAL: return metalF(m, wo, wi);
        default: return Vec3(0.f);
    }
}
inline float bsdfPdf(const Material& m, const Vec3& wo, const Vec3& wi) {
    switch (m.type) {
        case LAMBERTIAN: return uniformHemispherePDF(wi);
        case MICROFACET:
        case METAL: return microfacetPdf(m, wo, wi);
        default: return 0.f;
    }
}
inline BSDFSample bsdfSample(const Material& m, const Vec3& wo, Rng& rng) {
    switch (m.type) {
        case LAMBERTIAN: { const float a = rng.uniform(); const float b = rng.uniform(); return lambertSample(m, wo, a, b); }
        case MIRROR: return mirrorSample(wo);
        case GLASS: return glassSample(m, wo, rng.uniform());
        default: { const float a = rng.uniform(); const float b = rng.uniform(); return microfacetSample(m, wo, a, b); }
    }
}
// World::getEmit(materialID, record) (world.h:156-174): front-facing Lambertian only
inline Vec3 getEmit(const Scene& sc, const HitRecord& r) {
    const Material& m = sc.mats[r.materialID];
    if (m.type == LAMBERTIAN && r.isFront()) return m.emit;
    return Vec3(0.f);
}

// ---- lights (include/lights/sampler.h:20-183) -------------------------------------------
struct LightSample { Vec3 wi, normal; float distance, pdf; Vec3 emitted; };

inline float triangleArea(const Triangle& t) {
    const Vec3 c = cross(t.p1 - t.p0, t.p2 - t.p0);
    return fabsf(c.length() / 2.f);
}
inline float sphereArea(const Sphere& s) { return 4.f * M_PI * s.r * s.r; }

inline LightSample sampleDirectLights(const Scene& sc, const Vec3& hitPoint, float s0, float s1, float s2) {
    const int nl = (int)sc.lights.size();
    int choiceSize = nl + (sc.env.present ? 1 : 0);
    const int lightChoice = (int)fminf(choiceSize - 1, (int)floorf(s0 * choiceSize));
    const float choicePDF = 1.f / choiceSize;
    LightSample ls;
    if (lightChoice < nl) {
        const LightIndex li = sc.lights[lightChoice];
        Vec3 point, normal;
        float areaPdf;
        int matId;
        if (li.type == TRIANGLE) {
            const Triangle& t = sc.tris[li.index];
            const float a = 1 - sqrtf(s1);
            const float b = sqrtf(s1) * (1 - s2);
            const float c = 1 - a - b;
            point = t.p0 * a + t.p1 * b + t.p2 * c;
            normal = normalized(cross(t.p1 - t.p0, t.p2 - t.p0));
            areaPdf = 1.f / triangleArea(t);
            matId = t.mat;
        } else {
            const Sphere& s = sc.sphs[li.index];
            const Vec3 local = uniformSphere(s1, s2);
            point = local * s.r + s.c;
            normal = local;
            areaPdf = 1.f / sphereArea(s);
            matId = s.mat;
        }
        const Vec3 direction = point - hitPoint;
        const float distance = direction.length();
        // SurfaceSample::solidAnglePDF (surface_sample.h:13-24)
        const Vec3 lightWo = -normalized(direction);
        const float d2 = distance * distance;
        const float proj = fabsf(dot(normal, lightWo));
        const float sa = proj == 0.f ? 0.f : areaPdf * d2 / proj;
        ls.wi = normalized(direction);
        ls.normal = normal;
        ls.distance = distance;
        ls.pdf = sa * choicePDF;
        const Material& m = sc.mats[matId];
        ls.emitted = m.type == LAMBERTIAN ? m.emit : Vec3(0.f);
    } else {
        float pdf;
        const Vec3 w = sc.env.sample(&pdf, s1, s2);
        const Vec3 wi = normalized(w);
        ls.wi = wi;
        ls.normal = -wi;
        ls.distance = 1e16;
        ls.pdf = pdf * choicePDF;
        ls.emitted = sc.env.emit(w);
    }
    return ls;
}
inline float pdfSceneLights(const Scene& sc, const Vec3& ref, const HitRecord& lr) {
    const float areaPdf = lr.primType == SPHERE ? 1.f / sphereArea(sc.sphs[lr.primIndex])
                                                : 1.f / triangleArea(sc.tris[lr.primIndex]);
    // Measure::areaToSolidAngle (core/measure.h:8-23)
    const Vec3 sd = ref - lr.point;
    const Vec3 swo = normalized(sd);
    const float dist = sd.length();
    const float d2 = dist * dist;
    const float proj = fmaxf(0.f, dot(lr.normal, swo));
    const float sa = areaPdf * d2 / proj;
    int choiceCount = (int)sc.lights.size() + (sc.env.present ? 1 : 0);
    return sa / choiceCount;
}
inline float pdfEnvironmentLight(const Scene& sc, const Vec3& wi) {
    if (!sc.env.present) return 0.f;
    return sc.env.pdf(wi) * (1.f / (sc.lights.size() + 1));
}
inline float balance(float p1, float p2) { return (1 * p1) / (1 * p1 + 1 * p2); }

// ---- camera (include/core/camera.h:40-61, src/transform.cu:7-33) ------------------------
struct Camera {
    float m[3][4];
    float vfov;
    int rx, ry;
    void init(const float* o, const float* t, const float* u, float fov, bool flip, int w, int h) {
        const Vec3 src(o[0], o[1], o[2]), tgt(t[0], t[1], t[2]), up(u[0], u[1], u[2]);
        const Vec3 dir = normalized(src - tgt);
        const Vec3 xa = normalized(cross(normalized(up), dir));
        const Vec3 ya = normalized(cross(dir, xa));
        const float sign = flip ? -1.f : 1.f;
        const float mm[3][4] = {{sign * xa.x(), ya.x(), dir.x(), src.x()},
                                {sign * xa.y(), ya.y(), dir.y(), src.y()},
                                {sign * xa.z(), ya.z(), dir.z(), src.z()}};
        std::memcpy(m, mm, sizeof(m));
        vfov = fov;
        rx = w;
        ry = h;
    }
    Ray generate(int row, int col, float s0, float s1) const {
        const float top = tanf(vfov / 2.f);
        const float height = top * 2.f;
        const float aspect = 1.f * rx / ry;
        const float width = height * aspect;
        const float right = width / 2.f;
        const float xc = (col + s0) / rx;
        const float yc = (row + s1) / ry;
        const float y = yc * height - top;
        const float x = xc * width - right;
        const Vec3 d = normalized(Vec3(x, y, -1));
        Ray r;
        r.o = Vec3(m[0][3], m[1][3], m[2][3]);
        r.d = Vec3(m[0][0] * d.x() + m[0][1] * d.y() + m[0][2] * d.z(), m[1][0] * d.x() + m[1][1] * d.y() + m[1][2] * d.z(),
                   m[2][0] * d.x() + m[2][1] * d.y() + m[2][2] * d.z());
        return r;
    }
};

// ---- integrator (src/renderers/path_tracer.cu:38-233) -----------------------------------
// trace_once = 0: the reference's two traces per bounce (BSDF-direct at tMin 1e-4, :51, and
// continuation at 1e-3, :177). trace_once = 1: the CUDA path's rules: one trace at 1e-4 serves
// both unless its hit lies closer than 1e-3, when the direction is traced again from 1e-3 for
// the continuation (the same hits as the two traces), and paths that cannot add anything are
// dropped instead of traced.
// Canonical queries: camera + continuation closest hits, and shadow rays that can contribute.
// `duplicate` counts the reference's second trace of each BSDF direction (compat mode only).
struct Counters { uint64_t queries = 0, shadow = 0, duplicate = 0; };

// The BSDF sampler's own density of a direction: Microfacet::sample draws with alpha(wo)
// (microfacet.h:148-158) while Microfacet::pdf evaluates D with alpha(wi) (:124-134).
inline float bsdfSamplingPdf(const Material& m, const Vec3& wo, const Vec3& wi) {
    if (m.type != MICROFACET && m.type != METAL) return bsdfPdf(m, wo, wi);
    if (wo.z() < 0.f || wi.z() < 0.f) return 0.f;
    const Beckmann d{m.alpha};
    const Vec3 wh = normalized(wo + wi);
    return d.pdf(wo, wh) / (4.f * absDot(wo, wh));
}

// consistent: the light sample's MIS weight uses the BSDF's sampling density (an unbiased
// combination) instead of the reference's Microfacet::pdf.
Vec3 directLight(const Scene& sc, const HitRecord& rec, const BSDFSample& bs, Rng& rng, Counters& cnt,
                 int traceOnce, bool consistent = false) {
    // directSampleLights (:83-126)
    if (bs.isDelta) return Vec3(0.f);
    if (traceOnce && sc.lights.empty() && !sc.env.present) return Vec3(0.f);  // no emitter to sample
    const float x1 = rng.uniform(), x2 = rng.uniform(), x3 = rng.uniform();  // world.h:56-58
    const LightSample ls = sampleDirectLights(sc, rec.point, x1, x2, x3);
    if (dot(ls.normal, ls.wi) >= 0.f) return Vec3(0.f);
    if (traceOnce && !(ls.pdf > 0.f)) return Vec3(0.f);  // zero-density sample (0/0 in the reference)
    // The contribution is evaluated before the shadow query (same value as the reference's
    // order, :115-124); a shadow ray that cannot contribute is neither traced nor counted.
    const Vec3 wiLocal = Frame(rec.normal).toLocal(ls.wi);
    const Material& m = sc.mats[rec.materialID];
    const float bsdfPDF = consistent ? bsdfSamplingPdf(m, rec.wo, wiLocal) : bsdfPdf(m, rec.wo, wiLocal);
    const float lw = balance(ls.pdf, bsdfPDF);
    const Vec3 c = Vec3(1.f) * ls.emitted * lw * bsdfF(m, rec.wo, wiLocal) * fabsf(dot(rec.normal, ls.wi)) / ls.pdf;
    if (c.isZero()) return c;
    Ray shadow{rec.point, ls.wi};
    HitRecord occ;
    cnt.shadow++;
    if (worldHit(sc, shadow, 1e-4, ls.distance - 2e-4, occ, true)) return Vec3(0.f);
    return c;
}

Vec3 bsdfDirectFromHit(const Scene& sc, const HitRecord& rec, const BSDFSample& bs, bool hit, const HitRecord& br,
                       const Vec3& dir) {
    // directSampleBSDF (:38-81) given the traced hit
    if (bs.f.isZero()) return Vec3(0.f);
    if (hit) {
        const Vec3 emit = getEmit(sc, br);
        if (emit.isZero()) return Vec3(0.f);
        const float lightPDF = pdfSceneLights(sc, rec.point, br);
        const float w = bs.isDelta ? 1.f : balance(bs.pdf, lightPDF);
        return emit * w * bs.f * fabsf(bs.wiLocal.z()) / bs.pdf;
    }
    const float lightPDF = pdfEnvironmentLight(sc, dir);
    const float w = bs.isDelta ? 1.f : balance(bs.pdf, lightPDF);
    return sc.env.emit(dir) * w * bs.f * fabsf(bs.wiLocal.z()) / bs.pdf;
}

Vec3 LiNEE(const Scene& sc, const Ray& ray, int maxDepth, Rng& rng, int traceOnce, Counters& cnt,
           bool consistent = false) {
    if (maxDepth == 0) return Vec3(0.f);
    Vec3 beta(1.f), result(0.f);
    HitRecord rec;
    cnt.queries++;
    bool hit = worldHit(sc, ray, 0.f, FLT_MAX, rec);
    if (hit) {
        const Vec3 emit = getEmit(sc, rec);
        if (!emit.isZero()) result += emit * beta;
    } else {
        return sc.env.emit(ray.d);
    }
    for (int path = 1; path < maxDepth; path++) {
        const Frame fr(rec.normal);
        const BSDFSample bs = bsdfSample(sc.mats[rec.materialID], rec.wo, rng);
        Vec3 direct = directLight(sc, rec, bs, rng, cnt, traceOnce, consistent);
        const Vec3 bounceDir = fr.toWorld(bs.wiLocal);
        const Ray bounce{rec.point, bounceDir};
        HitRecord next;
        bool nhit;
        if (traceOnce) {
            // the CUDA path ends a path whose throughput becomes zero or non-finite instead
            // of tracing it further (nothing it could add is non-zero)
            const Vec3 nb = beta * (bs.f * fabsf(bs.wiLocal.z()) / bs.pdf);
            if (!(bs.pdf > 0.f) || nb.isZero() || !std::isfinite(nb.x() + nb.y() + nb.z())) {
                result += beta * direct;
                return result;
            }
            cnt.queries++;
            HitRecord dh;
            const bool dhit = worldHit(sc, bounce, 1e-4, FLT_MAX, dh);
            direct += bsdfDirectFromHit(sc, rec, bs, dhit, dh, bounceDir);
            // a triangle at t = tMin is inside the continuation's range, a sphere is not
            // (triangle.cu:34 accepts t >= tMin, sphere.cu:16,29 need t > tMin)
            const bool closer = dh.t < 1e-3f || (dh.primType == SPHERE && dh.t == 1e-3f);
            if (dhit && closer && path + 1 < maxDepth) {
                cnt.duplicate++;  // the continuation's own trace: not a canonical query
                nhit = worldHit(sc, bounce, 1e-3, FLT_MAX, next);
            } else {
                nhit = dhit;
                next = dh;
            }
        } else {
            if (!bs.f.isZero()) {
                HitRecord br;
                cnt.duplicate++;  // same direction traced again below: not a canonical query
                const bool bh = worldHit(sc, bounce, 1e-4, FLT_MAX, br);
                direct += bsdfDirectFromHit(sc, rec, bs, bh, br, bounceDir);
            }
            // a continuation whose throughput is already zero is wasted work, not canonical
            if ((beta * (bs.f * fabsf(bs.wiLocal.z()) / bs.pdf)).isZero()) cnt.duplicate++;
            else cnt.queries++;
            nhit = worldHit(sc, bounce, 1e-3, FLT_MAX, next);
        }
        result += beta * direct;
        beta *= bs.f * fabsf(bs.wiLocal.z()) / bs.pdf;
        if (!nhit) return result;
        rec = next;
    }
    return result;
}

Vec3 LiNaive(const Scene& sc, const Ray& ray, int maxDepth, Rng& rng, Counters& cnt) {
    if (maxDepth == 0) return Vec3(0.f);
    Vec3 beta(1.f), result(0.f);
    HitRecord rec;
    cnt.queries++;
    bool hit = worldHit(sc, ray, 0.f, FLT_MAX, rec);
    if (hit) {
        const Vec3 emit = getEmit(sc, rec);
        if (!emit.isZero()) result += emit * beta;
    } else {
        return sc.env.emit(ray.d);
    }
    for (int path = 1; path < maxDepth; path++) {
        const Frame fr(rec.normal);
        const BSDFSample bs = bsdfSample(sc.mats[rec.materialID], rec.wo, rng);
        beta *= Vec3(1.f) * bs.f * fabsf(bs.wiLocal.z()) / bs.pdf;
        const Vec3 bd = fr.toWorld(bs.wiLocal);
        const Ray bounce{rec.point, bd};
        cnt.queries++;
        hit = worldHit(sc, bounce, 1e-3, FLT_MAX, rec);
        if (hit) {
            const Vec3 emit = getEmit(sc, rec);
            if (!emit.isZero()) result += emit * beta;
        } else {
            return result + sc.env.emit(bounce.d) * beta;
        }
    }
    return result;
}

}  // namespace oracle

using namespace oracle;

extern "C" {

Scene* oracle_scene_create(int ntri, const float* tri_p, const float* tri_n, const int* tri_mat, int nsph,
                           const float* sph, const int* sph_mat, int nmat, const int* mtype, const float* albedo,
                           const float* emit, const float* ior, const float* alpha, int env_w, int env_h,
                           const float* env_rgba) {
    Scene* s = new Scene();
    for (int i = 0; i < ntri; i++) {
        const float* p = tri_p + (size_t)i * 9;
        const float* n = tri_n + (size_t)i * 9;
        s->tris.push_back(Triangle{Vec3(p[0], p[1], p[2]), Vec3(p[3], p[4], p[5]), Vec3(p[6], p[7], p[8]),
                                   Vec3(n[0], n[1], n[2]), Vec3(n[3], n[4], n[5]), Vec3(n[6], n[7], n[8]), tri_mat[i]});
    }
    for (int i = 0; i < nsph; i++) {
        const float* q = sph + (size_t)i * 4;
        s->sphs.push_back(Sphere{Vec3(q[0], q[1], q[2]), q[3], sph_mat[i]});
    }
    for (int i = 0; i < nmat; i++)
        s->mats.push_back(Material{mtype[i], Vec3(albedo[3 * i], albedo[3 * i + 1], albedo[3 * i + 2]),
                                   Vec3(emit[3 * i], emit[3 * i + 1], emit[3 * i + 2]), ior[i], alpha[i]});
    // emitter list (src/scene_data.cu:92-115)
    auto emitter = [&](int mat) { const Material& m = s->mats[mat]; return m.type == LAMBERTIAN && !m.emit.isZero(); };
    for (int i = 0; i < ntri; i++) if (emitter(s->tris[i].mat)) s->lights.push_back({TRIANGLE, i});
    for (int i = 0; i < nsph; i++) if (emitter(s->sphs[i].mat)) s->lights.push_back({SPHERE, i});
    if (env_rgba && env_w > 0 && env_h > 0) {
        s->env.present = true;
        s->env.w = env_w;
        s->env.h = env_h;
        s->env.rgba.assign(env_rgba, env_rgba + (size_t)env_w * env_h * 4);
        std::vector<float> inten((size_t)env_w * env_h);
        for (size_t i = 0; i < inten.size(); i++)  // environment_light.cu:44-47
            inten[i] = env_rgba[i * 4 + 0] + env_rgba[i * 4 + 1] + env_rgba[i * 4 + 2];
        s->env.dist = Distribution2D::build(inten.data(), env_w, env_h);
    }
    return s;
}

void oracle_scene_destroy(Scene* s) { delete s; }
// Build the parity accelerator: later queries on the scene give the linear scan's results
// through a BVH (buildAccel).
void oracle_scene_accel(Scene* s) { buildAccel(*s); }
// Triangles take the watertight test (1) or Triangle::hit's (0, the default).
void oracle_scene_watertight(Scene* s, int on) { s->watertight = on != 0; }
int oracle_num_lights(const Scene* s) { return (int)s->lights.size(); }

// Closest hit of n rays by the reference's linear scan. prim_type -1 on a miss.
void oracle_trace(const Scene* s, const float* o, const float* d, const float* tmin, const float* tmax, int n,
                  int* prim_type, int* prim_id, int* mat_id, float* t, int threads) {
    parallel_for(n, threads, 64, [&](int i, int) {
        Ray r{Vec3(o[3 * i], o[3 * i + 1], o[3 * i + 2]), Vec3(d[3 * i], d[3 * i + 1], d[3 * i + 2])};
        HitRecord rec;
        if (worldHit(*s, r, tmin[i], tmax[i], rec)) {
            prim_type[i] = rec.primType;
            prim_id[i] = rec.primIndex;
            mat_id[i] = rec.materialID;
            t[i] = rec.t;
        } else {
            prim_type[i] = -1;
            prim_id[i] = -1;
            mat_id[i] = -1;
            t[i] = 0.f;
        }
    });
}

// Per-pixel radiance over `spp` samples for the listed pixels (pixel = row * width + col).
// mean/var: 3 doubles per listed pixel, the FP64 sample mean and the variance of that mean.
// Returns query counts through `counts`: canonical closest-hit, canonical shadow, and the
// non-canonical extra traces of the reference's convention.
void oracle_render(const Scene* s, const float* cam, int width, int height, const int* pixels, int npix, int spp,
                   int max_depth, int nee, uint64_t seed, uint64_t sample_base, int trace_once, double* mean,
                   double* var, uint64_t* counts, int threads, int consistent_mis) {
    Camera c;
    c.init(cam, cam + 3, cam + 6, cam[9], cam[10] != 0.f, width, height);
    std::atomic<uint64_t> q{0}, sh{0}, dup{0};
    parallel_for(npix, threads, 4, [&](int k, int) {
        const int pixel = pixels[k];
        const int row = pixel / width, col = pixel % width;
        double m[3] = {0, 0, 0}, m2[3] = {0, 0, 0};
        Counters cnt;
        for (int sIdx = 0; sIdx < spp; sIdx++) {
            Rng rng = Rng::seeded(seed, sample_base + (uint64_t)sIdx, (uint32_t)pixel);
            const float x1 = rng.uniform(), x2 = rng.uniform();  // camera.cu:29-34
            const Ray r = c.generate(row, col, x1, x2);
            const Vec3 L = nee ? LiNEE(*s, r, max_depth, rng, trace_once, cnt, consistent_mis != 0)
                               : LiNaive(*s, r, max_depth, rng, cnt);
            for (int ch = 0; ch < 3; ch++) {  // Welford
                const double v = L.e[ch];
                const double dlt = v - m[ch];
                m[ch] += dlt / (sIdx + 1);
                m2[ch] += dlt * (v - m[ch]);
            }
        }
        for (int ch = 0; ch < 3; ch++) {
            mean[3 * (size_t)k + ch] = m[ch];
            var[3 * (size_t)k + ch] = spp > 1 ? m2[ch] / ((double)(spp - 1) * spp) : 0.0;
        }
        q += cnt.queries;
        sh += cnt.shadow;
        dup += cnt.duplicate;
    });
    if (counts) {
        counts[0] = q.load();
        counts[1] = sh.load();
        counts[2] = dup.load();
    }
}

// ---- unit entry points for pinning against the reference's own code ----------------------
// out: wi[3], pdf, f[3], delta
void oracle_bsdf_sample(int type, const float* albedo, float ior, float alpha, const float* wo, float xi1, float xi2,
                        float* out) {
    Material m{type, Vec3(albedo[0], albedo[1], albedo[2]), Vec3(0.f), ior, alpha};
    const Vec3 w(wo[0], wo[1], wo[2]);
    BSDFSample b;
    switch (type) {
        case LAMBERTIAN: b = lambertSample(m, w, xi1, xi2); break;
        case MIRROR: b = mirrorSample(w); break;
        case GLASS: b = glassSample(m, w, xi1); break;
        default: b = microfacetSample(m, w, xi1, xi2);
    }
    out[0] = b.wiLocal.x(); out[1] = b.wiLocal.y(); out[2] = b.wiLocal.z();
    out[3] = b.pdf;
    out[4] = b.f.x(); out[5] = b.f.y(); out[6] = b.f.z();
    out[7] = b.isDelta ? 1.f : 0.f;
}
// out: f[3], pdf
void oracle_bsdf_eval(int type, const float* albedo, float ior, float alpha, const float* wo, const float* wi,
                      float* out) {
    Material m{type, Vec3(albedo[0], albedo[1], albedo[2]), Vec3(0.f), ior, alpha};
    const Vec3 a(wo[0], wo[1], wo[2]), b(wi[0], wi[1], wi[2]);
    const Vec3 f = bsdfF(m, a, b);
    out[0] = f.x(); out[1] = f.y(); out[2] = f.z();
    out[3] = bsdfPdf(m, a, b);
}
// out: wi[3], normal[3], distance, pdf, emitted[3]
void oracle_light_sample(const Scene* s, const float* p, float x1, float x2, float x3, float* out) {
    const LightSample ls = sampleDirectLights(*s, Vec3(p[0], p[1], p[2]), x1, x2, x3);
    const float v[11] = {ls.wi.x(), ls.wi.y(), ls.wi.z(), ls.normal.x(), ls.normal.y(), ls.normal.z(),
                         ls.distance, ls.pdf, ls.emitted.x(), ls.emitted.y(), ls.emitted.z()};
    std::memcpy(out, v, sizeof(v));
}
// Normals G-buffer (src/renderers/g_buffer.cu:27-57): per pixel the pixel-centre camera ray
// (Camera::generateRay(row, col), src/core/camera.cu:24-27), World::hit over [0, FLT_MAX],
// and (normal + 1) / 2 of the closest hit, zero on a miss. out: width * height * 3 floats,
// pixel = row * width + col.
void oracle_normals(const Scene* s, const float* cam, int width, int height, float* out, int threads) {
    Camera c;
    c.init(cam, cam + 3, cam + 6, cam[9], cam[10] != 0.f, width, height);
    parallel_for(width * height, threads, 64, [&](int i, int) {
        const int row = i / width, col = i % width;
        const Ray r = c.generate(row, col, 0.5f, 0.5f);
        HitRecord rec;
        Vec3 v(0.f, 0.f, 0.f);
        if (worldHit(*s, r, 0.f, FLT_MAX, rec))
            v = Vec3((rec.normal.e[0] + 1.f) / 2.f, (rec.normal.e[1] + 1.f) / 2.f, (rec.normal.e[2] + 1.f) / 2.f);
        for (int k = 0; k < 3; k++) out[3 * (size_t)i + k] = v.e[k];
    });
}
// out: o[3], d[3]
void oracle_camera_ray(const float* cam, int width, int height, int row, int col, float x1, float x2, float* out) {
    Camera c;
    c.init(cam, cam + 3, cam + 6, cam[9], cam[10] != 0.f, width, height);
    const Ray r = c.generate(row, col, x1, x2);
    for (int k = 0; k < 3; k++) { out[k] = r.o.e[k]; out[3 + k] = r.d.e[k]; }
}
// 1-D distribution (DistributionParams::createDistribution + Distribution::pmf/sample)
void oracle_dist1d(const float* values, int n, const float* xis, int nxi, float* pmf_out, float* total_out,
                   int* idx_out, float* spmf_out) {
    const Distribution d = Distribution::build(values, n);
    for (int i = 0; i < n; i++) pmf_out[i] = d.pmf(i);
    *total_out = d.totalMass;
    for (int k = 0; k < nxi; k++) idx_out[k] = d.sample(&spmf_out[k], xis[k]);
}
// 2-D distribution (Distribution2DBuilder + Distribution2D::pmf/sample)
void oracle_dist2d(const float* values, int w, int h, const float* xis, int nxi, float* pmf_out, int* sx, int* sy,
                   float* spmf) {
    const Distribution2D d = Distribution2D::build(values, w, h);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) pmf_out[y * w + x] = d.pmf(x, y);
    for (int k = 0; k < nxi; k++) {
        if (!d.sample(&spmf[k], xis[2 * k], xis[2 * k + 1], &sx[k], &sy[k])) { sx[k] = sy[k] = -1; spmf[k] = 0.f; }
    }
}
// PhiThetaDistribution::pdf on canonical coordinates and on directions
void oracle_phitheta_pdf(const float* values, int w, int h, const float* canon, int ncanon, float* pdf_canon,
                         const float* dirs, int ndirs, float* pdf_dir) {
    Env e;
    e.present = true;
    e.w = w;
    e.h = h;
    e.dist = Distribution2D::build(values, w, h);
    for (int k = 0; k < ncanon; k++) pdf_canon[k] = e.pdfCanonical(canon[2 * k], canon[2 * k + 1]);
    for (int k = 0; k < ndirs; k++) pdf_dir[k] = e.pdf(Vec3(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]));
}
// Environment light sample/pdf/emit of a loaded scene. out: wi[3], pdf, emit[3]
void oracle_env_sample(const Scene* s, float x1, float x2, float* out) {
    float pdf;
    const Vec3 w = s->env.sample(&pdf, x1, x2);
    const Vec3 e = s->env.emit(w);
    const float v[7] = {w.x(), w.y(), w.z(), pdf, e.x(), e.y(), e.z()};
    std::memcpy(out, v, sizeof(v));
}
// PCG32 stream check: the first n variates of (seed, sample, pixel)
void oracle_rng(uint64_t seed, uint64_t sample, uint32_t pixel, int n, float* out) {
    Rng r = Rng::seeded(seed, sample, pixel);
    for (int i = 0; i < n; i++) out[i] = r.uniform();
}

}  // extern "C"

// ---- guide network in FP64 (checker of the guide kernels) ----------------------------------
// Network 80 -> 64 -> 64 -> 64 (ReLU) -> 40, parameters W1[80][64] b1 W2[64][64] b2
// W3[64][64] b3 W4[64][40] b4 concatenated; outputs per lobe (mu_raw.xyz, kappa_raw, logit).
namespace oracle {
namespace guide {
constexpr int IN = 80, H = 64, OUT = 40, L = 8;
constexpr int W1 = 0, B1 = W1 + IN * H, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H, B3 = W3 + H * H, W4 = B3 + H,
              B4 = W4 + H * OUT, NP = B4 + OUT;

inline float bf16(float x) {  // round to nearest even, to BF16 precision
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

inline bool is_bias(int i) { return i >= B4 || (i >= B1 && i < W2) || (i >= B2 && i < W3) || (i >= B3 && i < W4); }

struct Net {
    std::vector<double> w;
    // the kernels multiply with BF16-rounded weights and add FP32 biases
    explicit Net(const float* p) : w(NP) {
        for (int i = 0; i < NP; i++) w[i] = is_bias(i) ? (double)p[i] : (double)bf16(p[i]);
    }
};

// forward; act[l] holds post-ReLU activations of hidden layer l; quant: round layer inputs to BF16
inline void forward(const Net& n, const double* x, bool quant, double (&a1)[H], double (&a2)[H], double (&a3)[H],
                    double (&y)[OUT]) {
    auto q = [&](double v) { return quant ? (double)bf16((float)v) : v; };
    double xin[IN];
    for (int k = 0; k < IN; k++) xin[k] = q(x[k]);
    for (int j = 0; j < H; j++) {
        double s = n.w[B1 + j];
        for (int k = 0; k < IN; k++) s += xin[k] * n.w[W1 + k * H + j];
        a1[j] = s > 0 ? s : 0;
    }
    for (int j = 0; j < H; j++) {
        double s = n.w[B2 + j];
        for (int k = 0; k < H; k++) s += q(a1[k]) * n.w[W2 + k * H + j];
        a2[j] = s > 0 ? s : 0;
    }
    for (int j = 0; j < H; j++) {
        double s = n.w[B3 + j];
        for (int k = 0; k < H; k++) s += q(a2[k]) * n.w[W3 + k * H + j];
        a3[j] = s > 0 ? s : 0;
    }
    for (int j = 0; j < OUT; j++) {
        double s = n.w[B4 + j];
        for (int k = 0; k < H; k++) s += q(a3[k]) * n.w[W4 + k * OUT + j];
        y[j] = s;
    }
}

// -w log q(wi) and its gradient with respect to the raw outputs
inline double loss_and_grad(const double (&y)[OUT], const double* wi, double w, double (&dy)[OUT]) {
    double pi[L], kap[L], mu[L][3], len[L], dt[L], lf[L];
    double mx = -1e300;
    for (int j = 0; j < L; j++) mx = std::max(mx, y[5 * j + 4]);
    double se = 0;
    for (int j = 0; j < L; j++) se += std::exp(y[5 * j + 4] - mx);
    double lmax = -1e300;
    for (int j = 0; j < L; j++) {
        pi[j] = std::exp(y[5 * j + 4] - mx) / se;
        len[j] = std::sqrt(y[5 * j] * y[5 * j] + y[5 * j + 1] * y[5 * j + 1] + y[5 * j + 2] * y[5 * j + 2]) + 1e-12;
        for (int a = 0; a < 3; a++) mu[j][a] = y[5 * j + a] / len[j];
        kap[j] = std::exp(std::min(10.0, std::max(-4.0, y[5 * j + 3])));
        dt[j] = mu[j][0] * wi[0] + mu[j][1] * wi[1] + mu[j][2] * wi[2];
        const double lognorm = std::log(kap[j]) - std::log(2 * M_PI) - std::log1p(-std::exp(-2 * kap[j]));
        lf[j] = std::log(pi[j] + 1e-300) + lognorm + kap[j] * (dt[j] - 1);
        lmax = std::max(lmax, lf[j]);
    }
    double sq = 0;
    for (int j = 0; j < L; j++) sq += std::exp(lf[j] - lmax);
    const double logq = lmax + std::log(sq);
    for (int j = 0; j < L; j++) {
        const double s = std::exp(lf[j] - logq);
        dy[5 * j + 4] = -w * (s - pi[j]);
        const double kr = y[5 * j + 3], k = kap[j];
        const double dlogc = 1 / k - 2 * std::exp(-2 * k) / (-std::expm1(-2 * k));
        dy[5 * j + 3] = (kr > -4 && kr < 10) ? -w * s * (dlogc + dt[j] - 1) * k : 0.0;
        const double c = -w * s * k / len[j];
        for (int a = 0; a < 3; a++) dy[5 * j + a] = c * (wi[a] - dt[j] * mu[j][a]);
    }
    return -w * logq;
}
}  // namespace guide
}  // namespace oracle

extern "C" {

// Raw outputs (n x 40). quant = 1 rounds each layer's inputs to BF16 (as the inference
// kernel's operands are); FP64 accumulation. Inputs 78 and 79 are padding and read as zero.
void oracle_guide_forward(const float* params, const float* x, int n, int quant, double* out) {
    using namespace oracle::guide;
    const Net net(params);
    for (int i = 0; i < n; i++) {
        double xi[IN], a1[H], a2[H], a3[H], y[OUT];
        for (int k = 0; k < IN; k++) xi[k] = k < IN - 2 ? x[(size_t)i * IN + k] : 0.0;
        forward(net, xi, quant != 0, a1, a2, a3, y);
        for (int j = 0; j < OUT; j++) out[(size_t)i * OUT + j] = y[j];
    }
}

// Loss -sum_i min(w_i / sum w, 500 / n) log q_i and its gradient (16104 values) in FP64 on the BF16-rounded
// weights. quant = 1 also rounds every matrix-product operand to BF16 where the tensor-core
// training kernel does: the inputs and activations X, A1..A3 and the back-propagated dY,
// dZ3, dZ2, dZ1 (the ReLU masks use the unrounded activations). Inputs 78 and 79 are padding
// and read as zero.
double oracle_guide_grad(const float* params, const float* x, const float* wi, const float* w, int n, int quant,
                         double* grad) {
    using namespace oracle::guide;
    const Net net(params);
    auto q = [&](double v) { return quant ? (double)bf16((float)v) : v; };
    for (int i = 0; i < NP; i++) grad[i] = 0;
    double wsum = 0;
    for (int i = 0; i < n; i++) wsum += w[i];
    const double inv = wsum > 0 ? 1 / wsum : 0;
    double loss = 0;
    for (int i = 0; i < n; i++) {
        double xi[IN], a1[H], a2[H], a3[H], y[OUT], dy[OUT];
        for (int k = 0; k < IN; k++) xi[k] = k < IN - 2 ? q(x[(size_t)i * IN + k]) : 0.0;
        forward(net, xi, quant != 0, a1, a2, a3, y);
        const double d[3] = {wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]};
        if (w[i] == 0) continue;
        loss += loss_and_grad(y, d, std::min(w[i] * inv, 500.0 / n), dy);  // per-sample weight cap
        double d3[H], d2[H], d1[H];
        for (int j = 0; j < OUT; j++) dy[j] = q(dy[j]);
        for (int k = 0; k < H; k++) {
            double s = 0;
            for (int j = 0; j < OUT; j++) {
                grad[W4 + k * OUT + j] += q(a3[k]) * dy[j];
                s += dy[j] * net.w[W4 + k * OUT + j];
            }
            d3[k] = a3[k] > 0 ? q(s) : 0;
        }
        for (int j = 0; j < OUT; j++) grad[B4 + j] += dy[j];
        for (int k = 0; k < H; k++) {
            double s = 0;
            for (int j = 0; j < H; j++) {
                grad[W3 + k * H + j] += q(a2[k]) * d3[j];
                s += d3[j] * net.w[W3 + k * H + j];
            }
            d2[k] = a2[k] > 0 ? q(s) : 0;
        }
        for (int j = 0; j < H; j++) grad[B3 + j] += d3[j];
        for (int k = 0; k < H; k++) {
            double s = 0;
            for (int j = 0; j < H; j++) {
                grad[W2 + k * H + j] += q(a1[k]) * d2[j];
                s += d2[j] * net.w[W2 + k * H + j];
            }
            d1[k] = a1[k] > 0 ? q(s) : 0;
        }
        for (int j = 0; j < H; j++) grad[B2 + j] += d2[j];
        for (int k = 0; k < IN; k++)
            for (int j = 0; j < H; j++) grad[W1 + k * H + j] += xi[k] * d1[j];
        for (int j = 0; j < H; j++) grad[B1 + j] += d1[j];
    }
    return loss;
}

// Loss only (for finite differences): the parameters are used as given (no BF16 rounding).
double oracle_guide_loss_exact(const double* params, const float* x, const float* wi, const float* w, int n) {
    using namespace oracle::guide;
    std::vector<float> dummy(NP, 0.f);
    Net net(dummy.data());
    for (int i = 0; i < NP; i++) net.w[i] = params[i];
    double wsum = 0;
    for (int i = 0; i < n; i++) wsum += w[i];
    double loss = 0;
    for (int i = 0; i < n; i++) {
        double xi[IN], a1[H], a2[H], a3[H], y[OUT], dy[OUT];
        for (int k = 0; k < IN; k++) xi[k] = x[(size_t)i * IN + k];
        forward(net, xi, false, a1, a2, a3, y);
        const double d[3] = {wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]};
        if (w[i] == 0) continue;
        loss += loss_and_grad(y, d, std::min(w[i] / wsum, 500.0 / n), dy);
    }
    return loss;
}

}  // extern "C"
