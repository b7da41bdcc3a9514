// Ray queries against the wide BVH: closest hit and any hit.
//
// Primitive tests restate the reference's arithmetic with uncontracted IEEE single
// operations (__fmul_rn/__fadd_rn/__fsub_rn/__fdiv_rn/__fsqrt_rn):
//   Triangle::hit  src/primitives/triangle.cu:7-48   (Moller-Trumbore form, inclusive bounds)
//   Sphere::hit    src/primitives/sphere.cu:7-43     (near root, then far root, strict bounds)
// and World::hit's selection rule (src/world.cu:5-41): a linear scan of all triangles in index
// order accepting t <= tNear (so on an exact tie the higher triangle index wins), then all
// spheres accepting only t < tNear (so triangles win ties against spheres and, among spheres,
// the lower index wins). Here the same outcome is computed as the minimum of a total order
// (t, then the tie rank), which does not depend on the order the BVH visits leaves in.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dev_math.cuh"
#include "pt_types.h"

namespace pt {

constexpr int kMissPrim = 0x7fffffff;  // no hit
// Relative slack applied to box-interval ends: boxes are visited when they might contain a
// hit the primitive test would accept (never culls what the linear scan reports).
constexpr float kBoxSlack = 1.00006103515625f;  // 1 + 2^-14

struct Hit {
    float t, b1, b2;
    int prim;  // >= 0 triangle id, < 0 ~sphere id, kMissPrim: none
};

__device__ __forceinline__ float xdot(V a, V b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ V xcross(V a, V b) {
    return V{__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
             -__fsub_rn(__fmul_rn(a.x, b.z), __fmul_rn(a.z, b.x)),
             __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ __forceinline__ V xsub(V a, V b) {
    return V{__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}

// Triangle::hit arithmetic. e1 = p1 - p0 and e2 = p2 - p0 arrive precomputed (same FP32
// subtractions). Returns false on a miss; otherwise t, b1, b2. tmax is inclusive.
__device__ __forceinline__ bool tri_test(V p0, V e1, V e2, V o, V d, float tmin, float tmax,
                                         float& t, float& b1, float& b2) {
    const V s1 = xcross(d, e2);
    const float divisor = xdot(s1, e1);
    if (divisor == 0.f) return false;
    const float inv = __fdiv_rn(1.f, divisor);
    const V s = xsub(o, p0);
    b1 = __fmul_rn(xdot(s, s1), inv);
    if (b1 < 0.f || b1 > 1.f) return false;
    const V s2 = xcross(s, e1);
    b2 = __fmul_rn(xdot(d, s2), inv);
    if (b2 < 0.f || __fadd_rn(b1, b2) > 1.f) return false;
    t = __fmul_rn(xdot(e2, s2), inv);
    if (t < tmin || t > tmax) return false;
    return true;
}

// Component k (0, 1, 2) of a vector, by selects (no local memory).
__device__ __forceinline__ float vcomp(V v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Watertight ray/triangle test (Woop, Benthin and Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1), 2013), the opt-in alternative to Triangle::hit: no ray that
// passes through a shared edge or vertex of a closed mesh slips between its triangles.
// - Axes: kz is the largest component of |d| (first of x, y, z on ties), kx and ky the next two
//   cyclically, swapped when d[kz] < 0 so the winding is kept.
// - Shear: sz = 1 / d[kz], sx = d[kx] * sz, sy = d[ky] * sz (every operation rounded once).
// - Vertices relative to the origin, sheared so the ray runs along +z: ax = A[kx] - sx A[kz],
//   ay = A[ky] - sy A[kz] (likewise B, C).
// - Edge functions U = cx by - cy bx, V = ax cy - ay cx, W = bx ay - by ax; any that is exactly 0
//   is recomputed in FP64 from the same FP32 inputs (products exact, one rounding each).
// - Mixed signs miss; det = U + V + W, det = 0 misses; T = U sz A[kz] + V sz B[kz] + W sz C[kz],
//   t = T / det within [tmin, tmax] (inclusive, as Triangle::hit), b1 = V / det (weight of p1),
//   b2 = W / det (weight of p2). No backface culling, as the reference.
// Every FP32 operation is an explicit round-to-nearest intrinsic (no contraction), so the
// oracle's host restatement gives the same bits.
__device__ __forceinline__ bool tri_test_wt(V p0, V p1, V p2, V o, V d, float tmin, float tmax, float& t,
                                            float& b1, float& b2) {
    const float adx = fabsf(d.x), ady = fabsf(d.y), adz = fabsf(d.z);
    const int kz = adx >= ady ? (adx >= adz ? 0 : 2) : (ady >= adz ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    const float dz = vcomp(d, kz);
    if (dz < 0.f) {
        const int k = kx;
        kx = ky;
        ky = k;
    }
    const float sz = __fdiv_rn(1.f, dz);
    const float sx = __fmul_rn(vcomp(d, kx), sz), sy = __fmul_rn(vcomp(d, ky), sz);
    const V A = xsub(p0, o), B = xsub(p1, o), C = xsub(p2, o);
    const float Az = vcomp(A, kz), Bz = vcomp(B, kz), Cz = vcomp(C, kz);
    const float ax = __fsub_rn(vcomp(A, kx), __fmul_rn(sx, Az)), ay = __fsub_rn(vcomp(A, ky), __fmul_rn(sy, Az));
    const float bx = __fsub_rn(vcomp(B, kx), __fmul_rn(sx, Bz)), by = __fsub_rn(vcomp(B, ky), __fmul_rn(sy, Bz));
    const float cx = __fsub_rn(vcomp(C, kx), __fmul_rn(sx, Cz)), cy = __fsub_rn(vcomp(C, ky), __fmul_rn(sy, Cz));
    float U = __fsub_rn(__fmul_rn(cx, by), __fmul_rn(cy, bx));
    float Vv = __fsub_rn(__fmul_rn(ax, cy), __fmul_rn(ay, cx));
    float Ww = __fsub_rn(__fmul_rn(bx, ay), __fmul_rn(by, ax));
    if (U == 0.f || Vv == 0.f || Ww == 0.f) {
        U = __double2float_rn(__dsub_rn(__dmul_rn((double)cx, (double)by), __dmul_rn((double)cy, (double)bx)));
        Vv = __double2float_rn(__dsub_rn(__dmul_rn((double)ax, (double)cy), __dmul_rn((double)ay, (double)cx)));
        Ww = __double2float_rn(__dsub_rn(__dmul_rn((double)bx, (double)ay), __dmul_rn((double)by, (double)ax)));
    }
    if ((U < 0.f || Vv < 0.f || Ww < 0.f) && (U > 0.f || Vv > 0.f || Ww > 0.f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, Vv), Ww);
    if (det == 0.f) return false;
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, __fmul_rn(sz, Az)), __fmul_rn(Vv, __fmul_rn(sz, Bz))),
                              __fmul_rn(Ww, __fmul_rn(sz, Cz)));
    const float inv = __fdiv_rn(1.f, det);
    t = __fmul_rn(T, inv);
    if (!(t >= tmin && t <= tmax)) return false;
    b1 = __fmul_rn(Vv, inv);
    b2 = __fmul_rn(Ww, inv);
    return true;
}

// Sphere::hit root selection: the near root when it lies above tmin, else the far root.
// Returns false when neither root is above tmin (the caller applies the strict upper bound).
__device__ __forceinline__ bool sphere_candidate(V c, float r, V o, V d, float tmin, float& t) {
    const V oc = xsub(o, c);
    const float a = xdot(d, d);
    const float b = xdot(oc, d);
    const float cc = __fsub_rn(xdot(oc, oc), __fmul_rn(r, r));
    const float disc = __fsub_rn(__fmul_rn(b, b), __fmul_rn(a, cc));
    if (!(disc > 0.f)) return false;
    const float sq = __fsqrt_rn(disc);
    const float nb = -b;
    float tt = __fdiv_rn(__fsub_rn(nb, sq), a);
    if (tt > tmin) { t = tt; return true; }
    tt = __fdiv_rn(__fadd_rn(nb, sq), a);
    if (tt > tmin) { t = tt; return true; }
    return false;
}

struct RayPre {
    V o, d;
    float ix, iy, iz, ox, oy, oz;
};
__device__ __forceinline__ RayPre make_raypre(V o, V d) {
    RayPre r;
    r.o = o;
    r.d = d;
    const float dx = fabsf(d.x) < 1e-20f ? copysignf(1e-20f, d.x) : d.x;
    const float dy = fabsf(d.y) < 1e-20f ? copysignf(1e-20f, d.y) : d.y;
    const float dz = fabsf(d.z) < 1e-20f ? copysignf(1e-20f, d.z) : d.z;
    r.ix = 1.f / dx;
    r.iy = 1.f / dy;
    r.iz = 1.f / dz;
    r.ox = o.x * r.ix;
    r.oy = o.y * r.iy;
    r.oz = o.z * r.iz;
    return r;
}

// Slab test: the entry and exit distances of the box clipped to [tmin, tlim]; the box is
// visited when tn <= tf * kBoxSlack.
__device__ __forceinline__ void box_interval(const RayPre& r, float lx, float hx, float ly, float hy, float lz,
                                             float hz, float tmin, float tlim, float& tn, float& tf) {
    const float t0x = fmaf(lx, r.ix, -r.ox), t1x = fmaf(hx, r.ix, -r.ox);
    const float t0y = fmaf(ly, r.iy, -r.oy), t1y = fmaf(hy, r.iy, -r.oy);
    const float t0z = fmaf(lz, r.iz, -r.oz), t1z = fmaf(hz, r.iz, -r.oz);
    tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), tmin));
    tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), tlim));
}
// Slab test; returns the entry distance or +inf when the interval is empty.
__device__ __forceinline__ float box_entry(const RayPre& r, float lx, float hx, float ly, float hy,
                                           float lz, float hz, float tmin, float tlim) {
    float tn, tf;
    box_interval(r, lx, hx, ly, hy, lz, hz, tmin, tlim, tn, tf);
    return (tn <= tf * kBoxSlack) ? tn : __int_as_float(0x7f800000);
}

// Children are ordered by an integer sort key: the entry distance, clamped at zero, with its
// three low bits replaced by the child's slot (the slot breaks ties and travels with the
// key), or kMissKey | slot for a child that was not hit. Keys of hit children are below
// kMissKey, and for non-negative floats the bit patterns order like the values, so sorting the
// keys orders the children by their distance bucket key_dist(tn) (tn with the three low bits
// cleared: 8 ulp wide), nearest first.
constexpr uint32_t kMissKey = 0x7f800000u;
__device__ __forceinline__ float key_dist(float tn) { return __uint_as_float(__float_as_uint(fmaxf(tn, 0.f)) & ~7u); }
__device__ __forceinline__ void key_order(uint32_t& a, uint32_t& b) {
    const uint32_t lo = min(a, b);
    b = max(a, b);
    a = lo;
}
// Ascending sort of W keys by size-optimal sorting networks (1, 5 and 19 comparators; Knuth,
// TAOCP vol. 3, 5.3.4).
template <int W>
__device__ __forceinline__ void sort_keys(uint32_t (&k)[W]) {
    if constexpr (W == 2) {
        key_order(k[0], k[1]);
    } else if constexpr (W == 4) {
        key_order(k[0], k[1]); key_order(k[2], k[3]);
        key_order(k[0], k[2]); key_order(k[1], k[3]);
        key_order(k[1], k[2]);
    } else {
        static_assert(W == 8, "BVH width 2, 4 or 8");
        key_order(k[0], k[2]); key_order(k[1], k[3]); key_order(k[4], k[6]); key_order(k[5], k[7]);
        key_order(k[0], k[4]); key_order(k[1], k[5]); key_order(k[2], k[6]); key_order(k[3], k[7]);
        key_order(k[0], k[1]); key_order(k[2], k[3]); key_order(k[4], k[5]); key_order(k[6], k[7]);
        key_order(k[2], k[4]); key_order(k[3], k[5]);
        key_order(k[1], k[4]); key_order(k[3], k[6]);
        key_order(k[1], k[2]); key_order(k[3], k[4]); key_order(k[5], k[6]);
    }
}

// Closest-hit acceptance for one leaf entry (tie rules above). `tcur` is best.t or tmax.
// `wt`: the scene's triangle entries hold p0, p1, p2 and take the watertight test.
__device__ __forceinline__ void leaf_entry(const float4* __restrict__ prims, int e, const RayPre& r,
                                           float tmin, float tmax, Hit& best, bool wt) {
    const float4 a = __ldg(prims + 3 * e);
    const int id = __float_as_int(a.w);
    const float tcur = best.prim == kMissPrim ? tmax : best.t;
    if (id >= 0) {
        const float4 b = __ldg(prims + 3 * e + 1);
        const float4 c = __ldg(prims + 3 * e + 2);
        float t, b1, b2;
        const bool h = wt ? tri_test_wt(mkv(a), mkv(b), mkv(c), r.o, r.d, tmin, tcur, t, b1, b2)
                          : tri_test(mkv(a), mkv(b), mkv(c), r.o, r.d, tmin, tcur, t, b1, b2);
        if (h) {
            // equal t: the higher triangle index wins; a triangle beats a sphere
            if (t == tcur && best.prim != kMissPrim && best.prim >= 0 && id < best.prim) return;
            best.t = t;
            best.b1 = b1;
            best.b2 = b2;
            best.prim = id;
        }
    } else {
        const float4 b = __ldg(prims + 3 * e + 1);
        float t;
        if (sphere_candidate(mkv(a), b.x, r.o, r.d, tmin, t)) {
            const bool better = t < tcur ||
                                (t == tcur && best.prim != kMissPrim && best.prim < 0 && id > best.prim);
            // id = ~k: a larger id is a lower sphere index k
            if (better) {
                best.t = t;
                best.b1 = 0.f;
                best.b2 = 0.f;
                best.prim = id;
            }
        }
    }
}

// Any-hit acceptance for one leaf entry: true if the entry blocks [tmin, tmax].
__device__ __forceinline__ bool leaf_entry_any(const float4* __restrict__ prims, int e, const RayPre& r,
                                               float tmin, float tmax, bool wt) {
    const float4 a = __ldg(prims + 3 * e);
    const int id = __float_as_int(a.w);
    if (id >= 0) {
        const float4 b = __ldg(prims + 3 * e + 1);
        const float4 c = __ldg(prims + 3 * e + 2);
        float t, b1, b2;
        return wt ? tri_test_wt(mkv(a), mkv(b), mkv(c), r.o, r.d, tmin, tmax, t, b1, b2)
                  : tri_test(mkv(a), mkv(b), mkv(c), r.o, r.d, tmin, tmax, t, b1, b2);
    }
    const float4 b = __ldg(prims + 3 * e + 1);
    float t;
    return sphere_candidate(mkv(a), b.x, r.o, r.d, tmin, t) && t < tmax;
}

template <int W>
struct NodeView {
    float lo_x[W], hi_x[W], lo_y[W], hi_y[W], lo_z[W], hi_z[W];
    int child[W];
};

template <int W>
__device__ __forceinline__ void load_node(const float4* __restrict__ p, NodeView<W>& nv) {
    constexpr int kUsed = (7 * W + 3) / 4;  // float4s that hold bounds + children
    float4 raw[kUsed];
#pragma unroll
    for (int i = 0; i < kUsed; i++) raw[i] = __ldg(p + i);
    const float* f = reinterpret_cast<const float*>(raw);
#pragma unroll
    for (int k = 0; k < W; k++) {
        nv.lo_x[k] = f[0 * W + k];
        nv.hi_x[k] = f[1 * W + k];
        nv.lo_y[k] = f[2 * W + k];
        nv.hi_y[k] = f[3 * W + k];
        nv.lo_z[k] = f[4 * W + k];
        nv.hi_z[k] = f[5 * W + k];
        nv.child[k] = __float_as_int(f[6 * W + k]);
    }
}

// A float node (W = 4 or 8) read in the ray's octant order: per axis the near planes (the
// lower bounds where the ray's direction component is positive, the upper ones where it is
// negative) into lo_*, the far planes into hi_*. For a box with lower <= upper bound, the near
// plane's slab distance is the smaller one (fmaf is monotone in its first operand for a fixed
// nonzero factor), so the slab test needs no min/max per axis and gives the same entry and exit
// distances bit for bit. The choice of plane is an address offset per load.
template <int W>
__device__ __forceinline__ void load_node_oct(const float4* __restrict__ p, const RayPre& r, NodeView<W>& nv) {
    static_assert(W == 4 || W == 8, "octant loads need whole float4 planes");
    constexpr int A = W / 4;  // float4s per plane
    const int sx = __float_as_int(r.ix) < 0 ? A : 0;
    const int sy = __float_as_int(r.iy) < 0 ? A : 0;
    const int sz = __float_as_int(r.iz) < 0 ? A : 0;
    float4 raw[7 * A];
#pragma unroll
    for (int a = 0; a < A; a++) {
        raw[0 * A + a] = __ldg(p + 0 * A + sx + a);
        raw[1 * A + a] = __ldg(p + 1 * A - sx + a);
        raw[2 * A + a] = __ldg(p + 2 * A + sy + a);
        raw[3 * A + a] = __ldg(p + 3 * A - sy + a);
        raw[4 * A + a] = __ldg(p + 4 * A + sz + a);
        raw[5 * A + a] = __ldg(p + 5 * A - sz + a);
        raw[6 * A + a] = __ldg(p + 6 * A + a);
    }
    const float* f = reinterpret_cast<const float*>(raw);
#pragma unroll
    for (int k = 0; k < W; k++) {
        nv.lo_x[k] = f[0 * W + k];
        nv.hi_x[k] = f[1 * W + k];
        nv.lo_y[k] = f[2 * W + k];
        nv.hi_y[k] = f[3 * W + k];
        nv.lo_z[k] = f[4 * W + k];
        nv.hi_z[k] = f[5 * W + k];
        nv.child[k] = __float_as_int(f[6 * W + k]);
    }
}

// Slab test on near and far planes (load_node_oct): the entry distance, or +inf when empty.
__device__ __forceinline__ float box_entry_nf(const RayPre& r, float nx, float fx, float ny, float fy, float nz,
                                              float fz, float tmin, float tlim) {
    const float tnx = fmaf(nx, r.ix, -r.ox), tfx = fmaf(fx, r.ix, -r.ox);
    const float tny = fmaf(ny, r.iy, -r.oy), tfy = fmaf(fy, r.iy, -r.oy);
    const float tnz = fmaf(nz, r.iz, -r.oz), tfz = fmaf(fz, r.iz, -r.oz);
    const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
    const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tlim));
    return (tn <= tf * kBoxSlack) ? tn : __int_as_float(0x7f800000);
}

// Scale of a quantized node's axis: the FP32 power of two with biased exponent e.
__device__ __forceinline__ float qscale(uint32_t e) { return __uint_as_float((e & 0xFFu) << 23); }


// A quantized node (qnode_bytes(W) bytes, W = 4 or 8) decoded into the float view: each plane
// is fmaf(q, scale, origin), which contains the float box the build quantized.
template <int W>
__device__ __forceinline__ void load_qnode(const float4* __restrict__ p, NodeView<W>& nv) {
    constexpr int kF4 = qnode_bytes(W) / 16;
    float4 raw[kF4];
#pragma unroll
    for (int i = 0; i < kF4; i++) raw[i] = __ldg(p + i);
    const uint32_t e = __float_as_uint(raw[0].w);
    const float ox = raw[0].x, oy = raw[0].y, oz = raw[0].z;
    const float sx = qscale(e), sy = qscale(e >> 8), sz = qscale(e >> 16);
    const uint32_t* u = reinterpret_cast<const uint32_t*>(raw);
    auto q = [&](int a, int k) { return (float)((u[4 + (a * W + k) / 4] >> (8 * ((a * W + k) & 3))) & 0xFFu); };
#pragma unroll
    for (int k = 0; k < W; k++) {
        nv.lo_x[k] = __fmaf_rn(q(0, k), sx, ox);
        nv.hi_x[k] = __fmaf_rn(q(1, k), sx, ox);
        nv.lo_y[k] = __fmaf_rn(q(2, k), sy, oy);
        nv.hi_y[k] = __fmaf_rn(q(3, k), sy, oy);
        nv.lo_z[k] = __fmaf_rn(q(4, k), sz, oz);
        nv.hi_z[k] = __fmaf_rn(q(5, k), sz, oz);
        nv.child[k] = (int)u[qnode_child_offset(W) / 4 + k];
    }
}

// Per-query work counters (only maintained when the CNT template flag is set).
struct TraceWork {
    unsigned nodes = 0;  // wide nodes loaded
    unsigned prims = 0;  // leaf entries tested
};

// Next entry to process from the traversal stack, or kEmptyChild when it is empty.
// Stack entry: x = node index, y = (remaining count << 24) | 3-bit child slots, nearest first;
// the stack holds at most one entry per tree level. For closest-hit queries the popped child
// is re-tested against the current hit distance. When it is culled, the siblings behind it are
// dropped with it if its distance bucket already lies beyond the culling threshold: the
// siblings' buckets are no nearer, so each of them would be culled by its own test. Otherwise
// only the popped child is dropped and the next sibling is tested in turn.
template <int W, bool ANY>
__device__ __forceinline__ int stack_pop(const float4* __restrict__ nodes, bool quant, const RayPre& r, float tmin,
                                         float tmax, const Hit& best, int2* __restrict__ stk, int stride, int& sp) {
    constexpr int kNF4 = sizeof(BvhNode<W>) / 16;
    while (sp > 0) {
        const int2 ent = stk[(sp - 1) * stride];
        const int parent = ent.x;
        const uint32_t packed = (uint32_t)ent.y;
        const int cnt = (int)(packed >> 24);
        const uint32_t list = packed & 0xFFFFFFu;
        const int sl = (int)(list & 7u);
        if (cnt > 1) stk[(sp - 1) * stride] = make_int2(parent, (int)(((uint32_t)(cnt - 1) << 24) | (list >> 3)));
        else sp--;
        if (W >= 4 && quant) {
            const float4* pq = nodes + (size_t)parent * (qnode_bytes(W) / 16);
            const unsigned char* b = reinterpret_cast<const unsigned char*>(pq);
            if (!ANY) {
                const float4 h = __ldg(pq);
                const uint32_t e = __float_as_uint(h.w);
                const float sx = qscale(e), sy = qscale(e >> 8), sz = qscale(e >> 16);
                const float tc = best.prim == kMissPrim ? tmax : best.t;
                float tn, tf;
                box_interval(r, __fmaf_rn((float)__ldg(b + 16 + 0 * W + sl), sx, h.x),
                             __fmaf_rn((float)__ldg(b + 16 + 1 * W + sl), sx, h.x),
                             __fmaf_rn((float)__ldg(b + 16 + 2 * W + sl), sy, h.y),
                             __fmaf_rn((float)__ldg(b + 16 + 3 * W + sl), sy, h.y),
                             __fmaf_rn((float)__ldg(b + 16 + 4 * W + sl), sz, h.z),
                             __fmaf_rn((float)__ldg(b + 16 + 5 * W + sl), sz, h.z), tmin, tc * kBoxSlack, tn, tf);
                const float thr = tf * kBoxSlack;
                if (!(tn <= thr)) {
                    if (cnt > 1 && key_dist(tn) > fmaxf(thr, 0.f)) sp--;
                    continue;
                }
            }
            return __ldg(reinterpret_cast<const int*>(b + qnode_child_offset(W)) + sl);
        }
        const float* pf = reinterpret_cast<const float*>(nodes + (size_t)parent * kNF4);
        if (!ANY) {
            const float tc = best.prim == kMissPrim ? tmax : best.t;
            float tn, tf;
            box_interval(r, __ldg(pf + 0 * W + sl), __ldg(pf + 1 * W + sl), __ldg(pf + 2 * W + sl),
                         __ldg(pf + 3 * W + sl), __ldg(pf + 4 * W + sl), __ldg(pf + 5 * W + sl), tmin, tc * kBoxSlack,
                         tn, tf);
            const float thr = tf * kBoxSlack;
            if (!(tn <= thr)) {
                if (cnt > 1 && key_dist(tn) > fmaxf(thr, 0.f)) sp--;
                continue;
            }
        }
        return __float_as_int(__ldg(pf + 6 * W + sl));
    }
    return kEmptyChild;
}

// One internal-node visit of a live query (`cur` >= 0): test the node's children, push the
// farther hits (nearest first for closest hit; for any hit, nearest first with `near`, else in
// the node's order), descend into the first, or pop the stack when none was hit. The query ends (`alive` false) when the stack
// runs empty, or gives up with `overflow` set when it would exceed `max_depth` entries.
template <int W, bool ANY, bool CNT>
__device__ __forceinline__ void node_step(const float4* __restrict__ nodes, bool quant, const RayPre& r, float tmin,
                                          float tmax, int2* __restrict__ stk, int stride, int max_depth,
                                          const Hit& best, int& cur, int& sp, bool& alive, int& overflow,
                                          TraceWork* work, bool near = false) {
    constexpr int kNF4 = sizeof(BvhNode<W>) / 16;
    NodeView<W> nv;
    constexpr bool kOct = W >= 4 && !ANY;  // closest hit: float nodes read in octant order (near, far planes)
    if (quant) load_qnode<W>(nodes + (size_t)cur * (qnode_bytes(W) / 16), nv);
    else if constexpr (kOct) load_node_oct<W>(nodes + (size_t)cur * kNF4, r, nv);
    else load_node<W>(nodes + (size_t)cur * kNF4, nv);
    if (CNT) work->nodes++;
    const float tcur = best.prim == kMissPrim ? tmax : best.t;
    const float tlim = tcur * kBoxSlack;
    // sort keys: nearest first for closest hit (and any hit with `near`); otherwise hit
    // children first in slot order
    uint32_t key[W];
    int nhit = 0;
#pragma unroll
    for (int k = 0; k < W; k++) {
        const float te =
            kOct && !quant
                ? box_entry_nf(r, nv.lo_x[k], nv.hi_x[k], nv.lo_y[k], nv.hi_y[k], nv.lo_z[k], nv.hi_z[k], tmin, tlim)
                : box_entry(r, nv.lo_x[k], nv.hi_x[k], nv.lo_y[k], nv.hi_y[k], nv.lo_z[k], nv.hi_z[k], tmin, tlim);
        const bool hit = te != __int_as_float(0x7f800000) && nv.child[k] != kEmptyChild;
        if (ANY && !near) key[k] = hit ? (uint32_t)k : kMissKey | (uint32_t)k;
        else key[k] = hit ? (__float_as_uint(key_dist(te)) | (uint32_t)k) : kMissKey | (uint32_t)k;
        nhit += hit ? 1 : 0;
    }
    sort_keys<W>(key);
    int next = kEmptyChild;
    if (nhit > 0) {
        if (nhit > 1) {
            // slots of the hit children after the nearest, nearest in the low bits (entries
            // past nhit - 1 are never read)
            uint32_t list = 0;
#pragma unroll
            for (int k = W - 1; k >= 1; k--) list = (list << 3) | (key[k] & 7u);
            if (sp >= max_depth) {
                overflow = 1;
                alive = false;  // reported to the host; the query gives up
            } else {
                stk[sp * stride] = make_int2(cur, (int)(((uint32_t)(nhit - 1) << 24) | list));
                sp++;
            }
        }
        const int sel = (int)(key[0] & 7u);
#pragma unroll
        for (int k = 0; k < W; k++)
            if (k == sel) next = nv.child[k];
    }
    if (alive && next == kEmptyChild) next = stack_pop<W, ANY>(nodes, quant, r, tmin, tmax, best, stk, stride, sp);
    cur = next;
    if (cur == kEmptyChild) alive = false;
}

// Test the entries of one leaf (`leaf` a leaf code) against a query; an any-hit query stops
// at its first hit.
template <bool ANY, bool CNT>
__device__ __forceinline__ void leaf_test(const float4* __restrict__ prims, int leaf, const RayPre& r, float tmin,
                                          float tmax, Hit& best, bool& hit_any, TraceWork* work, bool wt) {
    const int first = leaf_first(leaf), cnt = leaf_count(leaf);
    if (CNT) work->prims += cnt;
    if (ANY) {
        for (int e = first; e < first + cnt; e++) {
            if (leaf_entry_any(prims, e, r, tmin, tmax, wt)) {
                hit_any = true;
                break;
            }
        }
    } else {
        for (int e = first; e < first + cnt; e++) leaf_entry(prims, e, r, tmin, tmax, best, wt);
    }
}

// One leaf visit of a live query (`cur` a leaf code): test its entries, then pop the stack.
// An any-hit query ends at its first hit (`hit_any`); every query ends on an empty stack.
template <int W, bool ANY, bool CNT>
__device__ __forceinline__ void leaf_step(const float4* __restrict__ nodes, const float4* __restrict__ prims,
                                          bool quant, const RayPre& r, float tmin, float tmax,
                                          int2* __restrict__ stk, int stride, Hit& best, int& cur, int& sp,
                                          bool& alive, bool& hit_any, TraceWork* work, bool wt) {
    leaf_test<ANY, CNT>(prims, cur, r, tmin, tmax, best, hit_any, work, wt);
    if (ANY && hit_any) alive = false;
    if (alive) {
        cur = stack_pop<W, ANY>(nodes, quant, r, tmin, tmax, best, stk, stride, sp);
        if (cur == kEmptyChild) alive = false;
    }
}

// One round of the warp-synchronous traversal; every lane of the warp calls it together.
// Phase 1 visits internal nodes until each live lane holds a leaf (or its query ended);
// phase 2 tests the leaves. With `spec` (speculative traversal, Aila and Laine 2009), a lane
// that reaches its first leaf parks it in `pend` and keeps descending while some lane of the
// warp has found no leaf yet, so the node phase runs with fuller warps; the parked leaf is
// tested in phase 2. Closest hits are the minimum of a total order, so the visiting order
// never changes a result; speculation only visits nodes that a tighter bound might have culled.
template <int W, bool ANY, bool CNT>
__device__ __forceinline__ void traverse_round(const float4* __restrict__ nodes, const float4* __restrict__ prims,
                                               bool quant, bool spec, const RayPre& r, float tmin, float tmax,
                                               int2* __restrict__ stk, int stride, int max_depth, Hit& best,
                                               int& cur, int& pend, int& sp, bool& alive, bool& hit_any,
                                               int& overflow, TraceWork* work, bool wt = false, bool near = false) {
    // ---- phase 1: internal nodes, while some live lane has found no leaf
    while (__any_sync(0xffffffffu, alive && cur >= 0 && pend == kEmptyChild)) {
        if (alive && cur >= 0) {
            node_step<W, ANY, CNT>(nodes, quant, r, tmin, tmax, stk, stride, max_depth, best, cur, sp, alive, overflow,
                                   work, near);
            if (spec) {
                if (!alive && !overflow && pend != kEmptyChild) {
                    alive = true;  // the stack ran empty: only the parked leaf is left
                    cur = pend;
                    pend = kEmptyChild;
                } else if (alive && cur < 0 && pend == kEmptyChild) {
                    pend = cur;  // park the first leaf and keep descending
                    cur = stack_pop<W, ANY>(nodes, quant, r, tmin, tmax, best, stk, stride, sp);
                    if (cur == kEmptyChild) {
                        cur = pend;
                        pend = kEmptyChild;
                    }
                }
            }
        }
    }
    // ---- phase 2: the parked leaf, then the current one (which pops the stack)
    if (alive && pend != kEmptyChild) {
        leaf_test<ANY, CNT>(prims, pend, r, tmin, tmax, best, hit_any, work, wt);
        pend = kEmptyChild;
        if (ANY && hit_any) alive = false;
    }
    if (alive && cur < 0)
        leaf_step<W, ANY, CNT>(nodes, prims, quant, r, tmin, tmax, stk, stride, best, cur, sp, alive, hit_any, work, wt);
}

// Warp-synchronous traversal: every lane of the warp calls this together (`active` marks the
// lanes that carry a query). Lanes advance through internal nodes in one phase and test
// leaves in the next, re-converging at each phase boundary (the while-while organisation of
// Aila and Laine, HPG 2009), so leaf tests and node visits execute as coherent SIMT
// instructions instead of drifting apart. Returns whether the query hit. Q: node format, 0 float
// nodes, 1 quantized nodes (W >= 4), -1 read from the scene at run time.
template <int W, bool ANY, bool CNT = false, int Q = -1>
__device__ __forceinline__ bool traverse(const SceneDevice& sc, const RayPre& r, float tmin, float tmax, bool active,
                                         int2* __restrict__ stk, int stride, int max_depth, Hit& best,
                                         int& overflow, TraceWork* work = nullptr) {
    const float4* __restrict__ nodes = sc.nodes;
    const float4* __restrict__ prims = sc.prims;
    const bool quant = Q < 0 ? (W >= 4 && sc.node_q != 0) : (W >= 4 && Q == 1);  // warp-uniform
    const bool wt = sc.watertight != 0;
    best.prim = kMissPrim;
    best.t = tmax;
    int sp = 0;
    int cur = active ? sc.root : kEmptyChild;
    bool alive = active;
    bool hit_any = false;
    int pend = kEmptyChild;
    while (__any_sync(0xffffffffu, alive))
        traverse_round<W, ANY, CNT>(nodes, prims, quant, false, r, tmin, tmax, stk, stride, max_depth, best, cur, pend,
                                    sp, alive, hit_any, overflow, work, wt);
    if (ANY) {
        if (hit_any) best.prim = 0;
        return hit_any;
    }
    return best.prim != kMissPrim;
}

}  // namespace pt
