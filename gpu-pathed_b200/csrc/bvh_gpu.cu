// GPU BVH construction: a binary tree over the Morton-sorted primitives, either a linear BVH
// (Karras 2012 radix tree) or agglomerative clustering (PLOC), collapsed to the same W-wide
// node format, padded boxes and leaf-entry layout as the host's binned-SAH builder
// (bvh_build.cpp), so every traversal kernel works on any of the trees unchanged and the
// closest-hit results stay identical (the tie rule lives in the leaf test, the padding keeps
// every child box conservative).
//
//   1. primitive boxes and centroids (triangles: vertex min/max; spheres: centre -/+ radius)
//   2. scene and centroid bounds (warp reduction + atomics on order-preserving integers)
//   3. 63-bit Morton codes of the centroids, sorted with their primitive ids (CUB radix sort)
//   4. LBVH: radix tree over the sorted codes (Karras, "Maximizing parallelism in the
//      construction of BVHs, octrees, and k-d trees", HPG 2012): each internal node finds its
//      range and split from the codes' common-prefix lengths;
//   5. bounds and primitive counts bottom-up (the second child to arrive at a node merges).
//   4'. PLOC instead (Meister and Bittner, "Parallel Locally-Ordered Clustering for Bounding
//      Volume Hierarchy Construction", TVCG 2018): starting from one cluster per primitive in
//      Morton order, each cluster finds the neighbour within kPlocRadius positions whose union
//      box has the smallest surface area; mutual nearest neighbours merge into a new node, and
//      the surviving clusters are compacted in order, until one is left. Leaves are then
//      numbered in the tree's depth-first order, so every subtree's primitives are contiguous.
//   6. top-down collapse, one launch per level: a wide node opens its largest-area children
//      that hold more than max_leaf primitives until it has W children; children with at
//      most max_leaf primitives become leaves (their primitives are contiguous in Morton order)
//   7. leaf entries in Morton order (LBVH) or depth-first order (PLOC)
#include "bvh_gpu.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cfloat>
#include <cmath>
#include <cstring>

namespace pt {

namespace {

__device__ __forceinline__ unsigned ord_float(float f) {  // order-preserving float -> uint
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float unord_float(unsigned u) {
    const unsigned v = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
    float f;
    memcpy(&f, &v, 4);
    return f;
}

struct PrimIn {
    const float4* tri_p;  // 3 per triangle
    const float4* sph;    // centre, radius
    int nt, ns;
};

__global__ void k_lb_bounds_init(unsigned* bounds) {
    const int k = threadIdx.x;
    if (k < 12) bounds[k] = ((k / 3) & 1) ? 0u : 0xFFFFFFFFu;  // min slots start high, max slots low
}

__global__ void k_lb_boxes(PrimIn in, float4* box_lo, float4* box_hi, float4* cen, unsigned* bounds) {
    const int n = in.nt + in.ns;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float bl[3], bh[3], c[3];
        if (i < in.nt) {
            const float4 a = in.tri_p[3 * i], b = in.tri_p[3 * i + 1], d = in.tri_p[3 * i + 2];
            bl[0] = fminf(fminf(a.x, b.x), d.x); bh[0] = fmaxf(fmaxf(a.x, b.x), d.x);
            bl[1] = fminf(fminf(a.y, b.y), d.y); bh[1] = fmaxf(fmaxf(a.y, b.y), d.y);
            bl[2] = fminf(fminf(a.z, b.z), d.z); bh[2] = fmaxf(fmaxf(a.z, b.z), d.z);
            for (int k = 0; k < 3; k++) c[k] = 0.5f * (bl[k] + bh[k]);
        } else {
            const float4 s = in.sph[i - in.nt];
            const float sc[3] = {s.x, s.y, s.z};
            for (int k = 0; k < 3; k++) {
                bl[k] = sc[k] - s.w;
                bh[k] = sc[k] + s.w;
                c[k] = sc[k];
            }
        }
        box_lo[i] = make_float4(bl[0], bl[1], bl[2], 0.f);
        box_hi[i] = make_float4(bh[0], bh[1], bh[2], 0.f);
        cen[i] = make_float4(c[0], c[1], c[2], 0.f);
        for (int k = 0; k < 3; k++) {
            lo[k] = fminf(lo[k], bl[k]);
            hi[k] = fmaxf(hi[k], bh[k]);
            clo[k] = fminf(clo[k], c[k]);
            chi[k] = fmaxf(chi[k], c[k]);
        }
    }
    for (int k = 0; k < 3; k++) {  // warp reduction, then one atomic per warp and value
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
            clo[k] = fminf(clo[k], __shfl_xor_sync(0xffffffffu, clo[k], o));
            chi[k] = fmaxf(chi[k], __shfl_xor_sync(0xffffffffu, chi[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; k++) {
            atomicMin(bounds + k, ord_float(lo[k]));
            atomicMax(bounds + 3 + k, ord_float(hi[k]));
            atomicMin(bounds + 6 + k, ord_float(clo[k]));
            atomicMax(bounds + 9 + k, ord_float(chi[k]));
        }
    }
}

__device__ __forceinline__ unsigned long long spread21(unsigned v) {  // 21 bits -> every third bit
    unsigned long long x = v & 0x1FFFFFu;
    x = (x | (x << 32)) & 0x1F00000000FFFFull;
    x = (x | (x << 16)) & 0x1F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

__global__ void k_lb_morton(const float4* cen, int n, const unsigned* bounds, unsigned long long* keys, int* ids) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 c = cen[i];
    const float cc[3] = {c.x, c.y, c.z};
    unsigned q[3];
    for (int k = 0; k < 3; k++) {
        const float lo = unord_float(bounds[6 + k]), hi = unord_float(bounds[9 + k]);
        const float ext = hi - lo;
        float u = ext > 0.f ? (cc[k] - lo) / ext : 0.f;
        u = fminf(fmaxf(u, 0.f), 1.f);
        q[k] = min(2097151u, (unsigned)(u * 2097152.f));
    }
    keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    ids[i] = i;
}

// Common-prefix length of sorted keys i and j (ties broken by index), -1 outside [0, n).
__device__ __forceinline__ int lb_delta(const unsigned long long* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const unsigned long long a = k[i], b = k[j];
    if (a == b) return 64 + __clz((unsigned)(i ^ j));
    return __clzll(a ^ b);
}

// Binary node ids: internal nodes 0 .. n-2, leaf e (sorted position e) = n - 1 + e.
__global__ void k_lb_tree(const unsigned long long* keys, int n, int* left, int* right, int* parent, int* first,
                          int* last) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = lb_delta(keys, n, i, i + 1) - lb_delta(keys, n, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = lb_delta(keys, n, i, i - d);
    int lmax = 2;
    while (lb_delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (lb_delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = lb_delta(keys, n, i, j);
    int s = 0;
    for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
        if (lb_delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    const int split = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    const int lc = lo == split ? n - 1 + split : split;
    const int rc = hi == split + 1 ? n - 1 + split + 1 : split + 1;
    left[i] = lc;
    right[i] = rc;
    parent[lc] = i;
    parent[rc] = i;
    first[i] = lo;
    last[i] = hi;
}

struct NodeBox {
    float4* lo;  // per binary node (internal and leaf); w = primitive count (int bits)
    float4* hi;
};

__global__ void k_lb_leaf_boxes(const int* ids, const float4* box_lo, const float4* box_hi, int n, NodeBox nb) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int p = ids[e];
    float4 lo = box_lo[p];
    lo.w = __int_as_float(1);
    nb.lo[n - 1 + e] = lo;
    nb.hi[n - 1 + e] = box_hi[p];
}

__global__ void k_lb_refit(int n, const int* left, const int* right, const int* parent, NodeBox nb, int* visits) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n || n == 1) return;
    int node = parent[n - 1 + e];
    while (true) {
        __threadfence();
        if (atomicAdd(visits + node, 1) == 0) return;  // the sibling subtree is not done yet
        __threadfence();
        const int a = left[node], b = right[node];
        const float4 la = nb.lo[a], ha = nb.hi[a], lb = nb.lo[b], hb = nb.hi[b];
        nb.lo[node] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z),
                                  __int_as_float(__float_as_int(la.w) + __float_as_int(lb.w)));
        nb.hi[node] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.f);
        if (node == 0) return;
        node = parent[node];
    }
}

__device__ __forceinline__ double box_area(float4 lo, float4 hi) {
    const double dx = (double)hi.x - lo.x, dy = (double)hi.y - lo.y, dz = (double)hi.z - lo.z;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

// Outward padding of a child box, as the host builder pads: (|coordinate| + abs_pad) * 2^-18
// in double, then one more float step outward.
__device__ __forceinline__ void pad_box(float4 lo, float4 hi, double abs_pad, float out_lo[3], float out_hi[3]) {
    const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
    for (int k = 0; k < 3; k++) {
        const double mag = fmax(fabs((double)l[k]), fabs((double)h[k]));
        const double pad = (mag + abs_pad) * (1.0 / 262144.0);
        out_lo[k] = nextafterf((float)((double)l[k] - pad), -INFINITY);
        out_hi[k] = nextafterf((float)((double)h[k] + pad), INFINITY);
    }
}

struct CollapseArgs {
    const int* left;
    const int* right;
    const int* first;  // every binary node: its first leaf entry
    NodeBox nb;
    int n;
    int max_leaf;
    double abs_pad;
    uint8_t* nodes;    // wide nodes
    const int2* qin;   // (binary node, wide index)
    int qn;
    int2* qout;
    int* qout_n;
    int* wide_count;
    int* max_leaf_seen;
};

template <int W>
__global__ void k_lb_collapse(CollapseArgs a) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.qn) return;
    const int2 job = a.qin[q];
    auto count_of = [&](int id) { return __float_as_int(a.nb.lo[id].w); };
    auto first_of = [&](int id) { return a.first[id]; };
    auto internal = [&](int id) { return id < a.n - 1; };
    int list[W];
    int cnt = 0;
    const int b = job.x;
    if (!internal(b) || count_of(b) <= a.max_leaf) {
        list[cnt++] = b;  // the whole tree is one leaf
    } else {
        list[cnt++] = a.left[b];
        list[cnt++] = a.right[b];
        while (cnt < W) {
            int pick = -1;
            double best = -1.0;
            for (int k = 0; k < cnt; k++) {
                const int c = list[k];
                if (internal(c) && count_of(c) > a.max_leaf) {
                    const double ar = box_area(a.nb.lo[c], a.nb.hi[c]);
                    if (ar > best) {
                        best = ar;
                        pick = k;
                    }
                }
            }
            if (pick < 0) break;
            const int c = list[pick];
            list[pick] = a.left[c];
            list[cnt++] = a.right[c];
        }
    }
    BvhNode<W> node;
    for (int k = 0; k < W; k++) {
        node.lo_x[k] = node.lo_y[k] = node.lo_z[k] = INFINITY;
        node.hi_x[k] = node.hi_y[k] = node.hi_z[k] = -INFINITY;
        node.child[k] = kEmptyChild;
    }
    for (int k = 0; k < (int)(sizeof(node.pad) / sizeof(int)); k++) node.pad[k] = 0;
    for (int k = 0; k < cnt; k++) {
        const int c = list[k];
        float lo[3], hi[3];
        pad_box(a.nb.lo[c], a.nb.hi[c], a.abs_pad, lo, hi);
        node.lo_x[k] = lo[0]; node.lo_y[k] = lo[1]; node.lo_z[k] = lo[2];
        node.hi_x[k] = hi[0]; node.hi_y[k] = hi[1]; node.hi_z[k] = hi[2];
        const int cc = count_of(c);
        if (!internal(c) || cc <= a.max_leaf) {
            node.child[k] = leaf_code(first_of(c), cc);
            atomicMax(a.max_leaf_seen, cc);
        } else {
            const int w = atomicAdd(a.wide_count, 1);
            node.child[k] = w;
            a.qout[atomicAdd(a.qout_n, 1)] = make_int2(c, w);
        }
    }
    reinterpret_cast<BvhNode<W>*>(a.nodes)[job.y] = node;
}

__global__ void k_lb_prims(const int* ids, int n, PrimIn in, float4* prims) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int p = ids[e];
    float4 r0, r1, r2;
    if (p < in.nt) {
        const float4 v0 = in.tri_p[3 * p], v1 = in.tri_p[3 * p + 1], v2 = in.tri_p[3 * p + 2];
        r0 = make_float4(v0.x, v0.y, v0.z, __int_as_float(p));
        // e1, e2: the single-precision subtractions Triangle::hit performs
        r1 = make_float4(__fsub_rn(v1.x, v0.x), __fsub_rn(v1.y, v0.y), __fsub_rn(v1.z, v0.z), 0.f);
        r2 = make_float4(__fsub_rn(v2.x, v0.x), __fsub_rn(v2.y, v0.y), __fsub_rn(v2.z, v0.z), 0.f);
    } else {
        const int si = p - in.nt;
        const float4 s = in.sph[si];
        r0 = make_float4(s.x, s.y, s.z, __int_as_float(~si));
        r1 = make_float4(s.w, 0.f, 0.f, 0.f);
        r2 = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    prims[3 * e] = r0;
    prims[3 * e + 1] = r1;
    prims[3 * e + 2] = r2;
}

template <class T>
cudaError_t grow(DevBuf& b, size_t count) {
    return b.alloc(count * sizeof(T));
}

// LBVH leaves are numbered in Morton order: leaf e starts at entry e.
__global__ void k_lb_leaf_first(int n, int* first) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) first[n - 1 + e] = e;
}

// ---- PLOC ----
constexpr int kPlocRadius = 16;

// Half the surface area of the union of two boxes (ordering only). Symmetric in its
// arguments, so both clusters of a pair compute the same value.
__device__ __forceinline__ float ploc_union_area(float4 alo, float4 ahi, float4 blo, float4 bhi) {
    const float dx = fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x);
    const float dy = fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y);
    const float dz = fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

// One cluster per primitive, in Morton order: binary leaf n - 1 + e and its box.
__global__ void k_ploc_init(int n, NodeBox nb, int* cnode, float4* clo, float4* chi) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    cnode[e] = n - 1 + e;
    clo[e] = nb.lo[n - 1 + e];
    chi[e] = nb.hi[n - 1 + e];
}

// Each cluster's nearest neighbour among the kPlocRadius clusters on either side. Pairs are
// ordered by (union area, lower index, higher index), a total order: scanning j upwards with
// a strict comparison keeps the smaller index on equal areas, which is the same order, so the
// pair that is smallest overall is always a mutual choice and every pass merges.
__global__ void k_ploc_nn(const float4* __restrict__ clo, const float4* __restrict__ chi, int m, int* nn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const float4 alo = clo[i], ahi = chi[i];
    float best = INFINITY;
    int bj = -1;
    const int j0 = max(0, i - kPlocRadius), j1 = min(m - 1, i + kPlocRadius);
    for (int j = j0; j <= j1; j++) {
        if (j == i) continue;
        const float a = ploc_union_area(alo, ahi, clo[j], chi[j]);
        if (a < best) {
            best = a;
            bj = j;
        }
    }
    nn[i] = bj;
}

// Mutual nearest neighbours i < j merge into a new internal node (ids n - 2 down to 0, so the
// last merge, the root, is node 0) that takes position i; position j is dropped. A cluster has
// one nearest neighbour, so it is in at most one pair, and the n - 1 merges of the whole build
// use exactly the ids n - 2 .. 0.
__global__ void k_ploc_merge(const int* __restrict__ nn, int m, const int* __restrict__ cnode,
                             const float4* __restrict__ clo, const float4* __restrict__ chi, int* next_id, int* left,
                             int* right, int* parent, NodeBox nb, int* keep, int* onode, float4* olo, float4* ohi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int j = nn[i];
    if (j >= 0 && nn[j] == i) {
        if (j < i) {
            keep[i] = 0;
            return;
        }
        const int id = atomicSub(next_id, 1) - 1;
        const int a = cnode[i], b = cnode[j];
        left[id] = a;
        right[id] = b;
        parent[a] = id;
        parent[b] = id;
        const float4 la = clo[i], ha = chi[i], lb = clo[j], hb = chi[j];
        const int cnt = __float_as_int(nb.lo[a].w) + __float_as_int(nb.lo[b].w);
        const float4 lo = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), __int_as_float(cnt));
        const float4 hi = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.f);
        nb.lo[id] = lo;
        nb.hi[id] = hi;
        keep[i] = 1;
        onode[i] = id;
        olo[i] = lo;
        ohi[i] = hi;
    } else {
        keep[i] = 1;
        onode[i] = cnode[i];
        olo[i] = clo[i];
        ohi[i] = chi[i];
    }
}

// The kept clusters, in order, into the next pass's arrays; the new count into *m_out.
__global__ void k_ploc_compact(const int* __restrict__ keep, const int* __restrict__ pos, int m,
                               const int* __restrict__ onode, const float4* __restrict__ olo,
                               const float4* __restrict__ ohi, int* cnode, float4* clo, float4* chi, int* m_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (i == m - 1) *m_out = pos[i] + keep[i];
    if (!keep[i]) return;
    const int k = pos[i];
    cnode[k] = onode[i];
    clo[k] = olo[i];
    chi[k] = ohi[i];
}

// The climbs below follow parent links that the merges wrote; each step checks the link
// (an internal node, a bounded number of steps) and raises *err instead of leaving the tree.
constexpr int kPlocMaxClimb = 1 << 16;

// Depth-first numbering of the leaves: a leaf's first entry is the primitive count of the
// left subtrees beside its path to the root (node 0).
__global__ void k_ploc_leaf_first(int n, const int* left, const int* parent, NodeBox nb, int* first, int* err) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    int node = n - 1 + e, pos = 0;
    for (int step = 0; node != 0; step++) {
        const int p = parent[node];
        if (p < 0 || p >= n - 1 || step >= kPlocMaxClimb) {
            atomicOr(err, 1);
            return;
        }
        if (left[p] != node) pos += __float_as_int(nb.lo[left[p]].w);
        node = p;
    }
    first[n - 1 + e] = pos;
}

// An internal node's first entry is its leftmost leaf's: each leaf climbs while it is a left
// child.
__global__ void k_ploc_node_first(int n, const int* left, const int* parent, int* first, int* err) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    int node = n - 1 + e;
    const int pos = first[node];
    for (int step = 0; node != 0; step++) {
        const int p = parent[node];
        if (p < 0 || p >= n - 1 || step >= kPlocMaxClimb) {
            atomicOr(err, 1);
            return;
        }
        if (left[p] != node) break;
        first[p] = pos;
        node = p;
    }
}

// Primitive ids in leaf-entry order: dfs_ids[first of leaf e] = sorted id e.
__global__ void k_ploc_order(int n, const int* sids, const int* first, int* dfs_ids, int* err) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int f = first[n - 1 + e];
    if (f < 0 || f >= n) {
        atomicOr(err, 1);
        return;
    }
    dfs_ids[f] = sids[e];
}

}  // namespace

cudaError_t gpu_build_bvh(const float4* tri_p, int nt, const float4* sph, int ns, int width, int max_leaf,
                          GpuBvhScratch& sc, DevBuf& nodes_out, DevBuf& prims_out, GpuBvhInfo& info,
                          cudaStream_t st, int algorithm) {
    const int n = nt + ns;
    if (n <= 0 || n >= (1 << 27) || max_leaf < 1 || max_leaf > kMaxLeafPrims ||
        (width != 2 && width != 4 && width != 8) || (algorithm != kGpuBvhLbvh && algorithm != kGpuBvhPloc))
        return cudaErrorInvalidValue;
    const bool ploc = algorithm == kGpuBvhPloc;
    cudaError_t e;
    if ((e = grow<float4>(sc.box_lo, n)) || (e = grow<float4>(sc.box_hi, n)) || (e = grow<float4>(sc.cen, n)) ||
        (e = grow<unsigned>(sc.bounds, 16)) || (e = grow<unsigned long long>(sc.keys, 2 * (size_t)n)) ||
        (e = grow<int>(sc.ids, 3 * (size_t)n)) || (e = grow<int>(sc.tree, 7 * (size_t)n + 4)) ||
        (e = grow<float4>(sc.nbox, 4 * (size_t)n)) || (e = grow<int>(sc.visits, n)) ||
        (e = grow<int2>(sc.queue, 2 * (size_t)n + 2)) || (e = grow<int>(sc.counters, 8)))
        return e;
    const size_t node_bytes = width == 2 ? sizeof(BvhNode<2>) : width == 4 ? sizeof(BvhNode<4>) : sizeof(BvhNode<8>);
    if ((e = nodes_out.alloc((size_t)n * node_bytes)) || (e = prims_out.alloc((size_t)n * 3 * sizeof(float4))))
        return e;
    const PrimIn in{tri_p, sph, nt, ns};
    unsigned* bounds = sc.bounds.as<unsigned>();
    k_lb_bounds_init<<<1, 32, 0, st>>>(bounds);
    k_lb_boxes<<<256, 256, 0, st>>>(in, sc.box_lo.as<float4>(), sc.box_hi.as<float4>(), sc.cen.as<float4>(), bounds);
    unsigned long long* keys = sc.keys.as<unsigned long long>();
    int* ids = sc.ids.as<int>();
    const int gb = (n + 255) / 256;
    k_lb_morton<<<gb, 256, 0, st>>>(sc.cen.as<float4>(), n, bounds, keys, ids);
    // sort (key, id) pairs by key into the second halves
    size_t tmp = 0;
    if ((e = cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys + n, ids, ids + n, n, 0, 64, st))) return e;
    if ((e = sc.sort_tmp.alloc(tmp + 16))) return e;
    if ((e = cub::DeviceRadixSort::SortPairs(sc.sort_tmp.p, tmp, keys, keys + n, ids, ids + n, n, 0, 64, st)))
        return e;
    const unsigned long long* skeys = keys + n;
    const int* sids = ids + n;
    int* left = sc.tree.as<int>();  // n - 1 internal nodes
    int* right = left + n;
    int* parent = right + n;        // 2n - 1 binary nodes
    int* first = parent + 2 * n;    // 2n - 1 binary nodes: first leaf entry
    int* last = first + 2 * n;      // internal nodes: range end (LBVH)
    const NodeBox nb{sc.nbox.as<float4>(), sc.nbox.as<float4>() + 2 * (size_t)n};
    k_lb_leaf_boxes<<<gb, 256, 0, st>>>(sids, sc.box_lo.as<float4>(), sc.box_hi.as<float4>(), n, nb);
    const int* entry_ids = sids;  // primitive of each leaf entry
    if (!ploc) {
        if (n > 1) k_lb_tree<<<(n - 1 + 255) / 256, 256, 0, st>>>(skeys, n, left, right, parent, first, last);
        k_lb_leaf_first<<<gb, 256, 0, st>>>(n, first);
        if ((e = cudaMemsetAsync(sc.visits.p, 0, (size_t)n * sizeof(int), st))) return e;
        k_lb_refit<<<gb, 256, 0, st>>>(n, left, right, parent, nb, sc.visits.as<int>());
    } else {
        if ((e = grow<float4>(sc.cbox, 6 * (size_t)n)) || (e = grow<int>(sc.cint, 7 * (size_t)n + 8))) return e;
        float4* clo[2] = {sc.cbox.as<float4>(), sc.cbox.as<float4>() + n};
        float4* chi[2] = {clo[1] + n, clo[1] + 2 * (size_t)n};
        float4* olo = chi[1] + n;
        float4* ohi = olo + n;
        int* cnode[2] = {sc.cint.as<int>(), sc.cint.as<int>() + n};
        int* nn = cnode[1] + n;
        int* keep = nn + n;
        int* pos = keep + n;
        int* onode = pos + n;
        int* ctr = onode + n;  // [0] next internal id, [1] next cluster count, [2] tree error
        size_t stmp = 0;
        if ((e = cub::DeviceScan::ExclusiveSum(nullptr, stmp, keep, pos, n, st))) return e;
        if ((e = sc.scan_tmp.alloc(stmp + 16))) return e;
        k_ploc_init<<<gb, 256, 0, st>>>(n, nb, cnode[0], clo[0], chi[0]);
        if ((e = cudaMemsetAsync(parent, 0xFF, 2 * (size_t)n * sizeof(int), st))) return e;  // -1: none
        if ((e = cudaMemsetAsync(first, 0xFF, 2 * (size_t)n * sizeof(int), st))) return e;
        const int ctr0[3] = {n - 1, 0, 0};
        if ((e = cudaMemcpyAsync(ctr, ctr0, sizeof(ctr0), cudaMemcpyHostToDevice, st))) return e;
        int m = n, cur = 0, passes = 0;
        while (m > 1) {
            if (++passes > 4096) return cudaErrorInvalidValue;  // every pass merges at least one pair
            const int g = (m + 255) / 256;
            k_ploc_nn<<<g, 256, 0, st>>>(clo[cur], chi[cur], m, nn);
            k_ploc_merge<<<g, 256, 0, st>>>(nn, m, cnode[cur], clo[cur], chi[cur], ctr, left, right, parent, nb, keep,
                                            onode, olo, ohi);
            if ((e = cub::DeviceScan::ExclusiveSum(sc.scan_tmp.p, stmp, keep, pos, m, st))) return e;
            k_ploc_compact<<<g, 256, 0, st>>>(keep, pos, m, onode, olo, ohi, cnode[cur ^ 1], clo[cur ^ 1],
                                              chi[cur ^ 1], ctr + 1);
            int m2 = 0;
            if ((e = cudaMemcpyAsync(&m2, ctr + 1, sizeof(int), cudaMemcpyDeviceToHost, st))) return e;
            if ((e = cudaStreamSynchronize(st))) return e;
            if (m2 >= m || m2 < 1) return cudaErrorInvalidValue;
            m = m2;
            cur ^= 1;
        }
        k_ploc_leaf_first<<<gb, 256, 0, st>>>(n, left, parent, nb, first, ctr + 2);
        k_ploc_node_first<<<gb, 256, 0, st>>>(n, left, parent, first, ctr + 2);
        int* dfs_ids = ids + 2 * (size_t)n;
        k_ploc_order<<<gb, 256, 0, st>>>(n, sids, first, dfs_ids, ctr + 2);
        int terr = 0;
        if ((e = cudaMemcpyAsync(&terr, ctr + 2, sizeof(int), cudaMemcpyDeviceToHost, st))) return e;
        if ((e = cudaStreamSynchronize(st))) return e;
        if (terr) return cudaErrorInvalidValue;
        entry_ids = dfs_ids;
    }
    k_lb_prims<<<gb, 256, 0, st>>>(entry_ids, n, in, prims_out.as<float4>());
    // abs_pad = 1e-3 x the scene diagonal, as the host builder
    unsigned hb[6];
    if ((e = cudaMemcpyAsync(hb, bounds, sizeof(hb), cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    double diag = 0;
    for (int k = 0; k < 3; k++) {
        const double ext = (double)unord_float(hb[3 + k]) - unord_float(hb[k]);
        diag += ext * ext;
    }
    const double abs_pad = 1e-3 * std::sqrt(diag);
    // top-down collapse, one tree level per launch
    int* cnt = sc.counters.as<int>();  // [0] wide nodes, [1] next queue length, [2] largest leaf
    int2* qa = sc.queue.as<int2>();
    int2* qb = qa + n + 1;
    const int one = 1;
    const int2 root = make_int2(0, 0);
    if ((e = cudaMemsetAsync(cnt, 0, 8 * sizeof(int), st))) return e;
    if ((e = cudaMemcpyAsync(cnt, &one, sizeof(int), cudaMemcpyHostToDevice, st))) return e;
    if ((e = cudaMemcpyAsync(qa, &root, sizeof(int2), cudaMemcpyHostToDevice, st))) return e;
    int qn = 1, depth = 0;
    while (qn > 0) {
        if (++depth > 64) return cudaErrorInvalidValue;  // a tree over < 2^27 primitives is shallower
        if ((e = cudaMemsetAsync(cnt + 1, 0, sizeof(int), st))) return e;
        const CollapseArgs a{left, right, first, nb, n, max_leaf, abs_pad, nodes_out.as<uint8_t>(), qa, qn, qb,
                             cnt + 1, cnt, cnt + 2};
        const int g = (qn + 127) / 128;
        if (width == 2) k_lb_collapse<2><<<g, 128, 0, st>>>(a);
        else if (width == 4) k_lb_collapse<4><<<g, 128, 0, st>>>(a);
        else k_lb_collapse<8><<<g, 128, 0, st>>>(a);
        if ((e = cudaMemcpyAsync(&qn, cnt + 1, sizeof(int), cudaMemcpyDeviceToHost, st))) return e;
        if ((e = cudaStreamSynchronize(st))) return e;
        int2* t = qa;
        qa = qb;
        qb = t;
    }
    int hc[3];
    if ((e = cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    info.root = 0;
    info.num_nodes = hc[0];
    info.depth = depth;
    info.max_leaf = hc[2];
    info.width = width;
    return cudaGetLastError();
}

namespace {

// One node per thread: per axis the origin is the smallest child lower plane, the scale the
// smallest power of two whose 255 steps reach the largest upper plane; each plane's q is then
// stepped until fmaf(q, scale, origin) lies outside the float plane (down for lower planes,
// up for upper planes). A larger scale is tried when an upper plane does not fit.
template <int W>
__global__ void k_quantize_nodes(const BvhNode<W>* __restrict__ in, int n, uint32_t* __restrict__ out, int* fail) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BvhNode<W> nd = in[i];
    uint32_t qb[6 * W / 4];
    for (int j = 0; j < 6 * W / 4; j++) qb[j] = 0u;
    float org[3] = {0.f, 0.f, 0.f};
    uint32_t ex[3] = {1u, 1u, 1u};
    bool all_ok = true;
    for (int a = 0; a < 3; a++) {
        const float* lo = a == 0 ? nd.lo_x : a == 1 ? nd.lo_y : nd.lo_z;
        const float* hi = a == 0 ? nd.hi_x : a == 1 ? nd.hi_y : nd.hi_z;
        float o = __int_as_float(0x7f800000), m = -__int_as_float(0x7f800000);
        bool any = false;
        for (int k = 0; k < W; k++)
            if (nd.child[k] != kEmptyChild) {
                o = fminf(o, lo[k]);
                m = fmaxf(m, hi[k]);
                any = true;
            }
        if (!any) o = m = 0.f;
        const double ext = (double)m - (double)o;
        int e = ext > 0.0 ? (int)ceil(log2(ext / 255.0)) + 127 : 1;
        e = e < 1 ? 1 : e > 254 ? 254 : e;
        bool ok = false;
        uint8_t ql[W], qh[W];
        for (; e <= 254 && !ok; e++) {
            const float sc = __uint_as_float((uint32_t)e << 23);
            ok = true;
            for (int k = 0; k < W; k++) {
                ql[k] = qh[k] = 0;
                if (nd.child[k] == kEmptyChild) continue;
                int l = (int)floor(((double)lo[k] - (double)o) / (double)sc);
                l = l < 0 ? 0 : l > 255 ? 255 : l;
                while (l > 0 && __fmaf_rn((float)l, sc, o) > lo[k]) l--;
                int h = (int)ceil(((double)hi[k] - (double)o) / (double)sc);
                h = h < 0 ? 0 : h;
                if (h > 255) {
                    ok = false;
                    break;
                }
                while (h < 255 && __fmaf_rn((float)h, sc, o) < hi[k]) h++;
                if (__fmaf_rn((float)l, sc, o) > lo[k] || __fmaf_rn((float)h, sc, o) < hi[k]) {
                    ok = false;
                    break;
                }
                ql[k] = (uint8_t)l;
                qh[k] = (uint8_t)h;
            }
            if (ok) ex[a] = (uint32_t)e;
        }
        if (!ok) all_ok = false;
        org[a] = o;
        for (int k = 0; k < W; k++) {
            const int bl = (2 * a) * W + k, bh = (2 * a + 1) * W + k;
            qb[bl / 4] |= (uint32_t)ql[k] << (8 * (bl & 3));
            qb[bh / 4] |= (uint32_t)qh[k] << (8 * (bh & 3));
        }
    }
    if (!all_ok) atomicOr(fail, 1);
    uint32_t* w = out + (size_t)i * (qnode_bytes(W) / 4);
    w[0] = __float_as_uint(org[0]);
    w[1] = __float_as_uint(org[1]);
    w[2] = __float_as_uint(org[2]);
    w[3] = ex[0] | (ex[1] << 8) | (ex[2] << 16);
    for (int j = 0; j < 6 * W / 4; j++) w[4 + j] = qb[j];
    for (int k = 0; k < W; k++) w[qnode_child_offset(W) / 4 + k] = (uint32_t)nd.child[k];
    for (int j = qnode_child_offset(W) / 4 + W; j < qnode_bytes(W) / 4; j++) w[j] = 0u;
}

}  // namespace

// Triangle leaf entries for the watertight test: (p0, id) (p1) (p2), the original vertices
// (tri_p, 3 float4 per triangle) in place of the edges e1, e2; sphere entries are unchanged.
// Shared vertices keep their exact values, which the test's watertightness relies on.
__global__ void k_prims_vertices(float4* __restrict__ prims, int n, const float4* __restrict__ tri_p) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int id = __float_as_int(prims[3 * e].w);
    if (id < 0) return;
    prims[3 * e + 1] = tri_p[3 * (size_t)id + 1];
    prims[3 * e + 2] = tri_p[3 * (size_t)id + 2];
}

cudaError_t prims_to_vertices(float4* prims, int n, const float4* tri_p, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_prims_vertices<<<(n + 255) / 256, 256, 0, st>>>(prims, n, tri_p);
    return cudaGetLastError();
}

cudaError_t quantize_bvh_nodes(const void* nodes, int num_nodes, int width, void* out, int* fail,
                               cudaStream_t stream) {
    if (num_nodes <= 0) return cudaSuccess;
    const int blocks = (num_nodes + 127) / 128;
    if (width == 4)
        k_quantize_nodes<4><<<blocks, 128, 0, stream>>>(static_cast<const BvhNode<4>*>(nodes), num_nodes,
                                                       static_cast<uint32_t*>(out), fail);
    else if (width == 8)
        k_quantize_nodes<8><<<blocks, 128, 0, stream>>>(static_cast<const BvhNode<8>*>(nodes), num_nodes,
                                                       static_cast<uint32_t*>(out), fail);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace pt
