#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <thread>

namespace pt {

namespace {

struct Box {
    float lo[3] = {std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
                   std::numeric_limits<float>::infinity()};
    float hi[3] = {-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
                   -std::numeric_limits<float>::infinity()};
    void grow(const Box& b) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], b.lo[k]);
            hi[k] = std::max(hi[k], b.hi[k]);
        }
    }
    void grow(const float* p) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], p[k]);
            hi[k] = std::max(hi[k], p[k]);
        }
    }
    bool empty() const { return !(lo[0] <= hi[0]); }
    double area() const {
        if (empty()) return 0.0;
        const double dx = (double)hi[0] - lo[0], dy = (double)hi[1] - lo[1], dz = (double)hi[2] - lo[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct Node2 {
    Box box;
    int left = -1, right = -1;
    int first = 0, count = 0;  // leaf when count > 0
};

constexpr int kBins = 32;
constexpr int kMaxDepth2 = 56;

struct Builder {
    const std::vector<Box>& pbox;
    const std::vector<float>& cen;  // 3 per prim
    std::vector<int>& idx;
    std::vector<Node2>& nodes;
    std::atomic<int>& next;
    int max_leaf;

    void make_leaf(int id, int begin, int end, const Box& b) {
        Node2& n = nodes[id];
        n.box = b;
        n.first = begin;
        n.count = end - begin;
    }

    void build(int id, int begin, int end, int depth, int par_budget) {
        Box b, cb;
        for (int i = begin; i < end; i++) {
            b.grow(pbox[idx[i]]);
            cb.grow(&cen[(size_t)idx[i] * 3]);
        }
        const int n = end - begin;
        if (n == 1) { make_leaf(id, begin, end, b); return; }

        int best_axis = -1, best_bin = -1;
        double best_cost = std::numeric_limits<double>::infinity();
        if (depth < kMaxDepth2) {
            for (int axis = 0; axis < 3; axis++) {
                const double ext = (double)cb.hi[axis] - cb.lo[axis];
                if (!(ext > 0)) continue;
                Box bins[kBins];
                int cnt[kBins] = {0};
                const double scale = kBins / ext;
                for (int i = begin; i < end; i++) {
                    int k = (int)(((double)cen[(size_t)idx[i] * 3 + axis] - cb.lo[axis]) * scale);
                    k = std::min(kBins - 1, std::max(0, k));
                    cnt[k]++;
                    bins[k].grow(pbox[idx[i]]);
                }
                double right_area[kBins];
                int right_cnt[kBins];
                Box acc;
                int c = 0;
                for (int k = kBins - 1; k > 0; k--) {
                    acc.grow(bins[k]);
                    c += cnt[k];
                    right_area[k] = acc.area();
                    right_cnt[k] = c;
                }
                Box lacc;
                int lc = 0;
                for (int k = 0; k < kBins - 1; k++) {
                    lacc.grow(bins[k]);
                    lc += cnt[k];
                    if (lc == 0 || right_cnt[k + 1] == 0) continue;
                    const double cost = lacc.area() * lc + right_area[k + 1] * right_cnt[k + 1];
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = axis;
                        best_bin = k;
                    }
                }
            }
        }
        const double area = b.area();
        const double split_cost = best_axis >= 0 && area > 0 ? 1.0 + best_cost / area : 1e300;
        if (n <= max_leaf && (double)n <= split_cost) { make_leaf(id, begin, end, b); return; }

        int mid;
        if (best_axis >= 0) {
            const double ext = (double)cb.hi[best_axis] - cb.lo[best_axis];
            const double scale = kBins / ext;
            const int axis = best_axis;
            auto* it = std::partition(idx.data() + begin, idx.data() + end, [&](int p) {
                int k = (int)(((double)cen[(size_t)p * 3 + axis] - cb.lo[axis]) * scale);
                k = std::min(kBins - 1, std::max(0, k));
                return k <= best_bin;
            });
            mid = (int)(it - idx.data());
            if (mid == begin || mid == end) mid = begin + n / 2;
        } else {
            if (n <= max_leaf) { make_leaf(id, begin, end, b); return; }
            // centroids coincide (or depth limit): median split along the widest axis
            int axis = 0;
            for (int k = 1; k < 3; k++)
                if (cb.hi[k] - cb.lo[k] > cb.hi[axis] - cb.lo[axis]) axis = k;
            mid = begin + n / 2;
            std::nth_element(idx.data() + begin, idx.data() + mid, idx.data() + end,
                             [&](int a, int c) { return cen[(size_t)a * 3 + axis] < cen[(size_t)c * 3 + axis]; });
        }
        const int left = next.fetch_add(2);
        const int right = left + 1;
        nodes[id].box = b;
        nodes[id].left = left;
        nodes[id].right = right;
        nodes[id].count = 0;
        if (par_budget > 0 && n > 65536) {
            auto fut = std::async(std::launch::async, [&, left, begin, mid, depth, par_budget] {
                build(left, begin, mid, depth + 1, par_budget / 2);
            });
            build(right, mid, end, depth + 1, par_budget / 2);
            fut.get();
        } else {
            build(left, begin, mid, depth + 1, 0);
            build(right, mid, end, depth + 1, 0);
        }
    }
};

// Pad a box outward so that FP rounding in the primitive tests cannot put a reported hit
// outside it (a few tens of ulps of the coordinate magnitudes).
void padded(const Box& b, double abs_pad, float lo[3], float hi[3]) {
    for (int k = 0; k < 3; k++) {
        const double mag = std::max(std::fabs((double)b.lo[k]), std::fabs((double)b.hi[k]));
        const double pad = (mag + abs_pad) * (1.0 / 262144.0);
        lo[k] = std::nextafter((float)((double)b.lo[k] - pad), -std::numeric_limits<float>::infinity());
        hi[k] = std::nextafter((float)((double)b.hi[k] + pad), std::numeric_limits<float>::infinity());
    }
}

template <int W>
struct Collapser {
    const std::vector<Node2>& n2;
    std::vector<BvhNode<W>>& out;
    double abs_pad;
    int max_depth = 0;
    int max_leaf = 0;

    int collapse(int id, int depth) {
        max_depth = std::max(max_depth, depth);
        int list[W];
        int cnt = 0;
        if (n2[id].count > 0) {
            list[cnt++] = id;  // single leaf root
        } else {
            list[cnt++] = n2[id].left;
            list[cnt++] = n2[id].right;
            while (cnt < W) {
                int pick = -1;
                double best = -1;
                for (int k = 0; k < cnt; k++) {
                    if (n2[list[k]].count == 0) {
                        const double a = n2[list[k]].box.area();
                        if (a > best) { best = a; pick = k; }
                    }
                }
                if (pick < 0) break;
                const int c = list[pick];
                list[pick] = n2[c].left;
                list[cnt++] = n2[c].right;
            }
        }
        const int me = (int)out.size();
        out.emplace_back();
        BvhNode<W> node;
        std::memset(&node, 0, sizeof(node));
        for (int k = 0; k < W; k++) {
            node.lo_x[k] = node.lo_y[k] = node.lo_z[k] = std::numeric_limits<float>::infinity();
            node.hi_x[k] = node.hi_y[k] = node.hi_z[k] = -std::numeric_limits<float>::infinity();
            node.child[k] = kEmptyChild;
        }
        for (int k = 0; k < cnt; k++) {
            const Node2& c = n2[list[k]];
            float lo[3], hi[3];
            padded(c.box, abs_pad, lo, hi);
            node.lo_x[k] = lo[0]; node.lo_y[k] = lo[1]; node.lo_z[k] = lo[2];
            node.hi_x[k] = hi[0]; node.hi_y[k] = hi[1]; node.hi_z[k] = hi[2];
            if (c.count > 0) {
                node.child[k] = leaf_code(c.first, c.count);
                max_leaf = std::max(max_leaf, c.count);
            } else {
                node.child[k] = collapse(list[k], depth + 1);
            }
        }
        out[me] = node;
        return me;
    }
};

template <int W>
void collapse_into(const std::vector<Node2>& n2, double abs_pad, BvhBuild& out) {
    std::vector<BvhNode<W>> wide;
    wide.reserve(n2.size() / 2 + 1);
    Collapser<W> c{n2, wide, abs_pad};
    out.root = c.collapse(0, 1);
    out.depth = c.max_depth;
    out.max_leaf = c.max_leaf;
    out.num_nodes = (int)wide.size();
    out.nodes.resize(wide.size() * sizeof(BvhNode<W>));
    std::memcpy(out.nodes.data(), wide.data(), out.nodes.size());
}

inline float bits_to_float(int v) {
    float f;
    std::memcpy(&f, &v, 4);
    return f;
}

}  // namespace

bool build_bvh(const HostScene& s, int width, int max_leaf, BvhBuild& out, std::string& err) {
    const auto t0 = std::chrono::steady_clock::now();
    if (width != 2 && width != 4 && width != 8) {
        err = "BVH width must be 2, 4 or 8";
        return false;
    }
    if (max_leaf < 1 || max_leaf > kMaxLeafPrims) {
        err = "BVH leaf size must be in [1, 16]";
        return false;
    }
    const int nt = s.num_tri(), ns = s.num_sph();
    const int n = nt + ns;
    if (n == 0) {
        err = "scene has no primitives";
        return false;
    }
    if (n >= (1 << 27)) {
        err = "scene has too many primitives for the leaf encoding";
        return false;
    }
    std::vector<Box> pbox(n);
    std::vector<float> cen((size_t)n * 3);
    Box scene;
    for (int i = 0; i < nt; i++) {
        Box b;
        for (int v = 0; v < 3; v++) b.grow(&s.tri_p[(size_t)i * 9 + v * 3]);
        pbox[i] = b;
        for (int k = 0; k < 3; k++) cen[(size_t)i * 3 + k] = 0.5f * (b.lo[k] + b.hi[k]);
        scene.grow(b);
    }
    for (int i = 0; i < ns; i++) {
        const float* sp = &s.sph[(size_t)i * 4];
        Box b;
        for (int k = 0; k < 3; k++) {
            b.lo[k] = sp[k] - sp[3];
            b.hi[k] = sp[k] + sp[3];
        }
        pbox[nt + i] = b;
        for (int k = 0; k < 3; k++) cen[(size_t)(nt + i) * 3 + k] = sp[k];
        scene.grow(b);
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::vector<Node2> n2((size_t)2 * n + 1);
    std::atomic<int> next{1};
    Builder b{pbox, cen, idx, n2, next, max_leaf};
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    b.build(0, 0, n, 0, (int)hw);
    n2.resize(next.load());

    double diag = 0;
    for (int k = 0; k < 3; k++) diag += ((double)scene.hi[k] - scene.lo[k]) * ((double)scene.hi[k] - scene.lo[k]);
    const double abs_pad = 1e-3 * std::sqrt(diag);
    out = BvhBuild();
    out.width = width;
    if (width == 2) collapse_into<2>(n2, abs_pad, out);
    else if (width == 4) collapse_into<4>(n2, abs_pad, out);
    else collapse_into<8>(n2, abs_pad, out);

    out.prims.resize((size_t)n * 12);
    out.prim_order.resize(n);
    for (int e = 0; e < n; e++) {
        const int p = idx[e];
        float* r = &out.prims[(size_t)e * 12];
        std::memset(r, 0, 12 * sizeof(float));
        if (p < nt) {
            const float* v = &s.tri_p[(size_t)p * 9];
            r[0] = v[0]; r[1] = v[1]; r[2] = v[2]; r[3] = bits_to_float(p);
            r[4] = v[3] - v[0]; r[5] = v[4] - v[1]; r[6] = v[5] - v[2];
            r[8] = v[6] - v[0]; r[9] = v[7] - v[1]; r[10] = v[8] - v[2];
            out.prim_order[e] = p;
        } else {
            const int si = p - nt;
            const float* sp = &s.sph[(size_t)si * 4];
            r[0] = sp[0]; r[1] = sp[1]; r[2] = sp[2]; r[3] = bits_to_float(~si);
            r[4] = sp[3];
            out.prim_order[e] = ~si;
        }
    }
    // SAH cost of the binary tree (traversal 1, intersection 1), for reporting.
    double cost = 0;
    const double ra = n2[0].box.area() > 0 ? n2[0].box.area() : 1.0;
    for (const Node2& nd : n2) cost += nd.box.area() / ra * (nd.count > 0 ? nd.count : 1.0);
    out.sah_cost = cost;
    out.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return true;
}

namespace {
template <int W>
bool check_wide(const HostScene& s, const BvhBuild& b, std::string& err) {
    const BvhNode<W>* nodes = reinterpret_cast<const BvhNode<W>*>(b.nodes.data());
    const int n = s.num_tri() + s.num_sph();
    std::vector<int> seen(n, 0);
    struct Item { int node; float lo[3], hi[3]; };
    std::vector<Item> stack;
    Item root{b.root, {-INFINITY, -INFINITY, -INFINITY}, {INFINITY, INFINITY, INFINITY}};
    stack.push_back(root);
    auto inside = [](const float* p, const float* lo, const float* hi) {
        for (int k = 0; k < 3; k++)
            if (p[k] < lo[k] || p[k] > hi[k]) return false;
        return true;
    };
    while (!stack.empty()) {
        Item it = stack.back();
        stack.pop_back();
        if (it.node < 0 || it.node >= b.num_nodes) { err = "child index out of range"; return false; }
        const BvhNode<W>& nd = nodes[it.node];
        for (int k = 0; k < W; k++) {
            const int c = nd.child[k];
            if (c == kEmptyChild) continue;
            const float lo[3] = {nd.lo_x[k], nd.lo_y[k], nd.lo_z[k]};
            const float hi[3] = {nd.hi_x[k], nd.hi_y[k], nd.hi_z[k]};
            if (child_is_leaf(c)) {
                const int first = leaf_first(c), cnt = leaf_count(c);
                if (first < 0 || first + cnt > n) { err = "leaf range out of bounds"; return false; }
                for (int e = first; e < first + cnt; e++) {
                    const int p = b.prim_order[e];
                    if (p >= 0) {
                        if (p >= s.num_tri()) { err = "triangle id out of range"; return false; }
                        seen[p]++;
                        for (int v = 0; v < 3; v++)
                            if (!inside(&s.tri_p[(size_t)p * 9 + v * 3], lo, hi) ||
                                !inside(&s.tri_p[(size_t)p * 9 + v * 3], it.lo, it.hi)) {
                                err = "triangle outside its leaf box";
                                return false;
                            }
                    } else {
                        const int si = ~p;
                        if (si >= s.num_sph()) { err = "sphere id out of range"; return false; }
                        seen[s.num_tri() + si]++;
                        const float* sp = &s.sph[(size_t)si * 4];
                        const float slo[3] = {sp[0] - sp[3], sp[1] - sp[3], sp[2] - sp[3]};
                        const float shi[3] = {sp[0] + sp[3], sp[1] + sp[3], sp[2] + sp[3]};
                        if (!inside(slo, lo, hi) || !inside(shi, lo, hi)) {
                            err = "sphere outside its leaf box";
                            return false;
                        }
                    }
                }
            } else {
                Item ch{c, {lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}};
                stack.push_back(ch);
            }
        }
    }
    for (int i = 0; i < n; i++)
        if (seen[i] != 1) { err = "primitive " + std::to_string(i) + " referenced " + std::to_string(seen[i]) + " times"; return false; }
    return true;
}
}  // namespace

bool check_bvh(const HostScene& s, const BvhBuild& b, std::string& err) {
    if (b.width == 2) return check_wide<2>(s, b, err);
    if (b.width == 4) return check_wide<4>(s, b, err);
    if (b.width == 8) return check_wide<8>(s, b, err);
    err = "bad width";
    return false;
}

// Append `b` (a scene's own BVH over its own primitive ids) to `into`, the BVH of a batch
// whose scenes share one node array, one leaf-entry array and one id space: internal child
// indices move by the node count already present, leaf ranges by the leaf entries present,
// triangle and sphere ids by the scene's first triangle and sphere. Returns the scene's root.
template <int W>
static int append_nodes(const BvhBuild& b, int node_base, int entry_base, BvhBuild& into) {
    const size_t nbytes = sizeof(BvhNode<W>);
    const size_t old = into.nodes.size();
    into.nodes.resize(old + (size_t)b.num_nodes * nbytes);
    for (int i = 0; i < b.num_nodes; i++) {
        BvhNode<W> nd;
        std::memcpy(&nd, b.nodes.data() + (size_t)i * nbytes, nbytes);
        for (int k = 0; k < W; k++) {
            const int c = nd.child[k];
            if (c == kEmptyChild) continue;
            if (child_is_leaf(c)) nd.child[k] = leaf_code(leaf_first(c) + entry_base, leaf_count(c));
            else nd.child[k] = c + node_base;
        }
        std::memcpy(into.nodes.data() + old + (size_t)i * nbytes, &nd, nbytes);
    }
    return b.root + node_base;
}

int append_bvh(const BvhBuild& b, int tri_base, int sph_base, BvhBuild& into) {
    const int node_base = into.num_nodes;
    const int entry_base = (int)(into.prims.size() / 12);
    if (node_base == 0 && into.prims.empty()) into.width = b.width;
    int root = 0;
    if (b.width == 2) root = append_nodes<2>(b, node_base, entry_base, into);
    else if (b.width == 4) root = append_nodes<4>(b, node_base, entry_base, into);
    else root = append_nodes<8>(b, node_base, entry_base, into);
    const size_t old = into.prims.size();
    into.prims.insert(into.prims.end(), b.prims.begin(), b.prims.end());
    for (size_t e = 0; e < b.prims.size() / 12; e++) {
        float* r = &into.prims[old + e * 12];
        int id;
        std::memcpy(&id, &r[3], 4);
        id = id >= 0 ? id + tri_base : ~(~id + sph_base);
        std::memcpy(&r[3], &id, 4);
        const int po = b.prim_order[e];
        into.prim_order.push_back(po >= 0 ? po + tri_base : ~(~po + sph_base));
    }
    into.num_nodes += b.num_nodes;
    into.depth = std::max(into.depth, b.depth);
    into.max_leaf = std::max(into.max_leaf, b.max_leaf);
    into.build_ms += b.build_ms;
    return root;
}

}  // namespace pt

namespace pt {

bool check_qnodes(const BvhBuild& b, const std::vector<uint8_t>& q, std::string& err) {
    const int w = b.width;
    if (w != 4 && w != 8) {
        err = "quantized nodes exist for widths 4 and 8";
        return false;
    }
    const size_t fb = w == 4 ? sizeof(BvhNode<4>) : sizeof(BvhNode<8>), qb = (size_t)qnode_bytes(w);
    if (b.nodes.size() != (size_t)b.num_nodes * fb || q.size() != (size_t)b.num_nodes * qb) {
        err = "node arrays have unexpected sizes";
        return false;
    }
    for (int i = 0; i < b.num_nodes; i++) {
        const float* f = reinterpret_cast<const float*>(b.nodes.data() + (size_t)i * fb);
        const uint8_t* n = q.data() + (size_t)i * qb;
        float org[3];
        uint32_t e;
        std::memcpy(org, n, 12);
        std::memcpy(&e, n + 12, 4);
        for (int k = 0; k < w; k++) {
            int fc, qc;
            std::memcpy(&fc, f + 6 * w + k, 4);
            std::memcpy(&qc, n + qnode_child_offset(w) + 4 * k, 4);
            if (fc != qc) {
                err = "node " + std::to_string(i) + ": child codes differ";
                return false;
            }
            if (fc == kEmptyChild) continue;
            for (int a = 0; a < 3; a++) {
                float sc;
                const uint32_t bits = ((e >> (8 * a)) & 0xFFu) << 23;
                std::memcpy(&sc, &bits, 4);
                const float lo = std::fmaf((float)n[16 + (2 * a) * w + k], sc, org[a]);
                const float hi = std::fmaf((float)n[16 + (2 * a + 1) * w + k], sc, org[a]);
                if (!(lo <= f[(2 * a) * w + k]) || !(hi >= f[(2 * a + 1) * w + k])) {
                    err = "node " + std::to_string(i) + " child " + std::to_string(k) + ": quantized box does not "
                          "contain the float box";
                    return false;
                }
            }
        }
    }
    return true;
}

}  // namespace pt
