// Wavefront path integrator: the reference's per-pixel megakernel
// (src/renderers/path_tracer.cu:142-264) split into stages over SoA ray queues.
//
//   camera   one thread per path of the wave: PCG stream, generateRay, queue slot
//   extend   persistent: closest hit for every queued ray (BVH, shared-memory stack)
//   sort     optional: bucket the queue by material class (miss, Lambert, mirror, glass,
//            Beckmann) so each warp of the shade stage runs one BSDF
//   shade    persistent: emission with MIS, BSDF sample, emitter sample (NEE) -> shadow
//            queue, continuation ray -> next queue (warp ballot/popc compaction)
//   shadow   persistent: any-hit for every shadow ray; unoccluded ones add their
//            contribution to the path radiance
//   accumulate  per pixel: mean over the frame's samples and the running mean across frames
//            (src/framebuffer.cu:7-41)
//
// Per bounce the reference traces the BSDF direction twice: directSampleBSDF with tMin 1e-4
// for the MIS emission term (path_tracer.cu:51) and the continuation with tMin 1e-3 (:177).
// Here the extend stage traces it once with tMin 1e-4. That hit serves both unless it lies
// closer than 1e-3: the closest hit at or beyond 1e-4 that is also at or beyond 1e-3 is the
// closest hit beyond 1e-3. Only then is the direction traced again from 1e-3, and the shade
// stage takes the emission term from the first hit and the next vertex from the second, as
// the reference does. With NEE off (calculateLiNaive, :186-233) there is one trace at 1e-3.
#include "wavefront.h"

#include <algorithm>
#include <cfloat>
#include <mutex>

#include "dev_math.cuh"
#include "dev_shade.cuh"
#include "dev_trace.cuh"
#include "guide_mlp.cuh"
#include "guide_tc.cuh"

#include <vector>

namespace pt {

namespace {

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated append: every lane of the full warp calls this; lanes with `want` get a
// slot index, computed from one atomic per warp.
__device__ __forceinline__ int warp_append(int* counter, bool want) {
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return want ? base + __popc(mask & lanemask_lt()) : -1;
}

// Persistent work fetch: one atomic per warp for n (default 32) consecutive items.
__device__ __forceinline__ int warp_fetch(int* cursor, int n = 32) {
    int base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(cursor, n);
    return __shfl_sync(0xffffffffu, base, 0);
}

// Warp-aggregated append of up to N items per lane with one atomic per warp: slot[k] is the
// slot of the lane's k-th item when want[k], -1 otherwise.
template <int N>
__device__ __forceinline__ void warp_append_n(int* counter, const bool (&want)[N], int (&slot)[N]) {
    unsigned m[N];
    int total = 0;
#pragma unroll
    for (int k = 0; k < N; k++) {
        m[k] = __ballot_sync(0xffffffffu, want[k]);
        total += __popc(m[k]);
    }
    int base = 0;
    if (total > 0 && (threadIdx.x & 31) == 0) base = atomicAdd(counter, total);
    base = __shfl_sync(0xffffffffu, base, 0);
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < N; k++) {
        slot[k] = want[k] ? base + __popc(m[k] & lt) : -1;
        base += __popc(m[k]);
    }
}

// Two warp-aggregated appends (counters ca and cb) whose atomics are both issued before
// either result is read, so their round trips overlap.
template <int N>
__device__ __forceinline__ void warp_append_pair(int* ca, const bool (&wa)[N], int (&sa)[N], int* cb,
                                                 const bool (&wb)[N], int (&sb)[N]) {
    unsigned ma[N], mb[N];
    int ta = 0, tb = 0;
#pragma unroll
    for (int k = 0; k < N; k++) {
        ma[k] = __ballot_sync(0xffffffffu, wa[k]);
        mb[k] = __ballot_sync(0xffffffffu, wb[k]);
        ta += __popc(ma[k]);
        tb += __popc(mb[k]);
    }
    int ba = 0, bb = 0;
    if ((threadIdx.x & 31) == 0) {
        if (ta > 0) ba = atomicAdd(ca, ta);
        if (tb > 0) bb = atomicAdd(cb, tb);
    }
    ba = __shfl_sync(0xffffffffu, ba, 0);
    bb = __shfl_sync(0xffffffffu, bb, 0);
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < N; k++) {
        sa[k] = wa[k] ? ba + __popc(ma[k] & lt) : -1;
        sb[k] = wb[k] ? bb + __popc(mb[k] & lt) : -1;
        ba += __popc(ma[k]);
        bb += __popc(mb[k]);
    }
}

__device__ __forceinline__ void prefetch_l2(const void* ptr) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

__device__ __forceinline__ int tag_path(int tag) { return tag & kTagPathMask; }
__device__ __forceinline__ int tag_scene(int tag) { return tag >> kTagPathBits; }

// Index s with base[s] <= v < base[s + 1] (binary search over a batch's prefix offsets).
__device__ __forceinline__ int batch_find(const long long* base, int n, long long v) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(base + mid) <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The scene a path belongs to: in batched frames its root, emitter range and environment come
// from the scene table (the geometry arrays are shared, with global primitive ids).
__device__ __forceinline__ SceneDevice batch_scene_view(const FrameParams& p, int sid) {
    SceneDevice sc = p.sc;
    const BatchScene& b = p.batch[sid];
    sc.root = b.root;
    sc.lights = p.sc.lights + b.light_first;
    sc.num_lights = b.num_lights;
    sc.env = b.env;
    return sc;
}

// The camera ray of path i of the wave (Camera::generateRay with the sample's two jitter
// draws, camera.h:40-61), its queue tag and the path's random state after the draws. k_camera
// queues it; in frames that do not queue camera rays (p.cam_fused) the closest-hit and shade
// stages of depth 0 each compute it from the path index instead: the same operations on the
// same inputs, so both stages see the same ray, and no camera stage writes 56 bytes per path.
template <bool B>
__device__ __forceinline__ void camera_path(const FrameParams& p, long long wave_first, int i, V& o, V& d,
                                            int& tag, uint64_t& st) {
    const long long gp = wave_first + i;
    long long local = gp;
    int sid = 0, spp = p.spp, width = p.width;
    const CameraParams* cp = &p.dyn->cam;
    uint64_t sd = p.dyn->seed, sb = p.dyn->sample_base;
    if (B) {
        sid = batch_find(p.batch_path_base, p.num_scenes, gp);
        const BatchScene& b = p.batch[sid];
        local = gp - b.path_base;
        spp = b.spp;
        width = b.width;
        cp = &b.cam;
        sd = b.seed;
        sb = b.sample_base;
    }
    const int pixel = (int)(local / spp);
    const int s = (int)(local - (long long)pixel * spp);
    const int row = pixel / width;
    const int col = pixel - row * width;
    const uint64_t inc = pcg_inc((uint32_t)pixel);
    st = pcg_seed(sd, sb + (uint64_t)s, (uint32_t)pixel);
    const float xi1 = pcg_uniform(st, inc);
    const float xi2 = pcg_uniform(st, inc);
    camera_ray(*cp, row, col, xi1, xi2, o, d);
    tag = i | (sid << kTagPathBits);
}

// The origin and direction records of queue slot `slot` at `depth` (depth 0 of a wave whose
// camera rays are not queued: the camera ray of path `slot`, with no MIS pdf).
template <bool B>
__device__ __forceinline__ void queue_ray(const FrameParams& p, const PathQueue& q, int depth, long long wave_first,
                                          int slot, float4& o4, float4& d4) {
    if (depth == 0 && p.cam_fused) {
        V o, d;
        int tag;
        uint64_t st;
        camera_path<B>(p, wave_first, slot, o, d, tag, st);
        o4 = make_float4(o.x, o.y, o.z, __int_as_float(tag));
        d4 = make_float4(d.x, d.y, d.z, 0.f);
    } else {
        o4 = q.o[slot];
        d4 = q.d[slot];
    }
}

// The depth-0 queue of a wave: its camera rays, unit throughput, random states, and zero
// radiance per path. Used when the shade kernel of the frame reads the queue at depth 0.
template <bool B>
__global__ void k_camera(FrameParams p, long long wave_first, int n) {
    const PathQueue q = p.q[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        V o, d;
        int tag;
        uint64_t st;
        camera_path<B>(p, wave_first, i, o, d, tag, st);
        q.o[i] = make_float4(o.x, o.y, o.z, __int_as_float(tag));
        q.d[i] = make_float4(d.x, d.y, d.z, 0.f);
        q.beta[i] = make_float4(1.f, 1.f, 1.f, __int_as_float(1));  // camera ray: no MIS
        q.rng[i] = make_uint2((uint32_t)st, (uint32_t)(st >> 32));
        p.L[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        p.counters->ray_count[0] = n;
        atomicAdd(&p.stats->rays_camera, (unsigned long long)n);
    }
}

// A wave's start when the frame's shade kernel computes its depth-0 rays itself (the kernel
// of all materials at 128 registers, plain frames: p.cam_fused): the closest-hit and shade
// stages of depth 0 take each camera ray from camera_path, so no queue records are written;
// the shade stage of depth 0 writes each path's first radiance. Without any depth, the paths'
// radiance is zero.
__global__ void k_wave_start(FrameParams p, int n) {
    if (p.max_depth == 0)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            p.L[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        p.counters->ray_count[0] = n;
        atomicAdd(&p.stats->rays_camera, (unsigned long long)n);
    }
}

__device__ __forceinline__ int material_class(const SceneDevice& sc, int prim) {
    if (prim == kMissPrim) return 0;
    const int mat = prim >= 0 ? __ldg(sc.tri_mat + prim) : __ldg(sc.sph_mat + ~prim);
    return sc.mats[mat].type + 1;
}

// Warp-sum of per-thread work counters, one 64-bit atomic per warp.
__device__ __forceinline__ void flush_work(const TraceWork& w, unsigned long long* nodes, unsigned long long* prims) {
    unsigned n = w.nodes, m = w.prims;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(0xffffffffu, n, o);
        m += __shfl_xor_sync(0xffffffffu, m, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(nodes, (unsigned long long)n);
        atomicAdd(prims, (unsigned long long)m);
    }
}

// Ray sorting (no counterpart in the reference, which traces each path's rays in pixel order,
// src/renderers/path_tracer.cu:140-190): continuation rays leave a shading point in all
// directions, so neighbouring queue slots traverse unrelated parts of the BVH. Grouping them
// by origin cell and direction octant before the closest-hit stage gives a warp's rays
// similar node sequences. Only the order in which the closest-hit stage visits the slots
// changes (it writes every hit back to the ray's own slot), so images are unchanged.
//
// Key: a 4x4x4 grid over the scene bounds (clamped, so any origin maps to a cell) times the
// octant, in [0, kRayBuckets). The shade stage that emits a continuation ray writes its key
// next to it and counts it in a block histogram (shared memory, one global atomic per
// non-empty bucket and block at the end of the persistent loop).
__device__ __forceinline__ int ray_sort_key(const GuideFrame& gf, float4 o, float4 d) {
    const float ov[3] = {o.x, o.y, o.z};
    int cell = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        // inv_ext = 2 / extent: u in [0, 4] inside the bounds; NaN clamps to 0
        const float u = fminf(fmaxf((ov[a] - gf.lo[a]) * gf.inv_ext[a] * 2.f, 0.f), 3.f);
        cell = cell * 4 + (int)u;
    }
    return (cell << 3) | (d.x < 0.f ? 1 : 0) | (d.y < 0.f ? 2 : 0) | (d.z < 0.f ? 4 : 0);
}

// Then, ahead of the closest-hit stage, every block scans the histogram (bucket offsets),
// counts its contiguous chunk of slots per bucket, reserves their ranges with one global
// atomic per bucket, and writes the slot indices into `ray_index`. Order within a bucket is
// unspecified.
__global__ void __launch_bounds__(kRaySortBlock) k_ray_scatter(FrameParams p, int depth) {
    __shared__ int off[kRayBuckets], loc[kRayBuckets], wsum[kRaySortBlock / 32];
    const int count = p.counters->ray_count[depth];
    const PathQueue q = p.q[depth & 1];
    const int* cnt = p.ray_hist + 2 * depth * kRayBuckets;
    int* fill = p.ray_hist + (2 * depth + 1) * kRayBuckets;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int c0 = cnt[2 * t], c1 = cnt[2 * t + 1];
    int x = c0 + c1;  // inclusive scan over the block's pairs
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, k);
        if (lane >= k) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    loc[2 * t] = loc[2 * t + 1] = 0;
    __syncthreads();
    int excl = x - c0 - c1;
    for (int w = 0; w < warp; w++) excl += wsum[w];
    off[2 * t] = excl;
    off[2 * t + 1] = excl + c0;
    const int per = (count + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * per, b1 = min(count, b0 + per);
    for (int i = b0 + t; i < b1; i += blockDim.x) atomicAdd(&loc[q.key[i]], 1);
    __syncthreads();
    for (int j = t; j < kRayBuckets; j += blockDim.x)
        if (loc[j]) loc[j] = off[j] + atomicAdd(&fill[j], loc[j]);
    __syncthreads();
    for (int i = b0 + t; i < b1; i += blockDim.x) p.ray_index[atomicAdd(&loc[q.key[i]], 1)] = i;
}

// Closest hit for the queue, persistent. Each lane carries one query through the
// warp-synchronous node and leaf phases (node_step / leaf_step, the while-while loop of
// Aila and Laine 2009). A lane whose query ends writes its hit at once. When shape.refill_idle
// or more lanes are idle, they take the next rays of the queue together (one atomic per warp),
// so a warp does not idle behind its longest query (Aila and Laine's replacement of
// terminated rays). With refill_idle = 32 a warp takes 32 new rays only after all of its
// queries ended. With kSpeculateExtend set, traverse_round parks each lane's first leaf and
// keeps descending while another lane of the warp still searches for one.
template <int W, bool CNT, bool B, int Q>
__global__ void k_extend(FrameParams p, int depth, long long wave_first) {
    extern __shared__ int2 stk[];
    __shared__ int s_class[8];  // the block's hits per material class
    const int count = p.counters->ray_count[depth];
    const PathQueue q = p.q[depth & 1];
    // NEE frames trace bounce rays from the BSDF-direct tMin and re-trace the rare ones whose
    // hit lies closer than the continuation's (see the file comment); at a path's last depth
    // only the emission term is needed, so no re-trace
    const bool two = depth > 0 && p.nee;
    const float tmin0 = depth == 0 ? kCameraTMin : (two ? kDirectTMin : kBounceTMin);
    const int lane = threadIdx.x & 31;
    const bool sorted = !B && depth > 0 && p.shape.sort_rays;
    const int refill_idle = p.shape.refill_idle;
    const bool spec = (p.shape.speculate & kSpeculateExtend) != 0;
    const bool quant = W >= 4 && Q == 1;
    if (threadIdx.x < 8) s_class[threadIdx.x] = 0;
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.stats->rays_extend, (unsigned long long)count);
    int2* const st = stk + threadIdx.x;
    const int stride = blockDim.x;
    TraceWork work;
    // the lane's query; slot < 0: none (then alive is false as well)
    int slot = -1, cur = kEmptyChild, pend = kEmptyChild, sp = 0, of = 0;
    bool alive = false, hit_any = false;  // hit_any: any-hit output, never set for closest hit
    bool retrace = false;  // the query may be traced again from kBounceTMin (two, not the last depth)
    bool second = false;   // the query is that second trace
    float tmin = tmin0;
    RayPre r = make_raypre(V{0.f, 0.f, 0.f}, V{0.f, 0.f, 1.f});
    Hit h{FLT_MAX, 0.f, 0.f, kMissPrim};
    SceneDevice scb;
    if (B) scb = p.sc;
    bool more = true;  // warp-uniform: the queue may hold rays not yet taken
    for (;;) {
        if (more) {
            const unsigned busy = __ballot_sync(0xffffffffu, slot >= 0);
            const int idle = 32 - __popc(busy);
            if (idle >= refill_idle) {  // refill_idle is in [1, 32]: an all-idle warp always fetches
                int base = 0;
                if (lane == 0) base = atomicAdd(&p.counters->work_extend[depth], idle);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base + idle >= count) more = false;
                const int k = base + __popc(~busy & lanemask_lt());
                if (slot < 0 && k < count) {
                    slot = sorted ? p.ray_index[k] : k;
                    float4 o, d;
                    queue_ray<B>(p, q, depth, wave_first, slot, o, d);
                    r = make_raypre(mkv(o), mkv(d));
                    int last = p.max_depth - 1;
                    if (B) {
                        const int sid = tag_scene(__float_as_int(o.w));
                        scb = batch_scene_view(p, sid);
                        last = p.batch[sid].max_depth - 1;
                    }
                    retrace = two && depth < last;
                    second = false;
                    tmin = tmin0;
                    h = Hit{FLT_MAX, 0.f, 0.f, kMissPrim};
                    cur = B ? scb.root : p.sc.root;
                    sp = 0;
                    pend = kEmptyChild;
                    of = 0;
                    alive = true;
                }
            }
        }
        // with no query left after a fetch, the queue is exhausted (more is false)
        if (!__any_sync(0xffffffffu, alive)) break;
        const SceneDevice& sc = B ? scb : p.sc;
        traverse_round<W, false, CNT>(sc.nodes, sc.prims, quant, spec, r, tmin, FLT_MAX, st, stride, p.stack_depth, h,
                                      cur, pend, sp, alive, hit_any, of, &work, Q == 2);
        // a triangle at t = tMin is inside the continuation's range, a sphere is not (triangle.cu:34
        // accepts t >= tMin, sphere.cu:16,29 need t > tMin)
        if (slot >= 0 && !alive && retrace && !second && h.prim != kMissPrim &&
            (h.t < kBounceTMin || (h.prim < 0 && h.t == kBounceTMin))) {
            // the BSDF-direct ray stopped closer than the continuation's tMin: keep its hit for
            // the emission term and trace the direction again from kBounceTMin
            if (of) atomicOr(&p.stats->error, 1);
            q.hitd[slot] = make_float4(h.t, h.b1, h.b2, __int_as_float(h.prim));
            second = true;
            tmin = kBounceTMin;
            h = Hit{FLT_MAX, 0.f, 0.f, kMissPrim};
            cur = B ? scb.root : p.sc.root;
            sp = 0;
            pend = kEmptyChild;
            of = 0;
            alive = true;
        }
        if (slot >= 0 && !alive) {  // the query ended: write its hit to the ray's own slot
            if (of) atomicOr(&p.stats->error, 1);
            q.hit[slot] = make_float4(second ? -h.t : h.t, h.b1, h.b2, __int_as_float(h.prim));
            if (p.shape.sort_materials) {
                const int key = material_class(p.sc, h.prim);
                q.key[slot] = key;
                atomicAdd(&s_class[key], 1);
            }
            slot = -1;
        }
    }
    __syncthreads();
    // one atomic per class and block for the whole persistent loop
    if (p.shape.sort_materials && threadIdx.x < kMaterialClasses && s_class[threadIdx.x] > 0)
        atomicAdd(&p.counters->sort_count[depth][threadIdx.x], s_class[threadIdx.x]);
    if (CNT) flush_work(work, &p.stats->extend_nodes, &p.stats->extend_prims);
}

constexpr int kSortItems = 4;  // queue entries per thread and chunk of the material sort
__global__ void k_sort(FrameParams p, int depth) {
    const int count = p.counters->ray_count[depth];
    const PathQueue q = p.q[depth & 1];
    int off[kMaterialClasses];
    int acc = 0;
#pragma unroll
    for (int c = 0; c < kMaterialClasses; c++) {
        off[c] = acc;
        acc += p.counters->sort_count[depth][c];
    }
    // Slots are reserved per block and chunk of kSortItems x blockDim.x entries: warps add
    // their class counts into shared counters, then one global atomic per class and chunk
    // reserves the chunk's range (the grid is capped at a few blocks per SM and strides over
    // the queue). Several entries per thread share each chunk's barriers and atomics.
    __shared__ int s_cnt[8], s_base[8];
    const int stride = gridDim.x * blockDim.x * kSortItems;
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    for (int base = blockIdx.x * blockDim.x * kSortItems; base < count; base += stride) {
        if (threadIdx.x < 8) s_cnt[threadIdx.x] = 0;
        __syncthreads();
        int key[kSortItems], b[kSortItems], leader[kSortItems];
        unsigned peers[kSortItems];
#pragma unroll
        for (int j = 0; j < kSortItems; j++) {
            const int i = base + j * blockDim.x + threadIdx.x;
            key[j] = i < count ? q.key[i] : 7;  // 7: no entry (no class uses it)
        }
#pragma unroll
        for (int j = 0; j < kSortItems; j++) {
            const int i = base + j * blockDim.x + threadIdx.x;
            peers[j] = __match_any_sync(0xffffffffu, key[j]);
            leader[j] = __ffs(peers[j]) - 1;
            b[j] = 0;
            if (i < count && lane == leader[j]) b[j] = atomicAdd(&s_cnt[key[j]], __popc(peers[j]));
        }
        __syncthreads();
        if (threadIdx.x < kMaterialClasses && s_cnt[threadIdx.x] > 0)
            s_base[threadIdx.x] = atomicAdd(&p.counters->sort_fill[depth][threadIdx.x], s_cnt[threadIdx.x]);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSortItems; j++) {
            const int i = base + j * blockDim.x + threadIdx.x;
            const int bj = __shfl_sync(0xffffffffu, b[j], leader[j]);
            if (i < count) {
                int ko = 0;
#pragma unroll
                for (int c = 0; c < kMaterialClasses; c++)
                    if (c == key[j]) ko = off[c] + s_base[c];
                p.sort_index[ko + bj + __popc(peers[j] & lt)] = i;
            }
        }
        __syncthreads();  // s_cnt / s_base are reused by the next chunk
    }
}

// Hit point, shading normal and material of a closest hit (Triangle::hit / Sphere::hit's
// record, src/primitives/*.cu): the triangle normal is the interpolated, unnormalised one.
__device__ __forceinline__ void hit_info(const SceneDevice& sc, V o, V dir, float4 h4, V& point, V& n, int& mat) {
    const int prim = __float_as_int(h4.w);
    if (prim >= 0) {
        const float b1 = h4.y, b2 = h4.z;
        const float w0 = 1.f - b1 - b2;
        const V p0 = mkv(__ldg(sc.tri_p + 3 * prim + 0));
        const V p1 = mkv(__ldg(sc.tri_p + 3 * prim + 1));
        const V p2 = mkv(__ldg(sc.tri_p + 3 * prim + 2));
        const V n0 = mkv(__ldg(sc.tri_n + 3 * prim + 0));
        const V n1 = mkv(__ldg(sc.tri_n + 3 * prim + 1));
        const V n2 = mkv(__ldg(sc.tri_n + 3 * prim + 2));
        point = p0 * w0 + p1 * b1 + p2 * b2;
        n = w0 * n0 + b1 * n1 + b2 * n2;
        mat = __ldg(sc.tri_mat + prim);
    } else {
        const float4 s = __ldg(sc.sph + ~prim);
        point = o + h4.x * dir;
        n = normalized((point - mkv(s.x, s.y, s.z)) / s.w);
        mat = __ldg(sc.sph_mat + ~prim);
    }
}

// The BSDF sampler's own density of a direction (the reference's Microfacet::pdf evaluates D
// with alpha(wi), microfacet.h:124-134, while sampling uses alpha(wo), :148-158).
__device__ __forceinline__ float bsdf_sampling_pdf(const Material& m, V wo, V wi) {
    if (m.type == kLambertian) return lambert_pdf(wi);
    if (m.type == kMicrofacet || m.type == kMetal) {
        const V wh = normalized(wo + wi);
        return mf_D(m.alpha, wo, wh) * fabsf(wh.z) / (4.f * fabsf(dot(wo, wh)));
    }
    return 0.f;
}

// The material functions with the type fixed at compile time (T >= 0) or read from the
// material (T < 0): a shade kernel specialised to one material class carries only its BSDF.
template <int T>
__device__ __forceinline__ V bsdf_f_t(const Material& m, V wo, V wi) {
    if constexpr (T == kLambertian) return lambert_f(m, wo, wi);
    else if constexpr (T == kMicrofacet) return mf_f(m.alpha, wo, wi);
    else if constexpr (T == kMetal) return mf_metal_f(m, wo, wi);
    else if constexpr (T == kMirror || T == kGlass) return mkv(0.f);
    else return bsdf_f(m, wo, wi);
}
template <int T>
__device__ __forceinline__ float bsdf_pdf_t(const Material& m, V wo, V wi) {
    if constexpr (T == kLambertian) return lambert_pdf(wi);
    else if constexpr (T == kMicrofacet || T == kMetal) return mf_pdf(m.alpha, wo, wi);
    else if constexpr (T == kMirror || T == kGlass) return 0.f;
    else return bsdf_pdf(m, wo, wi);
}
template <int T>
__device__ __forceinline__ float bsdf_sampling_pdf_t(const Material& m, V wo, V wi) {
    if constexpr (T == kLambertian) return lambert_pdf(wi);
    else if constexpr (T == kMicrofacet || T == kMetal) {
        const V wh = normalized(wo + wi);
        return mf_D(m.alpha, wo, wh) * fabsf(wh.z) / (4.f * fabsf(dot(wo, wh)));
    } else if constexpr (T == kMirror || T == kGlass) return 0.f;
    else return bsdf_sampling_pdf(m, wo, wi);
}

__device__ __forceinline__ float lum(V c) { return (c.x + c.y + c.z) * (1.f / 3.f); }

// Training index of a path: the path records training data when the index is a multiple of
// gstride, into slot index / gstride. A single scene: the wave-local path index. A batched
// frame: the path's position among the wave's paths of guided scenes (-1 for the paths of
// other scenes), so the training budget goes to the scenes that train a network.
template <bool B>
__device__ __forceinline__ long long train_index(const FrameParams& p, int sid, int path, long long wave_first,
                                                 long long gfirst) {
    if (!B) return path;
    const BatchScene& b = p.batch[sid];
    if (b.guide_net < 0) return -1;
    return b.guided_base + (wave_first + path - b.path_base) - gfirst;
}

// Per training path and depth: U (unweighted emission), R (NEE + MIS-weighted emission),
// W (MIS-weighted emission), luminance times throughput.
__device__ __forceinline__ void guide_account(const FrameParams& p, long long ti, int depth, float u, float r, float w) {
    if (p.guide_mode == 0 || ti < 0 || ti % p.gstride != 0) return;
    float* a = p.gacc + ((size_t)(ti / p.gstride) * p.max_depth + depth) * 3;
    a[0] += u;
    a[1] += r;
    a[2] += w;
}

// Emission term of a BSDF-direct ray that stopped closer than the continuation's tMin
// (directSampleBSDF's hit branch, path_tracer.cu:52-68, at the first hit): front-face
// emission of a Lambertian emitter with the MIS weight against the emitter sampler, else
// nothing. Rare, so kept out of line to spare the shade stage's registers.
// Returns the unweighted emission and its weight through `w`.
__device__ __noinline__ V direct_hit_emission(const SceneDevice& sc, V o, V dir, float4 hd, float bsdf_pdf,
                                              bool nomis, bool orthonormal, float& w) {
    V point, n;
    int mat;
    w = 0.f;
    hit_info(sc, o, dir, hd, point, n, mat);
    if (orthonormal) n = normalized(n);
    const Material m = sc.mats[mat];
    if (!m.emitting) return mkv(0.f);
    const Frame fr = make_frame(n);
    const V wo = normalized(to_local(fr, -dir));
    if (wo.z < 0.f) return mkv(0.f);
    w = nomis ? 1.f : balance(bsdf_pdf, pdf_scene_light(sc, o, point, n, __float_as_int(hd.w)));
    return mkv(m.emit[0], m.emit[1], m.emit[2]);
}

// GUIDE: compiled with the path-guiding code (used when guide_mode != 0); the plain
// instantiation keeps the reference integrator's register budget. B: batched frame (the
// scene, its depth, spp and guide come from the path's tag and the scene table).
// The guided instantiation runs 128-thread blocks, 8 per SM: capped at 64 registers (its
// spills stay in L1) it keeps twice the warps of the uncapped 127-register build resident,
// which measured 37% faster on the latency-bound guided shade (slit room, 1024^2).
constexpr int kShadeGuidedBlock = 128;
constexpr int kShadeGuidedBlocksPerSm = 8;
// Register budget of the per-class shade kernels (k_shade_class), measured on a B200 against
// 64, 80, 96 and 168: 64 for the Lambert, mirror, glass and miss classes (the slit room's
// Lambert walls shaded 24% faster than in the kernel of all materials), 96 for the two
// Beckmann classes (their sampling spills at 64; the icosphere shaded 12% faster).
__host__ __device__ constexpr int shade_class_regs(int cls) { return cls == kMicrofacet + 1 || cls == kMetal + 1 ? 96 : 64; }

// CLS: -1, every slot of the queue (in material-sorted order when sorting is on); >= 0, only
// the slots the sort put in material class CLS (0 miss, type + 1 otherwise), with that
// class's BSDF fixed at compile time, so each class kernel holds only its own registers.
// IPL items per lane per warp iteration: one fetch and one append atomic per warp serve
// 32 x IPL items (the queue counters are single addresses every warp of the grid hits).
// AHEAD (kernels with registers to spare): the warp claims its next chunk while the current
// one shades (lane 0's atomic is read at the top of the next iteration), loads a slot's
// random state with its other records, and issues the continuation and shadow appends'
// atomics together, so fewer global round trips are serialised per chunk. Under a tight
// register budget the extra live values spill and the stage slows down.
template <bool GUIDE, bool B, int CLS, int IPL, bool AHEAD = false>
__device__ __forceinline__ void shade_body(const FrameParams& p, int depth, long long wave_first, long long gfirst) {
    constexpr int kType = CLS > 0 ? CLS - 1 : -1;  // the material type of a class kernel
    int count = p.counters->ray_count[depth];
    int cls_first = 0;
    if constexpr (CLS >= 0) {  // the class's range of the sorted order
        for (int c = 0; c < CLS; c++) cls_first += p.counters->sort_count[depth][c];
        count = p.counters->sort_count[depth][CLS];
        if (count == 0) return;  // a class absent at this depth: no fetch, no atomics
    }
    int* const work = CLS >= 0 ? &p.counters->work_class[depth][CLS < 0 ? 0 : CLS] : &p.counters->work_shade[depth];
    const PathQueue q = p.q[depth & 1];
    const PathQueue qn = p.q[(depth + 1) & 1];
    const bool last_frame = depth >= p.max_depth - 1;
    const bool guided_frame = GUIDE && p.guide_mode == 2;
    // ray-sort keys of the continuation rays (uniform over the grid)
    const bool rsort = !B && p.shape.sort_rays && depth + 1 < p.max_depth;
    __shared__ int rhist[B ? 1 : kRayBuckets];
    if (rsort) {
        for (int j = threadIdx.x; j < kRayBuckets; j += blockDim.x) rhist[j] = 0;
        __syncthreads();
    }
    static_assert(!AHEAD || IPL == 1, "the claim-ahead loop shades one item per lane");
    const int lane = threadIdx.x & 31;
    auto slot_of = [&](int i) {
        return CLS >= 0 ? p.sort_index[cls_first + i] : (p.shape.sort_materials ? p.sort_index[i] : i);
    };
    // AHEAD: the chunk after next is claimed while a chunk shades (lane 0's atomic result,
    // read one chunk later), the next chunk's slots are loaded then too, and its queue records
    // are prefetched into L2 before this chunk's results are written
    int claimed = 0, cur_base = 0, next_base = 0, cur_slot = -1;
    if (AHEAD) {
        cur_base = warp_fetch(work);
        next_base = warp_fetch(work);
        if (cur_base + lane < count) cur_slot = slot_of(cur_base + lane);
    }
    for (;;) {
        const int base = AHEAD ? cur_base : warp_fetch(work, 32 * IPL);
        if (base >= count) break;
        int next_slot = -1;
        if (AHEAD) {
            if (lane == 0) claimed = atomicAdd(work, 32);
            if (next_base + lane < count) next_slot = slot_of(next_base + lane);
        }
        bool cont_[IPL], shadow_[IPL];
        float4 co_[IPL], cd_[IPL], cb_[IPL], so_[IPL], sd_[IPL], sc_[IPL];
        uint2 crng_[IPL];
#pragma unroll
        for (int item = 0; item < IPL; item++) {
        const int i = base + 32 * item + (threadIdx.x & 31);
        bool cont = false, shadow = false, record = false;
        float4 co, cd, cb, so, sd, sc4;
        uint2 crng;
        GuideRecord rec;
        if (i < count) {
            const int slot = AHEAD ? cur_slot : slot_of(i);
            float4 o4, d4, b4;
            float4 h4 = q.hit[slot];
            uint2 rng0 = make_uint2(0u, 0u);
            if (AHEAD && depth == 0) {  // camera ray of path `slot` (p.cam_fused): unit throughput, no MIS
                V o, d;
                int tg;
                uint64_t st0;
                camera_path<B>(p, wave_first, slot, o, d, tg, st0);
                o4 = make_float4(o.x, o.y, o.z, __int_as_float(tg));
                d4 = make_float4(d.x, d.y, d.z, 0.f);
                b4 = make_float4(1.f, 1.f, 1.f, __int_as_float(1));
                rng0 = make_uint2((uint32_t)st0, (uint32_t)(st0 >> 32));
            } else {
                o4 = q.o[slot];
                d4 = q.d[slot];
                b4 = q.beta[slot];
                if (AHEAD) rng0 = q.rng[slot];
            }
            // a negative t: the BSDF-direct ray stopped closer (hitd), this is the continuation's hit
            const bool split = __float_as_int(h4.x) < 0;
            h4.x = fabsf(h4.x);
            const int tag = __float_as_int(o4.w);
            const int path = tag_path(tag);
            const int sid = B ? tag_scene(tag) : 0;
            SceneDevice scb;
            if (B) scb = batch_scene_view(p, sid);
            const SceneDevice& sc = B ? scb : p.sc;
            const long long ti = GUIDE && p.guide_mode ? train_index<B>(p, sid, path, wave_first, gfirst) : -1;
            const bool last = B ? depth >= p.batch[sid].max_depth - 1 : last_frame;
            const bool guided = B ? GUIDE && p.batch[sid].guide_mode == 2 : guided_frame;
            const bool do_nee = p.nee && sc.num_lights + (sc.env.present ? 1 : 0) > 0;
            const int flags = __float_as_int(b4.w);
            const V o = mkv(o4), dir = mkv(d4), beta = mkv(b4);
            const int prim = __float_as_int(h4.w);
            const bool nomis = (flags & 1) || !p.nee;
            V Ladd = mkv(0.f);
            if (split) {
                const bool ortho = GUIDE && (B ? p.batch[sid].guide_mode : p.guide_mode);
                float w;
                const V Le = direct_hit_emission(sc, o, dir, q.hitd[slot], d4.w, nomis, ortho, w);
                if (!is_zero(Le)) {
                    Ladd = beta * Le * w;
                    if (GUIDE) guide_account(p, ti, depth, lum(beta * Le), lum(Ladd), lum(Ladd));
                }
            }
            // a class kernel knows whether its slots missed
            const bool miss = CLS == 0 ? true : (CLS > 0 ? false : prim == kMissPrim);
            if (miss) {
                // escaped: environment radiance (path_tracer.cu:68-79, :162, :206, :228); a
                // continuation that misses after a closer BSDF-direct hit adds nothing (:178-180)
                const V Le = split ? mkv(0.f) : env_emit(sc.env, dir);
                if (!is_zero(Le)) {
                    const float w = nomis ? 1.f : balance(d4.w, pdf_env_light(sc, dir));
                    Ladd = beta * Le * w;
                    if (GUIDE) guide_account(p, ti, depth, lum(beta * Le), lum(Ladd), lum(Ladd));
                }
            } else {
                V point, n;
                int mat;
                hit_info(sc, o, dir, h4, point, n, mat);
                // guided modes shade in an orthonormal frame (the reference's frame is built
                // from the unnormalised interpolated normal)
                if (GUIDE && (B ? p.batch[sid].guide_mode : p.guide_mode)) n = normalized(n);
                const Frame fr = make_frame(n);
                const V wo = normalized(to_local(fr, -dir));
                const Material m = sc.mats[mat];
                const int mtype = kType >= 0 ? kType : m.type;
                // front-face emission (lambertian.cu:5-11); only Lambertian materials emit
                if ((kType < 0 || kType == kLambertian) && !split && m.emitting && wo.z >= 0.f) {
                    const V Le = mkv(m.emit[0], m.emit[1], m.emit[2]);
                    const float w = nomis ? 1.f : balance(d4.w, pdf_scene_light(sc, o, point, n, prim));
                    Ladd = beta * Le * w;
                    if (GUIDE) guide_account(p, ti, depth, lum(beta * Le), lum(Ladd), lum(Ladd));
                }
                if (!last) {
                    const long long gp = wave_first + path;
                    const uint32_t pixel =
                        B ? (uint32_t)((gp - p.batch[sid].path_base) / p.batch[sid].spp) : (uint32_t)(gp / p.spp);
                    const uint64_t inc = pcg_inc(pixel);
                    if (!AHEAD) rng0 = q.rng[slot];
                    uint64_t st = ((uint64_t)rng0.y << 32) | rng0.x;
                    const bool delta_mat = mtype == kMirror || mtype == kGlass;
                    const bool use_guide = guided && !delta_mat;
                    const float* mix = use_guide ? p.gmix + (size_t)slot * kGuideOut : nullptr;
                    bool from_guide = false;
                    // one-sample MIS: the guide with probability gfrac (u in (0, 1])
                    if (use_guide) from_guide = pcg_uniform(st, inc) >= 1.f - p.gfrac;
                    BsdfSample bs;
                    V wworld;
                    if (from_guide) {
                        const float u0 = pcg_uniform(st, inc), u1 = pcg_uniform(st, inc), u2 = pcg_uniform(st, inc);
                        wworld = normalized(guide_sample(mix, u0, u1, u2));
                        bs.wi = to_local(fr, wworld);
                        bs.f = bsdf_f_t<kType>(m, wo, bs.wi);
                        bs.delta = false;
                    } else {
                        switch (mtype) {
                            case kLambertian: {
                                const float x1 = pcg_uniform(st, inc);
                                const float x2 = pcg_uniform(st, inc);
                                bs = lambert_sample(m, wo, x1, x2);
                                break;
                            }
                            case kMirror: bs = mirror_sample(wo); break;
                            case kGlass: bs = glass_sample(m, wo, pcg_uniform(st, inc)); break;
                            default: {  // Beckmann: kMicrofacet, kMetal
                                const float x1 = pcg_uniform(st, inc);
                                const float x2 = pcg_uniform(st, inc);
                                bs = mf_sample(m.alpha, wo, x1, x2);
                                if (mtype == kMetal) bs.f = mf_metal_f(m, wo, bs.wi);
                            }
                        }
                        wworld = to_world(fr, bs.wi);
                    }
                    if (use_guide) {
                        // mixture density of the direction, whichever strategy produced it
                        const float pb = bsdf_sampling_pdf_t<kType>(m, wo, bs.wi);
                        float pg = guide_pdf(mix, normalized(wworld));
                        if (!isfinite(pg)) pg = 0.f;
                        bs.pdf = (1.f - p.gfrac) * pb + p.gfrac * pg;
                    }
                    // mirror and glass samples are delta: no emitter sampling (:84)
                    if (kType != kMirror && kType != kGlass && do_nee && !bs.delta) {
                        // directSampleLights (path_tracer.cu:83-126)
                        const float x1 = pcg_uniform(st, inc);
                        const float x2 = pcg_uniform(st, inc);
                        const float x3 = pcg_uniform(st, inc);
                        const LightSample ls = sample_lights(sc, point, x1, x2, x3);
                        if (dot(ls.normal, ls.wi) < 0.f && ls.pdf > 0.f) {
                            const V wil = to_local(fr, ls.wi);
                            float bpdf = p.consistent_mis ? bsdf_sampling_pdf_t<kType>(m, wo, wil)
                                                          : bsdf_pdf_t<kType>(m, wo, wil);
                            if (use_guide) {
                                const float pg = guide_pdf(mix, ls.wi);
                                bpdf = (1.f - p.gfrac) * bpdf + p.gfrac * (isfinite(pg) ? pg : 0.f);
                            }
                            const float wl = balance(ls.pdf, bpdf);
                            const V f = bsdf_f_t<kType>(m, wo, wil);
                            const V contrib = beta * (ls.emitted * wl * f * fabsf(dot(n, ls.wi)) / ls.pdf);
                            if (!is_zero(contrib)) {
                                shadow = true;
                                so = make_float4(point.x, point.y, point.z, ls.distance - 2e-4f);
                                sd = make_float4(ls.wi.x, ls.wi.y, ls.wi.z, __int_as_float(tag));
                                sc4 = make_float4(contrib.x, contrib.y, contrib.z, 0.f);
                            }
                        }
                    }
                    // beta *= f * |cos| / pdf (path_tracer.cu:171-173)
                    if (bs.pdf > 0.f) {
                        const V fc = bs.f * fabsf(bs.wi.z) / bs.pdf;
                        const V nb = beta * fc;
                        if (!is_zero(nb) && isfinite(nb.x + nb.y + nb.z)) {
                            cont = true;
                            co = make_float4(point.x, point.y, point.z, __int_as_float(tag));
                            cd = make_float4(wworld.x, wworld.y, wworld.z, bs.pdf);
                            cb = make_float4(nb.x, nb.y, nb.z, __int_as_float(bs.delta ? 1 : 0));
                            crng = make_uint2((uint32_t)st, (uint32_t)(st >> 32));
                            if (GUIDE && p.guide_mode && !delta_mat && ti >= 0 && ti % p.gstride == 0) {
                                const V wn = normalized(wworld);
                                const V won = normalized(-dir);
                                rec = GuideRecord{{point.x, point.y, point.z}, {n.x, n.y, n.z}, {won.x, won.y, won.z},
                                                  {wn.x, wn.y, wn.z}, lum(fc), lum(nb), (int)(ti / p.gstride),
                                                  depth | (sid << 8)};
                                record = true;
                            }
                        }
                    }
                }
            }
            if (AHEAD && depth == 0) {  // the path's first radiance (p.cam_fused: no earlier stage wrote it)
                p.L[path] = make_float4(Ladd.x, Ladd.y, Ladd.z, 0.f);
            } else if (!is_zero(Ladd)) {
                float4 l = p.L[path];
                l.x += Ladd.x;
                l.y += Ladd.y;
                l.z += Ladd.z;
                p.L[path] = l;
            }
        }
        if (GUIDE && p.guide_mode) {
            const int r = warp_append(p.grec_count, record);
            if (record && r < p.grec_cap) p.grec[r] = rec;
        }
        cont_[item] = cont;
        shadow_[item] = shadow;
        co_[item] = co;
        cd_[item] = cd;
        cb_[item] = cb;
        crng_[item] = crng;
        so_[item] = so;
        sd_[item] = sd;
        sc_[item] = sc4;
        }
        if (AHEAD && next_slot >= 0) {
            prefetch_l2(q.o + next_slot);
            prefetch_l2(q.d + next_slot);
            prefetch_l2(q.beta + next_slot);
            prefetch_l2(q.hit + next_slot);
            prefetch_l2(q.rng + next_slot);
        }
        int cslot[IPL], sslot[IPL];
        if (AHEAD)
            warp_append_pair<IPL>(&p.counters->ray_count[depth + 1], cont_, cslot, &p.counters->shadow_count[depth],
                                  shadow_, sslot);
        else
            warp_append_n<IPL>(&p.counters->ray_count[depth + 1], cont_, cslot);
#pragma unroll
        for (int item = 0; item < IPL; item++) {
            if (!cont_[item]) continue;
            const int cs = cslot[item];
            qn.o[cs] = co_[item];
            qn.d[cs] = cd_[item];
            qn.beta[cs] = cb_[item];
            qn.rng[cs] = crng_[item];
            if (!B && rsort) {
                const int key = ray_sort_key(p.gframe, co_[item], cd_[item]);
                qn.key[cs] = key;
                atomicAdd(&rhist[key], 1);
            }
        }
        if (!AHEAD) warp_append_n<IPL>(&p.counters->shadow_count[depth], shadow_, sslot);
#pragma unroll
        for (int item = 0; item < IPL; item++) {
            if (!shadow_[item]) continue;
            const int ss = sslot[item];
            p.sq.o[ss] = so_[item];
            p.sq.d[ss] = sd_[item];
            p.sq.c[ss] = sc_[item];
        }
        if (AHEAD) {
            cur_base = next_base;
            next_base = __shfl_sync(0xffffffffu, claimed, 0);
            cur_slot = next_slot;
        }
    }
    if (!B && rsort) {
        __syncthreads();
        int* cnt = p.ray_hist + 2 * (depth + 1) * kRayBuckets;
        for (int j = threadIdx.x; j < kRayBuckets; j += blockDim.x)
            if (rhist[j]) atomicAdd(&cnt[j], rhist[j]);
    }
}

// The shade stage over every slot of the queue (all materials).
template <bool GUIDE, bool B>
__global__ void __launch_bounds__(GUIDE ? kShadeGuidedBlock : 512, GUIDE ? kShadeGuidedBlocksPerSm : 1)
    k_shade(FrameParams p, int depth, long long wave_first, long long gfirst) {
    shade_body<GUIDE, B, -1, 1>(p, depth, wave_first, gfirst);
}

// Items per lane of the plain shade kernels. 2 and 4 (one fetch and one append atomic per
// 64 or 128 items) measured slower on every configuration: the extra live state costs more
// warps than the contended queue counters do.
constexpr int kShadeIpl = 1;
// The plain shade stage over every slot of the queue (all materials) at a register budget
// of REGS: 128 (16 warps per SM at 128-thread blocks) or 80 (24 warps, with spills), the
// autotuner's choice per scene (the icosphere shaded 16% faster at 80, the spheres 7% slower).
template <bool B, int REGS>
__global__ void __maxnreg__(REGS) k_shade_all(FrameParams p, int depth, long long wave_first, long long gfirst) {
    shade_body<false, B, -1, kShadeIpl, REGS >= 128>(p, depth, wave_first, gfirst);
}
__host__ __device__ constexpr int shade_resident(int regs, int block) {
    return 65536 / (regs * block) < 2048 / block ? (65536 / (regs * block) > 0 ? 65536 / (regs * block) : 1)
                                                 : 2048 / block;
}

// The shade stage over one material class of a sorted queue (plain frames).
template <bool B, int CLS>
__global__ void __maxnreg__(shade_class_regs(CLS)) k_shade_class(FrameParams p, int depth, long long wave_first,
                                                                long long gfirst) {
    shade_body<false, B, CLS, kShadeIpl>(p, depth, wave_first, gfirst);
}

template <int W, bool CNT, bool B, int Q>
__global__ void k_shadow(FrameParams p, int depth, long long wave_first, long long gfirst) {
    extern __shared__ int2 stk[];
    const int count = p.counters->shadow_count[depth];
    const int lane = threadIdx.x & 31;
    const int refill_idle = p.shape.refill_idle;
    const bool spec = (p.shape.speculate & kSpeculateShadow) != 0;
    const bool near = p.shape.shadow_near != 0;  // children nearest first
    const bool quant = W >= 4 && Q == 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.stats->rays_shadow, (unsigned long long)count);
    int2* const st = stk + threadIdx.x;
    const int stride = blockDim.x;
    TraceWork work;
    // the lane's query, refilled as in k_extend; slot < 0: none
    int slot = -1, cur = kEmptyChild, pend = kEmptyChild, sp = 0, of = 0, tag = 0;
    bool alive = false, occ = false;
    float tmax = 0.f;
    RayPre r = make_raypre(V{0.f, 0.f, 0.f}, V{0.f, 0.f, 1.f});
    Hit h{0.f, 0.f, 0.f, kMissPrim};  // unused by any-hit queries
    SceneDevice scb;
    if (B) scb = p.sc;
    bool more = true;  // warp-uniform
    for (;;) {
        if (more) {
            const unsigned busy = __ballot_sync(0xffffffffu, slot >= 0);
            const int idle = 32 - __popc(busy);
            if (idle >= refill_idle) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&p.counters->work_shadow[depth], idle);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base + idle >= count) more = false;
                const int k = base + __popc(~busy & lanemask_lt());
                if (slot < 0 && k < count) {
                    slot = k;
                    const float4 o = p.sq.o[k], d = p.sq.d[k];
                    r = make_raypre(mkv(o), mkv(d));
                    tmax = o.w;
                    tag = __float_as_int(d.w);
                    if (B) scb = batch_scene_view(p, tag_scene(tag));
                    cur = B ? scb.root : p.sc.root;
                    sp = 0;
                    pend = kEmptyChild;
                    of = 0;
                    occ = false;
                    alive = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, alive)) break;
        const SceneDevice& sc = B ? scb : p.sc;
        traverse_round<W, true, CNT>(sc.nodes, sc.prims, quant, spec, r, kShadowTMin, tmax, st, stride, p.stack_depth,
                                     h, cur, pend, sp, alive, occ, of, &work, Q == 2, near);
        if (slot >= 0 && !alive) {  // the query ended: occluded, or the stack ran empty
            const int i = slot;
            slot = -1;
            if (of) atomicOr(&p.stats->error, 1);
            if (!occ) {
                const float4 c = p.sq.c[i];
                const int path = tag_path(tag);
                float4 l = p.L[path];
                l.x += c.x;
                l.y += c.y;
                l.z += c.z;
                p.L[path] = l;
                if (p.guide_mode) {
                    const long long ti = train_index<B>(p, tag_scene(tag), path, wave_first, gfirst);
                    guide_account(p, ti, depth, 0.f, (c.x + c.y + c.z) * (1.f / 3.f), 0.f);
                }
            }
        }
    }
    if (CNT) flush_work(work, &p.stats->shadow_nodes, &p.stats->shadow_prims);
}

// Guide inference for the rays of the queue consumed at `depth`: each lane computes the
// features of one hit, the warp runs the network on the tensor cores for its 32 rays (two
// 16-row groups sharing each weight fragment), each lane activates its own row and the warp
// writes the 32 mixtures of consecutive queue slots as one contiguous 5120-byte store.
constexpr int kInferWarps = 8;
constexpr int kInferSmemBytes = (kSWords + kInferWarps * 32 * kSXStride) * 4;  // 81 KB: 2 blocks per SM

// Features of one queued hit (zeros for a miss).
__device__ __forceinline__ bool guide_features(const FrameParams& p, const GuideFrame& gf, float4 o4, float4 d4,
                                               float4 h4, float x[kGuideIn]) {
    if (__float_as_int(h4.w) == kMissPrim) {
        for (int k = 0; k < kGuideIn; k++) x[k] = 0.f;
        return false;
    }
    h4.x = fabsf(h4.x);  // drop the mark of a split BSDF-direct hit
    V point, n;
    int mat;
    hit_info(p.sc, mkv(o4), mkv(d4), h4, point, n, mat);
    n = normalized(n);
    const V wo = normalized(-mkv(d4));
    const float pp[3] = {point.x, point.y, point.z}, nn[3] = {n.x, n.y, n.z}, ww[3] = {wo.x, wo.y, wo.z};
    guide_encode(gf, pp, nn, ww, x);
    return true;
}

// Raw outputs of row `lane` (left in the tile by guide_mlp_warp32) -> mixture, in place.
__device__ __forceinline__ float* guide_activate_row(uint32_t* sx, int lane) {
    float* row = reinterpret_cast<float*>(sx) + (lane >> 4) * 16 * kSXStride + (lane & 15) * kGuideOut;
    float raw[kGuideOut], mix[kGuideOut];
    for (int j = 0; j < kGuideOut; j++) raw[j] = row[j];
    guide_activate(raw, mix);
    for (int j = 0; j < kGuideOut; j++) row[j] = mix[j];
    return row;
}

// Guide inference for the rays of the queue consumed at `depth`: each lane computes the
// features of one hit, the warp runs the network on the tensor cores for its 32 rays (two
// 16-row groups sharing each weight fragment), each lane activates its own row and the warp
// writes the 32 mixtures of consecutive queue slots as one contiguous 5120-byte store.
// Batched frames (B): each scene has its own network (weights read through L1/L2); a warp
// evaluates each distinct network among its lanes in turn.
template <bool B>
__global__ void __launch_bounds__(32 * kInferWarps, 2) k_guide_infer(FrameParams p, int depth) {
    extern __shared__ __align__(16) uint32_t ism[];
    const int count = p.counters->ray_count[depth];
    const int groups = (count + 31) / 32;
    if (blockIdx.x * kInferWarps >= groups) return;  // no rays for this block: skip the weight copy
    uint32_t* sw = ism;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* sx = ism + kSWords + warp * 32 * kSXStride;
    // outputs overwrite the inputs of the same 16-row group: every lane has loaded its input
    // fragments into registers before the warp-synchronous mma chain reaches the output stores
    const float* sy = reinterpret_cast<const float*>(sx);
    if (!B) guide_load_weights(p.gwpack, sw);
    __syncthreads();
    const PathQueue q = p.q[depth & 1];
    for (int grp = blockIdx.x * kInferWarps + warp; grp < groups; grp += gridDim.x * kInferWarps) {
        const int slot = grp * 32 + lane;
        float x[kGuideIn];
        if (!B) {
            if (slot < count) guide_features(p, p.gframe, q.o[slot], q.d[slot], q.hit[slot], x);
            else
                for (int k = 0; k < kGuideIn; k++) x[k] = 0.f;
            guide_store_input(sx, lane, x);
            __syncwarp();
            guide_mlp_warp32(sw, sx);
            __syncwarp();
            guide_activate_row(sx, lane);
            __syncwarp();
            const int rows = count - grp * 32 < 32 ? count - grp * 32 : 32;
            float* dst = p.gmix + (size_t)grp * 32 * kGuideOut;
            for (int e = lane; e < rows * kGuideOut; e += 32)
                dst[e] = sy[(e / (16 * kGuideOut)) * 16 * kSXStride + e % (16 * kGuideOut)];
            __syncwarp();
        } else {
            int net = -1, sid = 0;
            float4 o4 = make_float4(0.f, 0.f, 0.f, 0.f), d4 = o4, h4 = o4;
            if (slot < count) {
                o4 = q.o[slot];
                d4 = q.d[slot];
                h4 = q.hit[slot];
                sid = tag_scene(__float_as_int(o4.w));
                const BatchScene& sb = p.batch[sid];
                if (sb.guide_mode == 2 && __float_as_int(h4.w) != kMissPrim) net = sb.guide_net;
            }
            unsigned pending = __ballot_sync(0xffffffffu, net >= 0);
            while (pending) {
                const int lnet = __shfl_sync(0xffffffffu, net, __ffs(pending) - 1);
                const bool mine = net == lnet;
                if (mine) guide_features(p, p.batch[sid].gframe, o4, d4, h4, x);
                else
                    for (int k = 0; k < kGuideIn; k++) x[k] = 0.f;
                __syncwarp();
                guide_store_input(sx, lane, x);
                __syncwarp();
                guide_mlp_warp32(p.gwpack + (size_t)lnet * kGuidePackWords, sx);
                __syncwarp();
                const float* row = guide_activate_row(sx, lane);
                if (mine) {
                    float4* dst = reinterpret_cast<float4*>(p.gmix + (size_t)slot * kGuideOut);
                    const float4* src = reinterpret_cast<const float4*>(row);
                    for (int j = 0; j < kGuideOut / 4; j++) dst[j] = src[j];
                }
                pending &= ~__ballot_sync(0xffffffffu, mine);
            }
            __syncwarp();
        }
    }
}

// Guide inference on the 5th-generation tensor cores: tiles of 256 queue slots (two MMA
// sub-tiles of 128), one thread per slot; the network runs as tcgen05.mma into tensor memory
// (guide_tc.cuh). 128 registers keep 2 CTAs (512 slots) resident per SM.
__global__ void __launch_bounds__(kTcThreads, 2) k_guide_infer_tc(FrameParams p, int depth) {
    extern __shared__ __align__(1024) uint8_t tsm[];
    TcSmem& s = *reinterpret_cast<TcSmem*>(tsm);
    const int count = p.counters->ray_count[depth];
    const int tiles = (count + kTcThreads - 1) / kTcThreads;
    if ((int)blockIdx.x >= tiles) return;  // no work: skip the setup and the TMEM allocation
    const uint32_t tmem = tc_setup(s, p.gwpack, p.gwpack + kPackWords);
    uint32_t phase = 0;
    const PathQueue q = p.q[depth & 1];
    const int t = threadIdx.x;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int slot = tile * kTcThreads + t;
        float x[kGuideIn];
        if (slot < count) guide_features(p, p.gframe, q.o[slot], q.d[slot], q.hit[slot], x);
        else
            for (int k = 0; k < kGuideIn; k++) x[k] = 0.f;
        tc_store_input(s.a[tc_sub()], tc_row(), x);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        float raw[kGuideOut];
        if (!tc_network(s, tmem, phase, raw, p.mma_test_polls)) {
            if (t == 0) atomicOr(&p.stats->error, 2);
            break;
        }
        if (slot < count) {
            float mix[kGuideOut];
            guide_activate(raw, mix);
            float4* dst = reinterpret_cast<float4*>(p.gmix + (size_t)slot * kGuideOut);
#pragma unroll
            for (int j = 0; j < kGuideOut / 4; j++)
                dst[j] = make_float4(mix[4 * j], mix[4 * j + 1], mix[4 * j + 2], mix[4 * j + 3]);
        }
    }
    tc_teardown(tmem);
}

// Resolve this wave's training records into samples: the radiance that arrived along each
// sampled direction is the path's later contributions (unweighted emission at the next
// vertex, everything after it) divided by the throughput after the vertex.
template <bool B>
__global__ void k_guide_collect(FrameParams p) {
    const int n = min(*p.grec_count, p.grec_cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const GuideRecord r = p.grec[i];
        const int net = B ? p.batch[r.depth >> 8].guide_net : 0;  // the record's scene's network
        if (net < 0) continue;
        const float* a = p.gacc + (size_t)r.tpath * p.max_depth * 3;
        float lin = 0.f;
        const int k1 = (r.depth & 0xFF) + 1;
        if (k1 < p.max_depth) {
            float sum_r = 0.f;
            for (int d = k1; d < p.max_depth; d++) sum_r += a[3 * d + 1];
            lin = (a[3 * k1] + sum_r - a[3 * k1 + 2]) / r.beta_next;
        }
        const float weight = r.fcos_over_p * lin;
        if (!(weight > 0.f) || !isfinite(weight)) continue;
        const int idx = atomicAdd(p.gring_count + net, 1);
        GuideSample smp;
        for (int k = 0; k < 3; k++) {
            smp.p[k] = r.p[k];
            smp.n[k] = r.n[k];
            smp.wo[k] = r.wo[k];
            smp.wi[k] = r.wi[k];
        }
        smp.weight = weight;
        smp.pad[0] = smp.pad[1] = smp.pad[2] = 0.f;
        p.gring[(size_t)net * p.gring_cap + (unsigned)idx % (unsigned)p.gring_cap] = smp;
    }
}

template <bool B>
__global__ void k_accumulate(FrameParams p, int first_pixel, int npix, long long wave_first) {
    const int pi = blockIdx.x * blockDim.x + threadIdx.x;
    if (pi >= npix) return;
    const int pixel = first_pixel + pi;
    int spp = p.spp, prev_spp;
    long long path0 = (long long)pi * p.spp;  // wave-local index of the pixel's first sample
    if (B) {
        const int sid = batch_find(p.batch_pixel_base, p.num_scenes, pixel);
        const BatchScene& sb = p.batch[sid];
        spp = sb.spp;
        path0 = sb.path_base + (pixel - sb.pixel_base) * (long long)spp - wave_first;
        prev_spp = sb.prev_spp;
    } else {
        prev_spp = p.dyn->prev_spp;
    }
    float r = 0.f, g = 0.f, b = 0.f;
    const float inv_spp = (float)spp;
    if ((spp & (spp - 1)) == 0) {
        // a power-of-two spp: x / spp and x * (1 / spp) are the same correctly rounded value
        // (the reciprocal is exact), without a division per sample
        const float rs = 1.f / inv_spp;
        for (int s = 0; s < spp; s++) {  // passRadiances += Li / spp (path_tracer.cu:258-262)
            const float4 l = p.L[path0 + s];
            r += l.x * rs;
            g += l.y * rs;
            b += l.z * rs;
        }
    } else {
        for (int s = 0; s < spp; s++) {
            const float4 l = p.L[path0 + s];
            r += l.x / inv_spp;
            g += l.y / inv_spp;
            b += l.z / inv_spp;
        }
    }
    p.pass_rgb[3 * (size_t)pixel + 0] = r;
    p.pass_rgb[3 * (size_t)pixel + 1] = g;
    p.pass_rgb[3 * (size_t)pixel + 2] = b;
    float nr = r, ng = g, nb = b;
    if (prev_spp > 0) {  // running mean (framebuffer.cu:23-33)
        const float prev = (float)prev_spp;
        const float total = (float)(prev_spp + spp);
        const float wpass = 1.f * spp / total;
        nr = p.accum_rgb[3 * (size_t)pixel + 0] * prev / total + r * wpass;
        ng = p.accum_rgb[3 * (size_t)pixel + 1] * prev / total + g * wpass;
        nb = p.accum_rgb[3 * (size_t)pixel + 2] * prev / total + b * wpass;
    }
    p.accum_rgb[3 * (size_t)pixel + 0] = nr;
    p.accum_rgb[3 * (size_t)pixel + 1] = ng;
    p.accum_rgb[3 * (size_t)pixel + 2] = nb;
    uchar4 c;
    c.x = (unsigned char)(fmaxf(0.f, fminf(1.f, to_srgb(nr))) * 255);
    c.y = (unsigned char)(fmaxf(0.f, fminf(1.f, to_srgb(ng))) * 255);
    c.z = (unsigned char)(fmaxf(0.f, fminf(1.f, to_srgb(nb))) * 255);
    c.w = 255;
    p.rgba8[pixel] = c;
}

// Records an event on its stream after each launch; a stage's time runs from the previous
// event on the same stream (stage -1 marks a point with no launch before it: a wave's start,
// or the end of a wait for the other stream).
struct Marker {
    StageMarks* m;
    cudaStream_t s;
    cudaError_t err = cudaSuccess;
    int last = -1;
    void operator()(int stage) {
        if (!m || err != cudaSuccess) return;
        if (m->used >= m->capacity) { err = cudaErrorInvalidValue; return; }
        m->stage[m->used] = stage;
        m->begin[m->used] = last;
        last = m->used;
        err = cudaEventRecord(m->events[m->used++], s);
    }
};

// The plain shade stage of material-sorted frames: one kernel per material class present
// (p.class_mask), each over its class's range of the sorted order. The class kernels hold
// fewer registers than the kernel of all materials; each persistent grid is as many blocks
// as the SMs keep resident at that register budget, and a class absent at a depth returns
// before its first fetch.
// With `par`, each class kernel runs on its own stream, forked from and joined back to
// `stream`: the classes touch disjoint paths and append through atomics, so they may run
// side by side, each filling the SMs the others' ramps and tails leave idle.
template <bool B>
cudaError_t enqueue_class_shades(const FrameParams& p, int d, long long wave_first, long long gfirst,
                                 cudaStream_t stream, const SideStream* par) {
    const int bs = p.shape.block_shade;
    auto grid = [&](int cls) {
        const int per_sm = std::max(1, std::min(65536 / (shade_class_regs(cls) * bs), 2048 / bs));
        return p.num_sms * per_sm;
    };
    cudaError_t e;
    if (par && (e = cudaEventRecord(par->cls_fork, stream))) return e;
    cudaError_t we = cudaSuccess;
    auto on = [&](int cls) -> cudaStream_t {
        if (!par) return stream;
        const cudaError_t w = cudaStreamWaitEvent(par->cls[cls], par->cls_fork, 0);
        if (w != cudaSuccess) we = w;
        return par->cls[cls];
    };
    if (p.class_mask & 1) k_shade_class<B, 0><<<grid(0), bs, 0, on(0)>>>(p, d, wave_first, gfirst);
    if (p.class_mask & 2) k_shade_class<B, 1><<<grid(1), bs, 0, on(1)>>>(p, d, wave_first, gfirst);
    if (p.class_mask & 4) k_shade_class<B, 2><<<grid(2), bs, 0, on(2)>>>(p, d, wave_first, gfirst);
    if (p.class_mask & 8) k_shade_class<B, 3><<<grid(3), bs, 0, on(3)>>>(p, d, wave_first, gfirst);
    if (p.class_mask & 16) k_shade_class<B, 4><<<grid(4), bs, 0, on(4)>>>(p, d, wave_first, gfirst);
    if (p.class_mask & 64) k_shade_class<B, 6><<<grid(6), bs, 0, on(6)>>>(p, d, wave_first, gfirst);
    if ((e = cudaGetLastError())) return e;
    if (we != cudaSuccess) return we;
    if (par)
        for (int c = 0; c < kMaterialClasses; c++) {
            if (!(p.class_mask & (1 << c))) continue;
            if ((e = cudaEventRecord(par->cls_done[c], par->cls[c]))) return e;
            if ((e = cudaStreamWaitEvent(stream, par->cls_done[c], 0))) return e;
        }
    return cudaSuccess;
}

template <int W, bool CNT, bool B>
cudaError_t enqueue_waves(const FrameParams& p_in, const WaveRange* waves, int nwaves, cudaStream_t stream,
                          StageMarks* marks, const SideStream* side) {
    // depth-0 rays are computed where they are used when every depth-0 stage can do so: plain
    // frames whose shade stage is the kernel of all materials at 128 registers
    FrameParams p = p_in;
    const bool classes = p.shape.shade_kernel == kShadeClasses && p.shape.sort_materials && p.class_mask;
    p.cam_fused = p.shape.fuse_camera && !p.guide_mode && !classes && p.shape.shade_kernel != kShadeAll80 ? 1 : 0;
    const int grid_e = p.num_sms * p.shape.blocks_per_sm;
    // shadow stage of depth d on the side stream: forked after the shade stage of d, joined
    // before the shade stage of d + 1 (which adds to the same path radiance after it); the
    // closest-hit stage of d + 1 runs beside it
    const bool concurrent = side && side->stream && p.shape.overlap_shadow;
    const bool overlap = concurrent && p.nee;
    const cudaStream_t sstream = overlap ? side->stream : stream;
    const size_t smem_e = stack_bytes(p.stack_depth, p.shape.block_extend);
    const size_t smem_s = stack_bytes(p.stack_depth, p.shape.block_shadow);
    Marker mark{marks, stream};
    Marker smark{marks, sstream};  // the side stream's shadow stages
    for (int wv = 0; wv < nwaves; wv++) {
        const WaveRange& w = waves[wv];
        const int n = w.npaths;
        const long long wave_first = w.first_path;
        cudaError_t e = cudaMemsetAsync(p.counters, 0, sizeof(WaveCounters), stream);
        if (e != cudaSuccess) return e;
        const bool sort_rays = !B && p.shape.sort_rays;
        if (sort_rays && (e = cudaMemsetAsync(p.ray_hist, 0, 2 * p.max_depth * kRayBuckets * sizeof(int), stream)))
            return e;
        if (p.guide_mode) {
            const size_t tpaths = (size_t)(w.guided_n + p.gstride - 1) / p.gstride;
            if ((e = cudaMemsetAsync(p.gacc, 0, tpaths * p.max_depth * 3 * sizeof(float), stream))) return e;
            if ((e = cudaMemsetAsync(p.grec_count, 0, sizeof(int), stream))) return e;
        }
        mark(-1);
        if (p.cam_fused) k_wave_start<<<p.max_depth == 0 ? (n + 255) / 256 : 1, 256, 0, stream>>>(p, n);
        else k_camera<B><<<(n + 255) / 256, 256, 0, stream>>>(p, wave_first, n);
        mark(kStageCamera);
        for (int d = 0; d < p.max_depth; d++) {
            if (sort_rays && d > 0) {  // keys and counts come from the previous shade launch
                k_ray_scatter<<<p.num_sms * 4, kRaySortBlock, 0, stream>>>(p, d);
                mark(kStageSort);
            }
            if (p.sc.watertight) {
                k_extend<W, CNT, B, 2><<<grid_e, p.shape.block_extend, smem_e, stream>>>(p, d, wave_first);
            } else if constexpr (W >= 4) {
                if (p.sc.node_q) k_extend<W, CNT, B, 1><<<grid_e, p.shape.block_extend, smem_e, stream>>>(p, d, wave_first);
                else k_extend<W, CNT, B, 0><<<grid_e, p.shape.block_extend, smem_e, stream>>>(p, d, wave_first);
            } else {
                k_extend<W, CNT, B, 0><<<grid_e, p.shape.block_extend, smem_e, stream>>>(p, d, wave_first);
            }
            mark(kStageExtend);
            if (p.shape.sort_materials) {
                k_sort<<<std::min((n + 256 * kSortItems - 1) / (256 * kSortItems), p.num_sms * 8), 256, 0, stream>>>(
                    p, d);
                mark(kStageSort);
            }
            if (p.guide_mode == 2 && d < p.max_depth - 1) {
                if (!B && p.guide_tc)
                    k_guide_infer_tc<<<p.num_sms * 2, kTcThreads, sizeof(TcSmem), stream>>>(p, d);
                else
                    k_guide_infer<B><<<p.num_sms * 2, 32 * kInferWarps, kInferSmemBytes, stream>>>(p, d);
                mark(kStageGuide);
            }
            if (overlap && d > 0) {
                if ((e = cudaStreamWaitEvent(stream, side->shadowed[d - 1], 0))) return e;
                mark(-1);  // the shade stage's time starts after the wait
            }
            if (p.guide_mode)
                k_shade<true, B><<<p.num_sms * kShadeGuidedBlocksPerSm, kShadeGuidedBlock, 0, stream>>>(
                    p, d, wave_first, w.guided_first);
            else if (p.shape.shade_kernel == kShadeClasses && p.shape.sort_materials && p.class_mask)
                e = enqueue_class_shades<B>(p, d, wave_first, w.guided_first, stream,
                                            concurrent && !marks && side->cls ? side : nullptr);
            else if (p.shape.shade_kernel == kShadeAll80)
                k_shade_all<B, 80><<<p.num_sms * shade_resident(80, p.shape.block_shade), p.shape.block_shade, 0,
                                     stream>>>(p, d, wave_first, w.guided_first);
            else
                k_shade_all<B, 128><<<p.num_sms * shade_resident(128, p.shape.block_shade), p.shape.block_shade, 0,
                                      stream>>>(p, d, wave_first, w.guided_first);
            if (e != cudaSuccess) return e;
            mark(kStageShade);
            if (p.nee && d < p.max_depth - 1) {
                if (overlap) {
                    if ((e = cudaEventRecord(side->shaded[d], stream))) return e;
                    if ((e = cudaStreamWaitEvent(sstream, side->shaded[d], 0))) return e;
                    smark(-1);
                }
                if (p.sc.watertight)
                    k_shadow<W, CNT, B, 2><<<grid_e, p.shape.block_shadow, smem_s, sstream>>>(p, d, wave_first,
                                                                                            w.guided_first);
                else if (W >= 4 && p.sc.node_q)
                    k_shadow<W, CNT, B, (W >= 4 ? 1 : 0)><<<grid_e, p.shape.block_shadow, smem_s, sstream>>>(
                        p, d, wave_first, w.guided_first);
                else
                    k_shadow<W, CNT, B, 0><<<grid_e, p.shape.block_shadow, smem_s, sstream>>>(p, d, wave_first,
                                                                                            w.guided_first);
                if (overlap) {
                    if ((e = cudaEventRecord(side->shadowed[d], sstream))) return e;
                    smark(kStageShadow);
                } else {
                    mark(kStageShadow);
                }
            }
        }
        k_accumulate<B><<<(w.npix + 127) / 128, 128, 0, stream>>>(p, w.first_pixel, w.npix, wave_first);
        mark(kStageAccum);
        if (p.guide_mode) {
            k_guide_collect<B><<<p.num_sms * 2, 256, 0, stream>>>(p);
            mark(kStageGuide);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (mark.err != cudaSuccess) return mark.err;
        if (smark.err != cudaSuccess) return smark.err;
    }
    return cudaSuccess;
}

// The hit record's normal (Triangle::hit's interpolated (1 - b1 - b2) n0 + b1 n1 + b2 n2,
// triangle.h:51-56; Sphere::hit's normalized((point - center) / radius), sphere.cu:19-24)
// with every operation rounded on its own, as the reference's arithmetic reads.
__device__ __forceinline__ V hit_normal_rn(const SceneDevice& sc, V o, V d, const Hit& h) {
    if (h.prim >= 0) {
        const float w0 = __fsub_rn(__fsub_rn(1.f, h.b1), h.b2);
        const V n0 = mkv(__ldg(sc.tri_n + 3 * h.prim + 0));
        const V n1 = mkv(__ldg(sc.tri_n + 3 * h.prim + 1));
        const V n2 = mkv(__ldg(sc.tri_n + 3 * h.prim + 2));
        return V{__fadd_rn(__fadd_rn(__fmul_rn(w0, n0.x), __fmul_rn(h.b1, n1.x)), __fmul_rn(h.b2, n2.x)),
                 __fadd_rn(__fadd_rn(__fmul_rn(w0, n0.y), __fmul_rn(h.b1, n1.y)), __fmul_rn(h.b2, n2.y)),
                 __fadd_rn(__fadd_rn(__fmul_rn(w0, n0.z), __fmul_rn(h.b1, n1.z)), __fmul_rn(h.b2, n2.z))};
    }
    const float4 s = __ldg(sc.sph + ~h.prim);
    const V q{__fdiv_rn(__fsub_rn(__fadd_rn(o.x, __fmul_rn(h.t, d.x)), s.x), s.w),
              __fdiv_rn(__fsub_rn(__fadd_rn(o.y, __fmul_rn(h.t, d.y)), s.y), s.w),
              __fdiv_rn(__fsub_rn(__fadd_rn(o.z, __fmul_rn(h.t, d.z)), s.z), s.w)};
    const float len = __fsqrt_rn(xdot(q, q));
    return V{__fdiv_rn(q.x, len), __fdiv_rn(q.y, len), __fdiv_rn(q.z, len)};
}

// Normals renderer (GBuffer with BufferType::Normals, src/renderers/g_buffer.cu:27-57): one
// pixel-centre camera ray per pixel (Camera::generateRay(row, col), camera.cu:24-27), the
// closest hit's (shading normal + 1) / 2, black on a miss; the accumulate kernel then treats
// it as a 1-spp frame, as updateFramebuffer does for the reference.
template <int W>
__global__ void k_normals(FrameParams p, int first_pixel, int npix) {
    extern __shared__ int2 stk[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < npix;  // every lane enters the warp-synchronous traversal
    const int pixel = first_pixel + (valid ? i : 0);
    const int row = pixel / p.width, col = pixel - row * p.width;
    V o, d;
    camera_ray(p.dyn->cam, row, col, 0.5f, 0.5f, o, d);
    const RayPre r = make_raypre(o, d);
    Hit h;
    int of = 0;
    traverse<W, false>(p.sc, r, kCameraTMin, FLT_MAX, valid, stk + threadIdx.x, blockDim.x, p.stack_depth, h, of);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.stats->rays_camera, (unsigned long long)npix);
    if (!valid) return;
    if (of) atomicOr(&p.stats->error, 1);
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    if (h.prim != kMissPrim) {
        const V n = hit_normal_rn(p.sc, o, d, h);
        out = make_float4(__fdiv_rn(__fadd_rn(n.x, 1.f), 2.f), __fdiv_rn(__fadd_rn(n.y, 1.f), 2.f),
                          __fdiv_rn(__fadd_rn(n.z, 1.f), 2.f), 0.f);
    }
    p.L[i] = out;
}

// Normals frame: waves of whole pixels, one pixel-centre ray each, then the accumulation.
template <int W>
cudaError_t enqueue_normals_w(const FrameParams& p, cudaStream_t stream, StageMarks* marks) {
    const int npixels = p.width * p.height;
    const int bs = p.shape.block_extend;  // the stack size the session configured covers this block
    const size_t smem = stack_bytes(p.stack_depth, bs);
    Marker mark{marks, stream};
    mark(-1);
    for (int first = 0; first < npixels; first += p.wave_pixels) {
        const int npix = npixels - first < p.wave_pixels ? npixels - first : p.wave_pixels;
        k_normals<W><<<(npix + bs - 1) / bs, bs, smem, stream>>>(p, first, npix);
        mark(kStageExtend);
        k_accumulate<false><<<(npix + 127) / 128, 128, 0, stream>>>(p, first, npix, (long long)first);
        mark(kStageAccum);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (mark.err != cudaSuccess) return mark.err;
    }
    return cudaSuccess;
}

// Single-scene frame: waves of whole pixels, p.wave_pixels each.
template <int W, bool CNT>
cudaError_t enqueue_frame_w(const FrameParams& p, cudaStream_t stream, StageMarks* marks, const SideStream* side) {
    const int npixels = p.width * p.height;
    const int nwaves = (npixels + p.wave_pixels - 1) / p.wave_pixels;
    WaveRange local[64];
    std::vector<WaveRange> heap;
    WaveRange* waves = local;
    if (nwaves > 64) {
        heap.resize(nwaves);
        waves = heap.data();
    }
    for (int k = 0; k < nwaves; k++) {
        const int first = k * p.wave_pixels;
        const int npix = npixels - first < p.wave_pixels ? npixels - first : p.wave_pixels;
        waves[k] = WaveRange{first, npix, (long long)first * p.spp, npix * p.spp, 0, 0, npix * p.spp, 0};
    }
    return enqueue_waves<W, CNT, false>(p, waves, nwaves, stream, marks, side);
}

template <int W>
cudaError_t set_smem_w(size_t bytes) {
    const int b = (int)bytes;
    cudaError_t e;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    constexpr int kQ = W >= 4 ? 1 : 0;  // the quantized-node variants (W >= 4)
    if ((e = cudaFuncSetAttribute(k_extend<W, false, false, 0>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_extend<W, true, false, 0>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_shadow<W, false, false, 0>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_shadow<W, true, false, 0>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_extend<W, false, true, 0>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_extend<W, true, true, 0>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_shadow<W, false, true, 0>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_shadow<W, true, true, 0>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_extend<W, false, false, kQ>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_extend<W, true, false, kQ>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_shadow<W, false, false, kQ>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_shadow<W, true, false, kQ>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_extend<W, false, true, kQ>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_extend<W, true, true, kQ>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_shadow<W, false, true, kQ>, a, b))) return e;
    if ((e = cudaFuncSetAttribute(k_shadow<W, true, true, kQ>, a, b))) return e;
    for (int cnt = 0; cnt < 2; cnt++)  // the watertight variants (Q = 2)
        for (int bt = 0; bt < 2; bt++) {
            const void* ke = cnt ? (bt ? (const void*)k_extend<W, true, true, 2> : (const void*)k_extend<W, true, false, 2>)
                                 : (bt ? (const void*)k_extend<W, false, true, 2> : (const void*)k_extend<W, false, false, 2>);
            const void* ks = cnt ? (bt ? (const void*)k_shadow<W, true, true, 2> : (const void*)k_shadow<W, true, false, 2>)
                                 : (bt ? (const void*)k_shadow<W, false, true, 2> : (const void*)k_shadow<W, false, false, 2>);
            if ((e = cudaFuncSetAttribute(ke, a, b))) return e;
            if ((e = cudaFuncSetAttribute(ks, a, b))) return e;
        }
    if ((e = cudaFuncSetAttribute(k_normals<W>, a, b))) return e;
    return cudaSuccess;
}

template <int W>
__global__ void k_trace_rays(SceneDevice sc, int stack_depth, const float* __restrict__ o,
                             const float* __restrict__ d, const float* __restrict__ tmin,
                             const float* __restrict__ tmax, int n, int* prim_type, int* prim_id, int* mat_id,
                             float* t, float* bary, int* overflow) {
    extern __shared__ int2 stk[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;  // every lane enters the warp-synchronous traversal
    const int j = valid ? i : 0;
    const RayPre r = make_raypre(mkv(o[3 * j], o[3 * j + 1], o[3 * j + 2]), mkv(d[3 * j], d[3 * j + 1], d[3 * j + 2]));
    Hit h;
    int of = 0;
    traverse<W, false>(sc, r, tmin[j], tmax[j], valid, stk + threadIdx.x, blockDim.x, stack_depth, h, of);
    if (!valid) return;
    if (of) atomicOr(overflow, 1);
    if (h.prim == kMissPrim) {
        prim_type[i] = -1;
        prim_id[i] = -1;
        mat_id[i] = -1;
        t[i] = 0.f;
        if (bary) { bary[2 * i] = 0.f; bary[2 * i + 1] = 0.f; }
    } else if (h.prim >= 0) {
        prim_type[i] = kTriangle;
        prim_id[i] = h.prim;
        mat_id[i] = sc.tri_mat[h.prim];
        t[i] = h.t;
        if (bary) { bary[2 * i] = h.b1; bary[2 * i + 1] = h.b2; }
    } else {
        prim_type[i] = kSphere;
        prim_id[i] = ~h.prim;
        mat_id[i] = sc.sph_mat[~h.prim];
        t[i] = h.t;
        if (bary) { bary[2 * i] = 0.f; bary[2 * i + 1] = 0.f; }
    }
}

template <int W>
__global__ void k_occluded(SceneDevice sc, int stack_depth, const float* __restrict__ o,
                           const float* __restrict__ d, const float* __restrict__ tmin,
                           const float* __restrict__ tmax, int n, int* occluded, int* overflow) {
    extern __shared__ int2 stk[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const int j = valid ? i : 0;
    const RayPre r = make_raypre(mkv(o[3 * j], o[3 * j + 1], o[3 * j + 2]), mkv(d[3 * j], d[3 * j + 1], d[3 * j + 2]));
    Hit h;
    int of = 0;
    const bool occ = traverse<W, true>(sc, r, tmin[j], tmax[j], valid, stk + threadIdx.x, blockDim.x, stack_depth, h, of);
    if (!valid) return;
    occluded[i] = occ ? 1 : 0;
    if (of) atomicOr(overflow, 1);
}

template <int W>
__global__ void k_hit_test(SceneDevice sc, CameraParams cam, int stack_depth, int x, int y, int* out, int* overflow) {
    extern __shared__ int2 stk[];
    V o, d;
    camera_ray(cam, y, x, 0.5f, 0.5f, o, d);
    const RayPre r = make_raypre(o, d);
    Hit h;
    int of = 0;
    // the whole warp enters the traversal; lane 0 carries the query and owns the stack
    traverse<W, false>(sc, r, 0.f, FLT_MAX, threadIdx.x == 0, stk, 1, stack_depth, h, of);
    if (threadIdx.x != 0) return;
    if (of) atomicOr(overflow, 1);
    if (h.prim == kMissPrim) *out = -1;
    else if (h.prim >= 0) *out = sc.tri_mat[h.prim];
    else *out = sc.sph_mat[~h.prim];
}

}  // namespace

cudaError_t enqueue_frame(const FrameParams& p, cudaStream_t stream, StageMarks* marks, const SideStream* side) {
    if (p.max_depth < 0 || p.max_depth > kMaxDepthLimit) return cudaErrorInvalidValue;
    if (p.renderer == 1) {
        if (p.spp != 1) return cudaErrorInvalidValue;
        switch (p.sc.bvh_width) {
            case 2: return enqueue_normals_w<2>(p, stream, marks);
            case 4: return enqueue_normals_w<4>(p, stream, marks);
            case 8: return enqueue_normals_w<8>(p, stream, marks);
            default: return cudaErrorInvalidValue;
        }
    }
    const bool cnt = p.count_work != 0;
    switch (p.sc.bvh_width) {
        case 2: return cnt ? enqueue_frame_w<2, true>(p, stream, marks, side) : enqueue_frame_w<2, false>(p, stream, marks, side);
        case 4: return cnt ? enqueue_frame_w<4, true>(p, stream, marks, side) : enqueue_frame_w<4, false>(p, stream, marks, side);
        case 8: return cnt ? enqueue_frame_w<8, true>(p, stream, marks, side) : enqueue_frame_w<8, false>(p, stream, marks, side);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t enqueue_batch_frame(const FrameParams& p, const WaveRange* waves, int nwaves, cudaStream_t stream,
                                StageMarks* marks, const SideStream* side) {
    if (p.max_depth < 0 || p.max_depth > kMaxDepthLimit || p.num_scenes <= 0) return cudaErrorInvalidValue;
    const bool cnt = p.count_work != 0;
    switch (p.sc.bvh_width) {
        case 2: return cnt ? enqueue_waves<2, true, true>(p, waves, nwaves, stream, marks, side)
                           : enqueue_waves<2, false, true>(p, waves, nwaves, stream, marks, side);
        case 4: return cnt ? enqueue_waves<4, true, true>(p, waves, nwaves, stream, marks, side)
                           : enqueue_waves<4, false, true>(p, waves, nwaves, stream, marks, side);
        case 8: return cnt ? enqueue_waves<8, true, true>(p, waves, nwaves, stream, marks, side)
                           : enqueue_waves<8, false, true>(p, waves, nwaves, stream, marks, side);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t configure_guide_infer() {
    cudaError_t e = cudaFuncSetAttribute(k_guide_infer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kInferSmemBytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_guide_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_guide_infer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmemBytes);
}

cudaError_t configure_traversal_smem(size_t bytes) {
    cudaError_t e;
    if ((e = set_smem_w<2>(bytes))) return e;
    if ((e = set_smem_w<4>(bytes))) return e;
    return set_smem_w<8>(bytes);
}

cudaError_t enqueue_trace_rays(const SceneDevice& sc, int stack_depth, const float* o, const float* d,
                               const float* tmin, const float* tmax, int n, int* prim_type, int* prim_id,
                               int* mat_id, float* t, float* bary, int* overflow, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int bs = 128;
    const size_t smem = stack_bytes(stack_depth, bs);
    const int grid = (n + bs - 1) / bs;
    switch (sc.bvh_width) {
        case 2: k_trace_rays<2><<<grid, bs, smem, stream>>>(sc, stack_depth, o, d, tmin, tmax, n, prim_type, prim_id, mat_id, t, bary, overflow); break;
        case 4: k_trace_rays<4><<<grid, bs, smem, stream>>>(sc, stack_depth, o, d, tmin, tmax, n, prim_type, prim_id, mat_id, t, bary, overflow); break;
        case 8: k_trace_rays<8><<<grid, bs, smem, stream>>>(sc, stack_depth, o, d, tmin, tmax, n, prim_type, prim_id, mat_id, t, bary, overflow); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t enqueue_occluded(const SceneDevice& sc, int stack_depth, const float* o, const float* d,
                             const float* tmin, const float* tmax, int n, int* occluded, int* overflow,
                             cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int bs = 128;
    const size_t smem = stack_bytes(stack_depth, bs);
    const int grid = (n + bs - 1) / bs;
    switch (sc.bvh_width) {
        case 2: k_occluded<2><<<grid, bs, smem, stream>>>(sc, stack_depth, o, d, tmin, tmax, n, occluded, overflow); break;
        case 4: k_occluded<4><<<grid, bs, smem, stream>>>(sc, stack_depth, o, d, tmin, tmax, n, occluded, overflow); break;
        case 8: k_occluded<8><<<grid, bs, smem, stream>>>(sc, stack_depth, o, d, tmin, tmax, n, occluded, overflow); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// ---- closest-hit queries without allocation ----------------------------------------------
// Staging area of trace_rays_static, one per device that loads the library (about 3.7 MB,
// held until the process exits): rays in (o, d, tmin, tmax), results out (type, id,
// material, t, barycentrics) and the traversal-overflow flag. Every call reuses it and it
// keeps the previous call's contents; the flag is cleared at the start of each call. Calls
// whose work overlaps on the GPU (other streams, other host threads) race on it.
namespace {
constexpr size_t kStaticRayWords = 14;  // 3 + 3 + 1 + 1 floats in, 1 + 1 + 1 + 1 + 2 words out
constexpr size_t kStaticScratchWords = (size_t)kStaticTraceMaxRays * kStaticRayWords + 64;
static __device__ __align__(256) float g_trace_scratch[kStaticScratchWords];

std::mutex g_scratch_mutex;
float* g_scratch_addr[64] = {};

cudaError_t static_scratch(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_trace_scratch);  // once per device, device current
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<float*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}
}  // namespace

cudaError_t trace_rays_static(const SceneDevice& sc, int stack_depth, const float* o, const float* d,
                              const float* tmin, const float* tmax, int n, int* prim_type, int* prim_id,
                              int* mat_id, float* t, float* bary, int* overflow, cudaStream_t stream) {
    if (n < 0 || n > kStaticTraceMaxRays) return cudaErrorInvalidValue;
    float* base = nullptr;
    cudaError_t e = static_scratch(&base);
    if (e != cudaSuccess) return e;
    const size_t N = kStaticTraceMaxRays;
    float* sO = base;
    float* sD = sO + 3 * N;
    float* sTmin = sD + 3 * N;
    float* sTmax = sTmin + N;
    int* sType = reinterpret_cast<int*>(sTmax + N);
    int* sId = sType + N;
    int* sMat = sId + N;
    float* sT = reinterpret_cast<float*>(sMat + N);
    float* sBary = sT + N;
    int* sFlag = reinterpret_cast<int*>(sBary + 2 * N);
    const size_t b = (size_t)n * sizeof(float);
    // Once a copy is queued, an error returns only after the stream has drained, so no copy
    // into the caller's arrays lands after the call has returned.
    auto enqueue = [&]() -> cudaError_t {
        cudaError_t x;
        if ((x = cudaMemsetAsync(sFlag, 0, sizeof(int), stream))) return x;
        if (n == 0) return cudaSuccess;
        if ((x = cudaMemcpyAsync(sO, o, 3 * b, cudaMemcpyHostToDevice, stream))) return x;
        if ((x = cudaMemcpyAsync(sD, d, 3 * b, cudaMemcpyHostToDevice, stream))) return x;
        if ((x = cudaMemcpyAsync(sTmin, tmin, b, cudaMemcpyHostToDevice, stream))) return x;
        if ((x = cudaMemcpyAsync(sTmax, tmax, b, cudaMemcpyHostToDevice, stream))) return x;
        if ((x = enqueue_trace_rays(sc, stack_depth, sO, sD, sTmin, sTmax, n, sType, sId, sMat, sT, sBary, sFlag,
                                    stream)))
            return x;
        if ((x = cudaMemcpyAsync(prim_type, sType, b, cudaMemcpyDeviceToHost, stream))) return x;
        if ((x = cudaMemcpyAsync(prim_id, sId, b, cudaMemcpyDeviceToHost, stream))) return x;
        if ((x = cudaMemcpyAsync(mat_id, sMat, b, cudaMemcpyDeviceToHost, stream))) return x;
        if ((x = cudaMemcpyAsync(t, sT, b, cudaMemcpyDeviceToHost, stream))) return x;
        if (bary && (x = cudaMemcpyAsync(bary, sBary, 2 * b, cudaMemcpyDeviceToHost, stream))) return x;
        return cudaMemcpyAsync(overflow, sFlag, sizeof(int), cudaMemcpyDeviceToHost, stream);
    };
    e = enqueue();
    const cudaError_t s = cudaStreamSynchronize(stream);
    return e != cudaSuccess ? e : s;
}

cudaError_t enqueue_hit_test(const SceneDevice& sc, const CameraParams& cam, int stack_depth, int x, int y,
                             int* out_material, int* overflow, cudaStream_t stream) {
    const size_t smem = stack_bytes(stack_depth, 1);
    switch (sc.bvh_width) {
        case 2: k_hit_test<2><<<1, 32, smem, stream>>>(sc, cam, stack_depth, x, y, out_material, overflow); break;
        case 4: k_hit_test<4><<<1, 32, smem, stream>>>(sc, cam, stack_depth, x, y, out_material, overflow); break;
        case 8: k_hit_test<8><<<1, 32, smem, stream>>>(sc, cam, stack_depth, x, y, out_material, overflow); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace pt
