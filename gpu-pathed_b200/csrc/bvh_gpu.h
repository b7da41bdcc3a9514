// GPU construction of the wide BVH (bvh_gpu.cu): a Morton-order linear BVH or PLOC clustering,
// collapsed to the host builder's node format.
#pragma once

#include <cuda_runtime.h>

#include "devbuf.h"
#include "pt_types.h"

namespace pt {

// Scratch buffers, kept between builds.
struct GpuBvhScratch {
    DevBuf box_lo, box_hi, cen, bounds, keys, ids, tree, nbox, visits, queue, counters, sort_tmp;
    DevBuf cbox, cint, scan_tmp;  // PLOC clusters
};

// Binary tree of the GPU build: Karras radix tree over the Morton codes, or PLOC clustering.
constexpr int kGpuBvhLbvh = 1;
constexpr int kGpuBvhPloc = 2;

struct GpuBvhInfo {
    int root = 0, num_nodes = 0, depth = 0, max_leaf = 0, width = 4;
};

// Build over nt triangles (3 float4 each: p0 p1 p2) and ns spheres (centre, radius) already on
// the device with the given binary-tree algorithm (kGpuBvhLbvh or kGpuBvhPloc): wide nodes into
// nodes_out, leaf entries (3 float4 each; Morton order for the LBVH, the tree's depth-first
// order for PLOC) into prims_out. Synchronises `st` once per tree level of the collapse and,
// for PLOC, once per clustering pass.
cudaError_t gpu_build_bvh(const float4* tri_p, int nt, const float4* sph, int ns, int width, int max_leaf,
                          GpuBvhScratch& scratch, DevBuf& nodes_out, DevBuf& prims_out, GpuBvhInfo& info,
                          cudaStream_t st, int algorithm = kGpuBvhLbvh);

// Rewrite the n leaf entries' triangles as (p0, id) (p1) (p2) for the watertight test.
cudaError_t prims_to_vertices(float4* prims, int n, const float4* tri_p, cudaStream_t st);

// Quantized copy (qnode_bytes(width) per node, width 4 or 8) of `num_nodes` BvhNode<width>
// nodes on the device. `fail` (device int) is set when a node cannot be quantized
// conservatively (it cannot happen for finite boxes; the check is kept).
cudaError_t quantize_bvh_nodes(const void* nodes, int num_nodes, int width, void* out, int* fail,
                               cudaStream_t stream);

}  // namespace pt
