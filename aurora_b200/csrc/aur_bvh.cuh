// aur_bvh.cuh — BVH layout shared by the device build and the traversal kernels.
//
// Replaces Embree's "bvh4.spatialsplit"/"triangle4" accelerator
// (Aurora/src/geometry/embreeAccelerator.cpp:19-35). Binary BVH, one 64-byte
// record per interior node holding BOTH children's boxes (so a node visit is
// four coalesced 128-bit loads and two slab tests):
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   d = (ref0, ref1, count0, count1)   ref >= 0: interior node index;
//        ref < 0: leaf; ~ref = start << 5 | count, triangles [start, start+count)
//        (so a leaf holds at most 31 triangles and a BVH at most 2^26 triangles)
// Triangles are stored in leaf order, 48 bytes each, as the exact inputs of the
// Moller-Trumbore test: (p1, prim id bits), (e1 = p2-p1, 0), (e2 = p3-p1, 0).
// Child boxes are padded outward by 2^-19 of their magnitude so that FP32
// rounding in the slab test can never cull a triangle the exact test accepts.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace aur {

struct BvhNode { float4 a, b, c, d; };
struct BvhTri { float4 p1, e1, e2; };

// 4-wide node (128 bytes, one cache line) collapsed from the binary tree: the
// four children's boxes as structure of arrays (lox = the four children's lo.x,
// ...) and their refs in the binary tree's encoding (>= 0: 4-wide node index;
// < 0: leaf ~(start << 5 | count)). The boxes are the binary tree's padded child
// boxes, bit for bit. Unused slots have +inf boxes (never entered) and ref ~0 (an
// empty leaf).
struct BvhNode4 { float4 lox, hix, loy, hiy, loz, hiz; int4 ref; int4 pad; };

struct DeviceBvh {
    BvhNode* nodes = nullptr;     // num_nodes records, root at 0
    BvhTri* tris = nullptr;       // num_tris records in leaf order
    int num_nodes = 0;
    int num_tris = 0;
    int depth = 0;                // longest root-to-leaf path (interior levels + 1)
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};   // scene bounds
    BvhNode4* nodes4 = nullptr;   // the 4-wide form, root at 0 (same triangles)
    int num_nodes4 = 0;
    int depth4 = 0;               // 4-wide levels on the longest path
};

struct BvhBuildOptions {
    int max_leaf = 4;             // triangles per leaf at most (<= 31)
    float cost_traverse = 1.0f;   // SAH node-visit cost
    float cost_intersect = 1.0f;  // SAH triangle-test cost
    int ploc_radius = 16;         // PLOC nearest-neighbour search radius
};

// Builds into freshly allocated device buffers (cudaMallocAsync on `stream`).
// verts: device float3[nvert]; idx: device uint32[3*ntri]. Returns cudaSuccess
// or the first CUDA error. ntri must be >= 1.
cudaError_t bvh_build_device(const float* verts, const uint32_t* idx, int ntri, const BvhBuildOptions& opt,
                             DeviceBvh* out, cudaStream_t stream);
void bvh_free_device(DeviceBvh* bvh, cudaStream_t stream);
// Collapses the binary tree of `bvh` into its 4-wide form (nodes4): each 4-wide node
// takes a binary node's two children and opens its largest-area interior child until
// it holds four, level by level from the root.
cudaError_t bvh_collapse4(DeviceBvh* bvh, cudaStream_t stream);

}  // namespace aur
