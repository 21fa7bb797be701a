// trace.cu — batched closest-hit / occlusion queries over the device BVH.
// The C-ABI entry points aur_trace_closest / aur_trace_occluded run these;
// they replace EmbreeAccelerator::intersect / intersectBinary
// (Aurora/src/geometry/embreeAccelerator.cpp:41-100) for arrays of rays.
#include "aur_kernels.h"
#include "aur_traverse.cuh"

namespace aur {
namespace {

constexpr int kTraceBlock = 128;

__global__ void __launch_bounds__(kTraceBlock) k_trace_closest(const BvhNode* __restrict__ nodes,
                                                               const BvhNode4* __restrict__ nodes4,
                                                               const BvhTri* __restrict__ tris,
                                                               const int* __restrict__ tri_attr,
                                                               const float4* __restrict__ rays, float* hits,
                                                               uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(&rays[2 * i]);
    const float4 b = __ldg(&rays[2 * i + 1]);
    Hit h;
    TraceWork w;
    const bool hit = bvh_closest(nodes, nodes4, tris, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w, &h, w);
    float* o = hits + 5 * (size_t)i;
    o[0] = hit ? h.t : b.w;
    o[1] = hit ? h.u : 0.f;
    o[2] = hit ? h.v : 0.f;
    o[3] = __int_as_float(hit ? h.prim : -1);
    o[4] = __int_as_float(hit ? (tri_attr ? tri_attr[h.prim] : 0) : -1);
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_occluded(const BvhNode* __restrict__ nodes,
                                                                const BvhNode4* __restrict__ nodes4,
                                                                const BvhTri* __restrict__ tris,
                                                                const float4* __restrict__ rays, uint8_t* occ,
                                                                uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(&rays[2 * i]);
    const float4 b = __ldg(&rays[2 * i + 1]);
    TraceWork w;
    occ[i] = bvh_occluded(nodes, nodes4, tris, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w, w) ? 1 : 0;
}

}  // namespace

cudaError_t launch_trace_closest(const DeviceBvh& bvh, const int* tri_attr, const void* rays, void* hits, uint32_t n,
                                 cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_trace_closest<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, s>>>(
        bvh.nodes, bvh.nodes4, bvh.tris, tri_attr, (const float4*)rays, (float*)hits, n);
    return cudaGetLastError();
}

cudaError_t launch_trace_occluded(const DeviceBvh& bvh, const void* rays, uint8_t* occ, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_trace_occluded<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, s>>>(bvh.nodes, bvh.nodes4, bvh.tris,
                                                                                 (const float4*)rays, occ, n);
    return cudaGetLastError();
}

}  // namespace aur
