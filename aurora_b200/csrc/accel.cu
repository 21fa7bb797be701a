// accel.cu — the full contract of EmbreeAccelerator::intersect for arrays of rays
// (Aurora/src/geometry/embreeAccelerator.cpp:41-91): closest hit, then the hit's
// post-process with the per-corner normals and uvs the mesh retains
// (EmbreeMesh::normals / uvs, geometry/embreeMesh.h:62-63):
//   w = 1. - u - v (in double, rounded to float)
//   hitP = org + dir * t
//   hitN = normalize(w n0 + u n1 + v n2), negated first when it faces along dir
//   st   = w st0 + u st1 + v st2
//   barCoords = (u, v, w); ray.maxt = t on a hit (embreeAccelerator.cpp:56)
// The arithmetic is the shading frame's (hit_frame), so a hit reported here and the
// same hit shaded by the renderers agree bit for bit.
#include "aur_capi_internal.h"

namespace aur {
namespace {

constexpr int kIsectBlock = 128;

__global__ void __launch_bounds__(kIsectBlock) k_intersect(const BvhNode* __restrict__ nodes,
                                                           const BvhNode4* __restrict__ nodes4,
                                                           const BvhTri* __restrict__ tris,
                                                           const int* __restrict__ tri_attr,
                                                           const float* __restrict__ corner_n,
                                                           const float* __restrict__ corner_uv, float4* rays,
                                                           aur_isect* out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = rays[2 * i];
    const float4 b = rays[2 * i + 1];
    const float3 o = mk(a.x, a.y, a.z), d = mk(b.x, b.y, b.z);
    Hit h;
    TraceWork work;
    aur_isect r;
    if (!bvh_closest(nodes, nodes4, tris, o, d, a.w, b.w, &h, work)) {
        r.t = b.w; r.u = r.v = 0.f; r.prim = -1; r.attr = -1;
        for (int k = 0; k < 3; ++k) { r.hitP[k] = 0.f; r.hitN[k] = 0.f; r.bar[k] = 0.f; }
        r.st[0] = r.st[1] = 0.f;
        out[i] = r;
        return;
    }
    const float w = (float)(1.0 - h.u - h.v);
    const float* nn = corner_n + (size_t)h.prim * 9;
    float3 N = mk(w * nn[0] + h.u * nn[3] + h.v * nn[6],
                  w * nn[1] + h.u * nn[4] + h.v * nn[7],
                  w * nn[2] + h.u * nn[5] + h.v * nn[8]);
    if (dot(N, d) > 0.f) N *= -1.f;
    N = normalize(N);
    const float3 P = o + d * h.t;
    float s = 0.f, t = 0.f;
    if (corner_uv) {
        const float* uv = corner_uv + (size_t)h.prim * 6;
        s = w * uv[0] + h.u * uv[2] + h.v * uv[4];
        t = w * uv[1] + h.u * uv[3] + h.v * uv[5];
    }
    r.t = h.t; r.u = h.u; r.v = h.v; r.prim = h.prim;
    r.attr = tri_attr ? tri_attr[h.prim] : 0;
    r.hitP[0] = P.x; r.hitP[1] = P.y; r.hitP[2] = P.z;
    r.hitN[0] = N.x; r.hitN[1] = N.y; r.hitN[2] = N.z;
    r.st[0] = s; r.st[1] = t;
    r.bar[0] = h.u; r.bar[1] = h.v; r.bar[2] = w;
    out[i] = r;
    rays[2 * i + 1].w = h.t;                 // ray->maxt = t
}

}  // namespace
}  // namespace aur

using namespace aur;

extern "C" aur_status aur_bvh_set_shading(aur_bvh* b, const float* corner_normals, const float* corner_uvs) {
    if (!b || !corner_normals) return fail(AUR_ERR_INVALID_ARG, "aur_bvh_set_shading: NULL argument");
    if (b->owned_by_scene) return fail(AUR_ERR_INVALID_ARG, "aur_bvh_set_shading: the BVH belongs to a scene, "
                                                            "which provides its normals and uvs");
    DeviceGuard g(b->ctx->device);
    cudaStream_t s = b->ctx->stream;
    const size_t ntri = (size_t)b->bvh.num_tris;
    if (b->owns_shading) {
        if (b->corner_n) cudaFreeAsync(b->corner_n, s);
        if (b->corner_uv) cudaFreeAsync(b->corner_uv, s);
        b->corner_n = b->corner_uv = nullptr;
        b->owns_shading = false;
    }
    float *cn = nullptr, *cu = nullptr;
    cudaError_t e = cudaMallocAsync(&cn, sizeof(float) * 9 * ntri, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cn, corner_normals, sizeof(float) * 9 * ntri, cudaMemcpyDefault, s);
    if (e == cudaSuccess && corner_uvs) e = cudaMallocAsync(&cu, sizeof(float) * 6 * ntri, s);
    if (e == cudaSuccess && corner_uvs) e = cudaMemcpyAsync(cu, corner_uvs, sizeof(float) * 6 * ntri, cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        if (cn) cudaFreeAsync(cn, s);
        if (cu) cudaFreeAsync(cu, s);
        cudaStreamSynchronize(s);
        return cuda_fail(e, "aur_bvh_set_shading");
    }
    b->corner_n = cn;
    b->corner_uv = cu;
    b->owns_shading = true;
    return AUR_OK;
}

extern "C" aur_status aur_bvh_intersect(aur_bvh* b, aur_ray* rays, aur_isect* isects, uint32_t n) {
    if (!b || (n && (!rays || !isects))) return fail(AUR_ERR_INVALID_ARG, "aur_bvh_intersect: NULL argument");
    if (!b->corner_n)
        return fail(AUR_ERR_INVALID_ARG, "aur_bvh_intersect: no per-corner normals (aur_bvh_set_shading)");
    if (n == 0) return AUR_OK;
    DeviceGuard g(b->ctx->device);
    cudaStream_t s = b->ctx->stream;
    DevOut dr, dh;   // rays are read and written (maxt), hits written
    CUDA_TRY(dr.init(rays, sizeof(aur_ray) * n, 16, s), "aur_bvh_intersect(rays)");
    if (dr.owned)
        CUDA_TRY(cudaMemcpyAsync(dr.ptr, rays, sizeof(aur_ray) * n, cudaMemcpyDefault, s), "aur_bvh_intersect(rays)");
    CUDA_TRY(dh.init(isects, sizeof(aur_isect) * n, 16, s), "aur_bvh_intersect(isects)");
    k_intersect<<<(n + kIsectBlock - 1) / kIsectBlock, kIsectBlock, 0, s>>>(
        b->bvh.nodes, b->bvh.nodes4, b->bvh.tris, b->tri_attr, b->corner_n, b->corner_uv, (float4*)dr.ptr,
        (aur_isect*)dh.ptr, n);
    CUDA_TRY(cudaGetLastError(), "aur_bvh_intersect");
    CUDA_TRY(dr.finish(), "aur_bvh_intersect(download)");
    CUDA_TRY(dh.finish(), "aur_bvh_intersect(download)");
    CUDA_TRY(cudaStreamSynchronize(s), "aur_bvh_intersect");
    return AUR_OK;
}
