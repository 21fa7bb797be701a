// gpu_accelerator.cpp — GpuAccelerator: EmbreeAccelerator's contract
// (Aurora/src/geometry/embreeAccelerator.cpp:19-123) on the device BVH, through the C ABI.
#include "gpu_accelerator.hpp"

#include <stdexcept>
#include <string>

namespace aurora_b200 {
namespace {

aur_ray to_aur(const Ray& r) {
    aur_ray a;
    a.org[0] = r.origin.x; a.org[1] = r.origin.y; a.org[2] = r.origin.z;
    a.dir[0] = r.direction.x; a.dir[1] = r.direction.y; a.dir[2] = r.direction.z;
    a.mint = r.mint;
    a.maxt = r.maxt;
    return a;
}

// EmbreeAccelerator::intersect's fill of Intersection (embreeAccelerator.cpp:58-90)
void fill(const aur_isect& h, Intersection* out) {
    out->hitP = Vec3{h.hitP[0], h.hitP[1], h.hitP[2]};
    out->hitN = Vec3{h.hitN[0], h.hitN[1], h.hitN[2]};
    out->attributesIndex = h.attr;
    out->shdGeo.P = out->hitP;
    out->shdGeo.Ng = out->hitN;
    out->shdGeo.st[0] = h.st[0];
    out->shdGeo.st[1] = h.st[1];
    out->shdGeo.triangleIndex = h.prim;
    out->shdGeo.barCoords = Vec3{h.bar[0], h.bar[1], h.bar[2]};
}

[[noreturn]] void raise(const char* what) {
    throw std::runtime_error(std::string(what) + ": " + aur_last_error());
}

}  // namespace

GpuAccelerator::GpuAccelerator(const MeshArrays& m, int device, const aur_bvh_opts* opts) {
    if (!m.vertices || !m.triangles || !m.normals || m.numTriangles == 0)
        throw std::runtime_error("GpuAccelerator: empty mesh or missing vertices, triangles or normals");
    vertices_.assign(m.vertices, m.vertices + 3 * (size_t)m.numVertices);
    triangles_.assign(m.triangles, m.triangles + 3 * (size_t)m.numTriangles);
    normals_.assign(m.normals, m.normals + 9 * (size_t)m.numTriangles);
    if (m.uvs) uvs_.assign(m.uvs, m.uvs + 6 * (size_t)m.numTriangles);
    if (aur_ctx_create(device, &ctx_) != AUR_OK) raise("GpuAccelerator(aur_ctx_create)");
    if (aur_bvh_build(ctx_, m.vertices, m.numVertices, m.triangles, m.id0, m.numTriangles, opts, &bvh_) != AUR_OK) {
        aur_ctx_destroy(ctx_);
        raise("GpuAccelerator(aur_bvh_build)");
    }
    if (aur_bvh_set_shading(bvh_, m.normals, m.uvs) != AUR_OK) {
        aur_bvh_destroy(bvh_);
        aur_ctx_destroy(ctx_);
        raise("GpuAccelerator(aur_bvh_set_shading)");
    }
}

GpuAccelerator::~GpuAccelerator() {
    if (bvh_) aur_bvh_destroy(bvh_);
    if (ctx_) aur_ctx_destroy(ctx_);
}

void GpuAccelerator::intersect(Ray* rays, Intersection* isects, bool* hit, size_t n) const {
    if (n == 0) return;
    std::vector<aur_ray> r(n);
    std::vector<aur_isect> h(n);
    for (size_t i = 0; i < n; ++i) r[i] = to_aur(rays[i]);
    status_ = aur_bvh_intersect(bvh_, r.data(), h.data(), (uint32_t)n);
    for (size_t i = 0; i < n; ++i) {
        hit[i] = status_ == AUR_OK && h[i].prim >= 0;
        if (!hit[i]) continue;
        rays[i].maxt = r[i].maxt;                  // ray->maxt = t (embreeAccelerator.cpp:56)
        fill(h[i], &isects[i]);
    }
}

bool GpuAccelerator::intersect(Ray* ray, Intersection* isect) const {
    bool hit = false;
    intersect(ray, isect, &hit, 1);
    return hit;
}

void GpuAccelerator::intersectBinary(const Ray* rays, bool* occluded, size_t n) const {
    if (n == 0) return;
    std::vector<aur_ray> r(n);
    std::vector<uint8_t> o(n);
    for (size_t i = 0; i < n; ++i) r[i] = to_aur(rays[i]);
    status_ = aur_trace_occluded(bvh_, r.data(), o.data(), (uint32_t)n);
    for (size_t i = 0; i < n; ++i) occluded[i] = status_ == AUR_OK && o[i] != 0;
}

bool GpuAccelerator::intersectBinary(Ray* ray) const {
    bool occ = false;
    intersectBinary(ray, &occ, 1);
    return occ;
}

// EmbreeAccelerator::getShadingTriangles (embreeAccelerator.cpp:102-123): corner k's
// position, normal (as Ng and Ns) and uv, read from the mesh kept on the host.
void GpuAccelerator::getShadingTriangles(int t, ShadingGeometry* shdGeo) const {
    for (int k = 0; k < 3; ++k) {
        const float* p = &vertices_[3 * (size_t)triangles_[3 * (size_t)t + k]];
        const float* nn = &normals_[9 * (size_t)t + 3 * k];
        shdGeo[k].P = Vec3{p[0], p[1], p[2]};
        shdGeo[k].Ng = Vec3{nn[0], nn[1], nn[2]};
        shdGeo[k].Ns = shdGeo[k].Ng;
        shdGeo[k].st[0] = uvs_.empty() ? 0.f : uvs_[6 * (size_t)t + 2 * k];
        shdGeo[k].st[1] = uvs_.empty() ? 0.f : uvs_[6 * (size_t)t + 2 * k + 1];
        shdGeo[k].triangleIndex = t;
    }
}

}  // namespace aurora_b200
