// gpu_accelerator.hpp — AccelerationStructure adapter over the C ABI.
//
// The reference renderer reaches its BVH through one interface,
// Aurora::AccelerationStructure (Aurora/src/geometry/accelerationStructure.h:17-27):
// intersect(Ray*, Intersection*), intersectBinary(Ray*) and getShadingTriangles(int,
// ShadingGeometry*), implemented by EmbreeAccelerator (embreeAccelerator.cpp:19-123)
// over the flattened mesh of EmbreeMesh::preRender (embreeMesh.h:30-58).
// GpuAccelerator keeps that contract on the device BVH of libaurora_b200:
//   * intersect: closest hit in [mint, maxt]; on a hit ray->maxt = t, hitP = org +
//     dir * t, hitN = shdGeo.Ng = the face-forwarded normalised interpolation of the
//     corner normals, shdGeo.st the interpolated uvs, shdGeo.barCoords = (u, v, w),
//     attributesIndex = id0, shdGeo.triangleIndex = id1 (the triangle's position);
//   * intersectBinary: any hit in [mint, maxt];
//   * getShadingTriangles: the triangle's three corners (P, Ng = Ns, st).
// The records below mirror the reference's fields that this contract fills (core/ray.h,
// attributes/intersection.h, attributes/shadingGeometry.h); a binding inside the
// reference copies them into its own types. Batched forms take arrays of rays: one
// device launch per call, which is how a renderer should use the GPU; the one-ray forms
// exist for callers that keep the reference's per-ray loop.
// Errors: the constructor throws std::runtime_error with aur_last_error()'s message; the
// queries return false / leave outputs unset and record the status (status()).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "aurora_b200.h"

namespace aurora_b200 {

struct Vec3 { float x, y, z; };
struct Ray { Vec3 origin, direction; float mint, maxt; };               // core/ray.h:25-30
struct ShadingGeometry {                                                // attributes/shadingGeometry.h:14-31
    Vec3 P, Ns, Ng;
    float st[2];
    Vec3 barCoords;
    int triangleIndex;
};
struct Intersection {                                                   // attributes/intersection.h:16-21
    ShadingGeometry shdGeo;
    Vec3 hitN, hitP;
    int attributesIndex;
};

// The flattened mesh, as EmbreeMesh holds it after preRender: camera-space vertices,
// triangles (v0, v1, v2) with their attribute index id0 (the triangle id id1 is the
// position), per-corner normals (9 floats per triangle) and uvs (6 per triangle, or null).
struct MeshArrays {
    const float* vertices;
    uint32_t numVertices;
    const uint32_t* triangles;
    const int32_t* id0;
    uint32_t numTriangles;
    const float* normals;
    const float* uvs;
};

class GpuAccelerator {
public:
    explicit GpuAccelerator(const MeshArrays& mesh, int device = 0, const aur_bvh_opts* opts = nullptr);
    ~GpuAccelerator();
    GpuAccelerator(const GpuAccelerator&) = delete;
    GpuAccelerator& operator=(const GpuAccelerator&) = delete;

    bool intersect(Ray* ray, Intersection* isect) const;
    bool intersectBinary(Ray* ray) const;
    void getShadingTriangles(int triangleIndex, ShadingGeometry* shdGeo) const;

    // n rays at once: hit[i] / occluded[i] as the one-ray forms return them
    void intersect(Ray* rays, Intersection* isects, bool* hit, size_t n) const;
    void intersectBinary(const Ray* rays, bool* occluded, size_t n) const;

    aur_status status() const { return status_; }
    aur_bvh* bvh() const { return bvh_; }

private:
    aur_ctx* ctx_ = nullptr;
    aur_bvh* bvh_ = nullptr;
    std::vector<float> vertices_, normals_, uvs_;
    std::vector<uint32_t> triangles_;
    mutable aur_status status_ = AUR_OK;
};

}  // namespace aurora_b200
