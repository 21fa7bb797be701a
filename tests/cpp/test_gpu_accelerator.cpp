// test_gpu_accelerator.cpp — drives GpuAccelerator (aurora_b200/adapters) the way the
// reference's Integrator drives its AccelerationStructure, for tests/test_gpu_accel.py.
//
// usage: test_gpu_accelerator IN OUT
// IN  (little endian): u32 nvert, ntri, nrays, nsingle, nshade, has_uvs; f32 vertices[3 nvert];
//     u32 triangles[3 ntri]; i32 id0[ntri]; f32 normals[9 ntri]; f32 uvs[6 ntri] (if has_uvs);
//     f32 rays[8 nrays] (org, mint, dir, maxt); i32 shade_ids[nshade]
// OUT: per ray the batched intersect: u8 hit, f32 maxt after, i32 attributesIndex,
//      i32 triangleIndex, f32 hitP[3], hitN[3], st[2], bar[3]  (53 bytes, packed);
//      then for the first nsingle rays the same record from the one-ray intersect;
//      then u8 occluded[nrays] from the batched intersectBinary and u8[nsingle] from the
//      one-ray form; then for each shade id 3 corners x (P[3], Ng[3], Ns[3], st[2], i32 id).
// Exit status 0 when every call succeeded.
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "gpu_accelerator.hpp"

using namespace aurora_b200;

template <class T>
static bool rd(FILE* f, T* p, size_t n) { return fread(p, sizeof(T), n, f) == n; }
template <class T>
static void wr(FILE* f, const T* p, size_t n) { fwrite(p, sizeof(T), n, f); }

static void put_isect(FILE* f, bool hit, const Ray& r, const Intersection& x) {
    const uint8_t h = hit ? 1 : 0;
    wr(f, &h, 1);
    wr(f, &r.maxt, 1);
    const int32_t a = hit ? x.attributesIndex : -1, t = hit ? x.shdGeo.triangleIndex : -1;
    wr(f, &a, 1);
    wr(f, &t, 1);
    const float zero[3] = {0.f, 0.f, 0.f};
    wr(f, hit ? &x.hitP.x : zero, 3);
    wr(f, hit ? &x.hitN.x : zero, 3);
    wr(f, hit ? x.shdGeo.st : zero, 2);
    wr(f, hit ? &x.shdGeo.barCoords.x : zero, 3);
}

int main(int argc, char** argv) {
    if (argc != 3) { fprintf(stderr, "usage: %s IN OUT\n", argv[0]); return 2; }
    FILE* in = fopen(argv[1], "rb");
    if (!in) { perror(argv[1]); return 2; }
    uint32_t hdr[6];
    if (!rd(in, hdr, 6)) return 2;
    const uint32_t nvert = hdr[0], ntri = hdr[1], nrays = hdr[2], nsingle = hdr[3], nshade = hdr[4];
    std::vector<float> verts(3 * (size_t)nvert), normals(9 * (size_t)ntri), uvs(hdr[5] ? 6 * (size_t)ntri : 0),
        rays(8 * (size_t)nrays);
    std::vector<uint32_t> tris(3 * (size_t)ntri);
    std::vector<int32_t> id0(ntri), shade(nshade);
    if (!rd(in, verts.data(), verts.size()) || !rd(in, tris.data(), tris.size()) || !rd(in, id0.data(), id0.size()) ||
        !rd(in, normals.data(), normals.size()) || (hdr[5] && !rd(in, uvs.data(), uvs.size())) ||
        !rd(in, rays.data(), rays.size()) || !rd(in, shade.data(), shade.size())) {
        fprintf(stderr, "short input\n");
        return 2;
    }
    fclose(in);
    MeshArrays m{verts.data(), nvert, tris.data(), id0.data(), ntri, normals.data(), hdr[5] ? uvs.data() : nullptr};
    try {
        GpuAccelerator acc(m);
        std::vector<Ray> rs(nrays);
        for (uint32_t i = 0; i < nrays; ++i) {
            const float* r = &rays[8 * (size_t)i];
            rs[i] = Ray{Vec3{r[0], r[1], r[2]}, Vec3{r[4], r[5], r[6]}, r[3], r[7]};
        }
        std::vector<Ray> batch = rs;
        std::vector<Intersection> isects(nrays);
        std::unique_ptr<bool[]> hit(new bool[nrays]);
        acc.intersect(batch.data(), isects.data(), hit.get(), nrays);
        if (acc.status() != AUR_OK) { fprintf(stderr, "intersect: %s\n", aur_last_error()); return 1; }
        FILE* out = fopen(argv[2], "wb");
        if (!out) { perror(argv[2]); return 2; }
        for (uint32_t i = 0; i < nrays; ++i) put_isect(out, hit[i], batch[i], isects[i]);
        for (uint32_t i = 0; i < nsingle; ++i) {
            Ray r = rs[i];
            Intersection x;
            const bool h = acc.intersect(&r, &x);
            if (acc.status() != AUR_OK) { fprintf(stderr, "intersect(1): %s\n", aur_last_error()); return 1; }
            put_isect(out, h, r, x);
        }
        std::unique_ptr<bool[]> occ(new bool[nrays]);
        acc.intersectBinary(rs.data(), occ.get(), nrays);
        if (acc.status() != AUR_OK) { fprintf(stderr, "intersectBinary: %s\n", aur_last_error()); return 1; }
        for (uint32_t i = 0; i < nrays; ++i) { const uint8_t o = occ[i] ? 1 : 0; wr(out, &o, 1); }
        for (uint32_t i = 0; i < nsingle; ++i) {
            Ray r = rs[i];
            const uint8_t o = acc.intersectBinary(&r) ? 1 : 0;
            wr(out, &o, 1);
        }
        for (uint32_t k = 0; k < nshade; ++k) {
            ShadingGeometry g[3];
            acc.getShadingTriangles(shade[k], g);
            for (int c = 0; c < 3; ++c) {
                wr(out, &g[c].P.x, 3);
                wr(out, &g[c].Ng.x, 3);
                wr(out, &g[c].Ns.x, 3);
                wr(out, g[c].st, 2);
                const int32_t id = g[c].triangleIndex;
                wr(out, &id, 1);
            }
        }
        fclose(out);
    } catch (const std::exception& ex) {
        fprintf(stderr, "%s\n", ex.what());
        return 1;
    }
    return 0;
}
