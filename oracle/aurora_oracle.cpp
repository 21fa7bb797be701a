// aurora_oracle.cpp — CPU restatement of Aurora's per-pixel MIS path-tracing
// loop. TEST INFRASTRUCTURE ONLY: it is the checker for the sm_100a kernels and
// the timed CPU baseline ("restatement, not the reference binary"); nothing in
// the product links or calls it.
//
// Written independently of the CUDA sources, in the reference's own structure
// (Vector/Color value types, virtual-free lobes), and compiled with
// -ffp-contract=off and IEEE division so every FP32 operation rounds exactly
// as written. Each function cites the reference file:line it restates
// (paths inside espennordahl/Aurora). Deliberate deviations:
//   * rand()/RAND_MAX is replaced by the counter-based SplitMix64 draw of the
//     product (same published algorithm, restated here), one fixed slot per
//     decision, so that CPU and GPU consume identical random numbers;
//   * Embree's BVH4 is replaced by (a) a brute-force scan for hit-ID parity and
//     (b) a binned-SAH binary BVH for the timed baseline; both use the
//     RenderableTriangle Moller-Trumbore test (renderableTriangle.cpp:68-98);
//   * the film is an FP64 running sum (the reference keeps half precision);
//   * the unshaded closest-hit ray after the last vertex (integrator.cpp:255-274)
//     is traced only when its miss adds radiance (a mirror ray in a scene with an
//     environment light); its hit is never shaded, so the radiance is the same.
// The adjoint restatement (oracle_adjoint) has no reference counterpart: it is the
// FP64 forward-mode derivative of this file's own estimator.
// Parity pinning: the reference ships no tests, golden vectors or fixtures and
// cannot be built here (Embree 1.x, TBB 4.1, OpenEXR 1.7, jsoncpp absent), so
// this restatement is pinned by its line-by-line correspondence and by the
// hand-derived known answers in tests/test_oracle.py.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#include "aurora_b200.h"   // plain-C record layouts only (aur_ray, aur_scene_desc, ...)

namespace oracle {

// ------------------------------------------------------------ constants.h
static const double CAUSTIC_BLUR = 0.2;
static const float FIREFLY = 200;
static const double ISBLACK = 0.0001;
static const double RAY_BIAS = 0.0005;
static const int COS_ENTRIES = 64, ROUGH_ENTRIES = 32, REFL_ENTRIES = 21;
#define M_PI_INV 1.f / M_PI

// ------------------------------------------------------------ core/vector.h, color.h
struct Vector {
    float x, y, z;
    Vector() : x(0), y(0), z(0) {}
    Vector(float a, float b, float c) : x(a), y(b), z(c) {}
    float lengthSquared() const { return x * x + y * y + z * z; }
    float length() const {                       // vector.h:65-71
        float l = sqrtf(lengthSquared());
        if (l == 0.) return 0.0001;
        return l;
    }
    Vector operator+(const Vector& v) const { return Vector(x + v.x, y + v.y, z + v.z); }
    Vector operator-(const Vector& v) const { return Vector(x - v.x, y - v.y, z - v.z); }
    Vector operator*(float f) const { return Vector(f * x, f * y, f * z); }
    Vector operator/(float f) const { float inv = 1.f / f; return Vector(x * inv, y * inv, z * inv); }
    Vector operator-() const { return Vector(-x, -y, -z); }
};
typedef Vector Point;

struct Color {
    float r, g, b;
    Color() : r(0), g(0), b(0) {}
    explicit Color(float c) : r(c), g(c), b(c) {}
    Color(float a, float b_, float c) : r(a), g(b_), b(c) {}
    Color operator+(const Color& c) const { return Color(r + c.r, g + c.g, b + c.b); }
    Color& operator+=(const Color& c) { r += c.r; g += c.g; b += c.b; return *this; }
    Color operator*(const Color& c) const { return Color(r * c.r, g * c.g, b * c.b); }
    Color& operator*=(const Color& c) { r *= c.r; g *= c.g; b *= c.b; return *this; }
    Color operator*(float f) const { return Color(r * f, g * f, b * f); }
    Color operator*(double d) const { return Color(r * d, g * d, b * d); }   // color.h:108-110
    Color& operator*=(float f) { r *= f; g *= f; b *= f; return *this; }
    Color operator/(float f) const { float d = 1 / f; return Color(r * d, g * d, b * d); }
    Color& operator/=(float f) { float d = 1 / f; r *= d; g *= d; b *= d; return *this; }
    bool isBlack() const { return r < ISBLACK && g < ISBLACK && b < ISBLACK; }          // color.h:149-151
    float lum() const { return 0.2126 * r + 0.7152 * g + 0.0722 * b; }                  // color.h:157-159
};

// ------------------------------------------------------------ core/math_utils.h
inline float dot(const Vector& a, const Vector& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vector normalize(const Vector& v) { return v / v.length(); }
inline Vector cross(const Vector& v1, const Vector& v2) {
    return Vector((v1.y * v2.z) - (v1.z * v2.y), (v1.z * v2.x) - (v1.x * v2.z), (v1.x * v2.y) - (v1.y * v2.x));
}
inline Vector SampleHemisphereUniform(float r1, float r2) {     // math_utils.h:70-78
    float z = r1;
    float r = sqrtf(fmax(0.f, 1.f - z * z));
    float phi = 2 * M_PI * r2;
    return Vector(r * cosf(phi), r * sinf(phi), z);
}
inline void coordinateSystem(const Vector& v1, Vector* v2, Vector* v3) {     // math_utils.h:107-129
    if (!v1.x && v1.y && !v1.z) *v2 = cross(v1, Vector(1.f, 0.f, 0.f));
    else *v2 = cross(v1, Vector(0.f, 1.f, 0.f));
    *v3 = cross(v1, *v2);
}
inline Vector tangentToWorld(const Vector& dir, const Vector& Nn) {           // math_utils.h:81-90
    Vector dPdu, dPdv;
    coordinateSystem(Nn, &dPdu, &dPdv);
    Vector RayDir = normalize(dPdu) * dir.x;
    RayDir = RayDir + (normalize(dPdv) * dir.y);
    RayDir = RayDir + (Nn * dir.z);
    return RayDir;
}
inline float schlick(float VdotH, float reflectance) { return reflectance + powf(1.f - VdotH, 5.f) * (1.f - reflectance); }
inline int afloor(float x) { return (int)x - (x < 0 && (int)x != x); }       // math_utils.h:252-254
inline float clampf(float x, float lo, float hi) { float r = x < lo ? lo : x; return r > hi ? hi : r; }

// ------------------------------------------------------------ RNG (SplitMix64, counter based)
inline uint64_t splitmix_fin(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
inline uint64_t key_of(uint32_t seed) { return splitmix_fin((uint64_t)seed * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull); }
inline float draw(uint64_t key, uint64_t counter) {
    return (float)(uint32_t)(splitmix_fin(key + counter * 0x9e3779b97f4a7c15ull) >> 40) * (1.0f / 16777216.0f);
}
struct Rng {
    uint64_t key, base;
    float operator()(uint32_t dim) const { return draw(key, base | dim); }
};
enum { DIM_LOBE = 0, DIM_LIGHTPICK = 1, DIM_LIGHTSAMPLE = 2, DIM_MISBRDF = 4, DIM_BRDF = 6, DIM_ROULETTE = 8 };
inline uint32_t vdim(int vertex, int slot) { return 2u + (uint32_t)vertex * 10u + (uint32_t)slot; }

// ------------------------------------------------------------ ray / sample
struct Ray { Vector direction; Point origin; float mint, maxt; };
struct Sample3D { Ray ray; Color color; float pdf; };

// ------------------------------------------------------------ RenderableTriangle (renderableTriangle.cpp:68-98)
inline bool triIntersect(const Point& p1, const Vector& e1, const Vector& e2, const Ray& ray, float* tout,
                         float* b1out, float* b2out) {
    Vector s1 = cross(ray.direction, e2);
    float divisor = dot(s1, e1);
    if (divisor == 0.) return false;
    float invDivisor = 1.f / divisor;
    Vector d = ray.origin - p1;
    float b1 = dot(d, s1) * invDivisor;
    if (b1 < 0. || b1 > 1.) return false;
    Vector s2 = cross(d, e1);
    float b2 = dot(ray.direction, s2) * invDivisor;
    if (b2 < 0. || (b1 + b2) > 1.) return false;
    float t = dot(e2, s2) * invDivisor;
    if (t < ray.mint || t > ray.maxt) return false;
    *tout = t; *b1out = b1; *b2out = b2;
    return true;
}

// ------------------------------------------------------------ scene as seen by the oracle
struct Tri { Point p1; Vector e1, e2; };
struct Mat {
    int type; Color diff, spec, gain; float rough, roughB, refl, mix;
    int diffTex, specTex, roughTex; int table; float ior;
    int normTex; Color normC;   // normal-map shader: texture, -1 none, -2 the constant colour normC
};
struct Light {
    int type; float xScale, yScale, radius; Point pCam[4]; Vector lightN; Color le; Point center; float m[16];
    Point tri[2][3];
    // environment light (InfiniteAreaLight): m = camera-to-world, minv = world-to-camera,
    // env map texture (or -1), 2^exposure, mean texel luminance
    float minv[16]; int tex; float escale; float pdfNorm;
};
// a texture shader: uv lookup (triScale 0) or triplanar projection with scale triScale
struct Tex { int w, h; const float* px; size_t offset; float triScale; };   // offset: first float in the texel array

struct BvhNode { float lo[3], hi[3]; int left, right, start, count; };   // leaf if count > 0

struct Scene {
    std::vector<Tri> tris;
    std::vector<int> triAttr;
    std::vector<float> cornerN, cornerUV;
    std::vector<int> attrMat;
    std::vector<Color> attrEmission;
    std::vector<Mat> mats;
    std::vector<Light> lights;
    std::vector<Tex> texs;
    std::vector<float> texels;
    std::vector<float> attrC2O;             // AttributeState::cameraToObject, 16 floats per attribute
    const float* albedo = nullptr;          // [table][64][32]
    float fov; int width, height;
    // CPU BVH (binned SAH) used by the timed baseline; brute force when empty
    std::vector<BvhNode> nodes;
    std::vector<int> order;
    bool hasEnv = false;                    // an InfiniteAreaLight is among the lights
};

// Whether the ray after vertex trueBounces - 1 is traced: always below maxDepth; the one
// after the last vertex only when an escaping mirror ray would see the environment
// (integrator.cpp:255-274 traces it always, shades no hit, and adds the environment for
// a mirror ray that misses).
static bool traceNext(const Scene& sc, int trueBounces, int maxDepth, int rayType) {
    return trueBounces < maxDepth || (rayType == 3 /* MirrorRay */ && sc.hasEnv);
}

// ------------------------------------------------------------ CPU BVH (baseline stand-in for Embree)
struct BuildPrim { float lo[3], hi[3], c[3]; };

static void boxOf(const Tri& t, float lo[3], float hi[3]) {
    Point p2 = t.p1 + t.e1, p3 = t.p1 + t.e2;   // only for bounds: the test uses (p1, e1, e2)
    const float* a = &t.p1.x; const float* b = &p2.x; const float* c = &p3.x;
    for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(std::min(a[k], b[k]), c[k]);
        hi[k] = std::max(std::max(a[k], b[k]), c[k]);
        float m = std::max(std::max(fabsf(lo[k]), fabsf(hi[k])), hi[k] - lo[k]);
        lo[k] -= m * 4e-6f + 1e-30f;   // p1+e1 is not exactly p2: pad the box
        hi[k] += m * 4e-6f + 1e-30f;
    }
}

static float halfArea(const float lo[3], const float hi[3]) {
    float d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
    return d0 * d1 + d1 * d2 + d2 * d0;
}

static int buildRec(Scene& sc, std::vector<BuildPrim>& bp, int begin, int end, int maxLeaf) {
    BvhNode node;
    for (int k = 0; k < 3; ++k) { node.lo[k] = FLT_MAX; node.hi[k] = -FLT_MAX; }
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = begin; i < end; ++i) {
        const BuildPrim& p = bp[sc.order[i]];
        for (int k = 0; k < 3; ++k) {
            node.lo[k] = std::min(node.lo[k], p.lo[k]); node.hi[k] = std::max(node.hi[k], p.hi[k]);
            clo[k] = std::min(clo[k], p.c[k]); chi[k] = std::max(chi[k], p.c[k]);
        }
    }
    const int idx = (int)sc.nodes.size();
    sc.nodes.push_back(node);
    const int n = end - begin;
    int bestAxis = -1, bestSplit = -1;
    float bestCost = FLT_MAX;
    const int NB = 16;
    if (n > maxLeaf) {
        for (int axis = 0; axis < 3; ++axis) {
            const float ext = chi[axis] - clo[axis];
            if (ext <= 0.f) continue;
            float blo[NB][3], bhi[NB][3]; int bc[NB] = {0};
            for (int b = 0; b < NB; ++b) for (int k = 0; k < 3; ++k) { blo[b][k] = FLT_MAX; bhi[b][k] = -FLT_MAX; }
            for (int i = begin; i < end; ++i) {
                const BuildPrim& p = bp[sc.order[i]];
                int b = std::min(NB - 1, (int)((p.c[axis] - clo[axis]) / ext * NB));
                ++bc[b];
                for (int k = 0; k < 3; ++k) { blo[b][k] = std::min(blo[b][k], p.lo[k]); bhi[b][k] = std::max(bhi[b][k], p.hi[k]); }
            }
            float rA[NB]; int rC[NB];
            float alo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ahi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX}; int ac = 0;
            for (int b = NB - 1; b > 0; --b) {
                for (int k = 0; k < 3; ++k) { alo[k] = std::min(alo[k], blo[b][k]); ahi[k] = std::max(ahi[k], bhi[b][k]); }
                ac += bc[b]; rA[b] = ac ? halfArea(alo, ahi) : 0.f; rC[b] = ac;
            }
            for (int k = 0; k < 3; ++k) { alo[k] = FLT_MAX; ahi[k] = -FLT_MAX; }
            ac = 0;
            for (int b = 0; b < NB - 1; ++b) {
                for (int k = 0; k < 3; ++k) { alo[k] = std::min(alo[k], blo[b][k]); ahi[k] = std::max(ahi[k], bhi[b][k]); }
                ac += bc[b];
                if (ac == 0 || rC[b + 1] == 0) continue;
                float cost = halfArea(alo, ahi) * ac + rA[b + 1] * rC[b + 1];
                if (cost < bestCost) { bestCost = cost; bestAxis = axis; bestSplit = b; }
            }
        }
    }
    const float leafCost = halfArea(node.lo, node.hi) * n;
    if (n <= maxLeaf || bestAxis < 0 || (n <= 16 && bestCost + halfArea(node.lo, node.hi) >= leafCost)) {
        if (n > 31 && bestAxis < 0) {   // identical centroids: split in the middle of the list
            const int mid = begin + n / 2;
            int l = buildRec(sc, bp, begin, mid, maxLeaf);
            int r = buildRec(sc, bp, mid, end, maxLeaf);
            sc.nodes[idx].left = l; sc.nodes[idx].right = r; sc.nodes[idx].start = 0; sc.nodes[idx].count = 0;
            return idx;
        }
        sc.nodes[idx].left = sc.nodes[idx].right = -1;
        sc.nodes[idx].start = begin; sc.nodes[idx].count = n;
        return idx;
    }
    const float ext = chi[bestAxis] - clo[bestAxis];
    int* mid = std::partition(sc.order.data() + begin, sc.order.data() + end, [&](int pi) {
        int b = std::min(NB - 1, (int)((bp[pi].c[bestAxis] - clo[bestAxis]) / ext * NB));
        return b <= bestSplit;
    });
    int m = (int)(mid - sc.order.data());
    if (m == begin || m == end) m = begin + n / 2;
    int l = buildRec(sc, bp, begin, m, maxLeaf);
    int r = buildRec(sc, bp, m, end, maxLeaf);
    sc.nodes[idx].left = l; sc.nodes[idx].right = r; sc.nodes[idx].start = 0; sc.nodes[idx].count = 0;
    return idx;
}

static void buildBvh(Scene& sc, int maxLeaf) {
    const int n = (int)sc.tris.size();
    std::vector<BuildPrim> bp(n);
    for (int i = 0; i < n; ++i) {
        boxOf(sc.tris[i], bp[i].lo, bp[i].hi);
        for (int k = 0; k < 3; ++k) bp[i].c[k] = 0.5f * (bp[i].lo[k] + bp[i].hi[k]);
    }
    sc.order.resize(n);
    for (int i = 0; i < n; ++i) sc.order[i] = i;
    sc.nodes.clear();
    sc.nodes.reserve(2 * n);
    buildRec(sc, bp, 0, n, maxLeaf);
}

static inline bool boxHit(const BvhNode& nd, const Ray& r, const float inv[3], float tmax, float* tnear) {
    float t0 = r.mint * 0.99999f, t1 = tmax * 1.00001f;
    const float o[3] = {r.origin.x, r.origin.y, r.origin.z};
    for (int k = 0; k < 3; ++k) {
        float a = (nd.lo[k] - o[k]) * inv[k], b = (nd.hi[k] - o[k]) * inv[k];
        if (a > b) std::swap(a, b);
        if (a != a) a = -FLT_MAX;
        if (b != b) b = FLT_MAX;
        t0 = a > t0 ? a : t0;
        t1 = b < t1 ? b : t1;
    }
    *tnear = t0;
    return t0 <= t1;
}

// closest hit (prim, t, b1, b2) in [mint, maxt]; ties resolved toward the later test
static bool sceneIntersect(const Scene& sc, const Ray& r, int* prim, float* t, float* u, float* v) {
    Ray ray = r;
    bool hit = false;
    if (sc.nodes.empty()) {
        for (size_t i = 0; i < sc.tris.size(); ++i) {
            float tt, b1, b2;
            if (triIntersect(sc.tris[i].p1, sc.tris[i].e1, sc.tris[i].e2, ray, &tt, &b1, &b2)) {
                ray.maxt = tt; *prim = (int)i; *t = tt; *u = b1; *v = b2; hit = true;
            }
        }
        return hit;
    }
    float inv[3];
    const float d[3] = {r.direction.x, r.direction.y, r.direction.z};
    for (int k = 0; k < 3; ++k) inv[k] = 1.f / (fabsf(d[k]) > 1e-20f ? d[k] : copysignf(1e-20f, d[k]));
    int stack[128]; int sp = 0; stack[sp++] = 0;
    while (sp) {
        const BvhNode& nd = sc.nodes[stack[--sp]];
        float tn;
        if (!boxHit(nd, ray, inv, ray.maxt, &tn)) continue;
        if (nd.count > 0) {
            for (int i = nd.start; i < nd.start + nd.count; ++i) {
                const int p = sc.order[i];
                float tt, b1, b2;
                if (triIntersect(sc.tris[p].p1, sc.tris[p].e1, sc.tris[p].e2, ray, &tt, &b1, &b2)) {
                    ray.maxt = tt; *prim = p; *t = tt; *u = b1; *v = b2; hit = true;
                }
            }
        } else {
            float tl, tr;
            bool hl = boxHit(sc.nodes[nd.left], ray, inv, ray.maxt, &tl);
            bool hr = boxHit(sc.nodes[nd.right], ray, inv, ray.maxt, &tr);
            if (hl && hr) {
                if (tl <= tr) { stack[sp++] = nd.right; stack[sp++] = nd.left; }
                else { stack[sp++] = nd.left; stack[sp++] = nd.right; }
            } else if (hl) stack[sp++] = nd.left;
            else if (hr) stack[sp++] = nd.right;
        }
    }
    return hit;
}

static bool sceneOccluded(const Scene& sc, const Ray& ray) {
    if (sc.nodes.empty()) {
        for (size_t i = 0; i < sc.tris.size(); ++i) {
            float tt, b1, b2;
            if (triIntersect(sc.tris[i].p1, sc.tris[i].e1, sc.tris[i].e2, ray, &tt, &b1, &b2)) return true;
        }
        return false;
    }
    float inv[3];
    const float d[3] = {ray.direction.x, ray.direction.y, ray.direction.z};
    for (int k = 0; k < 3; ++k) inv[k] = 1.f / (fabsf(d[k]) > 1e-20f ? d[k] : copysignf(1e-20f, d[k]));
    int stack[128]; int sp = 0; stack[sp++] = 0;
    while (sp) {
        const BvhNode& nd = sc.nodes[stack[--sp]];
        float tn;
        if (!boxHit(nd, ray, inv, ray.maxt, &tn)) continue;
        if (nd.count > 0) {
            for (int i = nd.start; i < nd.start + nd.count; ++i) {
                const int p = sc.order[i];
                float tt, b1, b2;
                if (triIntersect(sc.tris[p].p1, sc.tris[p].e1, sc.tris[p].e2, ray, &tt, &b1, &b2)) return true;
            }
        } else { stack[sp++] = nd.left; stack[sp++] = nd.right; }
    }
    return false;
}

// ------------------------------------------------------------ camera (camera.cpp:34-62)
static Ray convertSample(const Scene& sc, int x, int y, float j1, float j2) {
    float fovx = sc.fov;
    float fovy = ((float)sc.height / (float)sc.width) * fovx;
    float u = x + j1, v = y + j2;
    Ray r;
    r.direction.x = ((2 * u - sc.width) / (float)sc.width) * fovx;
    r.direction.y = ((-2 * v + sc.height) / (float)sc.height) * fovy;
    r.direction.z = -1.f;
    r.direction = normalize(r.direction);
    r.origin = Point(0, 0, 0);
    r.mint = 0.1f;
    r.maxt = 10000000.f;
    return r;
}

// ------------------------------------------------------------ BRDFs
// MirrorBrdf: SpecMirror; TransmitBrdf: SpecTransmit (the reference's type for both is MirrorBrdf)
enum { MatteBrdf = 0, SpecBrdf = 1, MirrorBrdf = 2, ConstantBrdf = 3, TransmitBrdf = 4 };
struct BrdfState { int type; Color color; float roughness; };   // TransmitBrdf: roughness holds the ior
inline bool isMirrorType(int t) { return t == MirrorBrdf || t == TransmitBrdf; }

static Sample3D lambertGetSample(const BrdfState& b, const Vector& Vn, const Vector& Nn, float r1, float r2) {   // lambert.h:44-62
    Vector dir = SampleHemisphereUniform(r1, r2);
    Sample3D s;
    s.ray.direction = normalize(tangentToWorld(dir, Nn));
    s.ray.origin = Point(0, 0, 0); s.ray.mint = RAY_BIAS; s.ray.maxt = 1000000.f;
    s.pdf = M_PI_INV * 0.5;
    s.color = b.color * M_PI_INV;
    return s;
}
static Color lambertEval(const BrdfState& b, const Vector& Ln, const Vector& Nn) {          // lambert.h:68-76
    float d = dot(Ln, Nn);
    if (d > 0.) return b.color * M_PI_INV;
    return Color(0);
}

static float ctD(float roughness, float cosalpha, float tanalpha) {                        // cookTorrance.cpp:40-45
    const float rough2 = std::max(0.001f, roughness * roughness);
    const float e = expf(-(tanalpha * tanalpha) / rough2);
    const float divisor = rough2 * M_PI * powf(cosalpha, 3.f);
    return e / divisor;
}
static Sample3D ctGetSample(const BrdfState& b, const Vector& Vn, const Vector& Nn, float r1, float r2) {  // cookTorrance.cpp:47-99
    float z = cosf(atanf(b.roughness * sqrtf(-log(1. - r1))));
    float r = sqrtf(fmax(0.f, 1.f - z * z));
    float phi = M_PI * 2 * r2;
    float x = r * cosf(phi);
    float y = r * sinf(phi);
    Vector dir = normalize(Vector(x, y, z));
    Vector Hn = normalize(tangentToWorld(dir, Nn));
    float vdoth = dot(Vn, Hn);
    Vector Ln = normalize(Vector((Hn * 2 * vdoth) - Vn));
    float ndoth = dot(Nn, Hn);
    Color result(0.f);
    float pdf = 1.f;
    if (vdoth > 0.0001) {
        const float tanalpha = (ndoth > 0.999) ? 0. : tanf(acosf(ndoth));
        float D = ctD(b.roughness, ndoth, tanalpha);
        D = std::min(D, 1000.f);
        pdf = D / (4 * vdoth);
        result = b.color * D / (4 * vdoth * vdoth);
        if (pdf > 100000) { pdf *= 0.01f; result *= 0.01f; }
    }
    Sample3D s;
    s.ray.direction = Ln; s.ray.origin = Point(0, 0, 0); s.ray.mint = RAY_BIAS; s.ray.maxt = 10000000.f;
    s.pdf = pdf; s.color = result;
    return s;
}
static float ctPdf(const BrdfState& b, const Vector& Ln, const Vector& Vn, const Vector& Nn) {   // cookTorrance.cpp:101-117
    Vector Hn = normalize(Ln + Vn);
    float vdoth = dot(Vn, Hn);
    float ndoth = dot(Nn, Hn);
    float D = ctD(b.roughness, ndoth, tanf(acosf(ndoth)));
    if (std::isnan(D)) D = 0.f;
    return D / (4 * vdoth);
}
static Color ctEval(const BrdfState& b, const Vector& Ln, const Vector& Vn, const Vector& Nn) {   // cookTorrance.cpp:125-144
    Vector Hn = normalize(Ln + Vn);
    const float vdoth = dot(Vn, Hn);
    const float vdotn = dot(Vn, Nn);
    const float ndoth = dot(Hn, Nn);
    const float ldotn = dot(Ln, Nn);
    const float roughnessSquared = b.roughness * b.roughness;
    const float D = (1.f / (roughnessSquared * M_PI * powf(ndoth, 3.f))) *
                    expf(-(tanf(acosf(ndoth)) * tanf(acosf(ndoth))) / roughnessSquared);
    if (vdoth <= 0.001 || ldotn <= 0.001 || vdotn <= 0.001 || std::isnan(D)) return Color(0.f);
    return b.color * D / (4. * vdoth * vdoth);
}

static Vector worldToTangent(const Vector& dir, const Vector& Nn) {            // math_utils.h:92-97
    Vector dPdu, dPdv;
    coordinateSystem(Nn, &dPdu, &dPdv);
    return Vector(dot(dir, dPdu), dot(dir, dPdv), dot(dir, Nn));
}
static Sample3D mirrorGetSample(const BrdfState& b, const Vector& Vn, const Vector& Nn) {   // specMirror.cpp:35-40
    Vector Vt = worldToTangent(Vn, Nn);
    Vector R = Vector(-Vt.x, -Vt.y, Vt.z);
    R = tangentToWorld(R, Nn);
    Sample3D s;
    s.ray.direction = normalize(R); s.ray.origin = Point(0, 0, 0); s.ray.mint = RAY_BIAS; s.ray.maxt = 100000000.f;
    s.pdf = 1.f; s.color = b.color;
    return s;
}
static Sample3D transmitGetSample(const BrdfState& b, const Vector& Vn, const Vector& Nn) { // specTransmit.cpp:33-56
    const float ior = b.roughness;
    float costheta = dot(Nn, Vn);
    float ei = 1, et = ior;
    if (costheta < 0.) { ei = ior; et = 1.; }
    float sini2 = std::max(0.f, 1 - costheta * costheta);
    float eta = ei / et;
    float sint2 = eta * eta * sini2;
    Sample3D s;
    if (sint2 >= 1.) {
        s.ray.direction = Vector(0, 0, 0); s.ray.origin = Point(); s.ray.mint = 0; s.ray.maxt = 0;
        s.pdf = 0.f; s.color = Color(0.f);
        return s;
    }
    float cost = sqrtf(std::max(0.f, 1 - sint2));
    if (costheta > 0.) cost = -cost;
    float sintOverSini = eta;
    Vector Vl = worldToTangent(Vn, Nn);
    Vector T = Vector(sintOverSini * -Vl.x, sintOverSini * -Vl.y, cost);
    T = tangentToWorld(T, Nn);
    s.ray.direction = normalize(T); s.ray.origin = Point(0, 0, 0); s.ray.mint = RAY_BIAS; s.ray.maxt = 10000000.f;
    s.pdf = 1.f; s.color = b.color;
    return s;
}

static Sample3D brdfGetSample(const BrdfState& b, const Vector& V, const Vector& N, float r1, float r2) {
    if (b.type == MatteBrdf) return lambertGetSample(b, V, N, r1, r2);
    if (b.type == SpecBrdf) return ctGetSample(b, V, N, r1, r2);
    if (b.type == MirrorBrdf) return mirrorGetSample(b, V, N);
    if (b.type == TransmitBrdf) return transmitGetSample(b, V, N);
    Sample3D s;                                   // Constant::getSample returns Sample3D() (constant.cpp:23-25)
    s.ray.direction = Vector(0, 1, 0); s.ray.origin = Point(); s.ray.mint = 0; s.ray.maxt = 0;
    s.pdf = 0; s.color = Color(0.f);
    return s;
}
static Color brdfEval(const BrdfState& b, const Vector& L, const Vector& V, const Vector& N) {
    if (b.type == MatteBrdf) return lambertEval(b, L, N);
    if (b.type == SpecBrdf) return ctEval(b, L, V, N);
    return Color(0.f);
}
static float brdfPdf(const BrdfState& b, const Vector& L, const Vector& V, const Vector& N) {
    if (b.type == MatteBrdf) return M_PI_INV * 0.5;   // lambert.h:78-80
    if (b.type == SpecBrdf) return ctPdf(b, L, V, N);
    return 0.f;
}

// ShadingGeometry + Integrator::LocalGeometry at a hit: Ng the interpolated face-forwarded
// normal, Nn the shading normal (normal map, back-facing fix)
struct LocalGeometry { Point P; Vector Vn, Nn, Ng; float su, sv; int attr; };

// ------------------------------------------------------------ textures (texture2DShader.h:28-31, texture2D.cpp:48-72)
static int texelOf(const Tex& t, float u, float v) {     // nearest texel (filter 0)
    float s = u - afloor(u);
    float tt = 1.f - (v - afloor(v));
    int x = afloor(s * t.w);
    int y = afloor(tt * t.h);
    if (y == t.h) y -= 1;
    if (x == t.w) x -= 1;
    x = std::max(0, std::min(x, t.w - 1));
    y = std::max(0, std::min(y, t.h - 1));
    return y * t.w + x;
}
static int texelAt(const Tex& t, float s, float tt) {    // Texture2D::read / ::pdf, filter 0
    int x = (int)floorf(s * t.w);
    int y = (int)floorf(tt * t.h);
    if (y == t.h) y -= 1;
    if (x == t.w) x -= 1;
    x = std::max(0, std::min(x, t.w - 1));
    y = std::max(0, std::min(y, t.h - 1));
    return y * t.w + x;
}

// TriplanarTextureShader<Color>::evaluate (triplanarTextureShader.h:29-51) and <float>
// (:71-93), as texel taps: axis i reads texel idx[i] with weight w[i] (w[i] = 0: skipped).
struct TriTaps { int idx[3]; float w[3]; };
static TriTaps triplanarTaps(const Scene& sc, const Tex& t, const LocalGeometry& lg, bool floatShader) {
    const float* m = &sc.attrC2O[16 * (size_t)lg.attr];
    float weights[3];
    float weightsum = 0.f;
    if (floatShader) {
        const float ng[3] = {lg.Ng.x, lg.Ng.y, lg.Ng.z};
        for (int i = 0; i < 3; ++i) {
            weights[i] = fabsf(ng[i]);
            weights[i] -= 0.2;
            weights[i] = std::max(weights[i], 0.f);
            weightsum += weights[i];
        }
    } else {
        Vector N = normalize(Vector(m[0] * lg.Ng.x + m[1] * lg.Ng.y + m[2] * lg.Ng.z,
                                    m[4] * lg.Ng.x + m[5] * lg.Ng.y + m[6] * lg.Ng.z,
                                    m[8] * lg.Ng.x + m[9] * lg.Ng.y + m[10] * lg.Ng.z));
        const float n[3] = {N.x, N.y, N.z};
        for (int i = 0; i < 3; ++i) {
            weights[i] = fabsf(n[i]);
            weights[i] -= 0.25;
            weights[i] = std::max(weights[i], 0.f);
            weightsum += weights[i];
        }
    }
    for (int i = 0; i < 3; ++i) weights[i] /= weightsum;
    float xp = m[0] * lg.P.x + m[1] * lg.P.y + m[2] * lg.P.z + m[3];
    float yp = m[4] * lg.P.x + m[5] * lg.P.y + m[6] * lg.P.z + m[7];
    float zp = m[8] * lg.P.x + m[9] * lg.P.y + m[10] * lg.P.z + m[11];
    float wp = m[12] * lg.P.x + m[13] * lg.P.y + m[14] * lg.P.z + m[15];
    if (wp != 1.f) { float iw = 1.f / wp; xp *= iw; yp *= iw; zp *= iw; }
    float inv = 1.f / t.triScale;                      // P /= m_scale
    const float P[3] = {xp * inv, yp * inv, zp * inv};
    TriTaps r;
    for (int i = 0; i < 3; ++i) {
        r.idx[i] = 0;
        r.w[i] = 0.f;
        if (weights[i] > 0) {
            float s = fabsf(fmodf(P[(i + 1) % 3], 1.f));
            float tt = fabsf(fmodf(P[(i + 2) % 3], 1.f));
            r.idx[i] = texelAt(t, s, tt);
            r.w[i] = weights[i];
        }
    }
    return r;
}
// Shader<Color>::evaluate of a texture shader
static Color shaderColor(const Scene& sc, int tex, const LocalGeometry& lg) {
    const Tex& t = sc.texs[tex];
    if (t.triScale == 0.f) {
        const float* p = t.px + 3 * texelOf(t, lg.su, lg.sv);
        return Color(p[0], p[1], p[2]);
    }
    const TriTaps k = triplanarTaps(sc, t, lg, false);
    Color result(0.f);
    for (int i = 0; i < 3; ++i)
        if (k.w[i] > 0) {
            const float* p = t.px + 3 * k.idx[i];
            result += Color(p[0], p[1], p[2]) * k.w[i];
        }
    return result;
}
// Shader<float>::evaluate: the red channel
static float shaderFloat(const Scene& sc, int tex, const LocalGeometry& lg) {
    const Tex& t = sc.texs[tex];
    if (t.triScale == 0.f) return t.px[3 * texelOf(t, lg.su, lg.sv)];
    const TriTaps k = triplanarTaps(sc, t, lg, true);
    float result = 0.f;
    for (int i = 0; i < 3; ++i)
        if (k.w[i] > 0) result += t.px[3 * k.idx[i]] * k.w[i];
    return result;
}

// ------------------------------------------------------------ KelemenMaterial::getAlbedo (kelemenMaterial.cpp:180-212)
static float getAlbedo(const float* table, float costheta, float roughness) {
    int i = afloor(costheta * (COS_ENTRIES - 1));
    int roughnessA = afloor(roughness * (ROUGH_ENTRIES - 1));
    int roughnessB = std::max(roughnessA + 1, ROUGH_ENTRIES - 1);
    i = std::max(0, std::min(i, COS_ENTRIES - 1));
    roughnessA = std::max(0, std::min(roughnessA, ROUGH_ENTRIES - 1));
    roughnessB = std::min(roughnessB, ROUGH_ENTRIES - 1);   // the reference reads past the table at roughness 1
    auto T = [&](int c, int r) { return table[c * ROUGH_ENTRIES + r]; };
    float valueA = T(i, roughnessA);
    float valueB = T(std::min(i + 1, COS_ENTRIES - 1), roughnessA);
    float mix = costheta * (COS_ENTRIES - 1) - i;
    float resultRoughnessA = (1. - mix) * valueA + mix * valueB;
    valueA = T(i, roughnessB);
    valueB = T(std::min(i + 1, COS_ENTRIES - 1), roughnessB);
    float resultRoughnessB = (1. - mix) * valueA + mix * valueB;
    float roughnessMix = roughness * (ROUGH_ENTRIES - 1) - roughnessA;
    return (1. - roughnessMix) * resultRoughnessA + roughnessMix * resultRoughnessB;
}

// Material::getBrdf (matteMaterial.cpp:30-35, kelemenMaterial.cpp:214-255, metalMaterial.cpp:32-62,
// constantMaterial.cpp:19-24)
static BrdfState getBrdf(const Scene& sc, int matId, const LocalGeometry& lg, bool mattePath, float lobeU) {
    const Vector& Vn = lg.Vn;
    const Vector& Nn = lg.Nn;
    const Mat& m = sc.mats[matId];
    BrdfState b;
    if (m.type == AUR_MAT_MATTE) {
        b.type = MatteBrdf; b.color = m.diffTex >= 0 ? shaderColor(sc, m.diffTex, lg) : m.diff; b.roughness = 0;
        return b;
    }
    if (m.type == AUR_MAT_KELEMEN || m.type == AUR_MAT_COOKTORRANCE) {
        float rough = m.roughTex >= 0 ? shaderFloat(sc, m.roughTex, lg) : m.rough;
        if (mattePath) rough = rough * (1. - CAUSTIC_BLUR) + CAUSTIC_BLUR;
        b.type = SpecBrdf; b.color = m.specTex >= 0 ? shaderColor(sc, m.specTex, lg) : m.spec; b.roughness = rough;
        if (m.type == AUR_MAT_KELEMEN && m.refl < 1.f) {
            float albedo = getAlbedo(sc.albedo + (size_t)m.table * COS_ENTRIES * ROUGH_ENTRIES,
                                     clampf(dot(Nn, Vn), 0., 1.), rough);
            if (lobeU > albedo) {
                b.type = MatteBrdf; b.color = m.diffTex >= 0 ? shaderColor(sc, m.diffTex, lg) : m.diff; b.roughness = 0;
            }
        }
        return b;
    }
    if (m.type == AUR_MAT_METAL) {
        float costheta = dot(Vn, Nn);
        Color sc_(schlick(costheta, m.spec.r), schlick(costheta, m.spec.g), schlick(costheta, m.spec.b));
        float rough = lobeU > m.mix ? m.rough : m.roughB;
        if (mattePath) rough = rough * (1. - CAUSTIC_BLUR) + CAUSTIC_BLUR;
        b.type = SpecBrdf; b.color = sc_ * m.gain; b.roughness = rough;
        return b;
    }
    if (m.type == AUR_MAT_GLASS) {                                   // glassMaterial.cpp:33-56
        b.type = MirrorBrdf; b.color = m.spec; b.roughness = 0;
        if (m.refl == 1.f) return b;
        float costheta = dot(Vn, Nn) * 0.5;
        if (costheta < 0.f) costheta = -costheta;
        float albedo = schlick(costheta, m.refl);
        if (lobeU > albedo) { b.type = TransmitBrdf; b.color = m.diff; b.roughness = m.ior; }
        return b;
    }
    b.type = ConstantBrdf; b.color = Color(0.f); b.roughness = 0;
    return b;
}

// ------------------------------------------------------------ lights (squareLight.h:57-122) + sphere extension
// Matrix4x4::inverse (core/matrix4x4.cpp:77-150): Gauss-Jordan with full pivoting, FP32
static bool invert4(const float* in, float* out) {
    int indxc[4], indxr[4];
    int ipiv[4] = {0, 0, 0, 0};
    float minv[4][4];
    memcpy(minv, in, 16 * sizeof(float));
    for (int i = 0; i < 4; i++) {
        int irow = -1, icol = -1;
        float big = 0.;
        for (int j = 0; j < 4; j++) {
            if (ipiv[j] != 1) {
                for (int k = 0; k < 4; k++) {
                    if (ipiv[k] == 0) {
                        if (fabsf(minv[j][k]) >= big) { big = float(fabsf(minv[j][k])); irow = j; icol = k; }
                    } else if (ipiv[k] > 1) {
                        return false;
                    }
                }
            }
        }
        if (icol < 0) return false;
        ++ipiv[icol];
        if (irow != icol) for (int k = 0; k < 4; ++k) std::swap(minv[irow][k], minv[icol][k]);
        indxr[i] = irow;
        indxc[i] = icol;
        if (minv[icol][icol] == 0.) return false;
        float pivinv = 1.f / minv[icol][icol];
        minv[icol][icol] = 1.f;
        for (int j = 0; j < 4; j++) minv[icol][j] *= pivinv;
        for (int j = 0; j < 4; j++) {
            if (j != icol) {
                float save = minv[j][icol];
                minv[j][icol] = 0;
                for (int k = 0; k < 4; k++) minv[j][k] -= minv[icol][k] * save;
            }
        }
    }
    for (int j = 3; j >= 0; j--) {
        if (indxr[j] != indxc[j]) {
            for (int k = 0; k < 4; k++) std::swap(minv[k][indxr[j]], minv[k][indxc[j]]);
        }
    }
    memcpy(out, minv, 16 * sizeof(float));
    return true;
}

static Point xformPoint(const float* m, const Point& p) {     // transform.cpp:196-204
    float xp = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
    float yp = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
    float zp = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
    float wp = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
    if (wp == 1.f) return Point(xp, yp, zp);
    return Point(xp, yp, zp) / wp;
}
// ---- environment light (geometry/infiniteAreaLight.cpp:35-106, frontend/texture2D.cpp)
static Vector xformVector(const float* m, const Vector& v) {      // transform.cpp:222-228
    return Vector(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z,
                  m[8] * v.x + m[9] * v.y + m[10] * v.z);
}
static Color envRead(const Scene& sc, const Light& l, float s, float tt) {
    const Tex& t = sc.texs[l.tex];
    const float* p = t.px + 3 * texelAt(t, s, tt);
    return Color(p[0], p[1], p[2]);
}
static float envMapPdf(const Scene& sc, const Light& l, float s, float tt) {   // p.a / m_pdf_normalization
    Color c = envRead(sc, l, s, tt);
    return ((c.r + c.g + c.b) / 3.f) / l.pdfNorm;
}
static void envUV(const Light& l, const Vector& camDir, float* u, float* v) {
    Vector dir = xformVector(l.m, camDir);
    *v = 0.5 * (1.f - dir.y);
    float uu = atan2f(dir.z, dir.x) / (M_PI * 2.f);
    if (uu < 0.f) uu += 1.f;
    *u = uu;
}
static Color lightEval(const Scene& sc, const Light& l, const Vector& dir) {    // Light::eval
    if (l.type != AUR_LIGHT_ENV || l.tex < 0) return l.le;
    float u, v;
    envUV(l, dir, &u, &v);
    return envRead(sc, l, u, v) * l.escale;
}

static bool lightVisible(const Light& l, const Point& P, const Vector& Nn) {
    if (l.type == AUR_LIGHT_ENV) return true;
    if (l.type == AUR_LIGHT_SQUARE) {
        for (int i = 0; i < 4; ++i) if (dot(l.pCam[i] - P, Nn) > 0.f) return true;
        return false;
    }
    return dot(l.center - P, Nn) > -l.radius;
}
static float sphereConeCos(const Light& l, const Point& P) {
    Vector wc = l.center - P;
    float s2 = l.radius * l.radius / dot(wc, wc);
    return sqrtf(std::max(0.f, 1.f - s2));
}
static bool sphereHit(const Light& l, const Point& o, const Vector& d, float mint, float* t) {
    Vector oc = o - l.center;
    float b = dot(oc, d);
    float c = dot(oc, oc) - l.radius * l.radius;
    float disc = b * b - c;
    if (disc < 0.f) { *t = -b; return false; }
    float sq = sqrtf(disc);
    float tt = -b - sq;
    if (tt < mint) tt = -b + sq;
    *t = tt;
    return tt >= mint;
}
static Sample3D lightGenerateSample(const Scene& sc, const Light& l, const Point& orig, const Vector& Nn, float x,
                                    float y) {
    Sample3D s;
    if (l.type == AUR_LIGHT_ENV) {                                  // InfiniteAreaLight::generateSample
        Vector dirW;
        float pdf = 1.f;
        if (l.tex >= 0) {
            float vy = 1.f - 2.f * y;
            float r = sqrtf(std::max(0.f, 1.f - vy * vy));
            float phi = 2.f * M_PI * x;
            float vx = r * cosf(phi);
            float vz = r * sinf(phi);
            dirW = xformVector(l.minv, Vector(vx, vy, vz));
            pdf = envMapPdf(sc, l, x, y);
        } else {
            pdf = 2.f;
            Vector dirT = SampleHemisphereUniform(x, y);
            dirW = tangentToWorld(dirT, Nn);
        }
        s.ray.direction = normalize(dirW); s.ray.origin = orig; s.ray.mint = RAY_BIAS; s.ray.maxt = 1000000.f;
        s.pdf = pdf / (M_PI * 4.);
        s.color = lightEval(sc, l, s.ray.direction);
        return s;
    }
    if (l.type == AUR_LIGHT_SQUARE) {
        Point lightP((x - 0.5) * l.xScale * 2, (y - 0.5) * l.yScale * 2, 0.f);
        lightP = xformPoint(l.m, lightP);
        Vector dir = lightP - orig;
        float sampleLength = dir.length();
        dir = normalize(dir);
        s.ray.direction = dir; s.ray.origin = orig; s.ray.mint = RAY_BIAS; s.ray.maxt = sampleLength - (RAY_BIAS * 10);
        float d = dot(l.lightN, -dir);
        if (!(d > 0.f)) d = 0.f;     // d *= 1-signbit(d): one-sided
        s.color = l.le;
        s.pdf = d == 0. ? 0.f : (float)((sampleLength * sampleLength) / (d * l.xScale * l.yScale * 4.));
        return s;
    }
    Vector wc = l.center - orig;
    float dc = wc.length();
    s.color = l.le;
    s.ray.origin = orig; s.ray.mint = RAY_BIAS;
    if (dc <= l.radius) { s.ray.direction = Vector(0, 1, 0); s.ray.maxt = 0; s.pdf = 0; return s; }
    Vector w = wc / dc;
    float cosmax = sphereConeCos(l, orig);
    float cost = (1.f - x) + x * cosmax;
    float sint = sqrtf(std::max(0.f, 1.f - cost * cost));
    float phi = 2 * M_PI * y;
    Vector dir = normalize(tangentToWorld(Vector(sint * cosf(phi), sint * sinf(phi), cost), w));
    float t;
    sphereHit(l, orig, dir, 0.f, &t);
    s.ray.direction = dir; s.ray.maxt = t - (float)(RAY_BIAS * 10);
    float solid = 2.f * (float)M_PI * (1.f - cosmax);
    s.pdf = solid > 0.f ? 1.f / solid : 0.f;
    return s;
}
static float lightPdf(const Scene& sc, const Light& l, Ray* ray) {   // SquareLight::pdf (squareLight.h:88-97)
    if (l.type == AUR_LIGHT_ENV) {                                  // InfiniteAreaLight::pdf, hemisphere
        if (l.tex < 0) return 1.f / (M_PI * 2.f);
        float u, v;
        envUV(l, ray->direction, &u, &v);
        float pdf = envMapPdf(sc, l, u, v);
        return pdf / (M_PI * 2.f);
    }
    if (l.type == AUR_LIGHT_SQUARE) {
        float t, b1, b2;
        bool hit = triIntersect(l.tri[0][0], l.tri[0][1], l.tri[0][2], *ray, &t, &b1, &b2);
        if (!hit) hit = triIntersect(l.tri[1][0], l.tri[1][1], l.tri[1][2], *ray, &t, &b1, &b2);
        if (!hit) return 0.f;
        ray->maxt = t;
        float d = dot(l.lightN, normalize(ray->direction));
        d *= (0 < d) - (d < 0);
        float pdf = (ray->maxt * ray->maxt) / (d * l.xScale * l.yScale * 4.);
        ray->maxt -= RAY_BIAS * 10;
        return pdf;
    }
    float t;
    if (!sphereHit(l, ray->origin, ray->direction, ray->mint, &t) || t > ray->maxt) return 0.f;
    Vector wc = l.center - ray->origin;
    if (dot(wc, wc) <= l.radius * l.radius) return 0.f;
    ray->maxt = t - (float)(RAY_BIAS * 10);
    float solid = 2.f * (float)M_PI * (1.f - sphereConeCos(l, ray->origin));
    return solid > 0.f ? 1.f / solid : 0.f;
}

inline float PowerHeuristic(int nf, float fPdf, int ng, float gPdf) {   // integrator.cpp:28-31
    float f = nf * fPdf, g = ng * gPdf;
    return (f * f) / (f * f + g * g);
}

// ------------------------------------------------------------ Integrator (integrator.cpp)
struct Counts { uint64_t closest = 0, shadow = 0; };

static LocalGeometry hitGeometry(const Scene& sc, const Ray& ray, int prim, float t, float u, float v) {
    // EmbreeAccelerator::intersect post-process (embreeAccelerator.cpp:49-90) + updateLocalGeometry (:132-150)
    LocalGeometry lg;
    float w = 1. - u - v;
    const float* n = &sc.cornerN[(size_t)prim * 9];
    Vector norm(w * n[0] + u * n[3] + v * n[6], w * n[1] + u * n[4] + v * n[7], w * n[2] + u * n[5] + v * n[8]);
    if (dot(norm, ray.direction) > 0.) norm = norm * -1;
    Vector hitN = normalize(norm);
    lg.P = ray.origin + (ray.direction * t);
    lg.su = lg.sv = 0.f;
    if (!sc.cornerUV.empty()) {
        const float* uv = &sc.cornerUV[(size_t)prim * 6];
        lg.su = w * uv[0] + u * uv[2] + v * uv[4];
        lg.sv = w * uv[1] + u * uv[3] + v * uv[5];
    }
    lg.attr = sc.triAttr[prim];
    lg.Ng = hitN;
    lg.Nn = hitN;
    const Mat& m = sc.mats[sc.attrMat[lg.attr]];
    if (m.normTex != -1) {                           // Material::runNormalShader (material.cpp:27-40)
        Color map = m.normTex == -2 ? m.normC : shaderColor(sc, m.normTex, lg);
        Vector Ns = tangentToWorld(Vector(map.r, map.g, map.b), lg.Ng);
        if (Ns.x || Ns.y || Ns.z) lg.Nn = normalize(Ns);
        else lg.Nn = lg.Ng;
    }
    lg.Vn = -normalize(ray.direction);
    if (dot(lg.Vn, lg.Nn) <= 0.) {
        Vector tmp = cross(lg.Nn, lg.Vn);
        lg.Nn = normalize(cross(lg.Vn, tmp));
    }
    return lg;
}

// Derivatives of one vertex's next-event estimate D (adjoint only, FP64): per channel
// dD_c/d(albedo_c) of a Lambert lobe and dD_c/d(roughness) of a Cook-Torrance lobe.
// Sampling pdfs and MIS weights are constants of the derivative.
struct DirectGrad { double dAlbedo[3] = {0, 0, 0}, dRough[3] = {0, 0, 0}; };

// d ln D / d roughness of the Beckmann term at the half vector (ndoth), FP64:
// D = exp(-tan^2/r^2) / (r^2 pi cos^3), tan^2 = (1 - cos^2) / cos^2.
static double dlnBeckmann(double r, double ndoth) {
    const double c2 = ndoth * ndoth;
    const double tan2 = (1.0 - c2) / c2;
    return 2.0 * tan2 / (r * r * r) - 2.0 / r;
}
// the same for a sampled direction (cookTorrance.cpp:47-99): ctD floors r^2 at 0.001 and
// the sample clamps D at 1000, where the sample's colour no longer depends on roughness
static double dlnBeckmannSampled(const BrdfState& b, const Vector& L, const Vector& V, const Vector& N) {
    const double hx = (double)L.x + V.x, hy = (double)L.y + V.y, hz = (double)L.z + V.z;
    const double hl = std::sqrt(hx * hx + hy * hy + hz * hz);
    const double ndoth = (hx * N.x + hy * N.y + hz * N.z) / hl;
    const double r = b.roughness;
    if (r * r <= 0.001) return 0.0;
    const double c2 = ndoth * ndoth;
    const double tan2 = ndoth > 0.999 ? 0.0 : (1.0 - c2) / c2;
    const double D = std::exp(-tan2 / (r * r)) / (r * r * M_PI * c2 * ndoth);
    if (D >= 1000.0) return 0.0;
    return 2.0 * tan2 / (r * r * r) - 2.0 / r;
}

static Color integrateDirect(const Scene& sc, const LocalGeometry& lg, const BrdfState& brdf, const Rng& rng, int vtx,
                             Counts& cnt, DirectGrad* grad = nullptr) {
    Color result(0.f);
    int numLights = 0;
    std::vector<int> idx;
    for (int i = 0; i < (int)sc.lights.size(); ++i) if (lightVisible(sc.lights[i], lg.P, lg.Nn)) idx.push_back(i);
    numLights = (int)idx.size();
    if (!numLights) return result;
    int k = std::min((int)(rng(vdim(vtx, DIM_LIGHTPICK)) * numLights), numLights - 1);
    const Light& light = sc.lights[idx[k]];
    float lx = rng(vdim(vtx, DIM_LIGHTSAMPLE)), ly = rng(vdim(vtx, DIM_LIGHTSAMPLE + 1));
    if (brdf.type == MatteBrdf) {                                         // integrateDirectLight :33-54
        Sample3D ls = lightGenerateSample(sc, light, lg.P, lg.Nn, lx, ly);
        float costheta = dot(lg.Nn, ls.ray.direction);
        if (costheta >= 0. && ls.pdf > 0.) {
            ++cnt.shadow;
            if (!sceneOccluded(sc, ls.ray)) {
                result += ls.color * brdfEval(brdf, ls.ray.direction, lg.Vn, lg.Nn) * costheta / ls.pdf;
                if (grad && dot(ls.ray.direction, lg.Nn) > 0.) {       // eval = albedo / pi
                    const double k = (double)costheta / ls.pdf / M_PI;
                    grad->dAlbedo[0] += ls.color.r * k; grad->dAlbedo[1] += ls.color.g * k; grad->dAlbedo[2] += ls.color.b * k;
                }
            }
        }
    } else if (brdf.type == SpecBrdf) {                                   // integrateDirectMIS :56-98
        Sample3D ls = lightGenerateSample(sc, light, lg.P, lg.Nn, lx, ly);
        float costheta = dot(lg.Nn, ls.ray.direction);
        if (costheta > 0. && ls.pdf > 0.) {
            float bp = brdfPdf(brdf, ls.ray.direction, lg.Vn, lg.Nn);
            if (bp > 0.) {
                ++cnt.shadow;
                if (!sceneOccluded(sc, ls.ray)) {
                    float weight = PowerHeuristic(1, ls.pdf, 1, bp);
                    Color c0 = ls.color * weight * brdfEval(brdf, ls.ray.direction, lg.Vn, lg.Nn) * costheta / ls.pdf;
                    result += c0;
                    if (grad) {
                        const Vector& L = ls.ray.direction;
                        const double hx = (double)L.x + lg.Vn.x, hy = (double)L.y + lg.Vn.y, hz = (double)L.z + lg.Vn.z;
                        const double ndoth = (hx * lg.Nn.x + hy * lg.Nn.y + hz * lg.Nn.z) / std::sqrt(hx * hx + hy * hy + hz * hz);
                        const double g = dlnBeckmann(brdf.roughness, ndoth);
                        grad->dRough[0] += c0.r * g; grad->dRough[1] += c0.g * g; grad->dRough[2] += c0.b * g;
                    }
                }
            }
        }
        Sample3D bs = brdfGetSample(brdf, lg.Vn, lg.Nn, rng(vdim(vtx, DIM_MISBRDF)), rng(vdim(vtx, DIM_MISBRDF + 1)));
        bs.ray.origin = lg.P;
        costheta = dot(lg.Nn, bs.ray.direction);
        if (costheta > 0.) {
            float lp = lightPdf(sc, light, &bs.ray);
            if (lp > 0. && bs.pdf > 0.) {
                ++cnt.shadow;
                if (!sceneOccluded(sc, bs.ray)) {
                    float weight = PowerHeuristic(1, bs.pdf, 1, lp);
                    Color c1 = bs.color * weight * lightEval(sc, light, bs.ray.direction) * costheta / bs.pdf;
                    result += c1;
                    if (grad) {
                        const double g = dlnBeckmannSampled(brdf, bs.ray.direction, lg.Vn, lg.Nn);
                        grad->dRough[0] += c1.r * g; grad->dRough[1] += c1.g * g; grad->dRough[2] += c1.b * g;
                    }
                }
            }
        }
    }
    result *= (float)numLights;
    if (grad)
        for (int c = 0; c < 3; ++c) { grad->dAlbedo[c] *= numLights; grad->dRough[c] *= numLights; }
    return result;
}

enum { CameraRay = 0, DiffuseRay = 1, SpecularRay = 2, MirrorRay = 3 };

// One path from the camera ray's first hit (prim, t, u, v of `ray`); returns its
// firefly-filtered radiance (integrator.cpp:169-285, one iteration of the numSamples loop).
static Color pathFromHit(const Scene& sc, Ray ray, int prim, float t, float u, float v, const Vector& camDir,
                         const Rng& rng, int maxDepth, int minDepth, Counts& cnt) {
    Color Lo(0.f);
    float continueProbability = 1.f;
    Color pathThroughput(1.f);
    bool mattePath = false;
    int rayType = CameraRay;
    int bounces = 0, trueBounces = 0;
    while (trueBounces < maxDepth) {
        LocalGeometry lg = hitGeometry(sc, ray, prim, t, u, v);
        const int vtx = trueBounces;
        if (rayType == DiffuseRay) mattePath = true;
        if (rayType == CameraRay || rayType == MirrorRay) Lo += pathThroughput * sc.attrEmission[lg.attr];
        BrdfState brdf = getBrdf(sc, sc.attrMat[lg.attr], lg, mattePath, rng(vdim(vtx, DIM_LOBE)));
        Lo += integrateDirect(sc, lg, brdf, rng, vtx, cnt) * pathThroughput;
        Sample3D cur = brdfGetSample(brdf, lg.Vn, lg.Nn, rng(vdim(vtx, DIM_BRDF)), rng(vdim(vtx, DIM_BRDF + 1)));
        if (cur.pdf <= 0.f) break;
        if (!isMirrorType(brdf.type)) {
            pathThroughput *= cur.color * dot(lg.Nn, cur.ray.direction) / cur.pdf;
            if (bounces > minDepth) continueProbability *= cur.color.lum() * dot(lg.Nn, cur.ray.direction) / cur.pdf;
            if (pathThroughput.isBlack()) break;
            rayType = brdf.type == SpecBrdf ? SpecularRay : DiffuseRay;
        } else {                                                           // integrator.cpp:233-239
            pathThroughput *= cur.color;
            if (bounces > minDepth) continueProbability *= cur.color.lum();
            rayType = MirrorRay;
        }
        if (bounces > minDepth) {
            if (rng(vdim(vtx, DIM_ROULETTE)) > continueProbability) break;
            pathThroughput /= continueProbability;
        }
        cur.ray.origin = lg.P;
        ++trueBounces;
        if (!isMirrorType(brdf.type)) ++bounces;
        if (!traceNext(sc, trueBounces, maxDepth, rayType)) break;
        ray = cur.ray;
        ++cnt.closest;
        if (!sceneIntersect(sc, ray, &prim, &t, &u, &v)) {
            // a mirror ray that escapes adds the environment along the CAMERA sample's
            // direction (integrator.cpp:262-274 evaluates `sample`, the camera ray)
            if (rayType == MirrorRay)
                for (const Light& l : sc.lights)
                    if (l.type == AUR_LIGHT_ENV) Lo += lightEval(sc, l, camDir) * pathThroughput;
            break;
        }
    }
    // firefly filter; a non-finite estimate (which would never leave the loop) is dropped
    if (!std::isfinite(Lo.r) || !std::isfinite(Lo.g) || !std::isfinite(Lo.b)) return Color(0.f);
    while (Lo.r > FIREFLY || Lo.g > FIREFLY || Lo.b > FIREFLY) Lo *= 0.2f;
    return Lo;
}

// Integrator::integrateCameraSample(sample, numSamples) (integrator.cpp:152-300) in pass
// `pass`: the first pass of a render traces one path (renderer.cpp:231-258 starts
// lightSamples at 1), later passes lightSamples paths from the camera ray's first hit,
// each added as Lo / numSamples. Sub-path j draws from sample index pass * L + j
// (L = max(1, lightSamples)); the camera ray from pass * L. *paths = paths traced.
static Color integrateCameraSample(const Scene& sc, int x, int y, uint64_t key, uint32_t pixel, int pass,
                                   int lightSamples, int maxDepth, int minDepth, float* alpha, Counts& cnt,
                                   int* paths) {
    const int lmax = lightSamples > 1 ? lightSamples : 1;
    const int n = pass == 0 ? 1 : lmax;
    *paths = n;
    Rng rng; rng.key = key;
    rng.base = ((uint64_t)pixel << 32) | ((uint64_t)(pass * lmax) << 12);
    Ray ray = convertSample(sc, x, y, rng(0), rng(1));
    const Vector camDir = ray.direction;
    *alpha = 0;
    ++cnt.closest;
    int prim; float t, u, v;
    if (!sceneIntersect(sc, ray, &prim, &t, &u, &v)) {   // camera miss: the environment lights (integrator.cpp:290-300)
        Color env(0.f);
        for (const Light& l : sc.lights)
            if (l.type == AUR_LIGHT_ENV) { env += lightEval(sc, l, camDir); *alpha = 1.f; }
        return env;
    }
    *alpha = 1.f;
    Color result(0.f);
    for (int j = 0; j < n; ++j) {
        Rng rj = rng;
        rj.base = ((uint64_t)pixel << 32) | ((uint64_t)(pass * lmax + j) << 12);
        const Color Lo = pathFromHit(sc, ray, prim, t, u, v, camDir, rj, maxDepth, minDepth, cnt);
        if (n == 1) result = Lo;
        else result += Lo / (float)n;
    }
    return result;
}

// ------------------------------------------------------------ adjoint restatement (FP64, forward mode)
// Derivative of integrateCameraSample's estimator with the sampling decisions held
// fixed (pdfs, MIS weights, lobe choice, roulette and the firefly factor are constants),
// carried FORWARD along the path in double:
//   L = sum_k T_k D_k,  T_{k+1} = T_k w_k / q_k
//   dT_{k+1} = (dT_k w_k + T_k dw_k) / q_k,   dL += dT_k D_k + T_k dD_k
// plus the score d ln P(lobe_k)/dr of Kelemen's lobe choice on every term from vertex k
// on. (The product evaluates the same quantity in reverse, by path replay.)
// Parameter vector: per material m (diffuse r, g, b, roughness) at 4m..4m+3, then the
// texel floats at 4 nmat + i.
// A vertex's parameter: n blocks base[k] weighted w[k] (a triplanar texture blends up to
// three texels; everything else is one block of weight 1).
struct ParamRef { int n = 0; long base[3] = {-1, -1, -1}; double w[3] = {1, 1, 1}; bool perChannel = false;
                  double chain = 1.0; };

static ParamRef paramOf(const Scene& sc, int matId, const BrdfState& b, const LocalGeometry& lg, bool mattePath,
                        float lobeU) {
    ParamRef p;
    const Mat& m = sc.mats[matId];
    if (b.type == MatteBrdf) {                       // albedo (matte, Kelemen's diffuse lobe)
        if (m.type != AUR_MAT_MATTE && m.type != AUR_MAT_KELEMEN) return p;
        p.perChannel = true;
        if (m.diffTex >= 0) {
            const Tex& t = sc.texs[m.diffTex];
            const long tbase = 4 * (long)sc.mats.size() + (long)t.offset;
            if (t.triScale == 0.f) {
                p.n = 1;
                p.base[0] = tbase + 3 * texelOf(t, lg.su, lg.sv);
            } else {                                 // d colour / d texel = the texel's weight
                const TriTaps k = triplanarTaps(sc, t, lg, false);
                for (int i = 0; i < 3; ++i)
                    if (k.w[i] > 0) { p.base[p.n] = tbase + 3 * (long)k.idx[i]; p.w[p.n] = k.w[i]; ++p.n; }
            }
        } else {
            p.n = 1;
            p.base[0] = 4 * matId;
        }
        return p;
    }
    if (b.type == SpecBrdf && m.roughTex < 0 &&
        (m.type == AUR_MAT_KELEMEN || m.type == AUR_MAT_COOKTORRANCE || (m.type == AUR_MAT_METAL && lobeU > m.mix))) {
        p.n = 1;
        p.base[0] = 4 * matId + 3;                   // roughness; blurred on matte paths (kelemenMaterial.cpp:232-234)
        p.chain = mattePath ? 1.0 - CAUSTIC_BLUR : 1.0;
    }
    return p;
}

// d ln P(chosen lobe) / d roughness of Kelemen's choice (kelemenMaterial.cpp:236-253):
// P(spec) = A(cos, r_eff) clamped to [0, 1]; getAlbedo is linear in r * 31 between
// column ra and column rb (rb = 31: the reference's max(ra + 1, 31)).
static double kelemenScore(const Scene& sc, const Mat& m, const LocalGeometry& lg, const BrdfState& b, bool mattePath) {
    if (m.type != AUR_MAT_KELEMEN || m.refl >= 1.f || m.roughTex >= 0) return 0.0;
    float rough = m.rough;
    if (mattePath) rough = rough * (1. - CAUSTIC_BLUR) + CAUSTIC_BLUR;
    const float* table = sc.albedo + (size_t)m.table * COS_ENTRIES * ROUGH_ENTRIES;
    const float c = clampf(dot(lg.Nn, lg.Vn), 0., 1.);
    const double A = getAlbedo(table, c, rough);
    int i = std::max(0, std::min(afloor(c * (COS_ENTRIES - 1)), COS_ENTRIES - 1));
    const int i1 = std::min(i + 1, COS_ENTRIES - 1);
    const int ra = std::max(0, std::min(afloor(rough * (ROUGH_ENTRIES - 1)), ROUGH_ENTRIES - 1));
    const int rb = ROUGH_ENTRIES - 1;
    const double mixc = (double)(c * (COS_ENTRIES - 1) - i);
    const double colA = (1.0 - mixc) * table[i * ROUGH_ENTRIES + ra] + mixc * table[i1 * ROUGH_ENTRIES + ra];
    const double colB = (1.0 - mixc) * table[i * ROUGH_ENTRIES + rb] + mixc * table[i1 * ROUGH_ENTRIES + rb];
    const double dA = (colB - colA) * (ROUGH_ENTRIES - 1) * (mattePath ? 1.0 - CAUSTIC_BLUR : 1.0);
    if (b.type == SpecBrdf) return (A > 0.0 && A < 1.0) ? dA / A : 0.0;
    return A < 1.0 ? -dA / (1.0 - A) : 0.0;
}

struct DThroughput { long base; bool perChannel; double d[3]; };

static void addDT(std::vector<DThroughput>& dT, long base, bool perChannel, const double v[3]) {
    for (auto& e : dT)
        if (e.base == base && e.perChannel == perChannel) { for (int c = 0; c < 3; ++c) e.d[c] += v[c]; return; }
    dT.push_back({base, perChannel, {v[0], v[1], v[2]}});
}

// One camera path: the forward arithmetic of integrateCameraSample, plus the derivative
// of <delta, L> added (times the firefly factor) to grad.
// A mirror ray that escapes: Lo += E T for every environment light along the camera
// direction, and its derivative dT E.
static void envMiss(const Scene& sc, const Vector& camDir, const Color& T, const std::vector<DThroughput>& dT,
                    const double delta[3], Color& Lo, std::vector<std::pair<long, double>>& contrib) {
    for (const Light& l : sc.lights) {
        if (l.type != AUR_LIGHT_ENV) continue;
        const Color E = lightEval(sc, l, camDir);
        Lo += E * T;
        for (const auto& e : dT) {
            if (e.perChannel) {
                contrib.push_back({e.base + 0, delta[0] * e.d[0] * E.r});
                contrib.push_back({e.base + 1, delta[1] * e.d[1] * E.g});
                contrib.push_back({e.base + 2, delta[2] * e.d[2] * E.b});
            } else {
                contrib.push_back({e.base, delta[0] * e.d[0] * E.r + delta[1] * e.d[1] * E.g + delta[2] * e.d[2] * E.b});
            }
        }
    }
}

// camRng draws the camera ray (with light samples the paths of a camera sample share it),
// rng the path's decisions; delta = dLoss/dpixel / spp (/ n for one of n light-sample paths).
static void adjointCameraSample(const Scene& sc, int x, int y, const Rng& camRng, const Rng& rng, int maxDepth,
                                int minDepth, const double delta[3], double* grad) {
    Counts cnt;
    Ray ray = convertSample(sc, x, y, camRng(0), camRng(1));
    const Vector camDir = ray.direction;
    int prim; float t, u, v;
    if (!sceneIntersect(sc, ray, &prim, &t, &u, &v)) return;   // the environment alone: no parameter
    Color Lo(0.f);
    float continueProbability = 1.f;
    Color pathThroughput(1.f);
    bool mattePath = false;
    int rayType = CameraRay;
    int bounces = 0, trueBounces = 0;
    std::vector<DThroughput> dT;
    std::vector<std::pair<long, double>> contrib;
    while (trueBounces < maxDepth) {
        LocalGeometry lg = hitGeometry(sc, ray, prim, t, u, v);
        const int vtx = trueBounces;
        if (rayType == DiffuseRay) mattePath = true;
        if (rayType == CameraRay || rayType == MirrorRay) {
            const Color& E = sc.attrEmission[lg.attr];
            Lo += pathThroughput * E;
            // emission seen through mirror / transmission vertices carries dT
            for (const auto& e : dT) {
                if (e.perChannel) {
                    contrib.push_back({e.base + 0, delta[0] * e.d[0] * E.r});
                    contrib.push_back({e.base + 1, delta[1] * e.d[1] * E.g});
                    contrib.push_back({e.base + 2, delta[2] * e.d[2] * E.b});
                } else {
                    contrib.push_back({e.base, delta[0] * e.d[0] * E.r + delta[1] * e.d[1] * E.g + delta[2] * e.d[2] * E.b});
                }
            }
        }
        const float lobeU = rng(vdim(vtx, DIM_LOBE));
        const int matId = sc.attrMat[lg.attr];
        BrdfState brdf = getBrdf(sc, matId, lg, mattePath, lobeU);
        const double T[3] = {pathThroughput.r, pathThroughput.g, pathThroughput.b};
        const double score = kelemenScore(sc, sc.mats[matId], lg, brdf, mattePath);
        if (score != 0.0) {
            const double s3[3] = {T[0] * score, T[1] * score, T[2] * score};
            addDT(dT, 4L * matId + 3, false, s3);
        }
        const ParamRef pr = paramOf(sc, matId, brdf, lg, mattePath, lobeU);
        DirectGrad dg;
        Color D = integrateDirect(sc, lg, brdf, rng, vtx, cnt, &dg);
        Lo += D * pathThroughput;
        const double Dd[3] = {D.r, D.g, D.b};
        for (const auto& e : dT) {
            if (e.perChannel) for (int c = 0; c < 3; ++c) contrib.push_back({e.base + c, delta[c] * e.d[c] * Dd[c]});
            else contrib.push_back({e.base, delta[0] * e.d[0] * Dd[0] + delta[1] * e.d[1] * Dd[1] + delta[2] * e.d[2] * Dd[2]});
        }
        for (int k = 0; k < pr.n; ++k) {
            if (pr.perChannel)
                for (int c = 0; c < 3; ++c) contrib.push_back({pr.base[k] + c, pr.w[k] * delta[c] * T[c] * dg.dAlbedo[c]});
            else contrib.push_back({pr.base[k], pr.chain * (delta[0] * T[0] * dg.dRough[0] + delta[1] * T[1] * dg.dRough[1] +
                                                             delta[2] * T[2] * dg.dRough[2])});
        }
        Sample3D cur = brdfGetSample(brdf, lg.Vn, lg.Nn, rng(vdim(vtx, DIM_BRDF)), rng(vdim(vtx, DIM_BRDF + 1)));
        if (cur.pdf <= 0.f) break;
        if (isMirrorType(brdf.type)) {     // delta lobe: T *= colour; no parameter of its own
            for (auto& e : dT) { e.d[0] *= cur.color.r; e.d[1] *= cur.color.g; e.d[2] *= cur.color.b; }
            pathThroughput *= cur.color;
            if (bounces > minDepth) continueProbability *= cur.color.lum();
            rayType = MirrorRay;
            if (bounces > minDepth) {
                if (rng(vdim(vtx, DIM_ROULETTE)) > continueProbability) break;
                pathThroughput /= continueProbability;
                for (auto& e : dT) for (int c = 0; c < 3; ++c) e.d[c] /= continueProbability;
            }
            cur.ray.origin = lg.P;
            ++trueBounces;
            if (!traceNext(sc, trueBounces, maxDepth, rayType)) break;
            ray = cur.ray;
            if (!sceneIntersect(sc, ray, &prim, &t, &u, &v)) {
                if (rayType == MirrorRay) envMiss(sc, camDir, pathThroughput, dT, delta, Lo, contrib);
                break;
            }
            continue;
        }
        const float cosl = dot(lg.Nn, cur.ray.direction);
        const double w[3] = {(double)cur.color.r * cosl / cur.pdf, (double)cur.color.g * cosl / cur.pdf,
                             (double)cur.color.b * cosl / cur.pdf};
        double dw[3] = {0, 0, 0};
        if (pr.n > 0) {
            if (pr.perChannel) {
                for (int c = 0; c < 3; ++c) dw[c] = (double)cosl / cur.pdf / M_PI;   // w_c = albedo_c / pi cos / pdf
            } else {
                const double g = dlnBeckmannSampled(brdf, cur.ray.direction, lg.Vn, lg.Nn) * pr.chain;
                for (int c = 0; c < 3; ++c) dw[c] = w[c] * g;
            }
        }
        for (auto& e : dT) for (int c = 0; c < 3; ++c) e.d[c] *= w[c];
        for (int k = 0; k < pr.n; ++k) {
            const double add[3] = {pr.w[k] * T[0] * dw[0], pr.w[k] * T[1] * dw[1], pr.w[k] * T[2] * dw[2]};
            addDT(dT, pr.base[k], pr.perChannel, add);
        }
        pathThroughput *= cur.color * dot(lg.Nn, cur.ray.direction) / cur.pdf;
        if (bounces > minDepth) continueProbability *= cur.color.lum() * dot(lg.Nn, cur.ray.direction) / cur.pdf;
        if (pathThroughput.isBlack()) break;
        rayType = brdf.type == SpecBrdf ? SpecularRay : DiffuseRay;
        if (bounces > minDepth) {
            if (rng(vdim(vtx, DIM_ROULETTE)) > continueProbability) break;
            pathThroughput /= continueProbability;
            for (auto& e : dT) for (int c = 0; c < 3; ++c) e.d[c] /= continueProbability;
        }
        cur.ray.origin = lg.P;
        ++trueBounces;
        ++bounces;
        if (!traceNext(sc, trueBounces, maxDepth, rayType)) break;
        ray = cur.ray;
        if (!sceneIntersect(sc, ray, &prim, &t, &u, &v)) {
                if (rayType == MirrorRay) envMiss(sc, camDir, pathThroughput, dT, delta, Lo, contrib);
                break;
            }
    }
    if (!std::isfinite(Lo.r) || !std::isfinite(Lo.g) || !std::isfinite(Lo.b)) return;   // dropped, as the forward
    double clamp = 1.0;
    while (Lo.r > FIREFLY || Lo.g > FIREFLY || Lo.b > FIREFLY) { Lo *= 0.2f; clamp *= 0.2; }
    for (const auto& c : contrib) grad[c.first] += clamp * c.second;
}

// ------------------------------------------------------------ scene import
static Scene* makeScene(const aur_scene_desc* d, const float* albedo) {
    Scene* sc = new Scene();
    sc->tris.resize(d->ntri);
    for (uint32_t i = 0; i < d->ntri; ++i) {
        const float* a = d->verts + 3 * d->tri_vidx[3 * i];
        const float* b = d->verts + 3 * d->tri_vidx[3 * i + 1];
        const float* c = d->verts + 3 * d->tri_vidx[3 * i + 2];
        Point p1(a[0], a[1], a[2]), p2(b[0], b[1], b[2]), p3(c[0], c[1], c[2]);
        sc->tris[i].p1 = p1; sc->tris[i].e1 = p2 - p1; sc->tris[i].e2 = p3 - p1;
    }
    sc->triAttr.assign(d->tri_attr, d->tri_attr + d->ntri);
    sc->cornerN.assign(d->corner_normals, d->corner_normals + 9 * (size_t)d->ntri);
    if (d->corner_uvs) sc->cornerUV.assign(d->corner_uvs, d->corner_uvs + 6 * (size_t)d->ntri);
    sc->attrMat.assign(d->attr_material, d->attr_material + d->nattr);
    for (uint32_t i = 0; i < d->nattr; ++i)
        sc->attrEmission.push_back(Color(d->attr_emission[3 * i], d->attr_emission[3 * i + 1], d->attr_emission[3 * i + 2]));
    for (uint32_t m = 0; m < d->nmat; ++m) {
        const aur_material_desc& md = d->materials[m];
        Mat mt;
        mt.type = md.type;
        mt.diff = Color(md.diffuse[0], md.diffuse[1], md.diffuse[2]);
        mt.spec = Color(md.specular[0], md.specular[1], md.specular[2]);
        mt.gain = Color(md.gain[0], md.gain[1], md.gain[2]);
        mt.rough = md.roughness; mt.roughB = md.roughness_b; mt.refl = md.reflectance; mt.mix = md.mix;
        mt.diffTex = md.diffuse_tex; mt.specTex = md.specular_tex; mt.roughTex = md.roughness_tex;
        mt.ior = md.ior;
        mt.normTex = md.normal_kind == AUR_NORMAL_TEXTURE ? md.normal_tex : md.normal_kind == AUR_NORMAL_CONSTANT ? -2 : -1;
        mt.normC = Color(md.normal[0], md.normal[1], md.normal[2]);
        // KelemenMaterial ctor: modrefl = roundf(reflectance*20)/20 selects the cache (kelemenMaterial.cpp:49-52)
        mt.table = md.type == AUR_MAT_KELEMEN ? std::max(0, std::min(REFL_ENTRIES - 1, (int)roundf(md.reflectance * (REFL_ENTRIES - 1)))) : 0;
        sc->mats.push_back(mt);
    }
    for (uint32_t i = 0; i < d->nlight; ++i) {           // SquareLight ctor (squareLight.cpp:20-52)
        const aur_light_desc& ld = d->lights[i];
        Light l = Light();
        l.type = ld.type;
        float intensity = powf(2, ld.exposure);
        l.le = Color(ld.color[0], ld.color[1], ld.color[2]) * intensity;
        memcpy(l.m, ld.object_to_camera, sizeof(l.m));
        l.tex = -1;
        if (ld.type == AUR_LIGHT_ENV) {                 // InfiniteAreaLight ctor; m = camera-to-world
            l.escale = pow(2, ld.exposure);             // eval: color * pow(2, m_exposure)
            l.le = Color(ld.color[0], ld.color[1], ld.color[2]) * l.escale;
            invert4(l.m, l.minv);
            l.tex = ld.tex;                             // pdf normalisation once the texels are in
            sc->hasEnv = true;
        } else if (ld.type == AUR_LIGHT_SQUARE) {
            l.xScale = ld.size_x; l.yScale = ld.size_y;
            Point p1 = xformPoint(l.m, Point(-l.xScale, -l.yScale, 0));
            Point p2 = xformPoint(l.m, Point(-l.xScale, l.yScale, 0));
            Point p3 = xformPoint(l.m, Point(l.xScale, l.yScale, 0));
            Point p4 = xformPoint(l.m, Point(l.xScale, -l.yScale, 0));
            l.lightN = normalize(cross(p1 - p2, p2 - p3));
            l.pCam[0] = p1; l.pCam[1] = p2; l.pCam[2] = p3; l.pCam[3] = p4;
            // m_tri1 = (p1, p2, p4), m_tri2 = (p3, p2, p4) stored as (p1, e1, e2)
            l.tri[0][0] = p1; l.tri[0][1] = p2 - p1; l.tri[0][2] = p4 - p1;
            l.tri[1][0] = p3; l.tri[1][1] = p2 - p3; l.tri[1][2] = p4 - p3;
        } else {
            l.center = Point(ld.center[0], ld.center[1], ld.center[2]);
            l.radius = ld.radius;
        }
        sc->lights.push_back(l);
    }
    size_t off = 0;
    for (uint32_t t = 0; t < d->ntex; ++t) {
        Tex tx; tx.w = d->tex_dims[2 * t]; tx.h = d->tex_dims[2 * t + 1]; tx.px = nullptr; tx.offset = off;
        tx.triScale = d->tex_triplanar_scale ? d->tex_triplanar_scale[t] : 0.f;
        sc->texs.push_back(tx);
        off += 3 * (size_t)tx.w * tx.h;
    }
    sc->texels.assign(d->texels ? d->texels : nullptr, d->texels ? d->texels + off : nullptr);
    off = 0;
    for (auto& tx : sc->texs) { tx.px = sc->texels.data() + off; off += 3 * (size_t)tx.w * tx.h; }
    for (auto& l : sc->lights) {                        // Texture2D::initPdf: m_pdf_normalization
        if (l.type != AUR_LIGHT_ENV || l.tex < 0) continue;
        const Tex& t = sc->texs[l.tex];
        float lum = 0;
        for (int i = 0; i < t.h; i++)
            for (int j = 0; j < t.w; j++) {
                const float* p = t.px + 3 * ((size_t)i * t.w + j);
                lum += (p[0] + p[1] + p[2]) / 3.f;
            }
        l.pdfNorm = lum / (t.w * t.h);
    }
    sc->attrC2O.assign(16 * (size_t)d->nattr, 0.f);
    if (d->attr_camera_to_object) {
        sc->attrC2O.assign(d->attr_camera_to_object, d->attr_camera_to_object + 16 * (size_t)d->nattr);
    } else {
        for (uint32_t i = 0; i < d->nattr; ++i)
            for (int k = 0; k < 4; ++k) sc->attrC2O[16 * (size_t)i + 5 * k] = 1.f;
    }
    sc->albedo = albedo;
    sc->fov = d->fov; sc->width = d->width; sc->height = d->height;
    return sc;
}

}  // namespace oracle

using namespace oracle;

extern "C" {

// ---------------------------------------------------------------- RNG probe
float oracle_rng_u01(uint32_t seed, uint32_t pixel, uint32_t sample, uint32_t dim) {
    return draw(key_of(seed), ((uint64_t)pixel << 32) | ((uint64_t)sample << 12) | dim);
}

// ---------------------------------------------------------------- triangle soup queries
// Brute-force closest hit over all triangles (renderableTriangle.cpp:68-98 per triangle,
// maxt shrinking as in the reference's accept-if-t<=maxt rule). hits: t,u,v,prim,attr
// (prim -1 on a miss); ties[i] = number of triangles whose t equals the minimum exactly.
int oracle_trace_brute(const float* verts, const uint32_t* idx, const int32_t* attr, uint32_t ntri, const aur_ray* rays,
                       uint32_t n, aur_hit* hits, int32_t* ties, int threads) {
    std::vector<Tri> tris(ntri);
    for (uint32_t i = 0; i < ntri; ++i) {
        const float* a = verts + 3 * idx[3 * i]; const float* b = verts + 3 * idx[3 * i + 1]; const float* c = verts + 3 * idx[3 * i + 2];
        Point p1(a[0], a[1], a[2]), p2(b[0], b[1], b[2]), p3(c[0], c[1], c[2]);
        tris[i].p1 = p1; tris[i].e1 = p2 - p1; tris[i].e2 = p3 - p1;
    }
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
    for (long long r = 0; r < (long long)n; ++r) {
        Ray ray;
        ray.origin = Point(rays[r].org[0], rays[r].org[1], rays[r].org[2]);
        ray.direction = Vector(rays[r].dir[0], rays[r].dir[1], rays[r].dir[2]);
        ray.mint = rays[r].mint; ray.maxt = rays[r].maxt;
        int best = -1; float bt = 0, bu = 0, bv = 0;
        for (uint32_t i = 0; i < ntri; ++i) {
            float t, u, v;
            if (triIntersect(tris[i].p1, tris[i].e1, tris[i].e2, ray, &t, &u, &v)) {
                ray.maxt = t; best = (int)i; bt = t; bu = u; bv = v;
            }
        }
        int tie = 0;
        if (best >= 0) {
            Ray probe = ray; probe.maxt = bt;
            for (uint32_t i = 0; i < ntri; ++i) {
                float t, u, v;
                if (triIntersect(tris[i].p1, tris[i].e1, tris[i].e2, probe, &t, &u, &v) && t == bt) ++tie;
            }
        }
        hits[r].t = best >= 0 ? bt : rays[r].maxt; hits[r].u = bu; hits[r].v = bv;
        hits[r].prim = best; hits[r].attr = best >= 0 ? (attr ? attr[best] : 0) : -1;
        if (ties) ties[r] = tie;
    }
    return 0;
}

int oracle_occluded_brute(const float* verts, const uint32_t* idx, uint32_t ntri, const aur_ray* rays, uint32_t n,
                          uint8_t* occ, int threads) {
    std::vector<Tri> tris(ntri);
    for (uint32_t i = 0; i < ntri; ++i) {
        const float* a = verts + 3 * idx[3 * i]; const float* b = verts + 3 * idx[3 * i + 1]; const float* c = verts + 3 * idx[3 * i + 2];
        Point p1(a[0], a[1], a[2]), p2(b[0], b[1], b[2]), p3(c[0], c[1], c[2]);
        tris[i].p1 = p1; tris[i].e1 = p2 - p1; tris[i].e2 = p3 - p1;
    }
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
    for (long long r = 0; r < (long long)n; ++r) {
        Ray ray;
        ray.origin = Point(rays[r].org[0], rays[r].org[1], rays[r].org[2]);
        ray.direction = Vector(rays[r].dir[0], rays[r].dir[1], rays[r].dir[2]);
        ray.mint = rays[r].mint; ray.maxt = rays[r].maxt;
        uint8_t o = 0;
        for (uint32_t i = 0; i < ntri && !o; ++i) {
            float t, u, v;
            if (triIntersect(tris[i].p1, tris[i].e1, tris[i].e2, ray, &t, &u, &v)) o = 1;
        }
        occ[r] = o;
    }
    return 0;
}

// ---------------------------------------------------------------- scene handle
void* oracle_scene_create(const aur_scene_desc* d, const float* albedo_tables, int use_bvh, int max_leaf) {
    Scene* sc = makeScene(d, albedo_tables);
    if (use_bvh) buildBvh(*sc, max_leaf > 0 ? max_leaf : 4);
    return sc;
}
void oracle_scene_destroy(void* h) { delete (Scene*)h; }
int oracle_scene_bvh_nodes(void* h) { return (int)((Scene*)h)->nodes.size(); }

int oracle_trace(void* h, const aur_ray* rays, uint32_t n, aur_hit* hits, int threads) {
    const Scene& sc = *(Scene*)h;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long r = 0; r < (long long)n; ++r) {
        Ray ray;
        ray.origin = Point(rays[r].org[0], rays[r].org[1], rays[r].org[2]);
        ray.direction = Vector(rays[r].dir[0], rays[r].dir[1], rays[r].dir[2]);
        ray.mint = rays[r].mint; ray.maxt = rays[r].maxt;
        int prim = -1; float t = rays[r].maxt, u = 0, v = 0;
        bool hit = sceneIntersect(sc, ray, &prim, &t, &u, &v);
        hits[r].t = hit ? t : rays[r].maxt; hits[r].u = hit ? u : 0; hits[r].v = hit ? v : 0;
        hits[r].prim = hit ? prim : -1; hits[r].attr = hit ? sc.triAttr[prim] : -1;
    }
    return 0;
}

// EmbreeAccelerator::intersect's post-process (embreeAccelerator.cpp:49-90) of given hits:
// out[8 i ..] = hitP xyz, hitN xyz (face-forwarded, normalised), st; zeros for a miss.
int oracle_isect_post(void* h, const aur_ray* rays, const aur_hit* hits, uint32_t n, float* out) {
    const Scene& sc = *(Scene*)h;
    for (uint32_t r = 0; r < n; ++r) {
        float* o = out + 8 * (size_t)r;
        for (int k = 0; k < 8; ++k) o[k] = 0.f;
        if (hits[r].prim < 0) continue;
        const int prim = hits[r].prim;
        const float u = hits[r].u, v = hits[r].v, t = hits[r].t;
        const Point org(rays[r].org[0], rays[r].org[1], rays[r].org[2]);
        const Vector dir(rays[r].dir[0], rays[r].dir[1], rays[r].dir[2]);
        float w = 1. - u - v;
        const float* nn = &sc.cornerN[(size_t)prim * 9];
        Vector norm(w * nn[0] + u * nn[3] + v * nn[6], w * nn[1] + u * nn[4] + v * nn[7],
                    w * nn[2] + u * nn[5] + v * nn[8]);
        if (dot(norm, dir) > 0.) norm = norm * -1;
        const Vector hitN = normalize(norm);
        const Point hitP = org + (dir * t);
        o[0] = hitP.x; o[1] = hitP.y; o[2] = hitP.z;
        o[3] = hitN.x; o[4] = hitN.y; o[5] = hitN.z;
        if (!sc.cornerUV.empty()) {
            const float* uv = &sc.cornerUV[(size_t)prim * 6];
            o[6] = w * uv[0] + u * uv[2] + v * uv[4];
            o[7] = w * uv[1] + u * uv[3] + v * uv[5];
        }
    }
    return 0;
}

// Renders pixels [x0, x0+w) x [y0, y0+h) of the full image with spp camera paths each.
// mean_rgba: w*h*4 doubles (RGB mean, alpha mean); m2_rgb: w*h*3 Welford sums of squared
// deviations (may be NULL); counts[0..2] += closest rays, shadow rays, paths.
int oracle_render(void* h, int spp, int sample_offset, int max_depth, int min_depth, uint32_t seed, int threads,
                  int x0, int y0, int w, int hgt, double* mean_rgba, double* m2_rgb, uint64_t* counts,
                  int light_samples) {
    const Scene& sc = *(Scene*)h;
    if (threads > 0) omp_set_num_threads(threads);
    const uint64_t key = key_of(seed);
    uint64_t cl = 0, sh = 0, np = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : cl, sh, np)
    for (long long i = 0; i < (long long)w * hgt; ++i) {
        const int x = x0 + (int)(i % w), y = y0 + (int)(i / w);
        const uint32_t pixel = (uint32_t)y * (uint32_t)sc.width + (uint32_t)x;
        double mean[3] = {0, 0, 0}, m2[3] = {0, 0, 0}, a = 0;
        Counts cnt;
        for (int s = 0; s < spp; ++s) {
            float alpha;
            int n;
            Color c = integrateCameraSample(sc, x, y, key, pixel, sample_offset + s, light_samples, max_depth, min_depth,
                                            &alpha, cnt, &n);
            np += (uint64_t)n;
            const double v[3] = {c.r, c.g, c.b};
            for (int k = 0; k < 3; ++k) {            // Welford
                const double dlt = v[k] - mean[k];
                mean[k] += dlt / (s + 1);
                m2[k] += dlt * (v[k] - mean[k]);
            }
            a += alpha;
        }
        for (int k = 0; k < 3; ++k) mean_rgba[4 * i + k] = mean[k];
        mean_rgba[4 * i + 3] = a / spp;
        if (m2_rgb) for (int k = 0; k < 3; ++k) m2_rgb[3 * i + k] = m2[k];
        cl += cnt.closest; sh += cnt.shadow;
    }
    if (counts) { counts[0] += cl; counts[1] += sh; counts[2] += np; }
    return 0;
}

// dLoss/dparams of <dfilm, image> restricted to pixels [x0, x0+w) x [y0, y0+h), with
// dfilm the full W*H*4 image gradient (alpha ignored) and the image the spp-sample mean.
// grad: 4*nmat + ntexel_floats doubles (overwritten).
// light_samples L > 1: camera sample s (s > 0) has L paths from its camera ray's first hit,
// drawing from sample indices s L + j and weighted 1 / L (integrateCameraSample(sample, L)).
int oracle_adjoint(void* h, int spp, int sample_offset, int max_depth, int min_depth, uint32_t seed, int threads,
                   int x0, int y0, int w, int hgt, const float* dfilm, double* grad, int light_samples) {
    const Scene& sc = *(Scene*)h;
    const size_t np = 4 * sc.mats.size() + sc.texels.size();
    if (threads > 0) omp_set_num_threads(threads);
    const uint64_t key = key_of(seed);
    std::fill(grad, grad + np, 0.0);
#pragma omp parallel
    {
        std::vector<double> local(np, 0.0);
#pragma omp for schedule(dynamic, 4)
        for (long long i = 0; i < (long long)w * hgt; ++i) {
            const int x = x0 + (int)(i % w), y = y0 + (int)(i / w);
            const uint32_t pixel = (uint32_t)y * (uint32_t)sc.width + (uint32_t)x;
            const double delta[3] = {(double)dfilm[4 * (size_t)pixel] / spp, (double)dfilm[4 * (size_t)pixel + 1] / spp,
                                     (double)dfilm[4 * (size_t)pixel + 2] / spp};
            if (delta[0] == 0 && delta[1] == 0 && delta[2] == 0) continue;
            const int lmax = light_samples > 1 ? light_samples : 1;
            for (int s = 0; s < spp; ++s) {
                const int pass = sample_offset + s;
                const int n = pass == 0 ? 1 : lmax;
                const double dn[3] = {delta[0] / n, delta[1] / n, delta[2] / n};
                Rng cam; cam.key = key;
                cam.base = ((uint64_t)pixel << 32) | ((uint64_t)(pass * lmax) << 12);
                for (int j = 0; j < n; ++j) {
                    Rng rng = cam;
                    rng.base = ((uint64_t)pixel << 32) | ((uint64_t)(pass * lmax + j) << 12);
                    adjointCameraSample(sc, x, y, cam, rng, max_depth, min_depth, dn, local.data());
                }
            }
        }
#pragma omp critical
        for (size_t k = 0; k < np; ++k) grad[k] += local[k];
    }
    return 0;
}

// ---------------------------------------------------------------- Kelemen table
// KelemenMaterial::preCalcAlbedo (kelemenMaterial.cpp:113-178) with `samples`
// draws per entry from an independent stream (seed); out[cos * 32 + rough].
int oracle_kelemen_table(float reflectance, int samples, uint32_t seed, float* out, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    const uint64_t key = key_of(seed);
#pragma omp parallel for schedule(dynamic, 1)
    for (int e = 0; e < COS_ENTRIES * ROUGH_ENTRIES; ++e) {
        const int i = e / ROUGH_ENTRIES, r = e % ROUGH_ENTRIES;
        float roughness = std::max(0.00001f, (float)r / (ROUGH_ENTRIES - 1.f));
        double albedo = 0;
        for (int j = 0; j < samples; ++j) {
            const uint64_t c = ((uint64_t)e << 32) | (uint64_t)(3 * j);
            float r1 = draw(key, c), r2 = draw(key, c + 1), r3 = draw(key, c + 2);
            float z = cosf(atanf(roughness * sqrtf(-log(1.f - r1))));
            float rr = sqrtf(fmax(0.f, 1.f - z * z));
            float phi = M_PI * 2 * r2;
            Vector Hn = normalize(Vector(rr * cosf(phi), rr * sinf(phi), z));
            Vector Nn(0, 0, 1);
            z = std::max(0.0001f, (float)i / (COS_ENTRIES - 1));
            rr = sqrtf(fmax(0.f, 1.f - z * z));
            phi = r3 * 2 * M_PI;
            Vector Vn = normalize(Vector(rr * cosf(phi), rr * sinf(phi), z));
            if (dot(Hn, Vn) < 0.) Hn = -Hn;
            float vdoth = dot(Vn, Hn);
            if (vdoth > 0.000001) {
                Vector Ln = normalize((Hn * 2 * vdoth) - Vn);
                float F = schlick(dot(Hn, Ln), reflectance);
                double a = F * std::max(0.f, dot(Ln, Nn)) / vdoth;
                albedo += a / ((float)samples / 100);
            }
        }
        out[i * ROUGH_ENTRIES + r] = albedo / 100.f;
    }
    return 0;
}

// ---------------------------------------------------------------- shading probes
// Record layouts (floats), shared with the device probe aur_shading_probe:
// kind 0 brdf_sample   in: lobe, color3, rough, V3, N3, r1, r2      (13) out: dir3, pdf, color3 (7)
// kind 1 brdf_eval     in: lobe, color3, rough, L3, V3, N3          (14) out: color3 (3)
// kind 2 brdf_pdf      in: lobe, color3, rough, L3, V3, N3          (14) out: pdf (1)
// kind 3 kelemen       in: table index, costheta, roughness          (3) out: albedo (1)
// kind 4 camera_ray    in: fov, w, h, px, py, j1, j2                 (7) out: dir3 (3)
// kind 5 power_heur.   in: f, g                                      (2) out: w (1)
// kind 6 light_sample  in: light, P3, u1, u2, N3                     (9) out: dir3, maxt, pdf, color3 (8)
// kind 7 light_pdf     in: light, o3, d3, mint, maxt                 (9) out: pdf, maxt (2)
// kind 8 light_visible in: light, P3, N3                             (7) out: visible (1)
// kind 9 get_brdf      in: material, V3, N3, su, sv, matte, lobe_u  (11) out: lobe, color3, rough (5)
// kind 10 shade_point  in: triangle, t, u, v, o3, d3, matte, lobe_u (12) out: N3, Ng3, lobe, color3, rough (11)
int oracle_shading_probe(void* h, int kind, const float* in, uint32_t n, float* out, const float* tables) {
    static const int kIn[11] = {13, 14, 14, 3, 7, 2, 9, 9, 7, 11, 12};
    static const int kOut[11] = {7, 3, 1, 1, 3, 1, 8, 2, 1, 5, 11};
    if (kind < 0 || kind > 10) return -1;
    const Scene* sc = (const Scene*)h;
    if (kind >= 6 && !sc) return -2;
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = in + (size_t)i * kIn[kind];
        float* o = out + (size_t)i * kOut[kind];
        if (kind <= 2) {
            BrdfState b; b.type = (int)q[0]; b.color = Color(q[1], q[2], q[3]); b.roughness = q[4];
            if (kind == 0) {
                Sample3D s = brdfGetSample(b, Vector(q[5], q[6], q[7]), Vector(q[8], q[9], q[10]), q[11], q[12]);
                o[0] = s.ray.direction.x; o[1] = s.ray.direction.y; o[2] = s.ray.direction.z;
                o[3] = s.pdf; o[4] = s.color.r; o[5] = s.color.g; o[6] = s.color.b;
            } else {
                Vector L(q[5], q[6], q[7]), V(q[8], q[9], q[10]), N(q[11], q[12], q[13]);
                if (kind == 1) { Color c = brdfEval(b, L, V, N); o[0] = c.r; o[1] = c.g; o[2] = c.b; }
                else o[0] = brdfPdf(b, L, V, N);
            }
        } else if (kind == 3) {
            o[0] = getAlbedo(tables + (size_t)q[0] * COS_ENTRIES * ROUGH_ENTRIES, q[1], q[2]);
        } else if (kind == 4) {
            Scene tmp; tmp.fov = q[0]; tmp.width = (int)q[1]; tmp.height = (int)q[2];
            Ray r = convertSample(tmp, (int)q[3], (int)q[4], q[5], q[6]);
            o[0] = r.direction.x; o[1] = r.direction.y; o[2] = r.direction.z;
        } else if (kind == 5) {
            o[0] = PowerHeuristic(1, q[0], 1, q[1]);
        } else if (kind == 6) {
            Sample3D s = lightGenerateSample(*sc, sc->lights[(int)q[0]], Point(q[1], q[2], q[3]), Vector(q[6], q[7], q[8]),
                                             q[4], q[5]);
            o[0] = s.ray.direction.x; o[1] = s.ray.direction.y; o[2] = s.ray.direction.z; o[3] = s.ray.maxt;
            o[4] = s.pdf; o[5] = s.color.r; o[6] = s.color.g; o[7] = s.color.b;
        } else if (kind == 7) {
            Ray r; r.origin = Point(q[1], q[2], q[3]); r.direction = Vector(q[4], q[5], q[6]); r.mint = q[7]; r.maxt = q[8];
            o[0] = lightPdf(*sc, sc->lights[(int)q[0]], &r); o[1] = r.maxt;
        } else if (kind == 8) {
            o[0] = lightVisible(sc->lights[(int)q[0]], Point(q[1], q[2], q[3]), Vector(q[4], q[5], q[6])) ? 1.f : 0.f;
        } else if (kind == 9) {
            LocalGeometry lg;
            lg.P = Point(0, 0, 0); lg.Vn = Vector(q[1], q[2], q[3]); lg.Nn = lg.Ng = Vector(q[4], q[5], q[6]);
            lg.su = q[7]; lg.sv = q[8]; lg.attr = 0;
            BrdfState b = getBrdf(*sc, (int)q[0], lg, q[9] != 0.f, q[10]);
            o[0] = (float)b.type; o[1] = b.color.r; o[2] = b.color.g; o[3] = b.color.b; o[4] = b.roughness;
        } else {
            Ray r; r.origin = Point(q[4], q[5], q[6]); r.direction = Vector(q[7], q[8], q[9]);
            LocalGeometry lg = hitGeometry(*sc, r, (int)q[0], q[1], q[2], q[3]);
            BrdfState b = getBrdf(*sc, sc->attrMat[lg.attr], lg, q[10] != 0.f, q[11]);
            o[0] = lg.Nn.x; o[1] = lg.Nn.y; o[2] = lg.Nn.z; o[3] = lg.Ng.x; o[4] = lg.Ng.y; o[5] = lg.Ng.z;
            o[6] = (float)b.type; o[7] = b.color.r; o[8] = b.color.g; o[9] = b.color.b; o[10] = b.roughness;
        }
    }
    return 0;
}

}  // extern "C"
