// aur_core.cuh — float3 math, constants and the counter-based path RNG shared by
// every sm_100a kernel of the Aurora path-tracing core.
//
// Semantics follow the reference's core math so that device results track the
// CPU restatement to a few ulp:
//   * dot/cross/normalize/length      Aurora/src/core/math_utils.h:31-60, vector.h:65-80
//     (length() returns 1e-4 for a zero vector; normalize multiplies by 1/len)
//   * coordinateSystem/tangentToWorld  Aurora/src/core/math_utils.h:81-129
//   * SampleHemisphereUniform          Aurora/src/core/math_utils.h:70-78
//   * schlick                          Aurora/src/core/math_utils.h:222-224
//   * Color::isBlack / lum             Aurora/src/core/color.h:149-159
//   * constants                        Aurora/constants.h:12-41
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <math.h>

#define AUR_HD __host__ __device__ __forceinline__

namespace aur {

// Aurora/constants.h
constexpr float kRayBias = 0.0005f;      // RAY_BIAS
constexpr float kFirefly = 200.f;        // FIREFLY
constexpr float kCausticBlur = 0.2f;     // CAUSTIC_BLUR
constexpr float kIsBlack = 0.0001f;      // ISBLACK
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr int kAlbedoCos = 64;           // SPECALBEDO_COSTHETA_ENTRIES
constexpr int kAlbedoRough = 32;         // SPECALBEDO_ROUGHNESSS_ENTRIES
constexpr int kAlbedoRefl = 21;          // SPECALBEDO_REFLECTANCE_ENTRIES

// Random-number dimensions consumed per path vertex. The reference draws
// rand() in this order (camera.cpp:47-48, kelemenMaterial.cpp:242,
// integrator.cpp:116, squareLight.h:63-64, cookTorrance.cpp:55-56,
// lambert.h:50-51, integrator.cpp:244); here each draw owns a fixed slot so
// that the plain kernel, the wavefront stages, the adjoint replay and the CPU
// oracle consume identical numbers.
constexpr int kDimCamera = 0;            // 2 dims: pixel jitter x, y
constexpr int kDimsPerVertex = 10;
constexpr int kDimLobe = 0;              // Kelemen lobe / metal mix choice
constexpr int kDimLightPick = 1;
constexpr int kDimLightSample = 2;       // 2 dims
constexpr int kDimMisBrdf = 4;           // 2 dims
constexpr int kDimBrdf = 6;              // 2 dims
constexpr int kDimRoulette = 8;
AUR_HD uint32_t vertex_dim(int vertex, int slot) { return 2u + (uint32_t)vertex * kDimsPerVertex + (uint32_t)slot; }

// ---------------------------------------------------------------- RNG
// SplitMix64 (Steele, Lea, Flood: "Fast splittable pseudorandom number
// generators", OOPSLA 2014) used as a counter-based generator: the state for a
// draw is key + counter * golden-gamma, and the output is its 64-bit finaliser.
// The finaliser is a bijection, so distinct counters never collide.
// counter = pixel << 32 | sample << 12 | dim  (sample < 2^20, dim < 4096).
AUR_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
AUR_HD uint64_t seed_key(uint32_t seed) { return mix64((uint64_t)seed * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull); }
AUR_HD uint64_t path_base(uint32_t pixel, uint32_t sample) { return ((uint64_t)pixel << 32) | ((uint64_t)sample << 12); }
AUR_HD float rng_u01(uint64_t key, uint64_t counter) {
    uint64_t z = mix64(key + counter * 0x9e3779b97f4a7c15ull);
    return (float)(uint32_t)(z >> 40) * (1.0f / 16777216.0f);   // [0, 1), exact in FP32
}
struct PathRng {
    uint64_t key, base;
    AUR_HD float u(uint32_t dim) const { return rng_u01(key, base | (uint64_t)dim); }
};

// ---------------------------------------------------------------- transcendentals
// The shading math is evaluated in double and rounded once to float, which is
// the correctly rounded float result in all but double-rounding cases. That is
// what the host's libm returns (to within its own <1 ulp), so device and CPU
// restatement agree on BRDF values even where the Beckmann lobe amplifies a
// 1-ulp difference (d ln D / d theta ~ 2 tan / m^2).
// A translation unit that defines AUR_MATH_OUT_OF_LINE before including this header gets
// them out of line: inlined at every call site, their double-precision bodies multiply the
// code of the adjoint kernels, whose warps then stall on instruction fetch. (The forward
// shading kernels are faster with them inlined.)
#ifdef AUR_MATH_OUT_OF_LINE
#define AUR_MATH static __host__ __device__ __noinline__
#else
#define AUR_MATH AUR_HD
#endif
AUR_MATH float xexpf(float x) { return (float)exp((double)x); }
AUR_MATH float xlogf(float x) { return (float)log((double)x); }
AUR_MATH float xpowf(float x, float y) { return (float)pow((double)x, (double)y); }
AUR_MATH float xacosf(float x) { return (float)acos((double)x); }
AUR_MATH float xtanf(float x) { return (float)tan((double)x); }
AUR_MATH float xatanf(float x) { return (float)atan((double)x); }
AUR_MATH float xcosf(float x) { return (float)cos((double)x); }
AUR_MATH float xsinf(float x) { return (float)sin((double)x); }
AUR_MATH float xatan2f(float y, float x) { return (float)atan2((double)y, (double)x); }

// ---------------------------------------------------------------- float3 helpers
AUR_HD float3 mk(float x, float y, float z) { float3 r; r.x = x; r.y = y; r.z = z; return r; }
AUR_HD float3 operator+(float3 a, float3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
AUR_HD float3 operator-(float3 a, float3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
AUR_HD float3 operator-(float3 a) { return mk(-a.x, -a.y, -a.z); }
AUR_HD float3 operator*(float3 a, float f) { return mk(a.x * f, a.y * f, a.z * f); }
AUR_HD float3 operator*(float3 a, float3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
AUR_HD float3& operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
AUR_HD float3& operator*=(float3& a, float3 b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
AUR_HD float3& operator*=(float3& a, float f) { a.x *= f; a.y *= f; a.z *= f; return a; }
// Color / float multiplies by the reciprocal (color.h operator/).
AUR_HD float3 cdiv(float3 a, float f) { float d = 1.f / f; return mk(a.x * d, a.y * d, a.z * d); }

AUR_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
AUR_HD float3 cross(float3 a, float3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
AUR_HD float length(float3 v) {
    float l = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return l == 0.f ? 0.0001f : l;
}
AUR_HD float3 normalize(float3 v) { float inv = 1.f / length(v); return mk(v.x * inv, v.y * inv, v.z * inv); }
AUR_HD float lum(float3 c) { return (float)(0.2126 * c.x + 0.7152 * c.y + 0.0722 * c.z); }   // double literals
AUR_HD bool is_black(float3 c) {   // compared with the double ISBLACK as in color.h:149-151
    return (double)c.x < 0.0001 && (double)c.y < 0.0001 && (double)c.z < 0.0001;
}
AUR_HD float schlick(float vdoth, float refl) { return refl + xpowf(1.f - vdoth, 5.f) * (1.f - refl); }

AUR_HD void coordinate_system(float3 v1, float3* v2, float3* v3) {
    if (!(v1.x != 0.f) && v1.y != 0.f && !(v1.z != 0.f)) *v2 = cross(v1, mk(1.f, 0.f, 0.f));
    else *v2 = cross(v1, mk(0.f, 1.f, 0.f));
    *v3 = cross(v1, *v2);
}
AUR_HD float3 tangent_to_world(float3 dir, float3 n) {
    float3 dpdu, dpdv;
    coordinate_system(n, &dpdu, &dpdv);
    float3 r = normalize(dpdu) * dir.x;
    r = r + normalize(dpdv) * dir.y;
    r = r + n * dir.z;
    return r;
}
AUR_HD float two_pi_times(float r) { return (float)(6.283185307179586 * (double)r); }   // 2 * M_PI * r in double
AUR_HD float3 sample_hemisphere_uniform(float r1, float r2) {
    float z = r1;
    float r = sqrtf(fmaxf(0.f, 1.f - z * z));
    float phi = two_pi_times(r2);
    return mk(r * xcosf(phi), r * xsinf(phi), z);
}

// Neumaier-compensated FP32 accumulator (film and gradient sums).
struct Kahan3 {
    float3 s, c;
    AUR_HD void init() { s = mk(0.f, 0.f, 0.f); c = s; }
    AUR_HD static void add1(float& s, float& c, float x) {
        float t = s + x;
        if (fabsf(s) >= fabsf(x)) c += (s - t) + x; else c += (x - t) + s;
        s = t;
    }
    AUR_HD void add(float3 x) { add1(s.x, c.x, x.x); add1(s.y, c.y, x.y); add1(s.z, c.z, x.z); }
    AUR_HD float3 total() const { return s + c; }
};

}  // namespace aur
