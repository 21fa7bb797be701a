// aur_shading.cuh — scene records and the per-vertex shading math of the
// Aurora path loop: camera rays, Lambert / Cook-Torrance(Beckmann) / Kelemen /
// metal lobes, square and sphere area lights, texture lookups and the exact
// FP32 Moller-Trumbore triangle test. Every function is __host__ __device__
// and stateless; random numbers are passed in by the caller.
//
// Reference semantics restated here (file:line in espennordahl/Aurora):
//   camera ray                Aurora/src/frontend/camera.cpp:34-62
//   Lambert                   Aurora/src/shading/bxdfs/lambert.h:44-80
//   Cook-Torrance (Beckmann)  Aurora/src/shading/bxdfs/cookTorrance.cpp:40-144
//   Kelemen lobe choice       Aurora/src/shading/materials/kelemenMaterial.cpp:180-255
//   metal lobe choice         Aurora/src/shading/materials/metalMaterial.cpp:32-62
//   matte / constant          matteMaterial.cpp:30-35, constantMaterial.cpp:19-24, bxdfs/constant.cpp:23-37
//   square light              Aurora/src/lights/squareLight.h:57-122, squareLight.cpp:20-52
//   triangle test             Aurora/src/geometry/renderableTriangle.cpp:33-123
//   texture2D (nearest)       Aurora/src/shading/shaders/texture2DShader.h:28-31, frontend/texture2D.cpp:48-72
//   triplanar texture         Aurora/src/shading/shaders/triplanarTextureShader.h:29-51 (colour), :71-93 (float)
//   normal map                Aurora/src/shading/materials/material.cpp:27-40, frontend/integrator.cpp:132-150
// The sphere light has no reference counterpart (uniform cone sampling of the
// subtended solid angle, as in Shirley & Wang 1994 / pbrt v3 section 14.2).
#pragma once
#include "aur_core.cuh"

namespace aur {

// ------------------------------------------------------------------ records
enum MatType : int { MAT_MATTE = 0, MAT_KELEMEN = 1, MAT_COOKTORRANCE = 2, MAT_METAL = 3, MAT_CONSTANT = 4,
                     MAT_GLASS = 5 };
// brdf.h BrdfType; LOBE_MIRROR (SpecMirror) and LOBE_TRANSMIT (SpecTransmit) are both the
// reference's MirrorBrdf: delta lobes without next-event estimation
enum LobeType : int { LOBE_MATTE = 0, LOBE_SPEC = 1, LOBE_MIRROR = 2, LOBE_CONSTANT = 3, LOBE_TRANSMIT = 4 };
enum LightType : int { LIGHT_SQUARE = 0, LIGHT_SPHERE = 1, LIGHT_ENV = 2 };

struct Material {            // 96 B
    int type;
    int diff_tex, spec_tex, rough_tex;   // texture index or -1
    float3 diff;             // matte colour / Kelemen diffusecolor
    float3 spec;             // Kelemen speccolor / CT colour / metal reflectance
    float3 gain;             // metal gain
    float rough, rough_b;    // roughness (metal: roughnessA, roughnessB)
    float refl;              // Kelemen reflectance (selects the albedo table)
    float mix;               // metal mix
    int table;               // Kelemen albedo table index (64x32 floats each)
    float ior;               // glass index of refraction
    int norm_tex;            // normal-map shader: texture index, kNormalNone or kNormalConst
    float3 norm;             // kNormalConst: the constant tangent-space map colour
};
constexpr int kNormalNone = -1, kNormalConst = -2;
struct Attr {                // AttributeState: material + emission (attributeState.h)
    int material;
    float3 emission;
};
struct Light {
    int type;
    float xs, ys, radius;
    float3 p[4];             // square corners in camera space (squareLight.cpp:28-48)
    float3 n;                // lightN = normalize(cross(p1-p2, p2-p3))
    float3 le;               // colour * 2^exposure
    float3 center;           // sphere centre (camera space)
    float m[16];             // square: object-to-camera, row major; env: camera-to-world
    float minv[16];          // env: world-to-camera (the FP32 Gauss-Jordan inverse of m)
    int tex;                 // env: env-map texture index, -1 for a constant colour
    float escale;            // env: 2^exposure (the map's texels are scaled by it)
    float pdf_norm;          // env: mean texel luminance (Texture2D::initPdf)
    int pad;
};
// A texture shader over one image (texels: RGB float, offset in floats): tri_scale 0 is
// the uv lookup (texture2DShader), > 0 the triplanar projection with that scale.
struct Texture { int w, h, offset; float tri_scale; };
struct Camera { float fov; int w, h; int pad; };

struct ShadeScene {          // device pointers for the shading stage
    const Material* mats;
    const Attr* attrs;
    const Light* lights;
    const Texture* texs;
    const float* texels;
    const float* albedo;     // Kelemen tables, [table][cos 64][rough 32]
    int nenv;                // environment lights among the lights
    const float* corner_n;   // per-corner normals, 9 floats per triangle
    const float* corner_uv;  // per-corner uvs, 6 floats per triangle
    const int* tri_attr;     // attribute index per triangle
    int nlights;
    int nnormal;             // materials with a normal map
    const float* attr_c2o;   // camera-to-object transform per attribute, 16 floats row major
};

// Shading point at a hit (ShadingGeometry + Integrator::LocalGeometry): P the hit point,
// Ng the interpolated face-forwarded normal, N the shading normal (normal map, then the
// back-facing fix), V = -normalize(dir), (su, sv) the interpolated uv.
struct Frame { float3 P, V, N, Ng; float su, sv; int attr; };

struct RayF { float3 o; float mint; float3 d; float maxt; };

// ------------------------------------------------------------------ camera
AUR_HD RayF camera_ray(const Camera& cam, int px, int py, float j1, float j2) {
    float fovx = cam.fov;
    float fovy = ((float)cam.h / (float)cam.w) * fovx;
    float u = (float)px + j1;
    float v = (float)py + j2;
    float3 d = mk(((2.f * u - (float)cam.w) / (float)cam.w) * fovx,
                  ((-2.f * v + (float)cam.h) / (float)cam.h) * fovy, -1.f);
    RayF r;
    r.d = normalize(d);
    r.o = mk(0.f, 0.f, 0.f);
    r.mint = 0.1f;
    r.maxt = 10000000.f;
    return r;
}

// ------------------------------------------------------------------ triangle
// Exact restatement of RenderableTriangle::intersect (renderableTriangle.cpp:68-98).
// The __f*_rn intrinsics forbid FMA contraction on the device, and the host
// build uses -ffp-contract=off, so both sides round every operation the same
// way. IEEE reciprocal (__frcp_rn) equals the reference's 1.f/divisor.
#ifdef __CUDA_ARCH__
#define AUR_MUL(a, b) __fmul_rn(a, b)
#define AUR_ADD(a, b) __fadd_rn(a, b)
#define AUR_SUB(a, b) __fsub_rn(a, b)
#define AUR_RCP(a) __frcp_rn(a)
#else
#define AUR_MUL(a, b) ((a) * (b))
#define AUR_ADD(a, b) ((a) + (b))
#define AUR_SUB(a, b) ((a) - (b))
#define AUR_RCP(a) (1.f / (a))
#endif
AUR_HD float xdot(float3 a, float3 b) { return AUR_ADD(AUR_ADD(AUR_MUL(a.x, b.x), AUR_MUL(a.y, b.y)), AUR_MUL(a.z, b.z)); }
AUR_HD float3 xcross(float3 a, float3 b) {
    return mk(AUR_SUB(AUR_MUL(a.y, b.z), AUR_MUL(a.z, b.y)),
              AUR_SUB(AUR_MUL(a.z, b.x), AUR_MUL(a.x, b.z)),
              AUR_SUB(AUR_MUL(a.x, b.y), AUR_MUL(a.y, b.x)));
}
AUR_HD float3 xsub(float3 a, float3 b) { return mk(AUR_SUB(a.x, b.x), AUR_SUB(a.y, b.y), AUR_SUB(a.z, b.z)); }
// Returns true and writes t, b1 (weight of vertex 1 = u), b2 (vertex 2 = v) on a hit in [mint, maxt].
AUR_HD bool tri_intersect(float3 p1, float3 e1, float3 e2, float3 o, float3 d, float mint, float maxt,
                          float* t_out, float* b1_out, float* b2_out) {
    float3 s1 = xcross(d, e2);
    float divisor = xdot(s1, e1);
    if (divisor == 0.f) return false;
    float inv = AUR_RCP(divisor);
    float3 dd = xsub(o, p1);
    float b1 = AUR_MUL(xdot(dd, s1), inv);
    if (b1 < 0.f || b1 > 1.f) return false;
    float3 s2 = xcross(dd, e1);
    float b2 = AUR_MUL(xdot(d, s2), inv);
    if (b2 < 0.f || AUR_ADD(b1, b2) > 1.f) return false;
    float t = AUR_MUL(xdot(e2, s2), inv);
    if (t < mint || t > maxt) return false;
    *t_out = t; *b1_out = b1; *b2_out = b2;
    return true;
}

// ------------------------------------------------------------------ textures
AUR_HD int aur_floor(float x) { return (int)x - (x < 0.f && (float)(int)x != x); }   // math_utils.h floor
// texel of the uv lookup (texture2DShader: wrap to [0, 1), flip t)
AUR_HD int uv_texel_index(const Texture& t, float su, float sv) {
    float fs = su - (float)aur_floor(su);
    float ft = 1.f - (sv - (float)aur_floor(sv));
    int x = aur_floor(fs * (float)t.w);
    int y = aur_floor(ft * (float)t.h);
    if (y == t.h) y -= 1;
    if (x == t.w) x -= 1;
    x = x < 0 ? 0 : (x > t.w - 1 ? t.w - 1 : x);
    y = y < 0 ? 0 : (y > t.h - 1 ? t.h - 1 : y);
    return y * t.w + x;
}
// Texture2D::read / ::pdf with filter 0 at (s, t) (texture2D.cpp:48-72, 112-134): the texel
// floor(s w), floor(t h), no wrap and no flip (unlike the uv shader lookup)
AUR_HD int texel_index(const Texture& t, float s, float v) {
    int x = (int)floorf(s * (float)t.w), y = (int)floorf(v * (float)t.h);
    if (y == t.h) y -= 1;
    if (x == t.w) x -= 1;
    x = x < 0 ? 0 : (x > t.w - 1 ? t.w - 1 : x);
    y = y < 0 ? 0 : (y > t.h - 1 ? t.h - 1 : y);
    return y * t.w + x;
}
AUR_HD float3 texel_rgb(const ShadeScene& s, const Texture& t, int i) {
    const float* p = s.texels + t.offset + 3 * i;
    return mk(p[0], p[1], p[2]);
}

// The texels a triplanar shader blends and their weights (triplanarTextureShader.h):
// the colour shader weighs the axes by |N_obj| - 0.25 of the object-space normal, the
// float shader by |Ng| - 0.2 of the camera-space normal; the texture is read at
// (|fmod(P_obj[i+1] / scale, 1)|, |fmod(P_obj[i+2] / scale, 1)|) for each axis i of
// positive weight. Tap i (axis i) is texel idx[i] with weight w[i]; w[i] = 0 skips it.
struct Taps { int idx[3]; float w[3]; };
AUR_HD Taps triplanar_taps(const float* c2o, const Texture& t, float3 P, float3 Ng, bool float_shader) {
    const float* m = c2o;
    float w[3];
    float3 N;
    double cut;
    if (float_shader) {
        N = Ng;
        cut = 0.2;
    } else {                                           // (*cameraToObject)(Ng), a vector
        N = normalize(mk(m[0] * Ng.x + m[1] * Ng.y + m[2] * Ng.z, m[4] * Ng.x + m[5] * Ng.y + m[6] * Ng.z,
                         m[8] * Ng.x + m[9] * Ng.y + m[10] * Ng.z));
        cut = 0.25;
    }
    const float n3[3] = {N.x, N.y, N.z};
    float sum = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float a = fabsf(n3[i]);
        a = (float)((double)a - cut);                  // weights[i] -= 0.25 (0.2): a double constant
        a = a > 0.f ? a : 0.f;                         // max(weights[i], 0.f)
        w[i] = a;
        sum = sum + a;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) w[i] = w[i] / sum;
    // (*cameraToObject)(P), a point (transform.cpp:206-214), then P /= scale
    float x = m[0] * P.x + m[1] * P.y + m[2] * P.z + m[3];
    float y = m[4] * P.x + m[5] * P.y + m[6] * P.z + m[7];
    float z = m[8] * P.x + m[9] * P.y + m[10] * P.z + m[11];
    const float wp = m[12] * P.x + m[13] * P.y + m[14] * P.z + m[15];
    if (wp != 1.f) {
        const float iw = 1.f / wp;
        x = x * iw; y = y * iw; z = z * iw;
    }
    const float inv = 1.f / t.tri_scale;
    const float p3[3] = {x * inv, y * inv, z * inv};
    Taps r;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        r.idx[i] = 0;
        r.w[i] = w[i] > 0.f ? w[i] : 0.f;              // if (weights[i] > 0): NaN weights skip too
        if (!(w[i] > 0.f)) continue;
        const float ss = fabsf(fmodf(p3[(i + 1) % 3], 1.f));
        const float tt = fabsf(fmodf(p3[(i + 2) % 3], 1.f));
        r.idx[i] = texel_index(t, ss, tt);
    }
    return r;
}
// The triplanar shaders' value (out of line: rare, and its arrays stay out of the callers'
// frames); `rgb` selects the colour shader, else the float shader's red channel in .x.
static __host__ __device__ __noinline__ float3 triplanar_eval(const float* texels, Texture t, const float* c2o, float3 P,
                                                              float3 Ng, bool rgb) {
    const Taps k = triplanar_taps(c2o, t, P, Ng, !rgb);
    float3 r = mk(0.f, 0.f, 0.f);
    float rf = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (!(k.w[i] > 0.f)) continue;
        const float* p = texels + t.offset + 3 * k.idx[i];
        if (rgb) r = r + mk(p[0], p[1], p[2]) * k.w[i];
        else rf = rf + p[0] * k.w[i];
    }
    return rgb ? r : mk(rf, 0.f, 0.f);
}
// Shader<Color>::evaluate of a texture shader at a shading point
AUR_HD float3 shader_color(const ShadeScene& s, int tex, const Frame& f) {
    const Texture t = s.texs[tex];
    if (t.tri_scale == 0.f) return texel_rgb(s, t, uv_texel_index(t, f.su, f.sv));
    return triplanar_eval(s.texels, t, s.attr_c2o + (size_t)f.attr * 16, f.P, f.Ng, true);
}
// Shader<float>::evaluate: the red channel
AUR_HD float shader_float(const ShadeScene& s, int tex, const Frame& f) {
    const Texture t = s.texs[tex];
    if (t.tri_scale == 0.f) return s.texels[t.offset + 3 * uv_texel_index(t, f.su, f.sv)];
    return triplanar_eval(s.texels, t, s.attr_c2o + (size_t)f.attr * 16, f.P, f.Ng, false).x;
}

// ------------------------------------------------------------------ BRDF lobes
struct Brdf {                // an instantiated lobe: BrdfState{Brdf*, bxdfParameters*}
    int lobe;                // LobeType
    float3 color;            // Lambert albedo, CT colour, mirror / transmission colour
    float rough;             // CT roughness; LOBE_TRANSMIT: the index of refraction
};

// worldToTangent (math_utils.h:92-97): components along the UNNORMALISED frame vectors
// of coordinateSystem (tangentToWorld normalises them), as the reference computes them.
AUR_HD float3 world_to_tangent(float3 dir, float3 n) {
    float3 dpdu, dpdv;
    coordinate_system(n, &dpdu, &dpdv);
    return mk(dot(dir, dpdu), dot(dir, dpdv), dot(dir, n));
}
struct BrdfSample { float3 dir; float pdf; float3 color; float maxt; };

// `albedo * M_PI_INV` with the reference's unparenthesised #define M_PI_INV 1.f/M_PI
// (math_utils.h:26) parses as (albedo * 1.f) / M_PI, i.e. Color::operator/(float)
// with (float)M_PI: a multiply by the float reciprocal 1/(float)pi.
constexpr float kInvPiMacro = 1.f / 3.14159265358979323846f;

AUR_HD float ct_d(float rough, float cosa, float tana) {        // cookTorrance.cpp:40-45
    float rough2 = fmaxf(0.001f, rough * rough);
    float e = xexpf(-(tana * tana) / rough2);
    float div = (float)((double)rough2 * 3.141592653589793 * (double)xpowf(cosa, 3.f));   // rough2 * M_PI in double
    return e / div;
}

AUR_HD BrdfSample brdf_sample(const Brdf& b, float3 V, float3 N, float r1, float r2) {
    BrdfSample s;
    if (b.lobe == LOBE_MATTE) {                                      // lambert.h:44-62
        float3 dir = sample_hemisphere_uniform(r1, r2);
        s.dir = normalize(tangent_to_world(dir, N));
        s.pdf = kInvPi * 0.5f;
        s.color = b.color * kInvPiMacro;
        s.maxt = 1000000.f;
        return s;
    }
    if (b.lobe == LOBE_SPEC) {                                       // cookTorrance.cpp:47-99
        float z = xcosf(xatanf(b.rough * sqrtf((float)(-log(1.0 - (double)r1)))));
        float r = sqrtf(fmaxf(0.f, 1.f - z * z));
        float phi = two_pi_times(r2);
        float3 dir = normalize(mk(r * xcosf(phi), r * xsinf(phi), z));
        float3 H = normalize(tangent_to_world(dir, N));
        float vdoth = dot(V, H);
        float3 L = normalize((H * 2.f) * vdoth - V);
        float ndoth = dot(N, H);
        s.color = mk(0.f, 0.f, 0.f);
        s.pdf = 1.f;
        if (vdoth > 0.0001f) {
            float tana = (ndoth > 0.999f) ? 0.f : xtanf(xacosf(ndoth));
            float D = ct_d(b.rough, ndoth, tana);
            D = fminf(D, 1000.f);
            s.pdf = D / (4.f * vdoth);
            s.color = cdiv(b.color * D, 4.f * vdoth * vdoth);
            if (s.pdf > 100000.f) { s.pdf *= 0.01f; s.color *= 0.01f; }
        }
        s.dir = L;
        s.maxt = 10000000.f;
        return s;
    }
    if (b.lobe == LOBE_MIRROR) {                                     // specMirror.cpp:35-40
        const float3 vt = world_to_tangent(V, N);
        s.dir = normalize(tangent_to_world(mk(-vt.x, -vt.y, vt.z), N));
        s.pdf = 1.f;
        s.color = b.color;
        s.maxt = 100000000.f;
        return s;
    }
    if (b.lobe == LOBE_TRANSMIT) {                                   // specTransmit.cpp:33-56
        const float costheta = dot(N, V);
        float ei = 1.f, et = b.rough;
        if (costheta < 0.f) { ei = b.rough; et = 1.f; }
        const float sini2 = fmaxf(0.f, 1.f - costheta * costheta);
        const float eta = ei / et;
        const float sint2 = eta * eta * sini2;
        if (sint2 >= 1.f) {   // total internal reflection: Sample3D(Ray(), 0, Color(0)) ends the path
            s.dir = mk(0.f, 0.f, 0.f); s.pdf = 0.f; s.color = mk(0.f, 0.f, 0.f); s.maxt = 0.f;
            return s;
        }
        float cost = sqrtf(fmaxf(0.f, 1.f - sint2));
        if (costheta > 0.f) cost = -cost;
        const float3 vl = world_to_tangent(V, N);
        s.dir = normalize(tangent_to_world(mk(eta * -vl.x, eta * -vl.y, cost), N));
        s.pdf = 1.f;
        s.color = b.color;
        s.maxt = 10000000.f;
        return s;
    }
    // constant (light geometry): Sample3D() -> pdf 0 ends the path (constant.cpp:23-25)
    s.dir = mk(0.f, 1.f, 0.f); s.pdf = 0.f; s.color = mk(0.f, 0.f, 0.f); s.maxt = 0.f;
    return s;
}

AUR_HD float3 brdf_eval(const Brdf& b, float3 L, float3 V, float3 N) {
    if (b.lobe == LOBE_MATTE) {                                      // lambert.h:68-76
        return dot(L, N) > 0.f ? b.color * kInvPiMacro : mk(0.f, 0.f, 0.f);
    }
    if (b.lobe == LOBE_SPEC) {                                       // cookTorrance.cpp:125-144
        float3 H = normalize(L + V);
        float vdoth = dot(V, H), vdotn = dot(V, N), ndoth = dot(H, N), ldotn = dot(L, N);
        float r2 = b.rough * b.rough;
        float ta = xtanf(xacosf(ndoth));
        float D = (float)((1.f / ((double)r2 * 3.141592653589793 * (double)xpowf(ndoth, 3.f))) *
                          (double)xexpf(-(ta * ta) / r2));
        if (vdoth <= 0.001f || ldotn <= 0.001f || vdotn <= 0.001f || isnan(D)) return mk(0.f, 0.f, 0.f);
        return cdiv(b.color * D, (float)(4.0 * vdoth * vdoth));
    }
    return mk(0.f, 0.f, 0.f);
}

AUR_HD float brdf_pdf(const Brdf& b, float3 L, float3 V, float3 N) {
    if (b.lobe == LOBE_MATTE) return kInvPi * 0.5f;                  // lambert.h:78-80
    if (b.lobe == LOBE_SPEC) {                                       // cookTorrance.cpp:101-117
        float3 H = normalize(L + V);
        float vdoth = dot(V, H), ndoth = dot(N, H);
        float D = ct_d(b.rough, ndoth, xtanf(xacosf(ndoth)));
        if (isnan(D)) D = 0.f;
        return D / (4.f * vdoth);
    }
    return 0.f;
}

// Kelemen directional-albedo lookup (kelemenMaterial.cpp:180-212). The
// reference's roughnessB = max(roughnessA+1, 31) is kept (it always reads the
// last roughness column); the column index is clamped to the table so that
// roughness 1 stays in bounds (the reference reads past the table there).
AUR_HD float kelemen_albedo(const float* table, float costheta, float roughness) {
    int i = aur_floor(costheta * (kAlbedoCos - 1));
    int ra = aur_floor(roughness * (kAlbedoRough - 1));
    int rb = ra + 1 > kAlbedoRough - 1 ? ra + 1 : kAlbedoRough - 1;
    i = i < 0 ? 0 : (i > kAlbedoCos - 1 ? kAlbedoCos - 1 : i);
    ra = ra < 0 ? 0 : (ra > kAlbedoRough - 1 ? kAlbedoRough - 1 : ra);
    rb = rb > kAlbedoRough - 1 ? kAlbedoRough - 1 : rb;
    int i1 = i + 1 < kAlbedoCos - 1 ? i + 1 : kAlbedoCos - 1;
    float va = table[i * kAlbedoRough + ra];
    float vb = table[i1 * kAlbedoRough + ra];
    float mixc = costheta * (kAlbedoCos - 1) - (float)i;
    float resA = (float)((1. - mixc) * va + (double)(mixc * vb));
    va = table[i * kAlbedoRough + rb];
    vb = table[i1 * kAlbedoRough + rb];
    float resB = (float)((1. - mixc) * va + (double)(mixc * vb));
    float rmix = roughness * (kAlbedoRough - 1) - (float)ra;
    return (float)((1. - rmix) * resA + (double)(rmix * resB));
}

// roughness * (1 - CAUSTIC_BLUR) + CAUSTIC_BLUR with the reference's double constants
AUR_HD float caustic_blur(float r) { return (float)((double)r * (1.0 - 0.2) + 0.2); }

// The Lambert lobe of a matte material (shading/materials/matteMaterial.h): its diffuse
// colour or texture.
AUR_HD Brdf matte_brdf(const ShadeScene& s, const Material& m, const Frame& f) {
    Brdf b;
    b.lobe = LOBE_MATTE;
    b.color = m.diff_tex >= 0 ? shader_color(s, m.diff_tex, f) : m.diff;
    b.rough = 0.f;
    return b;
}

// Material::getBrdf for every supported material at shading point `f`. `lobe_u` is the
// vertex's lobe-choice random number.
AUR_HD Brdf get_brdf(const ShadeScene& s, int mat_id, const Frame& f, bool matte_path, float lobe_u) {
    const float3 V = f.V, N = f.N;
    Material m = s.mats[mat_id];
    Brdf b;
    if (m.type == MAT_MATTE) return matte_brdf(s, m, f);
    if (m.type == MAT_KELEMEN || m.type == MAT_COOKTORRANCE) {
        float rough = m.rough_tex >= 0 ? shader_float(s, m.rough_tex, f) : m.rough;
        if (matte_path) rough = caustic_blur(rough);
        b.lobe = LOBE_SPEC;
        b.color = m.spec_tex >= 0 ? shader_color(s, m.spec_tex, f) : m.spec;
        b.rough = rough;
        if (m.type == MAT_KELEMEN && m.refl < 1.f) {
            float c = dot(N, V);
            c = c < 0.f ? 0.f : (c > 1.f ? 1.f : c);
            float albedo = kelemen_albedo(s.albedo + (size_t)m.table * (kAlbedoCos * kAlbedoRough), c, rough);
            if (lobe_u > albedo) {
                b.lobe = LOBE_MATTE;
                b.color = m.diff_tex >= 0 ? shader_color(s, m.diff_tex, f) : m.diff;
                b.rough = 0.f;
            }
        }
        return b;
    }
    if (m.type == MAT_METAL) {                                         // metalMaterial.cpp:32-62
        float costheta = dot(V, N);
        float3 sc = mk(schlick(costheta, m.spec.x), schlick(costheta, m.spec.y), schlick(costheta, m.spec.z));
        float rough = lobe_u > m.mix ? m.rough : m.rough_b;
        if (matte_path) rough = caustic_blur(rough);
        b.lobe = LOBE_SPEC;
        b.color = sc * m.gain;
        b.rough = rough;
        return b;
    }
    if (m.type == MAT_GLASS) {                                         // glassMaterial.cpp:33-56
        b.rough = 0.f;
        b.lobe = LOBE_MIRROR;
        b.color = m.spec;
        if (m.refl == 1.f) return b;
        float costheta = (float)((double)dot(V, N) * 0.5);            // the reference halves V.N
        if (costheta < 0.f) costheta = -costheta;
        const float albedo = schlick(costheta, m.refl);
        if (lobe_u > albedo) {
            b.lobe = LOBE_TRANSMIT;
            b.color = m.diff;                                          // transmitColor
            b.rough = m.ior;
        }
        return b;
    }
    b.lobe = LOBE_CONSTANT;
    b.color = mk(0.f, 0.f, 0.f);
    b.rough = 0.f;
    return b;
}

// ------------------------------------------------------------------ lights
struct LightSample { float3 dir; float maxt; float pdf; float3 color; };

// ---- environment light (InfiniteAreaLight, geometry/infiniteAreaLight.cpp:35-106)
AUR_HD float3 xform_vector(const float* m, float3 v) {                  // transform.cpp:222-228
    return mk(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z,
              m[8] * v.x + m[9] * v.y + m[10] * v.z);
}
AUR_HD float3 env_texel(const ShadeScene& sh, int tex, float s, float v) {
    const Texture t = sh.texs[tex];
    const float* p = sh.texels + t.offset + 3 * texel_index(t, s, v);
    return mk(p[0], p[1], p[2]);
}
// the map's pdf: texel luminance (r + g + b) / 3 over its mean (Texture2D::initPdf)
AUR_HD float env_texel_pdf(const ShadeScene& sh, const Light& l, float s, float v) {
    const float3 c = env_texel(sh, l.tex, s, v);
    return ((c.x + c.y + c.z) / 3.f) / l.pdf_norm;
}
// map coordinates of a camera-space direction (InfiniteAreaLight::eval / ::pdf)
AUR_HD void env_uv(const Light& l, float3 dir_cam, float* u, float* v) {
    const float3 dir = xform_vector(l.m, dir_cam);
    *v = (float)(0.5 * (double)(1.f - dir.y));
    float uu = (float)((double)xatan2f(dir.z, dir.x) / 6.283185307179586);   // / (M_PI * 2.f) in double
    if (uu < 0.f) uu += 1.f;
    *u = uu;
}
// radiance arriving along camera-space direction `dir` from a light (Light::eval): the
// square and sphere lights are constant, the environment reads its map
// (the environment's paths are kept out of line: inlined, they raise the register count of
// every shading kernel, with or without an environment in the scene)
// (their arguments are global pointers and values: an address of a local copy or of a
// kernel parameter would force that into local memory)
static __host__ __device__ __noinline__ float3 env_map_eval(const Texture* texs, const float* texels, const Light* l,
                                                            float3 dir) {
    ShadeScene sh;
    sh.texs = texs;
    sh.texels = texels;
    float u, v;
    env_uv(*l, dir, &u, &v);
    return env_texel(sh, l->tex, u, v) * l->escale;
}
// `l` must live in global memory (a reference into ShadeScene::lights)
AUR_HD float3 light_eval(const ShadeScene& sh, const Light& l, float3 dir) {
    if (l.type != LIGHT_ENV || l.tex < 0) return l.le;
    return env_map_eval(sh.texs, sh.texels, &l, dir);
}
// every environment light's radiance along `dir` (camera-ray and mirror-ray misses,
// integrator.cpp:262-288)
static __host__ __device__ __noinline__ float3 env_radiance_of(const Light* lights, int n, const Texture* texs,
                                                               const float* texels, float3 dir) {
    float3 r = mk(0.f, 0.f, 0.f);
    for (int i = 0; i < n; ++i) {
        const Light* l = &lights[i];
        if (l->type != LIGHT_ENV) continue;
        r += l->tex < 0 ? l->le : env_map_eval(texs, texels, l, dir);
    }
    return r;
}
AUR_HD float3 env_radiance(const ShadeScene& sh, float3 dir) {
    return env_radiance_of(sh.lights, sh.nlights, sh.texs, sh.texels, dir);
}

AUR_HD bool light_visible(const Light& l, float3 P, float3 N) {       // squareLight.h:99-110
    if (l.type == LIGHT_ENV) return true;
    if (l.type == LIGHT_SQUARE) {
        for (int i = 0; i < 4; ++i)
            if (dot(l.p[i] - P, N) > 0.f) return true;
        return false;
    }
    return dot(l.center - P, N) > -l.radius;
}

AUR_HD float3 xform_point(const float* m, float3 p) {                   // transform.cpp:196-204
    float xp = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
    float yp = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
    float zp = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
    float wp = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
    if (wp == 1.f) return mk(xp, yp, zp);
    return cdiv(mk(xp, yp, zp), wp);
}

// Sphere: distance along a unit ray to the near surface (tangent point if it misses).
AUR_HD float sphere_hit(float3 c, float radius, float3 o, float3 d, float mint, float* t_out) {
    float3 oc = o - c;
    float b = dot(oc, d);
    float cc = dot(oc, oc) - radius * radius;
    float disc = b * b - cc;
    if (disc < 0.f) { *t_out = -b; return false; }
    float sq = sqrtf(disc);
    float t = -b - sq;
    if (t < mint) t = -b + sq;
    *t_out = t;
    return t >= mint;
}
AUR_HD float sphere_cone_cos(const Light& l, float3 P) {
    float3 wc = l.center - P;
    float dc2 = dot(wc, wc);
    float s2 = l.radius * l.radius / dc2;
    return sqrtf(fmaxf(0.f, 1.f - s2));
}

static __host__ __device__ __noinline__ LightSample env_light_sample(const Texture* texs, const float* texels,
                                                                    const Light* lp, float3 N, float u1, float u2) {
    ShadeScene sh;
    sh.texs = texs;
    sh.texels = texels;
    const Light& l = *lp;
    LightSample s;
    {                                                                    // infiniteAreaLight.cpp:35-61
        float3 dirw;
        float pdf;
        if (l.tex >= 0) {   // a uniform direction on the sphere, weighted by the map's pdf at (u1, u2)
            const float vy = 1.f - 2.f * u2;
            const float r = sqrtf(fmaxf(0.f, 1.f - vy * vy));
            const float phi = two_pi_times(u1);
            dirw = xform_vector(l.minv, mk(r * xcosf(phi), vy, r * xsinf(phi)));
            pdf = env_texel_pdf(sh, l, u1, u2);
        } else {
            pdf = 2.f;
            dirw = tangent_to_world(sample_hemisphere_uniform(u1, u2), N);
        }
        s.dir = normalize(dirw);
        s.maxt = 1000000.f;
        s.pdf = (float)((double)pdf / 12.566370614359172);               // pdf / (M_PI * 4.)
        s.color = l.tex < 0 ? l.le : env_map_eval(texs, texels, lp, s.dir);
        return s;
    }
}

AUR_HD LightSample light_sample(const ShadeScene& sh, const Light& l, float3 P, float3 N, float u1, float u2) {
    LightSample s;
    if (l.type == LIGHT_ENV) return env_light_sample(sh.texs, sh.texels, &l, N, u1, u2);
    if (l.type == LIGHT_SQUARE) {                                        // squareLight.h:57-82
        float3 lp = mk((float)(((double)u1 - 0.5) * l.xs * 2.0), (float)(((double)u2 - 0.5) * l.ys * 2.0), 0.f);
        lp = xform_point(l.m, lp);
        float3 dir = lp - P;
        float len = length(dir);
        dir = normalize(dir);
        s.dir = dir;
        s.maxt = (float)((double)len - 0.005);                  // sampleLength - RAY_BIAS*10 (double)
        float d = dot(l.n, -dir);
        if (!(d > 0.f)) d = 0.f;
        s.color = l.le;
        s.pdf = d == 0.f ? 0.f : (float)((double)(len * len) / ((double)(d * l.xs * l.ys) * 4.0));
        return s;
    }
    float3 wc = l.center - P;                                            // sphere (extension)
    float dc = length(wc);
    s.color = l.le;
    if (dc <= l.radius) { s.dir = mk(0.f, 1.f, 0.f); s.maxt = 0.f; s.pdf = 0.f; return s; }
    float3 w = cdiv(wc, dc);
    float cosmax = sphere_cone_cos(l, P);
    float cost = (1.f - u1) + u1 * cosmax;
    float sint = sqrtf(fmaxf(0.f, 1.f - cost * cost));
    float phi = two_pi_times(u2);
    float3 dir = normalize(tangent_to_world(mk(sint * xcosf(phi), sint * xsinf(phi), cost), w));
    float t;
    sphere_hit(l.center, l.radius, P, dir, 0.f, &t);
    s.dir = dir;
    s.maxt = t - kRayBias * 10.f;
    float solid = 2.f * kPi * (1.f - cosmax);
    s.pdf = solid > 0.f ? 1.f / solid : 0.f;
    return s;
}

// SquareLight::pdf (squareLight.h:88-97): hits the two light triangles, shortens
// the ray to the light and returns the solid-angle pdf (two-sided, as in the reference).
static __host__ __device__ __noinline__ float env_light_pdf(const Texture* texs, const float* texels, const Light* lp,
                                                            float3 d) {
    // infiniteAreaLight.cpp:82-106, hemisphere domain
    const Light& l = *lp;
    if (l.tex < 0) return (float)(1.0 / 6.283185307179586);             // 1.f / (M_PI * 2.f)
    ShadeScene sh;
    sh.texs = texs;
    sh.texels = texels;
    float u, v;
    env_uv(l, d, &u, &v);
    return (float)((double)env_texel_pdf(sh, l, u, v) / 6.283185307179586);
}

AUR_HD float light_pdf(const ShadeScene& sh, const Light& l, float3 o, float3 d, float mint, float* maxt) {
    if (l.type == LIGHT_ENV) return env_light_pdf(sh.texs, sh.texels, &l, d);
    if (l.type == LIGHT_SQUARE) {
        float t, b1, b2;
        bool hit = tri_intersect(l.p[0], xsub(l.p[1], l.p[0]), xsub(l.p[3], l.p[0]), o, d, mint, *maxt, &t, &b1, &b2);
        if (!hit) hit = tri_intersect(l.p[2], xsub(l.p[1], l.p[2]), xsub(l.p[3], l.p[2]), o, d, mint, *maxt, &t, &b1, &b2);
        if (!hit) return 0.f;
        *maxt = t;
        float dd = dot(l.n, normalize(d));
        dd = dd > 0.f ? dd : (dd < 0.f ? -dd : 0.f);
        float pdf = (float)((double)(t * t) / ((double)(dd * l.xs * l.ys) * 4.0));
        *maxt = (float)((double)*maxt - 0.005);
        return pdf;
    }
    float t;
    if (!sphere_hit(l.center, l.radius, o, d, mint, &t) || t > *maxt) return 0.f;
    float3 wc = l.center - o;
    if (dot(wc, wc) <= l.radius * l.radius) return 0.f;
    *maxt = t - kRayBias * 10.f;
    float solid = 2.f * kPi * (1.f - sphere_cone_cos(l, o));
    return solid > 0.f ? 1.f / solid : 0.f;
}

AUR_HD float power_heuristic(float f, float g) { return (f * f) / (f * f + g * g); }  // integrator.cpp:28-31

// Material::runNormalShader (material.cpp:27-40): the map colour read as a tangent-space
// vector around Ng (tangentToWorld), normalised unless zero; out of line, as only scenes
// with normal maps take it (arguments by value or global pointer, so that nothing of the
// caller's moves to local memory).
static __host__ __device__ __noinline__ float3 normal_map(const Material* mats, const Texture* texs, const float* texels,
                                                          const float* attr_c2o, int mat, float3 P, float3 Ng,
                                                          float su, float sv, int attr) {
    const Material& m = mats[mat];
    float3 c = m.norm;
    if (m.norm_tex != kNormalConst) {
        ShadeScene s;
        s.texs = texs;
        s.texels = texels;
        s.attr_c2o = attr_c2o;
        Frame f;
        f.P = P; f.Ng = Ng; f.su = su; f.sv = sv; f.attr = attr;
        c = shader_color(s, m.norm_tex, f);
    }
    const float3 ns = tangent_to_world(c, Ng);
    if (!(ns.x != 0.f || ns.y != 0.f || ns.z != 0.f)) return Ng;
    return normalize(ns);
}

// Shading frame at a hit (embreeAccelerator.cpp:54-90 + integrator.cpp:132-150):
// interpolated, face-forwarded, normalised normal; the normal map; V = -normalize(dir);
// back-facing fix.
AUR_HD Frame hit_frame(const ShadeScene& s, int prim, float t, float u, float v, float3 o, float3 d, bool need_uv) {
    Frame f;
    const float* n = s.corner_n + (size_t)prim * 9;
    float w = (float)(1.0 - u - v);      // 1. - u - v in double (embreeAccelerator.cpp:54)
    float3 nn = mk(w * n[0] + u * n[3] + v * n[6],
                   w * n[1] + u * n[4] + v * n[7],
                   w * n[2] + u * n[5] + v * n[8]);
    if (dot(nn, d) > 0.f) nn *= -1.f;
    f.Ng = normalize(nn);
    f.N = f.Ng;
    f.P = o + d * t;
    f.attr = s.tri_attr[prim];
    f.su = f.sv = 0.f;
    if (need_uv && s.corner_uv) {
        const float* uv = s.corner_uv + (size_t)prim * 6;
        f.su = w * uv[0] + u * uv[2] + v * uv[4];
        f.sv = w * uv[1] + u * uv[3] + v * uv[5];
    }
    if (s.nnormal) {
        const int mat = s.attrs[f.attr].material;
        if (s.mats[mat].norm_tex != kNormalNone)
            f.N = normal_map(s.mats, s.texs, s.texels, s.attr_c2o, mat, f.P, f.Ng, f.su, f.sv, f.attr);
    }
    f.V = -normalize(d);
    if (dot(f.V, f.N) <= 0.f) {
        float3 tmp = cross(f.N, f.V);
        f.N = normalize(cross(f.V, tmp));
    }
    return f;
}

}  // namespace aur
