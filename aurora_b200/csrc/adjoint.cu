// adjoint.cu — path-replay backpropagation (Vicini, Speierer, Jakob, "Path Replay
// Backpropagation", SIGGRAPH 2021) for the Aurora path loop. No reference counterpart.
//
// Given dLoss/dFilm, every pixel replays its spp camera paths with the same
// counter-based random numbers as the forward renderer:
//   pass 1  the forward estimator of Integrator::integrateCameraSample
//           (integrator.cpp:152-300) with identical arithmetic; it records each
//           vertex's hit (prim, t, u, v) and the visibility of its next-event
//           rays in thread-local arrays, and yields the path radiance Lo;
//   pass 2  re-shades the recorded vertices (no ray tracing) and accumulates
//             dL/dtheta += delta . [ T_k dD_k/dtheta + L_after,k (dw_k/dtheta) / w_k ]
//           where D_k is the vertex's next-event estimate, w_k = f cos / pdf its
//           continuation weight, T_k the throughput and L_after,k = Lo minus the
//           radiance collected up to and including vertex k.
// Sampling decisions are detached: pdfs, MIS weights, the Kelemen/metal lobe
// choice, roulette probabilities and the firefly clamp factor are constants of
// the derivative (the discrete choices and the clamp make the estimator biased;
// the continuous parts are unbiased). Memory: O(pixels) — nothing is stored per path.
//
// Parameters: per material (diffuse rgb, roughness) and all texels. Diffuse
// colour drives Lambert lobes (matte, Kelemen's diffuse lobe); roughness drives
// Cook-Torrance lobes (Kelemen, Cook-Torrance, metal roughnessA); a diffuse
// texture receives the diffuse gradient of the texel the lookup used. Gradients
// are summed in FP32 with TwoSum-compensated atomics (shared, then global).
#define AUR_MATH_OUT_OF_LINE 1
#include "aur_capi_internal.h"

namespace aur {
namespace {

constexpr int kAdjBlock = 128;
constexpr int kAdjMaxDepth = 16;
constexpr int kAdjMaxMat = 64;

// hit record of one vertex: (t, u, v, prim | visibility of its next-event rays << 30)
__device__ __forceinline__ float4 pack_rec(const Hit& h, uint32_t vis) {
    return make_float4(h.t, h.u, h.v, __int_as_float(h.prim | (int)(vis << 30)));
}

// atomic add with the exact rounding error of that addition sent to a compensation slot
__device__ __forceinline__ void comp_add(float* sum, float* comp, float x) {
    if (x == 0.f) return;
    const float old = atomicAdd(sum, x);
    const float t = old + x;                        // what the atomic stored
    const float bp = t - old;
    const float err = (old - (t - bp)) + (x - bp);  // TwoSum(old, x) error
    if (err != 0.f) atomicAdd(comp, err);
}

// TwoSum step of a thread-local compensated sum
__device__ __forceinline__ void two_sum_add(float& sum, float& comp, float x) {
    const float t = sum + x;
    const float bp = t - sum;
    comp += (sum - (t - bp)) + (x - bp);
    sum = t;
}

// Per-thread compensated accumulators of the per-material gradients (diffuse rgb,
// roughness) of the two most recently touched materials. A pixel's paths mostly revisit
// the same materials, so the block's shared sums see one flush per eviction instead of
// one atomic per vertex (the megakernel: 11% faster; the replay kernel, one path per
// thread, is faster with DirectAcc). Register-resident: slots resolved by selects.
struct MatCache {
    int tag0 = -1, tag1 = -1;
    float s0[4] = {0.f, 0.f, 0.f, 0.f}, c0[4] = {0.f, 0.f, 0.f, 0.f};
    float s1[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};

    __device__ __forceinline__ static void flush_slot(int tag, const float* s, const float* c, float* s_g, float* s_c) {
        if (tag < 0) return;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (s[q] != 0.f) comp_add(&s_g[4 * tag + q], &s_c[4 * tag + q], s[q]);
            if (c[q] != 0.f) comp_add(&s_g[4 * tag + q], &s_c[4 * tag + q], c[q]);
        }
    }
    __device__ __forceinline__ void flush(float* s_g, float* s_c) {
        flush_slot(tag0, s0, c0, s_g, s_c);
        flush_slot(tag1, s1, c1, s_g, s_c);
        tag0 = tag1 = -1;
    }
    // makes `mat` the tag of slot 0 (evicting slot 1 to the shared sums if needed)
    __device__ __forceinline__ bool slot0(int mat, float* s_g, float* s_c) {
        if (tag0 == mat) return true;
        if (tag1 == mat) return false;
        flush_slot(tag1, s1, c1, s_g, s_c);
        tag1 = tag0;
#pragma unroll
        for (int q = 0; q < 4; ++q) { s1[q] = s0[q]; c1[q] = c0[q]; s0[q] = 0.f; c0[q] = 0.f; }
        tag0 = mat;
        return true;
    }
    template <int Q>
    __device__ __forceinline__ void add(int mat, float x, float* s_g, float* s_c) {
        if (x == 0.f) return;
        if (slot0(mat, s_g, s_c)) two_sum_add(s0[Q], c0[Q], x);
        else two_sum_add(s1[Q], c1[Q], x);
    }
    __device__ __forceinline__ void add3(int mat, float3 v, float* s_g, float* s_c) {
        if (v.x == 0.f && v.y == 0.f && v.z == 0.f) return;
        if (slot0(mat, s_g, s_c)) { two_sum_add(s0[0], c0[0], v.x); two_sum_add(s0[1], c0[1], v.y); two_sum_add(s0[2], c0[2], v.z); }
        else { two_sum_add(s1[0], c1[0], v.x); two_sum_add(s1[1], c1[1], v.y); two_sum_add(s1[2], c1[2], v.z); }
    }
};

// Accumulator that adds every contribution to the block's shared sums at once.
struct DirectAcc {
    template <int Q>
    __device__ __forceinline__ void add(int mat, float x, float* s_g, float* s_c) {
        if (x != 0.f) comp_add(&s_g[4 * mat + Q], &s_c[4 * mat + Q], x);
    }
    __device__ __forceinline__ void add3(int mat, float3 v, float* s_g, float* s_c) {
        add<0>(mat, v.x, s_g, s_c);
        add<1>(mat, v.y, s_g, s_c);
        add<2>(mat, v.z, s_g, s_c);
    }
    __device__ __forceinline__ void flush(float*, float*) {}
};

// ln D derivative w.r.t. roughness r of the Beckmann term, with tan^2(alpha) given
// and the reference's max(0.001, r^2) floor (eval uses r^2 unfloored).
__device__ __forceinline__ float dlnD_dr(float r, float tan2, bool floored) {
    const float r2 = r * r;
    if (floored && r2 <= 0.001f) return 0.f;
    return 2.f * tan2 / (r2 * r) - 2.f / r;
}
__device__ __forceinline__ float tan2_of(float ndoth) {
    const float t = xtanf(xacosf(ndoth));
    return t * t;
}

// d ln f / d roughness of a Cook-Torrance sample (cookTorrance.cpp:47-99): the sampled
// half vector is normalize(L + V); a clamped D (>= 1000) or the 0.001 floor on r^2
// makes the sample's colour independent of roughness.
__device__ __forceinline__ float sample_dlnD(const Brdf& b, const Frame& f, const BrdfSample& bs) {
    const float3 H = normalize(bs.dir + f.V);
    const float ndoth = dot(f.N, H);
    const float tana = ndoth > 0.999f ? 0.f : xtanf(xacosf(ndoth));
    if (ct_d(b.rough, ndoth, tana) >= 1000.f) return 0.f;
    return dlnD_dr(b.rough, tana * tana, true);
}

// Next-event estimation of one vertex (integrateDirect with integrateDirectLight /
// integrateDirectMIS). kTrace: traces the shadow rays and records their visibility
// in *vis; otherwise replays `vis`. With kGrad it also returns dD/dtheta of the lobe's
// parameter: per channel d/d(diffuse_c) for a Lambert lobe, d/d(roughness_eff) for a
// Cook-Torrance lobe (replicated in all channels).
template <bool kTrace, bool kGrad>
__device__ __forceinline__ float3 direct(const DevScene& sc, const Frame& f, const Brdf& brdf, const PathRng& rng,
                                         int vtx, RayCounts& rc, uint32_t* vis, float3* dD) {
    float3 res = mk(0.f, 0.f, 0.f), dres = res;
    if (kGrad) *dD = res;
    if (brdf.lobe != LOBE_MATTE && brdf.lobe != LOBE_SPEC) return res;
    int nvis;
    const int li = pick_visible_light(sc.sh, f.P, f.N, rng.u(vertex_dim(vtx, kDimLightPick)), &nvis);
    if (li < 0) return res;
    const Light& L = sc.sh.lights[li];   // global: the env paths take its address
    const LightSample ls = light_sample(sc.sh, L, f.P, f.N, rng.u(vertex_dim(vtx, kDimLightSample)),
                                        rng.u(vertex_dim(vtx, kDimLightSample + 1)));
    float cost = dot(f.N, ls.dir);
    if (brdf.lobe == LOBE_MATTE) {
        if (cost >= 0.f && ls.pdf > 0.f) {
            bool open;
            if (kTrace) { ++rc.shadow; open = !bvh_occluded(sc.nodes, sc.tris, f.P, ls.dir, kRayBias, ls.maxt, rc.shadow_work); if (open) *vis |= 1u; }
            else open = (*vis & 1u) != 0;
            if (open) {
                res += cdiv((ls.color * brdf_eval(brdf, ls.dir, f.V, f.N)) * cost, ls.pdf);
                if (kGrad && dot(ls.dir, f.N) > 0.f) dres += cdiv((ls.color * kInvPiMacro) * cost, ls.pdf);
            }
        }
    } else {
        if (cost > 0.f && ls.pdf > 0.f) {
            const float bp = brdf_pdf(brdf, ls.dir, f.V, f.N);
            if (bp > 0.f) {
                bool open;
                if (kTrace) { ++rc.shadow; open = !bvh_occluded(sc.nodes, sc.tris, f.P, ls.dir, kRayBias, ls.maxt, rc.shadow_work); if (open) *vis |= 1u; }
                else open = (*vis & 1u) != 0;
                if (open) {
                    const float w = power_heuristic(ls.pdf, bp);
                    const float3 c0 = cdiv(((ls.color * w) * brdf_eval(brdf, ls.dir, f.V, f.N)) * cost, ls.pdf);
                    res += c0;
                    if (kGrad) {
                        const float3 H = normalize(ls.dir + f.V);
                        dres += c0 * dlnD_dr(brdf.rough, tan2_of(dot(H, f.N)), false);
                    }
                }
            }
        }
        const BrdfSample bs = brdf_sample(brdf, f.V, f.N, rng.u(vertex_dim(vtx, kDimMisBrdf)),
                                          rng.u(vertex_dim(vtx, kDimMisBrdf + 1)));
        cost = dot(f.N, bs.dir);
        if (cost > 0.f) {
            float maxt = bs.maxt;
            const float lp = light_pdf(sc.sh, L, f.P, bs.dir, kRayBias, &maxt);
            if (lp > 0.f && bs.pdf > 0.f) {
                bool open;
                if (kTrace) { ++rc.shadow; open = !bvh_occluded(sc.nodes, sc.tris, f.P, bs.dir, kRayBias, maxt, rc.shadow_work); if (open) *vis |= 2u; }
                else open = (*vis & 2u) != 0;
                if (open) {
                    const float w = power_heuristic(bs.pdf, lp);
                    const float3 c1 = cdiv(((bs.color * w) * light_eval(sc.sh, L, bs.dir)) * cost, bs.pdf);
                    res += c1;
                    if (kGrad) dres += c1 * sample_dlnD(brdf, f, bs);
                }
            }
        }
    }
    if (kGrad) *dD = dres * (float)nvis;
    return res * (float)nvis;
}

// d A / d roughness of the Kelemen directional-albedo lookup (kelemen_albedo): the
// lookup is linear in roughness * 31 between the two columns it reads.
__device__ __forceinline__ float kelemen_dalbedo_dr(const float* table, float costheta, float roughness) {
    int i = aur_floor(costheta * (kAlbedoCos - 1));
    int ra = aur_floor(roughness * (kAlbedoRough - 1));
    int rb = ra + 1 > kAlbedoRough - 1 ? ra + 1 : kAlbedoRough - 1;
    i = i < 0 ? 0 : (i > kAlbedoCos - 1 ? kAlbedoCos - 1 : i);
    ra = ra < 0 ? 0 : (ra > kAlbedoRough - 1 ? kAlbedoRough - 1 : ra);
    rb = rb > kAlbedoRough - 1 ? kAlbedoRough - 1 : rb;
    const int i1 = i + 1 < kAlbedoCos - 1 ? i + 1 : kAlbedoCos - 1;
    const float mixc = costheta * (kAlbedoCos - 1) - (float)i;
    const float resA = (1.f - mixc) * table[i * kAlbedoRough + ra] + mixc * table[i1 * kAlbedoRough + ra];
    const float resB = (1.f - mixc) * table[i * kAlbedoRough + rb] + mixc * table[i1 * kAlbedoRough + rb];
    return (resB - resA) * (float)(kAlbedoRough - 1);
}

// Score-function factor d ln P(chosen lobe) / d roughness of Kelemen's lobe choice
// (kelemenMaterial.cpp:236-253): P(spec) = min(1, A(cos, r_eff)), P(diffuse) = 1 - A.
__device__ __forceinline__ float kelemen_score(const ShadeScene& sh, const Material& m, const Frame& f, const Brdf& b,
                                               bool matte) {
    float r = m.rough;
    if (matte) r = caustic_blur(r);
    float c = dot(f.N, f.V);
    c = c < 0.f ? 0.f : (c > 1.f ? 1.f : c);
    const float* table = sh.albedo + (size_t)m.table * (kAlbedoCos * kAlbedoRough);
    const float A = kelemen_albedo(table, c, r);
    const float dA = kelemen_dalbedo_dr(table, c, r) * (matte ? (float)(1.0 - 0.2) : 1.f);
    if (b.lobe == LOBE_SPEC) return A < 1.f && A > 0.f ? dA / A : 0.f;
    return A < 1.f ? -dA / (1.f - A) : 0.f;
}

// Which parameter a vertex's lobe depends on.
struct ParamRef {
    int kind;        // 0 none, 1 diffuse colour of material `index`, 2 texels `taps`, 3 roughness
    int index;
    float dr;        // roughness: d r_eff / d r (caustic blur on matte paths)
    Taps taps;       // kind 2: texel blocks (3 floats each, index from the texel array start) and
                     // the weights the shader blends them with (1 for the uv lookup; 0 = unused)
};

__device__ __forceinline__ ParamRef param_of(const ShadeScene& sh, int mat_id, const Brdf& b, const Frame& f,
                                             bool matte, float lobe_u) {
    ParamRef p;
    p.kind = 0; p.index = 0; p.dr = 0.f;
    for (int k = 0; k < 3; ++k) { p.taps.idx[k] = 0; p.taps.w[k] = 0.f; }
    const Material m = sh.mats[mat_id];
    if (b.lobe == LOBE_MATTE) {
        if (m.type != MAT_MATTE && m.type != MAT_KELEMEN) return p;
        if (m.diff_tex >= 0) {
            const Texture t = sh.texs[m.diff_tex];
            p.kind = 2;
            if (t.tri_scale == 0.f) {
                p.taps.idx[0] = uv_texel_index(t, f.su, f.sv);
                p.taps.w[0] = 1.f;
            } else {
                p.taps = triplanar_taps(sh.attr_c2o + (size_t)f.attr * 16, t, f.P, f.Ng, false);
            }
            for (int k = 0; k < 3; ++k) p.taps.idx[k] += t.offset / 3;
        } else {
            p.kind = 1;
            p.index = mat_id;
        }
        return p;
    }
    if (b.lobe == LOBE_SPEC && m.rough_tex < 0 &&
        (m.type == MAT_KELEMEN || m.type == MAT_COOKTORRANCE || (m.type == MAT_METAL && lobe_u > m.mix))) {
        p.kind = 3;
        p.index = mat_id;
        p.dr = matte ? (float)(1.0 - 0.2) : 1.f;
    }
    return p;
}

// Pass 2 of one camera path: re-shades the recorded vertices rec[0, nv) (no ray
// tracing) and accumulates dL/dtheta with delta = dLoss/dpixel / spp (/ n for one of the
// n paths of a camera sample with light samples). Lo is the path's unclamped radiance
// from pass 1; cam_rng draws the camera ray (the path's own rng but for light samples,
// whose paths share their sample's camera ray).
template <class Acc>
__device__ __forceinline__ void replay_path(const DevScene& sc, const PathParams& p, int px, int py,
                                            const PathRng& cam_rng, const PathRng& rng, const float4* rec, int nv,
                                            float3 Lo, float3 delta, Acc& mc, float* s_g, float* s_c, float* g_tex,
                                            float* g_tex_c, RayCounts& rc) {
    if (nv == 0 || !isfinite(Lo.x) || !isfinite(Lo.y) || !isfinite(Lo.z)) return;
    float clampf = 1.f;             // firefly clamp factor (detached)
    {
        float3 c = Lo;
        for (int k = 0; k < 64 && (c.x > kFirefly || c.y > kFirefly || c.z > kFirefly); ++k) { c *= 0.2f; clampf *= 0.2f; }
    }
    const float3 dp = delta * clampf;
    RayF ray = camera_ray(sc.cam, px, py, cam_rng.u(kDimCamera), cam_rng.u(kDimCamera + 1));
    float3 T = mk(1.f, 1.f, 1.f), collected = mk(0.f, 0.f, 0.f);
    float cont = 1.f;
    bool matte = false;
    int kind = RAY_CAMERA, bounces = 0;
    for (int vtx = 0; vtx < nv; ++vtx) {
        const float4 r = rec[vtx];
        const uint32_t bits = __float_as_uint(r.w);
        const int prim = (int)(bits & 0x3fffffffu);
        uint32_t vis = bits >> 30;
        const Frame f = hit_frame(sc.sh, prim, r.x, r.y, r.z, ray.o, ray.d, true);
        const Attr at = sc.sh.attrs[f.attr];
        if (kind == RAY_DIFFUSE) matte = true;
        if (collects_emission(kind)) collected += T * at.emission;
        const float lobe_u = rng.u(vertex_dim(vtx, kDimLobe));
        const Brdf brdf = get_brdf(sc.sh, at.material, f, matte, lobe_u);
        const ParamRef pr = param_of(sc.sh, at.material, brdf, f, matte, lobe_u);
        float3 dD;
        const float3 D = direct<false, true>(sc, f, brdf, rng, vtx, rc, &vis, &dD);
        collected += D * T;
        const float3 gdir = T * dD;
        const BrdfSample bs = brdf_sample(brdf, f.V, f.N, rng.u(vertex_dim(vtx, kDimBrdf)),
                                          rng.u(vertex_dim(vtx, kDimBrdf + 1)));
        float3 gcont = mk(0.f, 0.f, 0.f);
        float3 w = mk(0.f, 0.f, 0.f);
        const bool cont_ok = bs.pdf > 0.f;
        const float3 after = Lo - collected;
        const Material mat = sc.sh.mats[at.material];
        if (mat.type == MAT_KELEMEN && mat.refl < 1.f && mat.rough_tex < 0) {
            // the lobe choice depends on roughness: score-function term on the subtree radiance
            const float score = kelemen_score(sc.sh, mat, f, brdf, matte);
            const float3 sub = dp * (D * T + after);
            mc.template add<3>(at.material, score * (sub.x + sub.y + sub.z), s_g, s_c);
        }
        if (cont_ok && pr.kind != 0) {
            const float cosl = dot(f.N, bs.dir);
            w = cdiv(bs.color * cosl, bs.pdf);
            if (pr.kind == 3) {
                const float g = sample_dlnD(brdf, f, bs);   // dw/w = d ln f
                gcont = after * g;
            } else {
                const float dw = kInvPiMacro * cosl / bs.pdf;  // d w_c / d diffuse_c
                gcont = mk(w.x != 0.f ? after.x * dw / w.x : 0.f, w.y != 0.f ? after.y * dw / w.y : 0.f,
                           w.z != 0.f ? after.z * dw / w.z : 0.f);
            }
        }
        if (pr.kind == 1 || pr.kind == 2) {
            const float3 g = dp * (gdir + gcont);
            if (pr.kind == 1) {
                mc.add3(pr.index, g, s_g, s_c);
            } else {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int i = pr.taps.idx[k];
                    const float wk = pr.taps.w[k];
                    if (!(wk > 0.f)) continue;
                    comp_add(&g_tex[3 * i + 0], &g_tex_c[3 * i + 0], g.x * wk);
                    comp_add(&g_tex[3 * i + 1], &g_tex_c[3 * i + 1], g.y * wk);
                    comp_add(&g_tex[3 * i + 2], &g_tex_c[3 * i + 2], g.z * wk);
                }
            }
        } else if (pr.kind == 3) {
            const float3 g = dp * (gdir * pr.dr + gcont * pr.dr);
            mc.template add<3>(pr.index, g.x + g.y + g.z, s_g, s_c);
        }
        // the forward update, identical to pass 1
        if (!continue_path(brdf, bs, f.N, p.min_depth, rng, vtx, T, cont, kind, bounces)) break;
        ray.o = f.P; ray.d = bs.dir; ray.mint = kRayBias; ray.maxt = bs.maxt;
    }
}

// the block's material gradients (sum and compensation) go to the global ones
__device__ __forceinline__ void flush_block(const float* s_g, const float* s_c, int nmat, float* g_mat, float* g_mat_c) {
    __syncthreads();
    for (int i = threadIdx.x; i < nmat * 4; i += blockDim.x) {
        comp_add(&g_mat[i], &g_mat_c[i], s_g[i]);
        comp_add(&g_mat[i], &g_mat_c[i], s_c[i]);
    }
}

// The environment seen by a mirror ray traced after the last shaded vertex (zero when the ray
// hits anything in [RAY_BIAS, maxt]); out of line, as the case is rare.
__device__ __noinline__ float3 escape_after_last(const BvhNode* nodes, const BvhTri* tris, const Light* lights,
                                                 int nlights, const Texture* texs, const float* texels, float3 P,
                                                 float3 dir, float maxt, float3 cam_d) {
    TraceWork w;
    if (bvh_occluded(nodes, tris, P, dir, kRayBias, maxt, w)) return mk(0.f, 0.f, 0.f);
    return env_radiance_of(lights, nlights, texs, texels, cam_d);
}

// Megakernel form: one thread per pixel runs, for each of its camera samples, pass 1
// (forward with tracing, records in thread-local memory) and pass 2 of each path. With
// light samples a camera sample's n paths start at its camera ray's first hit (traced
// once) and draw from sample indices s * L + j (integrate_camera_sample). kMulti: light
// samples above one; the one-path form keeps a single path per sample (no inner loop), whose
// code is smaller and faster. kEnv: the scene has an environment light; only then is the ray
// after the last vertex traced (any code for it in the loop made the kernel 8% slower on
// scenes without one).
template <bool kMulti, bool kEnv>
__global__ void __launch_bounds__(kAdjBlock) k_adjoint(DevScene sc, PathParams p, const float4* __restrict__ dfilm,
                                                       int nmat, float* g_mat, float* g_mat_c, float* g_tex,
                                                       float* g_tex_c, unsigned long long* counters) {
    __shared__ float s_g[kAdjMaxMat * 4], s_c[kAdjMaxMat * 4];
    for (int i = threadIdx.x; i < nmat * 4; i += blockDim.x) { s_g[i] = 0.f; s_c[i] = 0.f; }
    __syncthreads();
    const int npix = sc.cam.w * sc.cam.h;
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    const int lmax = kMulti && p.light_samples > 1 ? p.light_samples : 1;
    RayCounts rc;
    MatCache mc;
    // paths traced for this pixel: the render's sample 0 has one, every other sample lmax
    const uint32_t paths = pixel < npix ? (uint32_t)(p.spp * lmax - (p.sample_offset == 0 ? lmax - 1 : 0)) : 0u;
    if (pixel < npix) {
        const float4 df = dfilm[pixel];
        const float inv = 1.f / (float)p.spp;
        const float3 delta = mk(df.x * inv, df.y * inv, df.z * inv);
        const int px = pixel % sc.cam.w, py = pixel / sc.cam.w;
        PathRng cam_rng;
        cam_rng.key = seed_key(p.seed);
        const bool any = delta.x != 0.f || delta.y != 0.f || delta.z != 0.f;
        for (int s = 0; any && s < p.spp; ++s) {
            const int pass = p.sample_offset + s;
            const int n = kMulti ? (pass == 0 ? 1 : lmax) : 1;
            cam_rng.base = path_base((uint32_t)pixel, (uint32_t)(pass * lmax));
            RayF ray0 = camera_ray(sc.cam, px, py, cam_rng.u(kDimCamera), cam_rng.u(kDimCamera + 1));
            const float3 cam_d = ray0.d;
            Hit h0;
            ++rc.closest;
            if (!bvh_closest(sc.nodes, sc.tris, ray0.o, ray0.d, ray0.mint, ray0.maxt, &h0, rc.work)) continue;
            const float3 dn = n > 1 ? delta * (1.f / (float)n) : delta;
            for (int j = 0; j < n; ++j) {
                PathRng rng = cam_rng;
                rng.base = path_base((uint32_t)pixel, (uint32_t)(pass * lmax + j));
                // ---------------- pass 1: forward, recording hits and visibility
                float4 rec[kAdjMaxDepth];
                int nv = 0;
                float3 Lo = mk(0.f, 0.f, 0.f);
                {
                    RayF ray = ray0;
                    Hit h = h0;
                    float3 T = mk(1.f, 1.f, 1.f);
                    float cont = 1.f;
                    bool matte = false;
                    int kind = RAY_CAMERA, bounces = 0;
                    for (int vtx = 0; vtx < p.max_depth; ++vtx) {
                        nv = vtx + 1;
                        const Frame f = hit_frame(sc.sh, h.prim, h.t, h.u, h.v, ray.o, ray.d, true);
                        const Attr at = sc.sh.attrs[f.attr];
                        if (kind == RAY_DIFFUSE) matte = true;
                        if (collects_emission(kind)) Lo += T * at.emission;
                        const Brdf brdf = get_brdf(sc.sh, at.material, f, matte,
                                                   rng.u(vertex_dim(vtx, kDimLobe)));
                        uint32_t vis = 0;
                        Lo += direct<true, false>(sc, f, brdf, rng, vtx, rc, &vis, nullptr) * T;
                        rec[vtx] = pack_rec(h, vis);
                        const BrdfSample bs = brdf_sample(brdf, f.V, f.N, rng.u(vertex_dim(vtx, kDimBrdf)),
                                                          rng.u(vertex_dim(vtx, kDimBrdf + 1)));
                        if (!continue_path(brdf, bs, f.N, p.min_depth, rng, vtx, T, cont, kind, bounces)) break;
                        if (vtx + 1 >= p.max_depth) {
                            // the reference's unshaded last ray: only an escaping mirror ray adds
                            // anything, the environment (integrator.cpp:256-274); replay sees it in Lo
                            if constexpr (kEnv) {
                                if (kind == RAY_MIRROR) {
                                    ++rc.closest;
                                    Lo += escape_after_last(sc.nodes, sc.tris, sc.sh.lights, sc.sh.nlights,
                                                            sc.sh.texs, sc.sh.texels, f.P, bs.dir, bs.maxt, cam_d) * T;
                                }
                            }
                            break;
                        }
                        ray.o = f.P; ray.d = bs.dir; ray.mint = kRayBias; ray.maxt = bs.maxt;
                        ++rc.closest;
                        if (!bvh_closest(sc.nodes, sc.tris, ray.o, ray.d, ray.mint, ray.maxt, &h, rc.work)) {
                            if (kEnv && kind == RAY_MIRROR) Lo += env_radiance(sc.sh, cam_d) * T;
                            break;
                        }
                    }
                }
                // ---------------- pass 2: re-shade the recorded vertices, accumulate gradients
                // one path per sample: its own generator drew the camera ray (cam_rng is no longer live)
                replay_path(sc, p, px, py, kMulti ? cam_rng : rng, rng, rec, nv, Lo, dn, mc, s_g, s_c, g_tex,
                            g_tex_c, rc);
            }
        }
    }
    mc.flush(s_g, s_c);
    flush_block(s_g, s_c, nmat, g_mat, g_mat_c);
    unsigned long long v[3] = {rc.closest, rc.shadow, paths};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; ++k) atomicAdd(&counters[k], v[k]);
}

// Replay form (pass 2 only): one thread per item of a record pass (sub-sample-major:
// q * npix + pixel with q = sl * L + j, L = max(1, light_samples), camera sample
// p.sample_offset + s0 + sl, random-number sample index (p.sample_offset + s0) * L + q).
// The wavefront engine's record pass wrote the hit records rec[item][p.max_depth] and
// lo_raw[item]; the sub-samples j > 0 of the render's sample 0 were not traced.
// 8 resident blocks of 128 threads (64 registers). (A grid-stride loop over a resident
// grid was 30% slower: the block scheduler already balances 128-thread blocks.)
__global__ void __launch_bounds__(kAdjBlock, 8) k_adjoint_replay(DevScene sc, PathParams p, int s0, uint32_t items,
                                                              const float4* __restrict__ rec,
                                                              const float4* __restrict__ lo_raw,
                                                              const float4* __restrict__ dfilm, int nmat, float* g_mat,
                                                              float* g_mat_c, float* g_tex, float* g_tex_c) {
    __shared__ float s_g[kAdjMaxMat * 4], s_c[kAdjMaxMat * 4];
    for (int i = threadIdx.x; i < nmat * 4; i += blockDim.x) { s_g[i] = 0.f; s_c[i] = 0.f; }
    __syncthreads();
    const uint32_t npix = (uint32_t)(sc.cam.w * sc.cam.h);
    RayCounts rc;
    DirectAcc mc;
    const uint32_t item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item < items) {
        const uint32_t lsub = p.light_samples > 1 ? (uint32_t)p.light_samples : 1u;
        const uint32_t pixel = item % npix, q = item / npix;
        const uint32_t j = q % lsub, sample = (uint32_t)(p.sample_offset + s0) + q / lsub;
        const uint32_t n = sample == 0 ? 1u : lsub;
        const float4 df = dfilm[pixel];
        const float inv = 1.f / (float)p.spp;
        float3 delta = mk(df.x * inv, df.y * inv, df.z * inv);
        if (n > 1) delta = delta * (1.f / (float)n);
        if (j < n && (delta.x != 0.f || delta.y != 0.f || delta.z != 0.f)) {
            const uint32_t first = (uint32_t)(p.sample_offset + s0) * lsub;
            PathRng rng, cam_rng;
            rng.key = cam_rng.key = seed_key(p.seed);
            rng.base = path_base(pixel, first + q);
            cam_rng.base = path_base(pixel, first + q - j);
            const float4 lo = lo_raw[item];
            replay_path(sc, p, (int)(pixel % (uint32_t)sc.cam.w), (int)(pixel / (uint32_t)sc.cam.w), cam_rng, rng,
                        rec + (size_t)item * p.max_depth, __float_as_int(lo.w), mk(lo.x, lo.y, lo.z), delta, mc, s_g,
                        s_c, g_tex, g_tex_c, rc);
        }
    }
    mc.flush(s_g, s_c);
    flush_block(s_g, s_c, nmat, g_mat, g_mat_c);
}

__global__ void k_add_comp(float* g, const float* c, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) g[i] += c[i];
}

}  // namespace
}  // namespace aur

using namespace aur;

extern "C" aur_status aur_render_adjoint(aur_scene* sc, const aur_render_opts* o, const float* dfilm, float* grad_mat,
                                         float* grad_tex, aur_render_stats* stats) {
    if (!sc || !o || !dfilm || !grad_mat) return fail(AUR_ERR_INVALID_ARG, "aur_render_adjoint: NULL argument");
    if (sc->ntexel_floats && !grad_tex) return fail(AUR_ERR_INVALID_ARG, "aur_render_adjoint: grad_tex is NULL");
    PathParams p;
    aur_status st = render_options(sc, o, &p);
    if (st != AUR_OK) return st;
    if (o->mode != AUR_RENDER_PLAIN && o->mode != AUR_RENDER_WAVEFRONT)
        return fail(AUR_ERR_INVALID_ARG, "aur_render_adjoint: unknown mode");
    const bool wavefront = o->mode == AUR_RENDER_WAVEFRONT;
    // the megakernel keeps a path's hit records in registers / local memory; the wavefront
    // form records them in device memory and takes any depth
    if (!wavefront && o->max_depth > kAdjMaxDepth)
        return fail(AUR_ERR_UNSUPPORTED, "aur_render_adjoint: max_depth above 16 needs mode AUR_RENDER_WAVEFRONT");
    if (sc->ntri >= (1u << 30)) return fail(AUR_ERR_UNSUPPORTED, "aur_render_adjoint: 2^30 triangles or more");
    const int nmat = (int)sc->h_mats.size();
    if (nmat > kAdjMaxMat) return fail(AUR_ERR_UNSUPPORTED, "aur_render_adjoint: more than 64 materials");
    DeviceGuard g(sc->ctx->device);
    cudaStream_t s = sc->ctx->stream;
    const size_t npix = (size_t)sc->cam.w * sc->cam.h;
    const int ntex = (int)sc->ntexel_floats;
    DevIn din;
    DevOut gm, gt;
    float *cm = nullptr, *ct = nullptr;
    cudaError_t e = din.init(dfilm, sizeof(float4) * npix, 16, s);
    if (e == cudaSuccess) e = gm.init(grad_mat, sizeof(float) * 4 * nmat, 4, s);
    if (e == cudaSuccess && ntex) e = gt.init(grad_tex, sizeof(float) * ntex, 4, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&cm, sizeof(float) * (4 * nmat + ntex), s);
    ct = cm ? cm + 4 * nmat : nullptr;
    if (e == cudaSuccess) e = cudaMemsetAsync(gm.ptr, 0, sizeof(float) * 4 * nmat, s);
    if (e == cudaSuccess && ntex) e = cudaMemsetAsync(gt.ptr, 0, sizeof(float) * ntex, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cm, 0, sizeof(float) * (4 * nmat + ntex), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(sc->ctx->counters, 0, sizeof(unsigned long long) * 8, s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    cudaEvent_t er0, er1;   // replay kernels alone (wavefront mode)
    cudaEventCreate(&er0);
    cudaEventCreate(&er1);
    double replay_ms = 0.0;
    uint64_t launches = 0;
    unsigned long long rays[2] = {0, 0};
    float4* rec = nullptr;
    if (wavefront) {
        // record passes (wavefront engine) + replay kernels over chunks of the samples, sized
        // so that the records stay within 2 GiB and item indices within 2^31
        const size_t lsub = (size_t)p.light_samples;   // items per pixel and camera sample
        const size_t per_item = sizeof(float4) * ((size_t)p.max_depth + 1);
        const size_t budget = (size_t)2 << 30;
        int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)p.spp, budget / (per_item * npix * lsub)));
        while (chunk > 1 && (size_t)chunk * npix * lsub * (p.max_depth + 1) >= (1ull << 31)) chunk /= 2;
        if ((size_t)chunk * npix * lsub * (p.max_depth + 1) >= (1ull << 31)) e = cudaErrorInvalidValue;
        if (e == cudaSuccess) e = ctx_scratch(sc->ctx, per_item * npix * lsub * chunk, (void**)&rec);
        float4* lo_raw = rec ? rec + (size_t)npix * lsub * chunk * p.max_depth : nullptr;
        for (int s0 = 0; s0 < p.spp && e == cudaSuccess; s0 += chunk) {
            const int n = std::min(chunk, p.spp - s0);
            aur_status rs = wf_record_pass(sc, p, s0, n, rec, lo_raw, &launches, rays);
            if (rs != AUR_OK) {
                if (cm) cudaFreeAsync(cm, s);
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                cudaEventDestroy(er0);
                cudaEventDestroy(er1);
                return rs;
            }
            const uint32_t items = (uint32_t)(npix * lsub * (size_t)n);
            cudaEventRecord(er0, s);
            k_adjoint_replay<<<(items + kAdjBlock - 1) / kAdjBlock, kAdjBlock, 0, s>>>(
                sc->dev(), p, s0, items, rec, lo_raw, (const float4*)din.ptr, nmat, (float*)gm.ptr, cm,
                ntex ? (float*)gt.ptr : nullptr, ct);
            ++launches;
            e = cudaGetLastError();
            cudaEventRecord(er1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(er1);
            float rms = 0.f;
            if (e == cudaSuccess && cudaEventElapsedTime(&rms, er0, er1) == cudaSuccess) replay_ms += rms;
        }
    } else if (e == cudaSuccess) {
        const unsigned grid = (unsigned)((npix + kAdjBlock - 1) / kAdjBlock);
        const DevScene dsc = sc->dev();
        auto kern = p.light_samples > 1 ? (dsc.sh.nenv ? k_adjoint<true, true> : k_adjoint<true, false>)
                                        : (dsc.sh.nenv ? k_adjoint<false, true> : k_adjoint<false, false>);
        kern<<<grid, kAdjBlock, 0, s>>>(dsc, p, (const float4*)din.ptr, nmat, (float*)gm.ptr, cm,
                                        ntex ? (float*)gt.ptr : nullptr, ct, sc->ctx->counters);
        ++launches;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_add_comp<<<(4 * nmat + 255) / 256, 256, 0, s>>>((float*)gm.ptr, cm, 4 * nmat);
        ++launches;
        if (ntex) { k_add_comp<<<(ntex + 255) / 256, 256, 0, s>>>((float*)gt.ptr, ct, ntex); ++launches; }
        e = cudaGetLastError();
    }
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = gm.finish();
    if (e == cudaSuccess && ntex) e = gt.finish();
    // paths traced: the render's sample 0 traces one path, every other camera sample L
    const unsigned long long lpaths = (unsigned long long)p.light_samples;
    unsigned long long cnt[3] = {rays[0], rays[1],
                                 (unsigned long long)npix * ((unsigned long long)p.spp * lpaths -
                                                             (p.sample_offset == 0 ? lpaths - 1 : 0))};
    if (e == cudaSuccess && !wavefront)
        e = cudaMemcpyAsync(cnt, sc->ctx->counters, sizeof(cnt), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(er0);
    cudaEventDestroy(er1);
    if (cm) cudaFreeAsync(cm, s);
    if (e != cudaSuccess) return cuda_fail(e, "aur_render_adjoint");
    if (stats) {
        *stats = aur_render_stats{};
        stats->closest_rays = cnt[0];
        stats->shadow_rays = cnt[1];
        stats->paths = cnt[2];
        stats->camera_rays = (unsigned long long)npix * p.spp;
        stats->launches = launches;
        stats->kernel_ms = ms;
        if (wavefront) {   // stage_ms[0]: record passes (and the rest), stage_ms[1]: replay kernels
            stats->stage_ms[1] = replay_ms;
            stats->stage_ms[0] = ms - replay_ms;
            if (sc->wf_tuned) { stats->wf_pool = sc->wf_pool; stats->wf_block = sc->wf_block; stats->wf_sort = sc->wf_sort; }
        }
    }
    return AUR_OK;
}
