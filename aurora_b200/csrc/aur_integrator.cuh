// aur_integrator.cuh — the per-path MIS loop of Integrator::integrateCameraSample
// (Aurora/src/frontend/integrator.cpp:152-300) for one camera path, as a
// device function shared by the plain megakernel and the tests' probes.
//
// Faithful to the reference: emission only on camera rays; one light chosen
// uniformly among the "visible" ones and the result scaled by their count
// (integrator.cpp:100-130); Lambert vertices use light sampling only
// (integrateDirectLight :33-54), specular vertices the power-heuristic MIS of
// integrateDirectMIS (:56-98); throughput f*cos/pdf; a cumulative continue
// probability and roulette when bounces > mindepth (:219-248); firefly clamp
// (:278-281). The reference traces one more closest-hit ray after the last
// shaded vertex; its hit is never shaded, and when it misses it adds the
// environment lights if it is a mirror ray (:256-274). That ray is traced here
// only when it can add something (a mirror ray in a scene with an environment
// light); its hit ends the path unshaded.
#pragma once
#include "aur_traverse.cuh"

namespace aur {

struct DevScene {
    const BvhNode* nodes;
    const BvhTri* tris;
    const BvhNode4* nodes4;   // the 4-wide form of the same tree, or null
    ShadeScene sh;
    Camera cam;
};

struct PathParams {
    int max_depth, min_depth;
    int spp, sample_offset;
    uint32_t seed;
    int light_samples;   // paths per camera sample after the first pass (1: one path)
};

struct RayCounts { uint32_t closest = 0, shadow = 0; TraceWork work, shadow_work; };

// Picks the k-th light for which light_visible() holds; returns -1 if none.
__device__ __forceinline__ int pick_visible_light(const ShadeScene& sh, float3 P, float3 N, float u, int* nvis) {
    int n = 0;
    for (int i = 0; i < sh.nlights; ++i) n += light_visible(sh.lights[i], P, N) ? 1 : 0;
    *nvis = n;
    if (n == 0) return -1;
    int k = (int)(u * (float)n);
    k = k < n ? k : n - 1;
    for (int i = 0; i < sh.nlights; ++i) {
        if (light_visible(sh.lights[i], P, N)) {
            if (k == 0) return i;
            --k;
        }
    }
    return -1;
}

// Traversal of the scene's binary (kWidth 2) or 4-wide (kWidth 4) tree.
template <int kWidth>
__device__ __forceinline__ bool trace_closest(const DevScene& sc, float3 o, float3 d, float mint, float maxt, Hit* h,
                                              TraceWork& w) {
    if constexpr (kWidth == 4) return bvh_trace4<false>(sc.nodes4, sc.tris, o, d, mint, maxt, h, w);
    else return bvh_trace<false>(sc.nodes, sc.tris, o, d, mint, maxt, h, w);
}
template <int kWidth>
__device__ __forceinline__ bool trace_occluded(const DevScene& sc, float3 o, float3 d, float mint, float maxt,
                                               TraceWork& w) {
    Hit h;
    if constexpr (kWidth == 4) return bvh_trace4<true>(sc.nodes4, sc.tris, o, d, mint, maxt, &h, w);
    else return bvh_trace<true>(sc.nodes, sc.tris, o, d, mint, maxt, &h, w);
}

// integrateDirect (integrator.cpp:100-130) with integrateDirectLight / integrateDirectMIS.
template <int kWidth>
__device__ __forceinline__ float3 integrate_direct(const DevScene& sc, const Frame& f, const Brdf& brdf,
                                                   const PathRng& rng, int vtx, RayCounts& rc) {
    float3 res = mk(0.f, 0.f, 0.f);
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
            ++rc.shadow;
            if (!trace_occluded<kWidth>(sc, f.P, ls.dir, kRayBias, ls.maxt, rc.shadow_work))
                res += cdiv((ls.color * brdf_eval(brdf, ls.dir, f.V, f.N)) * cost, ls.pdf);
        }
    } else {
        if (cost > 0.f && ls.pdf > 0.f) {
            const float bp = brdf_pdf(brdf, ls.dir, f.V, f.N);
            if (bp > 0.f) {
                ++rc.shadow;
                if (!trace_occluded<kWidth>(sc, f.P, ls.dir, kRayBias, ls.maxt, rc.shadow_work)) {
                    const float w = power_heuristic(ls.pdf, bp);
                    res += cdiv(((ls.color * w) * brdf_eval(brdf, ls.dir, f.V, f.N)) * cost, ls.pdf);
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
                ++rc.shadow;
                if (!trace_occluded<kWidth>(sc, f.P, bs.dir, kRayBias, maxt, rc.shadow_work)) {
                    const float w = power_heuristic(bs.pdf, lp);
                    res += cdiv(((bs.color * w) * light_eval(sc.sh, L, bs.dir)) * cost, bs.pdf);
                }
            }
        }
    }
    return res * (float)nvis;
}

enum RayKind : int { RAY_CAMERA = 0, RAY_DIFFUSE = 1, RAY_SPECULAR = 2, RAY_MIRROR = 3 };

// Emission is added at vertices reached by camera and mirror rays (integrator.cpp:184-187).
__device__ __forceinline__ bool collects_emission(int kind) { return kind == RAY_CAMERA || kind == RAY_MIRROR; }

// Continuation of Integrator::integrateCameraSample (integrator.cpp:202-243) after the
// BRDF sample `bs` of `brdf`: throughput, roulette probability, ray kind, roulette and the
// bounce count. Delta lobes (mirror, transmission) multiply by the sample colour only,
// skip the black test and do not count as bounces for roulette. Returns false when the
// path ends.
__device__ __forceinline__ bool continue_path(const Brdf& brdf, const BrdfSample& bs, float3 N, int min_depth,
                                              const PathRng& rng, int vtx, float3& T, float& cont, int& kind,
                                              int& bounces) {
    if (bs.pdf <= 0.f) return false;
    const bool delta = brdf.lobe == LOBE_MIRROR || brdf.lobe == LOBE_TRANSMIT;
    if (!delta) {
        const float cosl = dot(N, bs.dir);
        T *= cdiv(bs.color * cosl, bs.pdf);
        if (bounces > min_depth) cont *= lum(bs.color) * cosl / bs.pdf;
        if (is_black(T)) return false;
        kind = brdf.lobe == LOBE_SPEC ? RAY_SPECULAR : RAY_DIFFUSE;
    } else {
        T *= bs.color;
        if (bounces > min_depth) cont *= lum(bs.color);
        kind = RAY_MIRROR;
    }
    if (bounces > min_depth) {
        if (rng.u(vertex_dim(vtx, kDimRoulette)) > cont) return false;
        T = cdiv(T, cont);
    }
    if (!delta) ++bounces;
    return true;
}

// Firefly filter (integrator.cpp:278-281). A non-finite estimate would never
// leave the reference's loop; it is dropped (returned as black) instead, which
// also bounds the loop to at most ~50 iterations.
AUR_HD float3 firefly_clamp(float3 Lo) {
    if (!isfinite(Lo.x) || !isfinite(Lo.y) || !isfinite(Lo.z)) return mk(0.f, 0.f, 0.f);
    for (int k = 0; k < 64 && (Lo.x > kFirefly || Lo.y > kFirefly || Lo.z > kFirefly); ++k) Lo *= 0.2f;
    return Lo;
}

// The path from the camera ray's first hit `h` (ray `ray`, camera direction `cam_d`);
// returns its firefly-filtered radiance.
template <int kWidth>
__device__ __forceinline__ float3 path_from_hit(const DevScene& sc, const PathParams& p, RayF ray, Hit h,
                                                const float3 cam_d, const PathRng& rng, RayCounts& rc) {
    float3 Lo = mk(0.f, 0.f, 0.f);
    float3 T = mk(1.f, 1.f, 1.f);
    float cont = 1.f;
    bool matte_path = false;
    int kind = RAY_CAMERA;
    int bounces = 0;
    for (int vtx = 0; vtx < p.max_depth; ++vtx) {
        const Frame f = hit_frame(sc.sh, h.prim, h.t, h.u, h.v, ray.o, ray.d, true);
        const Attr at = sc.sh.attrs[f.attr];
        if (kind == RAY_DIFFUSE) matte_path = true;
        if (collects_emission(kind)) Lo += T * at.emission;
        const Brdf brdf = get_brdf(sc.sh, at.material, f, matte_path,
                                   rng.u(vertex_dim(vtx, kDimLobe)));
        Lo += integrate_direct<kWidth>(sc, f, brdf, rng, vtx, rc) * T;
        const BrdfSample bs = brdf_sample(brdf, f.V, f.N, rng.u(vertex_dim(vtx, kDimBrdf)),
                                          rng.u(vertex_dim(vtx, kDimBrdf + 1)));
        if (!continue_path(brdf, bs, f.N, p.min_depth, rng, vtx, T, cont, kind, bounces)) break;
        // after the last vertex the reference traces one more ray whose hit is never shaded and
        // whose miss adds the environment for a mirror ray (integrator.cpp:256-274): traced here
        // only when it can add something, through the same call as every other ray
        const bool last = vtx + 1 >= p.max_depth;
        if (last && !(kind == RAY_MIRROR && sc.sh.nenv)) break;
        ray.o = f.P;
        ray.d = bs.dir;
        ray.mint = kRayBias;
        ray.maxt = bs.maxt;
        ++rc.closest;
        if (!trace_closest<kWidth>(sc, ray.o, ray.d, ray.mint, ray.maxt, &h, rc.work)) {
            // a mirror ray that escapes sees the environment along the CAMERA ray's
            // direction, as integrator.cpp:262-274 evaluates it
            if (kind == RAY_MIRROR && sc.sh.nenv) Lo += env_radiance(sc.sh, cam_d) * T;
            break;
        }
        if (last) break;
    }
    return firefly_clamp(Lo);
}

// One camera path; returns the clamped radiance, sets *alpha to 1 on a camera hit.
template <int kWidth>
__device__ __forceinline__ float3 integrate_path(const DevScene& sc, const PathParams& p, int px, int py,
                                                 const PathRng& rng, RayCounts& rc, float* alpha) {
    RayF ray = camera_ray(sc.cam, px, py, rng.u(kDimCamera), rng.u(kDimCamera + 1));
    Hit h;
    ++rc.closest;
    *alpha = 0.f;
    const float3 cam_d = ray.d;
    if (!trace_closest<kWidth>(sc, ray.o, ray.d, ray.mint, ray.maxt, &h, rc.work)) {
        if (sc.sh.nenv == 0) return mk(0.f, 0.f, 0.f);
        *alpha = 1.f;                       // environment seen directly: not firefly-filtered
        return env_radiance(sc.sh, cam_d);
    }
    *alpha = 1.f;
    return path_from_hit<kWidth>(sc, p, ray, h, cam_d, rng, rc);
}

// Integrator::integrateCameraSample(sample, numSamples) (integrator.cpp:152-300) in pass
// `pass` (the sample index): the first pass traces one path per camera sample and later
// passes p.light_samples paths from the camera ray's first hit (renderer.cpp:231-258
// starts lightSamples at 1 and raises it after the first pass), each averaged in as
// Lo / numSamples. Sub-path j of pass s draws from sample index s * L + j (L =
// max(1, p.light_samples)); the camera ray from s * L. *paths = the paths traced.
template <int kWidth>
__device__ __forceinline__ float3 integrate_camera_sample(const DevScene& sc, const PathParams& p, int px, int py,
                                                          uint32_t pixel, uint64_t key, int pass, RayCounts& rc,
                                                          float* alpha, int* paths) {
    const int lmax = p.light_samples > 1 ? p.light_samples : 1;
    const int n = pass == 0 ? 1 : lmax;
    PathRng rng;
    rng.key = key;
    rng.base = path_base(pixel, (uint32_t)(pass * lmax));
    *paths = n;
    RayF ray = camera_ray(sc.cam, px, py, rng.u(kDimCamera), rng.u(kDimCamera + 1));
    Hit h;
    ++rc.closest;
    *alpha = 0.f;
    const float3 cam_d = ray.d;
    if (!trace_closest<kWidth>(sc, ray.o, ray.d, ray.mint, ray.maxt, &h, rc.work)) {
        if (sc.sh.nenv == 0) return mk(0.f, 0.f, 0.f);
        *alpha = 1.f;                       // environment seen directly: not firefly-filtered
        return env_radiance(sc.sh, cam_d);
    }
    *alpha = 1.f;
    // one call site of the path (one copy of its code) for any number of sub-paths
    float3 sum = mk(0.f, 0.f, 0.f);
    for (int j = 0; j < n; ++j) {
        PathRng rj = rng;
        rj.base = path_base(pixel, (uint32_t)(pass * lmax + j));
        const float3 v = path_from_hit<kWidth>(sc, p, ray, h, cam_d, rj, rc);
        if (n == 1) sum = v;                 // Lo / 1.f: unchanged
        else sum += cdiv(v, (float)n);
    }
    return sum;
}

}  // namespace aur
