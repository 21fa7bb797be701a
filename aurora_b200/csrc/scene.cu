// scene.cu — flattened scenes on the device and the render entry points.
//
// aur_scene_create takes the camera-space soup that
// Renderer::buildRenderEnvironment produces (Aurora/src/frontend/renderer.cpp:99-145):
// objects then light shapes, per-corner normals/uvs (EmbreeMesh, embreeMesh.h:30-63),
// AttributeState {material, emission} per object/light, materials, lights.
#include "aur_capi_internal.h"
#include "aur_host_math.h"
#include <cmath>
#include <cstring>
#include <thread>

using namespace aur;


namespace aur {

aur_status bvh_options(const aur_bvh_opts* o, BvhBuildOptions* out) {
    *out = BvhBuildOptions();
    if (!o) return AUR_OK;
    if (o->max_leaf) out->max_leaf = o->max_leaf;
    if (o->cost_traverse > 0.f) out->cost_traverse = o->cost_traverse;
    if (o->cost_intersect > 0.f) out->cost_intersect = o->cost_intersect;
    if (o->ploc_radius) out->ploc_radius = o->ploc_radius;
    if (out->max_leaf < 1 || out->max_leaf > 31) return fail(AUR_ERR_INVALID_ARG, "bvh options: max_leaf must be 1..31");
    if (out->ploc_radius < 1 || out->ploc_radius > 32)
        return fail(AUR_ERR_INVALID_ARG, "bvh options: ploc_radius must be 1..32");
    return AUR_OK;
}

// Square light set-up of SquareLight's constructor (squareLight.cpp:20-52); the
// environment light's (infiniteAreaLight.cpp:21-33, Texture2D::initPdf).
static Light make_light(const aur_light_desc& d, const std::vector<Texture>& texs, const float* texels) {
    Light l;
    memset(&l, 0, sizeof(l));
    l.type = d.type;
    l.tex = -1;
    const float inten = powf(2.f, d.exposure);
    l.le = mk(d.color[0] * inten, d.color[1] * inten, d.color[2] * inten);
    for (int k = 0; k < 16; ++k) l.m[k] = d.object_to_camera[k];
    if (d.type == AUR_LIGHT_ENV) {
        const float e = (float)pow(2.0, (double)d.exposure);             // pow(2, m_exposure) in eval
        l.le = mk(d.color[0] * e, d.color[1] * e, d.color[2] * e);
        l.escale = e;
        invert4_gj(l.m, l.minv);
        if (d.tex >= 0) {   // the pdf normalisation: the FP32 running sum of (r + g + b) / 3 over the map
            l.tex = d.tex;
            const Texture& t = texs[d.tex];
            float sum = 0.f;
            for (int y = 0; y < t.h; ++y)
                for (int x = 0; x < t.w; ++x) {
                    const float* p = texels + t.offset + 3 * ((size_t)y * t.w + x);
                    sum += (p[0] + p[1] + p[2]) / 3.f;
                }
            l.pdf_norm = sum / (float)(t.w * t.h);
        }
        return l;
    }
    if (d.type == AUR_LIGHT_SQUARE) {
        l.xs = d.size_x;
        l.ys = d.size_y;
        l.p[0] = xform_point(l.m, mk(-l.xs, -l.ys, 0.f));
        l.p[1] = xform_point(l.m, mk(-l.xs, l.ys, 0.f));
        l.p[2] = xform_point(l.m, mk(l.xs, l.ys, 0.f));
        l.p[3] = xform_point(l.m, mk(l.xs, -l.ys, 0.f));
        l.n = normalize(cross(l.p[0] - l.p[1], l.p[1] - l.p[2]));
    } else {
        l.center = mk(d.center[0], d.center[1], d.center[2]);
        l.radius = d.radius;
    }
    return l;
}

static Material make_material(const aur_material_desc& d) {
    Material m;
    memset(&m, 0, sizeof(m));
    m.type = d.type;
    m.diff_tex = d.diffuse_tex;
    m.spec_tex = d.specular_tex;
    m.rough_tex = d.roughness_tex;
    m.diff = mk(d.diffuse[0], d.diffuse[1], d.diffuse[2]);
    m.spec = mk(d.specular[0], d.specular[1], d.specular[2]);
    m.gain = mk(d.gain[0], d.gain[1], d.gain[2]);
    m.rough = d.roughness;
    m.rough_b = d.roughness_b;
    m.refl = d.reflectance;
    m.mix = d.mix;
    m.ior = d.ior;
    m.table = d.type == AUR_MAT_KELEMEN ? kelemen_index(d.reflectance) : 0;
    m.norm_tex = d.normal_kind == AUR_NORMAL_TEXTURE ? d.normal_tex
               : d.normal_kind == AUR_NORMAL_CONSTANT ? kNormalConst : kNormalNone;
    m.norm = mk(d.normal[0], d.normal[1], d.normal[2]);
    return m;
}

template <typename T>
static cudaError_t upload(T** dst, const void* src, size_t count, cudaStream_t s) {
    *dst = nullptr;
    if (!src || count == 0) return cudaSuccess;
    cudaError_t e = cudaMallocAsync((void**)dst, sizeof(T) * count, s);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, src, sizeof(T) * count,
                           is_device_ptr(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
}

static void scene_free(aur_scene* sc) {
    --sc->ctx->live;
    cudaStream_t s = sc->ctx->stream;
    cudaStreamSynchronize(s);
    bvh_free_device(&sc->bvh.bvh, s);
    cudaStreamSynchronize(s);
    void* bufs[] = {sc->bvh.tri_attr, sc->corner_n, sc->corner_uv, sc->attrs, sc->mats, sc->lights, sc->texs, sc->texels,
                    sc->attr_c2o};
    for (void* b : bufs) if (b) cudaFreeAsync(b, s);
    cudaStreamSynchronize(s);
    delete sc;
}

}  // namespace aur

DevScene aur_scene::dev() const {
    DevScene d;
    d.nodes = bvh.bvh.nodes;
    d.tris = bvh.bvh.tris;
    d.nodes4 = bvh.bvh.nodes4;
    d.sh.mats = mats;
    d.sh.attrs = attrs;
    d.sh.lights = lights;
    d.sh.texs = texs;
    d.sh.texels = texels;
    d.sh.albedo = ctx->kelemen;
    d.sh.corner_n = corner_n;
    // the per-corner uvs are read only where a uv-mapped shader (texture2DShader) needs them:
    // a scene without one skips their 24 bytes per shaded vertex
    bool uses_uv = false;
    auto uv_tex = [&](int t) { return t >= 0 && t < (int)h_texs.size() && h_texs[t].tri_scale == 0.f; };
    for (const Material& m : h_mats)
        uses_uv = uses_uv || uv_tex(m.diff_tex) || uv_tex(m.spec_tex) || uv_tex(m.rough_tex) || uv_tex(m.norm_tex);
    d.sh.corner_uv = uses_uv ? corner_uv : nullptr;
    d.sh.tri_attr = bvh.tri_attr;
    d.sh.nlights = (int)h_lights.size();
    d.sh.nenv = 0;
    for (const Light& l : h_lights) d.sh.nenv += l.type == LIGHT_ENV ? 1 : 0;
    d.sh.nnormal = 0;
    for (const Material& m : h_mats) d.sh.nnormal += m.norm_tex != kNormalNone ? 1 : 0;
    d.sh.attr_c2o = attr_c2o;
    d.cam = cam;
    return d;
}

extern "C" {

aur_status aur_scene_create(aur_ctx* ctx, const aur_scene_desc* d, const aur_bvh_opts* bvh_opts, aur_scene** out) {
    if (!ctx || !d || !out) return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: NULL argument");
    *out = nullptr;
    if (!d->verts || !d->tri_vidx || !d->tri_attr || !d->corner_normals || d->ntri == 0)
        return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: geometry arrays missing or empty");
    if (!d->attr_material || !d->attr_emission || d->nattr == 0)
        return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: attribute arrays missing");
    if (!d->materials || d->nmat == 0) return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: no materials");
    if (d->nlight && !d->lights) return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: lights missing");
    if (d->width <= 0 || d->height <= 0 || (long long)d->width * d->height > (1ll << 31) / 4)
        return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: bad resolution");
    if (d->ntex && (!d->tex_dims || !d->texels)) return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: textures missing");
    // the triangles' attribute indices are checked on the device after their upload (below);
    // the attributes' material indices here (device-resident attribute tables are trusted)
    for (uint32_t i = 0; i < d->nattr; ++i)
        if (!is_device_ptr(d->attr_material) && (d->attr_material[i] < 0 || (uint32_t)d->attr_material[i] >= d->nmat))
            return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: attribute material out of range");
    std::vector<Texture> texs(d->ntex);
    uint32_t texel_floats = 0;
    for (uint32_t t = 0; t < d->ntex; ++t) {
        const int w = d->tex_dims[2 * t], h = d->tex_dims[2 * t + 1];
        if (w <= 0 || h <= 0) return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: bad texture size");
        texs[t].w = w; texs[t].h = h; texs[t].offset = (int)texel_floats;
        texs[t].tri_scale = 0.f;
        if (d->tex_triplanar_scale) {
            if (is_device_ptr(d->tex_triplanar_scale))
                return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: triplanar scales must be host memory");
            const float sc = d->tex_triplanar_scale[t];
            if (!(sc >= 0.f) || !std::isfinite(sc))
                return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: triplanar scale must be finite and >= 0");
            texs[t].tri_scale = sc;
        }
        texel_floats += 3u * (uint32_t)w * (uint32_t)h;
    }
    std::vector<Material> mats(d->nmat);
    for (uint32_t m = 0; m < d->nmat; ++m) {
        const aur_material_desc& md = d->materials[m];
        if (md.type < AUR_MAT_MATTE || md.type > AUR_MAT_GLASS)
            return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: unknown material type");
        if (md.type == AUR_MAT_GLASS && !(md.ior > 0.f))
            return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: glass needs an index of refraction > 0");
        const int tx[3] = {md.diffuse_tex, md.specular_tex, md.roughness_tex};
        for (int k = 0; k < 3; ++k)
            if (tx[k] >= (int)d->ntex || tx[k] < -1) return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: texture index");
        if (md.normal_kind < AUR_NORMAL_NONE || md.normal_kind > AUR_NORMAL_CONSTANT)
            return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: unknown normal-map kind");
        if (md.normal_kind == AUR_NORMAL_TEXTURE && (md.normal_tex < 0 || md.normal_tex >= (int)d->ntex))
            return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: normal-map texture index");
        mats[m] = make_material(md);
    }
    std::vector<Light> lights(d->nlight);
    for (uint32_t l = 0; l < d->nlight; ++l) {
        const aur_light_desc& ld = d->lights[l];
        if (ld.type != AUR_LIGHT_SQUARE && ld.type != AUR_LIGHT_SPHERE && ld.type != AUR_LIGHT_ENV)
            return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: unknown light type");
        if (ld.type == AUR_LIGHT_ENV) {
            float inv[16];
            if (!invert4_gj(ld.object_to_camera, inv))
                return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: singular camera-to-world matrix");
            if (ld.tex >= (int)d->ntex || ld.tex < -1)
                return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: environment texture index");
            if (ld.tex >= 0 && is_device_ptr(d->texels))
                return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: an env map needs host texels");
            if (ld.tex >= 0 && texs[ld.tex].tri_scale != 0.f)
                return fail(AUR_ERR_INVALID_ARG, "aur_scene_create: an env map must be a plain (uv) texture");
        }
        lights[l] = make_light(ld, texs, d->texels);
    }

    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    // The per-corner normals and uvs (the largest inputs, 60 B per triangle) go up on
    // their own stream and host thread while the BVH builds.
    float *cn = nullptr, *cu = nullptr;
    cudaError_t up_err = cudaSuccess;
    cudaStream_t us = nullptr;
    std::thread uploader;
    if (cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking) == cudaSuccess) {
        uploader = std::thread([&]() {
            DeviceGuard g2(ctx->device);
            up_err = upload(&cn, d->corner_normals, 9 * (size_t)d->ntri, us);
            if (up_err == cudaSuccess) up_err = upload(&cu, d->corner_uvs, 6 * (size_t)d->ntri, us);
            cudaError_t se = cudaStreamSynchronize(us);
            if (up_err == cudaSuccess) up_err = se;
        });
    } else {
        cudaGetLastError();
        us = nullptr;                // uploaded below on the context's stream
    }
    aur_bvh* tmp = nullptr;
    aur_status st = aur_bvh_build(ctx, d->verts, d->nvert, d->tri_vidx, d->tri_attr, d->ntri, bvh_opts, &tmp);
    if (st == AUR_OK) {   // every triangle's attribute index below nattr (negative ones wrap above)
        bool in_range = true;
        const cudaError_t ce = indices_below((const uint32_t*)tmp->tri_attr, d->ntri, d->nattr, &in_range, s);
        if (ce != cudaSuccess) st = cuda_fail(ce, "aur_scene_create(check)");
        else if (!in_range) st = fail(AUR_ERR_INVALID_ARG, "aur_scene_create: triangle attribute out of range");
        if (st != AUR_OK) { aur_bvh_destroy(tmp); tmp = nullptr; }
    }
    if (uploader.joinable()) uploader.join();
    if (us) cudaStreamDestroy(us);
    if (st != AUR_OK) {
        if (cn) cudaFree(cn);
        if (cu) cudaFree(cu);
        return st;
    }
    aur_scene* sc = new aur_scene();
    sc->ctx = ctx;
    sc->bvh = *tmp;
    sc->bvh.owned_by_scene = true;
    delete tmp;                      // the scene takes over the BVH's place in ctx->live
    sc->ntri = d->ntri;
    sc->nattr = d->nattr;
    sc->ntexel_floats = texel_floats;
    sc->h_mats = mats;
    sc->h_lights = lights;
    sc->h_texs = texs;
    sc->cam.fov = d->fov;
    sc->cam.w = d->width;
    sc->cam.h = d->height;
    std::vector<Attr> attrs(d->nattr);
    {
        std::vector<int32_t> am(d->nattr);
        std::vector<float> ae(3 * d->nattr);
        cudaMemcpy(am.data(), d->attr_material, sizeof(int32_t) * d->nattr, cudaMemcpyDefault);
        cudaMemcpy(ae.data(), d->attr_emission, sizeof(float) * 3 * d->nattr, cudaMemcpyDefault);
        for (uint32_t i = 0; i < d->nattr; ++i) { attrs[i].material = am[i]; attrs[i].emission = mk(ae[3 * i], ae[3 * i + 1], ae[3 * i + 2]); }
    }
    // cameraToObject per attribute (identity when not given)
    std::vector<float> c2o(16 * (size_t)d->nattr, 0.f);
    if (d->attr_camera_to_object) {
        cudaMemcpy(c2o.data(), d->attr_camera_to_object, sizeof(float) * c2o.size(), cudaMemcpyDefault);
    } else {
        for (uint32_t i = 0; i < d->nattr; ++i)
            for (int k = 0; k < 4; ++k) c2o[16 * (size_t)i + 5 * k] = 1.f;
    }
    cudaError_t e = cudaSuccess;
    for (const Material& m : mats)
        if (m.type == MAT_KELEMEN && e == cudaSuccess) e = ctx_kelemen_ensure(ctx, m.table);
    if (us) {
        sc->corner_n = cn;
        sc->corner_uv = cu;
        if (e == cudaSuccess) e = up_err;
    } else {
        if (e == cudaSuccess) e = upload(&sc->corner_n, d->corner_normals, 9 * (size_t)d->ntri, s);
        if (e == cudaSuccess) e = upload(&sc->corner_uv, d->corner_uvs, 6 * (size_t)d->ntri, s);
    }
    if (e == cudaSuccess) e = upload(&sc->attrs, attrs.data(), attrs.size(), s);
    if (e == cudaSuccess) e = upload(&sc->mats, mats.data(), mats.size(), s);
    if (e == cudaSuccess) e = upload(&sc->lights, lights.data(), lights.size(), s);
    if (e == cudaSuccess) e = upload(&sc->texs, texs.data(), texs.size(), s);
    if (e == cudaSuccess) e = upload(&sc->texels, d->texels, texel_floats, s);
    if (e == cudaSuccess) e = upload(&sc->attr_c2o, c2o.data(), c2o.size(), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { scene_free(sc); return cuda_fail(e, "aur_scene_create"); }
    sc->bvh.corner_n = sc->corner_n;       // aur_bvh_intersect on aur_scene_bvh reads the scene's arrays
    sc->bvh.corner_uv = sc->corner_uv;
    *out = sc;
    return AUR_OK;
}

aur_status aur_scene_destroy(aur_scene* sc) {
    if (!sc) return AUR_OK;
    DeviceGuard g(sc->ctx->device);
    scene_free(sc);
    return AUR_OK;
}

aur_status aur_scene_info(const aur_scene* sc, int32_t* w, int32_t* h, uint32_t* ntri, uint32_t* nmat,
                          uint32_t* ntexel) {
    if (!sc) return fail(AUR_ERR_INVALID_ARG, "aur_scene_info: NULL scene");
    if (w) *w = sc->cam.w;
    if (h) *h = sc->cam.h;
    if (ntri) *ntri = sc->ntri;
    if (nmat) *nmat = (uint32_t)sc->h_mats.size();
    if (ntexel) *ntexel = sc->ntexel_floats;
    return AUR_OK;
}

aur_status aur_scene_bvh(aur_scene* sc, aur_bvh** b) {
    if (!sc || !b) return fail(AUR_ERR_INVALID_ARG, "aur_scene_bvh: NULL argument");
    *b = &sc->bvh;
    return AUR_OK;
}

aur_status aur_scene_set_params(aur_scene* sc, const float* mp, const float* texels) {
    if (!sc) return fail(AUR_ERR_INVALID_ARG, "aur_scene_set_params: NULL scene");
    DeviceGuard g(sc->ctx->device);
    cudaStream_t s = sc->ctx->stream;
    if (mp) {
        std::vector<float> h(4 * sc->h_mats.size());
        CUDA_TRY(cudaMemcpy(h.data(), mp, sizeof(float) * h.size(), cudaMemcpyDefault), "aur_scene_set_params");
        for (size_t m = 0; m < sc->h_mats.size(); ++m) {
            sc->h_mats[m].diff = mk(h[4 * m], h[4 * m + 1], h[4 * m + 2]);
            sc->h_mats[m].rough = h[4 * m + 3];
        }
        CUDA_TRY(cudaMemcpyAsync(sc->mats, sc->h_mats.data(), sizeof(Material) * sc->h_mats.size(),
                                 cudaMemcpyHostToDevice, s), "aur_scene_set_params");
    }
    if (texels && sc->ntexel_floats) {
        CUDA_TRY(cudaMemcpyAsync(sc->texels, texels, sizeof(float) * sc->ntexel_floats, cudaMemcpyDefault, s),
                 "aur_scene_set_params");
    }
    CUDA_TRY(cudaStreamSynchronize(s), "aur_scene_set_params");
    return AUR_OK;
}

aur_status aur_scene_get_params(aur_scene* sc, float* mp, float* texels) {
    if (!sc) return fail(AUR_ERR_INVALID_ARG, "aur_scene_get_params: NULL scene");
    DeviceGuard g(sc->ctx->device);
    if (mp) {
        std::vector<float> h(4 * sc->h_mats.size());
        for (size_t m = 0; m < sc->h_mats.size(); ++m) {
            h[4 * m] = sc->h_mats[m].diff.x; h[4 * m + 1] = sc->h_mats[m].diff.y;
            h[4 * m + 2] = sc->h_mats[m].diff.z; h[4 * m + 3] = sc->h_mats[m].rough;
        }
        CUDA_TRY(cudaMemcpy(mp, h.data(), sizeof(float) * h.size(), cudaMemcpyDefault), "aur_scene_get_params");
    }
    if (texels && sc->ntexel_floats)
        CUDA_TRY(cudaMemcpy(texels, sc->texels, sizeof(float) * sc->ntexel_floats, cudaMemcpyDefault),
                 "aur_scene_get_params");
    return AUR_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ render
namespace aur {

aur_status render_options(const aur_scene* sc, const aur_render_opts* o, PathParams* p) {
    if (!o) return fail(AUR_ERR_INVALID_ARG, "render: options are NULL");
    if (o->spp <= 0) return fail(AUR_ERR_INVALID_ARG, "render: spp must be positive");
    if (o->max_depth < 1 || o->max_depth > 400) return fail(AUR_ERR_INVALID_ARG, "render: max_depth must be 1..400");
    if (o->light_samples < 0 || o->light_samples > 4096)
        return fail(AUR_ERR_INVALID_ARG, "render: light_samples must be 0..4096");
    const long long lmax = o->light_samples > 1 ? o->light_samples : 1;
    if (o->sample_offset < 0 || ((long long)o->sample_offset + o->spp) * lmax > (1 << 20))
        return fail(AUR_ERR_INVALID_ARG, "render: sample indices (times light_samples) must stay below 2^20");
    if (lmax > 1 && o->count_work) return fail(AUR_ERR_UNSUPPORTED, "render: count_work with light_samples > 1");
    p->light_samples = (int)lmax;
    p->max_depth = o->max_depth;
    p->min_depth = o->min_depth;
    p->spp = o->spp;
    p->sample_offset = o->sample_offset;
    p->seed = o->seed;
    (void)sc;
    return AUR_OK;
}

}  // namespace aur

static aur_status render_plain_impl(aur_scene* sc, const aur_render_opts* o, void* film, bool f64,
                                    aur_render_stats* stats) {
    if (!sc || !o || !film) return fail(AUR_ERR_INVALID_ARG, "aur_render: NULL argument");
    PathParams p;
    aur_status st = render_options(sc, o, &p);
    if (st != AUR_OK) return st;
    DeviceGuard g(sc->ctx->device);
    cudaStream_t s = sc->ctx->stream;
    const size_t npix = (size_t)sc->cam.w * sc->cam.h;
    DevOut fo, fo64;
    double* d64 = nullptr;
    float4* f32 = nullptr;
    if (f64) {
        CUDA_TRY(fo64.init(film, sizeof(double) * 4 * npix, 8, s), "aur_render(film)");
        d64 = (double*)fo64.ptr;
        CUDA_TRY(cudaMallocAsync(&f32, sizeof(float4) * npix, s), "aur_render(film)");
    } else {
        const bool fp64_acc = o->fp64_film != 0;
        CUDA_TRY(fo.init(film, sizeof(float4) * npix, 16, s), "aur_render(film)");
        f32 = (float4*)fo.ptr;
        if (fp64_acc) CUDA_TRY(cudaMallocAsync(&d64, sizeof(double) * 4 * npix, s), "aur_render(film)");
    }
    CUDA_TRY(cudaMemsetAsync(sc->ctx->counters, 0, sizeof(unsigned long long) * 8, s), "aur_render");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    cudaError_t e = launch_render_plain(sc->dev(), p, f32, d64, sc->ctx->counters, o->count_work != 0, s);
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = f64 ? fo64.finish() : fo.finish();
    unsigned long long cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, sc->ctx->counters, sizeof(cnt), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (f64) cudaFreeAsync(f32, s);
    else if (d64) cudaFreeAsync(d64, s);
    if (e != cudaSuccess) return cuda_fail(e, "aur_render");
    if (stats) {
        stats->camera_rays = cnt[0];
        stats->closest_rays = cnt[1];
        stats->shadow_rays = cnt[2];
        stats->paths = cnt[3];
        stats->node_visits = cnt[4];
        stats->tri_tests = cnt[5];
        stats->shadow_node_visits = cnt[6];
        stats->shadow_tri_tests = cnt[7];
        stats->launches = 1;
        stats->kernel_ms = ms;
        stats->node_bytes = o->count_work && sc->bvh.bvh.nodes4 ? (int32_t)sizeof(BvhNode4) : (int32_t)sizeof(BvhNode);
    }
    return AUR_OK;
}

namespace {

// acc += pass mean * n (FP64 per channel); mean = acc / done
__global__ void k_progressive(const float4* __restrict__ pass, double4* acc, float4* mean, uint32_t npix, double n,
                              double done) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const float4 p = pass[i];
    double4 a = acc[i];
    a.x += (double)p.x * n; a.y += (double)p.y * n; a.z += (double)p.z * n; a.w += (double)p.w * n;
    acc[i] = a;
    mean[i] = make_float4((float)(a.x / done), (float)(a.y / done), (float)(a.z / done), (float)(a.w / done));
}

}  // namespace

extern "C" {

aur_status aur_render_progressive(aur_scene* sc, const aur_render_opts* o, int32_t pass_spp, aur_pass_fn on_pass,
                                  void* user, float* film, aur_render_stats* stats) {
    if (!sc || !o || !film) return fail(AUR_ERR_INVALID_ARG, "aur_render_progressive: NULL argument");
    if (pass_spp < 1) return fail(AUR_ERR_INVALID_ARG, "aur_render_progressive: pass_spp must be >= 1");
    if (o->spp < 1) return fail(AUR_ERR_INVALID_ARG, "aur_render_progressive: spp must be >= 1");
    if (o->count_work || o->fp64_film) return fail(AUR_ERR_INVALID_ARG, "aur_render_progressive: count_work / fp64_film");
    DeviceGuard g(sc->ctx->device);
    cudaStream_t s = sc->ctx->stream;
    const uint32_t npix = (uint32_t)sc->cam.w * (uint32_t)sc->cam.h;
    float4 *pass = nullptr, *mean = nullptr;
    double4* acc = nullptr;
    std::vector<float> host;
    cudaError_t e = cudaMallocAsync(&pass, sizeof(float4) * npix, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&mean, sizeof(float4) * npix, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&acc, sizeof(double4) * npix, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(double4) * npix, s);
    auto release = [&]() {
        if (pass) cudaFreeAsync(pass, s);
        if (mean) cudaFreeAsync(mean, s);
        if (acc) cudaFreeAsync(acc, s);
        cudaStreamSynchronize(s);
    };
    if (e != cudaSuccess) { release(); return cuda_fail(e, "aur_render_progressive"); }
    aur_render_stats total;
    memset(&total, 0, sizeof(total));
    int32_t done = 0;
    aur_status st = AUR_OK;
    while (done < o->spp) {
        aur_render_opts po = *o;
        po.spp = std::min(pass_spp, o->spp - done);
        po.sample_offset = o->sample_offset + done;
        aur_render_stats ps;
        memset(&ps, 0, sizeof(ps));
        st = aur_render(sc, &po, (float*)pass, &ps);
        if (st != AUR_OK) break;
        done += po.spp;
        k_progressive<<<(npix + 255) / 256, 256, 0, s>>>(pass, acc, mean, npix, (double)po.spp, (double)done);
        e = cudaGetLastError();
        total.camera_rays += ps.camera_rays; total.closest_rays += ps.closest_rays;
        total.shadow_rays += ps.shadow_rays; total.paths += ps.paths;
        total.launches += ps.launches + 1; total.kernel_ms += ps.kernel_ms;
        for (int k = 0; k < 5; ++k) total.stage_ms[k] += ps.stage_ms[k];
        total.wf_pool = ps.wf_pool; total.wf_block = ps.wf_block; total.wf_sort = ps.wf_sort;
        total.node_bytes = ps.node_bytes;
        const bool last = done >= o->spp;
        if (e == cudaSuccess && on_pass && !last) {
            host.resize(4 * (size_t)npix);
            e = cudaMemcpyAsync(host.data(), mean, sizeof(float4) * npix, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e == cudaSuccess && on_pass(user, host.data(), done) != 0) break;   // the caller stops here
        }
        if (e != cudaSuccess) break;
    }
    if (st == AUR_OK && e == cudaSuccess)
        e = cudaMemcpyAsync(film, mean, sizeof(float4) * npix, cudaMemcpyDefault, s);
    if (st == AUR_OK && e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (st == AUR_OK && e == cudaSuccess && on_pass && done >= o->spp) {
        host.resize(4 * (size_t)npix);
        e = cudaMemcpy(host.data(), mean, sizeof(float4) * npix, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) on_pass(user, host.data(), done);
    }
    release();
    if (st != AUR_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "aur_render_progressive");
    if (stats) *stats = total;
    return AUR_OK;
}

aur_status aur_render(aur_scene* sc, const aur_render_opts* o, float* film, aur_render_stats* stats) {
    if (o && o->mode == AUR_RENDER_WAVEFRONT) return aur::render_wavefront(sc, o, film, stats);
    if (o && o->mode != AUR_RENDER_PLAIN) return fail(AUR_ERR_INVALID_ARG, "aur_render: unknown mode");
    return render_plain_impl(sc, o, film, false, stats);
}

aur_status aur_render_f64(aur_scene* sc, const aur_render_opts* o, double* film, aur_render_stats* stats) {
    return render_plain_impl(sc, o, film, true, stats);
}

}  // extern "C"
