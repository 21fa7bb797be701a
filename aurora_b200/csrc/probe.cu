// probe.cu — aur_shading_probe: evaluates the device shading functions on
// caller-given inputs, one thread per record, so that BRDF values, pdfs, MIS
// weights, Kelemen lookups, camera and light sampling can be compared with a
// CPU restatement value by value. Record layouts are documented in aurora_b200.h.
#include "aur_capi_internal.h"

using namespace aur;

namespace {

constexpr int kKinds = 11;
constexpr int kInH[kKinds] = {13, 14, 14, 3, 7, 2, 9, 9, 7, 11, 12};
constexpr int kOutH[kKinds] = {7, 3, 1, 1, 3, 1, 8, 2, 1, 5, 11};
__constant__ int kIn[kKinds] = {13, 14, 14, 3, 7, 2, 9, 9, 7, 11, 12};
__constant__ int kOut[kKinds] = {7, 3, 1, 1, 3, 1, 8, 2, 1, 5, 11};

__global__ void k_probe(int kind, const float* in, uint32_t n, float* out, ShadeScene sh, const float* tables) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* q = in + (size_t)i * kIn[kind];
    float* o = out + (size_t)i * kOut[kind];
    if (kind <= 2) {
        Brdf b;
        b.lobe = (int)q[0];
        b.color = mk(q[1], q[2], q[3]);
        b.rough = q[4];
        if (kind == 0) {
            BrdfSample s = brdf_sample(b, mk(q[5], q[6], q[7]), mk(q[8], q[9], q[10]), q[11], q[12]);
            o[0] = s.dir.x; o[1] = s.dir.y; o[2] = s.dir.z; o[3] = s.pdf;
            o[4] = s.color.x; o[5] = s.color.y; o[6] = s.color.z;
        } else {
            const float3 L = mk(q[5], q[6], q[7]), V = mk(q[8], q[9], q[10]), N = mk(q[11], q[12], q[13]);
            if (kind == 1) { float3 c = brdf_eval(b, L, V, N); o[0] = c.x; o[1] = c.y; o[2] = c.z; }
            else o[0] = brdf_pdf(b, L, V, N);
        }
    } else if (kind == 3) {
        o[0] = kelemen_albedo(tables + (size_t)q[0] * kAlbedoCos * kAlbedoRough, q[1], q[2]);
    } else if (kind == 4) {
        Camera c; c.fov = q[0]; c.w = (int)q[1]; c.h = (int)q[2];
        RayF r = camera_ray(c, (int)q[3], (int)q[4], q[5], q[6]);
        o[0] = r.d.x; o[1] = r.d.y; o[2] = r.d.z;
    } else if (kind == 5) {
        o[0] = power_heuristic(q[0], q[1]);
    } else if (kind == 6) {
        LightSample s = light_sample(sh, sh.lights[(int)q[0]], mk(q[1], q[2], q[3]), mk(q[6], q[7], q[8]), q[4], q[5]);
        o[0] = s.dir.x; o[1] = s.dir.y; o[2] = s.dir.z; o[3] = s.maxt; o[4] = s.pdf;
        o[5] = s.color.x; o[6] = s.color.y; o[7] = s.color.z;
    } else if (kind == 7) {
        float maxt = q[8];
        o[0] = light_pdf(sh, sh.lights[(int)q[0]], mk(q[1], q[2], q[3]), mk(q[4], q[5], q[6]), q[7], &maxt);
        o[1] = maxt;
    } else if (kind == 8) {
        o[0] = light_visible(sh.lights[(int)q[0]], mk(q[1], q[2], q[3]), mk(q[4], q[5], q[6])) ? 1.f : 0.f;
    } else if (kind == 9) {
        Frame f;
        f.P = mk(0.f, 0.f, 0.f);
        f.V = mk(q[1], q[2], q[3]);
        f.N = f.Ng = mk(q[4], q[5], q[6]);
        f.su = q[7]; f.sv = q[8];
        f.attr = 0;
        Brdf b = get_brdf(sh, (int)q[0], f, q[9] != 0.f, q[10]);
        o[0] = (float)b.lobe; o[1] = b.color.x; o[2] = b.color.y; o[3] = b.color.z; o[4] = b.rough;
    } else {
        const Frame f = hit_frame(sh, (int)q[0], q[1], q[2], q[3], mk(q[4], q[5], q[6]), mk(q[7], q[8], q[9]), true);
        Brdf b = get_brdf(sh, sh.attrs[f.attr].material, f, q[10] != 0.f, q[11]);
        o[0] = f.N.x; o[1] = f.N.y; o[2] = f.N.z; o[3] = f.Ng.x; o[4] = f.Ng.y; o[5] = f.Ng.z;
        o[6] = (float)b.lobe; o[7] = b.color.x; o[8] = b.color.y; o[9] = b.color.z; o[10] = b.rough;
    }
}

}  // namespace

extern "C" aur_status aur_shading_probe(aur_ctx* ctx, aur_scene* scene, int kind, const float* in, uint32_t n,
                                        float* out) {
    if (!ctx || (n && (!in || !out))) return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: NULL argument");
    if (kind < 0 || kind >= kKinds) return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: unknown kind");
    if (kind >= 6 && !scene) return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: this kind needs a scene");
    if (n == 0) return AUR_OK;
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    // validate indices on the host before any device access
    std::vector<float> h((size_t)n * kInH[kind]);
    if (cudaMemcpy(h.data(), in, sizeof(float) * h.size(), cudaMemcpyDefault) != cudaSuccess)
        return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: cannot read inputs");
    for (uint32_t i = 0; i < n; ++i) {
        const float idx = h[(size_t)i * kInH[kind]];
        if (kind <= 2 && (idx < 0.f || idx > 4.f)) return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: bad lobe");
        if (kind == 3) {
            if (idx < 0.f || idx > 20.f) return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: bad table");
            cudaError_t e = ctx_kelemen_ensure(ctx, (int)idx);
            if (e != cudaSuccess) return cuda_fail(e, "aur_shading_probe");
        }
        if (kind >= 6 && kind <= 8 && (idx < 0.f || idx >= (float)scene->h_lights.size()))
            return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: bad light index");
        if (kind == 9 && (idx < 0.f || idx >= (float)scene->h_mats.size()))
            return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: bad material index");
        if (kind == 10 && (idx < 0.f || idx >= (float)scene->ntri))
            return fail(AUR_ERR_INVALID_ARG, "aur_shading_probe: bad triangle index");
    }
    DevIn di;
    DevOut dout;
    cudaError_t e = di.init(h.data(), sizeof(float) * h.size(), 4, s);
    if (e == cudaSuccess) e = dout.init(out, sizeof(float) * (size_t)n * kOutH[kind], 4, s);
    ShadeScene sh{};
    if (scene) sh = scene->dev().sh;
    if (e == cudaSuccess) {
        k_probe<<<(n + 127) / 128, 128, 0, s>>>(kind, (const float*)di.ptr, n, (float*)dout.ptr, sh, ctx->kelemen);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = dout.finish();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "aur_shading_probe");
    return AUR_OK;
}
