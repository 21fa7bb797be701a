// render_plain.cu — the plain renderer: one thread per pixel runs that pixel's
// spp camera paths back to back (Renderer::renderImage's spp passes of
// IntegrateParallel, Aurora/src/frontend/renderer.cpp:147-186,201-271, folded
// into one launch) and writes the running mean the reference keeps in
// OpenexrDisplay::appendValue (openexrDisplay.cpp:61-72). Accumulation is
// Neumaier-compensated FP32, or FP64 for oracle images.
#include "aur_kernels.h"

namespace aur {
namespace {

constexpr int kPlainBlock = 128;

// counters: camera rays, closest rays, shadow rays, paths, then (counting variant) node visits and
// triangle tests of closest-hit rays and of shadow rays
template <int kN>
__device__ __forceinline__ void add_counters(unsigned long long* counters, const uint32_t (&v_in)[kN]) {
    unsigned long long v[kN];
#pragma unroll
    for (int k = 0; k < kN; ++k) v[k] = v_in[k];
#pragma unroll
    for (int k = 0; k < kN; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < kN; ++k) atomicAdd(&counters[k], v[k]);
}

// kWidth: the tree traversed (2 binary, 4 four-wide). The timed kernels use the binary
// tree, on which this one-thread-per-path kernel is fastest (its code holds five
// traversals; the 4-wide ones made it 30% slower); the counting pass can use either, to
// count the work of the wavefront renderer's traversal.
// kMulti: light_samples > 1 (several paths per camera sample after the first pass); the
// one-path form keeps the single-path loop, whose code is smaller and 6% faster.
template <bool kFp64, bool kCount, int kWidth, bool kMulti>
__global__ void __launch_bounds__(kPlainBlock) k_render_plain(DevScene sc, PathParams p, float4* film,
                                                              double* film64, unsigned long long* counters) {
    const int npix = sc.cam.w * sc.cam.h;
    const int pixel = blockIdx.x * blockDim.x + threadIdx.x;
    RayCounts rc;
    uint32_t paths = 0;
    if (pixel < npix) {
        const int px = pixel % sc.cam.w, py = pixel / sc.cam.w;
        const uint64_t key = seed_key(p.seed);
        Kahan3 acc;
        acc.init();
        double d[3] = {0.0, 0.0, 0.0};
        float alpha_sum = 0.f;
        for (int s = 0; s < p.spp; ++s) {
            float a;
            int n = 1;
            float3 L;
            if (kMulti) {
                L = integrate_camera_sample<kWidth>(sc, p, px, py, (uint32_t)pixel, key, p.sample_offset + s, rc, &a, &n);
            } else {
                PathRng rng;
                rng.key = key;
                rng.base = path_base((uint32_t)pixel, (uint32_t)(p.sample_offset + s));
                L = integrate_path<kWidth>(sc, p, px, py, rng, rc, &a);
            }
            if (kFp64) { d[0] += L.x; d[1] += L.y; d[2] += L.z; }
            else acc.add(L);
            alpha_sum += a;
            paths += (uint32_t)n;
        }
        const float inv = 1.f / (float)p.spp;
        if (kFp64) {
            film64[4 * (size_t)pixel + 0] = d[0] / p.spp;
            film64[4 * (size_t)pixel + 1] = d[1] / p.spp;
            film64[4 * (size_t)pixel + 2] = d[2] / p.spp;
            film64[4 * (size_t)pixel + 3] = (double)alpha_sum / p.spp;
            film[pixel] = make_float4((float)(d[0] / p.spp), (float)(d[1] / p.spp), (float)(d[2] / p.spp),
                                      alpha_sum * inv);
        } else {
            const float3 t = acc.total();
            film[pixel] = make_float4(t.x * inv, t.y * inv, t.z * inv, alpha_sum * inv);
        }
    }
    if (kCount) {
        const uint32_t v[8] = {pixel < npix ? (uint32_t)p.spp : 0u, rc.closest, rc.shadow, paths, rc.work.nodes,
                               rc.work.tris, rc.shadow_work.nodes, rc.shadow_work.tris};
        add_counters<8>(counters, v);
    } else {
        const uint32_t v[4] = {pixel < npix ? (uint32_t)p.spp : 0u, rc.closest, rc.shadow, paths};
        add_counters<4>(counters, v);
    }
}

}  // namespace

cudaError_t launch_render_plain(const DevScene& sc, const PathParams& p, float4* film, double* film64,
                                unsigned long long* counters, bool count_work, cudaStream_t s) {
    const int npix = sc.cam.w * sc.cam.h;
    const int grid = (npix + kPlainBlock - 1) / kPlainBlock;
    const bool multi = p.light_samples > 1;
    if (film64 && multi) k_render_plain<true, false, 2, true><<<grid, kPlainBlock, 0, s>>>(sc, p, film, film64, counters);
    else if (film64) k_render_plain<true, false, 2, false><<<grid, kPlainBlock, 0, s>>>(sc, p, film, film64, counters);
    else if (count_work && multi) return cudaErrorNotSupported;   // the counting pass counts one path per sample
    else if (count_work && sc.nodes4)
        k_render_plain<false, true, 4, false><<<grid, kPlainBlock, 0, s>>>(sc, p, film, film64, counters);
    else if (count_work) k_render_plain<false, true, 2, false><<<grid, kPlainBlock, 0, s>>>(sc, p, film, film64, counters);
    else if (multi) k_render_plain<false, false, 2, true><<<grid, kPlainBlock, 0, s>>>(sc, p, film, film64, counters);
    else k_render_plain<false, false, 2, false><<<grid, kPlainBlock, 0, s>>>(sc, p, film, film64, counters);
    return cudaGetLastError();
}

}  // namespace aur
