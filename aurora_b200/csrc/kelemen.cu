// kelemen.cu — regenerates the Kelemen specular-albedo tables on the device.
//
// The reference loads 64x32 half-precision tables from EXR files that are not
// shipped (Aurora/src/shading/materials/kelemenMaterial.cpp:48-80); they were
// produced by KelemenMaterial::preCalcAlbedo (kelemenMaterial.cpp:113-178):
// for every (cos theta_i = max(1e-4, i/63), roughness_r = max(1e-5, r/31)),
// 250000 Beckmann half-vector samples estimate E[F(h.l) * max(0, l.n) / v.h]
// with Schlick F at reflectance k/20. This kernel restates that estimator with
// the counter-based RNG, FP64 accumulation and a fixed reduction order (so the
// table is bit-reproducible), then rounds to half like the EXR cache.
#include "aur_kernels.h"
#include <cuda_fp16.h>

namespace aur {
namespace {

constexpr int kSamples = 250000;     // SPECALBEDO_SAMPLES
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_kelemen_table(int refl_index, float* out) {
    const int entry = blockIdx.x;                 // i * 32 + r
    const int i = entry / kAlbedoRough, r = entry % kAlbedoRough;
    const float reflectance = (float)refl_index / (float)(kAlbedoRefl - 1);
    const float roughness = fmaxf(0.00001f, (float)r / (kAlbedoRough - 1.f));
    const float vz = fmaxf(0.0001f, (float)i / (float)(kAlbedoCos - 1));
    const uint64_t key = seed_key(0x4B454C00u + (uint32_t)refl_index);
    const uint64_t base = (uint64_t)entry << 32;
    double acc = 0.0;
    for (int j = threadIdx.x; j < kSamples; j += kThreads) {
        const uint64_t c = base | (uint64_t)(3 * j);
        const float r1 = rng_u01(key, c), r2 = rng_u01(key, c + 1), r3 = rng_u01(key, c + 2);
        float z = cosf(atanf(roughness * sqrtf(-logf(1.f - r1))));
        float rr = sqrtf(fmaxf(0.f, 1.f - z * z));
        float phi = kPi * 2.f * r2;
        float3 H = normalize(mk(rr * cosf(phi), rr * sinf(phi), z));
        const float3 N = mk(0.f, 0.f, 1.f);
        rr = sqrtf(fmaxf(0.f, 1.f - vz * vz));
        phi = r3 * 2.f * kPi;
        const float3 V = normalize(mk(rr * cosf(phi), rr * sinf(phi), vz));
        if (dot(H, V) < 0.f) H = -H;
        const float vdoth = dot(V, H);
        if (vdoth > 0.000001f) {
            const float3 L = normalize(H * 2.f * vdoth - V);
            const float F = schlick(dot(H, L), reflectance);
            const double a = (double)(F * fmaxf(0.f, dot(L, N)) / vdoth);
            acc += a / (double)((float)kSamples / 100.f);
        }
    }
    __shared__ double s[kThreads];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const float v = (float)(s[0] / 100.0);
        out[i * kAlbedoRough + r] = __half2float(__float2half_rn(v));
    }
}

}  // namespace

cudaError_t launch_kelemen_table(int refl_index, float* out, cudaStream_t s) {
    k_kelemen_table<<<kAlbedoCos * kAlbedoRough, kThreads, 0, s>>>(refl_index, out);
    return cudaGetLastError();
}

}  // namespace aur
