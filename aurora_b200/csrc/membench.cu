// membench.cu — read bandwidth of one memory level, the denominator of the traversal
// roofline. The traversal kernels fetch node and triangle records that the L1 and
// the L2 serve for the most part (a scene's BVH is reused by every ray), so their
// algorithmic bytes are set against the L2's read bandwidth as well as against HBM's.
// No reference counterpart (the reference has no device code).
//
// A buffer of `bytes` is read `reps` times by a resident grid with 128-bit loads that
// bypass L1 (ld.global.cg): below the L2's 126 MB every pass after the first is
// served by the L2, above it by HBM.
#include "aur_capi_internal.h"

namespace aur {
namespace {

constexpr int kBwBlock = 512;
constexpr int kBwUnroll = 4;

__global__ void __launch_bounds__(kBwBlock) k_read_bw(const float4* __restrict__ p, size_t n4, int reps,
                                                      float* __restrict__ sink) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    float acc = 0.f;
    for (int r = 0; r < reps; ++r) {
        size_t i = t;
        for (; i + (kBwUnroll - 1) * stride < n4; i += kBwUnroll * stride) {
            float4 v[kBwUnroll];
#pragma unroll
            for (int k = 0; k < kBwUnroll; ++k) v[k] = __ldcg(p + i + k * stride);
#pragma unroll
            for (int k = 0; k < kBwUnroll; ++k) acc += (v[k].x + v[k].y) + (v[k].z + v[k].w);
        }
        for (; i < n4; i += stride) {
            const float4 v = __ldcg(p + i);
            acc += (v.x + v.y) + (v.z + v.w);
        }
    }
    if (acc == 1.2345e-30f) sink[0] = acc;   // never true for the zero-filled buffer; keeps the loads
}

}  // namespace
}  // namespace aur

using namespace aur;

extern "C" aur_status aur_measure_read_bandwidth(aur_ctx* ctx, uint64_t bytes, int32_t reps, double* gb_per_s) {
    if (!ctx || !gb_per_s || reps < 1 || bytes < (1u << 20))
        return fail(AUR_ERR_INVALID_ARG, "aur_measure_read_bandwidth: NULL argument, reps < 1 or bytes < 1 MiB");
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t n4 = (size_t)(bytes / sizeof(float4));
    void* buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, n4 * sizeof(float4) + sizeof(float4), s);
    if (e != cudaSuccess) return cuda_fail(e, "aur_measure_read_bandwidth");
    float* sink = (float*)((float4*)buf + n4);
    e = cudaMemsetAsync(buf, 0, n4 * sizeof(float4) + sizeof(float4), s);
    int dev_sms = 0, per_sm = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_read_bw, kBwBlock, 0);
    const int grid = dev_sms * (per_sm > 0 ? per_sm : 1);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {   // one untimed pass brings the buffer into the L2 (when it fits)
        k_read_bw<<<grid, kBwBlock, 0, s>>>((const float4*)buf, n4, 1, sink);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) {
        k_read_bw<<<grid, kBwBlock, 0, s>>>((const float4*)buf, n4, reps, sink);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFreeAsync(buf, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_fail(e, "aur_measure_read_bandwidth");
    *gb_per_s = ms > 0.f ? (double)n4 * sizeof(float4) * reps / (ms * 1e-3) / 1e9 : 0.0;
    return AUR_OK;
}
