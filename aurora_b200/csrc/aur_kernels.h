// aur_kernels.h — host-side launch wrappers of the sm_100a kernels (internal).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "aur_bvh.cuh"
#include "aur_integrator.cuh"

namespace aur {

// trace.cu — batched ray queries (aur_ray / aur_hit layouts of aurora_b200.h)
cudaError_t launch_trace_closest(const DeviceBvh& bvh, const int* tri_attr, const void* rays, void* hits, uint32_t n,
                                 cudaStream_t s);
cudaError_t launch_trace_occluded(const DeviceBvh& bvh, const void* rays, uint8_t* occ, uint32_t n, cudaStream_t s);

// kelemen.cu — directional-albedo table for reflectance index 0..20 into out[2048]
cudaError_t launch_kelemen_table(int refl_index, float* out, cudaStream_t s);

// render_plain.cu — one thread per pixel, spp paths per thread.
// counters[0..3] = camera rays, closest rays, shadow rays, paths; with count_work
// also [4..5] interior-node visits / triangle tests of closest-hit rays and
// [6..7] those of shadow rays (accumulated).
cudaError_t launch_render_plain(const DevScene& sc, const PathParams& p, float4* film, double* film64,
                                unsigned long long* counters, bool count_work, cudaStream_t s);

}  // namespace aur
