// aur_capi_internal.h — handle layouts and helpers shared by the C-ABI sources.
#pragma once
#include "aurora_b200.h"
#include "aur_kernels.h"
#include <array>
#include <map>
#include <string>
#include <vector>

struct aur_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    float* kelemen = nullptr;                  // 21 tables x 2048 floats
    bool kel_ready[aur::kAlbedoRefl] = {};
    unsigned long long* counters = nullptr;    // 8 render counters
    cudaStream_t work_stream = nullptr;        // non-blocking stream for captured work (wavefront graphs)
    cudaEvent_t ev_order = nullptr;            // orders work_stream after `stream`
    std::map<uint64_t, std::array<int, 3>> wf_batch_tuned;   // autotuned batch configs (pool, block, sort)
    std::map<uint64_t, std::array<int, 3>> wf_scene_tuned;   // autotuned configs by scene signature
    int live = 0;                              // BVHs and scenes created on this context and not destroyed
    void* scratch = nullptr;                   // grow-only device scratch (adjoint hit records)
    size_t scratch_bytes = 0;
};

struct aur_bvh {
    aur_ctx* ctx = nullptr;
    aur::DeviceBvh bvh;
    int* tri_attr = nullptr;                   // device, per original triangle id
    bool owns_attr = false;
    bool owned_by_scene = false;
    // per-corner normals (9 floats) and uvs (6 floats) per triangle for aur_bvh_intersect:
    // the scene's arrays for a scene's BVH, else uploaded by aur_bvh_set_shading (owned)
    float* corner_n = nullptr;
    float* corner_uv = nullptr;
    bool owns_shading = false;
};

struct aur_scene {
    aur_ctx* ctx = nullptr;
    aur_bvh bvh;                               // owned_by_scene = true
    // device buffers
    float* corner_n = nullptr;
    float* corner_uv = nullptr;
    aur::Attr* attrs = nullptr;
    aur::Material* mats = nullptr;
    aur::Light* lights = nullptr;
    aur::Texture* texs = nullptr;
    float* texels = nullptr;
    float* attr_c2o = nullptr;                 // 16 floats per attribute
    // host copies
    std::vector<aur::Material> h_mats;
    std::vector<aur::Light> h_lights;
    std::vector<aur::Texture> h_texs;
    uint32_t ntri = 0, nattr = 0, ntexel_floats = 0;
    aur::Camera cam{};
    bool wf_tuned = false;                     // autotuned wavefront configuration
    int wf_pool = 0, wf_block = 0, wf_sort = 0;
    aur::DevScene dev() const;
};

#define CUDA_TRY(x, where) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return aur::cuda_fail(e_, where); } while (0)

namespace aur {

aur_status fail(aur_status s, const std::string& msg);
aur_status cuda_fail(cudaError_t e, const char* where);
bool is_device_ptr(const void* p);
// Checks on the device that v[0, n) < bound (device pointer v); synchronises the stream.
cudaError_t indices_below(const uint32_t* v, size_t n, uint32_t bound, bool* ok, cudaStream_t s);
cudaError_t ctx_kelemen_ensure(aur_ctx* ctx, int refl_index);
// The context's scratch buffer of at least `bytes` (kept and reused by later calls;
// freed with the context). Work on the context's stream must not still use it.
cudaError_t ctx_scratch(aur_ctx* ctx, size_t bytes, void** out);
int kelemen_index(float reflectance);
aur_status bvh_options(const aur_bvh_opts* o, BvhBuildOptions* out);
aur_status render_options(const aur_scene* sc, const aur_render_opts* o, PathParams* p);
aur_status render_wavefront(aur_scene* sc, const aur_render_opts* o, float* film, aur_render_stats* stats);
void wf_release_context(aur_ctx* ctx);   // frees the wavefront engines cached for a context
aur_status wf_record_pass(aur_scene* sc, const PathParams& p, int s0, int nsamples, float4* rec, float4* lo_raw,
                          uint64_t* launches, unsigned long long* rays);

struct DeviceGuard {
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
    int prev_ = 0;
};

struct DevIn {
    const void* ptr = nullptr;
    void* owned = nullptr;
    cudaStream_t stream = nullptr;
    cudaError_t init(const void* p, size_t bytes, size_t align, cudaStream_t s);
    ~DevIn();
};

struct DevOut {
    void* ptr = nullptr;
    void* owned = nullptr;
    void* user = nullptr;
    size_t size = 0;
    bool host = false;
    cudaStream_t stream = nullptr;
    cudaError_t init(void* p, size_t bytes, size_t align, cudaStream_t s);
    cudaError_t finish();
    ~DevOut();
};

}  // namespace aur
