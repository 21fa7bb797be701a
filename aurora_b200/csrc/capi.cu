// capi.cu — the C ABI of include/aurora_b200.h: contexts, the device BVH
// (EmbreeAccelerator replacement), flattened scenes and the render entry.
#include "aurora_b200.h"
#include "aur_kernels.h"
#include "aur_capi_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace aur;

// ------------------------------------------------------------------ errors
namespace {
thread_local std::string g_err;
}

namespace aur {
// flag |= 1 when any of the n indices is >= bound (a grid-stride scan; stream-ordered, no sync)
__global__ void k_check_below(const uint32_t* __restrict__ v, size_t n, uint32_t bound, uint32_t* flag) {
    uint32_t bad = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        bad |= v[i] >= bound ? 1u : 0u;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// Checks on the device that every index of v[0, n) is below bound (host or device inputs,
// after their upload). Synchronises the stream. *ok = false on an index out of range.
cudaError_t indices_below(const uint32_t* v, size_t n, uint32_t bound, bool* ok, cudaStream_t s) {
    *ok = true;
    if (n == 0) return cudaSuccess;
    uint32_t* flag = nullptr;
    cudaError_t e = cudaMallocAsync(&flag, sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) {
        const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 8);
        k_check_below<<<grid, 256, 0, s>>>(v, n, bound, flag);
        e = cudaGetLastError();
    }
    uint32_t h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (flag) cudaFreeAsync(flag, s);
    const cudaError_t se = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = se;
    *ok = h == 0;
    return e;
}
}  // namespace aur

namespace aur {
aur_status fail(aur_status s, const std::string& msg) {
    g_err = msg;
    return s;
}
aur_status cuda_fail(cudaError_t e, const char* where) {
    g_err = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? AUR_ERR_OOM : AUR_ERR_CUDA;
}

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

DeviceGuard::DeviceGuard(int dev) {
    cudaGetDevice(&prev_);
    if (prev_ != dev) cudaSetDevice(dev);
}
DeviceGuard::~DeviceGuard() { cudaSetDevice(prev_); }

// Device view of a caller array: the pointer itself when it already is device
// memory with the required alignment, else a stream-ordered staging copy.
cudaError_t DevIn::init(const void* p, size_t bytes, size_t align, cudaStream_t s) {
    stream = s;
    if (!p || bytes == 0) { ptr = nullptr; return cudaSuccess; }
    const bool dev = is_device_ptr(p);
    if (dev && ((uintptr_t)p % align) == 0) { ptr = p; return cudaSuccess; }
    cudaError_t e = cudaMallocAsync(&owned, bytes, s);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(owned, p, bytes, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
    ptr = owned;
    return e;
}
DevIn::~DevIn() { if (owned) cudaFreeAsync(owned, stream); }

cudaError_t DevOut::init(void* p, size_t bytes, size_t align, cudaStream_t s) {
    stream = s; user = p; size = bytes;
    if (is_device_ptr(p) && ((uintptr_t)p % align) == 0) { ptr = p; return cudaSuccess; }
    host = !is_device_ptr(p);
    cudaError_t e = cudaMallocAsync(&owned, bytes ? bytes : 1, s);
    ptr = owned;
    return e;
}
cudaError_t DevOut::finish() {
    if (!owned) return cudaSuccess;
    return cudaMemcpyAsync(user, owned, size, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, stream);
}
DevOut::~DevOut() { if (owned) cudaFreeAsync(owned, stream); }

cudaError_t ctx_kelemen_tables(aur_ctx* ctx) {
    if (!ctx->kelemen) {
        cudaError_t e = cudaMalloc(&ctx->kelemen, sizeof(float) * kAlbedoRefl * kAlbedoCos * kAlbedoRough);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
cudaError_t ctx_scratch(aur_ctx* ctx, size_t bytes, void** out) {
    if (bytes > ctx->scratch_bytes) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);   // the old buffer may still be in use
        if (e != cudaSuccess) return e;
        if (ctx->scratch) cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
        e = cudaMalloc(&ctx->scratch, bytes);
        if (e != cudaSuccess) return e;
        ctx->scratch_bytes = bytes;
    }
    *out = ctx->scratch;
    return cudaSuccess;
}

cudaError_t ctx_kelemen_ensure(aur_ctx* ctx, int refl_index) {
    cudaError_t e = ctx_kelemen_tables(ctx);
    if (e != cudaSuccess) return e;
    if (ctx->kel_ready[refl_index]) return cudaSuccess;
    e = launch_kelemen_table(refl_index, ctx->kelemen + (size_t)refl_index * kAlbedoCos * kAlbedoRough, ctx->stream);
    if (e == cudaSuccess) ctx->kel_ready[refl_index] = true;
    return e;
}
int kelemen_index(float reflectance) {
    int k = (int)roundf(reflectance * (kAlbedoRefl - 1));
    return k < 0 ? 0 : (k > kAlbedoRefl - 1 ? kAlbedoRefl - 1 : k);
}
}  // namespace aur


extern "C" {

const char* aur_last_error(void) { return g_err.c_str(); }

const char* aur_status_string(aur_status s) {
    switch (s) {
        case AUR_OK: return "AUR_OK";
        case AUR_ERR_INVALID_ARG: return "AUR_ERR_INVALID_ARG";
        case AUR_ERR_OOM: return "AUR_ERR_OOM";
        case AUR_ERR_CUDA: return "AUR_ERR_CUDA";
        case AUR_ERR_TIMEOUT: return "AUR_ERR_TIMEOUT";
        case AUR_ERR_QUEUE_OVERFLOW: return "AUR_ERR_QUEUE_OVERFLOW";
        case AUR_ERR_PARSE: return "AUR_ERR_PARSE";
        case AUR_ERR_IO: return "AUR_ERR_IO";
        case AUR_ERR_UNSUPPORTED: return "AUR_ERR_UNSUPPORTED";
    }
    return "AUR_ERR_UNKNOWN";
}

const char* aur_version(void) { return "aurora-b200 0.1 (sm_100a)"; }

aur_status aur_ctx_create(int device, aur_ctx** out) {
    if (!out) return fail(AUR_ERR_INVALID_ARG, "aur_ctx_create: out is NULL");
    *out = nullptr;
    int n = 0;
    CUDA_TRY(cudaGetDeviceCount(&n), "aur_ctx_create");
    if (device < 0 || device >= n) return fail(AUR_ERR_INVALID_ARG, "aur_ctx_create: no such CUDA device");
    DeviceGuard g(device);
    aur_ctx* c = new aur_ctx();
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return cuda_fail(e, "aur_ctx_create"); }
    c->own_stream = true;
    e = cudaMalloc(&c->counters, sizeof(unsigned long long) * 8);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->work_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        // Scene and BVH buffers come from the device's stream-ordered pool; keeping freed
        // blocks reserved (instead of trimming at every synchronisation) makes a new scene's
        // allocations reuse them rather than map fresh memory. aur_ctx_destroy trims it.
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_order, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (c->counters) cudaFree(c->counters);
        if (c->work_stream) cudaStreamDestroy(c->work_stream);
        cudaStreamDestroy(c->stream);
        delete c;
        return cuda_fail(e, "aur_ctx_create");
    }
    *out = c;
    return AUR_OK;
}


aur_status aur_ctx_destroy(aur_ctx* ctx) {
    if (!ctx) return AUR_OK;
    if (ctx->live > 0)
        return fail(AUR_ERR_INVALID_ARG, "aur_ctx_destroy: destroy the context's scenes and BVHs first");
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    wf_release_context(ctx);
    if (ctx->kelemen) cudaFree(ctx->kelemen);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->counters) cudaFree(ctx->counters);
    if (ctx->work_stream) { cudaStreamSynchronize(ctx->work_stream); cudaStreamDestroy(ctx->work_stream); }
    if (ctx->ev_order) cudaEventDestroy(ctx->ev_order);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(pool, 0);
    }
    cudaGetLastError();
    delete ctx;
    return AUR_OK;
}

aur_status aur_ctx_set_stream(aur_ctx* ctx, void* stream) {
    if (!ctx) return fail(AUR_ERR_INVALID_ARG, "aur_ctx_set_stream: ctx is NULL");
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    if (stream) { ctx->stream = (cudaStream_t)stream; ctx->own_stream = false; }
    else {
        CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "aur_ctx_set_stream");
        ctx->own_stream = true;
    }
    return AUR_OK;
}

aur_status aur_ctx_synchronize(aur_ctx* ctx) {
    if (!ctx) return fail(AUR_ERR_INVALID_ARG, "aur_ctx_synchronize: ctx is NULL");
    DeviceGuard g(ctx->device);
    CUDA_TRY(cudaStreamSynchronize(ctx->stream), "aur_ctx_synchronize");
    return AUR_OK;
}

// ------------------------------------------------------------------ BVH
aur_status aur_bvh_build(aur_ctx* ctx, const float* verts, uint32_t nvert, const uint32_t* tri_vidx,
                         const int32_t* tri_attr, uint32_t ntri, const aur_bvh_opts* opts, aur_bvh** out) {
    if (!ctx || !out || !verts || !tri_vidx) return fail(AUR_ERR_INVALID_ARG, "aur_bvh_build: NULL argument");
    *out = nullptr;
    if (ntri == 0 || nvert == 0) return fail(AUR_ERR_INVALID_ARG, "aur_bvh_build: empty triangle set");
    if (ntri >= (1u << 26)) return fail(AUR_ERR_UNSUPPORTED, "aur_bvh_build: more than 2^26 triangles");
    BvhBuildOptions bo;
    aur_status st = bvh_options(opts, &bo);
    if (st != AUR_OK) return st;
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    DevIn dv, di, da;
    CUDA_TRY(dv.init(verts, sizeof(float) * 3 * nvert, 4, s), "aur_bvh_build(upload)");
    CUDA_TRY(di.init(tri_vidx, sizeof(uint32_t) * 3 * ntri, 4, s), "aur_bvh_build(upload)");
    // vertex indices must be in range before any build kernel reads vertices through them:
    // checked on the device copy (host and device inputs alike)
    bool in_range = true;
    CUDA_TRY(indices_below((const uint32_t*)di.ptr, 3 * (size_t)ntri, nvert, &in_range, s), "aur_bvh_build(check)");
    if (!in_range) return fail(AUR_ERR_INVALID_ARG, "aur_bvh_build: vertex index out of range");
    aur_bvh* b = new aur_bvh();
    b->ctx = ctx;
    cudaError_t e = bvh_build_device((const float*)dv.ptr, (const uint32_t*)di.ptr, (int)ntri, bo, &b->bvh, s);
    if (e == cudaSuccess && b->bvh.depth >= kTraversalStack) {
        bvh_free_device(&b->bvh, s);
        delete b;
        return fail(AUR_ERR_UNSUPPORTED, "aur_bvh_build: tree deeper than the traversal stack");
    }
    if (e == cudaSuccess) e = bvh_collapse4(&b->bvh, s);
    if (e == cudaSuccess && 3 * b->bvh.depth4 + 1 > kTraversalStack4) {
        // a 4-wide node pushes up to three entries: too deep for its stack, keep the binary tree only
        cudaFreeAsync(b->bvh.nodes4, s);
        b->bvh.nodes4 = nullptr;
        b->bvh.num_nodes4 = 0;
    }
    if (e == cudaSuccess && tri_attr) {
        e = cudaMallocAsync(&b->tri_attr, sizeof(int) * ntri, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->tri_attr, tri_attr, sizeof(int) * ntri,
                                is_device_ptr(tri_attr) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
        b->owns_attr = true;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        bvh_free_device(&b->bvh, s);
        if (b->tri_attr) cudaFreeAsync(b->tri_attr, s);
        delete b;
        return cuda_fail(e, "aur_bvh_build");
    }
    ++ctx->live;
    *out = b;
    return AUR_OK;
}

aur_status aur_bvh_destroy(aur_bvh* b) {
    if (!b) return AUR_OK;
    if (b->owned_by_scene) return fail(AUR_ERR_INVALID_ARG, "aur_bvh_destroy: BVH belongs to a scene");
    --b->ctx->live;
    DeviceGuard g(b->ctx->device);
    bvh_free_device(&b->bvh, b->ctx->stream);
    if (b->owns_attr && b->tri_attr) cudaFreeAsync(b->tri_attr, b->ctx->stream);
    if (b->owns_shading && b->corner_n) cudaFreeAsync(b->corner_n, b->ctx->stream);
    if (b->owns_shading && b->corner_uv) cudaFreeAsync(b->corner_uv, b->ctx->stream);
    cudaStreamSynchronize(b->ctx->stream);
    delete b;
    return AUR_OK;
}

aur_status aur_bvh_info(const aur_bvh* b, uint32_t* num_nodes, uint32_t* depth, float bounds[6]) {
    if (!b) return fail(AUR_ERR_INVALID_ARG, "aur_bvh_info: NULL bvh");
    if (num_nodes) *num_nodes = (uint32_t)b->bvh.num_nodes;
    if (depth) *depth = (uint32_t)b->bvh.depth;
    if (bounds) for (int k = 0; k < 3; ++k) { bounds[k] = b->bvh.lo[k]; bounds[3 + k] = b->bvh.hi[k]; }
    return AUR_OK;
}

aur_status aur_trace_closest(aur_bvh* b, const aur_ray* rays, aur_hit* hits, uint32_t n) {
    if (!b || (n && (!rays || !hits))) return fail(AUR_ERR_INVALID_ARG, "aur_trace_closest: NULL argument");
    if (n == 0) return AUR_OK;
    DeviceGuard g(b->ctx->device);
    cudaStream_t s = b->ctx->stream;
    DevIn dr;
    DevOut dh;
    CUDA_TRY(dr.init(rays, sizeof(aur_ray) * n, 16, s), "aur_trace_closest(rays)");
    CUDA_TRY(dh.init(hits, sizeof(aur_hit) * n, 4, s), "aur_trace_closest(hits)");
    CUDA_TRY(launch_trace_closest(b->bvh, b->tri_attr, dr.ptr, dh.ptr, n, s), "aur_trace_closest");
    CUDA_TRY(dh.finish(), "aur_trace_closest(download)");
    CUDA_TRY(cudaStreamSynchronize(s), "aur_trace_closest");
    return AUR_OK;
}

aur_status aur_trace_occluded(aur_bvh* b, const aur_ray* rays, uint8_t* occluded, uint32_t n) {
    if (!b || (n && (!rays || !occluded))) return fail(AUR_ERR_INVALID_ARG, "aur_trace_occluded: NULL argument");
    if (n == 0) return AUR_OK;
    DeviceGuard g(b->ctx->device);
    cudaStream_t s = b->ctx->stream;
    DevIn dr;
    DevOut dh;
    CUDA_TRY(dr.init(rays, sizeof(aur_ray) * n, 16, s), "aur_trace_occluded(rays)");
    CUDA_TRY(dh.init(occluded, n, 1, s), "aur_trace_occluded(out)");
    CUDA_TRY(launch_trace_occluded(b->bvh, dr.ptr, (uint8_t*)dh.ptr, n, s), "aur_trace_occluded");
    CUDA_TRY(dh.finish(), "aur_trace_occluded(download)");
    CUDA_TRY(cudaStreamSynchronize(s), "aur_trace_occluded");
    return AUR_OK;
}

aur_status aur_kelemen_table(aur_ctx* ctx, float reflectance, float* out) {
    if (!ctx || !out) return fail(AUR_ERR_INVALID_ARG, "aur_kelemen_table: NULL argument");
    DeviceGuard g(ctx->device);
    const int k = kelemen_index(reflectance);
    CUDA_TRY(ctx_kelemen_ensure(ctx, k), "aur_kelemen_table");
    DevOut o;
    CUDA_TRY(o.init(out, sizeof(float) * kAlbedoCos * kAlbedoRough, 4, ctx->stream), "aur_kelemen_table");
    CUDA_TRY(cudaMemcpyAsync(o.ptr, ctx->kelemen + (size_t)k * kAlbedoCos * kAlbedoRough,
                             sizeof(float) * kAlbedoCos * kAlbedoRough, cudaMemcpyDeviceToDevice, ctx->stream),
             "aur_kelemen_table");
    CUDA_TRY(o.finish(), "aur_kelemen_table");
    CUDA_TRY(cudaStreamSynchronize(ctx->stream), "aur_kelemen_table");
    return AUR_OK;
}

}  // extern "C"
