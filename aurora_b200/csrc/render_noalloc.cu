// render_noalloc.cu — aur_render_fp64acc_noalloc: the plain renderer with FP64
// accumulation, for callers that cannot allocate device memory.
//
// Some host applications own every byte of device memory through their own
// allocator or a hard budget (a DCC or game-engine plugin host, a service that
// pre-reserves its GPU memory), and a library call that allocates behind their
// back would fail or break their accounting. This entry point writes into the
// caller's film and keeps its scratch — the per-pixel FP64 accumulators and
// the ray counters — in file-scope static device arrays that every GPU loading
// the library holds until process exit (2 MiB + 64 B). It calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// Limits and sharing rules:
//   * at most kMaxPixels = 65536 pixels (e.g. 256 x 256); larger films, and
//     cameras with no pixels, are rejected with AUR_ERR_INVALID_ARG;
//   * the film must be device memory of the scene's device (or managed
//     memory), 16-byte aligned; a film on another device is rejected;
//   * opts->fp64_film must be 1 (this renderer accumulates in FP64 only) and
//     opts->count_work 0 (it has no counting pass): other values are refused;
//   * every call looks up the arrays' device addresses (cudaGetSymbolAddress,
//     a host-side lookup) with the scene's device current, so a reset device
//     or another driver context of the same device gets its own addresses.
//     The first call on a device may load the library's device code there;
//     make that first call before any stream capture on the device;
//   * every call shares the same arrays and they keep the last call's
//     contents: the counters are cleared at the start of each call, the
//     accumulators are fully overwritten. Calls that overlap on the GPU (two
//     streams, two host threads) race on the arrays and must be serialised by
//     the caller.
#include "aur_capi_internal.h"

using namespace aur;

namespace {

constexpr int kMaxPixels = 256 * 256;

static __device__ __align__(256) double g_accum[4 * kMaxPixels];
static __device__ __align__(256) unsigned long long g_counters[8];

struct Addresses {
    double* accum = nullptr;
    unsigned long long* counters = nullptr;
};

// Host code must not hand the kernel the arrays' host-side names: their device
// addresses are looked up with the device current (the caller's DeviceGuard).
aur_status device_addresses(Addresses* out) {
    cudaError_t e = cudaGetSymbolAddress((void**)&out->accum, g_accum);
    if (e != cudaSuccess) return cuda_fail(e, "aur_render_fp64acc_noalloc(cudaGetSymbolAddress)");
    e = cudaGetSymbolAddress((void**)&out->counters, g_counters);
    if (e != cudaSuccess) return cuda_fail(e, "aur_render_fp64acc_noalloc(cudaGetSymbolAddress)");
    return AUR_OK;
}

// The film: device memory of `device` (or managed memory), 16-byte aligned.
bool film_ok(const void* film, int device) {
    if (((uintptr_t)film % 16) != 0) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, film) != cudaSuccess) { cudaGetLastError(); return false; }
    return (a.type == cudaMemoryTypeDevice && a.device == device) || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" aur_status aur_render_fp64acc_noalloc(aur_scene* sc, const aur_render_opts* o, float* film,
                                                 aur_render_stats* stats) {
    if (!sc || !o || !film) return fail(AUR_ERR_INVALID_ARG, "aur_render_fp64acc_noalloc: NULL argument");
    if (o->mode != AUR_RENDER_PLAIN)
        return fail(AUR_ERR_INVALID_ARG, "aur_render_fp64acc_noalloc: only the plain renderer is available");
    if (o->fp64_film != 1)
        return fail(AUR_ERR_UNSUPPORTED, "aur_render_fp64acc_noalloc: accumulates in FP64 only (set fp64_film = 1)");
    if (o->count_work)
        return fail(AUR_ERR_UNSUPPORTED, "aur_render_fp64acc_noalloc: no work-counting pass (count_work must be 0)");
    const long long npix = (long long)sc->cam.w * sc->cam.h;
    if (sc->cam.w <= 0 || sc->cam.h <= 0)
        return fail(AUR_ERR_INVALID_ARG, "aur_render_fp64acc_noalloc: the camera has no pixels");
    if (npix > kMaxPixels)
        return fail(AUR_ERR_INVALID_ARG, "aur_render_fp64acc_noalloc: film larger than 65536 pixels (the static "
                                         "scratch holds 256x256)");
    PathParams p;
    aur_status st = render_options(sc, o, &p);
    if (st != AUR_OK) return st;
    DeviceGuard g(sc->ctx->device);
    if (!film_ok(film, sc->ctx->device))
        return fail(AUR_ERR_INVALID_ARG, "aur_render_fp64acc_noalloc: film must be 16-byte aligned device memory "
                                         "of the scene's device");
    Addresses a;
    if ((st = device_addresses(&a)) != AUR_OK) return st;
    cudaStream_t s = sc->ctx->stream;
    cudaError_t e = cudaMemsetAsync(a.counters, 0, sizeof(unsigned long long) * 8, s);
    if (e == cudaSuccess) e = launch_render_plain(sc->dev(), p, (float4*)film, a.accum, a.counters, false, s);
    unsigned long long cnt[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, a.counters, sizeof(cnt), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "aur_render_fp64acc_noalloc");
    if (stats) {
        *stats = aur_render_stats{};
        stats->camera_rays = cnt[0];
        stats->closest_rays = cnt[1];
        stats->shadow_rays = cnt[2];
        stats->paths = cnt[3];
        stats->launches = 1;
        stats->kernel_ms = 0.0;   // no events are created here
    }
    return AUR_OK;
}
