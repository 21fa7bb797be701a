// render_wavefront.cu — the batched (wavefront) renderer.
//
// Same estimator as Integrator::integrateCameraSample (Aurora/src/frontend/
// integrator.cpp:152-300) and the plain kernel, reorganised for the GPU:
// a pool of P path slots lives in HBM (structure of arrays) and every
// iteration runs one bounce of every live path as separate stages:
//
//   regen   finished slots write their sample and take the next work item
//           (scene, pixel, sample) from a global counter -> camera ray
//   extend  closest hit for the extension queue (persistent warps, traversal only)
//   sort    optional: counting sort of the hits by material type
//   shade   emission, lobe choice, next-event rays + their contributions, BRDF
//           continuation, throughput and roulette -> next extension queue
//   shadow  occlusion for the next-event rays, Lo += direct * T
//
// Queue appends and work fetches are aggregated per block (one atomic per block). Many scenes of
// different resolution, spp and depth share one pool (batched launch). The
// per-iteration kernels are captured once into a CUDA graph and replayed.
// Every (pixel, sample) result goes to a per-sample buffer and is resolved in
// sample order with the plain kernel's compensated sum, so both renderers
// produce the same film for the same seed.
#include "aur_capi_internal.h"
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <type_traits>

namespace aur {
namespace {

enum : uint32_t { PS_EMPTY = 0, PS_ACTIVE = 1, PS_DONE = 2, PS_MASK = 3, PS_PENDING = 4 };
// lane refill: a warp takes new rays once this many lanes are idle, and runs kRounds
// traversal rounds (interior phase + leaf phase) between refill checks
// (swept on the 4-wide tree: rounds 2 / 3 / 4 / 6 / 8 at 16 idle lanes 479.6 / 481.8 /
// 488.1 / 472.7 / 463.8 M samples/s; refill 8-20 idle lanes within 0.5% at 4 rounds)
constexpr int kRefill = 16;
constexpr int kRounds = 4;
// resident 256-thread blocks per SM the traversal kernels are compiled for (register cap)
#ifndef AUR_TRAV_MINB
#define AUR_TRAV_MINB 4
#endif
enum : int { B_MISS = 0, B_MATTE = 1, B_KELEMEN = 2, B_CT = 3, B_METAL = 4, B_CONST = 5, kBuckets = 6 };
// counters
enum : int {
    C_EXT0 = 0, C_EXT1 = 1, C_SHADOW = 2, C_WORK = 3, C_TOTAL = 4, C_CUR_EXT = 5, C_CUR_SHADE = 6,
    C_CUR_SHADOW = 7, C_CUR_SORT = 8, C_CUR_SHADE2 = 9, C_BUCKET = 16, C_FILL = 24, kCounters = 32
};

struct WfScene {
    DevScene sc;
    PathParams p;          // spp = samples of this pass, sample_offset = first sample index of this pass
    uint64_t key;
    uint32_t npix, item_base, items, rec_depth;
    // Light samples: every camera sample of the pass has lsub sub-samples q = sl * lsub + j
    // (lsub = light_samples, 1 without them); sub-sample j of sample s traces the path j of
    // Integrator::integrateCameraSample(sample, numSamples) and draws from random-number sample
    // index s * lsub + j = rng_offset + q, its camera ray from s * lsub. The render's sample 0
    // has one path only (renderer.cpp:231-258): its sub-samples j > 0 are skipped.
    uint32_t lsub, rng_offset;
    float4* samples;       // [spp_pass * lsub][npix]
    // record mode (path-replay adjoint): per item (sample-major, sl * npix + pixel)
    float4* rec;           // [items][rec_depth] hit records (t, u, v, prim | visibility << 30)
    float4* lo_raw;        // [items] unclamped path radiance, w = number of recorded vertices
};

// Per-slot state in 32-byte pairs (one DRAM sector per slot and pair), structure of arrays
// over the slots: the stages gather slots in queue order (material buckets, not slot order),
// so a float4 of its own array would pull a half-used sector per field; a pair of fields that
// are read together fills its sector, and slot-order sweeps (regen) stay coalesced.
//   ray    origin + mint, direction + maxt        (extend, shade; written by regen, shade)
//   hitid  hit (t, u, v, prim), id (scene, pixel, sub-sample, flags)   (extend, sort, shade, regen)
//   tplo   throughput + roulette factor, radiance + alpha              (shade, regen)
//   neeA   shading point, first next-event direction + maxt            (shadow)
//   neeB   second next-event direction + maxt, its contribution        (shadow, regen)
//   neeC   first next-event contribution, throughput + nvis            (regen)
struct WfPool {
    float4 *ray, *hitid, *tplo, *neeA, *neeB, *neeC;   // [P][2] each
    uint32_t* state;            // PS_* in the low bits, PS_PENDING when next-event rays are in flight
    uint32_t* sh_vis;           // bit k: next-event ray k of the slot is unoccluded
    uint32_t* rec_cur;          // record mode: record index of the vertex whose next-event rays are in flight
    uint8_t* bucket;            // material bucket of the slot's last hit (written by the sorting extend)
    uint32_t *q_ext0, *q_ext1, *q_sort, *q_shadow;
    uint32_t* ctr;
    unsigned long long* rays;   // [0] closest-hit rays, [1] shadow rays
    const WfScene* scenes;
    int nscenes;                // table capacity; unused entries start at item UINT32_MAX
    uint32_t P;
    __device__ __forceinline__ float4& ray_o(uint32_t i) const { return ray[2 * (size_t)i]; }
    __device__ __forceinline__ float4& ray_d(uint32_t i) const { return ray[2 * (size_t)i + 1]; }
    __device__ __forceinline__ float4& hit(uint32_t i) const { return hitid[2 * (size_t)i]; }
    __device__ __forceinline__ uint4& id(uint32_t i) const { return reinterpret_cast<uint4*>(hitid)[2 * (size_t)i + 1]; }
    __device__ __forceinline__ float4& tp(uint32_t i) const { return tplo[2 * (size_t)i]; }
    __device__ __forceinline__ float4& lo(uint32_t i) const { return tplo[2 * (size_t)i + 1]; }
    __device__ __forceinline__ float4& sh_p(uint32_t i) const { return neeA[2 * (size_t)i]; }
    __device__ __forceinline__ float4& sh_d0(uint32_t i) const { return neeA[2 * (size_t)i + 1]; }
    __device__ __forceinline__ float4& sh_d1(uint32_t i) const { return neeB[2 * (size_t)i]; }
    __device__ __forceinline__ float4& sh_c1(uint32_t i) const { return neeB[2 * (size_t)i + 1]; }
    __device__ __forceinline__ float4& sh_c0(uint32_t i) const { return neeC[2 * (size_t)i]; }
    __device__ __forceinline__ float4& sh_t(uint32_t i) const { return neeC[2 * (size_t)i + 1]; }
};

// flags in id.w; kNoClamp: the sample is the environment seen by the camera ray, which
// the reference adds without the firefly filter
constexpr uint32_t kNoClamp = 1u << 21;
__device__ __forceinline__ uint32_t pack_flags(int vtx, int bounces, int kind, bool matte) {
    return (uint32_t)vtx | ((uint32_t)bounces << 9) | ((uint32_t)kind << 18) | ((uint32_t)matte << 20);
}
__device__ __forceinline__ int f_vtx(uint32_t f) { return f & 511; }
__device__ __forceinline__ int f_bounces(uint32_t f) { return (f >> 9) & 511; }
__device__ __forceinline__ int f_kind(uint32_t f) { return (f >> 18) & 3; }
__device__ __forceinline__ bool f_matte(uint32_t f) { return (f >> 20) & 1; }

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << lane_id()) - 1u; }

// Block-aggregated append to up to three queues: every thread of the block calls it
// (uniform control flow) with its flags; it returns each flagged thread's slot in the
// queue. One atomic per queue per block instead of one per warp.
struct BlockScan { uint32_t cnt[16][3]; uint32_t base[3]; };
__device__ __forceinline__ void block_reserve(BlockScan& sh, const bool (&p)[3], uint32_t* const (&ctr)[3],
                                              uint32_t (&pos)[3]) {
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t m[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) m[q] = __ballot_sync(0xffffffffu, p[q]);
    if (lane_id() == 0)
#pragma unroll
        for (int q = 0; q < 3; ++q) sh.cnt[warp][q] = __popc(m[q]);
    __syncthreads();
    if (threadIdx.x < 3) {
        const int q = threadIdx.x;
        uint32_t t = 0;
        for (int j = 0; j < nw; ++j) { const uint32_t c = sh.cnt[j][q]; sh.cnt[j][q] = t; t += c; }
        sh.base[q] = (t && ctr[q]) ? atomicAdd(ctr[q], t) : 0u;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 3; ++q) pos[q] = sh.base[q] + sh.cnt[warp][q] + __popc(m[q] & lanemask_lt());
    __syncthreads();   // sh is reused by the next call
}

// random-number sample index of sub-sample q, and that of its camera ray
__device__ __forceinline__ uint32_t rng_index(const WfScene& S, uint32_t q) { return S.rng_offset + q; }
__device__ __forceinline__ uint32_t cam_index(const WfScene& S, uint32_t q) {
    return S.lsub > 1 ? S.rng_offset + q - q % S.lsub : S.rng_offset + q;
}
// sub-samples j > 0 of the render's sample 0 trace nothing (one path in the first pass)
__device__ __forceinline__ bool skipped_sub(const WfScene& S, uint32_t q) {
    return S.lsub > 1 && q % S.lsub != 0 && (uint32_t)S.p.sample_offset + q / S.lsub == 0;
}

__device__ __forceinline__ int scene_of(const WfPool& w, uint32_t item) {
    int lo = 0, hi = w.nscenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (w.scenes[mid].item_base <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------------ regen
template <bool kRec>
__global__ void k_regen(WfPool w, int in_q) {
    __shared__ BlockScan s_scan;
    uint32_t* qin = in_q ? w.q_ext1 : w.q_ext0;
    uint32_t* cin = &w.ctr[in_q ? C_EXT1 : C_EXT0];
    const uint32_t total = w.ctr[C_TOTAL];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < w.P; base += stride) {
        const uint32_t i = base + threadIdx.x;
        const bool valid = i < w.P;
        uint32_t st = PS_ACTIVE, vis = 0;
        float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), t = lo, c0 = lo;
        uint4 id = make_uint4(0, 0, 0, 0);
        if (valid) {
            // the slot's records are loaded together, before its state says which of them it
            // uses, so that their latencies overlap (c0 and t share one 32-byte pair)
            st = w.state[i];
            vis = w.sh_vis[i];
            t = w.sh_t(i);
            c0 = w.sh_c0(i);
            lo = w.lo(i);
            id = w.id(i);
        }
        if (st & PS_PENDING) {
            // next-event estimate of the last vertex: Lo += ((vis0 c0 + vis1 c1) nvis) T, the
            // plain kernel's order of operations (integrate_direct)
            const float nvis = t.w;   // the number of visible lights rides in the throughput record
            float3 res = mk(0.f, 0.f, 0.f);
            if (vis & 1u) res += mk(c0.x, c0.y, c0.z);   // only unoccluded contributions are added
            if (vis & 2u) { const float4 c1 = w.sh_c1(i); res += mk(c1.x, c1.y, c1.z); }
            const float3 add = (res * nvis) * mk(t.x, t.y, t.z);
            lo.x += add.x; lo.y += add.y; lo.z += add.z;
            w.lo(i) = lo;
            st &= ~PS_PENDING;
            if (kRec) {   // the visibility of the vertex's next-event rays goes into its record
                float4* r = w.scenes[id.x].rec + w.rec_cur[i];
                r->w = __int_as_float(__float_as_int(r->w) | (int)(vis << 30));
            }
        }
        if (st == PS_DONE) {
            const WfScene& S = w.scenes[id.x];
            if (kRec) {
                S.lo_raw[(size_t)id.z * S.npix + id.y] = make_float4(lo.x, lo.y, lo.z, __int_as_float(f_vtx(id.w)));
            } else {
                const float3 L = (id.w & kNoClamp) ? mk(lo.x, lo.y, lo.z) : firefly_clamp(mk(lo.x, lo.y, lo.z));
                // with light samples, alpha 2 marks the environment seen by the camera ray: the
                // sample is that radiance, not the mean of its sub-samples (integrator.cpp:287-298)
                const float a = (S.lsub > 1 && (id.w & kNoClamp)) ? 2.f : lo.w;
                S.samples[(size_t)id.z * S.npix + id.y] = make_float4(L.x, L.y, L.z, a);
            }
            st = PS_EMPTY;
        }
        const bool want = st == PS_EMPTY && *(volatile uint32_t*)&w.ctr[C_WORK] < total;
        uint32_t item = 0xffffffffu;
        {
            const bool pw[3] = {want, false, false};
            uint32_t* const cw[3] = {&w.ctr[C_WORK], nullptr, nullptr};
            uint32_t pos[3];
            block_reserve(s_scan, pw, cw, pos);
            if (want) item = pos[0];
        }
        bool start = want && item < total;
        int s = 0;
        uint32_t pixel = 0, q = 0;
        if (start) {
            s = scene_of(w, item);
            const uint32_t local = item - w.scenes[s].item_base;
            pixel = local % w.scenes[s].npix;
            q = local / w.scenes[s].npix;
            start = !skipped_sub(w.scenes[s], q);
        }
        if (start) {
            const WfScene& S = w.scenes[s];
            PathRng rng;
            rng.key = S.key;
            rng.base = path_base(pixel, cam_index(S, q));
            const RayF r = camera_ray(S.sc.cam, (int)(pixel % (uint32_t)S.sc.cam.w), (int)(pixel / (uint32_t)S.sc.cam.w),
                                      rng.u(kDimCamera), rng.u(kDimCamera + 1));
            w.ray_o(i) = make_float4(r.o.x, r.o.y, r.o.z, r.mint);
            w.ray_d(i) = make_float4(r.d.x, r.d.y, r.d.z, r.maxt);
            w.tp(i) = make_float4(1.f, 1.f, 1.f, 1.f);
            w.lo(i) = make_float4(0.f, 0.f, 0.f, 0.f);
            w.id(i) = make_uint4((uint32_t)s, pixel, q, pack_flags(0, 0, RAY_CAMERA, false));
            st = PS_ACTIVE;
        }
        {
            const bool pp[3] = {start, false, false};
            uint32_t* const cp[3] = {cin, nullptr, nullptr};
            uint32_t pos[3];
            block_reserve(s_scan, pp, cp, pos);
            if (start) qin[pos[0]] = i;
        }
        if (valid) w.state[i] = st;
    }
}

// ------------------------------------------------------------------ extend
__device__ __forceinline__ int bucket_of(const ShadeScene& sh, int prim) {
    if (prim < 0) return B_MISS;
    const int mt = sh.mats[sh.attrs[sh.tri_attr[prim]].material].type;
    return mt == MAT_MATTE ? B_MATTE : mt == MAT_KELEMEN ? B_KELEMEN : mt == MAT_COOKTORRANCE ? B_CT
         : mt == MAT_METAL ? B_METAL : B_CONST;
}

// Closest hit for the extension queue. Each lane keeps a resumable traversal;
// finished lanes are refilled from the queue (one atomic per warp) while the
// others continue, so a warp is not held up by its slowest ray.
template <bool kSort, bool kWide>
__global__ void __launch_bounds__(256, AUR_TRAV_MINB) k_extend(WfPool w, int in_q) {
    using Stack = std::conditional_t<kWide, LaneStack4, LaneStack>;
    using Trace = std::conditional_t<kWide, TraceState4<false>, TraceState<false>>;
    using Node = std::conditional_t<kWide, BvhNode4, BvhNode>;
    const uint32_t* qin = in_q ? w.q_ext1 : w.q_ext0;
    const uint32_t n = w.ctr[in_q ? C_EXT1 : C_EXT0];
    // Outputs of the later stages start empty. Only counters that no block of
    // this kernel touches are reset here; the bucket counters this kernel
    // increments were reset by the previous next-event stage (or the pass start).
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.ctr[in_q ? C_EXT0 : C_EXT1] = 0;
        w.ctr[C_SHADOW] = 0;
        w.ctr[C_CUR_SHADE] = 0;
        w.ctr[C_CUR_SHADE2] = 0;
        w.ctr[C_CUR_SHADOW] = 0;
        w.ctr[C_CUR_SORT] = 0;
        w.rays[0] += n;
    }
    extern __shared__ int s_stack[];
    __shared__ uint32_t s_bucket[kBuckets];   // per-block material counts, added to the global ones at exit
    if (kSort && threadIdx.x < kBuckets) s_bucket[threadIdx.x] = 0;
    __syncthreads();
    Stack stack;
    stack.col = s_stack + threadIdx.x;
    stack.stride = blockDim.x;
    Trace ts;
    const Node* nodes = nullptr;
    const BvhTri* tris = nullptr;
    const WfScene* S = nullptr;
    uint32_t slot = 0;
    bool has = false, exhausted = false;
    while (true) {
        const bool need = !has && !exhausted;
        const uint32_t m = __ballot_sync(0xffffffffu, need);
        const uint32_t act = __ballot_sync(0xffffffffu, has);
        if (m && (__popc(m) >= kRefill || act == 0)) {
            const int leader = __ffs(m) - 1;
            uint32_t b = 0;
            if ((int)lane_id() == leader) b = atomicAdd(&w.ctr[C_CUR_EXT], (uint32_t)__popc(m));
            b = __shfl_sync(0xffffffffu, b, leader);
            if (need) {
                const uint32_t k = b + __popc(m & lanemask_lt());
                if (k < n) {
                    slot = qin[k];
                    S = &w.scenes[w.id(slot).x];
                    if constexpr (kWide) nodes = S->sc.nodes4;
                    else nodes = S->sc.nodes;
                    tris = S->sc.tris;
                    const float4 o = w.ray_o(slot), d = w.ray_d(slot);
                    ts.begin(mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), o.w, d.w);
                    has = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, has || !exhausted) == 0) break;
        bool done = false;
        for (int k = 0; k < kRounds; ++k) {          // all lanes take part in every round
            if (ts.round(nodes, tris, stack, has && !done)) done = true;
        }
        done = done && has;
        int bucket = -1;
        if (done) {
            w.hit(slot) = make_float4(ts.tbest, ts.bu, ts.bv, __int_as_float(ts.best));
            if (kSort) {
                bucket = bucket_of(S->sc.sh, ts.best);
                w.bucket[slot] = (uint8_t)bucket;   // the scatter reads it instead of the hit's material
            }
            has = false;
        }
        if (kSort) {   // per-bucket counts, one shared atomic per (warp, bucket)
            const uint32_t fin = __ballot_sync(0xffffffffu, bucket >= 0);
            if (bucket >= 0) {
                const uint32_t peers = __match_any_sync(fin, bucket);
                if ((int)lane_id() == __ffs(peers) - 1) atomicAdd(&s_bucket[bucket], (uint32_t)__popc(peers));
            }
        }
    }
    if (kSort) {
        __syncthreads();
        if (threadIdx.x < kBuckets && s_bucket[threadIdx.x]) atomicAdd(&w.ctr[C_BUCKET + threadIdx.x], s_bucket[threadIdx.x]);
    }
}

// counting-sort scatter of the extension queue into q_sort, grouped by bucket
__global__ void k_sort_scatter(WfPool w, int in_q) {
    const uint32_t* qin = in_q ? w.q_ext1 : w.q_ext0;
    const uint32_t n = w.ctr[in_q ? C_EXT1 : C_EXT0];
    __shared__ uint32_t s_ofs[kBuckets], s_cnt[kBuckets], s_base[kBuckets];
    __shared__ uint32_t s_fetch;
    if (threadIdx.x == 0) {
        uint32_t a = 0;
        for (int b = 0; b < kBuckets; ++b) { s_ofs[b] = a; a += w.ctr[C_BUCKET + b]; }
    }
    while (true) {   // a block takes blockDim entries at a time; one atomic per bucket per block
        if (threadIdx.x == 0) s_fetch = atomicAdd(&w.ctr[C_CUR_SORT], blockDim.x);
        if (threadIdx.x < kBuckets) s_cnt[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t b = s_fetch;
        if (b >= n) break;
        const uint32_t k = b + threadIdx.x;
        int bucket = -1;
        uint32_t slot = 0, local = 0;
        if (k < n) {
            slot = qin[k];
            bucket = w.bucket[slot];
        }
        const uint32_t active = __ballot_sync(0xffffffffu, bucket >= 0);
        if (bucket >= 0) {
            const uint32_t peers = __match_any_sync(active, bucket);
            const int leader = __ffs(peers) - 1;
            uint32_t wb = 0;
            if ((int)lane_id() == leader) wb = atomicAdd(&s_cnt[bucket], (uint32_t)__popc(peers));
            local = __shfl_sync(peers, wb, leader) + __popc(peers & lanemask_lt());
        }
        __syncthreads();
        if (threadIdx.x < kBuckets)
            s_base[threadIdx.x] = s_cnt[threadIdx.x] ? atomicAdd(&w.ctr[C_FILL + threadIdx.x], s_cnt[threadIdx.x]) : 0u;
        __syncthreads();
        if (bucket >= 0) w.q_sort[s_ofs[bucket] + s_base[bucket] + local] = slot;
        __syncthreads();   // s_fetch and s_cnt are rewritten next round
    }
}

// ------------------------------------------------------------------ shade
// A ray that missed in a scene with environment lights: the camera ray sees the
// environment (alpha 1, no firefly filter), an escaping mirror ray adds it times the
// throughput, both along the camera ray's direction (integrator.cpp:262-288). Out of line.
__device__ __noinline__ float4 shade_env_miss(const WfPool* w, const WfScene* S, uint32_t slot, uint4 id, int vtx,
                                              float4 lo) {
    PathRng rng;
    rng.key = S->key;
    rng.base = path_base(id.y, cam_index(*S, id.z));
    const RayF cr = camera_ray(S->sc.cam, (int)(id.y % (uint32_t)S->sc.cam.w), (int)(id.y / (uint32_t)S->sc.cam.w),
                               rng.u(kDimCamera), rng.u(kDimCamera + 1));
    const float3 e = env_radiance_of(S->sc.sh.lights, S->sc.sh.nlights, S->sc.sh.texs, S->sc.sh.texels, cr.d);
    if (vtx == 0) {
        w->id(slot).w = id.w | kNoClamp;
        return make_float4(e.x, e.y, e.z, 1.f);
    }
    const float4 t = w->tp(slot);
    const float3 a = e * mk(t.x, t.y, t.z);
    return make_float4(lo.x + a.x, lo.y + a.y, lo.z + a.z, lo.w);
}

// Three resident 256-thread blocks per SM (85 registers, some spilled) instead of the two that
// its 106 registers allow: 50.7 vs 52.3 ms per 1080p frame.
// kPart selects the entries: SHADE_ALL every queued one; with the queue sorted by bucket,
// SHADE_MATTE the matte bucket alone (its lobe known at compile time, so the glossy lobes'
// code and registers drop out) and SHADE_REST all others. The bucket counts stay in place
// until the next-event stage resets them, after both parts have read them.
enum : int { SHADE_ALL = 0, SHADE_MATTE = 1, SHADE_REST = 2 };
#ifndef AUR_SHADE_MATTE_MINB
#define AUR_SHADE_MATTE_MINB 4
#endif
template <bool kRec, int kPart>
__global__ void __launch_bounds__(256, kPart == SHADE_MATTE ? AUR_SHADE_MATTE_MINB : 3) k_shade(WfPool w, int in_q, int sorted) {
    const uint32_t* qin = sorted ? w.q_sort : (in_q ? w.q_ext1 : w.q_ext0);
    const uint32_t n_all = w.ctr[in_q ? C_EXT1 : C_EXT0];
    // the sorted queue holds the misses first, then the matte bucket
    const uint32_t nmiss = kPart == SHADE_ALL ? 0u : w.ctr[C_BUCKET + B_MISS];
    const uint32_t nm = kPart == SHADE_ALL ? 0u : w.ctr[C_BUCKET + B_MATTE];
    const uint32_t n = kPart == SHADE_ALL ? n_all : kPart == SHADE_MATTE ? nm : n_all - nm;
    uint32_t* qout = in_q ? w.q_ext0 : w.q_ext1;
    uint32_t* cout = &w.ctr[in_q ? C_EXT0 : C_EXT1];
    __shared__ BlockScan s_scan;
    __shared__ uint32_t s_fetch;
    while (true) {
        if (threadIdx.x == 0) s_fetch = atomicAdd(&w.ctr[kPart == SHADE_MATTE ? C_CUR_SHADE2 : C_CUR_SHADE], blockDim.x);
        __syncthreads();
        const uint32_t b = s_fetch;   // rewritten only after block_reserve's barriers below
        if (b >= n) break;
        const uint32_t k = b + threadIdx.x;
        bool push_ext = false, push_sh0 = false, push_sh1 = false;
        uint32_t slot = 0;
        if (k < n) {
            slot = qin[kPart == SHADE_ALL ? k : kPart == SHADE_MATTE ? nmiss + k : (k < nmiss ? k : k + nm)];
            const float4 hh = w.hit(slot);
            const int prim = __float_as_int(hh.w);
            float4 lo = w.lo(slot);
            if (prim < 0) {
                const uint4 id = w.id(slot);
                const WfScene& S = w.scenes[id.x];
                const int kind = f_kind(id.w), vtx = f_vtx(id.w);
                if (S.sc.sh.nenv && (vtx == 0 || kind == RAY_MIRROR))
                    lo = shade_env_miss(&w, &S, slot, id, vtx, lo);
                w.state[slot] = PS_DONE;
            } else if (f_vtx(w.id(slot).w) >= w.scenes[w.id(slot).x].p.max_depth) {
                // the reference's unshaded last ray hit something: the path ends
                w.state[slot] = PS_DONE;
            } else {
                const uint4 id = w.id(slot);
                const WfScene& S = w.scenes[id.x];
                const DevScene& sc = S.sc;
                const uint32_t flags = id.w;
                const int vtx = f_vtx(flags);
                int kind = f_kind(flags);
                bool matte = f_matte(flags);
                int bounces = f_bounces(flags);
                PathRng rng;
                rng.key = S.key;
                rng.base = path_base(id.y, rng_index(S, id.z));
                const float4 ro = w.ray_o(slot), rd = w.ray_d(slot);
                float4 tpv = w.tp(slot);
                float3 T = mk(tpv.x, tpv.y, tpv.z);
                float cont = tpv.w;
                float3 Lo = mk(lo.x, lo.y, lo.z);
                if (vtx == 0) lo.w = 1.f;   // camera ray hit: alpha
                const uint32_t rec_at = (id.z * S.npix + id.y) * S.rec_depth + (uint32_t)vtx;
                if (kRec) S.rec[rec_at] = make_float4(hh.x, hh.y, hh.z, __int_as_float(prim));
                const Frame f = hit_frame(sc.sh, prim, hh.x, hh.y, hh.z, mk(ro.x, ro.y, ro.z), mk(rd.x, rd.y, rd.z), true);
                const Attr at = sc.sh.attrs[f.attr];
                if (kind == RAY_DIFFUSE) matte = true;
                if (collects_emission(kind)) Lo += T * at.emission;
                const Brdf brdf = kPart == SHADE_MATTE
                                      ? matte_brdf(sc.sh, sc.sh.mats[at.material], f)
                                      : get_brdf(sc.sh, at.material, f, matte, rng.u(vertex_dim(vtx, kDimLobe)));
                // next-event estimation: rays and their unoccluded contributions
                if (brdf.lobe == LOBE_MATTE || brdf.lobe == LOBE_SPEC) {
                    int nvis;
                    const int li = pick_visible_light(sc.sh, f.P, f.N, rng.u(vertex_dim(vtx, kDimLightPick)), &nvis);
                    if (li >= 0) {
                        const Light& L = sc.sh.lights[li];   // global: the env paths take its address
                        const LightSample ls = light_sample(sc.sh, L, f.P, f.N, rng.u(vertex_dim(vtx, kDimLightSample)),
                                                            rng.u(vertex_dim(vtx, kDimLightSample + 1)));
                        float cost = dot(f.N, ls.dir);
                        float3 c0 = mk(0.f, 0.f, 0.f), c1 = c0;
                        float3 d0 = ls.dir, d1 = ls.dir;
                        float m0 = ls.maxt, m1 = 0.f;
                        bool r0 = false, r1 = false;
                        if (brdf.lobe == LOBE_MATTE) {
                            if (cost >= 0.f && ls.pdf > 0.f) {
                                r0 = true;
                                c0 = cdiv((ls.color * brdf_eval(brdf, ls.dir, f.V, f.N)) * cost, ls.pdf);
                            }
                        } else {
                            if (cost > 0.f && ls.pdf > 0.f) {
                                const float bp = brdf_pdf(brdf, ls.dir, f.V, f.N);
                                if (bp > 0.f) {
                                    r0 = true;
                                    const float wgt = power_heuristic(ls.pdf, bp);
                                    c0 = cdiv(((ls.color * wgt) * brdf_eval(brdf, ls.dir, f.V, f.N)) * cost, ls.pdf);
                                }
                            }
                            const BrdfSample bs = brdf_sample(brdf, f.V, f.N, rng.u(vertex_dim(vtx, kDimMisBrdf)),
                                                              rng.u(vertex_dim(vtx, kDimMisBrdf + 1)));
                            cost = dot(f.N, bs.dir);
                            if (cost > 0.f) {
                                float maxt = bs.maxt;
                                const float lp = light_pdf(sc.sh, L, f.P, bs.dir, kRayBias, &maxt);
                                if (lp > 0.f && bs.pdf > 0.f) {
                                    r1 = true;
                                    d1 = bs.dir;
                                    m1 = maxt;
                                    const float wgt = power_heuristic(bs.pdf, lp);
                                    c1 = cdiv(((bs.color * wgt) * light_eval(sc.sh, L, bs.dir)) * cost, bs.pdf);
                                }
                            }
                        }
                        if (r0 || r1) {
                            if (kRec) w.rec_cur[slot] = rec_at;
                            w.sh_p(slot) = make_float4(f.P.x, f.P.y, f.P.z, 0.f);
                            w.sh_d0(slot) = make_float4(d0.x, d0.y, d0.z, m0);
                            w.sh_d1(slot) = make_float4(d1.x, d1.y, d1.z, m1);
                            w.sh_c0(slot) = make_float4(c0.x, c0.y, c0.z, 0.f);
                            w.sh_c1(slot) = make_float4(c1.x, c1.y, c1.z, 0.f);
                            w.sh_t(slot) = make_float4(T.x, T.y, T.z, (float)nvis);
                            w.sh_vis[slot] = 0u;
                            push_sh0 = r0;
                            push_sh1 = r1;
                        }
                    }
                }
                // continuation (integrator.cpp:208-261)
                bool alive = false;
                const BrdfSample bs = brdf_sample(brdf, f.V, f.N, rng.u(vertex_dim(vtx, kDimBrdf)),
                                                  rng.u(vertex_dim(vtx, kDimBrdf + 1)));
                // after the last vertex the reference traces one more ray, which only an
                // escaping mirror ray in a scene with an environment light turns into radiance
                // (integrator.cpp:256-274): that ray is queued and its hit is not shaded
                if (continue_path(brdf, bs, f.N, S.p.min_depth, rng, vtx, T, cont, kind, bounces) &&
                    (vtx + 1 < S.p.max_depth || (kind == RAY_MIRROR && sc.sh.nenv))) {
                    alive = true;
                    w.ray_o(slot) = make_float4(f.P.x, f.P.y, f.P.z, kRayBias);
                    w.ray_d(slot) = make_float4(bs.dir.x, bs.dir.y, bs.dir.z, bs.maxt);
                    w.tp(slot) = make_float4(T.x, T.y, T.z, cont);
                    w.id(slot).w = pack_flags(vtx + 1, bounces, kind, matte);
                }
                lo = make_float4(Lo.x, Lo.y, Lo.z, lo.w);
                // a finished path's flags count its recorded vertices (a missed ray's vertex is not recorded)
                if (kRec && !alive) w.id(slot).w = pack_flags(vtx + 1, bounces, kind, matte);
                w.state[slot] = (alive ? PS_ACTIVE : PS_DONE) | (push_sh0 || push_sh1 ? PS_PENDING : 0u);
                push_ext = alive;
            }
            w.lo(slot) = lo;
        }
        {
            const bool pp[3] = {push_ext, push_sh0, push_sh1};
            uint32_t* const cp[3] = {cout, &w.ctr[C_SHADOW], &w.ctr[C_SHADOW]};
            uint32_t pos[3];
            block_reserve(s_scan, pp, cp, pos);
            if (push_ext) qout[pos[0]] = slot;
            if (push_sh0) w.q_shadow[pos[1]] = slot << 1;
            if (push_sh1) w.q_shadow[pos[2]] = (slot << 1) | 1u;
        }
    }
}

// ------------------------------------------------------------------ shadow
// Occlusion of the next-event rays (entries slot << 1 | ray); lanes are refilled as in
// k_extend. An unoccluded ray sets its bit in sh_vis; the next regen adds the light.
template <bool kWide>
__global__ void __launch_bounds__(256, AUR_TRAV_MINB) k_shadow(WfPool w) {
    using Stack = std::conditional_t<kWide, LaneStack4, LaneStack>;
    using Trace = std::conditional_t<kWide, TraceState4<true>, TraceState<true>>;
    using Node = std::conditional_t<kWide, BvhNode4, BvhNode>;
    const uint32_t n = w.ctr[C_SHADOW];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.rays[1] += n;
        // extend, scatter and shade are finished: reset their fetch and bucket counters
        w.ctr[C_CUR_EXT] = 0;
        for (int k = 0; k < kBuckets; ++k) { w.ctr[C_BUCKET + k] = 0; w.ctr[C_FILL + k] = 0; }
    }
    extern __shared__ int s_stack[];
    Stack stack;
    stack.col = s_stack + threadIdx.x;
    stack.stride = blockDim.x;
    Trace ts;
    const Node* nodes = nullptr;
    const BvhTri* tris = nullptr;
    uint32_t entry = 0;
    bool has = false, exhausted = false;
    while (true) {
        const bool need = !has && !exhausted;
        const uint32_t m = __ballot_sync(0xffffffffu, need);
        const uint32_t act = __ballot_sync(0xffffffffu, has);
        if (m && (__popc(m) >= kRefill || act == 0)) {
            const int leader = __ffs(m) - 1;
            uint32_t b = 0;
            if ((int)lane_id() == leader) b = atomicAdd(&w.ctr[C_CUR_SHADOW], (uint32_t)__popc(m));
            b = __shfl_sync(0xffffffffu, b, leader);
            if (need) {
                const uint32_t k = b + __popc(m & lanemask_lt());
                if (k < n) {
                    entry = w.q_shadow[k];
                    const uint32_t slot = entry >> 1;
                    const WfScene& S = w.scenes[w.id(slot).x];
                    if constexpr (kWide) nodes = S.sc.nodes4;
                    else nodes = S.sc.nodes;
                    tris = S.sc.tris;
                    const float4 p = w.sh_p(slot);
                    const float4 d = (entry & 1u) ? w.sh_d1(slot) : w.sh_d0(slot);
                    ts.begin(mk(p.x, p.y, p.z), mk(d.x, d.y, d.z), kRayBias, d.w);
                    has = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (__ballot_sync(0xffffffffu, has || !exhausted) == 0) break;
        bool done = false;
        for (int k = 0; k < kRounds; ++k) {
            if (ts.round(nodes, tris, stack, has && !done)) done = true;
        }
        if (done && has) {
            if (!ts.hit_any) atomicOr(&w.sh_vis[entry >> 1], 1u << (entry & 1u));
            has = false;
        }
    }
}

// ------------------------------------------------------------------ resolve
// Adds this pass's samples of every pixel, in sample order, to the per-pixel
// compensated sums (the plain kernel's accumulation order).
__global__ void k_resolve(const WfScene* scenes, int s, float4* acc_s, float4* acc_c) {
    const WfScene& S = scenes[s];
    const uint32_t pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= S.npix) return;
    const float4 a = acc_s[pixel], c = acc_c[pixel];
    Kahan3 k;
    k.s = mk(a.x, a.y, a.z);
    k.c = mk(c.x, c.y, c.z);
    float alpha = a.w;
    if (S.lsub <= 1) {
        for (int j = 0; j < S.p.spp; ++j) {
            const float4 v = S.samples[(size_t)j * S.npix + pixel];
            k.add(mk(v.x, v.y, v.z));
            alpha += v.w;
        }
    } else {
        // a camera sample with light samples is the mean of its n sub-samples, added in their
        // order as Lo / n (integrate_camera_sample); n = 1 for the render's sample 0
        for (int sl = 0; sl < S.p.spp; ++sl) {
            const float4* sub = S.samples + (size_t)sl * S.lsub * S.npix + pixel;
            const float4 v0 = sub[0];
            if (v0.w == 2.f) {               // the camera ray saw the environment
                k.add(mk(v0.x, v0.y, v0.z));
                alpha += 1.f;
                continue;
            }
            const int n = S.p.sample_offset + sl == 0 ? 1 : (int)S.lsub;
            float3 sum = mk(v0.x, v0.y, v0.z);
            if (n > 1) {
                sum = cdiv(sum, (float)n);
                for (int j = 1; j < n; ++j) {
                    const float4 v = sub[(size_t)j * S.npix];
                    sum += cdiv(mk(v.x, v.y, v.z), (float)n);
                }
            }
            k.add(sum);
            alpha += v0.w;
        }
    }
    acc_s[pixel] = make_float4(k.s.x, k.s.y, k.s.z, alpha);
    acc_c[pixel] = make_float4(k.c.x, k.c.y, k.c.z, 0.f);
}

__global__ void k_finish(const float4* acc_s, const float4* acc_c, uint32_t npix, int spp, float4* film) {
    const uint32_t pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= npix) return;
    const float inv = 1.f / (float)spp;
    const float4 a = acc_s[pixel], c = acc_c[pixel];
    const float3 t = mk(a.x, a.y, a.z) + mk(c.x, c.y, c.z);
    film[pixel] = make_float4(t.x * inv, t.y * inv, t.z * inv, a.w * inv);
}

}  // namespace

struct WfConfig {
    uint32_t pool = 1u << 21;
    int block = 128;
    int sort = 1;
    int record = 0;   // record mode: hit records + unclamped radiance per item instead of samples
    int wide = 0;     // traverse the 4-wide trees (every scene of the batch has one)
};

// The 4-wide traversal is used when every scene of a batch has a 4-wide tree.
#ifndef AUR_WIDE_TRAVERSAL
#define AUR_WIDE_TRAVERSAL 1
#endif
struct BatchItem;
static int wide_for(const std::vector<BatchItem>& items);

// ------------------------------------------------------------------ host driver
struct WfRun {
    // one wavefront engine: pool buffers + a captured graph of kItersPerGraph iterations
    WfConfig cfg;
    WfPool w{};
    void* mem = nullptr;
    WfScene* d_scenes = nullptr;
    int cap_scenes = 0;
    float4* samples = nullptr;                 // per-sample buffer, grown on demand
    size_t samples_bytes = 0;
    float4* acc = nullptr;                     // per-pixel compensated sums, grown on demand
    size_t acc_bytes = 0;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;
    int grid_regen = 0, grid_ext = 0, grid_shade = 0, grid_shade_m = 0, grid_shade_r = 0, grid_shadow = 0, grid_sort = 0;
    size_t stack_smem = 0;                     // shared traversal stack of one block
    uint32_t* h_ctr = nullptr;   // pinned
    static constexpr int kItersPerGraph = 8;
    static constexpr int kStages = 5;          // regen, extend, sort, shade, shadow
    cudaEvent_t ev[kItersPerGraph * kStages + 1] = {};
    int launches_per_graph = 0;
    double stage_ms[kStages] = {0, 0, 0, 0, 0};

    cudaError_t init(const WfConfig& c, int nscenes, cudaStream_t s) {
        cfg = c;
        stream = s;
        const size_t P = c.pool;
        const size_t bytes = P * (12 * sizeof(float4) + 8 * sizeof(uint32_t) + 1) + 21 * 256 +
                             kCounters * sizeof(uint32_t) + 2 * sizeof(unsigned long long);
        cudaError_t e = cudaMalloc(&mem, bytes);
        if (e != cudaSuccess) return e;
        char* p = (char*)mem;
        auto take = [&](size_t n) { char* r = p; p += (n + 255) & ~(size_t)255; return (void*)r; };
        float4** pairs[] = {&w.ray, &w.hitid, &w.tplo, &w.neeA, &w.neeB, &w.neeC};
        for (float4** q : pairs) *q = (float4*)take(2 * P * sizeof(float4));
        w.state = (uint32_t*)take(P * 4);
        w.q_ext0 = (uint32_t*)take(P * 4);
        w.q_ext1 = (uint32_t*)take(P * 4);
        w.q_sort = (uint32_t*)take(P * 4);
        w.q_shadow = (uint32_t*)take(2 * P * 4);   // up to two next-event rays per slot
        w.sh_vis = (uint32_t*)take(P * 4);
        w.rec_cur = (uint32_t*)take(P * 4);
        w.bucket = (uint8_t*)take(P);
        w.ctr = (uint32_t*)take(kCounters * 4);
        w.rays = (unsigned long long*)take(2 * sizeof(unsigned long long));
        if ((size_t)(p - (char*)mem) > bytes) return cudaErrorMemoryAllocation;
        cap_scenes = std::max(nscenes, 64);
        e = cudaMalloc(&d_scenes, sizeof(WfScene) * cap_scenes);
        if (e != cudaSuccess) return e;
        w.scenes = d_scenes;
        w.nscenes = cap_scenes;
        w.P = (uint32_t)P;
        e = cudaMallocHost(&h_ctr, kCounters * 4);
        if (e != cudaSuccess) return e;
        for (auto& x : ev) if ((e = cudaEventCreate(&x)) != cudaSuccess) return e;
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        stack_smem = (size_t)kSharedDepth * c.block * sizeof(int);
        auto persist = [&](const void* fn, size_t smem) {
            int nb = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, c.block, smem);
            return std::max(1, nb) * sms;
        };
        const void* ext = c.wide ? (c.sort ? (const void*)k_extend<true, true> : (const void*)k_extend<false, true>)
                                 : (c.sort ? (const void*)k_extend<true, false> : (const void*)k_extend<false, false>);
        grid_ext = persist(ext, stack_smem);
        grid_shade = persist(c.record ? (const void*)k_shade<true, SHADE_ALL> : (const void*)k_shade<false, SHADE_ALL>, 0);
        grid_shade_m = persist(c.record ? (const void*)k_shade<true, SHADE_MATTE> : (const void*)k_shade<false, SHADE_MATTE>, 0);
        grid_shade_r = persist(c.record ? (const void*)k_shade<true, SHADE_REST> : (const void*)k_shade<false, SHADE_REST>, 0);
        grid_shadow = persist(c.wide ? (const void*)k_shadow<true> : (const void*)k_shadow<false>, stack_smem);
        grid_sort = persist((const void*)k_sort_scatter, 0);
        // 64 blocks per SM (about 10 resident waves of the 40-register kernel): 14.8 ms per
        // 1080p frame against 15.3 at 16 and 16.5 at exactly the resident 6
        grid_regen = (int)std::min<size_t>((P + c.block - 1) / c.block, (size_t)sms * 64);
        return cudaSuccess;
    }

    // One iteration; an event after every stage so the graph reports per-stage device time.
    void enqueue_iteration(int in_q, int it) {
        // inside stream capture only an "external" record becomes an event-record node
        cudaEvent_t* e = &ev[it * kStages + 1];
        if (cfg.record) k_regen<true><<<grid_regen, cfg.block, 0, stream>>>(w, in_q);
        else k_regen<false><<<grid_regen, cfg.block, 0, stream>>>(w, in_q);
        cudaEventRecordWithFlags(e[0], stream, cudaEventRecordExternal);
        if (cfg.wide) {
            if (cfg.sort) k_extend<true, true><<<grid_ext, cfg.block, stack_smem, stream>>>(w, in_q);
            else k_extend<false, true><<<grid_ext, cfg.block, stack_smem, stream>>>(w, in_q);
        } else {
            if (cfg.sort) k_extend<true, false><<<grid_ext, cfg.block, stack_smem, stream>>>(w, in_q);
            else k_extend<false, false><<<grid_ext, cfg.block, stack_smem, stream>>>(w, in_q);
        }
        cudaEventRecordWithFlags(e[1], stream, cudaEventRecordExternal);
        if (cfg.sort) k_sort_scatter<<<grid_sort, cfg.block, 0, stream>>>(w, in_q);
        cudaEventRecordWithFlags(e[2], stream, cudaEventRecordExternal);
        if (cfg.sort) {   // the matte bucket, then the others
            if (cfg.record) {
                k_shade<true, SHADE_MATTE><<<grid_shade_m, cfg.block, 0, stream>>>(w, in_q, 1);
                k_shade<true, SHADE_REST><<<grid_shade_r, cfg.block, 0, stream>>>(w, in_q, 1);
            } else {
                k_shade<false, SHADE_MATTE><<<grid_shade_m, cfg.block, 0, stream>>>(w, in_q, 1);
                k_shade<false, SHADE_REST><<<grid_shade_r, cfg.block, 0, stream>>>(w, in_q, 1);
            }
        } else if (cfg.record) {
            k_shade<true, SHADE_ALL><<<grid_shade, cfg.block, 0, stream>>>(w, in_q, 0);
        } else {
            k_shade<false, SHADE_ALL><<<grid_shade, cfg.block, 0, stream>>>(w, in_q, 0);
        }
        cudaEventRecordWithFlags(e[3], stream, cudaEventRecordExternal);
        if (cfg.wide) k_shadow<true><<<grid_shadow, cfg.block, stack_smem, stream>>>(w);
        else k_shadow<false><<<grid_shadow, cfg.block, stack_smem, stream>>>(w);
        cudaEventRecordWithFlags(e[4], stream, cudaEventRecordExternal);
    }

    cudaError_t build_graph() {
        cudaGraph_t g;
        cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        cudaEventRecordWithFlags(ev[0], stream, cudaEventRecordExternal);
        for (int it = 0; it < kItersPerGraph; ++it) enqueue_iteration(it & 1, it);
        e = cudaStreamEndCapture(stream, &g);
        if (e != cudaSuccess) return e;
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        launches_per_graph = kItersPerGraph * (cfg.sort ? 6 : 4);
        return e;
    }

    // Runs one pass over `total` work items of the uploaded scene table.
    cudaError_t run_pass(uint32_t total, uint64_t* launches) {
        cudaError_t e = cudaMemsetAsync(w.ctr, 0, kCounters * 4, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(w.state, 0, (size_t)w.P * 4, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&w.ctr[C_TOTAL], &total, 4, cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return e;
        if (!exec && (e = build_graph()) != cudaSuccess) return e;
        // Bound on graph launches: each launch advances every live path by 8 bounces
        // and refills the pool, so a pass needs about total / P * depth / 8 launches.
        const uint64_t max_launches = (uint64_t)total * 64ull / ((uint64_t)w.P) + 4096ull;
        for (uint64_t it = 0; it < max_launches; ++it) {
            e = cudaGraphLaunch(exec, stream);
            if (e != cudaSuccess) return e;
            *launches += launches_per_graph;
            e = cudaMemcpyAsync(h_ctr, w.ctr, 8 * 4, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return e;
            for (int k = 0; k < kItersPerGraph * kStages; ++k) {
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, ev[k], ev[k + 1]) == cudaSuccess) stage_ms[k % kStages] += ms;
                else cudaGetLastError();   // timing is informational; never leave a stale error behind
            }
            if (h_ctr[C_WORK] >= total && h_ctr[C_EXT0] == 0) {
                // writes the last finished samples
                if (cfg.record) k_regen<true><<<grid_regen, cfg.block, 0, stream>>>(w, 0);
                else k_regen<false><<<grid_regen, cfg.block, 0, stream>>>(w, 0);
                *launches += 1;
                return cudaGetLastError();
            }
        }
        return cudaErrorLaunchTimeout;
    }

    cudaError_t ensure_samples(size_t bytes) {
        if (bytes <= samples_bytes) return cudaSuccess;
        if (samples) cudaFree(samples);
        samples = nullptr;
        samples_bytes = 0;
        cudaError_t e = cudaMalloc(&samples, bytes);
        if (e == cudaSuccess) samples_bytes = bytes;
        return e;
    }

    cudaError_t ensure_acc(size_t bytes) {
        if (bytes <= acc_bytes) return cudaSuccess;
        if (acc) cudaFree(acc);
        acc = nullptr;
        acc_bytes = 0;
        cudaError_t e = cudaMalloc(&acc, bytes);
        if (e == cudaSuccess) acc_bytes = bytes;
        return e;
    }

    void release() {
        if (acc) cudaFree(acc);
        acc = nullptr;
        acc_bytes = 0;
        if (exec) cudaGraphExecDestroy(exec);
        if (mem) cudaFree(mem);
        if (d_scenes) cudaFree(d_scenes);
        if (samples) cudaFree(samples);
        samples = nullptr;
        samples_bytes = 0;
        if (h_ctr) cudaFreeHost(h_ctr);
        for (auto& x : ev) if (x) cudaEventDestroy(x);
        exec = nullptr; mem = nullptr; d_scenes = nullptr; h_ctr = nullptr;
        for (auto& x : ev) x = nullptr;
    }
};

struct BatchItem {
    aur_scene* scene;
    PathParams p;
    uint32_t npix;
    float4* acc_s;
    float4* acc_c;
    uint32_t lsub() const { return p.light_samples > 1 ? (uint32_t)p.light_samples : 1u; }
    // work items (one per traced or skipped sub-sample) of one camera sample of every pixel
    uint64_t items_per_sample() const { return (uint64_t)npix * lsub(); }
    // paths traced for spp samples from sample_offset (the render's sample 0 traces one)
    uint64_t paths(int spp, int offset) const {
        return (uint64_t)npix * ((uint64_t)spp * lsub() - (offset == 0 && spp > 0 ? lsub() - 1 : 0));
    }
};

// Fills the scene table of one pass: samples [s0, s0 + chunk) of every scene.
static uint32_t fill_table(std::vector<BatchItem>& items, int s0, int chunk, float4* samples, std::vector<WfScene>& tab,
                           int capacity) {
    uint32_t base = 0;
    size_t off = 0;
    tab.assign(capacity, WfScene());
    for (int i = (int)items.size(); i < capacity; ++i) tab[i].item_base = 0xffffffffu;   // never selected
    for (size_t i = 0; i < items.size(); ++i) {
        WfScene& t = tab[i];
        memset(&t, 0, sizeof(t));
        t.sc = items[i].scene->dev();
        t.p = items[i].p;
        const int pass_spp = std::max(0, std::min(chunk, items[i].p.spp - s0));
        t.p.spp = pass_spp;
        t.p.sample_offset = items[i].p.sample_offset + s0;
        t.key = seed_key(items[i].p.seed);
        t.npix = items[i].npix;
        t.lsub = items[i].lsub();
        t.rng_offset = (uint32_t)t.p.sample_offset * t.lsub;
        t.item_base = base;
        t.items = (uint32_t)(items[i].items_per_sample() * (uint32_t)pass_spp);
        t.samples = samples ? samples + off : nullptr;
        base += t.items;
        off += (size_t)items[i].items_per_sample() * chunk;
    }
    return base;
}

// Autotuner: times every candidate (pool size x block size x material sort) on the
// same probe — the first `limit` work items of the real workload (at most 2^25) — and
// keeps the fastest. Pools larger than twice the probe are not tried. (On the 1080p
// depth-8 terrain, pools of 2^21 / 2^22 / 2^23 / 2^24 slots gave 475 / 491 / 504 / 509 M
// samples/s: more paths in flight hide more of the traversal's fetch latency.)
// Returns the chosen configuration.
static aur_status autotune(aur_ctx* ctx, std::vector<BatchItem>& items, WfConfig* best_out) {
    cudaStream_t s = ctx->work_stream;
    size_t per_sample = 0;
    uint64_t total = 0;
    for (auto& it : items) {
        per_sample += (size_t)it.items_per_sample() * sizeof(float4);
        total += it.items_per_sample() * it.p.spp;
    }
    const uint32_t limit = (uint32_t)std::min<uint64_t>(total, 1ull << 25);
    int chunk = 1;   // samples buffer large enough for the probe's first `limit` items
    {
        uint64_t covered = 0;
        while (covered < limit) {
            covered = 0;
            for (auto& it : items) covered += it.items_per_sample() * std::min(chunk, it.p.spp);
            ++chunk;
        }
    }
    float4* samples = nullptr;
    cudaError_t e = cudaMallocAsync(&samples, per_sample * chunk, s);
    if (e != cudaSuccess) return cuda_fail(e, "wavefront autotune");
    std::vector<WfScene> tab;
    fill_table(items, 0, chunk, samples, tab, std::max((int)items.size(), 64));
    constexpr int kPools = 5;
    const uint32_t pools[kPools] = {1u << 20, 1u << 21, 1u << 22, 1u << 23, 1u << 24};
    const int blocks[2] = {128, 256};
    double best = -1.0;
    WfConfig bestc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    bool warmed = false;
    for (int pi = 0; pi < kPools && e == cudaSuccess; ++pi) {
        if (pi > 0 && (uint64_t)pools[pi] > 2ull * limit) break;   // a pool that would stay mostly empty
        for (int bi = 0; bi < 2 && e == cudaSuccess; ++bi)
            for (int so = 0; so < 2 && e == cudaSuccess; ++so) {
                WfConfig c;
                c.pool = pools[pi];
                c.block = blocks[bi];
                c.sort = so;
                c.wide = wide_for(items);
                WfRun run;
                e = run.init(c, (int)items.size(), s);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(run.d_scenes, tab.data(), sizeof(WfScene) * tab.size(), cudaMemcpyHostToDevice, s);
                uint64_t l = 0;
                if (e == cudaSuccess && !warmed) { e = run.run_pass(std::min<uint32_t>(limit, 1u << 20), &l); warmed = true; }
                cudaEventRecord(e0, s);
                if (e == cudaSuccess) e = run.run_pass(limit, &l);
                cudaEventRecord(e1, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                float ms = 0.f;
                if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
                run.release();
                if (e == cudaErrorMemoryAllocation) { cudaGetLastError(); e = cudaSuccess; continue; }
                const double rate = ms > 0.f ? limit / ms : 0.0;
                if (e == cudaSuccess && rate > best) { best = rate; bestc = c; }
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(samples, s);
    cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "wavefront autotune");
    if (best < 0) return fail(AUR_ERR_OOM, "wavefront autotune: no configuration fits in device memory");
    *best_out = bestc;
    return AUR_OK;
}

// Engines (pool buffers, captured graph, events, sample buffer) are cached per
// (context, configuration) and reused by later calls; aur_ctx_destroy releases them.
static std::mutex g_engine_mutex;
static std::map<std::tuple<aur_ctx*, uint32_t, int, int, int, int>, std::unique_ptr<WfRun>> g_engines;

static WfRun* engine_for(aur_ctx* ctx, const WfConfig& cfg, int nscenes, cudaError_t* err) {
    std::lock_guard<std::mutex> lock(g_engine_mutex);
    const auto key = std::make_tuple(ctx, cfg.pool, cfg.block, cfg.sort, cfg.record, cfg.wide);
    auto it = g_engines.find(key);
    if (it != g_engines.end() && it->second->cap_scenes >= nscenes) return it->second.get();
    if (it != g_engines.end()) { it->second->release(); g_engines.erase(it); }
    std::unique_ptr<WfRun> r(new WfRun());
    *err = r->init(cfg, nscenes, ctx->work_stream);
    if (*err != cudaSuccess) { r->release(); return nullptr; }
    WfRun* raw = r.get();
    g_engines.emplace(key, std::move(r));
    return raw;
}

static void wf_drop_engine(aur_ctx* ctx, const WfConfig& cfg) {
    std::lock_guard<std::mutex> lock(g_engine_mutex);
    auto it = g_engines.find(std::make_tuple(ctx, cfg.pool, cfg.block, cfg.sort, cfg.record, cfg.wide));
    if (it != g_engines.end()) { it->second->release(); g_engines.erase(it); }
}

void wf_release_context(aur_ctx* ctx) {
    std::lock_guard<std::mutex> lock(g_engine_mutex);
    for (auto it = g_engines.begin(); it != g_engines.end();) {
        if (std::get<0>(it->first) == ctx) { it->second->release(); it = g_engines.erase(it); }
        else ++it;
    }
}

static int wide_for(const std::vector<BatchItem>& items) {
    if (!AUR_WIDE_TRAVERSAL) return 0;
    for (const BatchItem& it : items)
        if (!it.scene->bvh.bvh.nodes4) return 0;
    return 1;
}

// Renders a batch of scenes with the wavefront engine. films[i]: device float4[npix].
static aur_status wavefront_batch(aur_ctx* ctx, std::vector<BatchItem>& items, const WfConfig& cfg_in,
                                  std::vector<float4*>& films, aur_render_stats* stats, float* kernel_ms) {
    const int n = (int)items.size();
    WfConfig cfg = cfg_in;
    cfg.wide = wide_for(items);
    // The engine runs on the context's own non-blocking stream (graph capture is not
    // allowed on the legacy default stream), ordered after the caller's stream.
    cudaStream_t s = ctx->work_stream;
    cudaEventRecord(ctx->ev_order, ctx->stream);
    cudaStreamWaitEvent(s, ctx->ev_order, 0);
    cudaError_t e = cudaSuccess;
    WfRun* engine = engine_for(ctx, cfg, n, &e);
    if (!engine) return cuda_fail(e, "wavefront: pool allocation");
    WfRun& run = *engine;
    // sample-buffer budget: passes over the spp range when all samples do not fit
    const size_t budget = (size_t)3 << 30;
    size_t per_sample = 0;
    int max_spp = 0;
    for (auto& it : items) {
        per_sample += (size_t)it.items_per_sample() * sizeof(float4);
        max_spp = std::max(max_spp, it.p.spp);
    }
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)max_spp, budget / std::max<size_t>(per_sample, 1)));
    e = run.ensure_samples(per_sample * chunk);
    float4* samples = run.samples;
    size_t per_pixel_set = 0;
    for (auto& it : items) per_pixel_set += (size_t)it.npix * sizeof(float4);
    if (e == cudaSuccess) e = run.ensure_acc(2 * per_pixel_set);   // two float4 per pixel
    {
        size_t off = 0;
        for (auto& it : items) {
            it.acc_s = run.acc + off;
            it.acc_c = run.acc + off + it.npix;
            off += 2 * (size_t)it.npix;
        }
    }
    for (auto& it : items) {
        if (e == cudaSuccess) e = cudaMemsetAsync(it.acc_s, 0, sizeof(float4) * it.npix, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(it.acc_c, 0, sizeof(float4) * it.npix, s);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(run.w.rays, 0, 2 * sizeof(unsigned long long), s);
    for (double& x : run.stage_ms) x = 0.0;
    if (e != cudaSuccess) return cuda_fail(e, "wavefront: sample buffers");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    uint64_t launches = 0;
    std::vector<WfScene> tab;
    for (int s0 = 0; s0 < max_spp && e == cudaSuccess; s0 += chunk) {
        const uint32_t total = fill_table(items, s0, chunk, samples, tab, run.cap_scenes);
        e = cudaMemcpyAsync(run.d_scenes, tab.data(), sizeof(WfScene) * run.cap_scenes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = run.run_pass(total, &launches);
        for (int i = 0; i < n && e == cudaSuccess; ++i) {
            if (tab[i].p.spp == 0) continue;
            k_resolve<<<(items[i].npix + 255) / 256, 256, 0, s>>>(run.d_scenes, i, items[i].acc_s, items[i].acc_c);
            ++launches;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // the scene table is rewritten next pass
    }
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        k_finish<<<(items[i].npix + 255) / 256, 256, 0, s>>>(items[i].acc_s, items[i].acc_c, items[i].npix,
                                                             items[i].p.spp, films[i]);
        ++launches;
        e = cudaGetLastError();
    }
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    unsigned long long rays[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(rays, run.w.rays, sizeof(rays), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaEventRecord(ctx->ev_order, s);              // the caller's stream continues after this work
    cudaStreamWaitEvent(ctx->stream, ctx->ev_order, 0);
    double stage[WfRun::kStages];
    for (int k = 0; k < WfRun::kStages; ++k) stage[k] = run.stage_ms[k];
    if (e != cudaSuccess) wf_drop_engine(ctx, cfg);   // never reuse an engine left in an unknown state
    if (e == cudaErrorLaunchTimeout) return fail(AUR_ERR_TIMEOUT, "wavefront: the path pool did not drain");
    if (e != cudaSuccess) return cuda_fail(e, "wavefront");
    *kernel_ms = ms;
    if (stats) {
        uint64_t paths = 0, cams = 0;
        for (auto& it : items) { paths += it.paths(it.p.spp, it.p.sample_offset); cams += (uint64_t)it.npix * it.p.spp; }
        stats->paths = paths;
        stats->camera_rays = cams;   // camera samples; with light samples every path retraces its camera ray
        stats->closest_rays = rays[0];
        stats->shadow_rays = rays[1];
        stats->launches = launches;
        stats->kernel_ms = ms;
        for (int k = 0; k < WfRun::kStages; ++k) stats->stage_ms[k] = stage[k];
        stats->wf_pool = (int32_t)cfg.pool;
        stats->wf_block = cfg.block;
        stats->wf_sort = cfg.sort;
        stats->node_bytes = cfg.wide ? (int32_t)sizeof(BvhNode4) : (int32_t)sizeof(BvhNode);
    }
    return AUR_OK;
}

// Record pass of the path-replay adjoint: traces samples [s0, s0 + nsamples) of every
// pixel with the wavefront engine in record mode and writes, per item (sample-major:
// sl * npix + pixel), the hit records of its vertices (p.max_depth slots) and its
// unclamped radiance. Ordered after the caller's stream and before its later work.
aur_status wf_record_pass(aur_scene* sc, const PathParams& p, int s0, int nsamples, float4* rec, float4* lo_raw,
                          uint64_t* launches, unsigned long long* rays) {
    aur_ctx* ctx = sc->ctx;
    WfConfig cfg;
    if (sc->wf_tuned) { cfg.pool = (uint32_t)sc->wf_pool; cfg.block = sc->wf_block; cfg.sort = sc->wf_sort; }
    cfg.record = 1;
    std::vector<BatchItem> items(1);
    items[0] = {sc, p, (uint32_t)sc->cam.w * (uint32_t)sc->cam.h, nullptr, nullptr};
    cfg.wide = wide_for(items);
    cudaStream_t s = ctx->work_stream;
    cudaEventRecord(ctx->ev_order, ctx->stream);
    cudaStreamWaitEvent(s, ctx->ev_order, 0);
    cudaError_t e = cudaSuccess;
    WfRun* engine = engine_for(ctx, cfg, 1, &e);
    if (!engine) return cuda_fail(e, "adjoint record pass: pool allocation");
    WfRun& run = *engine;
    std::vector<WfScene> tab;
    const uint32_t total = fill_table(items, s0, nsamples, nullptr, tab, run.cap_scenes);
    tab[0].rec = rec;
    tab[0].lo_raw = lo_raw;
    tab[0].rec_depth = (uint32_t)p.max_depth;
    e = cudaMemsetAsync(run.w.rays, 0, 2 * sizeof(unsigned long long), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(run.d_scenes, tab.data(), sizeof(WfScene) * run.cap_scenes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = run.run_pass(total, launches);
    unsigned long long r[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(r, run.w.rays, sizeof(r), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // the host table and counters are read back
    cudaEventRecord(ctx->ev_order, s);
    cudaStreamWaitEvent(ctx->stream, ctx->ev_order, 0);
    if (e != cudaSuccess) wf_drop_engine(ctx, cfg);
    if (e == cudaErrorLaunchTimeout) return fail(AUR_ERR_TIMEOUT, "adjoint record pass: the path pool did not drain");
    if (e != cudaSuccess) return cuda_fail(e, "adjoint record pass");
    rays[0] += r[0];
    rays[1] += r[1];
    return AUR_OK;
}

static bool wants_tuning(const aur_render_opts* o) { return o->wf_pool == 0 && o->wf_block == 0 && o->wf_sort < 0; }

static WfConfig config_from(const aur_render_opts* o, const WfConfig& base) {
    WfConfig c = base;
    if (o->wf_pool > 0) c.pool = (uint32_t)o->wf_pool;
    if (o->wf_block > 0) c.block = o->wf_block;
    if (o->wf_sort >= 0) c.sort = o->wf_sort;
    return c;
}

static aur_status check_config(const WfConfig& c) {
    if (c.pool < 1024 || c.pool > (1u << 26) || (c.pool & 31))
        return fail(AUR_ERR_INVALID_ARG, "wavefront: pool must be a multiple of 32 in [1024, 2^26]");
    if (c.block != 64 && c.block != 128 && c.block != 256)   // the stage kernels take at most 256
        return fail(AUR_ERR_INVALID_ARG, "wavefront: block must be 64, 128 or 256");
    return AUR_OK;
}

aur_status render_wavefront(aur_scene* sc, const aur_render_opts* o, float* film, aur_render_stats* stats) {
    if (!sc || !o || !film) return fail(AUR_ERR_INVALID_ARG, "aur_render: NULL argument");
    PathParams p;
    aur_status st = render_options(sc, o, &p);
    if (st != AUR_OK) return st;
    if (o->count_work) return fail(AUR_ERR_UNSUPPORTED, "aur_render: count_work is implemented by the plain renderer");
    WfConfig cfg = config_from(o, WfConfig());
    if ((st = check_config(cfg)) != AUR_OK) return st;
    DeviceGuard g(sc->ctx->device);
    cudaStream_t s = sc->ctx->stream;
    const uint32_t npix = (uint32_t)sc->cam.w * sc->cam.h;
    if ((uint64_t)npix * o->spp * (uint64_t)p.light_samples >= (1ull << 31))
        return fail(AUR_ERR_INVALID_ARG, "aur_render: more than 2^31 paths");
    DevOut fo;
    cudaError_t e = fo.init(film, sizeof(float4) * npix, 16, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // film staging allocated on the caller's stream
    if (e != cudaSuccess) return cuda_fail(e, "aur_render(wavefront)");
    std::vector<BatchItem> items(1);
    items[0] = {sc, p, npix, nullptr, nullptr};
    if (wants_tuning(o)) {
        // Tuned once per render shape (triangles, materials, lights, resolution, spp, depths)
        // on this context: a scene rendered at another spp or depth is tuned for that too,
        // and a new scene of the same shape reuses the configuration.
        uint64_t sig = 1469598103934665603ull;
        const uint64_t parts[8] = {sc->ntri, sc->h_mats.size(), sc->h_lights.size(), (uint64_t)sc->cam.w,
                                   (uint64_t)sc->cam.h, (uint64_t)o->spp, (uint64_t)o->max_depth,
                                   (uint64_t)(int64_t)o->min_depth};
        for (uint64_t v : parts) sig = (sig ^ v) * 1099511628211ull;
        auto it = sc->ctx->wf_scene_tuned.find(sig);
        if (it == sc->ctx->wf_scene_tuned.end()) {
            WfConfig t;
            if ((st = autotune(sc->ctx, items, &t)) != AUR_OK) return st;
            it = sc->ctx->wf_scene_tuned.emplace(sig, std::array<int, 3>{(int)t.pool, t.block, t.sort}).first;
        }
        sc->wf_pool = it->second[0]; sc->wf_block = it->second[1]; sc->wf_sort = it->second[2];
        sc->wf_tuned = true;
        cfg.pool = sc->wf_pool; cfg.block = sc->wf_block; cfg.sort = sc->wf_sort;
    }
    std::vector<float4*> films = {(float4*)fo.ptr};
    float ms = 0.f;
    st = wavefront_batch(sc->ctx, items, cfg, films, stats, &ms);
    if (st == AUR_OK) {
        e = fo.finish();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "aur_render(wavefront download)");
    }
    return st;
}

}  // namespace aur

extern "C" aur_status aur_render_batch(aur_scene* const* scenes, const aur_render_opts* opts, uint32_t n,
                                       float* const* films, aur_render_stats* stats) {
    using namespace aur;
    if (!scenes || !opts || !films || n == 0) return fail(AUR_ERR_INVALID_ARG, "aur_render_batch: NULL argument");
    aur_ctx* ctx = scenes[0] ? scenes[0]->ctx : nullptr;
    if (!ctx) return fail(AUR_ERR_INVALID_ARG, "aur_render_batch: NULL scene");
    for (uint32_t i = 0; i < n; ++i)
        if (!scenes[i] || scenes[i]->ctx != ctx || !films[i])
            return fail(AUR_ERR_INVALID_ARG, "aur_render_batch: scenes must share one context and have films");
    WfConfig cfg = config_from(&opts[0], WfConfig());
    aur_status st = check_config(cfg);
    if (st != AUR_OK) return st;
    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    std::vector<BatchItem> items(n);
    std::vector<DevOut> outs(n);
    std::vector<float4*> fl(n);
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) {
        PathParams p;
        if ((st = render_options(scenes[i], &opts[i], &p)) != AUR_OK) return st;
        const uint32_t npix = (uint32_t)scenes[i]->cam.w * scenes[i]->cam.h;
        total += (uint64_t)npix * p.spp * (uint64_t)p.light_samples;
        items[i] = {scenes[i], p, npix, nullptr, nullptr};
    }
    if (total >= (1ull << 31)) return fail(AUR_ERR_INVALID_ARG, "aur_render_batch: more than 2^31 paths");
    cudaError_t e = cudaSuccess;
    for (uint32_t i = 0; i < n && e == cudaSuccess; ++i) {
        e = outs[i].init(films[i], sizeof(float4) * items[i].npix, 16, s);
        fl[i] = (float4*)outs[i].ptr;
    }
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && wants_tuning(&opts[0])) {
        // tuned once per (scene count, path count) on this context
        const uint64_t key = ((uint64_t)n << 40) ^ total;
        auto it = ctx->wf_batch_tuned.find(key);
        if (it == ctx->wf_batch_tuned.end()) {
            WfConfig t;
            st = autotune(ctx, items, &t);
            if (st == AUR_OK) it = ctx->wf_batch_tuned.emplace(key, std::array<int, 3>{(int)t.pool, t.block, t.sort}).first;
        }
        if (st == AUR_OK) { cfg.pool = (uint32_t)it->second[0]; cfg.block = it->second[1]; cfg.sort = it->second[2]; }
    }
    if (e == cudaSuccess && st == AUR_OK) st = wavefront_batch(ctx, items, cfg, fl, stats, &ms);
    else if (e != cudaSuccess) st = cuda_fail(e, "aur_render_batch");
    for (uint32_t i = 0; i < n && st == AUR_OK; ++i) {
        e = outs[i].finish();
        if (e != cudaSuccess) st = cuda_fail(e, "aur_render_batch(download)");
    }
    cudaStreamSynchronize(s);
    return st;
}
