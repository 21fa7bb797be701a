// aur_traverse.cuh — closest-hit and any-hit traversal of the device BVH.
//
// Replaces EmbreeAccelerator::intersect / intersectBinary
// (Aurora/src/geometry/embreeAccelerator.cpp:41-100): closest hit in
// [mint, maxt] returning (t, u, v, prim) with Embree's barycentric convention
// (u weights vertex 1, v vertex 2), and occlusion anywhere in [mint, maxt].
// Nodes and triangles are fetched with 128-bit read-only loads; the traversal
// stack lives in registers/local memory (64 entries, ample for PLOC trees).
// The triangle test is the exact FP32 Moller-Trumbore of tri_intersect, so the
// closest prim equals a brute-force scan's whenever the minimum is unique.
#pragma once
#include <climits>
#include "aur_bvh.cuh"
#include "aur_shading.cuh"

namespace aur {

struct Hit { float t, u, v; int prim; };

// Work counters of one or more traversals: interior-node visits (one 64-byte
// record each) and triangle tests (one 48-byte record each). Kernels that do
// not store them let the compiler drop the increments.
struct TraceWork { uint32_t nodes = 0, tris = 0; };

constexpr int kTraversalStack = 64;

__device__ __forceinline__ float safe_rcp(float x) {
    return __frcp_rn(fabsf(x) > 1e-20f ? x : copysignf(1e-20f, x));
}

// Slab test against one child box; tmin/tmax already carry the rounding slack.
__device__ __forceinline__ bool slab(float lox, float hix, float loy, float hiy, float loz, float hiz,
                                     float3 id, float3 ood, float tmin, float tmax, float* tnear) {
    const float x0 = fmaf(lox, id.x, -ood.x), x1 = fmaf(hix, id.x, -ood.x);
    const float y0 = fmaf(loy, id.y, -ood.y), y1 = fmaf(hiy, id.y, -ood.y);
    const float z0 = fmaf(loz, id.z, -ood.z), z1 = fmaf(hiz, id.z, -ood.z);
    const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
    const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax));
    *tnear = tn;
    return tn <= tf;
}

// Slab test with the near and far planes already chosen by the ray direction's signs
// (for a positive inverse direction the near plane is lo, else hi): the same entry and
// exit distances as slab(), without the per-axis min/max.
__device__ __forceinline__ bool slab_nf(float nx, float fx, float ny, float fy, float nz, float fz, float3 id,
                                        float3 ood, float tmin, float tmax, float* tnear) {
    const float tn = fmaxf(fmaxf(fmaf(nx, id.x, -ood.x), fmaf(ny, id.y, -ood.y)), fmaxf(fmaf(nz, id.z, -ood.z), tmin));
    const float tf = fminf(fminf(fmaf(fx, id.x, -ood.x), fmaf(fy, id.y, -ood.y)), fminf(fmaf(fz, id.z, -ood.z), tmax));
    *tnear = tn;
    return tn <= tf;
}

__device__ __forceinline__ float4 ld_node(const float4* a) { return __ldg(a); }

// 32 contiguous bytes in one 256-bit read-only load (sm_100: ld.global.nc.v8.f32, address
// 32-byte aligned): one L1 request per lane where two 128-bit loads take two.
__device__ __forceinline__ void ld_node2(const float4* a, float4& x, float4& y) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w), "=f"(y.x), "=f"(y.y), "=f"(y.z), "=f"(y.w)
        : "l"(a));
}

// The four children's near and far planes of a 4-wide node, by the direction's signs
// (lox, hix, loy, hiy, loz, hiz order). kLoad256: both planes of each axis in one 256-bit
// load, then chosen by sign in registers (3 load requests instead of 6). Measured on the
// 1080p terrain: the any-hit (next-event) traversal 57.6 vs 59.5 ms per frame with it, the
// closest-hit traversal 118.2 vs 109.2 ms (its 64-register budget spills), so only the
// any-hit traversals use it.
struct Planes4 { float4 nx, fx, ny, fy, nz, fz; };
template <bool kLoad256>
__device__ __forceinline__ Planes4 load_planes4(const BvhNode4* q, float3 id) {
    const float4* p = reinterpret_cast<const float4*>(q);
    Planes4 r;
    if constexpr (kLoad256) {
        float4 lx, hx, ly, hy, lz, hz;
        ld_node2(p, lx, hx);
        ld_node2(p + 2, ly, hy);
        ld_node2(p + 4, lz, hz);
        const bool nx = id.x < 0.f, ny = id.y < 0.f, nz = id.z < 0.f;
        r.nx = nx ? hx : lx; r.fx = nx ? lx : hx;
        r.ny = ny ? hy : ly; r.fy = ny ? ly : hy;
        r.nz = nz ? hz : lz; r.fz = nz ? lz : hz;
    } else {
        const int sx = id.x < 0.f, sy = id.y < 0.f, sz = id.z < 0.f;
        r.nx = ld_node(p + sx); r.fx = ld_node(p + 1 - sx);
        r.ny = ld_node(p + 2 + sy); r.fy = ld_node(p + 3 - sy);
        r.nz = ld_node(p + 4 + sz); r.fz = ld_node(p + 5 - sz);
    }
    return r;
}

// kAnyHit=false: closest hit, returns true when hit->prim >= 0.
// kAnyHit=true : returns true as soon as any triangle is hit in [mint, maxt].
template <bool kAnyHit>
__device__ __forceinline__ bool bvh_trace(const BvhNode* __restrict__ nodes, const BvhTri* __restrict__ tris,
                                          float3 o, float3 d, float mint, float maxt, Hit* hit, TraceWork& work) {
    const float3 id = mk(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z));
    const float3 ood = mk(o.x * id.x, o.y * id.y, o.z * id.z);
    const float box_tmin = mint > 0.f ? mint * 0.99999905f : mint * 1.00000095f;
    float tbest = maxt;
    float box_tmax = tbest * 1.00000095f;
    int best = -1;
    float bu = 0.f, bv = 0.f;
    int stack[kTraversalStack];
    int sp = 0;
    int node = 0;
    while (true) {
        if (node >= 0) {
            ++work.nodes;
            const float4 a = __ldg(&nodes[node].a);
            const float4 b = __ldg(&nodes[node].b);
            const float4 c = __ldg(&nodes[node].c);
            const float4 e = __ldg(&nodes[node].d);
            float t0, t1;
            const bool h0 = slab(a.x, a.y, a.z, a.w, c.x, c.y, id, ood, box_tmin, box_tmax, &t0);
            const bool h1 = slab(b.x, b.y, b.z, b.w, c.z, c.w, id, ood, box_tmin, box_tmax, &t1);
            const int r0 = __float_as_int(e.x), r1 = __float_as_int(e.y);
            if (h0 && h1) {
                const bool first0 = t0 <= t1;
                if (sp < kTraversalStack) stack[sp++] = first0 ? r1 : r0;   // depth <= 63 is checked at build
                node = first0 ? r0 : r1;
                continue;
            }
            if (h0) { node = r0; continue; }
            if (h1) { node = r1; continue; }
        } else {
            const int packed = ~node;
            const int start = packed >> 5, end = start + (packed & 31);
            for (int k = start; k < end; ++k) {
                ++work.tris;
                const float4 p = __ldg(&tris[k].p1);
                const float4 e1 = __ldg(&tris[k].e1);
                const float4 e2 = __ldg(&tris[k].e2);
                float t, u, v;
                if (tri_intersect(mk(p.x, p.y, p.z), mk(e1.x, e1.y, e1.z), mk(e2.x, e2.y, e2.z), o, d, mint, tbest,
                                  &t, &u, &v)) {
                    if (kAnyHit) return true;
                    tbest = t; bu = u; bv = v;
                    best = __float_as_int(p.w);
                    box_tmax = tbest * 1.00000095f;
                }
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    if (kAnyHit) return false;
    hit->t = tbest; hit->u = bu; hit->v = bv; hit->prim = best;
    return best >= 0;
}

// The same traversal over the 4-wide tree (one 128-byte record per node visit; hit
// children nearest first).
constexpr int kTraversalStack4Local = 96;
template <bool kAnyHit>
__device__ __forceinline__ bool bvh_trace4(const BvhNode4* __restrict__ nodes, const BvhTri* __restrict__ tris,
                                           float3 o, float3 d, float mint, float maxt, Hit* hit, TraceWork& work) {
    const float3 id = mk(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z));
    const float3 ood = mk(o.x * id.x, o.y * id.y, o.z * id.z);
    const float box_tmin = mint > 0.f ? mint * 0.99999905f : mint * 1.00000095f;
    const float kMiss = __int_as_float(0x7f800000);
    float tbest = maxt;
    float box_tmax = tbest * 1.00000095f;
    int best = -1;
    float bu = 0.f, bv = 0.f;
    int stack[kTraversalStack4Local];
    int sp = 0;
    int node = 0;
    while (true) {
        if (node >= 0) {
            ++work.nodes;
            const BvhNode4* q = nodes + node;
            const Planes4 pl = load_planes4<kAnyHit>(q, id);
            const int4 rf = __ldg(&q->ref);
            float t[4];
            int r[4] = {rf.x, rf.y, rf.z, rf.w};
            float tc;
            t[0] = slab_nf(pl.nx.x, pl.fx.x, pl.ny.x, pl.fy.x, pl.nz.x, pl.fz.x, id, ood, box_tmin, box_tmax, &tc) ? tc : kMiss;
            t[1] = slab_nf(pl.nx.y, pl.fx.y, pl.ny.y, pl.fy.y, pl.nz.y, pl.fz.y, id, ood, box_tmin, box_tmax, &tc) ? tc : kMiss;
            t[2] = slab_nf(pl.nx.z, pl.fx.z, pl.ny.z, pl.fy.z, pl.nz.z, pl.fz.z, id, ood, box_tmin, box_tmax, &tc) ? tc : kMiss;
            t[3] = slab_nf(pl.nx.w, pl.fx.w, pl.ny.w, pl.fy.w, pl.nz.w, pl.fz.w, id, ood, box_tmin, box_tmax, &tc) ? tc : kMiss;
            auto cx = [&](int i, int j) {   // nearest first, as the resumable traversal
                if (t[j] < t[i]) { const float tt = t[i]; t[i] = t[j]; t[j] = tt; const int rr = r[i]; r[i] = r[j]; r[j] = rr; }
            };
            cx(0, 1); cx(2, 3); cx(0, 2); cx(1, 3); cx(1, 2);
            if (t[0] != kMiss) {
                if (t[3] != kMiss && sp < kTraversalStack4Local) stack[sp++] = r[3];
                if (t[2] != kMiss && sp < kTraversalStack4Local) stack[sp++] = r[2];
                if (t[1] != kMiss && sp < kTraversalStack4Local) stack[sp++] = r[1];
                node = r[0];
                continue;
            }
        } else {
            const int packed = ~node;
            const int start = packed >> 5, end = start + (packed & 31);
            for (int k = start; k < end; ++k) {
                ++work.tris;
                const float4 p = __ldg(&tris[k].p1);
                const float4 e1 = __ldg(&tris[k].e1);
                const float4 e2 = __ldg(&tris[k].e2);
                float t, u, v;
                if (tri_intersect(mk(p.x, p.y, p.z), mk(e1.x, e1.y, e1.z), mk(e2.x, e2.y, e2.z), o, d, mint, tbest,
                                  &t, &u, &v)) {
                    if (kAnyHit) return true;
                    tbest = t; bu = u; bv = v;
                    best = __float_as_int(p.w);
                    box_tmax = tbest * 1.00000095f;
                }
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    if (kAnyHit) return false;
    hit->t = tbest; hit->u = bu; hit->v = bv; hit->prim = best;
    return best >= 0;
}

__device__ __forceinline__ bool bvh_closest(const BvhNode* nodes, const BvhTri* tris, float3 o, float3 d, float mint,
                                            float maxt, Hit* hit, TraceWork& work) {
    return bvh_trace<false>(nodes, tris, o, d, mint, maxt, hit, work);
}
__device__ __forceinline__ bool bvh_occluded(const BvhNode* nodes, const BvhTri* tris, float3 o, float3 d, float mint,
                                             float maxt, TraceWork& work) {
    Hit h;
    return bvh_trace<true>(nodes, tris, o, d, mint, maxt, &h, work);
}
// The 4-wide tree when there is one, else the binary tree.
__device__ __forceinline__ bool bvh_closest(const BvhNode* nodes, const BvhNode4* nodes4, const BvhTri* tris, float3 o,
                                            float3 d, float mint, float maxt, Hit* hit, TraceWork& work) {
    if (nodes4) return bvh_trace4<false>(nodes4, tris, o, d, mint, maxt, hit, work);
    return bvh_trace<false>(nodes, tris, o, d, mint, maxt, hit, work);
}
__device__ __forceinline__ bool bvh_occluded(const BvhNode* nodes, const BvhNode4* nodes4, const BvhTri* tris, float3 o,
                                             float3 d, float mint, float maxt, TraceWork& work) {
    Hit h;
    if (nodes4) return bvh_trace4<true>(nodes4, tris, o, d, mint, maxt, &h, work);
    return bvh_trace<true>(nodes, tris, o, d, mint, maxt, &h, work);
}

}  // namespace aur

namespace aur {

// Traversal stack of one thread: the first kSharedDepth entries live in shared
// memory laid out [depth][thread] (consecutive threads hit consecutive banks at
// any mix of depths, one wavefront per warp access), deeper entries in local memory.
constexpr int kSharedDepth = 24;   // all-local stacks measured 1.7% slower in k_extend
// A 4-wide node pushes up to three entries: the stack of its traversal holds 96
// (the collapse checks 3 x 4-wide depth + 1 against it).
constexpr int kTraversalStack4 = 96;
template <int kCap>
struct LaneStackT {
    int* col;                       // &s_stack[threadIdx.x]
    int stride;                     // blockDim.x
    int deep[kCap - kSharedDepth];
    __device__ __forceinline__ void set(int i, int v) {
        if (i < kSharedDepth) col[i * stride] = v; else deep[i - kSharedDepth] = v;
    }
    __device__ __forceinline__ int get(int i) const {
        return i < kSharedDepth ? col[i * stride] : deep[i - kSharedDepth];
    }
};
using LaneStack = LaneStackT<kTraversalStack>;
using LaneStack4 = LaneStackT<kTraversalStack4>;

// Resumable traversal of one ray, for persistent kernels whose lanes take a new
// ray as soon as theirs finishes (lane refill). Same visiting order, slack and
// exact triangle test as bvh_trace; round() advances every lane of a warp by one
// while-while round and returns true when this lane's ray is finished.
template <bool kAnyHit>
struct TraceState {
    float3 o, d, id, ood;
    float mint, tbest, box_tmin, box_tmax, bu, bv;
    int node, sp, best;
    bool hit_any;

    __device__ __forceinline__ void begin(float3 o_, float3 d_, float mint_, float maxt_) {
        o = o_; d = d_;
        id = mk(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z));
        ood = mk(o.x * id.x, o.y * id.y, o.z * id.z);
        mint = mint_;
        box_tmin = mint > 0.f ? mint * 0.99999905f : mint * 1.00000095f;
        tbest = maxt_;
        box_tmax = tbest * 1.00000095f;
        bu = bv = 0.f;
        node = 0; sp = 0; best = -1;
        leaf = kNone;
        hit_any = false;
    }

    // One round of "while-while" traversal with speculative leaf postponing (Aila &
    // Laine, "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009): the
    // interior loop runs until every lane of the warp holds a leaf (or has finished),
    // lanes that already hold one keep descending speculatively, then all lanes test
    // their leaf's triangles together. `live` marks lanes that have a ray; all 32
    // lanes of the warp must call round(). Returns true when this lane's ray is done.
    int leaf;        // postponed leaf reference, kNone if none
    static constexpr int kNone = INT_MIN;

    __device__ __forceinline__ bool round(const BvhNode* __restrict__ nodes, const BvhTri* __restrict__ tris,
                                          LaneStack& stack, bool live) {
        bool finished = !live;
        if (live && leaf == kNone && node == kNone) finished = true;
        // interior phase
        while (true) {
            bool searching = false;
            if (!finished && node != kNone && node >= 0) {
                const float4 a = __ldg(&nodes[node].a);
                const float4 b = __ldg(&nodes[node].b);
                const float4 c = __ldg(&nodes[node].c);
                const float4 e = __ldg(&nodes[node].d);
                float t0, t1;
                const bool h0 = slab(a.x, a.y, a.z, a.w, c.x, c.y, id, ood, box_tmin, box_tmax, &t0);
                const bool h1 = slab(b.x, b.y, b.z, b.w, c.z, c.w, id, ood, box_tmin, box_tmax, &t1);
                const int r0 = __float_as_int(e.x), r1 = __float_as_int(e.y);
                if (h0 && h1) {
                    const bool first0 = t0 <= t1;
                    if (sp < kTraversalStack) stack.set(sp++, first0 ? r1 : r0);   // depth <= 63 is checked at build
                    node = first0 ? r0 : r1;
                } else if (h0) node = r0;
                else if (h1) node = r1;
                else node = sp > 0 ? stack.get(--sp) : kNone;
            }
            if (!finished && node != kNone && node < 0 && leaf == kNone) {   // postpone this leaf
                leaf = node;
                node = sp > 0 ? stack.get(--sp) : kNone;
            }
            if (!finished) searching = leaf == kNone && node != kNone;   // still looking for a leaf
            if (!__any_sync(0xffffffffu, searching)) break;
        }
        // leaf phase
        if (!finished && leaf != kNone) {
            const int packed = ~leaf;
            const int start = packed >> 5, end = start + (packed & 31);
            leaf = kNone;
            for (int k = start; k < end; ++k) {
                const float4 p = __ldg(&tris[k].p1);
                const float4 e1 = __ldg(&tris[k].e1);
                const float4 e2 = __ldg(&tris[k].e2);
                float t, u, v;
                if (tri_intersect(mk(p.x, p.y, p.z), mk(e1.x, e1.y, e1.z), mk(e2.x, e2.y, e2.z), o, d, mint, tbest,
                                  &t, &u, &v)) {
                    if (kAnyHit) { hit_any = true; return true; }
                    tbest = t; bu = u; bv = v;
                    best = __float_as_int(p.w);
                    box_tmax = tbest * 1.00000095f;
                }
            }
        }
        if (finished) return live;
        return leaf == kNone && node == kNone;
    }
};

// The same resumable while-while traversal over the 4-wide tree: a node visit loads
// one 128-byte record, tests four boxes, and continues with the nearest hit child
// while the other hit children go on the stack, farthest first. Boxes and the triangle
// test are the binary tree's, so the closest hit equals it whenever the minimum is unique.
template <bool kAnyHit>
struct TraceState4 {
    float3 o, d, id, ood;
    float mint, tbest, box_tmin, box_tmax, bu, bv;
    int node, sp, best;
    bool hit_any;
    int leaf;
    static constexpr int kNone = INT_MIN;

    __device__ __forceinline__ void begin(float3 o_, float3 d_, float mint_, float maxt_) {
        o = o_; d = d_;
        id = mk(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z));
        ood = mk(o.x * id.x, o.y * id.y, o.z * id.z);
        mint = mint_;
        box_tmin = mint > 0.f ? mint * 0.99999905f : mint * 1.00000095f;
        tbest = maxt_;
        box_tmax = tbest * 1.00000095f;
        bu = bv = 0.f;
        node = 0; sp = 0; best = -1;
        leaf = kNone;
        hit_any = false;
    }

    __device__ __forceinline__ void visit(const BvhNode4* __restrict__ nodes, LaneStack4& stack) {
        const BvhNode4* q = nodes + node;
        const Planes4 pl = load_planes4<kAnyHit>(q, id);
        const float4 rff = ld_node(reinterpret_cast<const float4*>(&q->ref));
        const int4 rf = make_int4(__float_as_int(rff.x), __float_as_int(rff.y), __float_as_int(rff.z),
                                  __float_as_int(rff.w));
        const float kMiss = __int_as_float(0x7f800000);
        float t[4];
        int r[4] = {rf.x, rf.y, rf.z, rf.w};
        float tc;
        t[0] = slab_nf(pl.nx.x, pl.fx.x, pl.ny.x, pl.fy.x, pl.nz.x, pl.fz.x, id, ood, box_tmin, box_tmax, &tc) ? tc : kMiss;
        t[1] = slab_nf(pl.nx.y, pl.fx.y, pl.ny.y, pl.fy.y, pl.nz.y, pl.fz.y, id, ood, box_tmin, box_tmax, &tc) ? tc : kMiss;
        t[2] = slab_nf(pl.nx.z, pl.fx.z, pl.ny.z, pl.fy.z, pl.nz.z, pl.fz.z, id, ood, box_tmin, box_tmax, &tc) ? tc : kMiss;
        t[3] = slab_nf(pl.nx.w, pl.fx.w, pl.ny.w, pl.fy.w, pl.nz.w, pl.fz.w, id, ood, box_tmin, box_tmax, &tc) ? tc : kMiss;
        // ascending by entry distance (misses last): a five-exchange network. Any-hit rays
        // take the same order (nearest first measured 1.6% faster than slot order for the
        // next-event rays, whose occluders tend to lie near the shading point).
        auto cx = [&](int i, int j) {
            if (t[j] < t[i]) { const float tt = t[i]; t[i] = t[j]; t[j] = tt; const int rr = r[i]; r[i] = r[j]; r[j] = rr; }
        };
        cx(0, 1); cx(2, 3); cx(0, 2); cx(1, 3); cx(1, 2);
        if (t[0] == kMiss) { node = sp > 0 ? stack.get(--sp) : kNone; return; }
        if (t[3] != kMiss && sp < kTraversalStack4) stack.set(sp++, r[3]);
        if (t[2] != kMiss && sp < kTraversalStack4) stack.set(sp++, r[2]);
        if (t[1] != kMiss && sp < kTraversalStack4) stack.set(sp++, r[1]);
        node = r[0];
    }

    // As TraceState::round: interior phase until every live lane holds a leaf, then the
    // leaf phase. All 32 lanes of the warp must call it.
    __device__ __forceinline__ bool round(const BvhNode4* __restrict__ nodes, const BvhTri* __restrict__ tris,
                                          LaneStack4& stack, bool live) {
        bool finished = !live;
        if (live && leaf == kNone && node == kNone) finished = true;
        while (true) {
            bool searching = false;
            if (!finished && node != kNone && node >= 0) visit(nodes, stack);
            if (!finished && node != kNone && node < 0 && leaf == kNone) {   // postpone this leaf
                leaf = node;
                node = sp > 0 ? stack.get(--sp) : kNone;
            }
            if (!finished) searching = leaf == kNone && node != kNone;
            if (!__any_sync(0xffffffffu, searching)) break;
        }
        if (!finished && leaf != kNone) {
            const int packed = ~leaf;
            const int start = packed >> 5, end = start + (packed & 31);
            leaf = kNone;
            for (int k = start; k < end; ++k) {
                const float4 p = __ldg(&tris[k].p1);
                const float4 e1 = __ldg(&tris[k].e1);
                const float4 e2 = __ldg(&tris[k].e2);
                float t, u, v;
                if (tri_intersect(mk(p.x, p.y, p.z), mk(e1.x, e1.y, e1.z), mk(e2.x, e2.y, e2.z), o, d, mint, tbest,
                                  &t, &u, &v)) {
                    if (kAnyHit) { hit_any = true; return true; }
                    tbest = t; bu = u; bv = v;
                    best = __float_as_int(p.w);
                    box_tmax = tbest * 1.00000095f;
                }
            }
        }
        if (finished) return live;
        return leaf == kNone && node == kNone;
    }
};

}  // namespace aur
