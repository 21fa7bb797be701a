// bvh_build.cu — SAH-quality BVH built entirely on the device.
//
// Stands in for embree::rtcCreateAccel("bvh4.spatialsplit", "triangle4", ...)
// (Aurora/src/geometry/embreeAccelerator.cpp:24-32) over the flattened
// camera-space triangle soup of Renderer::buildRenderEnvironment
// (Aurora/src/frontend/renderer.cpp:99-145, triangleMesh.cpp:57-81).
//
// Pipeline (all kernels in this file, no library calls):
//   1. triangle boxes + centroid bounds            k_prim_setup
//   2. 30-bit Morton codes, stable LSD radix sort   k_morton, k_radix_hist/k_radix_scatter
//   3. PLOC agglomerative clustering (Meister & Bittner, "Parallel Locally-
//      Ordered Clustering for BVH Construction", IEEE TVCG 2018): every cluster
//      finds its nearest neighbour (smallest merged surface area) within a
//      window of the Morton order; mutual pairs merge; the list is compacted
//      with an order-preserving scan. Ties are broken on the index pair so that
//      the globally best pair is always mutual (guaranteed progress).
//   4. bottom-up SAH leaf collapse (atomic second-arrival walk)
//   5. deterministic depth-first layout: every node derives its output slot by
//      walking to the root, so the result is independent of thread timing.
//   6. the 4-wide tree: an SAH-optimal grouping of the binary nodes (a bottom-up
//      dynamic program), built level by level.
#include "aur_bvh.cuh"
#include "aur_shading.cuh"
#include <cfloat>
#include <vector>

namespace aur {
namespace {

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return e_; } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t n, cudaStream_t s) { return cudaMallocAsync((void**)p, sizeof(T) * (n ? n : 1), s); }
template <typename T>
void dfree(T*& p, cudaStream_t s) { if (p) cudaFreeAsync(p, s); p = nullptr; }

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// ------------------------------------------------------------ exclusive scan
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// In-place safe: each thread reads its own items before writing them.
__global__ void k_scan_tiles(const uint32_t* in, uint32_t* out, uint32_t* sums, int n) {
    __shared__ uint32_t s_warp[kScanThreads / 32];
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) { int i = base + k; v[k] = i < n ? in[i] : 0u; local += v[k]; }
    uint32_t incl = warp_incl_scan(local);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
        w = warp_incl_scan(w);
        if (lane < kScanThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    uint32_t excl = incl - local + (warp > 0 ? s_warp[warp - 1] : 0u);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) { int i = base + k; if (i < n) out[i] = excl; excl += v[k]; }
    if (sums && threadIdx.x == 0) sums[blockIdx.x] = s_warp[kScanThreads / 32 - 1];
}

__global__ void k_scan_add(uint32_t* out, const uint32_t* add, int n) {
    const int base = blockIdx.x * kScanTile;
    const uint32_t a = add[blockIdx.x];
    const int end = min(base + kScanTile, n);
    for (int i = base + threadIdx.x; i < end; i += blockDim.x) out[i] += a;
}

cudaError_t exclusive_scan(const uint32_t* in, uint32_t* out, int n, cudaStream_t s) {
    const int nb = div_up(n, kScanTile);
    if (nb <= 1) { k_scan_tiles<<<1, kScanThreads, 0, s>>>(in, out, nullptr, n); return cudaGetLastError(); }
    uint32_t* sums = nullptr;
    CK(dalloc(&sums, nb, s));
    k_scan_tiles<<<nb, kScanThreads, 0, s>>>(in, out, sums, n);
    CK(exclusive_scan(sums, sums, nb, s));
    k_scan_add<<<nb, 256, 0, s>>>(out, sums, n);
    dfree(sums, s);
    return cudaGetLastError();
}

// ------------------------------------------------------------ radix sort
// Stable LSD sort of (key, value) pairs, 8 bits per pass. One warp per block
// walks its 2048-key tile in order, so ranks within a digit follow input order.
constexpr int kSortTile = 2048;

__global__ void k_radix_hist(const uint32_t* keys, int n, int shift, uint32_t* hist, int nb) {
    __shared__ uint32_t s_h[256];
    const int lane = threadIdx.x;
    for (int d = lane; d < 256; d += 32) s_h[d] = 0;
    __syncwarp();
    const int base = blockIdx.x * kSortTile;
    for (int k = 0; k < kSortTile / 32; ++k) {
        int i = base + k * 32 + lane;
        if (i < n) atomicAdd(&s_h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncwarp();
    for (int d = lane; d < 256; d += 32) hist[d * nb + blockIdx.x] = s_h[d];
}

__global__ void k_radix_scatter(const uint32_t* keys, const uint32_t* vals, uint32_t* okeys, uint32_t* ovals,
                                int n, int shift, const uint32_t* offs, int nb) {
    __shared__ uint32_t s_off[256];
    const int lane = threadIdx.x;
    for (int d = lane; d < 256; d += 32) s_off[d] = offs[d * nb + blockIdx.x];
    __syncwarp();
    const int base = blockIdx.x * kSortTile;
    for (int k = 0; k < kSortTile / 32; ++k) {
        const int i = base + k * 32 + lane;
        const bool valid = i < n;
        const uint32_t active = __ballot_sync(0xffffffffu, valid);
        if (!active) break;
        if (valid) {
            const uint32_t key = keys[i], val = vals[i];
            const uint32_t d = (key >> shift) & 255u;
            const uint32_t peers = __match_any_sync(active, d);
            const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
            const int leader = __ffs(peers) - 1;
            const uint32_t b = s_off[d];
            __syncwarp(active);
            if (lane == leader) s_off[d] = b + __popc(peers);
            okeys[b + rank] = key;
            ovals[b + rank] = val;
        }
        __syncwarp();
    }
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, int n, int bits, cudaStream_t s) {
    const int nb = div_up(n, kSortTile);
    uint32_t *k2 = nullptr, *v2 = nullptr, *hist = nullptr;
    CK(dalloc(&k2, n, s)); CK(dalloc(&v2, n, s)); CK(dalloc(&hist, (size_t)256 * nb, s));
    uint32_t *ka = keys, *va = vals, *kb = k2, *vb = v2;
    for (int shift = 0; shift < bits; shift += 8) {
        k_radix_hist<<<nb, 32, 0, s>>>(ka, n, shift, hist, nb);
        CK(exclusive_scan(hist, hist, 256 * nb, s));
        k_radix_scatter<<<nb, 32, 0, s>>>(ka, va, kb, vb, n, shift, hist, nb);
        std::swap(ka, kb); std::swap(va, vb);
    }
    if (ka != keys) {
        CK(cudaMemcpyAsync(keys, ka, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
    dfree(k2, s); dfree(v2, s); dfree(hist, s);
    return cudaGetLastError();
}

// ------------------------------------------------------------ primitives
__device__ __forceinline__ int f2ord(float f) { int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7fffffff; }
__device__ __forceinline__ float ord2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__device__ __forceinline__ float3 ld3(const float* v, uint32_t i) { return mk(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }

__global__ void k_prim_setup(const float* verts, const uint32_t* idx, int n, float4* plo, float4* phi, float4* cent,
                             int* gb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float c[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, C[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    if (i < n) {
        float3 a = ld3(verts, idx[3 * i]), b = ld3(verts, idx[3 * i + 1]), d = ld3(verts, idx[3 * i + 2]);
        float3 lo = mk(fminf(fminf(a.x, b.x), d.x), fminf(fminf(a.y, b.y), d.y), fminf(fminf(a.z, b.z), d.z));
        float3 hi = mk(fmaxf(fmaxf(a.x, b.x), d.x), fmaxf(fmaxf(a.y, b.y), d.y), fmaxf(fmaxf(a.z, b.z), d.z));
        plo[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
        phi[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
        float3 ce = (lo + hi) * 0.5f;
        cent[i] = make_float4(ce.x, ce.y, ce.z, 0.f);
        c[0] = C[0] = ce.x; c[1] = C[1] = ce.y; c[2] = C[2] = ce.z;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            c[k] = fminf(c[k], __shfl_xor_sync(0xffffffffu, c[k], o));
            C[k] = fmaxf(C[k], __shfl_xor_sync(0xffffffffu, C[k], o));
        }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; ++k) { atomicMin(&gb[k], f2ord(c[k])); atomicMax(&gb[3 + k], f2ord(C[k])); }
}

__global__ void k_init_bounds(int* gb) {
    if (threadIdx.x < 3) { gb[threadIdx.x] = f2ord(FLT_MAX); gb[3 + threadIdx.x] = f2ord(-FLT_MAX); }
}

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_morton(const float4* cent, int n, const int* gb, uint32_t* keys, uint32_t* vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3], sc[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = ord2f(gb[k]);
        float ext = ord2f(gb[3 + k]) - lo[k];
        sc[k] = ext > 0.f ? 1023.f / ext : 0.f;
    }
    float4 c = cent[i];
    uint32_t q[3];
    float cc[3] = {c.x, c.y, c.z};
    for (int k = 0; k < 3; ++k) {
        float f = (cc[k] - lo[k]) * sc[k];
        f = fminf(fmaxf(f, 0.f), 1023.f);
        q[k] = (uint32_t)f;
    }
    keys[i] = (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
    vals[i] = (uint32_t)i;
}

// ------------------------------------------------------------ PLOC
struct Tree {
    float4 *lo, *hi;
    int *left, *right, *parent;
};

__global__ void k_init_leaves(const uint32_t* sorted, int n, const float4* plo, const float4* phi, Tree t, int* clusters) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t p = sorted[k];
    t.lo[k] = plo[p];
    t.hi[k] = phi[p];
    t.left[k] = -1;
    t.right[k] = -1;
    t.parent[k] = -1;
    clusters[k] = k;
}

__device__ __forceinline__ float half_area(float3 lo, float3 hi) {
    float3 d = hi - lo;
    return d.x * d.y + d.y * d.z + d.z * d.x;
}

constexpr int kNnBlock = 256;
constexpr int kPlocBatch = 8;
constexpr int kMaxRadius = 32;

// The cluster count m lives on the device (dm) so that several iterations run between host
// synchronisations; grids are sized for an upper bound of it.
__global__ void __launch_bounds__(kNnBlock) k_ploc_nn(const int* clusters, const int* dm, Tree t, int* nn, int r) {
    __shared__ float3 s_lo[kNnBlock + 2 * kMaxRadius], s_hi[kNnBlock + 2 * kMaxRadius];
    const int m = *dm;
    const int start = blockIdx.x * kNnBlock - r;
    const int count = kNnBlock + 2 * r;
    for (int k = threadIdx.x; k < count; k += kNnBlock) {
        const int g = start + k;
        if (g >= 0 && g < m) {
            const int c = clusters[g];
            float4 a = t.lo[c], b = t.hi[c];
            s_lo[k] = mk(a.x, a.y, a.z);
            s_hi[k] = mk(b.x, b.y, b.z);
        }
    }
    __syncthreads();
    const int i = blockIdx.x * kNnBlock + threadIdx.x;
    if (i >= m) return;
    const float3 mlo = s_lo[threadIdx.x + r], mhi = s_hi[threadIdx.x + r];
    float best = FLT_MAX;
    int bj = -1;
    const int j0 = max(0, i - r), j1 = min(m - 1, i + r);
    for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        const int sj = j - start;
        float3 lo = mk(fminf(mlo.x, s_lo[sj].x), fminf(mlo.y, s_lo[sj].y), fminf(mlo.z, s_lo[sj].z));
        float3 hi = mk(fmaxf(mhi.x, s_hi[sj].x), fmaxf(mhi.y, s_hi[sj].y), fmaxf(mhi.z, s_hi[sj].z));
        const float a = half_area(lo, hi);
        // strict order on unordered pairs: (area, min index, max index); j increases,
        // so for equal area the first j seen has the smaller pair key.
        if (a < best) { best = a; bj = j; }
    }
    nn[i] = bj;
}

__global__ void k_ploc_merge(int* clusters, const int* dm, int bound, const int* nn, Tree t, int* node_counter,
                             uint32_t* keep) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bound) return;
    if (i >= *dm) { keep[i] = 0u; return; }   // the scan runs over the bound
    const int j = nn[i];
    if (j >= 0 && nn[j] == i) {
        if (i < j) {
            const int a = clusters[i], b = clusters[j];
            const int node = atomicAdd(node_counter, 1);
            float4 la = t.lo[a], lb = t.lo[b], ha = t.hi[a], hb = t.hi[b];
            t.lo[node] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.f);
            t.hi[node] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.f);
            t.left[node] = a;
            t.right[node] = b;
            t.parent[node] = -1;
            t.parent[a] = node;
            t.parent[b] = node;
            clusters[i] = node;
            keep[i] = 1u;
        } else {
            keep[i] = 0u;
        }
    } else {
        keep[i] = 1u;
    }
}

__global__ void k_compact(const int* in, const uint32_t* keep, const uint32_t* pos, const int* dm, int* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < *dm && keep[i]) out[pos[i]] = in[i];
}

// The next cluster count: the kept clusters of the compaction.
__global__ void k_ploc_count(const uint32_t* keep, const uint32_t* pos, int* dm) {
    const int m = *dm;
    *dm = (int)(pos[m - 1] + keep[m - 1]);
}

// ------------------------------------------------------------ SAH collapse
struct Sah {
    int *cnt, *icount, *visit;
    float* cost;
    unsigned char* collapsed;
};

__global__ void k_bottom_up(int n, Tree t, Sah s, int max_leaf, float ct, float ci) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    {
        float4 a = t.lo[k], b = t.hi[k];
        s.cnt[k] = 1;
        s.cost[k] = ci * half_area(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z));
        s.icount[k] = 0;
        s.collapsed[k] = 1;
    }
    __threadfence();
    int node = t.parent[k];
    while (node >= 0) {
        if (atomicAdd(&s.visit[node], 1) == 0) return;
        __threadfence();
        const int l = t.left[node], r = t.right[node];
        const int cl = __ldcg(&s.cnt[l]), cr = __ldcg(&s.cnt[r]);
        const float kl = __ldcg(&s.cost[l]), kr = __ldcg(&s.cost[r]);
        const int il = __ldcg(&s.icount[l]), ir = __ldcg(&s.icount[r]);
        float4 a = t.lo[node], b = t.hi[node];
        const float A = half_area(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z));
        const int c = cl + cr;
        const float split = ct * A + kl + kr;
        const float leaf = c <= max_leaf ? ci * A * (float)c : FLT_MAX;
        s.cnt[node] = c;
        if (leaf <= split) { s.cost[node] = leaf; s.icount[node] = 0; s.collapsed[node] = 1; }
        else { s.cost[node] = split; s.icount[node] = 1 + il + ir; s.collapsed[node] = 0; }
        __threadfence();
        node = t.parent[node];
    }
}

__global__ void k_fix_root(int root, Tree t, Sah s) {
    if (s.collapsed[root]) {
        s.collapsed[root] = 0;
        s.icount[root] = 1 + s.icount[t.left[root]] + s.icount[t.right[root]];
    }
}

// ------------------------------------------------------------ layout
// Outward padding: 2^-19 of the box's own magnitude, and at least 2^-20 of the
// scene's magnitude (covers the rounding of slab distances for rays whose
// origin lies anywhere inside the scene bounds).
__device__ __forceinline__ void pad_box(float& lo, float& hi, float floor_pad) {
    const float m = fmaxf(fmaxf(fabsf(lo), fabsf(hi)), hi - lo);
    const float p = fmaxf(m * 1.9073486e-6f, floor_pad) + 1e-30f;
    lo -= p;
    hi += p;
}

__global__ void k_layout_tris(int n, Tree t, Sah s, const uint32_t* sorted, const float* verts, const uint32_t* idx,
                              BvhTri* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int pos = 0, x = k, p;
    while ((p = t.parent[x]) >= 0) {
        if (t.right[p] == x) pos += s.cnt[t.left[p]];
        x = p;
    }
    const uint32_t prim = sorted[k];
    float3 a = ld3(verts, idx[3 * prim]), b = ld3(verts, idx[3 * prim + 1]), c = ld3(verts, idx[3 * prim + 2]);
    float3 e1 = xsub(b, a), e2 = xsub(c, a);
    BvhTri tr;
    tr.p1 = make_float4(a.x, a.y, a.z, __int_as_float((int)prim));
    tr.e1 = make_float4(e1.x, e1.y, e1.z, 0.f);
    tr.e2 = make_float4(e2.x, e2.y, e2.z, 0.f);
    out[pos] = tr;
}

__global__ void k_layout_nodes(int n, int total, Tree t, Sah s, float floor_pad, BvhNode* out, int* max_depth) {
    const int x = n + blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= total || s.collapsed[x]) return;
    int idx = 0, start = 0, y = x, p, depth = 1;
    while ((p = t.parent[y]) >= 0) {
        if (s.collapsed[p]) return;      // inside a collapsed leaf subtree
        const int l = t.left[p];
        if (t.right[p] == y) { idx += 1 + s.icount[l]; start += s.cnt[l]; }
        else idx += 1;
        y = p;
        ++depth;
    }
    atomicMax(max_depth, depth);
    const int l = t.left[x], r = t.right[x];
    int ref[2], cnt[2];
    const int ch[2] = {l, r};
    const int cidx[2] = {idx + 1, idx + 1 + s.icount[l]};
    const int cstart[2] = {start, start + s.cnt[l]};
    float blo[2][3], bhi[2][3];
    for (int k = 0; k < 2; ++k) {
        const int c = ch[k];
        if (c < n || s.collapsed[c]) { ref[k] = ~((cstart[k] << 5) | s.cnt[c]); cnt[k] = s.cnt[c]; }
        else { ref[k] = cidx[k]; cnt[k] = 0; }
        float4 a = t.lo[c], b = t.hi[c];
        blo[k][0] = a.x; blo[k][1] = a.y; blo[k][2] = a.z;
        bhi[k][0] = b.x; bhi[k][1] = b.y; bhi[k][2] = b.z;
        for (int d = 0; d < 3; ++d) pad_box(blo[k][d], bhi[k][d], floor_pad);
    }
    BvhNode nd;
    nd.a = make_float4(blo[0][0], bhi[0][0], blo[0][1], bhi[0][1]);
    nd.b = make_float4(blo[1][0], bhi[1][0], blo[1][1], bhi[1][1]);
    nd.c = make_float4(blo[0][2], bhi[0][2], blo[1][2], bhi[1][2]);
    nd.d = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), __int_as_float(cnt[0]), __int_as_float(cnt[1]));
    out[idx] = nd;
}

// single triangle: one node with a leaf child and an empty child
__global__ void k_single(const float* verts, const uint32_t* idx, BvhNode* nodes, BvhTri* tris) {
    float3 a = ld3(verts, idx[0]), b = ld3(verts, idx[1]), c = ld3(verts, idx[2]);
    float lo[3] = {fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z)};
    float hi[3] = {fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z)};
    for (int d = 0; d < 3; ++d) pad_box(lo[d], hi[d], 0.f);
    BvhNode nd;
    nd.a = make_float4(lo[0], hi[0], lo[1], hi[1]);
    nd.b = make_float4(FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX);
    nd.c = make_float4(lo[2], hi[2], FLT_MAX, -FLT_MAX);
    nd.d = make_float4(__int_as_float(~1), __int_as_float(~0), __int_as_float(1), __int_as_float(0));
    nodes[0] = nd;
    float3 e1 = xsub(b, a), e2 = xsub(c, a);
    tris[0].p1 = make_float4(a.x, a.y, a.z, __int_as_float(0));
    tris[0].e1 = make_float4(e1.x, e1.y, e1.z, 0.f);
    tris[0].e2 = make_float4(e2.x, e2.y, e2.z, 0.f);
}

}  // namespace

cudaError_t bvh_build_device(const float* verts, const uint32_t* idx, int n, const BvhBuildOptions& opt,
                             DeviceBvh* out, cudaStream_t s) {
    if (n < 1) return cudaErrorInvalidValue;
    *out = DeviceBvh();
    out->num_tris = n;
    CK(dalloc(&out->tris, n, s));
    if (n == 1) {
        CK(dalloc(&out->nodes, 1, s));
        out->num_nodes = 1;
        out->depth = 1;
        k_single<<<1, 1, 0, s>>>(verts, idx, out->nodes, out->tris);
        return cudaGetLastError();
    }
    const int total = 2 * n - 1;
    const int T = 256;
    float4 *plo, *phi, *cent;
    uint32_t *keys, *vals;
    int* gb;
    CK(dalloc(&plo, n, s)); CK(dalloc(&phi, n, s)); CK(dalloc(&cent, n, s));
    CK(dalloc(&keys, n, s)); CK(dalloc(&vals, n, s)); CK(dalloc(&gb, 8, s));
    k_init_bounds<<<1, 32, 0, s>>>(gb);
    k_prim_setup<<<div_up(n, T), T, 0, s>>>(verts, idx, n, plo, phi, cent, gb);
    k_morton<<<div_up(n, T), T, 0, s>>>(cent, n, gb, keys, vals);
    CK(radix_sort_pairs(keys, vals, n, 32, s));

    Tree t;
    CK(dalloc(&t.lo, total, s)); CK(dalloc(&t.hi, total, s));
    CK(dalloc(&t.left, total, s)); CK(dalloc(&t.right, total, s)); CK(dalloc(&t.parent, total, s));
    int *ca, *cb, *nn, *counter;
    uint32_t *keep, *pos;
    CK(dalloc(&ca, n, s)); CK(dalloc(&cb, n, s)); CK(dalloc(&nn, n, s)); CK(dalloc(&counter, 1, s));
    CK(dalloc(&keep, n, s)); CK(dalloc(&pos, n, s));
    k_init_leaves<<<div_up(n, T), T, 0, s>>>(vals, n, plo, phi, t, ca);
    CK(cudaMemcpyAsync(counter, &n, sizeof(int), cudaMemcpyHostToDevice, s));
    const int r = opt.ploc_radius < 1 ? 1 : (opt.ploc_radius > kMaxRadius ? kMaxRadius : opt.ploc_radius);
    // kPlocBatch iterations between host reads of the count; once one cluster is left the
    // remaining iterations of a batch keep it as it is
    int m = n;
    int* dm = nullptr;
    CK(dalloc(&dm, 1, s));
    CK(cudaMemcpyAsync(dm, &n, sizeof(int), cudaMemcpyHostToDevice, s));
    while (m > 1) {
        for (int it = 0; it < kPlocBatch; ++it) {
            k_ploc_nn<<<div_up(m, kNnBlock), kNnBlock, 0, s>>>(ca, dm, t, nn, r);
            k_ploc_merge<<<div_up(m, T), T, 0, s>>>(ca, dm, m, nn, t, counter, keep);
            CK(exclusive_scan(keep, pos, m, s));
            k_compact<<<div_up(m, T), T, 0, s>>>(ca, keep, pos, dm, cb);
            k_ploc_count<<<1, 1, 0, s>>>(keep, pos, dm);
            std::swap(ca, cb);
        }
        int m2 = 0;
        CK(cudaMemcpyAsync(&m2, dm, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (m2 < 1 || (m2 > 1 && m2 >= m)) return cudaErrorUnknown;   // no progress: impossible with the strict pair order
        m = m2;
    }
    dfree(dm, s);
    int root = 0;
    CK(cudaMemcpyAsync(&root, ca, sizeof(int), cudaMemcpyDeviceToHost, s));

    Sah sah;
    CK(dalloc(&sah.cnt, total, s)); CK(dalloc(&sah.icount, total, s)); CK(dalloc(&sah.visit, total, s));
    CK(dalloc(&sah.cost, total, s)); CK(dalloc(&sah.collapsed, total, s));
    CK(cudaMemsetAsync(sah.visit, 0, sizeof(int) * total, s));
    k_bottom_up<<<div_up(n, T), T, 0, s>>>(n, t, sah, opt.max_leaf < 1 ? 1 : opt.max_leaf, opt.cost_traverse,
                                           opt.cost_intersect);
    CK(cudaStreamSynchronize(s));
    k_fix_root<<<1, 1, 0, s>>>(root, t, sah);
    int num_nodes = 0;
    CK(cudaMemcpyAsync(&num_nodes, sah.icount + root, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    out->num_nodes = num_nodes;
    CK(dalloc(&out->nodes, num_nodes, s));
    // scene bounds for the caller and the scene-relative box padding
    float4 rb[2];
    CK(cudaMemcpyAsync(&rb[0], t.lo + root, sizeof(float4), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&rb[1], t.hi + root, sizeof(float4), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    out->lo[0] = rb[0].x; out->lo[1] = rb[0].y; out->lo[2] = rb[0].z;
    out->hi[0] = rb[1].x; out->hi[1] = rb[1].y; out->hi[2] = rb[1].z;
    float scale = 0.f;
    for (int k = 0; k < 3; ++k) scale = fmaxf(scale, fmaxf(fabsf(out->lo[k]), fabsf(out->hi[k])));
    k_layout_tris<<<div_up(n, T), T, 0, s>>>(n, t, sah, vals, verts, idx, out->tris);
    int* dmax;
    CK(dalloc(&dmax, 1, s));
    CK(cudaMemsetAsync(dmax, 0, sizeof(int), s));
    k_layout_nodes<<<div_up(n - 1, T), T, 0, s>>>(n, total, t, sah, scale * 9.5367432e-7f, out->nodes, dmax);
    CK(cudaMemcpyAsync(&out->depth, dmax, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    dfree(dmax, s);

    dfree(plo, s); dfree(phi, s); dfree(cent, s); dfree(keys, s); dfree(vals, s); dfree(gb, s);
    dfree(t.lo, s); dfree(t.hi, s); dfree(t.left, s); dfree(t.right, s); dfree(t.parent, s);
    dfree(ca, s); dfree(cb, s); dfree(nn, s); dfree(counter, s); dfree(keep, s); dfree(pos, s);
    dfree(sah.cnt, s); dfree(sah.icount, s); dfree(sah.visit, s); dfree(sah.cost, s); dfree(sah.collapsed, s);
    return cudaGetLastError();
}

void bvh_free_device(DeviceBvh* bvh, cudaStream_t s) {
    if (bvh->nodes) cudaFreeAsync(bvh->nodes, s);
    if (bvh->tris) cudaFreeAsync(bvh->tris, s);
    if (bvh->nodes4) cudaFreeAsync(bvh->nodes4, s);
    *bvh = DeviceBvh();
}

namespace {

__device__ __forceinline__ void child_of(const BvhNode& nd, int k, float lo[3], float hi[3], int* ref) {
    if (k == 0) {
        lo[0] = nd.a.x; hi[0] = nd.a.y; lo[1] = nd.a.z; hi[1] = nd.a.w; lo[2] = nd.c.x; hi[2] = nd.c.y;
        *ref = __float_as_int(nd.d.x);
    } else {
        lo[0] = nd.b.x; hi[0] = nd.b.y; lo[1] = nd.b.z; hi[1] = nd.b.w; lo[2] = nd.c.z; hi[2] = nd.c.w;
        *ref = __float_as_int(nd.d.y);
    }
}

__device__ __forceinline__ float half_area(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// Writes the 4-wide node at index `at` with children (lo, hi, ref)[0..n): interior children
// get the next 4-wide indices and join the next level's front.
__device__ void write_node4(const float (&lo)[4][3], const float (&hi)[4][3], const int (&ref)[4], int n, int at,
                            BvhNode4* __restrict__ out, int* counters, int2* __restrict__ next, int cap) {
    float v[6][4];
    int r[4];
    for (int k = 0; k < 4; ++k) {
        if (k >= n) {
            for (int d = 0; d < 6; ++d) v[d][k] = __int_as_float(0x7f800000);   // +inf: never entered
            r[k] = ~0;
            continue;
        }
        v[0][k] = lo[k][0]; v[1][k] = hi[k][0]; v[2][k] = lo[k][1];
        v[3][k] = hi[k][1]; v[4][k] = lo[k][2]; v[5][k] = hi[k][2];
        if (ref[k] >= 0) {
            const int j = atomicAdd(&counters[0], 1);
            const int q = atomicAdd(&counters[1], 1);
            if (j < cap && q < cap) next[q] = make_int2(ref[k], j);
            r[k] = j;
        } else {
            r[k] = ref[k];
        }
    }
    if (at >= cap) return;
    BvhNode4 o;
    o.lox = make_float4(v[0][0], v[0][1], v[0][2], v[0][3]);
    o.hix = make_float4(v[1][0], v[1][1], v[1][2], v[1][3]);
    o.loy = make_float4(v[2][0], v[2][1], v[2][2], v[2][3]);
    o.hiy = make_float4(v[3][0], v[3][1], v[3][2], v[3][3]);
    o.loz = make_float4(v[4][0], v[4][1], v[4][2], v[4][3]);
    o.hiz = make_float4(v[5][0], v[5][1], v[5][2], v[5][3]);
    o.ref = make_int4(r[0], r[1], r[2], r[3]);
    o.pad = make_int4(0, 0, 0, 0);
    out[at] = o;
}

// SAH-optimal grouping of the binary tree into 4-wide nodes: a dynamic program over the
// binary tree, bottom up (the 8-wide form is in Ylitie, Karras and Laine, "Efficient
// Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017). The leaves are
// fixed, so groupings differ in SAH cost only by the summed surface area of the 4-wide
// nodes. S(x, j) is the least such sum for the subtree of binary node x when it may fill j
// of its parent's child slots (a leaf costs nothing): S(x, 1) = A(x) + D(x, 4), and for
// j > 1 S(x, j) = min(S(x, 1), D(x, j)), with D(x, j) = min over k in [1, j) of
// S(left, k) + S(right, j - k). dec(x, j) is the k that reaches S(x, j), or 0 where x fills
// one slot; dec(x, 4) is the split of x's slots when x roots a 4-wide node.
struct Dp4 {
    float4* S;          // S(x, 1..4)
    uchar4* dec;        // dec(x, 1..4) (dec(x, 1) = 0)
    int* parent;        // binary parent, -1 at the root
    int* visit;         // arrivals so far, started at the number of leaf children
};

__global__ void k_dp4_init(const BvhNode* __restrict__ n2, int nn, Dp4 d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const BvhNode nd = n2[i];
    const int r0 = __float_as_int(nd.d.x), r1 = __float_as_int(nd.d.y);
    d.visit[i] = (r0 < 0) + (r1 < 0);
    if (i == 0) d.parent[0] = -1;
    if (r0 >= 0) d.parent[r0] = i;
    if (r1 >= 0) d.parent[r1] = i;
}

__device__ void dp4_node(const BvhNode* __restrict__ n2, int x, Dp4 d) {
    const BvhNode nd = n2[x];
    float lo[2][3], hi[2][3];
    int r[2];
    child_of(nd, 0, lo[0], hi[0], &r[0]);
    child_of(nd, 1, lo[1], hi[1], &r[1]);
    float ulo[3], uhi[3];
    for (int a = 0; a < 3; ++a) { ulo[a] = fminf(lo[0][a], lo[1][a]); uhi[a] = fmaxf(hi[0][a], hi[1][a]); }
    float sc[2][5];
    for (int c = 0; c < 2; ++c) {
        sc[c][0] = 0.f;
        if (r[c] >= 0) {
            const float4 v = __ldcg(&d.S[r[c]]);
            sc[c][1] = v.x; sc[c][2] = v.y; sc[c][3] = v.z; sc[c][4] = v.w;
        } else {
            sc[c][1] = sc[c][2] = sc[c][3] = sc[c][4] = 0.f;
        }
    }
    float D[5] = {0.f, 0.f, FLT_MAX, FLT_MAX, FLT_MAX};
    int kd[5] = {0, 0, 0, 0, 0};
    for (int j = 2; j <= 4; ++j)
        for (int k = 1; k < j; ++k) {
            const float c = sc[0][k] + sc[1][j - k];
            if (c < D[j]) { D[j] = c; kd[j] = k; }
        }
    const float s1 = half_area(ulo, uhi) + D[4];
    float S[5];
    int dec[5];
    S[1] = s1; dec[1] = 0;
    for (int j = 2; j <= 3; ++j) {
        if (s1 <= D[j]) { S[j] = s1; dec[j] = 0; }
        else { S[j] = D[j]; dec[j] = kd[j]; }
    }
    S[4] = D[4]; dec[4] = kd[4];   // s1 = A + D(x, 4) > D(x, 4)
    d.S[x] = make_float4(S[1], S[2], S[3], S[4]);
    d.dec[x] = make_uchar4(0, (unsigned char)dec[2], (unsigned char)dec[3], (unsigned char)dec[4]);
}

// Bottom-up sweep: a thread starts at each node whose children are both leaves; the last
// child to finish carries on to the parent.
__global__ void k_dp4(const BvhNode* __restrict__ n2, int nn, Dp4 d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const BvhNode nd = n2[i];
    if (__float_as_int(nd.d.x) >= 0 || __float_as_int(nd.d.y) >= 0) return;
    int x = i;
    while (true) {
        dp4_node(n2, x, d);
        __threadfence();
        const int p = d.parent[x];
        if (p < 0) return;
        if (atomicAdd(&d.visit[p], 1) == 0) return;   // the sibling subtree is still running
        __threadfence();
        x = p;
    }
}

// Between two levels: the next front becomes the current one (c[2]) and a non-empty level
// is counted (c[3]).
constexpr int kCollapseBatch = 8;
__global__ void k_collapse_next(int* c) {
    if (c[2] > 0) ++c[3];
    c[2] = c[1];
    c[1] = 0;
}

__device__ __forceinline__ int dec_for(uchar4 v, int j) { return j == 2 ? v.y : j == 3 ? v.z : j == 4 ? v.w : 0; }

// One level of the collapse by the program's decisions: the node's four slots are split
// between its binary children by dec(x, 4), and a child given j > 1 slots is opened while
// dec(child, j) says so. Slots always add up to four, so a node gets at most four children.
__global__ void k_collapse4_dp(const BvhNode* __restrict__ n2, const uchar4* __restrict__ dec,
                               const int2* __restrict__ front, const int* nfront, BvhNode4* __restrict__ out,
                               int* counters, int2* __restrict__ next, int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *nfront) return;
    const int2 f = front[i];
    float lo[4][3], hi[4][3];
    int ref[4], bud[4];
    int n = 2;
    {
        const BvhNode nd = n2[f.x];
        child_of(nd, 0, lo[0], hi[0], &ref[0]);
        child_of(nd, 1, lo[1], hi[1], &ref[1]);
        const int k = dec[f.x].w;
        bud[0] = k;
        bud[1] = 4 - k;
    }
    while (n < 4) {
        int e = -1, dd = 0;
        for (int q = 0; q < n && e < 0; ++q) {
            if (ref[q] < 0 || bud[q] < 2) continue;
            const int v = dec_for(dec[ref[q]], bud[q]);
            if (v > 0) { e = q; dd = v; }
        }
        if (e < 0) break;
        const BvhNode c = n2[ref[e]];
        child_of(c, 1, lo[n], hi[n], &ref[n]);
        bud[n] = bud[e] - dd;
        child_of(c, 0, lo[e], hi[e], &ref[e]);
        bud[e] = dd;
        ++n;
    }
    write_node4(lo, hi, ref, n, f.y, out, counters, next, cap);
}

}  // namespace

cudaError_t bvh_collapse4(DeviceBvh* b, cudaStream_t s) {
    if (!b->nodes || b->num_nodes < 1) return cudaErrorInvalidValue;
    const int cap = b->num_nodes;             // a 4-wide tree has at most as many nodes as the binary one
    int2 *fa = nullptr, *fb = nullptr;
    int* counters = nullptr;
    CK(dalloc(&b->nodes4, cap, s));
    // every 4-wide node must start on a 128-byte line (the traversals read it in 32-byte and
    // 16-byte vector loads): the allocator's alignment, checked rather than assumed
    if ((uintptr_t)b->nodes4 % sizeof(BvhNode4) != 0) {
        cudaFreeAsync(b->nodes4, s);
        b->nodes4 = nullptr;
        return cudaErrorMisalignedAddress;
    }
    CK(dalloc(&fa, cap, s));
    CK(dalloc(&fb, cap, s));
    CK(dalloc(&counters, 4, s));
    Dp4 dp{};
    CK(dalloc(&dp.S, cap, s));
    CK(dalloc(&dp.dec, cap, s));
    CK(dalloc(&dp.parent, cap, s));
    CK(dalloc(&dp.visit, cap, s));
    k_dp4_init<<<div_up(cap, 256), 256, 0, s>>>(b->nodes, cap, dp);
    k_dp4<<<div_up(cap, 256), 256, 0, s>>>(b->nodes, cap, dp);
    CK(cudaGetLastError());
    const int2 root = make_int2(0, 0);
    // counters: next 4-wide index, next front's size, this front's size, non-empty levels.
    // kCollapseBatch levels run between host reads; the grid covers an upper bound of the
    // front (at most four times the previous one, and at most cap)
    const int init[4] = {1, 0, 1, 0};
    CK(cudaMemcpyAsync(fa, &root, sizeof(int2), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(counters, init, sizeof(init), cudaMemcpyHostToDevice, s));
    int bound = 1, launched = 0, hc[4] = {1, 0, 1, 0};
    while (true) {
        for (int it = 0; it < kCollapseBatch; ++it) {
            k_collapse4_dp<<<div_up(bound, 256), 256, 0, s>>>(b->nodes, dp.dec, fa, counters + 2, b->nodes4, counters,
                                                              fb, cap);
            k_collapse_next<<<1, 1, 0, s>>>(counters);
            std::swap(fa, fb);
            bound = (int)std::min<long long>(cap, 4ll * bound);
        }
        launched += kCollapseBatch;
        CK(cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (hc[0] > cap || hc[2] > cap) return cudaErrorUnknown;
        if (hc[2] == 0) break;
        if (launched > 64) return cudaErrorUnknown;   // the binary tree's depth is at most 63
        bound = hc[2];
    }
    b->num_nodes4 = hc[0];
    b->depth4 = hc[3];
    dfree(fa, s);
    dfree(fb, s);
    dfree(counters, s);
    dfree(dp.S, s);
    dfree(dp.dec, s);
    dfree(dp.parent, s);
    dfree(dp.visit, s);
    return cudaGetLastError();
}

}  // namespace aur
