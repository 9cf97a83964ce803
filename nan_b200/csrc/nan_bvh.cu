// nan_bvh.cu -- GPU scene flattening and BVH construction.
//
// Replaces the reference's driver-built BLAS/TLAS (scene.py:445-533): the
// instances are flattened into one world-space triangle array (each triangle
// keeps its (instance, primitive) identity), and a binary BVH is built over
// it entirely on the GPU:
//   1. per-instance triangle counts + exclusive scan (CUB),
//   2. flatten: transform every triangle to world space, write its box,
//   3. scene bounds of the centroids (block reduction + ordered-int atomics),
//   4. 63-bit Morton codes of the centroids, radix sort (CUB),
//   5. a binary hierarchy over the sorted triangles, by one of three builders
//      (NanTuning.bvh_builder):
//      0. top-down binned SAH (k_sah_*, the default),
//      1. LBVH from the sorted codes (Karras 2012, "Maximizing parallelism in
//         the construction of BVHs, octrees, and k-d trees") with a
//         bottom-up box refit (one atomic arrival counter per node),
//      2. PLOC clustering (k_ploc_*),
//   6. for 0 and 2: SAH leaf collapse (up to 3 triangles per leaf), depth-first
//      placement and the compressed 8-wide conversion,
//   7. emission of 64-byte two-box nodes and leaf-ordered triangles.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <vector>

#include "nan_internal.h"

namespace {

using nan_host::cuda_fail;
using nan_host::set_error;

constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t float_to_ordered(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_instance_counts(const uint4* __restrict__ instance_descs, const uint4* __restrict__ mesh_descs,
                                  uint32_t instance_count, uint32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > instance_count) return;
    if (i == instance_count) {
        counts[i] = 0u;
        return;
    }
    const uint4 id = instance_descs[i];
    counts[i] = mesh_descs[id.x].y / 3u;
}

// mul(M, float4(p, 1)).xyz, unfused, left to right (the CPU oracle's order).
__device__ __forceinline__ float3 xform(const float* __restrict__ m, float x, float y, float z) {
    return make_float3(((m[0] * x + m[1] * y) + m[2] * z) + m[3], ((m[4] * x + m[5] * y) + m[6] * z) + m[7],
                       ((m[8] * x + m[9] * y) + m[10] * z) + m[11]);
}

struct Bounds {
    uint32_t lo[3];  // ordered ints
    uint32_t hi[3];
    uint32_t max_abs;
};

__global__ void k_flatten(NanSceneDesc sd, const uint32_t* __restrict__ offsets, uint32_t tri_count,
                          float4* __restrict__ tris, uint2* __restrict__ refs, float4* __restrict__ box_lo,
                          float4* __restrict__ box_hi, Bounds* __restrict__ bounds) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    float c[3] = {INFINITY, INFINITY, INFINITY};
    float ch[3] = {-INFINITY, -INFINITY, -INFINITY};
    float mabs = 0.0f;
    if (f < tri_count) {
        // instance = last i with offsets[i] <= f
        uint32_t lo = 0, hi = sd.instance_count;  // search in [0, I]
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (offsets[mid] <= f) lo = mid; else hi = mid - 1u;
        }
        const uint32_t inst = lo;
        const uint32_t prim = f - offsets[inst];
        const uint4 id = reinterpret_cast<const uint4*>(sd.instance_descs)[inst];
        const uint4 md = reinterpret_cast<const uint4*>(sd.mesh_descs)[id.x];
        const float* m = sd.transforms + 16u * id.z;
        float3 w[3];
        for (int k = 0; k < 3; ++k) {
            const uint32_t vi = md.z + sd.indices[md.w + 3u * prim + (uint32_t)k];
            const float* v = sd.vertices + 8u * vi;
            w[k] = xform(m, v[0], v[1], v[2]);
        }
        tris[3u * f + 0] = make_float4(w[0].x, w[0].y, w[0].z, __uint_as_float(f));
        tris[3u * f + 1] = make_float4(w[1].x, w[1].y, w[1].z, 0.0f);
        tris[3u * f + 2] = make_float4(w[2].x, w[2].y, w[2].z, 0.0f);
        refs[f] = make_uint2(inst, prim);
        float3 l = make_float3(fminf(fminf(w[0].x, w[1].x), w[2].x), fminf(fminf(w[0].y, w[1].y), w[2].y),
                               fminf(fminf(w[0].z, w[1].z), w[2].z));
        float3 h = make_float3(fmaxf(fmaxf(w[0].x, w[1].x), w[2].x), fmaxf(fmaxf(w[0].y, w[1].y), w[2].y),
                               fmaxf(fmaxf(w[0].z, w[1].z), w[2].z));
        box_lo[f] = make_float4(l.x, l.y, l.z, 0.0f);
        box_hi[f] = make_float4(h.x, h.y, h.z, 0.0f);
        c[0] = ch[0] = 0.5f * (l.x + h.x);
        c[1] = ch[1] = 0.5f * (l.y + h.y);
        c[2] = ch[2] = 0.5f * (l.z + h.z);
        mabs = fmaxf(fmaxf(fmaxf(fabsf(l.x), fabsf(h.x)), fmaxf(fabsf(l.y), fabsf(h.y))),
                     fmaxf(fabsf(l.z), fabsf(h.z)));
    }
    typedef cub::BlockReduce<float, kThreads> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    for (int a = 0; a < 3; ++a) {
        const float mn = Reduce(tmp).Reduce(c[a], cub::Min());
        __syncthreads();
        const float mx = Reduce(tmp).Reduce(ch[a], cub::Max());
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicMin(&bounds->lo[a], float_to_ordered(mn));
            atomicMax(&bounds->hi[a], float_to_ordered(mx));
        }
    }
    const float ma = Reduce(tmp).Reduce(mabs, cub::Max());
    if (threadIdx.x == 0) atomicMax(&bounds->max_abs, float_to_ordered(ma));
}

__device__ __forceinline__ uint64_t expand21(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void k_morton(const float4* __restrict__ box_lo, const float4* __restrict__ box_hi, uint32_t n,
                         const Bounds* __restrict__ bounds, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 l = box_lo[i], h = box_hi[i];
    const float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        const float lo = ordered_to_float(bounds->lo[a]);
        const float hi = ordered_to_float(bounds->hi[a]);
        const float ext = hi - lo;
        float u = ext > 0.0f ? (c[a] - lo) / ext : 0.0f;
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        q[a] = min((uint32_t)(u * 2097152.0f), 2097151u);
    }
    keys[i] = (expand21(q[0]) << 2) | (expand21(q[1]) << 1) | expand21(q[2]);
    vals[i] = i;
}

__device__ __forceinline__ int delta(const uint64_t* __restrict__ k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = k[i], b = k[j];
    if (a == b) return 64 + __clz((uint32_t)(i ^ j));
    return __clzll((long long)(a ^ b));
}

// Interior node i of n-1; children < n-1 are interior, leaves are encoded as
// ~leaf. parent arrays: interior parents (n-1) and leaf parents (n).
__global__ void k_hierarchy(const uint64_t* __restrict__ keys, int n, int2* __restrict__ children,
                            int* __restrict__ node_parent, int* __restrict__ leaf_parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int left = (min(i, j) == gamma) ? ~gamma : gamma;
    const int right = (max(i, j) == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    children[i] = make_int2(left, right);
    if (left < 0) leaf_parent[~left] = i; else node_parent[left] = i;
    if (right < 0) leaf_parent[~right] = i; else node_parent[right] = i;
    if (i == 0) node_parent[0] = -1;
}

// Leaf-ordered triangles and boxes.
__global__ void k_gather_leaves(const uint32_t* __restrict__ order, uint32_t n, const float4* __restrict__ tris_flat,
                                const float4* __restrict__ lo_flat, const float4* __restrict__ hi_flat,
                                float4* __restrict__ tris, float4* __restrict__ leaf_lo, float4* __restrict__ leaf_hi) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t f = order[i];
    tris[3u * i + 0] = tris_flat[3u * f + 0];
    tris[3u * i + 1] = tris_flat[3u * f + 1];
    tris[3u * i + 2] = tris_flat[3u * f + 2];
    leaf_lo[i] = lo_flat[f];
    leaf_hi[i] = hi_flat[f];
}

__device__ __forceinline__ void child_box(int c, const float4* node_lo, const float4* node_hi, const float4* leaf_lo,
                                          const float4* leaf_hi, float4* lo, float4* hi) {
    if (c < 0) {
        *lo = leaf_lo[~c];
        *hi = leaf_hi[~c];
    } else {
        *lo = __ldcg(node_lo + c);
        *hi = __ldcg(node_hi + c);
    }
}

// Every walk from a leaf or node up to the root stops after kMaxWalk steps
// or at a parent index outside [0, interior): a malformed hierarchy then
// yields a depth above the traversal stack's (rejected by the host) instead of
// a walk that never ends. Valid trees have depth <= 96 here.
constexpr uint32_t kMaxWalk = 4096u;
__device__ __forceinline__ bool walk_on(int p, uint32_t interior, uint32_t steps) {
    return p >= 0 && (uint32_t)p < interior && steps < kMaxWalk;
}

// Bottom-up refit: the second thread to reach a node computes its box.
__global__ void k_refit(uint32_t n, const int2* __restrict__ children, const int* __restrict__ node_parent,
                        const int* __restrict__ leaf_parent, const float4* __restrict__ leaf_lo,
                        const float4* __restrict__ leaf_hi, float4* node_lo, float4* node_hi,
                        uint32_t* __restrict__ arrivals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = leaf_parent[i];
    for (uint32_t steps = 0; walk_on(p, n - 1u, steps); ++steps) {
        __threadfence();
        if (atomicAdd(&arrivals[p], 1u) == 0u) return;
        const int2 ch = children[p];
        float4 al, ah, bl, bh;
        child_box(ch.x, node_lo, node_hi, leaf_lo, leaf_hi, &al, &ah);
        child_box(ch.y, node_lo, node_hi, leaf_lo, leaf_hi, &bl, &bh);
        __stcg(node_lo + p, make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f));
        __stcg(node_hi + p, make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f));
        p = node_parent[p];
    }
}

// Depth of every leaf (steps to the root); max over leaves is the tree depth.
__global__ void k_depth(uint32_t n, const int* __restrict__ node_parent, const int* __restrict__ leaf_parent,
                        uint32_t* __restrict__ max_depth) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t depth = 1;
    int p = leaf_parent[i];
    while (walk_on(p, n - 1u, depth)) {
        ++depth;
        p = node_parent[p];
    }
    if (p >= 0) depth = kMaxWalk;  // a parent out of range or a walk too long: reject
    atomicMax(max_depth, depth);
}

__device__ __forceinline__ float half_area(float4 l, float4 h) {
    const float x = h.x - l.x, y = h.y - l.y, z = h.z - l.z;
    return x * y + y * z + z * x;
}

// 64-byte nodes with padded child boxes; also accumulates the SAH cost.
// Adds each lane's SAH term into *sah with one atomic per warp (a single
// address takes one atomic per node otherwise, which serialises millions of
// them). Every lane of the warp must call it.
__device__ __forceinline__ void add_sah(double* sah, double cost) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cost += __shfl_down_sync(0xffffffffu, cost, o);
    if ((threadIdx.x & 31u) == 0u && cost != 0.0) atomicAdd(sah, cost);
}

__global__ void k_emit(uint32_t interior, const int2* __restrict__ children, const float4* __restrict__ node_lo,
                       const float4* __restrict__ node_hi, const float4* __restrict__ leaf_lo,
                       const float4* __restrict__ leaf_hi, const Bounds* __restrict__ bounds,
                       float4* __restrict__ nodes, double* __restrict__ sah) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double cost = 0.0;
    if (i < interior) {
        const float pad = ordered_to_float(bounds->max_abs) * 3.814697265625e-6f + 1e-30f;  // 2^-18 relative
        const int2 ch = children[i];
        float4 al, ah, bl, bh;
        child_box(ch.x, node_lo, node_hi, leaf_lo, leaf_hi, &al, &ah);
        child_box(ch.y, node_lo, node_hi, leaf_lo, leaf_hi, &bl, &bh);
        nodes[4u * i + 0] = make_float4(al.x - pad, ah.x + pad, al.y - pad, ah.y + pad);
        nodes[4u * i + 1] = make_float4(bl.x - pad, bh.x + pad, bl.y - pad, bh.y + pad);
        nodes[4u * i + 2] = make_float4(al.z - pad, ah.z + pad, bl.z - pad, bh.z + pad);
        // leaves (single triangles in LBVH) as ~(first << 3 | count - 1)
        const int rx = ch.x < 0 ? ~((~ch.x) << 3) : ch.x;
        const int ry = ch.y < 0 ? ~((~ch.y) << 3) : ch.y;
        nodes[4u * i + 3] = make_float4(__int_as_float(rx), __int_as_float(ry), 0.0f, 0.0f);
        const float root_area = fmaxf(half_area(node_lo[0], node_hi[0]), 1e-30f);
        cost = (double)(half_area(node_lo[i], node_hi[i]) / root_area);  // one traversal step
        if (ch.x < 0) cost += (double)(half_area(al, ah) / root_area);   // one triangle per leaf
        if (ch.y < 0) cost += (double)(half_area(bl, bh) / root_area);
    }
    add_sah(sah, cost);
}


// ---------------------------------------------------------------------------
// PLOC: parallel locally-ordered clustering (Meister and Bittner 2018).
// Clusters start as the Morton-sorted triangles; every iteration each cluster
// finds the neighbour within +-kPlocRadius positions whose union box has the
// smallest surface area, mutual nearest neighbours merge into a new interior
// node, and the cluster list is compacted (order preserved).
// ---------------------------------------------------------------------------
constexpr int kPlocRadius = 64;
constexpr int kPlocBlock = 256;
constexpr int kPlocBatch = 8;       // PLOC iterations between two host checks of the count
constexpr int kWideBatch = 4;       // wide-conversion levels between two host checks
constexpr int kWideMaxLevels = 256;
constexpr int kMaxLeafTris = 3;  // the wide nodes' leaf encoding holds up to 3 triangles

__device__ __forceinline__ float area_union(float4 al, float4 ah, float4 bl, float4 bh) {
    const float x = fmaxf(ah.x, bh.x) - fminf(al.x, bl.x);
    const float y = fmaxf(ah.y, bh.y) - fminf(al.y, bl.y);
    const float z = fmaxf(ah.z, bh.z) - fminf(al.z, bl.z);
    return x * y + y * z + z * x;
}

__global__ void k_ploc_init(uint32_t n, int* __restrict__ idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) idx[i] = ~(int)i;
}

// The PLOC kernels read the current cluster count from device memory
// (*count), so that several iterations run back to back without the host;
// grids are sized for an upper bound of the count, and with one cluster left
// every kernel does nothing.
__global__ void __launch_bounds__(kPlocBlock) k_ploc_nn(const uint32_t* __restrict__ count,
                                                         const float4* __restrict__ lo,
                                                         const float4* __restrict__ hi, int* __restrict__ nn) {
    const int c = (int)*count;
    if (c <= 1) return;
    __shared__ float4 slo[kPlocBlock + 2 * kPlocRadius];
    __shared__ float4 shi[kPlocBlock + 2 * kPlocRadius];
    const int b0 = blockIdx.x * kPlocBlock;
    for (int k = threadIdx.x; k < kPlocBlock + 2 * kPlocRadius; k += blockDim.x) {
        const int g = b0 - kPlocRadius + k;
        if (g >= 0 && g < c) {
            slo[k] = lo[g];
            shi[k] = hi[g];
        }
    }
    __syncthreads();
    const int i = b0 + (int)threadIdx.x;
    if (i >= c) return;
    const float4 ml = slo[threadIdx.x + kPlocRadius], mh = shi[threadIdx.x + kPlocRadius];
    float best = INFINITY;
    int bj = -1;
    for (int dj = -kPlocRadius; dj <= kPlocRadius; ++dj) {
        const int j = i + dj;
        if (dj == 0 || j < 0 || j >= c) continue;
        const float a = area_union(ml, mh, slo[threadIdx.x + kPlocRadius + dj], shi[threadIdx.x + kPlocRadius + dj]);
        if (a < best) {  // ties keep the lower index (dj ascending)
            best = a;
            bj = j;
        }
    }
    nn[i] = bj;
}

// Also clears valid[c .. bound] (bound + 1 flags are scanned).
__global__ void k_ploc_merge(const uint32_t* __restrict__ count, int bound, const int* __restrict__ nn,
                             const int* __restrict__ idx,
                             const float4* __restrict__ lo, const float4* __restrict__ hi, int* __restrict__ idx2,
                             float4* __restrict__ lo2, float4* __restrict__ hi2, uint32_t* __restrict__ valid,
                             int2* __restrict__ children, int* __restrict__ node_parent, int* __restrict__ leaf_parent,
                             float4* __restrict__ node_lo, float4* __restrict__ node_hi, uint32_t* node_counter) {
    const int c = (int)*count;
    if (c <= 1) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > bound) return;
    if (i >= c) {
        valid[i] = 0u;
        return;
    }
    const int j = nn[i];
    if (j >= 0 && nn[j] == i) {
        if (i > j) {
            valid[i] = 0u;
            return;
        }
        const int id = (int)atomicAdd(node_counter, 1u);
        const int a = idx[i], b = idx[j];
        const float4 al = lo[i], ah = hi[i], bl = lo[j], bh = hi[j];
        const float4 l = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f);
        const float4 h = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
        children[id] = make_int2(a, b);
        if (a < 0) leaf_parent[~a] = id; else node_parent[a] = id;
        if (b < 0) leaf_parent[~b] = id; else node_parent[b] = id;
        node_lo[id] = l;
        node_hi[id] = h;
        idx2[i] = id;
        lo2[i] = l;
        hi2[i] = h;
    } else {
        idx2[i] = idx[i];
        lo2[i] = lo[i];
        hi2[i] = hi[i];
    }
    valid[i] = 1u;
}

// Also writes the next iteration's count (the kept clusters) to *next_count:
// the count is double-buffered, iteration k reading slot k & 1.
__global__ void k_ploc_compact(const uint32_t* __restrict__ count, uint32_t* __restrict__ next_count,
                               const uint32_t* __restrict__ valid, const uint32_t* __restrict__ pos,
                               const int* __restrict__ idx2, const float4* __restrict__ lo2,
                               const float4* __restrict__ hi2, int* __restrict__ idx, float4* __restrict__ lo,
                               float4* __restrict__ hi) {
    const int c = (int)*count;
    if (blockIdx.x == 0 && threadIdx.x == 0) *next_count = c <= 1 ? (uint32_t)c : pos[c];
    if (c <= 1) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c || !valid[i]) return;
    const uint32_t p = pos[i];
    idx[p] = idx2[i];
    lo[p] = lo2[i];
    hi[p] = hi2[i];
}

__device__ __forceinline__ float half_area4(float4 l, float4 h) {
    const float x = h.x - l.x, y = h.y - l.y, z = h.z - l.z;
    return x * y + y * z + z * x;
}

// Bottom-up: triangle count, kept-interior count and SAH cost (relative to
// the node's own area, C_trav = C_int = 1) of every subtree; a subtree of at
// most kMaxLeafTris triangles collapses into one leaf when that is cheaper.
struct SubtreeInfo {
    uint32_t tris;
    uint32_t interior;  // kept interior nodes (0 when collapsed)
    float cost;
    uint32_t collapsed;
};

__device__ __forceinline__ void child_info(int c, const SubtreeInfo* info, uint32_t* tris, uint32_t* interior,
                                           float* cost) {
    if (c < 0) {
        *tris = 1u;
        *interior = 0u;
        *cost = 1.0f;
    } else {
        const volatile SubtreeInfo* v = info + c;  // written by the sibling's thread
        *tris = v->tris;
        *interior = v->interior;
        *cost = v->cost;
    }
}

__global__ void k_subtree(uint32_t n, const int2* __restrict__ children, const int* __restrict__ node_parent,
                          const int* __restrict__ leaf_parent, const float4* __restrict__ leaf_lo,
                          const float4* __restrict__ leaf_hi, const float4* __restrict__ node_lo,
                          const float4* __restrict__ node_hi, SubtreeInfo* info, uint32_t* __restrict__ arrivals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = leaf_parent[i];
    for (uint32_t steps = 0; walk_on(p, n - 1u, steps); ++steps) {
        __threadfence();
        if (atomicAdd(&arrivals[p], 1u) == 0u) return;
        const int2 ch = children[p];
        uint32_t ta, ia, tb, ib;
        float ca, cb;
        child_info(ch.x, info, &ta, &ia, &ca);
        child_info(ch.y, info, &tb, &ib, &cb);
        const float ap = fmaxf(half_area4(node_lo[p], node_hi[p]), 1e-30f);
        const float aa = ch.x < 0 ? half_area4(leaf_lo[~ch.x], leaf_hi[~ch.x]) : half_area4(node_lo[ch.x], node_hi[ch.x]);
        const float ab = ch.y < 0 ? half_area4(leaf_lo[~ch.y], leaf_hi[~ch.y]) : half_area4(node_lo[ch.y], node_hi[ch.y]);
        const float split = 1.0f + (aa * ca + ab * cb) / ap;
        const uint32_t tris = ta + tb;
        SubtreeInfo v;
        v.tris = tris;
        if (tris <= (uint32_t)kMaxLeafTris && (float)tris <= split) {
            v.cost = (float)tris;
            v.interior = 0u;
            v.collapsed = 1u;
        } else {
            v.cost = split;
            v.interior = 1u + ia + ib;
            v.collapsed = 0u;
        }
        volatile SubtreeInfo* dst = info + p;
        dst->tris = v.tris;
        dst->interior = v.interior;
        dst->cost = v.cost;
        dst->collapsed = v.collapsed;
        p = node_parent[p];
    }
}

// Depth-first placement: walking up from a node or triangle to the root,
// every step from a right child skips the left sibling's interior nodes (for
// the node index) or triangles (for the triangle position). Nodes below a
// collapsed ancestor are not emitted (dfs = -1).
__global__ void k_dfs_nodes(uint32_t interior, const int2* __restrict__ children, const int* __restrict__ node_parent,
                            const SubtreeInfo* __restrict__ info, int* __restrict__ dfs, uint32_t* __restrict__ tri_off) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= interior) return;
    int node = (int)x;
    int index = 0;
    uint32_t toff = 0u;
    bool hidden = false;
    int p = node_parent[node];
    for (uint32_t steps = 0; walk_on(p, interior, steps); ++steps) {
        const SubtreeInfo pi = info[p];
        if (pi.collapsed) hidden = true;
        const int2 ch = children[p];
        index += 1;
        if (ch.y == node) {
            if (ch.x >= 0) {
                const SubtreeInfo li = info[ch.x];
                index += (int)li.interior;
                toff += li.tris;
            } else {
                toff += 1u;
            }
        }
        node = p;
        p = node_parent[p];
    }
    dfs[x] = hidden ? -1 : index;
    tri_off[x] = toff;
}

__global__ void k_dfs_leaves(uint32_t n, const int2* __restrict__ children, const int* __restrict__ node_parent,
                             const int* __restrict__ leaf_parent, const SubtreeInfo* __restrict__ info,
                             uint32_t* __restrict__ tri_pos) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int node = ~(int)i;
    uint32_t toff = 0u;
    int p = leaf_parent[i];
    for (uint32_t steps = 0; walk_on(p, n - 1u, steps); ++steps) {
        const int2 ch = children[p];
        if (ch.y == node) toff += ch.x >= 0 ? info[ch.x].tris : 1u;
        node = p;
        p = node_parent[p];
    }
    tri_pos[i] = toff;
}

__global__ void k_scatter_tris(uint32_t n, const uint32_t* __restrict__ tri_pos, const float4* __restrict__ src,
                               float4* __restrict__ dst) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t p = tri_pos[i];
    dst[3u * p] = src[3u * i];
    dst[3u * p + 1] = src[3u * i + 1];
    dst[3u * p + 2] = src[3u * i + 2];
}

__device__ __forceinline__ int child_ref(int c, const int* dfs, const uint32_t* tri_off, const uint32_t* tri_pos,
                                         const SubtreeInfo* info) {
    if (c < 0) return ~(int)(tri_pos[~c] << 3);
    const SubtreeInfo v = info[c];
    if (v.collapsed) return ~(int)((tri_off[c] << 3) | (v.tris - 1u));
    return dfs[c];
}

__global__ void k_emit_dfs(uint32_t interior, const int2* __restrict__ children, const float4* __restrict__ node_lo,
                           const float4* __restrict__ node_hi, const float4* __restrict__ leaf_lo,
                           const float4* __restrict__ leaf_hi, const Bounds* __restrict__ bounds,
                           const SubtreeInfo* __restrict__ info, const int* __restrict__ dfs,
                           const uint32_t* __restrict__ tri_off, const uint32_t* __restrict__ tri_pos, int root,
                           float4* __restrict__ nodes, double* __restrict__ sah) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const int slot = x < interior ? dfs[x] : -1;
    double cost = 0.0;
    if (slot >= 0 && !info[x].collapsed) {
        const float pad = ordered_to_float(bounds->max_abs) * 3.814697265625e-6f + 1e-30f;
        const int2 ch = children[x];
        float4 al, ah, bl, bh;
        child_box(ch.x, node_lo, node_hi, leaf_lo, leaf_hi, &al, &ah);
        child_box(ch.y, node_lo, node_hi, leaf_lo, leaf_hi, &bl, &bh);
        nodes[4u * slot + 0] = make_float4(al.x - pad, ah.x + pad, al.y - pad, ah.y + pad);
        nodes[4u * slot + 1] = make_float4(bl.x - pad, bh.x + pad, bl.y - pad, bh.y + pad);
        nodes[4u * slot + 2] = make_float4(al.z - pad, ah.z + pad, bl.z - pad, bh.z + pad);
        const int ra = child_ref(ch.x, dfs, tri_off, tri_pos, info);
        const int rb = child_ref(ch.y, dfs, tri_off, tri_pos, info);
        nodes[4u * slot + 3] = make_float4(__int_as_float(ra), __int_as_float(rb), 0.0f, 0.0f);
        const float root_area = fmaxf(half_area4(node_lo[root], node_hi[root]), 1e-30f);
        cost = (double)(half_area4(node_lo[x], node_hi[x]) / root_area);
        if (ra < 0) cost += (double)(half_area4(al, ah) / root_area) * (double)(((~ra) & 7) + 1);
        if (rb < 0) cost += (double)(half_area4(bl, bh) / root_area) * (double)(((~rb) & 7) + 1);
    }
    add_sah(sah, cost);
}


// ---------------------------------------------------------------------------
// Compressed 8-wide BVH (after Ylitie, Karras and Laine, "Efficient Incoherent
// Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017), converted
// top-down from the collapsed binary tree (binned SAH or PLOC): each wide
// node takes up to 8 subtrees by repeatedly opening the largest-area interior
// binary node, places them in slots ordered by octant direction, stores its
// interior children
// contiguously (child_base) and its leaf triangles contiguously (tri_base),
// and quantizes the children's boxes to 8 bits against the node's box.
// Node (80 B): w0 = (p.xyz, e.x | e.y << 8 | e.z << 16 | imask << 24)
//              w1 = (child_base, tri_base, meta[0..3], meta[4..7])
//              w2..w4 = qlo.x, qlo.y, qlo.z, qhi.x, qhi.y, qhi.z (8 bytes each)
// meta[slot]: 0 empty; interior slots are marked in imask; a leaf slot holds
// (unary triangle count) << 5 | (triangle offset from tri_base).
// ---------------------------------------------------------------------------
struct WideItem {
    int bnode;      // binary node (>= 0) or leaf code (~sorted leaf)
    uint32_t wnode;
};

__device__ __forceinline__ bool expandable(int c, const SubtreeInfo* info) { return c >= 0 && !info[c].collapsed; }

__device__ __forceinline__ void entry_box(int c, const float4* node_lo, const float4* node_hi, const float4* leaf_lo,
                                          const float4* leaf_hi, float4* lo, float4* hi) {
    if (c < 0) {
        *lo = leaf_lo[~c];
        *hi = leaf_hi[~c];
    } else {
        *lo = node_lo[c];
        *hi = node_hi[c];
    }
}

// The first level of the wide conversion: the binary root (the last cluster).
__global__ void k_wide_root(const int* __restrict__ root, WideItem* __restrict__ items) {
    items[0] = WideItem{root[0], 0u};
}

// One level of the wide conversion: *count_in items of this level in, the
// next level's items appended at *count_out (counters[0] and [1] count the
// wide nodes and triangles written so far).
__global__ void k_wide_level(const WideItem* __restrict__ items, const uint32_t* __restrict__ count_in,
                             WideItem* __restrict__ items_out, uint32_t* __restrict__ count_out,
                             uint32_t* __restrict__ counters, const int2* __restrict__ children,
                             const float4* __restrict__ node_lo, const float4* __restrict__ node_hi,
                             const float4* __restrict__ leaf_lo, const float4* __restrict__ leaf_hi,
                             const SubtreeInfo* __restrict__ info, const uint32_t* __restrict__ tri_off,
                             const uint32_t* __restrict__ tri_pos, const float4* __restrict__ tris_dfs,
                             const Bounds* __restrict__ bounds, uint4* __restrict__ wnodes,
                             float4* __restrict__ wtris) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *count_in) return;
    const WideItem it = items[k];
    int ent[8];
    float4 elo[8], ehi[8];
    int m = 0;
    if (expandable(it.bnode, info)) {
        const int2 ch = children[it.bnode];
        ent[0] = ch.x;
        ent[1] = ch.y;
        m = 2;
    } else {
        ent[0] = it.bnode;  // a root that is a single leaf
        m = 1;
    }
    for (int i = 0; i < m; ++i) entry_box(ent[i], node_lo, node_hi, leaf_lo, leaf_hi, &elo[i], &ehi[i]);
    while (m < 8) {
        int best = -1;
        float best_area = -1.0f;
        for (int i = 0; i < m; ++i) {
            if (!expandable(ent[i], info)) continue;
            const float a = half_area4(elo[i], ehi[i]);
            if (a > best_area) {
                best_area = a;
                best = i;
            }
        }
        if (best < 0) break;
        const int2 ch = children[ent[best]];
        ent[best] = ch.x;
        ent[m] = ch.y;
        entry_box(ent[best], node_lo, node_hi, leaf_lo, leaf_hi, &elo[best], &ehi[best]);
        entry_box(ent[m], node_lo, node_hi, leaf_lo, leaf_hi, &elo[m], &ehi[m]);
        ++m;
    }
    // node box and slot assignment by octant direction of each child's centre
    float4 plo = elo[0], phi = ehi[0];
    for (int i = 1; i < m; ++i) {
        plo = make_float4(fminf(plo.x, elo[i].x), fminf(plo.y, elo[i].y), fminf(plo.z, elo[i].z), 0.0f);
        phi = make_float4(fmaxf(phi.x, ehi[i].x), fmaxf(phi.y, ehi[i].y), fmaxf(phi.z, ehi[i].z), 0.0f);
    }
    const float pcx = 0.5f * (plo.x + phi.x), pcy = 0.5f * (plo.y + phi.y), pcz = 0.5f * (plo.z + phi.z);
    float score[8][8];
    for (int i = 0; i < m; ++i) {
        const float vx = 0.5f * (elo[i].x + ehi[i].x) - pcx;
        const float vy = 0.5f * (elo[i].y + ehi[i].y) - pcy;
        const float vz = 0.5f * (elo[i].z + ehi[i].z) - pcz;
        for (int sl = 0; sl < 8; ++sl)
            score[i][sl] = ((sl & 1) ? vx : -vx) + ((sl & 2) ? vy : -vy) + ((sl & 4) ? vz : -vz);
    }
    int slot_of[8];
    uint32_t used_slots = 0u, done = 0u;
    for (int r = 0; r < m; ++r) {
        float best = -INFINITY;
        int bi = -1, bs = -1;
        for (int i = 0; i < m; ++i) {
            if (done & (1u << i)) continue;
            for (int sl = 0; sl < 8; ++sl) {
                if (used_slots & (1u << sl)) continue;
                if (score[i][sl] > best || bi < 0) {
                    best = score[i][sl];
                    bi = i;
                    bs = sl;
                }
            }
        }
        slot_of[bi] = bs;
        done |= 1u << bi;
        used_slots |= 1u << bs;
    }
    int slot_ent[8];
    for (int sl = 0; sl < 8; ++sl) slot_ent[sl] = -1;
    for (int i = 0; i < m; ++i) slot_ent[slot_of[i]] = i;
    // allocation: interior children and leaf triangles, both in slot order
    uint32_t n_int = 0u, n_tri = 0u;
    for (int sl = 0; sl < 8; ++sl) {
        const int i = slot_ent[sl];
        if (i < 0) continue;
        if (expandable(ent[i], info)) ++n_int;
        else n_tri += ent[i] < 0 ? 1u : info[ent[i]].tris;
    }
    const uint32_t child_base = n_int ? atomicAdd(&counters[0], n_int) : 0u;
    const uint32_t tri_base = n_tri ? atomicAdd(&counters[1], n_tri) : 0u;
    const uint32_t out_base = n_int ? atomicAdd(count_out, n_int) : 0u;
    // quantization grid: p = node lo, scale 2^e with 255 * 2^e >= extent
    const float pad = ordered_to_float(bounds->max_abs) * 3.814697265625e-6f + 1e-30f;
    const double lo3[3] = {(double)plo.x - pad, (double)plo.y - pad, (double)plo.z - pad};
    const double hi3[3] = {(double)phi.x + pad, (double)phi.y + pad, (double)phi.z + pad};
    float p3[3];
    int e3[3];
    for (int a = 0; a < 3; ++a) {
        p3[a] = (float)lo3[a];
        if ((double)p3[a] > lo3[a]) p3[a] = nextafterf(p3[a], -INFINITY);  // p <= lo
        const double ext = hi3[a] - (double)p3[a];
        int e = -126;
        if (ext > 0.0) {
            e = (int)ceil(log2(ext / 255.0));
            while (ldexp(255.0, e) < ext) ++e;
            e = max(min(e, 127), -126);
        }
        e3[a] = e;
    }
    uint32_t imask = 0u, rank = 0u, toff = 0u;
    uint8_t meta[8], qlo[3][8], qhi[3][8];
    for (int sl = 0; sl < 8; ++sl) {
        meta[sl] = 0u;
        for (int a = 0; a < 3; ++a) {
            qlo[a][sl] = 1u;  // empty slot: an inverted box
            qhi[a][sl] = 0u;
        }
        const int i = slot_ent[sl];
        if (i < 0) continue;
        const double clo[3] = {(double)elo[i].x - pad, (double)elo[i].y - pad, (double)elo[i].z - pad};
        const double chi[3] = {(double)ehi[i].x + pad, (double)ehi[i].y + pad, (double)ehi[i].z + pad};
        for (int a = 0; a < 3; ++a) {
            const double sc = ldexp(1.0, e3[a]);
            const double ql = floor((clo[a] - (double)p3[a]) / sc);
            const double qh = ceil((chi[a] - (double)p3[a]) / sc);
            qlo[a][sl] = (uint8_t)fmax(0.0, fmin(255.0, ql));
            qhi[a][sl] = (uint8_t)fmax(0.0, fmin(255.0, qh));
        }
        const int c = ent[i];
        if (expandable(c, info)) {
            imask |= 1u << sl;
            items_out[out_base + rank] = WideItem{c, child_base + rank};
            ++rank;
        } else {
            const uint32_t cnt = c < 0 ? 1u : info[c].tris;
            const uint32_t src = c < 0 ? tri_pos[~c] : tri_off[c];
            for (uint32_t t = 0; t < cnt; ++t) {
                const uint32_t d = tri_base + toff + t;
                wtris[3u * d + 0] = tris_dfs[3u * (src + t) + 0];
                wtris[3u * d + 1] = tris_dfs[3u * (src + t) + 1];
                wtris[3u * d + 2] = tris_dfs[3u * (src + t) + 2];
            }
            const uint32_t unary = cnt == 1u ? 1u : (cnt == 2u ? 3u : 7u);
            meta[sl] = (uint8_t)((unary << 5) | toff);
            toff += cnt;
        }
    }
    auto pack4 = [](const uint8_t* b) {
        return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
    };
    const uint32_t ebits = (uint32_t)(e3[0] + 127) | ((uint32_t)(e3[1] + 127) << 8) |
                           ((uint32_t)(e3[2] + 127) << 16) | (imask << 24);
    uint4* w = wnodes + 5u * it.wnode;
    w[0] = make_uint4(__float_as_uint(p3[0]), __float_as_uint(p3[1]), __float_as_uint(p3[2]), ebits);
    w[1] = make_uint4(child_base, tri_base, pack4(meta), pack4(meta + 4));
    w[2] = make_uint4(pack4(qlo[0]), pack4(qlo[0] + 4), pack4(qlo[1]), pack4(qlo[1] + 4));
    w[3] = make_uint4(pack4(qlo[2]), pack4(qlo[2] + 4), pack4(qhi[0]), pack4(qhi[0] + 4));
    w[4] = make_uint4(pack4(qhi[1]), pack4(qhi[1] + 4), pack4(qhi[2]), pack4(qhi[2] + 4));
}

// ---------------------------------------------------------------------------
// Top-down binned SAH (Wald, "On fast construction of SAH-based bounding
// volume hierarchies", 2007): every node bins its triangles' centroids into
// kSahBins equal intervals of the node's centroid bounds on each axis and
// splits at the bin boundary of least (left area x left count + right area x
// right count), down to single triangles; the SAH leaf collapse and the
// depth-first emission above then run on this tree as on PLOC's.
// Nodes of more than kSahSeqMax triangles are split level by level over the
// whole GPU: bins accumulate with atomics (per block in shared memory for the
// block's main node), one thread per node picks the split, and a scan of the
// left flags partitions each node's range stably. Nodes of at most
// kSahSeqMax triangles are built by one thread each, with the same split rule.
// A node whose centroids coincide on every axis splits its range in half.
// ---------------------------------------------------------------------------
constexpr int kSahBins = 32;
constexpr uint32_t kSahSeqMax = 64;
constexpr int kSahBinWords = 13;  // box lo, hi, centroid lo, hi (ordered ints), count
constexpr int kSahTaskWords = 3 * kSahBins * kSahBinWords;
constexpr int kSahMaxLevels = 512;

struct SahTask {
    uint32_t first, count;
    int node;
    int axis;           // split axis, -1: halve the range
    uint32_t clo[3], chi[3];  // centroid bounds (ordered ints)
    uint32_t split_bin;       // bins <= split_bin go left
    uint32_t left_count;
    int child_task[2];  // next-level large task, or -1
};

struct SahSmall {
    uint32_t first, count;
    int node;
};

// interior nodes allocated, large tasks of the next level (appended), small
// tasks (appended), large tasks of the current level
struct SahCounters {
    uint32_t nodes, large, small, level;
    uint32_t overflow;  // nonzero: a bound below was exceeded (nothing was written past it)
};

// Capacities of the next-level task list, the small-task list and the
// interior nodes (n - 1).
struct SahLimits {
    uint32_t large, small, nodes;
};

__device__ __forceinline__ float sah_half_area(float lx, float ly, float lz, float hx, float hy, float hz) {
    const float dx = hx - lx, dy = hy - ly, dz = hz - lz;
    if (!(dx >= 0.0f)) return 0.0f;  // empty box
    return dx * dy + dy * dz + dz * dx;
}

// Bin of centroid c on an axis with centroid bounds [lo, hi]; every centroid
// lands in bin 0 when the bounds have no extent.
__device__ __forceinline__ int sah_bin(float c, float lo, float hi) {
    const float ext = hi - lo;
    if (!(ext > 0.0f)) return 0;
    const float scale = (float)kSahBins / ext;
    const int b = (int)((c - lo) * scale);
    return min(max(b, 0), kSahBins - 1);
}

__device__ __forceinline__ float3 sah_centroid(float4 lo, float4 hi) {
    return make_float3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z));
}

__global__ void k_sah_init(uint32_t n, int* __restrict__ ids, int* __restrict__ task_of, int first_task) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ids[i] = (int)i;
    task_of[i] = first_task;
}

__global__ void k_sah_root(uint32_t n, const Bounds* __restrict__ bounds, SahTask* __restrict__ tasks,
                           SahSmall* __restrict__ small, SahCounters* __restrict__ ctr) {
    ctr->nodes = 1u;
    ctr->large = 0u;
    ctr->level = n > kSahSeqMax ? 1u : 0u;
    ctr->overflow = 0u;
    if (n > kSahSeqMax) {
        SahTask t;
        t.first = 0u;
        t.count = n;
        t.node = 0;
        t.axis = -1;
        for (int a = 0; a < 3; ++a) {
            t.clo[a] = bounds->lo[a];
            t.chi[a] = bounds->hi[a];
        }
        t.split_bin = 0u;
        t.left_count = 0u;
        t.child_task[0] = t.child_task[1] = -1;
        tasks[0] = t;
        ctr->small = 0u;
    } else {
        small[0] = SahSmall{0u, n, 0};
        ctr->small = 1u;
    }
}

__global__ void k_sah_bins_reset(uint32_t words, uint32_t* __restrict__ bins) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= words) return;
    const uint32_t w = i % kSahBinWords;
    // min fields start at the largest ordered value, max fields and counts at 0
    bins[i] = (w < 3 || (w >= 6 && w < 9)) ? 0xffffffffu : 0u;
}

__device__ __forceinline__ void sah_bin_add(uint32_t* b, float4 lo, float4 hi, float3 c) {
    const uint32_t v[12] = {float_to_ordered(lo.x), float_to_ordered(lo.y), float_to_ordered(lo.z),
                            float_to_ordered(hi.x), float_to_ordered(hi.y), float_to_ordered(hi.z),
                            float_to_ordered(c.x),  float_to_ordered(c.y),  float_to_ordered(c.z),
                            float_to_ordered(c.x),  float_to_ordered(c.y),  float_to_ordered(c.z)};
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        if (k < 3 || (k >= 6 && k < 9)) atomicMin(b + k, v[k]);
        else atomicMax(b + k, v[k]);
    }
    atomicAdd(b + 12, 1u);
}

constexpr int kSahBinPerThread = 4;

// Bins of every triangle in a large node. A block covers kThreads x
// kSahBinPerThread consecutive positions and keeps the bins of the node at
// its first position in shared memory.
__global__ void __launch_bounds__(kThreads) k_sah_bin(uint32_t n, const int* __restrict__ ids,
                                                      const int* __restrict__ task_of,
                                                      const SahTask* __restrict__ tasks,
                                                      const float4* __restrict__ leaf_lo,
                                                      const float4* __restrict__ leaf_hi, uint32_t* __restrict__ bins) {
    __shared__ uint32_t s_bins[kSahTaskWords];
    __shared__ uint32_t s_first;
    const uint32_t base = blockIdx.x * (uint32_t)(kThreads * kSahBinPerThread);
    if (threadIdx.x == 0) s_first = 0xffffffffu;
    for (int i = threadIdx.x; i < kSahTaskWords; i += kThreads) {
        const int w = i % kSahBinWords;
        s_bins[i] = (w < 3 || (w >= 6 && w < 9)) ? 0xffffffffu : 0u;
    }
    __syncthreads();
    for (int k = 0; k < kSahBinPerThread; ++k) {
        const uint32_t p = base + (uint32_t)k * kThreads + threadIdx.x;
        if (p < n && task_of[p] >= 0) {
            atomicMin(&s_first, p);
            break;
        }
    }
    __syncthreads();
    if (s_first == 0xffffffffu) return;
    const int main_task = task_of[s_first];
    for (int k = 0; k < kSahBinPerThread; ++k) {
        const uint32_t p = base + (uint32_t)k * kThreads + threadIdx.x;
        if (p >= n) break;
        const int t = task_of[p];
        if (t < 0) continue;
        const int prim = ids[p];
        const float4 lo = leaf_lo[prim], hi = leaf_hi[prim];
        const float3 c = sah_centroid(lo, hi);
        const SahTask& task = tasks[t];
        const float cc[3] = {c.x, c.y, c.z};
        uint32_t* dst = t == main_task ? s_bins : bins + (size_t)t * kSahTaskWords;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int b = sah_bin(cc[a], ordered_to_float(task.clo[a]), ordered_to_float(task.chi[a]));
            sah_bin_add(dst + (a * kSahBins + b) * kSahBinWords, lo, hi, c);
        }
    }
    __syncthreads();
    uint32_t* g = bins + (size_t)main_task * kSahTaskWords;
    for (int i = threadIdx.x; i < kSahTaskWords; i += kThreads) {
        const int w = i % kSahBinWords;
        const uint32_t v = s_bins[i];
        if (w < 3 || (w >= 6 && w < 9)) {
            if (v != 0xffffffffu) atomicMin(g + i, v);
        } else if (v != 0u) {
            if (w == 12) atomicAdd(g + i, v);
            else atomicMax(g + i, v);
        }
    }
}

// One warp per large node, lane b holding bin b of each axis: the node's box
// (the union of its axis-0 bins), the best split (left and right sweeps as
// warp scans of the bins' ordered-int boxes and counts; the first minimum over
// axes 0..2, then bins 0..30), and the children, which lane 0 allocates:
// interior ids, next-level or small tasks.
static_assert(kSahBins == 32, "one bin per lane");
__global__ void __launch_bounds__(128) k_sah_split(const uint32_t* __restrict__ count, SahTask* __restrict__ tasks,
                            const uint32_t* __restrict__ bins, SahTask* __restrict__ next, SahSmall* __restrict__ small,
                            SahCounters* __restrict__ ctr, SahLimits lim, int2* __restrict__ children,
                            int* __restrict__ node_parent, float4* __restrict__ node_lo, float4* __restrict__ node_hi) {
    constexpr uint32_t kFull = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= *count) return;  // the whole warp leaves together
    SahTask task = tasks[t];
    const uint32_t* tb = bins + (size_t)t * kSahTaskWords;
    {
        const uint32_t* w = tb + lane * kSahBinWords;
        uint32_t box[6];
        for (int k = 0; k < 3; ++k) {
            box[k] = __reduce_min_sync(kFull, w[k]);
            box[3 + k] = __reduce_max_sync(kFull, w[3 + k]);
        }
        if (lane == 0) {
            node_lo[task.node] =
                make_float4(ordered_to_float(box[0]), ordered_to_float(box[1]), ordered_to_float(box[2]), 0.f);
            node_hi[task.node] =
                make_float4(ordered_to_float(box[3]), ordered_to_float(box[4]), ordered_to_float(box[5]), 0.f);
        }
    }
    float best_cost = INFINITY;
    int best_axis = -1, best_bin = 0;
    for (int a = 0; a < 3; ++a) {
        const float ext = ordered_to_float(task.chi[a]) - ordered_to_float(task.clo[a]);
        if (!(ext > 0.0f)) continue;  // uniform across the warp
        const uint32_t* w = tb + (a * kSahBins + lane) * kSahBinWords;
        // empty bins hold the identities (min fields all ones, max fields 0)
        uint32_t pl[3] = {w[0], w[1], w[2]}, ph[3] = {w[3], w[4], w[5]}, pn = w[12];
        uint32_t sl[3] = {w[0], w[1], w[2]}, sh[3] = {w[3], w[4], w[5]}, sn = w[12];
        for (uint32_t d = 1; d < 32u; d <<= 1) {
            uint32_t ul[3], uh[3], dl[3], dh[3];
            for (int k = 0; k < 3; ++k) {
                ul[k] = __shfl_up_sync(kFull, pl[k], d);
                uh[k] = __shfl_up_sync(kFull, ph[k], d);
                dl[k] = __shfl_down_sync(kFull, sl[k], d);
                dh[k] = __shfl_down_sync(kFull, sh[k], d);
            }
            const uint32_t un = __shfl_up_sync(kFull, pn, d), dn = __shfl_down_sync(kFull, sn, d);
            if (lane >= d) {
                for (int k = 0; k < 3; ++k) {
                    pl[k] = min(pl[k], ul[k]);
                    ph[k] = max(ph[k], uh[k]);
                }
                pn += un;
            }
            if (lane + d < 32u) {
                for (int k = 0; k < 3; ++k) {
                    sl[k] = min(sl[k], dl[k]);
                    sh[k] = max(sh[k], dh[k]);
                }
                sn += dn;
            }
        }
        // split after bin `lane`: left = bins 0..lane (prefix), right = bins lane+1..31
        uint32_t rl[3], rh[3];
        for (int k = 0; k < 3; ++k) {
            rl[k] = __shfl_down_sync(kFull, sl[k], 1);
            rh[k] = __shfl_down_sync(kFull, sh[k], 1);
        }
        const uint32_t rn = __shfl_down_sync(kFull, sn, 1);
        float cost = INFINITY;
        if (lane < 31u && pn != 0u && rn != 0u) {
            const float la = sah_half_area(ordered_to_float(pl[0]), ordered_to_float(pl[1]), ordered_to_float(pl[2]),
                                           ordered_to_float(ph[0]), ordered_to_float(ph[1]), ordered_to_float(ph[2]));
            const float ra = sah_half_area(ordered_to_float(rl[0]), ordered_to_float(rl[1]), ordered_to_float(rl[2]),
                                           ordered_to_float(rh[0]), ordered_to_float(rh[1]), ordered_to_float(rh[2]));
            cost = la * (float)pn + ra * (float)rn;
        }
        float m = cost;
        for (int d = 16; d > 0; d >>= 1) m = fminf(m, __shfl_xor_sync(kFull, m, d));
        if (m < best_cost) {  // strictly cheaper than the earlier axes' best
            best_cost = m;
            best_axis = a;
            best_bin = __ffs(__ballot_sync(kFull, cost == m)) - 1;  // the first bin reaching it
        }
    }
    uint32_t left = task.count / 2u;
    uint32_t cb[2][6];  // children's centroid bounds
    if (best_axis >= 0) {
        const uint32_t* w = tb + (best_axis * kSahBins + lane) * kSahBinWords;
        const bool in_left = (int)lane <= best_bin;
        left = __reduce_add_sync(kFull, in_left ? w[12] : 0u);
        for (int k = 0; k < 3; ++k) {
            cb[0][k] = __reduce_min_sync(kFull, in_left ? w[6 + k] : 0xffffffffu);
            cb[0][3 + k] = __reduce_max_sync(kFull, in_left ? w[9 + k] : 0u);
            cb[1][k] = __reduce_min_sync(kFull, in_left ? 0xffffffffu : w[6 + k]);
            cb[1][3 + k] = __reduce_max_sync(kFull, in_left ? 0u : w[9 + k]);
        }
    } else {
        for (int s = 0; s < 2; ++s)
            for (int k = 0; k < 3; ++k) {
                cb[s][k] = task.clo[k];
                cb[s][3 + k] = task.chi[k];
            }
    }
    if (lane != 0u) return;
    task.axis = best_axis;
    task.split_bin = (uint32_t)best_bin;
    task.left_count = left;
    const uint32_t counts[2] = {left, task.count - left};
    int refs[2] = {0, 0};
    for (int s = 0; s < 2; ++s) {
        task.child_task[s] = -1;
        if (counts[s] == 1u) continue;  // a leaf: the scatter writes it
        const int id = (int)atomicAdd(&ctr->nodes, 1u);
        if ((uint32_t)id >= lim.nodes) {
            atomicOr(&ctr->overflow, 1u);
            continue;
        }
        refs[s] = id;
        node_parent[id] = task.node;
        const uint32_t first = task.first + (s ? left : 0u);
        if (counts[s] > kSahSeqMax) {
            const uint32_t ti = atomicAdd(&ctr->large, 1u);
            if (ti >= lim.large) {
                atomicOr(&ctr->overflow, 2u);
                continue;
            }
            SahTask c;
            c.first = first;
            c.count = counts[s];
            c.node = id;
            c.axis = -1;
            for (int k = 0; k < 3; ++k) {
                c.clo[k] = cb[s][k];
                c.chi[k] = cb[s][3 + k];
            }
            c.split_bin = 0u;
            c.left_count = 0u;
            c.child_task[0] = c.child_task[1] = -1;
            next[ti] = c;
            task.child_task[s] = (int)ti;
        } else {
            const uint32_t si = atomicAdd(&ctr->small, 1u);
            if (si >= lim.small) {
                atomicOr(&ctr->overflow, 4u);
                continue;
            }
            small[si] = SahSmall{first, counts[s], id};
        }
    }
    if (counts[0] != 1u) children[task.node].x = refs[0];
    if (counts[1] != 1u) children[task.node].y = refs[1];
    tasks[t] = task;
}

__device__ __forceinline__ bool sah_goes_left(const SahTask& task, uint32_t p, const int* ids, const float4* leaf_lo,
                                              const float4* leaf_hi) {
    if (task.axis < 0) return p - task.first < task.left_count;
    const int prim = ids[p];
    const float3 c = sah_centroid(leaf_lo[prim], leaf_hi[prim]);
    const float cc = task.axis == 0 ? c.x : task.axis == 1 ? c.y : c.z;
    const int b = sah_bin(cc, ordered_to_float(task.clo[task.axis]), ordered_to_float(task.chi[task.axis]));
    return (uint32_t)b <= task.split_bin;
}

__global__ void k_sah_flags(uint32_t n, const int* __restrict__ ids, const int* __restrict__ task_of,
                            const SahTask* __restrict__ tasks, const float4* __restrict__ leaf_lo,
                            const float4* __restrict__ leaf_hi, uint32_t* __restrict__ flags) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > n) return;
    uint32_t f = 0u;
    if (p < n) {
        const int t = task_of[p];
        if (t >= 0) f = sah_goes_left(tasks[t], p, ids, leaf_lo, leaf_hi) ? 1u : 0u;
    }
    flags[p] = f;
}

// Stable partition of every large node's range (rank = left flags before the
// position, from an exclusive scan), and the leaves of its children.
__global__ void k_sah_scatter(uint32_t n, const int* __restrict__ ids, const int* __restrict__ task_of,
                              const SahTask* __restrict__ tasks, const uint32_t* __restrict__ flags,
                              const uint32_t* __restrict__ rank, int* __restrict__ ids_out,
                              int* __restrict__ task_of_out, int2* __restrict__ children,
                              int* __restrict__ leaf_parent, SahCounters* __restrict__ ctr) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int t = task_of[p];
    const int prim = ids[p];
    if (t < 0) {
        ids_out[p] = prim;
        task_of_out[p] = -1;
        return;
    }
    const SahTask& task = tasks[t];
    const uint32_t r = rank[p] - rank[task.first];
    const bool left = flags[p] != 0u;
    // a left rank past the left count (or a right rank past the right count)
    // means the flags and the bins disagree: stop before writing
    if (left ? r >= task.left_count : (p - task.first - r) >= task.count - task.left_count) {
        atomicOr(&ctr->overflow, 8u);
        return;
    }
    const uint32_t q = left ? task.first + r : task.first + task.left_count + (p - task.first - r);
    ids_out[q] = prim;
    const int s = left ? 0 : 1;
    task_of_out[q] = task.child_task[s];
    const uint32_t cn = left ? task.left_count : task.count - task.left_count;
    if (cn == 1u) {
        if (s == 0) children[task.node].x = ~prim;
        else children[task.node].y = ~prim;
        leaf_parent[prim] = task.node;
    }
}

// One thread builds the whole subtree of a small node, with the same split
// rule, partitioning its range of ids in place (stably, through a local copy).
__global__ void k_sah_small(const uint32_t* __restrict__ count, const SahSmall* __restrict__ small,
                            int* __restrict__ ids, const float4* __restrict__ leaf_lo,
                            const float4* __restrict__ leaf_hi, SahCounters* __restrict__ ctr, SahLimits lim,
                            int2* __restrict__ children, int* __restrict__ node_parent, int* __restrict__ leaf_parent,
                            float4* __restrict__ node_lo, float4* __restrict__ node_hi) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count || i >= lim.small) return;
    const SahSmall root = small[i];
    if (root.count < 2u || root.count > kSahSeqMax) {
        atomicOr(&ctr->overflow, 16u);
        return;
    }
    int next_id = root.count > 2u ? (int)atomicAdd(&ctr->nodes, root.count - 2u) : 0;
    if (root.count > 2u && (uint32_t)next_id + (root.count - 2u) > lim.nodes) {
        atomicOr(&ctr->overflow, 1u);
        return;
    }
    uint32_t st_first[kSahSeqMax], st_count[kSahSeqMax];
    int st_node[kSahSeqMax];
    int sp = 0;
    st_first[0] = root.first;
    st_count[0] = root.count;
    st_node[0] = root.node;
    sp = 1;
    int tmp[kSahSeqMax];
    while (sp > 0) {
        --sp;
        const uint32_t first = st_first[sp], cnt = st_count[sp];
        const int node = st_node[sp];
        float bl[3] = {INFINITY, INFINITY, INFINITY}, bh[3] = {-INFINITY, -INFINITY, -INFINITY};
        float cl[3] = {INFINITY, INFINITY, INFINITY}, ch[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t k = 0; k < cnt; ++k) {
            const int prim = ids[first + k];
            const float4 lo = leaf_lo[prim], hi = leaf_hi[prim];
            const float3 c = sah_centroid(lo, hi);
            bl[0] = fminf(bl[0], lo.x); bl[1] = fminf(bl[1], lo.y); bl[2] = fminf(bl[2], lo.z);
            bh[0] = fmaxf(bh[0], hi.x); bh[1] = fmaxf(bh[1], hi.y); bh[2] = fmaxf(bh[2], hi.z);
            cl[0] = fminf(cl[0], c.x); cl[1] = fminf(cl[1], c.y); cl[2] = fminf(cl[2], c.z);
            ch[0] = fmaxf(ch[0], c.x); ch[1] = fmaxf(ch[1], c.y); ch[2] = fmaxf(ch[2], c.z);
        }
        node_lo[node] = make_float4(bl[0], bl[1], bl[2], 0.0f);
        node_hi[node] = make_float4(bh[0], bh[1], bh[2], 0.0f);
        float best_cost = INFINITY;
        int best_axis = -1, best_bin = 0;
        for (int a = 0; a < 3; ++a) {
            if (!(ch[a] - cl[a] > 0.0f)) continue;
            float lo3[kSahBins][3], hi3[kSahBins][3];
            uint32_t nb[kSahBins];
            for (int b = 0; b < kSahBins; ++b) {
                nb[b] = 0u;
                for (int k = 0; k < 3; ++k) {
                    lo3[b][k] = INFINITY;
                    hi3[b][k] = -INFINITY;
                }
            }
            for (uint32_t k = 0; k < cnt; ++k) {
                const int prim = ids[first + k];
                const float4 lo = leaf_lo[prim], hi = leaf_hi[prim];
                const float3 c = sah_centroid(lo, hi);
                const float cc = a == 0 ? c.x : a == 1 ? c.y : c.z;
                const int b = sah_bin(cc, cl[a], ch[a]);
                nb[b]++;
                lo3[b][0] = fminf(lo3[b][0], lo.x); lo3[b][1] = fminf(lo3[b][1], lo.y); lo3[b][2] = fminf(lo3[b][2], lo.z);
                hi3[b][0] = fmaxf(hi3[b][0], hi.x); hi3[b][1] = fmaxf(hi3[b][1], hi.y); hi3[b][2] = fmaxf(hi3[b][2], hi.z);
            }
            float right_area[kSahBins];
            uint32_t right_n[kSahBins];
            float rl[3] = {INFINITY, INFINITY, INFINITY}, rh[3] = {-INFINITY, -INFINITY, -INFINITY};
            uint32_t rn = 0u;
            for (int b = kSahBins - 1; b >= 1; --b) {
                for (int k = 0; k < 3; ++k) {
                    rl[k] = fminf(rl[k], lo3[b][k]);
                    rh[k] = fmaxf(rh[k], hi3[b][k]);
                }
                rn += nb[b];
                right_area[b] = sah_half_area(rl[0], rl[1], rl[2], rh[0], rh[1], rh[2]);
                right_n[b] = rn;
            }
            float ll[3] = {INFINITY, INFINITY, INFINITY}, lh[3] = {-INFINITY, -INFINITY, -INFINITY};
            uint32_t ln = 0u;
            for (int b = 0; b < kSahBins - 1; ++b) {
                for (int k = 0; k < 3; ++k) {
                    ll[k] = fminf(ll[k], lo3[b][k]);
                    lh[k] = fmaxf(lh[k], hi3[b][k]);
                }
                ln += nb[b];
                if (ln == 0u || right_n[b + 1] == 0u) continue;
                const float c = sah_half_area(ll[0], ll[1], ll[2], lh[0], lh[1], lh[2]) * (float)ln +
                                right_area[b + 1] * (float)right_n[b + 1];
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = a;
                    best_bin = b;
                }
            }
        }
        // stable partition through tmp
        uint32_t left = 0u;
        if (best_axis >= 0) {
            uint32_t r = 0u;
            for (uint32_t k = 0; k < cnt; ++k) {
                const int prim = ids[first + k];
                const float3 c = sah_centroid(leaf_lo[prim], leaf_hi[prim]);
                const float cc = best_axis == 0 ? c.x : best_axis == 1 ? c.y : c.z;
                if (sah_bin(cc, cl[best_axis], ch[best_axis]) <= best_bin) ids[first + left++] = prim;
                else tmp[r++] = prim;
            }
            for (uint32_t k = 0; k < r; ++k) ids[first + left + k] = tmp[k];
        } else {
            left = cnt / 2u;
        }
        const uint32_t counts[2] = {left, cnt - left};
        int refs[2];
        for (int s = 0; s < 2; ++s) {
            const uint32_t f = first + (s ? left : 0u);
            if (counts[s] == 1u) {
                const int prim = ids[f];
                refs[s] = ~prim;
                leaf_parent[prim] = node;
            } else {
                const int id = next_id++;
                refs[s] = id;
                node_parent[id] = node;
                st_first[sp] = f;
                st_count[sp] = counts[s];
                st_node[sp] = id;
                ++sp;
            }
        }
        children[node] = make_int2(refs[0], refs[1]);
    }
}

template <class T> T* dmalloc(size_t count, cudaStream_t s, cudaError_t* err) {
    void* p = nullptr;
    cudaError_t e = nan_host::scratch_alloc(&p, std::max<size_t>(count, 1) * sizeof(T), s);
    if (e != cudaSuccess && *err == cudaSuccess) *err = e;
    return static_cast<T*>(p);
}

uint32_t blocks(uint64_t n) { return (uint32_t)((n + kThreads - 1) / kThreads); }

}  // namespace

namespace nan_host {

void forget_scene(NanContext* ctx) {
    ctx->wide_count = 0;
    ctx->wide_built = false;
    ctx->has_scene = false;
    ctx->tri_count = ctx->node_count = ctx->leaf_count = ctx->max_depth = 0;
}

void free_scene(NanContext* ctx) {
    if (!ctx->caller_owned_bvh) {
        cudaFree(ctx->nodes);
        cudaFree(ctx->tris);
        cudaFree(ctx->tri_refs);
    }
    cudaFree(ctx->wnodes);
    cudaFree(ctx->wtris);
    ctx->wnodes = nullptr;
    ctx->wtris = nullptr;
    ctx->caller_owned_bvh = false;
    ctx->nodes = nullptr;
    ctx->tris = nullptr;
    ctx->tri_refs = nullptr;
    ctx->bvh_capacity = ctx->wide_capacity = 0;
    ctx->device_bytes = 0;
    forget_scene(ctx);
}


int finish_binary(NanContext* ctx, uint32_t n, const float4* tris_sorted, const float4* leaf_lo,
                  const float4* leaf_hi, int2* children, int* node_parent, int* leaf_parent, float4* node_lo,
                  float4* node_hi, uint32_t* arrivals, uint32_t* depth, double* sah, const Bounds* bounds,
                  const int* root_dev, cudaStream_t s);

// Binned-SAH hierarchy over the leaves (kernels k_sah_*): large nodes level by
// level, one host readback of the next level's node count per level, then
// the small nodes in one launch; the root is interior node 0.
int build_binned(NanContext* ctx, uint32_t n, const float4* tris_sorted, const float4* leaf_lo,
                 const float4* leaf_hi, int2* children, int* node_parent, int* leaf_parent, float4* node_lo,
                 float4* node_hi, uint32_t* arrivals, uint32_t* depth, double* sah, const Bounds* bounds,
                 cudaStream_t s) {
    cudaError_t err = cudaSuccess;
    const uint32_t max_large = n / (kSahSeqMax + 1u) + 1u;
    const SahLimits lim{max_large, n / 2u + 1u, n - 1u};
    int* ids_a = dmalloc<int>(n, s, &err);
    int* ids_b = dmalloc<int>(n, s, &err);
    int* task_a = dmalloc<int>(n, s, &err);
    int* task_b = dmalloc<int>(n, s, &err);
    uint32_t* flags = dmalloc<uint32_t>(n + 1, s, &err);
    uint32_t* rank = dmalloc<uint32_t>(n + 1, s, &err);
    SahTask* level_a = dmalloc<SahTask>(max_large, s, &err);
    SahTask* level_b = dmalloc<SahTask>(max_large, s, &err);
    SahSmall* small = dmalloc<SahSmall>(n / 2u + 1u, s, &err);
    uint32_t* bins = dmalloc<uint32_t>((size_t)max_large * kSahTaskWords, s, &err);
    SahCounters* ctr = dmalloc<SahCounters>(1, s, &err);
    int* root_dev = dmalloc<int>(1, s, &err);
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flags, rank, n + 1, s);
    void* scan_tmp = dmalloc<uint8_t>(scan_bytes, s, &err);
    auto release = [&] {
        for (void* p : {(void*)ids_a, (void*)ids_b, (void*)task_a, (void*)task_b, (void*)flags, (void*)rank,
                        (void*)level_a, (void*)level_b, (void*)small, (void*)bins, (void*)ctr, (void*)root_dev,
                        scan_tmp})
            if (p) cudaFreeAsync(p, s);
    };
    // every exit releases the scratch
    auto fail = [&](cudaError_t e, const char* what) {
        release();
        return cuda_fail(e, what);
    };
    auto limit = [&](const char* what) {
        release();
        set_error(what);
        return NAN_ERR_LIMIT;
    };
    if (err != cudaSuccess) return fail(err, "binned SAH scratch allocation");
    cudaMemsetAsync(root_dev, 0, sizeof(int), s);
    cudaMemsetAsync(node_parent, 0xff, (n - 1u) * sizeof(int), s);  // the root's parent stays -1
    k_sah_init<<<blocks(n), kThreads, 0, s>>>(n, ids_a, task_a, n > kSahSeqMax ? 0 : -1);
    k_sah_root<<<1, 1, 0, s>>>(n, bounds, level_a, small, ctr);
    ctx->launches += 2;
    uint32_t large = n > kSahSeqMax ? 1u : 0u;
    int levels = 0;
    const uint32_t bin_grid = (uint32_t)((n + kThreads * kSahBinPerThread - 1) / (kThreads * kSahBinPerThread));
    while (large > 0u) {
        if (++levels > kSahMaxLevels) return limit("binned SAH build did not terminate");
        const uint32_t words = large * (uint32_t)kSahTaskWords;
        k_sah_bins_reset<<<blocks(words), kThreads, 0, s>>>(words, bins);
        k_sah_bin<<<bin_grid, kThreads, 0, s>>>(n, ids_a, task_a, level_a, leaf_lo, leaf_hi, bins);
        k_sah_split<<<(large * 32u + 127u) / 128u, 128, 0, s>>>(&ctr->level, level_a, bins, level_b, small, ctr, lim,
                                                                children, node_parent, node_lo, node_hi);
        k_sah_flags<<<blocks(n + 1), kThreads, 0, s>>>(n, ids_a, task_a, level_a, leaf_lo, leaf_hi, flags);
        cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, flags, rank, n + 1, s);
        k_sah_scatter<<<blocks(n), kThreads, 0, s>>>(n, ids_a, task_a, level_a, flags, rank, ids_b, task_b, children,
                                                     leaf_parent, ctr);
        ctx->launches += 6;
        // the next level's count becomes the current one
        SahCounters lc{};
        cudaMemcpyAsync(&ctr->level, &ctr->large, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        err = cudaMemcpyAsync(&lc, ctr, sizeof(SahCounters), cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaMemsetAsync(&ctr->large, 0, sizeof(uint32_t), s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) return fail(err, "binned SAH level");
        large = lc.large;
        if (lc.overflow != 0u || large > max_large) return limit("binned SAH build exceeded a bound of its node lists");
        std::swap(ids_a, ids_b);
        std::swap(task_a, task_b);
        std::swap(level_a, level_b);
    }
    SahCounters c{};
    err = cudaMemcpyAsync(&c, ctr, sizeof(SahCounters), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return fail(err, "binned SAH counters");
    if (c.small > 0u) {
        k_sah_small<<<(c.small + 127u) / 128u, 128, 0, s>>>(&ctr->small, small, ids_a, leaf_lo, leaf_hi, ctr, lim,
                                                             children, node_parent, leaf_parent, node_lo, node_hi);
        ctx->launches++;
    }
    err = cudaMemcpyAsync(&c, ctr, sizeof(SahCounters), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return fail(err, "binned SAH small nodes");
    if (c.overflow != 0u || c.nodes != n - 1u) return limit("binned SAH build made the wrong number of interior nodes");
    const int rc = finish_binary(ctx, n, tris_sorted, leaf_lo, leaf_hi, children, node_parent, leaf_parent, node_lo,
                                 node_hi, arrivals, depth, sah, bounds, root_dev, s);
    release();
    return rc;
}

// PLOC hierarchy over the Morton-sorted leaves, SAH leaf collapse, and a
// depth-first emission of nodes and triangles (see the kernels above).
int build_ploc(NanContext* ctx, uint32_t n, const float4* tris_sorted, const float4* leaf_lo, const float4* leaf_hi,
               int2* children, int* node_parent, int* leaf_parent, float4* node_lo, float4* node_hi,
               uint32_t* arrivals, uint32_t* depth, double* sah, const Bounds* bounds, cudaStream_t s) {
    cudaError_t err = cudaSuccess;
    const uint32_t interior = n - 1;
    int* idx_a = dmalloc<int>(n, s, &err);
    int* idx_b = dmalloc<int>(n, s, &err);
    float4* lo_a = dmalloc<float4>(n, s, &err);
    float4* hi_a = dmalloc<float4>(n, s, &err);
    float4* lo_b = dmalloc<float4>(n, s, &err);
    float4* hi_b = dmalloc<float4>(n, s, &err);
    int* nn = dmalloc<int>(n, s, &err);
    uint32_t* valid = dmalloc<uint32_t>(n + 1, s, &err);
    uint32_t* pos = dmalloc<uint32_t>(n + 1, s, &err);
    // [0] interior nodes made; [1], [2] live clusters (double-buffered)
    uint32_t* counter = dmalloc<uint32_t>(3, s, &err);
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, valid, pos, n + 1, s);
    void* scan_tmp = dmalloc<uint8_t>(scan_bytes, s, &err);
    if (err != cudaSuccess) return cuda_fail(err, "PLOC scratch allocation");
    cudaMemsetAsync(node_parent, 0xff, interior * sizeof(int), s);
    {
        const uint32_t init[3] = {0u, n, n};
        cudaMemcpyAsync(counter, init, sizeof(init), cudaMemcpyHostToDevice, s);
    }
    cudaMemsetAsync(valid, 0, (n + 1) * sizeof(uint32_t), s);
    k_ploc_init<<<blocks(n), kThreads, 0, s>>>(n, idx_a);
    cudaMemcpyAsync(lo_a, leaf_lo, n * sizeof(float4), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(hi_a, leaf_hi, n * sizeof(float4), cudaMemcpyDeviceToDevice, s);
    ctx->launches++;
    // Iterations run in batches of kPlocBatch without the host: each kernel
    // reads the live count (counter[1]); the host reads it back once per
    // batch to size the next batch's grids and to check progress.
    uint32_t c = n;
    int iterations = 0;
    while (c > 1) {
        if (iterations > 4096) {
            set_error("PLOC did not converge");
            return NAN_ERR_LIMIT;
        }
        const uint32_t grid = (c + kPlocBlock - 1) / kPlocBlock;
        for (int k = 0; k < kPlocBatch; ++k, ++iterations) {
            uint32_t* live = counter + 1 + (iterations & 1);
            uint32_t* next_live = counter + 1 + ((iterations + 1) & 1);
            k_ploc_nn<<<grid, kPlocBlock, 0, s>>>(live, lo_a, hi_a, nn);
            k_ploc_merge<<<blocks(c + 1), kThreads, 0, s>>>(live, (int)c, nn, idx_a, lo_a, hi_a, idx_b, lo_b, hi_b,
                                                            valid, children, node_parent, leaf_parent, node_lo,
                                                            node_hi, counter);
            cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, valid, pos, c + 1, s);
            k_ploc_compact<<<blocks(c), kThreads, 0, s>>>(live, next_live, valid, pos, idx_b, lo_b, hi_b, idx_a,
                                                          lo_a, hi_a);
            ctx->launches += 4;
        }
        uint32_t next = 0;
        // kPlocBatch is even, so after a batch the live count is in slot 1 + 0
        err = cudaMemcpyAsync(&next, counter + 1 + (iterations & 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) return cuda_fail(err, "PLOC iteration");
        if (next >= c) {
            set_error("PLOC made no progress");
            return NAN_ERR_LIMIT;
        }
        c = next;
    }
    const int rc = finish_binary(ctx, n, tris_sorted, leaf_lo, leaf_hi, children, node_parent, leaf_parent, node_lo,
                                 node_hi, arrivals, depth, sah, bounds, idx_a, s);
    for (void* p : {(void*)idx_a, (void*)idx_b, (void*)lo_a, (void*)hi_a, (void*)lo_b, (void*)hi_b, (void*)nn,
                    (void*)valid, (void*)pos, (void*)counter, scan_tmp})
        cudaFreeAsync(p, s);
    return rc;
}

// SAH leaf collapse, depth-first emission of nodes and triangles, and the
// compressed 8-wide conversion of a binary hierarchy over the n leaves
// (children / parents / interior boxes; root_dev[0] is the root's index).
int finish_binary(NanContext* ctx, uint32_t n, const float4* tris_sorted, const float4* leaf_lo,
                  const float4* leaf_hi, int2* children, int* node_parent, int* leaf_parent, float4* node_lo,
                  float4* node_hi, uint32_t* arrivals, uint32_t* depth, double* sah, const Bounds* bounds,
                  const int* root_dev, cudaStream_t s) {
    cudaError_t err = cudaSuccess;
    const uint32_t interior = n - 1;
    SubtreeInfo* info = dmalloc<SubtreeInfo>(interior, s, &err);
    int* dfs = dmalloc<int>(interior, s, &err);
    uint32_t* tri_off = dmalloc<uint32_t>(interior, s, &err);
    uint32_t* tri_pos = dmalloc<uint32_t>(n, s, &err);
    if (err != cudaSuccess) return cuda_fail(err, "BVH collapse scratch allocation");
    int root = 0;
    err = cudaMemcpyAsync(&root, root_dev, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_fail(err, "BVH root readback");
    cudaMemsetAsync(arrivals, 0, interior * sizeof(uint32_t), s);
    k_subtree<<<blocks(n), kThreads, 0, s>>>(n, children, node_parent, leaf_parent, leaf_lo, leaf_hi, node_lo, node_hi,
                                            info, arrivals);
    k_dfs_nodes<<<blocks(interior), kThreads, 0, s>>>(interior, children, node_parent, info, dfs, tri_off);
    k_dfs_leaves<<<blocks(n), kThreads, 0, s>>>(n, children, node_parent, leaf_parent, info, tri_pos);
    k_scatter_tris<<<blocks(n), kThreads, 0, s>>>(n, tri_pos, tris_sorted, ctx->tris);
    err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_fail(err, "BVH collapse");

    // compressed 8-wide BVH from the collapsed binary tree, level by level
    if (ctx->wide_capacity < n) {
        cudaFree(ctx->wnodes);
        cudaFree(ctx->wtris);
        ctx->wnodes = nullptr;
        ctx->wtris = nullptr;
        ctx->wide_capacity = 0;
        if (cudaMalloc(&ctx->wnodes, (size_t)n * 5 * sizeof(uint4)) != cudaSuccess ||
            cudaMalloc(&ctx->wtris, (size_t)n * 3 * sizeof(float4)) != cudaSuccess) {
            set_error("out of device memory for the wide BVH");
            return NAN_ERR_OUT_OF_MEMORY;
        }
        ctx->device_bytes += (uint64_t)n * (5 * sizeof(uint4) + 3 * sizeof(float4));
        ctx->wide_capacity = n;
    }
    WideItem* items_a = dmalloc<WideItem>(interior + 1, s, &err);
    WideItem* items_b = dmalloc<WideItem>(interior + 1, s, &err);
    // [0] wide nodes, [1] wide triangles, [2 + l] items of level l
    uint32_t* wcount = dmalloc<uint32_t>(2 + kWideMaxLevels + 1, s, &err);
    if (err != cudaSuccess) return cuda_fail(err, "wide BVH scratch allocation");
    {
        // the root item: the binary root; levels run in batches of
        // kWideBatch without the host, each grid bounded by 8x the last
        k_wide_root<<<1, 1, 0, s>>>(root_dev, items_a);
        cudaMemsetAsync(wcount, 0, (2 + kWideMaxLevels + 1) * sizeof(uint32_t), s);
        const uint32_t init[3] = {1u, 0u, 1u};
        cudaMemcpyAsync(wcount, init, sizeof(init), cudaMemcpyHostToDevice, s);
        uint64_t bound = 1;
        int level = 0;
        for (;;) {
            for (int k = 0; k < kWideBatch; ++k, ++level) {
                if (level >= kWideMaxLevels) {
                    set_error("wide BVH conversion did not terminate");
                    return NAN_ERR_LIMIT;
                }
                const WideItem* in = (level & 1) ? items_b : items_a;
                WideItem* out = (level & 1) ? items_a : items_b;
                k_wide_level<<<blocks(bound), kThreads, 0, s>>>(in, wcount + 2 + level, out, wcount + 3 + level,
                                                                wcount, children, node_lo, node_hi, leaf_lo, leaf_hi,
                                                                info, tri_off, tri_pos, ctx->tris, bounds,
                                                                ctx->wnodes, ctx->wtris);
                ctx->launches++;
                bound = std::min<uint64_t>(bound * 8u, (uint64_t)interior + 1u);
            }
            uint32_t pending = 0;
            err = cudaMemcpyAsync(&pending, wcount + 2 + level, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
            if (err == cudaSuccess) err = cudaMemcpyAsync(&ctx->wide_count, wcount, sizeof(uint32_t),
                                                          cudaMemcpyDeviceToHost, s);
            if (err == cudaSuccess) err = cudaStreamSynchronize(s);
            if (err != cudaSuccess) return cuda_fail(err, "wide BVH level");
            if (pending == 0u) break;
        }
        ctx->wide_built = true;
    }
    cudaFreeAsync(items_a, s);
    cudaFreeAsync(items_b, s);
    cudaFreeAsync(wcount, s);
    k_emit_dfs<<<blocks(interior), kThreads, 0, s>>>(interior, children, node_lo, node_hi, leaf_lo, leaf_hi, bounds,
                                                     info, dfs, tri_off, tri_pos, root, ctx->nodes, sah);
    k_depth<<<blocks(n), kThreads, 0, s>>>(n, node_parent, leaf_parent, depth);
    ctx->launches += 6;
    SubtreeInfo root_info;
    uint32_t max_depth = 0;
    double sah_host = 0.0;
    err = cudaMemcpyAsync(&root_info, info + root, sizeof(SubtreeInfo), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&max_depth, depth, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&sah_host, sah, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_fail(err, "BVH emit");
    for (void* p : {(void*)info, (void*)dfs, (void*)tri_off, (void*)tri_pos}) cudaFreeAsync(p, s);
    if (root_info.collapsed) {  // the whole scene is one leaf
        ctx->root = ~(int)(n - 1u);
        ctx->node_count = 0;
        ctx->sah_cost = (double)n;
    } else {
        ctx->root = 0;
        ctx->node_count = root_info.interior;
        ctx->sah_cost = sah_host;
    }
    ctx->leaf_count = n;
    ctx->max_depth = max_depth;
    return NAN_OK;
}

int build_scene(NanContext* ctx, const NanSceneDesc* sd, cudaStream_t s) {
    cudaError_t err = cudaSuccess;
    if (ctx->caller_owned_bvh) free_scene(ctx);  // never reuse caller memory
    else forget_scene(ctx);
    ctx->scene = *sd;
    const uint32_t I = sd->instance_count;

    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, s);

    // 1. flat offsets
    uint32_t* counts = dmalloc<uint32_t>(I + 1, s, &err);
    uint32_t* offsets = dmalloc<uint32_t>(I + 1, s, &err);
    if (err != cudaSuccess) return cuda_fail(err, "scene build allocation");
    k_instance_counts<<<blocks(I + 1), kThreads, 0, s>>>(reinterpret_cast<const uint4*>(sd->instance_descs),
                                                         reinterpret_cast<const uint4*>(sd->mesh_descs), I, counts);
    ctx->launches++;
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts, offsets, I + 1, s);
    void* scan_tmp = dmalloc<uint8_t>(scan_bytes, s, &err);
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, counts, offsets, I + 1, s);
    ctx->launches++;
    uint32_t total = 0;
    err = cudaMemcpyAsync(&total, offsets + I, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_fail(err, "scene build (triangle count)");
    cudaFreeAsync(scan_tmp, s);
    cudaFreeAsync(counts, s);
    if (total > (1u << 30)) {
        cudaFreeAsync(offsets, s);
        set_error("scene has more than 2^30 triangles");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    const uint32_t n = total;
    ctx->tri_count = n;

    // Persistent storage, kept from an earlier build when it is large enough.
    const uint32_t interior = n > 1 ? n - 1 : 0;
    const uint32_t cap = std::max<uint32_t>(n, 1);
    if (ctx->bvh_capacity < cap) {
        cudaFree(ctx->tris);
        cudaFree(ctx->tri_refs);
        cudaFree(ctx->nodes);
        ctx->tris = nullptr;
        ctx->tri_refs = nullptr;
        ctx->nodes = nullptr;
        ctx->bvh_capacity = 0;
        if (cudaMalloc(&ctx->tris, (size_t)cap * 3 * sizeof(float4)) != cudaSuccess ||
            cudaMalloc(&ctx->tri_refs, (size_t)cap * sizeof(uint2)) != cudaSuccess ||
            cudaMalloc(&ctx->nodes, (size_t)cap * 4 * sizeof(float4)) != cudaSuccess) {
            cudaFreeAsync(offsets, s);
            free_scene(ctx);
            set_error("out of device memory for the BVH");
            return NAN_ERR_OUT_OF_MEMORY;
        }
        ctx->bvh_capacity = cap;
    }
    ctx->device_bytes = (uint64_t)ctx->bvh_capacity * (3 * sizeof(float4) + sizeof(uint2) + 4 * sizeof(float4)) +
                        (uint64_t)ctx->wide_capacity * (5 * sizeof(uint4) + 3 * sizeof(float4));

    if (n == 0) {
        cudaFreeAsync(offsets, s);
        ctx->has_scene = true;
        ctx->root = 0;
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        return NAN_OK;
    }

    // Scratch.
    float4* tris_flat = dmalloc<float4>(3ull * n, s, &err);
    float4* lo_flat = dmalloc<float4>(n, s, &err);
    float4* hi_flat = dmalloc<float4>(n, s, &err);
    Bounds* bounds = dmalloc<Bounds>(1, s, &err);
    uint64_t* keys = dmalloc<uint64_t>(n, s, &err);
    uint64_t* keys_sorted = dmalloc<uint64_t>(n, s, &err);
    uint32_t* vals = dmalloc<uint32_t>(n, s, &err);
    uint32_t* order = dmalloc<uint32_t>(n, s, &err);
    float4* leaf_lo = dmalloc<float4>(n, s, &err);
    float4* leaf_hi = dmalloc<float4>(n, s, &err);
    int2* children = dmalloc<int2>(std::max<uint32_t>(interior, 1), s, &err);
    int* node_parent = dmalloc<int>(std::max<uint32_t>(interior, 1), s, &err);
    int* leaf_parent = dmalloc<int>(n, s, &err);
    float4* node_lo = dmalloc<float4>(std::max<uint32_t>(interior, 1), s, &err);
    float4* node_hi = dmalloc<float4>(std::max<uint32_t>(interior, 1), s, &err);
    uint32_t* arrivals = dmalloc<uint32_t>(std::max<uint32_t>(interior, 1), s, &err);
    uint32_t* depth = dmalloc<uint32_t>(1, s, &err);
    double* sah = dmalloc<double>(1, s, &err);
    if (err != cudaSuccess) return cuda_fail(err, "scene build scratch allocation");

    Bounds init;
    for (int a = 0; a < 3; ++a) {
        init.lo[a] = 0xffffffffu;
        init.hi[a] = 0u;
    }
    init.max_abs = 0u;
    cudaMemcpyAsync(bounds, &init, sizeof(Bounds), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(arrivals, 0, std::max<uint32_t>(interior, 1) * sizeof(uint32_t), s);
    cudaMemsetAsync(depth, 0, sizeof(uint32_t), s);
    cudaMemsetAsync(sah, 0, sizeof(double), s);

    // 2-3. flatten + bounds
    k_flatten<<<blocks(n), kThreads, 0, s>>>(*sd, offsets, n, tris_flat, ctx->tri_refs, lo_flat, hi_flat, bounds);
    // 4. Morton codes + sort
    k_morton<<<blocks(n), kThreads, 0, s>>>(lo_flat, hi_flat, n, bounds, keys, vals);
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys, keys_sorted, vals, order, (int)n, 0, 63, s);
    void* sort_tmp = dmalloc<uint8_t>(sort_bytes, s, &err);
    if (err != cudaSuccess) return cuda_fail(err, "scene build sort allocation");
    cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, keys, keys_sorted, vals, order, (int)n, 0, 63, s);
    // NanTuning.bvh_builder: 0 binned SAH, 1 LBVH, 2 PLOC
    const bool use_sah = ctx->tuning.bvh_builder == 0 && n > 1;
    const bool use_ploc = ctx->tuning.bvh_builder == 2 && n > 1;
    float4* tris_sorted = (use_sah || use_ploc) ? dmalloc<float4>(3ull * n, s, &err) : ctx->tris;
    if (err != cudaSuccess) return cuda_fail(err, "scene build scratch allocation");
    k_gather_leaves<<<blocks(n), kThreads, 0, s>>>(order, n, tris_flat, lo_flat, hi_flat, tris_sorted, leaf_lo, leaf_hi);
    ctx->launches += 4;
    if (n == 1) {
        ctx->root = ~0;
        ctx->node_count = 0;
        ctx->leaf_count = 1;
        ctx->max_depth = 1;
        ctx->sah_cost = 1.0;
    } else if (use_sah || use_ploc) {
        int rc = use_sah ? build_binned(ctx, n, tris_sorted, leaf_lo, leaf_hi, children, node_parent, leaf_parent,
                                        node_lo, node_hi, arrivals, depth, sah, bounds, s)
                         : build_ploc(ctx, n, tris_sorted, leaf_lo, leaf_hi, children, node_parent, leaf_parent,
                                      node_lo, node_hi, arrivals, depth, sah, bounds, s);
        cudaFreeAsync(tris_sorted, s);
        if (rc != NAN_OK) return rc;
    } else {
        // 5-7. hierarchy, refit, depth, emit
        k_hierarchy<<<blocks(interior), kThreads, 0, s>>>(keys_sorted, (int)n, children, node_parent, leaf_parent);
        k_refit<<<blocks(n), kThreads, 0, s>>>(n, children, node_parent, leaf_parent, leaf_lo, leaf_hi, node_lo,
                                               node_hi, arrivals);
        k_depth<<<blocks(n), kThreads, 0, s>>>(n, node_parent, leaf_parent, depth);
        k_emit<<<blocks(interior), kThreads, 0, s>>>(interior, children, node_lo, node_hi, leaf_lo, leaf_hi, bounds,
                                                     ctx->nodes, sah);
        ctx->launches += 4;
        ctx->root = 0;
        ctx->node_count = interior;
        ctx->leaf_count = n;
        uint32_t max_depth = 0;
        double sah_host = 0.0;
        err = cudaMemcpyAsync(&max_depth, depth, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(&sah_host, sah, sizeof(double), cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) return cuda_fail(err, "scene build (depth and SAH readback)");
        ctx->max_depth = max_depth;
        ctx->sah_cost = sah_host;
    }
    cudaEventRecord(ev1, s);
    for (void* p : {(void*)offsets, (void*)tris_flat, (void*)lo_flat, (void*)hi_flat, (void*)bounds, (void*)keys,
                    (void*)keys_sorted, (void*)vals, (void*)order, (void*)leaf_lo, (void*)leaf_hi, (void*)children,
                    (void*)node_parent, (void*)leaf_parent, (void*)node_lo, (void*)node_hi, (void*)arrivals,
                    (void*)depth, (void*)sah, sort_tmp})
        cudaFreeAsync(p, s);
    err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_fail(err, "scene build");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    ctx->build_ms = ms;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (ctx->max_depth > 96u) {
        set_error("BVH deeper than the traversal stack (96)");
        free_scene(ctx);
        return NAN_ERR_LIMIT;
    }
    ctx->has_scene = true;
    return NAN_OK;
}

namespace {
__global__ void k_world_tris(const float4* __restrict__ tris, uint32_t n, float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = tris[3u * i], b = tris[3u * i + 1], c = tris[3u * i + 2];
    const uint32_t f = __float_as_uint(a.w);
    float* o = out + 9ull * f;
    o[0] = a.x; o[1] = a.y; o[2] = a.z;
    o[3] = b.x; o[4] = b.y; o[5] = b.z;
    o[6] = c.x; o[7] = c.y; o[8] = c.z;
}
}  // namespace

int world_triangles(NanContext* ctx, float* out, cudaStream_t s) {
    if (ctx->tri_count == 0) return NAN_OK;
    k_world_tris<<<blocks(ctx->tri_count), kThreads, 0, s>>>(ctx->tris, ctx->tri_count, out);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "world triangles");
}

}  // namespace nan_host

// ---------------------------------------------------------------------------
// nan_scene_build_noalloc: the scene build for callers that cannot allocate
// device memory (code running where cudaMalloc is unavailable or forbidden,
// e.g. inside another framework's memory pool or a real-time loop that must
// never allocate). All scratch lives in the fixed array below; the BVH goes
// into caller-provided buffers.
// ---------------------------------------------------------------------------
namespace {

// Scratch shared by every nan_scene_build_noalloc call on a device. The CUDA
// loader places one copy on each GPU that loads this library, held until the
// process exits. Calls that overlap on the GPU race on it.
constexpr size_t kNoAllocScratchBytes = 64ull << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device ordinal. In host code the
// symbol is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, taken once per device with that device current. The
// cached address belongs to the device's primary context: after
// cudaDeviceReset it is stale, and the library must not be used for a
// no-alloc build on that device again in this process.
std::mutex g_noalloc_mutex;
void* g_noalloc_address[128] = {};

int noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= 128) {
        set_error("device ordinal out of range for the no-alloc scratch table");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_address[device] == nullptr) {
        void* p = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess) return cuda_fail(err, "cudaGetSymbolAddress(no-alloc scratch)");
        g_noalloc_address[device] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_address[device]);
    return NAN_OK;
}

// Bump carving of the static scratch, 256-byte aligned.
struct Carver {
    unsigned char* base;
    size_t used = 0;
    size_t capacity;
    template <class T> T* take(size_t count) {
        used = (used + 255u) & ~size_t(255u);
        T* p = reinterpret_cast<T*>(base + used);
        used += std::max<size_t>(count, 1) * sizeof(T);
        return p;
    }
    bool fits() const { return used <= capacity; }
};

}  // namespace

extern "C" NAN_B200_API int nan_scene_build_noalloc(NanContext* ctx, const NanSceneDesc* sd, float* out_nodes,
                                                    uint64_t nodes_bytes, float* out_tris, uint64_t tris_bytes,
                                                    uint32_t* out_refs, uint64_t refs_bytes, void* stream) {
    if (!ctx || !sd) {
        set_error("null context or scene description");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    cudaError_t err = cudaSetDevice(ctx->device);
    if (err != cudaSuccess) return cuda_fail(err, "cudaSetDevice");
    if (!ctx->caller_owned_bvh && (ctx->nodes || ctx->tris || ctx->tri_refs)) {
        set_error("context holds a BVH allocated by nan_scene_build; use a context without one");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    // Forget the previous caller-owned BVH without freeing anything.
    auto forget_bvh = [ctx]() {
        ctx->nodes = nullptr;
        ctx->tris = nullptr;
        ctx->tri_refs = nullptr;
        ctx->caller_owned_bvh = false;
        ctx->has_scene = false;
        ctx->tri_count = ctx->node_count = ctx->leaf_count = ctx->max_depth = 0;
        ctx->device_bytes = 0;
    };
    if (sd->instance_count == 0 || !sd->vertices || !sd->indices || !sd->mesh_descs || !sd->instance_descs ||
        !sd->transforms || !sd->inverse_transposes || !sd->materials) {
        set_error("scene needs at least one instance and non-null buffers");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    if (!out_nodes || !out_tris || !out_refs || (reinterpret_cast<uintptr_t>(out_nodes) & 15u) ||
        (reinterpret_cast<uintptr_t>(out_tris) & 15u) || (reinterpret_cast<uintptr_t>(out_refs) & 7u)) {
        set_error("output buffers must be non-null; nodes and tris 16-byte aligned, refs 8-byte aligned");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* scratch = nullptr;
    int rc = noalloc_scratch(ctx->device, &scratch);
    if (rc) return rc;
    const uint32_t I = sd->instance_count;

    // Triangle count (per-instance counts + scan in the scratch).
    Carver head{scratch, 0, kNoAllocScratchBytes};
    uint32_t* counts = head.take<uint32_t>(I + 1);
    uint32_t* offsets = head.take<uint32_t>(I + 1);
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts, offsets, I + 1, s);
    unsigned char* scan_tmp = head.take<unsigned char>(scan_bytes);
    if (!head.fits()) {
        set_error("too many instances for the no-alloc scratch (64 MiB)");
        return NAN_ERR_LIMIT;
    }
    k_instance_counts<<<blocks(I + 1), kThreads, 0, s>>>(reinterpret_cast<const uint4*>(sd->instance_descs),
                                                         reinterpret_cast<const uint4*>(sd->mesh_descs), I, counts);
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, counts, offsets, I + 1, s);
    ctx->launches += 2;
    uint32_t n = 0;
    err = cudaMemcpyAsync(&n, offsets + I, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return cuda_fail(err, "no-alloc scene build (triangle count)");
    if (n == 0) {
        set_error("scene has no triangles");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    const uint32_t interior = n > 1 ? n - 1 : 0;
    if (nodes_bytes < (uint64_t)std::max<uint32_t>(interior, 1) * 64u || tris_bytes < (uint64_t)n * 48u ||
        refs_bytes < (uint64_t)n * 8u) {
        set_error("output buffers too small: need 64*max(T-1,1) node, 48*T triangle and 8*T ref bytes");
        return NAN_ERR_INVALID_ARGUMENT;
    }

    // Carve the rest of the build's scratch after the offsets.
    Carver c = head;
    float4* tris_flat = c.take<float4>(3ull * n);
    float4* lo_flat = c.take<float4>(n);
    float4* hi_flat = c.take<float4>(n);
    Bounds* bounds = c.take<Bounds>(1);
    uint64_t* keys = c.take<uint64_t>(n);
    uint64_t* keys_sorted = c.take<uint64_t>(n);
    uint32_t* vals = c.take<uint32_t>(n);
    uint32_t* order = c.take<uint32_t>(n);
    float4* leaf_lo = c.take<float4>(n);
    float4* leaf_hi = c.take<float4>(n);
    int2* children = c.take<int2>(interior);
    int* node_parent = c.take<int>(interior);
    int* leaf_parent = c.take<int>(n);
    float4* node_lo = c.take<float4>(interior);
    float4* node_hi = c.take<float4>(interior);
    uint32_t* arrivals = c.take<uint32_t>(interior);
    uint32_t* depth = c.take<uint32_t>(1);
    double* sah = c.take<double>(1);
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys, keys_sorted, vals, order, (int)n, 0, 63, s);
    unsigned char* sort_tmp = c.take<unsigned char>(sort_bytes);
    if (!c.fits()) {
        set_error("scene too large for the no-alloc scratch (64 MiB, about 300k triangles)");
        return NAN_ERR_LIMIT;
    }

    // Previous calls leave their contents behind: clear what must start at zero.
    Bounds init;
    for (int a = 0; a < 3; ++a) {
        init.lo[a] = 0xffffffffu;
        init.hi[a] = 0u;
    }
    init.max_abs = 0u;
    err = cudaMemcpyAsync(bounds, &init, sizeof(Bounds), cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess) err = cudaMemsetAsync(arrivals, 0, std::max<uint32_t>(interior, 1) * sizeof(uint32_t), s);
    if (err == cudaSuccess) err = cudaMemsetAsync(depth, 0, sizeof(uint32_t), s);
    if (err == cudaSuccess) err = cudaMemsetAsync(sah, 0, sizeof(double), s);
    if (err != cudaSuccess) return cuda_fail(err, "no-alloc scene build (scratch clear)");

    forget_bvh();
    ctx->scene = *sd;
    ctx->caller_owned_bvh = true;
    ctx->nodes = reinterpret_cast<float4*>(out_nodes);
    ctx->tris = reinterpret_cast<float4*>(out_tris);
    ctx->tri_refs = reinterpret_cast<uint2*>(out_refs);
    ctx->tri_count = n;
    ctx->device_bytes = 0;

    k_flatten<<<blocks(n), kThreads, 0, s>>>(*sd, offsets, n, tris_flat, ctx->tri_refs, lo_flat, hi_flat, bounds);
    k_morton<<<blocks(n), kThreads, 0, s>>>(lo_flat, hi_flat, n, bounds, keys, vals);
    cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, keys, keys_sorted, vals, order, (int)n, 0, 63, s);
    k_gather_leaves<<<blocks(n), kThreads, 0, s>>>(order, n, tris_flat, lo_flat, hi_flat, ctx->tris, leaf_lo, leaf_hi);
    ctx->launches += 4;
    uint32_t max_depth = 1;
    double sah_host = 1.0;
    if (n == 1) {
        ctx->root = ~0;
        ctx->node_count = 0;
    } else {
        k_hierarchy<<<blocks(interior), kThreads, 0, s>>>(keys_sorted, (int)n, children, node_parent, leaf_parent);
        k_refit<<<blocks(n), kThreads, 0, s>>>(n, children, node_parent, leaf_parent, leaf_lo, leaf_hi, node_lo,
                                               node_hi, arrivals);
        k_depth<<<blocks(n), kThreads, 0, s>>>(n, node_parent, leaf_parent, depth);
        k_emit<<<blocks(interior), kThreads, 0, s>>>(interior, children, node_lo, node_hi, leaf_lo, leaf_hi, bounds,
                                                     ctx->nodes, sah);
        ctx->launches += 4;
        ctx->root = 0;
        ctx->node_count = interior;
        err = cudaMemcpyAsync(&max_depth, depth, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaMemcpyAsync(&sah_host, sah, sizeof(double), cudaMemcpyDeviceToHost, s);
        if (err != cudaSuccess) {
            forget_bvh();
            return cuda_fail(err, "no-alloc scene build (depth and SAH readback)");
        }
    }
    err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) {
        forget_bvh();
        return cuda_fail(err, "no-alloc scene build");
    }
    ctx->leaf_count = n;
    ctx->max_depth = max_depth;
    ctx->sah_cost = sah_host;
    ctx->build_ms = 0.0;
    if (ctx->max_depth > 96u) {
        forget_bvh();
        set_error("BVH deeper than the traversal stack (96)");
        return NAN_ERR_LIMIT;
    }
    ctx->has_scene = true;
    return NAN_OK;
}
