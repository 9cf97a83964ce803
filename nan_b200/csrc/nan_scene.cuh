// nan_scene.cuh -- device view of a built scene: BVH traversal, shading data,
// spawn offsets and lights. Included by translation units compiled with
// --fmad=false (see nan_math.cuh).
#pragma once

#include <cstdint>

#include "nan_math.cuh"

namespace nbd {

constexpr int kTraversalStack = 96;
constexpr uint32_t kStatusStackOverflow = 1u;

// Binary BVH node, 64 bytes: both children's boxes live in the parent so one
// node fetch tests two boxes.
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   d = (child0, child1, -, -): child >= 0 is an interior node; child < 0 a
//       leaf of triangles [first, first + count) in leaf order, encoded as
//       ~(first << 3 | (count - 1)) (1..8 triangles).
// Triangles in leaf order: 3 float4 each, (v0, flat index bits), (v1, 0),
// (v2, 0), world space.
struct SceneView {
    const float4* nodes;
    const float4* tris;
    const uint4* wnodes;            // compressed 8-wide nodes (null: use the binary nodes)
    const float4* wtris;            // triangles in the wide leaf order
    const uint2* tri_refs;          // flat index -> (instance, primitive)
    const float* vertices;          // f32[V][8]
    const uint32_t* indices;        // u32[T][3]
    const uint4* mesh_descs;
    const uint4* instance_descs;
    const float* transforms;        // f32[X][16]
    const float* inverse_transposes;
    const float* materials;         // f32[N][8]
    int root;
    uint32_t tri_count;
    uint32_t instance_count;
    uint32_t* status;               // device status word
    // emissive triangles for area-light NEE (4 float4 each: v0 + cdf, e1 + area,
    // e2 + luminance, emission); null when none were given
    const float4* lights;
    uint32_t light_count;
    float light_power;              // sum of area * luminance
};

constexpr uint32_t kStatusBadRecord = 4u;

// True when (instance, primitive) names a triangle of the scene; records that
// do not are skipped by the kernels and flagged in the status word.
__device__ __forceinline__ bool valid_prim(const SceneView& s, uint32_t inst, uint32_t prim) {
    if (inst >= s.instance_count) return false;
    const uint4 idesc = __ldg(s.instance_descs + inst);
    const uint4 mdesc = __ldg(s.mesh_descs + idesc.x);
    return prim < mdesc.y / 3u;
}

struct HitInfo {
    bool valid;
    uint32_t flat;
    float t;
    float b1, b2;  // weights of v1 and v2 (Slang HitInfo.bary)
};

// Per-ray constants of the watertight test (Woop, Benthin, Wald 2013).
struct WtRay {
    int kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ WtRay wt_setup(f3 d) {
    WtRay r;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0;
    float m = ax;
    if (ay > m) { kz = 1; m = ay; }
    if (az > m) kz = 2;
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    const float dz = comp(d, kz);
    if (dz < 0.0f) { int t = kx; kx = ky; ky = t; }
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.sx = comp(d, kx) / dz;
    r.sy = comp(d, ky) / dz;
    r.sz = 1.0f / dz;
    return r;
}

// Edge functions and scaled distance; returns false when the ray misses the
// closed triangle or the triangle is degenerate along the ray.
__device__ __forceinline__ bool wt_test(const WtRay& r, f3 o, f3 v0, f3 v1, f3 v2, float* t,
                                        float* out_v, float* out_w, float* out_det) {
    const f3 A = v0 - o, B = v1 - o, C = v2 - o;
    const float akz = comp(A, r.kz), bkz = comp(B, r.kz), ckz = comp(C, r.kz);
    const float ax = comp(A, r.kx) - r.sx * akz;
    const float ay = comp(A, r.ky) - r.sy * akz;
    const float bx = comp(B, r.kx) - r.sx * bkz;
    const float by = comp(B, r.ky) - r.sy * bkz;
    const float cx = comp(C, r.kx) - r.sx * ckz;
    const float cy = comp(C, r.ky) - r.sy * ckz;
    float U = cx * by - cy * bx;
    float V = ax * cy - ay * cx;
    float W = bx * ay - by * ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)cx * (double)by - (double)cy * (double)bx);
        V = (float)((double)ax * (double)cy - (double)ay * (double)cx);
        W = (float)((double)bx * (double)ay - (double)by * (double)ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = (U + V) + W;
    if (det == 0.0f) return false;
    const float tt = (U * (r.sz * akz) + V * (r.sz * bkz)) + W * (r.sz * ckz);
    *t = tt / det;
    *out_v = V;
    *out_w = W;
    *out_det = det;
    return true;
}

__device__ __forceinline__ void load_tri(const SceneView& s, int i, f3* v0, f3* v1, f3* v2, uint32_t* flat) {
    const float4 a = __ldg(s.tris + 3 * i);
    const float4 b = __ldg(s.tris + 3 * i + 1);
    const float4 c = __ldg(s.tris + 3 * i + 2);
    *v0 = mk3(a.x, a.y, a.z);
    *v1 = mk3(b.x, b.y, b.z);
    *v2 = mk3(c.x, c.y, c.z);
    *flat = __float_as_uint(a.w);
}

// Slab test of both children of a node. Node boxes are padded outward at
// build time by more than the rounding of the fused slab arithmetic, so the
// test never rejects a box the exact ray crosses.
struct BoxRay {
    float ix, iy, iz, ox, oy, oz;
};

__device__ __forceinline__ BoxRay box_setup(f3 o, f3 d) {
    BoxRay b;
    const float e = 1e-20f;
    b.ix = 1.0f / (fabsf(d.x) > e ? d.x : copysignf(e, d.x));
    b.iy = 1.0f / (fabsf(d.y) > e ? d.y : copysignf(e, d.y));
    b.iz = 1.0f / (fabsf(d.z) > e ? d.z : copysignf(e, d.z));
    b.ox = o.x * b.ix;
    b.oy = o.y * b.iy;
    b.oz = o.z * b.iz;
    return b;
}

// Three-input float min / max (PTX min.f32 / max.f32 with three sources,
// sm_100 and later). Both are exact, so any grouping gives the same value.
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

__device__ __forceinline__ void box2(const BoxRay& r, float4 na, float4 nb, float4 nc, float tmin, float tmax,
                                     float* t0, float* t1, bool* h0, bool* h1) {
    const float x0a = __fmaf_rn(na.x, r.ix, -r.ox), x0b = __fmaf_rn(na.y, r.ix, -r.ox);
    const float y0a = __fmaf_rn(na.z, r.iy, -r.oy), y0b = __fmaf_rn(na.w, r.iy, -r.oy);
    const float z0a = __fmaf_rn(nc.x, r.iz, -r.oz), z0b = __fmaf_rn(nc.y, r.iz, -r.oz);
    const float x1a = __fmaf_rn(nb.x, r.ix, -r.ox), x1b = __fmaf_rn(nb.y, r.ix, -r.ox);
    const float y1a = __fmaf_rn(nb.z, r.iy, -r.oy), y1b = __fmaf_rn(nb.w, r.iy, -r.oy);
    const float z1a = __fmaf_rn(nc.z, r.iz, -r.oz), z1b = __fmaf_rn(nc.w, r.iz, -r.oz);
    const float lo0 = max3f(fminf(x0a, x0b), fminf(y0a, y0b), fmaxf(fminf(z0a, z0b), tmin));
    const float hi0 = min3f(fmaxf(x0a, x0b), fmaxf(y0a, y0b), fminf(fmaxf(z0a, z0b), tmax));
    const float lo1 = max3f(fminf(x1a, x1b), fminf(y1a, y1b), fmaxf(fminf(z1a, z1b), tmin));
    const float hi1 = min3f(fmaxf(x1a, x1b), fmaxf(y1a, y1b), fminf(fmaxf(z1a, z1b), tmax));
    *t0 = lo0;
    *t1 = lo1;
    *h0 = lo0 <= hi0;
    *h1 = lo1 <= hi1;
}


// ---------------------------------------------------------------------------
// Compressed 8-wide traversal (node format in nan_bvh.cu). A group is
// (first child index, interior-slot mask, remaining children as bits at
// position slot ^ octant); popping the lowest bit visits the children of a
// node roughly front to back for the ray's direction octant.
// ---------------------------------------------------------------------------
constexpr int kWideStack = 64;

struct WideRay {
    f3 o;
    float ix, iy, iz;
    uint32_t oct;
};

__device__ __forceinline__ WideRay wide_setup(f3 o, f3 d) {
    WideRay r;
    const float e = 1e-20f;
    r.o = o;
    r.ix = 1.0f / (fabsf(d.x) > e ? d.x : copysignf(e, d.x));
    r.iy = 1.0f / (fabsf(d.y) > e ? d.y : copysignf(e, d.y));
    r.iz = 1.0f / (fabsf(d.z) > e ? d.z : copysignf(e, d.z));
    r.oct = (r.ix < 0.0f ? 1u : 0u) | (r.iy < 0.0f ? 2u : 0u) | (r.iz < 0.0f ? 4u : 0u);
    return r;
}

// Slot bits of m reordered by the ray's octant (bit i moves to i ^ oct), by
// selects: oct is fixed per ray but differs between the lanes of a warp.
__device__ __forceinline__ uint32_t octant_permute(uint32_t m, uint32_t oct) {
    m = (oct & 1u) ? (((m & 0x55u) << 1) | ((m & 0xaau) >> 1)) : m;
    m = (oct & 2u) ? (((m & 0x33u) << 2) | ((m & 0xccu) >> 2)) : m;
    m = (oct & 4u) ? (((m & 0x0fu) << 4) | ((m & 0xf0u) >> 4)) : m;
    return m;
}

// Slots of the node whose (conservatively dequantized) boxes the ray enters
// within [tmin, tmax].
__device__ __forceinline__ uint32_t wide_hits(const WideRay& r, uint4 w0, uint4 w2, uint4 w3, uint4 w4, float tmin,
                                              float tmax) {
    const uint32_t eb = w0.w;
    const float sx = __uint_as_float((eb & 0xffu) << 23);
    const float sy = __uint_as_float(((eb >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((eb >> 16) & 0xffu) << 23);
    const float ax = sx * r.ix, ay = sy * r.iy, az = sz * r.iz;
    const float bx = (__uint_as_float(w0.x) - r.o.x) * r.ix;
    const float by = (__uint_as_float(w0.y) - r.o.y) * r.iy;
    const float bz = (__uint_as_float(w0.z) - r.o.z) * r.iz;
    // near / far planes by direction sign: qlo.x = w2.xy, qlo.y = w2.zw,
    // qlo.z = w3.xy, qhi.x = w3.zw, qhi.y = w4.xy, qhi.z = w4.zw
    const bool nx = r.ix >= 0.0f, ny = r.iy >= 0.0f, nz = r.iz >= 0.0f;
    const uint32_t nxa = nx ? w2.x : w3.z, nxb = nx ? w2.y : w3.w, fxa = nx ? w3.z : w2.x, fxb = nx ? w3.w : w2.y;
    const uint32_t nya = ny ? w2.z : w4.x, nyb = ny ? w2.w : w4.y, fya = ny ? w4.x : w2.z, fyb = ny ? w4.y : w2.w;
    const uint32_t nza = nz ? w3.x : w4.z, nzb = nz ? w3.y : w4.w, fza = nz ? w4.z : w3.x, fzb = nz ? w4.w : w3.y;
    uint32_t hits = 0u;
#pragma unroll
    for (int sl = 0; sl < 8; ++sl) {
        const int sh = (sl & 3) * 8;
        const uint32_t qnx = ((sl < 4 ? nxa : nxb) >> sh) & 0xffu, qfx = ((sl < 4 ? fxa : fxb) >> sh) & 0xffu;
        const uint32_t qny = ((sl < 4 ? nya : nyb) >> sh) & 0xffu, qfy = ((sl < 4 ? fya : fyb) >> sh) & 0xffu;
        const uint32_t qnz = ((sl < 4 ? nza : nzb) >> sh) & 0xffu, qfz = ((sl < 4 ? fza : fzb) >> sh) & 0xffu;
        const float tn = fmaxf(fmaxf(__fmaf_rn((float)qnx, ax, bx), __fmaf_rn((float)qny, ay, by)),
                               fmaxf(__fmaf_rn((float)qnz, az, bz), tmin));
        const float tf = fminf(fminf(__fmaf_rn((float)qfx, ax, bx), __fmaf_rn((float)qfy, ay, by)),
                               fminf(__fmaf_rn((float)qfz, az, bz), tmax));
        if (tn <= tf) hits |= 1u << sl;
    }
    return hits;
}

__device__ __forceinline__ void load_wtri(const SceneView& s, uint32_t i, f3* v0, f3* v1, f3* v2, uint32_t* flat) {
    const float4 a = __ldg(s.wtris + 3u * i);
    const float4 b = __ldg(s.wtris + 3u * i + 1u);
    const float4 c = __ldg(s.wtris + 3u * i + 2u);
    *v0 = mk3(a.x, a.y, a.z);
    *v1 = mk3(b.x, b.y, b.z);
    *v2 = mk3(c.x, c.y, c.z);
    *flat = __float_as_uint(a.w);
}

template <bool kAnyHit>
__device__ __forceinline__ bool trace_wide(const SceneView& s, f3 o, f3 d, float tmin, float tmax, HitInfo* hit) {
    const WtRay wr = wt_setup(d);
    const WideRay r = wide_setup(o, d);
    uint2 stack[kWideStack];
    int sp = 0;
    uint32_t g_base = 0u, g_imask = 1u, g_mask = 1u << r.oct;  // the root as slot 0 of a virtual group
    float best_t = tmax;
    uint32_t best_key = 0xffffffffu, best_tri = 0xffffffffu;
    bool overflow = false;
    for (;;) {
        if (g_mask == 0u) {
            if (sp == 0) break;
            const uint2 e = stack[--sp];
            g_base = e.x;
            g_imask = e.y >> 8;
            g_mask = e.y & 0xffu;
            continue;
        }
        const uint32_t pos = (uint32_t)__ffs(g_mask) - 1u;
        g_mask &= g_mask - 1u;
        const uint32_t slot = pos ^ r.oct;
        const uint32_t child = g_base + (uint32_t)__popc(g_imask & ((1u << slot) - 1u));
        const bool push = g_mask != 0u && sp < kWideStack;
        overflow |= g_mask != 0u && sp >= kWideStack;
        if (push) stack[sp] = make_uint2(g_base, (g_imask << 8) | g_mask);
        sp += push ? 1 : 0;
        const uint4* w = s.wnodes + 5u * child;
        const uint4 w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2), w3 = __ldg(w + 3), w4 = __ldg(w + 4);
        const uint32_t imask = w0.w >> 24;
        const uint32_t hits = wide_hits(r, w0, w2, w3, w4, tmin, kAnyHit ? tmax : best_t);
        uint32_t leaf_hits = hits & ~imask;
        while (leaf_hits != 0u) {
            const uint32_t sl = (uint32_t)__ffs(leaf_hits) - 1u;
            leaf_hits &= leaf_hits - 1u;
            const uint32_t meta = ((sl < 4u ? w1.z : w1.w) >> ((sl & 3u) * 8u)) & 0xffu;
            if (meta == 0u) continue;
            const uint32_t first = w1.y + (meta & 31u);
            const uint32_t cnt = (uint32_t)__popc(meta >> 5);
            for (uint32_t k = 0; k < cnt; ++k) {
                f3 v0, v1, v2;
                uint32_t flat;
                load_wtri(s, first + k, &v0, &v1, &v2, &flat);
                float t, V, W, det;
                if (wt_test(wr, o, v0, v1, v2, &t, &V, &W, &det) && t >= tmin) {
                    if (kAnyHit) {
                        if (t <= tmax) {
                            if (overflow) atomicOr(s.status, kStatusStackOverflow);
                            return true;
                        }
                    } else if (t < best_t || (t == best_t && flat < best_key)) {
                        best_t = t;
                        best_key = flat;
                        best_tri = first + k;
                    }
                }
            }
        }
        g_base = w1.x;
        g_imask = imask;
        g_mask = octant_permute(hits & imask, r.oct);
    }
    if (overflow) atomicOr(s.status, kStatusStackOverflow);
    if (kAnyHit) return false;
    if (best_tri != 0xffffffffu) {
        f3 v0, v1, v2;
        uint32_t flat;
        load_wtri(s, best_tri, &v0, &v1, &v2, &flat);
        float t, V, W, det;
        wt_test(wr, o, v0, v1, v2, &t, &V, &W, &det);
        hit->valid = true;
        hit->flat = best_key;
        hit->t = best_t;
        hit->b1 = V / det;
        hit->b2 = W / det;
        return true;
    }
    return false;
}

// Traversal stacks. LocalStack: the whole stack in the thread's local
// memory. SplitStack: the first kShared entries in a shared-memory column of
// the thread (entry k at top[k * kStride]), the rest in local memory.
template <int kDepth>
struct LocalStack {
    int a[kDepth];
    __device__ __forceinline__ void put(int i, int v) { a[i] = v; }
    __device__ __forceinline__ int get(int i) const { return a[i]; }
};

template <int kShared, int kStride, int kDepth>
struct SplitStack {
    int* top;
    int spill[kDepth - kShared];
    __device__ __forceinline__ void put(int i, int v) {
        if (i < kShared) top[i * kStride] = v;
        else spill[i - kShared] = v;
    }
    __device__ __forceinline__ int get(int i) const { return i < kShared ? top[i * kStride] : spill[i - kShared]; }
};

// Closest hit in [tmin, tmax]; ties in t go to the lower flat triangle index
// (lexicographic (instance, primitive)), so the result does not depend on
// the traversal order. Binary-node traversal.
template <int kDepth, class Stk>
__device__ __forceinline__ HitInfo trace_closest_binary_s(const SceneView& s, Stk& stack, f3 o, f3 d, float tmin,
                                                          float tmax) {
    HitInfo hit;
    hit.valid = false;
    hit.flat = 0xffffffffu;
    hit.t = tmax;
    hit.b1 = 0.0f;
    hit.b2 = 0.0f;
    if (s.tri_count == 0) return hit;
    const WtRay wr = wt_setup(d);
    const BoxRay br = box_setup(o, d);
    int sp = 0;
    int node = s.root;
    float best_t = tmax;
    uint32_t best_key = 0xffffffffu;
    int best_tri = -1;
    bool overflow = false;
    for (;;) {
        if (node >= 0) {
            const float4* n = s.nodes + 4 * node;
            const float4 na = __ldg(n), nb = __ldg(n + 1), nc = __ldg(n + 2);
            const int4 nd = __ldg(reinterpret_cast<const int4*>(n + 3));
            float t0, t1;
            bool h0, h1;
            box2(br, na, nb, nc, tmin, best_t, &t0, &t1, &h0, &h1);
            if (h0 || h1) {
                // near child first; the far one is pushed when both are hit
                // (selects and a predicated push: one branch per node)
                const bool both = h0 && h1, swap = both && t1 < t0;
                const bool push = both && sp < kDepth;
                overflow |= both && sp >= kDepth;
                if (push) stack.put(sp, swap ? nd.x : nd.y);
                sp += push ? 1 : 0;
                node = (h0 && !swap) ? nd.x : nd.y;
                continue;
            }
        } else {
            const int leaf = ~node;
            const int first = leaf >> 3, last = first + (leaf & 7);
            for (int tri = first; tri <= last; ++tri) {
                f3 v0, v1, v2;
                uint32_t flat;
                load_tri(s, tri, &v0, &v1, &v2, &flat);
                float t, V, W, det;
                if (wt_test(wr, o, v0, v1, v2, &t, &V, &W, &det) && t >= tmin &&
                    (t < best_t || (t == best_t && flat < best_key))) {
                    best_t = t;
                    best_key = flat;
                    best_tri = tri;
                }
            }
        }
        if (sp == 0) break;
        node = stack.get(--sp);
    }
    if (overflow) atomicOr(s.status, kStatusStackOverflow);
    if (best_tri >= 0) {
        f3 v0, v1, v2;
        uint32_t flat;
        load_tri(s, best_tri, &v0, &v1, &v2, &flat);
        float t, V, W, det;
        wt_test(wr, o, v0, v1, v2, &t, &V, &W, &det);
        hit.valid = true;
        hit.flat = best_key;
        hit.t = best_t;
        hit.b1 = V / det;
        hit.b2 = W / det;
    }
    return hit;
}

template <int kDepth = kTraversalStack>
__device__ __forceinline__ HitInfo trace_closest_binary(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
    LocalStack<kDepth> stack;
    return trace_closest_binary_s<kDepth>(s, stack, o, d, tmin, tmax);
}

// Any hit in [tmin, tmax]. Binary-node traversal.
template <int kDepth, class Stk>
__device__ __forceinline__ bool trace_any_binary_s(const SceneView& s, Stk& stack, f3 o, f3 d, float tmin, float tmax) {
    if (s.tri_count == 0) return false;
    const WtRay wr = wt_setup(d);
    const BoxRay br = box_setup(o, d);
    int sp = 0;
    int node = s.root;
    bool overflow = false, blocked = false;
    for (;;) {
        if (node >= 0) {
            const float4* n = s.nodes + 4 * node;
            const float4 na = __ldg(n), nb = __ldg(n + 1), nc = __ldg(n + 2);
            const int4 nd = __ldg(reinterpret_cast<const int4*>(n + 3));
            float t0, t1;
            bool h0, h1;
            box2(br, na, nb, nc, tmin, tmax, &t0, &t1, &h0, &h1);
            if (h0 || h1) {
                const bool both = h0 && h1, swap = both && t1 < t0;
                const bool push = both && sp < kDepth;
                overflow |= both && sp >= kDepth;
                if (push) stack.put(sp, swap ? nd.x : nd.y);
                sp += push ? 1 : 0;
                node = (h0 && !swap) ? nd.x : nd.y;
                continue;
            }
        } else {
            const int leaf = ~node;
            const int first = leaf >> 3, last = first + (leaf & 7);
            for (int tri = first; tri <= last; ++tri) {
                f3 v0, v1, v2;
                uint32_t flat;
                load_tri(s, tri, &v0, &v1, &v2, &flat);
                float t, V, W, det;
                if (wt_test(wr, o, v0, v1, v2, &t, &V, &W, &det) && t >= tmin && t <= tmax) {
                    blocked = true;
                    break;
                }
            }
            if (blocked) break;
        }
        if (sp == 0) break;
        node = stack.get(--sp);
    }
    if (overflow) atomicOr(s.status, kStatusStackOverflow);
    return blocked;
}

template <int kDepth = kTraversalStack>
__device__ __forceinline__ bool trace_any_binary(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
    LocalStack<kDepth> stack;
    return trace_any_binary_s<kDepth>(s, stack, o, d, tmin, tmax);
}

// ---------------------------------------------------------------------------
// Speculative while-while walks (after Aila and Laine, "Understanding the
// efficiency of ray traversal on GPUs", HPG 2009). A lane that reaches a leaf
// parks it and keeps descending; once every lane still descending holds a
// parked leaf, the lanes test their leaves together. Leaf tests then run
// with more lanes active, at the price of some speculative node visits. The
// closest hit does not depend on the visit order (the (t, flat) tie-break),
// and an any-hit query answers the same either way.
// kWalkDone marks an ended walk: a leaf is ~(first << 3 | last - first)
// with at most 8 triangles, so no leaf encodes to it.
// ---------------------------------------------------------------------------
constexpr int kWalkDone = -2147483647 - 1;

template <int kDepth>
__device__ __forceinline__ int spec_pop(const int* stack, int& sp) {
    return sp ? stack[--sp] : kWalkDone;
}

// One interior node of a binary walk: the next node (near child, the other
// hit child, or a popped entry), pushing the far child when both are hit.
template <int kDepth>
__device__ __forceinline__ int spec_interior(const SceneView& s, const BoxRay& br, int node, float tmin, float tmax,
                                             int* stack, int& sp) {
    const float4* n = s.nodes + 4 * node;
    const float4 na = __ldg(n), nb = __ldg(n + 1), nc = __ldg(n + 2);
    const int4 nd = __ldg(reinterpret_cast<const int4*>(n + 3));
    float t0, t1;
    bool h0, h1;
    box2(br, na, nb, nc, tmin, tmax, &t0, &t1, &h0, &h1);
    if (h0 && h1) {
        int near_child = nd.x, far_child = nd.y;
        if (t1 < t0) { near_child = nd.y; far_child = nd.x; }
        if (sp < kDepth) stack[sp++] = far_child;
        else atomicOr(s.status, kStatusStackOverflow);
        return near_child;
    }
    if (h0) return nd.x;
    if (h1) return nd.y;
    return spec_pop<kDepth>(stack, sp);
}

template <int kDepth = kTraversalStack>
__device__ __forceinline__ HitInfo trace_closest_binary_spec(const SceneView& s, f3 o, f3 d, float tmin,
                                                             float tmax) {
    HitInfo hit;
    hit.valid = false;
    hit.flat = 0xffffffffu;
    hit.t = tmax;
    hit.b1 = 0.0f;
    hit.b2 = 0.0f;
    if (s.tri_count == 0) return hit;
    const WtRay wr = wt_setup(d);
    const BoxRay br = box_setup(o, d);
    int stack[kDepth];
    int sp = 0;
    int node = s.root;
    int leaf = 0;  // the parked leaf (< 0), or 0
    float best_t = tmax;
    uint32_t best_key = 0xffffffffu;
    int best_tri = -1;
    while (node != kWalkDone) {
        while (node >= 0) {
            node = spec_interior<kDepth>(s, br, node, tmin, best_t, stack, sp);
            if (node < 0 && node != kWalkDone && leaf == 0) {
                leaf = node;
                node = spec_pop<kDepth>(stack, sp);
            }
            if (!__any_sync(__activemask(), leaf == 0)) break;
        }
        if (leaf == 0 && node < 0 && node != kWalkDone) {
            leaf = node;
            node = spec_pop<kDepth>(stack, sp);
        }
        while (leaf < 0) {
            const int l = ~leaf;
            const int first = l >> 3, last = first + (l & 7);
            for (int tri = first; tri <= last; ++tri) {
                f3 v0, v1, v2;
                uint32_t flat;
                load_tri(s, tri, &v0, &v1, &v2, &flat);
                float t, V, W, det;
                if (wt_test(wr, o, v0, v1, v2, &t, &V, &W, &det) && t >= tmin &&
                    (t < best_t || (t == best_t && flat < best_key))) {
                    best_t = t;
                    best_key = flat;
                    best_tri = tri;
                }
            }
            leaf = 0;
            if (node < 0 && node != kWalkDone) {
                leaf = node;
                node = spec_pop<kDepth>(stack, sp);
            }
        }
    }
    if (best_tri >= 0) {
        f3 v0, v1, v2;
        uint32_t flat;
        load_tri(s, best_tri, &v0, &v1, &v2, &flat);
        float t, V, W, det;
        wt_test(wr, o, v0, v1, v2, &t, &V, &W, &det);
        hit.valid = true;
        hit.flat = best_key;
        hit.t = best_t;
        hit.b1 = V / det;
        hit.b2 = W / det;
    }
    return hit;
}

template <int kDepth = kTraversalStack>
__device__ __forceinline__ bool trace_any_binary_spec(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
    if (s.tri_count == 0) return false;
    const WtRay wr = wt_setup(d);
    const BoxRay br = box_setup(o, d);
    int stack[kDepth];
    int sp = 0;
    int node = s.root;
    int leaf = 0;
    while (node != kWalkDone) {
        while (node >= 0) {
            node = spec_interior<kDepth>(s, br, node, tmin, tmax, stack, sp);
            if (node < 0 && node != kWalkDone && leaf == 0) {
                leaf = node;
                node = spec_pop<kDepth>(stack, sp);
            }
            if (!__any_sync(__activemask(), leaf == 0)) break;
        }
        if (leaf == 0 && node < 0 && node != kWalkDone) {
            leaf = node;
            node = spec_pop<kDepth>(stack, sp);
        }
        while (leaf < 0) {
            const int l = ~leaf;
            const int first = l >> 3, last = first + (l & 7);
            for (int tri = first; tri <= last; ++tri) {
                f3 v0, v1, v2;
                uint32_t flat;
                load_tri(s, tri, &v0, &v1, &v2, &flat);
                float t, V, W, det;
                if (wt_test(wr, o, v0, v1, v2, &t, &V, &W, &det) && t >= tmin && t <= tmax) return true;
            }
            leaf = 0;
            if (node < 0 && node != kWalkDone) {
                leaf = node;
                node = spec_pop<kDepth>(stack, sp);
            }
        }
    }
    return false;
}

// ---------------------------------------------------------------------------
// Resumable binary walks: the state of trace_closest_binary /
// trace_any_binary between steps, so that a persistent kernel can advance a
// lane's ray one node (or leaf) at a time and hand a lane whose ray has ended
// a new one while the other lanes keep walking. A step does exactly what one
// pass of the per-lane loop does, so the hit is the same.
// ---------------------------------------------------------------------------
struct ClosestWalk {
    WtRay wr;
    BoxRay br;
    f3 o;
    float tmin;
    float best_t;
    uint32_t best_key;
    int best_tri;
    int node;
    int sp;
};

// False when there is nothing to walk (empty scene).
__device__ __forceinline__ bool closest_begin(const SceneView& s, ClosestWalk& w, f3 o, f3 d, float tmin, float tmax) {
    w.wr = wt_setup(d);
    w.br = box_setup(o, d);
    w.o = o;
    w.tmin = tmin;
    w.best_t = tmax;
    w.best_key = 0xffffffffu;
    w.best_tri = -1;
    w.node = s.root;
    w.sp = 0;
    return s.tri_count != 0;
}

// One node or leaf; false once the walk has ended.
template <int kDepth>
__device__ __forceinline__ bool closest_step(const SceneView& s, ClosestWalk& w, int* stack) {
    if (w.node >= 0) {
        const float4* n = s.nodes + 4 * w.node;
        const float4 na = __ldg(n), nb = __ldg(n + 1), nc = __ldg(n + 2);
        const int4 nd = __ldg(reinterpret_cast<const int4*>(n + 3));
        float t0, t1;
        bool h0, h1;
        box2(w.br, na, nb, nc, w.tmin, w.best_t, &t0, &t1, &h0, &h1);
        if (h0 && h1) {
            int near_child = nd.x, far_child = nd.y;
            if (t1 < t0) { near_child = nd.y; far_child = nd.x; }
            if (w.sp < kDepth) stack[w.sp++] = far_child;
            else atomicOr(s.status, kStatusStackOverflow);
            w.node = near_child;
            return true;
        }
        if (h0) { w.node = nd.x; return true; }
        if (h1) { w.node = nd.y; return true; }
    } else {
        const int leaf = ~w.node;
        const int first = leaf >> 3, last = first + (leaf & 7);
        for (int tri = first; tri <= last; ++tri) {
            f3 v0, v1, v2;
            uint32_t flat;
            load_tri(s, tri, &v0, &v1, &v2, &flat);
            float t, V, W, det;
            if (wt_test(w.wr, w.o, v0, v1, v2, &t, &V, &W, &det) && t >= w.tmin &&
                (t < w.best_t || (t == w.best_t && flat < w.best_key))) {
                w.best_t = t;
                w.best_key = flat;
                w.best_tri = tri;
            }
        }
    }
    if (w.sp == 0) return false;
    w.node = stack[--w.sp];
    return true;
}

__device__ __forceinline__ HitInfo closest_end(const SceneView& s, const ClosestWalk& w) {
    HitInfo hit;
    hit.valid = false;
    hit.flat = 0xffffffffu;
    hit.t = w.best_t;
    hit.b1 = 0.0f;
    hit.b2 = 0.0f;
    if (w.best_tri >= 0) {
        f3 v0, v1, v2;
        uint32_t flat;
        load_tri(s, w.best_tri, &v0, &v1, &v2, &flat);
        float t, V, W, det;
        wt_test(w.wr, w.o, v0, v1, v2, &t, &V, &W, &det);
        hit.valid = true;
        hit.flat = w.best_key;
        hit.b1 = V / det;
        hit.b2 = W / det;
    }
    return hit;
}

struct AnyWalk {
    WtRay wr;
    BoxRay br;
    f3 o;
    float tmin;
    float tmax;
    int node;
    int sp;
};

__device__ __forceinline__ bool any_begin(const SceneView& s, AnyWalk& w, f3 o, f3 d, float tmin, float tmax) {
    w.wr = wt_setup(d);
    w.br = box_setup(o, d);
    w.o = o;
    w.tmin = tmin;
    w.tmax = tmax;
    w.node = s.root;
    w.sp = 0;
    return s.tri_count != 0;
}

// One node or leaf: 0 = walk on, 1 = ended without a hit, 2 = hit.
template <int kDepth>
__device__ __forceinline__ int any_step(const SceneView& s, AnyWalk& w, int* stack) {
    if (w.node >= 0) {
        const float4* n = s.nodes + 4 * w.node;
        const float4 na = __ldg(n), nb = __ldg(n + 1), nc = __ldg(n + 2);
        const int4 nd = __ldg(reinterpret_cast<const int4*>(n + 3));
        float t0, t1;
        bool h0, h1;
        box2(w.br, na, nb, nc, w.tmin, w.tmax, &t0, &t1, &h0, &h1);
        if (h0 && h1) {
            int near_child = nd.x, far_child = nd.y;
            if (t1 < t0) { near_child = nd.y; far_child = nd.x; }
            if (w.sp < kDepth) stack[w.sp++] = far_child;
            else atomicOr(s.status, kStatusStackOverflow);
            w.node = near_child;
            return 0;
        }
        if (h0) { w.node = nd.x; return 0; }
        if (h1) { w.node = nd.y; return 0; }
    } else {
        const int leaf = ~w.node;
        const int first = leaf >> 3, last = first + (leaf & 7);
        for (int tri = first; tri <= last; ++tri) {
            f3 v0, v1, v2;
            uint32_t flat;
            load_tri(s, tri, &v0, &v1, &v2, &flat);
            float t, V, W, det;
            if (wt_test(w.wr, w.o, v0, v1, v2, &t, &V, &W, &det) && t >= w.tmin && t <= w.tmax) return 2;
        }
    }
    if (w.sp == 0) return 1;
    w.node = stack[--w.sp];
    return 0;
}

// Width-specialised entry points (kWidth 2: binary nodes, 8: compressed
// wide nodes) and a run-time dispatch for kernels that are not specialised.
template <int kWidth>
__device__ __forceinline__ HitInfo trace_closest_w(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
    if (kWidth == 8) {
        HitInfo hit;
        hit.valid = false;
        hit.flat = 0xffffffffu;
        hit.t = tmax;
        hit.b1 = 0.0f;
        hit.b2 = 0.0f;
        if (s.tri_count != 0) trace_wide<false>(s, o, d, tmin, tmax, &hit);
        return hit;
    }
    return trace_closest_binary(s, o, d, tmin, tmax);
}

template <int kWidth>
__device__ __forceinline__ bool trace_any_w(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
    if (kWidth == 8) {
        HitInfo unused;
        return s.tri_count != 0 && trace_wide<true>(s, o, d, tmin, tmax, &unused);
    }
    return trace_any_binary(s, o, d, tmin, tmax);
}

__device__ __forceinline__ HitInfo trace_closest(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
    return s.wnodes ? trace_closest_w<8>(s, o, d, tmin, tmax) : trace_closest_w<2>(s, o, d, tmin, tmax);
}

__device__ __forceinline__ bool trace_any(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
    return s.wnodes ? trace_any_w<8>(s, o, d, tmin, tmax) : trace_any_w<2>(s, o, d, tmin, tmax);
}

// Traversal policies for code templated on the tracer: the run-time
// dispatch, or binary nodes with a fixed stack depth (a depth below the
// BVH's must not be chosen: the overflow is flagged and the push dropped).
struct DefaultTracer {
    __device__ static HitInfo closest(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
        return trace_closest(s, o, d, tmin, tmax);
    }
    __device__ static bool any(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
        return trace_any(s, o, d, tmin, tmax);
    }
};

template <int kDepth>
struct BinaryTracer {
    __device__ static HitInfo closest(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
        return trace_closest_binary<kDepth>(s, o, d, tmin, tmax);
    }
    __device__ static bool any(const SceneView& s, f3 o, f3 d, float tmin, float tmax) {
        return trace_any_binary<kDepth>(s, o, d, tmin, tmax);
    }
};

// ---------------------------------------------------------------------------
// Shading (scene.slang:178-406, opaque and untextured materials).
// ---------------------------------------------------------------------------
struct Shading {
    f3 position;
    f3 origin_front;
    float offset;
    f3 face_normal;
    f3 diffuse;
    f3 emissive;
    Frame frame;     // shading frame
    bool back_side;  // double-sided material seen from its back
};

struct TriRefs {
    const float* v0;
    const float* v1;
    const float* v2;
    const float* m;
    const float* it;
    const float* mat;
    uint32_t flags;
};

__device__ __forceinline__ TriRefs tri_refs(const SceneView& s, uint32_t inst, uint32_t prim) {
    const uint4 idesc = __ldg(s.instance_descs + inst);
    const uint4 mdesc = __ldg(s.mesh_descs + idesc.x);
    const uint32_t base = mdesc.w + prim * 3u;
    TriRefs r;
    r.v0 = s.vertices + 8u * (mdesc.z + __ldg(s.indices + base));
    r.v1 = s.vertices + 8u * (mdesc.z + __ldg(s.indices + base + 1));
    r.v2 = s.vertices + 8u * (mdesc.z + __ldg(s.indices + base + 2));
    r.m = s.transforms + 16u * idesc.z;
    r.it = s.inverse_transposes + 16u * idesc.z;
    r.mat = s.materials + 8u * idesc.y;
    r.flags = idesc.w;
    return r;
}

// get_triangle_spawn_data, scene.slang:178-269.
__device__ __forceinline__ void triangle_spawn(f3 v0, f3 v1, f3 v2, float bx, float by, const float* m,
                                               const float* it, f3* pos, f3* nrm, float* off) {
    const float c0 = 5.9604644775390625e-8f;
    const float c1 = 1.7881397695873602e-7f;
    const float c2 = 1.1920931797249068e-7f;
    float M[12], I[16];
#pragma unroll
    for (int k = 0; k < 12; ++k) M[k] = __ldg(m + k);
#pragma unroll
    for (int k = 0; k < 16; ++k) I[k] = __ldg(it + k);
    const f3 e1 = v1 - v0, e2 = v2 - v0;
    const f3 op = mk3(v0.x + __fmaf_rn(bx, e1.x, by * e2.x), v0.y + __fmaf_rn(bx, e1.y, by * e2.y),
                      v0.z + __fmaf_rn(bx, e1.z, by * e2.z));
    const f3 on = cross3(e1, e2);
    f3 wp;
    wp.x = M[3] + __fmaf_rn(M[0], op.x, __fmaf_rn(M[1], op.y, M[2] * op.z));
    wp.y = M[7] + __fmaf_rn(M[4], op.x, __fmaf_rn(M[5], op.y, M[6] * op.z));
    wp.z = M[11] + __fmaf_rn(M[8], op.x, __fmaf_rn(M[9], op.y, M[10] * op.z));
    const f3 wnu = mk3((I[0] * on.x + I[1] * on.y) + I[2] * on.z, (I[4] * on.x + I[5] * on.y) + I[6] * on.z,
                       (I[8] * on.x + I[9] * on.y) + I[10] * on.z);
    const float ws = 1.0f / sqrtf(maxf(dot3(wnu, wnu), 1e-30f));
    const f3 wn = wnu * ws;
    const f3 ext3 = (abs3(e1) + abs3(e2)) + abs3(abs3(e1) - abs3(e2));
    const float ext = maxf(maxf(ext3.x, ext3.y), ext3.z);
    const f3 av0 = abs3(v0);
    f3 oe = mk3(c0 * av0.x + c1 * ext, c0 * av0.y + c1 * ext, c0 * av0.z + c1 * ext);
    const f3 aop = abs3(op);
    f3 we;
    we.x = c1 * dot3(abs3(mk3(M[0], M[1], M[2])), aop) + c2 * fabsf(M[3]);
    we.y = c1 * dot3(abs3(mk3(M[4], M[5], M[6])), aop) + c2 * fabsf(M[7]);
    we.z = c1 * dot3(abs3(mk3(M[8], M[9], M[10])), aop) + c2 * fabsf(M[11]);
    const f3 awp = abs3(wp);
    f3 te;
    te.x = ((fabsf(I[0]) * awp.x + fabsf(I[4]) * awp.y) + fabsf(I[8]) * awp.z) + fabsf(I[12]) * 1.0f;
    te.y = ((fabsf(I[1]) * awp.x + fabsf(I[5]) * awp.y) + fabsf(I[9]) * awp.z) + fabsf(I[13]) * 1.0f;
    te.z = ((fabsf(I[2]) * awp.x + fabsf(I[6]) * awp.y) + fabsf(I[10]) * awp.z) + fabsf(I[14]) * 1.0f;
    oe = oe + mk3(c2 * te.x, c2 * te.y, c2 * te.z);
    const float oo = dot3(oe, abs3(on));
    float wo = dot3(we, abs3(wn));
    wo = __fmaf_rn(ws, oo, wo);
    *pos = wp;
    *nrm = wn;
    *off = wo;
}

// get_shading_data, scene.slang:271-406.
__device__ __forceinline__ Shading shading_data(const SceneView& s, uint32_t inst, uint32_t prim, float bx,
                                                float by, f3 view) {
    const TriRefs r = tri_refs(s, inst, prim);
    const float b0 = (1.0f - bx) - by;
    const f3 p0 = ld3(r.v0), p1 = ld3(r.v1), p2 = ld3(r.v2);
    f3 pos, fn;
    float off;
    triangle_spawn(p0, p1, p2, bx, by, r.m, r.it, &pos, &fn, &off);
    const f3 n0 = ld3(r.v0 + 3), n1 = ld3(r.v1 + 3), n2 = ld3(r.v2 + 3);
    const f3 ni = (b0 * n0 + bx * n1) + by * n2;
    const float* it = r.it;
    const f3 gnu = mk3(((__ldg(it + 0) * ni.x + __ldg(it + 1) * ni.y) + __ldg(it + 2) * ni.z) + __ldg(it + 3) * 0.0f,
                       ((__ldg(it + 4) * ni.x + __ldg(it + 5) * ni.y) + __ldg(it + 6) * ni.z) + __ldg(it + 7) * 0.0f,
                       ((__ldg(it + 8) * ni.x + __ldg(it + 9) * ni.y) + __ldg(it + 10) * ni.z) + __ldg(it + 11) * 0.0f);
    f3 gn = normalize3(gnu);
    f3 sn = gn;
    const uint32_t mflags = __float_as_uint(__ldg(r.mat + 3));
    const bool double_sided = (mflags & 1u) != 0u;
    const bool front = dot3(fn, view) > 0.0f;
    const float sign = (double_sided && !front) ? -1.0f : 1.0f;
    fn = fn * sign;
    gn = gn * sign;
    sn = sn * sign;
    sn = adjust_shading_normal(sn, fn, -view);
    Shading sd;
    sd.position = pos;
    sd.origin_front = pos + off * fn;
    sd.offset = off;
    sd.face_normal = fn;
    sd.frame = Frame(sn);
    sd.diffuse = ld3(r.mat);
    sd.emissive = ld3(r.mat + 4);
    sd.back_side = double_sided && !front;
    return sd;
}

// get_world_flat_normal, texture_space_path_tracer.slang:39-55, with
// compute_flat_normal, common.slang:101-111.
__device__ __forceinline__ f3 world_flat_normal(const SceneView& s, uint32_t inst, uint32_t prim) {
    const TriRefs r = tri_refs(s, inst, prim);
    const f3 p0 = ld3(r.v0), p1 = ld3(r.v1), p2 = ld3(r.v2);
    f3 n = normalize3(cross3(p1 - p0, p2 - p0));
    if (r.flags & 1u) n = -n;
    const float* it = r.it;
    const f3 w = mk3((__ldg(it + 0) * n.x + __ldg(it + 1) * n.y) + __ldg(it + 2) * n.z,
                     (__ldg(it + 4) * n.x + __ldg(it + 5) * n.y) + __ldg(it + 6) * n.z,
                     (__ldg(it + 8) * n.x + __ldg(it + 9) * n.y) + __ldg(it + 10) * n.z);
    return normalize3(w);
}

// ---------------------------------------------------------------------------
// Lights (scene.slang:408-527, 940-1009). The sun transmittance is one value
// per frame (get_sun_transmittance_at_view reads the LUT at the fixed view
// position), so it arrives as a constant; the sky is a constant radiance or
// the sky-view LUT looked up per direction (sample_sky_lut).
// ---------------------------------------------------------------------------
struct LightParams {
    f3 sun_dir;
    float cos_half;
    f3 outer;   // color * intensity
    f3 trans;   // transmittance
    f3 illum;   // outer * trans
    f3 sky;
    float t_max;
    bool sun_disk;
    bool area_nee;  // screen tracer: NEE toward the emissive triangles, MIS with the BSDF
    // sky-view LUT (null: the constant sky): RGBA32F [height][width]
    const float4* sky_lut;
    uint32_t sky_w, sky_h;
    f3 sky_up;          // unit vector from the planet's centre to the view position
    float sky_horizon;  // horizon angle at the view height (scene.slang:474)
};

struct LightingRaw {  // layout of NanLighting
    float sun_direction[3];
    float sun_cos_half_angle;
    float sun_color[3];
    float sun_intensity;
    float sun_transmittance[3];
    float ray_t_max;
    float sky_radiance[3];
    uint32_t flags;
    const float* sky_view_lut;
    uint32_t sky_view_width;
    uint32_t sky_view_height;
    float sky_view_up[3];
    float sky_view_horizon_angle;
};

__device__ __forceinline__ LightParams make_light(const LightingRaw& p) {
    LightParams L;
    L.sun_dir = mk3(p.sun_direction[0], p.sun_direction[1], p.sun_direction[2]);
    L.cos_half = p.sun_cos_half_angle;
    L.outer = mk3(p.sun_color[0], p.sun_color[1], p.sun_color[2]) * p.sun_intensity;
    L.trans = mk3(p.sun_transmittance[0], p.sun_transmittance[1], p.sun_transmittance[2]);
    L.illum = L.outer * L.trans;
    L.sky = mk3(p.sky_radiance[0], p.sky_radiance[1], p.sky_radiance[2]);
    L.t_max = p.ray_t_max;
    L.sun_disk = (p.flags & 1u) != 0u;
    L.area_nee = (p.flags & 2u) != 0u;
    L.sky_lut = reinterpret_cast<const float4*>(p.sky_view_lut);
    L.sky_w = p.sky_view_width;
    L.sky_h = p.sky_view_height;
    L.sky_up = mk3(p.sky_view_up[0], p.sky_view_up[1], p.sky_view_up[2]);
    L.sky_horizon = p.sky_view_horizon_angle;
    return L;
}

// sample_sky_lut (scene.slang:469-518): altitude asin(d . up) clamped 0.01
// short of the poles, azimuth atan2 against the frame (right = sun x up,
// forward = up x right), the LUT's non-linear altitude mapping inverted,
// v = (1 -+ sqrt|adjV|) / 2, u = azimuth / 2pi + 1/2; a bilinear fetch with
// wrapped addressing (the default sampler), times the sun's outer-space
// illuminance. A direction with no azimuth (straight along up) takes u = 1/2.
__device__ __forceinline__ float4 sky_texel(const LightParams& L, int x, int y) {
    x %= (int)L.sky_w;
    y %= (int)L.sky_h;
    if (x < 0) x += (int)L.sky_w;
    if (y < 0) y += (int)L.sky_h;
    return __ldg(L.sky_lut + (size_t)y * L.sky_w + (size_t)x);
}

__device__ __forceinline__ f3 sky_radiance(const LightParams& L, f3 d) {
    if (!L.sky_lut) return L.sky;
    const float kHalfPiF = 1.57079632679489662f;
    const float altitude = fminf(fmaxf(nan_asin(dot3(d, L.sky_up)), -kHalfPiF + 1e-2f), kHalfPiF - 1e-2f);
    float azimuth = 0.0f;
    if (!(fabsf(altitude) > kHalfPiF - 1e-4f)) {
        const f3 right = cross3(L.sun_dir, L.sky_up);
        const f3 forward = cross3(L.sky_up, right);
        const f3 proj = normalize3(d - L.sky_up * dot3(d, L.sky_up));
        azimuth = nan_atan2(dot3(proj, right), dot3(proj, forward));
    }
    const float adj = (altitude + L.sky_horizon) / kHalfPiF;
    const float v = adj < 0.0f ? 0.5f * (1.0f - sqrtf(fminf(fmaxf(-adj, 0.0f), 1.0f)))
                               : 0.5f * (1.0f + sqrtf(fminf(fmaxf(adj, 0.0f), 1.0f)));
    float u = azimuth / (2.0f * 3.14159265358979324f) + 0.5f;
    if (!(u >= 0.0f && u <= 1.0f)) u = 0.5f;
    const float fx = u * (float)L.sky_w - 0.5f, fy = v * (float)L.sky_h - 0.5f;
    const float x0 = floorf(fx), y0 = floorf(fy);
    const float tx = fx - x0, ty = fy - y0;
    const float4 a = sky_texel(L, (int)x0, (int)y0), b = sky_texel(L, (int)x0 + 1, (int)y0);
    const float4 c = sky_texel(L, (int)x0, (int)y0 + 1), e = sky_texel(L, (int)x0 + 1, (int)y0 + 1);
    const f3 top = mk3(a.x + tx * (b.x - a.x), a.y + tx * (b.y - a.y), a.z + tx * (b.z - a.z));
    const f3 bot = mk3(c.x + tx * (e.x - c.x), c.y + tx * (e.y - c.y), c.z + tx * (e.z - c.z));
    const f3 rgb = mk3(top.x + ty * (bot.x - top.x), top.y + ty * (bot.y - top.y), top.z + ty * (bot.z - top.z));
    return rgb * L.outer;
}

// Area-light next-event estimation (no counterpart in the reference, whose
// path tracer reaches emitters by BSDF sampling only). A triangle is chosen
// with probability area * luminance / power, a point uniformly on it, and
// the estimate is weighted against the cosine BSDF pdf by the power
// heuristic (Veach 1997, ch. 9). Emitters count from both sides.
struct AreaSample {
    f3 dir;
    float tmax;
    f3 contrib;  // to be multiplied by the path throughput when visible
    bool valid;
};

__device__ __forceinline__ AreaSample area_nee_sample(const SceneView& s, const Shading& sd, float usel, float u0,
                                                      float u1) {
    AreaSample r;
    r.valid = false;
    if (s.light_count == 0u) return r;
    uint32_t lo = 0u, hi = s.light_count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (usel < __ldg(s.lights + 4u * mid).w) hi = mid; else lo = mid + 1u;
    }
    const float4 a = __ldg(s.lights + 4u * lo), b = __ldg(s.lights + 4u * lo + 1u);
    const float4 c = __ldg(s.lights + 4u * lo + 2u), e = __ldg(s.lights + 4u * lo + 3u);
    const float su = sqrtf(u0);
    const float wa = su * (1.0f - u1), wb = su * u1;
    const f3 p = mk3((a.x + b.x * wa) + c.x * wb, (a.y + b.y * wa) + c.y * wb, (a.z + b.z * wa) + c.z * wb);
    const f3 v = p - sd.origin_front;
    const float d2 = dot3(v, v);
    if (!(d2 > 0.0f)) return r;
    const float dist = sqrtf(d2);
    const f3 l = v * (1.0f / dist);
    const float cx = dot3(sd.frame.n, l);
    if (!(cx > 0.0f)) return r;
    const f3 nl = normalize3(cross3(mk3(b.x, b.y, b.z), mk3(c.x, c.y, c.z)));
    const float cl = fabsf(dot3(nl, l));
    if (!(cl > 1e-6f)) return r;
    const float pl = ((c.w / s.light_power) * d2) / cl;
    const float pb = cx * kInvPi;
    const float w = (pl * pl) / (pl * pl + pb * pb);
    const f3 f = sd.diffuse * kInvPi;
    r.contrib = (f * mk3(e.x, e.y, e.z)) * ((cx / pl) * w);
    r.dir = l;
    r.tmax = dist * 0.999f;
    r.valid = true;
    return r;
}

// Power-heuristic weight of emission reached by a cosine BSDF sample with
// pdf pdf_bsdf, at distance t along dir, on a triangle with face normal fn.
__device__ __forceinline__ float area_mis_weight(const SceneView& s, f3 emissive, f3 fn, f3 dir, float t,
                                                 float pdf_bsdf) {
    const float lum = (0.2126f * emissive.x + 0.7152f * emissive.y) + 0.0722f * emissive.z;
    if (!(lum > 0.0f) || s.light_count == 0u) return 1.0f;
    const float cl = fabsf(dot3(normalize3(fn), dir));
    if (!(cl > 1e-6f)) return 0.0f;
    const float pl = ((lum / s.light_power) * (t * t)) / cl;
    return (pdf_bsdf * pdf_bsdf) / (pdf_bsdf * pdf_bsdf + pl * pl);
}

// get_sun_disk_luminance, scene.slang:408-465.
__device__ __forceinline__ f3 sun_disk(const LightParams& L, f3 dir) {
    const f3 vp = mk3(0.0f, 6.360f + 0.0002f, 0.0f);
    const float a = dot3(dir, dir);
    const float b = 2.0f * dot3(vp, dir);
    const float gr = 6.360f;
    const float c = dot3(vp, vp) - gr * gr;
    const float disc = b * b - 4.0f * a * c;
    if (disc >= 0.0f) {
        const float sq = sqrtf(disc);
        const float t0 = (-b - sq) / (2.0f * a);
        const float t1 = (-b + sq) / (2.0f * a);
        if (t0 > 0.0f || t1 > 0.0f) return mk3(0.0f, 0.0f, 0.0f);
    }
    const float vdl = dot3(dir, L.sun_dir);
    if (vdl > L.cos_half) {
        const float solid = (2.0f * kPi) * (1.0f - L.cos_half);
        const f3 lum = L.outer / solid;
        const float soft = sat(2.0f * (vdl - L.cos_half) / (1.0f - L.cos_half));
        return (L.trans * lum) * soft;
    }
    return mk3(0.0f, 0.0f, 0.0f);
}

struct RayTally {
    uint32_t extend;
    uint32_t shadow;
};

// sample_directional_light_with_visibility(sd, u, 1, 0), scene.slang:954-990.
template <class Tr = DefaultTracer>
__device__ __forceinline__ f3 sun_nee(const SceneView& s, const LightParams& L, const Shading& sd, float ux,
                                      float uy, RayTally& tally) {
    const f3 l = sample_cone_direction(L.sun_dir, L.cos_half, ux, uy);
    tally.shadow++;
    const float vis = Tr::any(s, sd.origin_front, l, 0.0f, L.t_max) ? 0.0f : 1.0f;
    const float ndl = maxf(0.0f, dot3(sd.frame.n, l));
    const f3 f = sd.diffuse * kInvPi;
    return ((vis * f) * L.illum) * ndl;
}

// sample_directional_irradiance, scene.slang:940-952.
__device__ __forceinline__ f3 sun_irradiance(const SceneView& s, const LightParams& L, const Shading& sd,
                                             float ux, float uy, RayTally& tally) {
    const f3 l = sample_cone_direction(L.sun_dir, L.cos_half, ux, uy);
    tally.shadow++;
    const float vis = trace_any(s, sd.origin_front, l, 0.0f, L.t_max) ? 0.0f : 1.0f;
    const float ndl = maxf(0.0f, dot3(sd.frame.n, l));
    return (vis * L.illum) * ndl;
}

}  // namespace nbd
