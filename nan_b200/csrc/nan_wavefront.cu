// nan_wavefront.cu -- wavefront form of the integrators.
//
// A path lives in SoA state arrays between kernels. Each iteration runs:
//   extend   persistent warps pull path ids from a compacted queue and trace
//            the closest hit of each path's ray (all lanes do traversal);
//   shade    per path: emission, sun NEE shadow ray (queued), next direction;
//   shadow   persistent warps trace the queued any-hit rays and add the
//            contributions of the visible ones;
//   finalize per path: continue, or close the sample (and start the next
//            sample, the back side, or retire the path).
// The RNG of a path is the reference's per-thread stream, drawn in the same
// order, and every radiance sum is formed in the same order as the
// reference's loop, so the result equals the one-thread-per-unit kernels bit
// for bit. Compiled with --fmad=false (see nan_math.cuh).
#include <algorithm>
#include <cstring>

#include "nan_internal.h"
#include "nan_scene.cuh"
#include "nan_sinks.cuh"
#include "nan_probe.cuh"

namespace {

using namespace nbd;
using nan_host::cuda_fail;
using nan_host::set_error;

constexpr uint32_t kFlagBack = 1u << 0;
constexpr uint32_t kFlagEnd = 1u << 1;
constexpr uint32_t kFlagNoPath = 1u << 2;
constexpr uint32_t kFlagTwoSided = 1u << 3;
constexpr uint32_t kBounceShift = 4;
constexpr uint32_t kBounceMask = 0xffu << kBounceShift;
constexpr uint32_t kSampleShift = 12;

constexpr uint32_t kKindNee = 0u;  // shadow contribution goes to rad
constexpr uint32_t kKindSun = 1u;  // shadow contribution goes to si (screen: the area-light term)

struct WfState {
    uint32_t* unit;   // surface texel / probe index
    uint32_t* rng;
    uint32_t* flags;
    float4* surf;     // b1, b2, instance bits, primitive bits
    float4* ro;       // origin, w = t_min
    float4* rd;       // direction, w = t_max
    float4* thp;
    float4* rad;
    float4* si;
    float4* irr;
    float2* zpdf;     // |z| and pdf of the sample's first direction
    float4* hit;      // flat bits (~0 = miss), t, b1, b2
    float4* pa;       // probes: source instance bits, source primitive bits, source offset, first-hit distance
    uint4* pb;        // probes: self-hit suspects of the sample, of all samples, previous count, radial texel
    uint4* pc;        // probes: 2 per path, per-radial-texel sample counts (16 x u16)
};

struct WfQueues {
    uint32_t* ext[2];
    uint32_t* ext_sorted;  // the extend queue regrouped by direction octant (NanTuning ray_order 1)
    float4* shd[2];        // 3 float4 per entry: (o, path bits), (d, kind bits), (c, 0)
    uint32_t* ctl;         // per iteration k: [4k] ext count, [4k+1] ext fetch, [4k+2] shd count, [4k+3] shd fetch
    uint32_t* oct;         // per iteration k: [16k..16k+7] paths per octant, [16k+8..16k+15] placement cursors
};

constexpr size_t kBytesPerPath = 4 + 4 + 4 + 16 * 9 + 8 + 16 + 16 + 32 + 3 * 4 + 2 * 2 * 48;

// Warp-aggregated append: returns this lane's slot in the queue.
__device__ __forceinline__ uint32_t queue_slot(uint32_t* count, bool want) {
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, want);
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t base = 0u;
    const int leader = __ffs(mask) - 1;
    if (mask && (int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
    base = __shfl_sync(active, base, leader < 0 ? __ffs(active) - 1 : leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

// tmax 0: the ray runs to the scene's t_max
__device__ __forceinline__ void push_shadow(const WfQueues& q, int buf, uint32_t* count, uint32_t p, f3 o, f3 d,
                                            f3 c, uint32_t kind, float tmax = 0.0f) {
    const uint32_t slot = queue_slot(count, true);
    float4* e = q.shd[buf] + 3u * slot;
    e[0] = make_float4(o.x, o.y, o.z, __uint_as_float(p));
    e[1] = make_float4(d.x, d.y, d.z, __uint_as_float(kind));
    e[2] = make_float4(c.x, c.y, c.z, tmax);
}

__device__ __forceinline__ f3 xyz(float4 v) { return mk3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 f4(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// ---------------------------------------------------------------------------
// Generic traversal stages.
// ---------------------------------------------------------------------------
// Extend-queue regrouping by ray direction octant (x < 0 | y < 0 << 1 |
// z < 0 << 2): neighbouring lanes of the traversal then follow rays of one
// octant, in their previous order within it. Two passes over the queue:
// a histogram, then a placement with warp-aggregated cursors.
__device__ __forceinline__ uint32_t dir_octant(float4 d) {
    return (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
}

__global__ void __launch_bounds__(256) k_wf_octant_count(const uint32_t* __restrict__ queue, const uint32_t* ctl,
                                                         const float4* __restrict__ rd, uint32_t* oct) {
    const uint32_t count = *(volatile const uint32_t*)(ctl + 0);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t o = dir_octant(rd[queue[idx]]);
        const unsigned group = __match_any_sync(__activemask(), o);
        if ((threadIdx.x & 31u) == (uint32_t)(__ffs(group) - 1)) atomicAdd(oct + o, (uint32_t)__popc(group));
    }
}

__global__ void __launch_bounds__(256) k_wf_octant_place(const uint32_t* __restrict__ queue, const uint32_t* ctl,
                                                         const float4* __restrict__ rd, uint32_t* oct,
                                                         uint32_t* __restrict__ out) {
    const uint32_t count = *(volatile const uint32_t*)(ctl + 0);
    uint32_t base[8];
    uint32_t sum = 0u;
    for (int o = 0; o < 8; ++o) {
        base[o] = sum;
        sum += oct[o];
    }
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t p = queue[idx];
        const uint32_t o = dir_octant(rd[p]);
        const unsigned active = __activemask();
        const unsigned group = __match_any_sync(active, o);
        const int leader = __ffs(group) - 1;
        uint32_t first = 0u;
        if ((int)lane == leader) first = atomicAdd(oct + 8 + o, (uint32_t)__popc(group));
        first = __shfl_sync(active, first, leader);
        out[base[o] + first + (uint32_t)__popc(group & ((1u << lane) - 1u))] = p;
    }
}

// Scene of a path: one scene for the per-scene passes, the path's probe set
// for the multi-scene batch (set index per path).
struct OneScene {
    SceneView s;
    __device__ __forceinline__ const SceneView& of(uint32_t) const { return s; }
};

struct ManyScenes {
    const BatchSet* sets;
    const uint32_t* set_of;
    __device__ __forceinline__ const SceneView& of(uint32_t p) const { return sets[set_of[p]].s; }
};

template <int kWidth, class Src, int kShared = 0, bool kSpec = false>
// kShared > 0 (binary nodes): the first kShared traversal-stack entries of a
// thread live in a shared-memory column, the rest in local memory. kSpec
// (binary nodes): the speculative while-while walk.
// 10 resident blocks of 128 per SM (48 registers a thread, -Xptxas -v): measured
// 1,941 against 1,895 Mrays/s with the register count left free (9 blocks),
// 1,916 at 11 and 12 blocks, 1,639 at 16 (spills).
__global__ void __launch_bounds__(128, 10) k_wf_extend(Src src, const uint32_t* __restrict__ queue,
                                                   uint32_t* ctl, const float4* __restrict__ ro,
                                                   const float4* __restrict__ rd, const uint32_t* __restrict__ flags,
                                                   float4* __restrict__ hit, unsigned long long* counters) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    const uint32_t lane = threadIdx.x & 31u;
    RayTally tally{0u, 0u};
    __shared__ int stack_top[kShared > 0 ? kShared * 128 : 1];
    for (;;) {
        uint32_t base = 0u;
        if (lane == 0u) base = atomicAdd(ctl + 1, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t idx = base + lane;
        if (idx < count) {
            const uint32_t p = queue[idx];
            if (flags[p] & kFlagNoPath) {
                hit[p] = make_float4(__uint_as_float(0xffffffffu), 0.0f, 0.0f, 0.0f);
            } else {
                const SceneView s = src.of(p);
                const float4 o = ro[p], d = rd[p];
                tally.extend++;
                HitInfo h;
                if constexpr (kShared > 0 && kWidth == 2) {
                    SplitStack<kShared, 128, kTraversalStack> stk;
                    stk.top = stack_top + threadIdx.x;
                    h = trace_closest_binary_s<kTraversalStack>(s, stk, xyz(o), xyz(d), o.w, d.w);
                } else if constexpr (kSpec && kWidth == 2) {
                    h = trace_closest_binary_spec(s, xyz(o), xyz(d), o.w, d.w);
                } else {
                    h = trace_closest_w<kWidth>(s, xyz(o), xyz(d), o.w, d.w);
                }
                hit[p] = make_float4(__uint_as_float(h.valid ? h.flat : 0xffffffffu), h.t, h.b1, h.b2);
            }
        }
    }
    flush_tally(counters, tally, 0u, 0u);
}

template <int kWidth, class Src, int kShared = 0, bool kSpec = false>
__global__ void __launch_bounds__(128, 10) k_wf_shadow(Src src, const float4* __restrict__ queue, uint32_t* ctl,
                                                   float t_max, float4* __restrict__ rad, float4* __restrict__ si,
                                                   unsigned long long* counters) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 2);
    const uint32_t lane = threadIdx.x & 31u;
    RayTally tally{0u, 0u};
    __shared__ int stack_top[kShared > 0 ? kShared * 128 : 1];
    for (;;) {
        uint32_t base = 0u;
        if (lane == 0u) base = atomicAdd(ctl + 3, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t idx = base + lane;
        if (idx < count) {
            const float4 a = queue[3u * idx], b = queue[3u * idx + 1u], c = queue[3u * idx + 2u];
            tally.shadow++;
            const uint32_t p = __float_as_uint(a.w);
            const SceneView s = src.of(p);
            bool blocked;
            if constexpr (kShared > 0 && kWidth == 2) {
                SplitStack<kShared, 128, kTraversalStack> stk;
                stk.top = stack_top + threadIdx.x;
                blocked = trace_any_binary_s<kTraversalStack>(s, stk, xyz(a), xyz(b), 0.0f, c.w > 0.0f ? c.w : t_max);
            } else if constexpr (kSpec && kWidth == 2) {
                blocked = trace_any_binary_spec(s, xyz(a), xyz(b), 0.0f, c.w > 0.0f ? c.w : t_max);
            } else {
                blocked = trace_any_w<kWidth>(s, xyz(a), xyz(b), 0.0f, c.w > 0.0f ? c.w : t_max);
            }
            if (!blocked) {
                float4* target = (__float_as_uint(b.w) == kKindNee) ? rad : si;
                const float4 v = target[p];
                target[p] = make_float4(v.x + c.x, v.y + c.y, v.z + c.z, v.w);
            }
        }
    }
    flush_tally(counters, tally, 0u, 0u);
}

// Persistent traversal with lane refill. Each lane walks its own ray
// (closest_step / any_step); once at least kRefill lanes of the warp are
// idle, the warp takes that many new rays from the queue in one atomic and
// hands them to the idle lanes, while the other lanes keep their walks.
// Finished rays write their results in the same refill round, so ray set-up
// and result stores run for the idle lanes together. kBurst steps run
// between two refill checks. Without refill, a warp that took 32 rays runs
// until the slowest of them ends.
template <int kRefill, int kBurst, class Src>
__global__ void __launch_bounds__(128, 10) k_wf_extend_refill(Src src, const uint32_t* __restrict__ queue,
                                                          uint32_t* ctl, const float4* __restrict__ ro,
                                                          const float4* __restrict__ rd,
                                                          const uint32_t* __restrict__ flags,
                                                          float4* __restrict__ hit, unsigned long long* counters) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    RayTally tally{0u, 0u};
    ClosestWalk w;
    int stack[kTraversalStack];
    bool alive = false, pending = false, drained = false;
    uint32_t p = 0u;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, !alive);
        if (drained) {
            if (idle == 0xffffffffu) break;
        } else if (__popc(idle) >= kRefill) {
            if (pending) {
                const HitInfo h = closest_end(src.of(p), w);
                hit[p] = make_float4(__uint_as_float(h.valid ? h.flat : 0xffffffffu), h.t, h.b1, h.b2);
                pending = false;
            }
            const uint32_t n = (uint32_t)__popc(idle);
            uint32_t base = 0u;
            if (lane == 0u) base = atomicAdd(ctl + 1, n);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (!alive) {
                const uint32_t idx = base + (uint32_t)__popc(idle & below);
                if (idx < count) {
                    p = queue[idx];
                    if (flags[p] & kFlagNoPath) {
                        hit[p] = make_float4(__uint_as_float(0xffffffffu), 0.0f, 0.0f, 0.0f);
                    } else {
                        const float4 o = ro[p], d = rd[p];
                        tally.extend++;
                        alive = closest_begin(src.of(p), w, xyz(o), xyz(d), o.w, d.w);
                        pending = !alive;
                    }
                }
            }
            if (base + n >= count) drained = true;
            continue;
        }
        if (alive) {
            const SceneView& s = src.of(p);
#pragma unroll 1
            for (int k = 0; k < kBurst; ++k) {
                if (!closest_step<kTraversalStack>(s, w, stack)) {
                    alive = false;
                    pending = true;
                    break;
                }
            }
        }
    }
    if (pending) {
        const HitInfo h = closest_end(src.of(p), w);
        hit[p] = make_float4(__uint_as_float(h.valid ? h.flat : 0xffffffffu), h.t, h.b1, h.b2);
    }
    flush_tally(counters, tally, 0u, 0u);
}

template <int kRefill, int kBurst, class Src>
__global__ void __launch_bounds__(128, 10) k_wf_shadow_refill(Src src, const float4* __restrict__ queue, uint32_t* ctl,
                                                          float t_max, float4* __restrict__ rad,
                                                          float4* __restrict__ si, unsigned long long* counters) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 2);
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    RayTally tally{0u, 0u};
    AnyWalk w;
    int stack[kTraversalStack];
    bool alive = false, pending = false, drained = false;
    uint32_t p = 0u, e = 0u;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, !alive);
        if (drained) {
            if (idle == 0xffffffffu) break;
        } else if (__popc(idle) >= kRefill) {
            if (pending) {  // a ray that ended without a hit adds its contribution
                const float4 b = queue[3u * e + 1u], c = queue[3u * e + 2u];
                float4* target = (__float_as_uint(b.w) == kKindNee) ? rad : si;
                const float4 v = target[p];
                target[p] = make_float4(v.x + c.x, v.y + c.y, v.z + c.z, v.w);
                pending = false;
            }
            const uint32_t n = (uint32_t)__popc(idle);
            uint32_t base = 0u;
            if (lane == 0u) base = atomicAdd(ctl + 3, n);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (!alive) {
                const uint32_t idx = base + (uint32_t)__popc(idle & below);
                if (idx < count) {
                    e = idx;
                    const float4 a = queue[3u * idx], b = queue[3u * idx + 1u], c = queue[3u * idx + 2u];
                    tally.shadow++;
                    p = __float_as_uint(a.w);
                    alive = any_begin(src.of(p), w, xyz(a), xyz(b), 0.0f, c.w > 0.0f ? c.w : t_max);
                    pending = !alive;
                }
            }
            if (base + n >= count) drained = true;
            continue;
        }
        if (alive) {
            const SceneView& s = src.of(p);
#pragma unroll 1
            for (int k = 0; k < kBurst; ++k) {
                const int r = any_step<kTraversalStack>(s, w, stack);
                if (r != 0) {
                    alive = false;
                    pending = r == 1;
                    break;
                }
            }
        }
    }
    if (pending) {
        const float4 b = queue[3u * e + 1u], c = queue[3u * e + 2u];
        float4* target = (__float_as_uint(b.w) == kKindNee) ? rad : si;
        const float4 v = target[p];
        target[p] = make_float4(v.x + c.x, v.y + c.y, v.z + c.z, v.w);
    }
    flush_tally(counters, tally, 0u, 0u);
}

// The path-state stages (generate / shade / finalize) are bound by the
// latency of their gathers (scene records, path state) more than by
// bandwidth: their launch bound of 6 blocks of 128 per SM (at most 80
// registers, no spills in the texel stages; they used 111-128) doubles the
// resident warps. Measured on the 200k texel iteration: 5.54 -> 5.03 ms of
// stage time per step. Shade and finalize take 8 blocks (64 registers, about
// 112 B of spills each): 5.04 -> 4.92 ms; generate stays at 6.
// ---------------------------------------------------------------------------
// Texture-space integrator stages (texture_space_path_tracer.slang:57-216).
// ---------------------------------------------------------------------------
struct TexelArgs {
    McView mc;
    uint4* slots;
    uint32_t iteration;
    uint32_t n;  // samples per texel
    uint32_t max_bounces;
    int reset;
    // points mode (irradiance at given surface points instead of texels)
    const float4* points;  // (b1, b2, instance bits, primitive bits | back << 31)
    float4* point_out;     // (E rgb, 0), or (0, 0, 0, -1) for no point
    int indirect_only;     // points mode: leave out the direct sun irradiance term
};

// Start sample k of the current side: sun irradiance shadow ray, first
// direction (estimate_surface_irradiance, texture_space_path_tracer.slang:95-113).
__device__ __forceinline__ void texel_start_sample(const SceneView& s, const LightParams& L, const WfState& st,
                                                   const WfQueues& q, int buf, uint32_t* ctl_next, uint32_t p,
                                                   uint32_t flags, Rng& rng, bool direct = true) {
    const float4 sf = st.surf[p];
    const uint32_t inst = __float_as_uint(sf.z), prim = __float_as_uint(sf.w);
    f3 view = world_flat_normal(s, inst, prim);
    if (flags & kFlagBack) view = -view;
    const Shading sd = shading_data(s, inst, prim, sf.x, sf.y, view);
    const float u0 = rng.next_1d(), u1 = rng.next_1d();
    const f3 l = sample_cone_direction(L.sun_dir, L.cos_half, u0, u1);
    const float ndl = maxf(0.0f, dot3(sd.frame.n, l));
    // the two draws are taken either way, so the RNG streams stay aligned
    if (direct) push_shadow(q, buf, ctl_next + 2, p, sd.origin_front, l, L.illum * ndl, kKindSun);
    st.si[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    st.rad[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    st.thp[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    const float e0 = rng.next_1d(), e1 = rng.next_1d();
    float pdf;
    const f3 dir = cosine_sample_hemisphere(e0, e1, &pdf);
    flags &= ~(kFlagEnd | kFlagNoPath | kBounceMask);
    if (pdf > 1e-6f) {
        st.ro[p] = f4(sd.origin_front, 0.0f);
        st.rd[p] = f4(sd.frame.to_global(dir), L.t_max);
        st.zpdf[p] = make_float2(fabsf(dir.z), pdf);
    } else {
        flags |= kFlagNoPath;
    }
    st.flags[p] = flags;
    const uint32_t slot = queue_slot(ctl_next + 0, true);
    q.ext[buf][slot] = p;
}

__global__ void __launch_bounds__(128, 6) k_wf_texel_generate(SceneView s, LightingRaw lraw, TexelArgs a, WfState st,
                                                           WfQueues q, uint32_t begin, uint32_t count,
                                                           unsigned long long* counters) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    TexelSurface ts;
    Rng rng(0u, 0u, 0u);
    if (!texel_surface(s, a.mc, begin + p, a.iteration, a.n, &ts, &rng)) return;
    const LightParams L = make_light(lraw);
    st.unit[p] = begin + p;
    st.surf[p] = make_float4(ts.b1, ts.b2, __uint_as_float(ts.inst), __uint_as_float(ts.prim));
    st.irr[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const uint32_t flags = (ts.side.y & 1u) ? kFlagTwoSided : 0u;
    texel_start_sample(s, L, st, q, 0, q.ctl, p, flags, rng);
    st.rng[p] = rng.state;
    RayTally none{0u, 0u};
    flush_tally(counters, none, 1u, (ts.side.y & 1u) ? 2u * a.n : a.n);
}

// Surface points instead of texels: the same estimator at the listed points,
// with RNG(index, 0xFFFFFFFF, iteration * n) and view = the flat normal,
// negated for the back side.
__global__ void __launch_bounds__(128) k_wf_point_generate(SceneView s, LightingRaw lraw, TexelArgs a, WfState st,
                                                           WfQueues q, uint32_t begin, uint32_t count,
                                                           unsigned long long* counters) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const uint32_t u = begin + p;
    const float4 pt = a.points[u];
    const uint32_t inst = __float_as_uint(pt.z), primw = __float_as_uint(pt.w);
    const uint32_t prim = primw & 0x7fffffffu;
    if (inst == 0xffffffffu || !valid_prim(s, inst, prim)) {
        if (inst != 0xffffffffu) atomicOr(s.status, kStatusBadRecord);
        a.point_out[u] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        return;
    }
    const LightParams L = make_light(lraw);
    Rng rng(u, 0xffffffffu, a.iteration * a.n);
    st.unit[p] = u;
    st.surf[p] = make_float4(pt.x, pt.y, __uint_as_float(inst), __uint_as_float(prim));
    st.irr[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    texel_start_sample(s, L, st, q, 0, q.ctl, p, (primw >> 31) ? kFlagBack : 0u, rng, !a.indirect_only);
    st.rng[p] = rng.state;
    RayTally none{0u, 0u};
    flush_tally(counters, none, 1u, a.n);
}

// One bounce of trace_radiance (texture_space_path_tracer.slang:60-83) after
// the extend stage found the hit.
__global__ void __launch_bounds__(128, 8) k_wf_texel_shade(SceneView s, LightingRaw lraw, TexelArgs a, WfState st,
                                                        WfQueues q, int buf, uint32_t* ctl) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    const LightParams L = make_light(lraw);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t p = q.ext[buf][idx];
        uint32_t flags = st.flags[p];
        if (flags & kFlagNoPath) {
            st.flags[p] = flags | kFlagEnd;
            continue;
        }
        const float4 h = st.hit[p];
        const f3 d = xyz(st.rd[p]);
        f3 thp = xyz(st.thp[p]), rad = xyz(st.rad[p]);
        const uint32_t flat = __float_as_uint(h.x);
        if (flat == 0xffffffffu) {
            rad = rad + thp * sky_radiance(L, d);
            st.rad[p] = f4(rad, 0.0f);
            st.flags[p] = flags | kFlagEnd;
            continue;
        }
        Rng rng(0u, 0u, 0u);
        rng.state = st.rng[p];
        const uint2 ref = __ldg(s.tri_refs + flat);
        const Shading sd = shading_data(s, ref.x, ref.y, h.z, h.w, -d);
        rad = rad + thp * sd.emissive;
        const float u0 = rng.next_1d(), u1 = rng.next_1d();
        const f3 l = sample_cone_direction(L.sun_dir, L.cos_half, u0, u1);
        const float ndl = maxf(0.0f, dot3(sd.frame.n, l));
        const f3 f = sd.diffuse * kInvPi;
        push_shadow(q, buf, ctl + 2, p, sd.origin_front, l, thp * ((f * L.illum) * ndl), kKindNee);
        const float e0 = rng.next_1d(), e1 = rng.next_1d();
        float pdf;
        const f3 sdir = cosine_sample_hemisphere(e0, e1, &pdf);
        if (pdf <= 1e-6f) {
            flags |= kFlagEnd;
        } else {
            thp = thp * ((f * fabsf(sdir.z)) / pdf);
            st.ro[p] = f4(sd.origin_front, 0.0f);
            st.rd[p] = f4(sd.frame.to_global(sdir), L.t_max);
            const uint32_t bounce = ((flags & kBounceMask) >> kBounceShift) + 1u;
            flags = (flags & ~kBounceMask) | (bounce << kBounceShift);
            if (bounce >= a.max_bounces) flags |= kFlagEnd;
        }
        st.thp[p] = f4(thp, 0.0f);
        st.rad[p] = f4(rad, 0.0f);
        st.rng[p] = rng.state;
        st.flags[p] = flags;
    }
}

// Close finished samples: si += L*|z|/pdf, irr += si, next sample / side, or
// the running-mean store (texture_space_path_tracer.slang:111-138, 203-215).
__global__ void __launch_bounds__(128, 8) k_wf_texel_finalize(SceneView s, LightingRaw lraw, TexelArgs a, WfState st,
                                                           WfQueues q, int buf, uint32_t* ctl, uint32_t* ctl_next) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    const LightParams L = make_light(lraw);
    const int nbuf = buf ^ 1;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t p = q.ext[buf][idx];
        uint32_t flags = st.flags[p];
        if (!(flags & kFlagEnd)) {
            const uint32_t slot = queue_slot(ctl_next + 0, true);
            q.ext[nbuf][slot] = p;
            continue;
        }
        f3 si = xyz(st.si[p]);
        if (!(flags & kFlagNoPath)) {
            const float2 zp = st.zpdf[p];
            si = si + ((xyz(st.rad[p]) * zp.x) / zp.y);
        }
        f3 irr = xyz(st.irr[p]) + si;
        uint32_t k = (flags >> kSampleShift) + 1u;
        Rng rng(0u, 0u, 0u);
        rng.state = st.rng[p];
        if (k < a.n) {
            flags = (flags & ((1u << kSampleShift) - 1u)) | (k << kSampleShift);
            st.irr[p] = f4(irr, 0.0f);
            texel_start_sample(s, L, st, q, nbuf, ctl_next, p, flags, rng, !a.indirect_only);
            st.rng[p] = rng.state;
            continue;
        }
        const uint32_t u = st.unit[p];
        if (a.point_out) {
            a.point_out[u] = f4(irr / (float)a.n, 0.0f);
            continue;
        }
        // side complete: running mean into its slot
        const uint32_t inst = __float_as_uint(st.surf[p].z);
        const uint4 info = __ldg(a.mc.instance_infos + inst);
        const uint2 side = __ldg(a.mc.side_infos + inst);
        const uint32_t global_texel = info.z + (u - __ldg(a.mc.surface_prefix + inst));
        const uint32_t slot = (flags & kFlagBack) ? side.x + (global_texel - info.z) : global_texel;
        if (slot < a.mc.payload_count) store_running_mean(a.slots, slot, irr / (float)a.n, a.reset, a.mc.compensation);
        else atomicOr(s.status, 2u);
        if (!(flags & kFlagBack) && (flags & kFlagTwoSided)) {
            flags = (flags & ((1u << kSampleShift) - 1u)) | kFlagBack;
            st.irr[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            texel_start_sample(s, L, st, q, nbuf, ctl_next, p, flags, rng);
            st.rng[p] = rng.state;
        }
    }
}


// ---------------------------------------------------------------------------
// Screen path tracer stages (path_tracer.slang:40-130, camera.slang:201-236).
// ---------------------------------------------------------------------------
struct CameraWf {  // layout of NanCamera
    float position[3];
    float jitter_x;
    float image_u[3];
    float jitter_y;
    float image_v[3];
    float near_clip;
    float image_w[3];
    float far_clip;
};

// Cached frames: paths end at their second hit, which becomes a cache query
// (position and pixel, shading normal, weight = throughput * albedo / pi).
// Pixels (offset + i * stride) mod P for i < train_count also record the
// hit as training point i.
struct CachedArgs {
    float4* queries;  // 2 per query
    float4* weights;
    uint32_t* query_count;
    float4* train_points;
    float4* train_queries;  // 2 per training point
    uint32_t train_count, train_offset, train_inverse;
    uint32_t vertex;  // path vertex that queries the cache: 0 (indirect) or 1
};

struct ScreenArgs {
    CameraWf cam;
    float4* out;
    uint32_t width, height, frame, max_vertices;
    int cached;
    int area_nee;  // lighting flag bit 1 (the finalize stage has no lighting)
    CachedArgs cache;
};

__global__ void __launch_bounds__(128) k_wf_screen_generate(SceneView s, LightingRaw lraw, ScreenArgs a, WfState st,
                                                            WfQueues q, uint32_t begin, uint32_t count,
                                                            unsigned long long* counters) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const uint32_t pixel = begin + p;
    const uint32_t px = pixel % a.width, py = pixel / a.width;
    Rng rng(px, py, a.frame * 1u + 0u);
    rng.next_1d();
    rng.next_1d();  // the unused jitter draw (path_tracer.slang:121)
    const CameraWf& cam = a.cam;
    float pxf = ((float)px + 0.5f) / (float)a.width;
    float pyf = ((float)py + 0.5f) / (float)a.height;
    pxf = pxf + (-cam.jitter_x);
    pyf = pyf + cam.jitter_y;
    const float nx = 2.0f * pxf + -1.0f;
    const float ny = -2.0f * pyf + 1.0f;
    const f3 U = mk3(cam.image_u[0], cam.image_u[1], cam.image_u[2]);
    const f3 V = mk3(cam.image_v[0], cam.image_v[1], cam.image_v[2]);
    const f3 W = mk3(cam.image_w[0], cam.image_w[1], cam.image_w[2]);
    const f3 dir = normalize3((nx * U + ny * V) + W);
    const float inv_cos = 1.0f / dot3(normalize3(W), dir);
    st.unit[p] = pixel;
    st.rng[p] = rng.state;
    st.flags[p] = 0u;
    st.ro[p] = f4(mk3(cam.position[0], cam.position[1], cam.position[2]), cam.near_clip * inv_cos);
    st.rd[p] = f4(dir, cam.far_clip * inv_cos);
    st.thp[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    st.rad[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    st.si[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    st.zpdf[p] = make_float2(0.0f, 1.0f);
    const uint32_t slot = queue_slot(q.ctl + 0, true);
    q.ext[0][slot] = p;
    RayTally none{0u, 0u};
    flush_tally(counters, none, 1u, 1u);
}

// The area-light term of the previous vertex (kept apart by the shadow stage)
// joins the radiance after that vertex's sun term, as in the loop's order.
__device__ __forceinline__ f3 fold_area_term(const WfState& st, uint32_t p, f3 rad) {
    const float4 a = st.si[p];
    st.si[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return rad + xyz(a);
}

__global__ void __launch_bounds__(128, 6) k_wf_screen_shade(SceneView s, LightingRaw lraw, ScreenArgs a, WfState st,
                                                         WfQueues q, int buf, uint32_t* ctl) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    const LightParams L = make_light(lraw);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t p = q.ext[buf][idx];
        uint32_t flags = st.flags[p];
        const float4 h = st.hit[p];
        const f3 d = xyz(st.rd[p]);
        f3 thp = xyz(st.thp[p]), rad = xyz(st.rad[p]);
        if (L.area_nee) rad = fold_area_term(st, p, rad);
        const uint32_t vertex = (flags & kBounceMask) >> kBounceShift;
        const uint32_t flat = __float_as_uint(h.x);
        if (flat == 0xffffffffu) {
            f3 sky = sky_radiance(L, d);
            if (vertex == 0u && L.sun_disk) sky = sky + sun_disk(L, d);
            rad = rad + thp * sky;
            st.rad[p] = f4(rad, 0.0f);
            st.flags[p] = flags | kFlagEnd;
            continue;
        }
        Rng rng(0u, 0u, 0u);
        rng.state = st.rng[p];
        const uint2 ref = __ldg(s.tri_refs + flat);
        const Shading sd = shading_data(s, ref.x, ref.y, h.z, h.w, -d);
        if (L.area_nee && vertex > 0u)
            rad = rad + thp * (sd.emissive * area_mis_weight(s, sd.emissive, sd.face_normal, d, h.y, st.zpdf[p].y));
        else
            rad = rad + thp * sd.emissive;
        const f3 f = sd.diffuse * kInvPi;
        if (a.cached && vertex == a.cache.vertex) {
            // the rest of the path is the cache's irradiance at this point;
            // at vertex 0 the sun is still sampled (NEE) and the cache holds
            // the indirect irradiance only
            if (vertex == 0u) {
                const float u0 = rng.next_1d(), u1 = rng.next_1d();
                const f3 l = sample_cone_direction(L.sun_dir, L.cos_half, u0, u1);
                const float ndl = maxf(0.0f, dot3(sd.frame.n, l));
                push_shadow(q, buf, ctl + 2, p, sd.origin_front, l, thp * ((f * L.illum) * ndl), kKindNee);
            }
            const uint32_t pixel = st.unit[p];
            const uint32_t qi = queue_slot(a.cache.query_count, true);
            const float4 q0 = make_float4(sd.position.x, sd.position.y, sd.position.z, __uint_as_float(pixel));
            const float4 q1 = f4(sd.frame.n, 0.0f);
            a.cache.queries[2u * qi] = q0;
            a.cache.queries[2u * qi + 1u] = q1;
            a.cache.weights[qi] = f4(thp * f, 0.0f);
            const uint32_t P = a.width * a.height;
            const uint32_t rel = pixel >= a.cache.train_offset ? pixel - a.cache.train_offset
                                                               : pixel + (P - a.cache.train_offset);
            const uint32_t ti = (uint32_t)(((uint64_t)rel * a.cache.train_inverse) % P);
            if (ti < a.cache.train_count) {
                // a back side exists for double-sided materials only (as texel back slots)
                const bool two = (__float_as_uint(__ldg(tri_refs(s, ref.x, ref.y).mat + 3)) & 1u) != 0u;
                const bool back = two && dot3(world_flat_normal(s, ref.x, ref.y), -d) < 0.0f;
                a.cache.train_points[ti] = make_float4(h.z, h.w, __uint_as_float(ref.x),
                                                       __uint_as_float(ref.y | (back ? 0x80000000u : 0u)));
                a.cache.train_queries[2u * ti] = q0;
                a.cache.train_queries[2u * ti + 1u] = q1;
            }
            st.rad[p] = f4(rad, 0.0f);
            st.flags[p] = flags | kFlagEnd;
            continue;
        }
        const float u0 = rng.next_1d(), u1 = rng.next_1d();
        const f3 l = sample_cone_direction(L.sun_dir, L.cos_half, u0, u1);
        const float ndl = maxf(0.0f, dot3(sd.frame.n, l));
        push_shadow(q, buf, ctl + 2, p, sd.origin_front, l, thp * ((f * L.illum) * ndl), kKindNee);
        // light reached from this vertex lies on the next one: sampled only
        // where that vertex exists, so both strategies cover the same paths
        if (L.area_nee && vertex + 1u < a.max_vertices) {
            const float us = rng.next_1d(), a0 = rng.next_1d(), a1 = rng.next_1d();
            const AreaSample as = area_nee_sample(s, sd, us, a0, a1);
            if (as.valid) push_shadow(q, buf, ctl + 2, p, sd.origin_front, as.dir, thp * as.contrib, kKindSun, as.tmax);
        }
        const float e0 = rng.next_1d(), e1 = rng.next_1d();
        float pdf;
        const f3 wo = cosine_sample_hemisphere(e0, e1, &pdf);
        pdf = maxf(pdf, 1e-6f);
        st.zpdf[p] = make_float2(0.0f, pdf);
        thp = thp * ((f * fabsf(wo.z)) / pdf);
        st.ro[p] = f4(sd.origin_front, 0.0f);
        st.rd[p] = f4(sd.frame.to_global(wo), L.t_max);
        const uint32_t next = vertex + 1u;
        flags = (flags & ~kBounceMask) | (next << kBounceShift);
        if (next >= a.max_vertices) flags |= kFlagEnd;
        st.thp[p] = f4(thp, 0.0f);
        st.rad[p] = f4(rad, 0.0f);
        st.rng[p] = rng.state;
        st.flags[p] = flags;
    }
}

__global__ void __launch_bounds__(128) k_wf_screen_finalize(ScreenArgs a, WfState st, WfQueues q, int buf,
                                                            uint32_t* ctl, uint32_t* ctl_next) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t p = q.ext[buf][idx];
        if (!(st.flags[p] & kFlagEnd)) {
            const uint32_t slot = queue_slot(ctl_next + 0, true);
            q.ext[buf ^ 1][slot] = p;
            continue;
        }
        float4 r = st.rad[p];
        if (a.area_nee) {
            const float4 t = st.si[p];
            r = make_float4(r.x + t.x, r.y + t.y, r.z + t.z, r.w);
        }
        a.out[st.unit[p]] = make_float4(r.x, r.y, r.z, 1.0f);
    }
}

// ---------------------------------------------------------------------------
// Surface-probe baker stages (surface_probe_path_tracer.slang:151-315).
// ---------------------------------------------------------------------------
struct ProbeArgs {
    ProbeOut out;
    const float4* probes;
    const float4* pinst;
    uint32_t probe_instance_count;
    uint32_t iteration, n, spp, max_bounces;
    int reset;
};

// Shading of the probe's own surface point (estimate_surface_irradiance).
__device__ __forceinline__ Shading probe_surface(const SceneView& s, const ProbeArgs& a, uint32_t probe,
                                                 const float4& surf) {
    const float4 nrm = __ldg(a.probes + 3u * probe + 1u);
    const f3 view = normalize3(mk3(nrm.x, nrm.y, nrm.z));
    return shading_data(s, __float_as_uint(surf.z), __float_as_uint(surf.w), surf.x, surf.y, view);
}

// One cosine sample around the face normal (no sun at the probe itself).
__device__ __forceinline__ void probe_start_sample(const SceneView& s, const LightParams& L, const ProbeArgs& a,
                                                   const WfState& st, const WfQueues& q, int buf, uint32_t* ctl_next,
                                                   uint32_t p, uint32_t flags, Rng& rng) {
    const float4 surf = st.surf[p];
    const Shading sd = probe_surface(s, a, st.unit[p], surf);
    const float kr = st.si[p].w;
    const float e0 = rng.next_1d(), e1 = rng.next_1d();
    float pdf;
    const f3 dir = cosine_sample_hemisphere(e0, e1, &pdf);
    flags &= ~(kFlagEnd | kFlagNoPath | kBounceMask);
    if (pdf > 1e-6f) {
        const f3 o = sd.origin_front;
        st.ro[p] = f4(o, 0.0f);
        st.rd[p] = f4(Frame(normalize3(sd.face_normal)).to_global(dir), L.t_max);
        st.thp[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        st.rad[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        st.zpdf[p] = make_float2(fabsf(dir.z), pdf);
        st.pa[p] = make_float4(surf.z, surf.w, len3(o - sd.position), 2.0f * kr);
        uint4 b = st.pb[p];
        b.x = 0u;
        b.w = radial_texel(dir);
        st.pb[p] = b;
    } else {
        flags |= kFlagNoPath;
    }
    st.flags[p] = flags;
    const uint32_t slot = queue_slot(ctl_next + 0, true);
    q.ext[buf][slot] = p;
}

// Per-path bodies of the probe stages, shared by the one-scene kernels and the
// multi-scene batch kernels (which look up the path's probe set first).
__device__ __forceinline__ bool probe_generate_path(const SceneView& s, const LightParams& L, const ProbeArgs& a,
                                                    const WfState& st, const WfQueues& q, uint32_t probe, uint32_t p) {
    const uint4 meta = __ldg(reinterpret_cast<const uint4*>(a.probes) + 3u * probe + 2u);
    const uint32_t inst = meta.w >> 8;
    if (inst >= a.probe_instance_count || !valid_prim(s, inst, meta.x)) {
        atomicOr(s.status, kStatusBadRecord);
        return false;
    }
    const float4 params = __ldg(a.pinst + 3u * inst + 2u);
    st.unit[p] = probe;
    st.surf[p] = make_float4(__uint_as_float(meta.y), __uint_as_float(meta.z), __uint_as_float(inst),
                             __uint_as_float(meta.x));
    st.si[p] = make_float4(0.0f, 0.0f, 0.0f, maxf(params.x, 1e-6f));
    st.irr[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const uint32_t prev_iter = a.reset ? 0u : a.out.counts[probe];
    st.pb[p] = make_uint4(0u, 0u, prev_iter, 0u);
    st.pc[2u * p] = make_uint4(0u, 0u, 0u, 0u);
    st.pc[2u * p + 1u] = make_uint4(0u, 0u, 0u, 0u);
    if (a.reset)
        for (int t = 0; t < 16; ++t) a.out.radial[16u * probe + (uint32_t)t] = 0u;
    Rng rng(probe, inst, a.iteration * a.n);
    probe_start_sample(s, L, a, st, q, 0, q.ctl, p, 0u, rng);
    st.rng[p] = rng.state;
    return true;
}

__device__ __forceinline__ void probe_shade_path(const SceneView& s, const LightParams& L, const ProbeArgs& a,
                                                 const WfState& st, const WfQueues& q, int buf, uint32_t* ctl,
                                                 uint32_t p) {
    uint32_t flags = st.flags[p];
    if (flags & kFlagNoPath) {
        st.flags[p] = flags | kFlagEnd;
        return;
    }
    const float4 h = st.hit[p];
    const f3 d = xyz(st.rd[p]);
    f3 thp = xyz(st.thp[p]), rad = xyz(st.rad[p]);
    float4 pa = st.pa[p];  // src inst, src prim, src offset, first hit
    const uint32_t bounce = (flags & kBounceMask) >> kBounceShift;
    const float radial_max = 2.0f * st.si[p].w;
    const uint32_t flat = __float_as_uint(h.x);
    if (flat == 0xffffffffu) {
        if (bounce == 0u) pa.w = radial_max;
        rad = rad + thp * sky_radiance(L, d);
        st.pa[p] = pa;
        st.rad[p] = f4(rad, 0.0f);
        st.flags[p] = flags | kFlagEnd;
        return;
    }
    if (bounce == 0u) pa.w = minf(h.y, radial_max);
    const uint2 ref = __ldg(s.tri_refs + flat);
    const uint32_t src_inst = __float_as_uint(pa.x), src_prim = __float_as_uint(pa.y);
    const bool same_prim = ref.x == src_inst && ref.y == src_prim;
    const float thr = maxf(4.0f * pa.z, 1e-6f);
    const bool adjacent = ref.x == src_inst && h.y <= thr;
    if (same_prim || adjacent) {
        uint4 b = st.pb[p];
        b.x += 1u;
        st.pb[p] = b;
    }
    Rng rng(0u, 0u, 0u);
    rng.state = st.rng[p];
    const Shading sd = shading_data(s, ref.x, ref.y, h.z, h.w, -d);
    rad = rad + thp * sd.emissive;
    const float u0 = rng.next_1d(), u1 = rng.next_1d();
    const f3 l = sample_cone_direction(L.sun_dir, L.cos_half, u0, u1);
    const float ndl = maxf(0.0f, dot3(sd.frame.n, l));
    const f3 f = sd.diffuse * kInvPi;
    // the set's own t_max travels with the shadow ray (the batch mixes scenes)
    push_shadow(q, buf, ctl + 2, p, sd.origin_front, l, thp * ((f * L.illum) * ndl), kKindNee, L.t_max);
    const float e0 = rng.next_1d(), e1 = rng.next_1d();
    float pdf;
    const f3 sdir = cosine_sample_hemisphere(e0, e1, &pdf);
    if (pdf <= 1e-6f) {
        flags |= kFlagEnd;
    } else {
        thp = thp * ((f * fabsf(sdir.z)) / pdf);
        const f3 next_origin = sd.origin_front;
        st.ro[p] = f4(next_origin, 0.0f);
        st.rd[p] = f4(Frame(normalize3(sd.face_normal)).to_global(sdir), L.t_max);
        pa.x = __uint_as_float(ref.x);
        pa.y = __uint_as_float(ref.y);
        pa.z = len3(next_origin - sd.position);
        const uint32_t next = bounce + 1u;
        flags = (flags & ~kBounceMask) | (next << kBounceShift);
        if (next >= a.max_bounces) flags |= kFlagEnd;
    }
    st.pa[p] = pa;
    st.thp[p] = f4(thp, 0.0f);
    st.rad[p] = f4(rad, 0.0f);
    st.rng[p] = rng.state;
    st.flags[p] = flags;
}

__device__ __forceinline__ void probe_finalize_path(const SceneView& s, const LightParams& L, const ProbeArgs& a,
                                                    const WfState& st, const WfQueues& q, int buf,
                                                    uint32_t* ctl_next, uint32_t p) {
    const int nbuf = buf ^ 1;
    uint32_t flags = st.flags[p];
    if (!(flags & kFlagEnd)) {
        const uint32_t slot = queue_slot(ctl_next + 0, true);
        q.ext[nbuf][slot] = p;
        return;
    }
    const uint32_t probe = st.unit[p];
    f3 irr = xyz(st.irr[p]);
    uint4 b = st.pb[p];
    if (!(flags & kFlagNoPath)) {
        b.y += b.x;  // self-hit suspects of this sample
        const uint32_t texel = b.w;
        uint4 c = st.pc[2u * p + (texel >> 3)];
        const uint32_t word = (texel >> 1) & 3u, shift = (texel & 1u) * 16u;
        uint32_t* cw = word == 0u ? &c.x : (word == 1u ? &c.y : (word == 2u ? &c.z : &c.w));
        const uint32_t local = ((*cw >> shift) & 0xffffu) + 1u;
        *cw = (*cw & ~(0xffffu << shift)) | ((local & 0xffffu) << shift);
        st.pc[2u * p + (texel >> 3)] = c;
        const float kr = st.si[p].w;
        accumulate_radial_moment(a.out.radial, probe, texel, st.pa[p].w / maxf(kr, 1e-6f), b.z, local, a.spp);
        const float2 zp = st.zpdf[p];
        irr = irr + ((xyz(st.rad[p]) * zp.x) / zp.y);
    }
    st.pb[p] = b;
    const uint32_t k = (flags >> kSampleShift) + 1u;
    if (k < a.n) {
        st.irr[p] = f4(irr, 0.0f);
        Rng rng(0u, 0u, 0u);
        rng.state = st.rng[p];
        probe_start_sample(s, L, a, st, q, nbuf, ctl_next, p,
                           (flags & ((1u << kSampleShift) - 1u)) | (k << kSampleShift), rng);
        st.rng[p] = rng.state;
        return;
    }
    irr = irr / (float)a.n;
    const uint32_t prev = a.reset ? 0u : a.out.counts[probe];
    f3 pv = mk3(0.0f, 0.0f, 0.0f);
    if (prev != 0u)
        pv = mk3(a.out.values[3u * probe], a.out.values[3u * probe + 1u], a.out.values[3u * probe + 2u]);
    float4 comp = a.out.compensation ? a.out.compensation[probe] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const f3 acc = running_mean_step(pv, irr, prev, a.out.compensation ? &comp : nullptr);
    if (a.out.compensation) a.out.compensation[probe] = comp;
    a.out.values[3u * probe] = acc.x;
    a.out.values[3u * probe + 1u] = acc.y;
    a.out.values[3u * probe + 2u] = acc.z;
    a.out.counts[probe] = min(prev + 1u, 65535u);
    const uint32_t prev_self = a.reset ? 0u : a.out.self_hits[probe];
    a.out.self_hits[probe] = prev_self + b.y;
}

__global__ void __launch_bounds__(128) k_wf_probe_generate(SceneView s, LightingRaw lraw, ProbeArgs a, WfState st,
                                                           WfQueues q, uint32_t begin, uint32_t count,
                                                           unsigned long long* counters) {
    const uint32_t slot_p = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot_p >= count) return;
    if (!probe_generate_path(s, make_light(lraw), a, st, q, begin + slot_p, slot_p)) return;
    RayTally none{0u, 0u};
    flush_tally(counters, none, 1u, a.n);
}

__global__ void __launch_bounds__(128, 6) k_wf_probe_shade(SceneView s, LightingRaw lraw, ProbeArgs a, WfState st,
                                                        WfQueues q, int buf, uint32_t* ctl) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    const LightParams L = make_light(lraw);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x)
        probe_shade_path(s, L, a, st, q, buf, ctl, q.ext[buf][idx]);
}

__global__ void __launch_bounds__(128, 6) k_wf_probe_finalize(SceneView s, LightingRaw lraw, ProbeArgs a, WfState st,
                                                           WfQueues q, int buf, uint32_t* ctl, uint32_t* ctl_next) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    const LightParams L = make_light(lraw);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x)
        probe_finalize_path(s, L, a, st, q, buf, ctl_next, q.ext[buf][idx]);
}

// ---------------------------------------------------------------------------
// Multi-scene probe batch on the wavefront: every (set, probe) unit of the
// batch is one path in flight; each stage looks up the path's set (scene,
// lighting, records, outputs). The iteration and reset come from the batch's
// device control block, so a captured frame replays with the next iteration.
// ---------------------------------------------------------------------------
struct BatchWfArgs {
    const BatchSet* sets;
    const uint32_t* prefix;
    const BatchCtl* ctl;
    uint32_t* set_of;
    uint32_t set_count, total, n, spp, max_bounces;
    // independent samples: units [unit_begin, unit_begin + units) of this
    // chunk, one path per (unit, sample), and the per-sample results
    uint32_t unit_begin, units;
    ProbeSample* samples;
};

__device__ __forceinline__ uint32_t batch_set_of_unit(const BatchWfArgs& m, uint32_t u) {
    uint32_t lo = 0u, hi = m.set_count - 1u;  // set = last s with prefix[s] <= u
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (__ldg(m.prefix + mid) <= u) lo = mid;
        else hi = mid - 1u;
    }
    return lo;
}

__device__ __forceinline__ ProbeArgs batch_probe_args(const BatchWfArgs& m, const BatchSet& b) {
    ProbeArgs a;
    a.out = b.out;
    a.probes = b.probes;
    a.pinst = b.pinst;
    a.probe_instance_count = b.probe_instance_count;
    a.iteration = m.ctl->iteration;
    a.n = m.n;
    a.spp = m.spp;
    a.max_bounces = m.max_bounces;
    a.reset = m.ctl->reset ? 1 : 0;
    return a;
}

__global__ void __launch_bounds__(128) k_wfb_probe_generate(BatchWfArgs m, WfState st, WfQueues q,
                                                            unsigned long long* counters) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= m.total) return;
    uint32_t lo = 0u, hi = m.set_count - 1u;  // set = last s with prefix[s] <= u
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (__ldg(m.prefix + mid) <= u) lo = mid;
        else hi = mid - 1u;
    }
    m.set_of[u] = lo;
    const BatchSet& b = m.sets[lo];
    const ProbeArgs a = batch_probe_args(m, b);
    if (!probe_generate_path(b.s, make_light(b.light), a, st, q, u - __ldg(m.prefix + lo), u)) return;
    RayTally none{0u, 0u};
    flush_tally(counters, none, 1u, a.n);
}

// Independent samples (NAN_BATCH_WAVEFRONT_INDEPENDENT): sample k of a probe
// draws from RNG(probe, instance, iteration * n + k) and is its own path, so a
// frame is max_bounces rounds; every finished path stores its sample, and a
// last pass folds each probe's samples in sample order, as the
// independent-sample persistent kernel does.
__global__ void __launch_bounds__(128) k_wfi_probe_generate(BatchWfArgs m, WfState st, WfQueues q) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m.units * m.n) return;
    const uint32_t uoff = p / m.n, k = p - uoff * m.n;
    const uint32_t u = m.unit_begin + uoff;
    const uint32_t set = batch_set_of_unit(m, u);
    m.set_of[p] = set;
    const BatchSet& b = m.sets[set];
    const uint32_t probe = u - __ldg(m.prefix + set);
    const ProbeArgs a = batch_probe_args(m, b);
    const uint4 meta = __ldg(reinterpret_cast<const uint4*>(a.probes) + 3u * probe + 2u);
    const uint32_t inst = meta.w >> 8;
    if (inst >= a.probe_instance_count || !valid_prim(b.s, inst, meta.x)) {
        atomicOr(b.s.status, kStatusBadRecord);
        ProbeSample none;
        none.si = mk3(0.0f, 0.0f, 0.0f);
        none.self_hits = 0u;
        none.texel = 0u;
        none.nd = 0.0f;
        none.has_path = false;
        m.samples[p] = none;
        return;
    }
    const float4 params = __ldg(a.pinst + 3u * inst + 2u);
    st.unit[p] = probe;
    st.surf[p] = make_float4(__uint_as_float(meta.y), __uint_as_float(meta.z), __uint_as_float(inst),
                             __uint_as_float(meta.x));
    st.si[p] = make_float4(0.0f, 0.0f, 0.0f, maxf(params.x, 1e-6f));
    st.pb[p] = make_uint4(0u, 0u, 0u, 0u);
    Rng rng(probe, inst, a.iteration * m.n + k);
    probe_start_sample(b.s, make_light(b.light), a, st, q, 0, q.ctl, p, 0u, rng);
    st.rng[p] = rng.state;
}

__global__ void __launch_bounds__(128) k_wfi_probe_finalize(BatchWfArgs m, WfState st, WfQueues q, int buf,
                                                            uint32_t* ctl, uint32_t* ctl_next) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t p = q.ext[buf][idx];
        const uint32_t flags = st.flags[p];
        if (!(flags & kFlagEnd)) {
            const uint32_t slot = queue_slot(ctl_next + 0, true);
            q.ext[buf ^ 1][slot] = p;
            continue;
        }
        ProbeSample r;
        r.si = mk3(0.0f, 0.0f, 0.0f);
        r.self_hits = 0u;
        r.texel = 0u;
        r.nd = 0.0f;
        r.has_path = !(flags & kFlagNoPath);
        if (r.has_path) {
            const uint4 b = st.pb[p];
            const float2 zp = st.zpdf[p];
            r.si = r.si + ((xyz(st.rad[p]) * zp.x) / zp.y);
            r.self_hits = b.x;
            r.texel = b.w;
            r.nd = st.pa[p].w / maxf(st.si[p].w, 1e-6f);
        }
        m.samples[p] = r;
    }
}

__global__ void __launch_bounds__(128) k_wfi_probe_fold(BatchWfArgs m, unsigned long long* counters) {
    const uint32_t uoff = blockIdx.x * blockDim.x + threadIdx.x;
    if (uoff >= m.units) return;
    const uint32_t u = m.unit_begin + uoff;
    const uint32_t set = batch_set_of_unit(m, u);
    const BatchSet& b = m.sets[set];
    const uint32_t probe = u - __ldg(m.prefix + set);
    const uint4 meta = __ldg(reinterpret_cast<const uint4*>(b.probes) + 3u * probe + 2u);
    const uint32_t inst = meta.w >> 8;
    if (inst >= b.probe_instance_count || !valid_prim(b.s, inst, meta.x)) return;
    const int reset = m.ctl->reset ? 1 : 0;
    const uint32_t prev_iter = reset ? 0u : b.out.counts[probe];
    if (reset)
        for (int t = 0; t < 16; ++t) b.out.radial[16u * probe + (uint32_t)t] = 0u;
    ProbeAcc acc;
    probe_acc_init(acc);
    for (uint32_t k = 0; k < m.n; ++k) probe_fold(acc, b.out, probe, m.samples[uoff * m.n + k], prev_iter, m.spp);
    probe_store(b.out, probe, acc, m.n, reset);
    RayTally none{0u, 0u};
    flush_tally(counters, none, 1u, m.n);
}

__global__ void __launch_bounds__(128, 6) k_wfb_probe_shade(BatchWfArgs m, WfState st, WfQueues q, int buf,
                                                         uint32_t* ctl) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t p = q.ext[buf][idx];
        const BatchSet& b = m.sets[m.set_of[p]];
        probe_shade_path(b.s, make_light(b.light), batch_probe_args(m, b), st, q, buf, ctl, p);
    }
}

__global__ void __launch_bounds__(128, 6) k_wfb_probe_finalize(BatchWfArgs m, WfState st, WfQueues q, int buf,
                                                            uint32_t* ctl, uint32_t* ctl_next) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < count; idx += gridDim.x * blockDim.x) {
        const uint32_t p = q.ext[buf][idx];
        const BatchSet& b = m.sets[m.set_of[p]];
        probe_finalize_path(b.s, make_light(b.light), batch_probe_args(m, b), st, q, buf, ctl_next, p);
    }
}

LightingRaw to_raw(const NanLighting* l) {
    LightingRaw r;
    memcpy(&r, l, sizeof(r));
    return r;
}

SceneView scene_view(const NanContext* ctx) {
    SceneView v;
    v.nodes = ctx->nodes;
    v.tris = ctx->tris;
    const bool wide = ctx->wide_built && ctx->wnodes != nullptr && ctx->tuning.bvh_width == 8;
    v.wnodes = wide ? ctx->wnodes : nullptr;
    v.wtris = wide ? ctx->wtris : nullptr;
    v.tri_refs = ctx->tri_refs;
    v.vertices = ctx->scene.vertices;
    v.indices = ctx->scene.indices;
    v.mesh_descs = reinterpret_cast<const uint4*>(ctx->scene.mesh_descs);
    v.instance_descs = reinterpret_cast<const uint4*>(ctx->scene.instance_descs);
    v.transforms = ctx->scene.transforms;
    v.inverse_transposes = ctx->scene.inverse_transposes;
    v.materials = ctx->scene.materials;
    v.root = ctx->root;
    v.tri_count = ctx->tri_count;
    v.instance_count = ctx->scene.instance_count;
    v.status = ctx->d_status;
    v.lights = reinterpret_cast<const float4*>(ctx->lights);
    v.light_count = ctx->lights ? ctx->light_count : 0u;
    v.light_power = ctx->light_power;
    return v;
}

template <class T> T* carve(unsigned char*& cur, size_t count) {
    T* p = reinterpret_cast<T*>(cur);
    cur += ((count * sizeof(T) + 255u) / 256u) * 256u;
    return p;
}

// Traversal launches of one wavefront round: node width from the scene,
// the traversal form from the context's tuning (NanTuning.traversal).
template <class Src>
void launch_extend(const NanContext* ctx, int blocks, cudaStream_t st, bool wide, Src src, const uint32_t* queue,
                   uint32_t* ctl, const WfState& S) {
#define NAN_EXT_ARGS src, queue, ctl, S.ro, S.rd, S.flags, S.hit, ctx->d_counters
    if (wide) k_wf_extend<8><<<blocks, 128, 0, st>>>(NAN_EXT_ARGS);
    else switch (ctx->tuning.traversal) {
        case 1: k_wf_extend_refill<8, 1, Src><<<blocks, 128, 0, st>>>(NAN_EXT_ARGS); break;
        case 2: k_wf_extend_refill<16, 1, Src><<<blocks, 128, 0, st>>>(NAN_EXT_ARGS); break;
        case 3: k_wf_extend_refill<24, 1, Src><<<blocks, 128, 0, st>>>(NAN_EXT_ARGS); break;
        case 4: k_wf_extend_refill<16, 4, Src><<<blocks, 128, 0, st>>>(NAN_EXT_ARGS); break;
        case 5: k_wf_extend<2, Src, 16><<<blocks, 128, 0, st>>>(NAN_EXT_ARGS); break;
        case 6: k_wf_extend<2, Src, 0, true><<<blocks, 128, 0, st>>>(NAN_EXT_ARGS); break;
        default: k_wf_extend<2><<<blocks, 128, 0, st>>>(NAN_EXT_ARGS); break;
    }
#undef NAN_EXT_ARGS
}

template <class Src>
void launch_shadow(const NanContext* ctx, int blocks, cudaStream_t st, bool wide, Src src, const float4* queue,
                   uint32_t* ctl, float t_max, const WfState& S) {
#define NAN_SHD_ARGS src, queue, ctl, t_max, S.rad, S.si, ctx->d_counters
    if (wide) k_wf_shadow<8><<<blocks, 128, 0, st>>>(NAN_SHD_ARGS);
    else switch (ctx->tuning.traversal) {
        case 1: k_wf_shadow_refill<8, 1, Src><<<blocks, 128, 0, st>>>(NAN_SHD_ARGS); break;
        case 2: k_wf_shadow_refill<16, 1, Src><<<blocks, 128, 0, st>>>(NAN_SHD_ARGS); break;
        case 3: k_wf_shadow_refill<24, 1, Src><<<blocks, 128, 0, st>>>(NAN_SHD_ARGS); break;
        case 4: k_wf_shadow_refill<16, 4, Src><<<blocks, 128, 0, st>>>(NAN_SHD_ARGS); break;
        case 5: k_wf_shadow<2, Src, 16><<<blocks, 128, 0, st>>>(NAN_SHD_ARGS); break;
        case 6: k_wf_shadow<2, Src, 0, true><<<blocks, 128, 0, st>>>(NAN_SHD_ARGS); break;
        default: k_wf_shadow<2><<<blocks, 128, 0, st>>>(NAN_SHD_ARGS); break;
    }
#undef NAN_SHD_ARGS
}

struct Grid {
    int persistent_blocks;
    int stream_blocks;
};

Grid grid_for(const NanContext* ctx) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_wf_extend<2, OneScene>, 128, 0);
    Grid g;
    const int per_sm = ctx->tuning.trace_blocks_per_sm ? (int)ctx->tuning.trace_blocks_per_sm : std::max(occ, 1);
    g.persistent_blocks = sms * per_sm;
    g.stream_blocks = sms * 16;
    return g;
}

}  // namespace

namespace nan_host {

size_t wavefront_bytes_per_path() { return kBytesPerPath + 64; }

namespace {
cudaEvent_t pooled_event(NanContext* ctx) {
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}
}  // namespace

cudaEvent_t timing_begin(NanContext* ctx, cudaStream_t stream) {
    if (!ctx->tuning.kernel_timing) return nullptr;
    cudaEvent_t e = pooled_event(ctx);
    if (e && cudaEventRecord(e, stream) != cudaSuccess) {
        ctx->event_pool.push_back(e);
        return nullptr;
    }
    return e;
}

void timing_end(NanContext* ctx, int kind, cudaEvent_t start, cudaStream_t stream) {
    if (!start) return;
    cudaEvent_t e = pooled_event(ctx);
    if (!e || cudaEventRecord(e, stream) != cudaSuccess) {
        ctx->event_pool.push_back(start);
        if (e) ctx->event_pool.push_back(e);
        return;
    }
    ctx->timed.push_back({kind, start, e});
}

int read_kernel_times(NanContext* ctx, NanKernelTimes* out, int reset) {
    cudaError_t first = cudaSuccess;
    for (const NanContext::TimedLaunch& t : ctx->timed) {
        float ms = 0.0f;
        cudaError_t err = cudaEventSynchronize(t.stop);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, t.start, t.stop);
        if (err == cudaSuccess) {
            ctx->stage_ms[t.kind] += ms;
            ctx->stage_launches[t.kind]++;
        } else if (first == cudaSuccess) {
            first = err;
        }
        ctx->event_pool.push_back(t.start);
        ctx->event_pool.push_back(t.stop);
    }
    ctx->timed.clear();
    if (out) {
        out->extend_ms = ctx->stage_ms[0];
        out->shadow_ms = ctx->stage_ms[1];
        out->stage_ms = ctx->stage_ms[2];
        out->extend_launches = ctx->stage_launches[0];
        out->shadow_launches = ctx->stage_launches[1];
        out->stage_launches = ctx->stage_launches[2];
    }
    if (reset) {
        for (int k = 0; k < 3; ++k) {
            ctx->stage_ms[k] = 0.0;
            ctx->stage_launches[k] = 0;
        }
    }
    return cuda_fail(first, "kernel timing events");
}

void release_timing(NanContext* ctx) {
    for (const NanContext::TimedLaunch& t : ctx->timed) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
    }
    ctx->timed.clear();
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    ctx->event_pool.clear();
}

// Scratch plan shared by the integrators: control words for `iters`
// iterations plus as many paths as the arena holds (or the tuning cap).
int wf_plan(NanContext* ctx, uint64_t iters64, uint32_t* iters, uint64_t* cap) {
    if (iters64 > (1u << 20)) {
        set_error("samples * bounces too large for the wavefront schedule");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    *iters = (uint32_t)iters64;
    const size_t ctl_bytes = ((size_t)(*iters + 2) * 20 * sizeof(uint32_t) + 255u) / 256u * 256u;
    if (ctx->scratch_bytes <= ctl_bytes + 8192) {
        set_error("no wavefront scratch reserved on this context (nan_ctx_reserve)");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    *cap = (ctx->scratch_bytes - ctl_bytes - 8192) / wavefront_bytes_per_path();
    if (ctx->tuning.max_paths_in_flight) *cap = std::min<uint64_t>(*cap, ctx->tuning.max_paths_in_flight);
    if (*cap == 0) {
        set_error("wavefront scratch too small for one path");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    return NAN_OK;
}

void wf_carve(NanContext* ctx, uint32_t count, uint32_t iters, WfState& S, WfQueues& q) {
    unsigned char* cur = static_cast<unsigned char*>(ctx->scratch);
    q.ctl = carve<uint32_t>(cur, (size_t)(iters + 2) * 20);
    q.oct = q.ctl + (size_t)(iters + 2) * 4;
    S.unit = carve<uint32_t>(cur, count);
    S.rng = carve<uint32_t>(cur, count);
    S.flags = carve<uint32_t>(cur, count);
    S.surf = carve<float4>(cur, count);
    S.ro = carve<float4>(cur, count);
    S.rd = carve<float4>(cur, count);
    S.thp = carve<float4>(cur, count);
    S.rad = carve<float4>(cur, count);
    S.si = carve<float4>(cur, count);
    S.irr = carve<float4>(cur, count);
    S.zpdf = carve<float2>(cur, count);
    S.hit = carve<float4>(cur, count);
    S.pa = carve<float4>(cur, count);
    S.pb = carve<uint4>(cur, count);
    S.pc = carve<uint4>(cur, 2ull * count);
    q.ext[0] = carve<uint32_t>(cur, count);
    q.ext[1] = carve<uint32_t>(cur, count);
    q.ext_sorted = carve<uint32_t>(cur, count);
    q.shd[0] = carve<float4>(cur, 3ull * 2 * count);
    q.shd[1] = carve<float4>(cur, 3ull * 2 * count);
}

// Runs units [begin, end) in chunks: generate, then `iters` rounds of
// extend / shade / shadow / finalize. gen(S, q, first_unit, count),
// shade(S, q, buf, ctl) and fin(S, q, buf, ctl, ctl_next) launch the
// integrator's own stages.
template <class Gen, class Shade, class Fin>
int wf_run(NanContext* ctx, cudaStream_t st, uint64_t begin, uint64_t end, uint32_t iters, uint64_t cap, float t_max,
           Gen gen, Shade shade, Fin fin) {
    const SceneView s = scene_view(ctx);
    const Grid g = grid_for(ctx);
    for (uint64_t cb = begin; cb < end; cb += cap) {
        const uint32_t count = (uint32_t)std::min<uint64_t>(cap, end - cb);
        WfState S;
        WfQueues q;
        wf_carve(ctx, count, iters, S, q);
        cudaError_t err = cudaMemsetAsync(q.ctl, 0, (size_t)(iters + 2) * 20 * sizeof(uint32_t), st);
        if (err != cudaSuccess) return cuda_fail(err, "wavefront control reset");
        cudaEvent_t ev = timing_begin(ctx, st);
        gen(S, q, (uint32_t)cb, count);
        timing_end(ctx, 2, ev, st);
        ctx->launches++;
        for (uint32_t it = 0; it < iters; ++it) {
            const int buf = (int)(it & 1u);
            uint32_t* ctl = q.ctl + 4u * it;
            if (ctx->tuning.ray_order == 1u) {
                ev = timing_begin(ctx, st);
                uint32_t* oct = q.oct + 16u * it;
                k_wf_octant_count<<<g.stream_blocks, 256, 0, st>>>(q.ext[buf], ctl, S.rd, oct);
                k_wf_octant_place<<<g.stream_blocks, 256, 0, st>>>(q.ext[buf], ctl, S.rd, oct, q.ext_sorted);
                timing_end(ctx, 2, ev, st);
                std::swap(q.ext[buf], q.ext_sorted);
                ctx->launches += 2;
            }
            ev = timing_begin(ctx, st);
            launch_extend(ctx, g.persistent_blocks, st, s.wnodes != nullptr, OneScene{s}, q.ext[buf], ctl, S);
            timing_end(ctx, 0, ev, st);
            ev = timing_begin(ctx, st);
            shade(S, q, buf, ctl);
            timing_end(ctx, 2, ev, st);
            ev = timing_begin(ctx, st);
            launch_shadow(ctx, g.persistent_blocks, st, s.wnodes != nullptr, OneScene{s}, q.shd[buf], ctl, t_max, S);
            timing_end(ctx, 1, ev, st);
            ev = timing_begin(ctx, st);
            fin(S, q, buf, ctl, ctl + 4);
            timing_end(ctx, 2, ev, st);
            ctx->launches += 4;
        }
        err = cudaGetLastError();
        if (err != cudaSuccess) return cuda_fail(err, "wavefront launch");
    }
    return NAN_OK;
}

int launch_trace_texels_wavefront(NanContext* ctx, const NanMeshColorsDesc* lay, uint8_t* slots,
                                  uint32_t iteration, uint32_t spt, uint32_t max_bounces, int reset,
                                  const NanLighting* light, uint32_t begin, uint32_t end, cudaStream_t st) {
    if (end <= begin) return NAN_OK;
    const uint32_t n = std::max(spt, 1u);
    uint32_t iters = 0;
    uint64_t cap = 0;
    // a path may run its back side after its front: 2 sides x n samples x bounces
    int rc = wf_plan(ctx, 2ull * n * std::max(max_bounces, 1u), &iters, &cap);
    if (rc) return rc;
    const SceneView s = scene_view(ctx);
    const LightingRaw lr = to_raw(light);
    TexelArgs a;
    memset(&a, 0, sizeof(a));
    a.mc.compensation = reinterpret_cast<float4*>(lay->compensation);
    a.mc.face_infos = reinterpret_cast<const uint2*>(lay->face_infos);
    a.mc.instance_infos = reinterpret_cast<const uint4*>(lay->instance_infos);
    a.mc.side_infos = reinterpret_cast<const uint2*>(lay->side_infos);
    a.mc.surface_prefix = lay->surface_prefix;
    a.mc.instance_count = lay->instance_count;
    a.mc.payload_count = lay->payload_count;
    a.slots = reinterpret_cast<uint4*>(slots);
    a.iteration = iteration;
    a.n = n;
    a.max_bounces = std::max(max_bounces, 1u);
    a.reset = reset;
    const Grid g = grid_for(ctx);
    unsigned long long* counters = ctx->d_counters;
    return wf_run(
        ctx, st, begin, end, iters, cap, lr.ray_t_max,
        [&](const WfState& S, const WfQueues& q, uint32_t first, uint32_t count) {
            k_wf_texel_generate<<<(count + 127) / 128, 128, 0, st>>>(s, lr, a, S, q, first, count, counters);
        },
        [&](const WfState& S, const WfQueues& q, int buf, uint32_t* ctl) {
            k_wf_texel_shade<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl);
        },
        [&](const WfState& S, const WfQueues& q, int buf, uint32_t* ctl, uint32_t* ctl_next) {
            k_wf_texel_finalize<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl, ctl_next);
        });
}

namespace {
int screen_wavefront(NanContext* ctx, float* out, uint32_t w, uint32_t h, uint32_t frame, uint32_t max_vertices,
                     const NanCamera* cam, const NanLighting* light, const CachedArgs* cached, cudaStream_t st);
}  // namespace

int launch_trace_screen_wavefront(NanContext* ctx, float* out, uint32_t w, uint32_t h, uint32_t frame,
                                  uint32_t max_vertices, const NanCamera* cam, const NanLighting* light,
                                  cudaStream_t st) {
    return screen_wavefront(ctx, out, w, h, frame, max_vertices, cam, light, nullptr, st);
}

int launch_trace_screen_cached(NanContext* ctx, NanCache* cache, float* out, uint32_t w, uint32_t h,
                               uint32_t frame, const NanCamera* cam, const NanLighting* light,
                               const NanCachedFrame* fd, cudaStream_t st) {
    CachedArgs c;
    c.queries = reinterpret_cast<float4*>(fd->queries);
    c.weights = reinterpret_cast<float4*>(fd->query_weights);
    c.query_count = fd->query_count;
    c.train_points = reinterpret_cast<float4*>(fd->train_points);
    c.train_queries = reinterpret_cast<float4*>(fd->train_queries);
    c.train_count = fd->train_count;
    c.train_offset = fd->train_offset;
    c.train_inverse = fd->train_stride_inverse;
    c.vertex = fd->cache_vertex;
    cudaError_t err = cudaMemsetAsync(fd->query_count, 0, sizeof(uint32_t), st);
    if (err == cudaSuccess && fd->train_count)
        err = cudaMemsetAsync(fd->train_points, 0xff, (size_t)fd->train_count * 16u, st);
    if (err != cudaSuccess) return cuda_fail(err, "cached frame reset");
    int rc = screen_wavefront(ctx, out, w, h, frame, fd->cache_vertex + 1u, cam, light, &c, st);
    if (rc) return rc;
    return launch_cache_infer(cache, fd->queries, w * h, fd->query_count, nullptr, fd->query_weights, out, st);
}

int launch_trace_points_wavefront(NanContext* ctx, const float* points, uint32_t count, float* out,
                                  uint32_t iteration, uint32_t samples, uint32_t max_bounces, uint32_t flags,
                                  const NanLighting* light, cudaStream_t st) {
    if (count == 0) return NAN_OK;
    const uint32_t n = std::max(samples, 1u);
    uint32_t iters = 0;
    uint64_t cap = 0;
    int rc = wf_plan(ctx, (uint64_t)n * std::max(max_bounces, 1u), &iters, &cap);
    if (rc) return rc;
    const SceneView s = scene_view(ctx);
    const LightingRaw lr = to_raw(light);
    TexelArgs a;
    memset(&a, 0, sizeof(a));
    a.iteration = iteration;
    a.n = n;
    a.max_bounces = std::max(max_bounces, 1u);
    a.points = reinterpret_cast<const float4*>(points);
    a.point_out = reinterpret_cast<float4*>(out);
    a.indirect_only = (flags & NAN_POINTS_INDIRECT_ONLY) != 0u;
    const Grid g = grid_for(ctx);
    unsigned long long* counters = ctx->d_counters;
    return wf_run(
        ctx, st, 0, count, iters, cap, lr.ray_t_max,
        [&](const WfState& S, const WfQueues& q, uint32_t first, uint32_t cnt) {
            k_wf_point_generate<<<(cnt + 127) / 128, 128, 0, st>>>(s, lr, a, S, q, first, cnt, counters);
        },
        [&](const WfState& S, const WfQueues& q, int buf, uint32_t* ctl) {
            k_wf_texel_shade<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl);
        },
        [&](const WfState& S, const WfQueues& q, int buf, uint32_t* ctl, uint32_t* ctl_next) {
            k_wf_texel_finalize<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl, ctl_next);
        });
}

namespace {
int screen_wavefront(NanContext* ctx, float* out, uint32_t w, uint32_t h, uint32_t frame, uint32_t max_vertices,
                     const NanCamera* cam, const NanLighting* light, const CachedArgs* cached, cudaStream_t st) {
    const uint64_t pixels = (uint64_t)w * h;
    if (pixels == 0 || max_vertices == 0) return NAN_OK;
    uint32_t iters = 0;
    uint64_t cap = 0;
    int rc = wf_plan(ctx, max_vertices, &iters, &cap);
    if (rc) return rc;
    const SceneView s = scene_view(ctx);
    const LightingRaw lr = to_raw(light);
    ScreenArgs a;
    memcpy(&a.cam, cam, sizeof(a.cam));
    a.out = reinterpret_cast<float4*>(out);
    a.width = w;
    a.height = h;
    a.frame = frame;
    a.max_vertices = max_vertices;
    a.cached = cached != nullptr;
    a.area_nee = (light->flags & 2u) != 0u;
    if (cached) a.cache = *cached;
    else memset(&a.cache, 0, sizeof(a.cache));
    const Grid g = grid_for(ctx);
    unsigned long long* counters = ctx->d_counters;
    return wf_run(
        ctx, st, 0, pixels, iters, cap, lr.ray_t_max,
        [&](const WfState& S, const WfQueues& q, uint32_t first, uint32_t count) {
            k_wf_screen_generate<<<(count + 127) / 128, 128, 0, st>>>(s, lr, a, S, q, first, count, counters);
        },
        [&](const WfState& S, const WfQueues& q, int buf, uint32_t* ctl) {
            k_wf_screen_shade<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl);
        },
        [&](const WfState& S, const WfQueues& q, int buf, uint32_t* ctl, uint32_t* ctl_next) {
            k_wf_screen_finalize<<<g.stream_blocks, 128, 0, st>>>(a, S, q, buf, ctl, ctl_next);
        });
}
}  // namespace

size_t probe_sample_bytes() { return sizeof(ProbeSample); }

const void* wavefront_extend_kernel() { return reinterpret_cast<const void*>(&k_wf_extend<2, ManyScenes>); }

// The multi-scene probe batch on the wavefront: generate every (set, probe)
// unit as one path, then n * max_bounces rounds of extend / shade / shadow /
// finalize over all sets, with no host synchronisation (capturable). The
// context's scratch must hold `total` paths.
int launch_batch_wavefront(NanContext* ctx, const void* sets, const uint32_t* prefix, const void* batch_ctl,
                           uint32_t set_count, uint32_t total, uint32_t* set_of, uint32_t spp, uint32_t max_bounces,
                           float t_max, cudaStream_t st) {
    if (total == 0) return NAN_OK;
    const uint32_t n = std::max(spp, 1u);
    uint32_t iters = 0;
    uint64_t cap = 0;
    int rc = wf_plan(ctx, (uint64_t)n * std::max(max_bounces, 1u), &iters, &cap);
    if (rc) return rc;
    if (cap < total) {
        set_error("batch wavefront scratch holds fewer paths than the batch has probes");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    BatchWfArgs m;
    m.sets = static_cast<const BatchSet*>(sets);
    m.prefix = prefix;
    m.ctl = static_cast<const BatchCtl*>(batch_ctl);
    m.set_of = set_of;
    m.set_count = set_count;
    m.total = total;
    m.n = n;
    m.spp = spp;
    m.max_bounces = std::max(max_bounces, 1u);
    m.unit_begin = 0u;
    m.units = total;
    m.samples = nullptr;
    const ManyScenes src{m.sets, set_of};
    const Grid g = grid_for(ctx);
    WfState S;
    WfQueues q;
    wf_carve(ctx, total, iters, S, q);
    cudaError_t err = cudaMemsetAsync(q.ctl, 0, (size_t)(iters + 2) * 20 * sizeof(uint32_t), st);
    if (err != cudaSuccess) return cuda_fail(err, "batch wavefront control reset");
    k_wfb_probe_generate<<<(total + 127) / 128, 128, 0, st>>>(m, S, q, ctx->d_counters);
    ctx->launches++;
    for (uint32_t it = 0; it < iters; ++it) {
        const int buf = (int)(it & 1u);
        uint32_t* ctl = q.ctl + 4u * it;
        launch_extend(ctx, g.persistent_blocks, st, false, src, q.ext[buf], ctl, S);
        k_wfb_probe_shade<<<g.stream_blocks, 128, 0, st>>>(m, S, q, buf, ctl);
        launch_shadow(ctx, g.persistent_blocks, st, false, src, q.shd[buf], ctl, t_max, S);
        k_wfb_probe_finalize<<<g.stream_blocks, 128, 0, st>>>(m, S, q, buf, ctl, ctl + 4);
        ctx->launches += 4;
    }
    return cuda_fail(cudaGetLastError(), "batch wavefront launch");
}

int launch_batch_wavefront_independent(NanContext* ctx, const void* sets, const uint32_t* prefix,
                                       const void* batch_ctl, uint32_t set_count, uint32_t total, uint32_t* set_of,
                                       void* samples, uint64_t path_capacity, uint32_t spp, uint32_t max_bounces,
                                       float t_max, cudaStream_t st) {
    if (total == 0) return NAN_OK;
    const uint32_t n = std::max(spp, 1u);
    uint32_t iters = 0;
    uint64_t cap = 0;
    int rc = wf_plan(ctx, std::max(max_bounces, 1u), &iters, &cap);
    if (rc) return rc;
    cap = std::min(cap, path_capacity);
    const uint64_t chunk_units = cap / n;
    if (chunk_units == 0) {
        set_error("batch wavefront scratch holds fewer paths than one probe's samples");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    BatchWfArgs m;
    m.sets = static_cast<const BatchSet*>(sets);
    m.prefix = prefix;
    m.ctl = static_cast<const BatchCtl*>(batch_ctl);
    m.set_of = set_of;
    m.set_count = set_count;
    m.total = total;
    m.n = n;
    m.spp = spp;
    m.max_bounces = std::max(max_bounces, 1u);
    m.samples = static_cast<ProbeSample*>(samples);
    const ManyScenes src{m.sets, set_of};
    const Grid g = grid_for(ctx);
    for (uint64_t ub = 0; ub < total; ub += chunk_units) {
        m.unit_begin = (uint32_t)ub;
        m.units = (uint32_t)std::min<uint64_t>(chunk_units, total - ub);
        const uint32_t paths = m.units * n;
        WfState S;
        WfQueues q;
        wf_carve(ctx, paths, iters, S, q);
        cudaError_t err = cudaMemsetAsync(q.ctl, 0, (size_t)(iters + 2) * 20 * sizeof(uint32_t), st);
        if (err != cudaSuccess) return cuda_fail(err, "batch wavefront control reset");
        k_wfi_probe_generate<<<(paths + 127) / 128, 128, 0, st>>>(m, S, q);
        for (uint32_t it = 0; it < iters; ++it) {
            const int buf = (int)(it & 1u);
            uint32_t* ctl = q.ctl + 4u * it;
            launch_extend(ctx, g.persistent_blocks, st, false, src, q.ext[buf], ctl, S);
            k_wfb_probe_shade<<<g.stream_blocks, 128, 0, st>>>(m, S, q, buf, ctl);
            launch_shadow(ctx, g.persistent_blocks, st, false, src, q.shd[buf], ctl, t_max, S);
            k_wfi_probe_finalize<<<g.stream_blocks, 128, 0, st>>>(m, S, q, buf, ctl, ctl + 4);
        }
        k_wfi_probe_fold<<<(m.units + 127) / 128, 128, 0, st>>>(m, ctx->d_counters);
        ctx->launches += 2 + 4ull * iters;
    }
    return cuda_fail(cudaGetLastError(), "batch wavefront launch");
}

int launch_trace_probes_wavefront(NanContext* ctx, float* values, uint32_t* counts, uint32_t* self_hits,
                                  uint32_t* radial, const uint8_t* probes, uint32_t probe_count,
                                  const uint8_t* probe_instances, uint32_t probe_instance_count, uint32_t iteration,
                                  uint32_t spp, uint32_t max_bounces, int reset, const NanLighting* light,
                                  uint32_t begin, uint32_t end, float* compensation, cudaStream_t st) {
    end = std::min(end, probe_count);
    if (end <= begin) return NAN_OK;
    const uint32_t n = std::max(spp, 1u);
    uint32_t iters = 0;
    uint64_t cap = 0;
    int rc = wf_plan(ctx, (uint64_t)n * std::max(max_bounces, 1u), &iters, &cap);
    if (rc) return rc;
    const SceneView s = scene_view(ctx);
    const LightingRaw lr = to_raw(light);
    ProbeArgs a;
    a.out = ProbeOut{reinterpret_cast<float4*>(compensation), values, counts, self_hits, radial};
    a.probes = reinterpret_cast<const float4*>(probes);
    a.pinst = reinterpret_cast<const float4*>(probe_instances);
    a.probe_instance_count = probe_instance_count;
    a.iteration = iteration;
    a.n = n;
    a.spp = spp;
    a.max_bounces = std::max(max_bounces, 1u);
    a.reset = reset;
    const Grid g = grid_for(ctx);
    unsigned long long* counters = ctx->d_counters;
    return wf_run(
        ctx, st, begin, end, iters, cap, lr.ray_t_max,
        [&](const WfState& S, const WfQueues& q, uint32_t first, uint32_t count) {
            k_wf_probe_generate<<<(count + 127) / 128, 128, 0, st>>>(s, lr, a, S, q, first, count, counters);
        },
        [&](const WfState& S, const WfQueues& q, int buf, uint32_t* ctl) {
            k_wf_probe_shade<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl);
        },
        [&](const WfState& S, const WfQueues& q, int buf, uint32_t* ctl, uint32_t* ctl_next) {
            k_wf_probe_finalize<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl, ctl_next);
        });
}

}  // namespace nan_host
