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
constexpr uint32_t kKindSun = 1u;  // shadow contribution goes to si

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
};

struct WfQueues {
    uint32_t* ext[2];
    float4* shd[2];  // 3 float4 per entry: (o, path bits), (d, kind bits), (c, 0)
    uint32_t* ctl;   // per iteration k: [4k] ext count, [4k+1] ext fetch, [4k+2] shd count, [4k+3] shd fetch
};

constexpr size_t kBytesPerPath = 4 + 4 + 4 + 16 * 9 + 8 + 2 * 4 + 2 * 2 * 48;

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

__device__ __forceinline__ void push_shadow(const WfQueues& q, int buf, uint32_t* count, uint32_t p, f3 o, f3 d,
                                            f3 c, uint32_t kind) {
    const uint32_t slot = queue_slot(count, true);
    float4* e = q.shd[buf] + 3u * slot;
    e[0] = make_float4(o.x, o.y, o.z, __uint_as_float(p));
    e[1] = make_float4(d.x, d.y, d.z, __uint_as_float(kind));
    e[2] = make_float4(c.x, c.y, c.z, 0.0f);
}

__device__ __forceinline__ f3 xyz(float4 v) { return mk3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 f4(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// ---------------------------------------------------------------------------
// Generic traversal stages.
// ---------------------------------------------------------------------------
template <int kWidth>
__global__ void __launch_bounds__(128) k_wf_extend(SceneView s, const uint32_t* __restrict__ queue,
                                                   uint32_t* ctl, const float4* __restrict__ ro,
                                                   const float4* __restrict__ rd, const uint32_t* __restrict__ flags,
                                                   float4* __restrict__ hit, unsigned long long* counters) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 0);
    const uint32_t lane = threadIdx.x & 31u;
    RayTally tally{0u, 0u};
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
                const float4 o = ro[p], d = rd[p];
                tally.extend++;
                const HitInfo h = trace_closest_w<kWidth>(s, xyz(o), xyz(d), o.w, d.w);
                hit[p] = make_float4(__uint_as_float(h.valid ? h.flat : 0xffffffffu), h.t, h.b1, h.b2);
            }
        }
    }
    flush_tally(counters, tally, 0u, 0u);
}

template <int kWidth>
__global__ void __launch_bounds__(128) k_wf_shadow(SceneView s, const float4* __restrict__ queue, uint32_t* ctl,
                                                   float t_max, float4* __restrict__ rad, float4* __restrict__ si,
                                                   unsigned long long* counters) {
    const uint32_t count = *(volatile uint32_t*)(ctl + 2);
    const uint32_t lane = threadIdx.x & 31u;
    RayTally tally{0u, 0u};
    for (;;) {
        uint32_t base = 0u;
        if (lane == 0u) base = atomicAdd(ctl + 3, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t idx = base + lane;
        if (idx < count) {
            const float4 a = queue[3u * idx], b = queue[3u * idx + 1u], c = queue[3u * idx + 2u];
            tally.shadow++;
            if (!trace_any_w<kWidth>(s, xyz(a), xyz(b), 0.0f, t_max)) {
                const uint32_t p = __float_as_uint(a.w);
                float4* target = (__float_as_uint(b.w) == kKindNee) ? rad : si;
                const float4 v = target[p];
                target[p] = make_float4(v.x + c.x, v.y + c.y, v.z + c.z, v.w);
            }
        }
    }
    flush_tally(counters, tally, 0u, 0u);
}

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
};

// Start sample k of the current side: sun irradiance shadow ray, first
// direction (estimate_surface_irradiance, texture_space_path_tracer.slang:95-113).
__device__ __forceinline__ void texel_start_sample(const SceneView& s, const LightParams& L, const WfState& st,
                                                   const WfQueues& q, int buf, uint32_t* ctl_next, uint32_t p,
                                                   uint32_t flags, Rng& rng) {
    const float4 sf = st.surf[p];
    const uint32_t inst = __float_as_uint(sf.z), prim = __float_as_uint(sf.w);
    f3 view = world_flat_normal(s, inst, prim);
    if (flags & kFlagBack) view = -view;
    const Shading sd = shading_data(s, inst, prim, sf.x, sf.y, view);
    const float u0 = rng.next_1d(), u1 = rng.next_1d();
    const f3 l = sample_cone_direction(L.sun_dir, L.cos_half, u0, u1);
    const float ndl = maxf(0.0f, dot3(sd.frame.n, l));
    push_shadow(q, buf, ctl_next + 2, p, sd.origin_front, l, L.illum * ndl, kKindSun);
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

__global__ void __launch_bounds__(128) k_wf_texel_generate(SceneView s, LightingRaw lraw, TexelArgs a, WfState st,
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

// One bounce of trace_radiance (texture_space_path_tracer.slang:60-83) after
// the extend stage found the hit.
__global__ void __launch_bounds__(128) k_wf_texel_shade(SceneView s, LightingRaw lraw, TexelArgs a, WfState st,
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
            rad = rad + thp * L.sky;
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
__global__ void __launch_bounds__(128) k_wf_texel_finalize(SceneView s, LightingRaw lraw, TexelArgs a, WfState st,
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
            texel_start_sample(s, L, st, q, nbuf, ctl_next, p, flags, rng);
            st.rng[p] = rng.state;
            continue;
        }
        // side complete: running mean into its slot
        const uint32_t u = st.unit[p];
        const uint32_t inst = __float_as_uint(st.surf[p].z);
        const uint4 info = __ldg(a.mc.instance_infos + inst);
        const uint2 side = __ldg(a.mc.side_infos + inst);
        const uint32_t global_texel = info.z + (u - __ldg(a.mc.surface_prefix + inst));
        const uint32_t slot = (flags & kFlagBack) ? side.x + (global_texel - info.z) : global_texel;
        if (slot < a.mc.payload_count) store_running_mean(a.slots, slot, irr / (float)a.n, a.reset);
        else atomicOr(s.status, 2u);
        if (!(flags & kFlagBack) && (flags & kFlagTwoSided)) {
            flags = (flags & ((1u << kSampleShift) - 1u)) | kFlagBack;
            st.irr[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            texel_start_sample(s, L, st, q, nbuf, ctl_next, p, flags, rng);
            st.rng[p] = rng.state;
        }
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
    const bool wide = ctx->wnodes != nullptr && ctx->tuning.bvh_width == 8;
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
    return v;
}

template <class T> T* carve(unsigned char*& cur, size_t count) {
    T* p = reinterpret_cast<T*>(cur);
    cur += ((count * sizeof(T) + 255u) / 256u) * 256u;
    return p;
}

struct Grid {
    int persistent_blocks;
    int stream_blocks;
};

Grid grid_for(const NanContext* ctx) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_wf_extend<2>, 128, 0);
    Grid g;
    const int per_sm = ctx->tuning.trace_blocks_per_sm ? (int)ctx->tuning.trace_blocks_per_sm : std::max(occ, 1);
    g.persistent_blocks = sms * per_sm;
    g.stream_blocks = sms * 16;
    return g;
}

}  // namespace

namespace nan_host {

size_t wavefront_bytes_per_path() { return kBytesPerPath + 64; }

int launch_trace_texels_wavefront(NanContext* ctx, const NanMeshColorsDesc* lay, uint8_t* slots,
                                  uint32_t iteration, uint32_t spt, uint32_t max_bounces, int reset,
                                  const NanLighting* light, uint32_t begin, uint32_t end, cudaStream_t st) {
    if (end <= begin) return NAN_OK;
    const uint32_t n = std::max(spt, 1u);
    const uint32_t sides = 2u;  // a path may run its back side after its front
    const uint64_t iters64 = (uint64_t)sides * n * std::max(max_bounces, 1u);
    if (iters64 > (1u << 20)) {
        set_error("samples_per_texel * max_bounces too large for the wavefront schedule");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    const uint32_t iters = (uint32_t)iters64;
    const size_t ctl_bytes = ((size_t)(iters + 2) * 4 * sizeof(uint32_t) + 255u) / 256u * 256u;
    if (ctx->scratch_bytes <= ctl_bytes + 8192) {
        set_error("no wavefront scratch reserved on this context (nan_ctx_reserve)");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    uint64_t cap = (ctx->scratch_bytes - ctl_bytes - 8192) / wavefront_bytes_per_path();
    if (ctx->tuning.max_paths_in_flight) cap = std::min<uint64_t>(cap, ctx->tuning.max_paths_in_flight);
    if (cap == 0) {
        set_error("wavefront scratch too small for one path");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    const SceneView s = scene_view(ctx);
    const LightingRaw lr = to_raw(light);
    TexelArgs a;
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
    for (uint64_t cb = begin; cb < end; cb += cap) {
        const uint32_t count = (uint32_t)std::min<uint64_t>(cap, end - cb);
        unsigned char* cur = static_cast<unsigned char*>(ctx->scratch);
        WfQueues q;
        q.ctl = carve<uint32_t>(cur, (size_t)(iters + 2) * 4);
        WfState S;
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
        q.ext[0] = carve<uint32_t>(cur, count);
        q.ext[1] = carve<uint32_t>(cur, count);
        q.shd[0] = carve<float4>(cur, 3ull * 2 * count);
        q.shd[1] = carve<float4>(cur, 3ull * 2 * count);
        cudaError_t err = cudaMemsetAsync(q.ctl, 0, (size_t)(iters + 2) * 4 * sizeof(uint32_t), st);
        if (err != cudaSuccess) return cuda_fail(err, "wavefront control reset");
        k_wf_texel_generate<<<(count + 127) / 128, 128, 0, st>>>(s, lr, a, S, q, (uint32_t)cb, count, ctx->d_counters);
        ctx->launches++;
        for (uint32_t it = 0; it < iters; ++it) {
            const int buf = (int)(it & 1u);
            uint32_t* ctl = q.ctl + 4u * it;
            if (s.wnodes)
                k_wf_extend<8><<<g.persistent_blocks, 128, 0, st>>>(s, q.ext[buf], ctl, S.ro, S.rd, S.flags, S.hit,
                                                                   ctx->d_counters);
            else
                k_wf_extend<2><<<g.persistent_blocks, 128, 0, st>>>(s, q.ext[buf], ctl, S.ro, S.rd, S.flags, S.hit,
                                                                   ctx->d_counters);
            k_wf_texel_shade<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl);
            if (s.wnodes)
                k_wf_shadow<8><<<g.persistent_blocks, 128, 0, st>>>(s, q.shd[buf], ctl, lr.ray_t_max, S.rad, S.si,
                                                                   ctx->d_counters);
            else
                k_wf_shadow<2><<<g.persistent_blocks, 128, 0, st>>>(s, q.shd[buf], ctl, lr.ray_t_max, S.rad, S.si,
                                                                   ctx->d_counters);
            k_wf_texel_finalize<<<g.stream_blocks, 128, 0, st>>>(s, lr, a, S, q, buf, ctl, ctl + 4);
            ctx->launches += 4;
        }
        err = cudaGetLastError();
        if (err != cudaSuccess) return cuda_fail(err, "wavefront texel launch");
    }
    return NAN_OK;
}

}  // namespace nan_host
