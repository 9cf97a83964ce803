// nan_trace.cu -- ray queries, the three integrators, accumulation, RGB9E5.
// Compiled with --fmad=false (see nan_math.cuh).
#include <cuda_fp16.h>

#include <algorithm>

#include <cmath>

#include "nan_internal.h"
#include "nan_scene.cuh"
#include "nan_sinks.cuh"
#include "nan_probe.cuh"
#include "nan_probe_gather.cuh"

namespace {

using namespace nbd;
using nan_host::cuda_fail;
using nan_host::set_error;

struct CameraRaw {  // layout of NanCamera
    float position[3];
    float jitter_x;
    float image_u[3];
    float jitter_y;
    float image_v[3];
    float near_clip;
    float image_w[3];
    float far_clip;
};

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

__device__ __forceinline__ HitInfo closest(const SceneView& s, f3 o, f3 d, float tmin, float tmax, RayTally& t) {
    t.extend++;
    return trace_closest(s, o, d, tmin, tmax);
}

// ---------------------------------------------------------------------------
// Ray queries.
// ---------------------------------------------------------------------------
__global__ void k_intersect(SceneView s, const float4* __restrict__ rays, uint32_t n, uint4* __restrict__ ids,
                            float* __restrict__ tb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = rays[2u * i], b = rays[2u * i + 1];
    const HitInfo h = trace_closest(s, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), a.w, b.w);
    uint2 ref = make_uint2(0u, 0u);
    if (h.valid) ref = __ldg(s.tri_refs + h.flat);
    ids[i] = make_uint4(h.valid ? 1u : 0u, ref.x, ref.y, h.valid ? h.flat : 0xffffffffu);
    tb[3u * i + 0] = h.valid ? h.t : 0.0f;
    tb[3u * i + 1] = h.b1;
    tb[3u * i + 2] = h.b2;
}

__global__ void k_occluded(SceneView s, const float4* __restrict__ rays, uint32_t n, float* __restrict__ vis) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = rays[2u * i], b = rays[2u * i + 1];
    vis[i] = trace_any(s, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), a.w, b.w) ? 0.0f : 1.0f;
}


// ---------------------------------------------------------------------------
// PMR visibility caster (vertex_baker/cpp/tinybvh_visibility.cpp:145-230):
// per sample, the table's rays leave position + normalize(normal) * bias (a
// zero or non-finite normal: (0,0,1) and an origin one float nearer each
// ray, as tinybvh has no t_min) and are tested for any hit in
// [0, t_max]. One warp per sample: lanes take rays r = lane + 32 w, a ballot
// per 32 rays leaves mask word w in lane w; lanes 0-15 then sum coefficient
// `lane` of the unoccluded rays' weighted SH in the caster's order (64-ray
// batches, each summed in ray order, then added to the total).
// ---------------------------------------------------------------------------
constexpr uint32_t kVisTableStride = 20;  // floats per ray: direction xyz, 0, 16 weighted SH values

__device__ __forceinline__ float nudge_toward(float o, float d) {
    if (d > 0.0f) return nextafterf(o, __int_as_float(0x7f800000));
    if (d < 0.0f) return nextafterf(o, __int_as_float(0xff800000));
    return o;
}

// 10 blocks of 128 per SM (48 registers): 9.8 -> 9.3 ms for 65,536 samples x
// 512 rays on the 200k-triangle scene.
__global__ void __launch_bounds__(128, 10) k_visibility_sh16(SceneView s, const float* __restrict__ pos,
                                                         const float* __restrict__ nrm, uint32_t n,
                                                         const float* __restrict__ table, uint32_t rays, float tmax,
                                                         float bias, float* __restrict__ out,
                                                         uint32_t* __restrict__ counts, unsigned long long* counters) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t words = (rays + 31u) >> 5;
    RayTally tally{0u, 0u};
    for (uint32_t i = warp; i < n; i += warps) {
        const float px = __ldg(pos + 3ull * i), py = __ldg(pos + 3ull * i + 1), pz = __ldg(pos + 3ull * i + 2);
        const float nx = __ldg(nrm + 3ull * i), ny = __ldg(nrm + 3ull * i + 1), nz = __ldg(nrm + 3ull * i + 2);
        const float ls = nx * nx + ny * ny + nz * nz;
        const bool has_normal = isfinite(ls) && ls > 1.0e-16f;
        f3 u = mk3(0.0f, 0.0f, 1.0f);
        if (has_normal) {
            const float inv = 1.0f / sqrtf(ls);
            u = mk3(nx * inv, ny * inv, nz * inv);
        }
        const f3 o = mk3(px + u.x * bias, py + u.y * bias, pz + u.z * bias);
        uint32_t word = 0u;
        for (uint32_t w = 0; w < words; ++w) {
            const uint32_t r = 32u * w + lane;
            bool visible = false;
            if (r < rays) {
                const float* e = table + (size_t)kVisTableStride * r;
                const f3 d = mk3(__ldg(e), __ldg(e + 1), __ldg(e + 2));
                const f3 oo = has_normal ? o : mk3(nudge_toward(o.x, d.x), nudge_toward(o.y, d.y), nudge_toward(o.z, d.z));
                visible = !trace_any(s, oo, d, 0.0f, tmax);
                tally.shadow++;
            }
            const unsigned m = __ballot_sync(0xffffffffu, visible);
            if (lane == w) word = m;
        }
        const uint32_t seen = __reduce_add_sync(0xffffffffu, (uint32_t)__popc(word));
        float total = 0.0f;
        for (uint32_t b = 0; b < words; b += 2u) {
            float batch = 0.0f;
            const uint32_t wend = min(b + 2u, words);
            for (uint32_t w = b; w < wend; ++w) {
                unsigned m = __shfl_sync(0xffffffffu, word, w);
                while (m) {
                    const uint32_t j = (uint32_t)__ffs(m) - 1u;
                    m &= m - 1u;
                    if (lane < 16u) batch += __ldg(table + (size_t)kVisTableStride * (32u * w + j) + 4u + lane);
                }
            }
            total += batch;
        }
        if (lane < 16u) out[16ull * i + lane] = total;
        if (lane == 0u && counts) counts[i] = seen;
    }
    flush_tally(counters, tally, 0u, 0u);
}

// ---------------------------------------------------------------------------
// Screen path tracer: path_tracer.slang:40-130 and camera.slang:201-236.
// 128-thread blocks cover 16x8 pixel tiles; each warp an 8x4 tile.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_trace_screen(SceneView s, LightingRaw lraw, CameraRaw cam,
                                                      float4* __restrict__ out, uint32_t w, uint32_t h,
                                                      uint32_t frame, uint32_t max_vertices,
                                                      unsigned long long* counters) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = blockIdx.y * 8u + (warp >> 1) * 4u + (lane >> 3);
    if (px >= w || py >= h) return;
    const LightParams L = make_light(lraw);
    RayTally tally{0u, 0u};
    Rng rng(px, py, frame * 1u + 0u);
    rng.next_1d();
    rng.next_1d();  // the unused jitter draw (path_tracer.slang:121)
    float pxf = ((float)px + 0.5f) / (float)w;
    float pyf = ((float)py + 0.5f) / (float)h;
    pxf = pxf + (-cam.jitter_x);
    pyf = pyf + cam.jitter_y;
    const float nx = 2.0f * pxf + -1.0f;
    const float ny = -2.0f * pyf + 1.0f;
    const f3 U = mk3(cam.image_u[0], cam.image_u[1], cam.image_u[2]);
    const f3 V = mk3(cam.image_v[0], cam.image_v[1], cam.image_v[2]);
    const f3 W = mk3(cam.image_w[0], cam.image_w[1], cam.image_w[2]);
    f3 dir = normalize3((nx * U + ny * V) + W);
    const float inv_cos = 1.0f / dot3(normalize3(W), dir);
    float tmin = cam.near_clip * inv_cos;
    float tmax = cam.far_clip * inv_cos;
    f3 o = mk3(cam.position[0], cam.position[1], cam.position[2]);
    f3 thp = mk3(1.0f, 1.0f, 1.0f), Lr = mk3(0.0f, 0.0f, 0.0f);
    float prev_pdf = 1.0f;
    for (uint32_t vi = 0; vi < max_vertices; ++vi) {
        const HitInfo hit = closest(s, o, dir, tmin, tmax, tally);
        if (!hit.valid) {
            f3 sky = sky_radiance(L, dir);
            if (vi == 0u && L.sun_disk) sky = sky + sun_disk(L, dir);
            Lr = Lr + thp * sky;
            break;
        }
        const uint2 ref = __ldg(s.tri_refs + hit.flat);
        const Shading sd = shading_data(s, ref.x, ref.y, hit.b1, hit.b2, -dir);
        if (L.area_nee && vi > 0u)
            Lr = Lr + thp * (sd.emissive * area_mis_weight(s, sd.emissive, sd.face_normal, dir, hit.t, prev_pdf));
        else
            Lr = Lr + thp * sd.emissive;
        const float u0 = rng.next_1d(), u1 = rng.next_1d();
        Lr = Lr + thp * sun_nee(s, L, sd, u0, u1, tally);
        // light reached from vertex vi lies on vertex vi + 1: sampled only where
        // that vertex exists, so both strategies cover the same path lengths
        if (L.area_nee && vi + 1u < max_vertices) {
            const float us = rng.next_1d(), a0 = rng.next_1d(), a1 = rng.next_1d();
            const AreaSample as = area_nee_sample(s, sd, us, a0, a1);
            if (as.valid) {
                tally.shadow++;
                if (!trace_any(s, sd.origin_front, as.dir, 0.0f, as.tmax)) Lr = Lr + thp * as.contrib;
            }
        }
        const float e0 = rng.next_1d(), e1 = rng.next_1d();
        float pdf;
        const f3 wo = cosine_sample_hemisphere(e0, e1, &pdf);
        pdf = maxf(pdf, 1e-6f);
        prev_pdf = pdf;
        const f3 f = sd.diffuse * kInvPi;
        thp = thp * ((f * fabsf(wo.z)) / pdf);
        o = sd.origin_front;
        dir = sd.frame.to_global(wo);
        tmin = 0.0f;
        tmax = L.t_max;
    }
    out[(size_t)py * w + px] = make_float4(Lr.x, Lr.y, Lr.z, 1.0f);
    flush_tally(counters, tally, 1u, 1u);
}

// ---------------------------------------------------------------------------
// Mesh Colors resolve (mesh_colors_resolve.slang:29-73) and frozen RGB9E5
// resolve (mesh_colors_frozen_resolve.slang:93-135): one primary ray per
// pixel, the hit triangle's lattice colours interpolated
// (mesh_colors_sample_irradiance, mesh_colors.slang:365-426), shaded as
// emissive + albedo / pi * irradiance.
// ---------------------------------------------------------------------------
__device__ __forceinline__ f3 mc_load(const void* colors, bool packed, uint32_t texel) {
    if (packed) {
        const uint32_t p = __ldg(reinterpret_cast<const uint32_t*>(colors) + texel);
        // exp2(e - 24) for the 5-bit exponent e, built exactly
        const float scale = __int_as_float((int)(((p >> 27) - 24u + 127u) << 23));
        return mk3((float)(p & 0x1ffu) * scale, (float)((p >> 9) & 0x1ffu) * scale,
                   (float)((p >> 18) & 0x1ffu) * scale);
    }
    const float4 v = __ldg(reinterpret_cast<const float4*>(colors) + texel);
    return mk3(v.x, v.y, v.z);
}

__device__ __forceinline__ uint32_t mc_side_texel(uint32_t front, uint4 inst, uint2 side, bool back) {
    return back ? side.x + (front - inst.z) : front;
}

// mesh_colors_sample_irradiance (mesh_colors.slang:365-426) at barycentrics
// (b0, b1, b2) of a face, front or back side.
__device__ __forceinline__ f3 mc_sample(const void* colors, bool packed, float b0, float b1, float b2, uint4 inst,
                                        uint2 face, uint2 side, bool back) {
    const uint32_t R = face.y;
    const float rf = (float)R;
    const float s0 = sat(b0) * rf, s1 = sat(b1) * rf, s2 = sat(b2) * rf;
    uint32_t i = min((uint32_t)s0, R);
    uint32_t j = min((uint32_t)s1, R - i);
    float w0 = s0 - floorf(s0), w1 = s1 - floorf(s1), w2 = s2 - floorf(s2);
    const bool upper = fabsf(((w0 + w1) + w2) - 2.0f) <= 1e-3f;
    if (upper) {
        w0 = 1.0f - w0;
        w1 = 1.0f - w1;
        w2 = 1.0f - w2;
    }
    if ((w0 + w1) + w2 <= 1e-6f || i >= R || j >= R - i)
        return mc_load(colors, packed, mc_side_texel(mc_address(i, j, inst.z, face), inst, side, back));
    uint32_t ta, tb, tc;
    if (upper) {
        ta = mc_address(i, j + 1u, inst.z, face);
        tb = mc_address(i + 1u, j, inst.z, face);
        tc = mc_address(i + 1u, j + 1u, inst.z, face);
    } else {
        ta = mc_address(i + 1u, j, inst.z, face);
        tb = mc_address(i, j + 1u, inst.z, face);
        tc = mc_address(i, j, inst.z, face);
    }
    const f3 ca = mc_load(colors, packed, mc_side_texel(ta, inst, side, back));
    const f3 cb = mc_load(colors, packed, mc_side_texel(tb, inst, side, back));
    const f3 cc = mc_load(colors, packed, mc_side_texel(tc, inst, side, back));
    return (w0 * ca + w1 * cb) + w2 * cc;
}

template <bool kPacked>
__global__ void __launch_bounds__(128) k_resolve_mesh_colors(SceneView s, LightingRaw lraw, CameraRaw cam, McView mc,
                                                             const void* __restrict__ colors,
                                                             float4* __restrict__ out, uint32_t w, uint32_t h) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = blockIdx.y * 8u + (warp >> 1) * 4u + (lane >> 3);
    if (px >= w || py >= h) return;
    const LightParams L = make_light(lraw);
    // compute_ray_pinhole (camera.slang:223-236), as in the path tracer
    float pxf = ((float)px + 0.5f) / (float)w;
    float pyf = ((float)py + 0.5f) / (float)h;
    pxf = pxf + (-cam.jitter_x);
    pyf = pyf + cam.jitter_y;
    const float nx = 2.0f * pxf + -1.0f;
    const float ny = -2.0f * pyf + 1.0f;
    const f3 U = mk3(cam.image_u[0], cam.image_u[1], cam.image_u[2]);
    const f3 V = mk3(cam.image_v[0], cam.image_v[1], cam.image_v[2]);
    const f3 W = mk3(cam.image_w[0], cam.image_w[1], cam.image_w[2]);
    const f3 dir = normalize3((nx * U + ny * V) + W);
    const float inv_cos = 1.0f / dot3(normalize3(W), dir);
    const f3 o = mk3(cam.position[0], cam.position[1], cam.position[2]);
    const HitInfo hit = trace_closest(s, o, dir, cam.near_clip * inv_cos, cam.far_clip * inv_cos);
    const size_t pix = (size_t)py * w + px;
    if (!hit.valid) {
        f3 sky = sky_radiance(L, dir);
        if (L.sun_disk) sky = sky + sun_disk(L, dir);
        out[pix] = make_float4(sky.x, sky.y, sky.z, 1.0f);
        return;
    }
    const uint2 ref = __ldg(s.tri_refs + hit.flat);
    const bool back = dot3(world_flat_normal(s, ref.x, ref.y), -dir) <= 0.0f;
    if (ref.x >= mc.instance_count) {
        atomicOr(s.status, kStatusBadRecord);
        return;
    }
    const uint4 inst = __ldg(mc.instance_infos + ref.x);
    const uint2 side = __ldg(mc.side_infos + ref.x);
    if (back && !(side.y & 1u)) {
        out[pix] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        return;
    }
    const uint2 face = __ldg(mc.face_infos + inst.x + ref.y);
    const float b0 = (1.0f - hit.b1) - hit.b2;
    const f3 irr = mc_sample(colors, kPacked, b0, hit.b1, hit.b2, inst, face, side, back);
    const Shading sd = shading_data(s, ref.x, ref.y, hit.b1, hit.b2, -dir);
    const f3 c = sd.emissive + (sd.diffuse * kInvPi) * irr;
    out[pix] = make_float4(c.x, c.y, c.z, 1.0f);
}

// ---------------------------------------------------------------------------
// Surface-probe resolve (surface_probe_resolve.slang:325-472): per pixel one
// primary ray; at the hit the probes of the hit instance are gathered from its
// point octree and reconstructed (nan_probe_gather.cuh), optionally blended
// with the triangle's vertex-anchor probes and replaced by baked vertex
// lighting; shaded as emissive + real-time sun + albedo / pi * irradiance, or
// one of the seven debug views.
// ---------------------------------------------------------------------------
struct ProbeResolveArgs {
    ProbeLayoutView layout;
    ProbeFieldView field;
    const uint32_t* vl_rgbm;
    const float4* vl_target;
    const uint4* vl_tri_map;
    const uint2* vl_inst;
    uint32_t vl_vertex_count, vl_tri_map_count;
    uint32_t debug_view, min_gather, use_vertex_fallback, use_vertex_lighting, use_radial, frame;
    float max_density, vl_range;
};

__device__ __forceinline__ f3 decode_rgbm(uint32_t packed, float range) {
    const float x = (float)(packed & 255u) / 255.0f, y = (float)((packed >> 8) & 255u) / 255.0f;
    const float z = (float)((packed >> 16) & 255u) / 255.0f, w = (float)((packed >> 24) & 255u) / 255.0f;
    return (mk3(x, y, z) * w) * range;
}

__global__ void __launch_bounds__(128) k_resolve_probes(SceneView s, LightingRaw lraw, CameraRaw cam,
                                                        ProbeResolveArgs a, float4* __restrict__ out, uint32_t w,
                                                        uint32_t h) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = blockIdx.y * 8u + (warp >> 1) * 4u + (lane >> 3);
    if (px >= w || py >= h) return;
    const LightParams L = make_light(lraw);
    float pxf = ((float)px + 0.5f) / (float)w;
    float pyf = ((float)py + 0.5f) / (float)h;
    pxf = pxf + (-cam.jitter_x);
    pyf = pyf + cam.jitter_y;
    const float nx = 2.0f * pxf + -1.0f;
    const float ny = -2.0f * pyf + 1.0f;
    const f3 U = mk3(cam.image_u[0], cam.image_u[1], cam.image_u[2]);
    const f3 V = mk3(cam.image_v[0], cam.image_v[1], cam.image_v[2]);
    const f3 W = mk3(cam.image_w[0], cam.image_w[1], cam.image_w[2]);
    const f3 dir = normalize3((nx * U + ny * V) + W);
    const float inv_cos = 1.0f / dot3(normalize3(W), dir);
    const f3 o = mk3(cam.position[0], cam.position[1], cam.position[2]);
    const HitInfo hit = trace_closest(s, o, dir, cam.near_clip * inv_cos, cam.far_clip * inv_cos);
    const size_t pix = (size_t)py * w + px;
    const bool beauty = a.debug_view == 0u || a.debug_view == 6u;
    if (!hit.valid) {
        f3 c = mk3(0.02f, 0.02f, 0.02f);
        if (beauty) {
            c = sky_radiance(L, dir);
            if (L.sun_disk) c = c + sun_disk(L, dir);
        }
        out[pix] = make_float4(c.x, c.y, c.z, 1.0f);
        return;
    }
    const uint2 ref = __ldg(s.tri_refs + hit.flat);
    const Shading sd = shading_data(s, ref.x, ref.y, hit.b1, hit.b2, -dir);
    f3 sun = mk3(0.0f, 0.0f, 0.0f);
    if (beauty) {
        Rng rng(px, py, a.frame);
        const float ux = rng.next_1d();
        const float uy = rng.next_1d();
        RayTally tally{0u, 0u};
        sun = sun_nee<DefaultTracer>(s, L, sd, ux, uy, tally);
    }
    if (ref.x >= a.layout.instance_count) {
        atomicOr(s.status, kStatusBadRecord);
        return;
    }
    const ProbeInstance ins = load_probe_instance(a.layout, ref.x);
    if (ins.offsets.w == 0u) {
        const f3 c = beauty ? sd.emissive + sun : gather_count_color(0u);
        out[pix] = make_float4(c.x, c.y, c.z, 1.0f);
        return;
    }
    Candidates cand;
    const ProbeReconstruction r = probe_reconstruct(a.layout, a.field, ins, sd.position, normalize3(sd.face_normal),
                                                    a.min_gather, a.use_radial != 0u, cand, s.status);
    const uint32_t side = sd.back_side ? 1u : 0u;
    const float b0 = (1.0f - hit.b1) - hit.b2;
    const float bary[3] = {b0, hit.b1, hit.b2};
    // surface_probe_sample_vertex_fallback
    f3 vertex_irr = mk3(0.0f, 0.0f, 0.0f);
    bool has_fallback = false;
    if (a.use_vertex_fallback != 0u) {
        const uint32_t rec = ins.tri_map_offset + ref.y * 2u + side;
        if (rec >= a.layout.tri_map_count) {
            atomicOr(s.status, kStatusBadRecord);
        } else {
            const uint4 anchors = __ldg(a.layout.tri_vertex_probes + rec);
            if (anchors.w & 1u) {
                const uint32_t idx[3] = {anchors.x, anchors.y, anchors.z};
                f3 acc = mk3(0.0f, 0.0f, 0.0f);
                float avail = 0.0f;
                for (int c = 0; c < 3; ++c) {
                    if (idx[c] >= a.layout.probe_count) {
                        atomicOr(s.status, kStatusBadRecord);
                        continue;
                    }
                    if (__ldg(a.field.counts + idx[c]) == 0u) continue;
                    acc = acc + bary[c] * probe_irradiance(a.field, idx[c]);
                    avail = avail + bary[c];
                }
                if (avail > 1e-6f) {
                    vertex_irr = acc / avail;
                    has_fallback = true;
                }
            }
        }
    }
    const float target = (float)min(max(a.min_gather, 1u), 32u);
    float conf = minf(sat((float)r.gathered / target), sat(r.ess / target));
    if (r.weight_sum <= 1e-6f) conf = 0.0f;
    if (!has_fallback) conf = 1.0f;
    const float fallback_weight = 1.0f - conf;
    f3 irr = lerp3(vertex_irr, r.irradiance, conf);
    f3 c;
    if (a.debug_view == 1u) {
        c = gather_count_color(r.gathered);
    } else if (a.debug_view == 2u) {
        c = support_color(r.support);
    } else if (a.debug_view == 3u) {
        c = density_color(r.support, a.max_density);
    } else if (a.debug_view == 4u) {
        c = support_color(1.0f - fallback_weight);
    } else if (a.debug_view == 5u) {
        c = self_hit_color(r.self_hit_rate);
    } else {
        // surface_probe_sample_vertex_lighting
        bool has_vl = false;
        f3 vl = mk3(0.0f, 0.0f, 0.0f);
        float vl_conf = 0.0f;
        if (a.vl_rgbm != nullptr) {
            const uint2 io = __ldg(a.vl_inst + ref.x);
            const uint32_t rec = io.x + ref.y * 2u + side;
            if (rec >= a.vl_tri_map_count) {
                atomicOr(s.status, kStatusBadRecord);
            } else {
                const uint4 vv = __ldg(a.vl_tri_map + rec);
                if (vv.w != 0u) {
                    if (vv.x >= a.vl_vertex_count || vv.y >= a.vl_vertex_count || vv.z >= a.vl_vertex_count) {
                        atomicOr(s.status, kStatusBadRecord);
                    } else {
                        vl = (b0 * decode_rgbm(__ldg(a.vl_rgbm + vv.x), a.vl_range) +
                              hit.b1 * decode_rgbm(__ldg(a.vl_rgbm + vv.y), a.vl_range)) +
                             hit.b2 * decode_rgbm(__ldg(a.vl_rgbm + vv.z), a.vl_range);
                        vl_conf = (b0 * __ldg(a.vl_target + vv.x).w + hit.b1 * __ldg(a.vl_target + vv.y).w) +
                                  hit.b2 * __ldg(a.vl_target + vv.z).w;
                        has_vl = true;
                    }
                }
            }
        }
        if (a.debug_view == 6u) {
            c = has_vl ? (sd.emissive + sun) + (sd.diffuse * kInvPi) * vl : mk3(1.0f, 0.0f, 1.0f);
        } else if (a.debug_view == 7u) {
            c = has_vl ? support_color(vl_conf) : mk3(1.0f, 0.0f, 1.0f);
        } else {
            if (a.use_vertex_lighting != 0u && has_vl) irr = vl;
            c = (sd.emissive + sun) + (sd.diffuse * kInvPi) * irr;
        }
    }
    out[pix] = make_float4(c.x, c.y, c.z, 1.0f);
}

// ---------------------------------------------------------------------------
// Mesh Colors one-ring surface filter (mesh_colors_surface_filter.slang:
// 1-253): each texel's colour becomes the weighted mean of itself and its six
// lattice neighbours; neighbours across an edge are mapped into the adjacent
// face (mesh_colors_map_one_edge_tap, mesh_colors.slang:156-203), sampled
// there and weighted by the Gaussian in the angle between face normals. All
// instances in one launch (the reference dispatches per instance).
// ---------------------------------------------------------------------------
struct FilterArgs {
    McView mc;
    const uint4* adjacency;  // per face: packed edges 0..2
    const float4* normals;   // per face
    const float4* src;
    float4* dst;
    float neighbor_weight;
    float sigma;
    uint32_t total_texels;
};

__device__ __forceinline__ float normal_filter_weight(f3 c, f3 n, float sigma) {
    const float cosine = minf(maxf(dot3(c, n), 0.0f), 1.0f);
    if (sigma <= 1e-6f) return cosine >= 1.0f - 1e-6f ? 1.0f : 0.0f;
    const float angle = acosf(cosine);
    const float na = angle / sigma;
    return expf(-0.5f * na * na);
}

// Lattice point candidate (x, y) outside the face, across `edge`: its
// barycentrics in the adjacent face, or false.
__device__ __forceinline__ bool map_edge_tap(int x, int y, uint32_t R, uint32_t adj_edge, bool flip, uint32_t edge,
                                             float nb[3]) {
    const float inv = 1.0f / (float)R;
    const float sb[3] = {(float)x * inv, (float)y * inv, 1.0f - (float)(x + y) * inv};
    const uint32_t s_start = edge, s_end = (edge + 1u) % 3u, s_opp = (edge + 2u) % 3u;
    const uint32_t n_start = adj_edge, n_end = (adj_edge + 1u) % 3u, n_opp = (adj_edge + 2u) % 3u;
    const float outside = sb[s_opp];
    const uint32_t m_start = flip ? n_end : n_start, m_end = flip ? n_start : n_end;
    nb[0] = nb[1] = nb[2] = 0.0f;
    nb[m_start] = sb[s_start] + outside;
    nb[m_end] = sb[s_end] + outside;
    nb[n_opp] = -outside;
    for (int k = 0; k < 3; ++k)
        if (nb[k] < -1e-5f || nb[k] > 1.0f + 1e-5f) return false;
    for (int k = 0; k < 3; ++k) nb[k] = maxf(nb[k], 0.0f);
    const float sum = maxf((nb[0] + nb[1]) + nb[2], 1e-6f);
    for (int k = 0; k < 3; ++k) nb[k] = nb[k] / sum;
    return true;
}

__device__ __forceinline__ void filter_side(const FilterArgs& a, uint32_t front, int ci, int cj, uint4 inst,
                                            uint2 side, uint2 face, uint32_t prim, f3 cn, bool back) {
    const uint32_t center = mc_side_texel(front, inst, side, back);
    const float4 c = __ldg(a.src + center);
    f3 acc = mk3(c.x, c.y, c.z);
    float wsum = 1.0f;
    const int R = (int)face.y;
    const int off[6][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, -1}, {-1, 1}};
    for (int t = 0; t < 6; ++t) {
        const int x = ci + off[t][0], y = cj + off[t][1];
        if (x >= 0 && y >= 0 && x + y <= R) {
            const uint32_t ft = mc_address((uint32_t)x, (uint32_t)y, inst.z, face);
            const f3 v = mc_load(a.src, false, mc_side_texel(ft, inst, side, back));
            acc = acc + a.neighbor_weight * v;
            wsum = wsum + a.neighbor_weight;
            continue;
        }
        const uint32_t edge = x < 0 ? 1u : (y < 0 ? 2u : 0u);
        const uint4 adj4 = __ldg(a.adjacency + inst.x + prim);
        const uint32_t packed = edge == 0u ? adj4.x : (edge == 1u ? adj4.y : adj4.z);
        if (packed == 0xffffffffu) continue;
        const uint32_t adj_face = inst.x + (packed >> 3);
        float nb[3];
        if (!map_edge_tap(x, y, face.y, packed & 3u, (packed & 4u) != 0u, edge, nb)) continue;
        const float4 nn = __ldg(a.normals + adj_face);
        const float w = a.neighbor_weight * normal_filter_weight(cn, mk3(nn.x, nn.y, nn.z), a.sigma);
        const uint2 nface = __ldg(a.mc.face_infos + adj_face);
        const f3 v = mc_sample(a.src, false, nb[0], nb[1], nb[2], inst, nface, side, back);
        if (w > 0.0f) {
            acc = acc + w * v;
            wsum = wsum + w;
        }
    }
    const f3 r = acc / maxf(wsum, 1e-6f);
    a.dst[center] = make_float4(r.x, r.y, r.z, c.w);
}

__global__ void __launch_bounds__(128) k_filter_mesh_colors(FilterArgs a) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= a.total_texels) return;
    const McView& mc = a.mc;
    uint32_t lo = 0u, hi = mc.instance_count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (__ldg(mc.surface_prefix + mid) <= u) lo = mid; else hi = mid - 1u;
    }
    const uint32_t local = u - __ldg(mc.surface_prefix + lo);
    const uint4 inst = __ldg(mc.instance_infos + lo);
    if (local >= inst.w) return;
    // mesh_colors_find_face (mesh_colors.slang:272-305)
    int left = (int)inst.x, right = (int)(inst.x + inst.y) - 1;
    uint2 face = make_uint2(0u, 1u);
    uint32_t prim = 0u;
    bool found = false;
    while (left <= right) {
        const int mid = (left + right) / 2;
        face = __ldg(mc.face_infos + mid);
        const int loc = (int)local - (int)face.x;
        const int count = (int)((face.y + 1u) * (face.y + 2u) / 2u);
        if (loc < 0) right = mid - 1;
        else if (loc >= count) left = mid + 1;
        else {
            prim = (uint32_t)mid - inst.x;
            found = true;
            break;
        }
    }
    if (!found) return;
    const uint2 side = __ldg(mc.side_infos + lo);
    uint32_t ti, tj;
    mc_address_to_ij(local - face.x, face.y, &ti, &tj);
    const float4 n4 = __ldg(a.normals + inst.x + prim);
    const f3 cn = mk3(n4.x, n4.y, n4.z);
    const uint32_t front = inst.z + local;
    filter_side(a, front, (int)ti, (int)tj, inst, side, face, prim, cn, false);
    if (side.y & 1u) filter_side(a, front, (int)ti, (int)tj, inst, side, face, prim, cn, true);
}

// accumulator.slang:9-19
__global__ void k_accumulate(const float4* __restrict__ input, float4* __restrict__ output,
                             float4* __restrict__ history, uint32_t n, int reset) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 in = input[i];
    float4 a = reset ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : history[i];
    a = make_float4(a.x + in.x, a.y + in.y, a.z + in.z, a.w + 1.0f);
    history[i] = a;
    output[i] = make_float4(a.x / a.w, a.y / a.w, a.z / a.w, 1.0f);
}

// ---------------------------------------------------------------------------
// Mesh Colors lattice (mesh_colors.slang:37-65, 272-363).
// ---------------------------------------------------------------------------
// trace_radiance, texture_space_path_tracer.slang:57-84.
__device__ __forceinline__ f3 ts_trace_radiance(const SceneView& s, const LightParams& L, f3 o, f3 d, Rng& rng,
                                                uint32_t max_bounces, RayTally& tally) {
    f3 thp = mk3(1.0f, 1.0f, 1.0f), rad = mk3(0.0f, 0.0f, 0.0f);
    for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
        const HitInfo hit = closest(s, o, d, 0.0f, L.t_max, tally);
        if (!hit.valid) return rad + thp * sky_radiance(L, d);
        const uint2 ref = __ldg(s.tri_refs + hit.flat);
        const Shading sd = shading_data(s, ref.x, ref.y, hit.b1, hit.b2, -d);
        rad = rad + thp * sd.emissive;
        const float u0 = rng.next_1d(), u1 = rng.next_1d();
        rad = rad + thp * sun_nee(s, L, sd, u0, u1, tally);
        const float e0 = rng.next_1d(), e1 = rng.next_1d();
        float pdf;
        const f3 sdir = cosine_sample_hemisphere(e0, e1, &pdf);
        if (pdf <= 1e-6f) return rad;
        const f3 f = sd.diffuse * kInvPi;
        thp = thp * ((f * fabsf(sdir.z)) / pdf);
        o = sd.origin_front;
        d = sd.frame.to_global(sdir);
    }
    return rad;
}

// estimate_surface_irradiance, texture_space_path_tracer.slang:86-117.
__device__ __forceinline__ f3 ts_estimate(const SceneView& s, const LightParams& L, uint32_t inst, uint32_t prim,
                                          float bx, float by, f3 view, uint32_t n, Rng& rng, uint32_t max_bounces,
                                          RayTally& tally) {
    const Shading sd = shading_data(s, inst, prim, bx, by, view);
    f3 irr = mk3(0.0f, 0.0f, 0.0f);
    for (uint32_t k = 0; k < n; ++k) {
        const float u0 = rng.next_1d(), u1 = rng.next_1d();
        f3 si = sun_irradiance(s, L, sd, u0, u1, tally);
        const float e0 = rng.next_1d(), e1 = rng.next_1d();
        float pdf;
        const f3 dir = cosine_sample_hemisphere(e0, e1, &pdf);
        if (pdf > 1e-6f) {
            const f3 rad = ts_trace_radiance(s, L, sd.origin_front, sd.frame.to_global(dir), rng, max_bounces, tally);
            si = si + ((rad * fabsf(dir.z)) / pdf);
        }
        irr = irr + si;
    }
    return irr / (float)n;
}

// compute_main, texture_space_path_tracer.slang:140-216, one thread per
// surface texel of every instance.
__global__ void __launch_bounds__(128) k_trace_texels(SceneView s, LightingRaw lraw, McView mc,
                                                      uint4* __restrict__ slots, uint32_t iteration, uint32_t spt,
                                                      uint32_t max_bounces, int reset, uint32_t begin, uint32_t end,
                                                      unsigned long long* counters) {
    const uint32_t u = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= end) return;
    TexelSurface ts;
    Rng rng(0u, 0u, 0u);
    if (!texel_surface(s, mc, u, iteration, spt, &ts, &rng)) return;
    RayTally tally{0u, 0u};
    const uint32_t inst_index = ts.inst, prim = ts.prim, global_texel = ts.global_texel;
    const uint4 inst = ts.inst_info;
    const uint2 side = ts.side;
    const uint32_t n = max(spt, 1u);
    const float hb1 = ts.b1, hb2 = ts.b2;
    const LightParams L = make_light(lraw);
    const f3 fnrm = world_flat_normal(s, inst_index, prim);
    const f3 front = ts_estimate(s, L, inst_index, prim, hb1, hb2, fnrm, n, rng, max_bounces, tally);
    uint32_t paths = n;
    if (global_texel < mc.payload_count) store_running_mean(slots, global_texel, front, reset, mc.compensation);
    else atomicOr(s.status, 2u);
    if (side.y & 1u) {
        const f3 back = ts_estimate(s, L, inst_index, prim, hb1, hb2, -fnrm, n, rng, max_bounces, tally);
        const uint32_t bt = side.x + (global_texel - inst.z);
        if (bt < mc.payload_count) store_running_mean(slots, bt, back, reset, mc.compensation);
        else atomicOr(s.status, 2u);
        paths += n;
    }
    flush_tally(counters, tally, 1u, paths);
}

// The texel estimator at listed surface points (b1, b2, instance bits,
// primitive bits | back side << 31), one thread per point: RNG(index,
// 0xFFFFFFFF, iteration * n), view = the flat normal (negated for the back
// side); indirect_only drops the first vertex's sun term but still draws its
// two numbers. Out: (E, 0), or (0, 0, 0, -1) for a point whose instance is
// ~0. The same values as the wavefront points pass (k_wf_point_generate and
// the texel stages); one launch instead of a round of launches per bounce,
// for the small point sets that train the learned cache.
__global__ void __launch_bounds__(128) k_trace_points(SceneView s, LightingRaw lraw, const float4* __restrict__ points,
                                                      uint32_t count, float4* __restrict__ out, uint32_t iteration,
                                                      uint32_t n, uint32_t max_bounces, int indirect_only,
                                                      unsigned long long* counters) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= count) return;
    const float4 pt = points[u];
    const uint32_t inst = __float_as_uint(pt.z), primw = __float_as_uint(pt.w);
    const uint32_t prim = primw & 0x7fffffffu;
    if (inst == 0xffffffffu || !valid_prim(s, inst, prim)) {
        if (inst != 0xffffffffu) atomicOr(s.status, kStatusBadRecord);
        out[u] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        return;
    }
    const LightParams L = make_light(lraw);
    Rng rng(u, 0xffffffffu, iteration * n);
    RayTally tally{0u, 0u};
    f3 view = world_flat_normal(s, inst, prim);
    if (primw >> 31) view = -view;
    const Shading sd = shading_data(s, inst, prim, pt.x, pt.y, view);
    f3 irr = mk3(0.0f, 0.0f, 0.0f);
    for (uint32_t k = 0; k < n; ++k) {
        const float u0 = rng.next_1d(), u1 = rng.next_1d();
        f3 si = indirect_only ? mk3(0.0f, 0.0f, 0.0f) : sun_irradiance(s, L, sd, u0, u1, tally);
        const float e0 = rng.next_1d(), e1 = rng.next_1d();
        float pdf;
        const f3 dir = cosine_sample_hemisphere(e0, e1, &pdf);
        if (pdf > 1e-6f) {
            const f3 rad = ts_trace_radiance(s, L, sd.origin_front, sd.frame.to_global(dir), rng, max_bounces, tally);
            si = si + ((rad * fabsf(dir.z)) / pdf);
        }
        irr = irr + si;
    }
    const f3 e = irr / (float)n;
    out[u] = make_float4(e.x, e.y, e.z, 0.0f);
    flush_tally(counters, tally, 1u, n);
}

// ---------------------------------------------------------------------------
// Surface-probe baker: surface_probe_path_tracer.slang:47-315.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_trace_probes(SceneView s, LightingRaw lraw, ProbeOut out,
                                                      const float4* __restrict__ probes,
                                                      const float4* __restrict__ pinst, uint32_t probe_count,
                                                      uint32_t probe_instance_count, uint32_t iteration, uint32_t spp, uint32_t max_bounces,
                                                      int reset, uint32_t begin, uint32_t end,
                                                      unsigned long long* counters) {
    const uint32_t p = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= end || p >= probe_count) return;
    const LightParams L = make_light(lraw);
    RayTally tally{0u, 0u};
    if (probe_unit<DefaultTracer>(s, L, out, probes, pinst, probe_instance_count, iteration, spp, max_bounces, reset,
                                  p, tally))
        flush_tally(counters, tally, 1u, max(spp, 1u));
}

__global__ void __launch_bounds__(128) k_trace_probes_prt(SceneView s, LightingRaw lraw, PrtOut out,
                                                          const float4* __restrict__ probes,
                                                          const float4* __restrict__ pinst, uint32_t probe_count,
                                                          uint32_t probe_instance_count, uint32_t iteration,
                                                          uint32_t spp, uint32_t max_bounces, int reset,
                                                          uint32_t begin, uint32_t end, unsigned long long* counters) {
    const uint32_t p = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= end || p >= probe_count) return;
    const LightParams L = make_light(lraw);
    RayTally tally{0u, 0u};
    if (probe_prt_unit<DefaultTracer>(s, L, out, probes, pinst, probe_instance_count, iteration, spp, max_bounces,
                                      reset, p, tally))
        flush_tally(counters, tally, 1u, max(spp, 1u));
}

// ---------------------------------------------------------------------------
// PRT evaluation (surface_probe_prt_evaluate.slang:20-103). The lighting is
// projected on the SH L2 basis by a quasi-random sphere rule: sample i of n at
// y = 1 - 2 (i + 0.5) / n and phi = 2 pi radical_inverse(i); the radiance a
// path that escapes meets is the sky term. One thread per coefficient, the
// samples summed in order. Evaluation is static + sum_c T_c * L_c, clamped
// at 0, for probes with at least one sample.
// ---------------------------------------------------------------------------
// 256 threads: each chunk of 256 sample directions is evaluated in parallel
// into shared memory (sky * Y_c per coefficient and channel), then 27 threads
// each add their own (coefficient, channel) column in sample order, so every
// sum is the same sequential float sum as one loop over the samples.
__global__ void __launch_bounds__(256) k_prt_project_lighting(LightingRaw lraw, float4* __restrict__ sh,
                                                               uint32_t n) {
    __shared__ float terms[27][256];
    const uint32_t tid = threadIdx.x;
    const LightParams L = make_light(lraw);
    n = max(n, 1u);
    float acc = 0.0f;
    for (uint32_t base = 0; base < n; base += 256u) {
        const uint32_t i = base + tid;
        if (i < n) {
            const float u = (static_cast<float>(i) + 0.5f) / static_cast<float>(n);
            const float v = static_cast<float>(__brev(i)) * 2.3283064365386963e-10f;
            const float y = 1.0f - 2.0f * u;
            const float r = sqrtf(fmaxf(1.0f - y * y, 0.0f));
            float sn, cs;
            nan_sincos(kTwoPi * v, &sn, &cs);
            const f3 d = mk3(r * cs, y, r * sn);
            for (uint32_t c = 0; c < 9u; ++c) {
                const f3 t = sky_radiance(L, d) * sh_l2_basis(c, d);
                terms[3 * c][tid] = t.x;
                terms[3 * c + 1][tid] = t.y;
                terms[3 * c + 2][tid] = t.z;
            }
        }
        __syncthreads();
        if (tid < 27u) {
            const uint32_t m = min(256u, n - base);
            for (uint32_t k = 0; k < m; ++k) acc = acc + terms[tid][k];
        }
        __syncthreads();
    }
    if (tid < 27u) reinterpret_cast<float*>(sh)[4u * (tid / 3u) + tid % 3u] = acc * ((4.0f * kPi) / static_cast<float>(n));
    if (tid < 9u) reinterpret_cast<float*>(sh)[4u * tid + 3u] = 0.0f;
}

__global__ void k_prt_evaluate(const float* __restrict__ values, const uint32_t* __restrict__ counts,
                               const float* __restrict__ static_source, const float4* __restrict__ sh,
                               float* __restrict__ out, uint32_t* __restrict__ out_counts, uint32_t n) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t count = counts[p];
    f3 e = mk3(static_source[3 * p], static_source[3 * p + 1], static_source[3 * p + 2]);
    if (count > 0u) {
        const float* t = values + 27ull * p;
        for (int c = 0; c < 9; ++c) {
            const float4 l = sh[c];
            e = e + mk3(t[3 * c] * l.x, t[3 * c + 1] * l.y, t[3 * c + 2] * l.z);
        }
    }
    out[3 * p] = fmaxf(e.x, 0.0f);
    out[3 * p + 1] = fmaxf(e.y, 0.0f);
    out[3 * p + 2] = fmaxf(e.z, 0.0f);
    out_counts[p] = count;
}

// ---------------------------------------------------------------------------
// RGB9E5: mesh_colors.slang:218-253 and mesh_colors_rgb9e5_pack.slang:7-16.
// floor(log2(max)) is taken exactly from the binary exponent.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_rgb9e5(float r, float g, float b) {
    const float kMax = 65408.0f;
    float v[3] = {isnan(r) ? 0.0f : r, isnan(g) ? 0.0f : g, isnan(b) ? 0.0f : b};
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = fminf(fmaxf(v[i], 0.0f), kMax);
    const float m = fmaxf(v[0], fmaxf(v[1], v[2]));
    if (m < 0x1p-25f) return 0u;
    const int e2 = (int)((__float_as_uint(m) >> 23) & 0xffu) - 126;  // m is normal here
    const int exponent = max(-15, e2);
    uint32_t shared = (uint32_t)(exponent + 15);
    float scale = __uint_as_float((uint32_t)((int)shared - 24 + 127) << 23);
    uint32_t mant[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) mant[i] = (uint32_t)floorf(v[i] / scale + 0.5f);
    if (max(mant[0], max(mant[1], mant[2])) == 512u && shared < 31u) {
        shared += 1u;
        scale *= 2.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i) mant[i] = (uint32_t)floorf(v[i] / scale + 0.5f);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) mant[i] = min(mant[i], 511u);
    return mant[0] | (mant[1] << 9) | (mant[2] << 18) | (shared << 27);
}

__global__ void k_pack_rgb9e5(const uint4* __restrict__ slots, uint32_t* __restrict__ out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 s = slots[i];
    out[i] = pack_rgb9e5(__uint_as_float(s.x), __uint_as_float(s.y), __uint_as_float(s.z));
}

uint32_t blocks_for(uint64_t n, uint32_t threads) { return (uint32_t)((n + threads - 1) / threads); }

LightingRaw to_raw(const NanLighting* l) {
    LightingRaw r;
    static_assert(sizeof(LightingRaw) == sizeof(NanLighting), "lighting layout");
    memcpy(&r, l, sizeof(r));
    return r;
}

}  // namespace

namespace nan_host {

int launch_intersect(NanContext* ctx, const float* rays, uint32_t count, uint32_t* ids, float* tb, cudaStream_t st) {
    if (count == 0) return NAN_OK;
    k_intersect<<<blocks_for(count, 128), 128, 0, st>>>(scene_view(ctx), reinterpret_cast<const float4*>(rays), count,
                                                        reinterpret_cast<uint4*>(ids), tb);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "intersect launch");
}

// Direction table of the caster's make_ray_projections
// (tinybvh_visibility.cpp:81-101, 52-77): ray r has u0 = r / R, u1 = the
// bit-reversed r times 2^-32, phi = 2 pi u0, cos theta = 1 - 2 u1, direction
// (cos phi sin theta, cos theta, sin phi sin theta), and the real SH basis of
// bands 0-3 at that direction times 4 pi / R. Evaluated in float with the C
// library's cosf/sinf/sqrtf and the caster's operation order, so the rays
// and weights are the caster's own.
int visibility_ray_table(uint32_t ray_count, float* t) {
    constexpr float kPiF = 3.14159265358979323846f;
    const float weight = (4.0f * kPiF) / static_cast<float>(ray_count);
    for (uint32_t r = 0; r < ray_count; ++r) {
        uint32_t v = r;
        v = (v << 16) | (v >> 16);
        v = ((v & 0x55555555u) << 1) | ((v & 0xaaaaaaaau) >> 1);
        v = ((v & 0x33333333u) << 2) | ((v & 0xccccccccu) >> 2);
        v = ((v & 0x0f0f0f0fu) << 4) | ((v & 0xf0f0f0f0u) >> 4);
        v = ((v & 0x00ff00ffu) << 8) | ((v & 0xff00ff00u) >> 8);
        const float u0 = static_cast<float>(r) / static_cast<float>(ray_count);
        const float u1 = static_cast<float>(v) * 2.3283064365386963e-10f;
        const float phi = u0 * (2.0f * kPiF);
        const float ct = 1.0f - 2.0f * u1;
        const float st = std::sqrt(std::max(1.0f - ct * ct, 0.0f));
        const float x = std::cos(phi) * st, y = ct, z = std::sin(phi) * st;
        const float x2 = x * x, y2 = y * y, z2 = z * z;
        float* e = t + (size_t)kVisTableStride * r;
        e[0] = x;
        e[1] = y;
        e[2] = z;
        e[3] = 0.0f;
        float* sh = e + 4;
        sh[0] = weight * 0.282094791774f;
        sh[1] = weight * (-0.488602511903f * y);
        sh[2] = weight * (0.488602511903f * z);
        sh[3] = weight * (-0.488602511903f * x);
        sh[4] = weight * (1.09254843059f * x * y);
        sh[5] = weight * (-1.09254843059f * y * z);
        sh[6] = weight * (0.315391565253f * (-1.0f + 3.0f * z2));
        sh[7] = weight * (-1.09254843059f * x * z);
        sh[8] = weight * (0.546274215296f * (x2 - y2));
        sh[9] = weight * (-0.590043589927f * (3.0f * x2 * y - y2 * y));
        sh[10] = weight * (2.89061144264f * x * y * z);
        sh[11] = weight * (-0.457045799464f * y * (-1.0f + 5.0f * z2));
        sh[12] = weight * (0.37317633259f * z * (-3.0f + 5.0f * z2));
        sh[13] = weight * (-0.457045799464f * x * (-1.0f + 5.0f * z2));
        sh[14] = weight * (1.44530572132f * (x2 - y2) * z);
        sh[15] = weight * (-0.590043589927f * (x2 * x - 3.0f * x * y2));
    }
    return NAN_OK;
}

int launch_visibility_sh16(NanContext* ctx, const float* positions, const float* normals, uint32_t count,
                           const float* table, uint32_t ray_count, float max_distance, float self_bias, float* out,
                           uint32_t* visible, cudaStream_t st) {
    if (count == 0) return NAN_OK;
    int sms = 148, occ = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_visibility_sh16, 128, 0);
    const uint32_t grid = std::min<uint32_t>((uint32_t)sms * (uint32_t)std::max(occ, 1), (count + 3u) / 4u);
    k_visibility_sh16<<<grid, 128, 0, st>>>(scene_view(ctx), positions, normals, count, table, ray_count,
                                            max_distance, self_bias, out, visible, ctx->d_counters);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "visibility launch");
}

int launch_occluded(NanContext* ctx, const float* rays, uint32_t count, float* vis, cudaStream_t st) {
    if (count == 0) return NAN_OK;
    k_occluded<<<blocks_for(count, 128), 128, 0, st>>>(scene_view(ctx), reinterpret_cast<const float4*>(rays), count,
                                                       vis);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "occluded launch");
}

int launch_trace_screen(NanContext* ctx, float* out, uint32_t w, uint32_t h, uint32_t frame, uint32_t max_vertices,
                        const NanCamera* cam, const NanLighting* light, cudaStream_t st) {
    if (w == 0 || h == 0) return NAN_OK;
    CameraRaw c;
    static_assert(sizeof(CameraRaw) == sizeof(NanCamera), "camera layout");
    memcpy(&c, cam, sizeof(c));
    dim3 grid(blocks_for(w, 16), blocks_for(h, 8));
    k_trace_screen<<<grid, 128, 0, st>>>(scene_view(ctx), to_raw(light), c, reinterpret_cast<float4*>(out), w, h, frame,
                                         max_vertices, ctx->d_counters);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "trace_screen launch");
}

int launch_resolve_mesh_colors(NanContext* ctx, const NanMeshColorsDesc* lay, const void* colors, int packed,
                               float* out, uint32_t w, uint32_t h, const NanCamera* cam, const NanLighting* light,
                               cudaStream_t st) {
    if (w == 0 || h == 0) return NAN_OK;
    CameraRaw c;
    memcpy(&c, cam, sizeof(c));
    McView mc;
    memset(&mc, 0, sizeof(mc));
    mc.face_infos = reinterpret_cast<const uint2*>(lay->face_infos);
    mc.instance_infos = reinterpret_cast<const uint4*>(lay->instance_infos);
    mc.side_infos = reinterpret_cast<const uint2*>(lay->side_infos);
    mc.instance_count = lay->instance_count;
    mc.payload_count = lay->payload_count;
    dim3 grid(blocks_for(w, 16), blocks_for(h, 8));
    if (packed)
        k_resolve_mesh_colors<true><<<grid, 128, 0, st>>>(scene_view(ctx), to_raw(light), c, mc, colors,
                                                          reinterpret_cast<float4*>(out), w, h);
    else
        k_resolve_mesh_colors<false><<<grid, 128, 0, st>>>(scene_view(ctx), to_raw(light), c, mc, colors,
                                                           reinterpret_cast<float4*>(out), w, h);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "resolve_mesh_colors launch");
}

int launch_resolve_probes(NanContext* ctx, const NanProbeLayoutDesc* lay, const float* values,
                          const uint32_t* counts, const uint32_t* self_hits, const uint32_t* radial,
                          const NanProbeResolveOptions* opt, float* out, uint32_t w, uint32_t h,
                          const NanCamera* cam, const NanLighting* light, cudaStream_t st) {
    if (w == 0 || h == 0) return NAN_OK;
    CameraRaw c;
    memcpy(&c, cam, sizeof(c));
    ProbeResolveArgs a;
    memset(&a, 0, sizeof(a));
    a.layout.probes = reinterpret_cast<const float4*>(lay->probes);
    a.layout.nodes = reinterpret_cast<const uint4*>(lay->nodes);
    a.layout.instances = reinterpret_cast<const float4*>(lay->instances);
    a.layout.tri_vertex_probes = reinterpret_cast<const uint4*>(lay->triangle_vertex_probes);
    a.layout.probe_count = lay->probe_count;
    a.layout.node_count = lay->node_count;
    a.layout.instance_count = lay->instance_count;
    a.layout.tri_map_count = lay->triangle_vertex_probe_count;
    a.field = ProbeFieldView{values, counts, self_hits, radial};
    a.vl_rgbm = opt->vertex_lighting_rgbm;
    a.vl_target = reinterpret_cast<const float4*>(opt->vertex_lighting_target);
    a.vl_tri_map = reinterpret_cast<const uint4*>(opt->vertex_lighting_triangle_map);
    a.vl_inst = reinterpret_cast<const uint2*>(opt->vertex_lighting_instance_offsets);
    a.vl_vertex_count = opt->vertex_lighting_vertex_count;
    a.vl_tri_map_count = opt->vertex_lighting_triangle_record_count;
    a.debug_view = std::min(opt->debug_view, 7u);
    a.min_gather = opt->min_gather_count;
    a.use_vertex_fallback = opt->use_vertex_fallback;
    a.use_vertex_lighting = opt->use_vertex_lighting;
    a.use_radial = opt->use_radial_visibility;
    a.frame = opt->frame_index;
    a.max_density = opt->max_density_multiplier;
    a.vl_range = std::max(opt->vertex_lighting_rgbm_range, 1.0f);
    dim3 grid(blocks_for(w, 16), blocks_for(h, 8));
    k_resolve_probes<<<grid, 128, 0, st>>>(scene_view(ctx), to_raw(light), c, a, reinterpret_cast<float4*>(out), w,
                                           h);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "resolve_probes launch");
}

int launch_filter_mesh_colors(NanContext* ctx, const NanMeshColorsDesc* lay, const uint32_t* adjacency,
                              const float* face_normals, const uint8_t* src, uint8_t* dst, float neighbor_weight,
                              float sigma, cudaStream_t st) {
    if (lay->total_surface_texels == 0 || lay->instance_count == 0) return NAN_OK;
    FilterArgs a;
    memset(&a, 0, sizeof(a));
    a.mc.face_infos = reinterpret_cast<const uint2*>(lay->face_infos);
    a.mc.instance_infos = reinterpret_cast<const uint4*>(lay->instance_infos);
    a.mc.side_infos = reinterpret_cast<const uint2*>(lay->side_infos);
    a.mc.surface_prefix = lay->surface_prefix;
    a.mc.instance_count = lay->instance_count;
    a.mc.payload_count = lay->payload_count;
    a.adjacency = reinterpret_cast<const uint4*>(adjacency);
    a.normals = reinterpret_cast<const float4*>(face_normals);
    a.src = reinterpret_cast<const float4*>(src);
    a.dst = reinterpret_cast<float4*>(dst);
    a.neighbor_weight = neighbor_weight;
    a.sigma = sigma;
    a.total_texels = lay->total_surface_texels;
    k_filter_mesh_colors<<<blocks_for(a.total_texels, 128), 128, 0, st>>>(a);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "filter_mesh_colors launch");
}

int launch_accumulate(NanContext* ctx, const float* input, float* output, float* history, uint32_t w, uint32_t h,
                      int reset, cudaStream_t st) {
    const uint64_t n = (uint64_t)w * h;
    if (n == 0) return NAN_OK;
    k_accumulate<<<blocks_for(n, 256), 256, 0, st>>>(reinterpret_cast<const float4*>(input),
                                                     reinterpret_cast<float4*>(output),
                                                     reinterpret_cast<float4*>(history), (uint32_t)n, reset);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "accumulate launch");
}

int launch_trace_texels(NanContext* ctx, const NanMeshColorsDesc* lay, uint8_t* slots, uint32_t iteration,
                        uint32_t spt, uint32_t max_bounces, int reset, const NanLighting* light, uint32_t begin,
                        uint32_t end, cudaStream_t st) {
    if (end <= begin) return NAN_OK;
    McView mc;
    mc.compensation = reinterpret_cast<float4*>(lay->compensation);
    mc.face_infos = reinterpret_cast<const uint2*>(lay->face_infos);
    mc.instance_infos = reinterpret_cast<const uint4*>(lay->instance_infos);
    mc.side_infos = reinterpret_cast<const uint2*>(lay->side_infos);
    mc.surface_prefix = lay->surface_prefix;
    mc.instance_count = lay->instance_count;
    mc.payload_count = lay->payload_count;
    k_trace_texels<<<blocks_for(end - begin, 128), 128, 0, st>>>(scene_view(ctx), to_raw(light), mc,
                                                                  reinterpret_cast<uint4*>(slots), iteration, spt,
                                                                  max_bounces, reset, begin, end, ctx->d_counters);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "trace_texels launch");
}

int launch_trace_points(NanContext* ctx, const float* points, uint32_t count, float* out, uint32_t iteration,
                        uint32_t samples, uint32_t max_bounces, uint32_t flags, const NanLighting* light,
                        cudaStream_t st) {
    if (count == 0) return NAN_OK;
    k_trace_points<<<blocks_for(count, 128), 128, 0, st>>>(
        scene_view(ctx), to_raw(light), reinterpret_cast<const float4*>(points), count, reinterpret_cast<float4*>(out),
        iteration, std::max(samples, 1u), std::max(max_bounces, 1u), (flags & NAN_POINTS_INDIRECT_ONLY) ? 1 : 0,
        ctx->d_counters);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "trace_points launch");
}

int launch_trace_probes(NanContext* ctx, float* values, uint32_t* counts, uint32_t* self_hits, uint32_t* radial,
                        const uint8_t* probes, uint32_t probe_count, const uint8_t* probe_instances,
                        uint32_t probe_instance_count, uint32_t iteration, uint32_t spp, uint32_t max_bounces,
                        int reset, const NanLighting* light, uint32_t begin, uint32_t end, float* compensation,
                        cudaStream_t st) {
    end = std::min(end, probe_count);
    if (end <= begin) return NAN_OK;
    ProbeOut o{reinterpret_cast<float4*>(compensation), values, counts, self_hits, radial};
    k_trace_probes<<<blocks_for(end - begin, 128), 128, 0, st>>>(
        scene_view(ctx), to_raw(light), o, reinterpret_cast<const float4*>(probes),
        reinterpret_cast<const float4*>(probe_instances), probe_count, probe_instance_count, iteration, spp,
        max_bounces, reset, begin, end,
        ctx->d_counters);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "trace_probes launch");
}

int launch_trace_probes_prt(NanContext* ctx, float* values, uint32_t* counts, uint32_t* self_hits, uint32_t* radial,
                            float* static_source, const uint8_t* probes, uint32_t probe_count,
                            const uint8_t* probe_instances, uint32_t probe_instance_count, uint32_t iteration,
                            uint32_t spp, uint32_t max_bounces, int reset, const NanLighting* light, uint32_t begin,
                            uint32_t end, cudaStream_t st) {
    end = std::min(end, probe_count);
    if (end <= begin) return NAN_OK;
    PrtOut o{values, counts, self_hits, radial, static_source};
    k_trace_probes_prt<<<blocks_for(end - begin, 128), 128, 0, st>>>(
        scene_view(ctx), to_raw(light), o, reinterpret_cast<const float4*>(probes),
        reinterpret_cast<const float4*>(probe_instances), probe_count, probe_instance_count, iteration, spp,
        max_bounces, reset, begin, end, ctx->d_counters);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "trace_probes_prt launch");
}

int launch_prt_project_lighting(NanContext* ctx, float* sh, uint32_t samples, const NanLighting* light,
                                cudaStream_t st) {
    k_prt_project_lighting<<<1, 256, 0, st>>>(to_raw(light), reinterpret_cast<float4*>(sh), samples);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "prt_project_lighting launch");
}

int launch_prt_evaluate(NanContext* ctx, const float* values, const uint32_t* counts, const float* static_source,
                        const float* sh, float* out, uint32_t* out_counts, uint32_t n, cudaStream_t st) {
    if (n == 0) return NAN_OK;
    k_prt_evaluate<<<blocks_for(n, 256), 256, 0, st>>>(values, counts, static_source,
                                                       reinterpret_cast<const float4*>(sh), out, out_counts, n);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "prt_evaluate launch");
}

int launch_pack_rgb9e5(NanContext* ctx, const uint8_t* slots, uint32_t* out, uint32_t count, cudaStream_t st) {
    if (count == 0) return NAN_OK;
    k_pack_rgb9e5<<<blocks_for(count, 256), 256, 0, st>>>(reinterpret_cast<const uint4*>(slots), out, count);
    ctx->launches++;
    return cuda_fail(cudaGetLastError(), "pack_rgb9e5 launch");
}

}  // namespace nan_host
