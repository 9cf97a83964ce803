// nan_probe_gather.cuh -- surface-probe reconstruction at a surface point:
// the point-octree gather with its weights (surface_probes.slang:272-392),
// the Chebyshev radial-visibility prior (surface_probes.slang:478-535), the
// selection of the 32 strongest of up to 96 candidates (:394-416), the 2R
// fallback merge (:418-460) and the weighted reconstruction
// (surface_probe_irradiance_field.slang:28-81), as used by
// surface_probe_resolve.slang:122-226.
//
// Arithmetic follows nan_math.cuh (no contraction, IEEE division and sqrt);
// exp and log2 are nan_exp / nan_log2 and lerp(a, b, t) = a + t * (b - a).
// Every index read from the layout is checked against its buffer; a bad one
// sets kStatusBadRecord and is skipped.
#pragma once

#include <cuda_fp16.h>

#include "nan_scene.cuh"

namespace nbd {

constexpr uint32_t kProbeMaxGather = 32;
constexpr uint32_t kProbeMaxCandidates = 96;
constexpr uint32_t kProbeOctreeStack = 64;
constexpr float kProbeHardNormalCos = 0.17364818f;

struct ProbeLayoutView {
    const float4* probes;     // 3 x float4 per probe: position_radius, normal_side, meta (as uint)
    const uint4* nodes;       // (child_base, child_mask, probe_start, probe_count)
    const float4* instances;  // 3 x float4 per instance: root_center_extent, offsets (as uint), params
    const uint4* tri_vertex_probes;
    uint32_t probe_count, node_count, instance_count, tri_map_count;
};

struct ProbeFieldView {
    const float* values;  // irradiance f32[N][3]
    const uint32_t* counts;
    const uint32_t* self_hits;
    const uint32_t* radial;  // RG16F u32[N][16]
};

struct ProbeInstance {
    f3 root_center;
    float root_extent;
    uint4 offsets;  // node offset, node count, probe offset, probe count
    float kernel_radius, normal_cos, plane_sigma;
    uint32_t tri_map_offset;
};

__device__ __forceinline__ ProbeInstance load_probe_instance(const ProbeLayoutView& v, uint32_t i) {
    const float4 a = __ldg(v.instances + 3u * i);
    const float4 b = __ldg(v.instances + 3u * i + 1u);
    const float4 c = __ldg(v.instances + 3u * i + 2u);
    ProbeInstance r;
    r.root_center = mk3(a.x, a.y, a.z);
    r.root_extent = a.w;
    r.offsets = make_uint4(__float_as_uint(b.x), __float_as_uint(b.y), __float_as_uint(b.z), __float_as_uint(b.w));
    r.kernel_radius = c.x;
    r.normal_cos = c.y;
    r.plane_sigma = c.z;
    r.tri_map_offset = __float_as_uint(c.w);
    return r;
}

__device__ __forceinline__ f3 probe_position(const ProbeLayoutView& v, uint32_t p) {
    const float4 a = __ldg(v.probes + 3u * p);
    return mk3(a.x, a.y, a.z);
}

__device__ __forceinline__ float4 probe_normal_side(const ProbeLayoutView& v, uint32_t p) {
    return __ldg(v.probes + 3u * p + 1u);
}

__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + t * (b - a); }
__device__ __forceinline__ f3 lerp3(f3 a, f3 b, float t) { return a + t * (b - a); }

__device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
    const float t = sat((x - e0) / (e1 - e0));
    return (t * t) * (3.0f - 2.0f * t);
}

__device__ __forceinline__ float soft_normal_weight(float nc, float full_cos) {
    const float soft_end = maxf(full_cos, kProbeHardNormalCos + 1e-3f);
    return smoothstepf(kProbeHardNormalCos, soft_end, nc) * maxf(nc, 0.0f);
}

__device__ __forceinline__ bool sphere_meets_cube(f3 p, float r, f3 c, float e) {
    const f3 a = abs3(p - c);
    const f3 d = mk3(maxf(a.x - e, 0.0f), maxf(a.y - e, 0.0f), maxf(a.z - e, 0.0f));
    return dot3(d, d) <= r * r;
}

struct Candidates {
    uint32_t count;
    uint32_t index[kProbeMaxCandidates];
    float weight[kProbeMaxCandidates];
};

struct Gathered {
    uint32_t count;
    uint32_t index[kProbeMaxGather];
    float weight[kProbeMaxGather];
};

// surface_probe_gather: probes within the kernel radius (scaled), past the
// hard normal gate, weighted by (1 - d^2/R^2)^2, the plane-distance Gaussian
// and the soft normal gate; beyond 96 the weakest (first minimum) is replaced.
__device__ __noinline__ void probe_gather(const ProbeLayoutView& v, const ProbeInstance& ins, f3 q, f3 qn,
                                          float radius_scale, Candidates& out, uint32_t* status) {
    out.count = 0u;
    const float kr = maxf(ins.kernel_radius * maxf(radius_scale, 1.0f), 1e-6f);
    const float ncos = ins.normal_cos;
    const float ps = maxf(ins.plane_sigma, 1e-6f);
    const float kr2 = kr * kr;
    uint32_t st_node[kProbeOctreeStack];
    f3 st_center[kProbeOctreeStack];
    float st_extent[kProbeOctreeStack];
    uint32_t n = 1u;
    st_node[0] = ins.offsets.x;
    st_center[0] = ins.root_center;
    st_extent[0] = ins.root_extent;
    while (n > 0u) {
        n -= 1u;
        const uint32_t ni = st_node[n];
        const f3 c = st_center[n];
        const float e = st_extent[n];
        if (!sphere_meets_cube(q, kr, c, e)) continue;
        if (ni >= v.node_count) {
            atomicOr(status, kStatusBadRecord);
            continue;
        }
        const uint4 node = __ldg(v.nodes + ni);
        if (node.y == 0u) {
            if (node.z > v.probe_count || node.w > v.probe_count - node.z) {
                atomicOr(status, kStatusBadRecord);
                continue;
            }
            for (uint32_t k = 0; k < node.w; ++k) {
                const uint32_t p = node.z + k;
                const f3 delta = probe_position(v, p) - q;
                const float d2 = dot3(delta, delta);
                if (d2 > kr2) continue;
                const float4 ns = probe_normal_side(v, p);
                const float nc = dot3(qn, normalize3(mk3(ns.x, ns.y, ns.z)));
                if (nc < kProbeHardNormalCos) continue;
                const float pd = fabsf(dot3(delta, qn));
                const float pw = nan_exp((-0.5f * (pd / ps)) * (pd / ps));
                const float sp = maxf(1.0f - d2 / kr2, 0.0f);
                const float w = ((sp * sp) * pw) * soft_normal_weight(nc, ncos);
                if (w <= 1e-6f) continue;
                if (out.count < kProbeMaxCandidates) {
                    out.index[out.count] = p;
                    out.weight[out.count] = w;
                    out.count += 1u;
                } else {
                    uint32_t weakest = 0u;
                    for (uint32_t i = 1; i < kProbeMaxCandidates; ++i)
                        if (out.weight[i] < out.weight[weakest]) weakest = i;
                    if (w > out.weight[weakest]) {
                        out.index[weakest] = p;
                        out.weight[weakest] = w;
                    }
                }
            }
            continue;
        }
        const float ce = e * 0.5f;
        uint32_t compact = 0u;
        for (uint32_t o = 0; o < 8u; ++o) {
            if (!(node.y & (1u << o))) continue;
            const f3 off = mk3((o & 1u) ? 1.0f : -1.0f, (o & 2u) ? 1.0f : -1.0f, (o & 4u) ? 1.0f : -1.0f);
            const f3 cc = c + off * ce;
            if (sphere_meets_cube(q, kr, cc, ce) && n < kProbeOctreeStack) {
                st_node[n] = node.x + compact;
                st_center[n] = cc;
                st_extent[n] = ce;
                n += 1u;
            }
            compact += 1u;
        }
    }
}

__device__ __forceinline__ float2 load_radial(const uint32_t* radial, uint32_t p, uint32_t texel) {
    const uint32_t packed = __ldg(radial + 16u * p + min(texel, 15u));
    return make_float2(__half2float(__ushort_as_half((unsigned short)(packed & 0xffffu))),
                       __half2float(__ushort_as_half((unsigned short)(packed >> 16))));
}

// surface_probe_hemi_oct_encode (surface_probes.slang:134-155).
__device__ __forceinline__ float2 hemi_oct_encode(f3 d) {
    f3 h = mk3(d.x, d.y, maxf(d.z, 0.0f));
    const float l2 = dot3(h, h);
    if (l2 <= 1e-12f) return make_float2(0.5f, 0.5f);
    h = h * (1.0f / sqrtf(l2));
    const float inv_l1 = 1.0f / maxf((fabsf(h.x) + fabsf(h.y)) + h.z, 1e-6f);
    const float ox = h.x * inv_l1, oy = h.y * inv_l1;
    return make_float2(sat((ox + oy) * 0.5f + 0.5f), sat((ox - oy) * 0.5f + 0.5f));
}

// surface_probe_sample_radial_moments: bilinear over the 4x4 texels with
// centres at (n + 0.5)/4, only texels holding a second moment count.
__device__ __forceinline__ float2 sample_radial(const uint32_t* radial, uint32_t p, float2 uv, float* valid) {
    const float tx = sat(uv.x) * 4.0f - 0.5f, ty = sat(uv.y) * 4.0f - 0.5f;
    const float fx = floorf(tx), fy = floorf(ty);
    const int bx = (int)fx, by = (int)fy;
    const float ax = tx - fx, ay = ty - fy;
    const int x0 = max(min(bx, 3), 0), x1 = max(min(bx + 1, 3), 0);
    const int y0 = max(min(by, 3), 0), y1 = max(min(by + 1, 3), 0);
    const float w[4] = {(1.0f - ax) * (1.0f - ay), ax * (1.0f - ay), (1.0f - ax) * ay, ax * ay};
    const uint32_t t[4] = {(uint32_t)(y0 * 4 + x0), (uint32_t)(y0 * 4 + x1), (uint32_t)(y1 * 4 + x0),
                           (uint32_t)(y1 * 4 + x1)};
    float mx = 0.0f, my = 0.0f, vw = 0.0f;
    for (int i = 0; i < 4; ++i) {
        const float2 s = load_radial(radial, p, t[i]);
        if (s.y > 0.0f) {
            mx = mx + s.x * w[i];
            my = my + s.y * w[i];
            vw = vw + w[i];
        }
    }
    *valid = vw;
    return vw > 1e-6f ? make_float2(mx / vw, my / vw) : make_float2(0.0f, 0.0f);
}

__device__ __forceinline__ float chebyshev_visibility(float2 m, float nd) {
    if (m.y <= 0.0f) return 1.0f;
    const float mean = maxf(m.x, 0.0f);
    if (nd <= mean + 0.035f) return 1.0f;
    const float var = maxf(m.y - mean * mean, 2.5e-3f);
    const float diff = nd - mean;
    const float prob = var / (var + diff * diff);
    return maxf(sat((prob - 0.2f) / 0.8f), 0.05f);
}

__device__ __forceinline__ float radial_visibility(const ProbeLayoutView& v, const ProbeFieldView& f, uint32_t p,
                                                   f3 q, float kernel_radius, uint32_t sample_count,
                                                   bool enabled) {
    if (!enabled) return 1.0f;
    const f3 delta = q - probe_position(v, p);
    const float dist = len3(delta);
    if (dist <= 1e-6f) return 1.0f;
    const float4 ns = probe_normal_side(v, p);
    const f3 local = Frame(normalize3(mk3(ns.x, ns.y, ns.z))).to_local(delta / dist);
    const float nd = minf(dist / maxf(kernel_radius, 1e-6f), 2.0f);
    float valid;
    const float2 m = sample_radial(f.radial, p, hemi_oct_encode(local), &valid);
    if (valid <= 1e-6f) return 1.0f;
    const float vis = chebyshev_visibility(m, nd);
    const float tc = sat((float)sample_count / 32.0f);
    return lerpf(1.0f, vis, 0.75f * tc);
}

// surface_probe_select_strongest: repeatedly the first unconsumed candidate of
// the largest weight, up to 32.
__device__ __forceinline__ void select_strongest(const Candidates& c, Gathered& out) {
    out.count = 0u;
    uint32_t used[3] = {0u, 0u, 0u};
    for (uint32_t sel = 0; sel < c.count && out.count < kProbeMaxGather; ++sel) {
        uint32_t best = 0u;
        float bw = -1.0f;
        for (uint32_t i = 0; i < c.count; ++i) {
            const bool consumed = (used[i >> 5] >> (i & 31u)) & 1u;
            if (!consumed && c.weight[i] > bw) {
                best = i;
                bw = c.weight[i];
            }
        }
        used[best >> 5] |= 1u << (best & 31u);
        out.index[out.count] = c.index[best];
        out.weight[out.count] = bw;
        out.count += 1u;
    }
}

__device__ __forceinline__ void merge_fallback(const Gathered& fb, float scale, Gathered& g) {
    for (uint32_t k = 0; k < fb.count; ++k) {
        bool dup = false;
        for (uint32_t i = 0; i < g.count; ++i)
            if (g.index[i] == fb.index[k]) {
                dup = true;
                break;
            }
        if (dup) continue;
        const float w = fb.weight[k] * scale;
        if (w <= 1e-8f) continue;
        if (g.count < kProbeMaxGather) {
            g.index[g.count] = fb.index[k];
            g.weight[g.count] = w;
            g.count += 1u;
        } else {
            uint32_t weakest = 0u;
            for (uint32_t i = 1; i < g.count; ++i)
                if (g.weight[i] < g.weight[weakest]) weakest = i;
            if (w > g.weight[weakest]) {
                g.index[weakest] = fb.index[k];
                g.weight[weakest] = w;
            }
        }
    }
}

__device__ __forceinline__ float weight_ess(const Gathered& g) {
    float s = 0.0f, s2 = 0.0f;
    for (uint32_t i = 0; i < g.count; ++i) {
        const float w = maxf(g.weight[i], 0.0f);
        s = s + w;
        s2 = s2 + w * w;
    }
    return s2 > 1e-12f ? (s * s) / s2 : 0.0f;
}

__device__ __forceinline__ f3 probe_irradiance(const ProbeFieldView& f, uint32_t p) {
    return mk3(__ldg(f.values + 3u * p), __ldg(f.values + 3u * p + 1u), __ldg(f.values + 3u * p + 2u));
}

struct ProbeReconstruction {
    f3 irradiance;
    uint32_t gathered;
    float support, weight_sum, ess, self_hit_rate;
};

__device__ __forceinline__ void weight_by_visibility(const ProbeLayoutView& v, const ProbeFieldView& f,
                                                     Candidates& c, f3 q, float kernel_radius, bool radial) {
    for (uint32_t i = 0; i < c.count; ++i)
        c.weight[i] = c.weight[i] * radial_visibility(v, f, c.index[i], q, kernel_radius,
                                                      __ldg(f.counts + c.index[i]), radial);
}

// surface_probe_sample_irradiance (surface_probe_resolve.slang:122-226).
__device__ __forceinline__ ProbeReconstruction probe_reconstruct(const ProbeLayoutView& v, const ProbeFieldView& f,
                                                                 const ProbeInstance& ins, f3 q, f3 qn,
                                                                 uint32_t min_gather, bool radial,
                                                                 Candidates& cand, uint32_t* status) {
    Gathered g;
    probe_gather(v, ins, q, qn, 1.0f, cand, status);
    weight_by_visibility(v, f, cand, q, ins.kernel_radius, radial);
    select_strongest(cand, g);
    const uint32_t mg = min(max(min_gather, 1u), 32u);
    const float ess0 = weight_ess(g);
    const float fs = smoothstepf(0.0f, 1.0f, sat(((float)mg - ess0) / (float)mg));
    if (fs > 1e-4f) {
        Gathered fb;
        probe_gather(v, ins, q, qn, 2.0f, cand, status);
        weight_by_visibility(v, f, cand, q, ins.kernel_radius, radial);
        select_strongest(cand, fb);
        merge_fallback(fb, 0.25f * fs, g);
    }
    ProbeReconstruction r;
    float shs = 0.0f, shw = 0.0f;
    for (uint32_t i = 0; i < g.count; ++i) {
        const uint32_t p = g.index[i];
        const uint32_t sc = __ldg(f.counts + p);
        if (sc == 0u) continue;
        const float rate = (float)__ldg(f.self_hits + p) / (float)sc;
        shs = shs + g.weight[i] * rate;
        shw = shw + g.weight[i];
    }
    r.self_hit_rate = shw > 1e-6f ? shs / shw : 0.0f;
    // surface_probe_reconstruct_irradiance
    f3 acc = mk3(0.0f, 0.0f, 0.0f);
    float ws = 0.0f, wss = 0.0f, ss = 0.0f, ssw = 0.0f, best_w = -1.0f;
    f3 best = mk3(0.0f, 0.0f, 0.0f);
    for (uint32_t i = 0; i < g.count; ++i) {
        const uint32_t p = g.index[i];
        ss = ss + g.weight[i] * sat(probe_normal_side(v, p).w);
        ssw = ssw + g.weight[i];
        const f3 irr = probe_irradiance(f, p);
        const float conf = __ldg(f.counts + p) > 0u ? 1.0f : 0.0f;
        const float w = g.weight[i] * conf;
        acc = acc + w * irr;
        ws = ws + w;
        wss = wss + w * w;
        if (w > best_w) {
            best_w = w;
            best = irr;
        }
    }
    r.gathered = g.count;
    r.support = ssw > 1e-6f ? sat(ss / ssw) : 0.0f;
    r.weight_sum = ws;
    r.ess = wss > 1e-12f ? (ws * ws) / wss : 0.0f;
    if (ws > 1e-6f)
        r.irradiance = acc / ws;
    else if (best_w >= 0.0f)
        r.irradiance = best;
    else
        r.irradiance = mk3(0.0f, 0.0f, 0.0f);
    return r;
}

// Debug colours of surface_probe_resolve.slang:29-120.
__device__ __forceinline__ f3 gather_count_color(uint32_t n) {
    if (n == 0u) return mk3(1.0f, 0.0f, 1.0f);
    if (n < 4u) return lerp3(mk3(1.0f, 0.0f, 0.0f), mk3(1.0f, 0.5f, 0.0f), (float)(n - 1u) / 3.0f);
    if (n < 8u) return lerp3(mk3(1.0f, 1.0f, 0.0f), mk3(0.0f, 1.0f, 0.0f), (float)(n - 4u) / 4.0f);
    if (n < 16u) return lerp3(mk3(0.0f, 1.0f, 0.0f), mk3(0.0f, 1.0f, 1.0f), (float)(n - 8u) / 8.0f);
    if (n < 24u) return lerp3(mk3(0.0f, 1.0f, 1.0f), mk3(0.0f, 0.0f, 1.0f), (float)(n - 16u) / 8.0f);
    return lerp3(mk3(0.0f, 0.0f, 1.0f), mk3(1.0f, 1.0f, 1.0f), (float)(min(n, 32u) - 24u) / 8.0f);
}

__device__ __forceinline__ f3 support_color(float s) {
    const float v = sat(s);
    if (v < 0.25f) return lerp3(mk3(1.0f, 0.0f, 1.0f), mk3(1.0f, 0.0f, 0.0f), v * 4.0f);
    if (v < 0.5f) return lerp3(mk3(1.0f, 0.0f, 0.0f), mk3(1.0f, 1.0f, 0.0f), (v - 0.25f) * 4.0f);
    if (v < 0.75f) return lerp3(mk3(1.0f, 1.0f, 0.0f), mk3(0.0f, 1.0f, 0.0f), (v - 0.5f) * 4.0f);
    return lerp3(mk3(0.0f, 1.0f, 0.0f), mk3(0.0f, 0.25f, 1.0f), (v - 0.75f) * 4.0f);
}

__device__ __forceinline__ f3 density_color(float s, float max_density) {
    const float mx = maxf(max_density, 1.0f);
    const float density = minf(mx, 1.0f / maxf(sat(s), 1.0f / mx));
    const float normalized = mx > 1.0f ? nan_log2(density) / nan_log2(mx) : 0.0f;
    return support_color(1.0f - sat(normalized));
}

__device__ __forceinline__ f3 self_hit_color(float rate) {
    if (rate <= 0.0f) return mk3(0.0f, 0.0f, 0.25f);
    const float lr = nan_log2(maxf(rate, 1e-6f)) / nan_log2(10.0f);
    const float v = sat((lr + 6.0f) / 5.0f);
    if (v < 1.0f / 3.0f) return lerp3(mk3(0.0f, 0.0f, 0.25f), mk3(0.0f, 1.0f, 1.0f), v * 3.0f);
    if (v < 2.0f / 3.0f) return lerp3(mk3(0.0f, 1.0f, 1.0f), mk3(1.0f, 1.0f, 0.0f), (v - 1.0f / 3.0f) * 3.0f);
    return lerp3(mk3(1.0f, 1.0f, 0.0f), mk3(1.0f, 0.0f, 0.0f), (v - 2.0f / 3.0f) * 3.0f);
}

}  // namespace nbd
