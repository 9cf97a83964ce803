// nan_sinks.cuh -- the accumulation targets of the integrators: Mesh Colors
// lattice addressing and 16-byte running-mean slots, surface-probe radial
// depth moments, and warp-aggregated ray counters. Shared by the megakernel
// and the wavefront translation units (both compiled with --fmad=false).
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

#include "nan_scene.cuh"

namespace nbd {

// Warp-aggregated update of the context counters.
__device__ __forceinline__ void flush_tally(unsigned long long* counters, const RayTally& t, uint32_t units,
                                            uint32_t paths) {
    const unsigned mask = __activemask();
    const uint32_t e = __reduce_add_sync(mask, t.extend);
    const uint32_t s = __reduce_add_sync(mask, t.shadow);
    const uint32_t u = __reduce_add_sync(mask, units);
    const uint32_t p = __reduce_add_sync(mask, paths);
    if ((threadIdx.x & 31u) == (uint32_t)(__ffs(mask) - 1)) {
        atomicAdd(counters + 0, (unsigned long long)e);
        atomicAdd(counters + 1, (unsigned long long)s);
        atomicAdd(counters + 2, (unsigned long long)u);
        atomicAdd(counters + 3, (unsigned long long)p);
    }
}


// ---------------------------------------------------------------------------
// Mesh Colors lattice (mesh_colors.slang:37-65, 272-363).
// ---------------------------------------------------------------------------
struct McView {
    float4* compensation;  // optional Kahan terms of the running means, one per payload slot
    const uint2* face_infos;
    const uint4* instance_infos;
    const uint2* side_infos;
    const uint32_t* surface_prefix;
    uint32_t instance_count;
    uint32_t payload_count;
};

__device__ __forceinline__ uint32_t mc_address(uint32_t i, uint32_t j, uint32_t texel_offset, uint2 face) {
    const uint32_t row = i * (face.y + 1u) - i * (i - 1u) / 2u;
    return texel_offset + face.x + row + j;
}

__device__ __forceinline__ void mc_address_to_ij(uint32_t address, uint32_t r, uint32_t* oi, uint32_t* oj) {
    uint32_t left = 0u, right = r;
    while (left < right) {
        const uint32_t mid = (left + right + 1u) / 2u;
        const uint32_t ma = mid * (r + 1u) - mid * (mid - 1u) / 2u;
        if (ma <= address) left = mid; else right = mid - 1u;
    }
    *oi = left;
    *oj = address - (left * (r + 1u) - left * (left - 1u) / 2u);
}

__device__ __forceinline__ float fracf(float x) { return x - floorf(x); }

__device__ __forceinline__ uint32_t mc_nearest_texel(float b0, float b1, float b2, uint32_t texel_offset, uint2 face) {
    const uint32_t R = face.y;
    const float rf = (float)R;
    const float s0 = sat(b0) * rf, s1 = sat(b1) * rf, s2 = sat(b2) * rf;
    uint32_t i = (uint32_t)s0, j = (uint32_t)s1;
    i = min(i, R);
    j = min(j, R - i);
    float w0 = fracf(s0), w1 = fracf(s1), w2 = fracf(s2);
    const bool upper = fabsf(((w0 + w1) + w2) - 2.0f) <= 1e-3f;
    if (upper) {
        w0 = 1.0f - w0;
        w1 = 1.0f - w1;
        w2 = 1.0f - w2;
    }
    if ((w0 + w1) + w2 <= 1e-6f || i >= R || j >= R - i) return mc_address(i, j, texel_offset, face);
    const float largest = maxf(w0, maxf(w1, w2));
    if (upper) {
        if (fabsf(largest - w0) < 1e-3f) return mc_address(i, j + 1u, texel_offset, face);
        if (fabsf(largest - w1) < 1e-3f) return mc_address(i + 1u, j, texel_offset, face);
        return mc_address(i + 1u, j + 1u, texel_offset, face);
    }
    if (fabsf(largest - w0) < 1e-3f) return mc_address(i + 1u, j, texel_offset, face);
    if (fabsf(largest - w1) < 1e-3f) return mc_address(i, j + 1u, texel_offset, face);
    return mc_address(i, j, texel_offset, face);
}


// Surface point of surface texel u (texture_space_path_tracer.slang:144-200):
// instance by binary search over the surface prefix, face by
// mesh_colors_find_face, lattice (i, j), then up to 32 jittered candidates
// accepted when inside the triangle and nearest to this texel. Leaves the
// RNG where the reference's compute_main leaves it.
struct TexelSurface {
    uint32_t inst, prim, global_texel;
    float b1, b2;  // HitInfo.bary of the surface point
    uint4 inst_info;
    uint2 side;
};

__device__ __forceinline__ bool texel_surface(const SceneView& s, const McView& mc, uint32_t u, uint32_t iteration,
                                              uint32_t spt, TexelSurface* out, Rng* rng_out) {
    // instance = last i with surface_prefix[i] <= u
    uint32_t lo = 0u, hi = mc.instance_count - 1u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (__ldg(mc.surface_prefix + mid) <= u) lo = mid; else hi = mid - 1u;
    }
    const uint32_t inst_index = lo;
    const uint32_t local = u - __ldg(mc.surface_prefix + inst_index);
    const uint4 inst = __ldg(mc.instance_infos + inst_index);  // face off, face count, texel off, texel count
    const uint2 side = __ldg(mc.side_infos + inst_index);
    if (local >= inst.w) return false;
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
    if (!found) return false;
    if (!valid_prim(s, inst_index, prim)) {
        atomicOr(s.status, kStatusBadRecord);
        return false;
    }
    const uint32_t global_texel = inst.z + local;
    uint32_t ti, tj;
    mc_address_to_ij(local - face.x, face.y, &ti, &tj);
    const float rf = (float)face.y;
    const float base_x = (float)ti / rf, base_y = (float)tj / rf;
    const uint32_t n = max(spt, 1u);
    Rng rng(global_texel, inst_index, iteration * n);
    float bx = base_x, by = base_y;
    for (uint32_t attempt = 0; attempt < 32u; ++attempt) {
        const float r0 = rng.next_1d(), r1 = rng.next_1d();
        const float cx = base_x + (r0 - 0.5f) / rf;
        const float cy = base_y + (r1 - 0.5f) / rf;
        if (cx < 0.0f || cy < 0.0f || cx + cy > 1.0f) continue;
        if (mc_nearest_texel(cx, cy, (1.0f - cx) - cy, inst.z, face) == global_texel) {
            bx = cx;
            by = cy;
            break;
        }
    }
    out->inst = inst_index;
    out->prim = prim;
    out->global_texel = global_texel;
    out->b1 = by;
    out->b2 = maxf(0.0f, (1.0f - bx) - by);
    out->inst_info = inst;
    out->side = side;
    *rng_out = rng;
    return true;
}

// store_accumulated_irradiance, texture_space_path_tracer.slang:119-138.
// One step of the running mean m' = m + (x - m)/(n + 1). Without a
// compensation term this is the reference's lerp. With one, the increments
// are summed with Kahan compensation (the term lives beside the slot), so the
// mean does not drift by one rounding per sample over long accumulations.
__device__ __forceinline__ f3 running_mean_step(f3 m, f3 x, uint32_t prev, float4* comp) {
    if (comp == nullptr) {
        const float weight = 1.0f / (float)(prev + 1u);
        return m + weight * (x - m);
    }
    if (prev == 0u) {
        *comp = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return x;
    }
    const float weight = 1.0f / (float)(prev + 1u);
    const f3 inc = weight * (x - m);
    const f3 c = mk3(comp->x, comp->y, comp->z);
    const f3 y = inc - c;
    const f3 t = m + y;
    const f3 nc = (t - m) - y;
    *comp = make_float4(nc.x, nc.y, nc.z, 0.0f);
    return t;
}

__device__ __forceinline__ void store_running_mean(uint4* __restrict__ slots, uint32_t texel, f3 v, int reset,
                                                   float4* __restrict__ comp = nullptr) {
    uint4 old = make_uint4(0u, 0u, 0u, 0u);
    if (!reset) old = slots[texel];
    const uint32_t prev = reset ? 0u : old.w;
    f3 pv = mk3(0.0f, 0.0f, 0.0f);
    if (prev != 0u) pv = mk3(__uint_as_float(old.x), __uint_as_float(old.y), __uint_as_float(old.z));
    const uint32_t next = min(prev + 1u, 65535u);
    float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (comp) c = comp[texel];
    const f3 acc = running_mean_step(pv, v, prev, comp ? &c : nullptr);
    if (comp) comp[texel] = c;
    slots[texel] = make_uint4(__float_as_uint(acc.x), __float_as_uint(acc.y), __float_as_uint(acc.z), next);
}


// ---------------------------------------------------------------------------
// Surface-probe radial moments (surface_probe_path_tracer.slang:95-149,
// surface_probes.slang:84-167).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float radial_texel_cosine_probability(uint32_t texel) {
    const uint32_t cx = texel % 4u, cy = texel / 4u;
    const bool hb = cx == 0u || cx == 3u;
    const bool vb = cy == 0u || cy == 3u;
    if (hb && vb) return 0.02221812f;
    if (hb || vb) return 0.06578385f;
    return 0.09621418f;
}

// surface_probe_hemi_oct_encode + radial texel, surface_probes.slang:134-167.
__device__ __forceinline__ uint32_t radial_texel(f3 d) {
    f3 h = mk3(d.x, d.y, maxf(d.z, 0.0f));
    const float l2 = dot3(h, h);
    float u = 0.5f, v = 0.5f;
    if (!(l2 <= 1e-12f)) {
        h = h * (1.0f / sqrtf(l2));
        const float inv_l1 = 1.0f / maxf((fabsf(h.x) + fabsf(h.y)) + h.z, 1e-6f);
        const float ox = h.x * inv_l1, oy = h.y * inv_l1;
        u = sat((ox + oy) * 0.5f + 0.5f);
        v = sat((ox - oy) * 0.5f + 0.5f);
    }
    const uint32_t x = min((uint32_t)(sat(u) * 4.0f), 3u);
    const uint32_t y = min((uint32_t)(sat(v) * 4.0f), 3u);
    return y * 4u + x;
}

struct ProbeOut {
    float4* compensation;  // optional Kahan terms of the running means, one per probe
    float* values;
    uint32_t* counts;
    uint32_t* self_hits;
    uint32_t* radial;
};

// accumulate_radial_moment, surface_probe_path_tracer.slang:111-149.
__device__ __forceinline__ void accumulate_radial_moment(uint32_t* __restrict__ radial, uint32_t probe, uint32_t texel,
                                                         float nd, uint32_t prev_iter, uint32_t local_count,
                                                         uint32_t spp) {
    uint32_t* slot = radial + 16u * probe + texel;
    const uint32_t packed = *slot;
    float px = __half2float(__ushort_as_half((unsigned short)(packed & 0xffffu)));
    float py = __half2float(__ushort_as_half((unsigned short)(packed >> 16)));
    const float sample = minf(maxf(nd, 0.0f), 2.0f);
    const float smx = sample, smy = sample * sample;
    if (py <= 0.0f) {
        px = smx;
        py = smy;
    } else {
        const float pop = ((float)prev_iter * (float)max(spp, 1u)) * radial_texel_cosine_probability(texel);
        const uint32_t expected = prev_iter == 0u ? local_count - 1u : max((uint32_t)pop, 1u);
        const float alpha = 1.0f / (float)max(min(expected + local_count, 4096u), 1u);
        px = px + alpha * (smx - px);
        py = py + alpha * (smy - py);
    }
    px = minf(maxf(px, 0.0f), 4.0f);
    py = minf(maxf(py, 0.0f), 4.0f);
    *slot = (uint32_t)__half_as_ushort(__float2half_rn(px)) | ((uint32_t)__half_as_ushort(__float2half_rn(py)) << 16);
}


}  // namespace nbd
