// nan_probe.cuh -- one iteration of the surface-probe irradiance baker for
// one probe (surface_probe_path_tracer.slang:47-315), shared by the
// per-scene kernel and the multi-scene batched kernel. Templated on the
// traversal policy (nan_scene.cuh: DefaultTracer, BinaryTracer<depth>).
#pragma once

#include "nan_scene.cuh"
#include "nan_sinks.cuh"

namespace nbd {

template <class Tr>
__device__ __forceinline__ bool probe_unit(const SceneView& s, const LightParams& L, const ProbeOut& out,
                                           const float4* __restrict__ probes, const float4* __restrict__ pinst,
                                           uint32_t probe_instance_count, uint32_t iteration, uint32_t spp,
                                           uint32_t max_bounces, int reset, uint32_t p, RayTally& tally) {
    const float4 nrm = __ldg(probes + 3u * p + 1u);
    const uint4 meta = __ldg(reinterpret_cast<const uint4*>(probes) + 3u * p + 2u);
    const uint32_t inst = meta.w >> 8;
    if (inst >= probe_instance_count || !valid_prim(s, inst, meta.x)) {
        atomicOr(s.status, kStatusBadRecord);
        return false;
    }
    const float4 params = __ldg(pinst + 3u * inst + 2u);
    const float bx = __uint_as_float(meta.y), by = __uint_as_float(meta.z);
    const uint32_t prim = meta.x;
    const uint32_t n = max(spp, 1u);
    Rng rng(p, inst, iteration * n);
    const f3 view = normalize3(mk3(nrm.x, nrm.y, nrm.z));
    const float kr = maxf(params.x, 1e-6f);
    const Shading sd = shading_data(s, inst, prim, bx, by, view);
    f3 irr = mk3(0.0f, 0.0f, 0.0f);
    uint32_t self_total = 0u;
    const uint32_t prev_iter = reset ? 0u : out.counts[p];
    uint32_t local_counts[16];
#pragma unroll
    for (int t = 0; t < 16; ++t) local_counts[t] = 0u;
    if (reset)
        for (int t = 0; t < 16; ++t) out.radial[16u * p + (uint32_t)t] = 0u;
    const Frame surface_frame(normalize3(sd.face_normal));
    for (uint32_t k = 0; k < n; ++k) {
        f3 si = mk3(0.0f, 0.0f, 0.0f);
        const float e0 = rng.next_1d(), e1 = rng.next_1d();
        float pdf;
        const f3 dir = cosine_sample_hemisphere(e0, e1, &pdf);
        if (pdf > 1e-6f) {
            f3 o = sd.origin_front;
            f3 d = surface_frame.to_global(dir);
            f3 thp = mk3(1.0f, 1.0f, 1.0f), rad = mk3(0.0f, 0.0f, 0.0f);
            uint32_t src_inst = inst, src_prim = prim;
            float src_off = len3(o - sd.position);
            uint32_t self_hits = 0u;
            const float radial_max = 2.0f * kr;
            float first_hit = 2.0f * kr;
            // trace_radiance, surface_probe_path_tracer.slang:151-204
            for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
                tally.extend++;
                const HitInfo hit = Tr::closest(s, o, d, 0.0f, L.t_max);
                if (!hit.valid) {
                    if (bounce == 0u) first_hit = radial_max;
                    rad = rad + thp * L.sky;
                    break;
                }
                if (bounce == 0u) first_hit = minf(hit.t, radial_max);
                const uint2 ref = __ldg(s.tri_refs + hit.flat);
                const bool same_prim = ref.x == src_inst && ref.y == src_prim;
                const float thr = maxf(4.0f * src_off, 1e-6f);
                const bool adjacent = ref.x == src_inst && hit.t <= thr;
                if (same_prim || adjacent) self_hits += 1u;
                const Shading hs = shading_data(s, ref.x, ref.y, hit.b1, hit.b2, -d);
                rad = rad + thp * hs.emissive;
                const float u0 = rng.next_1d(), u1 = rng.next_1d();
                rad = rad + thp * sun_nee<Tr>(s, L, hs, u0, u1, tally);
                const float f0 = rng.next_1d(), f1 = rng.next_1d();
                float spdf;
                const f3 sdir = cosine_sample_hemisphere(f0, f1, &spdf);
                if (spdf <= 1e-6f) break;
                const f3 f = hs.diffuse * kInvPi;
                thp = thp * ((f * fabsf(sdir.z)) / spdf);
                const f3 next_origin = hs.origin_front;
                d = Frame(normalize3(hs.face_normal)).to_global(sdir);
                o = next_origin;
                src_inst = ref.x;
                src_prim = ref.y;
                src_off = len3(next_origin - hs.position);
            }
            self_total += self_hits;
            const uint32_t texel = radial_texel(dir);
            local_counts[texel] += 1u;
            accumulate_radial_moment(out.radial, p, texel, first_hit / maxf(kr, 1e-6f), prev_iter,
                                     local_counts[texel], spp);
            si = si + ((rad * fabsf(dir.z)) / pdf);
        }
        irr = irr + si;
    }
    irr = irr / (float)n;
    // store_accumulated_irradiance (:47-65)
    const uint32_t prev = reset ? 0u : out.counts[p];
    f3 pv = mk3(0.0f, 0.0f, 0.0f);
    if (prev != 0u) pv = mk3(out.values[3u * p], out.values[3u * p + 1u], out.values[3u * p + 2u]);
    float4 comp = out.compensation ? out.compensation[p] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const f3 acc = running_mean_step(pv, irr, prev, out.compensation ? &comp : nullptr);
    if (out.compensation) out.compensation[p] = comp;
    out.values[3u * p] = acc.x;
    out.values[3u * p + 1u] = acc.y;
    out.values[3u * p + 2u] = acc.z;
    out.counts[p] = min(prev + 1u, 65535u);
    // store_accumulated_self_hit_count (:67-79)
    const uint32_t prev_self = reset ? 0u : out.self_hits[p];
    out.self_hits[p] = prev_self + self_total;
    return true;
}

}  // namespace nbd
