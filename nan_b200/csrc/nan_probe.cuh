// nan_probe.cuh -- one iteration of the surface-probe irradiance baker for
// one probe (surface_probe_path_tracer.slang:47-315), shared by the
// per-scene kernel and the multi-scene batched kernel. Templated on the
// traversal policy (nan_scene.cuh: DefaultTracer, BinaryTracer<depth>).
#pragma once

#include "nan_scene.cuh"
#include "nan_sinks.cuh"

namespace nbd {

// One probe set of a multi-scene batch (nan_batch.cu): the scene, its
// lighting, the probe records and the outputs.
struct BatchSet {
    SceneView s;
    LightingRaw light;
    ProbeOut out;
    const float4* probes;
    const float4* pinst;
    uint32_t probe_count;
    uint32_t probe_instance_count;
};

// Device-side frame control of a batch: the work counter of the persistent
// launch, the iteration and the reset flag of the current frame.
struct BatchCtl {
    uint32_t next;
    uint32_t iteration;
    uint32_t reset;
    uint32_t pad;
};

// The probe's own surface point (estimate_surface_irradiance setup,
// surface_probe_path_tracer.slang:206-236).
struct ProbeSite {
    Shading sd;
    f3 normal;  // normalised face normal: the frame of the samples
    uint32_t inst, prim;
    float kr;
};

__device__ __forceinline__ bool probe_site(const SceneView& s, const float4* __restrict__ probes,
                                           const float4* __restrict__ pinst, uint32_t probe_instance_count,
                                           uint32_t p, ProbeSite* out) {
    const float4 nrm = __ldg(probes + 3u * p + 1u);
    const uint4 meta = __ldg(reinterpret_cast<const uint4*>(probes) + 3u * p + 2u);
    const uint32_t inst = meta.w >> 8;
    if (inst >= probe_instance_count || !valid_prim(s, inst, meta.x)) {
        atomicOr(s.status, kStatusBadRecord);
        return false;
    }
    const float4 params = __ldg(pinst + 3u * inst + 2u);
    const float bx = __uint_as_float(meta.y), by = __uint_as_float(meta.z);
    out->inst = inst;
    out->prim = meta.x;
    out->kr = maxf(params.x, 1e-6f);
    const f3 view = normalize3(mk3(nrm.x, nrm.y, nrm.z));
    out->sd = shading_data(s, inst, meta.x, bx, by, view);
    out->normal = normalize3(out->sd.face_normal);
    return true;
}

// One cosine sample of the probe: its irradiance term, self-hit suspects,
// radial texel and normalised first-hit distance (has_path false when the
// sample pdf is <= 1e-6 and the loop skips it).
struct ProbeSample {
    f3 si;
    uint32_t self_hits;
    uint32_t texel;
    float nd;
    bool has_path;
};

template <class Tr>
__device__ __forceinline__ ProbeSample probe_sample(const SceneView& s, const LightParams& L, const ProbeSite& site,
                                                    Rng& rng, uint32_t max_bounces, RayTally& tally) {
    ProbeSample r;
    r.si = mk3(0.0f, 0.0f, 0.0f);
    r.self_hits = 0u;
    r.texel = 0u;
    r.nd = 0.0f;
    r.has_path = false;
    const Shading& sd = site.sd;
    const float kr = site.kr;
    const float e0 = rng.next_1d(), e1 = rng.next_1d();
    float pdf;
    const f3 dir = cosine_sample_hemisphere(e0, e1, &pdf);
    if (pdf > 1e-6f) {
        f3 o = sd.origin_front;
        f3 d = Frame(site.normal).to_global(dir);
        f3 thp = mk3(1.0f, 1.0f, 1.0f), rad = mk3(0.0f, 0.0f, 0.0f);
        uint32_t src_inst = site.inst, src_prim = site.prim;
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
                rad = rad + thp * sky_radiance(L, d);
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
        r.self_hits = self_hits;
        r.texel = radial_texel(dir);
        r.nd = first_hit / maxf(kr, 1e-6f);
        r.si = r.si + ((rad * fabsf(dir.z)) / pdf);
        r.has_path = true;
    }
    return r;
}

// Per-probe sums of one iteration, folded in sample order.
struct ProbeAcc {
    f3 irr;
    uint32_t self_total;
    uint32_t local_counts[16];
};

__device__ __forceinline__ void probe_acc_init(ProbeAcc& a) {
    a.irr = mk3(0.0f, 0.0f, 0.0f);
    a.self_total = 0u;
#pragma unroll
    for (int t = 0; t < 16; ++t) a.local_counts[t] = 0u;
}

__device__ __forceinline__ void probe_fold(ProbeAcc& a, const ProbeOut& out, uint32_t p, const ProbeSample& smp,
                                           uint32_t prev_iter, uint32_t spp) {
    if (smp.has_path) {
        a.self_total += smp.self_hits;
        a.local_counts[smp.texel] += 1u;
        accumulate_radial_moment(out.radial, p, smp.texel, smp.nd, prev_iter, a.local_counts[smp.texel], spp);
    }
    a.irr = a.irr + smp.si;
}

// store_accumulated_irradiance and store_accumulated_self_hit_count
// (surface_probe_path_tracer.slang:47-79).
__device__ __forceinline__ void probe_store(const ProbeOut& out, uint32_t p, const ProbeAcc& a, uint32_t n,
                                            int reset) {
    const f3 irr = a.irr / (float)n;
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
    const uint32_t prev_self = reset ? 0u : out.self_hits[p];
    out.self_hits[p] = prev_self + a.self_total;
}

// The reference's baker: one RNG stream per probe, samples in sequence.
template <class Tr>
__device__ __forceinline__ bool probe_unit(const SceneView& s, const LightParams& L, const ProbeOut& out,
                                           const float4* __restrict__ probes, const float4* __restrict__ pinst,
                                           uint32_t probe_instance_count, uint32_t iteration, uint32_t spp,
                                           uint32_t max_bounces, int reset, uint32_t p, RayTally& tally) {
    ProbeSite site;
    if (!probe_site(s, probes, pinst, probe_instance_count, p, &site)) return false;
    const uint32_t n = max(spp, 1u);
    Rng rng(p, site.inst, iteration * n);
    const uint32_t prev_iter = reset ? 0u : out.counts[p];
    if (reset)
        for (int t = 0; t < 16; ++t) out.radial[16u * p + (uint32_t)t] = 0u;
    ProbeAcc acc;
    probe_acc_init(acc);
    for (uint32_t k = 0; k < n; ++k) {
        const ProbeSample smp = probe_sample<Tr>(s, L, site, rng, max_bounces, tally);
        probe_fold(acc, out, p, smp, prev_iter, spp);
    }
    probe_store(out, p, acc, n, reset);
    return true;
}

// ---------------------------------------------------------------------------
// PRT L2 field baker (surface_probe_prt_baker.slang:169-371): per probe, the
// transport of escaping light projected on the real SH L2 basis
// (surface_probe_sh.slang:5-21), and an RGB static source (emission and sun
// NEE along the paths), kept as running means; self-hit and radial moments as
// in the irradiance baker. One RNG stream per probe, samples in sequence.
// ---------------------------------------------------------------------------
struct PrtOut {
    float* values;         // f32[N][9][3]
    uint32_t* counts;
    uint32_t* self_hits;
    uint32_t* radial;
    float* static_source;  // f32[N][3]
};

__device__ __forceinline__ float sh_l2_basis(uint32_t c, f3 dir) {
    const f3 d = normalize3(dir);
    const float x = d.x, y = d.y, z = d.z;
    switch (c) {
        case 0: return 0.2820947918f;
        case 1: return 0.4886025119f * y;
        case 2: return 0.4886025119f * z;
        case 3: return 0.4886025119f * x;
        case 4: return 1.0925484306f * x * y;
        case 5: return 1.0925484306f * y * z;
        case 6: return 0.3153915653f * (3.0f * y * y - 1.0f);
        case 7: return 1.0925484306f * x * z;
        default: return 0.5462742153f * (x * x - z * z);
    }
}

template <class Tr>
__device__ __forceinline__ bool probe_prt_unit(const SceneView& s, const LightParams& L, const PrtOut& out,
                                               const float4* __restrict__ probes, const float4* __restrict__ pinst,
                                               uint32_t probe_instance_count, uint32_t iteration, uint32_t spp,
                                               uint32_t max_bounces, int reset, uint32_t p, RayTally& tally) {
    ProbeSite site;
    if (!probe_site(s, probes, pinst, probe_instance_count, p, &site)) return false;
    const uint32_t n = max(spp, 1u);
    Rng rng(p, site.inst, iteration * n);
    const Shading& sd = site.sd;
    const float kr = site.kr;
    const uint32_t prev_iter = reset ? 0u : out.counts[p];
    if (reset)
        for (int t = 0; t < 16; ++t) out.radial[16u * p + (uint32_t)t] = 0u;
    f3 transport[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) transport[c] = mk3(0.0f, 0.0f, 0.0f);
    f3 stat = mk3(0.0f, 0.0f, 0.0f);
    uint32_t self_total = 0u;
    uint32_t local_counts[16];
#pragma unroll
    for (int t = 0; t < 16; ++t) local_counts[t] = 0u;
    for (uint32_t k = 0; k < n; ++k) {
        const float e0 = rng.next_1d(), e1 = rng.next_1d();
        float pdf;
        const f3 dir = cosine_sample_hemisphere(e0, e1, &pdf);
        if (pdf <= 1e-6f) continue;
        f3 lt[9];
#pragma unroll
        for (int c = 0; c < 9; ++c) lt[c] = mk3(0.0f, 0.0f, 0.0f);
        f3 o = sd.origin_front;
        f3 d = Frame(site.normal).to_global(dir);
        f3 thp = mk3(1.0f, 1.0f, 1.0f), st = mk3(0.0f, 0.0f, 0.0f);
        uint32_t src_inst = site.inst, src_prim = site.prim;
        float src_off = len3(o - sd.position);
        uint32_t self_hits = 0u;
        const float radial_max = 2.0f * kr;
        float first_hit = 2.0f * kr;
        // trace_prt_transport (surface_probe_prt_baker.slang:164-230)
        for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
            tally.extend++;
            const HitInfo hit = Tr::closest(s, o, d, 0.0f, L.t_max);
            if (!hit.valid) {
                if (bounce == 0u) first_hit = radial_max;
#pragma unroll
                for (uint32_t c = 0; c < 9; ++c) lt[c] = lt[c] + thp * sh_l2_basis(c, d);
                break;
            }
            if (bounce == 0u) first_hit = minf(hit.t, radial_max);
            const uint2 ref = __ldg(s.tri_refs + hit.flat);
            const bool same_prim = ref.x == src_inst && ref.y == src_prim;
            const float thr = maxf(4.0f * src_off, 1e-6f);
            const bool adjacent = ref.x == src_inst && hit.t <= thr;
            if (same_prim || adjacent) self_hits += 1u;
            const Shading hs = shading_data(s, ref.x, ref.y, hit.b1, hit.b2, -d);
            st = st + thp * hs.emissive;
            const float u0 = rng.next_1d(), u1 = rng.next_1d();
            st = st + thp * sun_nee<Tr>(s, L, hs, u0, u1, tally);
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
        const float w = fabsf(dir.z) / pdf;
#pragma unroll
        for (int c = 0; c < 9; ++c) transport[c] = transport[c] + w * lt[c];
        stat = stat + w * st;
        const uint32_t texel = radial_texel(dir);
        local_counts[texel] += 1u;
        accumulate_radial_moment(out.radial, p, texel, first_hit / maxf(kr, 1e-6f), prev_iter, local_counts[texel],
                                 spp);
    }
    const float inv = 1.0f / (float)n;
    // store_accumulated_prt (surface_probe_prt_baker.slang:43-74)
    const uint32_t prev = reset ? 0u : out.counts[p];
    const float weight = 1.0f / (float)(prev + 1u);
#pragma unroll
    for (int c = 0; c < 9; ++c) {
        const f3 t = transport[c] * inv;
        float* v = out.values + 27u * p + 3u * (uint32_t)c;
        const f3 pv = prev == 0u ? mk3(0.0f, 0.0f, 0.0f) : mk3(v[0], v[1], v[2]);
        const f3 r = pv + weight * (t - pv);
        v[0] = r.x;
        v[1] = r.y;
        v[2] = r.z;
    }
    {
        const f3 t = stat * inv;
        float* v = out.static_source + 3u * p;
        const f3 pv = prev == 0u ? mk3(0.0f, 0.0f, 0.0f) : mk3(v[0], v[1], v[2]);
        const f3 r = pv + weight * (t - pv);
        v[0] = r.x;
        v[1] = r.y;
        v[2] = r.z;
    }
    out.counts[p] = min(prev + 1u, 65535u);
    const uint32_t prev_self = reset ? 0u : out.self_hits[p];
    out.self_hits[p] = prev_self + self_total;
    return true;
}

}  // namespace nbd
