// nan_batch.cu -- surface-probe baking of many scenes in one persistent
// launch (no counterpart in the reference, which bakes one scene per
// dispatch: surface_probe_path_tracer.py:49-83).
//
// The batch holds a device table of (scene view, lighting, probe set,
// outputs) and the exclusive prefix of the sets' probe counts. Warps pull
// 32 * grab (scene, probe) units per atomic from one counter, so scenes of
// very different size share the GPU without a launch per scene, and each
// unit runs the per-probe baker of nan_probe.cuh with the binary BVH at a
// fixed stack depth, or (NAN_BATCH_WAVEFRONT) every (scene, probe) unit
// becomes one path of a multi-scene wavefront (nan_wavefront.cu) with the
// same per-probe sample sequence. A frame is [reset counter, bake]; frames can be
// captured once into a CUDA graph whose last node advances the iteration
// on the device, and replayed. The autotuner times the launch shapes
// (stack depth, warps per SM, units per grab) on the batch itself.
#include <algorithm>
#include <cstring>
#include <vector>

#include "nan_internal.h"
#include "nan_probe.cuh"

namespace {

using namespace nbd;
using nan_host::cuda_fail;
using nan_host::set_error;


// kMinBlocks: the launch-bounds occupancy target that caps registers
// (0: the compiler's choice), one of the autotuned dimensions.
template <int kDepth, int kMinBlocks>
__global__ void __launch_bounds__(128, kMinBlocks) k_batch_probes(const BatchSet* __restrict__ sets,
                                                      const uint32_t* __restrict__ prefix, uint32_t set_count,
                                                      uint32_t total, BatchCtl* ctl, uint32_t spp,
                                                      uint32_t max_bounces, uint32_t grab,
                                                      unsigned long long* counters) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t iteration = ctl->iteration;
    const int reset = (int)ctl->reset;
    RayTally tally{0u, 0u};
    uint32_t units = 0u;
    for (;;) {
        uint32_t base = 0u;
        if (lane == 0u) base = atomicAdd(&ctl->next, 32u * grab);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        for (uint32_t j = 0; j < grab; ++j) {
            const uint32_t u = base + j * 32u + lane;
            if (u >= total) break;
            // set = last s with prefix[s] <= u (empty sets are skipped)
            uint32_t lo = 0u, hi = set_count - 1u;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1u) >> 1;
                if (__ldg(prefix + mid) <= u) lo = mid; else hi = mid - 1u;
            }
            const BatchSet& b = sets[lo];
            const LightParams L = make_light(b.light);
            if (probe_unit<BinaryTracer<kDepth>>(b.s, L, b.out, b.probes, b.pinst, b.probe_instance_count, iteration,
                                                 spp, max_bounces, reset, u - __ldg(prefix + lo), tally))
                units++;
        }
    }
    flush_tally(counters, tally, units, units * max(spp, 1u));
}

// Independent-sample mode: sample k of probe p draws from its own stream
// RNG(p, instance, iteration * n + k), so one warp traces 32 samples of one
// probe at once. Lane 0 then folds them in sample order, forming every sum
// exactly as the sequential loop does with those per-sample values.
template <int kDepth, int kMinBlocks>
__global__ void __launch_bounds__(128, kMinBlocks) k_batch_probes_ws(const BatchSet* __restrict__ sets,
                                                         const uint32_t* __restrict__ prefix, uint32_t set_count,
                                                         uint32_t total, BatchCtl* ctl, uint32_t spp,
                                                         uint32_t max_bounces, uint32_t grab,
                                                         unsigned long long* counters) {
    (void)grab;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t iteration = ctl->iteration;
    const int reset = (int)ctl->reset;
    const uint32_t n = max(spp, 1u);
    RayTally tally{0u, 0u};
    uint32_t units = 0u;
    for (;;) {
        uint32_t u = 0u;
        if (lane == 0u) u = atomicAdd(&ctl->next, 1u);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= total) break;
        uint32_t lo = 0u, hi = set_count - 1u;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (__ldg(prefix + mid) <= u) lo = mid; else hi = mid - 1u;
        }
        const BatchSet& b = sets[lo];
        const uint32_t p = u - __ldg(prefix + lo);
        const LightParams L = make_light(b.light);
        ProbeSite site;
        if (!probe_site(b.s, b.probes, b.pinst, b.probe_instance_count, p, &site)) continue;
        const uint32_t prev_iter = reset ? 0u : b.out.counts[p];
        if (reset && lane < 16u) b.out.radial[16u * p + lane] = 0u;
        __syncwarp();
        ProbeAcc acc;
        probe_acc_init(acc);
        for (uint32_t k0 = 0; k0 < n; k0 += 32u) {
            const uint32_t k = k0 + lane;
            ProbeSample smp;
            smp.si = mk3(0.0f, 0.0f, 0.0f);
            smp.self_hits = 0u;
            smp.texel = 0u;
            smp.nd = 0.0f;
            smp.has_path = false;
            if (k < n) {
                Rng rng(p, site.inst, iteration * n + k);
                smp = probe_sample<BinaryTracer<kDepth>>(b.s, L, site, rng, max_bounces, tally);
            }
            const uint32_t cnt = min(32u, n - k0);
            for (uint32_t j = 0; j < cnt; ++j) {
                ProbeSample q;
                q.si = mk3(__shfl_sync(0xffffffffu, smp.si.x, j), __shfl_sync(0xffffffffu, smp.si.y, j),
                           __shfl_sync(0xffffffffu, smp.si.z, j));
                q.self_hits = __shfl_sync(0xffffffffu, smp.self_hits, j);
                q.texel = __shfl_sync(0xffffffffu, smp.texel, j);
                q.nd = __shfl_sync(0xffffffffu, smp.nd, j);
                q.has_path = __shfl_sync(0xffffffffu, (int)smp.has_path, j) != 0;
                if (lane == 0u) probe_fold(acc, b.out, p, q, prev_iter, spp);
            }
        }
        if (lane == 0u) {
            probe_store(b.out, p, acc, n, reset);
            units++;
        }
        __syncwarp();
    }
    flush_tally(counters, tally, units, units * n);
}

__global__ void k_batch_begin(BatchCtl* ctl, uint32_t iteration, uint32_t reset) {
    ctl->next = 0u;
    ctl->iteration = iteration;
    ctl->reset = reset;
}

__global__ void k_batch_prepare(BatchCtl* ctl) { ctl->next = 0u; }

__global__ void k_batch_advance(BatchCtl* ctl) {
    ctl->iteration += 1u;
    ctl->reset = 0u;
}

constexpr uint32_t kDepths[] = {48u, 96u};
constexpr uint32_t kRegCaps[] = {0u, 4u, 6u};

template <int kDepth, int kMinBlocks>
const void* pick(uint32_t mode) {
    return mode == NAN_BATCH_INDEPENDENT_SAMPLES ? reinterpret_cast<const void*>(k_batch_probes_ws<kDepth, kMinBlocks>)
                                                 : reinterpret_cast<const void*>(k_batch_probes<kDepth, kMinBlocks>);
}

template <int kDepth>
const void* pick_caps(uint32_t mode, uint32_t cap) {
    switch (cap) {
        case 4: return pick<kDepth, 4>(mode);
        case 6: return pick<kDepth, 6>(mode);
        default: return pick<kDepth, 0>(mode);
    }
}

const void* kernel_for(uint32_t depth, uint32_t mode, uint32_t cap) {
    return depth <= 48u ? pick_caps<48>(mode, cap) : pick_caps<96>(mode, cap);
}

}  // namespace

namespace nan_host {

// The scene as the batched kernel traverses it: binary nodes.
SceneView scene_view_for_batch(const NanContext* ctx) {
    SceneView v;
    memset(&v, 0, sizeof(v));
    v.nodes = ctx->nodes;
    v.tris = ctx->tris;
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

struct BatchImpl {
    BatchSet* sets = nullptr;
    uint32_t* prefix = nullptr;
    BatchCtl* ctl = nullptr;
    uint32_t* set_of = nullptr;      // wavefront modes: probe set of each path
    uint64_t set_of_paths = 0;       // entries of set_of
    void* samples = nullptr;         // independent wavefront: one sample record per path
    uint64_t sample_paths = 0;       // paths the sample records and the scratch hold
    float t_max = 0.0f;              // largest ray t_max of the sets
    uint32_t set_count = 0;
    uint32_t total = 0;
    uint32_t min_depth = 32;  // smallest stack depth that covers every scene's BVH
    cudaStream_t capture_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

int launch_frame_kernel(NanBatch* b, uint32_t spp, uint32_t max_bounces, cudaStream_t st) {
    BatchImpl* m = b->impl;
    if (b->mode == NAN_BATCH_WAVEFRONT || b->mode == NAN_BATCH_WAVEFRONT_INDEPENDENT) {
        NanTuning& tt = b->ctx->tuning;
        tt.trace_blocks_per_sm = b->tuning.blocks_per_sm;
        if (b->mode == NAN_BATCH_WAVEFRONT_INDEPENDENT)
            return nan_host::launch_batch_wavefront_independent(b->ctx, m->sets, m->prefix, m->ctl, m->set_count,
                                                                m->total, m->set_of, m->samples, m->sample_paths,
                                                                spp, max_bounces, m->t_max, st);
        return nan_host::launch_batch_wavefront(b->ctx, m->sets, m->prefix, m->ctl, m->set_count, m->total, m->set_of,
                                                spp, max_bounces, m->t_max, st);
    }
    const NanBatchTuning& t = b->tuning;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->ctx->device);
    const uint32_t grid = (uint32_t)sms * std::max(t.blocks_per_sm, 1u);
    uint32_t grab = std::max(t.units_per_grab, 1u);
    uint32_t sc = m->set_count, total = m->total;
    BatchCtl* ctl = m->ctl;
    const BatchSet* sets = m->sets;
    const uint32_t* prefix = m->prefix;
    unsigned long long* counters = b->ctx->d_counters;
    void* args[] = {(void*)&sets, (void*)&prefix, &sc, &total, &ctl, &spp, &max_bounces, &grab, &counters};
    cudaError_t err = cudaLaunchKernel(kernel_for(t.stack_depth, b->mode, t.min_blocks_per_sm), dim3(grid), dim3(128),
                                       args, 0, st);
    b->ctx->launches++;
    return cuda_fail(err, "batched probe launch");
}

void drop_graph(BatchImpl* m) {
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->exec = nullptr;
    m->graph = nullptr;
}

}  // namespace

int batch_create(NanContext* ctx, const NanProbeSet* in, uint32_t count, NanBatch** out) {
    std::vector<BatchSet> sets(count);
    std::vector<uint32_t> prefix(count + 1u, 0u);
    uint32_t max_depth = 0;
    float t_max = 0.0f;
    for (uint32_t i = 0; i < count; ++i) {
        const NanProbeSet& p = in[i];
        if (const int lrc = check_lighting(&p.lighting)) return lrc;
        BatchSet& b = sets[i];
        b.s = scene_view_for_batch(p.scene);
        memcpy(&b.light, &p.lighting, sizeof(b.light));
        b.out = ProbeOut{reinterpret_cast<float4*>(p.compensation), p.values, p.sample_counts, p.self_hits, p.radial};
        b.probes = reinterpret_cast<const float4*>(p.probes);
        b.pinst = reinterpret_cast<const float4*>(p.probe_instances);
        b.probe_count = p.probe_count;
        b.probe_instance_count = p.probe_instance_count;
        const uint64_t next = (uint64_t)prefix[i] + p.probe_count;
        if (next > 0xffffffffull) {
            set_error("more than 2^32 probes in one batch");
            return NAN_ERR_INVALID_ARGUMENT;
        }
        prefix[i + 1] = (uint32_t)next;
        max_depth = std::max(max_depth, p.scene->max_depth);
        t_max = std::max(t_max, p.lighting.ray_t_max);
    }
    NanBatch* b = new NanBatch();
    b->ctx = ctx;
    b->impl = new BatchImpl();
    BatchImpl* m = b->impl;
    m->set_count = count;
    m->total = prefix[count];
    m->t_max = t_max;
    m->min_depth = max_depth + 2u <= 48u ? 48u : 96u;
    if (max_depth + 2u > 96u) {
        delete m;
        delete b;
        set_error("a scene's BVH is deeper than the batched traversal stack (94 levels)");
        return NAN_ERR_LIMIT;
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_probes<96, 0>, 128, 0);
    b->tuning.stack_depth = 96u;
    b->tuning.min_blocks_per_sm = 0u;
    b->tuning.blocks_per_sm = (uint32_t)std::max(occ, 1);
    b->tuning.units_per_grab = 1u;
    cudaError_t err = cudaMalloc(&m->sets, sizeof(BatchSet) * std::max(count, 1u));
    if (err == cudaSuccess) err = cudaMalloc(&m->prefix, sizeof(uint32_t) * (count + 1u));
    if (err == cudaSuccess) err = cudaMalloc(&m->ctl, sizeof(BatchCtl));
    if (err == cudaSuccess && count)
        err = cudaMemcpy(m->sets, sets.data(), sizeof(BatchSet) * count, cudaMemcpyHostToDevice);
    if (err == cudaSuccess)
        err = cudaMemcpy(m->prefix, prefix.data(), sizeof(uint32_t) * (count + 1u), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemset(m->ctl, 0, sizeof(BatchCtl));
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&m->capture_stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        batch_destroy(b);
        return cuda_fail(err, "batch allocation");
    }
    *out = b;
    return NAN_OK;
}

void batch_destroy(NanBatch* b) {
    if (!b) return;
    if (BatchImpl* m = b->impl) {
        drop_graph(m);
        if (m->capture_stream) cudaStreamDestroy(m->capture_stream);
        cudaFree(m->sets);
        cudaFree(m->prefix);
        cudaFree(m->ctl);
        cudaFree(m->set_of);
        cudaFree(m->samples);
        delete m;
    }
    delete b;
}

uint32_t batch_min_depth(const NanBatch* b) { return b->impl->min_depth; }

int batch_set_mode(NanBatch* b, uint32_t mode) {
    if (mode != NAN_BATCH_SEQUENTIAL_SAMPLES && mode != NAN_BATCH_INDEPENDENT_SAMPLES &&
        mode != NAN_BATCH_WAVEFRONT && mode != NAN_BATCH_WAVEFRONT_INDEPENDENT) {
        set_error("mode must be NAN_BATCH_SEQUENTIAL_SAMPLES, NAN_BATCH_INDEPENDENT_SAMPLES, NAN_BATCH_WAVEFRONT or "
                  "NAN_BATCH_WAVEFRONT_INDEPENDENT");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    if ((mode == NAN_BATCH_WAVEFRONT || mode == NAN_BATCH_WAVEFRONT_INDEPENDENT) && mode != b->mode) {
        BatchImpl* m = b->impl;
        NanContext* ctx = b->ctx;
        // WAVEFRONT: one path per probe; INDEPENDENT: one path per (probe,
        // sample), in chunks of at most 2^24 paths (64 samples of every probe
        // when the batch is smaller)
        const bool ind = mode == NAN_BATCH_WAVEFRONT_INDEPENDENT;
        const uint64_t paths = ind ? std::min<uint64_t>(std::max<uint64_t>((uint64_t)m->total * 64ull, 1ull << 15),
                                                        1ull << 24)
                                   : std::max<uint64_t>(m->total, 1u);
        const uint64_t need = paths * nan_host::wavefront_bytes_per_path() + (1ull << 22);
        cudaError_t err = cudaDeviceSynchronize();
        if (err == cudaSuccess && m->set_of_paths < paths) {
            cudaFree(m->set_of);
            m->set_of = nullptr;
            m->set_of_paths = 0;
            err = cudaMalloc(&m->set_of, sizeof(uint32_t) * paths);
            if (err == cudaSuccess) m->set_of_paths = paths;
        }
        if (err == cudaSuccess && ind && m->sample_paths < paths) {
            cudaFree(m->samples);
            m->samples = nullptr;
            m->sample_paths = 0;
            err = cudaMalloc(&m->samples, nan_host::probe_sample_bytes() * paths);
            if (err == cudaSuccess) m->sample_paths = paths;
        }
        if (err == cudaSuccess && ctx->scratch_bytes < need) err = nan_host::replace_context_scratch(ctx, need);
        if (err != cudaSuccess) return cuda_fail(err, "batch wavefront scratch");
        b->mode = mode;
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, nan_host::wavefront_extend_kernel(), 128, 0);
        b->tuning.blocks_per_sm = (uint32_t)std::max(occ, 1);
        b->tuning.units_per_grab = 1u;
        drop_graph(m);
        return NAN_OK;
    }
    if (mode != b->mode) {
        b->mode = mode;
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &occ, kernel_for(b->tuning.stack_depth, mode, b->tuning.min_blocks_per_sm), 128, 0);
        b->tuning.blocks_per_sm = (uint32_t)std::max(occ, 1);
        b->tuning.units_per_grab = 1u;
        drop_graph(b->impl);
    }
    return NAN_OK;
}
uint32_t batch_total(const NanBatch* b) { return b->impl->total; }

int batch_set_tuning(NanBatch* b, const NanBatchTuning* t) {
    if (t->stack_depth != 48 && t->stack_depth != 96) {
        set_error("stack_depth must be 48 or 96");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    if (t->min_blocks_per_sm != 0 && t->min_blocks_per_sm != 4 && t->min_blocks_per_sm != 6) {
        set_error("min_blocks_per_sm must be 0, 4 or 6");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    if (t->stack_depth < b->impl->min_depth) {
        set_error("stack_depth is below the depth a scene's BVH needs");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    if (t->blocks_per_sm == 0 || t->blocks_per_sm > 32 || t->units_per_grab == 0 || t->units_per_grab > 64) {
        set_error("blocks_per_sm must be in [1, 32] and units_per_grab in [1, 64]");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    b->tuning = *t;
    drop_graph(b->impl);  // a captured frame keeps the launch shape it was captured with
    return NAN_OK;
}

int batch_frame(NanBatch* b, uint32_t iteration, uint32_t spp, uint32_t max_bounces, int reset, cudaStream_t st) {
    BatchImpl* m = b->impl;
    if (m->total == 0) return NAN_OK;
    k_batch_begin<<<1, 1, 0, st>>>(m->ctl, iteration, reset ? 1u : 0u);
    b->ctx->launches++;
    return launch_frame_kernel(b, spp, max_bounces, st);
}

int batch_capture(NanBatch* b, uint32_t first_iteration, int reset_first, uint32_t spp, uint32_t max_bounces,
                  cudaStream_t st) {
    BatchImpl* m = b->impl;
    drop_graph(m);
    k_batch_begin<<<1, 1, 0, st>>>(m->ctl, first_iteration, reset_first ? 1u : 0u);
    b->ctx->launches++;
    cudaError_t err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) return cuda_fail(err, "batch capture (set frame)");
    cudaStream_t cs = m->capture_stream;
    err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return cuda_fail(err, "batch capture begin");
    k_batch_prepare<<<1, 1, 0, cs>>>(m->ctl);
    int rc = m->total ? launch_frame_kernel(b, spp, max_bounces, cs) : NAN_OK;
    k_batch_advance<<<1, 1, 0, cs>>>(m->ctl);
    cudaGraph_t g = nullptr;
    err = cudaStreamEndCapture(cs, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (err != cudaSuccess) return cuda_fail(err, "batch capture end");
    m->graph = g;
    err = cudaGraphInstantiate(&m->exec, g, 0);
    if (err != cudaSuccess) {
        drop_graph(m);
        return cuda_fail(err, "batch graph instantiate");
    }
    return NAN_OK;
}

int batch_replay(NanBatch* b, uint32_t frames, cudaStream_t st) {
    BatchImpl* m = b->impl;
    if (!m->exec) {
        set_error("no captured frame (nan_batch_capture)");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    for (uint32_t f = 0; f < frames; ++f) {
        cudaError_t err = cudaGraphLaunch(m->exec, st);
        if (err != cudaSuccess) return cuda_fail(err, "batch graph launch");
        b->ctx->launches += 3;
    }
    return NAN_OK;
}

// Times every admissible launch shape on one frame each (reset, iteration 0)
// and keeps the fastest. The outputs hold that last frame afterwards.
int batch_autotune(NanBatch* b, uint32_t spp, uint32_t max_bounces, cudaStream_t st, NanBatchTuning* chosen) {
    BatchImpl* m = b->impl;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    if (err != cudaSuccess) return cuda_fail(err, "autotune events");
    NanBatchTuning best = b->tuning;
    float best_ms = -1.0f;
    // one untimed frame first (first touch of the scenes' data)
    int rc = batch_frame(b, 0u, spp, max_bounces, 1, st);
    if (b->mode == NAN_BATCH_WAVEFRONT || b->mode == NAN_BATCH_WAVEFRONT_INDEPENDENT) {
        // the traversal grid of the wavefront: persistent blocks per SM
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, nan_host::wavefront_extend_kernel(), 128, 0);
        occ = std::max(occ, 1);
        for (uint32_t bps : {(uint32_t)std::max(occ / 2, 1), (uint32_t)std::max(3 * occ / 4, 1), (uint32_t)occ}) {
            if (rc) break;
            NanBatchTuning t = b->tuning;
            t.blocks_per_sm = bps;
            b->tuning = t;
            cudaEventRecord(e0, st);
            rc = batch_frame(b, 0u, spp, max_bounces, 1, st);
            cudaEventRecord(e1, st);
            if (rc) break;
            float ms = 0.0f;
            err = cudaEventSynchronize(e1);
            if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
            if (err != cudaSuccess) {
                rc = cuda_fail(err, "autotune timing");
                break;
            }
            if (best_ms < 0.0f || ms < best_ms) {
                best_ms = ms;
                best = t;
            }
        }
    }
    for (uint32_t depth : kDepths) {
        if (b->mode == NAN_BATCH_WAVEFRONT || b->mode == NAN_BATCH_WAVEFRONT_INDEPENDENT) break;
        if (rc) break;
        if (depth < m->min_depth) continue;
        for (uint32_t cap : kRegCaps) {
            if (rc) break;
            int occ = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel_for(depth, b->mode, cap), 128, 0);
            occ = std::max(occ, 1);
            const uint32_t blocks[] = {(uint32_t)std::max(occ / 2, 1), (uint32_t)occ};
            for (uint32_t bps : blocks) {
                for (uint32_t grab : {1u, 4u}) {
                    if (b->mode == NAN_BATCH_INDEPENDENT_SAMPLES && grab != 1u) continue;  // one probe per warp
                    NanBatchTuning t = b->tuning;
                    t.stack_depth = depth;
                    t.min_blocks_per_sm = cap;
                    t.blocks_per_sm = bps;
                    t.units_per_grab = grab;
                    b->tuning = t;
                    cudaEventRecord(e0, st);
                    rc = batch_frame(b, 0u, spp, max_bounces, 1, st);
                    cudaEventRecord(e1, st);
                    if (rc) break;
                    err = cudaEventSynchronize(e1);
                    float ms = 0.0f;
                    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
                    if (err != cudaSuccess) {
                        rc = cuda_fail(err, "autotune timing");
                        break;
                    }
                    if (best_ms < 0.0f || ms < best_ms) {
                        best_ms = ms;
                        best = t;
                    }
                }
                if (rc) break;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tuning = best;
    drop_graph(m);
    if (chosen) *chosen = best;
    b->tuned_ms = best_ms;
    return rc;
}

}  // namespace nan_host
