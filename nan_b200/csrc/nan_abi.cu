// nan_abi.cu -- the extern "C" entry points declared in include/nan_b200.h.
#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "nan_internal.h"

namespace nan_host {

thread_local std::string g_last_error;

namespace {
// One memory pool per device for the builders' stream-ordered scratch. The
// CUDA default pool returns unused memory to the driver at every
// synchronisation, so a build that synchronises between passes re-maps its
// scratch each time; this pool keeps it until a context is destroyed.
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[128] = {};
}  // namespace

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        if (!g_pools[dev]) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            err = cudaMemPoolCreate(&g_pools[dev], &props);
            if (err != cudaSuccess) {
                g_pools[dev] = nullptr;
                return err;
            }
            uint64_t keep = ~0ull;
            err = cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
            if (err != cudaSuccess) return err;
        }
        pool = g_pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

cudaError_t replace_context_scratch(NanContext* ctx, size_t bytes) {
    if (ctx->scratch) cudaFreeAsync(ctx->scratch, 0);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    if (bytes == 0) return cudaStreamSynchronize(0);
    cudaError_t err = scratch_alloc(&ctx->scratch, bytes, 0);
    if (err == cudaSuccess) err = cudaStreamSynchronize(0);  // usable from every stream once this returns
    if (err != cudaSuccess) {
        if (ctx->scratch) cudaFreeAsync(ctx->scratch, 0);
        ctx->scratch = nullptr;
        return err;
    }
    ctx->scratch_bytes = bytes;
    return cudaSuccess;
}

void trim_scratch(int device) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (device >= 0 && device < 128 && g_pools[device]) cudaMemPoolTrimTo(g_pools[device], 0);
}

void set_error(const std::string& msg) { g_last_error = msg; }

int cuda_fail(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return NAN_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(err));
    return err == cudaErrorMemoryAllocation ? NAN_ERR_OUT_OF_MEMORY : NAN_ERR_CUDA;
}

}  // namespace nan_host

namespace {

using nan_host::cuda_fail;
using nan_host::set_error;

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

int invalid(const char* msg) {
    set_error(msg);
    return NAN_ERR_INVALID_ARGUMENT;
}

int enter(NanContext* ctx) {
    if (!ctx) return invalid("null context");
    const cudaError_t err = cudaSetDevice(ctx->device);
    return cuda_fail(err, "cudaSetDevice");
}

int need_scene(NanContext* ctx) {
    if (!ctx->has_scene) {
        set_error("no scene has been built on this context");
        return NAN_ERR_NO_SCENE;
    }
    return NAN_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0u; }

}  // namespace


namespace {
int cache_enter(NanCache* k) {
    if (!k) return invalid("null cache");
    return enter(k->ctx);
}
int check_config(const NanCacheConfig* c) {
    if (!c) return invalid("null cache config");
    if (c->log2_table < 10 || c->log2_table > 24) return invalid("log2_table must be in [10, 24]");
    if (c->base_resolution < 2 || c->max_resolution < c->base_resolution || c->max_resolution > (1u << 20))
        return invalid("resolutions must satisfy 2 <= base <= max <= 2^20");
    for (int i = 0; i < 3; ++i)
        if (!(c->bounds_max[i] > c->bounds_min[i])) return invalid("cache bounds are empty");
    if (!(c->learning_rate > 0.0f) || !(c->beta1 >= 0.0f && c->beta1 < 1.0f) || !(c->beta2 >= 0.0f && c->beta2 < 1.0f) ||
        !(c->epsilon >= 0.0f) || !(c->loss_epsilon > 0.0f))
        return invalid("bad optimizer or loss parameter");
    if (c->table_update > 1) return invalid("table_update must be 0 (dense Adam) or 1 (lazy Adam)");
    return NAN_OK;
}
}  // namespace

extern "C" {

NAN_B200_API const char* nan_last_error(void) { return nan_host::g_last_error.c_str(); }

NAN_B200_API int nan_version(void) { return 1; }

NAN_B200_API int nan_ctx_create(int device, NanContext** out_ctx) {
    if (!out_ctx) return invalid("null output pointer");
    *out_ctx = nullptr;
    int count = 0;
    cudaError_t err = cudaGetDeviceCount(&count);
    if (err != cudaSuccess) return cuda_fail(err, "cudaGetDeviceCount");
    if (device < 0 || device >= count) return invalid("device ordinal out of range");
    err = cudaSetDevice(device);
    if (err != cudaSuccess) return cuda_fail(err, "cudaSetDevice");
    NanContext* ctx = new NanContext();
    ctx->device = device;
    if (cudaMalloc(&ctx->d_status, sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&ctx->d_counters, sizeof(NanCounters)) != cudaSuccess) {
        cudaFree(ctx->d_status);
        cudaFree(ctx->d_counters);
        delete ctx;
        set_error("out of device memory for the context");
        return NAN_ERR_OUT_OF_MEMORY;
    }
    cudaMemset(ctx->d_status, 0, sizeof(uint32_t));
    cudaMemset(ctx->d_counters, 0, sizeof(NanCounters));
    err = cudaDeviceSynchronize();
    if (err != cudaSuccess) return cuda_fail(err, "context init");
    *out_ctx = ctx;
    return NAN_OK;
}

NAN_B200_API int nan_ctx_destroy(NanContext* ctx) {
    if (!ctx) return NAN_OK;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    nan_host::free_scene(ctx);
    nan_host::release_timing(ctx);
    nan_host::replace_context_scratch(ctx, 0);
    cudaFree(ctx->d_status);
    cudaFree(ctx->d_counters);
    nan_host::trim_scratch(ctx->device);
    delete ctx;
    return NAN_OK;
}

NAN_B200_API int nan_ctx_check(NanContext* ctx, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    uint32_t status = 0;
    cudaError_t err = cudaMemcpyAsync(&status, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                      as_stream(stream));
    if (err == cudaSuccess) err = cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), as_stream(stream));
    if (err == cudaSuccess) err = cudaStreamSynchronize(as_stream(stream));
    if (err != cudaSuccess) return cuda_fail(err, "status read");
    if (status & 1u) {
        set_error("a traversal stack overflowed (device status 1)");
        return NAN_ERR_LIMIT;
    }
    if (status & 2u) {
        set_error("a slot index fell outside the payload buffer (device status 2)");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    if (status & 4u) {
        set_error("a texel or probe record names a triangle outside the scene (device status 4)");
        return NAN_ERR_INVALID_ARGUMENT;
    }
    if (status & 8u) {
        set_error("a tensor-core completion wait hit its iteration limit (device status 8)");
        return NAN_ERR_LIMIT;
    }
    return NAN_OK;
}

NAN_B200_API int nan_ctx_read_counters(NanContext* ctx, NanCounters* out, int reset, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out) return invalid("null counters pointer");
    cudaError_t err = cudaMemcpyAsync(out, ctx->d_counters, sizeof(NanCounters), cudaMemcpyDeviceToHost,
                                      as_stream(stream));
    if (err == cudaSuccess && reset)
        err = cudaMemsetAsync(ctx->d_counters, 0, sizeof(NanCounters), as_stream(stream));
    if (err == cudaSuccess) err = cudaStreamSynchronize(as_stream(stream));
    return cuda_fail(err, "counter read");
}

NAN_B200_API uint64_t nan_ctx_launch_count(NanContext* ctx) { return ctx ? ctx->launches : 0; }

NAN_B200_API int nan_ctx_read_kernel_times(NanContext* ctx, NanKernelTimes* out, int reset) {
    int rc = enter(ctx);
    if (rc) return rc;
    return nan_host::read_kernel_times(ctx, out, reset);
}

NAN_B200_API uint64_t nan_wavefront_bytes_per_path(void) { return nan_host::wavefront_bytes_per_path(); }

NAN_B200_API int nan_ctx_reserve(NanContext* ctx, uint64_t scratch_bytes) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (scratch_bytes <= ctx->scratch_bytes) return NAN_OK;
    cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) return cuda_fail(err, "reserve (synchronize)");
    err = nan_host::replace_context_scratch(ctx, scratch_bytes);
    if (err != cudaSuccess) return cuda_fail(err, "reserve wavefront scratch");
    return NAN_OK;
}

NAN_B200_API int nan_ctx_set_area_lights(NanContext* ctx, const float* lights, uint32_t count, float power) {
    if (!ctx) return invalid("null context");
    if (count && (!lights || !aligned16(lights))) return invalid("area lights must be a 16-byte aligned table");
    if (count && !(power > 0.0f)) return invalid("area light power must be positive");
    ctx->lights = count ? lights : nullptr;
    ctx->light_count = count;
    ctx->light_power = count ? power : 0.0f;
    return NAN_OK;
}

NAN_B200_API int nan_ctx_configure(NanContext* ctx, const NanTuning* tuning) {
    if (!ctx || !tuning) return invalid("null argument");
    if (tuning->integrator > 1) return invalid("integrator must be 0 (wavefront) or 1 (one thread per unit)");
    if (tuning->trace_blocks_per_sm > 64) return invalid("trace_blocks_per_sm above 64");
    if (tuning->bvh_builder > 2) return invalid("bvh_builder must be 0 (binned SAH), 1 (LBVH) or 2 (PLOC)");
    if (tuning->bvh_width != 0 && tuning->bvh_width != 2 && tuning->bvh_width != 8)
        return invalid("bvh_width must be 0 or 2 (binary) or 8 (compressed wide)");
    if (tuning->kernel_timing > 1) return invalid("kernel_timing must be 0 or 1");
    if (tuning->ray_order > 1) return invalid("ray_order must be 0 (path order) or 1 (by direction octant)");
    if (tuning->traversal > 6) return invalid("traversal must be 0..6");
    ctx->tuning = *tuning;
    return NAN_OK;
}

NAN_B200_API int nan_scene_build(NanContext* ctx, const NanSceneDesc* desc, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!desc) return invalid("null scene description");
    if (desc->instance_count > 0 &&
        (!desc->vertices || !desc->indices || !desc->mesh_descs || !desc->instance_descs || !desc->transforms ||
         !desc->inverse_transposes || !desc->materials))
        return invalid("null scene buffer");
    if (desc->mesh_descs && !aligned16(desc->mesh_descs)) return invalid("mesh_descs must be 16-byte aligned");
    if (desc->instance_descs && !aligned16(desc->instance_descs))
        return invalid("instance_descs must be 16-byte aligned");
    return nan_host::build_scene(ctx, desc, as_stream(stream));
}

NAN_B200_API int nan_scene_info(NanContext* ctx, NanSceneInfo* out) {
    if (!ctx || !out) return invalid("null argument");
    int rc = need_scene(ctx);
    if (rc) return rc;
    out->triangle_count = ctx->tri_count;
    out->node_count = ctx->node_count;
    out->leaf_count = ctx->leaf_count;
    out->max_depth = ctx->max_depth;
    out->device_bytes = ctx->device_bytes;
    out->build_ms = ctx->build_ms;
    out->sah_cost = ctx->sah_cost;
    return NAN_OK;
}

NAN_B200_API int nan_scene_world_triangles(NanContext* ctx, float* out, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if ((rc = need_scene(ctx))) return rc;
    if (!out) return invalid("null output");
    return nan_host::world_triangles(ctx, out, as_stream(stream));
}

NAN_B200_API int nan_intersect(NanContext* ctx, const float* rays, uint32_t count, uint32_t* hit_ids, float* hit_tb,
                               void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if ((rc = need_scene(ctx))) return rc;
    if (count && (!rays || !hit_ids || !hit_tb)) return invalid("null ray buffer");
    if (count && (!aligned16(rays) || !aligned16(hit_ids))) return invalid("rays and hit_ids must be 16-byte aligned");
    return nan_host::launch_intersect(ctx, rays, count, hit_ids, hit_tb, as_stream(stream));
}

NAN_B200_API int nan_occluded(NanContext* ctx, const float* rays, uint32_t count, float* visibility, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if ((rc = need_scene(ctx))) return rc;
    if (count && (!rays || !visibility)) return invalid("null ray buffer");
    if (count && !aligned16(rays)) return invalid("rays must be 16-byte aligned");
    return nan_host::launch_occluded(ctx, rays, count, visibility, as_stream(stream));
}

NAN_B200_API int nan_visibility_ray_table(uint32_t ray_count, float* host_table) {
    if (ray_count == 0 || ray_count > NAN_VISIBILITY_MAX_RAYS)
        return invalid("ray_count must be 1..1024 (NAN_VISIBILITY_MAX_RAYS)");
    if (!host_table) return invalid("null table");
    return nan_host::visibility_ray_table(ray_count, host_table);
}

NAN_B200_API int nan_visibility_sh16(NanContext* ctx, const float* sample_positions, const float* sample_normals,
                                     uint32_t sample_count, const float* ray_table, uint32_t ray_count,
                                     float max_distance, float self_bias, float* out_sh16,
                                     uint32_t* out_visible_counts, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if ((rc = need_scene(ctx))) return rc;
    if (ray_count == 0 || ray_count > NAN_VISIBILITY_MAX_RAYS)
        return invalid("ray_count must be 1..1024 (NAN_VISIBILITY_MAX_RAYS)");
    if (!ray_table) return invalid("null ray table");
    if (sample_count && (!sample_positions || !sample_normals || !out_sh16))
        return invalid("null sample or output buffer");
    if (!std::isfinite(self_bias)) return invalid("self_bias must be finite");
    if (!std::isfinite(max_distance) || max_distance <= 0.0f) max_distance = 1.0e30f;
    self_bias = std::max(0.0f, self_bias);
    return nan_host::launch_visibility_sh16(ctx, sample_positions, sample_normals, sample_count, ray_table, ray_count,
                                            max_distance, self_bias, out_sh16, out_visible_counts,
                                            as_stream(stream));
}

NAN_B200_API int nan_trace_screen(NanContext* ctx, float* out_rgba, uint32_t width, uint32_t height, uint32_t frame,
                                  uint32_t max_vertices, const NanCamera* camera, const NanLighting* lighting,
                                  void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if ((rc = need_scene(ctx))) return rc;
    if (!camera || !lighting) return invalid("null camera or lighting");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if ((width || height) && (!out_rgba || !aligned16(out_rgba))) return invalid("output must be 16-byte aligned");
    if (max_vertices > 64) return invalid("max_vertices above 64");
    if (ctx->tuning.integrator == 0)
        return nan_host::launch_trace_screen_wavefront(ctx, out_rgba, width, height, frame, max_vertices, camera,
                                                       lighting, as_stream(stream));
    return nan_host::launch_trace_screen(ctx, out_rgba, width, height, frame, max_vertices, camera, lighting,
                                         as_stream(stream));
}

NAN_B200_API int nan_accumulate(NanContext* ctx, const float* input, float* output, float* history, uint32_t width,
                                uint32_t height, int reset, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if ((width && height) && (!input || !output || !history)) return invalid("null image buffer");
    if ((width && height) && (!aligned16(input) || !aligned16(output) || !aligned16(history)))
        return invalid("image buffers must be 16-byte aligned");
    return nan_host::launch_accumulate(ctx, input, output, history, width, height, reset, as_stream(stream));
}

NAN_B200_API int nan_trace_texels(NanContext* ctx, const NanMeshColorsDesc* layout, uint8_t* slots,
                                  uint32_t iteration, uint32_t samples_per_texel, uint32_t max_bounces, int reset,
                                  const NanLighting* lighting, uint32_t texel_begin, uint32_t texel_end,
                                  void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if ((rc = need_scene(ctx))) return rc;
    if (!layout || !lighting) return invalid("null layout or lighting");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if (layout->instance_count == 0) return invalid("layout has no instances");
    if (!layout->face_infos || !layout->instance_infos || !layout->side_infos || !layout->surface_prefix || !slots)
        return invalid("null layout buffer");
    if (!aligned16(slots) || !aligned16(layout->instance_infos) ||
        (layout->compensation && !aligned16(layout->compensation)))
        return invalid("slots, instance_infos and compensation must be 16-byte aligned");
    if (texel_end > layout->total_surface_texels) return invalid("texel range beyond the layout");
    if (max_bounces > 64) return invalid("max_bounces above 64");
    if (ctx->tuning.integrator == 0)
        return nan_host::launch_trace_texels_wavefront(ctx, layout, slots, iteration, samples_per_texel, max_bounces,
                                                       reset, lighting, texel_begin, texel_end, as_stream(stream));
    return nan_host::launch_trace_texels(ctx, layout, slots, iteration, samples_per_texel, max_bounces, reset,
                                         lighting, texel_begin, texel_end, as_stream(stream));
}

NAN_B200_API int nan_trace_probes(NanContext* ctx, float* values, uint32_t* sample_counts, uint32_t* self_hits,
                                  uint32_t* radial, const uint8_t* probes, uint32_t probe_count,
                                  const uint8_t* probe_instances, uint32_t probe_instance_count,
                                  uint32_t iteration, uint32_t samples_per_probe, uint32_t max_bounces, int reset,
                                  const NanLighting* lighting, uint32_t probe_begin, uint32_t probe_end,
                                  float* compensation, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if ((rc = need_scene(ctx))) return rc;
    if (!lighting) return invalid("null lighting");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if (probe_count && (!values || !sample_counts || !self_hits || !radial || !probes || !probe_instances))
        return invalid("null probe buffer");
    if (probe_count && (!aligned16(probes) || !aligned16(probe_instances) ||
                        (compensation && !aligned16(compensation))))
        return invalid("probe records and compensation must be 16-byte aligned");
    if (probe_end > probe_count) return invalid("probe range beyond probe_count");
    if (max_bounces > 64) return invalid("max_bounces above 64");
    if (ctx->tuning.integrator == 0)
        return nan_host::launch_trace_probes_wavefront(ctx, values, sample_counts, self_hits, radial, probes,
                                                       probe_count, probe_instances, probe_instance_count, iteration,
                                                       samples_per_probe, max_bounces, reset, lighting, probe_begin,
                                                       probe_end, compensation, as_stream(stream));
    return nan_host::launch_trace_probes(ctx, values, sample_counts, self_hits, radial, probes, probe_count,
                                         probe_instances, probe_instance_count, iteration, samples_per_probe,
                                         max_bounces, reset, lighting, probe_begin, probe_end, compensation,
                                         as_stream(stream));
}

NAN_B200_API int nan_resolve_mesh_colors(NanContext* ctx, const NanMeshColorsDesc* layout, const void* colors,
                                         int packed, float* out, uint32_t width, uint32_t height,
                                         const NanCamera* camera, const NanLighting* lighting, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    rc = need_scene(ctx);
    if (rc) return rc;
    if (!layout || !colors || !out || !camera || !lighting) return invalid("null argument");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if (!layout->face_infos || !layout->instance_infos || !layout->side_infos) return invalid("null layout buffer");
    if (layout->instance_count < ctx->scene.instance_count)
        return invalid("the layout covers fewer instances than the scene");
    if (!aligned16(out) || (!packed && !aligned16(colors))) return invalid("out and slot colors must be 16-byte aligned");
    return nan_host::launch_resolve_mesh_colors(ctx, layout, colors, packed, out, width, height, camera, lighting,
                                                as_stream(stream));
}

NAN_B200_API int nan_filter_mesh_colors(NanContext* ctx, const NanMeshColorsDesc* layout, const uint32_t* adjacency,
                                        const float* face_normals, const uint8_t* source, uint8_t* destination,
                                        float neighbor_weight, float normal_sigma_radians, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!layout || !adjacency || !face_normals || !source || !destination) return invalid("null argument");
    if (!layout->face_infos || !layout->instance_infos || !layout->side_infos || !layout->surface_prefix)
        return invalid("null layout buffer");
    if (source == destination) return invalid("the surface filter needs distinct source and destination buffers");
    if (!aligned16(adjacency) || !aligned16(face_normals) || !aligned16(source) || !aligned16(destination))
        return invalid("adjacency, normals and slot buffers must be 16-byte aligned");
    if (!(neighbor_weight >= 0.0f) || !(normal_sigma_radians >= 0.0f)) return invalid("negative filter weight or sigma");
    return nan_host::launch_filter_mesh_colors(ctx, layout, adjacency, face_normals, source, destination,
                                               neighbor_weight, normal_sigma_radians, as_stream(stream));
}

NAN_B200_API int nan_trace_probes_prt(NanContext* ctx, float* values, uint32_t* sample_counts, uint32_t* self_hits,
                                      uint32_t* radial, float* static_source, const uint8_t* probes,
                                      uint32_t probe_count, const uint8_t* probe_instances,
                                      uint32_t probe_instance_count, uint32_t iteration, uint32_t samples_per_probe,
                                      uint32_t max_bounces, int reset, const NanLighting* lighting,
                                      uint32_t probe_begin, uint32_t probe_end, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    rc = need_scene(ctx);
    if (rc) return rc;
    if (probe_count && (!values || !sample_counts || !self_hits || !radial || !static_source || !probes ||
                        !probe_instances || !lighting))
        return invalid("null argument");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if (!aligned16(probes) || !aligned16(probe_instances)) return invalid("probe records must be 16-byte aligned");
    return nan_host::launch_trace_probes_prt(ctx, values, sample_counts, self_hits, radial, static_source, probes,
                                             probe_count, probe_instances, probe_instance_count, iteration,
                                             samples_per_probe, max_bounces, reset, lighting, probe_begin,
                                             probe_end, as_stream(stream));
}

NAN_B200_API int nan_prt_project_lighting(NanContext* ctx, float* lighting_sh, uint32_t sample_count,
                                          const NanLighting* lighting, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!lighting_sh || !lighting) return invalid("null argument");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if (!aligned16(lighting_sh)) return invalid("lighting_sh must be 16-byte aligned");
    return nan_host::launch_prt_project_lighting(ctx, lighting_sh, sample_count, lighting, as_stream(stream));
}

NAN_B200_API int nan_prt_evaluate(NanContext* ctx, const float* values, const uint32_t* sample_counts,
                                  const float* static_source, const float* lighting_sh, float* out_values,
                                  uint32_t* out_sample_counts, uint32_t probe_count, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (probe_count && (!values || !sample_counts || !static_source || !lighting_sh || !out_values ||
                        !out_sample_counts))
        return invalid("null argument");
    if (!aligned16(lighting_sh)) return invalid("lighting_sh must be 16-byte aligned");
    return nan_host::launch_prt_evaluate(ctx, values, sample_counts, static_source, lighting_sh, out_values,
                                         out_sample_counts, probe_count, as_stream(stream));
}

NAN_B200_API int nan_resolve_probes(NanContext* ctx, const NanProbeLayoutDesc* layout, const float* values,
                                    const uint32_t* sample_counts, const uint32_t* self_hits,
                                    const uint32_t* radial, const NanProbeResolveOptions* options, float* out,
                                    uint32_t width, uint32_t height, const NanCamera* camera,
                                    const NanLighting* lighting, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    rc = need_scene(ctx);
    if (rc) return rc;
    if (!layout || !options || !camera || !lighting) return invalid("null argument");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if ((uint64_t)width * height == 0) return NAN_OK;
    if (!out || !layout->instances || (layout->probe_count && (!layout->probes || !values || !sample_counts ||
                                                               !self_hits || !radial)) ||
        (layout->node_count && !layout->nodes) ||
        (layout->triangle_vertex_probe_count && !layout->triangle_vertex_probes))
        return invalid("null buffer");
    if (!aligned16(out) || !aligned16(layout->probes) || !aligned16(layout->nodes) ||
        !aligned16(layout->instances) || !aligned16(layout->triangle_vertex_probes))
        return invalid("probe layout buffers and out must be 16-byte aligned");
    if (options->vertex_lighting_rgbm &&
        (!options->vertex_lighting_target || !options->vertex_lighting_triangle_map ||
         !options->vertex_lighting_instance_offsets || !aligned16(options->vertex_lighting_target) ||
         !aligned16(options->vertex_lighting_triangle_map) ||
         (reinterpret_cast<uintptr_t>(options->vertex_lighting_instance_offsets) & 7u)))
        return invalid("vertex lighting needs target, triangle map and instance offsets (aligned)");
    return nan_host::launch_resolve_probes(ctx, layout, values, sample_counts, self_hits, radial, options, out, width,
                                           height, camera, lighting, as_stream(stream));
}

static int wse_entry(NanContext* ctx, const float* positions, const float* normals, const float* densities,
                     const uint32_t* set_offsets, uint32_t set_count, const uint32_t* output_counts,
                     const float* surface_areas, const NanWseOptions* options, uint8_t* keep, float* poisson_radii,
                     uint32_t* rounds, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!set_offsets || !options || (set_count && (!output_counts || !surface_areas)))
        return invalid("null argument");
    if (set_count > 65536u) return invalid("at most 65536 candidate sets per call");
    if (set_offsets[0] != 0u) return invalid("set_offsets[0] must be 0");
    for (uint32_t k = 0; k < set_count; ++k) {
        if (set_offsets[k + 1] < set_offsets[k]) return invalid("set_offsets must be non-decreasing");
        if (!(surface_areas[k] > 0.0f) || !std::isfinite(surface_areas[k]))
            return invalid("surface areas must be positive and finite");
    }
    if (!(options->normal_cosine_threshold >= -1.0f && options->normal_cosine_threshold <= 1.0f) ||
        !(options->plane_distance_scale > 0.0f) || !std::isfinite(options->plane_distance_scale))
        return invalid("normal cosine threshold must be in [-1, 1] and plane distance scale positive");
    const uint32_t n = set_offsets[set_count];
    if (n && (!positions || !normals || !keep)) return invalid("null buffer");
    return nan_host::launch_wse_eliminate(ctx, positions, normals, densities, set_offsets, set_count, output_counts,
                                          surface_areas, options, keep, poisson_radii, rounds, as_stream(stream));
}

NAN_B200_API int nan_wse_eliminate(NanContext* ctx, const float* positions, const float* normals,
                                   const uint32_t* set_offsets, uint32_t set_count, const uint32_t* output_counts,
                                   const float* surface_areas, const NanWseOptions* options, uint8_t* keep,
                                   float* poisson_radii, uint32_t* rounds, void* stream) {
    return wse_entry(ctx, positions, normals, nullptr, set_offsets, set_count, output_counts, surface_areas, options,
                     keep, poisson_radii, rounds, stream);
}

NAN_B200_API int nan_wse_eliminate_adaptive(NanContext* ctx, const float* positions, const float* normals,
                                            const float* relative_densities, const uint32_t* set_offsets,
                                            uint32_t set_count, const uint32_t* output_counts,
                                            const float* surface_areas, const NanWseOptions* options, uint8_t* keep,
                                            float* poisson_radii, uint32_t* rounds, void* stream) {
    if (set_offsets && set_count && set_offsets[set_count] && !relative_densities)
        return invalid("relative densities are required");
    return wse_entry(ctx, positions, normals, relative_densities, set_offsets, set_count, output_counts,
                     surface_areas, options, keep, poisson_radii, rounds, stream);
}

NAN_B200_API int nan_filter_audit_repair(NanContext* ctx, const float* candidate_positions,
                                         const float* candidate_normals, const uint32_t* candidate_sets,
                                         uint32_t candidate_count, const float* base_positions,
                                         const float* base_normals, const uint32_t* base_sets, uint32_t base_count,
                                         const uint32_t* base_selected_indices, uint32_t base_selected_count,
                                         uint32_t set_count, const double* audit_cell_sizes,
                                         double normal_cosine_threshold, uint32_t* audit_indices,
                                         uint32_t* audit_count, uint32_t* repair_indices, uint32_t* repair_count,
                                         void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!candidate_positions || !candidate_normals || !base_positions || !base_normals || !audit_indices ||
        !audit_count || !repair_indices || !repair_count || !audit_cell_sizes)
        return invalid("surface probe candidate filter received a null pointer");
    if (candidate_count == 0 || base_count == 0) return invalid("candidate_count and base_count must be positive");
    if (base_selected_count > 0 && !base_selected_indices)
        return invalid("base_selected_indices cannot be null when selections exist");
    if (set_count == 0 || set_count > 65536u) return invalid("set_count must be in 1..65536");
    if (set_count > 1 && (!candidate_sets || !base_sets)) return invalid("several sets need candidate and base sets");
    for (uint32_t k = 0; k < set_count; ++k)
        if (!std::isfinite(audit_cell_sizes[k]) || !(audit_cell_sizes[k] > 0.0))
            return invalid("invalid candidate filter cell size or normal threshold");
    if (!std::isfinite(normal_cosine_threshold) || normal_cosine_threshold < -1.0 || normal_cosine_threshold > 1.0)
        return invalid("invalid candidate filter cell size or normal threshold");
    if ((uint64_t)candidate_count + base_selected_count > 0x7fffffffull) return invalid("too many entries");
    return nan_host::launch_filter_audit_repair(
        ctx, candidate_positions, candidate_normals, candidate_sets, candidate_count, base_positions, base_normals,
        base_sets, base_count, base_selected_indices, base_selected_count, set_count, audit_cell_sizes,
        normal_cosine_threshold, audit_indices, audit_count, repair_indices, repair_count, as_stream(stream));
}

NAN_B200_API int nan_build_point_octrees(NanContext* ctx, const float* positions, const uint32_t* set_offsets,
                                         uint32_t set_count, uint32_t leaf_capacity, uint32_t max_depth,
                                         uint32_t* nodes, uint32_t node_capacity, uint32_t* node_offsets,
                                         uint32_t* order, double* roots, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!set_offsets || !node_offsets || !roots) return invalid("surface probe octree received a null pointer");
    if (set_count == 0 || set_count > 65536u) return invalid("set_count must be in 1..65536");
    if (leaf_capacity == 0 || max_depth == 0 || max_depth > 16u)
        return invalid("leaf_capacity must be positive and max_depth in 1..16");
    if (set_offsets[0] != 0u) return invalid("set_offsets[0] must be 0");
    for (uint32_t k = 0; k < set_count; ++k)
        if (set_offsets[k + 1] < set_offsets[k]) return invalid("set_offsets must be non-decreasing");
    const uint32_t n = set_offsets[set_count];
    if (n == 0) return invalid("the octrees need at least one position");
    if (!positions || !order || (node_capacity && !nodes)) return invalid("null buffer");
    return nan_host::launch_build_point_octrees(ctx, positions, set_offsets, set_count, leaf_capacity, max_depth,
                                                nodes, node_capacity, node_offsets, order, roots, as_stream(stream));
}

NAN_B200_API int nan_deficit_repair(NanContext* ctx, const float* base_positions, const float* base_normals,
                                    const uint32_t* base_instances, uint32_t base_count,
                                    const float* candidate_positions, const float* candidate_normals,
                                    const uint32_t* candidate_instances, uint32_t candidate_count,
                                    const float* audit_positions, const float* audit_normals,
                                    const uint32_t* audit_instances, uint32_t audit_count,
                                    const float* instance_radii, uint32_t instance_count,
                                    const NanRepairOptions* options, uint32_t* selected, uint32_t* repair_count,
                                    uint32_t* counts_before, uint32_t* counts_after, float* weight_sums_before,
                                    float* weight_sums_after, float* ess_before, float* ess_after,
                                    uint32_t* rounds, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!options || !repair_count || !instance_radii) return invalid("null argument");
    if (base_count == 0 || audit_count == 0 || instance_count == 0)
        return invalid("base_count, audit_count and instance_count must be positive");
    if (instance_count > 65535u) return invalid("at most 65535 instances");
    if (!base_positions || !base_normals || !base_instances || !audit_positions || !audit_normals ||
        !audit_instances || !counts_before || !counts_after || !weight_sums_before || !weight_sums_after ||
        !ess_before || !ess_after)
        return invalid("null buffer");
    if (candidate_count && (!candidate_positions || !candidate_normals || !candidate_instances))
        return invalid("non-empty repair candidates need their buffers");
    if (options->min_gather_count == 0 || options->min_gather_count > 32)
        return invalid("min_gather_count must be within [1, 32]");
    if (!std::isfinite(options->normal_cosine_threshold) || options->normal_cosine_threshold < -1.0f ||
        options->normal_cosine_threshold > 1.0f || !std::isfinite(options->weight_epsilon) ||
        options->weight_epsilon < 0.0f)
        return invalid("invalid deficit repair thresholds");
    if (std::min(options->max_repair_count, candidate_count) > 0 && !selected)
        return invalid("selected cannot be null when repairs are enabled");
    for (uint32_t k = 0; k < instance_count; ++k)
        if (!std::isfinite(instance_radii[k]) || !(instance_radii[k] > 0.0f))
            return invalid("instance radii must be positive and finite");
    const float* base[2] = {base_positions, base_normals};
    const float* cand[2] = {candidate_positions, candidate_normals};
    const float* audit[2] = {audit_positions, audit_normals};
    return nan_host::launch_deficit_repair(ctx, base, base_instances, base_count, cand, candidate_instances,
                                           candidate_count, audit, audit_instances, audit_count, instance_radii,
                                           instance_count, options, selected, repair_count, counts_before,
                                           counts_after, weight_sums_before, weight_sums_after, ess_before,
                                           ess_after, rounds, as_stream(stream));
}

NAN_B200_API int nan_estimate_support(NanContext* ctx, const float* reference_positions,
                                      const float* reference_normals, const uint32_t* reference_instances,
                                      const float* reference_area_weights, uint32_t reference_count,
                                      const float* query_positions, const float* query_normals,
                                      const uint32_t* query_instances, uint32_t query_count,
                                      const float* instance_radii, uint32_t instance_count,
                                      const NanSupportOptions* options, float* support_f, float* density_m,
                                      void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!options || !instance_radii) return invalid("null argument");
    if (instance_count == 0 || instance_count > 65535u) return invalid("instance_count must be in [1, 65535]");
    if (reference_count && (!reference_positions || !reference_normals || !reference_instances ||
                            !reference_area_weights))
        return invalid("null reference buffer");
    if (query_count && (!query_positions || !query_normals || !query_instances || !support_f || !density_m))
        return invalid("null query buffer");
    if (!std::isfinite(options->normal_cosine_threshold) || options->normal_cosine_threshold < -1.0f ||
        options->normal_cosine_threshold > 1.0f || !std::isfinite(options->weight_epsilon) ||
        options->weight_epsilon < 0.0f || !std::isfinite(options->max_density_multiplier))
        return invalid("invalid support options");
    for (uint32_t k = 0; k < instance_count; ++k)
        if (!std::isfinite(instance_radii[k]) || !(instance_radii[k] > 0.0f))
            return invalid("instance radii must be positive and finite");
    return nan_host::launch_estimate_support(ctx, reference_positions, reference_normals, reference_instances,
                                             reference_area_weights, reference_count, query_positions,
                                             query_normals, query_instances, query_count, instance_radii,
                                             instance_count, options, support_f, density_m, as_stream(stream));
}

NAN_B200_API int nan_pack_rgb9e5(NanContext* ctx, const uint8_t* slots, uint32_t* out, uint32_t count, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (count && (!slots || !out)) return invalid("null buffer");
    if (count && !aligned16(slots)) return invalid("slots must be 16-byte aligned");
    return nan_host::launch_pack_rgb9e5(ctx, slots, out, count, as_stream(stream));
}


NAN_B200_API int nan_cache_sizes(const NanCacheConfig* config, uint64_t* mlp_params, uint64_t* table_params) {
    int rc = check_config(config);
    if (rc) return rc;
    if (mlp_params) *mlp_params = nan_host::cache_mlp_params();
    if (table_params) *table_params = nan_host::cache_table_params(config);
    return NAN_OK;
}

NAN_B200_API int nan_cache_create(NanContext* ctx, const NanCacheConfig* config, NanCache** out) {
    if (!out) return invalid("null output pointer");
    *out = nullptr;
    int rc = enter(ctx);
    if (rc) return rc;
    rc = check_config(config);
    if (rc) return rc;
    return nan_host::cache_create(ctx, config, out);
}

NAN_B200_API int nan_cache_destroy(NanCache* cache) {
    if (!cache) return NAN_OK;
    cudaSetDevice(cache->ctx->device);
    cudaDeviceSynchronize();
    nan_host::cache_destroy(cache);
    return NAN_OK;
}

NAN_B200_API int nan_cache_set_params(NanCache* cache, const float* mlp, const float* table, void* stream) {
    int rc = cache_enter(cache);
    if (rc) return rc;
    if (!mlp || !table) return invalid("null parameter array");
    return nan_host::cache_set_params(cache, mlp, table, as_stream(stream));
}

NAN_B200_API int nan_cache_get_params(NanCache* cache, float* mlp, float* table, float* mlp_grad, float* table_grad,
                                      float* loss, void* stream) {
    int rc = cache_enter(cache);
    if (rc) return rc;
    return nan_host::cache_get_params(cache, mlp, table, mlp_grad, table_grad, loss, as_stream(stream));
}

NAN_B200_API int nan_cache_infer(NanCache* cache, const float* queries, uint32_t count, float* out, void* stream) {
    int rc = cache_enter(cache);
    if (rc) return rc;
    if (count && (!queries || !out)) return invalid("null query or output buffer");
    if (!aligned16(queries) || !aligned16(out)) return invalid("queries and out must be 16-byte aligned");
    return nan_host::launch_cache_infer(cache, queries, count, nullptr, out, nullptr, nullptr, as_stream(stream));
}

NAN_B200_API int nan_cache_backward(NanCache* cache, const float* queries, const float* targets, uint32_t count,
                                    uint32_t batch, void* stream) {
    int rc = cache_enter(cache);
    if (rc) return rc;
    if (count && (!queries || !targets)) return invalid("null query or target buffer");
    if (!aligned16(queries) || !aligned16(targets)) return invalid("queries and targets must be 16-byte aligned");
    if (batch == 0) return invalid("batch must be positive");
    return nan_host::launch_cache_backward(cache, queries, targets, count, batch, as_stream(stream));
}

NAN_B200_API int nan_cache_step(NanCache* cache, void* stream) {
    int rc = cache_enter(cache);
    if (rc) return rc;
    return nan_host::launch_cache_step(cache, as_stream(stream));
}

NAN_B200_API int nan_cache_set_learning_rate(NanCache* cache, float learning_rate) {
    if (!cache) return invalid("null cache");
    if (!(learning_rate >= 0.0f) || !std::isfinite(learning_rate)) return invalid("learning rate must be finite and >= 0");
    cache->cfg.learning_rate = learning_rate;
    return NAN_OK;
}

NAN_B200_API int nan_cache_train(NanCache* cache, const float* queries, const float* targets, uint32_t count,
                                 uint32_t batch, void* stream) {
    int rc = cache_enter(cache);
    if (rc) return rc;
    if (batch == 0) return invalid("batch must be positive");
    if (count && (!queries || !targets)) return invalid("null query or target buffer");
    if (!aligned16(queries) || !aligned16(targets)) return invalid("queries and targets must be 16-byte aligned");
    for (uint32_t b = 0; b < count; b += batch) {
        const uint32_t n = std::min(batch, count - b);
        rc = nan_host::launch_cache_backward(cache, queries + 8ull * b, targets + 4ull * b, n, n, as_stream(stream));
        if (rc) return rc;
        rc = nan_host::launch_cache_step(cache, as_stream(stream));
        if (rc) return rc;
    }
    return NAN_OK;
}

NAN_B200_API int nan_trace_points(NanContext* ctx, const float* points, uint32_t count, float* out,
                                  uint32_t iteration, uint32_t samples, uint32_t max_bounces, uint32_t flags,
                                  const NanLighting* lighting, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    rc = need_scene(ctx);
    if (rc) return rc;
    if (count && (!points || !out || !lighting)) return invalid("null argument");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if (!aligned16(points) || !aligned16(out)) return invalid("points and out must be 16-byte aligned");
    if (flags & ~(uint32_t)NAN_POINTS_INDIRECT_ONLY) return invalid("unknown points flag");
    // Up to kPointsPerThreadMax points (the learned cache's training sets) a
    // thread per point beats the wavefront's rounds of small launches.
    constexpr uint32_t kPointsPerThreadMax = 1u << 18;
    if (ctx->tuning.integrator != 0 || count <= kPointsPerThreadMax)
        return nan_host::launch_trace_points(ctx, points, count, out, iteration, samples, max_bounces, flags, lighting,
                                             as_stream(stream));
    return nan_host::launch_trace_points_wavefront(ctx, points, count, out, iteration, samples, max_bounces, flags,
                                                   lighting, as_stream(stream));
}

NAN_B200_API int nan_trace_screen_cached(NanContext* ctx, NanCache* cache, float* out, uint32_t width,
                                         uint32_t height, uint32_t frame, const NanCamera* camera,
                                         const NanLighting* lighting, const NanCachedFrame* fd, void* stream) {
    int rc = enter(ctx);
    if (rc) return rc;
    rc = need_scene(ctx);
    if (rc) return rc;
    if (!cache || !out || !camera || !lighting || !fd) return invalid("null argument");
    if (const int lrc = nan_host::check_lighting(lighting)) return lrc;
    if (cache->ctx->device != ctx->device) return invalid("cache and context are on different devices");
    const uint64_t P = (uint64_t)width * height;
    if (P == 0) return NAN_OK;
    if (P > 0x7fffffffull) return invalid("image too large");
    if (!fd->queries || !fd->query_weights || !fd->query_count) return invalid("null cached-frame scratch");
    if (fd->train_count && (!fd->train_points || !fd->train_queries)) return invalid("null training buffers");
    if (fd->train_count > P) return invalid("more training samples than pixels");
    if (fd->cache_vertex > 1) return invalid("cache_vertex must be 0 or 1");
    if (fd->train_offset >= P || fd->train_stride == 0 || fd->train_stride >= P + (P == 1 ? 1 : 0))
        return invalid("training offset and stride must lie in [0, W*H)");
    if ((uint64_t)fd->train_stride * fd->train_stride_inverse % P != 1 % P)
        return invalid("train_stride_inverse is not the inverse of train_stride modulo W*H");
    if (!aligned16(out) || !aligned16(fd->queries) || !aligned16(fd->query_weights) ||
        !aligned16(fd->train_points) || !aligned16(fd->train_queries))
        return invalid("image, query and training buffers must be 16-byte aligned");
    return nan_host::launch_trace_screen_cached(ctx, cache, out, width, height, frame, camera, lighting, fd,
                                                as_stream(stream));
}

NAN_B200_API int nan_batch_create(NanContext* ctx, const NanProbeSet* sets, uint32_t set_count, NanBatch** out) {
    if (!out) return invalid("null output pointer");
    *out = nullptr;
    int rc = enter(ctx);
    if (rc) return rc;
    if (set_count && !sets) return invalid("null probe sets");
    for (uint32_t i = 0; i < set_count; ++i) {
        const NanProbeSet& p = sets[i];
        if (!p.scene || p.scene->device != ctx->device) return invalid("probe set scene is null or on another device");
        if (!p.scene->has_scene) return invalid("probe set scene has no BVH");
        if (p.probe_count && (!p.probes || !p.probe_instances || !p.values || !p.sample_counts || !p.self_hits ||
                              !p.radial))
            return invalid("null probe buffer");
        if (!aligned16(p.probes) || !aligned16(p.probe_instances) || !aligned16(p.compensation))
            return invalid("probe records, instances and compensation must be 16-byte aligned");
    }
    return nan_host::batch_create(ctx, sets, set_count, out);
}

NAN_B200_API int nan_batch_destroy(NanBatch* batch) {
    if (!batch) return NAN_OK;
    cudaSetDevice(batch->ctx->device);
    cudaDeviceSynchronize();
    nan_host::batch_destroy(batch);
    return NAN_OK;
}

NAN_B200_API int nan_batch_info(NanBatch* batch, uint32_t* min_stack_depth, uint32_t* total_probes,
                                NanBatchTuning* tuning) {
    if (!batch) return invalid("null batch");
    if (min_stack_depth) *min_stack_depth = nan_host::batch_min_depth(batch);
    if (total_probes) *total_probes = nan_host::batch_total(batch);
    if (tuning) *tuning = batch->tuning;
    return NAN_OK;
}

NAN_B200_API int nan_batch_set_tuning(NanBatch* batch, const NanBatchTuning* tuning) {
    if (!batch || !tuning) return invalid("null argument");
    return nan_host::batch_set_tuning(batch, tuning);
}

NAN_B200_API int nan_batch_set_mode(NanBatch* batch, uint32_t mode) {
    if (!batch) return invalid("null batch");
    return nan_host::batch_set_mode(batch, mode);
}

NAN_B200_API int nan_batch_trace_probes(NanBatch* batch, uint32_t iteration, uint32_t samples_per_probe,
                                        uint32_t max_bounces, int reset, void* stream) {
    if (!batch) return invalid("null batch");
    int rc = enter(batch->ctx);
    if (rc) return rc;
    return nan_host::batch_frame(batch, iteration, samples_per_probe, max_bounces, reset, as_stream(stream));
}

NAN_B200_API int nan_batch_autotune(NanBatch* batch, uint32_t samples_per_probe, uint32_t max_bounces, void* stream,
                                    NanBatchTuning* chosen, float* frame_ms) {
    if (!batch) return invalid("null batch");
    int rc = enter(batch->ctx);
    if (rc) return rc;
    rc = nan_host::batch_autotune(batch, samples_per_probe, max_bounces, as_stream(stream), chosen);
    if (frame_ms) *frame_ms = batch->tuned_ms;
    return rc;
}

NAN_B200_API int nan_batch_capture(NanBatch* batch, uint32_t first_iteration, int reset_first,
                                   uint32_t samples_per_probe, uint32_t max_bounces, void* stream) {
    if (!batch) return invalid("null batch");
    int rc = enter(batch->ctx);
    if (rc) return rc;
    return nan_host::batch_capture(batch, first_iteration, reset_first, samples_per_probe, max_bounces,
                                   as_stream(stream));
}

NAN_B200_API int nan_batch_replay(NanBatch* batch, uint32_t frames, void* stream) {
    if (!batch) return invalid("null batch");
    int rc = enter(batch->ctx);
    if (rc) return rc;
    return nan_host::batch_replay(batch, frames, as_stream(stream));
}
}  // extern "C"
