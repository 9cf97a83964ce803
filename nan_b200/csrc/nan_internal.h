// nan_internal.h -- context object and host-side launchers shared by the
// translation units of libnan_b200.so (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/nan_b200.h"

struct NanContext {
    int device = 0;
    uint32_t* d_status = nullptr;              // device status word
    unsigned long long* d_counters = nullptr;  // NanCounters on the device
    // Scene (caller-owned buffers, read in place by the shading code).
    NanSceneDesc scene{};
    bool has_scene = false;
    // BVH storage owned by the context.
    bool caller_owned_bvh = false;  // BVH storage passed in by the caller (not freed here)
    float4* nodes = nullptr;        // 4 float4 per interior node
    float4* tris = nullptr;         // 3 float4 per triangle, leaf order
    uint2* tri_refs = nullptr;      // flat index -> (instance, primitive)
    uint4* wnodes = nullptr;        // compressed 8-wide nodes, 5 uint4 each (PLOC builds only)
    float4* wtris = nullptr;        // triangles in the wide nodes' leaf order
    uint32_t wide_count = 0;
    bool wide_built = false;        // wnodes/wtris hold this scene's wide BVH
    // Triangles the owned storage holds: nodes/tris/tri_refs, and the wide
    // nodes/triangles. A rebuild that fits reuses them (grow-only).
    uint32_t bvh_capacity = 0;
    uint32_t wide_capacity = 0;
    int root = 0;
    uint32_t tri_count = 0;
    uint32_t node_count = 0;
    uint32_t leaf_count = 0;
    uint32_t max_depth = 0;
    uint64_t device_bytes = 0;
    double build_ms = 0.0;
    double sah_cost = 0.0;
    uint64_t launches = 0;
    // Wavefront scratch arena (nan_ctx_reserve) and tuning (nan_ctx_configure).
    void* scratch = nullptr;
    uint64_t scratch_bytes = 0;
    NanTuning tuning{};
    // Area lights (nan_ctx_set_area_lights): caller-owned table.
    const float* lights = nullptr;
    uint32_t light_count = 0;
    float light_power = 0.0f;
    // Stage timing (NanTuning.kernel_timing): events pending a read, a pool
    // of free events, and the sums per stage kind (0 extend, 1 shadow, 2 other).
    struct TimedLaunch {
        int kind;
        cudaEvent_t start, stop;
    };
    std::vector<TimedLaunch> timed;
    std::vector<cudaEvent_t> event_pool;
    double stage_ms[3] = {0.0, 0.0, 0.0};
    uint64_t stage_launches[3] = {0, 0, 0};
};

// Learned radiance cache (nan_cache.cu): parameters, Adam moments and
// gradients in one block each: mlp = [p | m | v | g] x 16384 floats,
// table = [p | m | v | g] x table_params floats.
struct NanCache {
    NanContext* ctx = nullptr;
    NanCacheConfig cfg{};
    uint32_t resolutions[16] = {};
    size_t table_params = 0;
    uint64_t step = 0;
    float* mlp = nullptr;
    unsigned char* img = nullptr;  // bf16 weight images, interleaved tile layout
    float* table = nullptr;
    void* table16 = nullptr;       // fp16 feature pairs read by the encoding
    float* loss = nullptr;
    float* partials = nullptr;     // per-CTA weight gradients of one training launch
};

namespace nan_host {
struct BatchImpl;
}

// Multi-scene probe batch (nan_batch.cu).
struct NanBatch {
    NanContext* ctx = nullptr;  // device, counters and status of the batched launches
    nan_host::BatchImpl* impl = nullptr;
    NanBatchTuning tuning{};
    float tuned_ms = -1.0f;
    uint32_t mode = 0;  // NAN_BATCH_SEQUENTIAL_SAMPLES or NAN_BATCH_INDEPENDENT_SAMPLES
};

namespace nan_host {

void set_error(const std::string& msg);
// Stream-ordered scratch from this library's pool on the current device
// (freed with cudaFreeAsync; the memory stays in the pool until
// trim_scratch, which nan_ctx_destroy calls).
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t stream);
void trim_scratch(int device);
// The context's wavefront scratch replaced by `bytes` from the pool (0:
// released). The caller has synchronised the device: nothing still uses
// the old scratch.
cudaError_t replace_context_scratch(NanContext* ctx, size_t bytes);
int cuda_fail(cudaError_t err, const char* what);

// A lighting record the kernels can read: a sky-view LUT needs a size and a
// 16-byte aligned address. Returns NAN_OK or sets the error and returns
// NAN_ERR_INVALID_ARGUMENT.
inline int check_lighting(const NanLighting* l) {
    if (l && l->sky_view_lut) {
        if (l->sky_view_width == 0u || l->sky_view_height == 0u || l->sky_view_width > 16384u ||
            l->sky_view_height > 16384u) {
            set_error("sky_view_lut needs a width and height in 1..16384");
            return NAN_ERR_INVALID_ARGUMENT;
        }
        if (reinterpret_cast<uintptr_t>(l->sky_view_lut) & 15u) {
            set_error("sky_view_lut must be 16-byte aligned");
            return NAN_ERR_INVALID_ARGUMENT;
        }
    }
    return NAN_OK;
}

void free_scene(NanContext* ctx);
// Drops the scene's metadata but keeps owned BVH storage for a rebuild.
void forget_scene(NanContext* ctx);
// Stage timing: begin returns the start event (or nullptr when timing is
// off); end records the stop event and queues the pair.
cudaEvent_t timing_begin(NanContext* ctx, cudaStream_t stream);
void timing_end(NanContext* ctx, int kind, cudaEvent_t start, cudaStream_t stream);
int read_kernel_times(NanContext* ctx, NanKernelTimes* out, int reset);
void release_timing(NanContext* ctx);
int build_scene(NanContext* ctx, const NanSceneDesc* desc, cudaStream_t stream);
int world_triangles(NanContext* ctx, float* out, cudaStream_t stream);

int launch_intersect(NanContext* ctx, const float* rays, uint32_t count, uint32_t* ids, float* tb,
                     cudaStream_t stream);
int launch_occluded(NanContext* ctx, const float* rays, uint32_t count, float* vis, cudaStream_t stream);
int visibility_ray_table(uint32_t ray_count, float* host_table);
int launch_visibility_sh16(NanContext* ctx, const float* positions, const float* normals, uint32_t count,
                           const float* table, uint32_t ray_count, float max_distance, float self_bias, float* out,
                           uint32_t* visible, cudaStream_t stream);
int launch_trace_screen(NanContext* ctx, float* out, uint32_t w, uint32_t h, uint32_t frame,
                        uint32_t max_vertices, const NanCamera* cam, const NanLighting* light,
                        cudaStream_t stream);
int launch_accumulate(NanContext* ctx, const float* input, float* output, float* history, uint32_t w,
                      uint32_t h, int reset, cudaStream_t stream);
int launch_trace_texels(NanContext* ctx, const NanMeshColorsDesc* layout, uint8_t* slots, uint32_t iteration,
                        uint32_t spt, uint32_t max_bounces, int reset, const NanLighting* light,
                        uint32_t begin, uint32_t end, cudaStream_t stream);
int launch_trace_probes(NanContext* ctx, float* values, uint32_t* counts, uint32_t* self_hits,
                        uint32_t* radial, const uint8_t* probes, uint32_t probe_count,
                        const uint8_t* probe_instances, uint32_t probe_instance_count, uint32_t iteration,
                        uint32_t spp, uint32_t max_bounces, int reset, const NanLighting* light,
                        uint32_t begin, uint32_t end, float* compensation, cudaStream_t stream);
size_t wavefront_bytes_per_path();
int launch_trace_texels_wavefront(NanContext* ctx, const NanMeshColorsDesc* layout, uint8_t* slots,
                                  uint32_t iteration, uint32_t spt, uint32_t max_bounces, int reset,
                                  const NanLighting* light, uint32_t begin, uint32_t end, cudaStream_t stream);
int launch_trace_screen_wavefront(NanContext* ctx, float* out, uint32_t w, uint32_t h, uint32_t frame,
                                  uint32_t max_vertices, const NanCamera* cam, const NanLighting* light,
                                  cudaStream_t stream);
const void* wavefront_extend_kernel();  // for occupancy queries
int launch_batch_wavefront(NanContext* ctx, const void* sets, const uint32_t* prefix, const void* batch_ctl,
                           uint32_t set_count, uint32_t total, uint32_t* set_of, uint32_t spp, uint32_t max_bounces,
                           float t_max, cudaStream_t st);
int launch_batch_wavefront_independent(NanContext* ctx, const void* sets, const uint32_t* prefix,
                                       const void* batch_ctl, uint32_t set_count, uint32_t total, uint32_t* set_of,
                                       void* samples, uint64_t path_capacity, uint32_t spp, uint32_t max_bounces,
                                       float t_max, cudaStream_t st);
size_t probe_sample_bytes();
int launch_trace_probes_wavefront(NanContext* ctx, float* values, uint32_t* counts, uint32_t* self_hits,
                                  uint32_t* radial, const uint8_t* probes, uint32_t probe_count,
                                  const uint8_t* probe_instances, uint32_t probe_instance_count, uint32_t iteration,
                                  uint32_t spp, uint32_t max_bounces, int reset, const NanLighting* light,
                                  uint32_t begin, uint32_t end, float* compensation, cudaStream_t stream);
size_t cache_table_params(const NanCacheConfig* cfg);
size_t cache_mlp_params();
int cache_create(NanContext* ctx, const NanCacheConfig* cfg, NanCache** out);
void cache_destroy(NanCache* k);
int cache_set_params(NanCache* k, const float* mlp, const float* table, cudaStream_t st);
int cache_get_params(NanCache* k, float* mlp, float* table, float* mlp_grad, float* table_grad, float* loss,
                     cudaStream_t st);
int launch_cache_infer(NanCache* k, const float* queries, uint32_t count, const uint32_t* count_dev, float* out,
                       const float* weights, float* image, cudaStream_t st);
int launch_cache_backward(NanCache* k, const float* queries, const float* targets, uint32_t count, uint32_t batch,
                          cudaStream_t st);
int launch_cache_step(NanCache* k, cudaStream_t st);
int launch_trace_points_wavefront(NanContext* ctx, const float* points, uint32_t count, float* out,
                                  uint32_t iteration, uint32_t samples, uint32_t max_bounces, uint32_t flags,
                                  const NanLighting* light, cudaStream_t st);
// The same values with one thread per point (one launch): the choice for
// small point sets, whose wavefront rounds are bound by launch latency.
int launch_trace_points(NanContext* ctx, const float* points, uint32_t count, float* out, uint32_t iteration,
                        uint32_t samples, uint32_t max_bounces, uint32_t flags, const NanLighting* light,
                        cudaStream_t st);
int launch_trace_screen_cached(NanContext* ctx, NanCache* cache, float* out, uint32_t w, uint32_t h,
                               uint32_t frame, const NanCamera* cam, const NanLighting* light,
                               const NanCachedFrame* fd, cudaStream_t st);
int batch_create(NanContext* ctx, const NanProbeSet* sets, uint32_t count, NanBatch** out);
void batch_destroy(NanBatch* b);
uint32_t batch_min_depth(const NanBatch* b);
int batch_set_mode(NanBatch* b, uint32_t mode);
uint32_t batch_total(const NanBatch* b);
int batch_set_tuning(NanBatch* b, const NanBatchTuning* t);
int batch_frame(NanBatch* b, uint32_t iteration, uint32_t spp, uint32_t max_bounces, int reset, cudaStream_t st);
int batch_capture(NanBatch* b, uint32_t first_iteration, int reset_first, uint32_t spp, uint32_t max_bounces,
                  cudaStream_t st);
int batch_replay(NanBatch* b, uint32_t frames, cudaStream_t st);
int batch_autotune(NanBatch* b, uint32_t spp, uint32_t max_bounces, cudaStream_t st, NanBatchTuning* chosen);
int launch_resolve_mesh_colors(NanContext* ctx, const NanMeshColorsDesc* layout, const void* colors, int packed,
                               float* out, uint32_t w, uint32_t h, const NanCamera* cam, const NanLighting* light,
                               cudaStream_t st);
int launch_wse_eliminate(NanContext* ctx, const float* positions, const float* normals, const float* densities,
                         const uint32_t* set_offsets, uint32_t set_count, const uint32_t* output_counts,
                         const float* surface_areas, const NanWseOptions* opt, uint8_t* keep, float* poisson_radii,
                         uint32_t* rounds_out, cudaStream_t st);
int launch_filter_audit_repair(NanContext* ctx, const float* cand_pos, const float* cand_nrm, const uint32_t* cand_set,
                               uint32_t cand_count, const float* base_pos, const float* base_nrm,
                               const uint32_t* base_set, uint32_t base_count, const uint32_t* base_selected,
                               uint32_t base_selected_count, uint32_t set_count, const double* cell_sizes,
                               double ncos, uint32_t* audit_indices, uint32_t* audit_count, uint32_t* repair_indices,
                               uint32_t* repair_count, cudaStream_t st);
int launch_build_point_octrees(NanContext* ctx, const float* positions, const uint32_t* set_offsets,
                               uint32_t set_count, uint32_t leaf_capacity, uint32_t max_depth, uint32_t* nodes,
                               uint32_t node_capacity, uint32_t* node_offsets, uint32_t* order, double* roots,
                               cudaStream_t st);
int launch_estimate_support(NanContext* ctx, const float* ref_pos, const float* ref_nrm, const uint32_t* ref_inst,
                            const float* area_weights, uint32_t ref_count, const float* query_pos,
                            const float* query_nrm, const uint32_t* query_inst, uint32_t query_count,
                            const float* radii, uint32_t instance_count, const NanSupportOptions* opt,
                            float* support_f, float* density_m, cudaStream_t st);
int launch_deficit_repair(NanContext* ctx, const float* const* base, const uint32_t* base_instances, uint32_t base_count,
                          const float* const* cand, const uint32_t* cand_instances, uint32_t cand_count,
                          const float* const* audit, const uint32_t* audit_instances, uint32_t audit_count,
                          const float* radii, uint32_t instance_count, const NanRepairOptions* opt, uint32_t* selected,
                          uint32_t* repair_count, uint32_t* counts_before, uint32_t* counts_after,
                          float* sums_before, float* sums_after, float* ess_before, float* ess_after,
                          uint32_t* rounds_out, cudaStream_t st);
int launch_resolve_probes(NanContext* ctx, const NanProbeLayoutDesc* lay, const float* values,
                          const uint32_t* counts, const uint32_t* self_hits, const uint32_t* radial,
                          const NanProbeResolveOptions* opt, float* out, uint32_t w, uint32_t h,
                          const NanCamera* cam, const NanLighting* light, cudaStream_t st);
int launch_filter_mesh_colors(NanContext* ctx, const NanMeshColorsDesc* layout, const uint32_t* adjacency,
                              const float* face_normals, const uint8_t* src, uint8_t* dst, float neighbor_weight,
                              float sigma, cudaStream_t st);
int launch_trace_probes_prt(NanContext* ctx, float* values, uint32_t* counts, uint32_t* self_hits, uint32_t* radial,
                            float* static_source, const uint8_t* probes, uint32_t probe_count,
                            const uint8_t* probe_instances, uint32_t probe_instance_count, uint32_t iteration,
                            uint32_t spp, uint32_t max_bounces, int reset, const NanLighting* light, uint32_t begin,
                            uint32_t end, cudaStream_t st);
int launch_prt_project_lighting(NanContext* ctx, float* sh, uint32_t samples, const NanLighting* light,
                                cudaStream_t st);
int launch_prt_evaluate(NanContext* ctx, const float* values, const uint32_t* counts, const float* static_source,
                        const float* sh, float* out, uint32_t* out_counts, uint32_t n, cudaStream_t st);
int launch_pack_rgb9e5(NanContext* ctx, const uint8_t* slots, uint32_t* out, uint32_t count,
                       cudaStream_t stream);

}  // namespace nan_host
