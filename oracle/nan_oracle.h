/* nan_oracle.h -- CPU restatement of the reference's path-integration math.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path:
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load
 * it; the product (nan_b200/) never does.
 *
 * Every function restates a reference Slang/Python function; the citation
 * (path:line, relative to the reference project root) sits beside each
 * definition in nan_oracle.cpp.
 *
 * Two precisions:
 *   ORACLE_F32  float arithmetic in the reference's operation order (the
 *               "spec" mode the CUDA kernels are compared with bit for bit);
 *   ORACLE_F64  the same algorithm in double precision (the FP64 oracle the
 *               converged estimates are compared with).
 *
 * Record layouts are the reference's (all little-endian, 4-byte words):
 *   vertices        f32[V][8]   position, normal, uv      (scene.py:386-400)
 *   indices         u32[T][3]   mesh-local vertex indices
 *   mesh_descs      u32[M][4]   vertex_count, index_count, vertex_offset,
 *                               index_offset              (scene.py:84-98)
 *   instance_descs  u32[I][4]   mesh_id, material_id, transform_id, flags
 *   transforms      f32[X][16]  row-major float4x4 (mul(M, float4(p, 1)))
 *   inv_transposes  f32[X][16]  transpose(inverse(M))
 *   materials       f32[N][8]   base_color.rgb, flags(u32), emissive.rgb, pad
 */
#ifndef NAN_ORACLE_H
#define NAN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_F32 = 0, ORACLE_F64 = 1 };

typedef struct OracleLighting {
    float sun_direction[3];
    float sun_cos_half_angle;
    float sun_color[3];
    float sun_intensity;
    float sun_transmittance[3];
    float ray_t_max;
    float sky_radiance[3];
    uint32_t flags; /* bit 0: sun disk on primary misses */
    const float* sky_view_lut; /* host f32[height][width][4], or null: constant sky */
    uint32_t sky_view_width;
    uint32_t sky_view_height;
    float sky_view_up[3];
    float sky_view_horizon_angle;
} OracleLighting;

typedef struct OracleCamera {
    float position[3];
    float jitter_x;
    float image_u[3];
    float jitter_y;
    float image_v[3];
    float near_clip;
    float image_w[3];
    float far_clip;
} OracleCamera;

typedef struct OracleRayCounts {
    uint64_t extend_rays;
    uint64_t shadow_rays;
    uint64_t node_fetches;
    uint64_t triangle_tests;
} OracleRayCounts;

const char* oracle_last_error(void);

/* ---- scalar building blocks ------------------------------------------- */
void oracle_rng_sequence(uint32_t x, uint32_t y, uint32_t sample_index,
                         int count, float* out);
void oracle_sincos(const float* angles, int count, float* out_sin,
                   float* out_cos);
void oracle_pack_rgb9e5(const float* rgb, int count, uint32_t* out);
/* The own atan2 and asin (float) of the kernels, elementwise: atan2(y, x), asin(y). */
void oracle_atan2_asin(const float* y, const float* x, int count, float* out_atan2, float* out_asin);
/* sample_sky_lut (scene.slang:469-518) for unit directions f32[N][3] -> f32[N][3];
 * precision ORACLE_F32 (the kernels' operations) or ORACLE_F64. */
void oracle_sky_radiance(const OracleLighting* lighting, const float* dirs, int count, int precision, float* out);
void oracle_unpack_rgb9e5(const uint32_t* packed, int count, float* out_rgb);
void oracle_f32_to_f16(const float* values, int count, uint16_t* out);
void oracle_hemi_oct_encode(const float* dirs, int count, float* out_uv);
void oracle_hemi_oct_decode(const float* uv, int count, float* out_dirs);
void oracle_cosine_sample_hemisphere(const float* u, int count, float* out4);
void oracle_mesh_colors_address_to_ij(const uint32_t* address,
                                      const uint32_t* resolution, int count,
                                      uint32_t* out_ij);

/* ---- scenes ------------------------------------------------------------ */
void* oracle_scene_create(const float* vertices, int vertex_count,
                          const uint32_t* indices, int triangle_count,
                          const uint32_t* mesh_descs, int mesh_count,
                          const uint32_t* instance_descs, int instance_count,
                          const float* transforms,
                          const float* inverse_transposes,
                          int transform_count, const float* materials,
                          int material_count);
void oracle_scene_destroy(void* scene);
int oracle_scene_triangle_count(void* scene);
/* World-space triangles in flat order (instance-major), f32[T][9]. */
void oracle_scene_world_triangles(void* scene, float* out9);
/* Binned-SAH (8 bins) BVH statistics: node count, leaf count, SAH cost. */
void oracle_scene_bvh_stats(void* scene, double* out3);

/* rays f32[N][8] = origin, t_min, dir, t_max.
 * hits: u32[N][4] = valid, instance, primitive, flat index;
 *       f32[N][3] = t, bary.x, bary.y.
 * mode: 0 float BVH, 1 float brute force, 2 double brute force. */
void oracle_intersect(void* scene, const float* rays, int count, int mode,
                      uint32_t* out_hit_ids, float* out_hit_tb,
                      OracleRayCounts* counts);
void oracle_visibility(void* scene, const float* rays, int count, int mode,
                       float* out_visibility, OracleRayCounts* counts);

/* ---- integrators (float spec or FP64) ---------------------------------- */
/* Screen path tracer (path_tracer.slang:86-130) for the listed pixels
 * (u32 pairs x, y); writes float4 per listed pixel. */
int oracle_trace_screen(void* scene, const OracleLighting* lighting,
                        const OracleCamera* camera, uint32_t width,
                        uint32_t height, uint32_t frame,
                        uint32_t max_vertices, const uint32_t* pixels,
                        int pixel_count, int precision, int threads,
                        float* out_rgba, OracleRayCounts* counts);

/* Texture-space tracer (texture_space_path_tracer.slang:140-216) for the
 * listed (instance, instance-local texel) pairs. slots is the whole payload
 * buffer (u32[P][4], RGB f32 bits + count) and is updated in place. */
int oracle_trace_texels(void* scene, const OracleLighting* lighting,
                        uint8_t* slots, uint32_t payload_count,
                        const uint32_t* face_infos, uint32_t face_count,
                        const uint32_t* instance_infos,
                        const uint32_t* side_infos, uint32_t instance_count,
                        const uint32_t* units, int unit_count,
                        uint32_t iteration, uint32_t samples_per_texel,
                        uint32_t max_bounces, int reset, int precision,
                        int threads, OracleRayCounts* counts);

/* Mesh Colors resolve of the listed pixels (mesh_colors_resolve.slang:29-73;
 * packed = 1: the frozen RGB9E5 resolve, mesh_colors_frozen_resolve.slang:
 * 93-135). colors: 16-byte slots or RGB9E5 words. out f32[N][4]. */
int oracle_resolve_mesh_colors(void* scene, const OracleLighting* lighting,
                               const OracleCamera* camera, uint32_t width, uint32_t height,
                               const uint32_t* pixels, int pixel_count,
                               const uint32_t* face_infos, const uint32_t* instance_infos,
                               const uint32_t* side_infos, uint32_t instance_count,
                               const void* colors, int packed, int precision, int threads,
                               float* out);

/* Options of the surface-probe resolve (the layout of NanProbeResolveOptions,
 * host pointers). */
typedef struct OracleProbeResolveOptions {
    uint32_t debug_view;
    uint32_t min_gather_count;
    uint32_t use_vertex_fallback;
    uint32_t use_vertex_lighting;
    uint32_t use_radial_visibility;
    uint32_t frame_index;
    float max_density_multiplier;
    float vertex_lighting_rgbm_range;
    const uint32_t* vertex_lighting_rgbm;
    const float* vertex_lighting_target;
    const uint32_t* vertex_lighting_triangle_map;
    const uint32_t* vertex_lighting_instance_offsets;
    uint32_t vertex_lighting_vertex_count;
    uint32_t vertex_lighting_triangle_record_count;
} OracleProbeResolveOptions;

/* Surface-probe resolve (surface_probe_resolve.slang:325-472) of the listed
 * pixels u32[N][2] into out f32[N][4]; returns 4 when a layout index was out
 * of range (that access skipped), else 0. */
int oracle_resolve_probes(void* scene, const OracleLighting* lighting, const OracleCamera* camera,
                          uint32_t width, uint32_t height, const uint32_t* pixels, int pixel_count,
                          const float* probes, uint32_t probe_count, const uint32_t* nodes,
                          uint32_t node_count, const float* instances, uint32_t instance_count,
                          const uint32_t* triangle_vertex_probes, uint32_t triangle_vertex_probe_count,
                          const float* values, const uint32_t* sample_counts, const uint32_t* self_hits,
                          const uint32_t* radial, const OracleProbeResolveOptions* options, int threads,
                          float* out);

/* Weighted sample elimination (surface_probes.py:897-985), one candidate at
 * a time with a heap, for each contiguous candidate set: keep u8[N] marks
 * the survivors, poisson_radii f32[S] gets d_max / 2, order (optional
 * u32[N]) the eliminated candidates of each set in removal order from the
 * set's first slot. Contributions are rounded to 2^-50 units as in
 * nan_wse_eliminate. relative_densities (nullable, f32[N]) selects the
 * adaptive elimination: per-candidate d_max / sqrt(density), the Poisson
 * radius the base one. */
int oracle_wse_eliminate(const float* positions, const float* normals, const float* relative_densities,
                         const uint32_t* set_offsets, uint32_t set_count, const uint32_t* output_counts,
                         const float* surface_areas, float normal_cosine_threshold, float plane_distance_scale,
                         uint8_t* keep, float* poisson_radii, uint32_t* order, int threads);

/* Deficit repair (deficit_repair_python, surface_probe_sampler.py:990-1103),
 * one candidate at a time, with the float32 gather weights of the GPU
 * version. selected gets the chosen candidates in choice order. Returns 8
 * when an audit names an instance out of range. */
int oracle_deficit_repair(const float* base_p, const float* base_n, const uint32_t* base_i, uint32_t base_count,
                          const float* cand_p, const float* cand_n, const uint32_t* cand_i, uint32_t cand_count,
                          const float* audit_p, const float* audit_n, const uint32_t* audit_i, uint32_t audit_count,
                          const float* radii, uint32_t instance_count, uint32_t min_gather, uint32_t max_repair,
                          float normal_cosine_threshold, float eps, uint32_t* selected, uint32_t* repair_count,
                          uint32_t* counts_before, uint32_t* counts_after, float* sums_before, float* sums_after,
                          float* ess_before, float* ess_after);

/* Support estimate (estimate_support_python, surface_probe_sampler.py:
 * 1179-1260) with the float32 kernel of the GPU version; returns 8 when an
 * instance index is out of range. */
/* Audit/repair candidate filter (surface_probe_filter_audit_repair_candidates):
 * audit (u32[N]) the kept audit points, repair (u32[N]) the kept repair
 * candidates, both ascending. cs / bs per point set indices (nullable: one
 * set), cell_sizes f64[set_count]. Returns 1 for a selected base index out of
 * range, 2 for a set index out of range. */
int oracle_filter_audit_repair(const float* cp, const float* cn, const uint32_t* cs, uint32_t n, const float* bp,
                               const float* bn, const uint32_t* bs, uint32_t base_count, const uint32_t* selected,
                               uint32_t m, uint32_t set_count, const double* cell_sizes, double ncos,
                               uint32_t* audit, uint32_t* audit_count, uint32_t* repair, uint32_t* repair_count);
int oracle_estimate_support(const float* ref_p, const float* ref_n, const uint32_t* ref_i, const float* area,
                            uint32_t ref_count, const float* q_p, const float* q_n, const uint32_t* q_i,
                            uint32_t q_count, const float* radii, uint32_t instance_count,
                            float normal_cosine_threshold, float eps, float max_density, float* support_f,
                            float* density_m);

/* e^x and log2 x of the kernels' own float implementations (nan_exp,
 * nan_log2), for tests against the C library. */
float own_exp(float x);
float own_log2(float x);

/* One pass of the Mesh Colors one-ring surface filter over every texel of
 * every instance (mesh_colors_surface_filter.slang:1-253): source and
 * destination are 16-byte slot buffers. */
int oracle_filter_mesh_colors(const uint32_t* face_infos, const uint32_t* instance_infos,
                              const uint32_t* side_infos, uint32_t instance_count,
                              const uint32_t* adjacency, const float* face_normals,
                              const uint8_t* source, uint8_t* destination,
                              float neighbor_weight, float normal_sigma_radians, int threads);

/* PRT L2 field baker (surface_probe_prt_baker.slang:169-371) for the listed
 * probe indices: values f32[N][9][3], static_source f32[N][3] and the
 * baker's counts, self hits and radial moments, updated in place. */
int oracle_trace_probes_prt(void* scene, const OracleLighting* lighting, float* values,
                            uint32_t* sample_counts, uint32_t* self_hits, uint32_t* radial,
                            float* static_source, const uint8_t* probes, uint32_t probe_count,
                            const uint8_t* probe_instances, const uint32_t* units, int unit_count,
                            uint32_t iteration, uint32_t samples_per_probe, uint32_t max_bounces,
                            int reset, int precision, int threads);

/* PRT evaluation (surface_probe_prt_evaluate.slang:20-103): the SH L2
 * projection of the escape radiance, sh f32[9][4], and the per-probe
 * evaluation max(static + sum_c values[c] * sh[c], 0) into out f32[N][3]. */
void oracle_prt_project_lighting(const OracleLighting* lighting, uint32_t sample_count, float* sh);
void oracle_prt_evaluate(const float* values, const uint32_t* sample_counts, const float* static_source,
                         const float* sh, float* out, uint32_t* out_counts, uint32_t probe_count);

/* Area-light table of the screen tracer's NEE option (lighting flag bit 1),
 * the layout of nan_ctx_set_area_lights. */
void oracle_scene_set_area_lights(void* scene, const float* lights, int count, float power);

/* Irradiance at surface points: the texel estimator
 * (estimate_surface_irradiance, texture_space_path_tracer.slang:86-117) at
 * points f32[N][4] = (b1, b2, instance bits, primitive bits | back << 31),
 * with view = the flat normal (negated for back), RNG(index, 0xFFFFFFFF,
 * iteration * n). out f32[N][4] = (E rgb, 0), or (0, 0, 0, -1) where the
 * instance is ~0 (no point). flags bit 0: leave out the direct sun
 * irradiance term (its two RNG draws are still taken). The points pass of
 * the learned cache's training, checked bit for bit. */
int oracle_trace_points(void* scene, const OracleLighting* lighting, const float* points, int count,
                        uint32_t iteration, uint32_t samples, uint32_t max_bounces, uint32_t flags,
                        float* out, int precision, int threads, OracleRayCounts* counts);

/* Surface-probe irradiance baker (surface_probe_path_tracer.slang:280-315)
 * for the listed probe indices. Buffers are updated in place. */
int oracle_trace_probes(void* scene, const OracleLighting* lighting,
                        float* values, uint32_t* sample_counts,
                        uint32_t* self_hits, uint32_t* radial,
                        const uint8_t* probes, uint32_t probe_count,
                        const uint8_t* probe_instances,
                        uint32_t probe_instance_count,
                        const uint32_t* units, int unit_count,
                        uint32_t iteration, uint32_t samples_per_probe,
                        uint32_t max_bounces, int reset, int precision,
                        int threads, OracleRayCounts* counts);

/* The same with one RNG stream per sample, RNG(probe, instance, iteration * n
 * + k): the batched baker's independent-sample mode. */
int oracle_trace_probes_independent(void* scene, const OracleLighting* lighting,
                                    float* values, uint32_t* sample_counts,
                                    uint32_t* self_hits, uint32_t* radial,
                                    const uint8_t* probes, uint32_t probe_count,
                                    const uint8_t* probe_instances,
                                    uint32_t probe_instance_count,
                                    const uint32_t* units, int unit_count,
                                    uint32_t iteration, uint32_t samples_per_probe,
                                    uint32_t max_bounces, int reset, int precision,
                                    int threads, OracleRayCounts* counts);

#ifdef __cplusplus
}
#endif

#endif
