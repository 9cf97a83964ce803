/* nan_b200.h -- C ABI of libnan_b200.so, the B200 (sm_100a) path-integration
 * library: GPU BVH construction and traversal, Lambert path integration with
 * sun next-event estimation, and irradiance accumulation into screen pixels,
 * Mesh Colors texel slots and surface-probe sites.
 *
 * Conventions
 *   - Every call returns an int status (NAN_OK == 0). On failure
 *     nan_last_error() (thread-local) describes the error.
 *   - Every buffer argument is a DEVICE pointer owned by the caller, except
 *     the small parameter structs (NanLighting, NanCamera, NanSceneDesc,
 *     NanMeshColorsDesc, ...), which are read from host memory during the
 *     call. Record layouts are the reference's (4-byte little-endian words).
 *   - Work is enqueued on the given cudaStream_t (passed as void*; NULL is
 *     the legacy default stream). Calls return before the GPU finishes,
 *     except where noted ("synchronises").
 *   - Trace calls allocate nothing. nan_scene_build allocates the BVH it
 *     owns inside the context.
 *   - A context is not re-entrant from several host threads at once.
 *
 * The reference interfaces each call replaces are cited as path:line inside
 * the reference project (WeakKnight/Nan).
 */
#ifndef NAN_B200_H
#define NAN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NAN_B200_API __attribute__((visibility("default")))

enum NanStatus {
    NAN_OK = 0,
    NAN_ERR_INVALID_ARGUMENT = 1,
    NAN_ERR_OUT_OF_MEMORY = 2,
    NAN_ERR_LIMIT = 3,       /* a device loop or stack cap was hit */
    NAN_ERR_CUDA = 4,
    NAN_ERR_NO_SCENE = 5,
};

typedef struct NanContext NanContext;

/* Sun + sky lighting of the scene. Replaces Scene.bind()'s directional light
 * and sky bindings (scene.py:1338-1382, scene.slang:6-17); the sky-view LUT
 * (scene.slang:469-518) is reduced to a constant radiance and the sun
 * transmittance LUT (scene.slang:997-1009) to a constant RGB factor. */
typedef struct NanLighting {
    float sun_direction[3];     /* unit vector toward the sun */
    float sun_cos_half_angle;   /* cos of the sun disk's half apex angle */
    float sun_color[3];
    float sun_intensity;        /* outer-space illuminance = color * intensity */
    float sun_transmittance[3]; /* ground-level factor (LUT stand-in) */
    float ray_t_max;            /* t_max of bounce and shadow rays (Ray default 1000) */
    float sky_radiance[3];      /* constant sky radiance on misses */
    uint32_t flags;             /* bit 0: add the sun disk on primary misses; bit 1: screen
                                   tracer NEE toward the context's area lights with MIS
                                   (nan_ctx_set_area_lights; not in the reference) */
    /* Sky-view LUT (sample_sky_lut, scene.slang:469-518). Null: every miss sees the
     * constant sky_radiance. Otherwise device memory f32[height][width][4] (RGBA32F, the
     * reference's 200x200 sky-view LUT): a miss in direction d reads it bilinearly
     * (wrapped addressing) at u = azimuth / 2pi + 1/2 and the LUT's altitude mapping,
     * times sun_color * sun_intensity. */
    const float* sky_view_lut;
    uint32_t sky_view_width;
    uint32_t sky_view_height;
    float sky_view_up[3];        /* unit vector from the planet's centre to the view position */
    float sky_view_horizon_angle; /* acos(sqrt(h^2 - R^2) / h) - pi/2 at view height h, ground
                                     radius R (the reference's atmosphere: h = 6.3602, R = 6.36) */
} NanLighting;

/* Pinhole camera: the fields compute_ray_pinhole reads (camera.slang:173-236,
 * bound by Camera.bind camera.py:98-115). */
typedef struct NanCamera {
    float position[3];
    float jitter_x;
    float image_u[3];
    float jitter_y;
    float image_v[3];
    float near_clip;
    float image_w[3];
    float far_clip;
} NanCamera;

/* Scene buffers in the reference's layouts (scene.py:84-108, 386-436). */
typedef struct NanSceneDesc {
    const float* vertices;            /* f32[V][8]: position, normal, uv */
    uint32_t vertex_count;
    const uint32_t* indices;          /* u32[T][3], mesh-local */
    uint32_t index_triangle_count;    /* T */
    const uint32_t* mesh_descs;       /* u32[M][4]: vtx count, idx count, vtx off, idx off */
    uint32_t mesh_count;
    const uint32_t* instance_descs;   /* u32[I][4]: mesh, material, transform, flags */
    uint32_t instance_count;
    const float* transforms;          /* f32[X][16] row-major */
    const float* inverse_transposes;  /* f32[X][16] */
    uint32_t transform_count;
    const float* materials;           /* f32[N][8]: base rgb, flags(u32), emissive rgb, pad */
    uint32_t material_count;
} NanSceneDesc;

typedef struct NanSceneInfo {
    uint32_t triangle_count;   /* world triangles after flattening instances */
    uint32_t node_count;       /* BVH interior nodes */
    uint32_t leaf_count;
    uint32_t max_depth;
    uint64_t device_bytes;     /* BVH + triangle storage owned by the context */
    double build_ms;           /* device time of the last build */
    double sah_cost;           /* SAH cost of the BVH (C_trav = C_int = 1) */
} NanSceneInfo;

/* Mesh Colors layout buffers (mesh_colors.py:82-119, 310-337). */
typedef struct NanMeshColorsDesc {
    const uint32_t* face_infos;      /* u32[F][2]: address, resolution */
    uint32_t face_count;
    const uint32_t* instance_infos;  /* u32[I][4]: face off, face count, texel off, texel count */
    const uint32_t* side_infos;      /* u32[I][2]: back texel offset, flags */
    uint32_t instance_count;
    const uint32_t* surface_prefix;  /* u32[I+1]: exclusive prefix of texel_count */
    uint32_t total_surface_texels;
    uint32_t payload_count;          /* slots in the payload buffer */
    float* compensation;             /* optional f32[P][4] Kahan terms of the running means;
                                        NULL = the reference's plain lerp (bit-exact parity) */
} NanMeshColorsDesc;

/* Surface-probe layout (SurfaceProbeLayout, surface_probes.py:1490-1535, as
 * uploaded by surface_probe_resources.py:24-89): probe records 48 B
 * {position_radius, normal_side (xyz normal, w support), meta u32x4}; octree
 * nodes u32[M][4] (child_base, child_mask, probe_start, probe_count);
 * instance records 48 B {root_center_extent, offsets u32x4 (node offset, node
 * count, probe offset, probe count), params (kernel radius, normal cosine
 * threshold, plane sigma, triangle-map offset bits)}, one per scene instance;
 * triangle -> vertex-anchor probe map u32[R][4] (two records per triangle,
 * front and back; bit 0 of w marks a valid record). */
typedef struct NanProbeLayoutDesc {
    const uint8_t* probes;
    uint32_t probe_count;
    uint32_t node_count;
    const uint32_t* nodes;
    const uint8_t* instances;
    uint32_t instance_count;
    uint32_t triangle_vertex_probe_count;
    const uint32_t* triangle_vertex_probes;
} NanProbeLayoutDesc;

/* SurfaceProbeResolve.execute options (surface_probe_resolve.py:46-112).
 * Vertex lighting (SurfaceProbeVertexLighting's outputs) is optional:
 * vertex_lighting_rgbm = NULL means not built; otherwise rgbm u32[V], target
 * f32[V][4], triangle map u32[R][4] (xyz vertices, w valid) and instance
 * offsets u32[I][2] with one entry per probe-layout instance. */
typedef struct NanProbeResolveOptions {
    uint32_t debug_view;             /* 0 beauty, 1 gather count, 2 support, 3 density,
                                        4 reconstruction confidence, 5 self-hit rate,
                                        6 vertex lighting, 7 vertex-lighting confidence */
    uint32_t min_gather_count;       /* clamped to 1..32 */
    uint32_t use_vertex_fallback;
    uint32_t use_vertex_lighting;
    uint32_t use_radial_visibility;
    uint32_t frame_index;            /* RNG(pixel, frame) of the real-time sun sample */
    float max_density_multiplier;
    float vertex_lighting_rgbm_range;
    const uint32_t* vertex_lighting_rgbm;
    const float* vertex_lighting_target;
    const uint32_t* vertex_lighting_triangle_map;
    const uint32_t* vertex_lighting_instance_offsets;
    uint32_t vertex_lighting_vertex_count;
    uint32_t vertex_lighting_triangle_record_count;
} NanProbeResolveOptions;

/* Options of the weighted sample elimination (SurfaceProbeWSEOptions,
 * surface_probe_sampler.h:15-20, less the surface area, which is per set). */
typedef struct NanWseOptions {
    float normal_cosine_threshold;  /* 0.5 in the reference */
    float plane_distance_scale;     /* 0.35 in the reference */
} NanWseOptions;

/* Options of the deficit repair (SurfaceProbeRepairOptions,
 * surface_probe_sampler.h:50-56). */
typedef struct NanRepairOptions {
    uint32_t min_gather_count;     /* 1..32; 4 in the reference */
    uint32_t max_repair_count;     /* budget of chosen candidates */
    float normal_cosine_threshold; /* full-confidence cosine of the soft normal gate */
    float weight_epsilon;          /* 1e-6 in the reference */
} NanRepairOptions;

/* Options of the support estimate (SurfaceProbeSupportOptions,
 * surface_probe_sampler.h:87-92). */
typedef struct NanSupportOptions {
    float normal_cosine_threshold; /* full-confidence cosine of the soft normal gate (0.5) */
    float weight_epsilon;          /* kernel values at or below are 0 (1e-6) */
    float max_density_multiplier;  /* M (8) */
    float reserved;
} NanSupportOptions;

/* Execution choices of a context. The defaults (all zero) are the wavefront
 * integrator with occupancy-sized persistent traversal grids, as many paths
 * in flight as the reserved scratch holds, and the binned-SAH BVH builder. */
typedef struct NanTuning {
    uint32_t integrator;           /* 0: wavefront; 1: one thread per pixel/texel/probe */
    uint32_t trace_blocks_per_sm;  /* persistent traversal blocks per SM, 0 = occupancy limit */
    uint32_t max_paths_in_flight;  /* wavefront chunk size, 0 = as many as the scratch holds */
    uint32_t bvh_builder;          /* nan_scene_build: 0 = binned SAH, 1 = LBVH, 2 = PLOC; 0 and 2
                                      collapse subtrees of up to 3 triangles into leaves by SAH */
    uint32_t bvh_width;            /* traversed nodes: 0 or 2 = binary, 8 = compressed 8-wide (SAH or PLOC builds) */
    uint32_t kernel_timing;        /* 1: record CUDA events around each wavefront stage launch on the
                                      launching stream (read with nan_ctx_read_kernel_times); not for
                                      use under stream capture */
    uint32_t ray_order;            /* wavefront extend queue: 0 = path order, 1 = regrouped by ray
                                      direction octant before each extend launch */
    uint32_t traversal;            /* wavefront traversal over binary nodes, same results in every
                                      form: 0 = a warp takes 32 rays and walks until all have ended;
                                      1-4 = idle lanes are refilled from the queue;
                                      5 = stack top in shared memory;
                                      6 = speculative while-while walk (a lane parks its
                                      first leaf until every lane holds one) */
} NanTuning;

/* Device time of the wavefront stages since the last reset, from CUDA events
 * recorded on the launching stream while NanTuning.kernel_timing is 1. */
typedef struct NanKernelTimes {
    double extend_ms;          /* k_wf_extend: closest-hit traversal */
    double shadow_ms;          /* k_wf_shadow: any-hit traversal */
    double stage_ms;           /* generate / shade / finalize kernels */
    uint64_t extend_launches;
    uint64_t shadow_launches;
    uint64_t stage_launches;
} NanKernelTimes;

/* Device-side counters accumulated by the trace calls. */
typedef struct NanCounters {
    uint64_t extend_rays;   /* closest-hit rays */
    uint64_t shadow_rays;   /* any-hit rays */
    uint64_t units;         /* pixels / texels / probes processed */
    uint64_t paths;         /* light paths started */
} NanCounters;

NAN_B200_API const char* nan_last_error(void);
NAN_B200_API int nan_version(void);

/* Context: device ordinal, device status word and counters. */
NAN_B200_API int nan_ctx_create(int device, NanContext** out_ctx);
NAN_B200_API int nan_ctx_destroy(NanContext* ctx);
/* Synchronises `stream`, then reads (and clears) the device status word.
 * Returns NAN_ERR_LIMIT if a kernel hit its traversal-stack cap. */
NAN_B200_API int nan_ctx_check(NanContext* ctx, void* stream);
/* Synchronises `stream`, copies the counters, optionally zeroes them. */
NAN_B200_API int nan_ctx_read_counters(NanContext* ctx, NanCounters* out, int reset,
                                       void* stream);
/* Scratch arena for the wavefront integrator: path state and ray queues,
 * nan_wavefront_bytes_per_path() bytes per path in flight. Allocates (grow
 * only; never inside a trace call). Synchronises the device. */
NAN_B200_API int nan_ctx_reserve(NanContext* ctx, uint64_t scratch_bytes);
NAN_B200_API uint64_t nan_wavefront_bytes_per_path(void);
/* Emissive triangles for area-light NEE (lighting flag bit 1). lights is a
 * caller-owned device table f32[count][16]: v0 xyz, cdf (inclusive, last =
 * 1); e1 = v1 - v0, area; e2 = v2 - v0, luminance (0.2126 r + 0.7152 g +
 * 0.0722 b); emission rgb, 0. power = sum of area * luminance. It must list
 * every emissive triangle of the scene and stay alive while traced. No
 * counterpart in the reference (its path tracer reaches emitters by BSDF
 * sampling only). count 0 clears the table. */
NAN_B200_API int nan_ctx_set_area_lights(NanContext* ctx, const float* lights, uint32_t count, float power);
/* Select the integrator form and its launch shapes (see NanTuning). */
NAN_B200_API int nan_ctx_configure(NanContext* ctx, const NanTuning* tuning);
/* Number of kernels this context has launched. */
NAN_B200_API uint64_t nan_ctx_launch_count(NanContext* ctx);
/* Waits for the recorded stage events and sums their durations into `out`;
 * reset = 1 clears the sums. No counterpart in the reference (measurement). */
NAN_B200_API int nan_ctx_read_kernel_times(NanContext* ctx, NanKernelTimes* out, int reset);

/* Flatten the instances to world space and build the BVH on the GPU.
 * Replaces Scene.__init__'s buffer packing + build_blas/build_tlas
 * (scene.py:386-533). The scene buffers must stay alive and unchanged while
 * the context traces them (shading reads them in place). Synchronises. */
NAN_B200_API int nan_scene_build(NanContext* ctx, const NanSceneDesc* desc, void* stream);
/* nan_scene_build for callers that cannot allocate device memory: code that
 * runs inside another framework's memory pool, or a real-time loop that must
 * never call cudaMalloc/cudaFree. No counterpart in the reference (its BVH is
 * built by the graphics driver).
 *
 * It allocates nothing. Build scratch comes from one fixed 64 MiB array in
 * device memory (a file-scope __device__ array: every GPU that loads the
 * library holds it until the process exits), enough for scenes of about 300k
 * triangles; larger scenes return NAN_ERR_LIMIT. The tree is always an LBVH
 * (Karras 2012) with binary nodes: the context's NanTuning bvh_builder and
 * bvh_width are ignored. Hits equal nan_scene_build's (the closest hit is
 * chosen by (t, flat index) in any tree), but the LBVH has a higher SAH cost
 * than the default binned-SAH tree, so tracing it is slower. The BVH is written into the
 * caller's buffers, which must stay alive while the context traces them:
 *   out_nodes  >= 64 * max(T - 1, 1) bytes, 16-byte aligned
 *   out_tris   >= 48 * T bytes, 16-byte aligned
 *   out_refs   >= 8 * T bytes, 8-byte aligned
 * where T is the number of triangles over all instances. The context must
 * not hold a BVH from nan_scene_build. The first call on a device looks up
 * the scratch array's device address (cudaGetSymbolAddress); make that first
 * call before any stream capture. That address is cached for the process and
 * does not survive cudaDeviceReset on the device. Every call shares the scratch array, so
 * calls that overlap on the GPU (other streams, other host threads) race.
 * Synchronises `stream`. */
NAN_B200_API int nan_scene_build_noalloc(NanContext* ctx, const NanSceneDesc* desc, float* out_nodes,
                                         uint64_t nodes_bytes, float* out_tris, uint64_t tris_bytes,
                                         uint32_t* out_refs, uint64_t refs_bytes, void* stream);
NAN_B200_API int nan_scene_info(NanContext* ctx, NanSceneInfo* out);
/* World triangles in flat (instance-major) order, f32[T][9]; out may be a
 * device pointer of at least 36*T bytes. */
NAN_B200_API int nan_scene_world_triangles(NanContext* ctx, float* out, void* stream);

/* Closest hit per ray (Scene.intersect with t, scene.slang:1071-1124).
 * rays f32[N][8]: origin, t_min, dir, t_max.
 * hit_ids u32[N][4]: valid, instance, primitive, flat triangle index;
 * hit_tb f32[N][3]: t, bary.x, bary.y. */
NAN_B200_API int nan_intersect(NanContext* ctx, const float* rays, uint32_t count,
                               uint32_t* hit_ids, float* hit_tb, void* stream);
/* Any hit per ray: visibility 1.0 when nothing is hit in [t_min, t_max]
 * (Scene.get_visibility, scene.slang:1126-1172). */
NAN_B200_API int nan_occluded(NanContext* ctx, const float* rays, uint32_t count,
                              float* visibility, void* stream);

/* Most rays per sample of the PMR visibility caster below. */
#define NAN_VISIBILITY_MAX_RAYS 1024u
/* Ray table of the reference's PMR visibility caster, make_ray_projections
 * (vertex_baker/cpp/tinybvh_visibility.cpp:81-101, SH at :52-77): ray r of R
 * has u0 = r / R, u1 = bit-reversed r * 2^-32, phi = 2 pi u0,
 * cos theta = 1 - 2 u1, direction (cos phi sin theta, cos theta,
 * sin phi sin theta), and the real SH basis of bands 0-3 times 4 pi / R.
 * Writes host memory f32[R][20]: direction xyz, 0, the 16 weighted SH
 * values. Host only (the C library's cosf/sinf, as the caster uses);
 * 1 <= R <= NAN_VISIBILITY_MAX_RAYS. */
NAN_B200_API int nan_visibility_ray_table(uint32_t ray_count, float* host_table);
/* GPU form of the reference's PMR visibility caster,
 * vbake_pmr_visibility_sh_tinybvh (vertex_baker/cpp/vertex_baking_utils.h:73-90,
 * tinybvh_visibility.cpp:145-230), and of its hardware twin
 * HWRTPMRVisibilitySHSampler.sample (vertex_baker/hwrt_visibility_baker.py:145-240).
 * For every sample, the table's rays start at position + normalize(normal) *
 * self_bias (a zero or non-finite normal: direction (0,0,1) and the origin
 * moved one float towards each ray instead) and are tested for any hit in
 * [0, max_distance] (max_distance <= 0 or non-finite: 1e30; self_bias below
 * 0: 0) against the context's scene. The unoccluded rays' weighted SH values
 * are summed in the caster's order (64-ray batches), into out_sh16
 * f32[S][16]; out_visible_counts u32[S] (may be null) gets the number of
 * unoccluded rays. Device pointers: sample_positions/normals f32[S][3],
 * ray_table the table above copied to the device. The geometry is the built
 * scene (all instances, world space) rather than a positions/indices pair,
 * and the caster's thread count and BVH layout arguments have no meaning
 * here. Non-finite sample inputs are not checked (the caster rejects them). */
NAN_B200_API int nan_visibility_sh16(NanContext* ctx, const float* sample_positions, const float* sample_normals,
                                     uint32_t sample_count, const float* ray_table, uint32_t ray_count,
                                     float max_distance, float self_bias, float* out_sh16,
                                     uint32_t* out_visible_counts, void* stream);

/* One 1-spp frame of the screen path tracer into out_rgba f32[H][W][4]
 * (PathTracer.execute, path_tracer.py:21-40; path_tracer.slang:40-130).
 * max_vertices is the reference's hard-coded 5 (path_tracer.slang:42). */
NAN_B200_API int nan_trace_screen(NanContext* ctx, float* out_rgba, uint32_t width,
                                  uint32_t height, uint32_t frame, uint32_t max_vertices,
                                  const NanCamera* camera, const NanLighting* lighting,
                                  void* stream);

/* Running average of frames (Accumulator.execute, accumulator.py:32-58;
 * accumulator.slang:9-19). All buffers f32[H][W][4]. */
NAN_B200_API int nan_accumulate(NanContext* ctx, const float* input, float* output,
                                float* history, uint32_t width, uint32_t height, int reset,
                                void* stream);

/* One iteration of the texture-space tracer over surface texels
 * [texel_begin, texel_end) of the layout, all instances in ONE launch
 * (TextureSpacePathTracer.execute, texture_space_path_tracer.py:33-58;
 * texture_space_path_tracer.slang:57-216). slots u8[P][16]: RGB f32 + u32
 * count, updated in place as a running mean. */
NAN_B200_API int nan_trace_texels(NanContext* ctx, const NanMeshColorsDesc* layout,
                                  uint8_t* slots, uint32_t iteration,
                                  uint32_t samples_per_texel, uint32_t max_bounces, int reset,
                                  const NanLighting* lighting, uint32_t texel_begin,
                                  uint32_t texel_end, void* stream);

/* One iteration of the surface-probe irradiance baker over probes
 * [probe_begin, probe_end) (SurfaceProbeDiffuseIrradianceBaker.execute,
 * surface_probe_path_tracer.py:49-83; surface_probe_path_tracer.slang:47-315).
 * values f32[N][3], sample_counts u32[N], self_hits u32[N],
 * radial u32[N][16] (RG16F moments), probes u8[N][48],
 * probe_instances u8[I][48]; compensation: optional f32[N][4] Kahan terms of
 * the running means (NULL = the reference's plain lerp). */
NAN_B200_API int nan_trace_probes(NanContext* ctx, float* values, uint32_t* sample_counts,
                                  uint32_t* self_hits, uint32_t* radial,
                                  const uint8_t* probes, uint32_t probe_count,
                                  const uint8_t* probe_instances,
                                  uint32_t probe_instance_count, uint32_t iteration,
                                  uint32_t samples_per_probe, uint32_t max_bounces, int reset,
                                  const NanLighting* lighting, uint32_t probe_begin,
                                  uint32_t probe_end, float* compensation, void* stream);

/* MeshColorsResolve.execute / execute_frozen (mesh_colors_resolve.py:8-73;
 * mesh_colors_resolve.slang:29-73, mesh_colors_frozen_resolve.slang:93-135):
 * one primary ray per pixel, the hit triangle's lattice colours interpolated
 * (mesh_colors.slang:365-426) and shaded as emissive + albedo / pi *
 * irradiance into out f32[H][W][4]. colors is the 16-byte slot buffer
 * (packed = 0) or the RGB9E5 words of nan_pack_rgb9e5 (packed = 1); the
 * layout's face, instance and side buffers are read. */
NAN_B200_API int nan_resolve_mesh_colors(NanContext* ctx, const NanMeshColorsDesc* layout,
                                         const void* colors, int packed, float* out, uint32_t width,
                                         uint32_t height, const NanCamera* camera,
                                         const NanLighting* lighting, void* stream);

/* SurfaceProbeResolve.execute (surface_probe_resolve.py:16-112;
 * surface_probe_resolve.slang:325-472): one primary ray per pixel; the hit
 * instance's probes are gathered from its point octree (up to 96 candidates
 * weighted by distance, plane distance and normal, times the radial
 * Chebyshev visibility prior, the 32 strongest kept, a 2R fallback merged
 * when the gather's effective sample size is below min_gather_count) and
 * reconstructed from the irradiance field values f32[N][3] with its
 * sample_counts, self_hits and radial moments; out f32[H][W][4]. */
NAN_B200_API int nan_resolve_probes(NanContext* ctx, const NanProbeLayoutDesc* layout, const float* values,
                                    const uint32_t* sample_counts, const uint32_t* self_hits,
                                    const uint32_t* radial, const NanProbeResolveOptions* options, float* out,
                                    uint32_t width, uint32_t height, const NanCamera* camera,
                                    const NanLighting* lighting, void* stream);

/* MeshColorsSurfaceFilter.execute (mesh_colors_surface_filter.py:95-130;
 * mesh_colors_surface_filter.slang:1-253): one pass of the one-ring,
 * normal-aware filter from source slots to destination slots (distinct
 * buffers; counts are copied). adjacency u32[F][4]: per face the packed edges
 * 0..2 ((mesh-local adjacent face << 3) | adjacent edge | flip << 2, ~0 for
 * none); face_normals f32[F][4] in world space; neighbor_weight =
 * exp(-0.5 / spatial_sigma^2); normal_sigma in radians. All instances in one
 * launch. */
NAN_B200_API int nan_filter_mesh_colors(NanContext* ctx, const NanMeshColorsDesc* layout,
                                        const uint32_t* adjacency, const float* face_normals,
                                        const uint8_t* source, uint8_t* destination,
                                        float neighbor_weight, float normal_sigma_radians,
                                        void* stream);

/* SurfaceProbePrtBaker.execute (surface_probe_prt.py:62-128;
 * surface_probe_prt_baker.slang:169-371): one iteration of the PRT L2 field
 * baker over probes [probe_begin, probe_end). values f32[N][9][3] (SH L2
 * transport), static_source f32[N][3] (emission and sun along the paths),
 * sample_counts u32[N], self_hits u32[N], radial u32[N][16]. */
NAN_B200_API int nan_trace_probes_prt(NanContext* ctx, float* values, uint32_t* sample_counts,
                                      uint32_t* self_hits, uint32_t* radial, float* static_source,
                                      const uint8_t* probes, uint32_t probe_count,
                                      const uint8_t* probe_instances, uint32_t probe_instance_count,
                                      uint32_t iteration, uint32_t samples_per_probe,
                                      uint32_t max_bounces, int reset, const NanLighting* lighting,
                                      uint32_t probe_begin, uint32_t probe_end, void* stream);

/* SurfaceProbePrtEvaluator.execute (surface_probe_prt.py:131-248;
 * surface_probe_prt_evaluate.slang:20-103), first pass: the lighting's escape
 * radiance projected on SH L2 with sample_count quasi-random sphere
 * directions; lighting_sh f32[9][4] (rgb, 0), 16-byte aligned. */
NAN_B200_API int nan_prt_project_lighting(NanContext* ctx, float* lighting_sh, uint32_t sample_count,
                                          const NanLighting* lighting, void* stream);
/* Second pass: out_values f32[N][3] = max(static_source + sum_c values[c] *
 * lighting_sh[c], 0) (static only where sample_counts is 0); out_sample_counts
 * copies sample_counts. */
NAN_B200_API int nan_prt_evaluate(NanContext* ctx, const float* values, const uint32_t* sample_counts,
                                  const float* static_source, const float* lighting_sh, float* out_values,
                                  uint32_t* out_sample_counts, uint32_t probe_count, void* stream);

/* Weighted sample elimination of surface-probe candidates
 * (weighted_sample_elimination, surface_probes.py:897-985 and 1091-1123;
 * surface_probe_wse_eliminate, surface_probe_sampler.h:120-130) for
 * set_count candidate sets in one call. positions and normals are device
 * f32[N][3] with the sets contiguous: set k is [set_offsets[k],
 * set_offsets[k+1]). set_offsets (S+1), output_counts and surface_areas (S)
 * are host arrays. keep (device u8[N]) gets 1 for the survivors: per set the
 * output_count candidates (clamped to 1..count) that remain when, one at a
 * time, the candidate of largest weight (lowest index on ties) is removed.
 * poisson_radii (host f32[S], optional) gets d_max / 2 per set (the spacing
 * sqrt(area / count) when nothing is eliminated); rounds (optional) the
 * number of parallel elimination rounds. Contribution weights are rounded to
 * units of 2^-50 so the sums are exact (NAN_ERR_LIMIT past 8000 neighbours). Allocates scratch on the stream and
 * synchronizes it. */
NAN_B200_API int nan_wse_eliminate(NanContext* ctx, const float* positions, const float* normals,
                                   const uint32_t* set_offsets, uint32_t set_count, const uint32_t* output_counts,
                                   const float* surface_areas, const NanWseOptions* options, uint8_t* keep,
                                   float* poisson_radii, uint32_t* rounds, void* stream);

/* The adaptive elimination (_adaptive_weighted_sample_elimination_python,
 * surface_probes.py:988-1088 and 1126-1166; surface_probe_wse_eliminate_adaptive,
 * surface_probe_sampler.h:120-223), same arguments plus relative_densities
 * (device f32[N], finite and positive): candidate i is compared with its
 * neighbours within its own d_max_i = max(d_max / sqrt(density_i), 1e-6)
 * (plane limit max(d_max_i x plane_distance_scale, 1e-8)), so dense regions
 * keep more candidates. poisson_radii gets the base radius
 * sqrt(area / (2 sqrt(3) output_count)) per set. The reference's
 * partition_masses only shape its CPU partitioning and have no counterpart. */
NAN_B200_API int nan_wse_eliminate_adaptive(NanContext* ctx, const float* positions, const float* normals,
                                            const float* relative_densities, const uint32_t* set_offsets,
                                            uint32_t set_count, const uint32_t* output_counts,
                                            const float* surface_areas, const NanWseOptions* options, uint8_t* keep,
                                            float* poisson_radii, uint32_t* rounds, void* stream);

/* Audit/repair candidate filter (surface_probe_filter_audit_repair_candidates,
 * surface_probe_sampler.h:120-223; the Python form _deduplicate_audit_candidates
 * and _exclude_selected_duplicates, surface_probes.py:782-832) for set_count
 * candidate sets in one call. Candidates (device f32[N][3] positions and
 * normals, candidate_sets device u32[N] or null for one set) and base sites
 * (device f32[B][3], base_sets u32[B] or null) with the selected base sites
 * base_selected_indices (device u32[M]). audit_indices (device u32[N]) gets,
 * ascending, the candidates kept as audit points: per set and cell
 * floor(p / audit_cell_sizes[set]) (host f64[S]), in index order, those whose
 * normal dot with every earlier kept one of the cell stays below
 * normal_cosine_threshold. repair_indices (device u32[N]) gets, ascending,
 * the candidates whose (set, position bits, normal bits) match no selected
 * base site and no lower-indexed candidate. audit_count and repair_count are
 * host outputs. Allocates scratch on the stream and synchronizes it. */
NAN_B200_API int nan_filter_audit_repair(NanContext* ctx, const float* candidate_positions,
                                         const float* candidate_normals, const uint32_t* candidate_sets,
                                         uint32_t candidate_count, const float* base_positions,
                                         const float* base_normals, const uint32_t* base_sets, uint32_t base_count,
                                         const uint32_t* base_selected_indices, uint32_t base_selected_count,
                                         uint32_t set_count, const double* audit_cell_sizes,
                                         double normal_cosine_threshold, uint32_t* audit_indices,
                                         uint32_t* audit_count, uint32_t* repair_indices, uint32_t* repair_count,
                                         void* stream);

/* Point octrees of surface-probe sites (_build_point_octree_python,
 * surface_probes.py:1348-1438; surface_probe_build_point_octree,
 * surface_probe_sampler.h:120-223) for set_count point sets in one call.
 * positions: device f32[N][3], set k = [set_offsets[k], set_offsets[k+1])
 * (host u32[S+1]); empty sets get no nodes. Per set, nodes u32[4] =
 * (child_base, child_mask, probe_start, probe_count), numbered as the
 * reference's depth-first build numbers them (root 0, a split node's present
 * octants contiguous in ascending order from child_base), local to the set;
 * written to nodes (device u32[node_capacity][4]) from node_offsets[k] (host
 * u32[S+1] out). order (device u32[N]) gets, per set, the set-local input
 * index of each position in leaf order (each leaf ascending), which
 * probe_start and probe_count index. roots (host f64[S][4]) gets each root
 * cube's centre and half extent. leaf_capacity >= 1, max_depth 1..16.
 * NAN_ERR_LIMIT when the nodes exceed node_capacity, with
 * node_offsets[set_count] holding the count needed. Allocates scratch on the
 * stream and synchronizes it. */
NAN_B200_API int nan_build_point_octrees(NanContext* ctx, const float* positions, const uint32_t* set_offsets,
                                         uint32_t set_count, uint32_t leaf_capacity, uint32_t max_depth,
                                         uint32_t* nodes, uint32_t node_capacity, uint32_t* node_offsets,
                                         uint32_t* order, double* roots, void* stream);

/* Deficit repair (deficit_repair, surface_probes.py:1201-1253;
 * surface_probe_deficit_repair, surface_probe_sampler.h:120-223; the Python
 * form deficit_repair_python, surface_probe_sampler.py:990-1103). Each audit
 * point gathers the base probes of its own instance within that instance's
 * kernel radius (weights (1 - d^2/R^2)^2 x exp(-(plane distance / (R/4))^2 / 2)
 * x the soft normal gate, above weight_epsilon, the 32 largest); its deficit
 * is min_gather_count - count. Repair candidates are then chosen one at a
 * time by score sum (2 deficit - 1) over the deficient audits they reach,
 * highest first (lowest index on ties), each lowering those deficits by one,
 * until max_repair_count or no positive score. Positions and normals are
 * device f32[N][3], instances device u32[N]; instance_radii is a host
 * f32[instance_count]. selected (device u32[max_repair_count]) gets the
 * chosen candidates in choice order and *repair_count (host) their number;
 * counts, weight sums and effective sample sizes of every audit before and
 * after (device, audit_count each). Allocates scratch on the stream and
 * synchronizes it. */
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
                                    uint32_t* rounds, void* stream);

/* Support estimate (estimate_surface_support, surface_probes.py:1256-1299;
 * surface_probe_estimate_support, surface_probe_sampler.h:120-223; the
 * Python form estimate_support_python, surface_probe_sampler.py:1179-1260):
 * per query site, support = the float64 sum (ascending reference index,
 * numpy's pairwise scheme) of kernel x area weight over the reference points
 * of its instance within that instance's radius; f = clip(support / (pi R^2
 * / 3), 0, 1) and m = min(M, 1 / max(f, 1 / M)). Reference and query arrays
 * are device memory as in nan_deficit_repair; support_f and density_m are
 * device f32[query_count]. The float64 sum is numpy's for a float32 array:
 * buffers of 8192 terms, each summed pairwise, the buffer sums added in
 * order; no cap on the terms of a query. Allocates scratch on the stream and
 * synchronizes it. */
NAN_B200_API int nan_estimate_support(NanContext* ctx, const float* reference_positions,
                                      const float* reference_normals, const uint32_t* reference_instances,
                                      const float* reference_area_weights, uint32_t reference_count,
                                      const float* query_positions, const float* query_normals,
                                      const uint32_t* query_instances, uint32_t query_count,
                                      const float* instance_radii, uint32_t instance_count,
                                      const NanSupportOptions* options, float* support_f, float* density_m,
                                      void* stream);

/* 16-byte slots -> one RGB9E5 uint each (MeshColorsRGB9E5Packer.execute,
 * mesh_colors_rgb9e5.py:4-29; mesh_colors_rgb9e5_pack.slang:7-16). */
NAN_B200_API int nan_pack_rgb9e5(NanContext* ctx, const uint8_t* slots, uint32_t* out,
                                 uint32_t count, void* stream);

/* ------------------------------------------------------------------------
 * Multi-scene probe batches. No counterpart in the reference (one dispatch
 * per scene, surface_probe_path_tracer.py:49-83): the probe sets of many
 * scenes are baked by one persistent launch that balances (scene, probe)
 * units across the GPU, optionally replayed from a captured CUDA graph.
 * Each set has the buffers of nan_trace_probes. The batch keeps a snapshot of
 * every scene's BVH: rebuild the batch after rebuilding a scene.
 * ------------------------------------------------------------------------ */
typedef struct NanBatch NanBatch;

typedef struct NanProbeSet {
    NanContext* scene;               /* context whose scene (BVH) the probes sit in */
    const uint8_t* probes;           /* u8[N][48] */
    uint32_t probe_count;
    const uint8_t* probe_instances;  /* u8[I][48] */
    uint32_t probe_instance_count;
    float* values;                   /* f32[N][3] */
    uint32_t* sample_counts;         /* u32[N] */
    uint32_t* self_hits;             /* u32[N] */
    uint32_t* radial;                /* u32[N][16] */
    float* compensation;             /* optional f32[N][4] */
    NanLighting lighting;
} NanProbeSet;

typedef struct NanBatchTuning {
    uint32_t stack_depth;        /* traversal stack entries: 48 or 96 (>= every BVH's need) */
    uint32_t blocks_per_sm;      /* persistent 128-thread blocks per SM */
    uint32_t units_per_grab;     /* probes per lane taken from the work counter at once */
    uint32_t min_blocks_per_sm;  /* register cap of the kernel variant: 0 (compiler's), 4 or 6 */
} NanBatchTuning;

NAN_B200_API int nan_batch_create(NanContext* ctx, const NanProbeSet* sets, uint32_t set_count,
                                  NanBatch** out);
NAN_B200_API int nan_batch_destroy(NanBatch* batch);
/* Smallest admissible stack depth, the total probe count, the current tuning. */
NAN_B200_API int nan_batch_info(NanBatch* batch, uint32_t* min_stack_depth, uint32_t* total_probes,
                                NanBatchTuning* tuning);
NAN_B200_API int nan_batch_set_tuning(NanBatch* batch, const NanBatchTuning* tuning);
/* How a probe's samples draw random numbers. SEQUENTIAL (the default): one
 * stream per probe, samples in sequence, as the reference's baker
 * (surface_probe_path_tracer.slang:206-278) -- bit-exact with
 * nan_trace_probes. INDEPENDENT: sample k draws from RNG(probe, instance,
 * iteration * samples + k), so a warp traces 32 samples of one probe at once;
 * the per-probe sums are still formed in sample order. WAVEFRONT: the
 * sequential sample streams, run as one multi-scene wavefront (every probe of
 * every set one path in flight; extend / shade / shadow / finalize rounds
 * over all sets; bit-exact with SEQUENTIAL); allocates one path of scratch
 * per probe on the batch's context; the tuning's blocks_per_sm is the
 * traversal grid. WAVEFRONT_INDEPENDENT: the INDEPENDENT sample streams on
 * the wavefront, one path per (probe, sample), in chunks of up to 2^24 paths,
 * each finished sample stored and every probe's samples folded in sample
 * order (bit-exact with INDEPENDENT). Resets the launch shape to the new
 * kernel's defaults. */
enum {
    NAN_BATCH_SEQUENTIAL_SAMPLES = 0,
    NAN_BATCH_INDEPENDENT_SAMPLES = 1,
    NAN_BATCH_WAVEFRONT = 2,
    NAN_BATCH_WAVEFRONT_INDEPENDENT = 3
};
NAN_B200_API int nan_batch_set_mode(NanBatch* batch, uint32_t mode);
/* One iteration of every set (nan_trace_probes semantics per set). */
NAN_B200_API int nan_batch_trace_probes(NanBatch* batch, uint32_t iteration, uint32_t samples_per_probe,
                                        uint32_t max_bounces, int reset, void* stream);
/* Time each admissible launch shape on one frame (reset, iteration 0) and
 * keep the fastest; the outputs then hold that frame. */
NAN_B200_API int nan_batch_autotune(NanBatch* batch, uint32_t samples_per_probe, uint32_t max_bounces,
                                    void* stream, NanBatchTuning* chosen, float* frame_ms);
/* Capture one frame into a CUDA graph. The next replayed frame has
 * iteration first_iteration (reset if reset_first); each replay advances the
 * iteration on the device. Synchronises `stream` once. */
NAN_B200_API int nan_batch_capture(NanBatch* batch, uint32_t first_iteration, int reset_first,
                                   uint32_t samples_per_probe, uint32_t max_bounces, void* stream);
NAN_B200_API int nan_batch_replay(NanBatch* batch, uint32_t frames, void* stream);

/* ------------------------------------------------------------------------
 * Learned radiance cache. No counterpart in the reference: an online-trained
 * irradiance cache (multiresolution hash encoding, 16 levels x 2 FP16
 * features x 2^log2_table entries, feeding a 48-64-64-64-64-16 ReLU MLP whose
 * first 3 outputs are irradiance RGB) with BF16 tcgen05 forward and backward
 * kernels, a relative L2 loss and Adam.
 * Queries are f32[N][8]: position xyz, pad, shading normal xyz, pad.
 * Targets are f32[N][4]: irradiance rgb, w (w < 0: no sample, skipped).
 * All pointers are device memory.
 * ------------------------------------------------------------------------ */
typedef struct NanCache NanCache;

typedef struct NanCacheConfig {
    float bounds_min[3];       /* positions are normalised to this box */
    float bounds_max[3];
    uint32_t log2_table;       /* entries per level, 2^10 .. 2^24 */
    uint32_t base_resolution;  /* coarsest grid resolution */
    uint32_t max_resolution;   /* finest grid resolution */
    float learning_rate;       /* Adam */
    float beta1;
    float beta2;
    float epsilon;
    float loss_epsilon;        /* relative L2: (o - y)^2 / (o^2 + loss_epsilon) */
    uint32_t table_update;     /* hash-table optimizer step: 0 = Adam over every entry; 1 = lazy
                                  Adam, only entries whose gradient is nonzero in the step (their
                                  moments and parameters; bias correction by the global step) */
    uint32_t reserved[3];
} NanCacheConfig;

/* Scratch and outputs of one cached frame (nan_trace_screen_cached). */
typedef struct NanCachedFrame {
    float* queries;          /* f32[W*H][8] scratch: the frame's cache queries
                                (position, pixel bits; shading normal, 0) */
    float* query_weights;    /* f32[W*H][4] scratch: throughput * albedo / pi */
    uint32_t* query_count;   /* u32[1] scratch */
    float* train_points;     /* f32[T][4] out: (b1, b2, instance bits, primitive bits |
                                back << 31) of the training pixels' cache points,
                                instance ~0 where the path ended earlier */
    float* train_queries;    /* f32[T][8] out: their cache queries */
    uint32_t train_count;    /* T */
    uint32_t train_offset;   /* training pixel i is (offset + i * stride) mod (W*H) */
    uint32_t train_stride;   /* coprime with W*H */
    uint32_t train_stride_inverse;  /* stride^-1 mod (W*H) */
    uint32_t cache_vertex;   /* path vertex answered by the cache: 1 = the second hit (the
                                cache holds irradiance); 0 = the first hit, after its sun
                                NEE (the cache holds indirect irradiance) */
} NanCachedFrame;

/* Parameter counts: MLP weights (row-major per layer: 64x48, 3 x 64x64,
 * 16x64) and hash-table floats (levels x 2^log2_table x 2). */
NAN_B200_API int nan_cache_sizes(const NanCacheConfig* config, uint64_t* mlp_params,
                                 uint64_t* table_params);
NAN_B200_API int nan_cache_create(NanContext* ctx, const NanCacheConfig* config, NanCache** out);
NAN_B200_API int nan_cache_destroy(NanCache* cache);
/* Upload parameters (device f32 arrays) and reset the optimizer state. */
NAN_B200_API int nan_cache_set_params(NanCache* cache, const float* mlp, const float* table,
                                      void* stream);
/* Copy parameters, accumulated gradients and the accumulated loss into
 * device arrays; any output may be NULL. */
NAN_B200_API int nan_cache_get_params(NanCache* cache, float* mlp, float* table, float* mlp_grad,
                                      float* table_grad, float* loss, void* stream);
/* out f32[N][4] = network(queries). */
NAN_B200_API int nan_cache_infer(NanCache* cache, const float* queries, uint32_t count, float* out,
                                 void* stream);
/* Forward + backward of the loss averaged over `batch` samples; adds into
 * the gradients and the loss (no parameter change). */
NAN_B200_API int nan_cache_backward(NanCache* cache, const float* queries, const float* targets,
                                    uint32_t count, uint32_t batch, void* stream);
/* One Adam step from the accumulated gradients, which it then clears. */
NAN_B200_API int nan_cache_step(NanCache* cache, void* stream);
/* Train on `count` samples in batches of `batch`: backward + step each. */
/* Learning rate of the following optimizer steps (a schedule set by the
 * caller). Host state only. No counterpart in the reference. */
NAN_B200_API int nan_cache_set_learning_rate(NanCache* cache, float learning_rate);
NAN_B200_API int nan_cache_train(NanCache* cache, const float* queries, const float* targets,
                                 uint32_t count, uint32_t batch, void* stream);

/* Irradiance at surface points f32[N][4] (b1, b2, instance bits, primitive
 * bits | back << 31): the texel estimator (texture_space_path_tracer.slang:
 * 86-117) with RNG(index, 0xFFFFFFFF, iteration * samples) and view = the
 * flat normal (negated for back). out f32[N][4] = (E rgb, 0), or
 * (0, 0, 0, -1) where the instance is ~0. Produces the cache's training
 * targets; no counterpart in the reference's API. */
enum { NAN_POINTS_INDIRECT_ONLY = 1 }; /* leave out the direct sun irradiance term */
NAN_B200_API int nan_trace_points(NanContext* ctx, const float* points, uint32_t count, float* out,
                                  uint32_t iteration, uint32_t samples, uint32_t max_bounces,
                                  uint32_t flags, const NanLighting* lighting, void* stream);

/* A cached frame of the screen path tracer: the reference's path
 * (path_tracer.slang:40-84) up to vertex cache_vertex, whose remaining path
 * is replaced by throughput * albedo / pi * max(cache irradiance, 0).
 * Writes out f32[H][W][4] and the frame's training points. */
NAN_B200_API int nan_trace_screen_cached(NanContext* ctx, NanCache* cache, float* out, uint32_t width,
                                         uint32_t height, uint32_t frame, const NanCamera* camera,
                                         const NanLighting* lighting, const NanCachedFrame* frame_desc,
                                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NAN_B200_H */
