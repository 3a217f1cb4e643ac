/*
 * olcuda.h — C ABI of the B200 wavefront path tracer (libolcuda.so).
 *
 * Every entry point returns an int status (OLC_OK == 0).  On failure the
 * message is available from olc_last_error(ctx) (or olc_last_error(NULL)
 * for failures that happen before a context exists).  The Python layer maps
 * the codes to the exception types the reference renderer raises:
 *   OLC_ERR_VALUE   -> ValueError    (bad sizes / sample counts,
 *                                      ordinarylight/targets/vulkan/api.py:1267-1272,
 *                                      ordinarylight/renderers/reference/cpu.py:15-21)
 *   OLC_ERR_TYPE    -> TypeError
 *   OLC_ERR_CLOSED  -> RuntimeError  (closed renderer, cpu.py:60-62)
 *   OLC_ERR_RUNTIME / OLC_ERR_CUDA / OLC_ERR_MEMORY / OLC_ERR_TIMEOUT
 *                   -> RuntimeError / MemoryError
 *
 * Bulk arrays are plain pointers plus sizes.  Arguments documented as
 * "host" are read on the host; arguments documented as "device" must be
 * device pointers on the context's GPU (for example torch.Tensor.data_ptr()).
 * No entry point takes or returns framework (torch) types.
 */
#ifndef OLCUDA_H
#define OLCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OLC_ABI_VERSION 6

#if defined(__GNUC__)
#define OLC_API __attribute__((visibility("default")))
#else
#define OLC_API
#endif

enum olc_status {
  OLC_OK = 0,
  OLC_ERR_VALUE = 1,
  OLC_ERR_TYPE = 2,
  OLC_ERR_RUNTIME = 3,
  OLC_ERR_CUDA = 4,
  OLC_ERR_MEMORY = 5,
  OLC_ERR_CLOSED = 6,
  OLC_ERR_TIMEOUT = 7
};

/* Transport modes. */
enum olc_mode {
  /* GGX/Lambert BSDF, next-event estimation with power-heuristic MIS,
   * Russian roulette; the reference GPU wavefront's estimator
   * (ordinarylight/shaders/wavefront_shade.comp:262-596). */
  OLC_MODE_PRODUCTION = 0,
  /* The CPU reference's estimator: pure Lambert (albedo = base_color),
   * emission on every hit, CPU sky gradient, no NEE/RR, origin offset
   * 1e-4 along the facing normal and t_min 1e-4
   * (ordinarylight/renderers/reference/path_tracer.py:31-95). */
  OLC_MODE_REFERENCE_COMPATIBLE = 1
};

/* Camera projections (ordinarylight/cameras/). */
enum olc_projection {
  OLC_PROJECTION_PERSPECTIVE = 0,
  OLC_PROJECTION_ORTHOGRAPHIC = 1,
  OLC_PROJECTION_PANORAMIC = 2
};

/* Analytic light types; the codes of Scene.analytic_light_data
 * (ordinarylight/scene/_core.py:2578-2632). */
enum olc_light_type {
  OLC_LIGHT_POINT = 0,
  OLC_LIGHT_DIRECTIONAL = 1,
  OLC_LIGHT_SPOT = 2
};

/* Environment kinds: none (analytic sky of the mode), constant colour, or an
 * equirectangular float32 RGB image (path_tracer.py:185-202). */
enum olc_environment_kind {
  OLC_ENV_NONE = 0,
  OLC_ENV_CONSTANT = 1,
  OLC_ENV_EQUIRECT = 2
};

typedef struct olc_context olc_context;

/* Renderer configuration.  Mirrors ReferenceConfig
 * (ordinarylight/renderers/reference/cpu.py:9-21) plus the wavefront knobs of
 * RendererConfig (ordinarylight/targets/vulkan/api.py:27-717). */
typedef struct olc_config {
  int32_t device;               /* CUDA ordinal */
  uint32_t mode;                /* enum olc_mode */
  uint32_t max_bounces;         /* 1..64 */
  uint32_t seed;                /* added to frame_index, as cpu.py:64 does */
  uint32_t russian_roulette_start;   /* 0 disables RR (production mode) */
  float russian_roulette_min_survival;
  uint32_t restir;              /* 1 enables ReSTIR DI at the primary hit */
  uint32_t restir_candidates;   /* initial RIS candidates (1..64) */
  uint32_t restir_temporal;     /* temporal reuse passes (0/1) */
  uint32_t restir_spatial;      /* spatial reuse passes (0..2) */
  uint32_t restir_neighbours;   /* spatial neighbours per pass */
  float restir_radius;          /* spatial radius in pixels */
  uint32_t restir_max_history;  /* temporal M cap, multiple of the candidates */
  uint32_t block_size;          /* threads per block for the queue kernels */
  uint32_t stack_depth;         /* shared-memory traversal stack: 16, 24, 32 */
  uint32_t chunk_paths;         /* paths resident per wavefront chunk; 0 = auto */
  uint32_t use_graphs;          /* capture the bounce loop as a CUDA graph */
  uint32_t flatten_instances;   /* bake instances of meshes with <= 64 triangles
                                   into world-space triangles of the TLAS */
  uint32_t trace_scheduler;     /* 0: persistent lanes refilled from the queue
                                   as rays finish; 1: warps take 32 rays at a
                                   time and run them to completion */
  uint32_t disable_nee;         /* production mode without next-event
                                   estimation (pure BSDF sampling) */
  uint32_t trace_block;         /* threads per block of the traversal and
                                   shading kernels: 64, 128 or 256; 0 = 128 */
  uint32_t ray_sort;            /* reorder extension rays by origin cell and
                                   direction before tracing them (helps
                                   shading coherence on large scenes) */
  uint32_t serve_aging_steps;   /* serving: jobs queued this many steps go
                                   first, oldest first (0: shortest remaining
                                   work first only) */
  uint32_t sample_variance;     /* olc_render keeps each sample's luminance so
                                   olc_read_variance can return the per-pixel
                                   sample variance (4 bytes per path sample) */
  uint32_t reserved[1];
} olc_config;

/* Scene description: host arrays, copied at upload.  Geometry follows the
 * reference's instancing model: one bottom-level structure per MeshResource
 * (ordinarylight/targets/vulkan/scene.py:1493-1530), one instance per visible
 * Mesh in Scene.visible_meshes order (scene/_core.py:1029). */
typedef struct olc_scene_desc {
  /* bottom level: meshes in object space */
  uint32_t num_meshes;
  const uint32_t* mesh_vertex_offset;    /* [num_meshes + 1] */
  const uint32_t* mesh_triangle_offset;  /* [num_meshes + 1] */
  const float* vertices;                 /* [total_vertices * 3] */
  const float* normals;                  /* [total_vertices * 3] */
  const uint32_t* indices;               /* [total_triangles * 3], mesh-local */
  /* top level */
  uint32_t num_instances;
  const float* instance_object_to_world; /* [num_instances * 12], row-major 3x4 */
  const uint32_t* instance_mesh;         /* [num_instances] */
  const uint32_t* instance_material;     /* [num_instances] */
  const uint32_t* instance_id;           /* [num_instances] Mesh.id */
  const uint32_t* instance_primitive_offset; /* [num_instances] packed base */
  /* materials: 16 floats each:
   * base_color.rgb, roughness, emission.rgb, metallic, emission_two_sided,
   * material_id (as float bits), transmission, ior, 4 reserved */
  uint32_t num_materials;
  const float* materials;
  /* emissive triangles, 20 floats each, the layout of
   * Scene.emissive_triangle_data (scene/_core.py:2637-2691):
   * a.xyz,0  b.xyz,0  c.xyz,0  emission.rgb,area  cdf,pdf,two_sided,0 */
  uint32_t num_emitters;
  const float* emitters;
  float emissive_weight;                 /* Scene.emissive_light_weight */
  /* analytic lights, 16 floats each, Scene.analytic_light_data layout:
   * position.xyz,type  direction.xyz,range  color.rgb,intensity  cos_inner,cos_outer,0,0 */
  uint32_t num_lights;
  const float* lights;
  /* environment */
  uint32_t environment_kind;             /* enum olc_environment_kind */
  float environment_color[3];            /* colour * intensity */
  float environment_rotation;
  uint32_t environment_width, environment_height;
  const float* environment_image;        /* [h * w * 3] float32 */
  /* heterogeneous medium (one dense grid in a unit box; 0 = none) */
  uint32_t volume_present;
  uint32_t volume_dims[3];               /* nx, ny, nz */
  const float* volume_density;           /* [nz * ny * nx] */
  float volume_world_to_box[12];         /* row-major 3x4 world -> [0,1]^3 */
  float volume_sigma_t_scale;
  float volume_albedo;
  float volume_max_density;
  uint32_t reserved[7];
  /* textures (num_texture_bindings = 0: an untextured scene; the rest may
   * then be NULL) */
  const float* texcoords;                /* [total_vertices * 4]: uv0.xy, uv1.xy */
  const float* tangents;                 /* [total_vertices * 4]: object-space xyz, handedness */
  uint32_t num_texture_words;
  const uint32_t* texture_words;         /* Scene.texture_data layout: count, 8 words per
                                            texture (sRGB offset, linear offset, width, height,
                                            wrap/filter flags, levels, 0, 0), then RGBA8 mip
                                            pyramids (scene/_core.py:3005-3077) */
  uint32_t num_texture_bindings;
  const float* texture_bindings;         /* [n * 8]: texture, cos, sin, texcoord set, offset.xy,
                                            scale.xy (Scene.texture_binding_data) */
  const float* material_textures;        /* [num_materials * 12]: binding of the base colour,
                                            metallic-roughness, emissive, normal, occlusion and
                                            transmission maps (-1: none), normal scale, occlusion
                                            strength, uses texcoord set 1, 3 reserved */
  /* volumes in the reference's own model, which the reference-compatible mode
   * integrates along every ray segment (ReferencePathTracer.render_hdr,
   * renderers/reference/path_tracer.py:55-65; volume/_core.py:252-504); at
   * most 8, 72 floats each (integers as bit patterns):
   *   world->local unit cube rows (12), nx ny nz lut_len, grid offset,
   *   lut offset, address (0 clamp, 1 repeat, 2 mirror), linear filter,
   *   missing data, clip-plane count, Henyey-Greenstein phase, scattering
   *   orders, density scale, emission scale, step size, scattering scale,
   *   scattering colour rgb + anisotropy, scattering albedo rgb + 0,
   *   8 clip planes (a, b, c, d), 4 reserved */
  uint32_t num_ref_volumes;
  const float* ref_volume_records;       /* [n * 72] */
  uint64_t ref_grid_values;
  const float* ref_volume_grids;         /* Volume.normalized_data of each volume (z, y, x), concatenated */
  uint64_t ref_lut_entries;
  const float* ref_volume_luts;          /* transfer-function RGBA entries, concatenated */
} olc_scene_desc;

/* Camera basis computed by the caller in float32 exactly as the reference's
 * ReferencePathTracer._camera_rays does (path_tracer.py:110-151). */
typedef struct olc_camera {
  float position[3];
  float forward[3];
  float right[3];
  float up[3];
  float half_height;       /* tan(fov/2) or ortho half size */
  float horizontal_half;   /* panoramic: half horizontal angle (radians) */
  float vertical_half;     /* panoramic: half vertical angle (radians) */
  uint32_t projection;     /* enum olc_projection */
} olc_camera;

/* Per-frame statistics (host). */
typedef struct olc_render_stats {
  uint64_t camera_rays;
  uint64_t extension_rays;   /* closest-hit rays after the camera rays */
  uint64_t shadow_rays;
  uint64_t overflow;         /* queue overflows (paths terminated) */
  uint64_t traversal_errors; /* stack overflows (0 on a healthy run) */
  float gpu_ms;              /* CUDA-event time of the device work */
  /* raygen_ms stays 0: bounce-0 closest-hit traversal generates the camera
   * rays it traces, so their generation is part of trace_ms */
  float raygen_ms, trace_ms, shade_ms, shadow_ms, restir_ms, accumulate_ms;
  uint32_t chunks;
  uint32_t restir_history_used;
  uint32_t jobs_completed;   /* jobs resolved by the call */
  uint32_t reserved;
  uint64_t h2d_bytes;        /* host->device bytes of the call (chunk tables) */
  uint64_t d2h_bytes;        /* device->host bytes (counters, host outputs) */
} olc_render_stats;

/* ---- context --------------------------------------------------------- */

/* Create a context on cfg->device.  Replaces the construction of the
 * reference's GPU engine (_VulkanGlobalIlluminationEngine,
 * ordinarylight/targets/vulkan/api.py:844). */
OLC_API int olc_create(const olc_config* cfg, olc_context** out);

/* Release all device memory; ctx becomes invalid (RendererProtocol.close,
 * ordinarylight/renderers/base.py:69-71). */
OLC_API int olc_destroy(olc_context* ctx);

/* Last error message of ctx, or of the calling thread when ctx is NULL. */
OLC_API const char* olc_last_error(const olc_context* ctx);

/* Library ABI version (OLC_ABI_VERSION). */
OLC_API int olc_abi_version(void);

/* Update the mutable knobs of a live context (Renderer.reconfigure,
 * ordinarylight/renderer/_core.py:386-413). */
OLC_API int olc_reconfigure(olc_context* ctx, const olc_config* cfg);

/* ---- scene residency ------------------------------------------------- */

/* Upload a scene and build its two-level LBVH on the device
 * (replaces VulkanSceneUploader._build_scene,
 * ordinarylight/targets/vulkan/scene.py:1322-1560, and upload_window_scene,
 * ordinarylight/targets/vulkan/core.py:4574-4634).  Transactional: on
 * failure the previously resident scene stays resident. */
OLC_API int olc_upload_scene(olc_context* ctx, const olc_scene_desc* scene);

/* Device bytes held by the resident scene (for HBM admission). */
OLC_API int olc_scene_bytes(const olc_context* ctx, uint64_t* bytes);

/* ---- scene pool: several resident scenes ------------------------------ */

/* All resident scenes share one device pool (nodes, triangle slots,
 * instances, materials, emitters, lights), so one wavefront can mix rays of
 * different scenes.  olc_upload_scene replaces the context's default scene;
 * olc_add_scene makes an additional scene resident and returns its handle,
 * the way the reference keeps a scene resident across frames keyed by
 * Scene.revision (upload_window_scene, ordinarylight/targets/vulkan/core.py:4574-4634;
 * replace_scene, ordinarylight/targets/vulkan/api.py:913-917).
 * Transactional: on failure nothing becomes resident. */
OLC_API int olc_add_scene(olc_context* ctx, const olc_scene_desc* scene, uint32_t* handle);

/* Release a scene added by olc_add_scene.  Its pool ranges are reused by
 * later scenes.  Queued jobs that render it must have completed. */
OLC_API int olc_remove_scene(olc_context* ctx, uint32_t handle);

/* Handle that names the olc_upload_scene scene in olc_update_scene. */
#define OLC_DEFAULT_SCENE 0xffffffffu

/* Update a resident scene in place (animation, material or light edits)
 * from a description with the same layout: per-mesh vertex and triangle
 * counts, instance-to-mesh mapping, material/emitter/light counts and
 * environment image size.  Meshes flagged in mesh_changed ([num_meshes];
 * NULL = all) get their triangles rewritten and their BLAS refit with the
 * hierarchy unchanged; instance transforms, baked triangles, the TLAS,
 * materials, emitters, lights, environment and volume are rewritten.
 * *applied = 1 on success; 0 (nothing changed) when the layout differs, in
 * which case the caller uploads the scene again.  refitted (optional)
 * receives the number of refit BLAS.  Temporal ReSTIR history of the scene
 * is dropped.  Queued jobs that render the scene must have completed.
 * Replaces _try_update_window_scene (ordinarylight/targets/vulkan/core.py:4696-4868),
 * _refit_scene_blases and _rebuild_scene_tlas
 * (ordinarylight/targets/vulkan/scene.py:1217-1330). */
OLC_API int olc_update_scene(olc_context* ctx, uint32_t handle, const olc_scene_desc* scene,
                             const uint8_t* mesh_changed, int32_t* applied, uint32_t* refitted);

/* Statistics of one resident scene (handle from olc_add_scene). */
typedef struct olc_scene_stats {
  uint64_t bytes;            /* device bytes of the scene's data and hierarchy */
  uint32_t triangles;
  uint32_t blas_count;
  uint32_t blas_nodes;
  uint32_t tlas_nodes;
  uint32_t flattened_instances;
  uint32_t reserved;
  double build_ms;
} olc_scene_stats;
OLC_API int olc_scene_stats_get(const olc_context* ctx, uint32_t handle, olc_scene_stats* stats);

/* Device memory of the context, for admission by an HBM budget. */
typedef struct olc_pool_info {
  uint32_t resident_scenes;
  uint32_t queued_jobs;       /* served jobs not yet completed */
  uint64_t scene_bytes;       /* bytes the resident scenes use */
  uint64_t pool_bytes;        /* bytes the scene pool has allocated (capacity) */
  uint64_t wavefront_bytes;   /* queues, path state, reservoirs */
  uint64_t pixel_bytes;       /* allocated accumulator/output arena */
  uint64_t pixel_bytes_used;  /* arena bytes held by queued jobs */
  uint64_t reserved[3];
} olc_pool_info;
OLC_API int olc_pool_info_get(const olc_context* ctx, olc_pool_info* info);

/* ---- batched and served rendering ------------------------------------- */

/* One render job.  Its random numbers are keyed exactly as olc_render's
 * (pixel, sample, bounce, seed + frame_index), so a job renders the same
 * bits alone, in a batch or among served requests, and the same bits as
 * olc_render of the same scene, camera, size, samples and frame when that
 * frame uses no temporal history (first frame or after olc_reset_history). */
typedef struct olc_job {
  uint32_t scene;               /* handle from olc_add_scene */
  uint32_t width, height;
  uint32_t samples_per_pixel;   /* 1..65536 */
  uint32_t frame_index;
  uint32_t max_bounces;         /* 0: the context's max_bounces; else 1..64 */
  uint32_t first_sample;        /* RNG index of the job's first sample: a job
                                   with first_sample s renders samples
                                   s .. s + samples_per_pixel - 1 of the frame,
                                   so disjoint shards of one frame's samples
                                   can be rendered apart (other GPUs) */
  uint32_t reserved;
  olc_camera camera;
  float* out_rgba;              /* (height, width, 4) float32 mean of the job's
                                   samples, host or device; may be NULL when
                                   out_sums is set */
  uint64_t* out_sums;           /* optional (height, width, 3) fixed-point sums
                                   of the job's samples (scale 2^28), host or
                                   device like out_rgba: shards of a frame add
                                   exactly, and sum * 2^-28 / spp resolved in
                                   double and rounded to float equals the
                                   single-device image bit for bit */
  int32_t out_is_device;
  uint32_t reserved2;
} olc_job;

/* Render num_jobs jobs as one wavefront: every chunk of paths may hold
 * paths of several jobs and scenes, sharing the ray queues, and the chunk
 * sequence is replayed from a CUDA graph when the same mix recurs.  Returns
 * when every output is written.  Replaces rendering the jobs one at a time
 * through Renderer.render_async (ordinarylight/renderer/_core.py:614-651,
 * which serialises submissions on one worker). */
OLC_API int olc_render_batch(olc_context* ctx, const olc_job* jobs, uint32_t num_jobs,
                             olc_render_stats* stats);

/* Serving: queue a job (continuous batching).  Validates the job, reserves
 * its accumulator pixels and returns a ticket; the job's paths join the
 * shared wavefront at the next olc_serve_step.  job->out_rgba must stay
 * valid until the ticket is reported complete. */
OLC_API int olc_submit(olc_context* ctx, const olc_job* job, uint64_t* ticket);

/* One serving step: launch the next chunk (at most chunk_paths paths) drawn
 * from the queued jobs, shortest remaining work first (jobs queued for
 * serve_aging_steps steps or more go first, oldest first), then wait for the
 * chunk the previous step launched
 * and report the jobs whose last paths were in it (resolved and copied out).
 * Keeping one chunk in flight hides the host work of a step behind the
 * device work of the previous one.  done (host, capacity done_capacity)
 * receives the tickets and num_done their count; stats (may be NULL) the
 * collected chunk's statistics.  Jobs submitted between steps join the next
 * chunk; a job is queued until a step reports it. */
OLC_API int olc_serve_step(olc_context* ctx, uint64_t* done, uint32_t done_capacity,
                           uint32_t* num_done, olc_render_stats* stats);

/* Drop a queued job; its partial samples are discarded (RenderJob.cancel,
 * ordinarylight/renderer/_core.py:614-651). */
OLC_API int olc_cancel(olc_context* ctx, uint64_t ticket);

/* Tickets of the queued jobs in submission order (tickets may be NULL to
 * query the count).  After an olc_serve_step failure the jobs of the failed
 * chunk are no longer queued; this tells the caller which ones remain. */
OLC_API int olc_queued_jobs(const olc_context* ctx, uint64_t* tickets, uint32_t capacity, uint32_t* count);

/* Device bytes a job needs while queued (accumulator and output pixels),
 * for admission by an HBM budget. */
OLC_API int olc_job_bytes(const olc_context* ctx, const olc_job* job, uint64_t* bytes);

/* ---- rendering ------------------------------------------------------- */

/* Render width x height at spp samples for frame_index into out_rgba
 * ((height, width, 4) float32, linear HDR, channel 3 = 0 like the CPU
 * reference).  out_is_device selects a device or host destination.
 * Replaces render_wavefront_outputs (ordinarylight/targets/vulkan/api.py:1252-1451)
 * behind RendererProtocol.render_frame (ordinarylight/renderers/base.py:56-67). */
OLC_API int olc_render(olc_context* ctx, const olc_camera* camera, uint32_t width,
               uint32_t height, uint32_t spp, uint32_t frame_index,
               float* out_rgba, int out_is_device, olc_render_stats* stats);

/* Optional per-pixel products of the first sample's primary hit
 * (render_products, ordinarylight/renderer/_core.py:768-777).  Each pointer
 * may be NULL; all are host arrays of height*width entries (normal: *3).
 * Valid after olc_render with the same size. */
OLC_API int olc_read_products(olc_context* ctx, uint32_t width, uint32_t height,
                      float* depth, float* normal, uint32_t* instance_id,
                      uint32_t* material_id, uint32_t* primitive_id);

/* Unbiased per-pixel sample variance of the luminance
 * (0.2126 R + 0.7152 G + 0.0722 B) of the last olc_render's samples: the
 * "variance" product of render_wavefront_outputs
 * (ordinarylight/targets/vulkan/api.py:1400-1433), (sum(l^2) - sum(l)^2 / spp)
 * / (spp - 1) in double precision over the samples in order, clamped at 0,
 * and 0 for one sample.  Needs olc_config.sample_variance for that render.
 * variance: height*width floats, host or device (out_is_device). */
OLC_API int olc_read_variance(olc_context* ctx, uint32_t width, uint32_t height,
                              float* variance, int out_is_device);

/* World hit point (height*width*3 floats) and barycentrics (height*width*2,
 * (u, v) in the triangle's index order) of the last olc_render's first
 * sample's primary hits; host arrays, either may be NULL (the
 * primary_position / primary_barycentric readback of
 * render_wavefront_outputs, ordinarylight/targets/vulkan/api.py:1302-1397). */
OLC_API int olc_read_hit_geometry(olc_context* ctx, uint32_t width, uint32_t height,
                                  float* position, float* barycentric);

/* Denoiser path signals of the last olc_render's first sample (the
 * secondary path state, ordinarylight/wavefront/_core.py:75-87, written by
 * wavefront_shade.comp:406-410 and :561-568): signals, height*width*4
 * floats: the specular-lobe probability of the primary hit's material, 1
 * when that hit is opaque (0 for transmissive hits, misses and medium
 * events), 0, 0; secondary, height*width*4 floats: the world position of
 * the path's next surface vertex and 1, or zeros when it has none.  Host
 * arrays; either may be NULL. */
OLC_API int olc_read_path_signals(olc_context* ctx, uint32_t width, uint32_t height,
                                  float* signals, float* secondary);

/* Camera frame of the motion projection (_project_positions,
 * ordinarylight/targets/vulkan/api.py:1118-1136): origin, unit forward,
 * right and up, and tan(vertical fov / 2). */
typedef struct olc_motion_camera {
  double origin[3], forward[3], right[3], up[3];
  double scale;
} olc_motion_camera;

/* One visible mesh of the current frame: its packed triangles
 * [first, first + count) and the first packed triangle of the same mesh in
 * the captured frame (0xffffffff: the mesh has no motion history). */
typedef struct olc_motion_mesh {
  uint32_t first, count, previous_first, reserved;
} olc_motion_mesh;

/* Keep the default scene's world-space triangles (packed order) as the
 * previous frame of later olc_read_motion calls (_capture_motion_state,
 * ordinarylight/targets/vulkan/api.py:1139-1149). */
OLC_API int olc_capture_motion_state(olc_context* ctx);

/* Motion product (height*width*2 floats, host): for each pixel whose first
 * sample hit a triangle of a mesh with history, its projection now minus the
 * projection under `before` of the same barycentric point of that triangle
 * in the captured frame; 0 elsewhere (_motion_product,
 * ordinarylight/targets/vulkan/api.py:1151-1200).  meshes are sorted by
 * first. */
OLC_API int olc_read_motion(olc_context* ctx, uint32_t width, uint32_t height,
                            const olc_motion_mesh* meshes, uint32_t num_meshes,
                            const olc_motion_camera* now, const olc_motion_camera* before,
                            float* motion);

/* Material texture lookups of a resident scene (handle, or
 * OLC_DEFAULT_SCENE): for each of n points, the texture of `binding` at
 * uv0/uv1 (host, n*2 floats each) with ray-cone footprints fp0/fp1 (n
 * floats each), sRGB-decoded when srgb != 0, as the shading stage samples
 * it (sampleMaterialTexture, ordinarylight/shaders/wavefront_textures.glsl:134-204);
 * out: n*4 floats (host). */
OLC_API int olc_sample_texture(olc_context* ctx, uint32_t handle, int32_t binding, uint32_t n,
                               const float* uv0, const float* uv1, const float* fp0, const float* fp1,
                               int srgb, float* out);

/* Forget temporal history (Renderer.reset_sequence ->
 * reset_output_history, ordinarylight/renderer/_core.py:339-351, :447-451). */
OLC_API int olc_reset_history(olc_context* ctx);

/* Device timeline of the last olc_render: one record per kernel launch in
 * launch order, timed with CUDA events on the context's stream (the
 * per-stage timestamps of the reference's wavefront executor,
 * ordinarylight/targets/vulkan/core.py:2679-3116, "generate",
 * "intersect_shade.{b}", "resolve").  items = work units of the launch
 * (camera rays, rays, hits+misses, shadow rays, path samples, pixels);
 * misses = rays of the launch's bounce that left the scene. */
enum olc_stage {
  OLC_STAGE_RAYGEN = 0,   /* no longer recorded: part of bounce 0's OLC_STAGE_TRACE */
  OLC_STAGE_TRACE = 1,
  OLC_STAGE_RESTIR = 2,
  OLC_STAGE_SHADE = 3,
  OLC_STAGE_SHADOW = 4,
  OLC_STAGE_ACCUMULATE = 5,
  OLC_STAGE_RESOLVE = 6,
  OLC_STAGE_SORT = 7
};
typedef struct olc_launch_record {
  uint32_t stage;
  uint32_t bounce;
  uint32_t chunk;
  uint32_t misses;
  uint64_t items;
  float ms;
  uint32_t reserved;
} olc_launch_record;
OLC_API int olc_frame_profile(const olc_context* ctx, olc_launch_record* records, uint32_t capacity,
                              uint32_t* count);

/* The CUDA stream (cudaStream_t) the context launches on, for callers that
 * time or order work against it. */
OLC_API int olc_stream(const olc_context* ctx, void** stream);

/* ---- tracing primitives (parity and tests) --------------------------- */

/* Closest hit of n world-space rays against the resident scene.  Device
 * arrays: origins/directions [n*3] float32; outputs instance_id (Mesh.id,
 * 0xffffffff on miss), primitive (packed triangle index as in
 * Scene.triangles(), -1 on miss), t (inf on miss).  t_min applies strictly
 * (t > t_min).  Equal-t ties resolve to the lowest packed index, the rule of
 * ReferencePathTracer._intersect (path_tracer.py:154-176). */
OLC_API int olc_trace_closest(olc_context* ctx, uint32_t n, const float* origins,
                      const float* directions, float t_min,
                      uint32_t* instance_id, int32_t* primitive, float* t,
                      float* barycentrics);

/* Occlusion of n rays on (t_min, t_max[i]): occluded[i] = 1 if any hit. */
OLC_API int olc_trace_occluded(olc_context* ctx, uint32_t n, const float* origins,
                       const float* directions, float t_min,
                       const float* t_max, uint8_t* occluded);

/* Camera rays of one sample (device outputs origins/directions [w*h*3]) using
 * the renderer's counter-based jitter; jitter_override (host, may be NULL)
 * replaces the random jitter with a fixed (jx, jy) for every pixel. */
OLC_API int olc_camera_rays(olc_context* ctx, const olc_camera* camera, uint32_t width,
                    uint32_t height, uint32_t sample, uint32_t frame_index,
                    const float* jitter_override, float* origins,
                    float* directions);

/* ---- LBVH building blocks (exposed for bit-exact tests) --------------- */

/* 30-bit Morton codes of the AABB centres of n triangles (device arrays:
 * tri_vertices [n*9] float32 as a,b,c; codes [n]). */
OLC_API int olc_morton_codes(olc_context* ctx, uint32_t n, const float* tri_vertices,
                     uint32_t* codes);

/* Stable LSD radix sort of (key, value) pairs on the low key_bits bits.
 * Device arrays; in place (keys/values are overwritten with the sorted
 * sequence).  Ties keep input order, matching numpy.argsort(kind="stable"). */
OLC_API int olc_radix_sort_pairs(olc_context* ctx, uint32_t n, uint32_t key_bits,
                         uint32_t* keys, uint32_t* values);

/* Allocation-free variant of olc_radix_sort_pairs, for callers that must not
 * allocate device memory when they sort: code running while a stream is
 * captured into a CUDA graph, serving loops held to a fixed memory budget,
 * and hosts whose device allocator belongs to another runtime.  It needs no
 * context and calls no allocator: its scratch is one file-scope device array
 * of the library (about 8.5 MB per device that loads the library, held until
 * the process exits).  Limit: n <= 1048576 pairs per call (larger n returns
 * OLC_ERR_VALUE).  Asynchronous on `stream` (a cudaStream_t; NULL is the
 * default stream); message of a failure from olc_last_error(NULL).  The first
 * call on a device looks up the array's device address and should come before
 * any stream capture on that device.  All calls on a device share the array,
 * so calls whose device work overlaps race: order them on one stream.
 * This entry point has no counterpart in the reference. */
OLC_API int olc_radix_sort_pairs_noalloc(uint32_t n, uint32_t key_bits, uint32_t* keys, uint32_t* values,
                                         void* stream);

/* Statistics of the resident acceleration structure (host outputs). */
typedef struct olc_bvh_info {
  uint32_t blas_count;
  uint32_t blas_nodes;
  uint32_t tlas_nodes;
  uint32_t triangles;
  uint32_t max_depth;
  uint32_t reserved[3];
  double build_ms;
} olc_bvh_info;
OLC_API int olc_bvh_info_get(const olc_context* ctx, olc_bvh_info* info);

/* Verify the resident BVH: every triangle reachable once and every child box
 * inside its parent.  bad (host) receives the number of violations. */
OLC_API int olc_bvh_validate(olc_context* ctx, uint64_t* bad);

#ifdef __cplusplus
}
#endif

#endif /* OLCUDA_H */
