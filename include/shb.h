/*
 * shb.h - C ABI of the B200-native SH9 lightmap bake.
 *
 * This is the drop-in boundary for the bake hot path of sh-baker:
 *   RasterizeScene        (src/rasterizer.h:27-28)   -> shb_rasterize
 *   CreateValidityMask    (src/rasterizer.h:31-32)   -> shb_validity_mask
 *   DownsampleValidityMask(src/rasterizer.h:37-39)   -> shb_downsample_validity_mask
 *   BuildBVH / ReleaseBVH (src/scene.h:128-132)      -> shb_scene_upload / shb_scene_destroy
 *   FindOcclusion         (src/occlusion.h:27)       -> shb_find_occlusion (batched)
 *   BakeSHLightMap        (src/baker.h:25-28)        -> shb_bake
 *   DownsampleSHTexture   (src/baker.h:31)           -> shb_downsample (channels = 27)
 *   DownsampleEnvironmentVisibilityTexture
 *                         (src/baker.h:35-36)        -> shb_downsample (channels = 1)
 *   Dilate<T>             (src/dilation.h:14-16)     -> shb_dilate (kind = SH9 / F32 / U8)
 *   SaveSHLightMap        (src/saver.h:45-48)        -> shb_save_sh_lightmap
 *   LoadScene             (src/loader.h)             -> shb_load_gltf
 *
 * Plain C types only: host pointers are owned by the caller, device objects
 * are owned by the opaque handles.  Every entry point returns a shb_status;
 * shb_last_error() returns a thread-local message for the last failure.
 * One context owns one CUDA stream; use one context per host thread.
 * Entry points run on their context's device and give the calling thread
 * its previous current device back before they return.
 * Image arguments hold at most 2^31 - 1 texels (the G-buffer limit of
 * shb_rasterize) and shb_find_occlusion takes at most 2^31 - 1 rays per
 * call; larger sizes are SHB_ERR_INVALID_ARG.  A scene holds at most
 * 2^30 - 1 vertices, 2^30 - 1 triangles and 2^26 - 1 geometries, an albedo
 * texture at most 2^31 - 1 bytes and all of a scene's at most 2^32 - 1.
 *
 * Memory layouts are binary compatible with the reference's Eigen structs:
 *   shb_surface_point == sh_baker::SurfacePoint (64 bytes, Vector4f 16-byte
 *   aligned), an SH texel is 27 floats == sh_baker::SHCoeffs (9 x RGB).
 */
#ifndef SHB_H_
#define SHB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define SHB_API __declspec(dllexport)
#else
#define SHB_API __attribute__((visibility("default")))
#endif

#define SHB_ABI_VERSION 1

/* Every device loop and queue is bounded.  A bounded loop that runs out
 * (a ray's traversal steps) sets a device error flag and returns; the host
 * maps it to SHB_ERR_TIMEOUT.  A bounded capacity that is exceeded (the
 * traversal stack, a ray queue) maps to SHB_ERR_INTERNAL.  Either way the
 * kernels end, the context stays usable and shb_bake_stats.error_flags
 * holds the flags (1 stack, 2 queue, 4 traversal steps). */
typedef enum shb_status {
  SHB_OK = 0,
  SHB_ERR_INVALID_ARG = 1,
  SHB_ERR_OOM = 2,
  SHB_ERR_CUDA = 3,
  SHB_ERR_TIMEOUT = 4,
  SHB_ERR_INTERNAL = 5,
  SHB_ERR_NO_DEVICE = 6
} shb_status;

/* ---- scene description (mirrors src/scene.h:18-115) -------------------- */

/* Light::Type order of src/scene.h:71. */
typedef enum shb_light_type {
  SHB_LIGHT_POINT = 0,
  SHB_LIGHT_DIRECTIONAL = 1,
  SHB_LIGHT_SPOT = 2,
  SHB_LIGHT_AREA = 3
} shb_light_type;

/* One sh_baker::Geometry (src/scene.h:56-67), structure-of-arrays. */
typedef struct shb_geometry_desc {
  const float* vertices;     /* 3 * vertex_count, object space            */
  const float* normals;      /* 3 * vertex_count or NULL                   */
  const float* texture_uvs;  /* 2 * vertex_count or NULL                   */
  const float* lightmap_uvs; /* 2 * vertex_count or NULL (raster needs it) */
  const float* tangents;     /* 4 * vertex_count (xyz + sign) or NULL      */
  uint32_t vertex_count;
  const uint32_t* indices;   /* index_count, triangles                     */
  uint32_t index_count;
  int32_t material_id;       /* index into materials, -1 = none            */
  float transform[12];       /* Affine3f as row-major 3x4 [L | t]          */
} shb_geometry_desc;

/* One sh_baker::Material (src/scene.h:43-53); only the albedo texture and
 * the emission intensity are read by the bake (src/material.cpp:57-92). */
typedef struct shb_material_desc {
  const uint8_t* albedo_pixels; /* w*h*channels sRGB bytes or NULL        */
  uint32_t albedo_width;
  uint32_t albedo_height;
  uint32_t albedo_channels;     /* 3 or 4 (4 = alpha in A)                */
  float emission_intensity;
} shb_material_desc;

/* One sh_baker::Light (src/scene.h:70-87). */
typedef struct shb_light_desc {
  int32_t type; /* shb_light_type */
  float position[3];
  float direction[3];
  float color[3];
  float intensity;
  float cos_inner_cone;
  float cos_outer_cone;
  float area;
  int32_t material_index; /* area lights: Light::material            */
  int32_t geometry_index; /* area lights: Light::geometry_index      */
} shb_light_desc;

typedef struct shb_scene_desc {
  const shb_geometry_desc* geometries;
  uint32_t geometry_count;
  const shb_material_desc* materials;
  uint32_t material_count;
  const shb_light_desc* lights;
  uint32_t light_count;
} shb_scene_desc;

/* ---- raster / bake types (src/rasterizer.h:12-23, src/baker.h:10-19) ---- */

typedef struct shb_raster_config {
  int32_t width;
  int32_t height;
  int32_t supersample_scale;
} shb_raster_config;

/* sh_baker::SurfacePoint, 64 bytes, same offsets as the Eigen layout. */
typedef struct shb_surface_point {
  float position[3];
  float normal[3];
  float _pad0[2];
  float tangent[4];
  int32_t material_id; /* invalid if < 0 */
  int32_t _pad1[3];
} shb_surface_point;

typedef enum shb_rng_mode {
  SHB_RNG_PHILOX = 0 /* counter-based Philox4x32-10 stream */
} shb_rng_mode;

typedef struct shb_bake_config {
  int32_t samples;           /* BakeConfig::samples (default 128)          */
  int32_t bounces;           /* BakeConfig::bounces (default 3)            */
  int32_t num_light_samples; /* BakeConfig::num_light_samples (default 1)  */
  uint32_t seed;             /* RNG stream id (reference: fixed 12345+idx) */
  int32_t sample_offset;     /* first sample index (for split bakes)       */
  int32_t rng_mode;          /* shb_rng_mode                               */
  int32_t reserved[2];
} shb_bake_config;

/* Output of shb_bake.  Buffers are W*s x H*s texels (the supersampled size,
 * as BakeSHLightMap returns, src/baker.cpp:198-216).  sh: 27 floats per
 * texel (coeff-major RGB), env_visibility: 1 float per texel.  With
 * device_ptrs != 0 both pointers are CUDA device pointers on the context's
 * device, else host pointers. */
typedef struct shb_bake_output {
  float* sh;
  float* env_visibility;
  int32_t device_ptrs;
  int32_t reserved;
} shb_bake_output;

/* Ray / hit of FindOcclusion (src/occlusion.h:11-23). */
typedef struct shb_ray {
  float origin[3];
  float direction[3];
  float tnear;
  float tfar;
} shb_ray;

typedef struct shb_hit {
  float position[3];
  float uv[2];
  float normal[3];
  int32_t material_id;
  int32_t hit;          /* 0 = miss (nullopt) */
  float t;
  uint32_t prim_id;     /* global triangle id (geometry-major order) */
} shb_hit;

/* Per-bake counters filled by shb_bake when stats != NULL. */
typedef struct shb_bake_stats {
  uint64_t texel_samples;  /* valid texels x samples                      */
  uint64_t valid_texels;
  uint64_t extend_rays;    /* closest-hit rays traced                     */
  uint64_t shadow_rays;    /* any-hit rays traced                         */
  uint64_t kernel_launches;
  uint32_t error_flags;    /* device-side bounded-failure flags (0 = ok)  */
  uint32_t waves;
  double bvh_build_ms;     /* filled when profiling is on                 */
  double trace_ms;
  double extend_kernel_ms; /* sum of closest-hit kernel durations         */
  double shadow_kernel_ms;
  double shade_kernel_ms;   /* generate + shade + resolve kernel durations   */
  uint64_t extend_launches;
  uint64_t shadow_launches;
} shb_bake_stats;

typedef enum shb_dilate_kind {
  SHB_DILATE_SH9 = 0, /* 27 floats per texel (Dilate<SHCoeffs>) */
  SHB_DILATE_F32 = 1, /* 1 float per texel    (Dilate<float>)    */
  SHB_DILATE_U8 = 2   /* 1 byte per texel     (Dilate<uint8_t>)  */
} shb_dilate_kind;

typedef struct shb_options {
  int32_t device;      /* CUDA device ordinal                          */
  int32_t profiling;   /* 1: time kernel classes with CUDA events      */
  int32_t reserved[6];
} shb_options;

typedef struct shb_context shb_context;
typedef struct shb_scene shb_scene;
typedef struct shb_gbuffer shb_gbuffer;

/* ---- lifetime --------------------------------------------------------- */

SHB_API int32_t shb_abi_version(void);
SHB_API const char* shb_last_error(void);

/* Test hook (no counterpart in the reference): from now on, the device
 * allocation the library makes after `n` more successful ones fails with
 * SHB_ERR_OOM, once; n < 0 turns the hook off.  Host side only: the
 * allocation is refused before cudaMalloc is called. */
SHB_API void shb_test_fail_allocation_after(int32_t n);

/* SRGBToLinear (src/colorspace.h:10-14) of every 8-bit value, the table
 * GetAlbedo (src/material.cpp:69-85) reads: out[256] floats.  Host only. */
SHB_API void shb_srgb_to_linear_table(float* out);
SHB_API shb_status shb_context_create(const shb_options* options,
                                      shb_context** out);
/* Releases the handle and the context's scratch memory.  Scenes and
 * G-buffers made from the context keep it alive until they are destroyed,
 * in any order; the handle must not be used again. */
SHB_API shb_status shb_context_destroy(shb_context* ctx);
/* Replaces the context's stream with a caller-owned cudaStream_t (or 0 for
 * the context's own stream). */
SHB_API shb_status shb_context_set_stream(shb_context* ctx, void* stream);
SHB_API shb_status shb_context_synchronize(shb_context* ctx);
/* Number of kernels this context has launched so far. */
SHB_API uint64_t shb_context_kernel_launches(const shb_context* ctx);

/* Uploads the scene and builds the GPU BVH (binned SAH, compressed 8-wide
 * nodes).  Replaces BuildBVH (src/scene.cpp:209-262); the reference builds
 * it inside every BakeSHLightMap call (src/baker.cpp:258-259). */
SHB_API shb_status shb_scene_upload(shb_context* ctx, const shb_scene_desc* desc,
                                    shb_scene** out);
SHB_API shb_status shb_scene_destroy(shb_scene* scene);
/* Rebuilds the BVH of an uploaded scene (times the builder alone). */
SHB_API shb_status shb_scene_rebuild_bvh(shb_scene* scene);
SHB_API shb_status shb_scene_bvh_info(const shb_scene* scene, uint32_t* wide_nodes,
                                      uint32_t* triangles, uint32_t* depth);

/* The rotation that TransformedNormals / TransformedTangents
 * (src/scene.cpp:171-195) apply: the rotation part of a geometry's
 * transform (row-major 3x4 [L | t], as in shb_geometry_desc), that is
 * Eigen's Transform::rotation(), the orthogonal factor of L's polar
 * decomposition with a positive determinant; row-major 3x3 out.  The same
 * rotation the library applies to normals and tangents on upload.  Host
 * code only. */
SHB_API shb_status shb_rotation_part(const float transform[12], float rotation[9]);

/* ---- RasterizeScene (src/rasterizer.cpp:68-211) ----------------------- */

/* Rasterises every triangle's lightmap UVs into a (W*s) x (H*s) texel
 * G-buffer.  host_out (nullable) receives W*s*H*s surface points;
 * out_gbuffer (nullable) receives the device-resident G-buffer handle. */
SHB_API shb_status shb_rasterize(shb_scene* scene, const shb_raster_config* cfg,
                                 shb_surface_point* host_out,
                                 shb_gbuffer** out_gbuffer);
/* Device G-buffer from caller surface points (BakeSHLightMap takes them as
 * an argument, src/baker.h:25-28).  width/height are the texel dims. */
SHB_API shb_status shb_gbuffer_upload(shb_context* ctx, const shb_surface_point* points,
                                      int32_t width, int32_t height,
                                      shb_gbuffer** out);
SHB_API shb_status shb_gbuffer_download(const shb_gbuffer* g, shb_surface_point* points);
SHB_API shb_status shb_gbuffer_dims(const shb_gbuffer* g, int32_t* width, int32_t* height);
SHB_API shb_status shb_gbuffer_destroy(shb_gbuffer* g);

/* ---- CreateValidityMask / DownsampleValidityMask ---------------------- */

/* mask_out: width*height bytes (device pointer if device_ptr != 0). */
SHB_API shb_status shb_validity_mask(shb_context* ctx, const shb_gbuffer* g,
                                     uint8_t* mask_out, int32_t device_ptr);
/* src/rasterizer.cpp:222-241: out[y*w+x] = any(in block).  in: (w*s)x(h*s). */
SHB_API shb_status shb_downsample_validity_mask(shb_context* ctx, const uint8_t* in,
                                                int32_t width, int32_t height,
                                                int32_t scale, uint8_t* out,
                                                int32_t device_ptrs);

/* ---- BakeSHLightMap (src/baker.cpp:186-304) --------------------------- */

/* raster_cfg gives the base size and supersample scale of the G-buffer, as
 * in the reference; the G-buffer must be (W*s) x (H*s). */
SHB_API shb_status shb_bake(shb_scene* scene, const shb_gbuffer* g,
                            const shb_raster_config* raster_cfg,
                            const shb_bake_config* cfg, shb_bake_output* out,
                            shb_bake_stats* stats);

/* ---- batched bakes ------------------------------------------------------
 * Many independent BakeSHLightMap calls (different scenes, sizes, spp and
 * bounces) run through one shared sequence of wavefront launches: their
 * texels are cut into (bake, texel tile) work items that the host packs into
 * waves, small bakes sharing a wave, and each wave runs its per-depth
 * traversal and shading launches once for all of its paths; with use_graph
 * the whole launch sequence is captured in one CUDA graph.  Results are
 * bit-identical to one shb_bake call per item.  All scenes must belong to
 * `ctx`; outputs are device pointers of W*s x H*s texels. */
typedef struct shb_batch_item {
  shb_scene* scene;
  const shb_gbuffer* gbuffer;
  shb_raster_config raster;
  shb_bake_config config;
  float* sh;              /* device, 27 floats per texel */
  float* env_visibility;  /* device, 1 float per texel */
} shb_batch_item;

typedef struct shb_batch_options {
  int32_t use_graph;    /* 1: capture the waves in one CUDA graph            */
  int32_t autotune;     /* 1: pick wave/share/tile/grid per shape class,
                           cached                                          */
  int32_t wave_paths;   /* paths per wave (0: default or tuned)             */
  int32_t tile_texels;  /* texels per work tile (0: default or tuned)       */
  int32_t grid_scale;   /* traversal grid multiplier (0: default or tuned)  */
  int32_t share_paths;  /* bakes of fewer paths share waves with others;
                           larger ones get waves of their own (0: default
                           or tuned, which is half a wave; -1: no sharing) */
  int32_t nee_split;    /* next-event estimation of the forward bake: 0 its
                           own kernel where the light loop is long (punctual
                           lights + 4 x area lights >= 16), 1 inline in the
                           hit kernel, 2 its own kernel; results are
                           bit-identical either way                        */
  int32_t max_traversal_steps; /* bound of the traversal loop of one ray
                           (0: 4,194,304); a ray that reaches it ends the
                           bake with SHB_ERR_TIMEOUT                        */
  const char* tune_cache; /* tuning file; NULL: $SHB_TUNE_CACHE or
                             $HOME/.cache/sh_baker_b200/autotune.txt        */
  int32_t queue_capacity; /* entries of each ray queue (0: sized to the
                           wave); a smaller capacity drops the rays that do
                           not fit and ends the bake with SHB_ERR_INTERNAL */
  int32_t reserved[3];
} shb_batch_options;

SHB_API shb_status shb_bake_batch(shb_context* ctx, const shb_batch_item* items, int32_t count,
                                  const shb_batch_options* options, shb_bake_stats* stats);

/* ---- Differentiable bake (no counterpart in the reference) ------------ */

/* Adjoint parameters.  albedo_rgb (material_count x 3, nullable): a linear
 * base colour that replaces the albedo texture lookup of every material with
 * use_override[m] != 0 (use_override NULL: all materials; alpha still comes
 * from the texture).  light_intensity (light_count, nullable) replaces
 * shb_light_desc.intensity.  Materials without an override keep their
 * texture and get no gradient.  The BVH is not rebuilt. */
SHB_API shb_status shb_scene_set_params(shb_scene* scene, const float* albedo_rgb,
                                        const uint8_t* use_override, const float* light_intensity);

/* Path-replay adjoint of shb_bake with the same G-buffer and config:
 * regenerates every path from its counter-based random stream (nothing is
 * stored by the forward bake) and accumulates, for Loss with
 * dLoss/dSH = d_sh (27 floats per texel of the W*s x H*s G-buffer; device
 * memory when device_ptr, else host):
 *   d_albedo[3m + c] = dLoss / d albedo_rgb[3m + c]  (override materials,
 *                      through reflection, hit NEE, depth-0 emission and
 *                      area-light emission; 0 elsewhere)
 *   d_light[l]       = dLoss / d intensity of point, spot and directional
 *                      lights (area lights: 0, their radiance is the
 *                      emissive material's albedo x emission)
 * as host arrays.  Light-selection probabilities are held constant (the
 * estimator of the gradient of the expected bake).  At most 16 bounces and
 * 12288 parameters (3 x materials + lights). */
SHB_API shb_status shb_backward(shb_scene* scene, const shb_gbuffer* gbuffer,
                                const shb_raster_config* raster, const shb_bake_config* config,
                                const float* d_sh, int32_t device_ptr, double* d_albedo,
                                double* d_light, shb_bake_stats* stats);

/* ---- DownsampleTexture (src/baker.cpp:151-182) ------------------------ */

/* Box average over scale x scale blocks including invalid texels; channels
 * = 27 for SH, 1 for env visibility.  out: (in_w/scale) x (in_h/scale). */
SHB_API shb_status shb_downsample(shb_context* ctx, const float* in, int32_t in_width,
                                  int32_t in_height, int32_t channels, int32_t scale,
                                  float* out, int32_t device_ptrs);

/* ---- Dilate<T> (src/dilation.cpp:7-73) -------------------------------- */

/* pixels and mask are updated in place, like the reference. */
SHB_API shb_status shb_dilate(shb_context* ctx, int32_t kind, int32_t width,
                              int32_t height, void* pixels, uint8_t* mask,
                              int32_t passes, int32_t device_ptrs);

/* Dilation that allocates nothing.  No counterpart in the reference: it
 * exists for callers that cannot allocate device memory while they run (a
 * host application that owns and pre-reserves the GPU's memory, or a path
 * with a deadline where cudaMalloc's implicit synchronisation is not
 * acceptable).  Same passes and results as shb_dilate on device pointers
 * (pixels and mask on the context's device, updated in place).  The
 * ping-pong scratch lives in one fixed 16 MiB array inside the library.
 * Its device address is looked up by shb_context_create, so every device
 * that has had a context holds the array from then until the process
 * exits, and this call itself neither loads code nor reserves memory.  At
 * most about 153,000 texels of SH9, 3.3 million of float or 8.3 million of
 * uint8, and at most 4096 passes; larger requests return
 * SHB_ERR_INVALID_ARG.  The call only enqueues work on the context's
 * stream and returns: the results are ready once that stream has been
 * synchronised.  All calls share the array, so calls that overlap on the
 * GPU (other contexts, host threads or streams) race and must be ordered
 * by the caller; calls on one context's stream are ordered by the stream.
 * The calling thread's current device is the same on return. */
SHB_API shb_status shb_dilate_noalloc(shb_context* ctx, int32_t kind, int32_t width,
                                      int32_t height, void* pixels, uint8_t* mask,
                                      int32_t passes);

/* ---- the CLI's bake sequence (src/main.cpp:91-163) -------------------- */

typedef struct shb_pipeline_config {
  int32_t width;             /* --width  */
  int32_t height;            /* --height */
  int32_t supersample_scale; /* --supersample_scale */
  int32_t samples;           /* --samples */
  int32_t bounces;           /* --bounces */
  int32_t dilation;          /* --dilation (passes) */
  int32_t num_light_samples;
  uint32_t seed;
} shb_pipeline_config;

/* RasterizeScene -> BakeSHLightMap -> CreateValidityMask -> (s > 1)
 * DownsampleSHTexture / DownsampleEnvironmentVisibilityTexture /
 * DownsampleValidityMask -> (dilation > 0) Dilate(SH) then Dilate(env) with
 * the mask the first Dilate already updated, all on the device.  Host
 * outputs at width x height: sh (27 floats per texel), env_visibility,
 * mask (nullable).  The supersampled G-buffer and the intermediate
 * textures stay allocated in the context for the next call (released by
 * shb_context_destroy). */
SHB_API shb_status shb_bake_pipeline(shb_scene* scene, const shb_pipeline_config* cfg,
                                     float* sh_out, float* env_out, uint8_t* mask_out,
                                     shb_bake_stats* stats);

/* ---- SaveSHLightMap (src/saver.h:45-48, src/saver.cpp:108-401) -------- */

/* SaveMode (src/saver.h:21-25). */
typedef enum shb_save_mode {
  SHB_SAVE_COMBINED = 0,          /* one 28-channel file: L0.R .. L22.B, EnvVisibility */
  SHB_SAVE_SPLIT_CHANNELS = 1,    /* <stem>_L0 (RGB + A = env) .. <stem>_L22 (RGB)     */
  SHB_SAVE_LUMINANCE_PACKED = 2   /* <stem>_packed_0..2: L0 RGB + env; Rec. 709 luma of
                                     L1m1..L2m2; luma of L2m1..L22 (RGBA each)           */
} shb_save_mode;

/* Writes the SH lightmap (width x height texels of 27 floats) and the
 * environment visibility (nullable: written as 0) as OpenEXR, half storage,
 * ZIP compression, the files and channel names of the reference.  Device
 * pointers when device_ptrs, else host.  Empty dimensions are
 * SHB_ERR_INVALID_ARG (the reference logs and returns false). */
SHB_API shb_status shb_save_sh_lightmap(shb_context* ctx, const float* sh, const float* env,
                                        int32_t width, int32_t height, int32_t device_ptrs,
                                        const char* path, int32_t mode);

/* ---- SH previews (src/sh_cvt_main.cpp, glsl/viz.frag:42-99 as math) ---- */

typedef enum shb_preview_mode {
  SHB_PREVIEW_L0 = 0,        /* L0 coefficient as RGB (the EXR -> PNG tool)        */
  SHB_PREVIEW_SH = 1,        /* max(0, SH9 radiance towards the direction)          */
  SHB_PREVIEW_SH_PACKED = 2  /* the same from L0 + Rec. 709 luminance of L1/L2,
                                re-coloured with L0's chroma (luminance-packed) */
} shb_preview_mode;

/* width x height texels of 27 floats -> width x height x 3 bytes of
 * clamp(v) * 255 + 0.5 (optionally after Reinhard v / (1 + v)).  The
 * direction is normals[3 * texel] when normals != NULL (same memory kind
 * as sh), else direction[0..2].  sh / normals are device pointers when
 * device_ptrs, else host; rgb_out is always host memory. */
SHB_API shb_status shb_sh_preview(shb_context* ctx, const float* sh, int32_t width, int32_t height,
                                  const float* normals, const float direction[3], int32_t mode,
                                  int32_t reinhard, int32_t device_ptrs, uint8_t* rgb_out);

/* The named channels of a single-part scanline OpenEXR file (NONE, ZIPS or
 * ZIP compression; HALF, FLOAT or UINT samples) as float planes, count x
 * width x height (host); with out == NULL only width and height are
 * filled.  A missing channel is SHB_ERR_INVALID_ARG.  (The reference reads
 * EXR through tinyexr, src/sh_cvt_main.cpp:27-59.) */
SHB_API shb_status shb_exr_load_channels(const char* path, const char* const* names, int32_t count,
                                         int32_t* width, int32_t* height, float* out);

/* SaveTexture (src/saver.cpp:783-795): an 8-bit PNG of 1 to 4 channels. */
SHB_API shb_status shb_write_png(const char* path, int32_t width, int32_t height, int32_t channels,
                                 const uint8_t* pixels);

/* ---- LoadScene (src/loader.h, src/loader.cpp:144-844) ------------------ */

/* A scene read from a .gltf / .glb file and owned by the handle; its
 * shb_scene_desc (valid until shb_host_scene_destroy) feeds
 * shb_scene_upload.  Missing material / POSITION / NORMAL / TEXCOORD_0 on a
 * primitive, an unreadable file or an unsupported texture (neither PNG nor
 * Huffman-coded JPEG) are SHB_ERR_INVALID_ARG (the reference returns nullopt).
 * Emissive primitives become area lights; TEXCOORD_1 becomes the lightmap
 * UVs; a primitive without TANGENT gets tangents by the MikkTSpace method,
 * as the reference generates them (src/loader.cpp:363-385). */
typedef struct shb_host_scene shb_host_scene;
SHB_API shb_status shb_load_gltf(const char* path, shb_host_scene** out);
SHB_API const shb_scene_desc* shb_host_scene_desc(const shb_host_scene* scene);
SHB_API shb_status shb_host_scene_destroy(shb_host_scene* scene);
/* A loaded material's name and the absolute path of its albedo image file
 * (NULL when the albedo is not an external file); valid with the handle. */
SHB_API shb_status shb_host_scene_material_info(const shb_host_scene* scene, int32_t material,
                                                const char** name, const char** albedo_file);

/* SaveScene (src/saver.h:50-53, src/saver.cpp:423-781): writes `path`
 * (.gltf) and <stem>.bin beside it; albedo image files are copied next to
 * it.  material_names / albedo_files: one entry per material or NULL. */
SHB_API shb_status shb_save_gltf(const shb_scene_desc* scene, const char* const* material_names,
                                 const char* const* albedo_files, const char* path);

/* ---- CreateAtlasGeometries (src/atlas.h:28-53, src/atlas.cpp:95-250) --- */

/* atlas_internal::CalculateGeometryScales (src/atlas.h:22-24,
 * src/atlas.cpp:21-93): per geometry density * sqrt(albedo w*h) *
 * sqrt(texture-UV tile count), clamped to 5x the median.  scales_out holds
 * geometry_count floats.  A geometry without texture UVs or with a
 * material_id out of range is SHB_ERR_INVALID_ARG (the reference CHECKs). */
SHB_API shb_status shb_atlas_geometry_scales(const shb_scene_desc* scene, float density_multiplier,
                                             float* scales_out);

/* New lightmap UVs for every geometry, non-overlapping, in one page of
 * target_resolution^2 texels with at least `padding` empty texels between
 * charts.  Vertices on chart seams are split; each output vertex keeps the
 * position, normal, tangent and texture UV of its source vertex; faces keep
 * their order.  The result (geometries, copied materials and lights) is a
 * host scene owned by *out; width and height receive the page size.
 * Charts that cannot fit the page, an empty scene, or geometries without
 * texture UVs, normals or tangents are SHB_ERR_INVALID_ARG (the reference
 * returns nullopt or CHECKs).  xatlas is not used: the charts are built by
 * this library, so UVs differ from the reference's while keeping its
 * contract. */
SHB_API shb_status shb_create_atlas(const shb_scene_desc* scene, uint32_t target_resolution, uint32_t padding,
                                    float density_multiplier, shb_host_scene** out, int32_t* width,
                                    int32_t* height);

/* ---- FindOcclusion (src/occlusion.cpp:9-107), batched ----------------- */

SHB_API shb_status shb_find_occlusion(shb_scene* scene, const shb_ray* rays,
                                      int64_t count, shb_hit* hits,
                                      int32_t device_ptrs);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SHB_H_ */
