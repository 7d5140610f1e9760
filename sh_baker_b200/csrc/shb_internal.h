// shb_internal.h - host/device data structures shared by the CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/shb.h"

#define SHB_HD __host__ __device__ __forceinline__

namespace shb {

// ------------------------------------------------------------ errors ------

void set_error(const std::string& msg);
shb_status cuda_fail(cudaError_t e, const char* what);

// Runs the body of a C ABI entry point so that no C++ exception leaves it:
// a failed host allocation becomes SHB_ERR_OOM and any other exception
// SHB_ERR_INTERNAL, with its message in shb_last_error().  A C, ctypes or
// cgo caller cannot unwind a C++ exception.
template <class F>
shb_status guarded(const char* entry, F&& body) noexcept {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    try { set_error(std::string(entry) + ": host allocation failed"); } catch (...) {}
    return SHB_ERR_OOM;
  } catch (const std::exception& e) {
    try { set_error(std::string(entry) + ": " + e.what()); } catch (...) {}
    return SHB_ERR_INTERNAL;
  } catch (...) {
    try { set_error(std::string(entry) + ": unknown exception"); } catch (...) {}
    return SHB_ERR_INTERNAL;
  }
}

// Runs `work` on up to `threads` host threads, the calling one included,
// and joins them.  `work` must claim its items from a shared counter, so
// that any number of threads finishes them.  A std::thread that ends with
// an exception, or is destroyed unjoined, terminates the process, so an
// exception of any thread is kept and rethrown here once all have joined
// (for guarded to map), and a thread that cannot be started is skipped.
template <class F>
void run_host_threads(unsigned threads, F&& work) {
  std::mutex m;
  std::exception_ptr first;
  auto body = [&] {
    try {
      work();
    } catch (...) {
      std::lock_guard<std::mutex> lock(m);
      if (!first) first = std::current_exception();
    }
  };
  std::vector<std::thread> pool;
  try {
    pool.reserve(threads > 1 ? threads - 1 : 0);
    for (unsigned t = 1; t < threads; ++t) pool.emplace_back(body);
  } catch (...) {
    // fewer threads: those started, and this one, claim every item
  }
  body();
  for (auto& t : pool) t.join();
  if (first) std::rethrow_exception(first);
}

#define SHB_CUDA(call)                                             \
  do {                                                             \
    cudaError_t _e = (call);                                       \
    if (_e != cudaSuccess) return ::shb::cuda_fail(_e, #call);     \
  } while (0)

// Makes `dev` the calling thread's current device for the rest of the
// scope and gives the thread its previous current device back on exit, so
// that entry points of the C ABI leave the caller's device selection as
// they found it.
struct DeviceScope {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceScope(int dev) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) cur = -1;
    if (cur == dev) return;
    status = cudaSetDevice(dev);
    if (status == cudaSuccess) prev = cur;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};

// DeviceScope for the rest of the enclosing function; returns SHB_ERR_CUDA
// when the device cannot be made current.
#define SHB_ON_DEVICE(dev)                                                       \
  ::shb::DeviceScope _shb_device_scope(dev);                                     \
  do {                                                                           \
    if (_shb_device_scope.status != cudaSuccess)                                 \
      return ::shb::cuda_fail(_shb_device_scope.status, "cudaSetDevice");        \
  } while (0)

#define SHB_TRY(call)                      \
  do {                                     \
    shb_status _s = (call);                \
    if (_s != SHB_OK) return _s;           \
  } while (0)

// --------------------------------------------------------- device buffer --

// Owning device allocation (cudaMalloc), grown on demand, never shrunk.
// Device blocks given back by DevBuf::release are kept per device for reuse
// (shb_capi.cu) instead of being returned with cudaFree, which on shared
// machines has stalled the calling thread for up to a second.  A release
// first waits for the device, as cudaFree does, so a cached block is never
// still read or written by queued work when it is handed out again.
void block_release(int dev, void* ptr, size_t bytes);

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  int dev = -1;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) block_release(dev, ptr, bytes);
    ptr = nullptr;
    bytes = 0;
  }
  shb_status reserve(size_t n);  // keeps no contents
  void swap(DevBuf& o) {  // exchanges the blocks with their sizes
    std::swap(ptr, o.ptr);
    std::swap(bytes, o.bytes);
    std::swap(dev, o.dev);
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
};

// -------------------------------------------------------------- scene -----

struct DGeom {
  uint32_t vbase;      // first vertex in the global vertex arrays
  uint32_t prim_base;  // first triangle in global (geometry-major) order
  uint32_t tri_count;
  int32_t material_id;
  uint32_t flags;      // GEOM_* bits
  uint32_t pad[3];
};
enum : uint32_t { GEOM_HAS_NORMALS = 1, GEOM_HAS_TEXUV = 2, GEOM_HAS_TANGENTS = 4, GEOM_HAS_LMUV = 8 };

struct DMat {
  uint32_t pix_offset;
  uint32_t w, h, c;    // c == 0: no albedo texture (default 0.8 grey)
  float emission;
  int32_t use_override;  // 1: albedo := override (linear), adjoint parameter
  float override_rgb[3];
  float pad;
};

struct DLight {
  int32_t type;
  float px, py, pz;
  float dx, dy, dz;
  float cr, cg, cb;
  float intensity;
  float cos_inner, cos_outer;
  int32_t geom;      // area: geometry index
  int32_t mat;       // area: material index
  int32_t area_ord;  // area: ordinal among area lights (RNG slots)
  // area: emission when it is the same at every point (the material's
  // albedo is untextured, a 1x1 texture or an override), computed on the
  // host with the device's operations; emis_const 0: look it up per sample
  float er, eg, eb;
  int32_t emis_const;
  // area: the light's first triangle record (shade.cu sample_area) and its
  // triangle count | has-texture-uv << 31, so a sample reads them with the
  // light instead of from a separate table
  uint32_t area_first, area_count;
};

// Compressed 8-wide BVH node (80 bytes).  Children boxes are quantised on
// a per-node power-of-two grid anchored at p; slot s holds the child whose
// centroid lies in octant s of the parent (bit a set = positive side of
// axis a), so a ray visits slots in order i ^ octant(ray).
struct alignas(16) WideNode {
  float px, py, pz;
  uint32_t e_imask;   // ex | ey<<8 | ez<<16 | imask<<24
  uint32_t child_base;
  uint32_t tri_base;
  uint32_t meta_lo;   // meta of slots 0..3 (byte each)
  uint32_t meta_hi;   // meta of slots 4..7
  uint32_t qlo[6];    // qlo_x[8], qlo_y[8], qlo_z[8]
  uint32_t qhi[6];    // qhi_x[8], qhi_y[8], qhi_z[8]
};
static_assert(sizeof(WideNode) == 80, "WideNode must be 80 bytes");
// meta byte = count << 5 | position: the child contributes `count` bits
// from `position` to a node's hit mask.  Empty slot: 0.  Leaf: its
// triangle count and its first triangle's offset from tri_base (< 24).
// Internal child in slot s: count 1, position 24 + s (the traversal XORs s
// with the ray octant, so the hit mask's bits 24..31 are in visiting order).

struct BvhView {
  const WideNode* nodes;
  const float4* tris;   // 3 float4 per triangle in leaf order, v0.w = prim id
  uint32_t node_count;
  uint32_t tri_count;
};

struct SceneView {
  // per vertex (global)
  const float* obj_v;    // 3 per vertex
  const float* obj_n;    // 3 per vertex
  const float* tex_uv;   // 2 per vertex
  const float* world_v;  // 3 per vertex
  // per triangle (global order)
  const uint32_t* tri_vidx;  // 3 per triangle (global vertex ids)
  const uint32_t* tri_geom;  // geometry of each triangle
  const DGeom* geoms;
  const DMat* mats;
  const uint8_t* pixels;
  const DLight* lights;
  const float4* area_tris;  // 4 per area-light triangle (shade.cu sample_area)
  uint32_t geom_count, mat_count, light_count, area_light_count;
  uint32_t prim_count, vertex_count;
  int32_t has_alpha;     // any material with 4-channel albedo
};

}  // namespace shb

// Opaque handles of the C ABI.
struct shb_context {
  // One reference for the handle and one per live scene or G-buffer made
  // from it: shb_context_destroy drops the first, and the context (its
  // stream included) is freed when the last one goes, so destroying scenes
  // after their context stays valid.
  std::atomic<int> refs{1};
  int device = 0;
  int profiling = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  uint64_t launches = 0;
  // scratch reused across calls
  shb::DevBuf scratch[28];
  shb::DevBuf counters;
  // G-buffer of shb_bake_pipeline, kept between calls: allocating and
  // freeing hundreds of MB per call stalls the host for up to a second
  struct shb_gbuffer* pipe_gbuf = nullptr;
  void* host_pinned = nullptr;
  size_t host_pinned_bytes = 0;
};

struct shb_scene {
  shb_context* ctx = nullptr;
  // uploaded per-vertex arrays
  shb::DevBuf obj_v, obj_n, tex_uv, lm_uv, obj_t, world_v, world_n, world_t;
  shb::DevBuf tri_vidx, tri_geom, geoms, mats, pixels, lights, rot, lin, vgeom;
  shb::DevBuf area_tris;
  uint32_t vertex_count = 0, prim_count = 0, geom_count = 0, mat_count = 0, light_count = 0;
  uint32_t area_light_count = 0;
  int32_t has_alpha = 0;
  bool raster_ready = true;  // every geometry has normals, tangents, lightmap uvs
  std::string raster_error;
  std::vector<shb::DGeom> h_geoms;
  std::vector<shb::DMat> h_mats;      // host copies, edited by shb_scene_set_params
  std::vector<shb::DLight> h_lights;
  // per light: the albedo of a 1x1 or untextured material (3 floats) and
  // whether that albedo is constant, for the area-emission constants
  std::vector<float> h_light_albedo;
  std::vector<uint8_t> h_light_albedo_const;
  // BVH
  shb::DevBuf bvh_nodes, bvh_tris;
  uint32_t bvh_node_count = 0, bvh_tri_count = 0, bvh_depth = 0;
  double bvh_build_ms = 0.0;
  shb::SceneView view() const;
  shb::BvhView bvh() const;
};

struct shb_gbuffer {
  shb_context* ctx = nullptr;
  shb::DevBuf points;  // shb_surface_point per texel
  int32_t width = 0, height = 0;
};

namespace shb {

// Streaming multiprocessors of the calling thread's current device (cached
// per device); grids of the grid-stride kernels are sized in multiples of it.
int sm_count();

// launch bookkeeping
inline void count_launch(shb_context* c, uint64_t n = 1) { c->launches += n; }

// kernels implemented in the .cu files
shb_status transform_vertices(shb_scene* s);
shb_status build_bvh(shb_scene* s);
shb_status build_area_tris(shb_scene* s);
shb_status rasterize_device(shb_scene* s, int W, int H, shb_surface_point* d_out);
shb_status validity_mask_device(shb_context* c, const shb_surface_point* pts, int64_t n, uint8_t* out);
shb_status downsample_mask_device(shb_context* c, const uint8_t* in, int w, int h, int s, uint8_t* out);
shb_status downsample_device(shb_context* c, const float* in, int w, int h, int ch, int s, float* out);
shb_status dilate_device(shb_context* c, int kind, int w, int h, void* pixels, uint8_t* mask, int passes);
shb_status bake_device(shb_scene* s, const shb_surface_point* d_pts, int W, int H,
                       const shb_bake_config* cfg, float* d_sh, float* d_env, shb_bake_stats* stats);

// One bake of a batch, with device G-buffer and device outputs.
struct BakeSpec {
  shb_scene* scene;
  const shb_surface_point* pts;
  int W, H;  // supersampled texel dims
  shb_bake_config cfg;
  float* sh;
  float* env;
  const float* dsh = nullptr;  // backward: dLoss/dSH, 27 floats per texel (device)
};

// Launch-structure parameters (chosen by the autotuner for batches).
#ifndef SHB_WAVE_LOG2
#define SHB_WAVE_LOG2 25
#endif
struct BatchParams {
  int64_t wave_paths = int64_t(1) << SHB_WAVE_LOG2;  // paths in flight per wave (queue depth)
  int64_t tile_texels = int64_t(1) << 30; // texels per work tile
  int grid_scale = 1;                     // traversal grid = grid_scale x SMs x occupancy
  int64_t share_paths = -1;               // bakes of fewer paths share waves (-1: wave_paths / 2)
  int nee_split = 0;                      // next-event kernel: 0 by light-loop cost, 1 inline, 2 separate
  bool use_graph = false;                 // capture the waves in one CUDA graph
  uint32_t max_iters = 0;                 // traversal steps of one ray (0: default)
  int64_t queue_cap = 0;                  // entries per ray queue (0: sized to the wave)
  // Path-replay adjoint instead of the forward bake (one bake): gradients of
  // sum(dsh * SH) accumulate into grad[3 * mat_count + light_count] (device,
  // zeroed by the call).
  bool backward = false;
  double* grad = nullptr;
};

shb_status bake_batch_device(shb_context* c, const std::vector<BakeSpec>& specs, const BatchParams& prm,
                             shb_bake_stats* stats);
// Looks up the device address of shb_dilate_noalloc's fixed scratch array
// on `device` (current) and caches it (raster.cu).
shb_status noalloc_prepare(int device);
shb_status find_occlusion_device(shb_scene* s, const shb_ray* d_rays, int64_t n, shb_hit* d_hits);
// SaveSHLightMap (exr.cu): device SH (27 f32) and env (f32, nullable) texels.
shb_status save_sh_lightmap_device(shb_context* c, const float* d_sh, const float* d_env, int W, int H,
                                   const std::string& path, int mode);
shb_status exr_load_channels(const char* path, const char* const* names, int n, int* width, int* height, float* out);
// SH previews (preview.cu): d_out = n x 3 bytes (device).
shb_status sh_preview_device(shb_context* c, const float* d_sh, int64_t n, const float* d_normals, const float dir[3],
                             int mode, int reinhard, uint8_t* d_out);
bool write_png(const std::string& path, int w, int h, int channels, const uint8_t* px);
// Path-replay adjoint of bake_device: grad[3 * mat_count + light_count] (device).
shb_status backward_device(shb_scene* s, const shb_surface_point* d_pts, int W, int H, const shb_bake_config* cfg,
                           const float* d_dsh, double* d_grad, shb_bake_stats* stats);

// Rotation of the polar decomposition of a row-major 3x3 (Eigen's
// Transform::rotation()), shb_capi.cu.
void polar_rotation(const float L[9], float R[9]);

// sRGB -> linear table (computed on the host with powf, colorspace.h:10-14)
void srgb_table(float out[256]);

}  // namespace shb
