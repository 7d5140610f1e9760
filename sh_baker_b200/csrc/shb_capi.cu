// shb_capi.cu - the extern "C" boundary (include/shb.h): contexts, scene
// upload and validation, and dispatch of every entry point to its kernels.
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "shb_internal.h"

namespace shb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

shb_status cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " + what);
  return e == cudaErrorMemoryAllocation ? SHB_ERR_OOM : SHB_ERR_CUDA;
}

// ------------------------------------------------------- block cache ----

namespace {

struct CachedBlock {
  int dev;
  void* ptr;
  size_t bytes;
};

// Never destroyed: device buffers can still be released while the
// process tears down its statics at exit.
std::mutex& g_cache_mu = *new std::mutex;
std::vector<CachedBlock>& g_cache = *new std::vector<CachedBlock>;
int g_contexts = 0;  // live contexts; the cache is emptied with the last
constexpr size_t kCacheBytesPerDevice = size_t(8) << 30;

// Returns every cached block of `dev` (all devices: -1) with cudaFree.
void cache_flush(int dev) {
  std::vector<CachedBlock> keep, drop;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (const CachedBlock& b : g_cache) (dev < 0 || b.dev == dev ? drop : keep).push_back(b);
    g_cache.swap(keep);
  }
  int cur = 0;
  cudaGetDevice(&cur);
  for (const CachedBlock& b : drop) {
    cudaSetDevice(b.dev);
    cudaFree(b.ptr);
  }
  cudaSetDevice(cur);
}

// Takes the smallest cached block of `dev` that holds n bytes and is at
// most twice that (plus 1 MiB), so a small request does not pin a large block.
bool cache_take(int dev, size_t n, void** ptr, size_t* bytes) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  size_t best = g_cache.size();
  for (size_t i = 0; i < g_cache.size(); ++i) {
    const CachedBlock& b = g_cache[i];
    if (b.dev != dev || b.bytes < n || b.bytes > 2 * n + (size_t(1) << 20)) continue;
    if (best == g_cache.size() || b.bytes < g_cache[best].bytes) best = i;
  }
  if (best == g_cache.size()) return false;
  *ptr = g_cache[best].ptr;
  *bytes = g_cache[best].bytes;
  g_cache.erase(g_cache.begin() + (ptrdiff_t)best);
  return true;
}

}  // namespace

void block_release(int dev, void* ptr, size_t bytes) {
  int cur = 0;
  cudaGetDevice(&cur);
  if (dev >= 0 && dev != cur) cudaSetDevice(dev);
  cudaDeviceSynchronize();  // as cudaFree: no queued work still uses the block
  bool cached = false;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    size_t held = 0;
    for (const CachedBlock& b : g_cache)
      if (b.dev == dev) held += b.bytes;
    if (g_contexts > 0 && dev >= 0 && held + bytes <= kCacheBytesPerDevice) {
      g_cache.push_back(CachedBlock{dev, ptr, bytes});
      cached = true;
    }
  }
  if (!cached) cudaFree(ptr);
  if (dev >= 0 && dev != cur) cudaSetDevice(cur);
}

int sm_count() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
  if (dev < 64) {
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) {
    cudaGetLastError();
    sms = 1;
  }
  if (dev < 64) cache[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

void ctx_retain(shb_context* c) { c->refs.fetch_add(1); }

// Drops one reference; the last frees the context and its own stream.
void ctx_release(shb_context* c) {
  if (c->refs.fetch_sub(1) != 1) return;
  ::shb::DeviceScope _shb_device_scope(c->device);
  if (c->own_stream) {
    cudaStreamSynchronize(c->own_stream);
    cudaStreamDestroy(c->own_stream);
  }
  delete c;
  bool last = false;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    last = --g_contexts == 0;
  }
  if (last) cache_flush(-1);
}

// shb_test_fail_allocation_after: allocations left before one is refused
// (negative: off).
std::atomic<int> g_fail_alloc_countdown{-1};

shb_status DevBuf::reserve(size_t n) {
  if (n <= bytes && ptr) return SHB_OK;
  release();
  if (n == 0) n = 16;
  if (g_fail_alloc_countdown.load() >= 0 && g_fail_alloc_countdown.fetch_sub(1) == 0) {
    set_error("device allocation of " + std::to_string(n) + " bytes refused (shb_test_fail_allocation_after)");
    return SHB_ERR_OOM;
  }
  int d = 0;
  SHB_CUDA(cudaGetDevice(&d));
  if (cache_take(d, n, &ptr, &bytes)) {
    dev = d;
    return SHB_OK;
  }
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e == cudaErrorMemoryAllocation) {  // give the cached blocks back and retry
    cudaGetLastError();
    cache_flush(d);
    e = cudaMalloc(&ptr, n);
  }
  if (e != cudaSuccess) {
    ptr = nullptr;
    bytes = 0;
    return cuda_fail(e, "cudaMalloc");
  }
  bytes = n;
  dev = d;
  return SHB_OK;
}

void srgb_table(float out[256]) {
  // src/colorspace.h:10-14, evaluated once on the host.
  for (int i = 0; i < 256; ++i) {
    float v = (uint8_t)i / 255.0f;
    out[i] = v <= 0.04045f ? v / 12.92f : std::pow((v + 0.055f) / 1.055f, 2.4f);
  }
}

void srgb_upload(const float table[256]);

// Emission constants of the area lights (DLight::er/eg/eb, emis_const): for
// a material whose albedo does not vary over the surface, albedo *
// emission with the float products get_emission makes on the device.
void area_emission_consts(shb_scene* s) {
  for (uint32_t l = 0; l < s->light_count; ++l) {
    DLight& L = s->h_lights[l];
    L.emis_const = 0;
    L.er = L.eg = L.eb = 0.f;
    if (L.type != SHB_LIGHT_AREA) continue;
    if (L.mat < 0 || (uint32_t)L.mat >= s->mat_count) {  // load_mat's default: no emission
      L.emis_const = 1;
      continue;
    }
    const DMat& M = s->h_mats[L.mat];
    float a[3];
    if (M.use_override) {
      for (int c = 0; c < 3; ++c) a[c] = M.override_rgb[c];
    } else if (s->h_light_albedo_const[l]) {
      for (int c = 0; c < 3; ++c) a[c] = s->h_light_albedo[3 * l + c];
    } else {
      continue;
    }
    L.emis_const = 1;
    if (M.emission > 0.0f) {
      L.er = a[0] * M.emission;
      L.eg = a[1] * M.emission;
      L.eb = a[2] * M.emission;
    }
  }
}

// Rotation part of an affine map (Eigen Transform::rotation(): polar
// decomposition M = U S V^T, R = U diag(x,1,1) V^T, x = sign det(U V^T)),
// by cyclic Jacobi on M^T M in double precision.
void polar_rotation(const float Lf[9], float Rout[9]) {
  bool ident = true;
  for (int i = 0; i < 9; ++i) ident = ident && (Lf[i] == ((i % 4 == 0) ? 1.f : 0.f));
  if (ident) {
    for (int i = 0; i < 9; ++i) Rout[i] = (i % 4 == 0) ? 1.f : 0.f;
    return;
  }
  double M[3][3], A[3][3], V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i][j] = Lf[i * 3 + j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += M[k][i] * M[k][j];
      A[i][j] = s;
    }
  for (int sweep = 0; sweep < 60; ++sweep) {
    if (std::fabs(A[0][1]) + std::fabs(A[0][2]) + std::fabs(A[1][2]) < 1e-300) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (std::fabs(A[p][q]) < 1e-300) continue;
        double th = (A[q][q] - A[p][p]) / (2 * A[p][q]);
        double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1));
        double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 3; ++k) {
          double x = A[k][p], y = A[k][q];
          A[k][p] = c * x - s * y;
          A[k][q] = s * x + c * y;
        }
        for (int k = 0; k < 3; ++k) {
          double x = A[p][k], y = A[q][k];
          A[p][k] = c * x - s * y;
          A[q][k] = s * x + c * y;
        }
        for (int k = 0; k < 3; ++k) {
          double x = V[k][p], y = V[k][q];
          V[k][p] = c * x - s * y;
          V[k][q] = s * x + c * y;
        }
      }
  }
  int ord[3] = {0, 1, 2};
  double ev[3] = {A[0][0], A[1][1], A[2][2]};
  for (int i = 0; i < 3; ++i)
    for (int j = i + 1; j < 3; ++j)
      if (ev[ord[j]] > ev[ord[i]]) std::swap(ord[i], ord[j]);
  double Vs[3][3], U[3][3];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) Vs[i][j] = V[i][ord[j]];
  for (int j = 0; j < 3; ++j) {
    double col[3], n = 0;
    for (int i = 0; i < 3; ++i) {
      col[i] = M[i][0] * Vs[0][j] + M[i][1] * Vs[1][j] + M[i][2] * Vs[2][j];
      n += col[i] * col[i];
    }
    n = std::sqrt(n);
    for (int i = 0; i < 3; ++i) U[i][j] = n > 0 ? col[i] / n : 0.0;
  }
  auto det3 = [](double X[3][3]) {
    return X[0][0] * (X[1][1] * X[2][2] - X[1][2] * X[2][1]) - X[0][1] * (X[1][0] * X[2][2] - X[1][2] * X[2][0]) +
           X[0][2] * (X[1][0] * X[2][1] - X[1][1] * X[2][0]);
  };
  double x = (det3(U) * det3(Vs) < 0) ? -1.0 : 1.0;
  for (int i = 0; i < 3; ++i) U[i][0] *= x;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += U[i][k] * Vs[j][k];
      Rout[i * 3 + j] = (float)s;
    }
}

template <class T>
static shb_status upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  SHB_TRY(b.reserve(sizeof(T) * (v.empty() ? 1 : v.size())));
  if (!v.empty()) SHB_CUDA(cudaMemcpyAsync(b.ptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
  return SHB_OK;
}

static shb_status bad(const std::string& m) {
  set_error(m);
  return SHB_ERR_INVALID_ARG;
}

// Image arguments hold at most 2^31 - 1 texels, the G-buffer limit of
// shb_rasterize, and shb_find_occlusion takes at most that many rays, so that
// every byte count formed from them fits 64 bits and every texel index an
// int32.  The size checks come before the handle checks.
constexpr int64_t kMaxTexels = (1ll << 31) - 1;
static bool too_many_texels(int64_t w, int64_t h) {
  return w > 0 && h > 0 && (w > kMaxTexels || h > kMaxTexels || w * h > kMaxTexels);
}
static const char* kTooLarge = "image larger than 2^31 - 1 texels";

// Host<->device staging for the host-pointer variants.
struct Staging {
  shb_context* c;
  int slot;
  void* get(size_t n, shb_status* st) {
    *st = c->scratch[slot].reserve(n);
    return *st == SHB_OK ? c->scratch[slot].ptr : nullptr;
  }
};

}  // namespace shb

using namespace shb;

SceneView shb_scene::view() const {
  SceneView v;
  v.obj_v = obj_v.as<float>();
  v.obj_n = obj_n.as<float>();
  v.tex_uv = tex_uv.as<float>();
  v.world_v = world_v.as<float>();
  v.tri_vidx = tri_vidx.as<uint32_t>();
  v.tri_geom = tri_geom.as<uint32_t>();
  v.geoms = geoms.as<DGeom>();
  v.mats = mats.as<DMat>();
  v.pixels = pixels.as<uint8_t>();
  v.lights = lights.as<DLight>();
  v.area_tris = area_tris.as<float4>();
  v.geom_count = geom_count;
  v.mat_count = mat_count;
  v.light_count = light_count;
  v.area_light_count = area_light_count;
  v.prim_count = prim_count;
  v.vertex_count = vertex_count;
  v.has_alpha = has_alpha;
  return v;
}

BvhView shb_scene::bvh() const {
  BvhView b;
  b.nodes = bvh_nodes.as<WideNode>();
  b.tris = bvh_tris.as<float4>();
  b.node_count = bvh_node_count;
  b.tri_count = bvh_tri_count;
  return b;
}

extern "C" {

int32_t shb_abi_version(void) { return SHB_ABI_VERSION; }

const char* shb_last_error(void) { return g_last_error.c_str(); }

void shb_test_fail_allocation_after(int32_t n) { shb::g_fail_alloc_countdown.store(n < 0 ? -1 : n); }

void shb_srgb_to_linear_table(float* out) {
  if (out) srgb_table(out);
}

shb_status shb_context_create(const shb_options* options, shb_context** out) {
  return ::shb::guarded("shb_context_create", [&]() -> shb_status {
    if (!out) return bad("out is NULL");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
      set_error(std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0"));
      return SHB_ERR_NO_DEVICE;
    }
    int dev = options ? options->device : 0;
    if (dev < 0 || dev >= ndev) return bad("device ordinal out of range");
    SHB_ON_DEVICE(dev);
    cudaDeviceProp prop;
    SHB_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) {
      set_error("this library is built for sm_100a (B200); device is sm_" + std::to_string(prop.major) +
                std::to_string(prop.minor));
      return SHB_ERR_NO_DEVICE;
    }
    // owned here until it is handed out, so that no path (an exception
    // included) leaks it
    std::unique_ptr<shb_context> owner(new shb_context());
    shb_context* c = owner.get();
    c->device = dev;
    c->profiling = options ? options->profiling : 0;
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    c->stream = c->own_stream;
    float tab[256];
    srgb_table(tab);
    srgb_upload(tab);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      cudaStreamDestroy(c->own_stream);
      return cuda_fail(e, "sRGB table upload");
    }
    // shb_dilate_noalloc's fixed array: its address is resolved here, so that
    // the entry point itself never loads a module or reserves memory
    shb_status ns = noalloc_prepare(dev);
    if (ns != SHB_OK) {
      cudaStreamDestroy(c->own_stream);
      return ns;
    }
    {
      std::lock_guard<std::mutex> lk(g_cache_mu);
      ++g_contexts;
    }
    *out = owner.release();
    return SHB_OK;
  });
}

shb_status shb_context_destroy(shb_context* ctx) {
  return ::shb::guarded("shb_context_destroy", [&]() -> shb_status {
    if (!ctx) return SHB_OK;
    ::shb::DeviceScope _shb_device_scope(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& b : ctx->scratch) b.release();
    ctx->counters.release();
    delete ctx->pipe_gbuf;
    ctx->pipe_gbuf = nullptr;
    shb::ctx_release(ctx);
    return SHB_OK;
  });
}

shb_status shb_context_set_stream(shb_context* ctx, void* stream) {
  return ::shb::guarded("shb_context_set_stream", [&]() -> shb_status {
    if (!ctx) return bad("ctx is NULL");
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return SHB_OK;
  });
}

shb_status shb_context_synchronize(shb_context* ctx) {
  return ::shb::guarded("shb_context_synchronize", [&]() -> shb_status {
    if (!ctx) return bad("ctx is NULL");
    SHB_CUDA(cudaStreamSynchronize(ctx->stream));
    return SHB_OK;
  });
}

uint64_t shb_context_kernel_launches(const shb_context* ctx) { return ctx ? ctx->launches : 0; }

shb_status shb_rotation_part(const float transform[12], float rotation[9]) {
  return ::shb::guarded("shb_rotation_part", [&]() -> shb_status {
    if (!transform || !rotation) return bad("NULL argument");
    const float L[9] = {transform[0], transform[1], transform[2], transform[4], transform[5],
                        transform[6], transform[8], transform[9], transform[10]};
    polar_rotation(L, rotation);
    return SHB_OK;
  });
}

shb_status shb_scene_upload(shb_context* ctx, const shb_scene_desc* d, shb_scene** out) {
  return ::shb::guarded("shb_scene_upload", [&]() -> shb_status {
    if (!d || !out) return bad("NULL argument");
    *out = nullptr;
    if (d->geometry_count && !d->geometries) return bad("geometries is NULL");
    if (d->material_count && !d->materials) return bad("materials is NULL");
    if (d->light_count && !d->lights) return bad("lights is NULL");
    // The kernels index per-vertex arrays as up to 4 * vertex id, per-triangle
    // arrays as 3 * triangle id and the transforms as 12 * geometry id, all
    // in 32-bit arithmetic: these limits keep every such index in range.
    // (Checked from the counts alone, before the context.)
    static const char* kTooBig =
        "scene too large: at most 2^30 - 1 vertices, 2^30 - 1 triangles and 2^26 - 1 geometries";
    if (d->geometry_count >= (1u << 26)) return bad(kTooBig);
    uint64_t nv_total = 0, nt_total = 0;
    for (uint32_t g = 0; g < d->geometry_count; ++g) {
      const shb_geometry_desc& gd = d->geometries[g];
      nv_total += gd.vertex_count;
      nt_total += gd.index_count / 3;
    }
    if (nv_total >= (1ull << 30) || nt_total >= (1ull << 30)) return bad(kTooBig);
    if (!ctx) return bad("NULL argument");
    SHB_ON_DEVICE(ctx->device);
    cudaStream_t st = ctx->stream;
    std::vector<float> ov, on, tuv, luv, ot, lin, rot;
    std::vector<uint32_t> vidx, tgeom, vgeom;
    std::vector<DGeom> geoms;
    bool raster_ready = true;
    std::string raster_error;
    ov.reserve(3 * nv_total);
    on.assign(3 * nv_total, 0.f);
    tuv.assign(2 * nv_total, 0.f);
    luv.assign(2 * nv_total, 0.f);
    ot.assign(4 * nv_total, 0.f);
    uint32_t vbase = 0, pbase = 0;
    for (uint32_t g = 0; g < d->geometry_count; ++g) {
      const shb_geometry_desc& gd = d->geometries[g];
      if (gd.vertex_count && !gd.vertices) return bad("geometry " + std::to_string(g) + ": vertices is NULL");
      if (gd.index_count && !gd.indices) return bad("geometry " + std::to_string(g) + ": indices is NULL");
      if (gd.material_id < -1 || (gd.material_id >= 0 && (uint32_t)gd.material_id >= d->material_count))
        return bad("geometry " + std::to_string(g) + ": material_id out of range");
      uint32_t ntri = gd.index_count / 3;
      for (uint32_t i = 0; i < ntri * 3; ++i)
        if (gd.indices[i] >= gd.vertex_count) return bad("geometry " + std::to_string(g) + ": index out of range");
      DGeom G;
      std::memset(&G, 0, sizeof(G));
      G.vbase = vbase;
      G.prim_base = pbase;
      G.tri_count = ntri;
      G.material_id = gd.material_id;
      G.flags = (gd.normals ? GEOM_HAS_NORMALS : 0u) | (gd.texture_uvs ? GEOM_HAS_TEXUV : 0u) |
                (gd.tangents ? GEOM_HAS_TANGENTS : 0u) | (gd.lightmap_uvs ? GEOM_HAS_LMUV : 0u);
      geoms.push_back(G);
      if (gd.vertex_count == 0 || !gd.normals || !gd.tangents || !gd.lightmap_uvs) {
        if (raster_ready)
          raster_error = "geometry " + std::to_string(g) +
                         " lacks vertices, normals, tangents or lightmap_uvs (RasterizeScene requires them)";
        raster_ready = false;
      }
      for (uint32_t v = 0; v < gd.vertex_count; ++v) {
        uint64_t k = vbase + v;
        for (int a = 0; a < 3; ++a) ov.push_back(gd.vertices[3 * v + a]);
        if (gd.normals)
          for (int a = 0; a < 3; ++a) on[3 * k + a] = gd.normals[3 * v + a];
        if (gd.texture_uvs)
          for (int a = 0; a < 2; ++a) tuv[2 * k + a] = gd.texture_uvs[2 * v + a];
        if (gd.lightmap_uvs)
          for (int a = 0; a < 2; ++a) luv[2 * k + a] = gd.lightmap_uvs[2 * v + a];
        if (gd.tangents)
          for (int a = 0; a < 4; ++a) ot[4 * k + a] = gd.tangents[4 * v + a];
        vgeom.push_back(g);
      }
      for (uint32_t t = 0; t < ntri; ++t) {
        for (int k = 0; k < 3; ++k) vidx.push_back(vbase + gd.indices[3 * t + k]);
        tgeom.push_back(g);
      }
      for (int i = 0; i < 12; ++i) lin.push_back(gd.transform[i]);
      float L[9] = {gd.transform[0], gd.transform[1], gd.transform[2], gd.transform[4], gd.transform[5],
                    gd.transform[6], gd.transform[8], gd.transform[9], gd.transform[10]};
      float R[9];
      polar_rotation(L, R);
      for (int i = 0; i < 9; ++i) rot.push_back(R[i]);
      vbase += gd.vertex_count;
      pbase += ntri;
    }
    std::vector<DMat> mats;
    std::vector<uint8_t> pix;
    int has_alpha = 0;
    for (uint32_t m = 0; m < d->material_count; ++m) {
      const shb_material_desc& md = d->materials[m];
      DMat M;
      std::memset(&M, 0, sizeof(M));
      M.emission = md.emission_intensity;
      if (md.albedo_pixels && md.albedo_width && md.albedo_height && md.albedo_channels) {
        if (md.albedo_channels != 3 && md.albedo_channels != 4)
          return bad("material " + std::to_string(m) + ": albedo_channels must be 3 or 4");
        // a texel's byte offset is a 32-bit int inside its texture
        // (tex_index) and a 32-bit offset among all textures (pix_offset)
        const uint64_t n = (uint64_t)md.albedo_width * md.albedo_height * md.albedo_channels;
        if (n > 0x7FFFFFFFull || pix.size() + n > 0xFFFFFFFFull)
          return bad("material " + std::to_string(m) +
                     ": albedo texture above 2^31 - 1 bytes, or all textures above 2^32 - 1 bytes");
        M.pix_offset = (uint32_t)pix.size();
        M.w = md.albedo_width;
        M.h = md.albedo_height;
        M.c = md.albedo_channels;
        pix.insert(pix.end(), md.albedo_pixels, md.albedo_pixels + n);
        if (M.c == 4) has_alpha = 1;
      }
      mats.push_back(M);
    }
    std::vector<DLight> lights;
    int area_ord = 0;
    for (uint32_t l = 0; l < d->light_count; ++l) {
      const shb_light_desc& ld = d->lights[l];
      if (ld.type < SHB_LIGHT_POINT || ld.type > SHB_LIGHT_AREA)
        return bad("light " + std::to_string(l) + ": bad type");
      DLight L;
      std::memset(&L, 0, sizeof(L));
      L.type = ld.type;
      L.px = ld.position[0];
      L.py = ld.position[1];
      L.pz = ld.position[2];
      L.dx = ld.direction[0];
      L.dy = ld.direction[1];
      L.dz = ld.direction[2];
      L.cr = ld.color[0];
      L.cg = ld.color[1];
      L.cb = ld.color[2];
      L.intensity = ld.intensity;
      L.cos_inner = ld.cos_inner_cone;
      L.cos_outer = ld.cos_outer_cone;
      L.geom = -1;
      L.mat = -1;
      L.area_ord = -1;
      if (ld.type == SHB_LIGHT_AREA) {
        if (ld.geometry_index >= (int32_t)d->geometry_count)
          return bad("light " + std::to_string(l) + ": bad geometry");
        if (ld.material_index >= (int32_t)d->material_count)
          return bad("light " + std::to_string(l) + ": bad material");
        L.geom = ld.geometry_index;
        L.mat = ld.material_index;
        L.area_ord = area_ord++;
      }
      lights.push_back(L);
    }
    std::unique_ptr<shb_scene> owner(new shb_scene());  // owned here until handed out
    shb_scene* s = owner.get();
    s->ctx = ctx;
    s->vertex_count = vbase;
    s->prim_count = pbase;
    s->geom_count = d->geometry_count;
    s->mat_count = d->material_count;
    s->light_count = d->light_count;
    s->area_light_count = (uint32_t)area_ord;
    s->has_alpha = has_alpha;
    s->raster_ready = raster_ready;
    s->raster_error = raster_error;
    s->h_geoms = geoms;
    s->h_mats = mats;
    s->h_lights = lights;
    {
      float srgb[256];
      srgb_table(srgb);
      s->h_light_albedo.assign(3 * (size_t)s->light_count, 0.f);
      s->h_light_albedo_const.assign(s->light_count, 0);
      for (uint32_t l = 0; l < s->light_count; ++l) {
        const DLight& L = lights[l];
        if (L.type != SHB_LIGHT_AREA || L.mat < 0 || (uint32_t)L.mat >= s->mat_count) continue;
        const DMat& M = mats[L.mat];
        if (M.c == 0) {  // get_albedo's default grey
          for (int c = 0; c < 3; ++c) s->h_light_albedo[3 * l + c] = 0.8f;
          s->h_light_albedo_const[l] = 1;
        } else if (M.w == 1 && M.h == 1) {
          for (int c = 0; c < 3; ++c) s->h_light_albedo[3 * l + c] = srgb[pix[M.pix_offset + c]];
          s->h_light_albedo_const[l] = 1;
        }
      }
      area_emission_consts(s);
      lights = s->h_lights;
    }
    shb_status rc = SHB_OK;
    auto chk = [&](shb_status x) {
      if (rc == SHB_OK) rc = x;
    };
    chk(upload(s->obj_v, ov, st));
    chk(upload(s->obj_n, on, st));
    chk(upload(s->tex_uv, tuv, st));
    chk(upload(s->lm_uv, luv, st));
    chk(upload(s->obj_t, ot, st));
    chk(upload(s->tri_vidx, vidx, st));
    chk(upload(s->tri_geom, tgeom, st));
    chk(upload(s->vgeom, vgeom, st));
    chk(upload(s->geoms, geoms, st));
    chk(upload(s->mats, mats, st));
    chk(upload(s->pixels, pix, st));
    chk(upload(s->lights, lights, st));
    chk(upload(s->lin, lin, st));
    chk(upload(s->rot, rot, st));
    if (rc == SHB_OK) chk(s->world_v.reserve(sizeof(float) * 3 * (vbase ? vbase : 1)));
    if (rc == SHB_OK) chk(s->world_n.reserve(sizeof(float) * 3 * (vbase ? vbase : 1)));
    if (rc == SHB_OK) chk(s->world_t.reserve(sizeof(float) * 4 * (vbase ? vbase : 1)));
    if (rc == SHB_OK) chk(transform_vertices(s));
    if (rc == SHB_OK) chk(build_bvh(s));
    if (rc == SHB_OK) chk(build_area_tris(s));
    if (rc == SHB_OK) {
      cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) rc = cuda_fail(e, "scene upload");
    }
    if (rc != SHB_OK) return rc;
    ctx_retain(s->ctx);
    *out = owner.release();
    return SHB_OK;
  });
}

shb_status shb_scene_destroy(shb_scene* s) {
  return ::shb::guarded("shb_scene_destroy", [&]() -> shb_status {
    if (!s) return SHB_OK;
    shb_context* c = s->ctx;
    ::shb::DeviceScope _shb_device_scope(c->device);
    cudaStreamSynchronize(c->stream);
    delete s;
    ctx_release(c);
    return SHB_OK;
  });
}

shb_status shb_scene_rebuild_bvh(shb_scene* s) {
  return ::shb::guarded("shb_scene_rebuild_bvh", [&]() -> shb_status {
    if (!s) return bad("scene is NULL");
    SHB_ON_DEVICE(s->ctx->device);
    SHB_TRY(build_bvh(s));
    SHB_CUDA(cudaStreamSynchronize(s->ctx->stream));
    return SHB_OK;
  });
}

shb_status shb_scene_bvh_info(const shb_scene* s, uint32_t* wide_nodes, uint32_t* triangles, uint32_t* depth) {
  return ::shb::guarded("shb_scene_bvh_info", [&]() -> shb_status {
    if (!s) return bad("scene is NULL");
    if (wide_nodes) *wide_nodes = s->bvh_node_count;
    if (triangles) *triangles = s->bvh_tri_count;
    if (depth) *depth = s->bvh_depth;
    return SHB_OK;
  });
}

namespace {

// Rasterises into g (its storage grows as needed), optionally downloading
// the points to host_out, and waits for the stream.
shb_status rasterize_into(shb_scene* s, const shb_raster_config* cfg, shb_gbuffer* g, shb_surface_point* host_out) {
  if (!s->raster_ready) return bad(s->raster_error);
  if (cfg->width <= 0 || cfg->height <= 0 || cfg->supersample_scale <= 0)
    return bad("raster width, height and supersample_scale must be positive");
  int64_t W = (int64_t)cfg->width * cfg->supersample_scale, H = (int64_t)cfg->height * cfg->supersample_scale;
  if (W > 65535 || H > 65535 || W * H > (1ll << 31) - 1) return bad("raster size too large");
  SHB_ON_DEVICE(s->ctx->device);
  g->ctx = s->ctx;
  g->width = (int)W;
  g->height = (int)H;
  SHB_TRY(g->points.reserve(sizeof(shb_surface_point) * (size_t)(W * H)));
  SHB_TRY(rasterize_device(s, (int)W, (int)H, g->points.as<shb_surface_point>()));
  if (host_out)
    SHB_CUDA(cudaMemcpyAsync(host_out, g->points.ptr, sizeof(shb_surface_point) * (size_t)(W * H),
                             cudaMemcpyDeviceToHost, s->ctx->stream));
  cudaError_t e = cudaStreamSynchronize(s->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "rasterize");
  return SHB_OK;
}

}  // namespace

shb_status shb_rasterize(shb_scene* s, const shb_raster_config* cfg, shb_surface_point* host_out,
                         shb_gbuffer** out_gbuffer) {
  return ::shb::guarded("shb_rasterize", [&]() -> shb_status {
    if (!s || !cfg) return bad("NULL argument");
    if (out_gbuffer) *out_gbuffer = nullptr;
    std::unique_ptr<shb_gbuffer> owner(new shb_gbuffer());  // owned here until handed out
    shb_gbuffer* g = owner.get();
    shb_status rc = rasterize_into(s, cfg, g, host_out);
    if (rc != SHB_OK || !out_gbuffer) return rc;
    ctx_retain(g->ctx);
    *out_gbuffer = owner.release();
    return SHB_OK;
  });
}

shb_status shb_gbuffer_upload(shb_context* ctx, const shb_surface_point* points, int32_t width, int32_t height,
                              shb_gbuffer** out) {
  return ::shb::guarded("shb_gbuffer_upload", [&]() -> shb_status {
    if (width <= 0 || height <= 0) return bad("width and height must be positive");
    if (too_many_texels(width, height)) return bad(kTooLarge);
    if (!ctx || !points || !out) return bad("NULL argument");
    SHB_ON_DEVICE(ctx->device);
    std::unique_ptr<shb_gbuffer> owner(new shb_gbuffer());  // owned here until handed out
    shb_gbuffer* g = owner.get();
    g->ctx = ctx;
    g->width = width;
    g->height = height;
    size_t n = sizeof(shb_surface_point) * (size_t)width * height;
    shb_status rc = g->points.reserve(n);
    if (rc == SHB_OK) {
      cudaError_t e = cudaMemcpyAsync(g->points.ptr, points, n, cudaMemcpyHostToDevice, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) rc = cuda_fail(e, "G-buffer upload");
    }
    if (rc != SHB_OK) return rc;
    ctx_retain(g->ctx);
    *out = owner.release();
    return SHB_OK;
  });
}

shb_status shb_gbuffer_download(const shb_gbuffer* g, shb_surface_point* points) {
  return ::shb::guarded("shb_gbuffer_download", [&]() -> shb_status {
    if (!g || !points) return bad("NULL argument");
    SHB_ON_DEVICE(g->ctx->device);
    SHB_CUDA(cudaMemcpyAsync(points, g->points.ptr, sizeof(shb_surface_point) * (size_t)g->width * g->height,
                             cudaMemcpyDeviceToHost, g->ctx->stream));
    SHB_CUDA(cudaStreamSynchronize(g->ctx->stream));
    return SHB_OK;
  });
}

shb_status shb_gbuffer_dims(const shb_gbuffer* g, int32_t* width, int32_t* height) {
  return ::shb::guarded("shb_gbuffer_dims", [&]() -> shb_status {
    if (!g) return bad("gbuffer is NULL");
    if (width) *width = g->width;
    if (height) *height = g->height;
    return SHB_OK;
  });
}

shb_status shb_gbuffer_destroy(shb_gbuffer* g) {
  return ::shb::guarded("shb_gbuffer_destroy", [&]() -> shb_status {
    if (!g) return SHB_OK;
    shb_context* c = g->ctx;
    ::shb::DeviceScope _shb_device_scope(c->device);
    cudaStreamSynchronize(c->stream);
    delete g;
    ctx_release(c);
    return SHB_OK;
  });
}

shb_status shb_validity_mask(shb_context* ctx, const shb_gbuffer* g, uint8_t* mask_out, int32_t device_ptr) {
  return ::shb::guarded("shb_validity_mask", [&]() -> shb_status {
    if (!ctx || !g || !mask_out) return bad("NULL argument");
    SHB_ON_DEVICE(ctx->device);
    int64_t n = (int64_t)g->width * g->height;
    uint8_t* d = mask_out;
    if (!device_ptr) {
      SHB_TRY(ctx->scratch[18].reserve((size_t)n));
      d = ctx->scratch[18].as<uint8_t>();
    }
    SHB_TRY(validity_mask_device(ctx, g->points.as<shb_surface_point>(), n, d));
    if (!device_ptr) SHB_CUDA(cudaMemcpyAsync(mask_out, d, (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    SHB_CUDA(cudaStreamSynchronize(ctx->stream));
    return SHB_OK;
  });
}

shb_status shb_downsample_validity_mask(shb_context* ctx, const uint8_t* in, int32_t width, int32_t height,
                                        int32_t scale, uint8_t* out, int32_t device_ptrs) {
  return ::shb::guarded("shb_downsample_validity_mask", [&]() -> shb_status {
    if (width <= 0 || height <= 0 || scale <= 0) return bad("width, height and scale must be positive");
    if (too_many_texels((int64_t)width * scale, (int64_t)height * scale)) return bad(kTooLarge);
    if (!ctx || !in || !out) return bad("NULL argument");
    SHB_ON_DEVICE(ctx->device);
    size_t nin = (size_t)width * scale * height * scale, nout = (size_t)width * height;
    const uint8_t* din = in;
    uint8_t* dout = out;
    if (!device_ptrs) {
      SHB_TRY(ctx->scratch[18].reserve(nin));
      SHB_TRY(ctx->scratch[19].reserve(nout));
      SHB_CUDA(cudaMemcpyAsync(ctx->scratch[18].ptr, in, nin, cudaMemcpyHostToDevice, ctx->stream));
      din = ctx->scratch[18].as<uint8_t>();
      dout = ctx->scratch[19].as<uint8_t>();
    }
    SHB_TRY(downsample_mask_device(ctx, din, width, height, scale, dout));
    if (!device_ptrs) SHB_CUDA(cudaMemcpyAsync(out, dout, nout, cudaMemcpyDeviceToHost, ctx->stream));
    SHB_CUDA(cudaStreamSynchronize(ctx->stream));
    return SHB_OK;
  });
}

shb_status shb_bake(shb_scene* s, const shb_gbuffer* g, const shb_raster_config* rc, const shb_bake_config* cfg,
                    shb_bake_output* out, shb_bake_stats* stats) {
  return ::shb::guarded("shb_bake", [&]() -> shb_status {
    if (!s || !g || !rc || !cfg || !out || !out->sh || !out->env_visibility) return bad("NULL argument");
    if (cfg->samples <= 0) return bad("samples must be positive");
    if (cfg->bounces < 0 || cfg->bounces > 30) return bad("bounces must be in [0, 30]");
    if (cfg->num_light_samples <= 0) return bad("num_light_samples must be positive");
    if (cfg->rng_mode != SHB_RNG_PHILOX) return bad("unknown rng_mode");
    int64_t W = (int64_t)rc->width * rc->supersample_scale, H = (int64_t)rc->height * rc->supersample_scale;
    if (W != g->width || H != g->height) return bad("G-buffer size does not match raster_config (W*s x H*s)");
    if (s->bvh_depth > 64) return bad("BVH deeper than the traversal stack");
    SHB_ON_DEVICE(s->ctx->device);
    shb_context* c = s->ctx;
    uint64_t l0 = c->launches;
    size_t n = (size_t)W * H;
    float* dsh = out->sh;
    float* denv = out->env_visibility;
    if (!out->device_ptrs) {
      SHB_TRY(c->scratch[20].reserve(sizeof(float) * 28 * n));
      dsh = c->scratch[20].as<float>();
      denv = dsh + 27 * n;
    }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    SHB_TRY(bake_device(s, g->points.as<shb_surface_point>(), (int)W, (int)H, cfg, dsh, denv, stats));
    if (!out->device_ptrs) {
      SHB_CUDA(cudaMemcpyAsync(out->sh, dsh, sizeof(float) * 27 * n, cudaMemcpyDeviceToHost, c->stream));
      SHB_CUDA(cudaMemcpyAsync(out->env_visibility, denv, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    }
    SHB_CUDA(cudaStreamSynchronize(c->stream));
    if (stats) {
      stats->kernel_launches = c->launches - l0;
      stats->bvh_build_ms = s->bvh_build_ms;
    }
    return SHB_OK;
  });
}

shb_status shb_save_sh_lightmap(shb_context* ctx, const float* sh, const float* env, int32_t width, int32_t height,
                                int32_t device_ptrs, const char* path, int32_t mode) {
  return ::shb::guarded("shb_save_sh_lightmap", [&]() -> shb_status {
    if (too_many_texels(width, height)) return bad(kTooLarge);
    if (!ctx || !sh || !path || !*path) return bad("NULL argument");
    if (width <= 0 || height <= 0) return bad("Invalid SHTexture dimensions or empty pixels.");
    if (mode < SHB_SAVE_COMBINED || mode > SHB_SAVE_LUMINANCE_PACKED) return bad("unknown save mode");
    SHB_ON_DEVICE(ctx->device);
    const size_t n = (size_t)width * height;
    const float* dsh = sh;
    const float* denv = env;
    if (!device_ptrs) {
      SHB_TRY(ctx->scratch[27].reserve(sizeof(float) * 28 * n));
      float* d = ctx->scratch[27].as<float>();
      SHB_CUDA(cudaMemcpyAsync(d, sh, sizeof(float) * 27 * n, cudaMemcpyHostToDevice, ctx->stream));
      dsh = d;
      denv = nullptr;
      if (env) {
        SHB_CUDA(cudaMemcpyAsync(d + 27 * n, env, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
        denv = d + 27 * n;
      }
    }
    return save_sh_lightmap_device(ctx, dsh, denv, width, height, std::string(path), mode);
  });
}

shb_status shb_sh_preview(shb_context* ctx, const float* sh, int32_t width, int32_t height, const float* normals,
                          const float direction[3], int32_t mode, int32_t reinhard, int32_t device_ptrs,
                          uint8_t* rgb_out) {
  return ::shb::guarded("shb_sh_preview", [&]() -> shb_status {
    if (too_many_texels(width, height)) return bad(kTooLarge);
    if (!ctx || !sh || !rgb_out) return bad("NULL argument");
    if (width <= 0 || height <= 0) return bad("empty image");
    if (mode < SHB_PREVIEW_L0 || mode > SHB_PREVIEW_SH_PACKED) return bad("unknown preview mode");
    if (mode != SHB_PREVIEW_L0 && !normals && !direction) return bad("a direction or normals is needed");
    SHB_ON_DEVICE(ctx->device);
    const size_t n = (size_t)width * height;
    const size_t in_floats = 27 * n + (normals ? 3 * n : 0);
    SHB_TRY(ctx->scratch[27].reserve(sizeof(float) * in_floats + 3 * n));
    float* d_in = ctx->scratch[27].as<float>();
    uint8_t* d_out = reinterpret_cast<uint8_t*>(d_in + in_floats);
    const float* dsh = sh;
    const float* dn = normals;
    if (!device_ptrs) {
      SHB_CUDA(cudaMemcpyAsync(d_in, sh, sizeof(float) * 27 * n, cudaMemcpyHostToDevice, ctx->stream));
      dsh = d_in;
      if (normals) {
        SHB_CUDA(cudaMemcpyAsync(d_in + 27 * n, normals, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
        dn = d_in + 27 * n;
      }
    }
    const float zero[3] = {0.f, 0.f, 1.f};
    SHB_TRY(sh_preview_device(ctx, dsh, (int64_t)n, dn, direction ? direction : zero, mode, reinhard, d_out));
    SHB_CUDA(cudaMemcpyAsync(rgb_out, d_out, 3 * n, cudaMemcpyDeviceToHost, ctx->stream));
    SHB_CUDA(cudaStreamSynchronize(ctx->stream));
    return SHB_OK;
  });
}

shb_status shb_exr_load_channels(const char* path, const char* const* names, int32_t count, int32_t* width,
                                 int32_t* height, float* out) {
  return ::shb::guarded("shb_exr_load_channels", [&]() -> shb_status {
    if (!path || (count > 0 && !names)) return bad("NULL argument");
    for (int32_t k = 0; k < count; ++k)
      if (!names[k]) return bad("NULL channel name");
    return exr_load_channels(path, names, count, width, height, out);
  });
}

shb_status shb_write_png(const char* path, int32_t width, int32_t height, int32_t channels, const uint8_t* pixels) {
  return ::shb::guarded("shb_write_png", [&]() -> shb_status {
    if (!path || !pixels || width <= 0 || height <= 0 || channels < 1 || channels > 4) return bad("bad PNG arguments");
    if (!write_png(path, width, height, channels, pixels)) return bad(std::string("cannot write ") + path);
    return SHB_OK;
  });
}

shb_status shb_scene_set_params(shb_scene* s, const float* albedo_rgb, const uint8_t* use_override,
                                const float* light_intensity) {
  return ::shb::guarded("shb_scene_set_params", [&]() -> shb_status {
    if (!s) return bad("NULL scene");
    SHB_ON_DEVICE(s->ctx->device);
    if (albedo_rgb)
      for (uint32_t m = 0; m < s->mat_count; ++m)
        for (int c = 0; c < 3; ++c)
          if ((!use_override || use_override[m]) &&
              !(std::isfinite(albedo_rgb[3 * m + c]) && albedo_rgb[3 * m + c] >= 0.f))
            return bad("material " + std::to_string(m) + ": albedo override must be finite and >= 0");
    if (light_intensity)
      for (uint32_t l = 0; l < s->light_count; ++l)
        if (!std::isfinite(light_intensity[l])) return bad("light " + std::to_string(l) + ": intensity not finite");
    if (albedo_rgb)
      for (uint32_t m = 0; m < s->mat_count; ++m) {
        DMat& M = s->h_mats[m];
        M.use_override = (!use_override || use_override[m]) ? 1 : 0;
        for (int c = 0; c < 3; ++c) M.override_rgb[c] = albedo_rgb[3 * m + c];
      }
    if (light_intensity)
      for (uint32_t l = 0; l < s->light_count; ++l) s->h_lights[l].intensity = light_intensity[l];
    if (albedo_rgb) area_emission_consts(s);  // overrides change area emission
    cudaStream_t st = s->ctx->stream;
    if (albedo_rgb && s->mat_count)
      SHB_CUDA(cudaMemcpyAsync(s->mats.ptr, s->h_mats.data(), sizeof(DMat) * s->mat_count, cudaMemcpyHostToDevice, st));
    if ((light_intensity || albedo_rgb) && s->light_count)
      SHB_CUDA(cudaMemcpyAsync(s->lights.ptr, s->h_lights.data(), sizeof(DLight) * s->light_count,
                               cudaMemcpyHostToDevice, st));
    SHB_CUDA(cudaStreamSynchronize(st));
    return SHB_OK;
  });
}

shb_status shb_backward(shb_scene* s, const shb_gbuffer* g, const shb_raster_config* rc, const shb_bake_config* cfg,
                        const float* d_sh, int32_t device_ptr, double* d_albedo, double* d_light,
                        shb_bake_stats* stats) {
  return ::shb::guarded("shb_backward", [&]() -> shb_status {
    if (!s || !g || !rc || !cfg || !d_sh) return bad("NULL argument");
    if ((s->mat_count && !d_albedo) || (s->light_count && !d_light)) return bad("NULL gradient output");
    if (cfg->samples <= 0) return bad("samples must be positive");
    if (cfg->bounces < 0 || cfg->bounces > 30) return bad("bounces must be in [0, 30]");
    if (cfg->num_light_samples <= 0) return bad("num_light_samples must be positive");
    if (cfg->rng_mode != SHB_RNG_PHILOX) return bad("unknown rng_mode");
    int64_t W = (int64_t)rc->width * rc->supersample_scale, H = (int64_t)rc->height * rc->supersample_scale;
    if (W != g->width || H != g->height) return bad("G-buffer size does not match raster_config (W*s x H*s)");
    if (s->bvh_depth > 64) return bad("BVH deeper than the traversal stack");
    SHB_ON_DEVICE(s->ctx->device);
    shb_context* c = s->ctx;
    uint64_t l0 = c->launches;
    const size_t n = (size_t)W * H;
    const size_t np = 3 * (size_t)s->mat_count + s->light_count;
    SHB_TRY(c->scratch[21].reserve(sizeof(double) * std::max<size_t>(np, 1) +
                                   (device_ptr ? 0 : sizeof(float) * 27 * n)));
    double* dgrad = c->scratch[21].as<double>();
    const float* dsh = d_sh;
    if (!device_ptr) {
      float* tmp = reinterpret_cast<float*>(dgrad + std::max<size_t>(np, 1));
      SHB_CUDA(cudaMemcpyAsync(tmp, d_sh, sizeof(float) * 27 * n, cudaMemcpyHostToDevice, c->stream));
      dsh = tmp;
    }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    SHB_TRY(backward_device(s, g->points.as<shb_surface_point>(), (int)W, (int)H, cfg, dsh, dgrad, stats));
    std::vector<double> h(np);
    if (np) SHB_CUDA(cudaMemcpyAsync(h.data(), dgrad, sizeof(double) * np, cudaMemcpyDeviceToHost, c->stream));
    SHB_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < 3 * (size_t)s->mat_count; ++i) d_albedo[i] = h[i];
    for (size_t l = 0; l < s->light_count; ++l) d_light[l] = h[3 * (size_t)s->mat_count + l];
    if (stats) {
      stats->kernel_launches = c->launches - l0;
      stats->bvh_build_ms = s->bvh_build_ms;
    }
    return SHB_OK;
  });
}

shb_status shb_downsample(shb_context* ctx, const float* in, int32_t in_width, int32_t in_height, int32_t channels,
                          int32_t scale, float* out, int32_t device_ptrs) {
  return ::shb::guarded("shb_downsample", [&]() -> shb_status {
    if (in_width <= 0 || in_height <= 0 || channels <= 0 || scale <= 0) return bad("sizes must be positive");
    if (too_many_texels(in_width, in_height) || (int64_t)in_width * in_height * channels > 27 * kMaxTexels)
      return bad("image larger than 2^31 - 1 texels or 27 * (2^31 - 1) floats");
    if (!ctx || !in || !out) return bad("NULL argument");
    SHB_ON_DEVICE(ctx->device);
    size_t nin = (size_t)in_width * in_height * channels;
    size_t nout = scale <= 1 ? nin : (size_t)(in_width / scale) * (in_height / scale) * channels;
    const float* din = in;
    float* dout = out;
    if (!device_ptrs) {
      SHB_TRY(ctx->scratch[18].reserve(sizeof(float) * nin));
      SHB_TRY(ctx->scratch[19].reserve(sizeof(float) * (nout ? nout : 1)));
      SHB_CUDA(cudaMemcpyAsync(ctx->scratch[18].ptr, in, sizeof(float) * nin, cudaMemcpyHostToDevice, ctx->stream));
      din = ctx->scratch[18].as<float>();
      dout = ctx->scratch[19].as<float>();
    }
    SHB_TRY(downsample_device(ctx, din, in_width, in_height, channels, scale, dout));
    if (!device_ptrs && nout)
      SHB_CUDA(cudaMemcpyAsync(out, dout, sizeof(float) * nout, cudaMemcpyDeviceToHost, ctx->stream));
    SHB_CUDA(cudaStreamSynchronize(ctx->stream));
    return SHB_OK;
  });
}

shb_status shb_dilate(shb_context* ctx, int32_t kind, int32_t width, int32_t height, void* pixels, uint8_t* mask,
                      int32_t passes, int32_t device_ptrs) {
  return ::shb::guarded("shb_dilate", [&]() -> shb_status {
    if (too_many_texels(width, height)) return bad(kTooLarge);
    if (!ctx) return bad("ctx is NULL");
    if (kind < SHB_DILATE_SH9 || kind > SHB_DILATE_U8) return bad("bad dilate kind");
    if (width <= 0 || height <= 0 || passes <= 0) return SHB_OK;  // reference: nothing to do
    if (!pixels || !mask) return bad("NULL argument");
    SHB_ON_DEVICE(ctx->device);
    size_t n = (size_t)width * height;
    size_t pbytes = n * (kind == SHB_DILATE_SH9 ? 27 * 4 : (kind == SHB_DILATE_F32 ? 4 : 1));
    void* dp = pixels;
    uint8_t* dm = mask;
    if (!device_ptrs) {
      SHB_TRY(ctx->scratch[18].reserve(pbytes));
      SHB_TRY(ctx->scratch[19].reserve(n));
      SHB_CUDA(cudaMemcpyAsync(ctx->scratch[18].ptr, pixels, pbytes, cudaMemcpyHostToDevice, ctx->stream));
      SHB_CUDA(cudaMemcpyAsync(ctx->scratch[19].ptr, mask, n, cudaMemcpyHostToDevice, ctx->stream));
      dp = ctx->scratch[18].ptr;
      dm = ctx->scratch[19].as<uint8_t>();
    }
    SHB_TRY(dilate_device(ctx, kind, width, height, dp, dm, passes));
    if (!device_ptrs) {
      SHB_CUDA(cudaMemcpyAsync(pixels, dp, pbytes, cudaMemcpyDeviceToHost, ctx->stream));
      SHB_CUDA(cudaMemcpyAsync(mask, dm, n, cudaMemcpyDeviceToHost, ctx->stream));
    }
    SHB_CUDA(cudaStreamSynchronize(ctx->stream));
    return SHB_OK;
  });
}

shb_status shb_bake_pipeline(shb_scene* s, const shb_pipeline_config* cfg, float* sh_out, float* env_out,
                             uint8_t* mask_out, shb_bake_stats* stats) {
  return ::shb::guarded("shb_bake_pipeline", [&]() -> shb_status {
    if (!s || !cfg || !sh_out || !env_out) return bad("NULL argument");
    if (cfg->width <= 0 || cfg->height <= 0 || cfg->supersample_scale <= 0) return bad("sizes must be positive");
    shb_context* c = s->ctx;
    SHB_ON_DEVICE(c->device);
    const int ss = cfg->supersample_scale;
    shb_raster_config rc{cfg->width, cfg->height, ss};
    if (!c->pipe_gbuf) c->pipe_gbuf = new shb_gbuffer();
    shb_gbuffer* g = c->pipe_gbuf;
    SHB_TRY(rasterize_into(s, &rc, g, nullptr));
    const size_t W = (size_t)cfg->width * ss, H = (size_t)cfg->height * ss;
    const size_t n_hi = W * H, n_lo = (size_t)cfg->width * cfg->height;
    // device buffers: hi-res SH + env, hi-res mask, lo-res SH + env + mask
    SHB_TRY(c->scratch[21].reserve(sizeof(float) * 28 * n_hi + n_hi));
    SHB_TRY(c->scratch[22].reserve(sizeof(float) * 28 * n_lo + n_lo));
    float* sh_hi = c->scratch[21].as<float>();
    float* env_hi = sh_hi + 27 * n_hi;
    uint8_t* mask_hi = reinterpret_cast<uint8_t*>(env_hi + n_hi);
    float* sh_lo = c->scratch[22].as<float>();
    float* env_lo = sh_lo + 27 * n_lo;
    uint8_t* mask_lo = reinterpret_cast<uint8_t*>(env_lo + n_lo);
    shb_bake_config bc;
    std::memset(&bc, 0, sizeof(bc));
    bc.samples = cfg->samples;
    bc.bounces = cfg->bounces;
    bc.num_light_samples = cfg->num_light_samples > 0 ? cfg->num_light_samples : 1;
    bc.seed = cfg->seed;
    bc.rng_mode = SHB_RNG_PHILOX;
    shb_bake_output bo{sh_hi, env_hi, 1, 0};
    SHB_TRY(shb_bake(s, g, &rc, &bc, &bo, stats));
    SHB_TRY(validity_mask_device(c, g->points.as<shb_surface_point>(), (int64_t)n_hi, mask_hi));
    float* sh_fin = sh_hi;
    float* env_fin = env_hi;
    uint8_t* mask_fin = mask_hi;
    if (ss > 1) {
      SHB_TRY(downsample_device(c, sh_hi, (int)W, (int)H, 27, ss, sh_lo));
      SHB_TRY(downsample_device(c, env_hi, (int)W, (int)H, 1, ss, env_lo));
      SHB_TRY(downsample_mask_device(c, mask_hi, cfg->width, cfg->height, ss, mask_lo));
      sh_fin = sh_lo;
      env_fin = env_lo;
      mask_fin = mask_lo;
    }
    if (cfg->dilation > 0) {
      SHB_TRY(dilate_device(c, SHB_DILATE_SH9, cfg->width, cfg->height, sh_fin, mask_fin, cfg->dilation));
      SHB_TRY(dilate_device(c, SHB_DILATE_F32, cfg->width, cfg->height, env_fin, mask_fin, cfg->dilation));
    }
    SHB_CUDA(cudaMemcpyAsync(sh_out, sh_fin, sizeof(float) * 27 * n_lo, cudaMemcpyDeviceToHost, c->stream));
    SHB_CUDA(cudaMemcpyAsync(env_out, env_fin, sizeof(float) * n_lo, cudaMemcpyDeviceToHost, c->stream));
    if (mask_out) SHB_CUDA(cudaMemcpyAsync(mask_out, mask_fin, n_lo, cudaMemcpyDeviceToHost, c->stream));
    SHB_CUDA(cudaStreamSynchronize(c->stream));
    return SHB_OK;
  });
}

shb_status shb_find_occlusion(shb_scene* s, const shb_ray* rays, int64_t count, shb_hit* hits, int32_t device_ptrs) {
  return ::shb::guarded("shb_find_occlusion", [&]() -> shb_status {
    if (count > kMaxTexels) return bad("more than 2^31 - 1 rays in one call");
    if (!s || (count > 0 && (!rays || !hits))) return bad("NULL argument");
    if (count <= 0) return SHB_OK;
    shb_context* c = s->ctx;
    SHB_ON_DEVICE(c->device);
    const shb_ray* dr = rays;
    shb_hit* dh = hits;
    if (!device_ptrs) {
      SHB_TRY(c->scratch[18].reserve(sizeof(shb_ray) * (size_t)count));
      SHB_TRY(c->scratch[19].reserve(sizeof(shb_hit) * (size_t)count));
      SHB_CUDA(cudaMemcpyAsync(c->scratch[18].ptr, rays, sizeof(shb_ray) * (size_t)count, cudaMemcpyHostToDevice,
                               c->stream));
      dr = c->scratch[18].as<shb_ray>();
      dh = c->scratch[19].as<shb_hit>();
    }
    SHB_TRY(find_occlusion_device(s, dr, count, dh));
    if (!device_ptrs)
      SHB_CUDA(cudaMemcpyAsync(hits, dh, sizeof(shb_hit) * (size_t)count, cudaMemcpyDeviceToHost, c->stream));
    SHB_CUDA(cudaStreamSynchronize(c->stream));
    return SHB_OK;
  });
}

}  // extern "C"
