// sh_baker/sh_baker.h - C++ mirror of sh-baker's bake API over the C ABI
// (shb.h).  Header-only; link against libshb.so.
//
// Same names, structs, field order and argument meaning as the reference:
//   Texture, Texture32F, Material, Geometry, Light, Scene   (src/scene.h:18-115)
//   RasterConfig, SurfacePoint                              (src/rasterizer.h:12-23)
//   BakeConfig, BakeResult                                  (src/baker.h:10-19)
//   SHCoeffs, SHTexture                                     (src/sh_coeffs.h:10-23, src/saver.h:12-16)
//   RasterizeScene, CreateValidityMask, DownsampleValidityMask (src/rasterizer.h:27-39)
//   BakeSHLightMap, DownsampleSHTexture,
//   DownsampleEnvironmentVisibilityTexture                  (src/baker.h:25-36)
//   Dilate<T> for SHCoeffs, float, uint8_t                  (src/dilation.h:14-16)
//   SaveMode, SaveSHLightMap                                (src/saver.h:21-48)
//   CreateAtlasGeometries, atlas_internal::CalculateGeometryScales (src/atlas.h:10-53)
//   LoadScene, SaveScene                                    (src/loader.h:13, src/saver.h:50-53)
//   TransformedVertices / Normals / Tangents, SurfaceArea   (src/scene.h:117-123)
// Where the reference CHECK-fails these throw sh_baker::Error.  With Eigen
// available the vector types are Eigen's; otherwise small POD stand-ins with
// the same memory layout and accessors are used.
#ifndef SH_BAKER_B200_SH_BAKER_H_
#define SH_BAKER_B200_SH_BAKER_H_

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <type_traits>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../shb.h"

#if __has_include(<Eigen/Dense>)
#include <Eigen/Dense>
#define SH_BAKER_HAS_EIGEN 1
#endif

namespace sh_baker {

#ifdef SH_BAKER_HAS_EIGEN
using Vector2f = Eigen::Vector2f;
using Vector3f = Eigen::Vector3f;
using Vector4f = Eigen::Vector4f;
using Affine3f = Eigen::Affine3f;
inline void affine_rows(const Affine3f& a, float out[12]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) out[r * 4 + c] = a.matrix()(r, c);
}
#else
template <int N>
struct VecN {
  float v[N];
  VecN() { for (int i = 0; i < N; ++i) v[i] = 0.f; }
  template <class... T>
  VecN(T... xs) : v{static_cast<float>(xs)...} {}
  float& operator[](int i) { return v[i]; }
  float operator[](int i) const { return v[i]; }
  float& x() { return v[0]; }
  float& y() { return v[1]; }
  float x() const { return v[0]; }
  float y() const { return v[1]; }
  template <int M = N, class = std::enable_if_t<(M > 2)>>
  float z() const { return v[2]; }
  template <int M = N, class = std::enable_if_t<(M > 3)>>
  float w() const { return v[3]; }
  static VecN Zero() { return VecN(); }
};
using Vector2f = VecN<2>;
using Vector3f = VecN<3>;
struct alignas(16) Vector4f : VecN<4> {
  using VecN<4>::VecN;
};
struct Affine3f {
  float m[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};  // row-major [L | t]
  static Affine3f Identity() { return Affine3f(); }
};
inline void affine_rows(const Affine3f& a, float out[12]) { std::memcpy(out, a.m, sizeof(a.m)); }
#endif

struct Error : std::runtime_error {
  shb_status status;
  Error(shb_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(shb_status s) {
  if (s != SHB_OK) throw Error(s, std::string("shb: ") + shb_last_error());
}

// ---- src/scene.h:18-115 ----------------------------------------------------

struct Texture {
  std::optional<std::filesystem::path> file_path;
  uint32_t width = 0;
  uint32_t height = 0;
  uint32_t channels = 0;
  std::vector<uint8_t> pixel_data;
};

struct Texture32F {
  std::optional<std::filesystem::path> file_path;
  uint32_t width = 0;
  uint32_t height = 0;
  uint32_t channels = 0;
  std::vector<float> pixel_data;
};

struct Material {
  std::string name;
  Texture albedo;
  Texture normal_texture;
  Texture metallic_roughness_texture;
  float emission_intensity = 0.0f;
};

struct Geometry {
  std::vector<Vector3f> vertices;
  std::vector<Vector3f> normals;
  std::vector<Vector2f> texture_uvs;
  std::vector<Vector2f> lightmap_uvs;
  std::vector<Vector4f> tangents;
  std::vector<uint32_t> indices;
  int material_id = -1;
  Affine3f transform = Affine3f::Identity();
};

struct Light {
  enum class Type { Point, Directional, Spot, Area };
  Type type = Type::Point;
  Vector3f position = Vector3f(0.f, 0.f, 0.f);
  Vector3f direction = Vector3f(0.f, 0.f, -1.f);
  Vector3f color = Vector3f(1.f, 1.f, 1.f);
  float intensity = 1.0f;
  float cos_inner_cone = 1.0f;
  float cos_outer_cone = 0.70710678118654752440f;
  float area = 0.0f;
  const Material* material = nullptr;
  const Geometry* geometry = nullptr;
  int geometry_index = -1;
};

struct Scene {
  std::vector<Geometry> geometries;
  std::vector<Material> materials;
  std::vector<Light> lights;
};

// ---- src/rasterizer.h:12-23, src/baker.h:10-19, src/sh_coeffs.h ------------

struct RasterConfig {
  int width = 1024;
  int height = 1024;
  int supersample_scale = 1;
};

struct SurfacePoint {
  Vector3f position = Vector3f(0.f, 0.f, 0.f);
  Vector3f normal = Vector3f(0.f, 0.f, 0.f);
  Vector4f tangent = Vector4f(0.f, 0.f, 0.f, 0.f);
  int32_t material_id = -1;
};
static_assert(sizeof(SurfacePoint) == sizeof(shb_surface_point), "SurfacePoint layout");

struct SHCoeffs {
  Vector3f coeffs[9];
};
static_assert(sizeof(SHCoeffs) == 27 * sizeof(float), "SHCoeffs layout");

struct SHTexture {
  int width = 0;
  int height = 0;
  std::vector<SHCoeffs> pixels;
};

struct BakeConfig {
  int samples = 128;
  int bounces = 3;
  int num_light_samples = 1;
};

struct BakeResult {
  SHTexture sh_texture;
  Texture32F environment_visibility_texture;
};

// ---- device plumbing ---------------------------------------------------------

namespace detail {

// One context per host thread, on device 0 (SHB_DEVICE overrides).
inline shb_context* context() {
  struct Holder {
    shb_context* ctx = nullptr;
    ~Holder() {
      if (ctx) shb_context_destroy(ctx);
    }
  };
  static thread_local Holder h;
  if (!h.ctx) {
    shb_options o{};
    const char* d = std::getenv("SHB_DEVICE");
    const long dv = d ? std::strtol(d, nullptr, 10) : 0;  // outside int32: -1, refused
    o.device = dv < INT32_MIN || dv > INT32_MAX ? -1 : (int)dv;
    check(shb_context_create(&o, &h.ctx));
  }
  return h.ctx;
}

struct SceneHandle {
  shb_scene* s = nullptr;
  ~SceneHandle() { shb_scene_destroy(s); }
};

// A shb_scene_desc pointing into `scene` and the arrays below.
struct Desc {
  std::vector<shb_geometry_desc> g;
  std::vector<shb_material_desc> m;
  std::vector<shb_light_desc> l;
  shb_scene_desc d{};
};

inline void describe(const Scene& scene, Desc* out) {
  std::vector<shb_geometry_desc>& g = out->g;
  g.assign(scene.geometries.size(), shb_geometry_desc{});
  for (size_t i = 0; i < g.size(); ++i) {
    const Geometry& G = scene.geometries[i];
    shb_geometry_desc& d = g[i];
    std::memset(&d, 0, sizeof(d));
    d.vertices = G.vertices.empty() ? nullptr : reinterpret_cast<const float*>(G.vertices.data());
    d.normals = G.normals.empty() ? nullptr : reinterpret_cast<const float*>(G.normals.data());
    d.texture_uvs = G.texture_uvs.empty() ? nullptr : reinterpret_cast<const float*>(G.texture_uvs.data());
    d.lightmap_uvs = G.lightmap_uvs.empty() ? nullptr : reinterpret_cast<const float*>(G.lightmap_uvs.data());
    d.tangents = G.tangents.empty() ? nullptr : reinterpret_cast<const float*>(G.tangents.data());
    d.vertex_count = (uint32_t)G.vertices.size();
    d.indices = G.indices.data();
    d.index_count = (uint32_t)G.indices.size();
    d.material_id = G.material_id;
    affine_rows(G.transform, d.transform);
  }
  std::vector<shb_material_desc>& m = out->m;
  m.assign(scene.materials.size(), shb_material_desc{});
  for (size_t i = 0; i < m.size(); ++i) {
    const Material& M = scene.materials[i];
    m[i].albedo_pixels = M.albedo.pixel_data.empty() ? nullptr : M.albedo.pixel_data.data();
    m[i].albedo_width = M.albedo.width;
    m[i].albedo_height = M.albedo.height;
    m[i].albedo_channels = M.albedo.channels;
    m[i].emission_intensity = M.emission_intensity;
  }
  std::vector<shb_light_desc>& l = out->l;
  l.assign(scene.lights.size(), shb_light_desc{});
  for (size_t i = 0; i < l.size(); ++i) {
    const Light& L = scene.lights[i];
    shb_light_desc& d = l[i];
    d.type = (int32_t)L.type;
    for (int k = 0; k < 3; ++k) {
      d.position[k] = L.position[k];
      d.direction[k] = L.direction[k];
      d.color[k] = L.color[k];
    }
    d.intensity = L.intensity;
    d.cos_inner_cone = L.cos_inner_cone;
    d.cos_outer_cone = L.cos_outer_cone;
    d.area = L.area;
    d.geometry_index = L.geometry_index;
    if (d.geometry_index < 0 && L.geometry) d.geometry_index = (int32_t)(L.geometry - scene.geometries.data());
    d.material_index = L.material ? (int32_t)(L.material - scene.materials.data()) : -1;
  }
  out->d = shb_scene_desc{g.data(), (uint32_t)g.size(), m.data(), (uint32_t)m.size(), l.data(), (uint32_t)l.size()};
}

inline void upload(const Scene& scene, SceneHandle* out) {
  Desc D;
  describe(scene, &D);
  check(shb_scene_upload(context(), &D.d, &out->s));
}

}  // namespace detail

// ---- src/atlas.h:10-53 -----------------------------------------------------

namespace atlas_internal {

// Per geometry: density * sqrt(albedo w*h) * sqrt(UV tile count), clamped
// to 5x the median (shb_atlas_geometry_scales).
inline std::vector<float> CalculateGeometryScales(const std::vector<Geometry>& geometries,
                                                  const std::vector<Material>& materials, float density_multiplier) {
  std::vector<shb_geometry_desc> g(geometries.size(), shb_geometry_desc{});
  for (size_t i = 0; i < g.size(); ++i) {
    g[i].texture_uvs = geometries[i].texture_uvs.empty()
                           ? nullptr
                           : reinterpret_cast<const float*>(geometries[i].texture_uvs.data());
    g[i].vertex_count = (uint32_t)geometries[i].texture_uvs.size();
    g[i].material_id = geometries[i].material_id;
  }
  std::vector<shb_material_desc> m(materials.size(), shb_material_desc{});
  for (size_t i = 0; i < m.size(); ++i) {
    m[i].albedo_width = materials[i].albedo.width;
    m[i].albedo_height = materials[i].albedo.height;
  }
  shb_scene_desc d{g.data(), (uint32_t)g.size(), m.data(), (uint32_t)m.size(), nullptr, 0};
  std::vector<float> out(geometries.size());
  check(shb_atlas_geometry_scales(&d, density_multiplier, out.data()));
  return out;
}

}  // namespace atlas_internal

struct AtlasResult {
  std::vector<Geometry> geometries;
  int width;
  int height;
};

// New geometries with non-overlapping lightmap UVs (shb_create_atlas);
// nullopt when the charts do not fit one page, like the reference.
inline std::optional<AtlasResult> CreateAtlasGeometries(const Scene& scene, unsigned target_resolution,
                                                        unsigned padding, float density_multiplier = 1.0f) {
  detail::Desc D;
  detail::describe(scene, &D);
  shb_host_scene* hs = nullptr;
  int32_t w = 0, h = 0;
  if (shb_create_atlas(&D.d, target_resolution, padding, density_multiplier, &hs, &w, &h) != SHB_OK)
    return std::nullopt;
  const shb_scene_desc* out = shb_host_scene_desc(hs);
  AtlasResult r;
  r.width = w;
  r.height = h;
  for (uint32_t i = 0; i < out->geometry_count; ++i) {
    const shb_geometry_desc& d = out->geometries[i];
    Geometry G;
    G.material_id = d.material_id;
    G.transform = scene.geometries[i].transform;
    for (uint32_t v = 0; v < d.vertex_count; ++v) {
      G.vertices.push_back(Vector3f(d.vertices[3 * v], d.vertices[3 * v + 1], d.vertices[3 * v + 2]));
      G.normals.push_back(Vector3f(d.normals[3 * v], d.normals[3 * v + 1], d.normals[3 * v + 2]));
      G.texture_uvs.push_back(Vector2f(d.texture_uvs[2 * v], d.texture_uvs[2 * v + 1]));
      G.lightmap_uvs.push_back(Vector2f(d.lightmap_uvs[2 * v], d.lightmap_uvs[2 * v + 1]));
      G.tangents.push_back(
          Vector4f(d.tangents[4 * v], d.tangents[4 * v + 1], d.tangents[4 * v + 2], d.tangents[4 * v + 3]));
    }
    G.indices.assign(d.indices, d.indices + d.index_count);
    r.geometries.push_back(std::move(G));
  }
  shb_host_scene_destroy(hs);
  return r;
}

// ---- src/loader.h:13, src/saver.h:50-53 ------------------------------------

namespace detail {

inline Affine3f affine_from_rows(const float r[12]) {
#ifdef SH_BAKER_HAS_EIGEN
  Affine3f a = Affine3f::Identity();
  for (int i = 0; i < 3; ++i)
    for (int c = 0; c < 4; ++c) a.matrix()(i, c) = r[i * 4 + c];
  return a;
#else
  Affine3f a;
  std::memcpy(a.m, r, sizeof(a.m));
  return a;
#endif
}

// A geometry description as a Geometry; absent attributes stay empty.
inline Geometry geometry_from(const shb_geometry_desc& d) {
  Geometry G;
  G.material_id = d.material_id;
  G.transform = affine_from_rows(d.transform);
  for (uint32_t v = 0; v < d.vertex_count; ++v) {
    if (d.vertices) G.vertices.push_back(Vector3f(d.vertices[3 * v], d.vertices[3 * v + 1], d.vertices[3 * v + 2]));
    if (d.normals) G.normals.push_back(Vector3f(d.normals[3 * v], d.normals[3 * v + 1], d.normals[3 * v + 2]));
    if (d.texture_uvs) G.texture_uvs.push_back(Vector2f(d.texture_uvs[2 * v], d.texture_uvs[2 * v + 1]));
    if (d.lightmap_uvs) G.lightmap_uvs.push_back(Vector2f(d.lightmap_uvs[2 * v], d.lightmap_uvs[2 * v + 1]));
    if (d.tangents)
      G.tangents.push_back(
          Vector4f(d.tangents[4 * v], d.tangents[4 * v + 1], d.tangents[4 * v + 2], d.tangents[4 * v + 3]));
  }
  if (d.indices) G.indices.assign(d.indices, d.indices + d.index_count);
  return G;
}

}  // namespace detail

// A .gltf / .glb file through shb_load_gltf (host code, no GPU); nullopt
// on failure, like the reference, with the reason in shb_last_error().
// Each area light points at its material and geometry in the returned
// scene, as the reference fixes them up after loading
// (src/loader.cpp:835-839); moving the Scene keeps them valid, copying it
// does not.
inline std::optional<Scene> LoadScene(const std::filesystem::path& path) {
  shb_host_scene* hs = nullptr;
  if (shb_load_gltf(path.string().c_str(), &hs) != SHB_OK) return std::nullopt;
  struct Owned {
    shb_host_scene* h;
    ~Owned() { shb_host_scene_destroy(h); }
  } owned{hs};
  const shb_scene_desc* d = shb_host_scene_desc(hs);
  Scene scene;
  for (uint32_t g = 0; g < d->geometry_count; ++g) scene.geometries.push_back(detail::geometry_from(d->geometries[g]));
  for (uint32_t m = 0; m < d->material_count; ++m) {
    const shb_material_desc& md = d->materials[m];
    Material M;
    const char* name = nullptr;
    const char* file = nullptr;
    check(shb_host_scene_material_info(hs, (int32_t)m, &name, &file));
    M.name = name ? name : "";
    if (file) M.albedo.file_path = std::filesystem::path(file);
    M.albedo.width = md.albedo_width;
    M.albedo.height = md.albedo_height;
    M.albedo.channels = md.albedo_channels;
    if (md.albedo_pixels)
      M.albedo.pixel_data.assign(md.albedo_pixels,
                                 md.albedo_pixels + (size_t)md.albedo_width * md.albedo_height * md.albedo_channels);
    M.emission_intensity = md.emission_intensity;
    scene.materials.push_back(std::move(M));
  }
  for (uint32_t l = 0; l < d->light_count; ++l) {
    const shb_light_desc& ld = d->lights[l];
    Light L;
    L.type = static_cast<Light::Type>(ld.type);
    L.position = Vector3f(ld.position[0], ld.position[1], ld.position[2]);
    L.direction = Vector3f(ld.direction[0], ld.direction[1], ld.direction[2]);
    L.color = Vector3f(ld.color[0], ld.color[1], ld.color[2]);
    L.intensity = ld.intensity;
    L.cos_inner_cone = ld.cos_inner_cone;
    L.cos_outer_cone = ld.cos_outer_cone;
    L.area = ld.area;
    L.geometry_index = ld.geometry_index;
    scene.lights.push_back(L);
  }
  for (size_t l = 0; l < scene.lights.size(); ++l) {
    const shb_light_desc& ld = d->lights[l];
    if (ld.material_index >= 0 && (size_t)ld.material_index < scene.materials.size())
      scene.lights[l].material = &scene.materials[(size_t)ld.material_index];
    if (ld.geometry_index >= 0 && (size_t)ld.geometry_index < scene.geometries.size())
      scene.lights[l].geometry = &scene.geometries[(size_t)ld.geometry_index];
  }
  return std::optional<Scene>(std::move(scene));
}

// glTF + <stem>.bin through shb_save_gltf, with each material's name and
// albedo image file (copied beside the output); false on failure, like
// the reference.
inline bool SaveScene(const Scene& scene, const std::filesystem::path& path) {
  detail::Desc D;
  detail::describe(scene, &D);
  const size_t n = scene.materials.size();
  std::vector<std::string> files(n);
  std::vector<const char*> names(n), paths(n);
  for (size_t i = 0; i < n; ++i) {
    names[i] = scene.materials[i].name.c_str();
    if (scene.materials[i].albedo.file_path) files[i] = scene.materials[i].albedo.file_path->string();
    paths[i] = files[i].empty() ? nullptr : files[i].c_str();
  }
  return shb_save_gltf(&D.d, n ? names.data() : nullptr, n ? paths.data() : nullptr, path.string().c_str()) ==
         SHB_OK;
}

// ---- src/scene.h:117-123 ---------------------------------------------------
// World-space attributes (src/scene.cpp:162-207), with the float products
// in the order the library's upload uses: v' = L v + t, n' = normalize(R n),
// t' = (normalize(R t.xyz), t.w), R the rotation part of L
// (shb_rotation_part).

namespace detail {

inline Vector3f mat_vec(const float* m, int stride, float x, float y, float z) {
  return Vector3f(m[0] * x + (m[1] * y + m[2] * z), m[stride] * x + (m[stride + 1] * y + m[stride + 2] * z),
                  m[2 * stride] * x + (m[2 * stride + 1] * y + m[2 * stride + 2] * z));
}

inline Vector3f normalized(const Vector3f& v) {
  const float n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  return Vector3f(v[0] / n, v[1] / n, v[2] / n);
}

inline void rotation_of(const Affine3f& a, float R[9]) {
  float rows[12];
  affine_rows(a, rows);
  check(shb_rotation_part(rows, R));
}

}  // namespace detail

inline std::vector<Vector3f> TransformedVertices(const Geometry& geometry) {
  float rows[12];
  affine_rows(geometry.transform, rows);
  std::vector<Vector3f> out;
  out.reserve(geometry.vertices.size());
  for (const Vector3f& v : geometry.vertices) {
    const Vector3f m = detail::mat_vec(rows, 4, v[0], v[1], v[2]);
    out.push_back(Vector3f(m[0] + rows[3], m[1] + rows[7], m[2] + rows[11]));
  }
  return out;
}

inline std::vector<Vector3f> TransformedNormals(const Geometry& geometry) {
  float R[9];
  detail::rotation_of(geometry.transform, R);
  std::vector<Vector3f> out;
  out.reserve(geometry.normals.size());
  for (const Vector3f& n : geometry.normals) out.push_back(detail::normalized(detail::mat_vec(R, 3, n[0], n[1], n[2])));
  return out;
}

inline std::vector<Vector4f> TransformedTangents(const Geometry& geometry) {
  float R[9];
  detail::rotation_of(geometry.transform, R);
  std::vector<Vector4f> out;
  out.reserve(geometry.tangents.size());
  for (const Vector4f& t : geometry.tangents) {
    const Vector3f r = detail::normalized(detail::mat_vec(R, 3, t[0], t[1], t[2]));
    out.push_back(Vector4f(r[0], r[1], r[2], t[3]));
  }
  return out;
}

// Object-space area: the sum of 0.5 |(v1 - v0) x (v2 - v0)| over triangles.
inline float SurfaceArea(const Geometry& geometry) {
  float total = 0.0f;
  for (size_t i = 0; i + 2 < geometry.indices.size(); i += 3) {
    const Vector3f& a = geometry.vertices[geometry.indices[i]];
    const Vector3f& b = geometry.vertices[geometry.indices[i + 1]];
    const Vector3f& c = geometry.vertices[geometry.indices[i + 2]];
    const float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    const float x = e1[1] * e2[2] - e1[2] * e2[1], y = e1[2] * e2[0] - e1[0] * e2[2], z = e1[0] * e2[1] - e1[1] * e2[0];
    total += 0.5f * std::sqrt(x * x + y * y + z * z);
  }
  return total;
}

// ---- src/rasterizer.h:27-39 ------------------------------------------------

inline std::vector<SurfacePoint> RasterizeScene(const Scene& scene, const RasterConfig& config) {
  detail::SceneHandle s;
  detail::upload(scene, &s);
  std::vector<SurfacePoint> out((size_t)config.width * config.supersample_scale * config.height *
                                config.supersample_scale);
  shb_raster_config rc{config.width, config.height, config.supersample_scale};
  check(shb_rasterize(s.s, &rc, reinterpret_cast<shb_surface_point*>(out.data()), nullptr));
  return out;
}

inline std::vector<uint8_t> CreateValidityMask(const std::vector<SurfacePoint>& points) {
  std::vector<uint8_t> mask(points.size());
  if (points.empty()) return mask;
  shb_gbuffer* g = nullptr;
  check(shb_gbuffer_upload(detail::context(), reinterpret_cast<const shb_surface_point*>(points.data()),
                           (int32_t)points.size(), 1, &g));
  shb_status st = shb_validity_mask(detail::context(), g, mask.data(), 0);
  shb_gbuffer_destroy(g);
  check(st);
  return mask;
}

inline std::vector<uint8_t> DownsampleValidityMask(const std::vector<uint8_t>& high_res_mask, int width,
                                                   int height, int scale) {
  if (high_res_mask.size() != (size_t)width * height * scale * scale)
    throw Error(SHB_ERR_INVALID_ARG, "DownsampleValidityMask: size mismatch (CHECK_EQ in the reference)");
  std::vector<uint8_t> mask((size_t)width * height, 0);
  check(shb_downsample_validity_mask(detail::context(), high_res_mask.data(), width, height, scale, mask.data(), 0));
  return mask;
}

// ---- src/baker.h:25-36 -----------------------------------------------------

inline BakeResult BakeSHLightMap(const Scene& scene, const std::vector<SurfacePoint>& surface_points,
                                 const RasterConfig& raster_config, const BakeConfig& config,
                                 uint32_t seed = 12345) {
  detail::SceneHandle s;
  detail::upload(scene, &s);
  const int W = raster_config.width * raster_config.supersample_scale;
  const int H = raster_config.height * raster_config.supersample_scale;
  BakeResult r;
  r.sh_texture.width = W;
  r.sh_texture.height = H;
  r.sh_texture.pixels.resize((size_t)W * H);
  r.environment_visibility_texture.width = W;
  r.environment_visibility_texture.height = H;
  r.environment_visibility_texture.pixel_data.resize((size_t)W * H);
  shb_gbuffer* g = nullptr;
  check(shb_gbuffer_upload(detail::context(), reinterpret_cast<const shb_surface_point*>(surface_points.data()), W,
                           H, &g));
  shb_raster_config rc{raster_config.width, raster_config.height, raster_config.supersample_scale};
  shb_bake_config bc{};
  bc.samples = config.samples;
  bc.bounces = config.bounces;
  bc.num_light_samples = config.num_light_samples;
  bc.seed = seed;
  bc.rng_mode = SHB_RNG_PHILOX;
  shb_bake_output out{reinterpret_cast<float*>(r.sh_texture.pixels.data()),
                      r.environment_visibility_texture.pixel_data.data(), 0, 0};
  shb_status st = shb_bake(s.s, g, &rc, &bc, &out, nullptr);
  shb_gbuffer_destroy(g);
  check(st);
  return r;
}

inline SHTexture DownsampleSHTexture(const SHTexture& input, int scale) {
  SHTexture out;
  out.width = input.width / scale;
  out.height = input.height / scale;
  if (scale <= 1) {
    out.width = input.width;
    out.height = input.height;
  }
  out.pixels.resize((size_t)out.width * out.height);
  if (input.pixels.empty() || out.pixels.empty()) return out;
  check(shb_downsample(detail::context(), reinterpret_cast<const float*>(input.pixels.data()), input.width,
                       input.height, 27, scale, reinterpret_cast<float*>(out.pixels.data()), 0));
  return out;
}

inline Texture32F DownsampleEnvironmentVisibilityTexture(const Texture32F& input, int scale) {
  Texture32F out;
  out.width = scale <= 1 ? input.width : input.width / scale;
  out.height = scale <= 1 ? input.height : input.height / scale;
  out.pixel_data.resize((size_t)out.width * out.height);
  if (input.pixel_data.empty() || out.pixel_data.empty()) return out;
  check(shb_downsample(detail::context(), input.pixel_data.data(), (int)input.width, (int)input.height, 1, scale,
                       out.pixel_data.data(), 0));
  return out;
}

// ---- src/saver.h:21-48 -------------------------------------------------------

enum class SaveMode { kCombined, kSplitChannels, kLuminancePacked };

// Writes the SH lightmap as OpenEXR (half, ZIP) in the reference's layouts;
// false on an empty texture or a write failure (the reference logs those).
inline bool SaveSHLightMap(const SHTexture& sh_texture, const Texture32F& environment_visibility_texture,
                           const std::string& path, SaveMode mode = SaveMode::kCombined) {
  if (sh_texture.pixels.empty() || sh_texture.width <= 0 || sh_texture.height <= 0) return false;
  const size_t n = (size_t)sh_texture.width * sh_texture.height;
  std::vector<float> env(n, 0.0f);
  const auto& e = environment_visibility_texture.pixel_data;
  std::copy(e.begin(), e.begin() + std::min(e.size(), n), env.begin());
  return shb_save_sh_lightmap(detail::context(), reinterpret_cast<const float*>(sh_texture.pixels.data()),
                              env.data(), sh_texture.width, sh_texture.height, 0, path.c_str(),
                              (int32_t)mode) == SHB_OK;
}

// ---- differentiable bake (no counterpart in the reference) ------------------

// Adjoint parameters: a linear base colour per material that replaces its
// albedo texture, and an intensity per light.  Empty vectors keep the
// scene's own values.
struct BakeParams {
  std::vector<Vector3f> albedo;
  std::vector<float> light_intensity;
};

// dLoss / d BakeParams: 3 per material (materials without an override: 0)
// and 1 per light (area lights: 0; their radiance is the emissive
// material's albedo times its emission).
struct BakeGradients {
  std::vector<double> d_albedo;
  std::vector<double> d_light_intensity;
};

namespace detail {
inline void set_params(shb_scene* s, const Scene& scene, const BakeParams& p) {
  if (!p.albedo.empty() && p.albedo.size() != scene.materials.size())
    throw Error(SHB_ERR_INVALID_ARG, "BakeParams::albedo: one entry per material");
  if (!p.light_intensity.empty() && p.light_intensity.size() != scene.lights.size())
    throw Error(SHB_ERR_INVALID_ARG, "BakeParams::light_intensity: one entry per light");
  std::vector<float> rgb;
  for (const Vector3f& a : p.albedo)
    for (int k = 0; k < 3; ++k) rgb.push_back(a[k]);
  check(shb_scene_set_params(s, rgb.empty() ? nullptr : rgb.data(), nullptr,
                             p.light_intensity.empty() ? nullptr : p.light_intensity.data()));
}
inline shb_bake_config bake_config(const BakeConfig& config, uint32_t seed) {
  shb_bake_config bc{};
  bc.samples = config.samples;
  bc.bounces = config.bounces;
  bc.num_light_samples = config.num_light_samples;
  bc.seed = seed;
  bc.rng_mode = SHB_RNG_PHILOX;
  return bc;
}
}  // namespace detail

// BakeSHLightMap with adjoint parameters applied.
inline BakeResult BakeSHLightMap(const Scene& scene, const std::vector<SurfacePoint>& surface_points,
                                 const RasterConfig& raster_config, const BakeConfig& config,
                                 const BakeParams& params, uint32_t seed = 12345) {
  detail::SceneHandle s;
  detail::upload(scene, &s);
  detail::set_params(s.s, scene, params);
  const int W = raster_config.width * raster_config.supersample_scale;
  const int H = raster_config.height * raster_config.supersample_scale;
  BakeResult r;
  r.sh_texture.width = W;
  r.sh_texture.height = H;
  r.sh_texture.pixels.resize((size_t)W * H);
  r.environment_visibility_texture.width = W;
  r.environment_visibility_texture.height = H;
  r.environment_visibility_texture.pixel_data.resize((size_t)W * H);
  shb_gbuffer* g = nullptr;
  check(shb_gbuffer_upload(detail::context(), reinterpret_cast<const shb_surface_point*>(surface_points.data()), W,
                           H, &g));
  shb_raster_config rc{raster_config.width, raster_config.height, raster_config.supersample_scale};
  shb_bake_config bc = detail::bake_config(config, seed);
  shb_bake_output out{reinterpret_cast<float*>(r.sh_texture.pixels.data()),
                      r.environment_visibility_texture.pixel_data.data(), 0, 0};
  shb_status st = shb_bake(s.s, g, &rc, &bc, &out, nullptr);
  shb_gbuffer_destroy(g);
  check(st);
  return r;
}

// Path-replay adjoint of the bake above: d_sh = dLoss/dSH per texel of the
// supersampled G-buffer; returns dLoss/d params.  Same seed, same paths.
inline BakeGradients Backward(const Scene& scene, const std::vector<SurfacePoint>& surface_points,
                              const RasterConfig& raster_config, const BakeConfig& config,
                              const BakeParams& params, const SHTexture& d_sh, uint32_t seed = 12345) {
  const int W = raster_config.width * raster_config.supersample_scale;
  const int H = raster_config.height * raster_config.supersample_scale;
  if (d_sh.pixels.size() != (size_t)W * H || surface_points.size() != (size_t)W * H)
    throw Error(SHB_ERR_INVALID_ARG, "Backward: d_sh and surface_points must have W*s x H*s texels");
  detail::SceneHandle s;
  detail::upload(scene, &s);
  detail::set_params(s.s, scene, params);
  shb_gbuffer* g = nullptr;
  check(shb_gbuffer_upload(detail::context(), reinterpret_cast<const shb_surface_point*>(surface_points.data()), W,
                           H, &g));
  shb_raster_config rc{raster_config.width, raster_config.height, raster_config.supersample_scale};
  shb_bake_config bc = detail::bake_config(config, seed);
  BakeGradients out;
  out.d_albedo.assign(3 * scene.materials.size(), 0.0);
  out.d_light_intensity.assign(scene.lights.size(), 0.0);
  shb_status st = shb_backward(s.s, g, &rc, &bc, reinterpret_cast<const float*>(d_sh.pixels.data()), 0,
                               out.d_albedo.data(), out.d_light_intensity.data(), nullptr);
  shb_gbuffer_destroy(g);
  check(st);
  return out;
}

// ---- src/dilation.h:14-16 --------------------------------------------------

template <typename T>
inline void Dilate(int width, int height, std::vector<T>& pixels, std::vector<uint8_t>& mask, int passes = 1) {
  static_assert(std::is_same<T, SHCoeffs>::value || std::is_same<T, float>::value ||
                    std::is_same<T, uint8_t>::value,
                "Dilate is instantiated for SHCoeffs, float and uint8_t");
  if (pixels.empty() || mask.empty() || pixels.size() != mask.size()) return;
  int kind = std::is_same<T, SHCoeffs>::value ? SHB_DILATE_SH9
             : std::is_same<T, float>::value  ? SHB_DILATE_F32
                                              : SHB_DILATE_U8;
  check(shb_dilate(detail::context(), kind, width, height, pixels.data(), mask.data(), passes, 0));
}

}  // namespace sh_baker

#endif  // SH_BAKER_B200_SH_BAKER_H_
