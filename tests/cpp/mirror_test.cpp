// The reference's own unit tests, restated against the C++ mirror
// (include/sh_baker/sh_baker.h) so they run on the CUDA library:
//   src/rasterizer_test.cpp:7-126, src/dilation_test.cpp:11-58,
//   src/baker_test.cpp:10-88, src/atlas_test.cpp:9-170.
// Exit status 0 when every check passes; with --host only the host-side
// tests (atlas) run, no GPU needed.
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <string>

#include "sh_baker/sh_baker.h"

using namespace sh_baker;

static int failures = 0;
#define EXPECT(cond)                                                  \
  do {                                                                \
    if (!(cond)) {                                                    \
      std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);   \
      ++failures;                                                     \
    }                                                                 \
  } while (0)

static Geometry Quad() {
  Geometry quad;
  quad.material_id = 0;
  quad.vertices = {Vector3f(-1, -1, 0), Vector3f(1, -1, 0), Vector3f(1, 1, 0), Vector3f(-1, 1, 0)};
  quad.normals = {Vector3f(0, 0, 1), Vector3f(0, 0, 1), Vector3f(0, 0, 1), Vector3f(0, 0, 1)};
  quad.texture_uvs = {Vector2f(0, 0), Vector2f(1, 0), Vector2f(1, 1), Vector2f(0, 1)};
  quad.lightmap_uvs = quad.texture_uvs;
  quad.tangents = {Vector4f(1, 0, 0, 1), Vector4f(1, 0, 0, 1), Vector4f(1, 0, 0, 1), Vector4f(1, 0, 0, 1)};
  quad.indices = {0, 1, 2, 0, 2, 3};
  return quad;
}

static void RasterizeQuad() {
  Scene scene;
  scene.geometries.push_back(Quad());
  scene.materials.push_back(Material{});
  RasterConfig config;
  config.width = 4;
  config.height = 4;
  std::vector<SurfacePoint> result = RasterizeScene(scene, config);
  EXPECT(result.size() == 16);
  for (int i = 0; i < 16; ++i) EXPECT(result[i].material_id >= 0);
  EXPECT(std::fabs(result[5].position[0] + 0.25f) < 0.001f);
  EXPECT(std::fabs(result[5].position[1] + 0.25f) < 0.001f);
  EXPECT(std::fabs(result[5].normal[2] - 1.0f) < 0.001f);
  config.supersample_scale = 2;
  result = RasterizeScene(scene, config);
  EXPECT(result.size() == 64);
  for (int i = 0; i < 64; ++i) EXPECT(result[i].material_id >= 0);
}

static void Masks() {
  std::vector<SurfacePoint> points(3);
  points[0].material_id = 0;
  points[1].material_id = -1;
  points[2].material_id = 0;
  std::vector<uint8_t> mask = CreateValidityMask(points);
  EXPECT(mask.size() == 3 && mask[0] == 1 && mask[1] == 0 && mask[2] == 1);
  std::vector<uint8_t> hi(16, 0);
  hi[2] = hi[8] = hi[9] = hi[12] = hi[13] = hi[15] = 1;
  std::vector<uint8_t> lo = DownsampleValidityMask(hi, 2, 2, 2);
  EXPECT(lo.size() == 4 && lo[0] == 0 && lo[1] == 1 && lo[2] == 1 && lo[3] == 1);
}

static void Dilation() {
  std::vector<SHCoeffs> pixels(9);
  std::vector<uint8_t> mask(9, 0);
  mask[4] = 1;
  pixels[4].coeffs[0] = Vector3f(1.0f, 0.0f, 0.0f);
  Dilate(3, 3, pixels, mask, 1);
  EXPECT(mask[1] == 1 && std::fabs(pixels[1].coeffs[0][0] - 1.0f) < 0.001f);
  EXPECT(mask[0] == 1 && std::fabs(pixels[0].coeffs[0][0] - 1.0f) < 0.001f);
  std::vector<SHCoeffs> p2(9);
  std::vector<uint8_t> m2(9, 0);
  m2[3] = m2[5] = 1;
  p2[3].coeffs[0] = Vector3f(1.0f, 0.0f, 0.0f);
  p2[5].coeffs[0] = Vector3f(0.0f, 0.0f, 1.0f);
  Dilate(3, 3, p2, m2, 1);
  EXPECT(m2[4] == 1 && std::fabs(p2[4].coeffs[0][0] - 0.5f) < 0.001f && std::fabs(p2[4].coeffs[0][2] - 0.5f) < 0.001f);
  std::vector<float> f(9, 0.f);
  std::vector<uint8_t> m3(9, 0);
  m3[4] = 1;
  f[4] = 2.0f;
  Dilate(3, 3, f, m3, 1);
  EXPECT(m3[0] == 1 && f[0] == 2.0f);
}

static void BakeSimpleQuad() {
  Scene scene;
  Geometry quad = Quad();
  quad.tangents.clear();
  scene.geometries.push_back(quad);
  Material mat;
  mat.name = "white";
  mat.albedo.pixel_data = {255, 255, 255, 255};
  mat.albedo.width = 1;
  mat.albedo.height = 1;
  mat.albedo.channels = 4;
  scene.materials.push_back(mat);
  Light light;
  light.type = Light::Type::Directional;
  light.direction = Vector3f(0, 0, -1);
  light.color = Vector3f(1, 1, 1);
  light.intensity = 1.0f;
  scene.lights.push_back(light);
  std::vector<SurfacePoint> surface_points(16);
  RasterConfig raster_config;
  raster_config.width = 4;
  raster_config.height = 4;
  surface_points[5].material_id = 0;
  surface_points[5].position = Vector3f(-0.25f, -0.25f, 0.0f);
  surface_points[5].normal = Vector3f(0.0f, 0.0f, 1.0f);
  surface_points[5].tangent = Vector4f(1.0f, 0.0f, 0.0f, 1.0f);
  BakeConfig config;
  config.samples = 64;
  config.bounces = 0;
  BakeResult output = BakeSHLightMap(scene, surface_points, raster_config, config);
  EXPECT(output.sh_texture.pixels[5].coeffs[0][0] > 0.1f);

  SHTexture input;
  input.width = 2;
  input.height = 2;
  input.pixels.resize(4);
  for (auto& p : input.pixels)
    for (auto& c : p.coeffs) c = Vector3f(1.0f, 1.0f, 1.0f);
  SHTexture ds = DownsampleSHTexture(input, 2);
  EXPECT(ds.width == 1 && ds.height == 1 && ds.pixels.size() == 1);
  for (int c = 0; c < 9; ++c) EXPECT(ds.pixels[0].coeffs[c][0] == 1.0f);
}

// Backward(): a directional light on a quad with an overridden albedo.  The
// texel-level NEE does not see the albedo, so with bounces = 0 the loss
// sum(SH) is linear in the light intensity only: dLoss/dI = sum(SH) / I.
void BackwardLinearInIntensity() {
  Scene scene;
  scene.geometries.push_back(Quad());
  Material mat;
  mat.albedo.pixel_data = {200, 200, 200};
  mat.albedo.width = mat.albedo.height = 1;
  mat.albedo.channels = 3;
  scene.materials.push_back(mat);
  Light light;
  light.type = Light::Type::Directional;
  light.direction = Vector3f(0, 0, -1);
  light.intensity = 2.0f;
  scene.lights.push_back(light);
  RasterConfig rc;
  rc.width = rc.height = 8;
  std::vector<SurfacePoint> pts = RasterizeScene(scene, rc);
  BakeConfig config;
  config.samples = 16;
  config.bounces = 0;
  BakeParams params;
  params.albedo = {Vector3f(0.5f, 0.5f, 0.5f)};
  params.light_intensity = {2.0f};
  BakeResult r = BakeSHLightMap(scene, pts, rc, config, params);
  SHTexture ones;
  ones.width = ones.height = 8;
  ones.pixels.resize(64);
  for (auto& p : ones.pixels)
    for (auto& c : p.coeffs) c = Vector3f(1.0f, 1.0f, 1.0f);
  BakeGradients g = Backward(scene, pts, rc, config, params, ones);
  double total = 0.0;
  for (const auto& p : r.sh_texture.pixels)
    for (const auto& c : p.coeffs) total += (double)c[0] + c[1] + c[2];
  EXPECT(total > 1.0);
  EXPECT(std::fabs(g.d_light_intensity[0] - total / 2.0) <= 1e-4 * std::fabs(total));
  EXPECT(g.d_albedo.size() == 3);
}

// SaveSHLightMap: a 2x2 texture in each mode writes the reference's files.
void SaveModes() {
  SHTexture sh;
  sh.width = sh.height = 2;
  sh.pixels.resize(4);
  for (auto& p : sh.pixels)
    for (auto& c : p.coeffs) c = Vector3f(0.5f, 0.25f, 2.0f);
  Texture32F env;
  env.width = env.height = 2;
  env.pixel_data = {1.0f, 0.5f, 0.0f, 0.25f};
  const std::string dir = std::filesystem::temp_directory_path() / "shb_mirror_exr";
  std::filesystem::create_directories(dir);
  EXPECT(SaveSHLightMap(sh, env, dir + "/lightmap.exr"));
  EXPECT(SaveSHLightMap(sh, env, dir + "/lightmap.exr", SaveMode::kLuminancePacked));
  EXPECT(SaveSHLightMap(sh, env, dir + "/lightmap.exr", SaveMode::kSplitChannels));
  for (const char* f : {"lightmap.exr", "lightmap_packed_0.exr", "lightmap_packed_2.exr", "lightmap_L0.exr",
                        "lightmap_L22.exr"})
    EXPECT(std::filesystem::file_size(dir + "/" + f) > 100);
  EXPECT(!SaveSHLightMap(SHTexture{}, env, dir + "/empty.exr"));
  std::filesystem::remove_all(dir);
}

// src/atlas_test.cpp:9-65 (SimpleQuad) and :67-170 (geometry scales).
static void Atlas() {
  Geometry g;
  g.vertices = {Vector3f(-1, -1, 0), Vector3f(1, -1, 0), Vector3f(-1, 1, 0), Vector3f(1, 1, 0)};
  g.normals = {Vector3f(0, 0, 1), Vector3f(0, 0, 1), Vector3f(0, 0, 1), Vector3f(0, 0, 1)};
  g.tangents = {Vector4f(1, 0, 0, 1), Vector4f(1, 0, 0, 1), Vector4f(1, 0, 0, 1), Vector4f(1, 0, 0, 1)};
  g.texture_uvs = {Vector2f(0, 0), Vector2f(1, 0), Vector2f(0, 1), Vector2f(1, 1)};
  g.indices = {0, 1, 2, 2, 1, 3};
  g.material_id = 0;
  Scene scene;
  scene.geometries = {g};
  Material mat;
  mat.albedo.width = 256;
  mat.albedo.height = 256;
  scene.materials.push_back(mat);
  std::optional<AtlasResult> r = CreateAtlasGeometries(scene, 256, 2);
  EXPECT(r.has_value());
  if (r) {
    EXPECT(r->width >= 0 && r->height >= 0);
    EXPECT(r->geometries.size() == 1);
    const Geometry& o = r->geometries[0];
    EXPECT(o.lightmap_uvs.size() == o.vertices.size());
    for (const auto& uv : o.lightmap_uvs) EXPECT(uv.x() >= 0.f && uv.x() <= 1.f && uv.y() >= 0.f && uv.y() <= 1.f);
    EXPECT(o.indices.size() == g.indices.size());
    EXPECT(o.vertices.size() >= g.vertices.size());
  }
  auto one = [](std::vector<Vector2f> uvs, uint32_t w, float density) {
    std::vector<Geometry> gs(1);
    gs[0].material_id = 0;
    gs[0].texture_uvs = uvs;
    std::vector<Material> ms(1);
    ms[0].albedo.width = ms[0].albedo.height = w;
    return atlas_internal::CalculateGeometryScales(gs, ms, density);
  };
  EXPECT(std::fabs(one({Vector2f(0, 0), Vector2f(1, 0), Vector2f(0, 1)}, 100, 1.f)[0] - 100.f) <= 1e-4f);
  EXPECT(std::fabs(one({Vector2f(0, 0), Vector2f(2, 0), Vector2f(0, 2)}, 10, 1.f)[0] - 20.f) <= 1e-4f);
  EXPECT(std::fabs(one({Vector2f(0, 0), Vector2f(1, 1)}, 100, 2.f)[0] - 200.f) <= 1e-4f);
  std::vector<Geometry> gs(3);
  std::vector<Material> ms(3);
  for (int i = 0; i < 3; ++i) {
    gs[i].material_id = i;
    gs[i].texture_uvs = {Vector2f(0, 0), Vector2f(1, 1)};
    ms[i].albedo.width = ms[i].albedo.height = i == 2 ? 1000 : 10;
  }
  std::vector<float> s = atlas_internal::CalculateGeometryScales(gs, ms, 1.f);
  EXPECT(s.size() == 3 && std::fabs(s[0] - 10.f) <= 1e-4f && std::fabs(s[1] - 10.f) <= 1e-4f &&
         std::fabs(s[2] - 50.f) <= 1e-4f);
}

int main(int argc, char** argv) {
  const bool host_only = argc > 1 && std::string(argv[1]) == "--host";
  try {
    Atlas();
    if (host_only) {
      std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
      return failures ? 1 : 0;
    }
    RasterizeQuad();
    Masks();
    Dilation();
    BakeSimpleQuad();
    BackwardLinearInIntensity();
    SaveModes();
  } catch (const std::exception& e) {
    std::printf("exception: %s\n", e.what());
    return 2;
  }
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
  return failures ? 1 : 0;
}
