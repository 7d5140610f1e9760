// sh_baker::LoadScene / SaveScene of the C++ mirror (include/sh_baker/
// sh_baker.h) over shb_load_gltf / shb_save_gltf.  Host code only: no
// context is created.
//   scene_io_test roundtrip <dir>   save a scene, load it back, compare
//   scene_io_test emissive <file>   load a scene with one emissive primitive
//   scene_io_test missing <file>    a missing file gives nullopt
//   scene_io_test transforms -      TransformedVertices / Normals / Tangents
//                                   and SurfaceArea (src/scene_test.cpp:42-94)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "sh_baker/sh_baker.h"

using namespace sh_baker;

static int failures = 0;
#define EXPECT(c)                                                \
  do {                                                           \
    if (!(c)) {                                                  \
      std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c);    \
      ++failures;                                                \
    }                                                            \
  } while (0)

static bool near(float a, float b) { return std::fabs(a - b) <= 1e-6f; }

static int roundtrip(const std::string& dir) {
  Scene s;
  for (int i = 0; i < 2; ++i) {
    Material m;
    m.name = "Mat_" + std::to_string(i);
    m.albedo.width = m.albedo.height = 1;
    m.albedo.channels = 4;
    m.albedo.pixel_data = {255, 255, 255, 255};
    s.materials.push_back(m);
    Geometry g;
    g.vertices = {Vector3f(0.f, 0.f, 0.f), Vector3f(1.f, 0.f, 0.f), Vector3f(0.f, 1.f, 0.f)};
    g.normals = {Vector3f(0.f, 0.f, 1.f), Vector3f(0.f, 0.f, 1.f), Vector3f(0.f, 0.f, 1.f)};
    g.texture_uvs = {Vector2f(0.f, 0.f), Vector2f(1.f, 0.f), Vector2f(0.f, 1.f)};
    g.lightmap_uvs = {Vector2f(0.1f, 0.1f), Vector2f(0.9f, 0.1f), Vector2f(0.1f, 0.9f)};
    g.tangents = {Vector4f(1.f, 0.f, 0.f, -1.f), Vector4f(1.f, 0.f, 0.f, -1.f), Vector4f(1.f, 0.f, 0.f, -1.f)};
    g.indices = {0, 1, 2};
    g.material_id = i;
    s.geometries.push_back(g);
  }
  Light p;
  p.type = Light::Type::Point;
  p.position = Vector3f(1.f, 2.f, 3.f);
  p.intensity = 7.f;
  s.lights.push_back(p);
  const std::string out = dir + "/scene.gltf";
  EXPECT(SaveScene(s, out));
  std::optional<Scene> r = LoadScene(out);
  EXPECT(r.has_value());
  if (!r) return 1;
  EXPECT(r->geometries.size() == 2 && r->materials.size() == 2 && r->lights.size() == 1);
  for (size_t i = 0; i < r->materials.size(); ++i) EXPECT(r->materials[i].name == "Mat_" + std::to_string(i));
  for (const Geometry& g : r->geometries) {
    EXPECT(g.vertices.size() == 3 && g.indices.size() == 3);
    EXPECT(g.lightmap_uvs.size() == 3 && near(g.lightmap_uvs[1].x(), 0.9f));
    EXPECT(g.tangents.size() == 3 && near(g.tangents[0].w(), -1.f));  // TANGENT kept as written
    EXPECT(near(g.vertices[1].x(), 1.f) && near(g.normals[0].z(), 1.f));
  }
  EXPECT(r->lights[0].type == Light::Type::Point && near(r->lights[0].intensity, 7.f));
  EXPECT(near(r->lights[0].position[1], 2.f));
  return 0;
}

static int emissive(const std::string& file) {
  std::optional<Scene> r = LoadScene(file);
  EXPECT(r.has_value());
  if (!r) return 1;
  int areas = 0;
  for (const Light& l : r->lights) {
    if (l.type != Light::Type::Area) continue;
    ++areas;
    EXPECT(l.material != nullptr && l.geometry != nullptr);
    if (!l.material || !l.geometry) continue;
    // pointers into the returned scene's own vectors
    EXPECT(l.material >= r->materials.data() && l.material < r->materials.data() + r->materials.size());
    EXPECT(l.geometry == &r->geometries[(size_t)l.geometry_index]);
    EXPECT(l.material->emission_intensity > 0.f);
    EXPECT(l.material->name == "Glow");
  }
  EXPECT(areas == 1);
  return 0;
}

static bool approx3(const Vector3f& a, float x, float y, float z) {
  return std::fabs(a[0] - x) <= 1e-5f && std::fabs(a[1] - y) <= 1e-5f && std::fabs(a[2] - z) <= 1e-5f;
}

static int transforms() {
  const float pi = 3.14159265358979323846f;
  const float c = std::cos(pi / 2.0f), s = std::sin(pi / 2.0f);
  // src/scene_test.cpp:42-57 (TransformedVertices): translation by (1, 2, 3)
  Geometry g;
  g.vertices = {Vector3f(1.f, 0.f, 0.f), Vector3f(0.f, 1.f, 0.f)};
  const float trans[12] = {1, 0, 0, 1, 0, 1, 0, 2, 0, 0, 1, 3};
  g.transform = detail::affine_from_rows(trans);
  std::vector<Vector3f> v = TransformedVertices(g);
  EXPECT(v.size() == 2 && approx3(v[0], 2.f, 2.f, 3.f) && approx3(v[1], 1.f, 3.f, 3.f));
  // src/scene_test.cpp:59-75 (TransformedNormals): 90 degrees about Z
  const float rot[12] = {c, -s, 0, 0, s, c, 0, 0, 0, 0, 1, 0};
  g.transform = detail::affine_from_rows(rot);
  g.normals = {Vector3f(1.f, 0.f, 0.f), Vector3f(0.f, 1.f, 0.f)};
  std::vector<Vector3f> n = TransformedNormals(g);
  EXPECT(n.size() == 2 && approx3(n[0], 0.f, 1.f, 0.f) && approx3(n[1], -1.f, 0.f, 0.f));
  // src/scene_test.cpp:77-94 (TransformedTangents): rotated, sign kept
  g.tangents = {Vector4f(1.f, 0.f, 0.f, 1.f)};
  std::vector<Vector4f> t = TransformedTangents(g);
  EXPECT(t.size() == 1 && approx3(Vector3f(t[0][0], t[0][1], t[0][2]), 0.f, 1.f, 0.f) && t[0][3] == 1.0f);
  // the rotation part strips a non-uniform scale: L = Rz(90) diag(2, 3, 4)
  const float rs[12] = {2 * c, -3 * s, 0, 5, 2 * s, 3 * c, 0, 6, 0, 0, 4, 7};
  g.transform = detail::affine_from_rows(rs);
  g.vertices = {Vector3f(1.f, 1.f, 1.f)};
  v = TransformedVertices(g);
  EXPECT(approx3(v[0], 2 * c - 3 * s + 5, 2 * s + 3 * c + 6, 11.f));
  n = TransformedNormals(g);
  EXPECT(approx3(n[0], 0.f, 1.f, 0.f) && approx3(n[1], -1.f, 0.f, 0.f));
  // SurfaceArea (src/scene.cpp:197-207): object space, transform ignored
  g.vertices = {Vector3f(0.f, 0.f, 0.f), Vector3f(1.f, 0.f, 0.f), Vector3f(0.f, 1.f, 0.f), Vector3f(0.f, 0.f, 4.f)};
  g.indices = {0, 1, 2, 0, 1, 3};
  EXPECT(std::fabs(SurfaceArea(g) - 2.5f) <= 1e-6f);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string mode = argv[1], arg = argv[2];
  if (mode == "roundtrip") roundtrip(arg);
  else if (mode == "emissive") emissive(arg);
  else if (mode == "missing") EXPECT(!LoadScene(arg).has_value());
  else if (mode == "transforms") transforms();
  else return 2;
  std::printf(failures ? "scene io test failed\n" : "scene io test passed\n");
  return failures ? 1 : 0;
}
