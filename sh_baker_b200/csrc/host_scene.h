// host_scene.h - a scene description that owns its arrays: what LoadScene
// and CreateAtlasGeometries return through the C ABI (shb_host_scene).
#pragma once

#include <cstring>
#include <string>
#include <vector>

#include "../../include/shb.h"

struct shb_host_scene {
  struct Geo {
    std::vector<float> v, n, uv0, uv1, t;
    std::vector<uint32_t> idx;
    int material = -1;
    float transform[12];
  };
  struct Mat {
    std::vector<uint8_t> px;
    uint32_t w = 0, h = 0, c = 0;
    float emission = 0.f;
    std::string name;
    std::string albedo_file;  // absolute path of an external albedo image
  };
  std::vector<Geo> geos;
  std::vector<Mat> mats;
  std::vector<shb_light_desc> lights;
  std::vector<shb_geometry_desc> gd;
  std::vector<shb_material_desc> md;
  shb_scene_desc desc{};

  // Points `desc` at the owned arrays; call after the last change to them.
  void finish() {
    gd.clear();
    md.clear();
    for (auto& g : geos) {
      shb_geometry_desc d{};
      d.vertices = g.v.empty() ? nullptr : g.v.data();
      d.normals = g.n.empty() ? nullptr : g.n.data();
      d.texture_uvs = g.uv0.empty() ? nullptr : g.uv0.data();
      d.lightmap_uvs = g.uv1.empty() ? nullptr : g.uv1.data();
      d.tangents = g.t.empty() ? nullptr : g.t.data();
      d.vertex_count = (uint32_t)(g.v.size() / 3);
      d.indices = g.idx.empty() ? nullptr : g.idx.data();
      d.index_count = (uint32_t)g.idx.size();
      d.material_id = g.material;
      std::memcpy(d.transform, g.transform, sizeof(d.transform));
      gd.push_back(d);
    }
    for (auto& mt : mats) {
      shb_material_desc d{};
      d.albedo_pixels = mt.px.empty() ? nullptr : mt.px.data();
      d.albedo_width = mt.w;
      d.albedo_height = mt.h;
      d.albedo_channels = mt.c;
      d.emission_intensity = mt.emission;
      md.push_back(d);
    }
    desc = shb_scene_desc{gd.data(), (uint32_t)gd.size(), md.data(), (uint32_t)md.size(), lights.data(),
                          (uint32_t)lights.size()};
  }
};
