// sh_baker - the command line of the reference (src/main.cpp:14-193) over
// libshb: load a glTF scene, bake its SH9 lightmap on the GPU, and write
// lightmap.exr (or its split / luminance-packed forms) and scene.gltf to
// --output.  Same flags and defaults as the reference; --seed selects the
// random stream (the reference always uses the fixed stream 12345 + texel).
//
// Like the reference (src/main.cpp:71-91), the lightmap UVs are generated
// for every scene before rasterising: shb_create_atlas with --width as the
// page size, --dilation as the padding and --density_multiplier (the
// reference uses xatlas; the charts here are built by libshb, so UVs differ
// while following the same contract).  --keep_lightmap_uvs, not a reference
// flag, bakes with the input's TEXCOORD_1 instead.
#include <sys/stat.h>

#include <chrono>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "shb.h"

namespace {

struct Flags {
  std::string input, output;
  int width = 2048, height = 2048, samples = 128, bounces = 3, dilation = 16, supersample_scale = 1;
  bool split_channels = false, luminance_only = false, debug_output = false, keep_lightmap_uvs = false;
  double density_multiplier = 1.0;
  long long seed = 12345;
};

bool parse_bool(const std::string& v, bool& out) {
  if (v == "true" || v == "1" || v == "yes" || v == "t" || v == "y") out = true;
  else if (v == "false" || v == "0" || v == "no" || v == "f" || v == "n") out = false;
  else return false;
  return true;
}

// gflags syntax: --name=value, --name value, -name, --name (bool), --noname
bool parse(int argc, char** argv, Flags& f) {
  std::map<std::string, std::string*> strs = {{"input", &f.input}, {"output", &f.output}};
  std::map<std::string, int*> ints = {{"width", &f.width},       {"height", &f.height},
                                      {"samples", &f.samples},   {"bounces", &f.bounces},
                                      {"dilation", &f.dilation}, {"supersample_scale", &f.supersample_scale}};
  std::map<std::string, bool*> bools = {
      {"split_channels", &f.split_channels}, {"luminance_only", &f.luminance_only}, {"debug_output", &f.debug_output},
      {"keep_lightmap_uvs", &f.keep_lightmap_uvs}};
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a.size() < 2 || a[0] != '-') {
      std::fprintf(stderr, "unexpected argument: %s\n", a.c_str());
      return false;
    }
    a = a.substr(a[1] == '-' ? 2 : 1);
    std::string name = a, value;
    bool has_value = false;
    size_t eq = a.find('=');
    if (eq != std::string::npos) {
      name = a.substr(0, eq);
      value = a.substr(eq + 1);
      has_value = true;
    }
    if (bools.count(name)) {
      bool v = true;
      if (has_value && !parse_bool(value, v)) {
        std::fprintf(stderr, "bad value for --%s: %s\n", name.c_str(), value.c_str());
        return false;
      }
      *bools[name] = v;
      continue;
    }
    if (!has_value && name.rfind("no", 0) == 0 && bools.count(name.substr(2))) {
      *bools[name.substr(2)] = false;
      continue;
    }
    const bool known = strs.count(name) || ints.count(name) || name == "density_multiplier" || name == "seed";
    if (!known) {
      std::fprintf(stderr, "unknown flag: --%s\n", name.c_str());
      return false;
    }
    if (!has_value) {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for --%s\n", name.c_str());
        return false;
      }
      value = argv[++i];
    }
    char* end = nullptr;
    if (strs.count(name)) {
      *strs[name] = value;
      continue;
    }
    if (ints.count(name)) {
      errno = 0;
      long v = std::strtol(value.c_str(), &end, 10);
      // an int32 flag, as gflags parses it: no wrap-around of larger values
      if (value.empty() || *end || errno == ERANGE || v < INT32_MIN || v > INT32_MAX) {
        std::fprintf(stderr, "bad value for --%s: %s\n", name.c_str(), value.c_str());
        return false;
      }
      *ints[name] = (int)v;
    } else if (name == "density_multiplier") {
      f.density_multiplier = std::strtod(value.c_str(), &end);
    } else {
      f.seed = std::strtoll(value.c_str(), &end, 10);
    }
    if (value.empty() || (end && *end)) {
      std::fprintf(stderr, "bad value for --%s: %s\n", name.c_str(), value.c_str());
      return false;
    }
  }
  return true;
}

void log(const std::string& s) { std::fprintf(stderr, "I %s\n", s.c_str()); }
int fail(const std::string& s) {
  const char* e = shb_last_error();
  std::fprintf(stderr, "E %s%s%s\n", s.c_str(), (e && *e) ? ": " : "", e ? e : "");
  return 1;
}

bool mkdirs(const std::string& dir) {
  std::string cur;
  for (size_t i = 0; i <= dir.size(); ++i) {
    if ((i == dir.size() || dir[i] == '/') && !cur.empty()) {
      struct stat st;
      if (stat(cur.c_str(), &st) != 0 && mkdir(cur.c_str(), 0755) != 0) return false;
    }
    if (i < dir.size()) cur += dir[i];
  }
  return true;
}

// CreateMaterialMap (src/rasterizer.cpp:243-287): a colour per material id
// from an integer hash, lifted when all channels are dark.
std::vector<uint8_t> material_map(const std::vector<shb_surface_point>& pts) {
  std::vector<uint8_t> out(pts.size() * 3, 0);
  for (size_t i = 0; i < pts.size(); ++i) {
    if (pts[i].material_id < 0) continue;
    uint32_t id = (uint32_t)pts[i].material_id;
    id = ((id >> 16) ^ id) * 0x45d9f3bu;
    id = ((id >> 16) ^ id) * 0x45d9f3bu;
    id = (id >> 16) ^ id;
    uint8_t r = id & 0xFF, g = (id >> 8) & 0xFF, b = (id >> 16) & 0xFF;
    if (r < 50 && g < 50 && b < 50) {
      r += 50;
      g += 50;
      b += 50;
    }
    out[3 * i] = r;
    out[3 * i + 1] = g;
    out[3 * i + 2] = b;
  }
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  Flags F;
  if (!parse(argc, argv, F)) return 1;
  if (F.input.empty()) {
    std::fprintf(stderr, "Usage: %s --input <gltf_file>\n", argv[0]);
    return 1;
  }
  struct stat st;
  if (stat(F.input.c_str(), &st) != 0) return fail("Input file does not exist: " + F.input);
  if (F.width <= 0 || F.height <= 0 || F.supersample_scale <= 0 || F.samples <= 0 || F.bounces < 0 ||
      F.dilation < 0)
    return fail("bad --width/--height/--supersample_scale/--samples/--bounces/--dilation");
  log("Loading scene from: " + F.input);
  shb_host_scene* hs = nullptr;
  if (shb_load_gltf(F.input.c_str(), &hs) != SHB_OK) return fail("Failed to load scene.");
  const shb_scene_desc* desc = shb_host_scene_desc(hs);
  log("Scene loaded successfully.  Geometries: " + std::to_string(desc->geometry_count) +
      "  Materials: " + std::to_string(desc->material_count) + "  Lights: " + std::to_string(desc->light_count));
  if (desc->geometry_count == 0) return fail("No geometries found in scene.");
  shb_host_scene* atlas = nullptr;
  if (F.keep_lightmap_uvs) {
    for (uint32_t g = 0; g < desc->geometry_count; ++g)
      if (!desc->geometries[g].lightmap_uvs)
        return fail("geometry " + std::to_string(g) + " has no lightmap UVs (TEXCOORD_1) to keep");
  } else {
    log("Generating Lightmap UVs...");
    int32_t aw = 0, ah = 0;
    if (shb_create_atlas(desc, (uint32_t)F.width, (uint32_t)F.dilation, (float)F.density_multiplier, &atlas, &aw,
                         &ah) != SHB_OK)
      return fail(std::string("Atlas generation failed (possibly could not fit charts): ") + shb_last_error());
    desc = shb_host_scene_desc(atlas);
    log("Atlas generation complete.  Resolution: " + std::to_string(aw) + "x" + std::to_string(ah));
  }

  shb_options o{};
  const char* dev = std::getenv("SHB_DEVICE");
  // an ordinal outside int32 becomes -1, which context creation refuses
  const long dv = dev ? std::strtol(dev, nullptr, 10) : 0;
  o.device = dv < INT32_MIN || dv > INT32_MAX ? -1 : (int)dv;
  shb_context* ctx = nullptr;
  if (shb_context_create(&o, &ctx) != SHB_OK) return fail("no CUDA context");
  shb_scene* scene = nullptr;
  if (shb_scene_upload(ctx, desc, &scene) != SHB_OK) return fail("scene upload failed");

  if (F.debug_output) {
    const int sw = F.width * F.supersample_scale, sh = F.height * F.supersample_scale;
    std::vector<shb_surface_point> pts((size_t)sw * sh);
    shb_raster_config rc{F.width, F.height, F.supersample_scale};
    if (shb_rasterize(scene, &rc, pts.data(), nullptr) != SHB_OK) return fail("rasterisation failed");
    const std::string dir = F.output.empty() ? "." : F.output;
    mkdirs(dir);
    const std::string map_path = dir + "/material_map.png";
    const std::vector<uint8_t> mm = material_map(pts);
    if (shb_write_png(map_path.c_str(), sw, sh, 3, mm.data()) == SHB_OK) log("Material map saved to: " + map_path);
    else std::fprintf(stderr, "E Failed to save material map to: %s\n", map_path.c_str());
  }

  log("Starting Bake (" + std::to_string(F.samples) + " samples)...");
  shb_pipeline_config cfg{F.width, F.height, F.supersample_scale, F.samples, F.bounces, F.dilation, 1,
                          (uint32_t)F.seed};
  const size_t n = (size_t)F.width * F.height;
  std::vector<float> sh(n * 27), env(n);
  std::vector<uint8_t> mask(n);
  shb_bake_stats stats{};
  auto t0 = std::chrono::high_resolution_clock::now();
  if (shb_bake_pipeline(scene, &cfg, sh.data(), env.data(), mask.data(), &stats) != SHB_OK)
    return fail("bake failed");
  const double secs = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
  log("Bake complete in " + std::to_string(secs) + " seconds (" + std::to_string(stats.texel_samples) +
      " texel-samples).");

  if (!F.output.empty()) {
    log("Saving output to: " + F.output);
    if (!mkdirs(F.output)) return fail("cannot create " + F.output);
    const int mode = F.luminance_only ? SHB_SAVE_LUMINANCE_PACKED
                                      : (F.split_channels ? SHB_SAVE_SPLIT_CHANNELS : SHB_SAVE_COMBINED);
    if (shb_save_sh_lightmap(ctx, sh.data(), env.data(), F.width, F.height, 0, (F.output + "/lightmap.exr").c_str(),
                             mode) != SHB_OK)
      return fail("Failed to save output.");
    std::vector<const char*> names(desc->material_count), files(desc->material_count);
    for (uint32_t m = 0; m < desc->material_count; ++m)
      shb_host_scene_material_info(hs, (int32_t)m, &names[m], &files[m]);
    if (shb_save_gltf(desc, names.data(), files.data(), (F.output + "/scene.gltf").c_str()) != SHB_OK)
      return fail("Failed to save glTF.");
  }
  shb_scene_destroy(scene);
  shb_context_destroy(ctx);
  shb_host_scene_destroy(atlas);
  shb_host_scene_destroy(hs);
  return 0;
}
