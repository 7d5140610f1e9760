// sh_cvt - the reference's EXR -> PNG tool (src/sh_cvt_main.cpp) over
// libshb: every .exr file of --input (not recursive) whose L0.R/L0.G/L0.B
// channels (else R/G/B) exist becomes <stem>_L0.png beside it, the L0
// colour as bytes clamp(v) * 255 + 0.5, after Reinhard v / (1 + v) with
// --reinhard.  The conversion runs on the GPU (shb_sh_preview, L0 mode).
#include <dirent.h>
#include <sys/stat.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "shb.h"

namespace {

bool parse_bool(const std::string& v, bool& out) {
  if (v == "true" || v == "1" || v == "yes" || v == "t" || v == "y") out = true;
  else if (v == "false" || v == "0" || v == "no" || v == "f" || v == "n") out = false;
  else return false;
  return true;
}

void convert(shb_context* ctx, const std::string& path, bool reinhard) {
  const char* l0[3] = {"L0.R", "L0.G", "L0.B"};
  const char* rgb[3] = {"R", "G", "B"};
  const char* const* names = l0;
  int32_t w = 0, h = 0;
  if (shb_exr_load_channels(path.c_str(), l0, 3, &w, &h, nullptr) != SHB_OK) {
    names = rgb;
    if (shb_exr_load_channels(path.c_str(), rgb, 3, &w, &h, nullptr) != SHB_OK) {
      std::fprintf(stderr, "E Could not find L0 channels (L0.R/G/B) or standard RGB channels in %s\n", path.c_str());
      return;
    }
  }
  const size_t n = (size_t)w * h;
  std::vector<float> planes(3 * n), sh(27 * n, 0.0f);
  std::vector<uint8_t> out(3 * n);
  if (shb_exr_load_channels(path.c_str(), names, 3, &w, &h, planes.data()) != SHB_OK) {
    std::fprintf(stderr, "E Failed to load EXR image: %s (%s)\n", path.c_str(), shb_last_error());
    return;
  }
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) sh[27 * i + c] = planes[c * n + i];
  if (shb_sh_preview(ctx, sh.data(), w, h, nullptr, nullptr, SHB_PREVIEW_L0, reinhard ? 1 : 0, 0, out.data()) !=
      SHB_OK) {
    std::fprintf(stderr, "E conversion failed for %s: %s\n", path.c_str(), shb_last_error());
    return;
  }
  const size_t slash = path.find_last_of('/');
  const std::string dir = slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
  std::string stem = path.substr(dir.size());
  stem = stem.substr(0, stem.size() - 4);  // ".exr"
  const std::string png = dir + stem + "_L0.png";
  if (shb_write_png(png.c_str(), w, h, 3, out.data()) == SHB_OK) std::fprintf(stderr, "I Saved %s\n", png.c_str());
  else std::fprintf(stderr, "E Failed to write PNG to %s\n", png.c_str());
}

}  // namespace

int main(int argc, char** argv) {
  std::string input;
  bool reinhard = false;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a.size() < 2 || a[0] != '-') {
      std::fprintf(stderr, "unexpected argument: %s\n", a.c_str());
      return 1;
    }
    a = a.substr(a[1] == '-' ? 2 : 1);
    std::string name = a, value;
    const size_t eq = a.find('=');
    const bool has_value = eq != std::string::npos;
    if (has_value) {
      name = a.substr(0, eq);
      value = a.substr(eq + 1);
    }
    if (name == "reinhard") {
      if (has_value && !parse_bool(value, reinhard)) {
        std::fprintf(stderr, "bad value for --reinhard: %s\n", value.c_str());
        return 1;
      }
      if (!has_value) reinhard = true;
    } else if (name == "noreinhard" && !has_value) {
      reinhard = false;
    } else if (name == "input") {
      if (!has_value) {
        if (i + 1 >= argc) {
          std::fprintf(stderr, "missing value for --input\n");
          return 1;
        }
        value = argv[++i];
      }
      input = value;
    } else {
      std::fprintf(stderr, "unknown flag: --%s\n", name.c_str());
      return 1;
    }
  }
  if (input.empty()) {
    std::fprintf(stderr, "E Please provide --input_dir\n");
    return 1;
  }
  struct stat st;
  if (stat(input.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) {
    std::fprintf(stderr, "E Input path is not a valid directory: %s\n", input.c_str());
    return 1;
  }
  std::vector<std::string> files;
  if (DIR* d = opendir(input.c_str())) {
    while (dirent* e = readdir(d)) {
      const std::string f = e->d_name;
      const std::string p = input + (input.back() == '/' ? "" : "/") + f;
      struct stat fs;
      if (f.size() > 4 && f.compare(f.size() - 4, 4, ".exr") == 0 && stat(p.c_str(), &fs) == 0 &&
          S_ISREG(fs.st_mode))
        files.push_back(p);
    }
    closedir(d);
  }
  std::sort(files.begin(), files.end());
  shb_options o{};
  const char* dev = std::getenv("SHB_DEVICE");
  // an ordinal outside int32 becomes -1, which context creation refuses
  const long dv = dev ? std::strtol(dev, nullptr, 10) : 0;
  o.device = dv < INT32_MIN || dv > INT32_MAX ? -1 : (int)dv;
  shb_context* ctx = nullptr;
  if (shb_context_create(&o, &ctx) != SHB_OK) {
    std::fprintf(stderr, "E no CUDA context: %s\n", shb_last_error());
    return 1;
  }
  for (const std::string& f : files) convert(ctx, f, reinhard);
  shb_context_destroy(ctx);
  return 0;
}
