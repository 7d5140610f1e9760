// exr_ref_harness.cpp - TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own vendored EXR library (tinyexr + miniz, compiled
// from the reference tree into oracle/_ref by oracle/build.py) the way the
// reference's saver does, so that files written by the CUDA writer can be
// checked against files written by the reference's code path, and read
// back by the reference's reader.
//
//   ref_exr_save  restates src/saver.cpp:108-401 (SaveCombined, SaveSplit,
//                 SavePackedLuminance): channel names and order, FLOAT input
//                 stored as HALF, ZIP compression, file naming
//                 (src/saver.cpp:232-236, 306-317, src/saver.h:28-43).
//   ref_exr_load  LoadEXRImageFromFile with HALF kept as stored: the raw
//                 16-bit samples of every channel in file order.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tinyexr.h"

namespace {

const char* kCoeff[9] = {"L0", "L1m1", "L10", "L11", "L2m2", "L2m1", "L20", "L21", "L22"};

// Channel source: 0..26 SH channel, 100 + k luminance of coefficient k, 200 env.
int save_one(const float* sh, const float* env, int w, int h, const std::vector<std::string>& names,
             const std::vector<int>& src, const std::string& path) {
  const int n = (int)names.size();
  const size_t np = (size_t)w * h;
  std::vector<std::vector<float>> ch(n, std::vector<float>(np));
  for (int c = 0; c < n; ++c)
    for (size_t p = 0; p < np; ++p) {
      const float* q = sh + p * 27;
      float v;
      if (src[c] < 27) v = q[src[c]];
      else if (src[c] < 200) {
        const float* k = q + 3 * (src[c] - 100);
        // Eigen Vector3f::dot with Rec. 709 weights (src/saver.cpp:313)
        v = k[0] * 0.2126f + (k[1] * 0.7152f + k[2] * 0.0722f);
      } else v = env ? env[p] : 0.0f;
      ch[c][p] = v;
    }
  EXRHeader header;
  InitEXRHeader(&header);
  EXRImage image;
  InitEXRImage(&image);
  image.num_channels = n;
  std::vector<float*> ptr(n);
  for (int c = 0; c < n; ++c) ptr[c] = ch[c].data();
  header.channels = (EXRChannelInfo*)std::malloc(sizeof(EXRChannelInfo) * n);
  header.pixel_types = (int*)std::malloc(sizeof(int) * n);
  header.requested_pixel_types = (int*)std::malloc(sizeof(int) * n);
  for (int c = 0; c < n; ++c) {
    std::strncpy(header.channels[c].name, names[c].c_str(), 255);
    header.channels[c].name[255] = 0;
    header.pixel_types[c] = TINYEXR_PIXELTYPE_FLOAT;
    header.requested_pixel_types[c] = TINYEXR_PIXELTYPE_HALF;
  }
  image.images = (unsigned char**)ptr.data();
  image.width = w;
  image.height = h;
  header.num_channels = n;
  header.compression_type = TINYEXR_COMPRESSIONTYPE_ZIP;
  const char* err = nullptr;
  int ret = SaveEXRImageToFile(&image, &header, path.c_str(), &err);
  std::free(header.channels);
  std::free(header.pixel_types);
  std::free(header.requested_pixel_types);
  if (ret != TINYEXR_SUCCESS) {
    FreeEXRErrorMessage(err);
    return 1;
  }
  return 0;
}

void split(const std::string& path, std::string& base, std::string& ext) {
  size_t slash = path.find_last_of('/');
  size_t dot = path.find_last_of('.');
  size_t name0 = slash == std::string::npos ? 0 : slash + 1;
  if (dot != std::string::npos && dot > name0) {
    base = path.substr(0, dot);
    ext = path.substr(dot);
  } else {
    base = path;
    ext.clear();
  }
}

}  // namespace

extern "C" {

// mode 0 combined, 1 split channels, 2 luminance packed (src/saver.h:21-25)
int ref_exr_save(const float* sh, const float* env, int w, int h, const char* path, int mode) {
  if (!sh || w <= 0 || h <= 0) return 2;
  if (mode == 0) {
    std::vector<std::string> names;
    std::vector<int> src;
    const char* rgb[3] = {".R", ".G", ".B"};
    for (int i = 0; i < 9; ++i)
      for (int c = 0; c < 3; ++c) {
        names.push_back(std::string(kCoeff[i]) + rgb[c]);
        src.push_back(3 * i + c);
      }
    names.push_back("EnvVisibility");
    src.push_back(200);
    return save_one(sh, env, w, h, names, src, path);
  }
  std::string base, ext;
  split(path, base, ext);
  if (mode == 1) {
    for (int i = 0; i < 9; ++i) {
      std::vector<std::string> names = {"R", "G", "B"};
      std::vector<int> src = {3 * i, 3 * i + 1, 3 * i + 2};
      if (i == 0) {
        names.push_back("A");
        src.push_back(200);
      }
      if (save_one(sh, env, w, h, names, src, base + "_" + kCoeff[i] + ext)) return 1;
    }
    return 0;
  }
  if (mode == 2) {
    const std::vector<std::string> names = {"R", "G", "B", "A"};
    if (save_one(sh, env, w, h, names, {0, 1, 2, 200}, base + "_packed_0" + ext)) return 1;
    if (save_one(sh, env, w, h, names, {101, 102, 103, 104}, base + "_packed_1" + ext)) return 1;
    return save_one(sh, env, w, h, names, {105, 106, 107, 108}, base + "_packed_2" + ext);
  }
  return 2;
}

// Reads `path` with tinyexr.  Returns the channel count (or -1), fills
// width/height, names (256 bytes each, up to max_ch) and, when halves is
// not NULL, the raw half samples channel-major (max_ch x w x h).
int ref_exr_load(const char* path, int* width, int* height, int max_ch, char* names, uint16_t* halves) {
  EXRVersion version;
  if (ParseEXRVersionFromFile(&version, path) != TINYEXR_SUCCESS) return -1;
  EXRHeader header;
  InitEXRHeader(&header);
  const char* err = nullptr;
  if (ParseEXRHeaderFromFile(&header, &version, path, &err) != TINYEXR_SUCCESS) {
    FreeEXRErrorMessage(err);
    return -1;
  }
  EXRImage image;
  InitEXRImage(&image);
  if (LoadEXRImageFromFile(&image, &header, path, &err) != TINYEXR_SUCCESS) {
    FreeEXRErrorMessage(err);
    FreeEXRHeader(&header);
    return -1;
  }
  const int n = header.num_channels;
  *width = image.width;
  *height = image.height;
  for (int c = 0; c < n && c < max_ch; ++c) {
    std::strncpy(names + 256 * c, header.channels[c].name, 255);
    names[256 * c + 255] = 0;
    if (halves && header.pixel_types[c] == TINYEXR_PIXELTYPE_HALF) {
      const size_t np = (size_t)image.width * image.height;
      std::memcpy(halves + np * c, image.images[c], np * sizeof(uint16_t));
    }
  }
  FreeEXRImage(&image);
  FreeEXRHeader(&header);
  return n;
}

}  // extern "C"
