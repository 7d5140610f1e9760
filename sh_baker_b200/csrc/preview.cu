// preview.cu - headless SH lightmap previews as 8-bit RGB images, for
// looking at bakes without a graphics API:
//   SHB_PREVIEW_L0          the L0 (DC) coefficient as colour, as the
//                           reference's EXR -> PNG tool does
//                           (src/sh_cvt_main.cpp:99-117);
//   SHB_PREVIEW_SH          the SH9 radiance towards a direction, clamped at
//                           zero, as the viewer's EvalSHBasis
//                           (glsl/viz.frag:42-68, restated as arithmetic);
//   SHB_PREVIEW_SH_PACKED   the same from what the luminance-packed files
//                           keep: L1/L2 as Rec. 709 luminance re-coloured
//                           with the chroma of L0 (glsl/viz.frag:75-99).
// Optional Reinhard x / (1 + x); bytes are clamp(v) * 255 + 0.5 truncated
// (src/sh_cvt_main.cpp:21-24).  The direction is the texel's normal when
// normals are given, else one fixed direction.
#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "shb_internal.h"

namespace shb {
namespace {

__device__ __forceinline__ float to_byte(float v, bool reinhard) {
  if (reinhard) v = __fdiv_rn(v, __fadd_rn(1.0f, v));
  v = fmaxf(0.0f, fminf(1.0f, v));
  return __fadd_rn(__fmul_rn(v, 255.0f), 0.5f);
}

__global__ void k_sh_preview(const float* __restrict__ sh, int64_t n, const float* __restrict__ normals, float3 dir,
                             int mode, int reinhard, uint8_t* __restrict__ out) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const float* c = sh + p * 27;
    float rgb[3];
    if (mode == SHB_PREVIEW_L0) {
      rgb[0] = c[0];
      rgb[1] = c[1];
      rgb[2] = c[2];
    } else {
      float x = dir.x, y = dir.y, z = dir.z;
      if (normals) {
        x = normals[3 * p];
        y = normals[3 * p + 1];
        z = normals[3 * p + 2];
      }
      float b[9];
      b[0] = 0.282095f;
      b[1] = __fmul_rn(0.488603f, y);
      b[2] = __fmul_rn(0.488603f, z);
      b[3] = __fmul_rn(0.488603f, x);
      b[4] = __fmul_rn(__fmul_rn(1.092548f, x), y);
      b[5] = __fmul_rn(__fmul_rn(1.092548f, y), z);
      b[6] = __fmul_rn(0.315392f, __fsub_rn(__fmul_rn(__fmul_rn(3.0f, z), z), 1.0f));
      b[7] = __fmul_rn(__fmul_rn(1.092548f, x), z);
      b[8] = __fmul_rn(0.546274f, __fsub_rn(__fmul_rn(x, x), __fmul_rn(y, y)));
      float coef[27];
      for (int k = 0; k < 27; ++k) coef[k] = c[k];
      if (mode == SHB_PREVIEW_SH_PACKED) {
        // L0 kept in colour; L1/L2 as luminance times the chroma of L0
        const float l0 = __fadd_rn(__fadd_rn(__fmul_rn(coef[0], 0.2126f), __fmul_rn(coef[1], 0.7152f)),
                                   __fmul_rn(coef[2], 0.0722f));
        float chroma[3] = {1.0f, 1.0f, 1.0f};
        if (l0 > 1e-6f)
          for (int ch = 0; ch < 3; ++ch) chroma[ch] = __fdiv_rn(coef[ch], l0);
        for (int k = 1; k < 9; ++k) {
          const float* q = c + 3 * k;
          // the packed file holds x0*w0 + (x1*w1 + x2*w2) (src/saver.cpp:354-360)
          const float lum = __fadd_rn(__fmul_rn(q[0], 0.2126f), __fadd_rn(__fmul_rn(q[1], 0.7152f),
                                                                            __fmul_rn(q[2], 0.0722f)));
          for (int ch = 0; ch < 3; ++ch) coef[3 * k + ch] = __fmul_rn(lum, chroma[ch]);
        }
      }
      for (int ch = 0; ch < 3; ++ch) {
        float s = __fmul_rn(coef[ch], b[0]);
        for (int k = 1; k < 9; ++k) s = __fadd_rn(s, __fmul_rn(coef[3 * k + ch], b[k]));
        rgb[ch] = fmaxf(s, 0.0f);
      }
    }
    for (int ch = 0; ch < 3; ++ch) out[3 * p + ch] = (uint8_t)to_byte(rgb[ch], reinhard != 0);
  }
}

}  // namespace

shb_status sh_preview_device(shb_context* c, const float* d_sh, int64_t n, const float* d_normals, const float dir[3],
                             int mode, int reinhard, uint8_t* d_out) {
  const int grid = (int)std::min<int64_t>((n + 255) / 256, shb::sm_count() * 16);
  if (n > 0)
    k_sh_preview<<<grid, 256, 0, c->stream>>>(d_sh, n, d_normals, make_float3(dir[0], dir[1], dir[2]), mode,
                                              reinhard, d_out);
  count_launch(c, 1);
  SHB_CUDA(cudaGetLastError());
  return SHB_OK;
}

// 8-bit RGB / RGBA / gray PNG, filter type 0, zlib.
bool write_png(const std::string& path, int w, int h, int channels, const uint8_t* px) {
  const int ct = channels == 1 ? 0 : channels == 2 ? 4 : channels == 3 ? 2 : 6;
  const size_t stride = (size_t)w * channels;
  std::vector<uint8_t> raw;
  raw.reserve((stride + 1) * (size_t)h);
  for (int y = 0; y < h; ++y) {
    raw.push_back(0);
    raw.insert(raw.end(), px + (size_t)y * stride, px + (size_t)(y + 1) * stride);
  }
  uLongf zl = compressBound((uLong)raw.size());
  std::vector<uint8_t> z(zl);
  if (compress2(z.data(), &zl, raw.data(), (uLong)raw.size(), Z_DEFAULT_COMPRESSION) != Z_OK) return false;
  z.resize(zl);
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  auto be = [](uint32_t v, uint8_t* o) {
    o[0] = (uint8_t)(v >> 24);
    o[1] = (uint8_t)(v >> 16);
    o[2] = (uint8_t)(v >> 8);
    o[3] = (uint8_t)v;
  };
  bool ok = true;
  auto chunk = [&](const char* t, const uint8_t* d, size_t n) {
    uint8_t hdr[8];
    be((uint32_t)n, hdr);
    std::memcpy(hdr + 4, t, 4);
    uLong crc = crc32(0L, reinterpret_cast<const Bytef*>(t), 4);
    if (n) crc = crc32(crc, d, (uInt)n);
    uint8_t tail[4];
    be((uint32_t)crc, tail);
    ok = ok && std::fwrite(hdr, 1, 8, f) == 8 && (n == 0 || std::fwrite(d, 1, n, f) == n) &&
         std::fwrite(tail, 1, 4, f) == 4;
  };
  static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  ok = std::fwrite(sig, 1, 8, f) == 8;
  uint8_t ihdr[13];
  be((uint32_t)w, ihdr);
  be((uint32_t)h, ihdr + 4);
  ihdr[8] = 8;
  ihdr[9] = (uint8_t)ct;
  ihdr[10] = ihdr[11] = ihdr[12] = 0;
  chunk("IHDR", ihdr, 13);
  chunk("IDAT", z.data(), z.size());
  chunk("IEND", nullptr, 0);
  return (std::fclose(f) == 0) && ok;
}

}  // namespace shb
