// exr.cu - SaveSHLightMap (src/saver.cpp:108-401): the SH lightmap written
// as OpenEXR scanline files, half storage, ZIP compression, in the three
// layouts of the reference (combined 28 channels, 9 split RGB(A) files, 3
// luminance-packed RGBA files).
//
// The device does the per-sample work: channel selection, Rec. 709 luminance
// of L1/L2 (src/saver.cpp:313,354-360), float -> half, the EXR scanline
// layout of each 16-line chunk, and ZIP's byte reorder + delta predictor
// (the OpenEXR ZIP pre-pass).  The host deflates each chunk with zlib on all
// cores and writes header, offset table and chunks.
//
// File layout and choices follow what the reference's writer emits
// (tinyexr's SaveEXRImageToFile as called in src/saver.cpp): attributes
// channels, compression, dataWindow, displayWindow, lineOrder,
// pixelAspectRatio, screenWindowCenter, screenWindowWidth in that order; the
// channel list in the order the saver names them (not sorted); HALF
// storage; ZIP_COMPRESSION with 16 lines per chunk; a chunk whose deflate
// output is not smaller than its raw bytes is stored raw.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "shb_internal.h"

namespace shb {
namespace {

constexpr int kLinesPerChunk = 16;  // ZIP_COMPRESSION

// Output channel recipes: kind 0 = SH coefficient channel `src` (0..26),
// kind 1 = Rec. 709 luminance of SH coefficient `src` (0..8), kind 2 = env.
struct ChanSpec {
  int kind;
  int src;
};
constexpr int kMaxChannels = 28;
struct ChanTable {
  ChanSpec c[kMaxChannels];
  int n;
};

// float -> half with the rounding of the reference's writer (tinyexr's
// float_to_half_full, the public-domain conversion by F. Giesen after the
// ISPC reference): truncate the mantissa and add one unit when the first
// dropped bit is set (round half away from zero in magnitude), float
// denormals flush to zero, overflow gives infinity, NaN gives a quiet NaN.
__device__ __forceinline__ uint16_t half_bits(float f) {
  const uint32_t u = __float_as_uint(f);
  const uint32_t sign = (u >> 16) & 0x8000u;
  const int exp = (int)((u >> 23) & 0xFFu);
  const uint32_t man = u & 0x7FFFFFu;
  uint32_t h = 0;
  if (exp == 0) {
    h = 0;
  } else if (exp == 255) {
    h = (31u << 10) | (man ? 0x200u : 0u);
  } else {
    const int e = exp - 127 + 15;
    if (e >= 31) {
      h = 31u << 10;
    } else if (e <= 0) {
      if (14 - e <= 24) {
        const uint32_t m = man | 0x800000u;
        h = m >> (14 - e);
        if ((m >> (13 - e)) & 1u) h += 1u;
      }
    } else {
      h = ((uint32_t)e << 10) | (man >> 13);
      if (man & 0x1000u) h += 1u;
    }
  }
  return (uint16_t)((h & 0x7FFFu) | sign);
}

// One half sample per thread, written in the raw chunk layout:
// chunk k holds lines [16k, 16k + lines), each line holds every channel's
// `width` samples in table order (little-endian).
__global__ void k_exr_raw(const float* __restrict__ sh, const float* __restrict__ env, int W, int H, ChanTable t,
                          uint16_t* __restrict__ raw) {
  const int64_t total = (int64_t)W * H * t.n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    // i enumerates (y, c, x) in file order: chunks are contiguous lines
    const int64_t line = i / ((int64_t)W * t.n);
    const int rem = (int)(i - line * (int64_t)W * t.n);
    const int c = rem / W;
    const int x = rem - c * W;
    const int64_t p = line * W + x;
    const ChanSpec s = t.c[c];
    float v;
    if (s.kind == 0) {
      v = sh[p * 27 + s.src];
    } else if (s.kind == 1) {
      // Eigen dot: x0*y0 + (x1*y1 + x2*y2), Rec. 709 weights
      const float* q = sh + p * 27 + 3 * s.src;
      v = __fadd_rn(__fmul_rn(q[0], 0.2126f), __fadd_rn(__fmul_rn(q[1], 0.7152f), __fmul_rn(q[2], 0.0722f)));
      if (isnan(v)) {
        // The host (x86 SSE) result: a NaN operand propagates quieted with
        // its sign, the first in evaluation order (x0, then x1, then x2);
        // a NaN made from inf - inf is the negative default NaN.  The GPU's
        // own NaN is the positive canonical one.
        uint32_t bits = 0xFFC00000u;
        if (isnan(q[0])) bits = __float_as_uint(q[0]) | 0x400000u;
        else if (isnan(q[1])) bits = __float_as_uint(q[1]) | 0x400000u;
        else if (isnan(q[2])) bits = __float_as_uint(q[2]) | 0x400000u;
        v = __uint_as_float(bits);
      }
    } else {
      v = env ? env[p] : 0.0f;
    }
    raw[i] = half_bits(v);
  }
}

// ZIP pre-pass per chunk (OpenEXR ZIP compressor): bytes are reordered as
// [even-indexed bytes, odd-indexed bytes], then each byte after the first
// becomes (t[i] - t[i-1] + 128) mod 256.  One output byte per thread.
__global__ void k_exr_predict(const uint8_t* __restrict__ raw, int64_t line_bytes, int H, int64_t total,
                              uint8_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t chunk_bytes = line_bytes * kLinesPerChunk;
    const int64_t k = i / chunk_bytes;
    const int64_t base = k * chunk_bytes;
    const int lines = min(kLinesPerChunk, H - (int)(k * kLinesPerChunk));
    const int64_t n = line_bytes * lines;
    const int64_t j = i - base;
    const int64_t half = (n + 1) / 2;
    auto t = [&](int64_t q) -> int { return q < half ? raw[base + 2 * q] : raw[base + 2 * (q - half) + 1]; };
    out[i] = j == 0 ? (uint8_t)t(0) : (uint8_t)((t(j) - t(j - 1) + 128 + 256) & 0xFF);
  }
}

void put_attr(std::vector<uint8_t>& o, const char* name, const char* type, const void* data, int len) {
  o.insert(o.end(), name, name + std::strlen(name) + 1);
  o.insert(o.end(), type, type + std::strlen(type) + 1);
  const uint8_t* l = reinterpret_cast<const uint8_t*>(&len);
  o.insert(o.end(), l, l + 4);
  const uint8_t* d = static_cast<const uint8_t*>(data);
  o.insert(o.end(), d, d + len);
}

std::vector<uint8_t> exr_header(const std::vector<std::string>& names, int W, int H) {
  std::vector<uint8_t> o = {0x76, 0x2f, 0x31, 0x01, 2, 0, 0, 0};
  std::vector<uint8_t> ch;
  for (const std::string& n : names) {
    ch.insert(ch.end(), n.begin(), n.end());
    ch.push_back(0);
    const int32_t v[4] = {1 /* HALF */, 0 /* pLinear + reserved */, 1, 1};
    const uint8_t* b = reinterpret_cast<const uint8_t*>(v);
    ch.insert(ch.end(), b, b + 16);
  }
  ch.push_back(0);
  put_attr(o, "channels", "chlist", ch.data(), (int)ch.size());
  const uint8_t zip = 3;
  put_attr(o, "compression", "compression", &zip, 1);
  const int32_t win[4] = {0, 0, W - 1, H - 1};
  put_attr(o, "dataWindow", "box2i", win, 16);
  put_attr(o, "displayWindow", "box2i", win, 16);
  const uint8_t order = 0;
  put_attr(o, "lineOrder", "lineOrder", &order, 1);
  const float one = 1.0f, center[2] = {0.f, 0.f};
  put_attr(o, "pixelAspectRatio", "float", &one, 4);
  put_attr(o, "screenWindowCenter", "v2f", center, 8);
  put_attr(o, "screenWindowWidth", "float", &one, 4);
  o.push_back(0);
  return o;
}

// One file: channels of `t` named `names`.
shb_status write_exr(shb_context* c, const float* d_sh, const float* d_env, int W, int H, const ChanTable& t,
                     const std::vector<std::string>& names, const std::string& path) {
  cudaStream_t st = c->stream;
  const int64_t line_bytes = (int64_t)W * t.n * 2;
  const int64_t total = line_bytes * H;
  SHB_TRY(c->scratch[26].reserve((size_t)total * 2));
  uint8_t* d_raw = c->scratch[26].as<uint8_t>();
  uint8_t* d_pred = d_raw + total;
  const int64_t samples = (int64_t)W * H * t.n;
  const int grid = (int)std::min<int64_t>((samples + 255) / 256, shb::sm_count() * 16);
  k_exr_raw<<<grid, 256, 0, st>>>(d_sh, d_env, W, H, t, reinterpret_cast<uint16_t*>(d_raw));
  const int grid2 = (int)std::min<int64_t>((total + 255) / 256, shb::sm_count() * 16);
  k_exr_predict<<<grid2, 256, 0, st>>>(d_raw, line_bytes, H, total, d_pred);
  count_launch(c, 2);
  SHB_CUDA(cudaGetLastError());
  std::vector<uint8_t> raw((size_t)total), pred((size_t)total);
  SHB_CUDA(cudaMemcpyAsync(raw.data(), d_raw, (size_t)total, cudaMemcpyDeviceToHost, st));
  SHB_CUDA(cudaMemcpyAsync(pred.data(), d_pred, (size_t)total, cudaMemcpyDeviceToHost, st));
  SHB_CUDA(cudaStreamSynchronize(st));

  const int chunks = (H + kLinesPerChunk - 1) / kLinesPerChunk;
  std::vector<std::vector<uint8_t>> data((size_t)chunks);
  std::atomic<int> next{0}, failed{0};
  auto worker = [&]() {
    for (int k; (k = next.fetch_add(1)) < chunks;) {
      const int lines = std::min(kLinesPerChunk, H - k * kLinesPerChunk);
      const size_t n = (size_t)line_bytes * lines, off = (size_t)k * line_bytes * kLinesPerChunk;
      uLongf cap = compressBound((uLong)n);
      std::vector<uint8_t> z(cap);
      if (compress2(z.data(), &cap, pred.data() + off, (uLong)n, Z_DEFAULT_COMPRESSION) != Z_OK) {
        failed = 1;
        continue;
      }
      if (cap >= n) z.assign(raw.begin() + off, raw.begin() + off + n);  // stored raw
      else z.resize(cap);
      data[k] = std::move(z);
    }
  };
  run_host_threads((unsigned)std::max(1, std::min<int>(chunks, (int)std::thread::hardware_concurrency())), worker);
  if (failed) {
    set_error("zlib compression failed");
    return SHB_ERR_INTERNAL;
  }
  std::vector<uint8_t> head = exr_header(names, W, H);
  std::vector<uint64_t> offsets((size_t)chunks);
  uint64_t pos = head.size() + 8ull * chunks;
  for (int k = 0; k < chunks; ++k) {
    offsets[k] = pos;
    pos += 8 + data[k].size();
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    set_error("cannot open " + path + " for writing");
    return SHB_ERR_INVALID_ARG;
  }
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  ok = ok && std::fwrite(offsets.data(), 8, offsets.size(), f) == offsets.size();
  for (int k = 0; ok && k < chunks; ++k) {
    const int32_t y = k * kLinesPerChunk, sz = (int32_t)data[k].size();
    ok = std::fwrite(&y, 4, 1, f) == 1 && std::fwrite(&sz, 4, 1, f) == 1 &&
         std::fwrite(data[k].data(), 1, data[k].size(), f) == data[k].size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    set_error("write failed: " + path);
    return SHB_ERR_INVALID_ARG;
  }
  return SHB_OK;
}

const char* kCoeffNames[9] = {"L0", "L1m1", "L10", "L11", "L2m2", "L2m1", "L20", "L21", "L22"};

// path -> (parent/stem, extension) as std::filesystem::path would split it
void split_path(const std::string& path, std::string& base, std::string& ext) {
  const size_t slash = path.find_last_of('/');
  const size_t dot = path.find_last_of('.');
  const size_t name0 = slash == std::string::npos ? 0 : slash + 1;
  // a leading dot of the file name does not start an extension
  if (dot != std::string::npos && dot > name0 && path.size() - dot > 0) {
    base = path.substr(0, dot);
    ext = path.substr(dot);
  } else {
    base = path;
    ext.clear();
  }
}

// ------------------------------------------------------------- reader -----

float half_to_float(uint16_t h) {
  const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  uint32_t exp = (h >> 10) & 0x1Fu, man = h & 0x3FFu, bits;
  if (exp == 0) {
    if (man == 0) {
      bits = sign;
    } else {  // subnormal: renormalise
      int e = -1;
      do {
        ++e;
        man <<= 1;
      } while (!(man & 0x400u));
      bits = sign | ((uint32_t)(127 - 15 - e) << 23) | ((man & 0x3FFu) << 13);
    }
  } else if (exp == 31) {
    bits = sign | 0x7F800000u | (man << 13);
  } else {
    bits = sign | ((exp + 112u) << 23) | (man << 13);
  }
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

struct ExrFile {
  int W = 0, H = 0, comp = 0;
  std::vector<std::string> names;
  std::vector<int> types;
  std::vector<uint8_t> bytes;
  size_t chunk_table = 0;
};

bool read_exr_header(const std::string& path, ExrFile& e, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot read " + path;
    return false;
  }
  std::fseek(f, 0, SEEK_END);
  long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  e.bytes.resize(n > 0 ? (size_t)n : 0);
  size_t got = e.bytes.empty() ? 0 : std::fread(e.bytes.data(), 1, e.bytes.size(), f);
  std::fclose(f);
  const std::vector<uint8_t>& b = e.bytes;
  if (got != b.size() || b.size() < 8 || b[0] != 0x76 || b[1] != 0x2f || b[2] != 0x31 || b[3] != 0x01) {
    err = "not an OpenEXR file: " + path;
    return false;
  }
  if (b[4] != 2 || (b[5] & 0x1E)) {
    err = "only single-part scanline OpenEXR files are read";
    return false;
  }
  size_t i = 8;
  auto cstr = [&](std::string& out) {
    size_t j = i;
    while (j < b.size() && b[j]) ++j;
    if (j >= b.size()) return false;
    out.assign(reinterpret_cast<const char*>(&b[i]), j - i);
    i = j + 1;
    return true;
  };
  bool have_ch = false, have_dw = false;
  int x0 = 0, y0 = 0, x1 = -1, y1 = -1;
  while (i < b.size() && b[i]) {
    std::string name, type;
    int32_t size = 0;
    if (!cstr(name) || !cstr(type) || i + 4 > b.size()) break;
    std::memcpy(&size, &b[i], 4);
    i += 4;
    if (size < 0 || i + (size_t)size > b.size()) break;
    const uint8_t* v = &b[i];
    if (name == "channels") {
      size_t k = 0;
      while (k < (size_t)size && v[k]) {
        size_t z = k;
        while (z < (size_t)size && v[z]) ++z;
        if (z + 17 > (size_t)size) break;
        e.names.emplace_back(reinterpret_cast<const char*>(v + k), z - k);
        int32_t t;
        std::memcpy(&t, v + z + 1, 4);
        e.types.push_back(t);
        k = z + 17;
      }
      have_ch = true;
    } else if (name == "compression" && size >= 1) {
      e.comp = v[0];
    } else if (name == "dataWindow" && size >= 16) {
      int32_t w[4];
      std::memcpy(w, v, 16);
      x0 = w[0];
      y0 = w[1];
      x1 = w[2];
      y1 = w[3];
      have_dw = true;
    }
    i += (size_t)size;
  }
  if (!have_ch || !have_dw || i >= b.size() || x1 < x0 || y1 < y0) {
    err = "bad OpenEXR header: " + path;
    return false;
  }
  // in 64 bits: the window's corners are arbitrary int32 values
  const int64_t W = (int64_t)x1 - x0 + 1, H = (int64_t)y1 - y0 + 1;
  if (W > 2147483647 || H > 2147483647 || W * H > 2147483647) {
    err = "OpenEXR image larger than 2^31 - 1 pixels: " + path;
    return false;
  }
  e.W = (int)W;
  e.H = (int)H;
  e.chunk_table = i + 1;
  if (e.comp != 0 && e.comp != 2 && e.comp != 3) {
    err = "unsupported OpenEXR compression (NONE, ZIPS and ZIP are read)";
    return false;
  }
  for (int t : e.types)
    if (t < 0 || t > 2) {
      err = "bad OpenEXR channel type";
      return false;
    }
  return true;
}

bool read_exr_channels(ExrFile& e, const std::vector<int>& want, float* out, std::string& err) {
  const std::vector<uint8_t>& b = e.bytes;
  const int lpc = e.comp == 3 ? 16 : 1;
  const int chunks = (e.H + lpc - 1) / lpc;
  size_t line_bytes = 0;
  std::vector<size_t> off;
  for (int t : e.types) {
    off.push_back(line_bytes);
    line_bytes += (size_t)e.W * (t == 1 ? 2 : 4);
  }
  if (e.chunk_table + 8ull * chunks > b.size()) {
    err = "truncated OpenEXR offset table";
    return false;
  }
  std::vector<uint8_t> raw, tmp;
  for (int k = 0; k < chunks; ++k) {
    uint64_t pos;
    std::memcpy(&pos, &b[e.chunk_table + 8ull * k], 8);
    if (pos > b.size() || b.size() - pos < 8) {  // (pos + 8 can wrap)
      err = "bad OpenEXR chunk offset";
      return false;
    }
    int32_t y, size;
    std::memcpy(&y, &b[pos], 4);
    std::memcpy(&size, &b[pos + 4], 4);
    const int ly = k * lpc;
    const int lines = std::min(lpc, e.H - ly);
    const size_t n = line_bytes * lines;
    // a zlib stream inflates by at most about 1032:1, so a chunk of `size`
    // bytes cannot hold more: refuse before allocating its lines
    if (size < 0 || pos + 8 + (uint64_t)size > b.size() ||
        (e.comp == 0 ? (size_t)size != n : n > 1100 * (uint64_t)size + 1024)) {
      err = "bad OpenEXR chunk size";
      return false;
    }
    const uint8_t* d = b.data() + pos + 8;
    raw.resize(n);
    if (e.comp == 0 || (size_t)size == n) {
      if ((size_t)size != n) {
        err = "bad OpenEXR chunk size";
        return false;
      }
      std::memcpy(raw.data(), d, n);
    } else {
      tmp.resize(n);
      uLongf got = (uLongf)n;
      if (uncompress(tmp.data(), &got, d, (uLong)size) != Z_OK || got != n) {
        err = "OpenEXR chunk does not inflate";
        return false;
      }
      // undo the delta predictor, then re-interleave the two byte halves
      for (size_t q = 1; q < n; ++q) tmp[q] = (uint8_t)(tmp[q - 1] + tmp[q] - 128);
      const size_t half = (n + 1) / 2;
      for (size_t q = 0; q < n; ++q) raw[q] = (q & 1) ? tmp[half + q / 2] : tmp[q / 2];
    }
    for (int l = 0; l < lines; ++l)
      for (size_t c = 0; c < want.size(); ++c) {
        const int ch = want[c];
        const uint8_t* src = raw.data() + (size_t)l * line_bytes + off[(size_t)ch];
        float* dst = out + c * (size_t)e.W * e.H + (size_t)(ly + l) * e.W;
        for (int x = 0; x < e.W; ++x) {
          if (e.types[(size_t)ch] == 1) {
            uint16_t h;
            std::memcpy(&h, src + 2 * (size_t)x, 2);
            dst[x] = half_to_float(h);
          } else if (e.types[(size_t)ch] == 2) {
            std::memcpy(&dst[x], src + 4 * (size_t)x, 4);
          } else {
            uint32_t u;
            std::memcpy(&u, src + 4 * (size_t)x, 4);
            dst[x] = (float)u;
          }
        }
      }
  }
  return true;
}

}  // namespace

// Named channels of an OpenEXR file as float planes (n x width x height);
// with out == NULL only the dimensions are returned.
shb_status exr_load_channels(const char* path, const char* const* names, int n, int* width, int* height, float* out) {
  ExrFile e;
  std::string err;
  if (!read_exr_header(path, e, err)) {
    set_error(err);
    return SHB_ERR_INVALID_ARG;
  }
  std::vector<int> want;
  for (int k = 0; k < n; ++k) {
    int found = -1;
    for (size_t c = 0; c < e.names.size(); ++c)
      if (e.names[c] == names[k]) found = (int)c;
    if (found < 0) {
      set_error(std::string("no channel ") + names[k] + " in " + path);
      return SHB_ERR_INVALID_ARG;
    }
    want.push_back(found);
  }
  if (width) *width = e.W;
  if (height) *height = e.H;
  if (out && !read_exr_channels(e, want, out, err)) {
    set_error(err);
    return SHB_ERR_INVALID_ARG;
  }
  return SHB_OK;
}

shb_status save_sh_lightmap_device(shb_context* c, const float* d_sh, const float* d_env, int W, int H,
                                   const std::string& path, int mode) {
  if (mode == SHB_SAVE_COMBINED) {
    ChanTable t{};
    std::vector<std::string> names;
    const char* rgb[3] = {".R", ".G", ".B"};
    for (int i = 0; i < 9; ++i)
      for (int k = 0; k < 3; ++k) {
        t.c[t.n++] = ChanSpec{0, 3 * i + k};
        names.push_back(std::string(kCoeffNames[i]) + rgb[k]);
      }
    t.c[t.n++] = ChanSpec{2, 0};
    names.push_back("EnvVisibility");
    return write_exr(c, d_sh, d_env, W, H, t, names, path);
  }
  std::string base, ext;
  split_path(path, base, ext);
  if (mode == SHB_SAVE_SPLIT_CHANNELS) {
    for (int i = 0; i < 9; ++i) {
      ChanTable t{};
      std::vector<std::string> names = {"R", "G", "B"};
      for (int k = 0; k < 3; ++k) t.c[t.n++] = ChanSpec{0, 3 * i + k};
      if (i == 0) {
        t.c[t.n++] = ChanSpec{2, 0};
        names.push_back("A");
      }
      SHB_TRY(write_exr(c, d_sh, d_env, W, H, t, names, base + "_" + kCoeffNames[i] + ext));
    }
    return SHB_OK;
  }
  if (mode == SHB_SAVE_LUMINANCE_PACKED) {
    const std::vector<std::string> names = {"R", "G", "B", "A"};
    ChanTable t0{}, t1{}, t2{};
    t0.c[0] = ChanSpec{0, 0};
    t0.c[1] = ChanSpec{0, 1};
    t0.c[2] = ChanSpec{0, 2};
    t0.c[3] = ChanSpec{2, 0};
    t0.n = 4;
    for (int k = 0; k < 4; ++k) {
      t1.c[k] = ChanSpec{1, 1 + k};
      t2.c[k] = ChanSpec{1, 5 + k};
    }
    t1.n = t2.n = 4;
    SHB_TRY(write_exr(c, d_sh, d_env, W, H, t0, names, base + "_packed_0" + ext));
    SHB_TRY(write_exr(c, d_sh, d_env, W, H, t1, names, base + "_packed_1" + ext));
    return write_exr(c, d_sh, d_env, W, H, t2, names, base + "_packed_2" + ext);
  }
  set_error("unknown save mode");
  return SHB_ERR_INVALID_ARG;
}

}  // namespace shb
