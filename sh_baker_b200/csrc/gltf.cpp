// gltf.cpp - LoadScene (src/loader.cpp:144-844): a minimal glTF 2.0 reader
// producing the bake's scene description.
//
// Reads .gltf (JSON, buffers as data URIs or files beside it) and .glb, node
// hierarchies with matrix or TRS transforms, triangle primitives with
// POSITION / NORMAL / TEXCOORD_0 (required, as the reference requires them)
// and optional TEXCOORD_1 / TANGENT, materials with
// KHR_materials_emissive_strength and a PNG or JPEG base-colour texture or the
// baseColorFactor, and KHR_lights_punctual lights.  Behaviour follows the
// reference loader:
//   - a primitive without material, POSITION, NORMAL or TEXCOORD_0 fails the
//     load (src/loader.cpp:146-167); primitives without indices have no
//     triangles (:268-290); triangles with a repeated index are dropped
//     (:333-361);
//   - an emissive material makes each of its primitives an area light of its
//     object-space surface area (:385-406, src/scene.cpp:197-207);
//   - without a texture the albedo is a 1x1 RGBA texture of the
//     baseColorFactor through LinearToSRGB (:486-505, src/colorspace.h:17-21);
//     without materials a white default is used (:438-465);
//   - a light takes the node's translation and its rotation applied to -Z
//     (:541-560), cone angles become cosines (:587-598).
// Tangents missing from the file are built by the MikkTSpace method
// (tspace.cpp), as the reference builds them with that library.
// Differences: JPEG textures are decoded by jpeg.cpp (Huffman-coded
// sequential and progressive files) instead of stb_image.  The sky
// environment (:705-797) is not read: the bake never samples it.
#include <zlib.h>

#include "tspace.h"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "host_scene.h"
#include "shb_internal.h"

namespace shb {
// jpeg.cpp: sequential JPEG -> 8-bit RGB.
bool decode_jpeg(const std::vector<uint8_t>& f, std::vector<uint8_t>& out, uint32_t& W, uint32_t& H, uint32_t& C,
                 std::string& err);
}  // namespace shb

namespace shb {
namespace {

// ------------------------------------------------------------- JSON -------

struct Json {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;
  const Json* get(const std::string& k) const {
    if (kind != Obj) return nullptr;
    for (const auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
  double number(const std::string& k, double def) const {
    const Json* j = get(k);
    return j && j->kind == Num ? j->num : def;
  }
  // `def` when the key is absent or not a number; INT_MIN (an index no
  // array has) when the number is not an integer that fits an int.
  int integer(const std::string& k, int def) const {
    const Json* j = get(k);
    return j && j->kind == Num ? to_index(j->num, INT_MIN) : def;
  }
  // A JSON number as an int: the value when it is integral and fits an int,
  // else `bad` (an out-of-range double-to-int conversion is undefined).
  static int to_index(double x, int bad) {
    return x >= -2147483648.0 && x <= 2147483647.0 && x == std::floor(x) ? (int)x : bad;
  }
};

// An accessor or buffer-view size field (count, byteOffset, byteLength,
// byteStride): 0 when absent, false unless it is an integral number in
// [0, 2^53].
bool size_field(const Json& o, const char* k, size_t& out) {
  const Json* j = o.get(k);
  out = 0;
  if (!j) return true;
  if (j->kind != Json::Num || !(j->num >= 0.0 && j->num <= 9007199254740992.0) || j->num != std::floor(j->num))
    return false;
  out = (size_t)j->num;
  return true;
}

// A JSON number as a float: the nearest float, with magnitudes beyond the
// float range taken to infinity explicitly (C++ leaves that cast undefined).
float to_f32(double x) {
  if (std::isfinite(x) && std::fabs(x) > (double)FLT_MAX) return x > 0 ? INFINITY : -INFINITY;
  return (float)x;
}

struct Parser {
  const char* p;
  const char* end;
  std::string err;
  void ws() {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  bool fail(const char* m) {
    if (err.empty()) err = m;
    return false;
  }
  bool lit(const char* s) {
    size_t n = std::strlen(s);
    if ((size_t)(end - p) < n || std::strncmp(p, s, n) != 0) return fail("bad literal");
    p += n;
    return true;
  }
  static void utf8(std::string& o, uint32_t cp) {
    if (cp < 0x80) o += (char)cp;
    else if (cp < 0x800) {
      o += (char)(0xC0 | (cp >> 6));
      o += (char)(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
      o += (char)(0xE0 | (cp >> 12));
      o += (char)(0x80 | ((cp >> 6) & 0x3F));
      o += (char)(0x80 | (cp & 0x3F));
    } else {
      o += (char)(0xF0 | (cp >> 18));
      o += (char)(0x80 | ((cp >> 12) & 0x3F));
      o += (char)(0x80 | ((cp >> 6) & 0x3F));
      o += (char)(0x80 | (cp & 0x3F));
    }
  }
  bool hex4(uint32_t& v) {
    if (end - p < 4) return fail("bad escape");
    v = 0;
    for (int i = 0; i < 4; ++i, ++p) {
      char c = *p;
      v <<= 4;
      if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
      else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
      else return fail("bad escape");
    }
    return true;
  }
  bool string(std::string& o) {
    if (p >= end || *p != '"') return fail("expected string");
    ++p;
    while (p < end && *p != '"') {
      char c = *p++;
      if (c != '\\') {
        o += c;
        continue;
      }
      if (p >= end) return fail("bad escape");
      char e = *p++;
      switch (e) {
        case '"': o += '"'; break;
        case '\\': o += '\\'; break;
        case '/': o += '/'; break;
        case 'b': o += '\b'; break;
        case 'f': o += '\f'; break;
        case 'n': o += '\n'; break;
        case 'r': o += '\r'; break;
        case 't': o += '\t'; break;
        case 'u': {
          uint32_t cp;
          if (!hex4(cp)) return false;
          if (cp >= 0xD800 && cp < 0xDC00 && end - p >= 6 && p[0] == '\\' && p[1] == 'u') {
            p += 2;
            uint32_t lo;
            if (!hex4(lo)) return false;
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          }
          utf8(o, cp);
          break;
        }
        default: return fail("bad escape");
      }
    }
    if (p >= end) return fail("unterminated string");
    ++p;
    return true;
  }
  bool value(Json& j, int depth) {
    if (depth > 256) return fail("nesting too deep");
    ws();
    if (p >= end) return fail("unexpected end");
    char c = *p;
    if (c == '{') {
      j.kind = Json::Obj;
      ++p;
      ws();
      if (p < end && *p == '}') {
        ++p;
        return true;
      }
      while (true) {
        ws();
        std::string k;
        if (!string(k)) return false;
        ws();
        if (p >= end || *p != ':') return fail("expected ':'");
        ++p;
        j.obj.emplace_back(std::move(k), Json());
        if (!value(j.obj.back().second, depth + 1)) return false;
        ws();
        if (p < end && *p == ',') {
          ++p;
          continue;
        }
        if (p < end && *p == '}') {
          ++p;
          return true;
        }
        return fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      j.kind = Json::Arr;
      ++p;
      ws();
      if (p < end && *p == ']') {
        ++p;
        return true;
      }
      while (true) {
        j.arr.emplace_back();
        if (!value(j.arr.back(), depth + 1)) return false;
        ws();
        if (p < end && *p == ',') {
          ++p;
          continue;
        }
        if (p < end && *p == ']') {
          ++p;
          return true;
        }
        return fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      j.kind = Json::Str;
      return string(j.str);
    }
    if (c == 't') {
      j.kind = Json::Bool;
      j.b = true;
      return lit("true");
    }
    if (c == 'f') {
      j.kind = Json::Bool;
      return lit("false");
    }
    if (c == 'n') return lit("null");
    const char* s = p;
    if (p < end && (*p == '-' || *p == '+')) ++p;
    while (p < end && ((*p >= '0' && *p <= '9') || *p == '.' || *p == 'e' || *p == 'E' || *p == '-' || *p == '+'))
      ++p;
    if (p == s) return fail("unexpected character");
    j.kind = Json::Num;
    j.num = std::strtod(std::string(s, p).c_str(), nullptr);
    return true;
  }
};

// ------------------------------------------------------------- PNG --------

uint32_t be32(const uint8_t* b) { return (uint32_t)b[0] << 24 | (uint32_t)b[1] << 16 | (uint32_t)b[2] << 8 | b[3]; }

// PNG of any colour type, bit depth and interlace -> 3 (RGB) or 4 (RGBA)
// 8-bit channels.  The reference's textures come from tinygltf's image
// loader over stb_image (src/loader.cpp:415-432), whose 8-bit conversions
// are these: 1/2/4-bit grey is scaled to 0..255 (x255, x85, x17), palette
// indices are not; a tRNS colour key on a grey or RGB image adds an alpha
// channel that is 0 where the pixel's samples equal the key; a palette with
// tRNS gives its alphas.  An image without alpha has 3 channels here and 4
// (alpha 255) there: either way the bake sees alpha 1.  16-bit samples keep
// their high byte, stb_image's 8-bit conversion; tinygltf may instead keep
// 16-bit samples, which the reference's albedo lookup would read as bytes.
// Adam7-interlaced images are decoded pass by pass (each pass a filtered
// sub-image) and scattered to their pixels.
bool decode_png(const std::vector<uint8_t>& f, std::vector<uint8_t>& out, uint32_t& W, uint32_t& H, uint32_t& C,
                std::string& err) {
  static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (f.size() < 8 || std::memcmp(f.data(), sig, 8) != 0) {
    err = "not a PNG or JPEG (only PNG and JPEG textures are supported)";
    return false;
  }
  size_t i = 8;
  int depth = 0, ctype = -1, interlace = 0;
  std::vector<uint8_t> idat, plte, trns;
  while (i + 12 <= f.size()) {
    uint32_t len = be32(&f[i]);
    std::string type(reinterpret_cast<const char*>(&f[i + 4]), 4);
    if (i + 12 + (size_t)len > f.size()) break;
    const uint8_t* d = &f[i + 8];
    if (type == "IHDR" && len >= 13) {
      W = be32(d);
      H = be32(d + 4);
      depth = d[8];
      ctype = d[9];
      interlace = d[12];
    } else if (type == "PLTE") {
      plte.assign(d, d + len);
    } else if (type == "tRNS") {
      trns.assign(d, d + len);
    } else if (type == "IDAT") {
      idat.insert(idat.end(), d, d + len);
    } else if (type == "IEND") {
      break;
    }
    i += 12 + (size_t)len;
  }
  if (ctype < 0 || W == 0 || H == 0 || W > (1u << 15) || H > (1u << 15)) {
    err = "bad PNG header";
    return false;
  }
  const int ch = ctype == 0 ? 1 : ctype == 2 ? 3 : ctype == 3 ? 1 : ctype == 4 ? 2 : ctype == 6 ? 4 : 0;
  if (!ch) {
    err = "bad PNG colour type";
    return false;
  }
  // PNG 1.2 table 11.1: the bit depths each colour type allows
  const bool depth_ok = ctype == 0 ? (depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)
                        : ctype == 3 ? (depth == 1 || depth == 2 || depth == 4 || depth == 8)
                                     : (depth == 8 || depth == 16);
  if (!depth_ok || interlace > 1) {
    err = "unsupported PNG (bad bit depth for its colour type, or unknown interlace method)";
    return false;
  }
  // colour key (grey: one 16-bit sample, RGB: three) and the output channels
  const bool key = (ctype == 0 && trns.size() >= 2) || (ctype == 2 && trns.size() >= 6);
  uint16_t keyv[3] = {0, 0, 0};
  if (key)
    for (int k = 0; k < (ctype == 0 ? 1 : 3); ++k) keyv[k] = (uint16_t)(trns[2 * k] << 8 | trns[2 * k + 1]);
  const bool alpha = ctype == 4 || ctype == 6 || (ctype == 3 && !trns.empty()) || key;
  C = alpha ? 4 : 3;
  // passes: (x0, y0, dx, dy); one pass covering every pixel when not interlaced
  static const int adam7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                                  {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
  static const int whole[1][4] = {{0, 0, 1, 1}};
  const int npass = interlace ? 7 : 1;
  const int(*pass)[4] = interlace ? adam7 : whole;
  const size_t bitspp = (size_t)ch * depth, bpp = std::max<size_t>(1, bitspp / 8);
  auto pass_w = [&](int p) { return (W > (uint32_t)pass[p][0]) ? (W - pass[p][0] + pass[p][2] - 1) / pass[p][2] : 0u; };
  auto pass_h = [&](int p) { return (H > (uint32_t)pass[p][1]) ? (H - pass[p][1] + pass[p][3] - 1) / pass[p][3] : 0u; };
  size_t total = 0;
  for (int p = 0; p < npass; ++p)
    if (pass_w(p) && pass_h(p)) total += ((pass_w(p) * bitspp + 7) / 8 + 1) * pass_h(p);
  // a zlib stream inflates by at most about 1032:1: refuse a size the IDAT
  // data cannot hold before allocating it
  if (total > 1100 * (uint64_t)idat.size() + 1024) {
    err = "PNG inflate failed";
    return false;
  }
  std::vector<uint8_t> raw(total);
  uLongf rl = (uLongf)raw.size();
  if (uncompress(raw.data(), &rl, idat.data(), (uLong)idat.size()) != Z_OK || rl != raw.size()) {
    err = "PNG inflate failed";
    return false;
  }
  out.assign((size_t)W * H * C, 255);
  const int scale = ctype == 0 && depth < 8 ? 255 / ((1 << depth) - 1) : 1;
  auto b8 = [&](uint32_t v) { return (uint8_t)(depth == 16 ? v >> 8 : v * scale); };
  size_t off = 0;
  std::vector<uint8_t> cur, prev;
  for (int p = 0; p < npass; ++p) {
    const uint32_t pw = pass_w(p), ph = pass_h(p);
    if (!pw || !ph) continue;
    const size_t stride = (pw * bitspp + 7) / 8;
    cur.assign(stride, 0);
    prev.assign(stride, 0);  // the line above the first one is zero
    for (uint32_t y = 0; y < ph; ++y) {
      const uint8_t ft = raw[off];
      const uint8_t* s = &raw[off + 1];
      off += stride + 1;
      for (size_t x = 0; x < stride; ++x) {
        const int a = x >= bpp ? cur[x - bpp] : 0, b = prev[x], c = x >= bpp ? prev[x - bpp] : 0;
        int v = s[x];
        switch (ft) {
          case 0: break;
          case 1: v += a; break;
          case 2: v += b; break;
          case 3: v += (a + b) / 2; break;
          case 4: {
            const int pp = a + b - c, pa = std::abs(pp - a), pb = std::abs(pp - b), pc = std::abs(pp - c);
            v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
            break;
          }
          default:
            err = "bad PNG filter";
            return false;
        }
        cur[x] = (uint8_t)v;
      }
      for (uint32_t x = 0; x < pw; ++x) {
        uint32_t v[4] = {0, 0, 0, 0};
        for (int k = 0; k < ch; ++k) {
          const size_t bit = ((size_t)x * ch + k) * depth;
          if (depth == 16) v[k] = (uint32_t)cur[bit / 8] << 8 | cur[bit / 8 + 1];
          else if (depth == 8) v[k] = cur[bit / 8];
          else v[k] = (cur[bit / 8] >> (8 - depth - (bit & 7))) & ((1u << depth) - 1);
        }
        const size_t X = pass[p][0] + (size_t)x * pass[p][2], Y = pass[p][1] + (size_t)y * pass[p][3];
        uint8_t* o = &out[(Y * W + X) * C];
        if (ctype == 3) {
          if (3 * (size_t)v[0] + 2 >= plte.size()) {
            err = "PNG palette index out of range";
            return false;
          }
          for (int k = 0; k < 3; ++k) o[k] = plte[3 * v[0] + k];
          if (alpha) o[3] = v[0] < trns.size() ? trns[v[0]] : 255;
        } else if (ctype == 0 || ctype == 4) {
          o[0] = o[1] = o[2] = b8(v[0]);
          if (ctype == 4) o[3] = b8(v[1]);
          else if (key) o[3] = v[0] == keyv[0] ? 0 : 255;
        } else {
          for (int k = 0; k < 3; ++k) o[k] = b8(v[k]);
          if (ctype == 6) o[3] = b8(v[3]);
          else if (key) o[3] = v[0] == keyv[0] && v[1] == keyv[1] && v[2] == keyv[2] ? 0 : 255;
        }
      }
      cur.swap(prev);
    }
  }
  return true;
}

// ------------------------------------------------------------- glTF -------

bool read_file(const std::string& path, std::vector<uint8_t>& out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return true;
}

bool base64(const std::string& s, std::vector<uint8_t>& out) {
  auto val = [](char c) -> int {
    if (c >= 'A' && c <= 'Z') return c - 'A';
    if (c >= 'a' && c <= 'z') return c - 'a' + 26;
    if (c >= '0' && c <= '9') return c - '0' + 52;
    if (c == '+' || c == '-') return 62;
    if (c == '/' || c == '_') return 63;
    return -1;
  };
  uint32_t acc = 0;
  int bits = 0;
  for (char c : s) {
    if (c == '=' || c == '\n' || c == '\r') continue;
    int v = val(c);
    if (v < 0) return false;
    acc = (acc << 6) | (uint32_t)v;
    bits += 6;
    if (bits >= 8) {
      bits -= 8;
      out.push_back((uint8_t)(acc >> bits));
    }
  }
  return true;
}

std::string uri_decode(const std::string& s) {
  std::string o;
  for (size_t i = 0; i < s.size(); ++i) {
    if (s[i] == '%' && i + 2 < s.size()) {
      o += (char)std::strtol(s.substr(i + 1, 2).c_str(), nullptr, 16);
      i += 2;
    } else {
      o += s[i];
    }
  }
  return o;
}

// data: URI or a file relative to the glTF
bool load_uri(const std::string& uri, const std::string& dir, std::vector<uint8_t>& out, std::string& err) {
  if (uri.rfind("data:", 0) == 0) {
    size_t comma = uri.find(',');
    if (comma == std::string::npos || uri.substr(0, comma).find(";base64") == std::string::npos) {
      err = "unsupported data URI";
      return false;
    }
    if (!base64(uri.substr(comma + 1), out)) {
      err = "bad base64 data";
      return false;
    }
    return true;
  }
  const std::string path = (!uri.empty() && uri[0] == '/') ? uri : dir + uri_decode(uri);
  if (!read_file(path, out)) {
    err = "cannot read " + path;
    return false;
  }
  return true;
}

struct Model {
  Json j;
  std::vector<std::vector<uint8_t>> buffers;
  std::string dir;
};

const Json* arr_at(const Json& root, const char* key, int i) {
  const Json* a = root.get(key);
  if (!a || a->kind != Json::Arr || i < 0 || (size_t)i >= a->arr.size()) return nullptr;
  return &a->arr[(size_t)i];
}

// Accessor -> (pointer to the first element, element stride in bytes, count)
struct View {
  const uint8_t* data = nullptr;
  size_t stride = 0, count = 0;
  int comp_type = 0, comps = 0;
};

int type_comps(const std::string& t) {
  if (t == "SCALAR") return 1;
  if (t == "VEC2") return 2;
  if (t == "VEC3") return 3;
  if (t == "VEC4") return 4;
  if (t == "MAT4") return 16;
  return 0;
}
int comp_size(int ct) {
  return ct == 5120 || ct == 5121 ? 1 : ct == 5122 || ct == 5123 ? 2 : ct == 5125 || ct == 5126 ? 4 : 0;
}

bool accessor(const Model& m, int idx, View& v, std::string& err) {
  const Json* a = arr_at(m.j, "accessors", idx);
  if (!a) {
    err = "bad accessor index";
    return false;
  }
  if (a->get("sparse")) {
    err = "sparse accessors are not supported";
    return false;
  }
  v.comp_type = a->integer("componentType", 0);
  const Json* t = a->get("type");
  v.comps = t && t->kind == Json::Str ? type_comps(t->str) : 0;
  size_t a_off = 0;
  if (!size_field(*a, "count", v.count) || !size_field(*a, "byteOffset", a_off)) {
    err = "accessor count and byteOffset must be non-negative integers";
    return false;
  }
  const int cs = comp_size(v.comp_type);
  if (!cs || !v.comps) {
    err = "bad accessor type";
    return false;
  }
  const Json* bvi = a->get("bufferView");
  if (!bvi) {
    err = "accessor without bufferView";
    return false;
  }
  const Json* bv = bvi->kind == Json::Num ? arr_at(m.j, "bufferViews", Json::to_index(bvi->num, -1)) : nullptr;
  if (!bv) {
    err = "bad bufferView index";
    return false;
  }
  const int b = bv->integer("buffer", -1);
  if (b < 0 || (size_t)b >= m.buffers.size()) {
    err = "bad buffer index";
    return false;
  }
  size_t view_begin = 0, len = 0;
  if (!size_field(*bv, "byteOffset", view_begin) || !size_field(*bv, "byteLength", len) ||
      !size_field(*bv, "byteStride", v.stride)) {
    err = "bufferView byteOffset, byteLength and byteStride must be non-negative integers";
    return false;
  }
  const size_t elem = (size_t)cs * v.comps;
  if (!v.stride) v.stride = elem;
  // in 128 bits: counts and offsets up to 2^53 cannot wrap the check
  using u128 = unsigned __int128;
  const u128 need = v.count ? (u128)(v.count - 1) * v.stride + elem : 0;
  const u128 off = (u128)view_begin + a_off;
  if (off + need > (u128)view_begin + len || (u128)view_begin + len > m.buffers[b].size()) {
    err = "accessor exceeds its buffer";
    return false;
  }
  v.data = m.buffers[b].data() + (size_t)off;
  return true;
}

bool float_attr(const Model& m, int idx, int comps, std::vector<float>& out, size_t& count, std::string& err) {
  View v;
  if (!accessor(m, idx, v, err)) return false;
  if (v.comp_type != 5126 || v.comps != comps) {
    err = "vertex attribute must be FLOAT with " + std::to_string(comps) + " components";
    return false;
  }
  count = v.count;
  out.resize(v.count * comps);
  for (size_t i = 0; i < v.count; ++i) std::memcpy(&out[i * comps], v.data + i * v.stride, sizeof(float) * comps);
  return true;
}

// Column-major 4x4 (glTF) -> our 3x4 row-major [L | t]
void mat_from_gltf(const double m[16], float out[12]) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) out[r * 4 + c] = to_f32(m[c * 4 + r]);
}

// Eigen Affine3f composition: identity.translate(t).rotate(q).scale(s) = T R S
void node_local(const Json& node, float out[12]) {
  const Json* mat = node.get("matrix");
  if (mat && mat->kind == Json::Arr && mat->arr.size() == 16) {
    double m[16];
    for (int i = 0; i < 16; ++i) m[i] = mat->arr[i].num;
    mat_from_gltf(m, out);
    return;
  }
  float t[3] = {0, 0, 0}, q[4] = {0, 0, 0, 1}, s[3] = {1, 1, 1};
  const Json* tj = node.get("translation");
  if (tj && tj->kind == Json::Arr && tj->arr.size() == 3)
    for (int i = 0; i < 3; ++i) t[i] = to_f32(tj->arr[i].num);
  const Json* rj = node.get("rotation");
  bool has_r = rj && rj->kind == Json::Arr && rj->arr.size() == 4;
  if (has_r)
    for (int i = 0; i < 4; ++i) q[i] = to_f32(rj->arr[i].num);
  const Json* sj = node.get("scale");
  if (sj && sj->kind == Json::Arr && sj->arr.size() == 3)
    for (int i = 0; i < 3; ++i) s[i] = to_f32(sj->arr[i].num);
  // Eigen's quaternion -> matrix (expects a unit quaternion, not normalised)
  const float x = q[0], y = q[1], z = q[2], w = q[3];
  float R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (has_r) {
    const float tx = 2 * x, ty = 2 * y, tz = 2 * z, twx = tx * w, twy = ty * w, twz = tz * w, txx = tx * x,
                txy = ty * x, txz = tz * x, tyy = ty * y, tyz = tz * y, tzz = tz * z;
    R[0] = 1 - (tyy + tzz);
    R[1] = txy - twz;
    R[2] = txz + twy;
    R[3] = txy + twz;
    R[4] = 1 - (txx + tzz);
    R[5] = tyz - twx;
    R[6] = txz - twy;
    R[7] = tyz + twx;
    R[8] = 1 - (txx + tyy);
  }
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) out[r * 4 + c] = R[r * 3 + c] * s[c];
    out[r * 4 + 3] = t[r];
  }
}

void compose(const float a[12], const float b[12], float out[12]) {
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 4; ++c) {
      float v = a[r * 4 + 0] * b[0 * 4 + c] + a[r * 4 + 1] * b[1 * 4 + c] + a[r * 4 + 2] * b[2 * 4 + c];
      if (c == 3) v += a[r * 4 + 3];
      out[r * 4 + c] = v;
    }
  }
}

// The reference casts the rounded value straight to uint8_t, which C++
// leaves undefined outside [0, 255] (a baseColorFactor above 1 or below 0).
// Compiled for x86-64 that cast is a truncating conversion to a 32-bit
// integer (INT_MIN for values out of its range and for NaN) whose low byte
// is kept; the same steps are written out here without undefined behaviour.
uint8_t byte_of(float r) {
  const int32_t i = r >= -2147483648.0f && r < 2147483648.0f ? (int32_t)r : INT32_MIN;
  return (uint8_t)(uint32_t)i;
}

// src/colorspace.h:17-21
uint8_t linear_to_srgb(float x) {
  if (x <= 0.0031308f) return byte_of(std::rint(x * 12.92f * 255.0f));
  return byte_of(std::rint((1.055f * std::pow(x, 1.0f / 2.4f) - 0.055f) * 255.0f));
}


float surface_area(const shb_host_scene::Geo& g) {
  float total = 0.0f;
  for (size_t i = 0; i + 2 < g.idx.size(); i += 3) {
    const float* a = &g.v[3 * g.idx[i]];
    const float* b = &g.v[3 * g.idx[i + 1]];
    const float* c = &g.v[3 * g.idx[i + 2]];
    const float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    const float x = e1[1] * e2[2] - e1[2] * e2[1], y = e1[2] * e2[0] - e1[0] * e2[2],
                z = e1[0] * e2[1] - e1[1] * e2[0];
    total += 0.5f * std::sqrt(x * x + (y * y + z * z));
  }
  return total;
}

// Tangents of a primitive that has no TANGENT attribute
// (src/loader.cpp:363-385): the MikkTSpace method of tspace.cpp.
void build_tangents(shb_host_scene::Geo& g, size_t nv) {
  g.t.assign(4 * nv, 0.0f);
  shb::generate_tangent_frames(g.v.data(), g.n.data(), g.uv0.data(), nv, g.idx.data(), g.idx.size(), g.t.data());
}

struct Loader {
  Model m;
  shb_host_scene* s;
  std::string err;

  bool primitive(const Json& pr, const float xf[12]) {
    const Json* attrs = pr.get("attributes");
    const int mat = pr.integer("material", -1);
    if (mat < 0) return fail("Primitive missing material.");
    auto attr = [&](const char* k) -> int {
      const Json* a = attrs ? attrs->get(k) : nullptr;
      return a && a->kind == Json::Num ? Json::to_index(a->num, -1) : -1;
    };
    if (attr("POSITION") < 0) return fail("Primitive missing POSITION attribute.");
    if (attr("NORMAL") < 0) return fail("Primitive missing NORMAL attribute. Baking requires Vertex Normals.");
    if (attr("TEXCOORD_0") < 0) return fail("Primitive missing TEXCOORD_0 attribute. Baking requires UVs.");
    if ((size_t)mat >= s->mats.size()) return fail("primitive material out of range");
    shb_host_scene::Geo g;
    g.material = mat;
    std::memcpy(g.transform, xf, sizeof(g.transform));
    size_t nv = 0, c2 = 0;
    if (!float_attr(m, attr("POSITION"), 3, g.v, nv, err)) return false;
    if (!float_attr(m, attr("NORMAL"), 3, g.n, c2, err) || c2 != nv) return fail(err.empty() ? "NORMAL count" : err);
    if (!float_attr(m, attr("TEXCOORD_0"), 2, g.uv0, c2, err) || c2 != nv)
      return fail(err.empty() ? "TEXCOORD_0 count" : err);
    if (attr("TEXCOORD_1") >= 0 && (!float_attr(m, attr("TEXCOORD_1"), 2, g.uv1, c2, err) || c2 != nv))
      return fail(err.empty() ? "TEXCOORD_1 count" : err);
    if (attr("TANGENT") >= 0 && (!float_attr(m, attr("TANGENT"), 4, g.t, c2, err) || c2 != nv))
      return fail(err.empty() ? "TANGENT count" : err);
    const int ii = pr.integer("indices", -1);
    if (ii >= 0) {
      View v;
      if (!accessor(m, ii, v, err)) return false;
      if (v.comps != 1 || (v.comp_type != 5121 && v.comp_type != 5123 && v.comp_type != 5125))
        return fail("indices must be unsigned byte/short/int scalars");
      for (size_t i = 0; i < v.count; ++i) {
        const uint8_t* q = v.data + i * v.stride;
        uint32_t x = v.comp_type == 5121 ? *q : v.comp_type == 5123 ? (uint32_t)(q[0] | q[1] << 8)
                                                                     : (uint32_t)(q[0] | q[1] << 8 | q[2] << 16 |
                                                                                  (uint32_t)q[3] << 24);
        if (x >= nv) return fail("index out of range");
        g.idx.push_back(x);
      }
      g.idx.resize(g.idx.size() / 3 * 3);
      std::vector<uint32_t> keep;
      keep.reserve(g.idx.size());
      for (size_t i = 0; i < g.idx.size(); i += 3) {
        const uint32_t a = g.idx[i], b = g.idx[i + 1], c = g.idx[i + 2];
        if (a == b || a == c || b == c) continue;
        keep.insert(keep.end(), {a, b, c});
      }
      g.idx.swap(keep);
    }
    if (g.t.empty()) build_tangents(g, nv);
    s->geos.push_back(std::move(g));
    const shb_host_scene::Mat& M = s->mats[(size_t)mat];
    if (M.emission > 0.0f) {
      shb_light_desc L{};
      L.type = SHB_LIGHT_AREA;
      L.material_index = mat;
      L.geometry_index = (int32_t)s->geos.size() - 1;
      L.area = surface_area(s->geos.back());
      L.intensity = M.emission;
      L.color[0] = L.color[1] = L.color[2] = 1.0f;
      L.direction[2] = -1.0f;
      L.cos_inner_cone = 1.0f;
      L.cos_outer_cone = 0.70710678118654752440f;
      s->lights.push_back(L);
    }
    return true;
  }

  bool fail(const std::string& e) {
    if (err.empty()) err = e;
    return false;
  }

  void light(const Json& l, const float xf[12]) {
    shb_light_desc L{};
    L.type = SHB_LIGHT_POINT;
    L.color[0] = L.color[1] = L.color[2] = 1.0f;
    L.intensity = 1.0f;
    L.cos_inner_cone = 1.0f;
    L.cos_outer_cone = 0.70710678118654752440f;
    L.material_index = L.geometry_index = -1;
    for (int r = 0; r < 3; ++r) L.position[r] = xf[r * 4 + 3];
    float Lm[9], R[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) Lm[r * 3 + c] = xf[r * 4 + c];
    polar_rotation(Lm, R);
    float d[3] = {-R[2], -R[5], -R[8]};
    const float len_sq = d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]);
    if (len_sq > 1e-8f && std::isfinite(len_sq)) {
      const float n = std::sqrt(len_sq);
      for (float& x : d) x /= n;
    } else {
      d[0] = d[1] = 0.f;
      d[2] = -1.f;
    }
    std::memcpy(L.direction, d, sizeof(d));
    const Json* t = l.get("type");
    if (t && t->kind == Json::Str) {
      if (t->str == "directional") L.type = SHB_LIGHT_DIRECTIONAL;
      else if (t->str == "spot") L.type = SHB_LIGHT_SPOT;
    }
    const Json* c = l.get("color");
    if (c && c->kind == Json::Arr && c->arr.size() == 3)
      for (int k = 0; k < 3; ++k) L.color[k] = to_f32(c->arr[k].num);
    L.intensity = to_f32(l.number("intensity", 1.0));
    const Json* sp = l.get("spot");
    if (L.type == SHB_LIGHT_SPOT && sp) {
      if (sp->get("innerConeAngle")) L.cos_inner_cone = std::cos(to_f32(sp->number("innerConeAngle", 0)));
      if (sp->get("outerConeAngle")) L.cos_outer_cone = std::cos(to_f32(sp->number("outerConeAngle", 0)));
    }
    s->lights.push_back(L);
  }

  bool node(int idx, const float parent[12], int depth) {
    const Json* n = arr_at(m.j, "nodes", idx);
    if (!n || depth > 1024) return fail("bad node index");
    float local[12], xf[12];
    node_local(*n, local);
    compose(parent, local, xf);
    const int mesh = n->integer("mesh", -1);
    if (mesh >= 0) {
      const Json* me = arr_at(m.j, "meshes", mesh);
      const Json* prims = me ? me->get("primitives") : nullptr;
      if (!prims || prims->kind != Json::Arr) return fail("bad mesh");
      for (const Json& pr : prims->arr)
        if (!primitive(pr, xf)) return false;
    }
    const Json* ext = n->get("extensions");
    const Json* kl = ext ? ext->get("KHR_lights_punctual") : nullptr;
    if (kl && kl->get("light")) {
      const int li = kl->integer("light", -1);
      const Json* mext = m.j.get("extensions");
      const Json* mk = mext ? mext->get("KHR_lights_punctual") : nullptr;
      const Json* arr = mk ? mk->get("lights") : nullptr;
      if (arr && arr->kind == Json::Arr && li >= 0 && (size_t)li < arr->arr.size() &&
          arr->arr[(size_t)li].kind == Json::Obj)
        light(arr->arr[(size_t)li], xf);
    }
    const Json* ch = n->get("children");
    if (ch && ch->kind == Json::Arr)
      for (const Json& c : ch->arr)
        if (!node(c.kind == Json::Num ? Json::to_index(c.num, -1) : -1, xf, depth + 1)) return false;
    return true;
  }

  bool texture(int tex, shb_host_scene::Mat& M) {
    const Json* t = arr_at(m.j, "textures", tex);
    if (!t) return true;
    const Json* img = arr_at(m.j, "images", t->integer("source", -1));
    if (!img) return true;
    std::vector<uint8_t> bytes;
    const Json* uri = img->get("uri");
    if (uri && uri->kind == Json::Str) {
      if (!load_uri(uri->str, m.dir, bytes, err)) return false;
      if (uri->str.rfind("data:", 0) != 0)
        M.albedo_file = (!uri->str.empty() && uri->str[0] == '/') ? uri->str : m.dir + uri_decode(uri->str);
    } else if (img->get("bufferView")) {
      const Json* bv = arr_at(m.j, "bufferViews", img->integer("bufferView", -1));
      const int b = bv ? bv->integer("buffer", -1) : -1;
      if (b < 0 || (size_t)b >= m.buffers.size()) return fail("bad image bufferView");
      size_t off = 0, len = 0;
      if (!size_field(*bv, "byteOffset", off) || !size_field(*bv, "byteLength", len) ||
          off > m.buffers[b].size() || len > m.buffers[b].size() - off)
        return fail("image exceeds its buffer");
      bytes.assign(m.buffers[b].begin() + off, m.buffers[b].begin() + off + len);
    } else {
      return true;
    }
    if (bytes.size() >= 2 && bytes[0] == 0xFF && bytes[1] == 0xD8) return shb::decode_jpeg(bytes, M.px, M.w, M.h, M.c, err);
    return decode_png(bytes, M.px, M.w, M.h, M.c, err);
  }

  bool materials() {
    const Json* mats = m.j.get("materials");
    if (!mats || mats->kind != Json::Arr || mats->arr.empty()) {
      shb_host_scene::Mat M;
      M.w = M.h = 1;
      M.c = 4;
      M.px = {255, 255, 255, 255};
      s->mats.push_back(M);
      return true;
    }
    for (const Json& gm : mats->arr) {
      shb_host_scene::Mat M;
      const Json* nm = gm.get("name");
      if (nm && nm->kind == Json::Str) M.name = nm->str;
      const Json* ext = gm.get("extensions");
      const Json* es = ext ? ext->get("KHR_materials_emissive_strength") : nullptr;
      if (es && es->get("emissiveStrength")) M.emission = to_f32(es->number("emissiveStrength", 0.0));
      const Json* pbr = gm.get("pbrMetallicRoughness");
      const Json* bct = pbr ? pbr->get("baseColorTexture") : nullptr;
      if (bct && !texture(bct->integer("index", -1), M)) return false;
      if (M.px.empty()) {
        M.w = M.h = 1;
        M.c = 4;
        const Json* f = pbr ? pbr->get("baseColorFactor") : nullptr;
        if (f && f->kind == Json::Arr && f->arr.size() == 4) {
          M.px = {linear_to_srgb(to_f32(f->arr[0].num)), linear_to_srgb(to_f32(f->arr[1].num)),
                  linear_to_srgb(to_f32(f->arr[2].num)),
                  (uint8_t)std::rint(std::min(std::max(f->arr[3].num, 0.0), 1.0) * 255.0)};
        } else {
          M.px = {255, 255, 255, 255};
        }
      }
      s->mats.push_back(std::move(M));
    }
    return true;
  }

  bool load(const std::string& path) {
    const size_t slash = path.find_last_of('/');
    m.dir = slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
    std::vector<uint8_t> file;
    if (!read_file(path, file)) return fail("cannot read " + path);
    std::string json;
    std::vector<uint8_t> bin;
    bool glb = file.size() >= 12 && std::memcmp(file.data(), "glTF", 4) == 0;
    if (glb) {
      size_t i = 12;
      while (i + 8 <= file.size()) {
        uint32_t len, type;
        std::memcpy(&len, &file[i], 4);
        std::memcpy(&type, &file[i + 4], 4);
        if (i + 8 + (size_t)len > file.size()) return fail("truncated GLB chunk");
        if (type == 0x4E4F534Au) json.assign(reinterpret_cast<const char*>(&file[i + 8]), len);
        else if (type == 0x004E4942u) bin.assign(file.begin() + (long)i + 8, file.begin() + (long)(i + 8 + len));
        i += 8 + ((size_t)len + 3) / 4 * 4;
      }
    } else {
      json.assign(file.begin(), file.end());
    }
    Parser p{json.data(), json.data() + json.size(), ""};
    if (!p.value(m.j, 0) || m.j.kind != Json::Obj) return fail("glTF JSON: " + (p.err.empty() ? "not an object" : p.err));
    const Json* bufs = m.j.get("buffers");
    if (bufs && bufs->kind == Json::Arr) {
      for (size_t b = 0; b < bufs->arr.size(); ++b) {
        const Json* uri = bufs->arr[b].get("uri");
        std::vector<uint8_t> data;
        if (uri && uri->kind == Json::Str) {
          if (!load_uri(uri->str, m.dir, data, err)) return false;
        } else if (glb && b == 0) {
          data = bin;
        } else {
          return fail("buffer without data");
        }
        m.buffers.push_back(std::move(data));
      }
    }
    if (!materials()) return false;
    const Json* scenes = m.j.get("scenes");
    const int def = m.j.integer("scene", -1);
    const Json* sc = arr_at(m.j, "scenes", def > -1 ? def : 0);
    if (!scenes || !sc) return fail("no scene");
    const float I[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    const Json* nodes = sc->get("nodes");
    if (nodes && nodes->kind == Json::Arr)
      for (const Json& n : nodes->arr)
        if (!node(n.kind == Json::Num ? Json::to_index(n.num, -1) : -1, I, 0)) return false;
    return true;
  }
};

// ------------------------------------------------------------- writer -----

// SRGBToLinear (src/colorspace.h:10-14)
float srgb_to_linear(uint8_t x) {
  float v = x / 255.0f;
  if (v <= 0.04045f) return v / 12.92f;
  return std::pow((v + 0.055f) / 1.055f, 2.4f);
}

std::string jstr(const std::string& s) {
  std::string o = "\"";
  for (unsigned char c : s) {
    if (c == '"' || c == '\\') {
      o += '\\';
      o += (char)c;
    } else if (c < 0x20) {
      char b[8];
      std::snprintf(b, sizeof(b), "\\u%04x", c);
      o += b;
    } else {
      o += (char)c;
    }
  }
  return o + "\"";
}

std::string jnum(double v) {
  if (!std::isfinite(v)) v = 0.0;
  char b[32];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

// Shoemake's rotation-matrix -> quaternion (x, y, z, w), row-major m.
void quat_from_matrix(const float m[9], float q[4]) {
  const float tr = m[0] + m[4] + m[8];
  if (tr > 0.0f) {
    float t = std::sqrt(tr + 1.0f);
    q[3] = 0.5f * t;
    t = 0.5f / t;
    q[0] = (m[7] - m[5]) * t;
    q[1] = (m[2] - m[6]) * t;
    q[2] = (m[3] - m[1]) * t;
  } else {
    int i = 0;
    if (m[4] > m[0]) i = 1;
    if (m[8] > m[i * 4]) i = 2;
    const int j = (i + 1) % 3, k = (j + 1) % 3;
    float t = std::sqrt(m[i * 4] - m[j * 4] - m[k * 4] + 1.0f);
    q[i] = 0.5f * t;
    t = 0.5f / t;
    q[3] = (m[k * 3 + j] - m[j * 3 + k]) * t;
    q[j] = (m[j * 3 + i] + m[i * 3 + j]) * t;
    q[k] = (m[k * 3 + i] + m[i * 3 + k]) * t;
  }
}

void normalize3(float v[3]) {
  const float n = std::sqrt(v[0] * v[0] + (v[1] * v[1] + v[2] * v[2]));
  if (n > 0.0f)
    for (int k = 0; k < 3; ++k) v[k] /= n;
}
void cross3(const float a[3], const float b[3], float o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

std::string file_name(const std::string& p) {
  const size_t s = p.find_last_of('/');
  return s == std::string::npos ? p : p.substr(s + 1);
}

bool copy_file(const std::string& from, const std::string& to) {
  if (from == to) return true;
  std::vector<uint8_t> d;
  if (!read_file(from, d)) return false;
  std::ofstream f(to, std::ios::binary | std::ios::trunc);
  f.write(reinterpret_cast<const char*>(d.data()), (std::streamsize)d.size());
  return (bool)f;
}

// SaveScene (src/saver.cpp:423-781): one buffer in <stem>.bin beside the
// .gltf; per geometry a mesh of one triangle primitive (POSITION with
// min/max, NORMAL, TANGENT, TEXCOORD_0, TEXCOORD_1, u32 indices) and a node
// with its matrix; materials as baseColorFactor (1x1 albedo, linear) or a
// copied albedo image; non-area lights as KHR_lights_punctual nodes whose
// -Z axis is the light direction.  Like the reference, emission strength is
// not written.
bool save_gltf(const shb_scene_desc& sc, const char* const* names, const char* const* files, const std::string& path,
               std::string& err) {
  const size_t slash = path.find_last_of('/');
  const std::string dir = slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
  std::string stem = file_name(path);
  const size_t dot = stem.find_last_of('.');
  if (dot != std::string::npos && dot > 0) stem = stem.substr(0, dot);
  std::vector<uint8_t> bin;
  std::vector<std::string> views, accessors;
  auto add_view = [&](const void* data, size_t size, size_t stride, int target) {
    while (bin.size() % 4) bin.push_back(0);
    const size_t off = bin.size();
    const uint8_t* b = static_cast<const uint8_t*>(data);
    bin.insert(bin.end(), b, b + size);
    std::string v = "{\"buffer\":0,\"byteOffset\":" + std::to_string(off) + ",\"byteLength\":" + std::to_string(size);
    if (stride) v += ",\"byteStride\":" + std::to_string(stride);
    v += ",\"target\":" + std::to_string(target) + "}";
    views.push_back(v);
    return (int)views.size() - 1;
  };
  auto add_acc = [&](int view, int ctype, size_t count, const char* type, const std::string& extra) {
    accessors.push_back("{\"bufferView\":" + std::to_string(view) + ",\"byteOffset\":0,\"componentType\":" +
                        std::to_string(ctype) + ",\"count\":" + std::to_string(count) + ",\"type\":\"" + type +
                        "\"" + extra + "}");
    return (int)accessors.size() - 1;
  };
  // materials
  std::vector<std::string> mats, images, textures;
  std::map<std::string, int> tex_of;
  for (uint32_t m = 0; m < sc.material_count; ++m) {
    const shb_material_desc& md = sc.materials[m];
    std::string j = "{\"name\":" + jstr(names && names[m] ? names[m] : "") + ",\"pbrMetallicRoughness\":{";
    const char* f = files ? files[m] : nullptr;
    if (f && *f) {
      const std::string fn = file_name(f);
      auto it = tex_of.find(fn);
      if (it == tex_of.end()) {
        if (!copy_file(f, dir + fn)) {
          err = std::string("Failed to copy file from ") + f + " to " + dir + fn;
          return false;
        }
        images.push_back("{\"uri\":" + jstr(fn) + "}");
        textures.push_back("{\"source\":" + std::to_string(images.size() - 1) + "}");
        it = tex_of.emplace(fn, (int)textures.size() - 1).first;
      }
      j += "\"baseColorTexture\":{\"index\":" + std::to_string(it->second) + "}";
    } else if (md.albedo_width == 1 && md.albedo_height == 1 && md.albedo_pixels &&
               md.albedo_channels >= 4) {
      j += "\"baseColorFactor\":[" + jnum(srgb_to_linear(md.albedo_pixels[0])) + "," +
           jnum(srgb_to_linear(md.albedo_pixels[1])) + "," + jnum(srgb_to_linear(md.albedo_pixels[2])) + "," +
           jnum(md.albedo_pixels[3] / 255.0f) + "]";
    }
    mats.push_back(j + "}}");
  }
  std::vector<std::string> meshes, nodes;
  std::vector<int> roots;
  for (uint32_t gi = 0; gi < sc.geometry_count; ++gi) {
    const shb_geometry_desc& g = sc.geometries[gi];
    const size_t nv = g.vertex_count;
    std::string attrs;
    {
      double mn[3] = {1e9, 1e9, 1e9}, mx[3] = {-1e9, -1e9, -1e9};
      for (size_t v = 0; v < nv; ++v)
        for (int k = 0; k < 3; ++k) {
          mn[k] = std::min(mn[k], (double)g.vertices[3 * v + k]);
          mx[k] = std::max(mx[k], (double)g.vertices[3 * v + k]);
        }
      const int view = add_view(g.vertices, nv * 12, 12, 34962);
      attrs = "\"POSITION\":" + std::to_string(add_acc(view, 5126, nv, "VEC3",
                                                        ",\"min\":[" + jnum(mn[0]) + "," + jnum(mn[1]) + "," +
                                                            jnum(mn[2]) + "],\"max\":[" + jnum(mx[0]) + "," +
                                                            jnum(mx[1]) + "," + jnum(mx[2]) + "]"));
    }
    if (g.normals) attrs += ",\"NORMAL\":" + std::to_string(add_acc(add_view(g.normals, nv * 12, 12, 34962), 5126,
                                                                      nv, "VEC3", ""));
    if (g.tangents) attrs += ",\"TANGENT\":" + std::to_string(add_acc(add_view(g.tangents, nv * 16, 16, 34962),
                                                                        5126, nv, "VEC4", ""));
    if (g.texture_uvs) attrs += ",\"TEXCOORD_0\":" + std::to_string(add_acc(add_view(g.texture_uvs, nv * 8, 8, 34962),
                                                                              5126, nv, "VEC2", ""));
    if (g.lightmap_uvs)
      attrs += ",\"TEXCOORD_1\":" + std::to_string(add_acc(add_view(g.lightmap_uvs, nv * 8, 8, 34962), 5126, nv,
                                                             "VEC2", ""));
    const int iacc = add_acc(add_view(g.indices, (size_t)g.index_count * 4, 0, 34963), 5125, g.index_count,
                             "SCALAR", "");
    meshes.push_back("{\"primitives\":[{\"mode\":4,\"material\":" + std::to_string(g.material_id) +
                     ",\"attributes\":{" + attrs + "},\"indices\":" + std::to_string(iacc) + "}]}");
    std::string mat = "[";
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r) {
        const double v = r < 3 ? g.transform[r * 4 + c] : (c == 3 ? 1.0 : 0.0);
        mat += jnum(v) + (c == 3 && r == 3 ? "]" : ",");
      }
    nodes.push_back("{\"mesh\":" + std::to_string(meshes.size() - 1) + ",\"matrix\":" + mat + "}");
    roots.push_back((int)nodes.size() - 1);
  }
  std::vector<std::string> lights;
  for (uint32_t li = 0; li < sc.light_count; ++li) {
    const shb_light_desc& L = sc.lights[li];
    if (L.type == SHB_LIGHT_AREA) continue;
    const int k = (int)lights.size();
    std::string lj = "{\"color\":[" + jnum(L.color[0]) + "," + jnum(L.color[1]) + "," + jnum(L.color[2]) +
                     "],\"intensity\":" + jnum(L.intensity);
    const char* type = L.type == SHB_LIGHT_DIRECTIONAL ? "directional" : L.type == SHB_LIGHT_SPOT ? "spot" : "point";
    if (L.type == SHB_LIGHT_SPOT) {
      auto safe_acos = [](float c) -> double {
        if (c >= 1.0f) return 0.0;
        if (c <= -1.0f) return 3.14159265358979323846;
        return std::acos(c);
      };
      lj += ",\"spot\":{\"innerConeAngle\":" + jnum(safe_acos(L.cos_inner_cone)) +
            ",\"outerConeAngle\":" + jnum(safe_acos(L.cos_outer_cone)) + "}";
    }
    lj += std::string(",\"type\":\"") + type + "\",\"name\":\"Light_" + std::to_string(k) + "\"}";
    lights.push_back(lj);
    std::string nj = "{\"name\":\"LightNode_" + std::to_string(k) + "\",\"translation\":[" +
                     jnum(L.position[0]) + "," + jnum(L.position[1]) + "," + jnum(L.position[2]) + "]";
    if (L.type == SHB_LIGHT_DIRECTIONAL || L.type == SHB_LIGHT_SPOT) {
      float Z[3] = {-L.direction[0], -L.direction[1], -L.direction[2]};
      normalize3(Z);
      float up[3] = {0.f, 1.f, 0.f};
      if (std::fabs(Z[1]) > 0.99f) {
        up[0] = 1.f;
        up[1] = 0.f;
      }
      float X[3], Y[3];
      cross3(up, Z, X);
      normalize3(X);
      cross3(Z, X, Y);
      normalize3(Y);
      const float m[9] = {X[0], Y[0], Z[0], X[1], Y[1], Z[1], X[2], Y[2], Z[2]};
      float q[4];
      quat_from_matrix(m, q);
      nj += ",\"rotation\":[" + jnum(q[0]) + "," + jnum(q[1]) + "," + jnum(q[2]) + "," + jnum(q[3]) + "]";
    }
    nj += ",\"extensions\":{\"KHR_lights_punctual\":{\"light\":" + std::to_string(k) + "}}}";
    nodes.push_back(nj);
    roots.push_back((int)nodes.size() - 1);
  }
  auto join = [](const std::vector<std::string>& v) {
    std::string o;
    for (size_t i = 0; i < v.size(); ++i) o += (i ? "," : "") + v[i];
    return o;
  };
  std::string j = "{\"asset\":{\"generator\":\"sh_baker\",\"version\":\"2.0\"}";
  if (!lights.empty())
    j += ",\"extensionsUsed\":[\"KHR_lights_punctual\"],\"extensions\":{\"KHR_lights_punctual\":{\"lights\":[" +
         join(lights) + "]}}";
  j += ",\"buffers\":[{\"byteLength\":" + std::to_string(bin.size()) + ",\"uri\":" + jstr(stem + ".bin") + "}]";
  j += ",\"bufferViews\":[" + join(views) + "],\"accessors\":[" + join(accessors) + "]";
  j += ",\"materials\":[" + join(mats) + "],\"meshes\":[" + join(meshes) + "],\"nodes\":[" + join(nodes) + "]";
  if (!images.empty()) j += ",\"images\":[" + join(images) + "],\"textures\":[" + join(textures) + "]";
  std::string rs;
  for (size_t i = 0; i < roots.size(); ++i) rs += (i ? "," : "") + std::to_string(roots[i]);
  j += ",\"scenes\":[{\"nodes\":[" + rs + "]}],\"scene\":0}";
  std::ofstream fb(dir + stem + ".bin", std::ios::binary | std::ios::trunc);
  fb.write(reinterpret_cast<const char*>(bin.data()), (std::streamsize)bin.size());
  std::ofstream fj(path, std::ios::trunc);
  fj << j;
  if (!fb || !fj) {
    err = "cannot write " + path;
    return false;
  }
  return true;
}

}  // namespace
}  // namespace shb

extern "C" {

shb_status shb_save_gltf(const shb_scene_desc* scene, const char* const* material_names,
                         const char* const* albedo_files, const char* path) {
  return ::shb::guarded("shb_save_gltf", [&]() -> shb_status {
    if (!scene || !path || !*path) {
      shb::set_error("NULL argument");
      return SHB_ERR_INVALID_ARG;
    }
    std::string err;
    if (!shb::save_gltf(*scene, material_names, albedo_files, path, err)) {
      shb::set_error("SaveScene: " + err);
      return SHB_ERR_INVALID_ARG;
    }
    return SHB_OK;
  });
}

shb_status shb_host_scene_material_info(const shb_host_scene* s, int32_t material, const char** name,
                                        const char** albedo_file) {
  return ::shb::guarded("shb_host_scene_material_info", [&]() -> shb_status {
    if (!s || material < 0 || (size_t)material >= s->mats.size()) {
      shb::set_error("bad material index");
      return SHB_ERR_INVALID_ARG;
    }
    if (name) *name = s->mats[(size_t)material].name.c_str();
    if (albedo_file) {
      const std::string& f = s->mats[(size_t)material].albedo_file;
      *albedo_file = f.empty() ? nullptr : f.c_str();
    }
    return SHB_OK;
  });
}


shb_status shb_load_gltf(const char* path, shb_host_scene** out) {
  return ::shb::guarded("shb_load_gltf", [&]() -> shb_status {
    if (!path || !out) {
      shb::set_error("NULL argument");
      return SHB_ERR_INVALID_ARG;
    }
    *out = nullptr;
    std::unique_ptr<shb_host_scene> s(new shb_host_scene());
    shb::Loader L;
    L.s = s.get();
    if (!L.load(path)) {
      shb::set_error("LoadScene: " + L.err);
      return SHB_ERR_INVALID_ARG;
    }
    s->finish();
    *out = s.release();
    return SHB_OK;
  });
}

const shb_scene_desc* shb_host_scene_desc(const shb_host_scene* s) { return s ? &s->desc : nullptr; }

shb_status shb_host_scene_destroy(shb_host_scene* s) {
  return ::shb::guarded("shb_host_scene_destroy", [&]() -> shb_status {
    delete s;
    return SHB_OK;
  });
}

}  // extern "C"
