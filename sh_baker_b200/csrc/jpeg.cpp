// jpeg.cpp - JPEG base-colour textures for the glTF loader.  The reference
// reads every texture through tinygltf's image loader over stb_image
// (src/loader.cpp:415-432); this is an own decoder of Huffman-coded JPEG
// (ITU-T T.81 baseline, extended 8-bit and progressive: SOF0 / SOF1 / SOF2)
// with restart intervals, 1 or 3 components and any sampling factors up to
// 4x4:
//   - Huffman tables as canonical codes (T.81 annex C), DC prediction per
//     component, AC run/size symbols with EOB and ZRL (annex F.2.2);
//   - dequantisation, a separable floating-point inverse DCT (the
//     definition of annex A.3.3), level shift and clamping;
//   - chroma upsampled with the triangle filter libjpeg and stb_image call
//     "fancy" (3/4 of the nearer and 1/4 of the farther sample per axis) for
//     2x sampling, nearest sample otherwise;
//   - YCbCr to RGB with the JFIF coefficients (JFIF 1.02).
// Output is 8-bit RGB, grey replicated, which is what stb_image returns for
// three requested channels.  Pixel values can differ from libjpeg's or
// stb_image's by a level or two: those use integer inverse DCTs.
// Progressive files (SOF2, annex G: spectral selection and successive
// approximation, DC and AC first and refinement scans, end-of-band runs)
// keep every block's coefficients across scans and are transformed once
// all scans are read.  Lossless and arithmetic-coded files are rejected.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr int kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                             12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                             35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                             58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

struct Huff {
  bool set = false;
  int maxcode[18];   // largest code of each length (-1: none)
  int valptr[17];    // index of the first symbol of each length
  int mincode[17];
  uint8_t vals[256];
};

struct Comp {
  int id = 0, h = 1, v = 1, tq = 0, td = 0, ta = 0;
  int bw = 0, bh = 0;  // blocks per line / column, padded to whole MCUs
  std::vector<uint8_t> px;  // bw*8 x bh*8 samples
  std::vector<int> coef;    // progressive: 64 coefficients per block, zigzag order
  int pred = 0;
};

struct Reader {
  const uint8_t* p;
  size_t n, i = 0;
  uint32_t bits = 0;
  int nbits = 0;
  bool marker = false;  // a marker was reached inside entropy-coded data
  int bit() {
    if (nbits == 0) {
      uint8_t b = 0;
      if (!marker && i < n) {
        b = p[i];
        if (b == 0xFF) {
          uint8_t nx = i + 1 < n ? p[i + 1] : 0;
          if (nx == 0x00) {
            i += 2;
          } else {
            marker = true;  // leave the marker for the caller; feed zeros
            b = 0;
          }
        } else {
          i++;
        }
      }
      bits = b;
      nbits = 8;
    }
    nbits--;
    return (bits >> nbits) & 1;
  }
  int receive(int s) {
    int v = 0;
    for (int k = 0; k < s; ++k) v = (v << 1) | bit();
    return v;
  }
  void reset() {
    nbits = 0;
    marker = false;
  }
};

int extend(int v, int s) { return s == 0 ? 0 : (v < (1 << (s - 1)) ? v - (1 << s) + 1 : v); }

int decode_huff(Reader& r, const Huff& h) {
  int code = 0;
  for (int l = 1; l <= 16; ++l) {
    code = (code << 1) | r.bit();
    if (h.maxcode[l] >= 0 && code <= h.maxcode[l]) return h.vals[h.valptr[l] + code - h.mincode[l]];
  }
  return -1;
}

void idct8x8(const int coef[64], const uint16_t* q, uint8_t* out, int stride) {
  static double C[8][8];
  static bool init = false;
  if (!init) {
    for (int x = 0; x < 8; ++x)
      for (int u = 0; u < 8; ++u) C[x][u] = (u == 0 ? std::sqrt(0.5) : 1.0) * std::cos((2 * x + 1) * u * M_PI / 16.0);
    init = true;
  }
  double F[64], T[64];
  for (int k = 0; k < 64; ++k) F[kZigzag[k]] = (double)coef[k] * q[k];
  for (int y = 0; y < 8; ++y)  // rows: T[v][x] = 1/2 sum_u C[x][u] F[v][u]
    for (int x = 0; x < 8; ++x) {
      double s = 0;
      for (int u = 0; u < 8; ++u) s += C[x][u] * F[y * 8 + u];
      T[y * 8 + x] = 0.5 * s;
    }
  for (int x = 0; x < 8; ++x)
    for (int y = 0; y < 8; ++y) {
      double s = 0;
      for (int v = 0; v < 8; ++v) s += C[y][v] * T[v * 8 + x];
      int pv = (int)std::lround(0.5 * s + 128.0);
      out[y * stride + x] = (uint8_t)(pv < 0 ? 0 : (pv > 255 ? 255 : pv));
    }
}

uint8_t clamp8(double v) {
  long r = std::lround(v);
  return (uint8_t)(r < 0 ? 0 : (r > 255 ? 255 : r));
}

// Sample of component c at output pixel (x, y): the triangle filter for a
// factor-2 axis, the covering sample otherwise.
struct Upsampler {
  const Comp& c;
  int sx, sy;  // output pixels per component sample on each axis
  int sample(int x, int y) const { return c.px[(size_t)y * c.bw * 8 + x]; }
  double at(int X, int Y, int W, int H) const {
    const int cw = (W + sx - 1) / sx, ch = (H + sy - 1) / sy;
    auto axis = [](int P, int s, int n, int& a, int& b, double& wa) {
      if (s != 2) {
        a = b = P / s;
        wa = 1.0;
        return;
      }
      a = P >> 1;
      b = (P & 1) ? a + 1 : a - 1;  // the farther neighbour on the side of P
      if (b < 0) b = 0;
      if (b > n - 1) b = n - 1;
      wa = 0.75;
    };
    int xa, xb, ya, yb;
    double wx, wy;
    axis(X, sx, cw, xa, xb, wx);
    axis(Y, sy, ch, ya, yb, wy);
    return wy * (wx * sample(xa, ya) + (1 - wx) * sample(xb, ya)) +
           (1 - wy) * (wx * sample(xa, yb) + (1 - wx) * sample(xb, yb));
  }
};

}  // namespace

namespace shb {

// JPEG -> 8-bit RGB (C = 3).  Returns false with `err` set on unsupported or
// damaged files.
bool decode_jpeg(const std::vector<uint8_t>& f, std::vector<uint8_t>& out, uint32_t& W, uint32_t& H, uint32_t& C,
                 std::string& err) {
  if (f.size() < 4 || f[0] != 0xFF || f[1] != 0xD8) {
    err = "not a JPEG";
    return false;
  }
  uint16_t q[4][64];
  bool qset[4] = {false, false, false, false};
  Huff dc[4], ac[4];
  std::vector<Comp> comps;
  int width = 0, height = 0, hmax = 1, vmax = 1, restart = 0;
  bool frame = false, scanned = false, progressive = false;
  size_t i = 2;
  auto u16 = [&](size_t k) { return (int)f[k] << 8 | f[k + 1]; };
  while (i + 4 <= f.size()) {
    if (f[i] != 0xFF) {
      err = "JPEG: marker expected";
      return false;
    }
    const uint8_t mk = f[i + 1];
    if (mk == 0xFF) {  // fill byte
      i++;
      continue;
    }
    if (mk == 0xD9) break;  // EOI
    const int len = u16(i + 2);
    if (len < 2 || i + 2 + (size_t)len > f.size()) {
      err = "JPEG: truncated segment";
      return false;
    }
    const size_t s = i + 4, e = i + 2 + len;
    // the fixed part each segment reads before its own checks
    const size_t need = mk == 0xC0 || mk == 0xC1 || mk == 0xC2 ? 6 : (mk == 0xDD ? 2 : (mk == 0xDA ? 1 : 0));
    if (s + need > e) {
      err = "JPEG: truncated segment";
      return false;
    }
    if (mk == 0xDB) {  // DQT
      size_t k = s;
      while (k < e) {
        const int pq = f[k] >> 4, tq = f[k] & 15;
        k++;
        if (tq > 3 || k + (pq ? 128 : 64) > e) {
          err = "JPEG: bad quantisation table";
          return false;
        }
        for (int z = 0; z < 64; ++z) q[tq][z] = pq ? (uint16_t)u16(k + 2 * z) : f[k + z];
        k += pq ? 128 : 64;
        qset[tq] = true;
      }
    } else if (mk == 0xC4) {  // DHT
      size_t k = s;
      while (k + 17 <= e) {
        const int tc = f[k] >> 4, th = f[k] & 15;
        if (tc > 1 || th > 3) {
          err = "JPEG: bad Huffman table";
          return false;
        }
        Huff& h = tc ? ac[th] : dc[th];
        int counts[17], total = 0;
        for (int l = 1; l <= 16; ++l) total += counts[l] = f[k + l];
        if (total > 256 || k + 17 + total > e) {
          err = "JPEG: bad Huffman table";
          return false;
        }
        std::memcpy(h.vals, &f[k + 17], (size_t)total);
        int code = 0, idx = 0;
        for (int l = 1; l <= 16; ++l) {
          h.valptr[l] = idx;
          h.mincode[l] = code;
          code += counts[l];
          idx += counts[l];
          h.maxcode[l] = counts[l] ? code - 1 : -1;
          code <<= 1;
        }
        h.set = true;
        k += 17 + (size_t)total;
      }
    } else if (mk == 0xC0 || mk == 0xC1 || mk == 0xC2) {  // SOF0 / SOF1 / SOF2
      if (frame) {
        err = "JPEG: more than one frame";
        return false;
      }
      progressive = mk == 0xC2;
      if (f[s] != 8) {
        err = "JPEG: only 8-bit samples are supported";
        return false;
      }
      height = u16(s + 1);
      width = u16(s + 3);
      const int nc = f[s + 5];
      if ((nc != 1 && nc != 3) || width <= 0 || height <= 0 || s + 6 + 3 * (size_t)nc > e) {
        err = "JPEG: unsupported frame (1 or 3 components, nonzero size)";
        return false;
      }
      // the frame header alone sizes the sample (and coefficient) planes
      if ((int64_t)width * height > (1 << 28)) {
        err = "JPEG: images above 2^28 pixels are not read";
        return false;
      }
      comps.resize((size_t)nc);
      for (int c = 0; c < nc; ++c) {
        Comp& cp = comps[(size_t)c];
        cp.id = f[s + 6 + 3 * c];
        cp.h = f[s + 7 + 3 * c] >> 4;
        cp.v = f[s + 7 + 3 * c] & 15;
        cp.tq = f[s + 8 + 3 * c] & 3;
        if (cp.h < 1 || cp.h > 4 || cp.v < 1 || cp.v > 4) {
          err = "JPEG: bad sampling factors";
          return false;
        }
        hmax = std::max(hmax, cp.h);
        vmax = std::max(vmax, cp.v);
      }
      const int mcux = (width + 8 * hmax - 1) / (8 * hmax), mcuy = (height + 8 * vmax - 1) / (8 * vmax);
      for (Comp& cp : comps) {
        cp.bw = mcux * cp.h;
        cp.bh = mcuy * cp.v;
        cp.px.assign((size_t)cp.bw * 8 * cp.bh * 8, 0);
        if (progressive) cp.coef.assign((size_t)cp.bw * cp.bh * 64, 0);
      }
      frame = true;
    } else if (mk >= 0xC2 && mk <= 0xCF && mk != 0xC4 && mk != 0xC8 && mk != 0xCC) {
      err = "JPEG: only Huffman-coded sequential and progressive 8-bit files are supported";
      return false;
    } else if (mk == 0xDD) {  // DRI
      restart = u16(s);
    } else if (mk == 0xDA) {  // SOS
      if (!frame) {
        err = "JPEG: scan before frame";
        return false;
      }
      const int ns = f[s];
      if (ns < 1 || ns > (int)comps.size() || s + 1 + 2 * (size_t)ns + 3 > e) {
        err = "JPEG: bad scan header";
        return false;
      }
      // spectral selection and successive approximation (T.81 B.2.3): fixed
      // at 0, 63, 0, 0 in sequential files
      const size_t ps = s + 1 + 2 * (size_t)ns;
      const int Ss = f[ps], Se = f[ps + 1], Ah = f[ps + 2] >> 4, Al = f[ps + 2] & 15;
      if (progressive && (Ah > 13 || Al > 13 || (Ss == 0 ? Se != 0 : (Se < Ss || Se > 63 || ns != 1)))) {
        err = "JPEG: bad progressive scan parameters";
        return false;
      }
      // tables a scan decodes with: sequential DC and AC; a progressive DC
      // first scan DC, an AC scan AC, a DC refinement none
      const bool need_dc = !progressive || (Ss == 0 && Ah == 0), need_ac = !progressive || Ss > 0;
      std::vector<Comp*> sc;
      for (int c = 0; c < ns; ++c) {
        const int id = f[s + 1 + 2 * c], t = f[s + 2 + 2 * c];
        Comp* cp = nullptr;
        for (Comp& x : comps)
          if (x.id == id) cp = &x;
        if (!cp || (need_dc && !dc[t >> 4 & 3].set) || (need_ac && !ac[t & 3].set) || !qset[cp->tq]) {
          err = "JPEG: scan names a missing component or table";
          return false;
        }
        cp->td = t >> 4 & 3;
        cp->ta = t & 3;
        cp->pred = 0;
        sc.push_back(cp);
      }
      Reader r{f.data(), f.size(), e};
      const bool single = ns == 1;
      const int mcux = single ? (((width * sc[0]->h + hmax - 1) / hmax) + 7) / 8
                              : (width + 8 * hmax - 1) / (8 * hmax);
      const int mcuy = single ? (((height * sc[0]->v + vmax - 1) / vmax) + 7) / 8
                              : (height + 8 * vmax - 1) / (8 * vmax);
      int coef[64];
      auto block = [&](Comp& cp, int bx, int by) -> bool {
        std::memset(coef, 0, sizeof(coef));
        const int t = decode_huff(r, dc[cp.td]);
        if (t < 0 || t > 11) return false;
        cp.pred += extend(r.receive(t), t);
        coef[0] = cp.pred;
        for (int k = 1; k < 64;) {
          const int rs = decode_huff(r, ac[cp.ta]);
          if (rs < 0) return false;
          const int run = rs >> 4, sz = rs & 15;
          if (sz == 0) {
            if (run != 15) break;  // EOB
            k += 16;               // ZRL
            continue;
          }
          k += run;
          if (k > 63) return false;
          coef[k++] = extend(r.receive(sz), sz);
        }
        idct8x8(coef, q[cp.tq], &cp.px[((size_t)by * 8) * cp.bw * 8 + (size_t)bx * 8], cp.bw * 8);
        return true;
      };
      // Progressive scans (T.81 annex G.1.2) add to the block's stored
      // coefficients; the inverse DCT runs once all scans are read.
      int eobrun = 0;  // blocks left in the current end-of-band run
      auto prog_block = [&](Comp& cp, int bx, int by) -> bool {
        int* z = &cp.coef[((size_t)by * cp.bw + bx) * 64];
        if (Ss == 0) {  // DC: first scan (difference, shifted by Al) or one refinement bit
          if (Ah == 0) {
            const int t = decode_huff(r, dc[cp.td]);
            if (t < 0 || t > 11) return false;
            cp.pred += extend(r.receive(t), t);
            z[0] = cp.pred * (1 << Al);
          } else if (r.bit()) {
            z[0] |= 1 << Al;
          }
          return true;
        }
        if (Ah == 0) {  // AC first scan: run/size symbols, end-of-band runs
          if (eobrun > 0) {
            --eobrun;
            return true;
          }
          for (int k = Ss; k <= Se; ++k) {
            const int rs = decode_huff(r, ac[cp.ta]);
            if (rs < 0) return false;
            const int run = rs >> 4, sz = rs & 15;
            if (sz == 0) {
              if (run < 15) {  // EOB run of 2^run + extra bits blocks, this one included
                eobrun = (1 << run) - 1 + (run ? r.receive(run) : 0);
                break;
              }
              k += 15;  // ZRL: sixteen zeros
              continue;
            }
            k += run;
            if (k > Se) return false;
            z[k] = extend(r.receive(sz), sz) * (1 << Al);
          }
          return true;
        }
        // AC refinement (G.1.2.3): one correction bit for every coefficient
        // already nonzero, new coefficients of magnitude 2^Al placed after
        // `run` coefficients that are still zero
        const int p1 = 1 << Al, m1 = -p1;
        auto correct = [&](int& c) {
          if (r.bit() && (c & p1) == 0) c += c >= 0 ? p1 : m1;
        };
        int k = Ss;
        if (eobrun == 0) {
          for (; k <= Se; ++k) {
            const int rs = decode_huff(r, ac[cp.ta]);
            if (rs < 0) return false;
            int run = rs >> 4;
            const int sz = rs & 15;
            int value = 0;
            if (sz == 0) {
              if (run < 15) {  // EOB run, this block included: its rest is refined below
                eobrun = (1 << run) + (run ? r.receive(run) : 0);
                break;
              }  // else ZRL: pass sixteen zero coefficients
            } else {
              if (sz != 1) return false;
              value = r.bit() ? p1 : m1;
            }
            while (k <= Se) {
              int& c = z[k];
              if (c != 0) {
                correct(c);
              } else {
                if (run == 0) {
                  if (value) c = value;
                  break;
                }
                --run;
              }
              ++k;
            }
            if (k > Se && value) return false;  // no zero coefficient left for the new one
          }
        }
        if (eobrun > 0) {
          for (; k <= Se; ++k)
            if (z[k] != 0) correct(z[k]);
          --eobrun;
        }
        return true;
      };
      auto unit = [&](Comp& cp, int bx, int by) { return progressive ? prog_block(cp, bx, by) : block(cp, bx, by); };
      int todo = restart;
      for (int my = 0; my < mcuy; ++my)
        for (int mx = 0; mx < mcux; ++mx) {
          if (restart && todo == 0) {  // expect RSTn: byte-align and reset predictions
            r.reset();
            while (r.i + 1 < f.size() && !(f[r.i] == 0xFF && f[r.i + 1] >= 0xD0 && f[r.i + 1] <= 0xD7)) r.i++;
            r.i += 2;
            for (Comp* cp : sc) cp->pred = 0;
            eobrun = 0;
            todo = restart;
          }
          bool ok = true;
          if (single) {
            ok = unit(*sc[0], mx, my);
          } else {
            for (Comp* cp : sc)
              for (int v = 0; v < cp->v && ok; ++v)
                for (int h = 0; h < cp->h && ok; ++h) ok = unit(*cp, mx * cp->h + h, my * cp->v + v);
          }
          if (!ok) {
            err = "JPEG: damaged entropy-coded data";
            return false;
          }
          if (restart) todo--;
        }
      // the scan ends at the next marker
      i = r.i;
      while (i + 1 < f.size() && !(f[i] == 0xFF && f[i + 1] != 0x00 && !(f[i + 1] >= 0xD0 && f[i + 1] <= 0xD7))) i++;
      scanned = true;
      continue;
    }
    i = e;
  }
  if (!scanned) {
    err = "JPEG: no image data";
    return false;
  }
  if (progressive)
    for (Comp& cp : comps)
      for (int by = 0; by < cp.bh; ++by)
        for (int bx = 0; bx < cp.bw; ++bx)
          idct8x8(&cp.coef[((size_t)by * cp.bw + bx) * 64], q[cp.tq],
                  &cp.px[((size_t)by * 8) * cp.bw * 8 + (size_t)bx * 8], cp.bw * 8);
  W = (uint32_t)width;
  H = (uint32_t)height;
  C = 3;
  out.assign((size_t)W * H * 3, 0);
  if (comps.size() == 1) {
    const Comp& g = comps[0];
    for (uint32_t y = 0; y < H; ++y)
      for (uint32_t x = 0; x < W; ++x) {
        const uint8_t v = g.px[(size_t)y * g.bw * 8 + x];
        uint8_t* o = &out[3 * ((size_t)y * W + x)];
        o[0] = o[1] = o[2] = v;
      }
    return true;
  }
  Upsampler up[3] = {{comps[0], hmax / comps[0].h, vmax / comps[0].v}, {comps[1], hmax / comps[1].h, vmax / comps[1].v},
                     {comps[2], hmax / comps[2].h, vmax / comps[2].v}};
  for (int c = 0; c < 3; ++c)
    if (hmax % comps[c].h || vmax % comps[c].v) {
      err = "JPEG: sampling factors that do not divide the largest";
      return false;
    }
  for (int Y = 0; Y < height; ++Y)
    for (int X = 0; X < width; ++X) {
      const double y = up[0].at(X, Y, width, height);
      const double cb = up[1].at(X, Y, width, height) - 128.0, cr = up[2].at(X, Y, width, height) - 128.0;
      uint8_t* o = &out[3 * ((size_t)Y * W + X)];
      o[0] = clamp8(y + 1.402 * cr);
      o[1] = clamp8(y - 0.344136 * cb - 0.714136 * cr);
      o[2] = clamp8(y + 1.772 * cb);
    }
  return true;
}

}  // namespace shb
