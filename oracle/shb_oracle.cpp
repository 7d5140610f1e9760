// shb_oracle.cpp - CPU oracle of the SH9 lightmap bake.
//
// TEST INFRASTRUCTURE ONLY: this file is the checker of the CUDA path and the
// timed CPU baseline.  The product never links, imports or calls it.
//
// It restates, step by step, the reference algorithm:
//   rasterizer.cpp:18-33,68-241   Barycentric, RasterizeScene, masks
//   baker.cpp:38-46,70-182,186-304 SampleHemisphereUniform, Trace,
//                                 DownsampleTexture, BakeSHLightMap
//   light.h:28-203, light.cpp:16-293  light radiance, SampleAreaLight, NEE
//   material.cpp:57-92,113-162    GetAlpha/GetAlbedo/GetEmission,
//                                 SampleMaterial, EvalMaterial
//   colorspace.h:10-14            SRGBToLinear
//   sh_coeffs.cpp:27-78           AccumulateRadiance
//   occlusion.cpp:9-107           FindOcclusion hit attributes
//   dilation.cpp:7-73             Dilate<T>
//   scene.cpp:162-207             TransformedVertices/Normals/Tangents
//
// Floating-point order: sums of Eigen expressions are evaluated left to
// right; 3-term dot products follow Eigen's unrolled reduction
// x0*y0 + (x1*y1 + x2*y2).  Built with -ffp-contract=off so no FMA is formed;
// the CUDA path computes the same operations in the same order.
//
// Ray queries use this file's own binned-SAH binary BVH and the watertight
// ray/triangle test of Woop, Benthin and Wald (JCGT 2013); Embree (absent
// here) is not reproducible bit for bit.  Two random streams are offered:
// std::mt19937(12345 + idx) with libstdc++'s distributions, which is the
// stream the reference consumes (baker.cpp:254), and Philox4x32-10 (Salmon
// et al., SC'11) addressed by (seed, texel, sample, path vertex, event, block),
// which is the stream the GPU consumes.  The whole tracer is a template over
// float / double; the double instance is the FP64 oracle.

#include "shb_oracle.h"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <thread>
#include <type_traits>
#include <vector>

namespace {

// ---------------------------------------------------------------- vectors --

template <class R>
struct V2 {
  R x = 0, y = 0;
};
template <class R>
struct V3 {
  R x = 0, y = 0, z = 0;
  R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class R>
struct V4 {
  R x = 0, y = 0, z = 0, w = 0;
};

template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline V3<R>& operator+=(V3<R>& a, V3<R> b) { a = a + b; return a; }
template <class R> inline V3<R> cmul(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
template <class R> inline R sqnorm(V3<R> a) { return dot(a, a); }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline V3<R> normalized(V3<R> a) {
  R n = sqnorm(a);
  if (n > R(0)) return a / std::sqrt(n);
  return a;
}
template <class R> inline R max_coeff(V3<R> a) { return std::max(a.x, std::max(a.y, a.z)); }

template <class R> inline V2<R> operator+(V2<R> a, V2<R> b) { return {a.x + b.x, a.y + b.y}; }
template <class R> inline V2<R> operator-(V2<R> a, V2<R> b) { return {a.x - b.x, a.y - b.y}; }
template <class R> inline V2<R> operator*(R s, V2<R> a) { return {s * a.x, s * a.y}; }
template <class R> inline V2<R> operator*(V2<R> a, R s) { return {a.x * s, a.y * s}; }
template <class R> inline R dot2(V2<R> a, V2<R> b) { return a.x * b.x + a.y * b.y; }

template <class R> inline V4<R> operator+(V4<R> a, V4<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class R> inline V4<R> operator*(V4<R> a, R s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }

// x86 cvttss2si semantics of (int)f, which the reference relies on.
inline int cvt_trunc(float f) {
  if (f >= -2147483648.0f && f < 2147483648.0f) return (int)f;
  return INT_MIN;
}

constexpr double kPi = 3.14159265358979323846;

// --------------------------------------------------------------- scene ----

struct Geo {
  std::vector<V3<float>> vertices, normals;  // object space
  std::vector<V2<float>> texture_uvs, lightmap_uvs;
  std::vector<V4<float>> tangents;
  std::vector<uint32_t> indices;
  int material_id = -1;
  float L[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  float t[3] = {0, 0, 0};
  float Rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::vector<V3<float>> world_vertices, world_normals;
  std::vector<V4<float>> world_tangents;
  uint32_t prim_base = 0;
};

struct Mat {
  std::vector<uint8_t> pixels;
  uint32_t w = 0, h = 0, c = 0;
  float emission = 0.f;
  int use_override = 0;  // adjoint parameter: linear base colour replaces the texture
  float ovr[3] = {0.f, 0.f, 0.f};
};

struct Lgt {
  int type = 0;
  V3<float> position, direction{0, 0, -1}, color{1, 1, 1};
  float intensity = 1.f, cos_inner = 1.f, cos_outer = 0.70710678f, area = 0.f;
  int material = -1, geometry = -1;
};

// Polar-decomposition rotation of a 3x3 (Eigen Transform::rotation()):
// M = U S V^T, rotation = U diag(x,1,1) V^T with x = sign(det U V^T), via a
// cyclic Jacobi eigen solve of M^T M in double.
void polar_rotation(const float Lf[9], float Rout[9]) {
  bool ident = true;
  for (int i = 0; i < 9; ++i) ident &= (Lf[i] == ((i % 4 == 0) ? 1.f : 0.f));
  if (ident) {
    for (int i = 0; i < 9; ++i) Rout[i] = (i % 4 == 0) ? 1.f : 0.f;
    return;
  }
  double M[3][3], A[3][3], V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i][j] = Lf[i * 3 + j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += M[k][i] * M[k][j];
      A[i][j] = s;
    }
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = std::fabs(A[0][1]) + std::fabs(A[0][2]) + std::fabs(A[1][2]);
    if (off < 1e-300) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (std::fabs(A[p][q]) < 1e-300) continue;
        double theta = (A[q][q] - A[p][p]) / (2 * A[p][q]);
        double tt = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(tt * tt + 1), s = tt * c;
        for (int k = 0; k < 3; ++k) {
          double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  // Sort singular values descending (JacobiSVD order).
  double ev[3] = {A[0][0], A[1][1], A[2][2]};
  int ord[3] = {0, 1, 2};
  std::sort(ord, ord + 3, [&](int a, int b) { return ev[a] > ev[b]; });
  double Vs[3][3], U[3][3];
  for (int j = 0; j < 3; ++j) {
    for (int i = 0; i < 3; ++i) Vs[i][j] = V[i][ord[j]];
  }
  for (int j = 0; j < 3; ++j) {
    double col[3];
    for (int i = 0; i < 3; ++i) col[i] = M[i][0] * Vs[0][j] + M[i][1] * Vs[1][j] + M[i][2] * Vs[2][j];
    double n = std::sqrt(col[0] * col[0] + col[1] * col[1] + col[2] * col[2]);
    for (int i = 0; i < 3; ++i) U[i][j] = n > 0 ? col[i] / n : 0.0;
  }
  auto det3 = [](double X[3][3]) {
    return X[0][0] * (X[1][1] * X[2][2] - X[1][2] * X[2][1]) -
           X[0][1] * (X[1][0] * X[2][2] - X[1][2] * X[2][0]) +
           X[0][2] * (X[1][0] * X[2][1] - X[1][1] * X[2][0]);
  };
  double x = (det3(U) * det3(Vs) < 0) ? -1.0 : 1.0;
  for (int i = 0; i < 3; ++i) U[i][0] *= x;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += U[i][k] * Vs[j][k];
      Rout[i * 3 + j] = (float)s;
    }
}

// Eigen 3x3 * vector, coefficient i = m(i,0)*v0 + (m(i,1)*v1 + m(i,2)*v2).
inline V3<float> mat_vec(const float m[9], V3<float> v) {
  return {m[0] * v.x + (m[1] * v.y + m[2] * v.z), m[3] * v.x + (m[4] * v.y + m[5] * v.z),
          m[6] * v.x + (m[7] * v.y + m[8] * v.z)};
}

}  // namespace

struct BvhF;
struct BvhD;

struct oracle_scene {
  std::vector<Geo> geos;
  std::vector<Mat> mats;
  std::vector<Lgt> lights;
  uint32_t prim_count = 0;
  std::vector<uint32_t> prim_geo;  // global prim -> geometry
  float srgb_lut[256];
  std::mutex mu;
  std::shared_ptr<void> bvh_f, bvh_d;
};

namespace {

// ------------------------------------------------------------- materials --

// colorspace.h:10-14
inline float srgb_to_linear(uint8_t x) {
  float v = x / 255.0f;
  if (v <= 0.04045f) return v / 12.92f;
  return std::pow((v + 0.055f) / 1.055f, 2.4f);
}
inline double srgb_to_linear_d(uint8_t x) {
  double v = x / 255.0;
  if (v <= 0.04045) return v / 12.92;
  return std::pow((v + 0.055) / 1.055, 2.4);
}

template <class R>
inline int tex_index(const Mat& m, V2<R> uv) {
  int tx = std::clamp(cvt_trunc((float)(uv.x * (R)m.w)), 0, (int)m.w - 1);
  int ty = std::clamp(cvt_trunc((float)(uv.y * (R)m.h)), 0, (int)m.h - 1);
  return (ty * (int)m.w + tx) * (int)m.c;
}

// material.cpp:57-67
template <class R>
R get_alpha(const Mat& m, V2<R> uv) {
  if (m.pixels.empty()) return R(1);
  if (m.c < 4) return R(1);
  int idx = tex_index(m, uv);
  return (R)m.pixels[idx + 3] / R(255);
}

// material.cpp:69-85
template <class R>
V3<R> get_albedo(const Mat& m, V2<R> uv) {
  if (m.use_override) return V3<R>{(R)m.ovr[0], (R)m.ovr[1], (R)m.ovr[2]};
  V3<R> albedo{R(0.8), R(0.8), R(0.8)};
  if (!m.pixels.empty()) {
    int idx = tex_index(m, uv);
    if constexpr (std::is_same<R, float>::value) {
      albedo = {srgb_to_linear(m.pixels[idx]), srgb_to_linear(m.pixels[idx + 1]),
                srgb_to_linear(m.pixels[idx + 2])};
    } else {
      albedo = {srgb_to_linear_d(m.pixels[idx]), srgb_to_linear_d(m.pixels[idx + 1]),
                srgb_to_linear_d(m.pixels[idx + 2])};
    }
  }
  return albedo;
}

// material.cpp:87-92
template <class R>
V3<R> get_emission(const Mat& m, V2<R> uv) {
  if (m.emission > 0.0f) return get_albedo(m, uv) * (R)m.emission;
  return V3<R>{};
}

// Eigen isZero(): every |coefficient| <= 1e-5.
template <class R>
inline bool is_zero(V3<R> v) {
  const R p = R(1e-5);
  return std::fabs(v.x) <= p && std::fabs(v.y) <= p && std::fabs(v.z) <= p;
}

// material.cpp:148-162
template <class R>
V3<R> eval_material(const Mat& m, V2<R> uv, V3<R> N, V3<R> incident, V3<R> reflected) {
  if (dot(N, reflected) <= R(0) || dot(N, incident) <= R(0)) return V3<R>{};
  V3<R> a = get_albedo(m, uv);
  if constexpr (std::is_same<R, float>::value) return a / (float)kPi;
  return a / (R)kPi;
}

// sh_coeffs.cpp:50-78
template <class R>
inline void accumulate_radiance(V3<R> L, V3<R> d, V3<R> acc[9]) {
  const R k0 = R(0.282095), k1 = R(0.488603), k21 = R(1.092548), k20 = R(0.315392),
          k22 = R(0.546274);
  R x = d.x, y = d.y, z = d.z;
  R sh[9];
  sh[0] = k0;
  sh[1] = k1 * y;
  sh[2] = k1 * z;
  sh[3] = k1 * x;
  sh[4] = k21 * x * y;
  sh[5] = k21 * y * z;
  sh[6] = k20 * (R(3) * z * z - R(1));
  sh[7] = k21 * x * z;
  sh[8] = k22 * (x * x - y * y);
  for (int i = 0; i < 9; ++i) acc[i] += L * sh[i];
}

// ------------------------------------------------------------- philox ----

inline void philox10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Event types of the counter stream (ctr[2]).
enum : uint32_t { EV_HEMI = 0, EV_NEE = 1, EV_BSDF = 2 };

// One event's uniforms: key = (seed, texel), ctr = (sample, vertex, type, block).
struct PhiloxEvent {
  uint32_t key[2];
  uint32_t ctr[3];
  uint32_t cache[4];
  int block = -1;
  uint32_t bits(int i) {
    int b = i >> 2;
    if (b != block) {
      uint32_t c[4] = {ctr[0], ctr[1], ctr[2], (uint32_t)b};
      philox10(c, key, cache);
      block = b;
    }
    return cache[i & 3];
  }
  float u(int i) { return (float)(bits(i) >> 8) * (1.0f / 16777216.0f); }
  size_t tri(int i, size_t n) { return (size_t)(((uint64_t)bits(i) * (uint64_t)n) >> 32); }
  struct Picker {
    PhiloxEvent* ev;
    const std::vector<float>* w;
    float sum;
    int base;
    int pick(int j) {
      float target = ev->u(base + j) * sum;
      float cum = 0.f;
      int last = -1;
      for (size_t i = 0; i < w->size(); ++i) {
        float wi = (*w)[i];
        cum += wi;
        if (wi > 0.f) last = (int)i;
        if (target < cum) return (int)i;
      }
      return last;
    }
  };
  Picker picker(const std::vector<float>& w, float sum, int base) { return Picker{this, &w, sum, base}; }
};

struct PhiloxRng {
  uint32_t seed, texel, sample;
  PhiloxEvent event(uint32_t vertex, uint32_t type) const {
    PhiloxEvent e;
    e.key[0] = seed;
    e.key[1] = texel;
    e.ctr[0] = sample;
    e.ctr[1] = vertex;
    e.ctr[2] = type;
    return e;
  }
};

// The reference stream: every draw advances one std::mt19937.
struct MtEvent {
  std::mt19937* g;
  float u(int) { return std::uniform_real_distribution<float>(0.0f, 1.0f)(*g); }
  size_t tri(int, size_t n) { return std::uniform_int_distribution<size_t>(0, n - 1)(*g); }
  struct Picker {
    std::mt19937* g;
    std::discrete_distribution<int> d;
    int pick(int) { return d(*g); }
  };
  Picker picker(const std::vector<float>& w, float, int) {
    return Picker{g, std::discrete_distribution<int>(w.begin(), w.end())};
  }
};
struct MtRng {
  std::mt19937* g;
  MtEvent event(uint32_t, uint32_t) const { return MtEvent{g}; }
};

// ------------------------------------------------------------- BVH --------

template <class R>
struct Tri {
  V3<R> v0, v1, v2;
};

template <class R>
struct Hit {
  bool hit = false;
  R t = 0, u = 0, v = 0;
  uint32_t prim = 0;
};

template <class R>
struct RayPre {
  V3<R> o, d, inv;
  int kx, ky, kz;
  R Sx, Sy, Sz;
};

template <class R>
RayPre<R> precompute(V3<R> o, V3<R> d) {
  RayPre<R> r;
  r.o = o;
  r.d = d;
  r.inv = {R(1) / d.x, R(1) / d.y, R(1) / d.z};
  R ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
  int kz = 0;
  if (ay > ax) kz = 1;
  if (az > (kz == 0 ? ax : ay)) kz = 2;
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  if (d[kz] < R(0)) std::swap(kx, ky);
  r.kx = kx; r.ky = ky; r.kz = kz;
  r.Sx = d[kx] / d[kz];
  r.Sy = d[ky] / d[kz];
  r.Sz = R(1) / d[kz];
  return r;
}

// Watertight ray/triangle test (Woop, Benthin, Wald 2013).  Accepts
// tnear < t < tfar with t in units of |d|; u, v weight v1, v2 (Embree).
template <class R>
bool tri_test(const RayPre<R>& r, const Tri<R>& tr, R tnear, R tfar, R& t, R& u, R& v) {
  V3<R> A = tr.v0 - r.o, B = tr.v1 - r.o, C = tr.v2 - r.o;
  R Ax = A[r.kx] - r.Sx * A[r.kz];
  R Ay = A[r.ky] - r.Sy * A[r.kz];
  R Bx = B[r.kx] - r.Sx * B[r.kz];
  R By = B[r.ky] - r.Sy * B[r.kz];
  R Cx = C[r.kx] - r.Sx * C[r.kz];
  R Cy = C[r.ky] - r.Sy * C[r.kz];
  R U = Cx * By - Cy * Bx;
  R V = Ax * Cy - Ay * Cx;
  R W = Bx * Ay - By * Ax;
  if constexpr (std::is_same<R, float>::value) {
    if (U == 0.f || V == 0.f || W == 0.f) {
      U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
      V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
      W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
  }
  if ((U < R(0) || V < R(0) || W < R(0)) && (U > R(0) || V > R(0) || W > R(0))) return false;
  R det = U + V + W;
  if (det == R(0)) return false;
  R Az = r.Sz * A[r.kz], Bz = r.Sz * B[r.kz], Cz = r.Sz * C[r.kz];
  R T = U * Az + V * Bz + W * Cz;
  if (det < R(0)) {
    T = -T;
    det = -det;
    U = -U;
    V = -V;
    W = -W;
  }
  if (!(T > tnear * det && T < tfar * det)) return false;
  t = T / det;
  u = V / det;
  v = W / det;
  return true;
}

template <class R>
struct Bvh {
  struct Node {
    R lo[3], hi[3];
    int left = -1, right = -1;  // left<0: leaf
    int start = 0, count = 0;
  };
  std::vector<Node> nodes;
  std::vector<Tri<R>> tris;       // leaf order
  std::vector<uint32_t> prim_of;  // leaf order -> global prim

  void build(const std::vector<Tri<R>>& in) {
    uint32_t n = (uint32_t)in.size();
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::vector<V3<R>> lo(n), hi(n), ce(n);
    for (uint32_t i = 0; i < n; ++i) {
      const Tri<R>& t = in[i];
      lo[i] = {std::min({t.v0.x, t.v1.x, t.v2.x}), std::min({t.v0.y, t.v1.y, t.v2.y}),
               std::min({t.v0.z, t.v1.z, t.v2.z})};
      hi[i] = {std::max({t.v0.x, t.v1.x, t.v2.x}), std::max({t.v0.y, t.v1.y, t.v2.y}),
               std::max({t.v0.z, t.v1.z, t.v2.z})};
      ce[i] = {(lo[i].x + hi[i].x) * R(0.5), (lo[i].y + hi[i].y) * R(0.5),
               (lo[i].z + hi[i].z) * R(0.5)};
    }
    nodes.clear();
    nodes.reserve(2 * std::max<uint32_t>(n, 1));
    if (n == 0) return;
    struct Job { int node, start, count; };
    std::vector<Job> stack;
    nodes.push_back(Node{});
    stack.push_back({0, 0, (int)n});
    while (!stack.empty()) {
      Job j = stack.back();
      stack.pop_back();
      Node nd;
      for (int a = 0; a < 3; ++a) {
        nd.lo[a] = std::numeric_limits<R>::infinity();
        nd.hi[a] = -std::numeric_limits<R>::infinity();
      }
      R clo[3], chi[3];
      for (int a = 0; a < 3; ++a) {
        clo[a] = std::numeric_limits<R>::infinity();
        chi[a] = -std::numeric_limits<R>::infinity();
      }
      for (int k = j.start; k < j.start + j.count; ++k) {
        uint32_t p = idx[k];
        for (int a = 0; a < 3; ++a) {
          nd.lo[a] = std::min(nd.lo[a], lo[p][a]);
          nd.hi[a] = std::max(nd.hi[a], hi[p][a]);
          clo[a] = std::min(clo[a], ce[p][a]);
          chi[a] = std::max(chi[a], ce[p][a]);
        }
      }
      nd.start = j.start;
      nd.count = j.count;
      int split_axis = -1;
      R split_pos = 0;
      if (j.count > 4) {
        constexpr int K = 16;
        R best = std::numeric_limits<R>::infinity();
        for (int a = 0; a < 3; ++a) {
          R ext = chi[a] - clo[a];
          if (!(ext > R(0))) continue;
          int cnt[K] = {};
          R blo[K][3], bhi[K][3];
          for (int b = 0; b < K; ++b)
            for (int c = 0; c < 3; ++c) {
              blo[b][c] = std::numeric_limits<R>::infinity();
              bhi[b][c] = -std::numeric_limits<R>::infinity();
            }
          for (int k = j.start; k < j.start + j.count; ++k) {
            uint32_t p = idx[k];
            int b = std::min(K - 1, (int)((ce[p][a] - clo[a]) * R(K) / ext));
            cnt[b]++;
            for (int c = 0; c < 3; ++c) {
              blo[b][c] = std::min(blo[b][c], lo[p][c]);
              bhi[b][c] = std::max(bhi[b][c], hi[p][c]);
            }
          }
          auto area = [](const R* l, const R* h) {
            R dx = h[0] - l[0], dy = h[1] - l[1], dz = h[2] - l[2];
            if (!(dx >= 0)) return R(0);
            return dx * dy + dy * dz + dz * dx;
          };
          R lA[K], rA[K];
          int lC[K], rC[K];
          R cl[3], ch[3];
          for (int c = 0; c < 3; ++c) { cl[c] = std::numeric_limits<R>::infinity(); ch[c] = -cl[c]; }
          int cc = 0;
          for (int b = 0; b < K; ++b) {
            for (int c = 0; c < 3; ++c) { cl[c] = std::min(cl[c], blo[b][c]); ch[c] = std::max(ch[c], bhi[b][c]); }
            cc += cnt[b];
            lA[b] = area(cl, ch);
            lC[b] = cc;
          }
          for (int c = 0; c < 3; ++c) { cl[c] = std::numeric_limits<R>::infinity(); ch[c] = -cl[c]; }
          cc = 0;
          for (int b = K - 1; b >= 0; --b) {
            for (int c = 0; c < 3; ++c) { cl[c] = std::min(cl[c], blo[b][c]); ch[c] = std::max(ch[c], bhi[b][c]); }
            cc += cnt[b];
            rA[b] = area(cl, ch);
            rC[b] = cc;
          }
          for (int b = 0; b < K - 1; ++b) {
            if (lC[b] == 0 || rC[b + 1] == 0) continue;
            R cost = lA[b] * lC[b] + rA[b + 1] * rC[b + 1];
            if (cost < best) {
              best = cost;
              split_axis = a;
              split_pos = clo[a] + ext * R(b + 1) / R(K);
            }
          }
        }
      }
      int mid = -1;
      if (j.count > 4) {
        if (split_axis >= 0) {
          auto it = std::partition(idx.begin() + j.start, idx.begin() + j.start + j.count,
                                   [&](uint32_t p) { return ce[p][split_axis] < split_pos; });
          mid = (int)(it - idx.begin());
          if (mid == j.start || mid == j.start + j.count) mid = -1;
        }
        if (mid < 0) mid = j.start + j.count / 2;
      }
      if (mid < 0) {
        nodes[j.node] = nd;
        continue;
      }
      int l = (int)nodes.size();
      nodes.push_back(Node{});
      nodes.push_back(Node{});
      nd.left = l;
      nd.right = l + 1;
      nodes[j.node] = nd;
      stack.push_back({l, j.start, mid - j.start});
      stack.push_back({l + 1, mid, j.start + j.count - mid});
    }
    tris.resize(n);
    prim_of = idx;
    for (uint32_t i = 0; i < n; ++i) tris[i] = in[idx[i]];
  }

  static bool box(const Node& nd, const RayPre<R>& r, R tnear, R tfar, R& tentry) {
    R t0 = tnear, t1 = tfar;
    for (int a = 0; a < 3; ++a) {
      R ta = (nd.lo[a] - r.o[a]) * r.inv[a];
      R tb = (nd.hi[a] - r.o[a]) * r.inv[a];
      if (ta > tb) std::swap(ta, tb);
      tb *= R(1) + R(4) * std::numeric_limits<R>::epsilon();
      t0 = ta > t0 ? ta : t0;
      t1 = tb < t1 ? tb : t1;
      if (t0 > t1) return false;
    }
    tentry = t0;
    return true;
  }

  // any_hit: stop at the first triangle in (tnear, tfar).
  Hit<R> trace(V3<R> o, V3<R> d, R tnear, R tfar, bool any_hit) const {
    Hit<R> h;
    if (nodes.empty()) return h;
    RayPre<R> r = precompute(o, d);
    int stack[128];
    int sp = 0;
    R best = tfar;
    R te;
    if (!box(nodes[0], r, tnear, best, te)) return h;
    stack[sp++] = 0;
    while (sp > 0) {
      const Node& nd = nodes[stack[--sp]];
      if (nd.left < 0) {
        for (int k = nd.start; k < nd.start + nd.count; ++k) {
          R t, u, v;
          if (tri_test(r, tris[k], tnear, best, t, u, v)) {
            best = t;
            h.hit = true;
            h.t = t;
            h.u = u;
            h.v = v;
            h.prim = prim_of[k];
            if (any_hit) return h;
          }
        }
        continue;
      }
      R tl, tr;
      bool hl = box(nodes[nd.left], r, tnear, best, tl);
      bool hr = box(nodes[nd.right], r, tnear, best, tr);
      if (hl && hr) {
        if (tl <= tr) {
          stack[sp++] = nd.right;
          stack[sp++] = nd.left;
        } else {
          stack[sp++] = nd.left;
          stack[sp++] = nd.right;
        }
      } else if (hl) {
        stack[sp++] = nd.left;
      } else if (hr) {
        stack[sp++] = nd.right;
      }
    }
    return h;
  }
};

template <class R>
std::shared_ptr<Bvh<R>> get_bvh(const oracle_scene* cs) {
  oracle_scene* s = const_cast<oracle_scene*>(cs);
  std::lock_guard<std::mutex> lk(s->mu);
  std::shared_ptr<void>& slot = std::is_same<R, float>::value ? s->bvh_f : s->bvh_d;
  if (!slot) {
    std::vector<Tri<R>> tris;
    tris.reserve(s->prim_count);
    for (const Geo& g : s->geos) {
      for (size_t i = 0; i + 2 < g.indices.size(); i += 3) {
        const V3<float>& a = g.world_vertices[g.indices[i]];
        const V3<float>& b = g.world_vertices[g.indices[i + 1]];
        const V3<float>& c = g.world_vertices[g.indices[i + 2]];
        tris.push_back(Tri<R>{{(R)a.x, (R)a.y, (R)a.z}, {(R)b.x, (R)b.y, (R)b.z}, {(R)c.x, (R)c.y, (R)c.z}});
      }
    }
    auto b = std::make_shared<Bvh<R>>();
    b->build(tris);
    slot = b;
  }
  return std::static_pointer_cast<Bvh<R>>(slot);
}

// Hit attributes (occlusion.cpp:70-133).
template <class R>
struct Occ {
  bool hit = false;
  V3<R> position;
  V2<R> uv;
  V3<R> normal;
  int material_id = -1;
  R t = 0;
  uint32_t prim = 0;
};

template <class R>
Occ<R> find_occlusion(const oracle_scene* s, const Bvh<R>& bvh, V3<R> o, V3<R> d, R tnear,
                      R tfar) {
  Occ<R> occ;
  Hit<R> h = bvh.trace(o, d, tnear, tfar, false);
  if (!h.hit) return occ;
  occ.hit = true;
  occ.t = h.t;
  occ.prim = h.prim;
  occ.position = o + d * h.t;
  const Geo& g = s->geos[s->prim_geo[h.prim]];
  occ.material_id = g.material_id;
  R u = h.u, v = h.v;
  R w = R(1) - u - v;
  uint32_t local = h.prim - g.prim_base;
  uint32_t i0 = g.indices[local * 3], i1 = g.indices[local * 3 + 1], i2 = g.indices[local * 3 + 2];
  auto cv = [](const V3<float>& a) { return V3<R>{(R)a.x, (R)a.y, (R)a.z}; };
  if (!g.normals.empty()) {
    occ.normal = normalized(w * cv(g.normals[i0]) + u * cv(g.normals[i1]) + v * cv(g.normals[i2]));
  } else {
    V3<R> a = cv(g.world_vertices[i0]), b = cv(g.world_vertices[i1]), c = cv(g.world_vertices[i2]);
    occ.normal = normalized(cross(b - a, c - a));
  }
  if (!g.texture_uvs.empty()) {
    auto c2 = [](const V2<float>& a) { return V2<R>{(R)a.x, (R)a.y}; };
    occ.uv = w * c2(g.texture_uvs[i0]) + u * c2(g.texture_uvs[i1]) + v * c2(g.texture_uvs[i2]);
  }
  return occ;
}

template <class R>
bool occluded(const Bvh<R>& bvh, V3<R> o, V3<R> d, R tnear, R tfar) {
  return bvh.trace(o, d, tnear, tfar, true).hit;
}

// ------------------------------------------------------------- lights -----

template <class R>
struct AreaSample {
  V3<R> point, normal, radiance;
  R pdf = 0;
};

template <class R, class Ev>
AreaSample<R> sample_area_light(const oracle_scene* s, const Lgt& L, Ev& ev, int ubase) {
  AreaSample<R> out;
  if (L.geometry < 0 || L.material < 0) return out;
  const Geo& g = s->geos[L.geometry];
  if (g.indices.empty()) return out;
  size_t n = g.indices.size() / 3;
  size_t tri = ev.tri(ubase, n);
  uint32_t i0 = g.indices[tri * 3], i1 = g.indices[tri * 3 + 1], i2 = g.indices[tri * 3 + 2];
  float u1f = ev.u(ubase + 1);
  float u2f = ev.u(ubase + 2);
  R u1 = u1f, u2 = u2f;
  if (u1 + u2 > R(1)) {
    u1 = R(1) - u1;
    u2 = R(1) - u2;
  }
  R w = R(1) - u1 - u2;
  auto cv = [](const V3<float>& a) { return V3<R>{(R)a.x, (R)a.y, (R)a.z}; };
  V3<R> v0 = cv(g.vertices[i0]), v1 = cv(g.vertices[i1]), v2 = cv(g.vertices[i2]);
  out.point = w * v0 + u1 * v1 + u2 * v2;
  out.normal = {0, 1, 0};
  if (!g.normals.empty())
    out.normal = normalized(w * cv(g.normals[i0]) + u1 * cv(g.normals[i1]) + u2 * cv(g.normals[i2]));
  V2<R> uv;
  if (!g.texture_uvs.empty()) {
    auto c2 = [](const V2<float>& a) { return V2<R>{(R)a.x, (R)a.y}; };
    uv = w * c2(g.texture_uvs[i0]) + u1 * c2(g.texture_uvs[i1]) + u2 * c2(g.texture_uvs[i2]);
  }
  out.radiance = get_emission<R>(s->mats[L.material], uv);
  R area = std::sqrt(sqnorm(cross(v0 - v1, v0 - v2))) / R(2);
  out.pdf = std::max(R(1e-6), R(1) / (R)n * R(1) / area);
  return out;
}

template <class R>
struct LightEval {
  V3<R> radiance;
  V3<R> ray_o, ray_d;
  R tnear = R(0.001), tfar = R(0);
  R area_pdf = R(1);
  V3<R> incident;  // unit direction to the light
  R cos_n = 0;
};

// Incoming radiance without visibility (light.h:34-49,72-95,117-144,166-188).
template <class R>
LightEval<R> incoming(const Lgt& L, V3<R> P, V3<R> N, const AreaSample<R>* as) {
  LightEval<R> e;
  auto cv = [](const V3<float>& a) { return V3<R>{(R)a.x, (R)a.y, (R)a.z}; };
  V3<R> color = cv(L.color);
  R I = L.intensity;
  if (L.type == SHB_LIGHT_DIRECTIONAL) {
    V3<R> dir = cv(L.direction);
    e.ray_o = P;
    e.ray_d = -dir;
    e.tfar = R(1.0e10);
    e.cos_n = dot(N, -dir);
    e.incident = -dir;
    e.radiance = e.cos_n < R(0) ? V3<R>{} : I * color;
    return e;
  }
  V3<R> target = (L.type == SHB_LIGHT_AREA) ? as->point : cv(L.position);
  V3<R> Lv = target - P;
  R dist_sq = sqnorm(Lv);
  R dist = std::sqrt(dist_sq);
  e.ray_o = P;
  e.ray_d = target - P;
  e.tfar = dist - R(0.001);
  Lv = Lv / dist;
  e.incident = Lv;
  e.cos_n = dot(N, Lv);
  if (L.type == SHB_LIGHT_POINT) {
    e.radiance = e.cos_n < R(0) ? V3<R>{} : I * color / (dist * dist);
  } else if (L.type == SHB_LIGHT_SPOT) {
    R cos_l = dot(cv(L.direction), -Lv);
    R falloff = (cos_l - (R)L.cos_outer) / ((R)L.cos_inner - (R)L.cos_outer);
    falloff = std::clamp(falloff, R(0), R(1));
    e.radiance = e.cos_n < R(0) ? V3<R>{} : I * color / (dist * dist) * falloff;
  } else {
    e.radiance = e.cos_n < R(0) ? V3<R>{} : as->radiance / (dist * dist);
    e.area_pdf = as->pdf;
  }
  return e;
}

struct BakeCtx {
  const oracle_scene* s;
  int max_depth;
  unsigned nls;
  uint64_t rays = 0;
};

// EvaluateLightSamples (light.cpp:82-189).
template <class R, class Ev>
V3<R> evaluate_light_samples(BakeCtx& c, const Bvh<R>& bvh, V3<R> P, V3<R> N, V3<R> wo,
                             const Mat& mat, V2<R> uv, Ev ev) {
  const oracle_scene* s = c.s;
  size_t nl = s->lights.size();
  std::vector<LightEval<R>> evs(nl);
  std::vector<float> weights(nl);
  int area_ord = 0;
  for (size_t i = 0; i < nl; ++i) {
    const Lgt& L = s->lights[i];
    AreaSample<R> as;
    if (L.type == SHB_LIGHT_AREA) as = sample_area_light<R>(s, L, ev, 3 * area_ord++);
    LightEval<R> e = incoming<R>(L, P, N, &as);
    // light.h:51-64,97-109,146-158,190-203: radiance x cos x BRDF.
    if (e.cos_n < R(0)) {
      e.radiance = V3<R>{};
    } else {
      V3<R> brdf = eval_material<R>(mat, uv, N, e.incident, wo);
      V3<R> cos_brdf = e.cos_n * brdf;
      e.radiance = cmul(e.radiance, cos_brdf);
    }
    evs[i] = e;
    weights[i] = (float)max_coeff(e.radiance);
  }
  float sum = std::accumulate(weights.begin(), weights.end(), 0.0f);
  V3<R> result{};
  if (sum < 1e-6f) return result;
  int total_area = 0;
  for (const Lgt& L : s->lights) total_area += (L.type == SHB_LIGHT_AREA);
  auto picker = ev.picker(weights, sum, 3 * total_area);
  for (unsigned i = 0; i < c.nls; ++i) {
    int idx = picker.pick((int)i);
    const LightEval<R>& e = evs[idx];
    c.rays++;
    if (occluded(bvh, e.ray_o, e.ray_d, e.tnear, e.tfar)) continue;
    R pdf = (R)weights[idx] / (R)sum;
    R joint = pdf * e.area_pdf;
    if (joint < R(1e-3)) continue;
    result += e.radiance / joint;
  }
  return result / (R)c.nls;
}

// AccumulateIncomingLightSamples (light.cpp:191-293).
template <class R, class Ev>
void accumulate_incoming(BakeCtx& c, const Bvh<R>& bvh, V3<R> P, V3<R> N, Ev ev, V3<R> acc[9],
                         V3<R>* acc2) {
  const oracle_scene* s = c.s;
  size_t nl = s->lights.size();
  std::vector<LightEval<R>> evs(nl);
  std::vector<float> weights(nl);
  int area_ord = 0;
  for (size_t i = 0; i < nl; ++i) {
    const Lgt& L = s->lights[i];
    AreaSample<R> as;
    if (L.type == SHB_LIGHT_AREA) as = sample_area_light<R>(s, L, ev, 3 * area_ord++);
    evs[i] = incoming<R>(L, P, N, &as);
    weights[i] = (float)max_coeff(evs[i].radiance);
  }
  float sum = std::accumulate(weights.begin(), weights.end(), 0.0f);
  if (sum < 1e-6f) return;
  int total_area = area_ord;
  auto picker = ev.picker(weights, sum, 3 * total_area);
  for (unsigned i = 0; i < c.nls; ++i) {
    int idx = picker.pick((int)i);
    const LightEval<R>& e = evs[idx];
    c.rays++;
    if (occluded(bvh, e.ray_o, e.ray_d, e.tnear, e.tfar)) continue;
    R pdf = (R)weights[idx] / (R)sum;
    R joint = pdf * e.area_pdf;
    if (joint < R(1e-3)) continue;
    V3<R> Li = e.radiance / (joint * (R)c.nls);
    accumulate_radiance(Li, e.ray_d, acc);
    if (acc2) accumulate_radiance(Li, e.ray_d, acc2);
  }
}

template <class R>
struct ReflSample {
  V3<R> direction;
  R pdf = 0;
};

// SampleMaterial (material.cpp:113-146).
template <class R, class Ev>
ReflSample<R> sample_material(V3<R> N, Ev ev) {
  V3<R> t, b;
  if (std::fabs(N.x) > std::fabs(N.z)) t = {-N.y, N.x, R(0)};
  else t = {R(0), -N.z, N.y};
  t = normalized(t);
  b = cross(N, t);
  float r1 = ev.u(0);
  float r2 = ev.u(1);
  R phi, theta, sin_theta;
  if constexpr (std::is_same<R, float>::value) {
    phi = (float)(2.0 * kPi * (double)r1);
    theta = std::acos(std::sqrt(r2));
    sin_theta = std::sin(theta);
  } else {
    phi = 2.0 * kPi * (double)r1;
    theta = std::acos(std::sqrt((double)r2));
    sin_theta = std::sin(theta);
  }
  V3<R> local{std::cos(phi) * sin_theta, std::sin(phi) * sin_theta, std::cos(theta)};
  V3<R> world = t * local.x + b * local.y + N * local.z;
  ReflSample<R> smp;
  smp.direction = normalized(world);
  if constexpr (std::is_same<R, float>::value) smp.pdf = (float)((double)local.z / kPi);
  else smp.pdf = local.z / kPi;
  return smp;
}

// Trace (baker.cpp:70-149).
template <class R, class Rng>
V3<R> trace(BakeCtx& c, const Bvh<R>& bvh, const Rng& rng, V3<R> origin, V3<R> dir, int depth,
            uint32_t vertex, float* env) {
  if (depth > c.max_depth) return V3<R>{};
  c.rays++;
  Occ<R> occ = find_occlusion<R>(c.s, bvh, origin, dir, R(0.001), std::numeric_limits<R>::infinity());
  if (!occ.hit) {
    if (depth == 0) *env += 1.0f;
    return V3<R>{};
  }
  static const Mat kDefault{};
  const Mat& mat = (occ.material_id >= 0 && occ.material_id < (int)c.s->mats.size())
                       ? c.s->mats[occ.material_id]
                       : kDefault;
  R alpha = get_alpha(mat, occ.uv);
  V3<R> color{};
  if (alpha < R(1)) {
    V3<R> hp = occ.position + dir * R(0.001);
    V3<R> transmission = trace<R>(c, bvh, rng, hp, dir, depth + 1, 2 * vertex + 1, env);
    color += (R(1) - alpha) * transmission;
  }
  if (alpha == R(0)) return color;
  V3<R> emission = get_emission(mat, occ.uv);
  if (!is_zero(emission)) {
    if (depth == 0) color += alpha * emission;
  }
  V3<R> hit_pos = occ.position + occ.normal * R(0.001);
  V3<R> L_direct = evaluate_light_samples<R>(c, bvh, hit_pos, occ.normal, -dir, mat, occ.uv,
                                             rng.event(vertex, EV_NEE));
  color += alpha * L_direct;
  ReflSample<R> smp = sample_material<R>(occ.normal, rng.event(vertex, EV_BSDF));
  if (smp.pdf < R(1e-3)) return color;
  V3<R> inc = trace<R>(c, bvh, rng, hit_pos, smp.direction, depth + 1, 2 * vertex, env);
  V3<R> brdf = eval_material<R>(mat, occ.uv, occ.normal, smp.direction, -dir);
  R cos_term = dot(occ.normal, smp.direction);
  V3<R> L_ind = cmul(inc, brdf) * (cos_term / smp.pdf);
  color += alpha * L_ind;
  return color;
}

template <class R>
V3<R> pt_pos(const shb_surface_point& p) { return {(R)p.position[0], (R)p.position[1], (R)p.position[2]}; }
template <class R>
V3<R> pt_nrm(const shb_surface_point& p) { return {(R)p.normal[0], (R)p.normal[1], (R)p.normal[2]}; }

// One texel of BakeSHLightMap (baker.cpp:244-295).
template <class R, class Rng>
void bake_texel(BakeCtx& c, const Bvh<R>& bvh, const shb_surface_point& sp, int samples,
                int sample_offset, Rng make_rng, float* sh_out, float* env_out, double* var_out,
                double* mean64_out, uint64_t texel) {
  V3<R> acc[9];
  float env = 0.0f;
  V3<R> P = pt_pos<R>(sp), N = pt_nrm<R>(sp);
  V3<R> T{(R)sp.tangent[0], (R)sp.tangent[1], (R)sp.tangent[2]};
  R Tw = sp.tangent[3];
  V3<R> origin = P + N * R(0.001);
  const R inv_pdf_uniform = std::is_same<R, float>::value ? (R)(float)(2.0f * kPi) : (R)(2.0 * kPi);
  double s1[27] = {}, s2[27] = {};
  bool stats = var_out || mean64_out;
  for (int s = 0; s < samples; ++s) {
    auto rng = make_rng(texel, (uint32_t)(s + sample_offset));
    auto hev = rng.event(0, EV_HEMI);
    float u1 = hev.u(0);
    float u2 = hev.u(1);
    R r, phi;
    if constexpr (std::is_same<R, float>::value) {
      r = std::sqrt(1.0f - u1 * u1);
      phi = (float)(2.0 * kPi * (double)u2);
    } else {
      r = std::sqrt(1.0 - (double)u1 * (double)u1);
      phi = 2.0 * kPi * (double)u2;
    }
    V3<R> dl{r * std::cos(phi), r * std::sin(phi), (R)u1};
    V3<R> bitangent = cross(N, T) * Tw;
    V3<R> dw = T * dl.x + bitangent * dl.y + N * dl.z;
    V3<R> tmp[9];
    accumulate_incoming<R>(c, bvh, P, N, rng.event(0, EV_NEE), acc, stats ? tmp : nullptr);
    V3<R> Li = trace<R>(c, bvh, rng, origin, dw, 0, 1, &env) * inv_pdf_uniform;
    accumulate_radiance(Li, dw, acc);
    if (stats) {
      accumulate_radiance(Li, dw, tmp);
      for (int i = 0; i < 9; ++i) {
        double v[3] = {(double)tmp[i].x, (double)tmp[i].y, (double)tmp[i].z};
        for (int k = 0; k < 3; ++k) {
          s1[i * 3 + k] += v[k];
          s2[i * 3 + k] += v[k] * v[k];
        }
      }
    }
  }
  R scale = std::is_same<R, float>::value ? (R)(1.0f / (float)samples) : R(1) / (R)samples;
  for (int i = 0; i < 9; ++i) {
    V3<R> v = acc[i] * scale;
    if (sh_out) {
      sh_out[i * 3 + 0] = (float)v.x;
      sh_out[i * 3 + 1] = (float)v.y;
      sh_out[i * 3 + 2] = (float)v.z;
    }
  }
  if (env_out) *env_out = env * (1.0f / samples);
  if (stats) {
    for (int k = 0; k < 27; ++k) {
      double m = s1[k] / samples;
      if (mean64_out) mean64_out[k] = m;
      if (var_out) var_out[k] = samples > 1 ? std::max(0.0, (s2[k] - samples * m * m) / (samples - 1)) : 0.0;
    }
  }
}

template <class R>
int bake_impl(const oracle_scene* s, const shb_surface_point* pts, const shb_raster_config* rc,
              oracle_bake_args* a) {
  auto bvh = get_bvh<R>(s);
  int64_t W = (int64_t)rc->width * rc->supersample_scale;
  int64_t H = (int64_t)rc->height * rc->supersample_scale;
  int64_t total = W * H;
  std::vector<int64_t> work;
  if (a->texel_subset) work.assign(a->texel_subset, a->texel_subset + a->subset_count);
  else {
    work.resize(total);
    std::iota(work.begin(), work.end(), 0);
  }
  int nthreads = a->threads > 0 ? a->threads : (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int64_t> next{0};
  std::atomic<uint64_t> rays{0}, ts{0};
  auto worker = [&]() {
    BakeCtx c{s, a->bounces, (unsigned)a->num_light_samples};
    uint64_t local_ts = 0;
    while (true) {
      int64_t begin = next.fetch_add(16);
      if (begin >= (int64_t)work.size()) break;
      int64_t end = std::min<int64_t>(begin + 16, work.size());
      for (int64_t k = begin; k < end; ++k) {
        int64_t idx = work[k];
        if (idx < 0 || idx >= total) continue;
        const shb_surface_point& sp = pts[idx];
        if (sp.material_id < 0) continue;
        float* sh = a->sh_out ? a->sh_out + idx * 27 : nullptr;
        float* env = a->env_out ? a->env_out + idx : nullptr;
        double* var = a->sh_var_out ? a->sh_var_out + idx * 27 : nullptr;
        double* m64 = a->sh_mean64_out ? a->sh_mean64_out + idx * 27 : nullptr;
        if (a->rng_mode == ORACLE_RNG_MT19937) {
          std::mt19937 g((std::mt19937::result_type)(12345 + (size_t)idx));
          auto mk = [&g](uint64_t, uint32_t) { return MtRng{&g}; };
          bake_texel<R>(c, *bvh, sp, a->samples, a->sample_offset, mk, sh, env, var, m64, idx);
        } else {
          uint32_t seed = a->seed;
          auto mk = [seed](uint64_t texel, uint32_t sample) {
            return PhiloxRng{seed, (uint32_t)texel, sample};
          };
          bake_texel<R>(c, *bvh, sp, a->samples, a->sample_offset, mk, sh, env, var, m64, idx);
        }
        local_ts += (uint64_t)a->samples;
      }
    }
    rays += c.rays;
    ts += local_ts;
  };
  std::vector<std::thread> th;
  for (int i = 0; i < nthreads; ++i) th.emplace_back(worker);
  for (auto& t : th) t.join();
  a->rays_traced = rays.load();
  a->texel_samples = ts.load();
  return 0;
}

}  // namespace

namespace {
// rasterizer.cpp:18-33
bool barycentric(V2<float> p, V2<float> a, V2<float> b, V2<float> c, float& u, float& v, float& w) {
  V2<float> v0 = b - a, v1 = c - a, v2 = p - a;
  float d00 = dot2(v0, v0);
  float d01 = dot2(v0, v1);
  float d11 = dot2(v1, v1);
  float d20 = dot2(v2, v0);
  float d21 = dot2(v2, v1);
  float denom = d00 * d11 - d01 * d01;
  if (std::fabs(denom) < 1e-8f) return false;
  v = (d11 * d20 - d01 * d21) / denom;
  w = (d00 * d21 - d01 * d20) / denom;
  u = 1.0f - v - w;
  return (v >= 0.0f) && (w >= 0.0f) && (u >= 0.0f);
}

shb_surface_point make_point(const Geo& g, uint32_t i0, uint32_t i1, uint32_t i2, float u, float v,
                             float w) {
  shb_surface_point sp;
  std::memset(&sp, 0, sizeof(sp));
  sp.material_id = g.material_id;
  V3<float> pos = g.world_vertices[i0] * u + g.world_vertices[i1] * v + g.world_vertices[i2] * w;
  V3<float> nrm = normalized(g.world_normals[i0] * u + g.world_normals[i1] * v + g.world_normals[i2] * w);
  V4<float> t4 = g.world_tangents[i0] * u + g.world_tangents[i1] * v + g.world_tangents[i2] * w;
  V3<float> t3{t4.x, t4.y, t4.z};
  t3 = normalized(t3 - nrm * dot(nrm, t3));
  sp.position[0] = pos.x; sp.position[1] = pos.y; sp.position[2] = pos.z;
  sp.normal[0] = nrm.x; sp.normal[1] = nrm.y; sp.normal[2] = nrm.z;
  sp.tangent[0] = t3.x; sp.tangent[1] = t3.y; sp.tangent[2] = t3.z; sp.tangent[3] = t4.w;
  return sp;
}
}  // namespace

namespace {
template <class T, int C>
void dilate_t(int w, int h, T* pixels, uint8_t* mask, int passes) {
  size_t n = (size_t)w * h;
  if (n == 0) return;
  std::vector<T> next(pixels, pixels + n * C);
  std::vector<uint8_t> nmask(mask, mask + n);
  for (int p = 0; p < passes; ++p) {
    bool changed = false;
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        size_t idx = (size_t)y * w + x;
        if (mask[idx]) continue;
        T acc[C];
        for (int c = 0; c < C; ++c) acc[c] = T();
        int count = 0;
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            if (dx == 0 && dy == 0) continue;
            int nx = x + dx, ny = y + dy;
            if (nx >= 0 && nx < w && ny >= 0 && ny < h) {
              size_t ni = (size_t)ny * w + nx;
              if (mask[ni]) {
                for (int c = 0; c < C; ++c) acc[c] += pixels[ni * C + c];
                count++;
              }
            }
          }
        if (count > 0) {
          float inv = 1.0f / count;
          for (int c = 0; c < C; ++c) next[idx * C + c] = (T)(acc[c] * inv);
          nmask[idx] = 1;
          changed = true;
        }
      }
    std::copy(next.begin(), next.end(), pixels);
    std::copy(nmask.begin(), nmask.end(), mask);
    if (!changed) break;
  }
}
}  // namespace


// ============================================================ gradient ===
//
// FP64 forward-mode derivative of the Philox-stream bake with respect to the
// adjoint parameters: 3 per material (linear base colour, only materials
// with an override; channel c of the radiance depends on channel c of the
// albedo only) and 1 per light (intensity of point, spot and directional
// lights).  A recursive tracer of its own, structured like trace() above,
// that carries next to every radiance value its dense tangent.  The
// light-selection weights are the forward's values and are held constant,
// so this is the derivative of the estimator of the expected bake.  The loss
// is linear in the SH output: Loss = sum(dsh * SH).

namespace {

using V3d = V3<double>;

struct GradCtx {
  const oracle_scene* s;
  const Bvh<double>* bvh;
  int max_depth;
  unsigned nls;
  int n_mat3, P;
};

struct Dual {
  V3d v{};
  std::vector<V3d> d;
  explicit Dual(int P) : d((size_t)P) {}
};

inline void add_scaled(Dual& y, const Dual& x, double a) {
  y.v += x.v * a;
  for (size_t p = 0; p < y.d.size(); ++p) y.d[p] += x.d[p] * a;
}

inline void add_channel(std::vector<V3d>& d, int base, V3d v) {
  d[base + 0].x += v.x;
  d[base + 1].y += v.y;
  d[base + 2].z += v.z;
}

inline bool is_param(const GradCtx& c, int mat) {
  return mat >= 0 && mat < (int)c.s->mats.size() && c.s->mats[mat].use_override;
}

// d(incoming radiance before the BRDF) / d(light parameter): per channel.
// light = true: the light's intensity (parameter n_mat3 + l); else the
// emissive material's albedo (parameters 3 mL + c), when it is a parameter.
struct LightDeriv {
  V3d dv{};
  int param = -1;
  bool light = false;
};

LightDeriv light_deriv(const GradCtx& c, int li, V3d P, const AreaSample<double>& as, const LightEval<double>& e) {
  const Lgt& L = c.s->lights[li];
  LightDeriv out;
  if (e.cos_n < 0.0) return out;
  V3d color{L.color.x, L.color.y, L.color.z};
  if (L.type == SHB_LIGHT_DIRECTIONAL) {
    out.dv = color;
    out.param = c.n_mat3 + li;
    out.light = true;
    return out;
  }
  V3d target = L.type == SHB_LIGHT_AREA ? as.point : V3d{L.position.x, L.position.y, L.position.z};
  V3d Lv = target - P;
  double dist = std::sqrt(sqnorm(Lv));
  if (L.type == SHB_LIGHT_POINT || L.type == SHB_LIGHT_SPOT) {
    double falloff = 1.0;
    if (L.type == SHB_LIGHT_SPOT) {
      V3d u = Lv / dist;
      double cos_l = dot(V3d{L.direction.x, L.direction.y, L.direction.z}, -u);
      falloff = std::clamp((cos_l - (double)L.cos_outer) / ((double)L.cos_inner - (double)L.cos_outer), 0.0, 1.0);
    }
    out.dv = color / (dist * dist) * falloff;
    out.param = c.n_mat3 + li;
    out.light = true;
    return out;
  }
  if (is_param(c, L.material) && c.s->mats[L.material].emission > 0.0f) {
    double em = c.s->mats[L.material].emission;
    out.dv = V3d{em, em, em} / (dist * dist);
    out.param = 3 * L.material;
  }
  return out;
}

inline void add_light_deriv(std::vector<V3d>& d, const LightDeriv& ld, V3d dv) {
  if (ld.param < 0) return;
  if (ld.light) d[ld.param] += dv;
  else add_channel(d, ld.param, dv);
}

inline void sh_basis(V3d dir, double Y[9]) {
  V3d acc[9];
  accumulate_radiance<double>(V3d{1.0, 1.0, 1.0}, dir, acc);
  for (int k = 0; k < 9; ++k) Y[k] = acc[k].x;
}

// sum_k g[3k + c] Y_k(dir) * scale, per channel
inline V3d sh_adjoint(const float* g, V3d dir, double scale) {
  double Y[9];
  sh_basis(dir, Y);
  V3d a{};
  for (int k = 0; k < 9; ++k) {
    a.x += (double)g[3 * k] * Y[k];
    a.y += (double)g[3 * k + 1] * Y[k];
    a.z += (double)g[3 * k + 2] * Y[k];
  }
  return a * scale;
}

// EvaluateLightSamples (light.cpp:82-189) with tangents.
Dual light_samples_grad(GradCtx& c, V3d P, V3d N, V3d wo, int mat_id, const Mat& mat, V2<double> uv,
                        PhiloxEvent ev) {
  const oracle_scene* s = c.s;
  size_t nl = s->lights.size();
  std::vector<LightEval<double>> evs(nl);
  std::vector<AreaSample<double>> ass(nl);
  std::vector<float> weights(nl);
  std::vector<V3d> brdfs(nl);
  int area_ord = 0;
  for (size_t i = 0; i < nl; ++i) {
    const Lgt& L = s->lights[i];
    if (L.type == SHB_LIGHT_AREA) ass[i] = sample_area_light<double>(s, L, ev, 3 * area_ord++);
    LightEval<double> e = incoming<double>(L, P, N, &ass[i]);
    if (e.cos_n < 0.0) {
      e.radiance = V3d{};
    } else {
      brdfs[i] = eval_material<double>(mat, uv, N, e.incident, wo);
      e.radiance = cmul(e.radiance, e.cos_n * brdfs[i]);
    }
    evs[i] = e;
    weights[i] = (float)max_coeff(e.radiance);
  }
  Dual out(c.P);
  float sum = std::accumulate(weights.begin(), weights.end(), 0.0f);
  if (sum < 1e-6f) return out;
  auto picker = ev.picker(weights, sum, 3 * area_ord);
  const bool own = is_param(c, mat_id);
  for (unsigned j = 0; j < c.nls; ++j) {
    int idx = picker.pick((int)j);
    const LightEval<double>& e = evs[idx];
    if (occluded(*c.bvh, e.ray_o, e.ray_d, e.tnear, e.tfar)) continue;
    double joint = (double)weights[idx] / (double)sum * e.area_pdf;
    if (joint < 1e-3) continue;
    out.v += e.radiance / joint;
    if (e.cos_n < 0.0) continue;
    const bool lit = !(dot(N, wo) <= 0.0 || dot(N, e.incident) <= 0.0);
    if (own && lit) {
      LightEval<double> pre = incoming<double>(s->lights[idx], P, N, &ass[idx]);
      add_channel(out.d, 3 * mat_id, pre.radiance * (e.cos_n / kPi / joint));
    }
    LightDeriv ld = light_deriv(c, idx, P, ass[idx], e);
    add_light_deriv(out.d, ld, cmul(ld.dv, e.cos_n * brdfs[idx]) / joint);
  }
  out.v = out.v / (double)c.nls;
  for (V3d& x : out.d) x = x / (double)c.nls;
  return out;
}

// Trace (baker.cpp:70-149) with tangents.
Dual trace_grad(GradCtx& c, const PhiloxRng& rng, V3d origin, V3d dir, int depth, uint32_t vertex) {
  Dual color(c.P);
  if (depth > c.max_depth) return color;
  Occ<double> occ = find_occlusion<double>(c.s, *c.bvh, origin, dir, 0.001, std::numeric_limits<double>::infinity());
  if (!occ.hit) return color;
  static const Mat kDefault{};
  const bool valid = occ.material_id >= 0 && occ.material_id < (int)c.s->mats.size();
  const Mat& mat = valid ? c.s->mats[occ.material_id] : kDefault;
  const int mid = valid ? occ.material_id : -1;
  double alpha = get_alpha(mat, occ.uv);
  if (alpha < 1.0) {
    Dual tr = trace_grad(c, rng, occ.position + dir * 0.001, dir, depth + 1, 2 * vertex + 1);
    add_scaled(color, tr, 1.0 - alpha);
  }
  if (alpha == 0.0) return color;
  V3d emission = get_emission(mat, occ.uv);
  if (!is_zero(emission) && depth == 0) {
    color.v += alpha * emission;
    if (is_param(c, mid)) add_channel(color.d, 3 * mid, V3d{1.0, 1.0, 1.0} * (alpha * (double)mat.emission));
  }
  V3d hit_pos = occ.position + occ.normal * 0.001;
  Dual direct = light_samples_grad(c, hit_pos, occ.normal, -dir, mid, mat, occ.uv, rng.event(vertex, EV_NEE));
  add_scaled(color, direct, alpha);
  ReflSample<double> smp = sample_material<double>(occ.normal, rng.event(vertex, EV_BSDF));
  if (smp.pdf < 1e-3) return color;
  Dual inc = trace_grad(c, rng, hit_pos, smp.direction, depth + 1, 2 * vertex);
  V3d brdf = eval_material<double>(mat, occ.uv, occ.normal, smp.direction, -dir);
  double k = dot(occ.normal, smp.direction) / smp.pdf;
  color.v += cmul(inc.v, brdf) * (k * alpha);
  for (int p = 0; p < c.P; ++p) color.d[p] += cmul(inc.d[p], brdf) * (k * alpha);
  const bool lit = !(dot(occ.normal, -dir) <= 0.0 || dot(occ.normal, smp.direction) <= 0.0);
  if (is_param(c, mid) && lit) add_channel(color.d, 3 * mid, inc.v * (k * alpha / kPi));
  return color;
}

// One texel: gradient of sum_k,c dsh[k,c] SH[k,c] (baker.cpp:244-295).
void texel_grad(GradCtx& c, const shb_surface_point& sp, int samples, int sample_offset, uint32_t seed,
                uint32_t texel, const float* g, std::vector<double>& grad) {
  V3d P = pt_pos<double>(sp), N = pt_nrm<double>(sp);
  V3d T{(double)sp.tangent[0], (double)sp.tangent[1], (double)sp.tangent[2]};
  double Tw = sp.tangent[3];
  V3d origin = P + N * 0.001;
  const double inv = 1.0 / (double)samples;
  for (int s = 0; s < samples; ++s) {
    PhiloxRng rng{seed, texel, (uint32_t)(s + sample_offset)};
    auto hev = rng.event(0, EV_HEMI);
    float u1 = hev.u(0);
    float u2 = hev.u(1);
    double r = std::sqrt(1.0 - (double)u1 * (double)u1);
    double phi = 2.0 * kPi * (double)u2;
    V3d dl{r * std::cos(phi), r * std::sin(phi), (double)u1};
    V3d bitangent = cross(N, T) * Tw;
    V3d dw = T * dl.x + bitangent * dl.y + N * dl.z;
    // texel-level NEE (light.cpp:191-293): no BRDF, unnormalised direction
    {
      PhiloxEvent ev = rng.event(0, EV_NEE);
      size_t nl = c.s->lights.size();
      std::vector<LightEval<double>> evs(nl);
      std::vector<AreaSample<double>> ass(nl);
      std::vector<float> weights(nl);
      int area_ord = 0;
      for (size_t i = 0; i < nl; ++i) {
        const Lgt& L = c.s->lights[i];
        if (L.type == SHB_LIGHT_AREA) ass[i] = sample_area_light<double>(c.s, L, ev, 3 * area_ord++);
        evs[i] = incoming<double>(L, P, N, &ass[i]);
        weights[i] = (float)max_coeff(evs[i].radiance);
      }
      float sum = std::accumulate(weights.begin(), weights.end(), 0.0f);
      if (!(sum < 1e-6f)) {
        auto picker = ev.picker(weights, sum, 3 * area_ord);
        for (unsigned j = 0; j < c.nls; ++j) {
          int idx = picker.pick((int)j);
          const LightEval<double>& e = evs[idx];
          if (occluded(*c.bvh, e.ray_o, e.ray_d, e.tnear, e.tfar)) continue;
          double joint = (double)weights[idx] / (double)sum * e.area_pdf;
          if (joint < 1e-3) continue;
          LightDeriv ld = light_deriv(c, idx, P, ass[idx], e);
          if (ld.param < 0) continue;
          V3d a = sh_adjoint(g, e.ray_d, inv);
          V3d dLi = ld.dv / (joint * (double)c.nls);
          if (ld.light) grad[ld.param] += a.x * dLi.x + a.y * dLi.y + a.z * dLi.z;
          else {
            grad[ld.param] += a.x * dLi.x;
            grad[ld.param + 1] += a.y * dLi.y;
            grad[ld.param + 2] += a.z * dLi.z;
          }
        }
      }
    }
    Dual Li = trace_grad(c, rng, origin, dw, 0, 1);
    V3d a = sh_adjoint(g, dw, 2.0 * kPi * inv);
    for (int p = 0; p < c.P; ++p) grad[p] += a.x * Li.d[p].x + a.y * Li.d[p].y + a.z * Li.d[p].z;
  }
}

}  // namespace

// ================================================================ C API ===

extern "C" {

oracle_scene* oracle_scene_create(const shb_scene_desc* d) {
  auto* s = new oracle_scene();
  for (int i = 0; i < 256; ++i) s->srgb_lut[i] = srgb_to_linear((uint8_t)i);
  uint32_t prim = 0;
  for (uint32_t gi = 0; gi < d->geometry_count; ++gi) {
    const shb_geometry_desc& gd = d->geometries[gi];
    Geo g;
    uint32_t nv = gd.vertex_count;
    g.vertices.resize(nv);
    for (uint32_t v = 0; v < nv; ++v) g.vertices[v] = {gd.vertices[3 * v], gd.vertices[3 * v + 1], gd.vertices[3 * v + 2]};
    if (gd.normals) {
      g.normals.resize(nv);
      for (uint32_t v = 0; v < nv; ++v) g.normals[v] = {gd.normals[3 * v], gd.normals[3 * v + 1], gd.normals[3 * v + 2]};
    }
    if (gd.texture_uvs) {
      g.texture_uvs.resize(nv);
      for (uint32_t v = 0; v < nv; ++v) g.texture_uvs[v] = {gd.texture_uvs[2 * v], gd.texture_uvs[2 * v + 1]};
    }
    if (gd.lightmap_uvs) {
      g.lightmap_uvs.resize(nv);
      for (uint32_t v = 0; v < nv; ++v) g.lightmap_uvs[v] = {gd.lightmap_uvs[2 * v], gd.lightmap_uvs[2 * v + 1]};
    }
    if (gd.tangents) {
      g.tangents.resize(nv);
      for (uint32_t v = 0; v < nv; ++v)
        g.tangents[v] = {gd.tangents[4 * v], gd.tangents[4 * v + 1], gd.tangents[4 * v + 2], gd.tangents[4 * v + 3]};
    }
    g.indices.assign(gd.indices, gd.indices + gd.index_count);
    g.material_id = gd.material_id;
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) g.L[r * 3 + c] = gd.transform[r * 4 + c];
      g.t[r] = gd.transform[r * 4 + 3];
    }
    polar_rotation(g.L, g.Rot);
    // scene.cpp:162-195
    g.world_vertices.resize(nv);
    for (uint32_t v = 0; v < nv; ++v) {
      V3<float> m = mat_vec(g.L, g.vertices[v]);
      g.world_vertices[v] = {m.x + g.t[0], m.y + g.t[1], m.z + g.t[2]};
    }
    g.world_normals.resize(g.normals.size());
    for (size_t v = 0; v < g.normals.size(); ++v) g.world_normals[v] = normalized(mat_vec(g.Rot, g.normals[v]));
    g.world_tangents.resize(g.tangents.size());
    for (size_t v = 0; v < g.tangents.size(); ++v) {
      V3<float> tv{g.tangents[v].x, g.tangents[v].y, g.tangents[v].z};
      V3<float> r = normalized(mat_vec(g.Rot, tv));
      g.world_tangents[v] = {r.x, r.y, r.z, g.tangents[v].w};
    }
    g.prim_base = prim;
    uint32_t ntri = gd.index_count / 3;
    for (uint32_t t = 0; t < ntri; ++t) s->prim_geo.push_back(gi);
    prim += ntri;
    s->geos.push_back(std::move(g));
  }
  s->prim_count = prim;
  for (uint32_t mi = 0; mi < d->material_count; ++mi) {
    const shb_material_desc& md = d->materials[mi];
    Mat m;
    m.w = md.albedo_width;
    m.h = md.albedo_height;
    m.c = md.albedo_channels;
    if (md.albedo_pixels && m.w && m.h && m.c)
      m.pixels.assign(md.albedo_pixels, md.albedo_pixels + (size_t)m.w * m.h * m.c);
    m.emission = md.emission_intensity;
    s->mats.push_back(std::move(m));
  }
  for (uint32_t li = 0; li < d->light_count; ++li) {
    const shb_light_desc& ld = d->lights[li];
    Lgt L;
    L.type = ld.type;
    L.position = {ld.position[0], ld.position[1], ld.position[2]};
    L.direction = {ld.direction[0], ld.direction[1], ld.direction[2]};
    L.color = {ld.color[0], ld.color[1], ld.color[2]};
    L.intensity = ld.intensity;
    L.cos_inner = ld.cos_inner_cone;
    L.cos_outer = ld.cos_outer_cone;
    L.area = ld.area;
    L.material = ld.material_index;
    L.geometry = ld.geometry_index;
    s->lights.push_back(L);
  }
  return s;
}

void oracle_scene_destroy(oracle_scene* s) { delete s; }

// ------------------------------------------------------------ raster -----


// rasterizer.cpp:68-211, geometries in order (the reference runs them in
// parallel; writes to a shared texel race, so order is defined here as
// geometry-major, triangle-minor last writer).
int oracle_rasterize(const oracle_scene* s, const shb_raster_config* cfg, shb_surface_point* out) {
  int W = cfg->width * cfg->supersample_scale;
  int H = cfg->height * cfg->supersample_scale;
  if (W <= 0 || H <= 0) return 1;
  shb_surface_point empty;
  std::memset(&empty, 0, sizeof(empty));
  empty.material_id = -1;
  for (int64_t i = 0; i < (int64_t)W * H; ++i) out[i] = empty;
  for (const Geo& g : s->geos) {
    if (g.vertices.empty() || g.normals.empty() || g.tangents.empty()) return 2;
    if (g.lightmap_uvs.size() != g.vertices.size()) return 3;
    size_t tri_count = g.indices.size() / 3;
    for (size_t i = 0; i < tri_count; ++i) {
      uint32_t i0 = g.indices[i * 3], i1 = g.indices[i * 3 + 1], i2 = g.indices[i * 3 + 2];
      V2<float> uv0 = g.lightmap_uvs[i0], uv1 = g.lightmap_uvs[i1], uv2 = g.lightmap_uvs[i2];
      float min_u = std::min({uv0.x, uv1.x, uv2.x});
      float max_u = std::max({uv0.x, uv1.x, uv2.x});
      float min_v = std::min({uv0.y, uv1.y, uv2.y});
      float max_v = std::max({uv0.y, uv1.y, uv2.y});
      int min_x = std::max(0, cvt_trunc(min_u * W));
      int max_x = std::min(W - 1, cvt_trunc(std::ceil(max_u * W)));
      int min_y = std::max(0, cvt_trunc(min_v * H));
      int max_y = std::min(H - 1, cvt_trunc(std::ceil(max_v * H)));
      bool any = false;
      for (int y = min_y; y <= max_y; ++y) {
        for (int x = min_x; x <= max_x; ++x) {
          V2<float> p{(x + 0.5f) / W, (y + 0.5f) / H};
          float u, v, w;
          if (!barycentric(p, uv0, uv1, uv2, u, v, w)) continue;
          any = true;
          out[(int64_t)y * W + x] = make_point(g, i0, i1, i2, u, v, w);
        }
      }
      if (!any) {
        float cu = (uv0.x + uv1.x + uv2.x) / 3.0f;
        float cvv = (uv0.y + uv1.y + uv2.y) / 3.0f;
        int cx = cvt_trunc(cu * W);
        int cy = cvt_trunc(cvv * H);
        if (cx >= 0 && cx < W && cy >= 0 && cy < H) {
          int64_t pi = (int64_t)cy * W + cx;
          if (out[pi].material_id < 0) {
            float t = 1.0f / 3.0f;
            out[pi] = make_point(g, i0, i1, i2, t, t, t);
          }
        }
      }
    }
  }
  return 0;
}

void oracle_validity_mask(const shb_surface_point* pts, int64_t n, uint8_t* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = pts[i].material_id >= 0;
}

int oracle_downsample_validity_mask(const uint8_t* in, int w, int h, int scale, uint8_t* out) {
  int stride = w * scale;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      uint8_t any = 0;
      for (int sy = y * scale; sy < (y + 1) * scale && !any; ++sy)
        for (int sx = x * scale; sx < (x + 1) * scale; ++sx)
          if (in[(int64_t)sy * stride + sx]) { any = 1; break; }
      out[(int64_t)y * w + x] = any;
    }
  return 0;
}

void oracle_downsample(const float* in, int in_w, int in_h, int ch, int scale, float* out) {
  if (scale <= 1) {
    std::memcpy(out, in, sizeof(float) * (size_t)in_w * in_h * ch);
    return;
  }
  int ow = in_w / scale, oh = in_h / scale;
  std::vector<float> avg(ch);
  for (int y = 0; y < oh; ++y)
    for (int x = 0; x < ow; ++x) {
      std::fill(avg.begin(), avg.end(), 0.0f);
      int count = 0;
      for (int dy = 0; dy < scale; ++dy)
        for (int dx = 0; dx < scale; ++dx) {
          int sx = x * scale + dx, sy = y * scale + dy;
          if (sx < in_w && sy < in_h) {
            const float* p = in + ((int64_t)sy * in_w + sx) * ch;
            for (int c = 0; c < ch; ++c) avg[c] += p[c];
            count++;
          }
        }
      float* o = out + ((int64_t)y * ow + x) * ch;
      if (count > 0) {
        float inv = 1.f / float(count);
        for (int c = 0; c < ch; ++c) o[c] = avg[c] * inv;
      } else {
        for (int c = 0; c < ch; ++c) o[c] = 0.0f;
      }
    }
}


void oracle_dilate(int kind, int w, int h, void* pixels, uint8_t* mask, int passes) {
  if (kind == SHB_DILATE_SH9) dilate_t<float, 27>(w, h, (float*)pixels, mask, passes);
  else if (kind == SHB_DILATE_F32) dilate_t<float, 1>(w, h, (float*)pixels, mask, passes);
  else dilate_t<uint8_t, 1>(w, h, (uint8_t*)pixels, mask, passes);
}

void oracle_scene_set_params(oracle_scene* s, const float* albedo_rgb, const uint8_t* use_override,
                             const float* light_intensity) {
  if (albedo_rgb)
    for (size_t m = 0; m < s->mats.size(); ++m) {
      s->mats[m].use_override = (!use_override || use_override[m]) ? 1 : 0;
      for (int c = 0; c < 3; ++c) s->mats[m].ovr[c] = albedo_rgb[3 * m + c];
    }
  if (light_intensity)
    for (size_t l = 0; l < s->lights.size(); ++l) s->lights[l].intensity = light_intensity[l];
}

int oracle_bake_grad(const oracle_scene* s, const shb_surface_point* pts, const shb_raster_config* rc,
                     oracle_bake_args* a, const float* dsh, double* d_albedo, double* d_light) {
  if (a->samples <= 0 || !dsh) return 1;
  auto bvh = get_bvh<double>(s);
  const int64_t total = (int64_t)rc->width * rc->supersample_scale * rc->height * rc->supersample_scale;
  std::vector<int64_t> work;
  if (a->texel_subset) work.assign(a->texel_subset, a->texel_subset + a->subset_count);
  else {
    work.resize(total);
    std::iota(work.begin(), work.end(), 0);
  }
  const int n_mat3 = 3 * (int)s->mats.size();
  const int P = n_mat3 + (int)s->lights.size();
  int nthreads = a->threads > 0 ? a->threads : (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int64_t> next{0};
  std::vector<std::vector<double>> part((size_t)nthreads, std::vector<double>((size_t)P, 0.0));
  auto worker = [&](int t) {
    GradCtx c{s, bvh.get(), a->bounces, (unsigned)a->num_light_samples, n_mat3, P};
    while (true) {
      int64_t begin = next.fetch_add(8);
      if (begin >= (int64_t)work.size()) break;
      int64_t end = std::min<int64_t>(begin + 8, work.size());
      for (int64_t k = begin; k < end; ++k) {
        int64_t idx = work[k];
        if (idx < 0 || idx >= total || pts[idx].material_id < 0) continue;
        texel_grad(c, pts[idx], a->samples, a->sample_offset, a->seed, (uint32_t)idx, dsh + idx * 27, part[t]);
      }
    }
  };
  std::vector<std::thread> th;
  for (int i = 0; i < nthreads; ++i) th.emplace_back(worker, i);
  for (auto& t : th) t.join();
  for (int p = 0; p < P; ++p) {
    double v = 0.0;
    for (int t = 0; t < nthreads; ++t) v += part[t][p];
    if (p < n_mat3) d_albedo[p] = v;
    else d_light[p - n_mat3] = v;
  }
  return 0;
}

int oracle_bake(const oracle_scene* s, const shb_surface_point* pts, const shb_raster_config* raster,
                oracle_bake_args* a) {
  if (a->samples <= 0) return 1;
  if (a->fp64) return bake_impl<double>(s, pts, raster, a);
  return bake_impl<float>(s, pts, raster, a);
}

void oracle_find_occlusion(const oracle_scene* s, const shb_ray* rays, int64_t n, shb_hit* hits) {
  auto bvh = get_bvh<float>(s);
  for (int64_t i = 0; i < n; ++i) {
    const shb_ray& r = rays[i];
    Occ<float> o = find_occlusion<float>(s, *bvh, {r.origin[0], r.origin[1], r.origin[2]},
                                         {r.direction[0], r.direction[1], r.direction[2]}, r.tnear, r.tfar);
    shb_hit h;
    std::memset(&h, 0, sizeof(h));
    h.hit = o.hit;
    if (o.hit) {
      h.position[0] = o.position.x; h.position[1] = o.position.y; h.position[2] = o.position.z;
      h.uv[0] = o.uv.x; h.uv[1] = o.uv.y;
      h.normal[0] = o.normal.x; h.normal[1] = o.normal.y; h.normal[2] = o.normal.z;
      h.material_id = o.material_id;
      h.t = o.t;
      h.prim_id = o.prim;
    }
    hits[i] = h;
  }
}

void oracle_accumulate_radiance(const float radiance[3], const float dir[3], float out27[27]) {
  V3<float> acc[9];
  for (int i = 0; i < 9; ++i) acc[i] = {out27[i * 3], out27[i * 3 + 1], out27[i * 3 + 2]};
  accumulate_radiance<float>({radiance[0], radiance[1], radiance[2]}, {dir[0], dir[1], dir[2]}, acc);
  for (int i = 0; i < 9; ++i) {
    out27[i * 3] = acc[i].x;
    out27[i * 3 + 1] = acc[i].y;
    out27[i * 3 + 2] = acc[i].z;
  }
}

float oracle_srgb_to_linear(uint8_t x) { return srgb_to_linear(x); }

void oracle_get_albedo(const oracle_scene* s, int m, const float uv[2], float out[3]) {
  V3<float> a = get_albedo<float>(s->mats[m], {uv[0], uv[1]});
  out[0] = a.x; out[1] = a.y; out[2] = a.z;
}
float oracle_get_alpha(const oracle_scene* s, int m, const float uv[2]) {
  return get_alpha<float>(s->mats[m], {uv[0], uv[1]});
}
void oracle_get_emission(const oracle_scene* s, int m, const float uv[2], float out[3]) {
  V3<float> a = get_emission<float>(s->mats[m], {uv[0], uv[1]});
  out[0] = a.x; out[1] = a.y; out[2] = a.z;
}

void oracle_evaluate_light_samples(const oracle_scene* s, const float p[3], const float n[3],
                                   const float wo[3], int mat, const float uv[2], unsigned num_samples,
                                   uint32_t seed, int empty_bvh, float out[3]) {
  static const Bvh<float> kEmpty{};
  auto holder = empty_bvh ? std::shared_ptr<Bvh<float>>() : get_bvh<float>(s);
  const Bvh<float>* bvh = empty_bvh ? &kEmpty : holder.get();
  BakeCtx c{s, 0, num_samples};
  std::mt19937 g(seed);
  static const Mat kDefault{};
  const Mat& m = (mat >= 0 && mat < (int)s->mats.size()) ? s->mats[mat] : kDefault;
  V3<float> r = evaluate_light_samples<float>(c, *bvh, {p[0], p[1], p[2]}, {n[0], n[1], n[2]},
                                              {wo[0], wo[1], wo[2]}, m, {uv[0], uv[1]}, MtEvent{&g});
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

void oracle_sample_area_light(const oracle_scene* s, int light, uint32_t seed, float out10[10]) {
  std::mt19937 g(seed);
  MtEvent ev{&g};
  AreaSample<float> a = sample_area_light<float>(s, s->lights[light], ev, 0);
  float v[10] = {a.point.x, a.point.y, a.point.z, a.normal.x, a.normal.y, a.normal.z,
                 a.radiance.x, a.radiance.y, a.radiance.z, a.pdf};
  std::memcpy(out10, v, sizeof(v));
}

void oracle_light_radiance_unit_brdf(const oracle_scene* s, int light, const float p[3], const float n[3],
                                     float out_rad[3], shb_ray* out_ray) {
  const Lgt& L = s->lights[light];
  AreaSample<float> as;
  LightEval<float> e = incoming<float>(L, {p[0], p[1], p[2]}, {n[0], n[1], n[2]}, &as);
  V3<float> rad{};
  if (!(e.cos_n < 0.f)) rad = cmul(e.radiance, e.cos_n * V3<float>{1, 1, 1});
  out_rad[0] = rad.x; out_rad[1] = rad.y; out_rad[2] = rad.z;
  out_ray->origin[0] = e.ray_o.x; out_ray->origin[1] = e.ray_o.y; out_ray->origin[2] = e.ray_o.z;
  out_ray->direction[0] = e.ray_d.x; out_ray->direction[1] = e.ray_d.y; out_ray->direction[2] = e.ray_d.z;
  out_ray->tnear = e.tnear;
  out_ray->tfar = e.tfar;
}

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  philox10(ctr, key, out);
}

}  // extern "C"
