// shade.cu - wavefront stages of BakeSHLightMap (src/baker.cpp:186-304):
//   generate  one path per (texel, sample): uniform-hemisphere primary ray
//             and texel-level next-event estimation (src/light.cpp:191-293)
//   shade     per closest hit: alpha, emission, NEE with BRDF
//             (src/light.cpp:82-189), cosine BSDF sample (material.cpp:113-162)
//   resolve   one warp per texel: SH9 projection of every sample in
//             registers, warp-shuffle reduction, one coalesced store
// plus the host loop that drives the waves.  Compiled with -fmad=false so
// the arithmetic rounds like the CPU restatement.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "shb_math.cuh"
#include "wavefront.h"

namespace shb {

// sRGB -> linear table (constant memory; measured faster on the atrium
// than an L1-cached global table).
__constant__ float g_srgb[256];

namespace {

constexpr int kThreads = 256;
// Launch bounds of k_shade when next-event estimation runs in k_nee:
// SHB_SHADE_BLOCKS_PER_SM > 0 asks the compiler to fit that many resident
// blocks per SM, 4 by default (it then uses 64 registers, 56 without the
// bound; 1 % faster shading on the atrium).  With
// k_generate also held to 64 registers the atrium's shading measured 1.2 %
// faster but the room's (5 lights) 1.9 % slower, so k_generate follows
// SHB_GEN_BLOCKS_PER_SM (0: the compiler's choice).  The adjoint k_shade
// (SHB_BWD_BLOCKS_PER_SM) and the k_shade with next-event estimation inline
// are bounded to 2 blocks (at most 128 registers), the compiler's own
// choice for them: with a bound of 1 block the adjoint k_shade took 160
// registers and its backward pass ran 14 % slower.
#ifndef SHB_SHADE_BLOCKS_PER_SM
#define SHB_SHADE_BLOCKS_PER_SM 4
#endif
#ifndef SHB_BWD_BLOCKS_PER_SM
#define SHB_BWD_BLOCKS_PER_SM 2
#endif
#ifndef SHB_GEN_BLOCKS_PER_SM
#define SHB_GEN_BLOCKS_PER_SM 0
#endif
#if SHB_SHADE_BLOCKS_PER_SM > 0
#define SHB_SHADE_BOUNDS \
  __launch_bounds__(kThreads, BWD ? SHB_BWD_BLOCKS_PER_SM : (!SPLIT ? 2 : SHB_SHADE_BLOCKS_PER_SM))
#else
#define SHB_SHADE_BOUNDS __launch_bounds__(kThreads)
#endif
#if SHB_GEN_BLOCKS_PER_SM > 0
#define SHB_GEN_BOUNDS __launch_bounds__(kThreads, BWD ? SHB_BWD_BLOCKS_PER_SM : SHB_GEN_BLOCKS_PER_SM)
#else
#define SHB_GEN_BOUNDS __launch_bounds__(kThreads)
#endif
// Alpha branches per path kept apart for deterministic accumulation: the
// wave is shrunk by 2^min(bounces, kMaxBranchLog).  Branch slots beyond that
// (more than six transmissive bounces) fall back to atomic accumulation.
constexpr int kMaxBranchLog = 6;
// Light-loop cost from which the forward bake runs next-event estimation as
// a kernel of its own (k_nee): punctual lights count 1, area lights 4 (each
// samples a triangle and a point and looks up its emission).
constexpr uint32_t kSplitNeeCost = 16;
// Adjoint limits: the per-block gradient accumulator lives in shared memory
// (3 x materials + lights floats) and a throughput tangent list holds at
// most one entry per bounce.
constexpr size_t kMaxGradSmem = 48 * 1024;
constexpr int kMaxTangents = 16;
constexpr double kTwoPiD = 6.283185307179586;

struct MatInfo {
  f3 albedo_over_pi;
  float alpha;
  f3 emission;
};

__device__ __forceinline__ DMat load_mat(const SceneView& sc, int id) {
  if (id < 0 || (uint32_t)id >= sc.mat_count) {
    DMat d;
    d.pix_offset = 0;
    d.w = d.h = d.c = 0;
    d.emission = 0.f;
    d.use_override = 0;
    d.override_rgb[0] = d.override_rgb[1] = d.override_rgb[2] = 0.f;
    d.pad = 0.f;
    return d;
  }
  return sc.mats[id];
}

__device__ __forceinline__ int tex_index(const DMat& m, f2 uv) {
  int tx = min(max(cvt_trunc(uv.x * (float)m.w), 0), (int)m.w - 1);
  int ty = min(max(cvt_trunc(uv.y * (float)m.h), 0), (int)m.h - 1);
  return (ty * (int)m.w + tx) * (int)m.c;
}

// src/material.cpp:69-85
__device__ __forceinline__ f3 get_albedo(const SceneView& sc, const DMat& m, f2 uv) {
  if (m.use_override) return {m.override_rgb[0], m.override_rgb[1], m.override_rgb[2]};
  if (m.c == 0) return {0.8f, 0.8f, 0.8f};
  const uint8_t* px = sc.pixels + m.pix_offset + tex_index(m, uv);
  return {g_srgb[px[0]], g_srgb[px[1]], g_srgb[px[2]]};
}
// src/material.cpp:57-67
__device__ __forceinline__ float get_alpha(const SceneView& sc, const DMat& m, f2 uv) {
  if (m.c < 4) return 1.0f;
  const uint8_t* px = sc.pixels + m.pix_offset + tex_index(m, uv);
  return (float)px[3] / 255.0f;
}
// src/material.cpp:87-92
__device__ __forceinline__ f3 get_emission(const SceneView& sc, const DMat& m, f2 uv) {
  if (m.emission > 0.0f) return get_albedo(sc, m, uv) * m.emission;
  return {0.f, 0.f, 0.f};
}

// std::max(a.x, std::max(a.y, a.z)) with std::max(a, b) = a < b ? b : a.
__device__ __forceinline__ float max_coeff_std(f3 a) {
  float m = a.y < a.z ? a.z : a.y;
  return a.x < m ? m : a.x;
}

// Area-light triangle records (built once per scene by build_area_tris):
// float4 {v0, pdf}, {v1, uv0.x}, {v2, uv0.y}, {uv1, uv2} with object-space
// vertices and pdf = max(1e-6, 1 / (n * area)) computed by the expressions
// of SampleAreaLight, so a sample reads one 64-byte record instead of the
// index, vertex and uv gathers.  The light record carries its first record
// and its triangle count | has-texture-uv << 31.
constexpr uint32_t kAreaHasUv = 0x80000000u;
// 1: the record's uv float4 is read only by a sample that looks up a
// textured emission (an emitter of constant emission never reads it);
// 0: all four are read up front.
#ifndef SHB_AREA_UV_LATE
#define SHB_AREA_UV_LATE 1
#endif
constexpr bool kAreaUvLate = SHB_AREA_UV_LATE != 0;

__device__ __forceinline__ float area_pdf(f3 v0, f3 v1, f3 v2, uint32_t n) {
  float area = sqrtf(sqnorm(cross(v0 - v1, v0 - v2))) / 2.f;
  float x = 1.f / (float)n * 1.f / area;
  return 1e-6f < x ? x : 1e-6f;
}

// src/light.cpp:16-78; uniforms ubase (triangle), ubase+1, ubase+2.
__device__ void sample_area(const SceneView& sc, const DLight& L, Event& ev, int ubase, f3& point, f3& rad,
                            float& pdf) {
  point = {0.f, 0.f, 0.f};
  rad = {0.f, 0.f, 0.f};
  pdf = 0.f;
  if (L.geom < 0 || L.mat < 0) return;
  const uint32_t n = L.area_count & ~kAreaHasUv;
  if (n == 0) return;
  uint32_t tri = ev.tri(ubase, n);
  const float4* r = sc.area_tris + 4 * ((size_t)L.area_first + tri);
  const float4 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2);
  float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
  if (!kAreaUvLate) d = __ldg(r + 3);
  float u1 = ev.u(ubase + 1);
  float u2 = ev.u(ubase + 2);
  if (u1 + u2 > 1.0f) {
    u1 = 1.0f - u1;
    u2 = 1.0f - u2;
  }
  float w = 1.0f - u1 - u2;
  f3 v0 = {a.x, a.y, a.z}, v1 = {b.x, b.y, b.z}, v2 = {c.x, c.y, c.z};
  point = w * v0 + u1 * v1 + u2 * v2;
  if (L.emis_const) {
    rad = {L.er, L.eg, L.eb};
  } else {
    f2 uv = {0.f, 0.f};
    if (L.area_count & kAreaHasUv) {
      if (kAreaUvLate) d = __ldg(r + 3);
      uv = w * f2{b.w, c.w} + u1 * f2{d.x, d.y} + u2 * f2{d.z, d.w};
    }
    rad = get_emission(sc, load_mat(sc, L.mat), uv);
  }
  pdf = a.w;
}

// entries: (global triangle, triangle count of its light, has uv, 0)
__global__ void k_area_tris(SceneView sc, const uint4* __restrict__ entries, int count, float4* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint4 e = entries[i];
    const uint32_t p = e.x;
    const uint32_t i0 = sc.tri_vidx[3 * p], i1 = sc.tri_vidx[3 * p + 1], i2 = sc.tri_vidx[3 * p + 2];
    const f3 v0 = ld3(sc.obj_v, i0), v1 = ld3(sc.obj_v, i1), v2 = ld3(sc.obj_v, i2);
    f2 t0 = {0.f, 0.f}, t1 = t0, t2 = t0;
    if (e.z) {
      t0 = ld2(sc.tex_uv, i0);
      t1 = ld2(sc.tex_uv, i1);
      t2 = ld2(sc.tex_uv, i2);
    }
    out[4 * (size_t)i] = make_float4(v0.x, v0.y, v0.z, area_pdf(v0, v1, v2, e.y));
    out[4 * (size_t)i + 1] = make_float4(v1.x, v1.y, v1.z, t0.x);
    out[4 * (size_t)i + 2] = make_float4(v2.x, v2.y, v2.z, t0.y);
    out[4 * (size_t)i + 3] = make_float4(t1.x, t1.y, t2.x, t2.y);
  }
}

struct LightEval {
  f3 rad;
  f3 ray_d;
  float tfar;
  float apdf;
  float w;
  // Adjoint only (BWD): light index; d rad / d(light parameter) per channel
  // (point/spot/directional: intensity, lpar = 1; area: the emissive
  // material's linear albedo, pmat >= 0 when that material is a parameter);
  // d rad_c / d albedo_c of the receiving material (HIT).
  uint32_t idx;
  int lpar, pmat;
  f3 dpar, dalb;
};

// Incoming radiance without visibility (src/light.h:34-49,72-95,117-144,
// 166-188); with HIT, times cos x BRDF (src/light.h:51-203).
template <bool HIT, bool BWD = false>
__device__ LightEval eval_light(const SceneView& sc, const DLight* lights, uint32_t li, f3 P, f3 N, Event& ev,
                                bool wo_back, f3 aop) {
  const DLight& L = lights[li];
  LightEval e;
  e.apdf = 1.0f;
  if (BWD) {
    e.idx = li;
    e.lpar = 0;
    e.pmat = -1;
    e.dpar = {0.f, 0.f, 0.f};
    e.dalb = {0.f, 0.f, 0.f};
  }
  f3 color = {L.cr, L.cg, L.cb};
  float cos_n;
  f3 incident;
  if (L.type == SHB_LIGHT_DIRECTIONAL) {
    f3 dir = {L.dx, L.dy, L.dz};
    e.ray_d = -dir;
    e.tfar = 1.0e10f;
    cos_n = dot(N, -dir);
    incident = -dir;
    e.rad = cos_n < 0.f ? f3{0.f, 0.f, 0.f} : L.intensity * color;
    if (BWD) {
      e.lpar = 1;
      e.dpar = cos_n < 0.f ? f3{0.f, 0.f, 0.f} : color;
    }
  } else if (L.type == SHB_LIGHT_POINT || L.type == SHB_LIGHT_SPOT || L.type == SHB_LIGHT_AREA) {
    f3 target, arad = {0.f, 0.f, 0.f};
    if (L.type == SHB_LIGHT_AREA) sample_area(sc, L, ev, 3 * L.area_ord, target, arad, e.apdf);
    else target = {L.px, L.py, L.pz};
    f3 Lv = target - P;
    float dist_sq = sqnorm(Lv);
    float dist = sqrtf(dist_sq);
    e.ray_d = target - P;
    e.tfar = dist - 0.001f;
    Lv = Lv / dist;
    incident = Lv;
    cos_n = dot(N, Lv);
    if (L.type == SHB_LIGHT_POINT) {
      e.rad = cos_n < 0.f ? f3{0.f, 0.f, 0.f} : L.intensity * color / (dist * dist);
      if (BWD) {
        e.lpar = 1;
        e.dpar = cos_n < 0.f ? f3{0.f, 0.f, 0.f} : color / (dist * dist);
      }
    } else if (L.type == SHB_LIGHT_SPOT) {
      float cos_l = dot(f3{L.dx, L.dy, L.dz}, -Lv);
      float falloff = (cos_l - L.cos_outer) / (L.cos_inner - L.cos_outer);
      falloff = fminf(fmaxf(falloff, 0.0f), 1.0f);
      e.rad = cos_n < 0.f ? f3{0.f, 0.f, 0.f} : L.intensity * color / (dist * dist) * falloff;
      if (BWD) {
        e.lpar = 1;
        e.dpar = cos_n < 0.f ? f3{0.f, 0.f, 0.f} : color / (dist * dist) * falloff;
      }
    } else {
      e.rad = cos_n < 0.f ? f3{0.f, 0.f, 0.f} : arad / (dist * dist);
      if (BWD && L.mat >= 0 && (uint32_t)L.mat < sc.mat_count) {
        const DMat& em = sc.mats[L.mat];
        if (em.use_override && em.emission > 0.0f && cos_n >= 0.f) {
          e.pmat = L.mat;
          e.dpar = f3{em.emission, em.emission, em.emission} / (dist * dist);
        }
      }
    }
  } else {
    e.rad = {0.f, 0.f, 0.f};
    e.ray_d = {0.f, 0.f, 1.f};
    e.tfar = 0.f;
    cos_n = -1.f;
    incident = {0.f, 0.f, 1.f};
  }
  if (HIT) {
    if (cos_n < 0.f) {
      e.rad = {0.f, 0.f, 0.f};
      if (BWD) e.dpar = {0.f, 0.f, 0.f};
    } else {
      bool zero = wo_back || dot(N, incident) <= 0.0f;
      f3 brdf = zero ? f3{0.f, 0.f, 0.f} : aop;
      if (BWD) {
        e.dpar = cmul(e.dpar, cos_n * brdf);
        e.dalb = zero ? f3{0.f, 0.f, 0.f} : e.rad * (cos_n / 3.14159265358979323846f);
      }
      e.rad = cmul(e.rad, cos_n * brdf);
    }
  }
  e.w = max_coeff_std(e.rad);
  return e;
}

// One light pick of the discrete distribution over weights (the counter
// stream's uniform `u` against the running float sum; zero-weight lights
// are never picked).
// Weights of up to kWeightCache lights are kept from the summing pass, so
// the pick only re-evaluates the chosen light; beyond that every light is
// re-evaluated (same values either way: evaluation is deterministic).  The
// cache of a thread is wcache[i * ws]: a local array (ws 1) or the thread's
// column of a block-wide array in shared memory (ws = threads per block).
// `lights` is the bake's light table in global memory or the block's copy
// of it in shared memory.
constexpr uint32_t kWeightCache = 32;
// 1: the picked light is evaluated after the weight scan (one convergent
// evaluation per warp); 0: inside the scan, where the lane's pick is found.
#ifndef SHB_PICK_AFTER_LOOP
#define SHB_PICK_AFTER_LOOP 1
#endif
constexpr bool kPickAfterLoop = SHB_PICK_AFTER_LOOP != 0;
// The same for the adjoint's picks (whose light evaluation carries the
// parameter derivatives).
#ifndef SHB_PICK_AFTER_LOOP_BWD
#define SHB_PICK_AFTER_LOOP_BWD 1
#endif
// Texel next-event estimation shares the punctual lights' weights across a
// warp of one texel's samples also in scenes with area lights.
#ifndef SHB_TEXEL_COOP_AREA
#define SHB_TEXEL_COOP_AREA 1
#endif

template <bool HIT, bool BWD = false>
__device__ bool pick_light(const SceneView& sc, const DLight* lights, f3 P, f3 N, Event& ev, bool wo_back, f3 aop,
                           float sum,
                           float u, const float* wcache, int ws, LightEval& out) {
  float target = u * sum;
  float cum = 0.f;
  int last = -1;
  const bool cached = sc.light_count <= kWeightCache;
  if (cached && kPickAfterLoop && (!BWD || SHB_PICK_AFTER_LOOP_BWD)) {
    // Find the index first and evaluate the picked light once, after the
    // loop: evaluated inside it, the warp would run the evaluation once for
    // every distinct pick among its lanes, each time with those lanes only.
    int pick = -1;
    for (uint32_t i = 0; i < sc.light_count; ++i) {
      const float w = wcache[i * ws];
      cum += w;
      if (w > 0.f) last = (int)i;
      if (target < cum) {
        pick = (int)i;
        break;
      }
    }
    if (pick < 0) pick = last;
    if (pick < 0) return false;
    out = eval_light<HIT, BWD>(sc, lights, (uint32_t)pick, P, N, ev, wo_back, aop);
    return true;
  }
  for (uint32_t i = 0; i < sc.light_count; ++i) {
    float w;
    LightEval e;
    if (cached) {
      w = wcache[i * ws];
    } else {
      e = eval_light<HIT, BWD>(sc, lights, i, P, N, ev, wo_back, aop);
      w = e.w;
    }
    cum += w;
    if (w > 0.f) last = (int)i;
    if (target < cum) {
      out = cached ? eval_light<HIT, BWD>(sc, lights, i, P, N, ev, wo_back, aop) : e;
      return true;
    }
  }
  if (last < 0) return false;
  out = eval_light<HIT, BWD>(sc, lights, (uint32_t)last, P, N, ev, wo_back, aop);
  return true;
}

template <bool HIT>
__device__ float light_weight_sum(const SceneView& sc, const DLight* lights, f3 P, f3 N, Event& ev, bool wo_back,
                                  f3 aop,
                                  float* wcache, int ws) {
  float sum = 0.0f;
  const bool cached = sc.light_count <= kWeightCache;
  for (uint32_t i = 0; i < sc.light_count; ++i) {
    float w = eval_light<HIT>(sc, lights, i, P, N, ev, wo_back, aop).w;
    if (cached) wcache[i * ws] = w;
    sum += w;
  }
  return sum;
}

// Forward next-event kernels keep the light table of a one-bake wave in
// shared memory (measured 3 % faster shading on the atrium than reading the
// records through L1; a per-thread weight cache in shared memory, 3 % slower
// than the local array, is not used).
constexpr uint32_t kSmemLights = 64;

// The table of bake `bake` in the block's shared copy `s` when the wave has
// one bake and few enough lights, else the global table.  Every thread of
// the block calls this once, before any early exit.
__device__ __forceinline__ const DLight* stage_lights(const BakeItem* bakes, int bake, DLight* s) {
  if (bake < 0) return nullptr;
  const SceneView& sc = bakes[bake].sc;
  if (sc.light_count > kSmemLights) return sc.lights;
  const uint32_t* src = reinterpret_cast<const uint32_t*>(sc.lights);
  uint32_t* dst = reinterpret_cast<uint32_t*>(s);
  const uint32_t words = sc.light_count * (uint32_t)(sizeof(DLight) / 4);
  for (uint32_t k = threadIdx.x; k < words; k += blockDim.x) dst[k] = __ldg(src + k);
  __syncthreads();
  return s;
}

// Dynamic shared memory of the forward next-event kernels: the staged light
// table.
constexpr size_t kNeeSmemBytes = kSmemLights * sizeof(DLight);

// Warp-aggregated queue slot: every lane of the warp must call this.
__device__ __forceinline__ int warp_push(int* counter, bool pred) {
  unsigned b = __ballot_sync(0xFFFFFFFFu, pred);
  if (b == 0) return -1;
  int lane = threadIdx.x & 31;
  int leader = __ffs(b) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(b));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  return pred ? base + __popc(b & ((1u << lane) - 1u)) : -1;
}

struct SP {
  f3 pos, nrm, tan;
  float tw;
  int mat;
};
__device__ __forceinline__ SP load_sp(const shb_surface_point* pts, uint32_t texel) {
  const float4* q = reinterpret_cast<const float4*>(pts + texel);
  float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
  SP s;
  s.pos = {a.x, a.y, a.z};
  s.nrm = {a.w, b.x, b.y};
  s.tan = {c.x, c.y, c.z};
  s.tw = c.w;
  s.mat = __float_as_int(d.x);
  return s;
}

// src/baker.cpp:38-46,266-271
__device__ __forceinline__ f3 primary_dir(const SP& sp, uint32_t seed, uint32_t texel, uint32_t sample) {
  Event e;
  e.init(seed, texel, sample, 0, EV_HEMI);
  float u1 = e.u(0), u2 = e.u(1);
  float r = sqrtf(1.0f - u1 * u1);
  float phi = (float)(kTwoPiD * (double)u2);
  f3 dl = {r * cosf(phi), r * sinf(phi), u1};
  f3 bit = cross(sp.nrm, sp.tan) * sp.tw;
  return sp.tan * dl.x + bit * dl.y + sp.nrm * dl.z;
}

struct WaveArgs {
  const BakeItem* bakes;  // device table
  int n_bakes;
  int one_bake;           // the one bake of this wave's tiles, else -1
  const Tile* tiles;      // this wave's tiles (device)
  int n_tiles;
  int64_t P;              // paths in the wave
  int64_t n_tex;          // texels in the wave
  int NLS;                // max num_light_samples over the batch (NEE slot stride)
  ExtQueue ext[2];
  float4* hits;
  ShadowQueue sh;
  PathInfo* info;
  float4* path_L;
  float4* nee_li;
  float4* nee_dir;
  int* cnt;
  int ext_cap;  // capacity of each extend queue
  int sh_cap;   // capacity of the shadow queue
  // With several light samples or alpha branching a path gets more than one
  // hit-NEE contribution per depth; they then go to fixed slots
  // (path, branch, sample) and k_commit adds them in that order, so results
  // do not depend on atomic ordering.
  int det;
  int slots;    // branch slots per path (1 without alpha)
  float4* pend;
  // Forward bake: k_shade leaves one next-event record per opaque hit,
  // five float4 planes of ext_cap entries: (position, path), (normal,
  // vertex), (ray direction, alpha), (albedo / pi, beta.x), (beta.yz).
  float4* nee_rec;
  // Adjoint (path replay).  path_L holds each path's adjoint weight
  // dLoss/dL (RGB).  Every extend-queue entry carries the forward-mode
  // tangent of its throughput, d beta_c / d albedo_{m,c}, as a list of
  // (rgb, material) float4 in tan[queue][k * ext_cap + i], k < beta.w bits.
  // Every shadow ray carries a gradient packet pk[k * sh_cap + slot],
  // k < count in pend[slot].x bits: (value rgb, parameter) per material or
  // (value, 0, 0, light | kLightFlag); k_shadow clears the count when the
  // ray is occluded and k_apply adds the visible packets.
  const float* dsh;   // dLoss/dSH of the bake, 27 per texel
  float4* tan[2];
  float4* pk;
  int ntan, npk;
  int n_mat3;         // 3 * mat_count: first light parameter
  int n_params;       // 3 * mat_count + light_count
  double* grad;
};

constexpr uint32_t kLightFlag = 0x80000000u;

// sum_k g[3k + c] Y_k(d): the adjoint of sh_accumulate for one direction.
__device__ __forceinline__ f3 sh_adjoint(const float* __restrict__ g, f3 d) {
  const float x = d.x, y = d.y, z = d.z;
  float sh[9];
  sh[0] = 0.282095f;
  sh[1] = 0.488603f * y;
  sh[2] = 0.488603f * z;
  sh[3] = 0.488603f * x;
  sh[4] = 1.092548f * x * y;
  sh[5] = 1.092548f * y * z;
  sh[6] = 0.315392f * (3.0f * z * z - 1.0f);
  sh[7] = 1.092548f * x * z;
  sh[8] = 0.546274f * (x * x - y * y);
  f3 a = {0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    a.x += __ldg(g + 3 * i) * sh[i];
    a.y += __ldg(g + 3 * i + 1) * sh[i];
    a.z += __ldg(g + 3 * i + 2) * sh[i];
  }
  return a;
}

// Warp-aggregated gradient add into the block's shared accumulator: lanes
// holding the same parameter are summed with shuffles and one lane adds the
// sum.  Every lane of the warp must call this.
__device__ __forceinline__ void warp_grad_add(float* sg, int pid, float v, bool act) {
  const int lane = threadIdx.x & 31;
  unsigned pending = __ballot_sync(0xFFFFFFFFu, act && v != 0.f);
  while (pending) {
    const int leader = __ffs(pending) - 1;
    const int key = __shfl_sync(0xFFFFFFFFu, pid, leader);
    const bool mine = ((pending >> lane) & 1u) && pid == key;
    float sum = mine ? v : 0.f;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, off);
    if (lane == leader) atomicAdd(sg + key, sum);
    pending &= ~__ballot_sync(0xFFFFFFFFu, mine);
  }
}

// One packet entry: material m adds rgb to parameters 3m..3m+2, light l
// adds x to parameter n_mat3 + l.  Every lane of the warp must call this.
__device__ __forceinline__ void warp_grad_entry(float* sg, const WaveArgs& a, float4 e, bool act) {
  const uint32_t id = __float_as_uint(e.w);
  const bool light = (id & kLightFlag) != 0u;
  const int p0 = light ? a.n_mat3 + (int)(id & ~kLightFlag) : 3 * (int)id;
  act = act && p0 >= 0 && p0 + (light ? 0 : 2) < a.n_params;
  warp_grad_add(sg, p0, e.x, act);
  warp_grad_add(sg, p0 + 1, e.y, act && !light);
  warp_grad_add(sg, p0 + 2, e.z, act && !light);
}

__device__ __forceinline__ void grad_zero(float* sg, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) sg[i] = 0.f;
  __syncthreads();
}
__device__ __forceinline__ void grad_flush(const float* sg, int n, double* g) {
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    if (sg[i] != 0.f) atomicAdd(g + i, (double)sg[i]);
}

// Queue slot within capacity, else the error flag is raised and the ray dropped.
__device__ __forceinline__ bool slot_ok(const WaveArgs& a, int slot, int cap) {
  if (slot < cap) return true;
  atomicOr(a.cnt + CNT_ERROR, ERR_QUEUE);
  return false;
}

// Tile containing wave position `x` (a path when BY_PATH, else a texel).
template <bool BY_PATH>
__device__ __forceinline__ int find_tile(const WaveArgs& a, int64_t x) {
  int lo = 0, hi = a.n_tiles;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    int64_t off = BY_PATH ? a.tiles[mid].path_off : a.tiles[mid].tex_off;
    if (off <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ------------------------------------------------------------- generate --
template <bool BWD>
__global__ void SHB_GEN_BOUNDS k_generate(WaveArgs a) {
  extern __shared__ float dyn_smem[];
  const DLight* wave_lights = BWD ? nullptr : stage_lights(a.bakes, a.one_bake, reinterpret_cast<DLight*>(dyn_smem));
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t warp_id = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  for (int64_t base = warp_id * 32; base < a.P; base += warps * 32) {
    int64_t p = base + lane;
    bool active = p < a.P;
    f3 o = {0.f, 0.f, 0.f}, dw = {0.f, 0.f, 1.f}, P0 = o, N = o;
    uint32_t texel = 0, sample = 0, b = 0;
    const BakeItem* B = a.bakes;
    const float* g = nullptr;
    float inv = 0.f;
    if (active) {
      const Tile t = a.tiles[find_tile<true>(a, p)];
      b = t.bake;
      B = a.bakes + b;
      int64_t local = p - t.path_off;
      uint32_t slot = t.t0 + (uint32_t)(local / t.spp);
      sample = (uint32_t)(local % t.spp) + B->sample_offset;
      texel = B->valid[slot];
      SP sp = load_sp(B->pts, texel);
      P0 = sp.pos;
      N = sp.nrm;
      dw = primary_dir(sp, B->seed, texel, sample);
      o = sp.pos + sp.nrm * 0.001f;
      a.info[p] = make_uint4(b, texel, sample, 0u);
      if (BWD) {
        // dLoss/dL of this path: sh_out = (1/spp) sum 2pi L Y(dw) (k_resolve)
        g = a.dsh + (int64_t)texel * 27;
        inv = 1.0f / (float)t.spp;
        f3 adj = sh_adjoint(g, dw) * ((float)kTwoPiD * inv);
        a.path_L[p] = make_float4(adj.x, adj.y, adj.z, 0.f);
      } else {
        a.path_L[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a.det)
          for (int k = 0; k < a.slots * a.NLS; ++k) a.pend[p * a.slots * a.NLS + k] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    // texel-level NEE (src/light.cpp:191-293), origin without offset
    Event ev;
    ev.init(active ? B->seed : 0u, texel, sample, 0, EV_NEE);
    const f3 zero3 = {0.f, 0.f, 0.f};
    float wcache[kWeightCache];
    const int ws = 1;
    const DLight* lights = wave_lights ? wave_lights : B->sc.lights;
    float sum = 0.f;
    // The weights of point, spot and directional lights depend on the texel
    // only.  When the warp's paths all belong to one texel (spp >= 32
    // mostly), lane j evaluates light j if it is one of those and the lanes
    // share the weights by shuffle; area lights, which sample a point per
    // path, are evaluated by every lane for its own path.  Each lane still
    // sums the weights in light order, so the result is the same.
    const unsigned act = __ballot_sync(0xFFFFFFFFu, active);
    const uint64_t key = active ? ((uint64_t)b << 32 | texel) : ~0ull;
    const int lead = act ? __ffs(act) - 1 : 0;
    const uint64_t key0 = __shfl_sync(0xFFFFFFFFu, key, lead);
    const bool coop = act && __all_sync(0xFFFFFFFFu, !active || (key == key0 &&
                                                                 (SHB_TEXEL_COOP_AREA || B->sc.area_light_count == 0) &&
                                                                 B->sc.light_count <= kWeightCache));
    if (coop) {
      const BakeItem* BL = a.bakes + (uint32_t)(key0 >> 32);
      const f3 Pl = {__shfl_sync(0xFFFFFFFFu, P0.x, lead), __shfl_sync(0xFFFFFFFFu, P0.y, lead),
                     __shfl_sync(0xFFFFFFFFu, P0.z, lead)};
      const f3 Nl = {__shfl_sync(0xFFFFFFFFu, N.x, lead), __shfl_sync(0xFFFFFFFFu, N.y, lead),
                     __shfl_sync(0xFFFFFFFFu, N.z, lead)};
      const uint32_t nl = BL->sc.light_count;
      const DLight* ll = wave_lights ? wave_lights : BL->sc.lights;
      const float mine = (uint32_t)lane < nl && ll[lane].type != SHB_LIGHT_AREA
                             ? eval_light<false>(BL->sc, ll, (uint32_t)lane, Pl, Nl, ev, true, zero3).w
                             : 0.f;
      for (uint32_t i = 0; i < nl; ++i) {
        float w;
        if (ll[i].type != SHB_LIGHT_AREA) w = __shfl_sync(0xFFFFFFFFu, mine, (int)i);
        else w = active ? eval_light<false>(BL->sc, ll, i, P0, N, ev, true, zero3).w : 0.f;
        wcache[i * ws] = w;
        sum += w;
      }
      if (!active) sum = 0.f;
    } else if (active) {
      sum = light_weight_sum<false>(B->sc, lights, P0, N, ev, true, zero3, wcache, ws);
    }
    bool any_light = active && !(sum < 1e-6f);
    const int nls = active ? B->nls : 0;
    for (int j = 0; j < a.NLS; ++j) {
      LightEval e;
      bool ok = false;
      float joint = 1.f;
      if (any_light && j < nls) {
        ok = pick_light<false, BWD>(B->sc, lights, P0, N, ev, true, zero3, sum,
                                    ev.u(3 * (int)B->sc.area_light_count + j), wcache, ws, e);
        if (ok) {
          float pdf = e.w / sum;
          joint = pdf * e.apdf;
          ok = !(joint < 1e-3f);
          if (ok && !BWD) {
            f3 Li = e.rad / (joint * (float)nls);
            a.nee_li[p * a.NLS + j] = make_float4(Li.x, Li.y, Li.z, 0.f);
            a.nee_dir[p * a.NLS + j] = make_float4(e.ray_d.x, e.ray_d.y, e.ray_d.z, 0.f);
          }
        }
      }
      if (!BWD && active && !ok) a.nee_li[p * a.NLS + j] = make_float4(0.f, 0.f, 0.f, 0.f);
      int slot = warp_push(a.cnt + CNT_SHADOW, ok);
      if (ok && slot_ok(a, slot, a.sh_cap)) {
        a.sh.o[slot] = make_float4(P0.x, P0.y, P0.z, e.tfar);
        if (BWD) {
          // Li = rad / (joint nls) projected along the unnormalised ray
          // direction (k_resolve); the selection pdf is held constant.
          f3 adj = sh_adjoint(g, e.ray_d) * inv;
          const float k = 1.0f / (joint * (float)nls);
          uint32_t n = 0;
          if (e.lpar) {
            a.pk[(int64_t)n++ * a.sh_cap + slot] =
                make_float4(dot(adj, e.dpar) * k, 0.f, 0.f, __uint_as_float(e.idx | kLightFlag));
          } else if (e.pmat >= 0) {
            f3 v = cmul(adj, e.dpar) * k;
            a.pk[(int64_t)n++ * a.sh_cap + slot] = make_float4(v.x, v.y, v.z, __uint_as_float((uint32_t)e.pmat));
          }
          a.pend[slot] = make_float4(__uint_as_float(n), 0.f, 0.f, 0.f);
          a.sh.d[slot] = make_float4(e.ray_d.x, e.ray_d.y, e.ray_d.z, __uint_as_float((uint32_t)slot));
          a.sh.c[slot] = make_float4(0.f, 0.f, 0.f, __uint_as_float(2u | (b << 2)));
        } else {
          a.sh.d[slot] = make_float4(e.ray_d.x, e.ray_d.y, e.ray_d.z, __uint_as_float((uint32_t)(p * a.NLS + j)));
          a.sh.c[slot] = make_float4(0.f, 0.f, 0.f, __uint_as_float(1u | (b << 2)));
        }
      }
    }
    int slot = warp_push(a.cnt + CNT_EXT0, active);
    if (active && slot_ok(a, slot, a.ext_cap)) {
      a.ext[0].o[slot] = make_float4(o.x, o.y, o.z, __uint_as_float((uint32_t)p));
      a.ext[0].d[slot] = make_float4(dw.x, dw.y, dw.z, __uint_as_float(1u));
      a.ext[0].beta[slot] = make_float4(1.f, 1.f, 1.f, 0.f);  // w: tangent count 0
    }
  }
}

// --------------------------------------------------------------- shade ---
// Next-event estimation at a path vertex (src/light.cpp:82-189): the light
// weights, NLS picks and one shadow-queue entry per visible candidate.  All
// lanes of the warp call it (queue pushes are warp-aggregated); lanes with
// opaque_hit false take part without work.  BWD adds the gradient packets.
template <bool BWD>
__device__ __forceinline__ void nee_hit(const WaveArgs& a, const BakeItem* B, uint32_t b, f3 hit_pos, f3 N, f3 wo,
                                        f3 aop, f3 beta, float alpha, uint32_t path, uint32_t vertex,
                                        uint32_t texel, uint32_t sample, int depth, bool opaque_hit, uint32_t ntan,
                                        f3 adj, bool param, int mat_id, int cur, int i, const DLight* lights) {
  Event ev;
  ev.init(opaque_hit ? B->seed : 0u, texel, sample, vertex, EV_NEE);
  float wcache[kWeightCache];
  const int ws = 1;
  // dot(N, wo) <= 0 zeroes the BRDF of every light alike: evaluated once
  const bool wo_back = dot(N, wo) <= 0.0f;
  float sum = opaque_hit ? light_weight_sum<true>(B->sc, lights, hit_pos, N, ev, wo_back, aop, wcache, ws) : 0.f;
  bool any_light = opaque_hit && !(sum < 1e-6f);
  const int nls = opaque_hit ? B->nls : 0;
  for (int j = 0; j < a.NLS; ++j) {
    LightEval e;
    bool ok = false;
    f3 c = {0.f, 0.f, 0.f};
    float scale = 0.f;
    if (any_light && j < nls) {
      ok = pick_light<true, BWD>(B->sc, lights, hit_pos, N, ev, wo_back, aop, sum,
                                 ev.u(3 * (int)B->sc.area_light_count + j), wcache, ws, e);
      if (ok) {
        float pdf = e.w / sum;
        float joint = pdf * e.apdf;
        ok = !(joint < 1e-3f);
        if (ok) c = cmul(beta, alpha * ((e.rad / joint) / (float)nls));
        scale = alpha / (joint * (float)nls);
      }
    }
    int slot = warp_push(a.cnt + CNT_SHADOW, ok);
    if (ok && slot_ok(a, slot, a.sh_cap)) {
      uint32_t target = path, kind = 0u;
      if (BWD) {
        // packet: tangents x X, own albedo, light parameter
        const f3 X = e.rad * scale;
        uint32_t np = 0;
        for (uint32_t k = 0; k < ntan; ++k) {
          float4 t = a.tan[cur][(int64_t)k * a.ext_cap + i];
          f3 v = cmul(adj, cmul(f3{t.x, t.y, t.z}, X));
          a.pk[(int64_t)np++ * a.sh_cap + slot] = make_float4(v.x, v.y, v.z, t.w);
        }
        if (param) {
          f3 v = cmul(adj, cmul(beta, e.dalb * scale));
          a.pk[(int64_t)np++ * a.sh_cap + slot] = make_float4(v.x, v.y, v.z, __uint_as_float((uint32_t)mat_id));
        }
        if (e.lpar) {
          a.pk[(int64_t)np++ * a.sh_cap + slot] =
              make_float4(dot(cmul(adj, beta), e.dpar) * scale, 0.f, 0.f, __uint_as_float(e.idx | kLightFlag));
        } else if (e.pmat >= 0) {
          f3 v = cmul(adj, cmul(beta, e.dpar * scale));
          a.pk[(int64_t)np++ * a.sh_cap + slot] = make_float4(v.x, v.y, v.z, __uint_as_float((uint32_t)e.pmat));
        }
        a.pend[slot] = make_float4(__uint_as_float(np), 0.f, 0.f, 0.f);
        target = (uint32_t)slot;
        kind = 2u;
      } else {
        const uint32_t vslot = vertex - (1u << depth);
        if (a.det && vslot < (uint32_t)a.slots) {
          target = ((path * (uint32_t)a.slots + vslot) * (uint32_t)a.NLS + (uint32_t)j);
          a.pend[target] = make_float4(c.x, c.y, c.z, 0.f);
          kind = 2u;
        }
      }
      a.sh.o[slot] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, e.tfar);
      a.sh.d[slot] = make_float4(e.ray_d.x, e.ray_d.y, e.ray_d.z, __uint_as_float(target));
      a.sh.c[slot] = make_float4(c.x, c.y, c.z, __uint_as_float(kind | (b << 2)));
    }
  }
}

// One path vertex of Trace (src/baker.cpp:70-149) in throughput form.
// BWD: the same vertex replayed for the adjoint.  The contributions are
// multilinear in the parameters once the light-selection pdfs are held
// constant, so the gradient follows from the throughput tangents: d(beta X)
// = D X + beta dX for a collected term X, and the child tangent of a bounce
// with factor f = alpha rho h is D f + [m] beta alpha h.
// SPLIT (forward only): next-event estimation is left to k_nee through a
// record per opaque hit instead of running inline.
template <bool BWD, bool SPLIT = false>
__global__ void SHB_SHADE_BOUNDS k_shade(WaveArgs a, int cur, int depth) {
  extern __shared__ float sgrad[];
  if (BWD) grad_zero(sgrad, a.n_params);
  // forward inline next-event estimation: the staged light table and weight cache
  const DLight* wave_lights =
      (BWD || SPLIT) ? nullptr : stage_lights(a.bakes, a.one_bake, reinterpret_cast<DLight*>(sgrad));
  const int n = min(a.cnt[cur], a.ext_cap);
  const int nxt = cur ^ 1;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int warp_id = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const ExtQueue q = a.ext[cur];
  const ExtQueue qn = a.ext[nxt];
  for (int base = warp_id * 32; base < n; base += warps * 32) {
    int i = base + lane;
    bool active = i < n;
    bool hit = false;
    uint32_t path = 0, vertex = 0, texel = 0, sample = 0, b = 0, ntan = 0;
    const BakeItem* B = a.bakes;
    f3 d = {0.f, 0.f, 1.f}, beta = {0.f, 0.f, 0.f}, pos = {0.f, 0.f, 0.f}, N = {0.f, 0.f, 1.f};
    f3 adj = {0.f, 0.f, 0.f};
    f2 uv = {0.f, 0.f};
    float alpha = 1.f;
    bool can_extend = false;
    int mat_id = -1;
    DMat mat{};
    if (active) {
      float4 qo = q.o[i], qd = q.d[i], qb = q.beta[i], h = a.hits[i];
      path = __float_as_uint(qo.w);
      vertex = __float_as_uint(qd.w);
      d = {qd.x, qd.y, qd.z};
      beta = {qb.x, qb.y, qb.z};
      if (BWD) {
        ntan = __float_as_uint(qb.w);
        float4 ad = a.path_L[path];
        adj = {ad.x, ad.y, ad.z};
      }
      uint32_t prim = __float_as_uint(h.w);
      if (prim == kMissPrim) {
        if (!BWD && depth == 0) a.path_L[path].w += 1.0f;
      } else {
        hit = true;
        PathInfo pi = a.info[path];
        b = pi.x;
        B = a.bakes + b;
        texel = pi.y;
        sample = pi.z;
        can_extend = depth < B->bounces;
        const SceneView& sc = B->sc;
        f3 o = {qo.x, qo.y, qo.z};
        pos = o + d * h.x;
        float u = h.y, v = h.z;
        float w = 1.0f - u - v;
        uint32_t g = sc.tri_geom[prim];
        DGeom G = sc.geoms[g];
        uint32_t i0 = sc.tri_vidx[3 * prim], i1 = sc.tri_vidx[3 * prim + 1], i2 = sc.tri_vidx[3 * prim + 2];
        if (G.flags & GEOM_HAS_NORMALS) {
          N = normalized(w * ld3(sc.obj_n, i0) + u * ld3(sc.obj_n, i1) + v * ld3(sc.obj_n, i2));
        } else {
          f3 v0 = ld3(sc.world_v, i0), v1 = ld3(sc.world_v, i1), v2 = ld3(sc.world_v, i2);
          N = normalized(cross(v1 - v0, v2 - v0));
        }
        if (G.flags & GEOM_HAS_TEXUV)
          uv = w * ld2(sc.tex_uv, i0) + u * ld2(sc.tex_uv, i1) + v * ld2(sc.tex_uv, i2);
        mat = load_mat(sc, G.material_id);
        mat_id = G.material_id;
        alpha = get_alpha(sc, mat, uv);
      }
    }
    // is the hit material an adjoint parameter
    const bool param = BWD && hit && mat_id >= 0 && (uint32_t)mat_id < B->sc.mat_count && mat.use_override;
    // transmission (src/baker.cpp:99-105)
    if (__any_sync(0xFFFFFFFFu, hit && B->sc.has_alpha)) {
      bool tr = hit && alpha < 1.0f && can_extend;
      int slot = warp_push(a.cnt + nxt, tr);
      if (tr && slot_ok(a, slot, a.ext_cap)) {
        f3 hp = pos + d * 0.001f;
        f3 bt = beta * (1.0f - alpha);
        qn.o[slot] = make_float4(hp.x, hp.y, hp.z, __uint_as_float(path));
        qn.d[slot] = make_float4(d.x, d.y, d.z, __uint_as_float(2u * vertex + 1u));
        qn.beta[slot] = make_float4(bt.x, bt.y, bt.z, __uint_as_float(BWD ? ntan : 0u));
        if (BWD)
          for (uint32_t k = 0; k < ntan; ++k) {
            float4 t = a.tan[cur][(int64_t)k * a.ext_cap + i];
            a.tan[nxt][(int64_t)k * a.ext_cap + slot] =
                make_float4(t.x * (1.0f - alpha), t.y * (1.0f - alpha), t.z * (1.0f - alpha), t.w);
          }
      }
    }
    bool opaque_hit = hit && alpha != 0.0f;
    f3 hit_pos = pos, aop = {0.f, 0.f, 0.f};
    if (opaque_hit) {
      f3 alb = get_albedo(B->sc, mat, uv);
      aop = alb / 3.14159265358979323846f;
      if (depth == 0) {
        f3 em = mat.emission > 0.0f ? alb * mat.emission : f3{0.f, 0.f, 0.f};
        if (!is_zero_eigen(em) && !BWD) {
          f3 c = cmul(beta, alpha * em);
          float4 L = a.path_L[path];
          a.path_L[path] = make_float4(L.x + c.x, L.y + c.y, L.z + c.z, L.w);
        }
      }
      hit_pos = pos + N * 0.001f;
    }
    if (BWD) {
      // emission at depth 0: d(beta alpha rho e)/d rho = beta alpha e (no tangents yet)
      bool em_on = param && opaque_hit && depth == 0 && mat.emission > 0.0f &&
                   !is_zero_eigen(get_albedo(B->sc, mat, uv) * mat.emission);
      f3 v = cmul(adj, beta) * (alpha * mat.emission);
      warp_grad_entry(sgrad, a, make_float4(v.x, v.y, v.z, __uint_as_float((uint32_t)max(mat_id, 0))), em_on);
    }
    // NEE at the hit (src/light.cpp:82-189): inline, or (SPLIT) a record per
    // opaque hit for k_nee
    f3 wo = -d;
    if (BWD || !SPLIT) {
      nee_hit<BWD>(a, B, b, hit_pos, N, wo, aop, beta, alpha, path, vertex, texel, sample, depth, opaque_hit, ntan,
                   adj, param, mat_id, cur, i, wave_lights ? wave_lights : B->sc.lights);
    } else {
      const int rs = warp_push(a.cnt + CNT_NEE, opaque_hit);
      if (opaque_hit && slot_ok(a, rs, a.ext_cap)) {
        const int64_t C = a.ext_cap;
        a.nee_rec[rs] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, __uint_as_float(path));
        a.nee_rec[C + rs] = make_float4(N.x, N.y, N.z, __uint_as_float(vertex));
        a.nee_rec[2 * C + rs] = make_float4(d.x, d.y, d.z, alpha);
        a.nee_rec[3 * C + rs] = make_float4(aop.x, aop.y, aop.z, beta.x);
        a.nee_rec[4 * C + rs] = make_float4(beta.y, beta.z, 0.f, 0.f);
      }
    }
    // indirect (src/material.cpp:113-162, src/baker.cpp:131-148)
    bool ext = false;
    f3 nd = {0.f, 0.f, 1.f}, nb = {0.f, 0.f, 0.f}, fac = {0.f, 0.f, 0.f};
    float hscale = 0.f;
    if (opaque_hit && can_extend) {
      Event eb;
      eb.init(B->seed, texel, sample, vertex, EV_BSDF);
      f3 t = fabsf(N.x) > fabsf(N.z) ? f3{-N.y, N.x, 0.0f} : f3{0.0f, -N.z, N.y};
      t = normalized(t);
      f3 bb = cross(N, t);
      float r1 = eb.u(0), r2 = eb.u(1);
      float phi = (float)(kTwoPiD * (double)r1);
      float theta = acosf(sqrtf(r2));
      float sin_theta = sinf(theta);
      f3 local = {cosf(phi) * sin_theta, sinf(phi) * sin_theta, cosf(theta)};
      nd = normalized(t * local.x + bb * local.y + N * local.z);
      float pdf = (float)((double)local.z / 3.14159265358979323846);
      if (!(pdf < 1e-3f)) {
        bool zero = dot(N, nd) <= 0.0f || dot(N, wo) <= 0.0f;
        f3 brdf = zero ? f3{0.f, 0.f, 0.f} : aop;
        float cos_term = dot(N, nd);
        fac = alpha * (brdf * (cos_term / pdf));
        nb = cmul(beta, fac);
        ext = !(nb.x == 0.f && nb.y == 0.f && nb.z == 0.f);
        if (BWD && !zero) hscale = alpha * ((cos_term / pdf) / 3.14159265358979323846f);
      }
    }
    int slot = warp_push(a.cnt + nxt, ext);
    if (ext && slot_ok(a, slot, a.ext_cap)) {
      uint32_t nt = 0;
      if (BWD) {
        // child tangents: D f, plus beta alpha h for the own albedo (merged)
        bool merged = false;
        for (uint32_t k = 0; k < ntan; ++k) {
          float4 t = a.tan[cur][(int64_t)k * a.ext_cap + i];
          f3 v = cmul(f3{t.x, t.y, t.z}, fac);
          if (param && __float_as_uint(t.w) == (uint32_t)mat_id) {
            v = v + beta * hscale;
            merged = true;
          }
          a.tan[nxt][(int64_t)nt++ * a.ext_cap + slot] = make_float4(v.x, v.y, v.z, t.w);
        }
        if (param && !merged) {
          if ((int)nt < a.ntan) {
            f3 v = beta * hscale;
            a.tan[nxt][(int64_t)nt++ * a.ext_cap + slot] = make_float4(v.x, v.y, v.z, __uint_as_float((uint32_t)mat_id));
          } else {
            atomicOr(a.cnt + CNT_ERROR, ERR_QUEUE);
          }
        }
      }
      qn.o[slot] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, __uint_as_float(path));
      qn.d[slot] = make_float4(nd.x, nd.y, nd.z, __uint_as_float(2u * vertex));
      qn.beta[slot] = make_float4(nb.x, nb.y, nb.z, __uint_as_float(nt));
    }
  }
  if (BWD) grad_flush(sgrad, a.n_params, a.grad);
}

// Next-event estimation of the forward bake over the dense record queue
// k_shade filled (CNT_NEE): the same arithmetic as the inline call of the
// adjoint, with fewer live registers and every lane on an opaque hit.
// k_nee is register-limited to SHB_NEE_BLOCKS_PER_SM resident blocks per
// SM (0: the compiler's choice, 116 registers and 2 blocks).  4 blocks (64
// registers, the light loop partly in local memory) measured 4.6 % faster
// on the atrium's shading than 2, and 3 blocks 2 %.
#ifndef SHB_NEE_BLOCKS_PER_SM
#define SHB_NEE_BLOCKS_PER_SM 4
#endif
#if SHB_NEE_BLOCKS_PER_SM > 0
#define SHB_NEE_BOUNDS __launch_bounds__(kThreads, SHB_NEE_BLOCKS_PER_SM)
#else
#define SHB_NEE_BOUNDS __launch_bounds__(kThreads)
#endif
__global__ void SHB_NEE_BOUNDS k_nee(WaveArgs a, int cur, int depth) {
  extern __shared__ float dyn_smem[];
  const DLight* wave_lights = stage_lights(a.bakes, a.one_bake, reinterpret_cast<DLight*>(dyn_smem));
  const int n = min(a.cnt[CNT_NEE], a.ext_cap);
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int warp_id = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const int64_t C = a.ext_cap;
  for (int base = warp_id * 32; base < n; base += warps * 32) {
    const int i = base + lane;
    const bool active = i < n;
    f3 hit_pos = {0.f, 0.f, 0.f}, N = {0.f, 0.f, 1.f}, d = {0.f, 0.f, 1.f}, aop = {0.f, 0.f, 0.f},
       beta = {0.f, 0.f, 0.f};
    float alpha = 0.f;
    uint32_t path = 0, vertex = 0, texel = 0, sample = 0, b = 0;
    const BakeItem* B = a.bakes;
    if (active) {
      const float4 r0 = a.nee_rec[i], r1 = a.nee_rec[C + i], r2 = a.nee_rec[2 * C + i],
                   r3 = a.nee_rec[3 * C + i];
      hit_pos = {r0.x, r0.y, r0.z};
      path = __float_as_uint(r0.w);
      N = {r1.x, r1.y, r1.z};
      vertex = __float_as_uint(r1.w);
      d = {r2.x, r2.y, r2.z};
      aop = {r3.x, r3.y, r3.z};
      const float4 r4 = a.nee_rec[4 * C + i];
      alpha = r2.w;
      beta = {r3.w, r4.x, r4.y};
      const PathInfo pi = a.info[path];
      b = pi.x;
      B = a.bakes + b;
      texel = pi.y;
      sample = pi.z;
    }
    const f3 wo = -d;
    nee_hit<false>(a, B, b, hit_pos, N, wo, aop, beta, alpha, path, vertex, texel, sample, depth, active, 0u,
                   f3{0.f, 0.f, 0.f}, false, -1, cur, i, wave_lights ? wave_lights : B->sc.lights);
  }
}

// Adds the gradient packets of the visible shadow rays (BWD): count in
// pend[slot].x, cleared by k_shadow for occluded rays.
__global__ void __launch_bounds__(kThreads) k_apply(WaveArgs a) {
  extern __shared__ float sgrad[];
  grad_zero(sgrad, a.n_params);
  const int n = min(a.cnt[CNT_SHADOW], a.sh_cap);
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
    const int i = base + (threadIdx.x & 31);
    const bool active = i < n;
    const uint32_t cnt = active ? min(__float_as_uint(a.pend[i].x), (uint32_t)a.npk) : 0u;
    for (int k = 0; k < a.npk; ++k) {
      const bool act = (uint32_t)k < cnt;
      float4 e = act ? a.pk[(int64_t)k * a.sh_cap + i] : make_float4(0.f, 0.f, 0.f, 0.f);
      warp_grad_entry(sgrad, a, e, act);
    }
  }
  grad_flush(sgrad, a.n_params, a.grad);
}

// Adds the pending hit-NEE contributions of one depth to the path radiance
// in (branch, light sample) order and clears them: the same sum however the
// shadow rays were scheduled.  Unoccluded slots keep the value k_shade
// wrote, occluded ones were cleared by k_shadow, unused ones stay zero.
__global__ void __launch_bounds__(kThreads) k_commit(WaveArgs a, int depth) {
  const int used = min(1 << min(depth, 30), a.slots);
  const int stride = a.slots * a.NLS;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < a.P; p += (int64_t)gridDim.x * blockDim.x) {
    float4* pend = a.pend + p * stride;
    float4 L = a.path_L[p];
    bool any = false;
    for (int v = 0; v < used; ++v) {
      f3 s = {0.f, 0.f, 0.f};
      for (int j = 0; j < a.NLS; ++j) {
        float4 c = pend[v * a.NLS + j];
        if (c.x != 0.f || c.y != 0.f || c.z != 0.f || __float_as_uint(c.w) != 0u) {
          s = s + f3{c.x, c.y, c.z};
          pend[v * a.NLS + j] = make_float4(0.f, 0.f, 0.f, 0.f);
          any = true;
        }
      }
      L.x += s.x;
      L.y += s.y;
      L.z += s.z;
    }
    if (any) a.path_L[p] = L;
  }
}

// ------------------------------------------------------------- resolve ---
__device__ __forceinline__ void sh_accumulate(f3 L, f3 d, float acc[27]) {
  const float x = d.x, y = d.y, z = d.z;
  float sh[9];
  sh[0] = 0.282095f;
  sh[1] = 0.488603f * y;
  sh[2] = 0.488603f * z;
  sh[3] = 0.488603f * x;
  sh[4] = 1.092548f * x * y;
  sh[5] = 1.092548f * y * z;
  sh[6] = 0.315392f * (3.0f * z * z - 1.0f);
  sh[7] = 1.092548f * x * z;
  sh[8] = 0.546274f * (x * x - y * y);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    acc[3 * i] += L.x * sh[i];
    acc[3 * i + 1] += L.y * sh[i];
    acc[3 * i + 2] += L.z * sh[i];
  }
}

// One warp per texel: each lane projects its samples into SH9 in registers
// (src/sh_coeffs.cpp:50-78), the warp reduces with shuffles, and lanes
// 0..27 store the 27 coefficients and the environment visibility.
__global__ void __launch_bounds__(kThreads) k_resolve(WaveArgs a) {
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t warp_id = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const float two_pi = (float)kTwoPiD;
  for (int64_t wt = warp_id; wt < a.n_tex; wt += warps) {
    const Tile t = a.tiles[find_tile<false>(a, wt)];
    const BakeItem* B = a.bakes + t.bake;
    const int64_t local = wt - t.tex_off;
    const uint32_t texel = B->valid[t.t0 + (uint32_t)local];
    const int64_t pbase = t.path_off + local * t.spp;
    const int nls = B->nls;
    SP sp = load_sp(B->pts, texel);
    float acc[27];
#pragma unroll
    for (int k = 0; k < 27; ++k) acc[k] = 0.f;
    float env = 0.f;
    for (uint32_t s = lane; s < t.spp; s += 32) {
      int64_t p = pbase + s;
      for (int j = 0; j < nls; ++j) {
        float4 li = a.nee_li[p * a.NLS + j];
        if (li.x != 0.f || li.y != 0.f || li.z != 0.f) {
          float4 nd = a.nee_dir[p * a.NLS + j];
          sh_accumulate(f3{li.x, li.y, li.z}, f3{nd.x, nd.y, nd.z}, acc);
        }
      }
      float4 L = a.path_L[p];
      f3 dw = primary_dir(sp, B->seed, texel, s + B->sample_offset);
      sh_accumulate(f3{L.x, L.y, L.z} * two_pi, dw, acc);
      env += L.w;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
      for (int k = 0; k < 27; ++k) acc[k] += __shfl_xor_sync(0xFFFFFFFFu, acc[k], off);
      env += __shfl_xor_sync(0xFFFFFFFFu, env, off);
    }
    const float inv = 1.0f / (float)t.spp;
    float mine = 0.f;
#pragma unroll
    for (int k = 0; k < 27; ++k)
      if (lane == k) mine = acc[k];
    if (lane < 27) B->sh_out[(int64_t)texel * 27 + lane] = mine * inv;
    else if (lane == 27) B->env_out[texel] = env * inv;
  }
}

// Hit attributes of FindOcclusion (src/occlusion.cpp:70-133).
__global__ void k_occ_attrs(SceneView sc, const shb_ray* __restrict__ rays, const float4* __restrict__ hits, int64_t n,
                            shb_hit* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float4 h = hits[i];
    uint32_t prim = __float_as_uint(h.w);
    shb_hit r;
    r.position[0] = r.position[1] = r.position[2] = 0.f;
    r.uv[0] = r.uv[1] = 0.f;
    r.normal[0] = r.normal[1] = r.normal[2] = 0.f;
    r.material_id = 0;
    r.hit = 0;
    r.t = 0.f;
    r.prim_id = 0;
    if (prim != kMissPrim) {
      const shb_ray& ray = rays[i];
      f3 o = {ray.origin[0], ray.origin[1], ray.origin[2]};
      f3 d = {ray.direction[0], ray.direction[1], ray.direction[2]};
      f3 pos = o + d * h.x;
      float u = h.y, v = h.z, w = 1.0f - u - v;
      DGeom G = sc.geoms[sc.tri_geom[prim]];
      uint32_t i0 = sc.tri_vidx[3 * prim], i1 = sc.tri_vidx[3 * prim + 1], i2 = sc.tri_vidx[3 * prim + 2];
      f3 N;
      if (G.flags & GEOM_HAS_NORMALS) {
        N = normalized(w * ld3(sc.obj_n, i0) + u * ld3(sc.obj_n, i1) + v * ld3(sc.obj_n, i2));
      } else {
        f3 v0 = ld3(sc.world_v, i0), v1 = ld3(sc.world_v, i1), v2 = ld3(sc.world_v, i2);
        N = normalized(cross(v1 - v0, v2 - v0));
      }
      f2 uv = {0.f, 0.f};
      if (G.flags & GEOM_HAS_TEXUV) uv = w * ld2(sc.tex_uv, i0) + u * ld2(sc.tex_uv, i1) + v * ld2(sc.tex_uv, i2);
      r.position[0] = pos.x;
      r.position[1] = pos.y;
      r.position[2] = pos.z;
      r.uv[0] = uv.x;
      r.uv[1] = uv.y;
      r.normal[0] = N.x;
      r.normal[1] = N.y;
      r.normal[2] = N.z;
      r.material_id = G.material_id;
      r.hit = 1;
      r.t = h.x;
      r.prim_id = prim;
    }
    out[i] = r;
  }
}

struct ValidPred {
  const shb_surface_point* pts;
  __device__ __forceinline__ bool operator()(uint32_t i) const { return pts[i].material_id >= 0; }
};

inline int grid_for(int64_t n) {
  int64_t g = (n + kThreads - 1) / kThreads;
  if (g > sm_count() * 8) g = sm_count() * 8;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace

void srgb_upload(const float table[256]) { cudaMemcpyToSymbol(g_srgb, table, sizeof(float) * 256); }

// Area-light triangle records of a scene (see sample_area).
shb_status build_area_tris(shb_scene* s) {
  std::vector<uint4> entries;
  for (DLight& L : s->h_lights) {
    L.area_first = 0;
    L.area_count = 0;
    if (L.type != SHB_LIGHT_AREA || L.area_ord < 0) continue;
    if (L.geom < 0 || L.mat < 0 || (size_t)L.geom >= s->h_geoms.size()) continue;
    const DGeom& g = s->h_geoms[(size_t)L.geom];
    const uint32_t has_uv = (g.flags & GEOM_HAS_TEXUV) ? 1u : 0u;
    L.area_first = (uint32_t)entries.size();
    L.area_count = g.tri_count | (has_uv ? kAreaHasUv : 0u);
    for (uint32_t t = 0; t < g.tri_count; ++t) entries.push_back(make_uint4(g.prim_base + t, g.tri_count, has_uv, 0u));
  }
  cudaStream_t st = s->ctx->stream;
  if (!s->h_lights.empty())
    SHB_CUDA(cudaMemcpyAsync(s->lights.ptr, s->h_lights.data(), sizeof(DLight) * s->h_lights.size(),
                             cudaMemcpyHostToDevice, st));
  SHB_TRY(s->area_tris.reserve(sizeof(float4) * 4 * std::max<size_t>(entries.size(), 1)));
  if (!entries.empty()) {
    DevBuf tmp;
    SHB_TRY(tmp.reserve(sizeof(uint4) * entries.size()));
    SHB_CUDA(cudaMemcpyAsync(tmp.ptr, entries.data(), sizeof(uint4) * entries.size(), cudaMemcpyHostToDevice, st));
    const int n = (int)entries.size();
    k_area_tris<<<std::min((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(s->view(), tmp.as<uint4>(), n,
                                                                      s->area_tris.as<float4>());
    count_launch(s->ctx, 1);
    SHB_CUDA(cudaGetLastError());
    SHB_CUDA(cudaStreamSynchronize(st));  // tmp is freed on return
  }
  return SHB_OK;
}

// Status of a bake or query whose kernels raised device error flags: a
// bounded loop that ran out is SHB_ERR_TIMEOUT, an exceeded capacity
// SHB_ERR_INTERNAL.
shb_status device_error(int err) {
  set_error(std::string("bounded device failure:") + (err & ERR_STACK ? " traversal stack overflow" : "") +
            (err & ERR_QUEUE ? " ray queue overflow" : "") + (err & ERR_ITER ? " traversal step limit reached" : ""));
  return (err & (ERR_STACK | ERR_QUEUE)) ? SHB_ERR_INTERNAL : SHB_ERR_TIMEOUT;
}

shb_status find_occlusion_device(shb_scene* s, const shb_ray* d_rays, int64_t n, shb_hit* d_hits) {
  shb_context* c = s->ctx;
  if (n <= 0) return SHB_OK;
  SHB_TRY(c->scratch[9].reserve(sizeof(float4) * (size_t)n));
  SHB_TRY(c->counters.reserve(sizeof(int) * CNT_COUNT + sizeof(Counters64)));
  int* cnt = c->counters.as<int>();
  SHB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * CNT_COUNT, c->stream));
  float4* hits = c->scratch[9].as<float4>();
  launch_closest_rays(c->stream, s->bvh(), d_rays, n, hits, cnt + CNT_ERROR);
  k_occ_attrs<<<grid_for(n), kThreads, 0, c->stream>>>(s->view(), d_rays, hits, n, d_hits);
  count_launch(c, 2);
  SHB_CUDA(cudaGetLastError());
  int err = 0;
  SHB_CUDA(cudaMemcpyAsync(&err, cnt + CNT_ERROR, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SHB_CUDA(cudaStreamSynchronize(c->stream));
  if (err) return device_error(err);
  return SHB_OK;
}

// ------------------------------------------------------------ batches ----

namespace {

uint32_t nee_cost(const shb_scene& sc) {
  return (sc.light_count - sc.area_light_count) + 4u * sc.area_light_count;
}

struct Wave {
  int tile_begin, n_tiles;
  int64_t P, n_tex;
  int max_bounces;
  int bake;  // the one bake whose tiles fill the wave, else -1
  uint32_t nee_cost;  // largest light-loop cost (nee_cost) of its bakes
};

// Splits every bake's valid texels into tiles of whole texels (all their
// samples) and packs tiles into waves of at most `wave_paths` paths.  A bake
// of at least `share_paths` paths gets waves of its own, split evenly (no
// short last wave), so that traversal runs with that bake's BVH bound for
// the whole launch; smaller bakes share waves in their order.
void plan_waves(const std::vector<BakeSpec>& specs, const std::vector<int>& n_valid, int64_t wave_paths,
                int64_t tile_texels, int64_t share_paths, std::vector<Tile>& tiles, std::vector<Wave>& waves) {
  tiles.clear();
  waves.clear();
  Wave cur{0, 0, 0, 0, 0, -1, 0};
  auto flush = [&] {
    if (cur.n_tiles > 0) waves.push_back(cur);
    cur = Wave{(int)tiles.size(), 0, 0, 0, 0, -1, 0};
  };
  auto add = [&](size_t b, int64_t cap) {
    const int64_t spp = specs[b].cfg.samples;
    const int64_t per_tile = std::max<int64_t>(1, std::min<int64_t>(tile_texels, cap / spp));
    for (int64_t t0 = 0; t0 < n_valid[b]; t0 += per_tile) {
      const int64_t nt = std::min<int64_t>(per_tile, n_valid[b] - t0);
      const int64_t paths = nt * spp;
      if (cur.n_tiles > 0 && cur.P + paths > cap) flush();
      Tile t;
      t.bake = (uint32_t)b;
      t.t0 = (uint32_t)t0;
      t.n_tex = (uint32_t)nt;
      t.spp = (uint32_t)spp;
      t.path_off = cur.P;
      t.tex_off = cur.n_tex;
      tiles.push_back(t);
      cur.bake = (cur.n_tiles == 0 || cur.bake == (int)b) ? (int)b : -1;
      cur.n_tiles++;
      cur.P += paths;
      cur.n_tex += nt;
      cur.max_bounces = std::max(cur.max_bounces, specs[b].cfg.bounces);
      cur.nee_cost = std::max(cur.nee_cost, nee_cost(*specs[b].scene));
    }
  };
  for (size_t b = 0; b < specs.size(); ++b) {
    const int64_t spp = specs[b].cfg.samples, paths = n_valid[b] * spp;
    if (paths == 0 || paths < share_paths) continue;
    flush();
    const int64_t n_w = (paths + wave_paths - 1) / wave_paths;
    const int64_t tex = (n_valid[b] + n_w - 1) / n_w;
    add(b, std::min(wave_paths, tex * spp));
    flush();
  }
  for (size_t b = 0; b < specs.size(); ++b)
    if ((int64_t)n_valid[b] * specs[b].cfg.samples < share_paths) add(b, wave_paths);
  flush();
}

}  // namespace

// Runs a batch of bakes.  Each bake's outputs are zeroed, its valid texels
// compacted, and then all bakes share waves of paths.
shb_status bake_batch_device(shb_context* c, const std::vector<BakeSpec>& specs, const BatchParams& prm,
                             shb_bake_stats* stats) {
  cudaStream_t st = c->stream;
  const int nb = (int)specs.size();
  if (nb == 0) return SHB_OK;
  const bool bwd = prm.backward;
  int n_params = 0;
  if (bwd) {
    if (nb != 1 || !specs[0].dsh || !prm.grad) {
      set_error("backward takes one bake with dLoss/dSH and a gradient buffer");
      return SHB_ERR_INVALID_ARG;
    }
    n_params = 3 * (int)specs[0].scene->mat_count + (int)specs[0].scene->light_count;
    if ((size_t)n_params * sizeof(float) > kMaxGradSmem) {
      set_error("backward: more than " + std::to_string(kMaxGradSmem / 4) + " parameters (3 x materials + lights)");
      return SHB_ERR_INVALID_ARG;
    }
    if (specs[0].cfg.bounces > kMaxTangents) {
      set_error("backward: at most " + std::to_string(kMaxTangents) + " bounces");
      return SHB_ERR_INVALID_ARG;
    }
  }
  int NLS = 1;
  int64_t total_texels = 0;
  bool any_alpha = false;
  int max_b = 0;
  for (const BakeSpec& s : specs) {
    NLS = std::max(NLS, s.cfg.num_light_samples);
    total_texels += (int64_t)s.W * s.H;
    any_alpha = any_alpha || s.scene->has_alpha;
    max_b = std::max(max_b, s.cfg.bounces);
  }
  // outputs and valid-texel lists
  SHB_TRY(c->scratch[10].reserve(sizeof(uint32_t) * (size_t)(total_texels + nb)));
  SHB_TRY(c->counters.reserve(sizeof(int) * CNT_COUNT + sizeof(Counters64) + sizeof(int) * (size_t)nb));
  int* cnt = c->counters.as<int>();
  Counters64* c64 = reinterpret_cast<Counters64*>(cnt + CNT_COUNT);
  int* nsel = reinterpret_cast<int*>(c64 + 1);
  SHB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * CNT_COUNT + sizeof(Counters64) + sizeof(int) * (size_t)nb, st));
  std::vector<BakeItem> items(nb);
  uint32_t* valid_all = c->scratch[10].as<uint32_t>();
  int64_t voff = 0;
  thrust::counting_iterator<uint32_t> it(0);
  for (int b = 0; b < nb; ++b) {
    const BakeSpec& s = specs[b];
    const int64_t n = (int64_t)s.W * s.H;
    if (!bwd) {
      SHB_CUDA(cudaMemsetAsync(s.sh, 0, sizeof(float) * 27 * (size_t)n, st));
      SHB_CUDA(cudaMemsetAsync(s.env, 0, sizeof(float) * (size_t)n, st));
    }
    size_t tb = 0;
    cub::DeviceSelect::If(nullptr, tb, it, valid_all + voff, nsel + b, (int)n, ValidPred{s.pts}, st);
    SHB_TRY(c->scratch[11].reserve(tb));
    SHB_CUDA(cub::DeviceSelect::If(c->scratch[11].ptr, tb, it, valid_all + voff, nsel + b, (int)n, ValidPred{s.pts},
                                   st));
    count_launch(c, 1);
    BakeItem& I = items[b];
    I.sc = s.scene->view();
    I.bvh = s.scene->bvh();
    I.pts = s.pts;
    I.valid = valid_all + voff;
    I.sh_out = s.sh;
    I.env_out = s.env;
    I.spp = (uint32_t)s.cfg.samples;
    I.seed = s.cfg.seed;
    I.sample_offset = (uint32_t)s.cfg.sample_offset;
    I.nls = s.cfg.num_light_samples;
    I.bounces = s.cfg.bounces;
    I.pad = 0;
    voff += n;
  }
  std::vector<int> n_valid(nb, 0);
  SHB_CUDA(cudaMemcpyAsync(n_valid.data(), nsel, sizeof(int) * (size_t)nb, cudaMemcpyDeviceToHost, st));
  SHB_TRY(c->scratch[19].reserve(sizeof(BakeItem) * (size_t)nb));
  BakeItem* d_items = c->scratch[19].as<BakeItem>();
  SHB_CUDA(cudaMemcpyAsync(d_items, items.data(), sizeof(BakeItem) * (size_t)nb, cudaMemcpyHostToDevice, st));
  SHB_CUDA(cudaStreamSynchronize(st));

  // plan tiles and waves
  int64_t wave_paths = prm.wave_paths;
  int64_t mult = 1;
  if (any_alpha) {
    int shift = max_b < kMaxBranchLog ? max_b : kMaxBranchLog;
    mult = (int64_t)1 << shift;
    wave_paths = std::max<int64_t>(wave_paths / mult, 1 << 16);
  }
  // Several hit-NEE contributions per path and depth (light samples or
  // alpha branches) are summed in a fixed order by k_commit.
  const bool det = !bwd && (NLS > 1 || any_alpha);
  const int slots = (int)mult;
  std::vector<Tile> tiles;
  std::vector<Wave> waves;
  const int64_t share = prm.share_paths < 0 ? wave_paths / 2 : prm.share_paths;
  plan_waves(specs, n_valid, wave_paths, prm.tile_texels, share, tiles, waves);
  int64_t Pmax = 0;
  for (const Wave& w : waves) Pmax = std::max(Pmax, w.P);
  int64_t ext_cap = std::max<int64_t>(Pmax * mult, 1);
  int64_t sh_cap = (Pmax + ext_cap) * NLS;
  if (prm.queue_cap > 0) {  // a smaller queue drops what does not fit (ERR_QUEUE)
    ext_cap = std::min(ext_cap, prm.queue_cap);
    sh_cap = std::min(sh_cap, prm.queue_cap);
  }
  if (ext_cap > INT32_MAX || sh_cap > INT32_MAX) {
    set_error("wave too large");
    return SHB_ERR_INVALID_ARG;
  }
  SHB_TRY(c->scratch[12].reserve(sizeof(float4) * 3 * (size_t)ext_cap));
  SHB_TRY(c->scratch[13].reserve(sizeof(float4) * 3 * (size_t)ext_cap));
  SHB_TRY(c->scratch[14].reserve(sizeof(float4) * (size_t)ext_cap));
  SHB_TRY(c->scratch[15].reserve(sizeof(float4) * 3 * (size_t)sh_cap));
  SHB_TRY(c->scratch[16].reserve(sizeof(float4) * (size_t)std::max<int64_t>(Pmax, 1)));
  SHB_TRY(c->scratch[17].reserve(sizeof(float4) * 2 * (size_t)std::max<int64_t>(Pmax, 1) * NLS));
  SHB_TRY(c->scratch[18].reserve(sizeof(PathInfo) * (size_t)std::max<int64_t>(Pmax, 1)));
  if (det) SHB_TRY(c->scratch[24].reserve(sizeof(float4) * (size_t)std::max<int64_t>(Pmax, 1) * slots * NLS));
  const int ntan = bwd ? std::max(max_b, 1) : 0, npk = ntan + 2;
  if (bwd) {
    SHB_TRY(c->scratch[24].reserve(sizeof(float4) * (size_t)sh_cap));
    SHB_TRY(c->scratch[25].reserve(sizeof(float4) * ((size_t)2 * ntan * ext_cap + (size_t)npk * sh_cap)));
    SHB_CUDA(cudaMemsetAsync(prm.grad, 0, sizeof(double) * (size_t)n_params, st));
  }
  SHB_TRY(c->scratch[23].reserve(sizeof(Tile) * std::max<size_t>(tiles.size(), 1)));
  Tile* d_tiles = c->scratch[23].as<Tile>();
  if (!tiles.empty())
    SHB_CUDA(cudaMemcpyAsync(d_tiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, st));
  WaveArgs a;
  a.bakes = d_items;
  a.n_bakes = nb;
  a.NLS = NLS;
  for (int k = 0; k < 2; ++k) {
    float4* base = c->scratch[12 + k].as<float4>();
    a.ext[k] = ExtQueue{base, base + ext_cap, base + 2 * ext_cap};
  }
  a.hits = c->scratch[14].as<float4>();
  {
    float4* base = c->scratch[15].as<float4>();
    a.sh = ShadowQueue{base, base + sh_cap, base + 2 * sh_cap};
  }
  a.path_L = c->scratch[16].as<float4>();
  a.nee_li = c->scratch[17].as<float4>();
  a.nee_dir = a.nee_li + std::max<int64_t>(Pmax, 1) * NLS;
  a.info = c->scratch[18].as<PathInfo>();
  a.cnt = cnt;
  a.ext_cap = (int)ext_cap;
  a.sh_cap = (int)sh_cap;
  a.det = det ? 1 : 0;
  a.slots = slots;
  a.pend = (det || bwd) ? c->scratch[24].as<float4>() : nullptr;
  // Next-event estimation runs as its own kernel in waves whose light loop
  // dominates shading (cost kSplitNeeCost or more): the hit kernel then
  // needs 56 registers instead of 118 and every k_nee lane is on an opaque
  // hit.  With a short loop the record round trip costs more (room, 5
  // punctual lights: shading +18 %; atrium, 9 punctual + 15 area: -10 %).
  bool any_split = false;
  auto splits = [&](const Wave& w) {
    return !bwd && (prm.nee_split == 2 || (prm.nee_split == 0 && w.nee_cost >= kSplitNeeCost));
  };
  for (const Wave& w : waves) any_split = any_split || splits(w);
  a.nee_rec = nullptr;
  if (any_split) {
    SHB_TRY(c->scratch[0].reserve(sizeof(float4) * 5 * (size_t)ext_cap));
    a.nee_rec = c->scratch[0].as<float4>();
  }
  a.dsh = bwd ? specs[0].dsh : nullptr;
  a.ntan = ntan;
  a.npk = npk;
  a.tan[0] = a.tan[1] = nullptr;
  a.pk = nullptr;
  if (bwd) {
    float4* base = c->scratch[25].as<float4>();
    a.tan[0] = base;
    a.tan[1] = base + (size_t)ntan * ext_cap;
    a.pk = base + (size_t)2 * ntan * ext_cap;
  }
  a.n_mat3 = bwd ? 3 * (int)specs[0].scene->mat_count : 0;
  a.n_params = n_params;
  a.grad = prm.grad;
  const size_t gsmem = bwd ? sizeof(float) * (size_t)n_params : 0;

  const int tgrid = traversal_grid(c->device, false) * std::max(1, prm.grid_scale);
  const int tgrid_sh = traversal_grid(c->device, true) * std::max(1, prm.grid_scale);
  const int sgrid = sm_count() * 8;
  const bool timed = c->profiling && !prm.use_graph;
  struct Pair {
    cudaEvent_t a, b;
    int kind;
  };
  std::vector<Pair> timed_pairs;
  auto stamp = [&](int kind) -> Pair {
    Pair p{nullptr, nullptr, kind};
    if (timed) {
      cudaEventCreate(&p.a);
      cudaEventCreate(&p.b);
      cudaEventRecord(p.a, st);
    }
    return p;
  };
  auto close_stamp = [&](Pair p) {
    if (timed) {
      cudaEventRecord(p.b, st);
      timed_pairs.push_back(p);
    }
  };
  uint64_t ext_launches = 0, sh_launches = 0;
  cudaEvent_t t_begin = nullptr, t_end = nullptr;
  if (c->profiling) {
    cudaEventCreate(&t_begin);
    cudaEventCreate(&t_end);
    cudaEventRecord(t_begin, st);
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (prm.use_graph) SHB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  uint64_t launches = 0;
  for (const Wave& w : waves) {
    a.tiles = d_tiles + w.tile_begin;
    a.n_tiles = w.n_tiles;
    a.P = w.P;
    a.n_tex = w.n_tex;
    const bool split_nee = splits(w);
    // traversal of a one-bake wave skips the per-ray bake lookup
    const BakeItem* bk = w.bake >= 0 ? d_items + w.bake : d_items;
    const int nbk = w.bake >= 0 ? 1 : nb;
    cudaMemsetAsync(cnt, 0, sizeof(int) * (CNT_FETCH_SHADOW + 1), st);
    Pair pg = stamp(2);
    a.one_bake = w.bake;
    if (bwd) k_generate<true><<<grid_for(w.P), kThreads, 0, st>>>(a);
    else k_generate<false><<<grid_for(w.P), kThreads, kNeeSmemBytes, st>>>(a);
    close_stamp(pg);
    launches++;
    for (int k = 0; k <= w.max_bounces; ++k) {
      int cur = k & 1, nxt = cur ^ 1;
      cudaMemsetAsync(cnt + nxt, 0, sizeof(int), st);
      cudaMemsetAsync(cnt + CNT_FETCH_EXT, 0, sizeof(int) * 2, st);
      Pair pe = stamp(0);
      launch_extend(st, tgrid, bk, nbk, a.info, a.ext[cur], cnt + cur, a.ext_cap, a.hits, cnt + CNT_FETCH_EXT,
                    cnt + CNT_ERROR, c64, prm.max_iters);
      close_stamp(pe);
      Pair pd = stamp(2);
      if (bwd) {
        k_shade<true><<<sgrid, kThreads, gsmem, st>>>(a, cur, k);
      } else if (split_nee) {
        cudaMemsetAsync(cnt + CNT_NEE, 0, sizeof(int), st);
        k_shade<false, true><<<sgrid, kThreads, 0, st>>>(a, cur, k);
        k_nee<<<sgrid, kThreads, kNeeSmemBytes, st>>>(a, cur, k);
        launches++;
      } else {
        k_shade<false><<<sgrid, kThreads, kNeeSmemBytes, st>>>(a, cur, k);
      }
      close_stamp(pd);
      Pair ps = stamp(1);
      launch_shadow(st, tgrid_sh, bk, nbk, a.sh, cnt + CNT_SHADOW, a.sh_cap, a.path_L, a.nee_li, a.pend,
                    cnt + CNT_FETCH_SHADOW, cnt + CNT_ERROR, c64, prm.max_iters);
      close_stamp(ps);
      if (bwd) {
        k_apply<<<sgrid, kThreads, gsmem, st>>>(a);
        launches++;
      }
      cudaMemsetAsync(cnt + CNT_SHADOW, 0, sizeof(int), st);
      launches += 3;
      if (det) {
        k_commit<<<grid_for(w.P), kThreads, 0, st>>>(a, k);
        launches++;
      }
      ext_launches++;
      sh_launches++;
    }
    if (!bwd) {
      Pair pr = stamp(2);
      k_resolve<<<grid_for(w.n_tex * 32), kThreads, 0, st>>>(a);
      close_stamp(pr);
      launches++;
    }
  }
  if (prm.use_graph) {
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(graph);
      return cuda_fail(e, "cudaGraphInstantiate");
    }
    e = cudaGraphLaunch(exec, st);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
  }
  count_launch(c, launches);
  SHB_CUDA(cudaGetLastError());
  int err = 0;
  Counters64 h64{0, 0};
  SHB_CUDA(cudaMemcpyAsync(&err, cnt + CNT_ERROR, sizeof(int), cudaMemcpyDeviceToHost, st));
  SHB_CUDA(cudaMemcpyAsync(&h64, c64, sizeof(Counters64), cudaMemcpyDeviceToHost, st));
  if (c->profiling) cudaEventRecord(t_end, st);
  SHB_CUDA(cudaStreamSynchronize(st));
  double ext_ms = 0.0, sh_ms = 0.0, shade_ms = 0.0;
  float total_ms = 0.f;
  if (c->profiling) {
    cudaEventElapsedTime(&total_ms, t_begin, t_end);
    cudaEventDestroy(t_begin);
    cudaEventDestroy(t_end);
    for (auto& pr : timed_pairs) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, pr.a, pr.b);
      if (pr.kind == 0) ext_ms += ms;
      else if (pr.kind == 1) sh_ms += ms;
      else shade_ms += ms;
      cudaEventDestroy(pr.a);
      cudaEventDestroy(pr.b);
    }
  }
  if (stats) {
    uint64_t ts = 0, vt = 0;
    for (int b = 0; b < nb; ++b) {
      ts += (uint64_t)n_valid[b] * (uint64_t)specs[b].cfg.samples;
      vt += (uint64_t)n_valid[b];
    }
    stats->texel_samples = ts;
    stats->valid_texels = vt;
    stats->extend_rays = h64.extend_rays;
    stats->shadow_rays = h64.shadow_rays;
    stats->error_flags = (uint32_t)err;
    stats->waves = (uint32_t)waves.size();
    stats->trace_ms = total_ms;
    stats->extend_kernel_ms = ext_ms;
    stats->shadow_kernel_ms = sh_ms;
    stats->shade_kernel_ms = shade_ms;
    stats->extend_launches = ext_launches;
    stats->shadow_launches = sh_launches;
  }
  if (err) return device_error(err);
  return SHB_OK;
}

// BakeSHLightMap on a device G-buffer: a batch of one.
shb_status bake_device(shb_scene* s, const shb_surface_point* d_pts, int W, int H, const shb_bake_config* cfg,
                       float* d_sh, float* d_env, shb_bake_stats* stats) {
  BakeSpec spec{s, d_pts, W, H, *cfg, d_sh, d_env};
  BatchParams prm;
  return bake_batch_device(s->ctx, {spec}, prm, stats);
}

shb_status backward_device(shb_scene* s, const shb_surface_point* d_pts, int W, int H, const shb_bake_config* cfg,
                           const float* d_dsh, double* d_grad, shb_bake_stats* stats) {
  BakeSpec spec{s, d_pts, W, H, *cfg, nullptr, nullptr, d_dsh};
  BatchParams prm;
  prm.backward = true;
  prm.grad = d_grad;
  return bake_batch_device(s->ctx, {spec}, prm, stats);
}

}  // namespace shb
