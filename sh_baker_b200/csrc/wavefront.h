// wavefront.h - ray queues and per-path state of the wavefront path tracer.
#pragma once

#include "shb_internal.h"

namespace shb {

constexpr uint32_t kMissPrim = 0xFFFFFFFFu;

// Extend (closest-hit) queue entry, structure of arrays:
//   o    = (origin.xyz, path index bits)
//   d    = (direction.xyz, path-vertex id bits)
//   beta = (throughput.xyz, unused)
struct ExtQueue {
  float4* o;
  float4* d;
  float4* beta;
};

// Shadow (any-hit) queue entry: tnear is 0.001 for every shadow ray
// (src/light.h:40,83,128,177).
//   o = (origin.xyz, tfar), d = (direction.xyz, target bits),
//   c = (contribution.xyz, kind bits): kind 0 adds c to the path radiance
//   of `target` when unoccluded; kind 1 clears texel-NEE slot `target`
//   when occluded; kind 2 clears pending hit-NEE slot `target` when
//   occluded (deterministic accumulation, see k_commit).
struct ShadowQueue {
  float4* o;
  float4* d;
  float4* c;
};

// Device counters of one bake.
enum CounterSlot {
  CNT_EXT0 = 0,
  CNT_EXT1 = 1,
  CNT_SHADOW = 2,
  CNT_FETCH_EXT = 3,
  CNT_FETCH_SHADOW = 4,
  CNT_ERROR = 5,
  CNT_NEE = 6,  // next-event records of the current depth (forward bake)
  CNT_COUNT = 8
};
enum ErrorBits : int { ERR_STACK = 1, ERR_QUEUE = 2, ERR_ITER = 4 };

struct Counters64 {
  unsigned long long extend_rays;
  unsigned long long shadow_rays;
};

// One bake of a batch (device table entry).  A single BakeSHLightMap call
// is a batch of one.
struct BakeItem {
  SceneView sc;
  BvhView bvh;
  const shb_surface_point* pts;  // (W*s) x (H*s) G-buffer
  const uint32_t* valid;         // compacted indices of valid texels
  float* sh_out;                 // 27 floats per texel
  float* env_out;
  uint32_t spp, seed, sample_offset;
  int32_t nls, bounces, pad;
};

// A tile of a wave: texel slots [t0, t0 + n_tex) of bake `bake` with all
// their samples; its paths start at `path_off` and its texels at `tex_off`
// within the wave.
struct Tile {
  uint32_t bake, t0, n_tex, spp;
  int64_t path_off;
  int64_t tex_off;
};

// Per-path record written by generate: (bake, texel, sample, unused).
using PathInfo = uint4;

// Shadow-queue kind bits: bits 0-1 = kind (0 path radiance, 1 texel-NEE
// slot, 2 pending hit-NEE slot), bits 2.. = bake index.

// Launch helpers for the persistent traversal kernels (traverse.cu).
// max_iters bounds the traversal steps of one ray (0: the default,
// 2^22); a ray that reaches it sets ERR_ITER and ends.
void launch_extend(cudaStream_t st, int grid, const BakeItem* bakes, int n_bakes, const PathInfo* info, ExtQueue q,
                   const int* n, int cap, float4* hits, int* fetch, int* err, Counters64* stats, uint32_t max_iters);
void launch_shadow(cudaStream_t st, int grid, const BakeItem* bakes, int n_bakes, ShadowQueue q, const int* n, int cap,
                   float4* path_L, float4* nee_li, float4* pend, int* fetch, int* err, Counters64* stats,
                   uint32_t max_iters);
void launch_closest_rays(cudaStream_t st, const BvhView& bvh, const shb_ray* rays, int64_t n, float4* hits,
                         int* err);
int traversal_grid(int device, bool shadow);

}  // namespace shb
