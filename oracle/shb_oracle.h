/*
 * shb_oracle.h - C entry points of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++ restatement of the
 * reference's bake path (src/rasterizer.cpp, src/baker.cpp, src/light.{h,cpp},
 * src/material.cpp, src/sh_coeffs.cpp, src/dilation.cpp, src/occlusion.cpp).
 * It is the checker of the CUDA path and the timed CPU baseline; nothing in
 * the product links or calls it.  It takes the same shb_scene_desc as the
 * product C ABI so both run on identical inputs.
 */
#ifndef SHB_ORACLE_H_
#define SHB_ORACLE_H_

#include "../include/shb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_scene oracle_scene;

/* RNG modes of the oracle bake. */
enum {
  ORACLE_RNG_MT19937 = 0, /* std::mt19937(12345 + idx) + std distributions,
                             exactly the stream of src/baker.cpp:254 */
  ORACLE_RNG_PHILOX = 1   /* the counter-based stream the GPU consumes  */
};

typedef struct oracle_bake_args {
  int32_t samples;
  int32_t bounces;
  int32_t num_light_samples;
  uint32_t seed;
  int32_t sample_offset;
  int32_t rng_mode;     /* ORACLE_RNG_* */
  int32_t fp64;         /* 1: whole path tracer in double */
  int32_t threads;      /* 0: hardware_concurrency */
  const int64_t* texel_subset; /* NULL: all texels; else list of indices */
  int64_t subset_count;
  float* sh_out;        /* 27 per texel (full G-buffer size), nullable */
  float* env_out;       /* 1 per texel, nullable */
  double* sh_var_out;   /* 27 per texel: per-sample variance, nullable */
  double* sh_mean64_out;/* 27 per texel: mean accumulated in double, nullable */
  uint64_t rays_traced; /* out */
  uint64_t texel_samples; /* out */
} oracle_bake_args;

oracle_scene* oracle_scene_create(const shb_scene_desc* desc);
void oracle_scene_destroy(oracle_scene* s);

/* src/rasterizer.cpp:68-211 (sequential, geometry-major). Returns 0 on ok. */
int oracle_rasterize(const oracle_scene* s, const shb_raster_config* cfg,
                     shb_surface_point* out);
void oracle_validity_mask(const shb_surface_point* pts, int64_t n, uint8_t* out);
int oracle_downsample_validity_mask(const uint8_t* in, int w, int h, int scale,
                                    uint8_t* out);
/* src/baker.cpp:151-182 for a texture of `channels` floats per texel. */
void oracle_downsample(const float* in, int in_w, int in_h, int channels,
                       int scale, float* out);
/* src/dilation.cpp:7-73. kind: SHB_DILATE_*. */
void oracle_dilate(int kind, int w, int h, void* pixels, uint8_t* mask, int passes);

/* src/baker.cpp:186-304 on the given surface points (W*s x H*s). */
int oracle_bake(const oracle_scene* s, const shb_surface_point* pts,
                const shb_raster_config* raster, oracle_bake_args* args);

/* Adjoint parameters, as shb_scene_set_params: per material a linear base
 * colour replacing the albedo texture (use_override NULL: all), per light
 * an intensity.  NULL arrays leave the values unchanged. */
void oracle_scene_set_params(oracle_scene* s, const float* albedo_rgb, const uint8_t* use_override,
                             const float* light_intensity);

/* FP64 forward-mode gradient of Loss = sum(dsh * SH) over the texels of
 * args (Philox stream, fp64 regardless of args->fp64; sh/env outputs
 * unused): d_albedo[3m + c] (override materials), d_light[l] (intensity of
 * point/spot/directional lights).  Light-selection weights are held
 * constant, as in the GPU adjoint. */
int oracle_bake_grad(const oracle_scene* s, const shb_surface_point* pts,
                     const shb_raster_config* raster, oracle_bake_args* args,
                     const float* dsh, double* d_albedo, double* d_light);

/* src/occlusion.cpp:9-107 for a batch of rays. */
void oracle_find_occlusion(const oracle_scene* s, const shb_ray* rays, int64_t n,
                           shb_hit* hits);

/* ---- known-answer helpers (the reference's unit tests call these) ------ */
/* src/sh_coeffs.cpp:50-78: out27 += radiance x Y(direction). */
void oracle_accumulate_radiance(const float radiance[3], const float dir[3],
                                float out27[27]);
/* src/colorspace.h:10-14 */
float oracle_srgb_to_linear(uint8_t x);
/* src/material.cpp:57-92 on material `m` at uv. */
void oracle_get_albedo(const oracle_scene* s, int m, const float uv[2], float out[3]);
float oracle_get_alpha(const oracle_scene* s, int m, const float uv[2]);
void oracle_get_emission(const oracle_scene* s, int m, const float uv[2], float out[3]);
/* src/light.cpp:82-189 with an mt19937 seeded by `seed`; empty_bvh = 1
 * traces shadow rays against an empty scene (as src/light_test.cpp does). */
void oracle_evaluate_light_samples(const oracle_scene* s, const float p[3],
                                   const float n[3], const float wo[3], int mat,
                                   const float uv[2], unsigned num_samples,
                                   uint32_t seed, int empty_bvh, float out[3]);
/* src/light.cpp:16-78: point, normal, radiance, pdf (10 floats). */
void oracle_sample_area_light(const oracle_scene* s, int light, uint32_t seed,
                              float out10[10]);
/* src/light.h:51-203 with a constant BRDF of 1: radiance x cos and the
 * pending visibility ray. */
void oracle_light_radiance_unit_brdf(const oracle_scene* s, int light, const float p[3],
                                     const float n[3], float out_rad[3],
                                     shb_ray* out_ray);
/* Philox4x32-10 (Salmon et al., SC'11) block function. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif

#endif
