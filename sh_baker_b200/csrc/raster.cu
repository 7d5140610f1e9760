// raster.cu - texel G-buffer rasteriser, validity masks, box downsample and
// dilation.  Compiled with -fmad=false: every result is bit-exact against
// the sequential CPU restatement of src/rasterizer.cpp, src/baker.cpp:151-182
// and src/dilation.cpp.
#include <cub/cub.cuh>

#include <mutex>

#include "shb_internal.h"
#include "shb_math.cuh"

namespace shb {

namespace {

constexpr int kThreads = 256;

inline int grid_for(int64_t n, int threads = kThreads) {
  int64_t g = (n + threads - 1) / threads;
  if (g > sm_count() * 64) g = sm_count() * 64;
  return (int)(g < 1 ? 1 : g);
}

// ---------------------------------------------------- vertex transform ----
// src/scene.cpp:162-195: v' = L v + t, n' = normalize(R n),
// t' = (normalize(R t.xyz), t.w), with R the polar rotation of L.
__device__ __forceinline__ f3 mat_vec(const float* m, f3 v) {
  return {m[0] * v.x + (m[1] * v.y + m[2] * v.z), m[3] * v.x + (m[4] * v.y + m[5] * v.z),
          m[6] * v.x + (m[7] * v.y + m[8] * v.z)};
}

__global__ void k_transform(uint32_t nv, const uint32_t* __restrict__ vgeom, const float* __restrict__ lin,
                            const float* __restrict__ rot, const DGeom* __restrict__ geoms,
                            const float* __restrict__ ov, const float* __restrict__ on,
                            const float* __restrict__ ot, float* __restrict__ wv, float* __restrict__ wn,
                            float* __restrict__ wt) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    uint32_t g = vgeom[i];
    const float* L = lin + 12 * g;
    const float* R = rot + 9 * g;
    float Lm[9] = {L[0], L[1], L[2], L[4], L[5], L[6], L[8], L[9], L[10]};
    f3 v = ld3(ov, i);
    f3 m = mat_vec(Lm, v);
    wv[3 * i] = m.x + L[3];
    wv[3 * i + 1] = m.y + L[7];
    wv[3 * i + 2] = m.z + L[11];
    uint32_t fl = geoms[g].flags;
    if (fl & GEOM_HAS_NORMALS) {
      f3 n = normalized(mat_vec(R, ld3(on, i)));
      wn[3 * i] = n.x;
      wn[3 * i + 1] = n.y;
      wn[3 * i + 2] = n.z;
    }
    if (fl & GEOM_HAS_TANGENTS) {
      f3 t = {ot[4 * i], ot[4 * i + 1], ot[4 * i + 2]};
      f3 r = normalized(mat_vec(R, t));
      wt[4 * i] = r.x;
      wt[4 * i + 1] = r.y;
      wt[4 * i + 2] = r.z;
      wt[4 * i + 3] = ot[4 * i + 3];
    }
  }
}

// -------------------------------------------------------------- raster ----

struct RasterArgs {
  const uint32_t* tri_vidx;
  const uint32_t* tri_geom;
  const DGeom* geoms;
  const float* lm_uv;
  const float* wv;
  const float* wn;
  const float* wt;
  int W, H;
  uint32_t T;
};

__device__ __forceinline__ float min3(float a, float b, float c) {
  float m = a;
  if (b < m) m = b;
  if (c < m) m = c;
  return m;
}
__device__ __forceinline__ float max3(float a, float b, float c) {
  float m = a;
  if (m < b) m = b;
  if (m < c) m = c;
  return m;
}

// src/rasterizer.cpp:18-33
__device__ __forceinline__ bool barycentric(f2 p, f2 a, f2 b, f2 c, float& u, float& v, float& w) {
  f2 v0 = b - a, v1 = c - a, v2 = p - a;
  float d00 = dot2(v0, v0);
  float d01 = dot2(v0, v1);
  float d11 = dot2(v1, v1);
  float d20 = dot2(v2, v0);
  float d21 = dot2(v2, v1);
  float denom = d00 * d11 - d01 * d01;
  if (fabsf(denom) < 1e-8f) return false;
  v = (d11 * d20 - d01 * d21) / denom;
  w = (d00 * d21 - d01 * d20) / denom;
  u = 1.0f - v - w;
  return (v >= 0.0f) && (w >= 0.0f) && (u >= 0.0f);
}

// Per triangle: clamped UV bounding box in texels (src/rasterizer.cpp:97-112).
__global__ void k_tri_bbox(RasterArgs a, int4* __restrict__ box, int64_t* __restrict__ area) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.T; p += gridDim.x * blockDim.x) {
    uint32_t i0 = a.tri_vidx[3 * p], i1 = a.tri_vidx[3 * p + 1], i2 = a.tri_vidx[3 * p + 2];
    f2 uv0 = ld2(a.lm_uv, i0), uv1 = ld2(a.lm_uv, i1), uv2 = ld2(a.lm_uv, i2);
    float min_u = min3(uv0.x, uv1.x, uv2.x), max_u = max3(uv0.x, uv1.x, uv2.x);
    float min_v = min3(uv0.y, uv1.y, uv2.y), max_v = max3(uv0.y, uv1.y, uv2.y);
    int min_x = max(0, cvt_trunc(min_u * (float)a.W));
    int max_x = min(a.W - 1, cvt_trunc(ceilf(max_u * (float)a.W)));
    int min_y = max(0, cvt_trunc(min_v * (float)a.H));
    int max_y = min(a.H - 1, cvt_trunc(ceilf(max_v * (float)a.H)));
    int bw = max_x - min_x + 1, bh = max_y - min_y + 1;
    box[p] = make_int4(min_x, min_y, bw, bh);
    area[p] = (bw > 0 && bh > 0) ? (int64_t)bw * (int64_t)bh : 0;
  }
}

// One thread per candidate (triangle, texel) pair of all bounding boxes; the
// last writer in geometry-major triangle order wins (atomicMax of the order).
__global__ void k_cover(RasterArgs a, const int4* __restrict__ box, const int64_t* __restrict__ offs,
                        int64_t total, int* __restrict__ owner, uint8_t* __restrict__ hit) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < total;
       c += (int64_t)gridDim.x * blockDim.x) {
    // upper_bound over the exclusive offsets
    uint32_t lo = 0, hi = a.T;
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (__ldg(offs + mid) <= c) lo = mid + 1;
      else hi = mid;
    }
    uint32_t p = lo - 1;
    int4 b = box[p];
    int64_t local = c - offs[p];
    int x = b.x + (int)(local % b.z);
    int y = b.y + (int)(local / b.z);
    uint32_t i0 = a.tri_vidx[3 * p], i1 = a.tri_vidx[3 * p + 1], i2 = a.tri_vidx[3 * p + 2];
    f2 uv0 = ld2(a.lm_uv, i0), uv1 = ld2(a.lm_uv, i1), uv2 = ld2(a.lm_uv, i2);
    f2 pt = {((float)x + 0.5f) / (float)a.W, ((float)y + 0.5f) / (float)a.H};
    float u, v, w;
    if (!barycentric(pt, uv0, uv1, uv2, u, v, w)) continue;
    hit[p] = 1;
    atomicMax(owner + (int64_t)y * a.W + x, (int)p);
  }
}

__device__ __forceinline__ int prim_material(const RasterArgs& a, uint32_t p) {
  return a.geoms[a.tri_geom[p]].material_id;
}

// Triangles that cover no texel centre try their centroid texel
// (src/rasterizer.cpp:160-205).  With sequential semantics the write that
// survives is: the last covering triangle if its material is valid; else
// the first later fallback with a valid material, else the last later
// fallback (writes with material < 0 leave the texel looking empty).
__global__ void k_fallback(RasterArgs a, const uint8_t* __restrict__ hit, const int* __restrict__ owner,
                           int* __restrict__ fb_pos, int* __restrict__ fb_neg) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.T; p += gridDim.x * blockDim.x) {
    if (hit[p]) continue;
    uint32_t i0 = a.tri_vidx[3 * p], i1 = a.tri_vidx[3 * p + 1], i2 = a.tri_vidx[3 * p + 2];
    f2 uv0 = ld2(a.lm_uv, i0), uv1 = ld2(a.lm_uv, i1), uv2 = ld2(a.lm_uv, i2);
    float cu = (uv0.x + uv1.x + uv2.x) / 3.0f;
    float cv = (uv0.y + uv1.y + uv2.y) / 3.0f;
    int cx = cvt_trunc(cu * (float)a.W);
    int cy = cvt_trunc(cv * (float)a.H);
    if (!(cx >= 0 && cx < a.W && cy >= 0 && cy < a.H)) continue;
    int64_t t = (int64_t)cy * a.W + cx;
    int n = owner[t];
    if (n >= 0 && (prim_material(a, (uint32_t)n) >= 0 || (int)p < n)) continue;
    if (prim_material(a, p) >= 0) atomicMin(fb_pos + t, (int)p);
    else atomicMax(fb_neg + t, (int)p);
  }
}

__device__ void make_point(const RasterArgs& a, uint32_t p, float u, float v, float w,
                           shb_surface_point* out) {
  uint32_t i0 = a.tri_vidx[3 * p], i1 = a.tri_vidx[3 * p + 1], i2 = a.tri_vidx[3 * p + 2];
  f3 pos = ld3(a.wv, i0) * u + ld3(a.wv, i1) * v + ld3(a.wv, i2) * w;
  f3 nrm = normalized(ld3(a.wn, i0) * u + ld3(a.wn, i1) * v + ld3(a.wn, i2) * w);
  float4 t0 = __ldg(reinterpret_cast<const float4*>(a.wt) + i0);
  float4 t1 = __ldg(reinterpret_cast<const float4*>(a.wt) + i1);
  float4 t2 = __ldg(reinterpret_cast<const float4*>(a.wt) + i2);
  f3 t3 = {t0.x * u + t1.x * v + t2.x * w, t0.y * u + t1.y * v + t2.y * w, t0.z * u + t1.z * v + t2.z * w};
  float tw = t0.w * u + t1.w * v + t2.w * w;
  t3 = normalized(t3 - nrm * dot(nrm, t3));
  float4* o = reinterpret_cast<float4*>(out);
  o[0] = make_float4(pos.x, pos.y, pos.z, nrm.x);
  o[1] = make_float4(nrm.y, nrm.z, 0.f, 0.f);
  o[2] = make_float4(t3.x, t3.y, t3.z, tw);
  o[3] = make_float4(__int_as_float(a.geoms[a.tri_geom[p]].material_id), 0.f, 0.f, 0.f);
}

__global__ void k_resolve_raster(RasterArgs a, const int* __restrict__ owner, const int* __restrict__ fb_pos,
                                 const int* __restrict__ fb_neg, shb_surface_point* __restrict__ out) {
  int64_t n = (int64_t)a.W * a.H;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int own = owner[t], fp = fb_pos[t], fn = fb_neg[t];
    int p = -1;
    bool fallback = false;
    if (own >= 0 && prim_material(a, (uint32_t)own) >= 0) {
      p = own;
    } else if (fp != 0x7FFFFFFF) {
      p = fp;
      fallback = true;
    } else if (fn >= 0) {
      p = fn;
      fallback = true;
    } else if (own >= 0) {
      p = own;
    }
    if (p < 0) {
      float4* o = reinterpret_cast<float4*>(out + t);
      o[0] = make_float4(0.f, 0.f, 0.f, 0.f);
      o[1] = o[0];
      o[2] = o[0];
      o[3] = make_float4(__int_as_float(-1), 0.f, 0.f, 0.f);
      continue;
    }
    float u, v, w;
    if (fallback) {
      u = v = w = 1.0f / 3.0f;
    } else {
      int x = (int)(t % a.W), y = (int)(t / a.W);
      uint32_t i0 = a.tri_vidx[3 * p], i1 = a.tri_vidx[3 * p + 1], i2 = a.tri_vidx[3 * p + 2];
      f2 pt = {((float)x + 0.5f) / (float)a.W, ((float)y + 0.5f) / (float)a.H};
      barycentric(pt, ld2(a.lm_uv, i0), ld2(a.lm_uv, i1), ld2(a.lm_uv, i2), u, v, w);
    }
    make_point(a, (uint32_t)p, u, v, w, out + t);
  }
}

__global__ void k_fill_i32(int* p, int64_t n, int v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// --------------------------------------------------------------- masks ----

__global__ void k_validity(const shb_surface_point* __restrict__ pts, int64_t n, uint8_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = pts[i].material_id >= 0;
}

// src/rasterizer.cpp:222-241
__global__ void k_mask_down(const uint8_t* __restrict__ in, int w, int h, int s, uint8_t* __restrict__ out) {
  int64_t n = (int64_t)w * h;
  int stride = w * s;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int x = (int)(i % w), y = (int)(i / w);
    uint8_t any = 0;
    for (int sy = y * s; sy < (y + 1) * s && !any; ++sy)
      for (int sx = x * s; sx < (x + 1) * s; ++sx)
        if (in[(int64_t)sy * stride + sx]) {
          any = 1;
          break;
        }
    out[i] = any;
  }
}

// src/baker.cpp:151-182, one thread per (output texel, channel).
__global__ void k_downsample(const float* __restrict__ in, int in_w, int in_h, int ch, int s,
                             float* __restrict__ out) {
  int ow = in_w / s, oh = in_h / s;
  int64_t n = (int64_t)ow * oh * ch;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)(i % ch);
    int64_t texel = i / ch;
    int x = (int)(texel % ow), y = (int)(texel / ow);
    float avg = 0.0f;
    int count = 0;
    for (int dy = 0; dy < s; ++dy)
      for (int dx = 0; dx < s; ++dx) {
        int sx = x * s + dx, sy = y * s + dy;
        if (sx < in_w && sy < in_h) {
          avg += in[((int64_t)sy * in_w + sx) * ch + c];
          count++;
        }
      }
    out[i] = count > 0 ? avg * (1.f / float(count)) : 0.0f;
  }
}

// One dilation pass (src/dilation.cpp:25-66), one thread per (texel,
// channel).  Pass p is skipped when pass p-1 changed nothing: from then on
// every pass is the identity, and both ping-pong buffers hold the result.
template <class T>
__global__ void k_dilate(const T* __restrict__ pin, const uint8_t* __restrict__ min, T* __restrict__ pout,
                         uint8_t* __restrict__ mout, int w, int h, int ch, int* changed, int pass) {
  if (pass > 0 && *(volatile int*)(changed + pass - 1) == 0) return;
  int64_t n = (int64_t)w * h * ch;
  bool any = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)(i % ch);
    int64_t idx = i / ch;
    T v = pin[i];
    uint8_t m = min[idx];
    if (!m) {
      int x = (int)(idx % w), y = (int)(idx / w);
      T acc = T();
      int count = 0;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          if (dx == 0 && dy == 0) continue;
          int nx = x + dx, ny = y + dy;
          if (nx >= 0 && nx < w && ny >= 0 && ny < h) {
            int64_t ni = (int64_t)ny * w + nx;
            if (min[ni]) {
              acc = (T)(acc + pin[ni * ch + c]);
              count++;
            }
          }
        }
      if (count > 0) {
        v = (T)(acc * (1.0f / count));
        m = 1;
        any = true;
      }
    }
    pout[i] = v;
    if (c == 0) mout[idx] = m;
  }
  if (any) changed[pass] = 1;
}

}  // namespace

// ================================================================ host ====

shb_status transform_vertices(shb_scene* s) {
  if (s->vertex_count == 0) return SHB_OK;
  shb_context* c = s->ctx;
  k_transform<<<grid_for(s->vertex_count), kThreads, 0, c->stream>>>(
      s->vertex_count, s->vgeom.as<uint32_t>(), s->lin.as<float>(), s->rot.as<float>(), s->geoms.as<DGeom>(),
      s->obj_v.as<float>(), s->obj_n.as<float>(), s->obj_t.as<float>(), s->world_v.as<float>(),
      s->world_n.as<float>(), s->world_t.as<float>());
  count_launch(c);
  SHB_CUDA(cudaGetLastError());
  return SHB_OK;
}

shb_status rasterize_device(shb_scene* s, int W, int H, shb_surface_point* d_out) {
  shb_context* c = s->ctx;
  cudaStream_t st = c->stream;
  int64_t n = (int64_t)W * H;
  uint32_t T = s->prim_count;
  RasterArgs a{s->tri_vidx.as<uint32_t>(), s->tri_geom.as<uint32_t>(), s->geoms.as<DGeom>(),
               s->lm_uv.as<float>(), s->world_v.as<float>(), s->world_n.as<float>(),
               s->world_t.as<float>(), W, H, T};
  SHB_TRY(c->scratch[1].reserve(sizeof(int) * n * 3));
  int* owner = c->scratch[1].as<int>();
  int* fb_pos = owner + n;
  int* fb_neg = owner + 2 * n;
  k_fill_i32<<<grid_for(n), kThreads, 0, st>>>(owner, n, -1);
  k_fill_i32<<<grid_for(n), kThreads, 0, st>>>(fb_pos, n, 0x7FFFFFFF);
  k_fill_i32<<<grid_for(n), kThreads, 0, st>>>(fb_neg, n, -1);
  count_launch(c, 3);
  if (T > 0) {
    SHB_TRY(c->scratch[2].reserve(sizeof(int4) * T));
    SHB_TRY(c->scratch[3].reserve(sizeof(int64_t) * (T + 1) * 2));
    SHB_TRY(c->scratch[4].reserve(T));
    int4* box = c->scratch[2].as<int4>();
    int64_t* area = c->scratch[3].as<int64_t>();
    int64_t* offs = area + (T + 1);
    uint8_t* hit = c->scratch[4].as<uint8_t>();
    SHB_CUDA(cudaMemsetAsync(hit, 0, T, st));
    SHB_CUDA(cudaMemsetAsync(area + T, 0, sizeof(int64_t), st));
    k_tri_bbox<<<grid_for(T), kThreads, 0, st>>>(a, box, area);
    count_launch(c);
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, area, offs, (int64_t)T + 1, st);
    SHB_TRY(c->scratch[5].reserve(tmp_bytes));
    SHB_CUDA(cub::DeviceScan::ExclusiveSum(c->scratch[5].ptr, tmp_bytes, area, offs, (int64_t)T + 1, st));
    count_launch(c, 2);
    int64_t total = 0;
    SHB_CUDA(cudaMemcpyAsync(&total, offs + T, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SHB_CUDA(cudaStreamSynchronize(st));
    if (total > 0) {
      k_cover<<<grid_for(total), kThreads, 0, st>>>(a, box, offs, total, owner, hit);
      count_launch(c);
    }
    k_fallback<<<grid_for(T), kThreads, 0, st>>>(a, hit, owner, fb_pos, fb_neg);
    count_launch(c);
  }
  k_resolve_raster<<<grid_for(n), kThreads, 0, st>>>(a, owner, fb_pos, fb_neg, d_out);
  count_launch(c);
  SHB_CUDA(cudaGetLastError());
  return SHB_OK;
}

shb_status validity_mask_device(shb_context* c, const shb_surface_point* pts, int64_t n, uint8_t* out) {
  if (n <= 0) return SHB_OK;
  k_validity<<<grid_for(n), kThreads, 0, c->stream>>>(pts, n, out);
  count_launch(c);
  SHB_CUDA(cudaGetLastError());
  return SHB_OK;
}

shb_status downsample_mask_device(shb_context* c, const uint8_t* in, int w, int h, int s, uint8_t* out) {
  int64_t n = (int64_t)w * h;
  if (n <= 0) return SHB_OK;
  k_mask_down<<<grid_for(n), kThreads, 0, c->stream>>>(in, w, h, s, out);
  count_launch(c);
  SHB_CUDA(cudaGetLastError());
  return SHB_OK;
}

shb_status downsample_device(shb_context* c, const float* in, int w, int h, int ch, int s, float* out) {
  if (s <= 1) {
    SHB_CUDA(cudaMemcpyAsync(out, in, sizeof(float) * (size_t)w * h * ch, cudaMemcpyDeviceToDevice, c->stream));
    return SHB_OK;
  }
  int64_t n = (int64_t)(w / s) * (h / s) * ch;
  if (n <= 0) return SHB_OK;
  k_downsample<<<grid_for(n), kThreads, 0, c->stream>>>(in, w, h, ch, s, out);
  count_launch(c);
  SHB_CUDA(cudaGetLastError());
  return SHB_OK;
}

shb_status dilate_device(shb_context* c, int kind, int w, int h, void* pixels, uint8_t* mask, int passes) {
  int64_t n = (int64_t)w * h;
  if (n <= 0 || passes <= 0) return SHB_OK;
  int ch = kind == SHB_DILATE_SH9 ? 27 : 1;
  size_t esz = kind == SHB_DILATE_U8 ? 1 : 4;
  size_t pbytes = esz * (size_t)n * ch;
  SHB_TRY(c->scratch[6].reserve(pbytes));
  SHB_TRY(c->scratch[7].reserve((size_t)n));
  SHB_TRY(c->scratch[8].reserve(sizeof(int) * (size_t)passes));
  int* changed = c->scratch[8].as<int>();
  SHB_CUDA(cudaMemsetAsync(changed, 0, sizeof(int) * (size_t)passes, c->stream));
  void* bufs[2] = {pixels, c->scratch[6].ptr};
  uint8_t* masks[2] = {mask, c->scratch[7].as<uint8_t>()};
  int64_t work = n * ch;
  for (int p = 0; p < passes; ++p) {
    int src = p & 1, dst = src ^ 1;
    if (kind == SHB_DILATE_U8)
      k_dilate<uint8_t><<<grid_for(work), kThreads, 0, c->stream>>>(
          (const uint8_t*)bufs[src], masks[src], (uint8_t*)bufs[dst], masks[dst], w, h, ch, changed, p);
    else
      k_dilate<float><<<grid_for(work), kThreads, 0, c->stream>>>(
          (const float*)bufs[src], masks[src], (float*)bufs[dst], masks[dst], w, h, ch, changed, p);
    count_launch(c);
  }
  if (passes & 1) {
    SHB_CUDA(cudaMemcpyAsync(pixels, bufs[1], pbytes, cudaMemcpyDeviceToDevice, c->stream));
    SHB_CUDA(cudaMemcpyAsync(mask, masks[1], (size_t)n, cudaMemcpyDeviceToDevice, c->stream));
  }
  SHB_CUDA(cudaGetLastError());
  return SHB_OK;
}

}  // namespace shb

// ============================================= allocation-free dilation ====
//
// Some callers cannot allocate device memory while they run: a host
// application that owns the GPU's memory budget and reserves all of it up
// front (an editor or content tool baking lightmaps beside its renderer),
// and callers on a deadline path, where cudaMalloc's implicit device-wide
// synchronisation and unpredictable latency are not acceptable.  For them
// shb_dilate_noalloc runs the same dilation passes as shb_dilate, but the
// ping-pong copy of the pixels and mask and the per-pass change flags live
// in the fixed array below.  Its device address is looked up when a
// context is created on a device (noalloc_prepare), so the array is held on
// every device that has had a context, from then until the process exits.

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;  // 16 MiB
constexpr int kNoAllocMaxPasses = 4096;
constexpr size_t kNoAllocFlagBytes = sizeof(int) * kNoAllocMaxPasses;  // 16 KiB
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_device_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (current).  The name is
// only a host-side stand-in for the symbol, so the address comes from
// cudaGetSymbolAddress once per device and is cached.
shb_status noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) {
    shb::set_error("shb_dilate_noalloc: device ordinal out of range");
    return SHB_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_device_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return shb::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_device_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_device_addr[device]);
  return SHB_OK;
}

}  // namespace

namespace shb {
shb_status noalloc_prepare(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) return SHB_OK;  // the entry point reports it
  unsigned char* p = nullptr;
  return noalloc_scratch(device, &p);
}
}  // namespace shb

extern "C" SHB_API shb_status shb_dilate_noalloc(shb_context* ctx, int32_t kind, int32_t width, int32_t height,
                                                 void* pixels, uint8_t* mask, int32_t passes) {
  return ::shb::guarded("shb_dilate_noalloc", [&]() -> shb_status {
    using namespace shb;
    if (!ctx) {
      set_error("ctx is NULL");
      return SHB_ERR_INVALID_ARG;
    }
    if (kind < SHB_DILATE_SH9 || kind > SHB_DILATE_U8) {
      set_error("bad dilate kind");
      return SHB_ERR_INVALID_ARG;
    }
    if (width <= 0 || height <= 0 || passes <= 0) return SHB_OK;  // nothing to do, as Dilate<T>
    if (!pixels || !mask) {
      set_error("NULL argument");
      return SHB_ERR_INVALID_ARG;
    }
    const int64_t n = (int64_t)width * height;  // width, height > 0 and < 2^31: no overflow
    const int ch = kind == SHB_DILATE_SH9 ? 27 : 1;
    const size_t esz = kind == SHB_DILATE_U8 ? 1 : 4;
    auto too_large = [&](const std::string& need) {
      set_error("shb_dilate_noalloc: " + std::to_string(width) + "x" + std::to_string(height) + " texels need " + need +
                " bytes of scratch; the fixed array holds " + std::to_string(kNoAllocScratchBytes) +
                " (about 153,000 texels of SH9, 3.3 M of float, 8.3 M of uint8)");
      return SHB_ERR_INVALID_ARG;
    };
    // every texel needs at least one mask byte of scratch: bound n before the
    // byte counts below are formed
    if (n > (int64_t)kNoAllocScratchBytes) return too_large("more than " + std::to_string(n));
    const size_t pbytes = esz * (size_t)n * ch;
    const size_t pbytes_aligned = (pbytes + 255) & ~size_t(255);
    const size_t need = kNoAllocFlagBytes + pbytes_aligned + (size_t)n;
    if (passes > kNoAllocMaxPasses) {
      set_error("shb_dilate_noalloc: at most " + std::to_string(kNoAllocMaxPasses) + " passes");
      return SHB_ERR_INVALID_ARG;
    }
    if (need > kNoAllocScratchBytes) return too_large(std::to_string(need));
    SHB_ON_DEVICE(ctx->device);
    unsigned char* base = nullptr;
    SHB_TRY(noalloc_scratch(ctx->device, &base));
    int* changed = reinterpret_cast<int*>(base);
    void* pbuf = base + kNoAllocFlagBytes;
    uint8_t* mbuf = base + kNoAllocFlagBytes + pbytes_aligned;
    cudaStream_t st = ctx->stream;
    // the array keeps the previous call's contents: the change flags must start at zero
    SHB_CUDA(cudaMemsetAsync(changed, 0, sizeof(int) * (size_t)passes, st));
    void* bufs[2] = {pixels, pbuf};
    uint8_t* masks[2] = {mask, mbuf};
    const int64_t work = n * ch;
    for (int p = 0; p < passes; ++p) {
      int src = p & 1, dst = src ^ 1;
      if (kind == SHB_DILATE_U8)
        k_dilate<uint8_t><<<grid_for(work), kThreads, 0, st>>>((const uint8_t*)bufs[src], masks[src],
                                                               (uint8_t*)bufs[dst], masks[dst], width, height, ch,
                                                               changed, p);
      else
        k_dilate<float><<<grid_for(work), kThreads, 0, st>>>((const float*)bufs[src], masks[src], (float*)bufs[dst],
                                                             masks[dst], width, height, ch, changed, p);
      count_launch(ctx);
    }
    if (passes & 1) {
      SHB_CUDA(cudaMemcpyAsync(pixels, bufs[1], pbytes, cudaMemcpyDeviceToDevice, st));
      SHB_CUDA(cudaMemcpyAsync(mask, masks[1], (size_t)n, cudaMemcpyDeviceToDevice, st));
    }
    SHB_CUDA(cudaGetLastError());
    return SHB_OK;
  });
}
