// traverse.cu - closest-hit and any-hit traversal of the compressed 8-wide
// BVH; replaces rtcIntersect1 (src/occlusion.cpp:37) for path rays and for
// shadow rays (src/light.cpp:173,275).
//
// Persistent kernels: a grid sized to fill every SM once; each warp takes
// 32 queue entries at a time from an atomic counter until the queue (whose
// length lives in device memory) is drained.  Children are visited in the
// ray-octant order of their slots; the watertight triangle test (Woop,
// Benthin, Wald 2013) is written with explicit round-to-nearest intrinsics
// so it rounds exactly like the CPU restatement even though this file is
// compiled with FMA contraction enabled for the box tests.
#include "wavefront.h"

namespace shb {

namespace {

constexpr int kStack = 64;
constexpr int kTravThreads = 128;

struct TravRay {
  float ox, oy, oz, dx, dy, dz;
  // watertight test
  int kx, ky, kz;
  float Sx, Sy, Sz;
  // box test
  float ix, iy, iz;
  uint32_t oct;
};

__device__ __forceinline__ float comp(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

__device__ __forceinline__ void prepare(TravRay& r) {
  float ax = fabsf(r.dx), ay = fabsf(r.dy), az = fabsf(r.dz);
  int kz = 0;
  if (ay > ax) kz = 1;
  if (az > (kz == 0 ? ax : ay)) kz = 2;
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  float dkz = comp(r.dx, r.dy, r.dz, kz);
  if (dkz < 0.f) {
    int t = kx;
    kx = ky;
    ky = t;
  }
  r.kx = kx;
  r.ky = ky;
  r.kz = kz;
  r.Sx = __fdiv_rn(comp(r.dx, r.dy, r.dz, kx), dkz);
  r.Sy = __fdiv_rn(comp(r.dx, r.dy, r.dz, ky), dkz);
  r.Sz = __fdiv_rn(1.0f, dkz);
  const float tiny = 1e-20f;
  r.ix = 1.0f / (fabsf(r.dx) > tiny ? r.dx : copysignf(tiny, r.dx));
  r.iy = 1.0f / (fabsf(r.dy) > tiny ? r.dy : copysignf(tiny, r.dy));
  r.iz = 1.0f / (fabsf(r.dz) > tiny ? r.dz : copysignf(tiny, r.dz));
  r.oct = (r.dx < 0.f ? 1u : 0u) | (r.dy < 0.f ? 2u : 0u) | (r.dz < 0.f ? 4u : 0u);
}

// Watertight ray/triangle test; accepts tnear < t < tfar (t in units of
// |d|); u, v are the weights of v1, v2.
__device__ __forceinline__ bool tri_test(const TravRay& r, float4 a, float4 b, float4 c, float tnear, float tfar,
                                         float& t, float& u, float& v) {
  float Ax_ = __fsub_rn(a.x, r.ox), Ay_ = __fsub_rn(a.y, r.oy), Az_ = __fsub_rn(a.z, r.oz);
  float Bx_ = __fsub_rn(b.x, r.ox), By_ = __fsub_rn(b.y, r.oy), Bz_ = __fsub_rn(b.z, r.oz);
  float Cx_ = __fsub_rn(c.x, r.ox), Cy_ = __fsub_rn(c.y, r.oy), Cz_ = __fsub_rn(c.z, r.oz);
  float Akz = comp(Ax_, Ay_, Az_, r.kz), Bkz = comp(Bx_, By_, Bz_, r.kz), Ckz = comp(Cx_, Cy_, Cz_, r.kz);
  float Ax = __fsub_rn(comp(Ax_, Ay_, Az_, r.kx), __fmul_rn(r.Sx, Akz));
  float Ay = __fsub_rn(comp(Ax_, Ay_, Az_, r.ky), __fmul_rn(r.Sy, Akz));
  float Bx = __fsub_rn(comp(Bx_, By_, Bz_, r.kx), __fmul_rn(r.Sx, Bkz));
  float By = __fsub_rn(comp(Bx_, By_, Bz_, r.ky), __fmul_rn(r.Sy, Bkz));
  float Cx = __fsub_rn(comp(Cx_, Cy_, Cz_, r.kx), __fmul_rn(r.Sx, Ckz));
  float Cy = __fsub_rn(comp(Cx_, Cy_, Cz_, r.ky), __fmul_rn(r.Sy, Ckz));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.f || V == 0.f || W == 0.f) {
    U = __double2float_rn(__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx)));
    V = __double2float_rn(__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx)));
    W = __double2float_rn(__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax)));
  }
  if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
  float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.f) return false;
  float Az = __fmul_rn(r.Sz, Akz), Bz = __fmul_rn(r.Sz, Bkz), Cz = __fmul_rn(r.Sz, Ckz);
  float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
  if (det < 0.f) {
    T = -T;
    det = -det;
    V = -V;
    W = -W;
  }
  if (!(T > __fmul_rn(tnear, det) && T < __fmul_rn(tfar, det))) return false;
  t = __fdiv_rn(T, det);
  u = __fdiv_rn(V, det);
  v = __fdiv_rn(W, det);
  return true;
}

__device__ __forceinline__ float byte_f(uint32_t w, int k) {
  return __uint_as_float(0x4B000000u | ((w >> (8 * k)) & 0xFFu)) - 8388608.0f;
}

// Returns true on a hit; for ANY the first hit ends the walk.
template <bool ANY>
__device__ bool traverse(const BvhView& bvh, const TravRay& r, float tnear, float tfar, float& t_out, float& u_out,
                         float& v_out, uint32_t& prim_out, int* err) {
  if (bvh.node_count == 0) return false;
  uint2 stack[kStack];
  int sp = 0;
  const uint32_t oct = r.oct;
  uint32_t ng_base = 0, ng_hits = 1u << oct, ng_imask = 1u;
  uint32_t tg_base = 0, tg_hits = 0;
  float tmax = tfar;
  bool hit = false;
  const uint4* nodes = reinterpret_cast<const uint4*>(bvh.nodes);
  // Every child index is larger than its parent's, so the walk ends; the
  // bound only turns a corrupted tree into an error flag.
  uint32_t iters = 0;
  while (true) {
    if (++iters > (1u << 22)) {
      atomicOr(err, ERR_ITER);
      break;
    }
    while (tg_hits) {
      int k = __ffs(tg_hits) - 1;
      tg_hits &= tg_hits - 1;
      const float4* tp = bvh.tris + 3 * (size_t)(tg_base + k);
      float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
      float t, u, v;
      if (tri_test(r, a, b, c, tnear, tmax, t, u, v)) {
        hit = true;
        tmax = t;
        t_out = t;
        u_out = u;
        v_out = v;
        prim_out = __float_as_uint(a.w);
        if (ANY) return true;
      }
    }
    if (ng_hits == 0) {
      if (sp == 0) break;
      --sp;
      ng_base = stack[sp].x;
      ng_hits = stack[sp].y & 0xFFu;
      ng_imask = stack[sp].y >> 8;
    }
    int bpos = __ffs(ng_hits) - 1;
    ng_hits &= ng_hits - 1;
    uint32_t slot = (uint32_t)bpos ^ oct;
    uint32_t node = ng_base + __popc(ng_imask & ((1u << slot) - 1u));
    if (ng_hits) {
      if (sp < kStack) {
        stack[sp++] = make_uint2(ng_base, ng_hits | (ng_imask << 8));
      } else {
        atomicOr(err, ERR_STACK);
      }
    }
    const uint4* np = nodes + 5 * (size_t)node;
    uint4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
    float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    uint32_t eim = n0.w;
    float sx = __uint_as_float((eim & 0xFFu) << 23) * r.ix;
    float sy = __uint_as_float(((eim >> 8) & 0xFFu) << 23) * r.iy;
    float sz = __uint_as_float(((eim >> 16) & 0xFFu) << 23) * r.iz;
    float ax = (px - r.ox) * r.ix, ay = (py - r.oy) * r.iy, az = (pz - r.oz) * r.iz;
    uint32_t imask = eim >> 24;
    // near / far quantised planes per axis (octant select)
    uint32_t lx0 = n2.x, lx1 = n2.y, ly0 = n2.z, ly1 = n2.w, lz0 = n3.x, lz1 = n3.y;
    uint32_t hx0 = n3.z, hx1 = n3.w, hy0 = n4.x, hy1 = n4.y, hz0 = n4.z, hz1 = n4.w;
    if (oct & 1u) { uint32_t t0 = lx0, t1 = lx1; lx0 = hx0; lx1 = hx1; hx0 = t0; hx1 = t1; }
    if (oct & 2u) { uint32_t t0 = ly0, t1 = ly1; ly0 = hy0; ly1 = hy1; hy0 = t0; hy1 = t1; }
    if (oct & 4u) { uint32_t t0 = lz0, t1 = lz1; lz0 = hz0; lz1 = hz1; hz0 = t0; hz1 = t1; }
    uint32_t hits_int = 0, hits_tri = 0;
    const float tlim = tmax * 1.0000004f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      uint32_t meta = ((j < 4 ? n1.z : n1.w) >> (8 * (j & 3))) & 0xFFu;
      int k = j & 3;
      float nx = byte_f(j < 4 ? lx0 : lx1, k), fx = byte_f(j < 4 ? hx0 : hx1, k);
      float ny = byte_f(j < 4 ? ly0 : ly1, k), fy = byte_f(j < 4 ? hy0 : hy1, k);
      float nz = byte_f(j < 4 ? lz0 : lz1, k), fz = byte_f(j < 4 ? hz0 : hz1, k);
      float t0x = fmaf(nx, sx, ax), t1x = fmaf(fx, sx, ax);
      float t0y = fmaf(ny, sy, ay), t1y = fmaf(fy, sy, ay);
      float t0z = fmaf(nz, sz, az), t1z = fmaf(fz, sz, az);
      float tmin_c = fmaxf(fmaxf(t0x, t0y), fmaxf(t0z, tnear));
      float tmax_c = fminf(fminf(t1x, t1y), fminf(t1z, tlim));
      bool h = meta != 0u && tmin_c <= tmax_c;
      if (h) {
        if (imask & (1u << j)) {
          hits_int |= 1u << ((uint32_t)j ^ oct);
        } else {
          uint32_t cnt = meta >> 5, off = meta & 31u;
          hits_tri |= ((1u << cnt) - 1u) << off;
        }
      }
    }
    ng_base = n1.x;
    ng_hits = hits_int;
    ng_imask = imask;
    tg_base = n1.y;
    tg_hits = hits_tri;
  }
  return hit;
}

__device__ __forceinline__ void load_ray(TravRay& r, float4 o, float4 d) {
  r.ox = o.x;
  r.oy = o.y;
  r.oz = o.z;
  r.dx = d.x;
  r.dy = d.y;
  r.dz = d.z;
  prepare(r);
}

__global__ void __launch_bounds__(kTravThreads) k_extend(BvhView bvh, ExtQueue q, const int* __restrict__ n_ptr, int cap,
                                                        float4* __restrict__ hits, int* fetch, int* err,
                                                        Counters64* stats) {
  const int n = min(*n_ptr, cap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(&stats->extend_rays, (unsigned long long)n);
  const int lane = threadIdx.x & 31;
  while (true) {
    int base = 0;
    if (lane == 0) base = atomicAdd(fetch, 32);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base >= n) break;
    int i = base + lane;
    if (i < n) {
      TravRay r;
      load_ray(r, q.o[i], q.d[i]);
      float t = 0.f, u = 0.f, v = 0.f;
      uint32_t prim = kMissPrim;
      bool h = traverse<false>(bvh, r, 0.001f, INFINITY, t, u, v, prim, err);
      hits[i] = h ? make_float4(t, u, v, __uint_as_float(prim)) : make_float4(0.f, 0.f, 0.f, __uint_as_float(kMissPrim));
    }
  }
}

__global__ void __launch_bounds__(kTravThreads) k_shadow(BvhView bvh, ShadowQueue q, const int* __restrict__ n_ptr, int cap,
                                                        float4* __restrict__ path_L, float4* __restrict__ nee_li,
                                                        int* fetch, int* err, Counters64* stats) {
  const int n = min(*n_ptr, cap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(&stats->shadow_rays, (unsigned long long)n);
  const int lane = threadIdx.x & 31;
  while (true) {
    int base = 0;
    if (lane == 0) base = atomicAdd(fetch, 32);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base >= n) break;
    int i = base + lane;
    if (i < n) {
      float4 o = q.o[i], d = q.d[i];
      TravRay r;
      load_ray(r, o, d);
      float t, u, v;
      uint32_t prim;
      bool occ = traverse<true>(bvh, r, 0.001f, o.w, t, u, v, prim, err);
      float4 c = q.c[i];
      uint32_t target = __float_as_uint(d.w);
      if (__float_as_uint(c.w) == 0u) {
        if (!occ) {
          float4* L = path_L + target;
          atomicAdd(&L->x, c.x);
          atomicAdd(&L->y, c.y);
          atomicAdd(&L->z, c.z);
        }
      } else if (occ) {
        nee_li[target] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }
}

__global__ void k_closest_rays(BvhView bvh, const shb_ray* __restrict__ rays, int64_t n, float4* __restrict__ hits,
                               int* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const shb_ray& sr = rays[i];
    TravRay r;
    r.ox = sr.origin[0];
    r.oy = sr.origin[1];
    r.oz = sr.origin[2];
    r.dx = sr.direction[0];
    r.dy = sr.direction[1];
    r.dz = sr.direction[2];
    prepare(r);
    float t = 0.f, u = 0.f, v = 0.f;
    uint32_t prim = kMissPrim;
    bool h = traverse<false>(bvh, r, sr.tnear, sr.tfar, t, u, v, prim, err);
    hits[i] = h ? make_float4(t, u, v, __uint_as_float(prim)) : make_float4(0.f, 0.f, 0.f, __uint_as_float(kMissPrim));
  }
}

}  // namespace

int traversal_grid(int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_extend, kTravThreads, 0);
  if (per_sm < 1) per_sm = 1;
  if (sms < 1) sms = 1;
  return sms * per_sm;
}

void launch_extend(cudaStream_t st, int grid, const BvhView& bvh, ExtQueue q, const int* n, int cap, float4* hits, int* fetch,
                   int* err, Counters64* stats) {
  k_extend<<<grid, kTravThreads, 0, st>>>(bvh, q, n, cap, hits, fetch, err, stats);
}

void launch_shadow(cudaStream_t st, int grid, const BvhView& bvh, ShadowQueue q, const int* n, int cap, float4* path_L,
                   float4* nee_li, int* fetch, int* err, Counters64* stats) {
  k_shadow<<<grid, kTravThreads, 0, st>>>(bvh, q, n, cap, path_L, nee_li, fetch, err, stats);
}

void launch_closest_rays(cudaStream_t st, const BvhView& bvh, const shb_ray* rays, int64_t n, float4* hits, int* err) {
  if (n <= 0) return;
  int64_t g = (n + 127) / 128;
  if (g > 148 * 16) g = 148 * 16;
  k_closest_rays<<<(int)g, 128, 0, st>>>(bvh, rays, n, hits, err);
}

}  // namespace shb
