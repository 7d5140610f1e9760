// traverse.cu - closest-hit and any-hit traversal of the compressed 8-wide
// BVH; replaces rtcIntersect1 (src/occlusion.cpp:37) for path rays and for
// shadow rays (src/light.cpp:173,275).
//
// Persistent kernels with per-lane ray replacement: the grid fills every SM
// once; a lane whose ray finishes takes the next queue entry (one atomic per
// warp for all lanes that refill), so lanes do not wait for the slowest ray
// of a batch.  Within a ray, children are visited in the ray-octant order of
// their slots.  Triangle groups can be postponed on the stack while too few
// lanes of the warp want to test triangles (Ylitie, Karras, Laine 2017);
// measured here that only slows both kernels down (the any-hit kernel most,
// it ends on the first triangle it hits), so SHB_POSTPONE defaults to off.
// The watertight triangle test (Woop, Benthin, Wald 2013) uses explicit
// round-to-nearest intrinsics so it rounds exactly like the CPU restatement
// even though this file is compiled with FMA contraction for the box tests.
#include "wavefront.h"

namespace shb {

namespace {

constexpr int kStack = 64;
constexpr int kTravThreads = 128;
// Resident blocks per SM the traversal kernels are register-limited to
// (0: the compiler's choice).
#ifndef SHB_TRAV_MIN_BLOCKS
#define SHB_TRAV_MIN_BLOCKS 0
#endif
#if SHB_TRAV_MIN_BLOCKS > 0
#define SHB_TRAV_BOUNDS __launch_bounds__(kTravThreads, SHB_TRAV_MIN_BLOCKS)
#else
#define SHB_TRAV_BOUNDS __launch_bounds__(kTravThreads)
#endif
#ifndef SHB_POSTPONE
#define SHB_POSTPONE 0
#endif
constexpr int kPostpone = SHB_POSTPONE;  // fewer lanes than this on triangles: postpone them
constexpr uint32_t kNodeGroup = 0x80000000u;
constexpr uint32_t kMaxIters = 1u << 22;  // default bound of one ray's traversal steps

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

// Byte k of w as a float (exact): one byte permute builds the bit pattern
// 0x4B0000bb = 2^23 + bb, from which 2^23 is subtracted.
__device__ __forceinline__ float byte_f(uint32_t w, int k) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | (uint32_t)k)) - 8388608.0f;
}


// Traversal state of one ray.  Groups are (base, bits): a node group has
// kNodeGroup set, the internal-child mask in bits 8..15 and the remaining
// hit slots (in ray-octant order) in bits 0..7; a triangle group has the
// remaining triangle bits 0..23.
struct Walk {
  TravRay r;
  float tnear, tmax;
  uint2 G, T;
  int sp;
  uint32_t iters;
  bool hit;
  float u, v;
  uint32_t prim;
};

__device__ __forceinline__ void walk_init(Walk& w, const BvhView& bvh, float tnear, float tfar) {
  w.tnear = tnear;
  w.tmax = tfar;
  w.G = bvh.node_count ? make_uint2(0u, kNodeGroup | (1u << 8) | (1u << w.r.oct)) : make_uint2(0u, 0u);
  w.T = make_uint2(0u, 0u);
  w.sp = 0;
  w.iters = 0;
  w.hit = false;
  w.u = w.v = 0.f;
  w.prim = kMissPrim;
}

// max / min of three floats, NaN operands ignored like fmaxf / fminf
// (PTX three-input max.f32 / min.f32).
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
// Mask of `width` bits from bit `pos` (both taken modulo 32 / clamped like
// PTX bmsk.clamp: width 0 gives 0).
__device__ __forceinline__ uint32_t bit_mask(uint32_t pos, uint32_t width) {
  uint32_t r;
  asm("bmsk.clamp.b32 %0, %1, %2;" : "=r"(r) : "r"(pos), "r"(width));
  return r;
}
__device__ __forceinline__ uint32_t bfe(uint32_t x, uint32_t pos, uint32_t len) {
  uint32_t r;
  asm("bfe.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(pos), "r"(len));
  return r;
}

// Tests the 8 children of `node`; returns the internal children as a node
// group and the hit leaf triangles as a triangle group.
//
// Every child adds its meta byte's bits to one 32-bit hit mask (triangles
// in bits 0..23, internal children at 24 + slot): the internal children's
// slots are first XORed with the ray octant, four at a time, so bits
// 24..31 come out in visiting order (the compressed wide BVH traversal of
// Ylitie, Karras and Laine 2017).
__device__ __forceinline__ void intersect_node(const BvhView& bvh, const Walk& w, uint32_t node, uint2& Gn,
                                               uint2& Tn) {
  const TravRay& r = w.r;
  const uint4* np = reinterpret_cast<const uint4*>(bvh.nodes) + 5 * (size_t)node;
  uint4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
  uint32_t eim = n0.w;
  float sx = __uint_as_float((eim & 0xFFu) << 23) * r.ix;
  float sy = __uint_as_float(((eim >> 8) & 0xFFu) << 23) * r.iy;
  float sz = __uint_as_float(((eim >> 16) & 0xFFu) << 23) * r.iz;
  float ax = (__uint_as_float(n0.x) - r.ox) * r.ix;
  float ay = (__uint_as_float(n0.y) - r.oy) * r.iy;
  float az = (__uint_as_float(n0.z) - r.oz) * r.iz;
  uint32_t imask = eim >> 24;
  const uint32_t oct = r.oct;
  uint32_t lx0 = n2.x, lx1 = n2.y, ly0 = n2.z, ly1 = n2.w, lz0 = n3.x, lz1 = n3.y;
  uint32_t hx0 = n3.z, hx1 = n3.w, hy0 = n4.x, hy1 = n4.y, hz0 = n4.z, hz1 = n4.w;
  if (oct & 1u) { uint32_t t0 = lx0, t1 = lx1; lx0 = hx0; lx1 = hx1; hx0 = t0; hx1 = t1; }
  if (oct & 2u) { uint32_t t0 = ly0, t1 = ly1; ly0 = hy0; ly1 = hy1; hy0 = t0; hy1 = t1; }
  if (oct & 4u) { uint32_t t0 = lz0, t1 = lz1; lz0 = hz0; lz1 = hz1; hz0 = t0; hz1 = t1; }
  const float tlim = w.tmax * 1.0000004f;
  const uint32_t oct4 = oct * 0x01010101u;
  // internal children have position bits 3 and 4 both set (24..31)
  const uint32_t m_lo = n1.z ^ (__vcmpeq4(n1.z & 0x18181818u, 0x18181818u) & oct4);
  const uint32_t m_hi = n1.w ^ (__vcmpeq4(n1.w & 0x18181818u, 0x18181818u) & oct4);
  uint32_t hm = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int k = j & 3;
    const uint32_t mw = j < 4 ? m_lo : m_hi;
    float t0x = fmaf(byte_f(j < 4 ? lx0 : lx1, k), sx, ax), t1x = fmaf(byte_f(j < 4 ? hx0 : hx1, k), sx, ax);
    float t0y = fmaf(byte_f(j < 4 ? ly0 : ly1, k), sy, ay), t1y = fmaf(byte_f(j < 4 ? hy0 : hy1, k), sy, ay);
    float t0z = fmaf(byte_f(j < 4 ? lz0 : lz1, k), sz, az), t1z = fmaf(byte_f(j < 4 ? hz0 : hz1, k), sz, az);
    const float tmin_c = fmaxf(max3f(t0x, t0y, t0z), w.tnear);
    const float tmax_c = fminf(min3f(t1x, t1y, t1z), tlim);
    const uint32_t bits = bit_mask(bfe(mw, 8 * k, 5), bfe(mw, 8 * k + 5, 3));
    if (tmin_c <= tmax_c) hm |= bits;
  }
  Gn = make_uint2(n1.x, kNodeGroup | (imask << 8) | (hm >> 24));
  Tn = make_uint2(n1.y, hm & 0x00FFFFFFu);
}

// One step: visit one node (or take a popped triangle group) and test the
// current triangle group.  Returns true when the ray is finished.
template <bool ANY>
__device__ __forceinline__ bool walk_step(const BvhView& bvh, Walk& w, uint2* stack, int* err, uint32_t max_iters) {
  if (++w.iters > max_iters) {
    atomicOr(err, ERR_ITER);
    return true;
  }
  bool descended = false;
  if ((w.G.y & kNodeGroup) && (w.G.y & 0xFFu)) {
    uint32_t hits = w.G.y & 0xFFu;
    uint32_t imask = (w.G.y >> 8) & 0xFFu;
    int bpos = __ffs(hits) - 1;
    hits &= hits - 1;
    uint32_t slot = (uint32_t)bpos ^ w.r.oct;
    uint32_t node = w.G.x + __popc(imask & ((1u << slot) - 1u));
    if (hits) {
      if (w.sp < kStack) stack[w.sp++] = make_uint2(w.G.x, kNodeGroup | (imask << 8) | hits);
      else atomicOr(err, ERR_STACK);
    }
    uint2 Tn;
    intersect_node(bvh, w, node, w.G, Tn);
    w.T = Tn;
    descended = true;
  } else if (!(w.G.y & kNodeGroup)) {
    w.T = w.G;  // a popped triangle group
    w.G = make_uint2(0u, 0u);
  } else {
    w.G = make_uint2(0u, 0u);
  }
  while (w.T.y) {
    // postpone when few lanes test triangles and this ray still has nodes to visit
    if (descended && (w.G.y & 0xFFu) && __popc(__activemask()) < kPostpone) {
      if (w.sp < kStack) {
        stack[w.sp++] = w.T;
        w.T.y = 0;
        break;
      }
    }
    int k = __ffs(w.T.y) - 1;
    w.T.y &= w.T.y - 1;
    const float4* tp = bvh.tris + 3 * (size_t)(w.T.x + k);
    float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
    float t, u, v;
    if (tri_test(w.r, a, b, c, w.tnear, w.tmax, t, u, v)) {
      w.hit = true;
      w.tmax = t;
      w.u = u;
      w.v = v;
      w.prim = __float_as_uint(a.w);
      if (ANY) return true;
    }
  }
  bool g_empty = !((w.G.y & kNodeGroup) ? (w.G.y & 0xFFu) : w.G.y);
  if (g_empty) {
    if (w.sp == 0) return true;
    w.G = stack[--w.sp];
  }
  return false;
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

// Persistent queue consumer: lanes refill from the queue as their rays end.
// `bvh_of(i, o, d)` gives the BVH of queue entry i (its bake's).
template <bool SHADOW, class Q, class B, class Fin>
__device__ __forceinline__ void consume(const Q& q, int n, int* fetch, int* err, uint32_t max_iters, B&& bvh_of,
                                       Fin&& finish) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  uint2 stack[kStack];
  Walk w;
  BvhView bvh;
  int ray = -1;
  bool exhausted = false;
  while (true) {
    bool need = ray < 0 && !exhausted;
    unsigned needm = __ballot_sync(0xFFFFFFFFu, need);
    if (needm) {
      int leader = __ffs(needm) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(fetch, __popc(needm));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (need) {
        int r = base + __popc(needm & lt);
        if (r < n) {
          ray = r;
          float4 o = q.o[r], d = q.d[r];
          bvh = bvh_of(r, o, d);
          load_ray(w.r, o, d);
          walk_init(w, bvh, 0.001f, SHADOW ? o.w : INFINITY);
        } else {
          exhausted = true;
        }
      }
    }
    if (!__any_sync(0xFFFFFFFFu, ray >= 0)) break;
    if (ray >= 0) {
      if (walk_step<SHADOW>(bvh, w, stack, err, max_iters)) {
        finish(ray, w);
        ray = -1;
      }
    }
  }
}

__global__ void SHB_TRAV_BOUNDS k_extend(const BakeItem* __restrict__ bakes, int n_bakes,
                                                        const PathInfo* __restrict__ info, ExtQueue q,
                                                        const int* __restrict__ n_ptr, int cap,
                                                        float4* __restrict__ hits, int* fetch, int* err,
                                                        Counters64* stats, uint32_t max_iters) {
  const int n = min(*n_ptr, cap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(&stats->extend_rays, (unsigned long long)n);
  const BvhView bvh0 = bakes[0].bvh;
  auto bvh_of = [&](int, float4 o, float4) {
    return n_bakes == 1 ? bvh0 : bakes[info[__float_as_uint(o.w)].x].bvh;
  };
  consume<false>(q, n, fetch, err, max_iters, bvh_of, [&](int i, const Walk& w) {
    hits[i] = w.hit ? make_float4(w.tmax, w.u, w.v, __uint_as_float(w.prim))
                    : make_float4(0.f, 0.f, 0.f, __uint_as_float(kMissPrim));
  });
}

__global__ void SHB_TRAV_BOUNDS k_shadow(const BakeItem* __restrict__ bakes, int n_bakes, ShadowQueue q,
                                                        const int* __restrict__ n_ptr, int cap,
                                                        float4* __restrict__ path_L, float4* __restrict__ nee_li,
                                                        float4* __restrict__ pend, int* fetch, int* err,
                                                        Counters64* stats, uint32_t max_iters) {
  const int n = min(*n_ptr, cap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(&stats->shadow_rays, (unsigned long long)n);
  const BvhView bvh0 = bakes[0].bvh;
  auto bvh_of = [&](int i, float4, float4) {
    return n_bakes == 1 ? bvh0 : bakes[__float_as_uint(q.c[i].w) >> 2].bvh;
  };
  consume<true>(q, n, fetch, err, max_iters, bvh_of, [&](int i, const Walk& w) {
    float4 c = q.c[i];
    uint32_t target = __float_as_uint(q.d[i].w);
    const uint32_t kind = __float_as_uint(c.w) & 3u;
    if (kind == 0u) {
      if (!w.hit) {
        float4* L = path_L + target;
        atomicAdd(&L->x, c.x);
        atomicAdd(&L->y, c.y);
        atomicAdd(&L->z, c.z);
      }
    } else if (w.hit) {
      (kind == 1u ? nee_li : pend)[target] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  });
}

__global__ void k_closest_rays(BvhView bvh, const shb_ray* __restrict__ rays, int64_t n, float4* __restrict__ hits,
                               int* err) {
  uint2 stack[kStack];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const shb_ray& sr = rays[i];
    Walk w;
    w.r.ox = sr.origin[0];
    w.r.oy = sr.origin[1];
    w.r.oz = sr.origin[2];
    w.r.dx = sr.direction[0];
    w.r.dy = sr.direction[1];
    w.r.dz = sr.direction[2];
    prepare(w.r);
    walk_init(w, bvh, sr.tnear, sr.tfar);
    while (!walk_step<false>(bvh, w, stack, err, kMaxIters)) {
    }
    hits[i] = w.hit ? make_float4(w.tmax, w.u, w.v, __uint_as_float(w.prim))
                    : make_float4(0.f, 0.f, 0.f, __uint_as_float(kMissPrim));
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

void launch_extend(cudaStream_t st, int grid, const BakeItem* bakes, int n_bakes, const PathInfo* info, ExtQueue q,
                   const int* n, int cap, float4* hits, int* fetch, int* err, Counters64* stats, uint32_t max_iters) {
  k_extend<<<grid, kTravThreads, 0, st>>>(bakes, n_bakes, info, q, n, cap, hits, fetch, err, stats,
                                          max_iters ? max_iters : kMaxIters);
}

void launch_shadow(cudaStream_t st, int grid, const BakeItem* bakes, int n_bakes, ShadowQueue q, const int* n, int cap,
                   float4* path_L, float4* nee_li, float4* pend, int* fetch, int* err, Counters64* stats,
                   uint32_t max_iters) {
  k_shadow<<<grid, kTravThreads, 0, st>>>(bakes, n_bakes, q, n, cap, path_L, nee_li, pend, fetch, err, stats,
                                          max_iters ? max_iters : kMaxIters);
}

void launch_closest_rays(cudaStream_t st, const BvhView& bvh, const shb_ray* rays, int64_t n, float4* hits, int* err) {
  if (n <= 0) return;
  int64_t g = (n + 127) / 128;
  if (g > sm_count() * 16) g = sm_count() * 16;
  k_closest_rays<<<(int)g, 128, 0, st>>>(bvh, rays, n, hits, err);
}

}  // namespace shb
