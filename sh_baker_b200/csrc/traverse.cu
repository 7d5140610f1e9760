// traverse.cu - closest-hit and any-hit traversal of the compressed 8-wide
// BVH; replaces rtcIntersect1 (src/occlusion.cpp:37) for path rays and for
// shadow rays (src/light.cpp:173,275).
//
// Persistent kernels with per-lane ray replacement: the grid fills every SM
// once; lanes whose rays finished take the next queue entries together (one
// atomic per warp) once enough of them wait, so lanes do not wait for the
// slowest ray of a batch.  Within a ray, children are visited in the
// ray-octant order of their slots.
//
// Each traversal step is a node visit per lane followed by a triangle phase
// for the whole warp: the triangles that the visited nodes' hit leaves hold
// (a few lanes have several, most have none) are spread over all 32 lanes,
// one test per lane, instead of each lane looping over its own.  Each ray's
// lane then replays its accepted tests in triangle order against its
// shrinking tmax, which gives exactly the hit a sequential loop gives.
// The watertight triangle test (Woop, Benthin, Wald 2013) uses explicit
// round-to-nearest intrinsics so it rounds exactly like the CPU restatement
// even though this file is compiled with FMA contraction for the box tests.
#include "wavefront.h"

namespace shb {

namespace {

constexpr int kStack = 64;
constexpr int kTravThreads = 128;
// Resident blocks per SM the closest-hit and any-hit kernels are
// register-limited to (0: the compiler's choice).  The any-hit kernel runs
// 5 % faster at 10 blocks (48 registers, a few spilled) than at the
// compiler's 8; the closest-hit kernel 6 % slower.
#ifndef SHB_TRAV_MIN_BLOCKS
#define SHB_TRAV_MIN_BLOCKS 0
#endif
#ifndef SHB_SHADOW_MIN_BLOCKS
#define SHB_SHADOW_MIN_BLOCKS 10
#endif
#if SHB_TRAV_MIN_BLOCKS > 0
#define SHB_TRAV_BOUNDS __launch_bounds__(kTravThreads, SHB_TRAV_MIN_BLOCKS)
#else
#define SHB_TRAV_BOUNDS __launch_bounds__(kTravThreads)
#endif
#if SHB_SHADOW_MIN_BLOCKS > 0
#define SHB_SHADOW_BOUNDS __launch_bounds__(kTravThreads, SHB_SHADOW_MIN_BLOCKS)
#else
#define SHB_SHADOW_BOUNDS __launch_bounds__(kTravThreads)
#endif
// A warp refills its idle lanes from the queue once at least this many
// lanes wait for a ray (or none of its lanes has one left): the refill
// (queue atomic, ray load and setup) then runs once for several lanes.
#ifndef SHB_REFILL_MIN
#define SHB_REFILL_MIN 8
#endif
constexpr int kRefillMin = SHB_REFILL_MIN;
// 1: the warp-cooperative triangle phase; 0: each lane tests its own
// triangles in a loop.
#ifndef SHB_TRI_COOP
#define SHB_TRI_COOP 1
#endif
constexpr bool kTriCoop = SHB_TRI_COOP != 0;
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
// |d|).  On acceptance gives T, det, V, W with det > 0: t = T / det, and
// V / det, W / det are the weights of v1, v2 (the divisions are left to the
// caller: only the last accepted triangle of a ray needs its weights).
// `k` holds the ray's axes kx | ky << 2 | kz << 4.
__device__ __forceinline__ bool tri_core(float ox, float oy, float oz, uint32_t k, float Sx, float Sy, float Sz,
                                         float4 a, float4 b, float4 c, float tnear, float tfar, float& T_,
                                         float& det_, float& V_, float& W_) {
  const int kx = (int)(k & 3u), ky = (int)((k >> 2) & 3u), kz = (int)(k >> 4);
  float Ax_ = __fsub_rn(a.x, ox), Ay_ = __fsub_rn(a.y, oy), Az_ = __fsub_rn(a.z, oz);
  float Bx_ = __fsub_rn(b.x, ox), By_ = __fsub_rn(b.y, oy), Bz_ = __fsub_rn(b.z, oz);
  float Cx_ = __fsub_rn(c.x, ox), Cy_ = __fsub_rn(c.y, oy), Cz_ = __fsub_rn(c.z, oz);
  float Akz = comp(Ax_, Ay_, Az_, kz), Bkz = comp(Bx_, By_, Bz_, kz), Ckz = comp(Cx_, Cy_, Cz_, kz);
  float Ax = __fsub_rn(comp(Ax_, Ay_, Az_, kx), __fmul_rn(Sx, Akz));
  float Ay = __fsub_rn(comp(Ax_, Ay_, Az_, ky), __fmul_rn(Sy, Akz));
  float Bx = __fsub_rn(comp(Bx_, By_, Bz_, kx), __fmul_rn(Sx, Bkz));
  float By = __fsub_rn(comp(Bx_, By_, Bz_, ky), __fmul_rn(Sy, Bkz));
  float Cx = __fsub_rn(comp(Cx_, Cy_, Cz_, kx), __fmul_rn(Sx, Ckz));
  float Cy = __fsub_rn(comp(Cx_, Cy_, Cz_, ky), __fmul_rn(Sy, Ckz));
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
  float Az = __fmul_rn(Sz, Akz), Bz = __fmul_rn(Sz, Bkz), Cz = __fmul_rn(Sz, Ckz);
  float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
  if (det < 0.f) {
    T = -T;
    det = -det;
    V = -V;
    W = -W;
  }
  if (!(T > __fmul_rn(tnear, det) && T < __fmul_rn(tfar, det))) return false;
  T_ = T;
  det_ = det;
  V_ = V;
  W_ = W;
  return true;
}

__device__ __forceinline__ uint32_t axes(const TravRay& r) {
  return (uint32_t)r.kx | ((uint32_t)r.ky << 2) | ((uint32_t)r.kz << 4);
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
  float hV, hW, hdet;  // barycentric numerators and determinant of the hit
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
  w.hV = w.hW = 0.f;
  w.hdet = 1.f;
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

// The node part of one step: visit one node (or take a popped triangle
// group) and leave the triangles to test in w.T.  Returns true when the ray
// ran out of steps (w.T is then empty).
__device__ __forceinline__ bool walk_node(const BvhView& bvh, Walk& w, uint2* stack, int* err, uint32_t max_iters) {
  if (++w.iters > max_iters) {
    atomicOr(err, ERR_ITER);
    w.T.y = 0;
    return true;
  }
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
    intersect_node(bvh, w, node, w.G, w.T);
  } else if (!(w.G.y & kNodeGroup)) {
    w.T = w.G;  // a popped triangle group
    w.G = make_uint2(0u, 0u);
  } else {
    w.G = make_uint2(0u, 0u);
  }
  return false;
}

// The end of a step: take the next group from the stack when the current
// one is used up.  Returns true when the ray is finished.
__device__ __forceinline__ bool walk_pop(Walk& w, const uint2* stack) {
  bool g_empty = !((w.G.y & kNodeGroup) ? (w.G.y & 0xFFu) : w.G.y);
  if (g_empty) {
    if (w.sp == 0) return true;
    w.G = stack[--w.sp];
  }
  return false;
}

// Accepts a test that passed against the tmax of its step if it still
// passes against the ray's current tmax (the sequential loop's test with
// the tmax of the triangles before it).
__device__ __forceinline__ void accept(Walk& w, float T, float det, float V, float W, float prim_bits) {
  if (T < __fmul_rn(w.tmax, det)) {
    w.hit = true;
    w.tmax = __fdiv_rn(T, det);
    w.hV = V;
    w.hW = W;
    w.hdet = det;
    w.prim = __float_as_uint(prim_bits);
  }
}

// The triangle part of one step, one lane: its own triangles in bit order.
template <bool ANY>
__device__ __forceinline__ void tri_seq(Walk& w, const float4* tris) {
  const uint32_t k = axes(w.r);
  while (w.T.y) {
    int b = __ffs(w.T.y) - 1;
    w.T.y &= w.T.y - 1;
    const float4* tp = tris + 3 * (size_t)(w.T.x + b);
    float4 a = __ldg(tp), bb = __ldg(tp + 1), c = __ldg(tp + 2);
    float T, det, V, W;
    if (tri_core(w.r.ox, w.r.oy, w.r.oz, k, w.r.Sx, w.r.Sy, w.r.Sz, a, bb, c, w.tnear, w.tmax, T, det, V, W)) {
      accept(w, T, det, V, W, a.w);
      if (ANY) {
        w.T.y = 0;
        return;
      }
    }
  }
}

// Position of the n-th (from 0) set bit of x; x has more than n set bits.
__device__ __forceinline__ uint32_t nth_bit(uint32_t x, uint32_t n) {
  uint32_t pos = 0, c;
  c = __popc(x & 0xFFFFu);
  if (n >= c) { n -= c; x >>= 16; pos += 16; }
  c = __popc(x & 0xFFu);
  if (n >= c) { n -= c; x >>= 8; pos += 8; }
  c = __popc(x & 0xFu);
  if (n >= c) { n -= c; x >>= 4; pos += 4; }
  c = __popc(x & 0x3u);
  if (n >= c) { n -= c; x >>= 2; pos += 2; }
  if (n >= (x & 1u)) pos += 1;
  return pos;
}

// Per-warp shared tables of the cooperative triangle phase: each lane's ray
// (written when the lane takes the ray), the lane owning each slot window
// start, and the accepted tests of a window.
struct CoopWarp {
  float4 r0[32];   // ox, oy, oz, tnear
  float4 r1[32];   // Sx, Sy, Sz, axes
  float4 hit[32];  // T, det, V, W
  float hprim[32];
  int own[32];
};

__device__ __forceinline__ void coop_store_ray(CoopWarp& s, int lane, const Walk& w) {
  s.r0[lane] = make_float4(w.r.ox, w.r.oy, w.r.oz, w.tnear);
  s.r1[lane] = make_float4(w.r.Sx, w.r.Sy, w.r.Sz, __uint_as_float(axes(w.r)));
}

// The triangle part of one step for the whole warp (every lane calls it;
// lanes without a ray have an empty w.T).  The warp's pending tests,
// ordered by lane and then by triangle bit, are dealt out 32 at a time, one
// per lane; each owner lane then replays its accepted tests in bit order
// (accept), so the result is the sequential loop's.  For ANY, an accepted
// test ends the ray (w.hit).
template <bool ANY>
__device__ __forceinline__ void tri_coop(CoopWarp& s, Walk& w, const float4* tris, int lane) {
  const uint32_t full = 0xFFFFFFFFu;
  const uint32_t cnt = __popc(w.T.y);
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t x = __shfl_up_sync(full, incl, o);
    if (lane >= o) incl += x;
  }
  const uint32_t total = __shfl_sync(full, incl, 31);
  if (total == 0) return;
  const uint32_t excl = incl - cnt;
  const unsigned long long tb = (unsigned long long)(tris + 3 * (size_t)w.T.x);
  for (uint32_t base = 0; base < total; base += 32) {
    // the lane whose tests cover the window's first slot, and the lanes
    // whose tests start inside the window
    const bool c0 = cnt && excl <= base && base < excl + cnt;
    const bool st = cnt && excl > base && excl < base + 32;
    if (c0) s.own[0] = lane;
    if (st) s.own[excl - base] = lane;
    const uint32_t starts = __reduce_or_sync(full, c0 ? 1u : (st ? 1u << (excl - base) : 0u));
    __syncwarp();
    const uint32_t g = base + (uint32_t)lane;
    const bool act = g < total;
    const int owner = act ? s.own[31 - __clz(starts & (full >> (31 - lane)))] : lane;
    const uint32_t oty = __shfl_sync(full, w.T.y, owner);
    const uint32_t oex = __shfl_sync(full, excl, owner);
    const float otmax = __shfl_sync(full, w.tmax, owner);
    const unsigned long long otb = __shfl_sync(full, tb, owner);
    bool hit = false;
    if (act) {
      const float4* tp = reinterpret_cast<const float4*>(otb) + 3 * nth_bit(oty, g - oex);
      const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
      const float4 r0 = s.r0[owner], r1 = s.r1[owner];
      float T, det, V, W;
      hit = tri_core(r0.x, r0.y, r0.z, __float_as_uint(r1.w), r1.x, r1.y, r1.z, a, b, c, r0.w, otmax, T, det, V, W);
      if (hit && !ANY) {
        s.hit[lane] = make_float4(T, det, V, W);
        s.hprim[lane] = a.w;
      }
    }
    const uint32_t hm = __ballot_sync(full, hit);
    if (hm) {
      __syncwarp();
      const int lo = (int)excl - (int)base, hi = (int)(excl + cnt) - (int)base;
      if (cnt && hi > 0 && lo < 32) {
        const int l0 = lo < 0 ? 0 : lo, l1 = hi > 32 ? 32 : hi;
        uint32_t m = hm & bit_mask((uint32_t)l0, (uint32_t)(l1 - l0));
        if (ANY) {
          if (m) w.hit = true;
        } else {
          while (m) {
            const int sl = __ffs(m) - 1;
            m &= m - 1;
            const float4 h = s.hit[sl];
            accept(w, h.x, h.y, h.z, h.w, s.hprim[sl]);
          }
        }
      }
    }
    __syncwarp();  // the tables are rewritten by the next window
  }
  w.T.y = 0;
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

__device__ __forceinline__ float4 hit_record(const Walk& w) {
  return w.hit ? make_float4(w.tmax, __fdiv_rn(w.hV, w.hdet), __fdiv_rn(w.hW, w.hdet), __uint_as_float(w.prim))
               : make_float4(0.f, 0.f, 0.f, __uint_as_float(kMissPrim));
}

// Persistent queue consumer: lanes refill from the queue as their rays end.
// `bvh_of(i, o, d)` gives the BVH of queue entry i (its bake's).
template <bool SHADOW, class Q, class B, class Fin>
__device__ __forceinline__ void consume(CoopWarp& s, const Q& q, int n, int* fetch, int* err, uint32_t max_iters,
                                        B&& bvh_of, Fin&& finish) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  uint2 stack[kStack];
  Walk w;
  w.T = make_uint2(0u, 0u);
  BvhView bvh;
  bvh.tris = nullptr;
  int ray = -1;
  bool exhausted = false;
  while (true) {
    bool need = ray < 0 && !exhausted;
    unsigned needm = __ballot_sync(0xFFFFFFFFu, need);
    if (kRefillMin > 1 && __popc(needm) < kRefillMin && __any_sync(0xFFFFFFFFu, ray >= 0)) needm = 0;
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
          if (kTriCoop) coop_store_ray(s, lane, w);
        } else {
          exhausted = true;
        }
      }
    }
    if (!__any_sync(0xFFFFFFFFu, ray >= 0)) break;
    bool done = false;
    if (ray >= 0) done = walk_node(bvh, w, stack, err, max_iters);
    if (kTriCoop) tri_coop<SHADOW>(s, w, bvh.tris, lane);
    else if (ray >= 0) tri_seq<SHADOW>(w, bvh.tris);
    if (ray >= 0) {
      if (!done) done = (SHADOW && w.hit) || walk_pop(w, stack);
      if (done) {
        finish(ray, w);
        ray = -1;
        w.T = make_uint2(0u, 0u);
      }
    }
  }
}

__global__ void SHB_TRAV_BOUNDS k_extend(const BakeItem* __restrict__ bakes, int n_bakes,
                                         const PathInfo* __restrict__ info, ExtQueue q,
                                         const int* __restrict__ n_ptr, int cap, float4* __restrict__ hits,
                                         int* fetch, int* err, Counters64* stats, uint32_t max_iters) {
  __shared__ CoopWarp coop[kTriCoop ? kTravThreads / 32 : 1];
  const int n = min(*n_ptr, cap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(&stats->extend_rays, (unsigned long long)n);
  const BvhView bvh0 = bakes[0].bvh;
  auto bvh_of = [&](int, float4 o, float4) {
    return n_bakes == 1 ? bvh0 : bakes[info[__float_as_uint(o.w)].x].bvh;
  };
  consume<false>(coop[kTriCoop ? threadIdx.x / 32 : 0], q, n, fetch, err, max_iters, bvh_of,
                 [&](int i, const Walk& w) { hits[i] = hit_record(w); });
}

__global__ void SHB_SHADOW_BOUNDS k_shadow(const BakeItem* __restrict__ bakes, int n_bakes, ShadowQueue q,
                                         const int* __restrict__ n_ptr, int cap, float4* __restrict__ path_L,
                                         float4* __restrict__ nee_li, float4* __restrict__ pend, int* fetch,
                                         int* err, Counters64* stats, uint32_t max_iters) {
  __shared__ CoopWarp coop[kTriCoop ? kTravThreads / 32 : 1];
  const int n = min(*n_ptr, cap);
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(&stats->shadow_rays, (unsigned long long)n);
  const BvhView bvh0 = bakes[0].bvh;
  auto bvh_of = [&](int i, float4, float4) {
    return n_bakes == 1 ? bvh0 : bakes[__float_as_uint(q.c[i].w) >> 2].bvh;
  };
  consume<true>(coop[kTriCoop ? threadIdx.x / 32 : 0], q, n, fetch, err, max_iters, bvh_of,
                [&](int i, const Walk& w) {
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

// One thread per ray, the per-lane triangle loop (FindOcclusion queries).
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
    while (true) {
      if (walk_node(bvh, w, stack, err, kMaxIters)) break;
      tri_seq<false>(w, bvh.tris);
      if (walk_pop(w, stack)) break;
    }
    hits[i] = hit_record(w);
  }
}

}  // namespace

int traversal_grid(int device, bool shadow) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (shadow) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_shadow, kTravThreads, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_extend, kTravThreads, 0);
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
