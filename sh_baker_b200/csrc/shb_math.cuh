// shb_math.cuh - device arithmetic that must round exactly like the CPU
// restatement of the reference.  Translation units that include this file
// are compiled with -fmad=false, so every expression below rounds once per
// operation, in the order written.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace shb {

struct f3 {
  float x, y, z;
};
struct f2 {
  float x, y;
};

__device__ __forceinline__ f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ f3 cmul(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
// Eigen's unrolled 3-term reduction: x0*y0 + (x1*y1 + x2*y2).
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
__device__ __forceinline__ float sqnorm(f3 a) { return dot(a, a); }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// Eigen normalized(): v / sqrt(|v|^2) when |v|^2 > 0, else v unchanged.
__device__ __forceinline__ f3 normalized(f3 a) {
  float n = sqnorm(a);
  if (n > 0.0f) {
    float r = sqrtf(n);
    return {a.x / r, a.y / r, a.z / r};
  }
  return a;
}
__device__ __forceinline__ float max_coeff(f3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__device__ __forceinline__ bool is_zero_eigen(f3 a) {
  return fabsf(a.x) <= 1e-5f && fabsf(a.y) <= 1e-5f && fabsf(a.z) <= 1e-5f;
}

__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ f2 operator*(float s, f2 a) { return {s * a.x, s * a.y}; }
__device__ __forceinline__ float dot2(f2 a, f2 b) { return a.x * b.x + a.y * b.y; }

__device__ __forceinline__ f3 ld3(const float* p, uint32_t i) {
  return {__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2)};
}
__device__ __forceinline__ f2 ld2(const float* p, uint32_t i) {
  return {__ldg(p + 2 * i), __ldg(p + 2 * i + 1)};
}

// (int)f with x86 cvttss2si semantics: out-of-range and NaN give INT_MIN.
__device__ __forceinline__ int cvt_trunc(float f) {
  if (f >= -2147483648.0f && f < 2147483648.0f) return __float2int_rz(f);
  return (int)0x80000000;
}

// ------------------------------------------------------------ Philox ------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
struct u4 {
  uint32_t x, y, z, w;
};
__device__ __forceinline__ u4 philox10(u4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = u4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
  }
  return c;
}

// Event types of the counter stream.
enum : uint32_t { EV_HEMI = 0, EV_NEE = 1, EV_BSDF = 2 };

// The uniforms of one event: key = (seed, texel), counter = (sample, path
// vertex, event type, block of four).
struct Event {
  uint32_t k0, k1, c0, c1, c2;
  int block;
  u4 cache;
  __device__ __forceinline__ void init(uint32_t seed, uint32_t texel, uint32_t sample, uint32_t vertex,
                                       uint32_t type) {
    k0 = seed; k1 = texel; c0 = sample; c1 = vertex; c2 = type; block = -1;
  }
  __device__ __forceinline__ uint32_t bits(int i) {
    int b = i >> 2;
    if (b != block) {
      cache = philox10(u4{c0, c1, c2, (uint32_t)b}, k0, k1);
      block = b;
    }
    int l = i & 3;
    return l == 0 ? cache.x : (l == 1 ? cache.y : (l == 2 ? cache.z : cache.w));
  }
  __device__ __forceinline__ float u(int i) { return (float)(bits(i) >> 8) * (1.0f / 16777216.0f); }
  __device__ __forceinline__ uint32_t tri(int i, uint32_t n) { return __umulhi(bits(i), n); }
};

}  // namespace shb
