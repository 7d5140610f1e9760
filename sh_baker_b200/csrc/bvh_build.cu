// bvh_build.cu - GPU BVH builder: binned-SAH binary BVH built top-down one
// level at a time, then collapsed into compressed 8-wide nodes.
//
// Replaces BuildBVH (src/scene.cpp:209-262), which hands the transformed
// triangles to Embree with RTC_BUILD_QUALITY_HIGH.  Every step is
// deterministic: bounds are reduced with integer min/max on order-preserving
// float bits, bin counts with integer adds, partitions are stable scans, and
// ties are broken by index, so the same scene always gives the same tree.
#include <cub/cub.cuh>

#include <chrono>

#include "shb_internal.h"

namespace shb {

namespace {

// Binned SAH: bins per axis, largest leaf, and the cost of a node visit
// relative to a triangle test in the leaf decision.
#ifndef SHB_BVH_BINS
#define SHB_BVH_BINS 32
#endif
#ifndef SHB_BVH_MAX_LEAF
#define SHB_BVH_MAX_LEAF 3
#endif
#ifndef SHB_BVH_NODE_COST
#define SHB_BVH_NODE_COST 1.0f
#endif
constexpr int kBins = SHB_BVH_BINS;
constexpr int kMaxLeaf = SHB_BVH_MAX_LEAF;  // triangles per leaf child of a wide node
// A wide node's triangle group is a 24-bit mask (bit 31 marks node groups in
// the traversal), so its 8 leaf children hold at most 24 triangles.
static_assert(kMaxLeaf >= 1 && kMaxLeaf * 8 <= 24, "leaf triangles must fit the 24-bit triangle group");
constexpr int kMaxDepth = 40;  // deeper nodes use median splits
constexpr int kThreads = 256;

inline int grid_for(int64_t n) {
  int64_t g = (n + kThreads - 1) / kThreads;
  if (g > sm_count() * 32) g = sm_count() * 32;
  return (int)(g < 1 ? 1 : g);
}

struct BNode {
  float lo[3], hi[3];
  int left, right;  // left < 0: leaf
  int begin, count;
};

__device__ __forceinline__ int f2o(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

constexpr int kPosInf = 0x7F800000;             // f2o(+inf)
constexpr int kNegInf = (int)(0xFF800000u ^ 0x7FFFFFFFu);  // f2o(-inf)

// Slot accumulators: [0..2] node lo, [3..5] node hi, [6..8] centroid lo,
// [9..11] centroid hi (order-preserving ints).
constexpr int kSlotBounds = 12;
// Bins per slot: per axis per bin: count + 6 bound ints.
constexpr int kBinInts = 7;
constexpr int kSlotBinInts = 3 * kBins * kBinInts;

__global__ void k_prim_bounds(uint32_t T, const uint32_t* __restrict__ vidx, const float* __restrict__ wv,
                              float4* __restrict__ plo, float4* __restrict__ phi) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < T; p += gridDim.x * blockDim.x) {
    float3 v[3];
    for (int k = 0; k < 3; ++k) {
      uint32_t i = vidx[3 * p + k];
      v[k] = make_float3(wv[3 * i], wv[3 * i + 1], wv[3 * i + 2]);
    }
    float3 lo = make_float3(fminf(v[0].x, fminf(v[1].x, v[2].x)), fminf(v[0].y, fminf(v[1].y, v[2].y)),
                            fminf(v[0].z, fminf(v[1].z, v[2].z)));
    float3 hi = make_float3(fmaxf(v[0].x, fmaxf(v[1].x, v[2].x)), fmaxf(v[0].y, fmaxf(v[1].y, v[2].y)),
                            fmaxf(v[0].z, fmaxf(v[1].z, v[2].z)));
    plo[p] = make_float4(lo.x, lo.y, lo.z, 0.f);
    phi[p] = make_float4(hi.x, hi.y, hi.z, 0.f);
  }
}

// Slot bounds start as [+inf x3 | -inf x3 | +inf x3 | -inf x3]; bins as
// [count 0 | lo +inf x3 | hi -inf x3].
__global__ void k_init_slots(int n_act, int* __restrict__ sb, int* __restrict__ bins) {
  int64_t nb = (int64_t)n_act * kSlotBounds;
  int64_t nbin = (int64_t)n_act * kSlotBinInts;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nb + nbin;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i < nb) {
      int k = (int)(i % kSlotBounds);
      sb[i] = ((k / 3) & 1) ? kNegInf : kPosInf;
    } else {
      int k = (int)((i - nb) % kBinInts);
      bins[i - nb] = k == 0 ? 0 : (k <= 3 ? kPosInf : kNegInf);
    }
  }
}

__device__ __forceinline__ float centroid(const float4& lo, const float4& hi, int a) {
  float l = a == 0 ? lo.x : (a == 1 ? lo.y : lo.z);
  float h = a == 0 ? hi.x : (a == 1 ? hi.y : hi.z);
  return (l + h) * 0.5f;
}

// Warp-aggregated atomic min/max: lanes with the same key reduce first.
__device__ __forceinline__ void agg_min(unsigned peers, int* addr, int v) {
  int r = __reduce_min_sync(peers, v);
  if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicMin(addr, r);
}
__device__ __forceinline__ void agg_max(unsigned peers, int* addr, int v) {
  int r = __reduce_max_sync(peers, v);
  if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicMax(addr, r);
}

// Node and centroid bounds of every active slot.
__global__ void k_slot_bounds(uint32_t T, const uint32_t* __restrict__ idx, const int* __restrict__ pslot,
                              const float4* __restrict__ plo, const float4* __restrict__ phi,
                              int* __restrict__ sb) {
  uint32_t stride = gridDim.x * blockDim.x;
  uint32_t n_iter = (T + stride - 1) / stride;
  for (uint32_t it = 0; it < n_iter; ++it) {
    uint32_t i = it * stride + blockIdx.x * blockDim.x + threadIdx.x;
    int s = -1;
    float4 lo = make_float4(0, 0, 0, 0), hi = lo;
    if (i < T) {
      s = pslot[i];
      if (s >= 0) {
        uint32_t p = idx[i];
        lo = plo[p];
        hi = phi[p];
      }
    }
    unsigned peers = __match_any_sync(0xFFFFFFFFu, s);
    if (s >= 0) {
      int* b = sb + (int64_t)s * kSlotBounds;
      agg_min(peers, b + 0, f2o(lo.x));
      agg_min(peers, b + 1, f2o(lo.y));
      agg_min(peers, b + 2, f2o(lo.z));
      agg_max(peers, b + 3, f2o(hi.x));
      agg_max(peers, b + 4, f2o(hi.y));
      agg_max(peers, b + 5, f2o(hi.z));
      for (int a = 0; a < 3; ++a) {
        float c = centroid(lo, hi, a);
        agg_min(peers, b + 6 + a, f2o(c));
        agg_max(peers, b + 9 + a, f2o(c));
      }
    }
  }
}

__device__ __forceinline__ int bin_of(float c, float cmin, float scale) {
  int b = (int)((c - cmin) * scale);
  return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
}

__device__ __forceinline__ void slot_axis(const int* sb, int a, float& cmin, float& ext, float& scale) {
  cmin = o2f(sb[6 + a]);
  float cmax = o2f(sb[9 + a]);
  ext = cmax - cmin;
  scale = ext > 0.f ? (float)kBins / ext : 0.f;
}

__global__ void k_bins(uint32_t T, const uint32_t* __restrict__ idx, const int* __restrict__ pslot,
                       const float4* __restrict__ plo, const float4* __restrict__ phi,
                       const int* __restrict__ sb, int* __restrict__ bins) {
  uint32_t stride = gridDim.x * blockDim.x;
  uint32_t n_iter = (T + stride - 1) / stride;
  for (uint32_t it = 0; it < n_iter; ++it) {
    uint32_t i = it * stride + blockIdx.x * blockDim.x + threadIdx.x;
    int s = -1;
    float4 lo = make_float4(0, 0, 0, 0), hi = lo;
    if (i < T) {
      s = pslot[i];
      if (s >= 0) {
        uint32_t p = idx[i];
        lo = plo[p];
        hi = phi[p];
      }
    }
    for (int a = 0; a < 3; ++a) {
      int key = -1;
      if (s >= 0) {
        float cmin, ext, scale;
        slot_axis(sb + (int64_t)s * kSlotBounds, a, cmin, ext, scale);
        if (ext > 0.f) key = (s * 3 + a) * kBins + bin_of(centroid(lo, hi, a), cmin, scale);
      }
      unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
      if (key >= 0) {
        int* b = bins + (int64_t)key * kBinInts;
        if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(b, __popc(peers));
        agg_min(peers, b + 1, f2o(lo.x));
        agg_min(peers, b + 2, f2o(lo.y));
        agg_min(peers, b + 3, f2o(lo.z));
        agg_max(peers, b + 4, f2o(hi.x));
        agg_max(peers, b + 5, f2o(hi.y));
        agg_max(peers, b + 6, f2o(hi.z));
      }
    }
  }
}

__device__ __forceinline__ float half_area(const float* l, const float* h) {
  float dx = h[0] - l[0], dy = h[1] - l[1], dz = h[2] - l[2];
  if (!(dx >= 0.f)) return 0.f;
  return dx * dy + dy * dz + dz * dx;
}

// Per active slot: write the node bounds and choose leaf / SAH split / median.
// split[s] = (axis or -1 median or -2 leaf, split bin, nL, is_split)
__global__ void k_split(int n_act, int depth, const int* __restrict__ act, BNode* __restrict__ nodes,
                        const int* __restrict__ sb, const int* __restrict__ bins, int4* __restrict__ split,
                        int* __restrict__ is_split) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_act; s += gridDim.x * blockDim.x) {
    BNode& nd = nodes[act[s]];
    const int* b = sb + (int64_t)s * kSlotBounds;
    for (int a = 0; a < 3; ++a) {
      nd.lo[a] = o2f(b[a]);
      nd.hi[a] = o2f(b[3 + a]);
    }
    int count = nd.count;
    int4 out = make_int4(-2, 0, 0, 0);
    if (count > 1) {
      float best = INFINITY;
      int best_axis = -1, best_bin = 0, best_nl = 0;
      if (depth < kMaxDepth) {
        for (int a = 0; a < 3; ++a) {
          float cmin, ext, scale;
          slot_axis(b, a, cmin, ext, scale);
          if (!(ext > 0.f)) continue;
          const int* bb = bins + (int64_t)((s * 3 + a) * kBins) * kBinInts;
          float lA[kBins];
          int lC[kBins];
          float cl[3] = {INFINITY, INFINITY, INFINITY}, ch[3] = {-INFINITY, -INFINITY, -INFINITY};
          int cc = 0;
          for (int k = 0; k < kBins; ++k) {
            const int* e = bb + k * kBinInts;
            if (e[0] > 0) {
              for (int c = 0; c < 3; ++c) {
                cl[c] = fminf(cl[c], o2f(e[1 + c]));
                ch[c] = fmaxf(ch[c], o2f(e[4 + c]));
              }
            }
            cc += e[0];
            lA[k] = half_area(cl, ch);
            lC[k] = cc;
          }
          float rl[3] = {INFINITY, INFINITY, INFINITY}, rh[3] = {-INFINITY, -INFINITY, -INFINITY};
          int rc = 0;
          for (int k = kBins - 1; k >= 1; --k) {
            const int* e = bb + k * kBinInts;
            if (e[0] > 0) {
              for (int c = 0; c < 3; ++c) {
                rl[c] = fminf(rl[c], o2f(e[1 + c]));
                rh[c] = fmaxf(rh[c], o2f(e[4 + c]));
              }
            }
            rc += e[0];
            int nl = lC[k - 1];
            if (nl == 0 || rc == 0) continue;
            float cost = lA[k - 1] * (float)nl + half_area(rl, rh) * (float)rc;
            if (cost < best) {
              best = cost;
              best_axis = a;
              best_bin = k;
              best_nl = nl;
            }
          }
        }
      }
      bool leaf = false;
      if (count <= kMaxLeaf) {
        float A = half_area(nd.lo, nd.hi);
        float split_cost = best_axis >= 0 && A > 0.f ? SHB_BVH_NODE_COST + best / A : INFINITY;
        leaf = (float)count <= split_cost;
      }
      if (!leaf) {
        if (best_axis >= 0) out = make_int4(best_axis, best_bin, best_nl, 1);
        else out = make_int4(-1, 0, count / 2, 1);
      }
    }
    split[s] = out;
    is_split[s] = out.w;
  }
}

__global__ void k_flags(uint32_t T, const uint32_t* __restrict__ idx, const int* __restrict__ pslot,
                        const float4* __restrict__ plo, const float4* __restrict__ phi,
                        const int* __restrict__ sb, const int4* __restrict__ split, const int* __restrict__ act,
                        const BNode* __restrict__ nodes, int* __restrict__ flag) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
    int s = pslot[i];
    int f = 0;
    if (s >= 0) {
      int4 sp = split[s];
      if (sp.w) {
        if (sp.x >= 0) {
          uint32_t p = idx[i];
          float cmin, ext, scale;
          slot_axis(sb + (int64_t)s * kSlotBounds, sp.x, cmin, ext, scale);
          f = bin_of(centroid(plo[p], phi[p], sp.x), cmin, scale) < sp.y;
        } else {
          f = (int)i - nodes[act[s]].begin < sp.z;
        }
      }
    }
    flag[i] = f;
  }
}

__global__ void k_scatter(uint32_t T, const uint32_t* __restrict__ idx, const int* __restrict__ pslot,
                          const int4* __restrict__ split, const int* __restrict__ rank, const int* __restrict__ act,
                          const BNode* __restrict__ nodes, const int* __restrict__ flag, const int* __restrict__ scanL,
                          uint32_t* __restrict__ idx_out, int* __restrict__ pslot_out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
    int s = pslot[i];
    if (s < 0 || !split[s].w) {
      idx_out[i] = idx[i];
      pslot_out[i] = -1;
      continue;
    }
    int4 sp = split[s];
    int begin = nodes[act[s]].begin;
    int rl = scanL[i] - scanL[begin];
    bool left = flag[i] != 0;
    int pos = left ? begin + rl : begin + sp.z + ((int)i - begin - rl);
    idx_out[pos] = idx[i];
    pslot_out[pos] = 2 * rank[s] + (left ? 0 : 1);
  }
}

__global__ void k_children(int n_act, const int* __restrict__ act, BNode* __restrict__ nodes,
                           const int4* __restrict__ split, const int* __restrict__ rank, int node_base,
                           int* __restrict__ next_act) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_act; s += gridDim.x * blockDim.x) {
    int4 sp = split[s];
    BNode& nd = nodes[act[s]];
    if (!sp.w) {
      nd.left = -1;
      nd.right = -1;
      continue;
    }
    int l = node_base + 2 * rank[s];
    nd.left = l;
    nd.right = l + 1;
    BNode c;
    for (int a = 0; a < 3; ++a) {
      c.lo[a] = 0.f;
      c.hi[a] = 0.f;
    }
    c.left = c.right = -1;
    c.begin = nd.begin;
    c.count = sp.z;
    nodes[l] = c;
    c.begin = nd.begin + sp.z;
    c.count = nd.count - sp.z;
    nodes[l + 1] = c;
    next_act[2 * rank[s]] = l;
    next_act[2 * rank[s] + 1] = l + 1;
  }
}

// ------------------------------------------------------------ collapse ----

struct Collapse {
  int child[8];
  int slot[8];  // slot of child k
  int n;
  int n_int;
  int n_tri;
  int leaf_mask;  // bit k: child k is a leaf slot (a binary leaf, or a small subtree merged into one)
};

// SAH-optimal collapse (Ylitie, Karras and Laine 2017, section 4.1): for
// every binary node n and i = 1..7, C(n, i) is the least SAH cost of the
// subtree at n spread over at most i child slots of its wide parent:
//   C(n, 1) = min(leaf(n), A(n) c_node + D(n, 8)),
//   C(n, i) = min(C(n, i - 1), D(n, i)),
//   D(n, j) = min over 0 < k < j of C(left, k) + C(right, j - k),
// leaf(n) = A(n) |n| for |n| <= kMaxLeaf triangles.  dec[n][i] records the
// choice (kDecLeaf, kDecNode, kDecFewer or the split k), dec[n][8] the split
// of D(n, 8); the collapse then reads the wide nodes off the decisions.
#ifndef SHB_BVH_SAH_COLLAPSE
#define SHB_BVH_SAH_COLLAPSE 1
#endif
constexpr int8_t kDecLeaf = -1, kDecNode = -2, kDecFewer = -3;
struct DpCost {
  float c[8];  // c[i] = C(n, i), i = 1..7
};
struct DpDec {
  int8_t d[9];  // d[i], i = 1..8
};

__device__ __forceinline__ float node_area(const BNode& n) { return half_area(n.lo, n.hi); }

// One level of binary nodes [begin, end), after all deeper levels.
__global__ void k_dp(int begin, int end, const BNode* __restrict__ nodes, DpCost* __restrict__ cost,
                     DpDec* __restrict__ dec) {
  for (int n = begin + blockIdx.x * blockDim.x + threadIdx.x; n < end; n += gridDim.x * blockDim.x) {
    const BNode& nd = nodes[n];
    const float A = half_area(nd.lo, nd.hi);
    DpCost C;
    DpDec D;
    C.c[0] = 0.f;
    D.d[0] = 0;
    if (nd.left < 0) {
      const float leaf = A * (float)nd.count;
      for (int i = 1; i < 8; ++i) {
        C.c[i] = leaf;
        D.d[i] = kDecLeaf;
      }
      D.d[8] = 0;
    } else {
      const DpCost L = cost[nd.left], R = cost[nd.right];
      float dist[9];
      int8_t arg[9];
      for (int j = 2; j <= 8; ++j) {
        float best = INFINITY;
        int8_t bk = 1;
        for (int k = 1; k < j; ++k) {
          const float v = L.c[k] + R.c[j - k];
          if (v < best) {
            best = v;
            bk = (int8_t)k;
          }
        }
        dist[j] = best;
        arg[j] = bk;
      }
      const float internal = A * SHB_BVH_NODE_COST + dist[8];
      const float leaf = nd.count <= kMaxLeaf ? A * (float)nd.count : INFINITY;
      C.c[1] = leaf <= internal ? leaf : internal;
      D.d[1] = leaf <= internal ? kDecLeaf : kDecNode;
      for (int i = 2; i < 8; ++i) {
        if (C.c[i - 1] <= dist[i]) {
          C.c[i] = C.c[i - 1];
          D.d[i] = kDecFewer;
        } else {
          C.c[i] = dist[i];
          D.d[i] = arg[i];
        }
      }
      D.d[8] = arg[8];
    }
    cost[n] = C;
    dec[n] = D;
  }
}

// Children of the wide node rooted at binary node r: the 8 slots of D(r, 8)
// spread down the recorded decisions.
__device__ void sah_children(int r, const BNode* __restrict__ nodes, const DpDec* __restrict__ dec, Collapse& c) {
  int st_n[16], st_i[16], sp = 0;
  const BNode& root = nodes[r];
  const int k8 = dec[r].d[8];
  st_n[sp] = root.left;
  st_i[sp++] = k8;
  st_n[sp] = root.right;
  st_i[sp++] = 8 - k8;
  c.n = 0;
  c.leaf_mask = 0;
  while (sp > 0) {
    const int n = st_n[--sp];
    int i = st_i[sp];
    const BNode& nd = nodes[n];
    const DpDec& D = dec[n];
    while (i > 1 && D.d[i] == kDecFewer) --i;
    // a split k outside 1..i-1 cannot occur; such an entry (or a full child
    // list or stack) would end the spreading at n rather than overrun
    const bool stop = i <= 1 || nd.left < 0 || D.d[i] < 1 || D.d[i] >= i || sp + 2 > 16 || c.n + sp + 2 > 8;
    if (stop) {
      if (nd.left < 0 || D.d[1] == kDecLeaf) c.leaf_mask |= 1 << c.n;
      c.child[c.n++] = n;
    } else {
      const int k = D.d[i];
      st_n[sp] = nd.left;
      st_i[sp++] = k;
      st_n[sp] = nd.right;
      st_i[sp++] = i - k;
    }
  }
}

__global__ void k_collapse(int n_level, const int* __restrict__ level, const BNode* __restrict__ nodes,
                           const DpDec* __restrict__ dec, Collapse* __restrict__ out, int* __restrict__ n_int,
                           int* __restrict__ n_tri) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n_level; w += gridDim.x * blockDim.x) {
    const BNode& root = nodes[level[w]];
    Collapse c;
    c.leaf_mask = 0;
    if (root.left < 0) {
      c.n = 1;
      c.child[0] = level[w];
      c.leaf_mask = 1;
    } else if (SHB_BVH_SAH_COLLAPSE) {
      sah_children(level[w], nodes, dec, c);
    } else {
      c.n = 2;
      c.child[0] = root.left;
      c.child[1] = root.right;
      while (c.n < 8) {
        int best = -1;
        float best_a = -1.f;
        for (int k = 0; k < c.n; ++k) {
          const BNode& ch = nodes[c.child[k]];
          if (ch.left < 0) continue;
          float a = node_area(ch);
          if (a > best_a) {
            best_a = a;
            best = k;
          }
        }
        if (best < 0) break;
        const BNode& ch = nodes[c.child[best]];
        c.child[best] = ch.left;
        c.child[c.n++] = ch.right;
      }
      for (int k = 0; k < c.n; ++k)
        if (nodes[c.child[k]].left < 0) c.leaf_mask |= 1 << k;
    }
    // octant slot assignment (greedy on centroid offsets)
    float pc[3];
    for (int a = 0; a < 3; ++a) pc[a] = 0.5f * (root.lo[a] + root.hi[a]);
    float cost[8][8];
    for (int k = 0; k < c.n; ++k) {
      const BNode& ch = nodes[c.child[k]];
      float d[3];
      for (int a = 0; a < 3; ++a) d[a] = 0.5f * (ch.lo[a] + ch.hi[a]) - pc[a];
      for (int s = 0; s < 8; ++s)
        cost[k][s] = ((s & 1) ? d[0] : -d[0]) + ((s & 2) ? d[1] : -d[1]) + ((s & 4) ? d[2] : -d[2]);
    }
    unsigned used_child = 0, used_slot = 0;
    for (int it = 0; it < c.n; ++it) {
      float bv = -INFINITY;
      int bk = -1, bs = -1;
      for (int k = 0; k < c.n; ++k) {
        if (used_child & (1u << k)) continue;
        for (int s = 0; s < 8; ++s) {
          if (used_slot & (1u << s)) continue;
          if (bk < 0 || cost[k][s] > bv) {
            bv = cost[k][s];
            bk = k;
            bs = s;
          }
        }
      }
      used_child |= 1u << bk;
      used_slot |= 1u << bs;
      c.slot[bk] = bs;
    }
    c.n_int = 0;
    c.n_tri = 0;
    for (int k = 0; k < c.n; ++k) {
      const BNode& ch = nodes[c.child[k]];
      if (!((c.leaf_mask >> k) & 1)) c.n_int++;
      else c.n_tri += ch.count;
    }
    out[w] = c;
    n_int[w] = c.n_int;
    n_tri[w] = c.n_tri;
  }
}

__device__ __forceinline__ uint32_t set_byte(uint32_t word, int k, uint32_t v) {
  return (word & ~(0xFFu << (8 * k))) | ((v & 0xFFu) << (8 * k));
}

__global__ void k_emit(int n_level, int wide_base, int child_wide_base, int tri_base_all,
                       const Collapse* __restrict__ col, const int* __restrict__ int_off, const int* __restrict__ tri_off,
                       const BNode* __restrict__ nodes, const uint32_t* __restrict__ idx,
                       const uint32_t* __restrict__ vidx, const float* __restrict__ wv, const int* __restrict__ level,
                       WideNode* __restrict__ wide, float4* __restrict__ tris, int* __restrict__ next_level) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < n_level; w += gridDim.x * blockDim.x) {
    const Collapse& c = col[w];
    const BNode& root = nodes[level[w]];
    int by_slot[8];
    unsigned leaf_slots = 0;
    for (int s = 0; s < 8; ++s) by_slot[s] = -1;
    for (int k = 0; k < c.n; ++k) {
      by_slot[c.slot[k]] = c.child[k];
      if ((c.leaf_mask >> k) & 1) leaf_slots |= 1u << c.slot[k];
    }
    WideNode nd;
    nd.px = root.lo[0];
    nd.py = root.lo[1];
    nd.pz = root.lo[2];
    float scale[3];
    uint32_t ebits = 0;
    for (int a = 0; a < 3; ++a) {
      float ext = __fsub_ru(root.hi[a], root.lo[a]);
      float sv = __fdiv_ru(ext, 255.0f);
      int e = 0;
      frexpf(sv, &e);
      if (!(sv > 0.f)) e = -126;
      e = e < -126 ? -126 : (e > 127 ? 127 : e);
      ebits |= (uint32_t)(e + 127) << (8 * a);
      scale[a] = __int_as_float((e + 127) << 23);
    }
    uint32_t imask = 0, meta_lo = 0, meta_hi = 0;
    uint32_t qlo[6] = {0, 0, 0, 0, 0, 0}, qhi[6] = {0, 0, 0, 0, 0, 0};
    int child_base = child_wide_base + int_off[w];
    int tri_base = tri_base_all + tri_off[w];
    int r_int = 0, t_off = 0;
    float p[3] = {nd.px, nd.py, nd.pz};
    for (int s = 0; s < 8; ++s) {
      int b = by_slot[s];
      if (b < 0) continue;
      const BNode& ch = nodes[b];
      uint32_t meta;
      if (!((leaf_slots >> s) & 1u)) {
        imask |= 1u << s;
        meta = (1u << 5) | (24u + (uint32_t)s);  // one bit at 24 + slot (see WideNode)
        next_level[int_off[w] + r_int] = b;
        r_int++;
      } else {
        meta = ((uint32_t)ch.count << 5) | (uint32_t)t_off;
        for (int k = 0; k < ch.count; ++k) {
          uint32_t prim = idx[ch.begin + k];
          int64_t o = 3 * (int64_t)(tri_base + t_off + k);
          for (int v = 0; v < 3; ++v) {
            uint32_t vi = vidx[3 * prim + v];
            tris[o + v] = make_float4(wv[3 * vi], wv[3 * vi + 1], wv[3 * vi + 2],
                                      v == 0 ? __uint_as_float(prim) : 0.f);
          }
        }
        t_off += ch.count;
      }
      if (s < 4) meta_lo = set_byte(meta_lo, s, meta);
      else meta_hi = set_byte(meta_hi, s - 4, meta);
      for (int a = 0; a < 3; ++a) {
        float l = floorf(__fdiv_rd(__fsub_rd(ch.lo[a], p[a]), scale[a]));
        float h = ceilf(__fdiv_ru(__fsub_ru(ch.hi[a], p[a]), scale[a]));
        int ql = l < 0.f ? 0 : (l > 255.f ? 255 : (int)l);
        int qh = h < 0.f ? 0 : (h > 255.f ? 255 : (int)h);
        while (ql > 0 && __fadd_rn(p[a], __fmul_rn((float)ql, scale[a])) > ch.lo[a]) ql--;
        while (qh < 255 && __fadd_rn(p[a], __fmul_rn((float)qh, scale[a])) < ch.hi[a]) qh++;
        int word = a * 2 + (s >> 2);
        qlo[word] = set_byte(qlo[word], s & 3, (uint32_t)ql);
        qhi[word] = set_byte(qhi[word], s & 3, (uint32_t)qh);
      }
    }
    nd.e_imask = ebits | (imask << 24);
    nd.child_base = (uint32_t)child_base;
    nd.tri_base = (uint32_t)tri_base;
    nd.meta_lo = meta_lo;
    nd.meta_hi = meta_hi;
    for (int k = 0; k < 6; ++k) {
      nd.qlo[k] = qlo[k];
      nd.qhi[k] = qhi[k];
    }
    wide[wide_base + w] = nd;
  }
}

}  // namespace

shb_status build_bvh(shb_scene* s) {
  shb_context* c = s->ctx;
  cudaStream_t st = c->stream;
  uint32_t T = s->prim_count;
  auto t0 = std::chrono::high_resolution_clock::now();
  s->bvh_node_count = 0;
  s->bvh_tri_count = 0;
  s->bvh_depth = 0;
  if (T == 0) {
    s->bvh_build_ms = 0.0;
    return SHB_OK;
  }
  DevBuf plo, phi, idx, idx2, pslot, pslot2, nodes, sb, bins, split, is_split, rank, act, act2, flag, scanL, tmp;
  SHB_TRY(plo.reserve(sizeof(float4) * T));
  SHB_TRY(phi.reserve(sizeof(float4) * T));
  SHB_TRY(idx.reserve(sizeof(uint32_t) * T));
  SHB_TRY(idx2.reserve(sizeof(uint32_t) * T));
  SHB_TRY(pslot.reserve(sizeof(int) * T));
  SHB_TRY(pslot2.reserve(sizeof(int) * T));
  SHB_TRY(nodes.reserve(sizeof(BNode) * 2 * (size_t)T));
  SHB_TRY(split.reserve(sizeof(int4) * T));
  SHB_TRY(is_split.reserve(sizeof(int) * (T + 1)));
  SHB_TRY(rank.reserve(sizeof(int) * (T + 1)));
  SHB_TRY(act.reserve(sizeof(int) * 2 * (size_t)T));
  SHB_TRY(act2.reserve(sizeof(int) * 2 * (size_t)T));
  SHB_TRY(flag.reserve(sizeof(int) * (T + 1)));
  SHB_TRY(scanL.reserve(sizeof(int) * (T + 1)));
  size_t tmp_bytes = 0, tb2 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flag.as<int>(), scanL.as<int>(), (int)T + 1, st);
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, is_split.as<int>(), rank.as<int>(), (int)T + 1, st);
  tmp_bytes = tmp_bytes > tb2 ? tmp_bytes : tb2;
  SHB_TRY(tmp.reserve(tmp_bytes + 256));

  k_prim_bounds<<<grid_for(T), kThreads, 0, st>>>(T, s->tri_vidx.as<uint32_t>(), s->world_v.as<float>(),
                                                  plo.as<float4>(), phi.as<float4>());
  count_launch(c);
  {
    std::vector<uint32_t> h(T);
    for (uint32_t i = 0; i < T; ++i) h[i] = i;
    SHB_CUDA(cudaMemcpyAsync(idx.ptr, h.data(), sizeof(uint32_t) * T, cudaMemcpyHostToDevice, st));
    SHB_CUDA(cudaMemsetAsync(pslot.ptr, 0, sizeof(int) * T, st));
    BNode root;
    for (int a = 0; a < 3; ++a) {
      root.lo[a] = 0.f;
      root.hi[a] = 0.f;
    }
    root.left = root.right = -1;
    root.begin = 0;
    root.count = (int)T;
    SHB_CUDA(cudaMemcpyAsync(nodes.ptr, &root, sizeof(BNode), cudaMemcpyHostToDevice, st));
    int zero = 0;
    SHB_CUDA(cudaMemcpyAsync(act.ptr, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
    SHB_CUDA(cudaStreamSynchronize(st));
  }
  int n_act = 1, node_count = 1, depth = 0;
  std::vector<int> level_begin = {0};  // binary nodes of depth d: [level_begin[d], level_begin[d + 1])
  size_t slot_cap = 0;
  while (n_act > 0) {
    if ((size_t)n_act > slot_cap) {
      slot_cap = (size_t)n_act;
      SHB_TRY(sb.reserve(sizeof(int) * kSlotBounds * slot_cap));
      SHB_TRY(bins.reserve(sizeof(int) * (size_t)kSlotBinInts * slot_cap));
    }
    k_init_slots<<<grid_for((int64_t)n_act * (kSlotBounds + kSlotBinInts)), kThreads, 0, st>>>(
        n_act, sb.as<int>(), bins.as<int>());
    k_slot_bounds<<<grid_for(T), kThreads, 0, st>>>(T, idx.as<uint32_t>(), pslot.as<int>(), plo.as<float4>(),
                                                   phi.as<float4>(), sb.as<int>());
    k_bins<<<grid_for(T), kThreads, 0, st>>>(T, idx.as<uint32_t>(), pslot.as<int>(), plo.as<float4>(),
                                            phi.as<float4>(), sb.as<int>(), bins.as<int>());
    k_split<<<grid_for(n_act), kThreads, 0, st>>>(n_act, depth, act.as<int>(), nodes.as<BNode>(), sb.as<int>(),
                                                  bins.as<int>(), split.as<int4>(), is_split.as<int>());
    SHB_CUDA(cudaMemsetAsync(is_split.as<int>() + n_act, 0, sizeof(int), st));
    SHB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tmp_bytes, is_split.as<int>(), rank.as<int>(), n_act + 1, st));
    count_launch(c, 6);
    int n_split = 0;
    SHB_CUDA(cudaMemcpyAsync(&n_split, rank.as<int>() + n_act, sizeof(int), cudaMemcpyDeviceToHost, st));
    SHB_CUDA(cudaStreamSynchronize(st));
    if (n_split > 0) {
      k_flags<<<grid_for(T), kThreads, 0, st>>>(T, idx.as<uint32_t>(), pslot.as<int>(), plo.as<float4>(),
                                               phi.as<float4>(), sb.as<int>(), split.as<int4>(), act.as<int>(),
                                               nodes.as<BNode>(), flag.as<int>());
      SHB_CUDA(cudaMemsetAsync(flag.as<int>() + T, 0, sizeof(int), st));
      SHB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tmp_bytes, flag.as<int>(), scanL.as<int>(), (int)T + 1, st));
      k_scatter<<<grid_for(T), kThreads, 0, st>>>(T, idx.as<uint32_t>(), pslot.as<int>(), split.as<int4>(),
                                                 rank.as<int>(), act.as<int>(), nodes.as<BNode>(), flag.as<int>(),
                                                 scanL.as<int>(), idx2.as<uint32_t>(), pslot2.as<int>());
      count_launch(c, 4);
    }
    k_children<<<grid_for(n_act), kThreads, 0, st>>>(n_act, act.as<int>(), nodes.as<BNode>(), split.as<int4>(),
                                                     rank.as<int>(), node_count, act2.as<int>());
    count_launch(c);
    SHB_CUDA(cudaGetLastError());
    if (n_split > 0) {
      idx.swap(idx2);
      pslot.swap(pslot2);
    }
    act.swap(act2);
    level_begin.push_back(node_count);
    node_count += 2 * n_split;
    n_act = 2 * n_split;
    depth++;
  }
  level_begin.push_back(node_count);
  // ---- SAH costs of spreading each subtree over 1..7 wide-node slots, bottom up
  DevBuf dp_cost, dp_dec;
  SHB_TRY(dp_cost.reserve(sizeof(DpCost) * (size_t)node_count));
  SHB_TRY(dp_dec.reserve(sizeof(DpDec) * (size_t)node_count));
  if (SHB_BVH_SAH_COLLAPSE) {
    for (int d = (int)level_begin.size() - 2; d >= 0; --d) {
      const int b0 = level_begin[(size_t)d], b1 = level_begin[(size_t)d + 1];
      if (b1 <= b0) continue;
      k_dp<<<grid_for(b1 - b0), kThreads, 0, st>>>(b0, b1, nodes.as<BNode>(), dp_cost.as<DpCost>(),
                                                    dp_dec.as<DpDec>());
      count_launch(c);
    }
  }
  // ---- collapse into 8-wide nodes
  DevBuf col, nint, ntri, ioff, toff, lev, lev2;
  size_t cap = (size_t)node_count;
  SHB_TRY(col.reserve(sizeof(Collapse) * cap));
  SHB_TRY(nint.reserve(sizeof(int) * (cap + 1)));
  SHB_TRY(ntri.reserve(sizeof(int) * (cap + 1)));
  SHB_TRY(ioff.reserve(sizeof(int) * (cap + 1)));
  SHB_TRY(toff.reserve(sizeof(int) * (cap + 1)));
  SHB_TRY(lev.reserve(sizeof(int) * cap));
  SHB_TRY(lev2.reserve(sizeof(int) * cap));
  SHB_TRY(s->bvh_nodes.reserve(sizeof(WideNode) * cap));
  SHB_TRY(s->bvh_tris.reserve(sizeof(float4) * 3 * (size_t)T));
  size_t tb3 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb3, nint.as<int>(), ioff.as<int>(), (int)cap + 1, st);
  SHB_TRY(tmp.reserve(tb3 + tmp_bytes + 256));
  size_t tmp_all = tmp.bytes;
  {
    int zero = 0;
    SHB_CUDA(cudaMemcpyAsync(lev.ptr, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
  }
  int n_level = 1, wide_count = 1, tri_count = 0, wdepth = 0;
  while (n_level > 0) {
    k_collapse<<<grid_for(n_level), kThreads, 0, st>>>(n_level, lev.as<int>(), nodes.as<BNode>(),
                                                       dp_dec.as<DpDec>(), col.as<Collapse>(), nint.as<int>(),
                                                       ntri.as<int>());
    SHB_CUDA(cudaMemsetAsync(nint.as<int>() + n_level, 0, sizeof(int), st));
    SHB_CUDA(cudaMemsetAsync(ntri.as<int>() + n_level, 0, sizeof(int), st));
    size_t tb = tmp_all;
    SHB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, nint.as<int>(), ioff.as<int>(), n_level + 1, st));
    tb = tmp_all;
    SHB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, ntri.as<int>(), toff.as<int>(), n_level + 1, st));
    int totals[2] = {0, 0};
    SHB_CUDA(cudaMemcpyAsync(&totals[0], ioff.as<int>() + n_level, sizeof(int), cudaMemcpyDeviceToHost, st));
    SHB_CUDA(cudaMemcpyAsync(&totals[1], toff.as<int>() + n_level, sizeof(int), cudaMemcpyDeviceToHost, st));
    k_emit<<<grid_for(n_level), kThreads, 0, st>>>(
        n_level, wide_count - n_level, wide_count, tri_count, col.as<Collapse>(), ioff.as<int>(), toff.as<int>(),
        nodes.as<BNode>(), idx.as<uint32_t>(), s->tri_vidx.as<uint32_t>(), s->world_v.as<float>(), lev.as<int>(),
        s->bvh_nodes.as<WideNode>(), s->bvh_tris.as<float4>(), lev2.as<int>());
    count_launch(c, 4);
    SHB_CUDA(cudaStreamSynchronize(st));
    SHB_CUDA(cudaGetLastError());
    tri_count += totals[1];
    wide_count += totals[0];
    n_level = totals[0];
    lev.swap(lev2);
    wdepth++;
  }
  s->bvh_node_count = (uint32_t)wide_count;
  s->bvh_tri_count = (uint32_t)tri_count;
  s->bvh_depth = (uint32_t)wdepth;
  auto t1 = std::chrono::high_resolution_clock::now();
  s->bvh_build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  if ((uint32_t)tri_count != T) {
    set_error("BVH build lost triangles");
    return SHB_ERR_INTERNAL;
  }
  return SHB_OK;
}

}  // namespace shb
