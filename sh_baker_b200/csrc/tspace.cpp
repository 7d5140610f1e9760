// tspace.cpp - tangent frames by the MikkTSpace method.
//
// The reference builds missing tangents with MikkTSpace's
// genTangSpaceDefault (src/loader.cpp:88-109, called at :363-368; the
// library is fetched at configure time from github.com/mmikk/MikkTSpace,
// branch master, and is not part of the reference tree).  This file
// restates the method as Mikkelsen describes it ("Simulation of wrinkled
// surfaces revisited", 2008, and the library's interface notes), in its own
// code:
//   1. Corners are welded: two corners are one vertex when position, normal
//      and texture UV compare equal.
//   2. Each triangle gets the direction of dP/du (the UV-space tangent) and
//      an orientation: whether its UV triangle winds counter-clockwise
//      (positive signed UV area).  A triangle with zero UV area has no
//      tangent of its own and takes the orientation of the first group that
//      reaches it.
//   3. Around each welded vertex, triangles that share an edge through it
//      (opposite winding, as in a consistently wound manifold) and have the
//      same orientation form one group.  The default angular threshold of
//      180 degrees never splits a group further.
//   4. A group's tangent is the normalised sum, over its corners, of the
//      triangle tangent projected onto the plane of the vertex normal and
//      normalised, weighted by the corner's angle measured between the two
//      edges projected onto that plane.  The sign is +1 for an
//      orientation-preserving group, -1 otherwise.
//   5. The frames are written per corner in face order to the corner's
//      vertex index, so a vertex index used by corners of several groups
//      keeps the last one, as the reference's SetTSpaceBasic callback does
//      (src/loader.cpp:73-86).
// Deliberate differences, for inputs the library treats as degenerate: a
// triangle two of whose corners weld together contributes and writes
// nothing; a group whose sum vanishes, and a vertex that no triangle
// writes, get the reference's geometric fallback (src/loader.cpp:370-385)
// instead of a zero tangent (with a zero tangent the reference's hemisphere
// frame, src/baker.cpp:266-271, collapses onto the normal).
#include "tspace.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

namespace shb {
namespace {

struct V3 {
  float x, y, z;
};

V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 scale(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Unit vector along `a`, or `a` itself when its length is zero.
V3 unit_or_same(V3 a) {
  const float l2 = dot(a, a);
  if (!(l2 > 0.0f)) return a;
  return scale(a, 1.0f / std::sqrt(l2));
}

// `a` with its component along the unit normal `n` removed, then unit.
V3 in_plane(V3 a, V3 n) { return unit_or_same(sub(a, scale(n, dot(n, a)))); }

bool is_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }

// The reference's tangent for a vertex without a UV frame: X (or Y when the
// normal is close to X) with its normal component removed, normalised.
void geometric_fallback(const float* n, float* t) {
  const float a[3] = {std::fabs(n[0]) < 0.9f ? 1.0f : 0.0f, std::fabs(n[0]) < 0.9f ? 0.0f : 1.0f, 0.0f};
  const float na = n[0] * a[0] + n[1] * a[1] + n[2] * a[2];
  float v[3] = {a[0] - n[0] * na, a[1] - n[1] * na, a[2] - n[2] * na};
  const float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const float r = l > 0.0f ? 1.0f / l : 1.0f;
  t[0] = v[0] * r;
  t[1] = v[1] * r;
  t[2] = v[2] * r;
  t[3] = 1.0f;
}

// Welded vertex id of every vertex index: equal position, normal and UV give
// one id.  Values compare by their bits with -0 taken as +0, which is float
// equality for every value but NaN.
std::vector<uint32_t> weld(const float* pos, const float* nrm, const float* uv, size_t nv) {
  auto key = [&](uint32_t v, int k) -> uint32_t {
    const float x = k < 3 ? pos[3 * v + k] : k < 6 ? nrm[3 * v + k - 3] : uv[2 * v + k - 6];
    uint32_t b;
    std::memcpy(&b, &x, 4);
    return b == 0x80000000u ? 0u : b;
  };
  std::vector<uint32_t> order(nv);
  std::iota(order.begin(), order.end(), 0u);
  auto less = [&](uint32_t a, uint32_t b) {
    for (int k = 0; k < 8; ++k) {
      const uint32_t x = key(a, k), y = key(b, k);
      if (x != y) return x < y;
    }
    return a < b;
  };
  std::sort(order.begin(), order.end(), less);
  std::vector<uint32_t> id(nv);
  for (size_t i = 0; i < nv; ++i) {
    const uint32_t v = order[i];
    bool same = i > 0;
    for (int k = 0; same && k < 8; ++k) same = key(v, k) == key(order[i - 1], k);
    id[v] = same ? id[order[i - 1]] : v;
  }
  return id;
}

struct Group {
  V3 sum;
  bool orient;
};

}  // namespace

void generate_tangent_frames(const float* pos, const float* nrm, const float* uv, size_t nv, const uint32_t* idx,
                             size_t n_idx, float* out) {
  for (size_t v = 0; v < nv; ++v) geometric_fallback(nrm + 3 * v, out + 4 * v);
  const size_t nt = n_idx / 3;
  if (nt == 0) return;
  const std::vector<uint32_t> wid = weld(pos, nrm, uv, nv);
  auto P = [&](uint32_t v) { return V3{pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]}; };
  auto N = [&](uint32_t v) { return V3{nrm[3 * v], nrm[3 * v + 1], nrm[3 * v + 2]}; };
  std::vector<uint32_t> w(3 * nt);
  for (size_t c = 0; c < 3 * nt; ++c) w[c] = wid[idx[c]];

  // 2. Per-triangle UV tangent and orientation (-1: undetermined).
  std::vector<V3> tan(nt, V3{0.0f, 0.0f, 0.0f});
  std::vector<int8_t> orient(nt, -1);
  std::vector<uint8_t> degen(nt, 0);
  for (size_t t = 0; t < nt; ++t) {
    const uint32_t* c = &w[3 * t];
    degen[t] = c[0] == c[1] || c[1] == c[2] || c[0] == c[2];
    const uint32_t i0 = idx[3 * t], i1 = idx[3 * t + 1], i2 = idx[3 * t + 2];
    const V3 e1 = sub(P(i1), P(i0)), e2 = sub(P(i2), P(i0));
    const float du1 = uv[2 * i1] - uv[2 * i0], dv1 = uv[2 * i1 + 1] - uv[2 * i0 + 1];
    const float du2 = uv[2 * i2] - uv[2 * i0], dv2 = uv[2 * i2 + 1] - uv[2 * i0 + 1];
    const float area2 = du1 * dv2 - dv1 * du2;
    if (area2 != 0.0f) {
      // dP/du = (dv2 e1 - dv1 e2) / area2: its direction
      const V3 s = sub(scale(e1, dv2), scale(e2, dv1));
      tan[t] = unit_or_same(area2 > 0.0f ? s : scale(s, -1.0f));
      orient[t] = area2 > 0.0f ? 1 : 0;
    }
  }

  // 3a. Neighbour across each edge (corner e -> corner e+1): the lowest-index
  // triangle holding the same welded edge in the opposite direction.
  struct Edge {
    uint32_t a, b, tri;
  };
  std::vector<Edge> edges;
  edges.reserve(3 * nt);
  for (size_t t = 0; t < nt; ++t)
    if (!degen[t])
      for (int e = 0; e < 3; ++e) edges.push_back({w[3 * t + e], w[3 * t + (e + 1) % 3], (uint32_t)t});
  std::sort(edges.begin(), edges.end(), [](const Edge& x, const Edge& y) {
    return x.a != y.a ? x.a < y.a : x.b != y.b ? x.b < y.b : x.tri < y.tri;
  });
  std::vector<int64_t> nb(3 * nt, -1);
  for (size_t t = 0; t < nt; ++t) {
    if (degen[t]) continue;
    for (int e = 0; e < 3; ++e) {
      const Edge want{w[3 * t + (e + 1) % 3], w[3 * t + e], 0};
      auto it = std::lower_bound(edges.begin(), edges.end(), want, [](const Edge& x, const Edge& y) {
        return x.a != y.a ? x.a < y.a : x.b < y.b;
      });
      for (; it != edges.end() && it->a == want.a && it->b == want.b; ++it)
        if (it->tri != t) {
          nb[3 * t + e] = it->tri;
          break;
        }
    }
  }

  // 3b. Groups: around the welded vertex of a corner, flood across the two
  // edges through it to triangles of the same orientation.
  std::vector<int32_t> grp(3 * nt, -1);
  std::vector<Group> groups;
  std::vector<std::pair<uint32_t, int>> stack;
  for (size_t t = 0; t < nt; ++t) {
    if (degen[t]) continue;
    for (int k = 0; k < 3; ++k) {
      if (grp[3 * t + k] >= 0) continue;
      if (orient[t] < 0) orient[t] = 0;  // no group reached it: not orientation-preserving
      const int32_t g = (int32_t)groups.size();
      groups.push_back({V3{0.0f, 0.0f, 0.0f}, orient[t] == 1});
      const uint32_t vert = w[3 * t + k];
      grp[3 * t + k] = g;
      stack.assign(1, {(uint32_t)t, k});
      while (!stack.empty()) {
        const auto [u, c] = stack.back();
        stack.pop_back();
        for (int e : {c, (c + 2) % 3}) {
          const int64_t n = nb[3 * (size_t)u + e];
          if (n < 0) continue;
          int cn = 0;
          while (cn < 3 && w[3 * n + cn] != vert) ++cn;
          if (cn == 3) continue;
          if (orient[n] < 0) orient[n] = groups[g].orient ? 1 : 0;  // adopts the group's orientation
          if ((orient[n] == 1) != groups[g].orient || grp[3 * n + cn] >= 0) continue;
          grp[3 * n + cn] = g;
          stack.push_back({(uint32_t)n, cn});
        }
      }
    }
  }

  // 4. Angle-weighted sum of the in-plane triangle tangents per group.
  for (size_t t = 0; t < nt; ++t) {
    if (degen[t] || is_zero(tan[t])) continue;
    for (int k = 0; k < 3; ++k) {
      const uint32_t i = idx[3 * t + k], i1 = idx[3 * t + (k + 1) % 3], i2 = idx[3 * t + (k + 2) % 3];
      const V3 n = N(i), p = P(i);
      const V3 a = in_plane(sub(P(i1), p), n), b = in_plane(sub(P(i2), p), n);
      const float cosv = std::min(1.0f, std::max(-1.0f, dot(a, b)));
      const float angle = std::acos(cosv);
      Group& G = groups[(size_t)grp[3 * t + k]];
      G.sum = add(G.sum, scale(in_plane(tan[t], n), angle));
    }
  }

  // 5. Per corner in face order, to the corner's vertex index.
  for (size_t t = 0; t < nt; ++t) {
    if (degen[t]) continue;
    for (int k = 0; k < 3; ++k) {
      const uint32_t i = idx[3 * t + k];
      const Group& G = groups[(size_t)grp[3 * t + k]];
      const V3 d = unit_or_same(G.sum);
      float* o = out + 4 * (size_t)i;
      if (is_zero(d) || !std::isfinite(d.x + d.y + d.z)) {
        geometric_fallback(nrm + 3 * (size_t)i, o);
        continue;
      }
      o[0] = d.x;
      o[1] = d.y;
      o[2] = d.z;
      o[3] = G.orient ? 1.0f : -1.0f;
    }
  }
}

}  // namespace shb
