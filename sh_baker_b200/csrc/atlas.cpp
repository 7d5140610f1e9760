// atlas.cpp - CreateAtlasGeometries and CalculateGeometryScales
// (src/atlas.h:28-53, src/atlas.cpp:21-250): new, non-overlapping lightmap
// UVs for every geometry, packed into one square page.
//
// The reference hands the transformed, per-geometry scaled meshes to xatlas,
// a third-party library fetched at configure time (absent here).  This file
// is a chart builder of its own with the same contract:
//   - per-geometry scale = density * sqrt(albedo w*h) * sqrt(UV tile count),
//     clamped to 5x the median (CalculateGeometryScales, restated exactly);
//   - charts never cross geometries; a vertex on a chart seam is split, and
//     every output vertex keeps the attributes of its source vertex (xatlas'
//     xref, src/atlas.cpp:187-229); face order and corner order are kept,
//     vertices no face uses are dropped;
//   - all charts land in one page of target_resolution^2 texels with at
//     least `padding` empty texels between the texels of two charts; a scene
//     that does not fit fails (the reference's atlasCount > 1 error);
//   - lightmap UVs are texel positions / page size, in [0, 1].
// Charts: faces grow from the largest unassigned face over shared edges
// (vertices welded by position), best-aligned neighbour first, while the
// face normal stays within acos(0.8) ~ 37 deg of the chart's area-weighted
// mean normal; the chart is projected onto the plane of that mean.  A chart
// whose projection shrinks a face below 0.7 of its area (or flips it) or
// overlaps itself is cut back to the faces grown before the first offending
// one, and the rest grow again.  Each chart
// is turned to its minimum-area bounding rectangle (rotating calipers over
// its convex hull); a skyline bottom-left packer places the rectangles, and a
// bisection on texels per unit finds the largest scale that fits the page.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <queue>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "host_scene.h"
#include "shb_internal.h"

namespace shb {
namespace {

constexpr float kMinScale = 0.001f;     // src/atlas.cpp:15
constexpr float kMaxScaleFactor = 5.0f; // src/atlas.cpp:16
constexpr double kChartCos = 0.8;       // face normal vs chart mean normal
constexpr double kMinProjCos = 0.7;     // least projected / true face area in a chart

struct D3 {
  double x, y, z;
};
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double len(D3 a) { return std::sqrt(dot(a, a)); }

struct D2 {
  double x, y;
};
inline double cross2(D2 o, D2 a, D2 b) { return (a.x - o.x) * (b.y - o.y) - (a.y - o.y) * (b.x - o.x); }

// One chart of one geometry: its faces, the chart-plane coordinates of each
// face corner (scaled world units, aligned to the minimum-area rectangle
// whose lower-left corner is the origin) and the rectangle's extent.
struct Chart {
  std::vector<uint32_t> faces;
  std::vector<D2> corner;  // 3 per face, in the order of `faces`
  double w = 0, h = 0;
  // placement: texel offset of the footprint, 90-degree turn
  int ox = 0, oy = 0;
  bool turned = false;
};

struct GeoCharts {
  std::vector<Chart> charts;
  std::vector<uint32_t> chart_of;  // per face
  std::vector<uint32_t> slot_of;   // per face: its index within its chart
};

// ---------------------------------------------------- geometry scales ----

bool geometry_scales(const shb_scene_desc* d, float density, std::vector<float>& out, std::string& err) {
  out.clear();
  for (uint32_t g = 0; g < d->geometry_count; ++g) {
    const shb_geometry_desc& G = d->geometries[g];
    if (G.material_id < 0 || (uint32_t)G.material_id >= d->material_count) {
      err = "geometry " + std::to_string(g) + ": material_id out of range";
      return false;
    }
    if (!G.texture_uvs || G.vertex_count == 0) {
      err = "geometry " + std::to_string(g) + ": texture_uvs required";
      return false;
    }
    const shb_material_desc& M = d->materials[G.material_id];
    const float width = (float)M.albedo_width, height = (float)M.albedo_height;
    const float target = density * std::sqrt(width * height);
    float u0 = std::numeric_limits<float>::max(), u1 = std::numeric_limits<float>::lowest();
    float v0 = u0, v1 = u1;
    for (uint32_t v = 0; v < G.vertex_count; ++v) {
      u0 = std::min(u0, G.texture_uvs[2 * v]);
      u1 = std::max(u1, G.texture_uvs[2 * v]);
      v0 = std::min(v0, G.texture_uvs[2 * v + 1]);
      v1 = std::max(v1, G.texture_uvs[2 * v + 1]);
    }
    const float ur = std::max(u1 - u0, 0.001f), vr = std::max(v1 - v0, 0.001f);
    const float tiles = ur * vr;
    out.push_back(target * std::sqrt(tiles));
  }
  if (!out.empty()) {
    std::vector<float> sorted = out;
    std::sort(sorted.begin(), sorted.end());
    const float median = std::max(sorted[sorted.size() / 2], 0.001f);
    const float cap = kMaxScaleFactor * median;
    for (float& s : out) s = std::min(s, cap);
  }
  return true;
}

// ------------------------------------------------------------ charts ----

struct Mesh {
  std::vector<D3> p;         // welded positions (scaled world space)
  std::vector<uint32_t> wv;  // per face corner: welded vertex id
  std::vector<D3> n;         // per face: unit normal (zero when degenerate)
  std::vector<double> area;  // per face
  std::vector<uint32_t> adj_off, adj;
};

struct Bits3Hash {
  size_t operator()(const std::array<uint64_t, 3>& k) const {
    uint64_t h = k[0] * 0x9E3779B97F4A7C15ull;
    h ^= k[1] + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
    h ^= k[2] + 0x85EBCA77C2B2AE63ull + (h << 6) + (h >> 2);
    return (size_t)h;
  }
};

void build_mesh(const shb_geometry_desc& G, float scale, Mesh& m) {
  const float* T = G.transform;
  const uint32_t nf = G.index_count / 3;
  std::unordered_map<std::array<uint64_t, 3>, uint32_t, Bits3Hash> weld;
  std::vector<uint32_t> wid(G.vertex_count, UINT32_MAX);
  m.wv.resize(3 * (size_t)nf);
  for (uint32_t f = 0; f < nf; ++f)
    for (int k = 0; k < 3; ++k) {
      const uint32_t v = G.indices[3 * f + k];
      if (wid[v] == UINT32_MAX) {
        const double x = G.vertices[3 * v], y = G.vertices[3 * v + 1], z = G.vertices[3 * v + 2];
        D3 w{T[0] * x + T[1] * y + T[2] * z + T[3], T[4] * x + T[5] * y + T[6] * z + T[7],
             T[8] * x + T[9] * y + T[10] * z + T[11]};
        w = w * (double)scale;
        w = w + D3{0.0, 0.0, 0.0};  // -0 and +0 weld together
        std::array<uint64_t, 3> key;
        std::memcpy(&key[0], &w.x, 8);
        std::memcpy(&key[1], &w.y, 8);
        std::memcpy(&key[2], &w.z, 8);
        auto it = weld.emplace(key, (uint32_t)m.p.size());
        if (it.second) m.p.push_back(w);
        wid[v] = it.first->second;
      }
      m.wv[3 * (size_t)f + k] = wid[v];
    }
  m.n.resize(nf);
  m.area.resize(nf);
  for (uint32_t f = 0; f < nf; ++f) {
    const D3 a = m.p[m.wv[3 * f]], b = m.p[m.wv[3 * f + 1]], c = m.p[m.wv[3 * f + 2]];
    const D3 e1 = b - a, e2 = c - a, x = cross(e1, e2);
    const double l = len(x);
    const bool degen = !(l > 1e-12 * len(e1) * len(e2)) || m.wv[3 * f] == m.wv[3 * f + 1] ||
                       m.wv[3 * f + 1] == m.wv[3 * f + 2] || m.wv[3 * f] == m.wv[3 * f + 2];
    m.n[f] = degen ? D3{0, 0, 0} : x * (1.0 / l);
    m.area[f] = degen ? 0.0 : 0.5 * l;
  }
  // faces sharing an edge (welded), through a sorted edge list
  std::vector<std::pair<uint64_t, uint32_t>> edges;
  edges.reserve(3 * (size_t)nf);
  for (uint32_t f = 0; f < nf; ++f)
    for (int k = 0; k < 3; ++k) {
      uint32_t a = m.wv[3 * f + k], b = m.wv[3 * f + (k + 1) % 3];
      if (a == b) continue;
      if (a > b) std::swap(a, b);
      edges.push_back({((uint64_t)a << 32) | b, f});
    }
  std::sort(edges.begin(), edges.end());
  std::vector<std::pair<uint32_t, uint32_t>> links;
  for (size_t i = 0; i < edges.size();) {
    size_t j = i;
    while (j < edges.size() && edges[j].first == edges[i].first) ++j;
    for (size_t a = i; a < j; ++a)
      for (size_t b = i; b < j; ++b)
        if (edges[a].second != edges[b].second) links.push_back({edges[a].second, edges[b].second});
    i = j;
  }
  std::sort(links.begin(), links.end());
  links.erase(std::unique(links.begin(), links.end()), links.end());
  m.adj_off.assign(nf + 1, 0);
  for (auto& l : links) m.adj_off[l.first + 1]++;
  for (uint32_t f = 0; f < nf; ++f) m.adj_off[f + 1] += m.adj_off[f];
  m.adj.resize(links.size());
  for (size_t i = 0; i < links.size(); ++i) m.adj[i] = links[i].second;  // sorted by first: CSR order
}

// Plane basis for a projection axis: u, v with u x v = axis.
void basis(D3 n, D3& u, D3& v) {
  const D3 a = std::fabs(n.x) < std::fabs(n.y) ? (std::fabs(n.x) < std::fabs(n.z) ? D3{1, 0, 0} : D3{0, 0, 1})
                                               : (std::fabs(n.y) < std::fabs(n.z) ? D3{0, 1, 0} : D3{0, 0, 1});
  u = cross(a, n);
  u = u * (1.0 / len(u));
  v = cross(n, u);
}

// Strict interior overlap of two 2-D triangles (separating axis, with a
// tolerance that lets them touch).
bool tri_overlap(const D2* a, const D2* b, double eps) {
  for (int pass = 0; pass < 2; ++pass) {
    const D2* t = pass ? b : a;
    const D2* o = pass ? a : b;
    for (int k = 0; k < 3; ++k) {
      const D2 p = t[k], q = t[(k + 1) % 3];
      const double nx = q.y - p.y, ny = p.x - q.x;
      double tmin = 1e300, tmax = -1e300, omin = 1e300, omax = -1e300;
      for (int i = 0; i < 3; ++i) {
        const double s = nx * t[i].x + ny * t[i].y, r = nx * o[i].x + ny * o[i].y;
        tmin = std::min(tmin, s);
        tmax = std::max(tmax, s);
        omin = std::min(omin, r);
        omax = std::max(omax, r);
      }
      const double e = eps * std::sqrt(nx * nx + ny * ny);
      if (tmax <= omin + e || omax <= tmin + e) return false;
    }
  }
  return true;
}

// Projects a chart's faces (growth order) onto the plane of their mean
// normal.  Returns the index of the first face to cut (faces.size() when
// the projection is one-to-one).
size_t project(const Mesh& m, const std::vector<uint32_t>& faces, std::vector<D2>& corner) {
  D3 ns{0, 0, 0};
  for (uint32_t f : faces) ns = ns + m.n[f] * m.area[f];
  const double l = len(ns);
  D3 axis = l > 0 ? ns * (1.0 / l) : D3{0, 0, 1};
  if (!(l > 0)) {
    for (uint32_t f : faces)
      if (m.area[f] > 0) {
        axis = m.n[f];
        break;
      }
  }
  D3 u, v;
  basis(axis, u, v);
  corner.resize(3 * faces.size());
  double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
  for (size_t i = 0; i < faces.size(); ++i)
    for (int k = 0; k < 3; ++k) {
      const D3 p = m.p[m.wv[3 * faces[i] + k]];
      const D2 q{dot(p, u), dot(p, v)};
      corner[3 * i + k] = q;
      x0 = std::min(x0, q.x);
      y0 = std::min(y0, q.y);
      x1 = std::max(x1, q.x);
      y1 = std::max(y1, q.y);
    }
  size_t cut = faces.size();
  for (size_t i = 0; i < faces.size(); ++i) {
    const uint32_t f = faces[i];
    if (m.area[f] <= 0) continue;
    const double a2 = cross2(corner[3 * i], corner[3 * i + 1], corner[3 * i + 2]);
    if (!(a2 > 2.0 * kMinProjCos * m.area[f])) {
      cut = i;
      break;
    }
  }
  // overlaps among the faces before `cut`, through a uniform grid
  const size_t n = cut;
  if (n < 2) return cut;
  const double span = std::max(x1 - x0, y1 - y0);
  const double eps = 1e-9 * std::max(span, 1e-30);
  double sum_a = 0;
  for (size_t i = 0; i < n; ++i) sum_a += m.area[faces[i]];
  double cell = std::sqrt(std::max(sum_a, 1e-300) / (double)n) * 2.0;
  if (!(cell > 0)) cell = std::max(span, 1e-30);
  const int gx = (int)std::min<double>(std::max(1.0, std::ceil((x1 - x0) / cell)), 2048.0);
  const int gy = (int)std::min<double>(std::max(1.0, std::ceil((y1 - y0) / cell)), 2048.0);
  const double cx = std::max(x1 - x0, 1e-300) / gx, cy = std::max(y1 - y0, 1e-300) / gy;
  auto cell_of = [&](double x, double y, int& i, int& j) {
    i = std::min(gx - 1, std::max(0, (int)((x - x0) / cx)));
    j = std::min(gy - 1, std::max(0, (int)((y - y0) / cy)));
  };
  std::vector<std::vector<uint32_t>> grid((size_t)gx * gy);
  std::vector<std::array<double, 4>> box(n);
  for (size_t t = 0; t < n; ++t) {
    const D2* c = &corner[3 * t];
    box[t] = {std::min({c[0].x, c[1].x, c[2].x}), std::min({c[0].y, c[1].y, c[2].y}),
              std::max({c[0].x, c[1].x, c[2].x}), std::max({c[0].y, c[1].y, c[2].y})};
    if (m.area[faces[t]] <= 0) continue;
    int i0, j0, i1, j1;
    cell_of(box[t][0], box[t][1], i0, j0);
    cell_of(box[t][2], box[t][3], i1, j1);
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) grid[(size_t)j * gx + i].push_back((uint32_t)t);
  }
  for (int j = 0; j < gy; ++j)
    for (int i = 0; i < gx; ++i) {
      const auto& c = grid[(size_t)j * gx + i];
      for (size_t a = 0; a < c.size(); ++a)
        for (size_t b = a + 1; b < c.size(); ++b) {
          const uint32_t s = c[a], t = c[b];
          const size_t later = std::max(s, t);
          if (later >= cut) continue;
          // test each pair once: in the cell holding the corner of the
          // boxes' intersection
          const double ix = std::max(box[s][0], box[t][0]), iy = std::max(box[s][1], box[t][1]);
          if (ix > std::min(box[s][2], box[t][2]) || iy > std::min(box[s][3], box[t][3])) continue;
          int ci, cj;
          cell_of(ix, iy, ci, cj);
          if (ci != i || cj != j) continue;
          int shared = 0;
          for (int p = 0; p < 3; ++p)
            for (int q = 0; q < 3; ++q) shared += m.wv[3 * faces[s] + p] == m.wv[3 * faces[t] + q];
          if (shared >= 2) continue;  // edge neighbours lie on either side (both unflipped)
          if (tri_overlap(&corner[3 * s], &corner[3 * t], eps)) cut = later;
        }
    }
  return cut;
}

// Turns a projected chart to its minimum-area bounding rectangle, lower
// left corner at the origin, wider than high.
void fit_rectangle(Chart& ch) {
  std::vector<D2> pts = ch.corner;
  std::sort(pts.begin(), pts.end(), [](D2 a, D2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
  pts.erase(std::unique(pts.begin(), pts.end(), [](D2 a, D2 b) { return a.x == b.x && a.y == b.y; }), pts.end());
  std::vector<D2> hull;
  if (pts.size() >= 3) {
    hull.resize(2 * pts.size());
    size_t k = 0;
    for (size_t i = 0; i < pts.size(); ++i) {
      while (k >= 2 && cross2(hull[k - 2], hull[k - 1], pts[i]) <= 0) --k;
      hull[k++] = pts[i];
    }
    for (size_t i = pts.size() - 1, t = k + 1; i > 0; --i) {
      while (k >= t && cross2(hull[k - 2], hull[k - 1], pts[i - 1]) <= 0) --k;
      hull[k++] = pts[i - 1];
    }
    hull.resize(k - 1);
  } else {
    hull = pts;
  }
  double best = 1e300, bx = 1, by = 0;
  for (size_t i = 0; i < hull.size(); ++i) {
    const D2 p = hull[i], q = hull[(i + 1) % hull.size()];
    double ex = q.x - p.x, ey = q.y - p.y;
    const double l = std::sqrt(ex * ex + ey * ey);
    if (!(l > 0)) continue;
    ex /= l;
    ey /= l;
    double a0 = 1e300, a1 = -1e300, b0 = 1e300, b1 = -1e300;
    for (const D2& h : hull) {
      const double a = h.x * ex + h.y * ey, b = -h.x * ey + h.y * ex;
      a0 = std::min(a0, a);
      a1 = std::max(a1, a);
      b0 = std::min(b0, b);
      b1 = std::max(b1, b);
    }
    const double area = (a1 - a0) * (b1 - b0);
    if (area < best * (1.0 - 1e-12)) {
      best = area;
      bx = ex;
      by = ey;
    }
  }
  double a0 = 1e300, a1 = -1e300, b0 = 1e300, b1 = -1e300;
  for (D2& c : ch.corner) {
    const D2 r{c.x * bx + c.y * by, -c.x * by + c.y * bx};
    c = r;
    a0 = std::min(a0, r.x);
    a1 = std::max(a1, r.x);
    b0 = std::min(b0, r.y);
    b1 = std::max(b1, r.y);
  }
  if (ch.corner.empty()) a0 = a1 = b0 = b1 = 0;
  ch.w = a1 - a0;
  ch.h = b1 - b0;
  for (D2& c : ch.corner) c = D2{c.x - a0, c.y - b0};
  if (ch.h > ch.w) {  // quarter turn: (x, y) -> (h - y, x)
    for (D2& c : ch.corner) c = D2{ch.h - c.y, c.x};
    std::swap(ch.w, ch.h);
  }
}

void build_charts(const shb_geometry_desc& G, float scale, GeoCharts& out) {
  Mesh m;
  build_mesh(G, scale, m);
  const uint32_t nf = G.index_count / 3;
  out.charts.clear();
  out.chart_of.assign(nf, UINT32_MAX);
  out.slot_of.assign(nf, 0);
  std::vector<uint32_t> order(nf);
  for (uint32_t f = 0; f < nf; ++f) order[f] = f;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return m.area[a] > m.area[b]; });
  std::vector<uint8_t> taken(nf, 0);
  using Item = std::pair<double, uint32_t>;
  for (bool again = true; again;) {
    again = false;
    for (uint32_t seed : order) {
      if (taken[seed]) continue;
      std::vector<uint32_t> faces{seed};
      taken[seed] = 1;
      D3 ns = m.n[seed] * m.area[seed];
      std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
      auto push_adj = [&](uint32_t f) {
        const double l = len(ns);
        for (uint32_t k = m.adj_off[f]; k < m.adj_off[f + 1]; ++k) {
          const uint32_t g = m.adj[k];
          if (taken[g]) continue;
          const double cost = m.area[g] <= 0 ? -1.0 : (l > 0 ? 1.0 - dot(m.n[g], ns) / l : 0.0);
          heap.push({cost, g});
        }
      };
      push_adj(seed);
      while (!heap.empty()) {
        const uint32_t f = heap.top().second;
        heap.pop();
        if (taken[f]) continue;
        const double l = len(ns);
        if (m.area[f] > 0 && l > 0 && dot(m.n[f], ns) < kChartCos * l) continue;
        taken[f] = 1;
        faces.push_back(f);
        ns = ns + m.n[f] * m.area[f];
        push_adj(f);
      }
      Chart ch;
      for (;;) {
        size_t cut = project(m, faces, ch.corner);
        if (cut == faces.size()) break;
        if (cut == 0) cut = 1;  // a face alone is always one-to-one
        for (size_t i = cut; i < faces.size(); ++i) taken[faces[i]] = 0;
        faces.resize(cut);
        again = true;
      }
      const uint32_t id = (uint32_t)out.charts.size();
      for (size_t i = 0; i < faces.size(); ++i) {
        out.chart_of[faces[i]] = id;
        out.slot_of[faces[i]] = (uint32_t)i;
      }
      ch.faces = std::move(faces);
      fit_rectangle(ch);
      out.charts.push_back(std::move(ch));
    }
  }
}

// ----------------------------------------------------------- packing ----

// Skyline bottom-left packing of (w + pad) x (h + pad) footprints into a
// (W + pad) x (H + pad) page (the trailing pad may leave the page).
struct Skyline {
  struct Seg {
    int x, y, w;
  };
  std::vector<Seg> seg;
  int W, H;
  Skyline(int w, int h) : seg{{0, 0, w}}, W(w), H(h) {}
  // lowest top edge for a rw x rh footprint; false if none fits
  bool find(int rw, int rh, int& bx, int& by, int& top) const {
    bool ok = false;
    for (size_t i = 0; i < seg.size(); ++i) {
      const int x = seg[i].x;
      if (x + rw > W) break;
      int y = 0, reach = 0;
      for (size_t j = i; j < seg.size() && reach < rw; ++j) {
        y = std::max(y, seg[j].y);
        reach = seg[j].x + seg[j].w - x;
      }
      if (y + rh > H) continue;
      if (!ok || y + rh < top || (y + rh == top && x < bx)) {
        ok = true;
        bx = x;
        by = y;
        top = y + rh;
      }
    }
    return ok;
  }
  void add(int x, int y, int rw, int rh) {
    std::vector<Seg> out;
    out.reserve(seg.size() + 2);
    bool placed = false;
    for (const Seg& s : seg) {
      const int s1 = s.x + s.w;
      if (s1 <= x) {  // left of the footprint
        out.push_back(s);
        continue;
      }
      if (s.x >= x + rw) {  // right of it
        if (!placed) out.push_back({x, y + rh, rw});
        placed = true;
        out.push_back(s);
        continue;
      }
      if (s.x < x) out.push_back({s.x, s.y, x - s.x});
      if (!placed) out.push_back({x, y + rh, rw});
      placed = true;
      if (s1 > x + rw) out.push_back({x + rw, s.y, s1 - (x + rw)});
    }
    if (!placed) out.push_back({x, y + rh, rw});
    seg.clear();  // merge neighbours of equal height
    for (const Seg& s : out) {
      if (!seg.empty() && seg.back().y == s.y && seg.back().x + seg.back().w == s.x) seg.back().w += s.w;
      else seg.push_back(s);
    }
  }
};

struct Rect {
  uint32_t geo, chart;
  double w, h;
};

// Footprint of a chart of extent (w, h) units at `s` texels per unit.  An
// extent beyond 2^30 texels, or not a number, gets a footprint of 2^30,
// which no page holds, so packing fails instead of casting out of int range.
inline int foot(double e, double s) {
  const double f = std::ceil(e * s - 1e-9);
  if (f != f || f >= 1073741824.0) return 1073741824;
  return f < 1.0 ? 1 : (int)f;
}

bool pack(std::vector<Rect>& rects, double s, int W, int H, int pad, std::vector<std::array<int, 3>>* place) {
  std::vector<uint32_t> order(rects.size());
  for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    const int ha = foot(rects[a].h, s), hb = foot(rects[b].h, s);
    if (ha != hb) return ha > hb;
    return foot(rects[a].w, s) > foot(rects[b].w, s);
  });
  Skyline sky(W + pad, H + pad);
  if (place) place->assign(rects.size(), {0, 0, 0});
  for (uint32_t i : order) {
    const int fw = foot(rects[i].w, s) + pad, fh = foot(rects[i].h, s) + pad;
    int x0 = 0, y0 = 0, t0 = 0, x1 = 0, y1 = 0, t1 = 0;
    const bool a = sky.find(fw, fh, x0, y0, t0);
    const bool b = fw != fh && sky.find(fh, fw, x1, y1, t1);
    if (!a && !b) return false;
    const bool turn = b && (!a || t1 < t0);
    if (turn) sky.add(x1, y1, fh, fw);
    else sky.add(x0, y0, fw, fh);
    if (place) (*place)[i] = {turn ? x1 : x0, turn ? y1 : y0, turn ? 1 : 0};
  }
  return true;
}

}  // namespace
}  // namespace shb

using namespace shb;

extern "C" {

shb_status shb_atlas_geometry_scales(const shb_scene_desc* scene, float density_multiplier, float* scales_out) {
  return ::shb::guarded("shb_atlas_geometry_scales", [&]() -> shb_status {
    if (!scene || (scene->geometry_count && (!scene->geometries || !scales_out))) {
      set_error("NULL argument");
      return SHB_ERR_INVALID_ARG;
    }
    std::vector<float> s;
    std::string err;
    if (!geometry_scales(scene, density_multiplier, s, err)) {
      set_error("CalculateGeometryScales: " + err);
      return SHB_ERR_INVALID_ARG;
    }
    if (!s.empty()) std::memcpy(scales_out, s.data(), sizeof(float) * s.size());
    return SHB_OK;
  });
}

shb_status shb_create_atlas(const shb_scene_desc* scene, uint32_t target_resolution, uint32_t padding,
                            float density_multiplier, shb_host_scene** out, int32_t* width, int32_t* height) {
  return ::shb::guarded("shb_create_atlas", [&]() -> shb_status {
    if (!scene || !out) {
      set_error("NULL argument");
      return SHB_ERR_INVALID_ARG;
    }
    *out = nullptr;
    auto fail = [](const std::string& m) {
      set_error("CreateAtlasGeometries: " + m);
      return SHB_ERR_INVALID_ARG;
    };
    if (scene->geometry_count == 0 || !scene->geometries) return fail("no geometries");
    if (target_resolution == 0 || target_resolution > 65536 || padding > 65536)
      return fail("target_resolution must be 1..65536 and padding at most 65536");
    std::vector<float> scales;
    std::string err;
    if (!geometry_scales(scene, density_multiplier, scales, err)) return fail(err);
    const uint32_t ng = scene->geometry_count;
    for (uint32_t g = 0; g < ng; ++g) {
      const shb_geometry_desc& G = scene->geometries[g];
      if (!G.vertices || !G.normals || !G.tangents)
        return fail("geometry " + std::to_string(g) + ": vertices, normals and tangents required");
      if (G.index_count && !G.indices) return fail("geometry " + std::to_string(g) + ": indices is NULL");
      for (uint32_t i = 0; i < G.index_count / 3 * 3; ++i)
        if (G.indices[i] >= G.vertex_count) return fail("geometry " + std::to_string(g) + ": index out of range");
      // a scale of zero (an albedo of 0 texels) would collapse every chart
      if (!(scales[g] >= kMinScale)) scales[g] = kMinScale;
    }
    // charts, geometries in parallel
    std::vector<GeoCharts> gc(ng);
    {
      std::atomic<uint32_t> next{0};
      auto work = [&] {
        for (uint32_t g; (g = next.fetch_add(1)) < ng;) build_charts(scene->geometries[g], scales[g], gc[g]);
      };
      ::shb::run_host_threads(std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), ng)), work);
    }
    std::vector<Rect> rects;
    double sum_area = 0;
    for (uint32_t g = 0; g < ng; ++g)
      for (uint32_t c = 0; c < gc[g].charts.size(); ++c) {
        const Chart& ch = gc[g].charts[c];
        rects.push_back(Rect{g, c, ch.w, ch.h});
        sum_area += ch.w * ch.h;
      }
    const int W = (int)target_resolution, H = (int)target_resolution, pad = (int)padding;
    double s = 1.0;
    if (!rects.empty()) {
      // texels per unit: the largest that fits, by bisection (area bound above)
      double hi = sum_area > 0 ? std::sqrt((double)W * H / sum_area) : 1.0;
      double lo = hi;
      bool fits = false;
      for (int i = 0; i < 64 && !fits; ++i) {
        lo *= 0.5;
        fits = pack(rects, lo, W, H, pad, nullptr);
        if (!fits) {
          bool all_unit = true;
          for (const Rect& r : rects) all_unit = all_unit && foot(r.w, lo) == 1 && foot(r.h, lo) == 1;
          if (all_unit) break;  // every chart is one texel: smaller scales cannot help
        }
      }
      if (!fits)
        return fail("could not fit " + std::to_string(rects.size()) + " charts into one " + std::to_string(W) + "x" +
                    std::to_string(H) + " atlas with padding " + std::to_string(pad));
      if (sum_area > 0)
        for (int i = 0; i < 30; ++i) {
          const double mid = 0.5 * (lo + hi);
          if (pack(rects, mid, W, H, pad, nullptr)) lo = mid;
          else hi = mid;
        }
      s = lo;
      std::vector<std::array<int, 3>> place;
      pack(rects, s, W, H, pad, &place);
      for (size_t i = 0; i < rects.size(); ++i) {
        Chart& ch = gc[rects[i].geo].charts[rects[i].chart];
        ch.ox = place[i][0];
        ch.oy = place[i][1];
        ch.turned = place[i][2] != 0;
      }
    }
    std::unique_ptr<shb_host_scene> hs(new shb_host_scene());
    hs->geos.resize(ng);
    for (uint32_t g = 0; g < ng; ++g) {
      const shb_geometry_desc& G = scene->geometries[g];
      shb_host_scene::Geo& o = hs->geos[g];
      o.material = G.material_id;
      std::memcpy(o.transform, G.transform, sizeof(o.transform));
      const uint32_t nf = G.index_count / 3;
      std::unordered_map<uint64_t, uint32_t> vmap;
      o.idx.resize(3 * (size_t)nf);
      for (uint32_t f = 0; f < nf; ++f) {
        const uint32_t c = gc[g].chart_of[f];
        const Chart& ch = gc[g].charts[c];
        const double fw = foot(ch.w, s), fh = foot(ch.h, s);
        for (int k = 0; k < 3; ++k) {
          const uint32_t v = G.indices[3 * f + k];
          auto it = vmap.emplace(((uint64_t)c << 32) | v, (uint32_t)(o.v.size() / 3));
          if (it.second) {
            for (int a = 0; a < 3; ++a) {
              o.v.push_back(G.vertices[3 * v + a]);
              o.n.push_back(G.normals[3 * v + a]);
            }
            for (int a = 0; a < 4; ++a) o.t.push_back(G.tangents[4 * v + a]);
            for (int a = 0; a < 2; ++a) o.uv0.push_back(G.texture_uvs[2 * v + a]);
            // texel position: chart centred in its footprint
            const D2 q = ch.corner[3 * (size_t)gc[g].slot_of[f] + k];
            double x = q.x * s + 0.5 * (fw - ch.w * s), y = q.y * s + 0.5 * (fh - ch.h * s);
            if (ch.turned) {  // quarter turn inside the placed footprint: (x, y) -> (fh - y, x)
              const double t = x;
              x = fh - y;
              y = t;
            }
            const float u = (float)((ch.ox + x) / W), w = (float)((ch.oy + y) / H);
            o.uv1.push_back(std::min(1.0f, std::max(0.0f, u)));
            o.uv1.push_back(std::min(1.0f, std::max(0.0f, w)));
          }
          o.idx[3 * (size_t)f + k] = it.first->second;
        }
      }
    }
    for (uint32_t m = 0; m < scene->material_count; ++m) {
      const shb_material_desc& M = scene->materials[m];
      shb_host_scene::Mat mt;
      mt.w = M.albedo_width;
      mt.h = M.albedo_height;
      mt.c = M.albedo_channels;
      mt.emission = M.emission_intensity;
      if (M.albedo_pixels) mt.px.assign(M.albedo_pixels, M.albedo_pixels + (size_t)mt.w * mt.h * mt.c);
      hs->mats.push_back(std::move(mt));
    }
    if (scene->light_count && scene->lights) hs->lights.assign(scene->lights, scene->lights + scene->light_count);
    hs->finish();
    if (width) *width = W;
    if (height) *height = H;
    *out = hs.release();
    return SHB_OK;
  });
}

}  // extern "C"
