// batch.cu - shb_bake_batch: many bakes run through one shared sequence of
// wavefront launches, and the autotuner that picks its launch structure per
// shape class.
//
// The bakes' valid texels are cut into work tiles of whole texels, and the
// tiles packed into waves of paths on the host (shade.cu plan_waves): a
// bake large enough to fill waves gets waves of its own, smaller bakes share
// waves, so the per-depth traversal and shading launches of one wave carry
// paths of several bakes.  The whole sequence can be captured in one CUDA
// graph.
//
// The tuned parameters are the queue depth (paths per wave), the size below
// which bakes share waves (larger bakes get waves of their own), the
// work-tile size (texels per tile) and the traversal grid (a multiple of
// SMs x resident blocks).  A shape class is (bake count, total paths, max
// bounces, mean triangles, max lights), each bucketed by powers of two.
// Tuning is a coordinate descent over those four parameters, each candidate
// timed with CUDA events on the whole batch (sample counts thinned evenly
// when the batch holds more than 2^30 paths); the fastest per path is
// appended as "<gpu>|v2|<class> wave tile grid share ms" to the tuning file so
// later batches of the same class skip the search.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "shb_internal.h"

namespace shb {
namespace {

int log2_bucket(double x) { return x <= 1.0 ? 0 : (int)std::floor(std::log2(x) + 0.5); }

std::string shape_class(const std::vector<BakeSpec>& specs) {
  double paths = 0, tris = 0;
  int max_b = 0;
  uint32_t max_l = 0;
  for (const BakeSpec& s : specs) {
    paths += (double)s.W * s.H * s.cfg.samples;
    tris += s.scene->prim_count;
    max_b = std::max(max_b, s.cfg.bounces);
    max_l = std::max(max_l, s.scene->light_count);
  }
  std::ostringstream os;
  os << "n" << log2_bucket((double)specs.size()) << "-p" << log2_bucket(paths) << "-b" << max_b << "-t"
     << log2_bucket(tris / std::max<size_t>(1, specs.size())) << "-l" << log2_bucket(max_l);
  return os.str();
}

std::string tune_path(const char* opt) {
  if (opt && *opt) return opt;
  if (const char* e = std::getenv("SHB_TUNE_CACHE")) return e;
  const char* home = std::getenv("HOME");
  std::string dir = std::string(home ? home : "/tmp") + "/.cache/sh_baker_b200";
  mkdir((std::string(home ? home : "/tmp") + "/.cache").c_str(), 0755);
  mkdir(dir.c_str(), 0755);
  return dir + "/autotune.txt";
}

std::string device_name(int dev) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return "unknown";
  std::string n = p.name;
  for (char& ch : n)
    if (ch == ' ' || ch == '|') ch = '_';
  return n;
}

bool lookup(const std::string& file, const std::string& key, BatchParams* out) {
  std::ifstream in(file);
  std::string line;
  bool found = false;
  while (std::getline(in, line)) {
    std::istringstream is(line);
    std::string k;
    long long wave = 0, tile = 0, share = 0;
    int grid = 0;
    double ms = 0;
    if (!(is >> k >> wave >> tile >> grid >> share >> ms)) continue;
    if (k == key && wave > 0 && tile > 0 && grid > 0 && share >= 0) {
      out->wave_paths = wave;
      out->tile_texels = tile;
      out->grid_scale = grid;
      out->share_paths = share;
      found = true;  // the last entry wins
    }
  }
  return found;
}

shb_status time_batch(shb_context* c, const std::vector<BakeSpec>& specs, const BatchParams& p, double* ms) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, c->stream);
  shb_status st = bake_batch_device(c, specs, p, nullptr);
  cudaEventRecord(b, c->stream);
  cudaEventSynchronize(b);
  float f = 0.f;
  cudaEventElapsedTime(&f, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = f;
  return st;
}

// Coordinate descent from the defaults: queue depth, then the sharing
// threshold, then the tile size, then the traversal grid, keeping the best
// of each sweep.  The probe is the whole batch, with every bake's sample
// count scaled by the same factor when the batch holds more than 2^30 paths.
shb_status tune(shb_context* c, const std::vector<BakeSpec>& specs, BatchParams* best, double* best_cost) {
  std::vector<BakeSpec> probe = specs;
  double paths = 0;
  for (const BakeSpec& s : probe) paths += (double)s.W * s.H * s.cfg.samples;
  if (paths > double(1 << 30)) {
    const double f = double(1 << 30) / paths;
    paths = 0;
    for (BakeSpec& s : probe) {
      s.cfg.samples = std::max(1, (int)(s.cfg.samples * f));
      paths += (double)s.W * s.H * s.cfg.samples;
    }
  }
  BatchParams cur;
  cur.tile_texels = int64_t(1) << 13;
  double ms = 0;
  {  // the first run pays allocation of the largest wave buffers
    BatchParams w = cur;
    w.wave_paths = int64_t(1) << 24;
    SHB_TRY(time_batch(c, probe, w, &ms));
  }
  *best_cost = 1e300;
  auto trial = [&](const BatchParams& p) -> shb_status {
    SHB_TRY(time_batch(c, probe, p, &ms));
    const double cost = ms / std::max(paths, 1.0) * 1e6;  // ms per million paths
    if (cost < *best_cost) {
      *best_cost = cost;
      *best = p;
    }
    return SHB_OK;
  };
  SHB_TRY(trial(cur));
  for (int64_t w : {int64_t(1) << 22, int64_t(1) << 24}) {
    BatchParams p = cur;
    p.wave_paths = w;
    SHB_TRY(trial(p));
  }
  cur = *best;
  for (int64_t sh : {int64_t(0), cur.wave_paths / 8, int64_t(1) << 40}) {
    BatchParams p = cur;
    p.share_paths = sh;
    SHB_TRY(trial(p));
  }
  cur = *best;
  {
    BatchParams p = cur;
    p.tile_texels = int64_t(1) << 30;
    SHB_TRY(trial(p));
  }
  cur = *best;
  {
    BatchParams p = cur;
    p.grid_scale = 2;
    SHB_TRY(trial(p));
  }
  if (best->share_paths < 0) best->share_paths = best->wave_paths / 2;
  return SHB_OK;
}

}  // namespace
}  // namespace shb

using namespace shb;

extern "C" shb_status shb_bake_batch(shb_context* ctx, const shb_batch_item* items, int32_t count,
                                     const shb_batch_options* options, shb_bake_stats* stats) {
  return ::shb::guarded("shb_bake_batch", [&]() -> shb_status {
    if (!ctx || (count > 0 && !items)) {
      set_error("NULL argument");
      return SHB_ERR_INVALID_ARG;
    }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (count <= 0) return SHB_OK;
    SHB_ON_DEVICE(ctx->device);
    std::vector<BakeSpec> specs;
    specs.reserve(count);
    for (int i = 0; i < count; ++i) {
      const shb_batch_item& it = items[i];
      std::string where = "batch item " + std::to_string(i) + ": ";
      if (!it.scene || !it.gbuffer || !it.sh || !it.env_visibility) {
        set_error(where + "NULL scene, gbuffer or output");
        return SHB_ERR_INVALID_ARG;
      }
      if (it.scene->ctx != ctx || it.gbuffer->ctx != ctx) {
        set_error(where + "scene and G-buffer must belong to the context");
        return SHB_ERR_INVALID_ARG;
      }
      const shb_bake_config& cfg = it.config;
      if (cfg.samples <= 0 || cfg.bounces < 0 || cfg.bounces > 30 || cfg.num_light_samples <= 0 ||
          cfg.rng_mode != SHB_RNG_PHILOX) {
        set_error(where + "bad bake config");
        return SHB_ERR_INVALID_ARG;
      }
      int64_t W = (int64_t)it.raster.width * it.raster.supersample_scale;
      int64_t H = (int64_t)it.raster.height * it.raster.supersample_scale;
      if (W != it.gbuffer->width || H != it.gbuffer->height) {
        set_error(where + "G-buffer size does not match raster config");
        return SHB_ERR_INVALID_ARG;
      }
      if (it.scene->bvh_depth > 64) {
        set_error(where + "BVH deeper than the traversal stack");
        return SHB_ERR_INVALID_ARG;
      }
      specs.push_back(BakeSpec{it.scene, it.gbuffer->points.as<shb_surface_point>(), (int)W, (int)H, cfg, it.sh,
                               it.env_visibility});
    }
    BatchParams prm;
    prm.use_graph = options && options->use_graph;
    // defaults for batches: tiles of 8192 texels so that bakes mix in a wave
    prm.tile_texels = int64_t(1) << 13;
    if (options && options->autotune) {
      const std::string file = tune_path(options->tune_cache);
      const std::string key = device_name(ctx->device) + "|v2|" + shape_class(specs);
      if (!lookup(file, key, &prm)) {
        double cost = 0;
        BatchParams best;
        SHB_TRY(tune(ctx, specs, &best, &cost));
        prm.wave_paths = best.wave_paths;
        prm.tile_texels = best.tile_texels;
        prm.grid_scale = best.grid_scale;
        prm.share_paths = best.share_paths;
        std::ofstream out(file, std::ios::app);
        out << key << " " << prm.wave_paths << " " << prm.tile_texels << " " << prm.grid_scale << " "
            << prm.share_paths << " " << cost << "\n";
      }
    }
    if (options && options->wave_paths > 0) prm.wave_paths = options->wave_paths;
    if (options && options->tile_texels > 0) prm.tile_texels = options->tile_texels;
    if (options && options->grid_scale > 0) prm.grid_scale = options->grid_scale;
    if (options && options->share_paths > 0) prm.share_paths = options->share_paths;
    if (options && options->share_paths < 0) prm.share_paths = 0;
    if (options && options->nee_split >= 0 && options->nee_split <= 2) prm.nee_split = options->nee_split;
    if (options && options->max_traversal_steps < 0) {
      set_error("max_traversal_steps must not be negative");
      return SHB_ERR_INVALID_ARG;
    }
    if (options && options->queue_capacity < 0) {
      set_error("queue_capacity must not be negative");
      return SHB_ERR_INVALID_ARG;
    }
    if (options) prm.max_iters = (uint32_t)options->max_traversal_steps;
    if (options) prm.queue_cap = options->queue_capacity;
    uint64_t l0 = ctx->launches;
    SHB_TRY(bake_batch_device(ctx, specs, prm, stats));
    if (stats) stats->kernel_launches = ctx->launches - l0;
    return SHB_OK;
  });
}
