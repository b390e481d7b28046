// autotune.cc -- picks d, the lane-to-rank mapping and CTAs per SM of the
// Hogwild epoch by timing candidate configurations on the caller's data.
//
// No reference counterpart (the reference takes d from --tasks-per-rank).
// For each candidate the data is blocked for that d, `epochs` epochs run after
// one warm-up epoch, and the median device time of an epoch is kept.  The
// factors are reset to the caller's for every candidate, so tuning does not
// advance the run.  Candidates that fail to build (unsupported shape, out of
// memory) are skipped.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/dsgdpp.h"

namespace {

struct Shape {
  uint32_t lanes, vecs, ctas;
};

double time_config(const dsgdpp_config& cfg, uint64_t nnz, const uint32_t* rows,
                   const uint32_t* cols, const double* vals, const double* W, const double* H,
                   uint32_t epochs, double eps) {
  dsgdpp_ctx* ctx = nullptr;
  if (dsgdpp_create(&cfg, &ctx) != DSGDPP_OK) return -1;
  double best = -1;
  if (dsgdpp_set_matrix(ctx, DSGDPP_TRAIN, nnz, rows, cols, vals) == DSGDPP_OK &&
      dsgdpp_set_factors(ctx, W, H) == DSGDPP_OK && dsgdpp_seed(ctx, 1) == DSGDPP_OK &&
      dsgdpp_epoch(ctx, eps) == DSGDPP_OK) {
    std::vector<double> ms;
    for (uint32_t e = 0; e < epochs; ++e) {
      double t = 0;
      if (dsgdpp_epoch(ctx, eps) != DSGDPP_OK || dsgdpp_last_epoch_ms(ctx, &t) != DSGDPP_OK) {
        ms.clear();
        break;
      }
      ms.push_back(t);
    }
    if (!ms.empty()) {
      std::sort(ms.begin(), ms.end());
      best = ms[ms.size() / 2];
    }
  }
  dsgdpp_destroy(ctx);
  return best;
}

}  // namespace

extern "C" int dsgdpp_autotune(const dsgdpp_config* base, uint64_t nnz, const uint32_t* rows,
                               const uint32_t* cols, const double* vals, const double* W,
                               const double* H, const uint32_t* d_candidates, uint32_t nd,
                               uint32_t epochs, double eps, dsgdpp_config* best,
                               double* best_ms) {
  if (!base || !best || !rows || !cols || !vals || !W || !H || epochs == 0)
    return DSGDPP_E_INVALID;
  if (base->exec != DSGDPP_EXEC_HOGWILD) return DSGDPP_E_UNSUPPORTED;
  std::vector<uint32_t> ds(d_candidates, d_candidates + nd);
  if (ds.empty()) ds = {64, 128, 256, 512};
  // lane mappings: the automatic one, and the other of (one vector per lane,
  // two vectors per lane on half the lanes)
  const std::vector<Shape> shapes = {{0, 0, 0}, {0, 0, 4}, {0, 0, 3}};
  double top = -1;
  dsgdpp_config chosen = *base;
  for (uint32_t d : ds) {
    for (const Shape& sh : shapes) {
      dsgdpp_config c = *base;
      c.d = d;
      c.lanes_per_nnz = sh.lanes;
      c.vecs_per_lane = sh.vecs;
      c.ctas_per_sm = sh.ctas;
      const double t = time_config(c, nnz, rows, cols, vals, W, H, epochs, eps);
      if (t > 0 && (top < 0 || t < top)) {
        top = t;
        chosen = c;
      }
    }
    // the alternative lane mapping at this d
    dsgdpp_config c = *base;
    c.d = d;
    dsgdpp_ctx* probe = nullptr;
    if (dsgdpp_create(&c, &probe) == DSGDPP_OK) {
      uint32_t lanes = 0, vecs = 0, grid = 0;
      dsgdpp_launch_shape(probe, &lanes, &vecs, &grid);
      dsgdpp_destroy(probe);
      // the other mapping: back to one vector per lane where the automatic
      // one takes two, else half the lanes with twice the vectors
      const bool wide = vecs == 2 && lanes <= 16;
      if (wide || lanes >= 4) {
        c.lanes_per_nnz = wide ? lanes * 2 : lanes / 2;
        c.vecs_per_lane = wide ? 1 : vecs * 2;
        const double t = time_config(c, nnz, rows, cols, vals, W, H, epochs, eps);
        if (t > 0 && (top < 0 || t < top)) {
          top = t;
          chosen = c;
        }
      }
    }
  }
  if (top < 0) return DSGDPP_E_UNSUPPORTED;
  *best = chosen;
  if (best_ms) *best_ms = top;
  return DSGDPP_OK;
}
