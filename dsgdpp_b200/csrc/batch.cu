// batch.cu -- many independent DSGD++ factorizations advanced together.
//
// No reference counterpart: the reference runs one factorization per job.
// Problems are grouped by padded rank (their factor rows have the same width);
// each group keeps all its problems' entries, factors and inverse counts in
// shared buffers, indices shifted so one kernel addresses all of them.  An
// epoch of every problem is one sequence of Hogwild launches: launch (group,
// s) works on the union of sub-epoch s of every problem of the group that has
// one (problems with a smaller d simply drop out of later launches); each
// segment carries its problem's step size and lazy-L2 scales.  The launch
// tables keep their shape from epoch to epoch, so the whole epoch is captured
// once as a CUDA graph and replayed with new table contents.  BoldDriver runs
// per problem on per-problem training losses, computed by a deterministic
// segmented reduction (fixed-size chunks, then one CTA per problem).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <new>
#include <string>
#include <vector>

#include "../../include/dsgdpp.h"
#include "context.h"
#include "kernels.cuh"
#include "schedule.h"

using namespace dsgdpp;

namespace {

constexpr uint64_t kLossChunk = 16384;  // entries or factor elements per reduction chunk
constexpr uint32_t kSmemSegs = 256;     // largest launch table staged in shared memory

struct Problem {
  uint64_t m = 0, n = 0;
  uint32_t r = 0, d = 0, group = 0;
  uint64_t w0 = 0, h0 = 0;          // first W / H row in the group buffers
  uint64_t nnz = 0, tnnz = 0;
  std::vector<uint64_t> block_ptr;  // d * 2d + 1, group-wide entry offsets
  uint64_t trec0 = 0;               // first test entry in the group test arrays
  Random32 master{0};
  double eps = 0, prev = 0, cur = 0, test = 0;
  uint32_t wslot = 0, hslot0 = 0;   // lazy-L2 scale slots of W and the 2d H blocks
  uint32_t nchunk_begin = 0, tchunk_begin = 0, wchunk_begin = 0, hchunk_begin = 0;
};

struct Group {
  uint32_t rp = 0, lanes = 0, vecs = 0, grid = 0;
  uint32_t smem_segs = 0;  // > 0: the launch tables are staged in shared memory
  std::vector<uint32_t> probs;
  uint64_t wrows = 0, hrows = 0, nnz = 0, tnnz = 0;
  void* W = nullptr;
  void* H = nullptr;
  void* inv1 = nullptr;
  void* inv2 = nullptr;
  uint32_t* row = nullptr;
  uint32_t* col = nullptr;
  void* val = nullptr;
  uint32_t* trow = nullptr;
  uint32_t* tcol = nullptr;
  void* tval = nullptr;
  uint32_t* w_slot = nullptr;  // per W row: its scale slot
  uint32_t* h_slot = nullptr;  // per H row
  uint32_t nslots = 0;
  float* d_scales = nullptr;
  float* h_scales = nullptr;
  uint32_t launch0 = 0, nlaunch = 0;  // this group's launches in the epoch
  // segmented loss reductions: chunk tables and per-problem chunk ranges
  RangeChunk* d_nchunks = nullptr;
  RangeChunk* d_tchunks = nullptr;
  RangeChunk* d_wchunks = nullptr;
  RangeChunk* d_hchunks = nullptr;
  uint32_t nn = 0, nt = 0, nw = 0, nh = 0;
  uint32_t* d_nown = nullptr;  // per problem of the group: first chunk (+1 sentinel)
  uint32_t* d_town = nullptr;
  uint32_t* d_wown = nullptr;
  uint32_t* d_hown = nullptr;
};

}  // namespace

struct dsgdpp_batch {
  dsgdpp_config cfg{};
  int layout_key = 0;  // kLayout* shared by every problem (a launch has one kernel)
  std::string err;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  std::vector<Problem> probs;
  std::vector<Group> groups;
  // epoch tables
  std::vector<LaunchDesc> launches;  // host copy (shapes fixed)
  LaunchDesc* d_launches = nullptr;
  Segment* h_segs = nullptr;
  Segment* d_segs = nullptr;
  uint64_t nsegs = 0;
  uint32_t* d_counters = nullptr;
  EpochParams* h_params = nullptr;
  EpochParams* d_params = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // loss scratch
  double* d_partials = nullptr;
  double* d_losses = nullptr;   // per problem: nzsl, test nzsl, |W|^2, |H|^2
  double* h_losses = nullptr;
  uint32_t max_chunks = 0;
  uint32_t epoch_counter = 0;
  double epoch_ms = 0;
};

namespace {

void free_group(Group& g) {
  for (void* p : {g.W, g.H, g.inv1, g.inv2, (void*)g.row, (void*)g.col, g.val, (void*)g.trow,
                  (void*)g.tcol, g.tval, (void*)g.w_slot, (void*)g.h_slot, (void*)g.d_scales,
                  (void*)g.d_nchunks, (void*)g.d_tchunks, (void*)g.d_wchunks, (void*)g.d_hchunks,
                  (void*)g.d_nown, (void*)g.d_town, (void*)g.d_wown, (void*)g.d_hown})
    if (p) cudaFree(p);
  if (g.h_scales) cudaFreeHost(g.h_scales);
  g = Group{};
}

void destroy_impl(dsgdpp_batch* b) {
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (auto& g : b->groups) free_group(g);
  for (void* p : {(void*)b->d_launches, (void*)b->d_segs, (void*)b->d_counters,
                  (void*)b->d_params, (void*)b->d_partials, (void*)b->d_losses})
    if (p) cudaFree(p);
  for (void* p : {(void*)b->h_segs, (void*)b->h_params, (void*)b->h_losses})
    if (p) cudaFreeHost(p);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
}

// d of a problem: the largest d <= 16 with at least ~2048 entries per block of
// a sub-epoch on average, within the blocking's limits (d <= m, 2d <= n)
uint32_t choose_d(uint64_t m, uint64_t n, uint64_t nnz, uint32_t dmax) {
  uint32_t d = 1;
  while (2 * d <= dmax && nnz / (2ull * (2 * d) * (2 * d)) >= 2048 && 2 * d <= m && 4 * d <= n)
    d *= 2;
  return d;
}

template <typename T>
T* dnew(size_t count, const char* what) {
  return dalloc<T>(count, what);
}

std::vector<RangeChunk> chunk_ranges(const std::vector<std::pair<uint64_t, uint64_t>>& ranges,
                                     std::vector<uint32_t>& owner_begin) {
  std::vector<RangeChunk> out;
  owner_begin.clear();
  for (const auto& rg : ranges) {
    owner_begin.push_back((uint32_t)out.size());
    for (uint64_t a = rg.first; a < rg.second; a += kLossChunk)
      out.push_back(RangeChunk{a, std::min(rg.second, a + kLossChunk)});
  }
  owner_begin.push_back((uint32_t)out.size());
  return out;
}

template <typename T>
void upload(T*& dst, const std::vector<T>& v, const char* what) {
  dst = dnew<T>(std::max<size_t>(v.size(), 1), what);
  if (!v.empty())
    check_cuda(cudaMemcpy(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), what);
}

void create_impl(dsgdpp_batch* b, const dsgdpp_config* common, uint32_t count,
                 const dsgdpp_problem* ps) {
  if (!common || !ps || count == 0) throw Error(DSGDPP_E_INVALID, "no problems");
  if (common->exec != DSGDPP_EXEC_HOGWILD)
    throw Error(DSGDPP_E_UNSUPPORTED, "the batched form runs the Hogwild path");
  if (common->truncate) throw Error(DSGDPP_E_UNSUPPORTED, "the batched form does not truncate");
  if (common->method != DSGDPP_METHOD_DSGDPP)
    throw Error(DSGDPP_E_UNSUPPORTED, "the batched form runs DSGD++ (d x 2d blocks)");
  if (common->loss == DSGDPP_LOSS_NZSL_NZL2)
    throw Error(DSGDPP_E_UNSUPPORTED, "the batched form computes the Nzsl and Nzsl_L2 losses");
  b->cfg = *common;
  // one record order for all problems: the automatic choice is column runs
  if (b->cfg.layout == DSGDPP_LAYOUT_RUNS) b->cfg.layout = DSGDPP_LAYOUT_COL_RUNS;
  b->layout_key = b->cfg.layout == DSGDPP_LAYOUT_COL_RUNS   ? kLayoutColRuns
                  : b->cfg.layout == DSGDPP_LAYOUT_ROW_RUNS ? kLayoutRowRuns
                                                            : kLayoutShuffled;
  check_cuda(cudaSetDevice(common->device), "cudaSetDevice");
  check_cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
  check_cuda(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, common->device),
             "attribute");
  const int prec = common->precision;
  const uint32_t vw = prec == kFp64 ? 2 : (prec == kFp32 ? 4 : 8);
  const size_t es = prec == kFp64 ? 8 : (prec == kFp32 ? 4 : 2);
  const size_t vs = prec == kFp64 ? 8 : 4;  // entry value / inverse count size
  b->probs.resize(count);
  // groups by padded rank
  for (uint32_t p = 0; p < count; ++p) {
    const auto& q = ps[p];
    if (q.m == 0 || q.n < 2 || q.rank == 0 || !q.W || !q.H || (q.nnz && (!q.rows || !q.cols || !q.vals)))
      throw Error(DSGDPP_E_INVALID, "problem " + std::to_string(p) + " is malformed");
    Problem& P = b->probs[p];
    P.m = q.m; P.n = q.n; P.r = q.rank;
    P.d = q.d ? q.d : choose_d(q.m, q.n, q.nnz, 16);
    if (P.d > P.m || 2 * P.d > P.n) throw Error(DSGDPP_E_INVALID, "problem d too large");
    const uint32_t rp = (q.rank + vw - 1) / vw * vw;
    uint32_t gi = 0;
    for (; gi < b->groups.size(); ++gi)
      if (b->groups[gi].rp == rp) break;
    if (gi == b->groups.size()) {
      b->groups.emplace_back();
      b->groups.back().rp = rp;
    }
    P.group = gi;
    b->groups[gi].probs.push_back(p);
    P.master.seed_with(q.seed);
    P.eps = q.eps0;
  }
  // per group: gather every problem's blocked entries through a per-problem context
  for (uint32_t gi = 0; gi < b->groups.size(); ++gi) {
    Group& G = b->groups[gi];
    for (uint32_t p : G.probs) {
      Problem& P = b->probs[p];
      P.w0 = G.wrows; P.h0 = G.hrows;
      G.wrows += P.m; G.hrows += P.n;
      P.nnz = ps[p].nnz; P.tnnz = ps[p].nnz_test;
      G.nnz += P.nnz; G.tnnz += P.tnnz;
    }
    if (G.wrows > 0xFFFFFFFFull || G.hrows > 0xFFFFFFFFull)
      throw Error(DSGDPP_E_INVALID, "a rank group's rows must fit in 32 bits");
    G.W = dnew<unsigned char>(G.wrows * G.rp * es, "W");
    G.H = dnew<unsigned char>(G.hrows * G.rp * es, "H");
    G.inv1 = dnew<unsigned char>(G.wrows * vs, "inv1");
    G.inv2 = dnew<unsigned char>(G.hrows * vs, "inv2");
    G.row = dnew<uint32_t>(G.nnz, "rows");
    G.col = dnew<uint32_t>(G.nnz, "cols");
    G.val = dnew<unsigned char>(std::max<uint64_t>(G.nnz, 1) * vs, "vals");
    G.trow = dnew<uint32_t>(G.tnnz, "test rows");
    G.tcol = dnew<uint32_t>(G.tnnz, "test cols");
    G.tval = dnew<unsigned char>(std::max<uint64_t>(G.tnnz, 1) * vs, "test vals");
    uint64_t rec = 0, trec = 0;
    for (uint32_t p : G.probs) {
      Problem& P = b->probs[p];
      const auto& q = ps[p];
      dsgdpp_config c = b->cfg;
      c.m = P.m; c.n = P.n; c.rank = P.r; c.d = P.d;
      c.launch = DSGDPP_LAUNCH_STREAM;
      dsgdpp_ctx* ctx = nullptr;
      int rc = dsgdpp_create(&c, &ctx);
      if (rc != DSGDPP_OK)
        throw Error(rc, "problem " + std::to_string(p) + ": " + dsgdpp_create_error());
      struct Guard { dsgdpp_ctx* c; ~Guard() { dsgdpp_destroy(c); } } guard{ctx};
      if ((rc = dsgdpp_set_matrix(ctx, DSGDPP_TRAIN, q.nnz, q.rows, q.cols, q.vals)) != DSGDPP_OK ||
          (q.nnz_test &&
           (rc = dsgdpp_set_matrix(ctx, DSGDPP_TEST, q.nnz_test, q.trows, q.tcols, q.tvals)) !=
               DSGDPP_OK) ||
          (rc = dsgdpp_set_factors(ctx, q.W, q.H)) != DSGDPP_OK)
        throw Error(rc, "problem " + std::to_string(p) + ": " + dsgdpp_last_error(ctx));
      if ((rc = dsgdpp_sync(ctx)) != DSGDPP_OK) throw Error(rc, dsgdpp_last_error(ctx));
      const DevMatrix& M = ctx->mat[0];
      const DevMatrix& T = ctx->mat[1];
      P.nnz = M.nnz;
      P.tnnz = T.nnz;
      check_cuda(launch_offset_copy(M.row, M.col, M.nnz, (uint32_t)P.w0, (uint32_t)P.h0,
                                    G.row + rec, G.col + rec, b->stream), "entries");
      check_cuda(cudaMemcpyAsync((unsigned char*)G.val + rec * vs, M.val, M.nnz * vs,
                                 cudaMemcpyDeviceToDevice, b->stream), "values");
      if (T.nnz) {
        check_cuda(launch_offset_copy(T.row, T.col, T.nnz, (uint32_t)P.w0, (uint32_t)P.h0,
                                      G.trow + trec, G.tcol + trec, b->stream), "test entries");
        check_cuda(cudaMemcpyAsync((unsigned char*)G.tval + trec * vs, T.val, T.nnz * vs,
                                   cudaMemcpyDeviceToDevice, b->stream), "test values");
      }
      check_cuda(cudaMemcpyAsync((unsigned char*)G.inv1 + P.w0 * vs, ctx->inv1, P.m * vs,
                                 cudaMemcpyDeviceToDevice, b->stream), "inv1");
      check_cuda(cudaMemcpyAsync((unsigned char*)G.inv2 + P.h0 * vs, ctx->inv2, P.n * vs,
                                 cudaMemcpyDeviceToDevice, b->stream), "inv2");
      check_cuda(cudaMemcpyAsync((unsigned char*)G.W + P.w0 * G.rp * es, ctx->W, P.m * G.rp * es,
                                 cudaMemcpyDeviceToDevice, b->stream), "W");
      check_cuda(cudaMemcpyAsync((unsigned char*)G.H + P.h0 * G.rp * es, ctx->H, P.n * G.rp * es,
                                 cudaMemcpyDeviceToDevice, b->stream), "H");
      P.block_ptr = M.h_block_ptr;
      for (auto& v : P.block_ptr) v += rec;
      P.trec0 = trec;
      rec += M.nnz;
      trec += T.nnz;
      check_cuda(cudaStreamSynchronize(b->stream), "sync");
    }
    G.nnz = rec;
    G.tnnz = trec;
    // lazy-L2 scale slots: one per problem for W, one per H column block
    std::vector<uint32_t> wslot(G.wrows), hslot(G.hrows);
    uint32_t slot = 0;
    for (uint32_t p : G.probs) {
      Problem& P = b->probs[p];
      P.wslot = slot++;
      P.hslot0 = slot;
      slot += 2 * P.d;
      std::fill(wslot.begin() + P.w0, wslot.begin() + P.w0 + P.m, P.wslot);
      std::vector<uint64_t> off = block_offsets(P.n, 2 * P.d);
      for (uint32_t b2 = 0; b2 < 2 * P.d; ++b2) {
        const uint64_t lo = off[b2], hi = b2 + 1 < 2 * P.d ? off[b2 + 1] : P.n;
        std::fill(hslot.begin() + P.h0 + lo, hslot.begin() + P.h0 + hi, P.hslot0 + b2);
      }
    }
    G.nslots = slot;
    upload(G.w_slot, wslot, "w slots");
    upload(G.h_slot, hslot, "h slots");
    G.d_scales = dnew<float>(G.nslots, "scales");
    G.h_scales = halloc<float>(G.nslots, "scales");
    // loss chunk tables
    std::vector<std::pair<uint64_t, uint64_t>> rn, rt, rw, rh;
    for (uint32_t p : G.probs) {
      const Problem& P = b->probs[p];
      rn.push_back({P.block_ptr.front(), P.block_ptr.back()});
      rt.push_back({P.trec0, P.trec0 + P.tnnz});
      rw.push_back({P.w0 * G.rp, (P.w0 + P.m) * G.rp});
      rh.push_back({P.h0 * G.rp, (P.h0 + P.n) * G.rp});
    }
    std::vector<uint32_t> on, ot, ow, oh;
    auto cn = chunk_ranges(rn, on), ct = chunk_ranges(rt, ot), cw = chunk_ranges(rw, ow),
         ch = chunk_ranges(rh, oh);
    G.nn = (uint32_t)cn.size(); G.nt = (uint32_t)ct.size();
    G.nw = (uint32_t)cw.size(); G.nh = (uint32_t)ch.size();
    upload(G.d_nchunks, cn, "chunks"); upload(G.d_tchunks, ct, "chunks");
    upload(G.d_wchunks, cw, "chunks"); upload(G.d_hchunks, ch, "chunks");
    upload(G.d_nown, on, "owners"); upload(G.d_town, ot, "owners");
    upload(G.d_wown, ow, "owners"); upload(G.d_hown, oh, "owners");
    b->max_chunks = std::max({b->max_chunks, G.nn, G.nt, G.nw, G.nh});
    // launch shape of the group
    const uint32_t nvec = G.rp / vw;
    uint32_t lanes = common->lanes_per_nnz;
    if (!lanes) {
      lanes = 2;
      while (lanes < nvec && lanes < 32) lanes <<= 1;
    }
    uint32_t vecs = common->vecs_per_lane ? common->vecs_per_lane : (nvec + lanes - 1) / lanes;
    if (vecs == 3) vecs = 4;
    G.lanes = lanes;
    G.vecs = vecs;
    if ((uint64_t)lanes * vecs < nvec)
      throw Error(DSGDPP_E_INVALID, "lanes_per_nnz x vecs_per_lane does not cover the rank");
  }
  // launch tables: group by group, sub-epoch by sub-epoch
  uint64_t seg = 0;
  for (uint32_t gi = 0; gi < b->groups.size(); ++gi) {
    Group& G = b->groups[gi];
    uint32_t smax = 0;
    for (uint32_t p : G.probs) smax = std::max(smax, 2 * b->probs[p].d);
    G.launch0 = (uint32_t)b->launches.size();
    G.nlaunch = smax;
    uint32_t most = 0;
    for (uint32_t s = 0; s < smax; ++s) {
      uint32_t nseg = 0;
      for (uint32_t p : G.probs)
        if (s < 2 * b->probs[p].d) nseg += b->probs[p].d;
      b->launches.push_back(LaunchDesc{seg, nseg, (uint32_t)b->launches.size()});
      seg += nseg + 1;
      most = std::max(most, nseg + 1);
    }
    G.smem_segs = most <= kSmemSegs ? most : 0;
    const bool atomic = common->write_mode != DSGDPP_WRITE_STORE;
    int per_sm = hogwild_ctas_per_sm(prec, G.lanes, G.vecs, atomic, G.smem_segs,
                                     b->layout_key != kLayoutShuffled);
    if (per_sm <= 0)
      throw Error(DSGDPP_E_INVALID, "no Hogwild kernel for lanes_per_nnz=" +
                                        std::to_string(G.lanes) + ", vecs_per_lane=" +
                                        std::to_string(G.vecs));
    if (common->ctas_per_sm)  // counted in CTAs of 256 threads
      per_sm = std::min<int>(per_sm, (int)common->ctas_per_sm * hogwild_cta_scale(prec, G.lanes));
    G.grid = (uint32_t)per_sm * (uint32_t)b->num_sms;
  }
  b->nsegs = seg;
  upload(b->d_launches, b->launches, "launches");
  b->h_segs = halloc<Segment>(b->nsegs, "segments");
  b->d_segs = dnew<Segment>(b->nsegs, "segments");
  b->d_counters = dnew<uint32_t>(b->launches.size(), "counters");
  b->h_params = halloc<EpochParams>(1, "params");
  b->d_params = dnew<EpochParams>(1, "params");
  b->d_partials = dnew<double>(std::max<uint32_t>(b->max_chunks, 1), "partials");
  b->d_losses = dnew<double>(4 * (size_t)count, "losses");
  b->h_losses = halloc<double>(4 * (size_t)count, "losses");
  check_cuda(cudaEventCreate(&b->ev0), "event");
  check_cuda(cudaEventCreate(&b->ev1), "event");
}

bool lazy_l2(const dsgdpp_config& c) {
  return c.regularize == DSGDPP_REGULARIZE_L2 && c.regularize_lambda != 0;
}

// host: the epoch's schedules, segment tables and lazy-L2 scales
void fill_tables(dsgdpp_batch* b) {
  const bool l2 = lazy_l2(b->cfg);
  std::vector<uint32_t> sched, seeds;
  std::vector<std::vector<uint32_t>> scheds(b->probs.size());
  uint32_t key0 = 0, key1 = 0;
  for (uint32_t p = 0; p < b->probs.size(); ++p) {
    Problem& P = b->probs[p];
    sched.assign((size_t)2 * P.d * P.d, 0);
    seeds.assign(P.d, 0);
    dsgdpp_schedule(P.master, P.d, b->cfg.stratum_order, sched.data(), seeds.data());
    scheds[p] = sched;
    key0 ^= seeds[0] * 2654435761u + p;
    key1 = key1 * 31u + seeds[P.d - 1];
  }
  for (Group& G : b->groups) {
    // scales: sigma_W(s) = f^s, sigma_H[b2] = f^(earlier visits of b2)
    std::vector<std::vector<double>> sh(G.probs.size());
    std::vector<double> sw(G.probs.size(), 1.0), fac(G.probs.size(), 1.0);
    for (size_t k = 0; k < G.probs.size(); ++k) {
      const Problem& P = b->probs[G.probs[k]];
      sh[k].assign(2 * P.d, 1.0);
      if (l2) {
        double f = 1 - (P.eps / P.d) * 2 * b->cfg.regularize_lambda;
        if (f < 0.5) f = 0.25 / (1 - f);
        fac[k] = f;
      }
    }
    for (uint32_t s = 0; s < G.nlaunch; ++s) {
      const LaunchDesc& L = b->launches[G.launch0 + s];
      Segment* out = b->h_segs + L.seg_begin;
      uint32_t k = 0, chunks = 0;
      for (size_t gp = 0; gp < G.probs.size(); ++gp) {
        const Problem& P = b->probs[G.probs[gp]];
        if (s >= 2 * P.d) continue;
        const uint32_t* S = scheds[G.probs[gp]].data();
        for (uint32_t id = 0; id < P.d; ++id) {
          const uint32_t b2 = S[(size_t)s * P.d + id];
          const uint64_t blk = (uint64_t)id * 2 * P.d + b2;
          Segment g;
          g.rec_begin = P.block_ptr[blk];
          g.count = (uint32_t)(P.block_ptr[blk + 1] - P.block_ptr[blk]);
          g.chunk_begin = chunks;
          chunks += (g.count + kChunk - 1) / kChunk;
          g.cwh = (float)(sw[gp] * sh[gp][b2]);
          g.rho_w = (float)(sh[gp][b2] / sw[gp]);
          g.rho_h = (float)(sw[gp] / sh[gp][b2]);
          g.col_block = b2;
          g.eps = P.eps;
          out[k++] = g;
        }
        sw[gp] *= fac[gp];
        for (uint32_t id = 0; id < P.d; ++id) sh[gp][S[(size_t)s * P.d + id]] *= fac[gp];
      }
      Segment e{};
      e.chunk_begin = chunks;
      out[k] = e;
    }
    for (size_t gp = 0; gp < G.probs.size(); ++gp) {
      const Problem& P = b->probs[G.probs[gp]];
      G.h_scales[P.wslot] = (float)sw[gp];
      for (uint32_t b2 = 0; b2 < 2 * P.d; ++b2) G.h_scales[P.hslot0 + b2] = (float)sh[gp][b2];
    }
  }
  EpochParams ep{};
  ep.eps = 0;  // per segment
  ep.key0 = key0;
  ep.key1 = key1;
  ep.epoch = b->epoch_counter++;
  *b->h_params = ep;
}

void enqueue_epoch(dsgdpp_batch* b) {
  cudaStream_t st = b->stream;
  const bool l2 = lazy_l2(b->cfg);
  check_cuda(cudaMemcpyAsync(b->d_segs, b->h_segs, b->nsegs * sizeof(Segment),
                             cudaMemcpyHostToDevice, st), "segments");
  check_cuda(cudaMemcpyAsync(b->d_params, b->h_params, sizeof(EpochParams), cudaMemcpyHostToDevice,
                             st), "params");
  check_cuda(cudaMemsetAsync(b->d_counters, 0, b->launches.size() * 4, st), "counters");
  for (Group& G : b->groups) {
    if (l2)
      check_cuda(cudaMemcpyAsync(G.d_scales, G.h_scales, G.nslots * 4, cudaMemcpyHostToDevice, st),
                 "scales");
    HogwildArgs a{};
    a.row = G.row; a.col = G.col; a.val = G.val;
    a.inv1 = G.inv1; a.inv2 = G.inv2;
    a.W = G.W; a.H = G.H;
    a.runs = b->layout_key != kLayoutShuffled;
    if (b->layout_key == kLayoutRowRuns) {  // the kernel caches its "H" side: hand it W
      a.row = G.col; a.col = G.row;
      a.inv1 = G.inv2; a.inv2 = G.inv1;
      a.W = G.H; a.H = G.W;
      a.swap_sides = 1;
    }
    a.segs = b->d_segs; a.launches = b->d_launches; a.counters = b->d_counters;
    a.params = b->d_params; a.smem_segs = G.smem_segs;
    a.r = G.rp; a.rp = G.rp;
    a.update = b->cfg.update; a.truncate = 0; a.sgd_order = b->cfg.sgd_order;
    a.atomic = b->cfg.write_mode != DSGDPP_WRITE_STORE;
    a.lambda = b->cfg.update_lambda;
    for (uint32_t s = 0; s < G.nlaunch; ++s)  // a group's launches overlap start and end
      check_cuda(launch_hogwild(b->cfg.precision, G.lanes, G.vecs, a, G.launch0 + s, G.grid, st,
                                s > 0), "batched hogwild");
    if (l2)
      check_cuda(launch_scale_rows(b->cfg.precision, G.W, G.wrows, G.H, G.hrows, G.rp, G.w_slot,
                                   G.h_slot, G.d_scales, st), "scales");
  }
}

void run_epoch(dsgdpp_batch* b) {
  fill_tables(b);
  cudaStream_t st = b->stream;
  check_cuda(cudaEventRecord(b->ev0, st), "event");
  if (b->cfg.launch == DSGDPP_LAUNCH_GRAPH) {
    if (!b->graph) {
      cudaGraph_t g = nullptr;
      check_cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
      try {
        enqueue_epoch(b);
      } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      check_cuda(cudaStreamEndCapture(st, &g), "capture");
      cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      check_cuda(e, "instantiate");
    }
    check_cuda(cudaGraphLaunch(b->graph, st), "graph launch");
  } else {
    enqueue_epoch(b);
  }
  check_cuda(cudaEventRecord(b->ev1, st), "event");
  check_cuda(cudaEventSynchronize(b->ev1), "event sync");  // the host tables are reused
  float ms = 0;
  check_cuda(cudaEventElapsedTime(&ms, b->ev0, b->ev1), "elapsed");
  b->epoch_ms += ms;
}

// per problem: nzsl(train), nzsl(test), |W|^2, |H|^2 into h_losses[4 p + k]
void losses(dsgdpp_batch* b, bool test) {
  cudaStream_t st = b->stream;
  const int prec = b->cfg.precision;
  for (Group& G : b->groups) {
    // the per-problem output slots of this group are gathered through owner
    // tables in group order; write them to a group-local area, then scatter
    const uint32_t np = (uint32_t)G.probs.size();
    double* out = b->d_losses;  // [4][np] for this group, reused per group
    check_cuda(launch_nzsl_chunks(prec, G.d_nchunks, G.nn, G.row, G.col, G.val, G.W, G.H, G.rp,
                                  G.rp, b->d_partials, st), "loss");
    check_cuda(launch_owner_sums(b->d_partials, G.d_nown, np, out, st), "loss");
    if (test) {
      check_cuda(launch_nzsl_chunks(prec, G.d_tchunks, G.nt, G.trow, G.tcol, G.tval, G.W, G.H,
                                    G.rp, G.rp, b->d_partials, st), "test loss");
      check_cuda(launch_owner_sums(b->d_partials, G.d_town, np, out + np, st), "test loss");
    }
    check_cuda(launch_sumsq_chunks(prec, G.d_wchunks, G.nw, G.W, b->d_partials, st), "l2");
    check_cuda(launch_owner_sums(b->d_partials, G.d_wown, np, out + 2 * np, st), "l2");
    check_cuda(launch_sumsq_chunks(prec, G.d_hchunks, G.nh, G.H, b->d_partials, st), "l2");
    check_cuda(launch_owner_sums(b->d_partials, G.d_hown, np, out + 3 * np, st), "l2");
    std::vector<double> h(4 * (size_t)np);
    check_cuda(cudaMemcpyAsync(h.data(), out, h.size() * 8, cudaMemcpyDeviceToHost, st), "D2H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    for (uint32_t k = 0; k < np; ++k) {
      const uint32_t p = G.probs[k];
      for (int q = 0; q < 4; ++q) b->h_losses[4 * (size_t)p + q] = h[(size_t)q * np + k];
    }
  }
}

double train_loss(const dsgdpp_batch* b, uint32_t p) {
  const double* l = b->h_losses + 4 * (size_t)p;
  const auto& c = b->cfg;
  if (c.loss == DSGDPP_LOSS_NZSL_L2) return l[0] + c.loss_lambda * (l[2] + l[3]);
  return l[0];  // Nzsl (the Nzl2 loss is not batched)
}

int guard(dsgdpp_batch* b, const std::function<void()>& f) {
  if (!b) return DSGDPP_E_INVALID;
  try {
    b->err.clear();
    check_cuda(cudaSetDevice(b->cfg.device), "cudaSetDevice");
    f();
    return DSGDPP_OK;
  } catch (const Error& e) {
    b->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    b->err = "host allocation failed";
    return DSGDPP_E_NOMEM;
  }
}
}  // namespace

extern "C" {

int dsgdpp_batch_create(const dsgdpp_config* common, uint32_t count,
                        const dsgdpp_problem* problems, dsgdpp_batch** out) {
  if (!out) return DSGDPP_E_INVALID;
  *out = nullptr;
  auto* b = new (std::nothrow) dsgdpp_batch();
  if (!b) return DSGDPP_E_NOMEM;
  int rc;
  try {
    create_impl(b, common, count, problems);
    rc = DSGDPP_OK;
  } catch (const Error& e) {
    b->err = e.msg;
    rc = e.code;
  } catch (const std::bad_alloc&) {
    rc = DSGDPP_E_NOMEM;
  }
  if (rc != DSGDPP_OK) {
    std::fprintf(stderr, "dsgdpp_batch_create: %s\n", b->err.c_str());
    destroy_impl(b);
    delete b;
    return rc;
  }
  *out = b;
  return DSGDPP_OK;
}

void dsgdpp_batch_destroy(dsgdpp_batch* b) {
  if (!b) return;
  destroy_impl(b);
  delete b;
}

const char* dsgdpp_batch_last_error(const dsgdpp_batch* b) {
  return b ? b->err.c_str() : "null batch";
}

int dsgdpp_batch_run(dsgdpp_batch* b, uint32_t epochs, double decrease, double increase,
                     double* train, double* test, double* epoch_ms) {
  return guard(b, [&]() {
    const uint32_t np = (uint32_t)b->probs.size();
    b->epoch_ms = 0;
    losses(b, epochs == 0);
    for (uint32_t p = 0; p < np; ++p) b->probs[p].cur = train_loss(b, p);
    for (uint32_t e = 0; e < epochs; ++e) {
      if (e > 0)  // BoldDriver per problem (decay_bolddriver.h:59-67)
        for (Problem& P : b->probs) P.eps *= (P.prev <= P.cur) ? decrease : increase;
      run_epoch(b);
      losses(b, e + 1 == epochs);
      for (uint32_t p = 0; p < np; ++p) {
        b->probs[p].prev = b->probs[p].cur;
        b->probs[p].cur = train_loss(b, p);
      }
    }
    for (uint32_t p = 0; p < np; ++p) {
      if (train) train[p] = b->probs[p].cur;
      if (test) test[p] = b->h_losses[4 * (size_t)p + 1];
    }
    if (epoch_ms) *epoch_ms = b->epoch_ms;
  });
}

int dsgdpp_batch_autotune(const dsgdpp_config* common, uint32_t count,
                          const dsgdpp_problem* problems, uint32_t sample_stride, uint32_t epochs,
                          uint32_t* d_out, uint32_t* ctas_per_sm, double* best_ms) {
  if (!common || !problems || count == 0 || !d_out || !ctas_per_sm) return DSGDPP_E_INVALID;
  if (sample_stride == 0) sample_stride = 1;
  if (epochs == 0) epochs = 2;
  static const uint32_t kCaps[] = {4, 8, 16, 32};
  static const uint32_t kCtas[] = {0, 3, 2};  // 0: as many as fit
  std::vector<dsgdpp_problem> sample;
  for (uint32_t p = 0; p < count; p += sample_stride) sample.push_back(problems[p]);
  double best = INFINITY;
  uint32_t best_cap = 16, best_ctas = 0;
  int last_rc = DSGDPP_OK;
  for (uint32_t cap : kCaps) {
    for (dsgdpp_problem& q : sample) q.d = choose_d(q.m, q.n, q.nnz, cap);
    for (uint32_t ctas : kCtas) {
      dsgdpp_config c = *common;
      c.ctas_per_sm = ctas;
      dsgdpp_batch* b = nullptr;
      int rc = dsgdpp_batch_create(&c, (uint32_t)sample.size(), sample.data(), &b);
      if (rc != DSGDPP_OK) {
        last_rc = rc;
        continue;
      }
      double ms = 0;
      rc = dsgdpp_batch_run(b, 1, 1.0, 1.0, nullptr, nullptr, nullptr);  // warm-up, graph capture
      if (rc == DSGDPP_OK) rc = dsgdpp_batch_run(b, epochs, 1.0, 1.0, nullptr, nullptr, &ms);
      dsgdpp_batch_destroy(b);
      if (rc != DSGDPP_OK) {
        last_rc = rc;
        continue;
      }
      if (ms < best) {
        best = ms;
        best_cap = cap;
        best_ctas = ctas;
      }
    }
  }
  if (!(best < INFINITY)) return last_rc != DSGDPP_OK ? last_rc : DSGDPP_E_CUDA;
  for (uint32_t p = 0; p < count; ++p)
    d_out[p] = problems[p].d ? problems[p].d
                             : choose_d(problems[p].m, problems[p].n, problems[p].nnz, best_cap);
  *ctas_per_sm = best_ctas;
  if (best_ms) *best_ms = best / epochs;
  return DSGDPP_OK;
}

int dsgdpp_batch_problem_d(dsgdpp_batch* b, uint32_t p, uint32_t* d) {
  return guard(b, [&]() {
    if (p >= b->probs.size() || !d) throw Error(DSGDPP_E_INVALID, "no such problem");
    *d = b->probs[p].d;
  });
}

int dsgdpp_batch_get_factors(dsgdpp_batch* b, uint32_t p, double* W, double* H) {
  return guard(b, [&]() {
    if (p >= b->probs.size()) throw Error(DSGDPP_E_INVALID, "no such problem");
    const Problem& P = b->probs[p];
    const Group& G = b->groups[P.group];
    const size_t es = b->cfg.precision == kFp64 ? 8 : (b->cfg.precision == kFp32 ? 4 : 2);
    double* tmp = dnew<double>((P.m + P.n) * P.r, "staging");
    struct F { double* p; ~F() { cudaFree(p); } } f{tmp};
    check_cuda(launch_factor_to_host(b->cfg.precision, (unsigned char*)G.W + P.w0 * G.rp * es,
                                     P.m, P.r, G.rp, tmp, b->stream), "W");
    check_cuda(launch_factor_to_host(b->cfg.precision, (unsigned char*)G.H + P.h0 * G.rp * es,
                                     P.n, P.r, G.rp, tmp + P.m * P.r, b->stream), "H");
    if (W) check_cuda(cudaMemcpyAsync(W, tmp, P.m * P.r * 8, cudaMemcpyDeviceToHost, b->stream), "D2H");
    if (H)
      check_cuda(cudaMemcpyAsync(H, tmp + P.m * P.r, P.n * P.r * 8, cudaMemcpyDeviceToHost,
                                 b->stream), "D2H");
    check_cuda(cudaStreamSynchronize(b->stream), "sync");
  });
}

}  // extern "C"
