// capi.cu -- the C ABI of include/dsgdpp.h: context, data upload, epochs,
// losses and the defaultRunner loop.
#include <cub/cub.cuh>

#include <functional>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dsgdpp.h"
#include "context.h"
#include "rm_device.h"
#include "kernels.cuh"
#include "trace_ranges.h"
#include "schedule.h"

using namespace dsgdpp;

// The master generator's draws of one epoch: DsgdPpRunner::epoch
// (mf/sgd/dsgdpp_impl.h:289-344) or DsgdRunner::epoch (mf/sgd/dsgd_impl.h:
// 328-350: the d x d schedule of computeDsgdSchedule, then one seed per task).
void dsgdpp::draw_epoch(dsgdpp_ctx* c, uint32_t* sched, uint32_t* seeds) {
  if (c->cfg.method == DSGDPP_METHOD_DSGD) {
    const std::vector<uint32_t> S = dsgd_schedule(1, c->d, c->cfg.stratum_order, c->master);
    std::copy(S.begin(), S.end(), sched);
    for (uint32_t id = 0; id < c->d; ++id) seeds[id] = c->master.next();
  } else {
    dsgdpp_schedule(c->master, c->d, c->cfg.stratum_order, sched, seeds);
  }
}


namespace {

template <typename F>
int guarded(dsgdpp_ctx* ctx, F&& f) {
  if (!ctx) return DSGDPP_E_INVALID;
  try {
    ctx->err.clear();
    return f();
  } catch (const Error& e) {
    ctx->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    ctx->err = "host allocation failed";
    return DSGDPP_E_NOMEM;
  }
}

void release_graph(dsgdpp_ctx* c) {
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  c->graph_exec = nullptr;
}

int resolve_layout(int layout, uint64_t m, uint64_t n) {
  switch (layout) {
    case DSGDPP_LAYOUT_COL_RUNS: return kLayoutColRuns;
    case DSGDPP_LAYOUT_ROW_RUNS: return kLayoutRowRuns;
    case DSGDPP_LAYOUT_RUNS: return n <= m ? kLayoutColRuns : kLayoutRowRuns;
    default: return kLayoutShuffled;
  }
}

void choose_hogwild_shape(dsgdpp_ctx* c) {
  const uint32_t nvec = c->rp / vec_width(c->cfg.precision);
  uint32_t lanes = c->cfg.lanes_per_nnz, vecs = c->cfg.vecs_per_lane;
  if (lanes == 0) {
    lanes = 2;
    while (lanes < nvec && lanes < 32) lanes <<= 1;
    // FP32 rows of 8 vectors or more: half the lanes with two vectors each,
    // twice the groups per warp (measured faster at ranks 32 and 128: 7.6 vs
    // 8.8 ms and 18.5 vs 22.2 ms per epoch on the 100M-entry and
    // Netflix-shaped workloads)
    if (c->cfg.precision == kFp32 && vecs == 0 && nvec >= 8 && lanes >= 4) lanes /= 2;
  }
  if (vecs == 0) vecs = (nvec + lanes - 1) / lanes;
  if (vecs == 3) vecs = 4;
  c->lanes = lanes;
  c->vecs = vecs;
  if ((uint64_t)lanes * vecs < nvec)
    throw Error(DSGDPP_E_INVALID, "lanes_per_nnz x vecs_per_lane does not cover the rank");
  int per_sm = hogwild_ctas_per_sm(c->cfg.precision, lanes, vecs, c->atomic_writes != 0,
                                   c->d + 1, c->layout_key != kLayoutShuffled);
  if (per_sm <= 0)
    throw Error(DSGDPP_E_INVALID, "no Hogwild kernel for lanes_per_nnz=" + std::to_string(lanes) +
                                      ", vecs_per_lane=" + std::to_string(vecs));
  if (c->cfg.launch == DSGDPP_LAUNCH_PERSISTENT) {
    per_sm = hogwild_epoch_ctas_per_sm(c->cfg.precision, lanes, vecs, c->nb2);
    if (per_sm <= 0) throw Error(DSGDPP_E_INVALID, "no persistent epoch kernel for this rank");
  }
  if (c->cfg.ctas_per_sm) {  // counted in CTAs of 256 threads
    const int scale =
        c->cfg.launch == DSGDPP_LAUNCH_PERSISTENT ? 1 : hogwild_cta_scale(c->cfg.precision, lanes);
    per_sm = std::min<int>(per_sm, (int)c->cfg.ctas_per_sm * scale);
  }
  c->grid = (uint32_t)(per_sm * c->num_sms);
}

void validate_config(const dsgdpp_config* c) {
  if (!c) throw Error(DSGDPP_E_INVALID, "config is null");
  if (c->m == 0 || c->n == 0) throw Error(DSGDPP_E_INVALID, "m and n must be positive");
  if (c->m > 0xFFFFFFFFull || c->n > 0xFFFFFFFFull)
    throw Error(DSGDPP_E_INVALID, "m and n must fit in 32 bits");
  if (c->d < 1 || c->d > 1024) throw Error(DSGDPP_E_INVALID, "d must be in [1, 1024]");
  if (c->method != DSGDPP_METHOD_DSGDPP && c->method != DSGDPP_METHOD_DSGD)
    throw Error(DSGDPP_E_INVALID, "unknown method");
  const uint64_t nb2 = c->method == DSGDPP_METHOD_DSGD ? c->d : 2ull * c->d;
  if (nb2 > c->n || c->d > c->m)
    throw Error(DSGDPP_E_INVALID, c->method == DSGDPP_METHOD_DSGD
                                      ? "the d x d blocking needs m >= d and n >= d"
                                      : "the d x 2d blocking needs m >= d and n >= 2d");
  if (c->rank < 1) throw Error(DSGDPP_E_INVALID, "rank must be positive");
  if (c->precision < 0 || c->precision > 2) throw Error(DSGDPP_E_INVALID, "unknown precision");
  if (c->exec != DSGDPP_EXEC_REPLAY && c->exec != DSGDPP_EXEC_HOGWILD)
    throw Error(DSGDPP_E_INVALID, "unknown exec mode");
  if (c->exec == DSGDPP_EXEC_REPLAY && c->precision != DSGDPP_FP64)
    throw Error(DSGDPP_E_UNSUPPORTED, "replay mode runs FP64 factors only");
  if (c->exec == DSGDPP_EXEC_REPLAY && c->rank > 256)
    throw Error(DSGDPP_E_UNSUPPORTED, "replay mode supports rank <= 256");
  if (c->launch != DSGDPP_LAUNCH_STREAM && c->launch != DSGDPP_LAUNCH_GRAPH &&
      c->launch != DSGDPP_LAUNCH_PERSISTENT)
    throw Error(DSGDPP_E_INVALID, "unknown launch form");
  if (c->write_mode < 0 || c->write_mode > 2) throw Error(DSGDPP_E_INVALID, "unknown write mode");
  if (c->layout < 0 || c->layout > 3) throw Error(DSGDPP_E_INVALID, "unknown layout");
  if (c->update < 0 || c->update > 2) throw Error(DSGDPP_E_INVALID, "unknown update");
  if (c->regularize < 0 || c->regularize > 1) throw Error(DSGDPP_E_INVALID, "unknown regularize");
  if (c->loss < 0 || c->loss > 2) throw Error(DSGDPP_E_INVALID, "unknown loss");
  if (c->sgd_order < 0 || c->sgd_order > 2) throw Error(DSGDPP_E_INVALID, "unknown sgd order");
  if (c->stratum_order < 0 || c->stratum_order > 4)
    throw Error(DSGDPP_E_INVALID, "unknown stratum order");
  if (c->truncate && c->regularize == DSGDPP_REGULARIZE_L2 && c->exec == DSGDPP_EXEC_HOGWILD)
    throw Error(DSGDPP_E_UNSUPPORTED, "truncation with L2 regularization needs replay mode");
  const uint64_t vw = vec_width(c->precision);
  if ((c->rank + vw - 1) / vw > 128) throw Error(DSGDPP_E_UNSUPPORTED, "rank too large");
}

void create_impl(dsgdpp_ctx* c, const dsgdpp_config* cfg) {
  validate_config(cfg);
  c->cfg = *cfg;
  int ndev = 0;
  check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (cfg->device < 0 || cfg->device >= ndev) throw Error(DSGDPP_E_CUDA, "no such CUDA device");
  check_cuda(cudaSetDevice(cfg->device), "cudaSetDevice");
  check_cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  check_cuda(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, cfg->device),
             "cudaDeviceGetAttribute");
  c->d = cfg->d;
  c->nb2 = cfg->method == DSGDPP_METHOD_DSGD ? cfg->d : 2 * cfg->d;
  c->task_lo = 0;
  c->task_hi = cfg->d;
  c->r = cfg->rank;
  const uint32_t vw = vec_width(cfg->precision);
  c->rp = (c->r + vw - 1) / vw * vw;
  const uint32_t d = c->d, d2 = c->nb2;
  c->off1 = block_offsets(cfg->m, d);
  c->off1.push_back(cfg->m);
  c->off2 = block_offsets(cfg->n, d2);
  c->off2.push_back(cfg->n);
  c->d_off1 = dalloc<uint64_t>(d + 1, "off1");
  c->d_off2 = dalloc<uint64_t>(d2 + 1, "off2");
  check_cuda(cudaMemcpy(c->d_off1, c->off1.data(), (d + 1) * 8, cudaMemcpyHostToDevice), "off1");
  check_cuda(cudaMemcpy(c->d_off2, c->off2.data(), (d2 + 1) * 8, cudaMemcpyHostToDevice), "off2");
  const size_t es = elem_size(cfg->precision);
  check_cuda(cudaMalloc(&c->W, cfg->m * c->rp * es), "W");
  check_cuda(cudaMalloc(&c->H, cfg->n * c->rp * es), "H");
  check_cuda(cudaMemset(c->W, 0, cfg->m * c->rp * es), "W");
  check_cuda(cudaMemset(c->H, 0, cfg->n * c->rp * es), "H");
  c->cnt1 = dalloc<uint32_t>(cfg->m, "cnt1");
  c->cnt2 = dalloc<uint32_t>(cfg->n, "cnt2");
  check_cuda(cudaMemset(c->cnt1, 0, cfg->m * 4), "cnt1");
  check_cuda(cudaMemset(c->cnt2, 0, cfg->n * 4), "cnt2");
  if (cfg->exec == DSGDPP_EXEC_HOGWILD) {
    const size_t cs = cfg->precision == kFp64 ? 8 : 4;
    check_cuda(cudaMalloc(&c->inv1, cfg->m * cs), "inv1");
    check_cuda(cudaMalloc(&c->inv2, cfg->n * cs), "inv2");
  }
  c->h_schedule = halloc<uint32_t>((size_t)d2 * d, "schedule");
  c->d_schedule = dalloc<uint32_t>((size_t)d2 * d, "schedule");
  c->h_params = halloc<EpochParams>(1, "params");
  c->d_params = dalloc<EpochParams>(1, "params");
  c->h_sigma = halloc<float>((size_t)d2 * d * 3, "sigma");
  c->d_sigma = dalloc<float>((size_t)d2 * d * 3, "sigma");
  c->h_scales = halloc<float>(d2 + 1, "scales");
  c->d_scales = dalloc<float>(d2 + 1, "scales");
  c->d_segs = dalloc<Segment>((size_t)d2 * (d + 1), "segments");
  c->d_counters = dalloc<uint32_t>(d2, "counters");
  {  // launch s covers the d segments of sub-epoch s, counter s
    std::vector<LaunchDesc> ld(d2);
    for (uint32_t s = 0; s < d2; ++s) ld[s] = LaunchDesc{(uint64_t)s * (d + 1), d, s};
    c->d_launches = dalloc<LaunchDesc>(d2, "launches");
    check_cuda(cudaMemcpy(c->d_launches, ld.data(), d2 * sizeof(LaunchDesc), cudaMemcpyHostToDevice),
               "launches");
  }
  c->h_pos_offset = halloc<uint64_t>((size_t)d2 * d + 1, "pos_offset");
  c->d_pos_offset = dalloc<uint64_t>((size_t)d2 * d + 1, "pos_offset");
  c->h_mask = halloc<uint8_t>((size_t)d2 * d2, "mask");
  c->d_mask = dalloc<uint8_t>((size_t)d2 * d2, "mask");
  // one resident wave of the loss kernel; fixed per context, so every loss
  // of the context is reduced in the same order
  const int loss_per_sm = nzsl_ctas_per_sm(cfg->precision, c->rp);
  c->loss_grid = (uint32_t)c->num_sms * (uint32_t)std::max(2, std::min(8, loss_per_sm));
  c->d_partials = dalloc<double>(3 * (size_t)c->loss_grid, "partials");
  c->d_out = dalloc<double>(4, "loss out");
  c->h_out = halloc<double>(4, "loss out");
  check_cuda(cudaEventCreate(&c->ev_begin), "event");
  check_cuda(cudaEventCreate(&c->ev_end), "event");
  check_cuda(cudaEventCreateWithFlags(&c->ev_inputs, cudaEventDisableTiming), "event");
  check_cuda(cudaEventRecord(c->ev_inputs, c->stream), "event");
  if (cfg->write_mode == DSGDPP_WRITE_ATOMIC && cfg->truncate)
    throw Error(DSGDPP_E_UNSUPPORTED, "atomic writes cannot truncate");
  c->atomic_writes = cfg->write_mode == DSGDPP_WRITE_ATOMIC ||
                     (cfg->write_mode == DSGDPP_WRITE_AUTO && !cfg->truncate);
  c->layout_key = resolve_layout(cfg->layout, cfg->m, cfg->n);
  if (cfg->launch == DSGDPP_LAUNCH_PERSISTENT) {
    if (cfg->exec != DSGDPP_EXEC_HOGWILD || !c->atomic_writes ||
        c->layout_key == kLayoutShuffled || cfg->sgd_order == DSGDPP_SGD_WR)
      throw Error(DSGDPP_E_UNSUPPORTED,
                  "the persistent epoch runs the Hogwild path with atomic writes, a run layout "
                  "and the SEQ or WOR order");
    c->d_done = dalloc<uint32_t>((size_t)d2 * d, "segment counters");
    c->d_dep_col = dalloc<int32_t>((size_t)d2 * d, "column dependencies");
    c->h_dep_col = halloc<int32_t>((size_t)d2 * d, "column dependencies");
    c->d_ticket = dalloc<uint32_t>(2, "ticket");  // [0] ticket, [1] error flag
    c->h_error = halloc<uint32_t>(1, "error flag");
    *c->h_error = 0;
  }
  if (cfg->exec == DSGDPP_EXEC_HOGWILD) choose_hogwild_shape(c);
}

void destroy_impl(dsgdpp_ctx* c) {
  if (c->stream) cudaStreamSynchronize(c->stream);
  release_graph(c);
  for (auto& m : c->mat) {
    dfree(m.row); dfree(m.col); dfree(m.val); dfree(m.block_ptr);
  }
  dfree(c->d_off1); dfree(c->d_off2);
  dfree(c->W); dfree(c->H); dfree(c->cnt1); dfree(c->cnt2); dfree(c->inv1); dfree(c->inv2);
  dfree(c->staging);
  dfree(c->scratch);
  dfree(c->W_saved); dfree(c->H_saved);
  hfree(c->h_schedule); dfree(c->d_schedule); hfree(c->h_params); dfree(c->d_params);
  hfree(c->h_sigma); dfree(c->d_sigma); hfree(c->h_scales); dfree(c->d_scales);
  dfree(c->d_segs); dfree(c->d_counters); dfree(c->d_launches);
  dfree(c->d_done); dfree(c->d_dep_col); hfree(c->h_dep_col); dfree(c->d_ticket);
  hfree(c->h_error);
  hfree(c->h_positions); dfree(c->d_positions); hfree(c->h_pos_offset); dfree(c->d_pos_offset);
  hfree(c->h_mask); dfree(c->d_mask);
  dfree(c->d_partials); dfree(c->d_out); hfree(c->h_out);
  for (auto e : c->prof_ev) cudaEventDestroy(e);
  c->prof_ev.clear();
  if (c->ev_begin) cudaEventDestroy(c->ev_begin);
  if (c->ev_end) cudaEventDestroy(c->ev_end);
  if (c->ev_inputs) cudaEventDestroy(c->ev_inputs);
  if (c->ev_coords) cudaEventDestroy(c->ev_coords);
  if (c->ev_vals) cudaEventDestroy(c->ev_vals);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
}

// ---- blocking on the GPU ----------------------------------------------------------
int bit_length(uint64_t v) {
  int b = 0;
  while (v) { ++b; v >>= 1; }
  return b;
}

// Bump allocation inside one scratch buffer (256-byte aligned pieces); with a
// null base it only adds up the size.
struct Carver {
  char* base = nullptr;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += std::max<size_t>(count, 1) * sizeof(T);
    return p;
  }
};

// record arrays of a matrix, grown only when a larger matrix arrives
void reserve_records(DevMatrix& M, uint64_t u, bool as_double) {
  u = std::max<uint64_t>(u, 1);
  if (M.row && M.cap >= u) return;
  dfree(M.row); dfree(M.col); dfree(M.val);
  M.cap = 0;
  M.row = dalloc<uint32_t>(u, "row");
  M.col = dalloc<uint32_t>(u, "col");
  check_cuda(cudaMalloc(&M.val, u * (as_double ? 8 : 4)), "val");
  M.cap = u;
}

// Fills the device input arrays (rows, cols, values) of the blocking: the
// entries generated on the device instead of copied from the host.
using DeviceFill = std::function<void(uint32_t*, uint32_t*, double*, cudaStream_t)>;

void set_matrix_impl(dsgdpp_ctx* c, int which, uint64_t nnz, const uint32_t* rows,
                     const uint32_t* cols, const double* vals,
                     const DeviceFill* fill = nullptr) {
  if (which != DSGDPP_TRAIN && which != DSGDPP_TEST) throw Error(DSGDPP_E_INVALID, "which");
  if (nnz > 0 && !fill && (!rows || !cols || !vals)) throw Error(DSGDPP_E_INVALID, "null input array");
  if (nnz >= 0x7FFFFFFFull) throw Error(DSGDPP_E_UNSUPPORTED, "nnz must be below 2^31");
  check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
  check_cuda(cudaStreamSynchronize(c->stream), "sync");
  release_graph(c);
  cudaStream_t st = c->stream;
  const uint32_t d = c->d, d2 = c->nb2, nblocks = d * d2;
  uint64_t mB = 0, nB = 0;
  for (uint32_t b = 0; b < d; ++b) mB = std::max(mB, c->off1[b + 1] - c->off1[b]);
  for (uint32_t b = 0; b < d2; ++b) nB = std::max(nB, c->off2[b + 1] - c->off2[b]);
  const uint64_t span = mB * nB;
  if (span == 0 || (double)nblocks * (double)span >= 1.8e19)
    throw Error(DSGDPP_E_UNSUPPORTED, "m x n too large for the 64-bit block key");
  const bool as_double = c->cfg.precision == kFp64;
  const bool shuffled = which == DSGDPP_TRAIN && c->cfg.exec == DSGDPP_EXEC_HOGWILD;

  DevMatrix& M = c->mat[which];
  M.present = false;
  M.nnz = 0;
  if (!M.block_ptr || M.nblocks != nblocks) {
    dfree(M.block_ptr);
    M.block_ptr = dalloc<uint64_t>(nblocks + 1, "block_ptr");
    M.nblocks = nblocks;
  }
  M.h_block_ptr.assign(nblocks + 1, 0);
  if (nnz == 0) {
    check_cuda(cudaMemset(M.block_ptr, 0, (nblocks + 1) * 8), "block_ptr");
    reserve_records(M, 1, as_double);
    M.present = true;
    if (which == DSGDPP_TRAIN) {
      check_cuda(cudaMemset(c->cnt1, 0, c->cfg.m * 4), "cnt1");
      check_cuda(cudaMemset(c->cnt2, 0, c->cfg.n * 4), "cnt2");
    }
    return;
  }

  // The blocking key (kernels.cuh: BlockingGeom).  For the Hogwild training
  // records its position part is the in-block layout order, so the one sort
  // both blocks and lays out the records; a key that would pass 64 bits keeps
  // the plain positions and lays the records out with a second sort.
  BlockingGeom g{c->cfg.m, c->cfg.n, d, d2, mB, nB, c->d_off1, c->d_off2};
  g.stride = span;
  bool layout_in_key = false;
  if (shuffled) {
    const int mode = c->layout_key;
    const uint64_t permuted = mode == kLayoutColRuns ? mB : mode == kLayoutRowRuns ? nB : span;
    const uint64_t major = mode == kLayoutColRuns ? nB : mode == kLayoutRowRuns ? mB : 1;
    const int pb = bit_length(permuted - 1);
    if (pb + bit_length(major) < 63 &&
        (double)nblocks * (double)(major << pb) < 1.8e19) {
      g.layout = mode;
      g.pbits = pb;
      g.stride = major << pb;
      g.seed = c->cfg.layout_seed;
      layout_in_key = true;
    }
  }

  // Scratch for the blocking: sized for nnz, kept by the context and reused
  // by later calls (a matrix of the same size allocates nothing).
  const int end_bit = bit_length((uint64_t)nblocks * g.stride - 1);
  const int blk_bits = bit_length((uint64_t)nblocks - 1);
  const int shuffle_bits = 32 + blk_bits;  // (block, 32-bit hash) layout keys
  size_t sort_bytes = 0, sort2_bytes = 0, scan_bytes = 0;
  {
    cub::DoubleBuffer<uint64_t> kb(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
    check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, kb, vb, (int)nnz, 0, end_bit,
                                               st), "sort size");
    check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, sort2_bytes, kb, vb, (int)nnz, 0,
                                               shuffle_bits, st), "sort size");
    check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t*)nullptr,
                                             (uint32_t*)nullptr, (int)nnz, st), "scan size");
  }
  Carver plan;
  plan.take<uint32_t>(nnz); plan.take<uint32_t>(nnz); plan.take<double>(nnz);   // input
  plan.take<uint64_t>(nnz); plan.take<uint64_t>(nnz);                          // keys
  plan.take<uint32_t>(nnz); plan.take<uint32_t>(nnz);                          // idx
  plan.take<uint32_t>(nnz);                                                    // pos
  plan.take<uint32_t>(nnz); plan.take<uint32_t>(nnz); plan.take<uint32_t>(nnz);  // merged
  plan.take<uint64_t>(nnz);                                                    // layout keys
  plan.take<unsigned long long>(1);
  plan.take<char>(std::max({sort_bytes, sort2_bytes, scan_bytes}));
  if (plan.off > c->scratch_bytes) {
    dfree(c->scratch);
    c->scratch_bytes = 0;
    c->scratch = dalloc<char>(plan.off, "blocking scratch");
    c->scratch_bytes = plan.off;
  }
  Carver cv{static_cast<char*>(c->scratch)};
  uint32_t* t_rows = cv.take<uint32_t>(nnz);
  uint32_t* t_cols = cv.take<uint32_t>(nnz);
  double* t_vals = cv.take<double>(nnz);
  uint64_t* keys[2] = {cv.take<uint64_t>(nnz), cv.take<uint64_t>(nnz)};
  uint32_t* idx[2] = {cv.take<uint32_t>(nnz), cv.take<uint32_t>(nnz)};
  uint32_t* pos = cv.take<uint32_t>(nnz);
  uint32_t* urow = cv.take<uint32_t>(nnz);
  uint32_t* ucol = cv.take<uint32_t>(nnz);
  uint32_t* head_at = cv.take<uint32_t>(nnz);
  uint64_t* lkeys = cv.take<uint64_t>(nnz);
  unsigned long long* d_bad = cv.take<unsigned long long>(1);
  void* tmp = cv.take<char>(std::max({sort_bytes, sort2_bytes, scan_bytes}));

  // The coordinates are copied first; the values (half the bytes) follow on
  // a side stream while everything that needs only the coordinates runs --
  // keys, the sort, duplicate runs, block pointers, the in-block layout (on
  // the key, or a second sort), the final coordinates and the counts -- and
  // are waited for only by the
  // last step, which sums each record's run of values into place.  The guard
  // waits for that copy on every exit, so no copy outlives the call (the
  // caller may free its arrays).
  struct SideGuard {
    cudaStream_t s = nullptr;
    ~SideGuard() {
      if (s) cudaStreamSynchronize(s);
    }
  } side_guard;
  bool vals_on_side = false;
  if (fill) {
    (*fill)(t_rows, t_cols, t_vals, st);
  } else {
    if (!c->side) {
      check_cuda(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking), "side stream");
      check_cuda(cudaEventCreateWithFlags(&c->ev_coords, cudaEventDisableTiming), "event");
      check_cuda(cudaEventCreateWithFlags(&c->ev_vals, cudaEventDisableTiming), "event");
    }
    check_cuda(cudaMemcpyAsync(t_rows, rows, nnz * 4, cudaMemcpyHostToDevice, st), "H2D rows");
    check_cuda(cudaMemcpyAsync(t_cols, cols, nnz * 4, cudaMemcpyHostToDevice, st), "H2D cols");
    check_cuda(cudaEventRecord(c->ev_coords, st), "event");
    check_cuda(cudaStreamWaitEvent(c->side, c->ev_coords, 0), "wait");
    side_guard.s = c->side;
    check_cuda(cudaMemcpyAsync(t_vals, vals, nnz * 8, cudaMemcpyHostToDevice, c->side), "H2D vals");
    check_cuda(cudaEventRecord(c->ev_vals, c->side), "event");
    vals_on_side = true;
  }
  check_cuda(cudaMemsetAsync(d_bad, 0, 8, st), "memset");
  check_cuda(launch_make_keys(g, t_rows, t_cols, nnz, keys[0], idx[0], d_bad, st), "make_keys");
  unsigned long long bad = 0;
  check_cuda(cudaMemcpyAsync(&bad, d_bad, 8, cudaMemcpyDeviceToHost, st), "D2H");
  check_cuda(cudaStreamSynchronize(st), "sync");
  if (bad) throw Error(DSGDPP_E_INVALID, std::to_string(bad) + " entries lie outside the matrix");

  cub::DoubleBuffer<uint64_t> kb(keys[0], keys[1]);
  cub::DoubleBuffer<uint32_t> vb(idx[0], idx[1]);
  check_cuda(cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, kb, vb, (int)nnz, 0, end_bit, st),
             "sort");
  uint64_t* skeys = kb.Current();
  uint32_t* sidx = vb.Current();
  uint64_t* okeys = kb.Alternate();
  uint32_t* oidx = vb.Alternate();

  // run heads -> output positions (reuse the alternate index buffer)
  uint32_t* flags = oidx;
  check_cuda(launch_head_flags(skeys, nnz, flags, st), "head_flags");
  check_cuda(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, flags, pos, (int)nnz, st), "scan");
  uint32_t last_pos = 0, last_flag = 0;
  check_cuda(cudaMemcpyAsync(&last_pos, pos + nnz - 1, 4, cudaMemcpyDeviceToHost, st), "D2H");
  check_cuda(cudaMemcpyAsync(&last_flag, flags + nnz - 1, 4, cudaMemcpyDeviceToHost, st), "D2H");
  check_cuda(cudaStreamSynchronize(st), "sync");
  const uint64_t u = (uint64_t)last_pos + last_flag;

  // duplicate runs -> one record each (key, coordinates, where its run starts)
  uint64_t* ukeys = okeys;
  check_cuda(launch_merge_keys(skeys, sidx, pos, nnz, t_rows, t_cols, ukeys, urow, ucol, head_at,
                               st), "merge_keys");
  check_cuda(launch_block_ptr(ukeys, u, g.stride, nblocks, M.block_ptr, st), "block_ptr");

  reserve_records(M, u, as_double);
  const uint32_t* perm = nullptr;  // final record k = merged record perm[k]
  if (shuffled && !layout_in_key) {
    // in-block layout: key = (block, 32-bit hash(layout_seed, k)), or
    // (block, local column | local row, hash) for runs; the sorted keys and
    // indices of the first sort stay for the values
    check_cuda(launch_shuffle_keys(ukeys, u, span, nB, c->layout_key, c->cfg.layout_seed, lkeys,
                                   pos, st), "shuffle");
    cub::DoubleBuffer<uint64_t> kb2(lkeys, ukeys);
    cub::DoubleBuffer<uint32_t> vb2(pos, flags);
    check_cuda(cub::DeviceRadixSort::SortPairs(tmp, sort2_bytes, kb2, vb2, (int)u, 0,
                                               shuffle_bits, st), "sort");
    perm = vb2.Current();
  }
  check_cuda(launch_gather_coords(perm, u, urow, ucol, M.row, M.col, st), "gather");
  check_cuda(cudaMemcpyAsync(M.h_block_ptr.data(), M.block_ptr, (nblocks + 1) * 8,
                             cudaMemcpyDeviceToHost, st), "D2H block_ptr");
  if (which == DSGDPP_TRAIN) {
    check_cuda(cudaMemsetAsync(c->cnt1, 0, c->cfg.m * 4, st), "cnt1");
    check_cuda(cudaMemsetAsync(c->cnt2, 0, c->cfg.n * 4, st), "cnt2");
    check_cuda(launch_count_nnz12(M.row, M.col, u, c->cnt1, c->cnt2, st), "nnz12");
    if (c->inv1) {
      check_cuda(launch_inverse_counts(c->cnt1, c->cfg.m, c->inv1, as_double, st), "inv1");
      check_cuda(launch_inverse_counts(c->cnt2, c->cfg.n, c->inv2, as_double, st), "inv2");
    }
  }
  if (vals_on_side) check_cuda(cudaStreamWaitEvent(st, c->ev_vals, 0), "wait values");
  check_cuda(launch_gather_values(perm, u, head_at, skeys, sidx, nnz, t_vals, M.val, as_double,
                                  st), "gather values");
  check_cuda(cudaStreamSynchronize(st), "sync");
  M.nnz = u;
  M.present = true;
}

void ensure_staging(dsgdpp_ctx* c) {
  if (!c->staging) c->staging = dalloc<double>((c->cfg.m + c->cfg.n) * c->r, "staging");
}

// ---- epochs --------------------------------------------------------------------------
void wait_inputs_free(dsgdpp_ctx* c) {
  check_cuda(cudaEventSynchronize(c->ev_inputs), "event sync");
}

void fill_epoch_params(dsgdpp_ctx* c, double eps, const uint32_t* seeds) {
  EpochParams p{};
  p.eps = eps;
  p.key0 = seeds[0];
  p.key1 = c->d > 1 ? seeds[1] : (seeds[0] ^ 0x5bd1e995u);
  p.epoch = c->epoch_counter++;
  *c->h_params = p;
}

// lazy L2 scales of the Hogwild path: sigma_W before sub-epoch s is f^s; the
// scale of H block b2 is f^(earlier visits of b2); both are folded into the
// update and applied to the factors once at the end of the epoch.
void fill_sigma(dsgdpp_ctx* c, double eps) {
  const uint32_t d = c->d, d2 = c->nb2;
  const bool l2 = c->cfg.regularize == DSGDPP_REGULARIZE_L2 && c->cfg.regularize_lambda != 0;
  double factor = 1.0;
  if (l2) {
    const double er = eps / d;
    factor = 1 - er * 2 * c->cfg.regularize_lambda;
    if (factor < 0.5) factor = 0.25 / (1 - factor);
  }
  std::vector<double> sh(d2, 1.0);
  double sw = 1.0;
  for (uint32_t s = 0; s < d2; ++s) {
    for (uint32_t id = 0; id < d; ++id) {
      const uint32_t b2 = c->h_schedule[(size_t)s * d + id];
      float* o = c->h_sigma + ((size_t)s * d + id) * 3;
      o[0] = (float)(sw * sh[b2]);
      o[1] = (float)(sh[b2] / sw);
      o[2] = (float)(sw / sh[b2]);
    }
    sw *= factor;
    for (uint32_t id = 0; id < d; ++id) sh[c->h_schedule[(size_t)s * d + id]] *= factor;
  }
  for (uint32_t b = 0; b < d2; ++b) c->h_scales[b] = (float)sh[b];
  c->h_scales[d2] = (float)sw;
}

// persistent epoch: for segment (s, i) the last earlier segment of the epoch
// that worked on the same column block of H (flat index s2 * d + j), or -1
void fill_deps(dsgdpp_ctx* c) {
  const uint32_t d = c->d, d2 = c->nb2;
  std::vector<int32_t> last(d2, -1);
  for (uint32_t s = 0; s < d2; ++s) {
    for (uint32_t i = 0; i < d; ++i)
      c->h_dep_col[(size_t)s * d + i] = last[c->h_schedule[(size_t)s * d + i]];
    for (uint32_t i = 0; i < d; ++i)
      last[c->h_schedule[(size_t)s * d + i]] = (int32_t)(s * d + i);
  }
}

bool lazy_l2(const dsgdpp_ctx* c) {
  return c->cfg.regularize == DSGDPP_REGULARIZE_L2 && c->cfg.regularize_lambda != 0;
}

// Sub-epochs [s0, s1) of the epoch; the epoch's inputs are uploaded and its
// segment tables built with the part that starts at 0, the end-of-epoch
// normalization runs with the part that ends at nb2.
void enqueue_hogwild_epoch(dsgdpp_ctx* c, uint32_t s0, uint32_t s1) {
  cudaStream_t st = c->stream;
  const uint32_t d = c->d, d2 = c->nb2;
  const bool l2 = lazy_l2(c);
  const bool persistent = c->cfg.launch == DSGDPP_LAUNCH_PERSISTENT;
  if (s0 == 0) {
  check_cuda(cudaMemcpyAsync(c->d_schedule, c->h_schedule, (size_t)d2 * d * 4,
                             cudaMemcpyHostToDevice, st), "H2D schedule");
  check_cuda(cudaMemcpyAsync(c->d_params, c->h_params, sizeof(EpochParams),
                             cudaMemcpyHostToDevice, st), "H2D params");
  if (l2) {
    check_cuda(cudaMemcpyAsync(c->d_sigma, c->h_sigma, (size_t)d2 * d * 3 * 4,
                               cudaMemcpyHostToDevice, st), "H2D sigma");
    check_cuda(cudaMemcpyAsync(c->d_scales, c->h_scales, (d2 + 1) * 4, cudaMemcpyHostToDevice,
                               st), "H2D scales");
  }
  SegBuildArgs sb{c->d_params, c->d_schedule, c->mat[0].block_ptr, l2 ? c->d_sigma : nullptr,
                  c->d_segs, c->d_counters, d, d2};
  check_cuda(launch_build_segments(sb, st), "build_segments");
  if (persistent) {
    check_cuda(cudaMemcpyAsync(c->d_dep_col, c->h_dep_col, (size_t)d2 * d * 4,
                               cudaMemcpyHostToDevice, st), "H2D dependencies");
    check_cuda(cudaMemsetAsync(c->d_done, 0, (size_t)d2 * d * 4, st), "segment counters");
    check_cuda(cudaMemsetAsync(c->d_ticket, 0, 8, st), "ticket");
  }
  }
  HogwildArgs a{};
  const DevMatrix& M = c->mat[0];
  a.row = M.row; a.col = M.col; a.val = M.val;
  a.inv1 = c->inv1; a.inv2 = c->inv2;
  a.W = c->W; a.H = c->H;
  a.runs = c->layout_key != kLayoutShuffled;
  if (c->layout_key == kLayoutRowRuns) {  // the kernel caches its "H" side: hand it W
    a.row = M.col; a.col = M.row;
    a.inv1 = c->inv2; a.inv2 = c->inv1;
    a.W = c->H; a.H = c->W;
    a.swap_sides = 1;
  }
  a.segs = c->d_segs; a.launches = c->d_launches; a.counters = c->d_counters;
  a.params = c->d_params; a.smem_segs = d + 1;
  a.r = c->r; a.rp = c->rp;
  a.update = c->cfg.update; a.truncate = c->cfg.truncate; a.sgd_order = c->cfg.sgd_order;
  a.atomic = c->atomic_writes;
  a.lambda = c->cfg.update_lambda; a.tmin = c->cfg.truncate_min; a.tmax = c->cfg.truncate_max;
  const bool prof = c->profiling && c->prof_ev.size() == d2 + 1 && s0 == 0 && s1 == d2;
  if (persistent) {
    EpochDeps dp{c->d_dep_col, c->d_done, c->d_ticket, c->d_ticket + 1, d, d2, c->wait_ns};
    if (prof) check_cuda(cudaEventRecord(c->prof_ev[0], st), "event");
    check_cuda(launch_hogwild_epoch(c->cfg.precision, c->lanes, c->vecs, a, dp, c->grid, st),
               "hogwild_epoch");
    if (prof) check_cuda(cudaEventRecord(c->prof_ev[d2], st), "event");
    check_cuda(cudaMemcpyAsync(c->h_error, c->d_ticket + 1, 4, cudaMemcpyDeviceToHost, st),
               "D2H error flag");
  }
  for (uint32_t s = s0; s < s1 && !persistent; ++s) {
    if (prof) check_cuda(cudaEventRecord(c->prof_ev[s], st), "event");
    // launches back to back (no timing event between) overlap start and end
    check_cuda(launch_hogwild(c->cfg.precision, c->lanes, c->vecs, a, s, c->grid, st,
                              s > s0 && !prof), "hogwild_subepoch");
  }
  if (prof && !persistent) check_cuda(cudaEventRecord(c->prof_ev[d2], st), "event");
  if (l2 && s1 == d2)
    check_cuda(launch_normalize(c->cfg.precision, c->W, c->H, c->cfg.m, c->cfg.n, c->rp,
                                c->d_scales, c->d_off2, d2, st), "normalize");
}

void collect_profile(dsgdpp_ctx* c) {
  if (!c->prof_pending) return;
  c->prof_pending = false;
  const uint32_t d2 = c->nb2;
  check_cuda(cudaEventSynchronize(c->prof_ev[d2]), "event sync");
  if (c->cfg.launch == DSGDPP_LAUNCH_PERSISTENT) {  // one launch per epoch
    float f = 0;
    check_cuda(cudaEventElapsedTime(&f, c->prof_ev[0], c->prof_ev[d2]), "elapsed");
    c->prof_ms += f;
    c->prof_launches += 1;
    return;
  }
  for (uint32_t s = 0; s < d2; ++s) {
    float f = 0;
    check_cuda(cudaEventElapsedTime(&f, c->prof_ev[s], c->prof_ev[s + 1]), "elapsed");
    c->prof_ms += f;
  }
  c->prof_launches += d2;
}

void run_hogwild_epoch(dsgdpp_ctx* c, double eps, uint32_t s0, uint32_t s1) {
  const bool whole = s0 == 0 && s1 == c->nb2;
  const bool persistent = c->cfg.launch == DSGDPP_LAUNCH_PERSISTENT;
  if (!whole && persistent)
    throw Error(DSGDPP_E_UNSUPPORTED, "the persistent launch runs whole epochs only");
  if (s0 == 0 && lazy_l2(c)) fill_sigma(c, eps);
  cudaStream_t st = c->stream;
  if (!whole) {  // a part: stream launches, timed from its first to its last part
    if (s0 == 0) check_cuda(cudaEventRecord(c->ev_begin, st), "event");
    enqueue_hogwild_epoch(c, s0, s1);
    if (s1 == c->nb2) {
      check_cuda(cudaEventRecord(c->ev_end, st), "event");
      c->epoch_timed = true;
    }
    check_cuda(cudaEventRecord(c->ev_inputs, st), "event");
    return;
  }
  if (persistent) fill_deps(c);
  collect_profile(c);
  check_cuda(cudaEventRecord(c->ev_begin, st), "event");
  if ((c->cfg.launch == DSGDPP_LAUNCH_GRAPH || persistent) && !c->profiling) {
    if (!c->graph_exec) {
      cudaGraph_t g = nullptr;
      check_cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
      try {
        enqueue_hogwild_epoch(c, 0, c->nb2);
      } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      check_cuda(cudaStreamEndCapture(st, &g), "capture end");
      cudaError_t e = cudaGraphInstantiate(&c->graph_exec, g, 0);
      cudaGraphDestroy(g);
      check_cuda(e, "graph instantiate");
    }
    check_cuda(cudaGraphLaunch(c->graph_exec, st), "graph launch");
  } else {
    enqueue_hogwild_epoch(c, 0, c->nb2);
    c->prof_pending = c->profiling;
  }
  check_cuda(cudaEventRecord(c->ev_end, st), "event");
  check_cuda(cudaEventRecord(c->ev_inputs, st), "event");
  c->epoch_timed = true;
  if (persistent) {  // a dependency wait that gave up leaves the epoch incomplete
    check_cuda(cudaEventSynchronize(c->ev_end), "event sync");
    if (*c->h_error) {
      *c->h_error = 0;
      throw Error(DSGDPP_E_CUDA, "persistent epoch: a dependency wait gave up after " +
                                     std::to_string(c->wait_ns / 1000) +
                                     " us; the epoch is incomplete");
    }
  }
}

void run_replay_epoch(dsgdpp_ctx* c, double eps, const uint32_t* seeds, uint32_t s0, uint32_t s1) {
  const uint32_t d = c->d, d2 = c->nb2;
  const DevMatrix& M = c->mat[0];
  const bool l2 = c->cfg.regularize == DSGDPP_REGULARIZE_L2;
  cudaStream_t st = c->stream;
  if (s0 == 0) {  // the epoch's inputs, with its first part
  // point orders, one generator per task (mf/sgd/dsgdpp_impl.h:79,112)
  uint64_t total = 0;
  for (uint32_t s = 0; s < d2; ++s)
    for (uint32_t id = 0; id < d; ++id) {
      c->h_pos_offset[(size_t)s * d + id] = total;
      const uint64_t blk = (uint64_t)id * d2 + c->h_schedule[(size_t)s * d + id];
      total += M.h_block_ptr[blk + 1] - M.h_block_ptr[blk];
    }
  c->h_pos_offset[(size_t)d2 * d] = total;
  if (total > c->positions_cap) {
    hfree(c->h_positions);
    dfree(c->d_positions);
    c->positions_cap = std::max<uint64_t>(total, 1);
    c->h_positions = halloc<uint32_t>(c->positions_cap, "positions");
    c->d_positions = dalloc<uint32_t>(c->positions_cap, "positions");
  }
  const unsigned hw = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), d));
  auto work = [&](unsigned t) {
    for (uint32_t id = t; id < d; id += hw) {
      TaskOrder order(seeds[id]);
      for (uint32_t s = 0; s < d2; ++s) {
        const uint64_t blk = (uint64_t)id * d2 + c->h_schedule[(size_t)s * d + id];
        const uint64_t n = M.h_block_ptr[blk + 1] - M.h_block_ptr[blk];
        order.next_block(c->cfg.sgd_order, n, c->h_positions + c->h_pos_offset[(size_t)s * d + id]);
      }
    }
  };
  if (hw > 1 && total > 100000) {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < hw; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  } else {
    for (unsigned t = 0; t < hw; ++t) work(t);
  }
  if (l2) {  // the H blocks each sub-epoch's tasks (those run here) regularize
    std::memset(c->h_mask, 0, (size_t)d2 * d2);
    for (uint32_t s = 0; s < d2; ++s)
      for (uint32_t id = c->task_lo; id < c->task_hi; ++id)
        c->h_mask[(size_t)s * d2 + c->h_schedule[(size_t)s * d + id]] = 1;
  }
  check_cuda(cudaEventRecord(c->ev_begin, st), "event");
  check_cuda(cudaMemcpyAsync(c->d_schedule, c->h_schedule, (size_t)d2 * d * 4,
                             cudaMemcpyHostToDevice, st), "H2D schedule");
  check_cuda(cudaMemcpyAsync(c->d_params, c->h_params, sizeof(EpochParams),
                             cudaMemcpyHostToDevice, st), "H2D params");
  check_cuda(cudaMemcpyAsync(c->d_pos_offset, c->h_pos_offset, ((size_t)d2 * d + 1) * 8,
                             cudaMemcpyHostToDevice, st), "H2D pos_offset");
  if (total)
    check_cuda(cudaMemcpyAsync(c->d_positions, c->h_positions, total * 4, cudaMemcpyHostToDevice,
                               st), "H2D positions");
  if (l2)
    check_cuda(cudaMemcpyAsync(c->d_mask, c->h_mask, (size_t)d2 * d2, cudaMemcpyHostToDevice, st),
               "H2D mask");
  }
  ReplayArgs a{};
  a.row = M.row; a.col = M.col; a.val = static_cast<const double*>(M.val);
  a.cnt1 = c->cnt1; a.cnt2 = c->cnt2;
  a.W = static_cast<double*>(c->W); a.H = static_cast<double*>(c->H);
  a.block_ptr = M.block_ptr; a.schedule = c->d_schedule;
  a.positions = c->d_positions; a.pos_offset = c->d_pos_offset; a.params = c->d_params;
  a.d = d; a.r = c->r; a.rp = c->rp; a.nb2 = d2;
  a.update = c->cfg.update; a.truncate = c->cfg.truncate;
  a.lambda = c->cfg.update_lambda; a.tmin = c->cfg.truncate_min; a.tmax = c->cfg.truncate_max;
  for (uint32_t s = s0; s < s1; ++s) {
    check_cuda(launch_replay_subepoch(a, s, st), "replay_subepoch");
    // the W row blocks of the tasks run here
    double* w0 = a.W + c->off1[c->task_lo] * c->rp;
    const uint64_t wrows = c->off1[c->task_hi] - c->off1[c->task_lo];
    if (l2 && c->cfg.regularize_lambda != 0)
      check_cuda(launch_regularize_exact(w0, a.H, wrows, c->cfg.n, c->rp, c->r, c->d_off2,
                                         c->d_mask + (size_t)s * d2, d, d2, c->d_params,
                                         c->cfg.regularize_lambda, c->cfg.truncate,
                                         c->cfg.truncate_min, c->cfg.truncate_max, st),
                 "regularize");
  }
  if (s1 == d2) {
    check_cuda(cudaEventRecord(c->ev_end, st), "event");
    c->epoch_timed = true;
  }
  check_cuda(cudaEventRecord(c->ev_inputs, st), "event");
}

// Sub-epochs [s0, s1) of the epoch given by (eps, schedule, seeds); the
// whole epoch is the range [0, nb2).  Parts run in order: a part starting at
// 0 begins an epoch, later parts must continue it with the same arguments.
void epoch_part_impl(dsgdpp_ctx* c, double eps, const uint32_t* schedule, const uint32_t* seeds,
                     uint32_t s0, uint32_t s1) {
  if (!schedule || !seeds) throw Error(DSGDPP_E_INVALID, "schedule and task seeds are required");
  if (!c->mat[0].present) throw Error(DSGDPP_E_STATE, "no training matrix");
  if (!c->factors_set) throw Error(DSGDPP_E_STATE, "factors not set");
  if (!std::isfinite(eps)) throw Error(DSGDPP_E_INVALID, "step size is not finite");
  const uint32_t d = c->d, d2 = c->nb2;
  if (s0 >= s1 || s1 > d2) throw Error(DSGDPP_E_INVALID, "sub-epoch range out of order or bounds");
  if (s0 != c->part_next)
    throw Error(DSGDPP_E_STATE, s0 == 0 ? "the epoch given in parts is unfinished"
                                        : "parts of an epoch must follow one another");
  if (s0 == 0) {
    for (size_t k = 0; k < (size_t)d2 * d; ++k)
      if (schedule[k] >= d2) throw Error(DSGDPP_E_INVALID, "schedule entry out of range");
  } else if (eps != c->h_params->eps ||
             std::memcmp(schedule, c->h_schedule, (size_t)d2 * d * 4) != 0 ||
             std::memcmp(seeds, c->part_seeds.data(), (size_t)d * 4) != 0) {
    throw Error(DSGDPP_E_INVALID, "a later part of an epoch must repeat its step size, schedule and seeds");
  }
  if (s0 == 0 && (c->task_lo != 0 || c->task_hi != d)) {
    for (int which = 0; which < 2; ++which) {
      const DevMatrix& M = c->mat[which];
      if (!M.present) continue;
      for (uint32_t b1 = 0; b1 < d; ++b1)
        if ((b1 < c->task_lo || b1 >= c->task_hi) &&
            M.h_block_ptr[(size_t)(b1 + 1) * d2] != M.h_block_ptr[(size_t)b1 * d2])
          throw Error(DSGDPP_E_STATE, std::string(which ? "test" : "training") +
                                          " entries in row block " + std::to_string(b1) +
                                          ", whose task does not run here (dsgdpp_set_tasks)");
    }
  }
  check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
  if (s0 == 0) {
    wait_inputs_free(c);
    std::memcpy(c->h_schedule, schedule, (size_t)d2 * d * 4);
    fill_epoch_params(c, eps, seeds);
    c->part_seeds.assign(seeds, seeds + d);
  }
  c->part_next = s1 == d2 ? 0 : s1;
  try {
    if (c->cfg.exec == DSGDPP_EXEC_REPLAY) run_replay_epoch(c, eps, seeds, s0, s1);
    else run_hogwild_epoch(c, eps, s0, s1);
  } catch (...) {
    c->part_next = 0;  // a failed part abandons its epoch
    throw;
  }
}

void epoch_explicit_impl(dsgdpp_ctx* c, double eps, const uint32_t* schedule,
                         const uint32_t* seeds) {
  epoch_part_impl(c, eps, schedule, seeds, 0, c->nb2);
}

// ---- losses --------------------------------------------------------------------------
double finish_sum(dsgdpp_ctx* c, uint32_t count) {
  check_cuda(launch_sum_partials(c->d_partials, count, c->d_out, c->stream), "sum_partials");
  check_cuda(cudaMemcpyAsync(c->h_out, c->d_out, 8, cudaMemcpyDeviceToHost, c->stream), "D2H");
  check_cuda(cudaStreamSynchronize(c->stream), "sync");
  return c->h_out[0];
}

// Sums n consecutive runs of loss_grid partials into d_out[0..n) and reads
// them back with one copy and one synchronisation.
void finish_sums(dsgdpp_ctx* c, uint32_t n, double* out) {
  for (uint32_t k = 0; k < n; ++k)
    check_cuda(launch_sum_partials(c->d_partials + (size_t)k * c->loss_grid, c->loss_grid,
                                   c->d_out + k, c->stream), "sum_partials");
  check_cuda(cudaMemcpyAsync(c->h_out, c->d_out, 8 * (size_t)n, cudaMemcpyDeviceToHost, c->stream),
             "D2H");
  check_cuda(cudaStreamSynchronize(c->stream), "sync");
  for (uint32_t k = 0; k < n; ++k) out[k] = c->h_out[k];
}

// The squared errors of the training or test entries as loss_grid partials.
void nzsl_partials(dsgdpp_ctx* c, int which, double* partials) {
  if (which != DSGDPP_TRAIN && which != DSGDPP_TEST) throw Error(DSGDPP_E_INVALID, "which");
  const DevMatrix& M = c->mat[which];
  if (!M.present) throw Error(DSGDPP_E_STATE, which ? "no test matrix" : "no training matrix");
  check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
  if (M.nnz == 0) {
    check_cuda(cudaMemsetAsync(partials, 0, sizeof(double) * c->loss_grid, c->stream), "memset");
    return;
  }
  check_cuda(launch_nzsl_partials(c->cfg.precision, M.row, M.col, M.val, M.nnz, c->W, c->H, c->r,
                                  c->rp, partials, c->loss_grid, c->stream), "nzsl");
}

double nzsl_impl(dsgdpp_ctx* c, int which) {
  nzsl_partials(c, which, c->d_partials);
  double v = 0;
  finish_sums(c, 1, &v);
  return v;
}

double sumsq_impl(dsgdpp_ctx* c, const void* X, uint64_t count) {
  check_cuda(launch_sumsq_partials(c->cfg.precision, X, count, c->d_partials, c->loss_grid,
                                   c->stream), "l2");
  return finish_sum(c, c->loss_grid);
}

double nzl2_impl(dsgdpp_ctx* c, const void* X, uint64_t rows, const uint32_t* cnt) {
  check_cuda(launch_nzl2_partials(c->cfg.precision, X, rows, c->rp, cnt, c->d_partials,
                                  c->loss_grid, c->stream), "nzl2");
  return finish_sum(c, c->loss_grid);
}

// The configured loss (mf/loss/loss.h:88-112 SumLoss of Nzsl and L2/Nzl2):
// its two or three reductions run back to back and come back in one copy.
double loss_impl(dsgdpp_ctx* c) {
  const uint32_t G = c->loss_grid;
  nzsl_partials(c, DSGDPP_TRAIN, c->d_partials);
  uint32_t n = 1;
  if (c->cfg.loss == DSGDPP_LOSS_NZSL_L2) {
    check_cuda(launch_sumsq_partials(c->cfg.precision, c->W, c->cfg.m * c->rp, c->d_partials + G,
                                     G, c->stream), "l2");
    check_cuda(launch_sumsq_partials(c->cfg.precision, c->H, c->cfg.n * c->rp,
                                     c->d_partials + 2 * (size_t)G, G, c->stream), "l2");
    n = 3;
  } else if (c->cfg.loss == DSGDPP_LOSS_NZSL_NZL2) {
    check_cuda(launch_nzl2_partials(c->cfg.precision, c->W, c->cfg.m, c->rp, c->cnt1,
                                    c->d_partials + G, G, c->stream), "nzl2");
    check_cuda(launch_nzl2_partials(c->cfg.precision, c->H, c->cfg.n, c->rp, c->cnt2,
                                    c->d_partials + 2 * (size_t)G, G, c->stream), "nzl2");
    n = 3;
  }
  double v[3] = {0, 0, 0};
  finish_sums(c, n, v);
  double l = v[0];
  if (n == 3) l = l + c->cfg.loss_lambda * (v[1] + v[2]);
  return l;
}

double elapsed_ns(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return (double)std::chrono::duration_cast<std::chrono::nanoseconds>(b - a).count();
}

}  // namespace

// ---- exported ------------------------------------------------------------------------
namespace {
thread_local std::string g_create_error;  // message of this thread's last failed dsgdpp_create
}

extern "C" {

int dsgdpp_abi_version(void) { return DSGDPP_ABI_VERSION; }

const char* dsgdpp_create_error(void) { return g_create_error.c_str(); }

const char* dsgdpp_status_string(int s) {
  switch (s) {
    case DSGDPP_OK: return "ok";
    case DSGDPP_E_INVALID: return "invalid argument";
    case DSGDPP_E_CUDA: return "CUDA error";
    case DSGDPP_E_IO: return "I/O error";
    case DSGDPP_E_UNSUPPORTED: return "not supported";
    case DSGDPP_E_STATE: return "call out of order";
    case DSGDPP_E_NOMEM: return "out of memory";
    default: return "unknown status";
  }
}

void dsgdpp_config_init(dsgdpp_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->rank = 10;
  c->d = 1;
  c->precision = DSGDPP_FP32;
  c->exec = DSGDPP_EXEC_HOGWILD;
  c->launch = DSGDPP_LAUNCH_GRAPH;
  c->update = DSGDPP_UPDATE_NZSL_L2;
  c->update_lambda = 1.0;
  c->regularize = DSGDPP_REGULARIZE_NONE;
  c->loss = DSGDPP_LOSS_NZSL_L2;
  c->loss_lambda = 1.0;
  c->truncate = 0;
  c->truncate_min = NAN;
  c->truncate_max = NAN;
  c->sgd_order = DSGDPP_SGD_WOR;
  c->stratum_order = DSGDPP_STRATUM_COWOR;
  c->device = 0;
  c->layout_seed = 0x5eed5eedull;
  c->layout = DSGDPP_LAYOUT_RUNS;
}

int dsgdpp_create(const dsgdpp_config* cfg, dsgdpp_ctx** out) {
  if (!out) return DSGDPP_E_INVALID;
  *out = nullptr;
  dsgdpp_ctx* c = new (std::nothrow) dsgdpp_ctx();
  if (!c) return DSGDPP_E_NOMEM;
  int rc = guarded(c, [&]() {
    create_impl(c, cfg);
    return DSGDPP_OK;
  });
  if (rc != DSGDPP_OK) {
    g_create_error = c->err;
    destroy_impl(c);
    delete c;
    return rc;
  }
  *out = c;
  return DSGDPP_OK;
}

void dsgdpp_destroy(dsgdpp_ctx* c) {
  if (!c) return;
  destroy_impl(c);
  delete c;
}

const char* dsgdpp_last_error(const dsgdpp_ctx* c) { return c ? c->err.c_str() : "null context"; }

int dsgdpp_set_matrix(dsgdpp_ctx* c, int which, uint64_t nnz, const uint32_t* rows,
                      const uint32_t* cols, const double* vals) {
  return guarded(c, [&]() {
    set_matrix_impl(c, which, nnz, rows, cols, vals);
    return DSGDPP_OK;
  });
}

// small device buffer freed on scope exit (set-up calls only)
struct TempDev {
  void* p = nullptr;
  explicit TempDev(size_t bytes) { check_cuda(cudaMalloc(&p, bytes ? bytes : 1), "cudaMalloc"); }
  ~TempDev() { cudaFree(p); }
};

int dsgdpp_set_blocks(dsgdpp_ctx* c, int which, const uint64_t* block_nnz,
                      const uint32_t* local_rows, const uint32_t* local_cols,
                      const double* vals) {
  return guarded(c, [&]() {
    if (!block_nnz) throw Error(DSGDPP_E_INVALID, "null block_nnz");
    const uint32_t nblocks = c->d * c->nb2;
    std::vector<uint64_t> start(nblocks + 1, 0);
    for (uint32_t b = 0; b < nblocks; ++b) start[b + 1] = start[b] + block_nnz[b];
    const uint64_t nnz = start[nblocks];
    if (nnz > 0 && (!local_rows || !local_cols || !vals))
      throw Error(DSGDPP_E_INVALID, "null input array");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    const DeviceFill fill = [&](uint32_t* r, uint32_t* col, double* v, cudaStream_t st) {
      TempDev tmp((nblocks + 1) * 8 + 8);
      uint64_t* d_start = static_cast<uint64_t*>(tmp.p);
      unsigned long long* d_bad = reinterpret_cast<unsigned long long*>(d_start + nblocks + 1);
      check_cuda(cudaMemcpyAsync(r, local_rows, nnz * 4, cudaMemcpyHostToDevice, st), "H2D rows");
      check_cuda(cudaMemcpyAsync(col, local_cols, nnz * 4, cudaMemcpyHostToDevice, st), "H2D cols");
      check_cuda(cudaMemcpyAsync(v, vals, nnz * 8, cudaMemcpyHostToDevice, st), "H2D vals");
      check_cuda(cudaMemcpyAsync(d_start, start.data(), (nblocks + 1) * 8, cudaMemcpyHostToDevice,
                                 st), "H2D block starts");
      check_cuda(cudaMemsetAsync(d_bad, 0, 8, st), "memset");
      check_cuda(launch_shift_blocks(d_start, nblocks, c->nb2, c->d_off1, c->d_off2, nnz, r, col,
                                     d_bad, st), "shift_blocks");
      unsigned long long bad = 0;
      check_cuda(cudaMemcpyAsync(&bad, d_bad, 8, cudaMemcpyDeviceToHost, st), "D2H");
      check_cuda(cudaStreamSynchronize(st), "sync");
      if (bad)
        throw Error(DSGDPP_E_INVALID, std::to_string(bad) + " entries lie outside their block");
    };
    set_matrix_impl(c, which, nnz, nullptr, nullptr, nullptr, &fill);
    return DSGDPP_OK;
  });
}

int dsgdpp_set_counts(dsgdpp_ctx* c, const uint64_t* nnz1, const uint64_t* nnz2) {
  return guarded(c, [&]() {
    if (!nnz1 || !nnz2) throw Error(DSGDPP_E_INVALID, "null count array");
    if (!c->mat[DSGDPP_TRAIN].present) throw Error(DSGDPP_E_STATE, "no training matrix");
    const uint64_t m = c->cfg.m, n = c->cfg.n;
    for (uint64_t i = 0; i < m; ++i)
      if (nnz1[i] >> 32) throw Error(DSGDPP_E_INVALID, "a row count exceeds 2^32 - 1");
    for (uint64_t j = 0; j < n; ++j)
      if (nnz2[j] >> 32) throw Error(DSGDPP_E_INVALID, "a column count exceeds 2^32 - 1");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    cudaStream_t st = c->stream;
    check_cuda(cudaStreamSynchronize(st), "sync");
    TempDev tmp((m + n) * 8);
    uint64_t* d = static_cast<uint64_t*>(tmp.p);
    check_cuda(cudaMemcpyAsync(d, nnz1, m * 8, cudaMemcpyHostToDevice, st), "H2D nnz1");
    check_cuda(cudaMemcpyAsync(d + m, nnz2, n * 8, cudaMemcpyHostToDevice, st), "H2D nnz2");
    check_cuda(launch_counts_to_u32(d, m, c->cnt1, st), "nnz1");
    check_cuda(launch_counts_to_u32(d + m, n, c->cnt2, st), "nnz2");
    if (c->inv1) {
      const bool as_double = c->cfg.precision == kFp64;
      check_cuda(launch_inverse_counts(c->cnt1, m, c->inv1, as_double, st), "inv1");
      check_cuda(launch_inverse_counts(c->cnt2, n, c->inv2, as_double, st), "inv2");
    }
    check_cuda(cudaStreamSynchronize(st), "sync");
    return DSGDPP_OK;
  });
}

int dsgdpp_set_matrix_rm(dsgdpp_ctx* c, int which, const dsgdpp_rm* rm) {
  return guarded(c, [&]() {
    if (!rm) throw Error(DSGDPP_E_INVALID, "null descriptor");
    const RmDesc& d = rm->d;
    if (!d.has_data()) throw Error(DSGDPP_E_INVALID, "the descriptor holds no data matrix");
    if (d.size1 != c->cfg.m || d.size2 != c->cfg.n)
      throw Error(DSGDPP_E_INVALID, "descriptor size " + std::to_string(d.size1) + " x " +
                                        std::to_string(d.size2) + " differs from the context's");
    const uint64_t nnz = rm_count(d, which == DSGDPP_TEST ? 1 : 0);
    const DeviceFill fill = [&](uint32_t* r, uint32_t* col, double* v, cudaStream_t st) {
      try {
        rm_data_device(d, which == DSGDPP_TEST ? 1 : 0, r, col, v, st);
      } catch (const std::invalid_argument& e) {
        throw Error(DSGDPP_E_INVALID, e.what());
      } catch (const std::runtime_error& e) {
        throw Error(DSGDPP_E_CUDA, e.what());
      }
    };
    set_matrix_impl(c, which, nnz, nullptr, nullptr, nullptr, &fill);
    return DSGDPP_OK;
  });
}

int dsgdpp_set_factors_rm(dsgdpp_ctx* c, const dsgdpp_rm* rm) {
  return guarded(c, [&]() {
    if (!rm) throw Error(DSGDPP_E_INVALID, "null descriptor");
    const RmDesc& d = rm->d;
    if (d.size1 != c->cfg.m || d.size2 != c->cfg.n || d.rank != c->r)
      throw Error(DSGDPP_E_INVALID, "descriptor " + std::to_string(d.size1) + " x " +
                                        std::to_string(d.size2) + ", rank " +
                                        std::to_string(d.rank) + " does not fit the context");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    ensure_staging(c);
    const uint64_t m = c->cfg.m, r = c->r;
    cudaStream_t st = c->stream;
    try {
      rm_factors_device(d, c->staging, c->staging + m * r, st);
    } catch (const std::runtime_error& e) {
      throw Error(DSGDPP_E_CUDA, e.what());
    }
    check_cuda(launch_factor_to_device(c->cfg.precision, c->staging, m, c->r, c->rp, c->W, st), "W");
    check_cuda(launch_factor_to_device(c->cfg.precision, c->staging + m * r, c->cfg.n, c->r, c->rp,
                                       c->H, st), "H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    c->factors_set = true;
    return DSGDPP_OK;
  });
}

int dsgdpp_set_factors(dsgdpp_ctx* c, const double* W, const double* H) {
  return guarded(c, [&]() {
    if (!W || !H) throw Error(DSGDPP_E_INVALID, "null factor array");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    ensure_staging(c);
    const uint64_t m = c->cfg.m, n = c->cfg.n, r = c->r;
    cudaStream_t st = c->stream;
    check_cuda(cudaMemcpyAsync(c->staging, W, m * r * 8, cudaMemcpyHostToDevice, st), "H2D W");
    check_cuda(cudaMemcpyAsync(c->staging + m * r, H, n * r * 8, cudaMemcpyHostToDevice, st), "H2D H");
    check_cuda(launch_factor_to_device(c->cfg.precision, c->staging, m, c->r, c->rp, c->W, st), "W");
    check_cuda(launch_factor_to_device(c->cfg.precision, c->staging + m * r, n, c->r, c->rp, c->H,
                                       st), "H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    c->factors_set = true;
    return DSGDPP_OK;
  });
}

int dsgdpp_get_factors(dsgdpp_ctx* c, double* W, double* H) {
  return guarded(c, [&]() {
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    ensure_staging(c);
    const uint64_t m = c->cfg.m, n = c->cfg.n, r = c->r;
    cudaStream_t st = c->stream;
    check_cuda(launch_factor_to_host(c->cfg.precision, c->W, m, c->r, c->rp, c->staging, st), "W");
    check_cuda(launch_factor_to_host(c->cfg.precision, c->H, n, c->r, c->rp, c->staging + m * r,
                                     st), "H");
    if (W) check_cuda(cudaMemcpyAsync(W, c->staging, m * r * 8, cudaMemcpyDeviceToHost, st), "D2H W");
    if (H)
      check_cuda(cudaMemcpyAsync(H, c->staging + m * r, n * r * 8, cudaMemcpyDeviceToHost, st),
                 "D2H H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    return DSGDPP_OK;
  });
}

int dsgdpp_block_nnz(dsgdpp_ctx* c, int which, uint64_t* out) {
  return guarded(c, [&]() {
    if (which != DSGDPP_TRAIN && which != DSGDPP_TEST) throw Error(DSGDPP_E_INVALID, "which");
    const DevMatrix& M = c->mat[which];
    if (!M.present) throw Error(DSGDPP_E_STATE, "matrix not set");
    const size_t nb = (size_t)c->d * c->nb2;
    for (size_t b = 0; b < nb; ++b) out[b] = M.h_block_ptr[b + 1] - M.h_block_ptr[b];
    return DSGDPP_OK;
  });
}

int dsgdpp_nnz12(dsgdpp_ctx* c, uint64_t* nnz1, uint64_t* nnz2, uint64_t* nnz12max) {
  return guarded(c, [&]() {
    if (!c->mat[0].present) throw Error(DSGDPP_E_STATE, "no training matrix");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    std::vector<uint32_t> a(c->cfg.m), b(c->cfg.n);
    check_cuda(cudaMemcpy(a.data(), c->cnt1, c->cfg.m * 4, cudaMemcpyDeviceToHost), "D2H");
    check_cuda(cudaMemcpy(b.data(), c->cnt2, c->cfg.n * 4, cudaMemcpyDeviceToHost), "D2H");
    uint64_t mx = 0;
    for (uint64_t i = 0; i < c->cfg.m; ++i) {
      if (nnz1) nnz1[i] = a[i];
      mx = std::max<uint64_t>(mx, a[i]);
    }
    for (uint64_t j = 0; j < c->cfg.n; ++j) {
      if (nnz2) nnz2[j] = b[j];
      mx = std::max<uint64_t>(mx, b[j]);
    }
    if (nnz12max) *nnz12max = mx;
    return DSGDPP_OK;
  });
}

int dsgdpp_seed(dsgdpp_ctx* c, uint32_t seed) {
  return guarded(c, [&]() {
    c->master.seed_with(seed);
    return DSGDPP_OK;
  });
}

int dsgdpp_epoch(dsgdpp_ctx* c, double eps) {
  TraceRange range("epoch");
  return guarded(c, [&]() {
    const uint32_t d = c->d;
    std::vector<uint32_t> sched((size_t)c->nb2 * d), seeds(d);
    draw_epoch(c, sched.data(), seeds.data());
    epoch_explicit_impl(c, eps, sched.data(), seeds.data());
    return DSGDPP_OK;
  });
}

int dsgdpp_epoch_explicit(dsgdpp_ctx* c, double eps, const uint32_t* schedule,
                          const uint32_t* task_seeds) {
  TraceRange range("epoch");
  return guarded(c, [&]() {
    epoch_explicit_impl(c, eps, schedule, task_seeds);
    return DSGDPP_OK;
  });
}

int dsgdpp_epoch_part(dsgdpp_ctx* c, double eps, const uint32_t* schedule,
                      const uint32_t* task_seeds, uint32_t s_begin, uint32_t s_end) {
  TraceRange range(s_end - s_begin == 1 ? "subepoch" : "epoch");
  return guarded(c, [&]() {
    epoch_part_impl(c, eps, schedule, task_seeds, s_begin, s_end);
    return DSGDPP_OK;
  });
}

int dsgdpp_set_tasks(dsgdpp_ctx* c, uint32_t first, uint32_t count) {
  return guarded(c, [&]() {
    if (count == 0 || first >= c->d || count > c->d - first)
      throw Error(DSGDPP_E_INVALID, "task range out of bounds");
    if (c->part_next != 0) throw Error(DSGDPP_E_STATE, "an epoch given in parts is unfinished");
    c->task_lo = first;
    c->task_hi = first + count;
    return DSGDPP_OK;
  });
}

int dsgdpp_h_block_bytes(dsgdpp_ctx* c, uint32_t b2, uint64_t* bytes) {
  return guarded(c, [&]() {
    if (!bytes || b2 >= c->nb2) throw Error(DSGDPP_E_INVALID, "column block out of range");
    *bytes = (c->off2[b2 + 1] - c->off2[b2]) * c->rp * elem_size(c->cfg.precision);
    return DSGDPP_OK;
  });
}

int dsgdpp_h_block_copy(dsgdpp_ctx* c, uint32_t b2, void* device_buf, int to_context) {
  return guarded(c, [&]() {
    if (!device_buf || b2 >= c->nb2) throw Error(DSGDPP_E_INVALID, "column block out of range");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    const size_t es = elem_size(c->cfg.precision);
    const size_t bytes = (c->off2[b2 + 1] - c->off2[b2]) * c->rp * es;
    char* blk = static_cast<char*>(c->H) + c->off2[b2] * c->rp * es;
    cudaStream_t st = c->stream;
    if (to_context)
      check_cuda(cudaMemcpyAsync(blk, device_buf, bytes, cudaMemcpyDefault, st), "copy into H");
    else
      check_cuda(cudaMemcpyAsync(device_buf, blk, bytes, cudaMemcpyDefault, st), "copy from H");
    check_cuda(cudaStreamSynchronize(st), "sync");
    return DSGDPP_OK;
  });
}

int dsgdpp_last_epoch_ms(dsgdpp_ctx* c, double* ms) {
  return guarded(c, [&]() {
    if (!ms) throw Error(DSGDPP_E_INVALID, "null output");
    if (!c->epoch_timed) throw Error(DSGDPP_E_STATE, "no epoch has run");
    check_cuda(cudaEventSynchronize(c->ev_end), "event sync");
    float f = 0;
    check_cuda(cudaEventElapsedTime(&f, c->ev_begin, c->ev_end), "elapsed");
    *ms = f;
    return DSGDPP_OK;
  });
}

int dsgdpp_set_wait_limit(dsgdpp_ctx* c, double seconds) {
  return guarded(c, [&]() {
    if (!(seconds >= 0) || seconds > 3600)
      throw Error(DSGDPP_E_INVALID, "the wait limit must be in [0, 3600] seconds");
    const uint64_t ns = (uint64_t)(seconds * 1e9);
    if (ns != c->wait_ns) {
      c->wait_ns = ns;
      release_graph(c);  // the limit is a launch argument: capture the epoch again
    }
    return DSGDPP_OK;
  });
}

int dsgdpp_set_kernel_timing(dsgdpp_ctx* c, int on) {
  return guarded(c, [&]() {
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    collect_profile(c);
    if (on && c->prof_ev.empty()) {
      c->prof_ev.resize(c->nb2 + 1);
      for (auto& e : c->prof_ev) check_cuda(cudaEventCreate(&e), "event");
    }
    c->profiling = on != 0;
    c->prof_ms = 0;
    c->prof_launches = 0;
    return DSGDPP_OK;
  });
}

int dsgdpp_kernel_timing(dsgdpp_ctx* c, double* total_ms, uint64_t* launches) {
  return guarded(c, [&]() {
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    collect_profile(c);
    if (total_ms) *total_ms = c->prof_ms;
    if (launches) *launches = c->prof_launches;
    return DSGDPP_OK;
  });
}

int dsgdpp_launch_shape(dsgdpp_ctx* c, uint32_t* lanes, uint32_t* vecs, uint32_t* grid) {
  return guarded(c, [&]() {
    if (lanes) *lanes = c->lanes;
    if (vecs) *vecs = c->vecs;
    if (grid) *grid = c->grid;
    return DSGDPP_OK;
  });
}

int dsgdpp_loss(dsgdpp_ctx* c, double* out) {
  TraceRange range("loss");
  return guarded(c, [&]() {
    if (!out) throw Error(DSGDPP_E_INVALID, "null output");
    *out = loss_impl(c);
    return DSGDPP_OK;
  });
}

int dsgdpp_nzsl(dsgdpp_ctx* c, int which, double* out) {
  TraceRange range("loss");
  return guarded(c, [&]() {
    if (!out) throw Error(DSGDPP_E_INVALID, "null output");
    *out = nzsl_impl(c, which);
    return DSGDPP_OK;
  });
}

int dsgdpp_l2(dsgdpp_ctx* c, double* w2, double* h2) {
  TraceRange range("loss");
  return guarded(c, [&]() {
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    if (w2) *w2 = sumsq_impl(c, c->W, c->cfg.m * c->rp);
    if (h2) *h2 = sumsq_impl(c, c->H, c->cfg.n * c->rp);
    return DSGDPP_OK;
  });
}

int dsgdpp_nzl2(dsgdpp_ctx* c, double* w, double* h) {
  TraceRange range("loss");
  return guarded(c, [&]() {
    if (!c->mat[0].present) throw Error(DSGDPP_E_STATE, "no training matrix");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    if (w) *w = nzl2_impl(c, c->W, c->cfg.m, c->cnt1);
    if (h) *h = nzl2_impl(c, c->H, c->cfg.n, c->cnt2);
    return DSGDPP_OK;
  });
}

int dsgdpp_run(dsgdpp_ctx* c, uint32_t epochs, int decay, double eps0, double decrease,
               double increase, dsgdpp_trace_row* trace) {
  return guarded(c, [&]() {
    if (decay != DSGDPP_DECAY_CONST && decay != DSGDPP_DECAY_BOLDDRIVER)
      throw Error(DSGDPP_E_INVALID, "unknown decay");
    using clock = std::chrono::steady_clock;
    const bool has_test = c->mat[1].present;
    auto t0 = clock::now();
    double cur = loss_impl(c);
    auto t1 = clock::now();
    double test = has_test ? nzsl_impl(c, DSGDPP_TEST) : NAN;
    auto t2 = clock::now();
    if (trace) {
      trace[0] = dsgdpp_trace_row{0, cur, test, NAN, 0, 0, elapsed_ns(t0, t1),
                                  has_test ? elapsed_ns(t1, t2) : 0.0};
    }
    double prev = 0, eps_state = eps0;
    const uint32_t d = c->d;
    std::vector<uint32_t> sched((size_t)c->nb2 * d), seeds(d);
    for (uint32_t e = 0; e < epochs; ++e) {
      auto a = clock::now();
      double eps;
      if (decay == DSGDPP_DECAY_CONST) {
        eps = eps0;
      } else if (e == 0) {
        eps = eps_state;  // BoldDriver: the first call returns the initial step
      } else {
        eps_state *= (prev <= cur) ? decrease : increase;  // decay_bolddriver.h:59-67
        eps = eps_state;
      }
      auto b = clock::now();
      draw_epoch(c, sched.data(), seeds.data());
      epoch_explicit_impl(c, eps, sched.data(), seeds.data());
      check_cuda(cudaEventSynchronize(c->ev_end), "event sync");
      auto e1 = clock::now();
      prev = cur;
      cur = loss_impl(c);
      auto e2 = clock::now();
      test = has_test ? nzsl_impl(c, DSGDPP_TEST) : NAN;
      auto e3 = clock::now();
      if (trace)
        trace[e + 1] = dsgdpp_trace_row{e + 1u, cur, test, eps, elapsed_ns(a, b), elapsed_ns(b, e1),
                                        elapsed_ns(e1, e2), has_test ? elapsed_ns(e2, e3) : 0.0};
    }
    return DSGDPP_OK;
  });
}

int dsgdpp_save_factors(dsgdpp_ctx* c) {
  return guarded(c, [&]() {
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    const size_t es = elem_size(c->cfg.precision);
    if (!c->W_saved) {
      check_cuda(cudaMalloc(&c->W_saved, c->cfg.m * c->rp * es), "W snapshot");
      check_cuda(cudaMalloc(&c->H_saved, c->cfg.n * c->rp * es), "H snapshot");
    }
    check_cuda(cudaMemcpyAsync(c->W_saved, c->W, c->cfg.m * c->rp * es, cudaMemcpyDeviceToDevice,
                               c->stream), "save W");
    check_cuda(cudaMemcpyAsync(c->H_saved, c->H, c->cfg.n * c->rp * es, cudaMemcpyDeviceToDevice,
                               c->stream), "save H");
    return DSGDPP_OK;
  });
}

int dsgdpp_restore_factors(dsgdpp_ctx* c) {
  return guarded(c, [&]() {
    if (!c->W_saved) throw Error(DSGDPP_E_STATE, "no saved factors");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    const size_t es = elem_size(c->cfg.precision);
    check_cuda(cudaMemcpyAsync(c->W, c->W_saved, c->cfg.m * c->rp * es, cudaMemcpyDeviceToDevice,
                               c->stream), "restore W");
    check_cuda(cudaMemcpyAsync(c->H, c->H_saved, c->cfg.n * c->rp * es, cudaMemcpyDeviceToDevice,
                               c->stream), "restore H");
    return DSGDPP_OK;
  });
}

int dsgdpp_update_norms(dsgdpp_ctx* c, double* mean, double* max) {
  return guarded(c, [&]() {
    if (!c->W_saved) throw Error(DSGDPP_E_STATE, "no saved factors");
    check_cuda(cudaSetDevice(c->cfg.device), "cudaSetDevice");
    double sum = 0, mx = 0;
    const struct { const void* x; const void* old; uint64_t rows; } parts[2] = {
        {c->W, c->W_saved, c->cfg.m}, {c->H, c->H_saved, c->cfg.n}};
    for (const auto& p : parts) {
      check_cuda(launch_update_norms(c->cfg.precision, p.x, p.old, p.rows, c->rp, c->d_partials,
                                     c->loss_grid, c->d_out, c->stream), "update norms");
      check_cuda(cudaMemcpyAsync(c->h_out, c->d_out, 16, cudaMemcpyDeviceToHost, c->stream), "D2H");
      check_cuda(cudaStreamSynchronize(c->stream), "sync");
      sum += c->h_out[0];
      mx = std::max(mx, c->h_out[1]);
    }
    if (mean) *mean = sum / (double)(c->cfg.m + c->cfg.n);
    if (max) *max = mx;
    return DSGDPP_OK;
  });
}

int dsgdpp_sync(dsgdpp_ctx* c) {
  return guarded(c, [&]() {
    check_cuda(cudaStreamSynchronize(c->stream), "sync");
    return DSGDPP_OK;
  });
}

// ---- host utilities ------------------------------------------------------------------
struct dsgdpp_rng {
  Random32 r;
};

dsgdpp_rng* dsgdpp_rng_create(uint32_t seed) {
  auto* g = new (std::nothrow) dsgdpp_rng();
  if (g) g->r.seed_with(seed);
  return g;
}
void dsgdpp_rng_destroy(dsgdpp_rng* g) { delete g; }
uint32_t dsgdpp_rng_next(dsgdpp_rng* g) { return g->r.next(); }
uint32_t dsgdpp_rng_next_int(dsgdpp_rng* g, uint32_t n) { return g->r.next_int(n); }

void dsgdpp_draw_schedule(dsgdpp_rng* g, uint32_t d, int order, uint32_t* schedule,
                          uint32_t* seeds) {
  dsgdpp_schedule(g->r, d, order, schedule, seeds);
}

void dsgdpp_dsgd_schedule(dsgdpp_rng* g, uint32_t w, uint32_t t, int order, uint32_t* out) {
  std::vector<uint32_t> s = dsgd_schedule(w, t, order, g->r);
  std::copy(s.begin(), s.end(), out);
}

uint64_t dsgdpp_point_orders(uint32_t d, int sgd_order, const uint64_t* block_nnz,
                             const uint32_t* schedule, const uint32_t* seeds, uint32_t* out) {
  const uint32_t d2 = 2 * d;
  std::vector<TaskOrder> tasks;
  tasks.reserve(d);
  for (uint32_t id = 0; id < d; ++id) tasks.emplace_back(seeds[id]);
  uint64_t at = 0;
  std::vector<uint32_t> tmp;
  for (uint32_t s = 0; s < d2; ++s)
    for (uint32_t id = 0; id < d; ++id) {
      const uint64_t n = block_nnz[(size_t)id * d2 + schedule[(size_t)s * d + id]];
      uint32_t* dst = out;
      if (out) dst = out + at;
      else { tmp.resize(n); dst = tmp.data(); }
      tasks[id].next_block(sgd_order, n, dst);
      at += n;
    }
  return at;
}

void dsgdpp_block_offsets(uint64_t size, uint32_t blocks, uint64_t* out) {
  std::vector<uint64_t> o = block_offsets(size, blocks);
  std::copy(o.begin(), o.end(), out);
}

void dsgdpp_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  Philox4 r = philox4x32_10(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
  for (int k = 0; k < 4; ++k) out[k] = r.v[k];
}

}  // extern "C"
