// context.h -- the device-side state behind a dsgdpp_ctx (internal to the library).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/dsgdpp.h"
#include "kernels.cuh"
#include "schedule.h"

namespace dsgdpp {

struct DevMatrix {
  bool present = false;
  uint64_t nnz = 0;
  uint32_t* row = nullptr;
  uint32_t* col = nullptr;
  void* val = nullptr;
  uint64_t* block_ptr = nullptr;
  uint32_t nblocks = 0;  // entries of block_ptr minus one
  uint64_t cap = 0;      // records the row/col/val arrays hold
  std::vector<uint64_t> h_block_ptr;
};

class Error {
 public:
  Error(int code, std::string msg) : code(code), msg(std::move(msg)) {}
  int code;
  std::string msg;
};

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw Error(e == cudaErrorMemoryAllocation ? DSGDPP_E_NOMEM : DSGDPP_E_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
inline T* dalloc(size_t count, const char* what) {
  void* p = nullptr;
  if (count == 0) count = 1;
  check_cuda(cudaMalloc(&p, count * sizeof(T)), what);
  return static_cast<T*>(p);
}
template <typename T>
inline T* halloc(size_t count, const char* what) {
  void* p = nullptr;
  if (count == 0) count = 1;
  check_cuda(cudaMallocHost(&p, count * sizeof(T)), what);
  return static_cast<T*>(p);
}
template <typename T>
inline void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}
template <typename T>
inline void hfree(T*& p) {
  if (p) cudaFreeHost((void*)p);
  p = nullptr;
}

inline uint32_t vec_width(int precision) { return precision == kFp64 ? 2 : (precision == kFp32 ? 4 : 8); }
inline size_t elem_size(int precision) { return precision == kFp64 ? 8 : (precision == kFp32 ? 4 : 2); }

}  // namespace dsgdpp

struct dsgdpp_ctx {
  using DevMatrix = dsgdpp::DevMatrix;
  using EpochParams = dsgdpp::EpochParams;
  using Segment = dsgdpp::Segment;
  using Random32 = dsgdpp::Random32;
  dsgdpp_config cfg{};
  std::string err;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  uint32_t d = 0, r = 0, rp = 0;
  uint32_t nb2 = 0;  // column blocks = sub-epochs per epoch: 2d (DSGD++) or d (DSGD)
  std::vector<uint64_t> off1, off2;  // with the end offset appended
  uint64_t* d_off1 = nullptr;
  uint64_t* d_off2 = nullptr;
  DevMatrix mat[2];
  void* W = nullptr;
  void* H = nullptr;
  bool factors_set = false;
  uint32_t* cnt1 = nullptr;
  uint32_t* cnt2 = nullptr;
  void* inv1 = nullptr;
  void* inv2 = nullptr;
  double* staging = nullptr;  // (m + n) * r doubles, factor upload / download
  void* scratch = nullptr;    // blocking scratch of set_matrix, grown on demand
  size_t scratch_bytes = 0;
  void* W_saved = nullptr;    // factor snapshot (dsgdpp_save_factors)
  void* H_saved = nullptr;
  // per-epoch inputs (pinned host copies feed the device copies)
  uint32_t* h_schedule = nullptr;
  uint32_t* d_schedule = nullptr;
  EpochParams* h_params = nullptr;
  EpochParams* d_params = nullptr;
  float* h_sigma = nullptr;   // [2d][d][3]
  float* d_sigma = nullptr;
  float* h_scales = nullptr;  // [2d + 1]
  float* d_scales = nullptr;
  Segment* d_segs = nullptr;
  dsgdpp::LaunchDesc* d_launches = nullptr;
  uint32_t* d_counters = nullptr;
  // persistent epoch
  uint32_t* d_done = nullptr;     // [2d][d] finished chunks per segment
  int32_t* d_dep_col = nullptr;   // [2d][d] last earlier segment on the same H block
  int32_t* h_dep_col = nullptr;
  uint32_t* d_ticket = nullptr;   // [0] chunk ticket, [1] error flag
  uint32_t* h_error = nullptr;    // error flag read back after each epoch
  uint64_t wait_ns = 1000000000ull;  // dependency wait limit (dsgdpp_set_wait_limit)
  // replay
  uint32_t* h_positions = nullptr;
  uint32_t* d_positions = nullptr;
  uint64_t positions_cap = 0;
  uint64_t* h_pos_offset = nullptr;
  uint64_t* d_pos_offset = nullptr;
  uint8_t* h_mask = nullptr;  // [2d][2d]
  uint8_t* d_mask = nullptr;
  // losses
  double* d_partials = nullptr;
  double* d_out = nullptr;
  double* h_out = nullptr;
  uint32_t loss_grid = 0;
  // Hogwild launch shape
  uint32_t lanes = 0, vecs = 0, grid = 0;
  int atomic_writes = 0;
  int layout_key = 0;  // kLayout* of the Hogwild training records
  // graph of one Hogwild epoch
  cudaGraphExec_t graph_exec = nullptr;
  // timing / ordering
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr, ev_inputs = nullptr;
  // set_matrix: the values travel on a side stream while the keys are sorted
  cudaStream_t side = nullptr;
  cudaEvent_t ev_coords = nullptr, ev_vals = nullptr;
  bool epoch_timed = false;
  // an epoch given in parts: the next sub-epoch to run (0 = none pending) and
  // the task seeds of its first part
  uint32_t part_next = 0;
  std::vector<uint32_t> part_seeds;
  // per-kernel timing of the Hogwild sub-epoch kernels (stream launch only)
  bool profiling = false;
  std::vector<cudaEvent_t> prof_ev;  // 2d + 1 events around the sub-epoch kernels
  double prof_ms = 0;                // summed sub-epoch kernel time of profiled epochs
  uint64_t prof_launches = 0;
  bool prof_pending = false;
  Random32 master{0};
  uint32_t epoch_counter = 0;
  // tasks [task_lo, task_hi) run here (dsgdpp_set_tasks; all d by default)
  uint32_t task_lo = 0, task_hi = 0;
};

namespace dsgdpp {
// The master generator's draws of one epoch (schedule [nb2][d], d task seeds).
void draw_epoch(dsgdpp_ctx* c, uint32_t* sched, uint32_t* seeds);
}  // namespace dsgdpp

