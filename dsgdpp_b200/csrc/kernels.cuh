// kernels.cuh -- argument blocks and host launchers of the DSGD++ kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"

namespace dsgdpp {

enum Precision : int { kFp64 = 0, kFp32 = 1, kBf16 = 2 };
enum UpdateKind : int { kUpdNzsl = 0, kUpdNzslL2 = 1, kUpdNzslNzl2 = 2 };

// Parameters that change every epoch live in device memory so a captured
// graph of the epoch stays valid.
struct EpochParams {
  double eps;
  uint32_t key0, key1;  // Philox key: drawn from the task seeds of the epoch
  uint32_t epoch;       // epoch counter (Philox counter word)
  uint32_t pad;
};

// Hogwild sub-epoch: all records of the sub-epoch's d conflict-free blocks are
// one work list of 32-record chunks; a warp takes a chunk, and 32/LPN groups
// of LPN lanes update 32/LPN records at a time, lanes spanning the rank.
struct HogwildArgs {
  const uint32_t* row;
  const uint32_t* col;
  const void* val;       // float (fp32/bf16 factors) or double (fp64 factors)
  const void* inv1;      // 1/nnz1 per row (float or double, as the compute type)
  const void* inv2;      // 1/nnz2 per column
  void* W;               // m x rp
  void* H;               // n x rp (column j of H is contiguous)
  const Segment* segs;          // segment tables of all launches
  const LaunchDesc* launches;   // per launch: its segments and work counter
  uint32_t* counters;           // work counters (zeroed before the launches)
  const EpochParams* params;
  uint32_t smem_segs;           // > 0: every launch's table (at most this many entries) is
                                // staged in shared memory; 0: searched in global memory
  uint32_t r, rp;
  int update, truncate, sgd_order;
  int atomic;                   // 1: write the update atomically (vector atomic add)
  int runs;                     // 1: records come in runs of one H row (see the kernel)
  int swap_sides;               // 1: W/H (and row/col, inv1/inv2) are passed swapped
  double lambda, tmin, tmax;
};

// Deterministic FP64 replay: one warp per task walks its block in the
// host-generated point order; d blocks of a sub-epoch run side by side.
struct ReplayArgs {
  const uint32_t* row;
  const uint32_t* col;
  const double* val;
  const uint32_t* cnt1;  // nnz1 per row
  const uint32_t* cnt2;  // nnz2 per column
  double* W;
  double* H;
  const uint64_t* block_ptr;  // d*nb2+1
  const uint32_t* schedule;   // [nb2][d]
  const uint32_t* positions;  // point order, concatenated per (sub-epoch, task)
  const uint64_t* pos_offset; // [nb2*d+1]
  const EpochParams* params;
  uint32_t d, r, rp;
  uint32_t nb2;               // column blocks (2d for DSGD++, d for DSGD)
  int update, truncate;
  double lambda, tmin, tmax;
};

struct SegBuildArgs {
  const EpochParams* params;  // eps of the epoch
  const uint32_t* schedule;   // [nb2][d]
  const uint64_t* block_ptr;  // d*nb2+1
  const float* sigma;         // [nb2][d][3] lazy L2 scales, or null (all ones)
  Segment* segs;              // [nb2][d+1]
  uint32_t* counters;         // [nb2]
  uint32_t d;
  uint32_t nb2;               // column blocks = sub-epochs (2d for DSGD++, d for DSGD)
};

// Persistent epoch: one launch walks every sub-epoch; a chunk of segment
// (s, i) starts once segment (s-1, i) -- the task's previous block, on the same
// rows of W -- and the last earlier segment on the same column block of H
// (dep_col) have finished all their chunks.
struct EpochDeps {
  const int32_t* dep_col;  // [nsub][d]: s2 * d + j of that segment, or -1
  uint32_t* done;          // [nsub][d] chunks finished per segment (zeroed per epoch)
  uint32_t* ticket;        // chunks handed out (zeroed per epoch)
  uint32_t* error;         // set when a dependency wait gave up
  uint32_t d;
  uint32_t nsub;           // sub-epochs (2d for DSGD++, d for DSGD)
  uint64_t wait_ns;        // a dependency wait gives up after this long
};

// Threads per CTA of a Hogwild sub-epoch kernel instance.  Registers are
// allocated per warp, so small CTAs pack more warps onto an SM when a
// CTA's registers do not divide the SM's: CTAs of 4 warps for FP32 and FP64
// (72 registers fit 28 warps per SM in CTAs of 4 warps, 24 in CTAs of 8;
// measured 6.9 against 7.5 ms per epoch at rank 32) and for BF16 with up to
// 4 lanes per entry (held to 73 registers without spills: 6.55 against 6.81
// ms at rank 32); CTAs of 8 warps for wider BF16 mappings (held to 64
// registers, 4 CTAs per SM, which measured faster at ranks 64 and 128).  A
// cap of CTAs per SM in a configuration counts CTAs of 256 threads, so it is
// scaled by hogwild_cta_scale.
constexpr int hogwild_threads(int precision, uint32_t lanes) {
  return precision == kBf16 && lanes > 4 ? 256 : 128;
}
constexpr int hogwild_cta_scale(int precision, uint32_t lanes) {
  return 256 / hogwild_threads(precision, lanes);
}

// ---- launchers (return cudaError_t) -------------------------------------------
cudaError_t launch_build_segments(const SegBuildArgs& a, cudaStream_t st);
// after_subepoch: the launch directly follows the sub-epoch launch before it
// in the stream (nothing in between), so its start may overlap that launch's
// end (programmatic dependent launch; the kernel waits for the previous grid
// before it touches a factor)
cudaError_t launch_hogwild(int precision, uint32_t lanes, uint32_t vecs, const HogwildArgs& a,
                           uint32_t launch_index, uint32_t grid, cudaStream_t st,
                           bool after_subepoch = false);
// CTAs per SM that the Hogwild kernel sustains for this configuration
int hogwild_ctas_per_sm(int precision, uint32_t lanes, uint32_t vecs, bool atomic,
                        uint32_t smem_segs, bool runs);
// the persistent epoch (column / row runs, atomic writes, SEQ or WOR order)
cudaError_t launch_hogwild_epoch(int precision, uint32_t lanes, uint32_t vecs, const HogwildArgs& a,
                                 const EpochDeps& dp, uint32_t grid, cudaStream_t st);
int hogwild_epoch_ctas_per_sm(int precision, uint32_t lanes, uint32_t vecs, uint32_t nsub);
cudaError_t launch_replay_subepoch(const ReplayArgs& a, uint32_t s, cudaStream_t st);
// RegularizeL2 after sub-epoch s, exactly as the reference (all W, stratum H)
cudaError_t launch_regularize_exact(double* W, double* H, uint64_t m, uint64_t n, uint32_t rp,
                                    uint32_t r, const uint64_t* off2, const uint8_t* mask,
                                    uint32_t d, uint32_t nb2, const EpochParams* params, double lambda,
                                    int truncate, double tmin, double tmax, cudaStream_t st);
// Lazy-L2 normalisation at the end of a Hogwild epoch: H column block b2 is
// multiplied by scales[b2], all of W by scales[nb2] (device memory)
cudaError_t launch_normalize(int precision, void* W, void* H, uint64_t m, uint64_t n,
                             uint32_t rp, const float* scales, const uint64_t* off2,
                             uint32_t nb2, cudaStream_t st);
// Batched lazy-L2 normalisation: W row i is multiplied by scales[w_slot[i]],
// H row j by scales[h_slot[j]]
cudaError_t launch_scale_rows(int precision, void* W, uint64_t wrows, void* H, uint64_t hrows,
                              uint32_t rp, const uint32_t* w_slot, const uint32_t* h_slot,
                              const float* scales, cudaStream_t st);

// Loss partial sums (FP64); `partials` holds `grid` doubles, then sum_partials
// writes the total to out[0].
cudaError_t launch_nzsl_partials(int precision, const uint32_t* row, const uint32_t* col,
                                 const void* val, uint64_t nnz, const void* W, const void* H,
                                 uint32_t r, uint32_t rp, double* partials, uint32_t grid,
                                 cudaStream_t st);
// CTAs per SM of the training-loss kernel for this precision and row width
int nzsl_ctas_per_sm(int precision, uint32_t rp);
cudaError_t launch_sumsq_partials(int precision, const void* X, uint64_t count,
                                  double* partials, uint32_t grid, cudaStream_t st);
cudaError_t launch_nzl2_partials(int precision, const void* X, uint64_t rows, uint32_t rp,
                                 const uint32_t* cnt, double* partials, uint32_t grid,
                                 cudaStream_t st);
cudaError_t launch_sum_partials(const double* partials, uint32_t count, double* out,
                                cudaStream_t st);

// Per-problem sums of the batched form: one CTA per range chunk writes
// partials[chunk]; owner_sums adds partials[owner_begin[p] .. owner_begin[p+1])
// in order into out[p] for p < owners.
struct RangeChunk {
  uint64_t begin, end;
};
cudaError_t launch_nzsl_chunks(int precision, const RangeChunk* chunks, uint32_t nchunks,
                               const uint32_t* row, const uint32_t* col, const void* val,
                               const void* W, const void* H, uint32_t r, uint32_t rp,
                               double* partials, cudaStream_t st);
cudaError_t launch_sumsq_chunks(int precision, const RangeChunk* chunks, uint32_t nchunks,
                                const void* X, double* partials, cudaStream_t st);
cudaError_t launch_owner_sums(const double* partials, const uint32_t* owner_begin,
                              uint32_t owners, double* out, cudaStream_t st);

// Sum (out2[0]) and maximum (out2[1]) over rows of |X_i - Xold_i|; partials
// holds 2 * grid doubles.
cudaError_t launch_update_norms(int precision, const void* X, const void* Xold, uint64_t rows,
                                uint32_t rp, double* partials, uint32_t grid, double* out2,
                                cudaStream_t st);

// ---- step-size controller network (16 -> 64 -> 64 -> 1, GELU) -----------------------
int mlp_param_count();
int mlp_input_count();
cudaError_t launch_mlp(const float* P, const float* X, const float* Y, int batch, float* out,
                       float* grads, float* losses, cudaStream_t st);
cudaError_t launch_mlp_reduce(const float* grads, int batch, float* grad, cudaStream_t st);
cudaError_t launch_adam(float* P, const float* g, float* m, float* v, float lr, float b1,
                        float b2, float eps, int step, cudaStream_t st);

// ---- data preparation -----------------------------------------------------------
// The blocking key of an entry is block * stride + its position in the block.
// The position is local row * nB + local column (the reference's (i, j) order
// within a block; stride = mB * nB), or, for the Hogwild training records, the
// in-block layout order itself: (local column, keyed permutation of the local
// row) for column runs, (local row, permuted local column) for row runs, a
// permutation of local row * nB + local column for the shuffled layout, the
// permuted part `pbits` wide.  A permutation keeps one position per (i, j), so
// duplicate entries still meet, and the one sort both blocks the entries and
// lays them out.
constexpr int kKeyPlain = -1;
struct BlockingGeom {
  uint64_t m, n;
  uint32_t nb1, nb2;      // d, 2d
  uint64_t mB, nB;        // largest block extent in rows / columns
  const uint64_t* off1;   // nb1+1 (last = m)
  const uint64_t* off2;   // nb2+1 (last = n)
  uint64_t stride = 0;    // key distance between consecutive blocks
  int layout = kKeyPlain;  // kKeyPlain or a LayoutKey
  int pbits = 0;           // width of the permuted part of the position
  uint64_t seed = 0;       // layout seed (the permutation's key)
};
cudaError_t launch_make_keys(const BlockingGeom& g, const uint32_t* rows, const uint32_t* cols,
                             uint64_t nnz, uint64_t* keys, uint32_t* idx,
                             unsigned long long* bad, cudaStream_t st);
cudaError_t launch_head_flags(const uint64_t* keys, uint64_t nnz, uint32_t* flags,
                              cudaStream_t st);
// merges runs of equal keys (values summed in input order) into compact arrays
cudaError_t launch_merge_keys(const uint64_t* keys, const uint32_t* idx, const uint32_t* pos,
                              uint64_t nnz, const uint32_t* rows_in, const uint32_t* cols_in,
                              uint64_t* ukeys, uint32_t* urow, uint32_t* ucol, uint32_t* head_at,
                              cudaStream_t st);
cudaError_t launch_block_ptr(const uint64_t* ukeys, uint64_t u, uint64_t block_span,
                             uint32_t nblocks, uint64_t* block_ptr, cudaStream_t st);
// in-block layout keys of the Hogwild matrix for a second sort, when the
// layout cannot ride on the blocking key (more than 64 key bits): (block,
// hash) for a shuffled layout; (block, local column, hash) or (block, local
// row, hash) for runs
enum LayoutKey : int { kLayoutShuffled = 0, kLayoutColRuns = 1, kLayoutRowRuns = 2 };
cudaError_t launch_shuffle_keys(const uint64_t* ukeys, uint64_t u, uint64_t block_span,
                                uint64_t nB, int mode, uint64_t seed, uint64_t* keys2,
                                uint32_t* idx2, cudaStream_t st);
cudaError_t launch_gather_coords(const uint32_t* perm, uint64_t u, const uint32_t* urow,
                                 const uint32_t* ucol, uint32_t* row, uint32_t* col,
                                 cudaStream_t st);
cudaError_t launch_gather_values(const uint32_t* perm, uint64_t u, const uint32_t* head_at,
                                 const uint64_t* keys, const uint32_t* idx, uint64_t nnz,
                                 const double* vals_in, void* val, int val_is_double,
                                 cudaStream_t st);
// rows_out[k] = rows_in[k] + row0, cols_out[k] = cols_in[k] + col0
cudaError_t launch_offset_copy(const uint32_t* rows_in, const uint32_t* cols_in, uint64_t nnz,
                               uint32_t row0, uint32_t col0, uint32_t* rows_out,
                               uint32_t* cols_out, cudaStream_t st);
// block-local -> global coordinates of concatenated blocks (start: nblocks+1
// prefix of the block sizes, row-major blocks); counts entries outside their block
cudaError_t launch_shift_blocks(const uint64_t* start, uint32_t nblocks, uint32_t nb2,
                                const uint64_t* off1, const uint64_t* off2, uint64_t nnz,
                                uint32_t* rows, uint32_t* cols, unsigned long long* bad,
                                cudaStream_t st);
cudaError_t launch_counts_to_u32(const uint64_t* in, uint64_t len, uint32_t* out,
                                 cudaStream_t st);
cudaError_t launch_count_nnz12(const uint32_t* row, const uint32_t* col, uint64_t nnz,
                               uint32_t* cnt1, uint32_t* cnt2, cudaStream_t st);
cudaError_t launch_inverse_counts(const uint32_t* cnt, uint64_t len, void* inv,
                                  int as_double, cudaStream_t st);
cudaError_t launch_factor_to_device(int precision, const double* src, uint64_t rows,
                                    uint32_t r, uint32_t rp, void* dst, cudaStream_t st);
cudaError_t launch_factor_to_host(int precision, const void* src, uint64_t rows, uint32_t r,
                                  uint32_t rp, double* dst, cudaStream_t st);

}  // namespace dsgdpp
