/*
 * dsgdpp.h -- C ABI of the B200 DSGD++ epoch.
 *
 * The reference exposes this path as C++ templates, not as a runtime ABI:
 *   - DsgdPpRunner::run / DsgdPpRunner::epoch      mf/sgd/dsgdpp.h:102-130
 *   - the update functors (UpdateConcept)           mf/sgd/functions/functions.h:21-45
 *   - the regularize functors (RegularizeConcept)   mf/sgd/functions/functions.h:47-63
 *   - the losses (LossConcept)                      mf/loss/loss.h:30-57
 *   - the adaptive decays (AdaptiveDecayConcept)    mf/sgd/decay/decay.h:35-67
 * The entry points below replace those for one GPU: plain C types, every
 * call returns an int status (0 = DSGDPP_OK, negative = error class) and
 * dsgdpp_last_error(ctx) gives the message; no C++ exception crosses the ABI.
 * One host thread drives a context; its work is ordered on one CUDA stream.
 * The context owns all device memory; host buffers are caller-owned and
 * copied.  There is no CPU fallback: without a usable GPU dsgdpp_create
 * fails with DSGDPP_E_CUDA.
 *
 * Layouts follow the reference (mf/types.h:33-42): V is given as a global
 * 0-based coordinate list; W is m x r row-major (DenseMatrix); H is r x n
 * column-major (DenseMatrixCM), i.e. column j's r entries are contiguous.
 */
#ifndef DSGDPP_H
#define DSGDPP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSGDPP_ABI_VERSION 1

typedef struct dsgdpp_ctx dsgdpp_ctx;

/* status codes */
#define DSGDPP_OK 0
#define DSGDPP_E_INVALID (-1)     /* rg::InvalidArgumentException */
#define DSGDPP_E_CUDA (-2)        /* CUDA runtime error, no device */
#define DSGDPP_E_IO (-3)          /* rg::IOException */
#define DSGDPP_E_UNSUPPORTED (-4) /* rg::NotImplementedException */
#define DSGDPP_E_STATE (-5)       /* call out of order (e.g. epoch before data) */
#define DSGDPP_E_NOMEM (-6)       /* device allocation failed */

/* --update / --loss / --regularize functors (tools/mfdsgdpp.cc:162-359) */
#define DSGDPP_UPDATE_NZSL 0       /* UpdateNzsl        update-nzsl.h:33-50     */
#define DSGDPP_UPDATE_NZSL_L2 1    /* UpdateNzslL2(l)   update-nzsl-l2.h:34-57  */
#define DSGDPP_UPDATE_NZSL_NZL2 2  /* UpdateNzslNzl2(l) update-nzsl-nzl2.h:34-53 */
#define DSGDPP_REGULARIZE_NONE 0   /* RegularizeNone    regularize-none.h:22-34 */
#define DSGDPP_REGULARIZE_L2 1     /* RegularizeL2(l)   regularize-l2.h:26-50   */
#define DSGDPP_LOSS_NZSL 0         /* NzslLoss                                  */
#define DSGDPP_LOSS_NZSL_L2 1      /* SumLoss<NzslLoss, L2Loss(l)>              */
#define DSGDPP_LOSS_NZSL_NZL2 2    /* SumLoss<NzslLoss, Nzl2Loss(l)>            */
/* --sgd-order (mf/sgd/sgd.h:39) and --stratum-order (mf/sgd/dsgd.h:29) */
#define DSGDPP_SGD_SEQ 0
#define DSGDPP_SGD_WR 1
#define DSGDPP_SGD_WOR 2
#define DSGDPP_STRATUM_SEQ 0
#define DSGDPP_STRATUM_RSEQ 1
#define DSGDPP_STRATUM_WR 2
#define DSGDPP_STRATUM_WOR 3
#define DSGDPP_STRATUM_COWOR 4
/* factor storage; arithmetic is FP64 for FP64 storage, FP32 otherwise */
#define DSGDPP_FP64 0
#define DSGDPP_FP32 1
#define DSGDPP_BF16 2 /* stochastic rounding on every store */
/* execution of a block's records */
#define DSGDPP_EXEC_REPLAY 0  /* sequential per block, reference point order, FP64 only */
#define DSGDPP_EXEC_HOGWILD 1 /* all SMs on the sub-epoch's records (Hogwild within a block) */
/* launch form of an epoch */
#define DSGDPP_LAUNCH_STREAM 0 /* 2d kernel launches per epoch */
#define DSGDPP_LAUNCH_GRAPH 1  /* the epoch captured once as a CUDA graph and replayed */
#define DSGDPP_LAUNCH_PERSISTENT 2 /* one launch per epoch (graph-captured): a block of
                                      sub-epoch s starts when the blocks it depends on in
                                      earlier sub-epochs are done (Hogwild, atomic writes,
                                      a run layout, SEQ or WOR order) */
/* how a Hogwild update is written back */
#define DSGDPP_WRITE_AUTO 0   /* ATOMIC without truncation, else STORE */
#define DSGDPP_WRITE_STORE 1  /* store the new row/column (concurrent updates may be lost) */
#define DSGDPP_WRITE_ATOMIC 2 /* add the update atomically: vector atomic add (FP32/FP64);
                                 BF16 adds the increment to the stochastically rounded value */
/* the stratified method (DsgdPpRunner, DsgdRunner) */
#define DSGDPP_METHOD_DSGDPP 0 /* d x 2d blocks, 2d sub-epochs (mf/sgd/dsgdpp_impl.h)        */
#define DSGDPP_METHOD_DSGD 1   /* d x d blocks, d sub-epochs (mf/sgd/dsgd_impl.h:80-234,328-350) */
/* order of the Hogwild training records inside each block */
#define DSGDPP_LAYOUT_SHUFFLED 0 /* random order (a permutation keyed by layout_seed) */
#define DSGDPP_LAYOUT_COL_RUNS 1 /* by column, random within a column: runs of one H row */
#define DSGDPP_LAYOUT_ROW_RUNS 2 /* by row, random within a row: runs of one W row */
#define DSGDPP_LAYOUT_RUNS 3     /* COL_RUNS when n <= m (more records per column), else ROW_RUNS */
/* matrices */
#define DSGDPP_TRAIN 0
#define DSGDPP_TEST 1
/* decays (mf/sgd/decay) */
#define DSGDPP_DECAY_CONST 0      /* DecayConstant(eps)              decay_constant.h:31-63 */
#define DSGDPP_DECAY_BOLDDRIVER 1 /* BoldDriver(eps, dec, inc)        decay_bolddriver.h:33-92 */

typedef struct dsgdpp_config {
  uint64_t m, n;          /* size of V: rows (of W) and columns (of H) */
  uint32_t rank;          /* r */
  uint32_t d;             /* tasks = row blocks; V is blocked d x 2d (1 <= d <= 1024) */
  int32_t precision;      /* DSGDPP_FP64 / FP32 / BF16 */
  int32_t exec;           /* DSGDPP_EXEC_* */
  int32_t launch;         /* DSGDPP_LAUNCH_* */
  int32_t update;         /* DSGDPP_UPDATE_* */
  double update_lambda;
  int32_t regularize;     /* DSGDPP_REGULARIZE_* */
  double regularize_lambda;
  int32_t loss;           /* DSGDPP_LOSS_* */
  double loss_lambda;
  int32_t truncate;       /* UpdateTruncate / RegularizeTruncate when nonzero */
  double truncate_min, truncate_max;
  int32_t sgd_order;      /* DSGDPP_SGD_* */
  int32_t stratum_order;  /* DSGDPP_STRATUM_* */
  int32_t device;         /* CUDA device ordinal */
  uint32_t lanes_per_nnz; /* Hogwild lanes per record: 0 = auto, else 2..32 */
  uint32_t vecs_per_lane; /* Hogwild 16-byte vectors per lane: 0 = auto */
  uint32_t ctas_per_sm;   /* Hogwild CTAs of 256 threads per SM (FP32/FP64 launch CTAs of
                             128, twice as many): 0 = occupancy limit */
  uint64_t layout_seed;   /* seeds the one-off shuffle of the Hogwild record layout */
  int32_t write_mode;     /* Hogwild factor writes: DSGDPP_WRITE_* */
  int32_t layout;         /* Hogwild record order in a block: DSGDPP_LAYOUT_* */
  int32_t method;         /* DSGDPP_METHOD_*: d x 2d (default) or d x d blocking */
} dsgdpp_config;

/* One row of the run trace (SgdTraceEntry, mf/trace.h:84-116); times in ns. */
typedef struct dsgdpp_trace_row {
  uint64_t epoch;
  double loss, test_loss, eps;
  double time_eps, time_epoch, time_loss, time_test_loss;
} dsgdpp_trace_row;

/* ---- context ------------------------------------------------------------ */
/* Fills c with the reference defaults: WOR / COWOR, Nzsl_L2(1) update and
 * loss, regularize None, FP32 Hogwild, graph launch, automatic lane mapping,
 * DSGDPP_LAYOUT_RUNS record order. */
void dsgdpp_config_init(dsgdpp_config* c);
/* replaces: DsgdPpJob / DsgdPpFactorizationData construction
 * (mf/sgd/dsgdpp.h:38-59, mf/sgd/dsgdpp-factorization.h:58-64) */
int dsgdpp_create(const dsgdpp_config* c, dsgdpp_ctx** out);
/* message of the calling thread's last failed dsgdpp_create */
const char* dsgdpp_create_error(void);
void dsgdpp_destroy(dsgdpp_ctx* ctx);
const char* dsgdpp_last_error(const dsgdpp_ctx* ctx);
const char* dsgdpp_status_string(int status);
int dsgdpp_abi_version(void);

/* ---- data --------------------------------------------------------------- */
/* replaces: getDataMatrices / loadMatrix blocking (mf/matrix/io/
 * generateDistributedMatrix_impl.h:692-744, read_impl.h:364-486).  Global
 * 0-based coordinates from host memory; blocked d x 2d and sorted (i, j)
 * inside each block on the GPU, duplicate entries summed.  For the training
 * matrix this also counts nnz1 / nnz2 (mf/matrix/op/nnz.h:124-163). */
int dsgdpp_set_matrix(dsgdpp_ctx* ctx, int which, uint64_t nnz, const uint32_t* rows,
                      const uint32_t* cols, const double* vals);
/* replaces: the blocked DistributedMatrix the runner works on (block-local
 * coordinates, read_impl.h:421): the d x 2d (d x d for DSGD) blocks one after
 * another in row-major block order, block b holding block_nnz[b] entries with
 * 0-based coordinates inside the block.  The block extents must be the
 * context's (computeDefaultBlockOffsets); an entry outside its block is an
 * error (DSGDPP_E_INVALID).  Otherwise the same as dsgdpp_set_matrix. */
int dsgdpp_set_blocks(dsgdpp_ctx* ctx, int which, const uint64_t* block_nnz,
                      const uint32_t* local_rows, const uint32_t* local_cols,
                      const double* vals);
/* replaces: the nnz12 counts of DistributedFactorizationData::init
 * (mf/factorization.h:202-208) with counts the caller holds (m and n
 * entries, each below 2^32), e.g. counted over more data than this context
 * holds.  Call after dsgdpp_set_matrix of the training matrix, which counts
 * them itself and would replace them. */
int dsgdpp_set_counts(dsgdpp_ctx* ctx, const uint64_t* nnz1, const uint64_t* nnz2);
/* replaces: getFactors (generateDistributedMatrix_impl.h:655-690) */
int dsgdpp_set_factors(dsgdpp_ctx* ctx, const double* W, const double* H);
/* replaces: unblock + the factor arrays read by writeMatrix (tools/mfdsgdpp.cc:145-159) */
int dsgdpp_get_factors(dsgdpp_ctx* ctx, double* W, double* H);
/* nnz per block of the blocked matrix: d x 2d row-major (DSGD++), d x d (DSGD) */
int dsgdpp_block_nnz(dsgdpp_ctx* ctx, int which, uint64_t* out);
/* per-row / per-column counts of the training matrix (nnz12) */
int dsgdpp_nnz12(dsgdpp_ctx* ctx, uint64_t* nnz1, uint64_t* nnz2, uint64_t* nnz12max);

/* ---- epoch -------------------------------------------------------------- */
/* Seeds the master generator (the Random32 of DsgdPpRunner, tools/mfdsgdpp.cc:542). */
int dsgdpp_seed(dsgdpp_ctx* ctx, uint32_t seed);
/* replaces: DsgdPpRunner::epoch(job, eps) (mf/sgd/dsgdpp_impl.h:282-349):
 * draws the red/blue split, the stratum schedule and the task seeds from the
 * master generator, then runs the 2d sub-epochs on the GPU. */
int dsgdpp_epoch(dsgdpp_ctx* ctx, double eps);
/* The same with a caller-given schedule (2d x d, row = sub-epoch, column =
 * task id, entry = column block) and task seeds (d). */
int dsgdpp_epoch_explicit(dsgdpp_ctx* ctx, double eps, const uint32_t* schedule,
                          const uint32_t* task_seeds);
/* Sub-epochs [s_begin, s_end) of the epoch given by eps, schedule and
 * task_seeds, as dsgdpp_epoch_explicit runs all of them: the parts of one
 * epoch follow one another from 0 to 2d (d for DSGD) with the same arguments,
 * and an epoch is finished (end-of-epoch work done) by the part that reaches
 * the end.  Between parts the caller may exchange H column blocks
 * (dsgdpp_h_block_copy) -- the hand-off of DsgdPpTask::run between
 * sub-epochs when the tasks live on several ranks (mf/sgd/dsgdpp_impl.h:
 * 153-263).  Stream launches; not for the persistent launch form. */
int dsgdpp_epoch_part(dsgdpp_ctx* ctx, double eps, const uint32_t* schedule,
                      const uint32_t* task_seeds, uint32_t s_begin, uint32_t s_end);
/* H column block b2 (columns off2[b2] .. off2[b2+1] of H, each rank-padded,
 * in the factor precision) copied from the context into device_buf
 * (to_context = 0) or from device_buf into the context (1); the caller's
 * buffer holds dsgdpp_h_block_bytes bytes and may live on any device the
 * context's device can reach.  Synchronous. */
int dsgdpp_h_block_bytes(dsgdpp_ctx* ctx, uint32_t b2, uint64_t* bytes);
int dsgdpp_h_block_copy(dsgdpp_ctx* ctx, uint32_t b2, void* device_buf, int to_context);
/* The context runs tasks first .. first+count-1 of the d tasks: one rank's
 * share of a job whose tasks are spread over several ranks, as an MPI rank of
 * the reference runs its tasksPerRank tasks (tools/mfdsgdpp.cc:41-42,76-77).
 * The entries of the other tasks' row blocks must be absent (an epoch with
 * such entries returns DSGDPP_E_STATE); the replay's per-sub-epoch
 * RegularizeL2 scales only these tasks' W row blocks and H blocks, as each
 * task of DsgdPpTask::run regularizes its own pair (mf/sgd/dsgdpp_impl.h:
 * 241-243).  Default: all d tasks. */
int dsgdpp_set_tasks(dsgdpp_ctx* ctx, uint32_t first, uint32_t count);

/* ---- one job over several ranks --------------------------------------------
 * replaces: the H-block hand-off of DsgdPpTask::run between sub-epochs over MPI
 * (mf/sgd/dsgdpp_impl.h:141-263: igetCopy / irecv / isend of the next
 * block, red/blue double buffering, a barrier per sub-epoch).  Rank r of G
 * drives a context holding its tasks' rows (dsgdpp_set_tasks(ctx, r d/G, d/G),
 * the nnz12 weights of the whole matrix given with dsgdpp_set_counts, the W
 * rows of other ranks zero).  A block that another rank needs next is sent
 * from H to H right after the sub-epoch that last used it, on a transfer
 * stream, while the next sub-epoch (the other colour) computes; only the
 * sub-epoch that uses it waits for it.  Transports: NCCL (one rank per GPU and
 * process, NCCL loaded at run time) or device copies between the contexts of
 * one process (emulated ranks on one GPU).  Not for the persistent launch. */
typedef struct dsgdpp_shard dsgdpp_shard;
#define DSGDPP_SHARD_ID_BYTES 128
/* A new NCCL unique id (rank 0 makes it and hands the bytes to every rank). */
int dsgdpp_shard_unique_id(void* id);
/* Rank `rank` of `world` over NCCL; every rank calls it with the same id. */
int dsgdpp_shard_create_nccl(dsgdpp_ctx* ctx, int rank, int world, const void* id,
                             dsgdpp_shard** out);
/* `world` emulated ranks in this process: ctxs[r] is rank r's context. */
int dsgdpp_shard_create_local(dsgdpp_ctx* const* ctxs, int world, dsgdpp_shard** out);
void dsgdpp_shard_destroy(dsgdpp_shard* sh);
const char* dsgdpp_shard_last_error(const dsgdpp_shard* sh);
/* Bound on a host wait for NCCL work (default 300 s); a wait that runs out
 * aborts the communicator and returns DSGDPP_E_CUDA (a rank left or hung). */
int dsgdpp_shard_set_wait_limit(dsgdpp_shard* sh, double seconds);
/* One epoch on every rank (DsgdPpRunner::epoch, mf/sgd/dsgdpp_impl.h:282-349):
 * the given schedule and task seeds, or (both null) the draws of the master
 * generator of the (first) context, the same on every rank seeded alike. */
int dsgdpp_shard_epoch(dsgdpp_shard* sh, double eps, const uint32_t* schedule,
                       const uint32_t* task_seeds);
/* Every H block's latest version to every rank (broadcast from its holder);
 * needed before losses or dsgdpp_get_factors of H. */
int dsgdpp_shard_share(dsgdpp_shard* sh);
/* The job's training loss (the configured loss over all ranks' entries, the
 * regularizer over all of W and H) and test loss (NaN without test entries);
 * after dsgdpp_shard_share. */
int dsgdpp_shard_losses(dsgdpp_shard* sh, double* loss, double* test_loss);
/* Every rank's W rows to every rank, so that dsgdpp_get_factors returns the
 * whole W (with NCCL a sum over the ranks: each rank's W is zero outside its
 * own rows).  For reading the result: afterwards the contexts hold all of W,
 * so no further epoch or loss of this shard is valid. */
int dsgdpp_shard_gather_w(dsgdpp_shard* sh);
/* Blocks (and bytes) the ranks driven here received in the last epoch. */
int dsgdpp_shard_moved(dsgdpp_shard* sh, uint64_t* moves, uint64_t* bytes);
/* Timeline of the next epochs: when on, events around every sub-epoch and
 * every transfer group; dsgdpp_shard_timeline gives, for the driven rank at
 * `index`, [begin, end] in ms from the epoch's start of each sub-epoch
 * (compute, 2 nb2 values) and of each transfer group posted before the epoch
 * and after sub-epochs 0 .. nb2-2 (transfer, 2 nb2 values; NaN where the
 * rank's transfer stream carried none of the group: emulated ranks copy on
 * the receiver's stream, NCCL sends and receives on both ranks'). */
int dsgdpp_shard_set_timeline(dsgdpp_shard* sh, int on);
int dsgdpp_shard_timeline(dsgdpp_shard* sh, uint32_t index, double* compute, double* transfer);
/* The hand-off plan of one epoch (host only, no GPU): moves as (group, block,
 * from rank, to rank) quadruples, group 0 = before the epoch and s + 1 = after
 * sub-epoch s; holder[nb2] (-1 = every rank) is the state before the epoch and
 * is updated.  Returns the number of moves (written when out is not null). */
uint64_t dsgdpp_shard_plan(uint32_t d, uint32_t nb2, int world, const uint32_t* schedule,
                           int32_t* holder, uint32_t* out);
/* How long one dependency wait of the persistent epoch (DSGDPP_LAUNCH_PERSISTENT)
 * may last before the epoch gives up, in seconds (default 1; 0 gives up at the
 * first unmet dependency).  A wait that runs out sets an error flag; every
 * warp then stops, dsgdpp_epoch returns DSGDPP_E_CUDA with a message, the
 * epoch is left incomplete, and the context stays usable.  Replaces the
 * unbounded barrier(channels) that ends a sub-epoch in the reference
 * (mf/sgd/dsgdpp_impl.h:259-263); the other launch forms do not wait. */
int dsgdpp_set_wait_limit(dsgdpp_ctx* ctx, double seconds);
/* Device time of the last epoch's kernels in milliseconds. */
int dsgdpp_last_epoch_ms(dsgdpp_ctx* ctx, double* ms);
/* Per-kernel timing of the Hogwild sub-epoch kernels: when on, epochs launch
 * on the stream (no graph) with an event around every sub-epoch kernel;
 * dsgdpp_kernel_timing returns their summed time and launch count since the
 * timing was switched on.  No reference counterpart (instrumentation). */
int dsgdpp_set_kernel_timing(dsgdpp_ctx* ctx, int on);
int dsgdpp_kernel_timing(dsgdpp_ctx* ctx, double* total_ms, uint64_t* launches);
/* The Hogwild launch shape chosen: lanes per record, 16-byte vectors per lane,
 * CTAs in the grid. */
int dsgdpp_launch_shape(dsgdpp_ctx* ctx, uint32_t* lanes, uint32_t* vecs, uint32_t* grid);

/* ---- losses (FP64 accumulation) ------------------------------------------- */
/* replaces: the configured training loss, SumLoss<NzslLoss, L2Loss|Nzl2Loss>
 * or NzslLoss (mf/loss/loss.h:88-112) */
int dsgdpp_loss(dsgdpp_ctx* ctx, double* out);
/* replaces: NzslLoss (mf/loss/nzsl.h:160-185); which = TRAIN or TEST */
int dsgdpp_nzsl(dsgdpp_ctx* ctx, int which, double* out);
/* replaces: l2 over W and over H (mf/loss/l2.h:134-145) */
int dsgdpp_l2(dsgdpp_ctx* ctx, double* w2, double* h2);
/* replaces: nzl2 over W and over H (mf/loss/nzl2.h:246-289) */
int dsgdpp_nzl2(dsgdpp_ctx* ctx, double* w, double* h);

/* Capacity of the fixed scratch of dsgdpp_nzsl_fp32_noalloc, in partial sums
 * (4096 doubles = 32 KiB of device memory per GPU that loads this library). */
#define DSGDPP_NOALLOC_MAX_PARTIALS 4096
/* Widest factor row dsgdpp_nzsl_fp32_noalloc takes, in floats (128 vectors:
 * the widest lane mapping of the loss kernel). */
#define DSGDPP_NOALLOC_MAX_LD 512
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- code running inside another framework's memory pool, or under an
 * allocator it does not own -- this computes the same sum of squared errors
 * as dsgdpp_nzsl, sum over k < nnz of (vals[k] - W[rows[k]] . H[cols[k]])^2
 * accumulated in FP64, from caller-owned device buffers: FP32 values, W and H
 * as FP32 rows of `ld` floats (ld a multiple of 4, >= rank rounded up to 4
 * and <= DSGDPP_NOALLOC_MAX_LD; W and H 16-byte aligned; only the first
 * `rank` entries of a row count).  The call takes no matrix shape, so it
 * cannot check the indices: every rows[k] must name a row of W and every
 * cols[k] a row of H -- that is the caller's contract.  The result is written
 * to the device double *out, ordered on `stream` (a cudaStream_t; NULL is the
 * default stream).  The call allocates and frees nothing: its scratch is a
 * fixed device array of DSGDPP_NOALLOC_MAX_PARTIALS doubles, one per CTA;
 * `partials` sets the CTA count (0 = 4 per SM).  A CTA count above the
 * capacity, or an ld outside the limits above, returns DSGDPP_E_INVALID with
 * a message on stderr.  The first call in a CUDA context (per device, the
 * runtime's primary context unless the caller made another current) looks up
 * the scratch address there (set-up); make that first call before any stream
 * capture.  A cudaDeviceReset ends the library's use of that device, as for
 * every other entry point.  All calls in a context share the scratch, which
 * keeps the last call's contents; calls that overlap on the GPU race on it. */
int dsgdpp_nzsl_fp32_noalloc(const uint32_t* rows, const uint32_t* cols, const float* vals,
                             uint64_t nnz, const float* W, const float* H, uint32_t rank,
                             uint32_t ld, uint32_t partials, double* out, void* stream);

/* ---- runner --------------------------------------------------------------- */
/* replaces: DsgdPpRunner::run -> detail::defaultRunner (mf/sgd/sgd_impl.h:34-145):
 * loss and test loss, then per epoch: decay, epoch, loss, test loss.  trace
 * receives epochs+1 rows (row 0 = the initial losses, eps NaN).  The test loss
 * is skipped (NaN) when no test matrix was set. */
int dsgdpp_run(dsgdpp_ctx* ctx, uint32_t epochs, int decay, double eps0, double decrease,
               double increase, dsgdpp_trace_row* trace);
int dsgdpp_sync(dsgdpp_ctx* ctx);

/* ---- step-size control ------------------------------------------------------
 * No reference counterpart (the reference's adaptive rule is BoldDriver with no
 * rollback, mf/sgd/decay/decay_bolddriver.h:59-67).  Device-side snapshot of
 * the factors, for rejecting an epoch whose proposed step raised the training
 * loss, and the per-row update norms |x_i - x_i(snapshot)| over W and H rows
 * (mean and maximum) used as controller features. */
int dsgdpp_save_factors(dsgdpp_ctx* ctx);
int dsgdpp_restore_factors(dsgdpp_ctx* ctx);
int dsgdpp_update_norms(dsgdpp_ctx* ctx, double* mean, double* max);

/* The controller network: 16 features -> 64 -> 64 -> 1 (GELU), FP32, output a
 * log step multiplier clipped to [-1, 1].  Inputs and outputs are host arrays
 * (batch x 16 features row-major); parameters live on the device. */
typedef struct dsgdpp_mlp dsgdpp_mlp;
int dsgdpp_mlp_create(int device, uint64_t seed, dsgdpp_mlp** out);
void dsgdpp_mlp_destroy(dsgdpp_mlp* mlp);
int dsgdpp_mlp_param_count(void);
int dsgdpp_mlp_get_params(dsgdpp_mlp* mlp, float* params);
int dsgdpp_mlp_set_params(dsgdpp_mlp* mlp, const float* params);
int dsgdpp_mlp_forward(dsgdpp_mlp* mlp, const float* x, int batch, float* out);
/* mean squared error of the unclipped output against y, and its gradient
 * w.r.t. the parameters */
int dsgdpp_mlp_gradient(dsgdpp_mlp* mlp, const float* x, const float* y, int batch, float* loss,
                        float* grad);
/* one Adam step (lr, betas 0.9/0.999, eps 1e-8) on the batch; returns the loss */
int dsgdpp_mlp_train_step(dsgdpp_mlp* mlp, const float* x, const float* y, int batch, float lr,
                          float* loss);
/* defaultRunner with the controller choosing each step: the network proposes
 * eps * exp(m).  If that epoch raises the training loss, BoldDriver takes
 * over (a fallback event): a rise of at most 1% is kept and the next step is
 * the proposal times `decrease`; a larger rise, or a non-finite loss, is
 * rolled back and the epoch re-run at the proposal times decrease^k
 * (k = 1..8) until the rise is at most 1%.  From the second decision on, an
 * epoch in which one factor row moved more than 40 times the mean row
 * movement and more than 4 times the median largest movement of the last
 * three kept epochs is rolled back the same way, whatever the loss did.  Once a step
 * has raised the loss, proposals are capped at 0.9 times the smallest such
 * step, a cap that grows by 5% with every decision that does not raise the
 * loss.  Stops after `epochs` or once the test loss is at most
 * target_test_loss (> 0).  trace gets epochs_done + 1 rows (time_epoch
 * includes the training losses the decisions need). */
int dsgdpp_run_controlled(dsgdpp_ctx* ctx, dsgdpp_mlp* mlp, uint32_t epochs, double eps0,
                          double decrease, double increase, double target_test_loss,
                          dsgdpp_trace_row* trace, uint32_t* epochs_done, uint32_t* fallbacks);
/* The 16 controller features from the run history: train/test losses of the
 * last 5 evaluations (index 0 = newest; NaN where missing), the current step,
 * the mean/max factor-update norms of the last epoch, the epoch fraction, the
 * last applied log multiplier and the smallest step that has raised the
 * training loss so far in this run (fail_eps; 0 = none), as log(fail_eps/eps). */
void dsgdpp_controller_features(const double* train_hist, const double* test_hist, double eps,
                                double upd_mean, double upd_max, double epoch_frac,
                                double last_log_mult, double fail_eps, float* out16);

/* ---- autotuning ------------------------------------------------------------- */
/* No reference counterpart (the reference takes d from --tasks-per-rank).
 * Times Hogwild epochs of `base` on the given training entries and factors
 * for each d in d_candidates (NULL/0: 64, 128, 256, 512) and several
 * lane-to-rank mappings and CTA counts per SM; writes the fastest
 * configuration to *best and its median epoch time to *best_ms. */
int dsgdpp_autotune(const dsgdpp_config* base, uint64_t nnz, const uint32_t* rows,
                    const uint32_t* cols, const double* vals, const double* W, const double* H,
                    const uint32_t* d_candidates, uint32_t nd, uint32_t epochs, double eps,
                    dsgdpp_config* best, double* best_ms);

/* ---- batched form: many independent factorizations ----------------------- */
/* No reference counterpart (the reference runs one factorization per job).
 * Problems are grouped by padded rank; one epoch of every problem is one
 * sequence of Hogwild launches, launch s of a group covering sub-epoch s of
 * all its problems (captured once as a CUDA graph under DSGDPP_LAUNCH_GRAPH).
 * Step sizes follow BoldDriver per problem on per-problem training losses. */
typedef struct dsgdpp_batch dsgdpp_batch;
typedef struct dsgdpp_problem {
  uint64_t m, n;       /* rows, columns */
  uint32_t rank;
  uint32_t d;          /* 0: chosen from the problem's size (at most 16) */
  uint64_t nnz;        /* training entries (0-based COO, duplicates summed) */
  const uint32_t* rows;
  const uint32_t* cols;
  const double* vals;
  uint64_t nnz_test;   /* test entries (may be 0) */
  const uint32_t* trows;
  const uint32_t* tcols;
  const double* tvals;
  const double* W;     /* m x rank row-major initial factors */
  const double* H;     /* n x rank row-major (row j = column j of H) */
  uint32_t seed;       /* master generator seed (dsgdpp_seed) */
  double eps0;         /* first step size */
} dsgdpp_problem;
/* `common` supplies precision, update/regularize/loss functions and their
 * lambdas, stratum and SGD orders, device, launch mode, write mode and the
 * lane mapping (0 = per group); its m, n, rank and d are ignored.  Only the
 * Hogwild path without truncation is batched (DSGDPP_E_UNSUPPORTED else). */
int dsgdpp_batch_create(const dsgdpp_config* common, uint32_t count,
                        const dsgdpp_problem* problems, dsgdpp_batch** out);
void dsgdpp_batch_destroy(dsgdpp_batch* b);
const char* dsgdpp_batch_last_error(const dsgdpp_batch* b);
/* Runs `epochs` epochs of every problem (BoldDriver per problem from eps0 as
 * dsgdpp_run, training loss after every epoch, test loss after the last).
 * train/test get one value per problem (may be NULL); *epoch_ms the summed
 * device time of the epochs' launches. */
int dsgdpp_batch_run(dsgdpp_batch* b, uint32_t epochs, double decrease, double increase,
                     double* train, double* test, double* epoch_ms);
/* The batched form's autotuner.  Times `epochs` epochs of the problems
 * problems[0], problems[sample_stride], ... for each cap on the automatic d
 * (4, 8, 16, 32) and each CTA count per SM (as many as fit, 3, 2), and writes
 * the fastest choice: d_out[p] for every problem (a problem's own nonzero d
 * is kept) and *ctas_per_sm (0 = as many as fit) for dsgdpp_config, with the
 * sample's epoch time in *best_ms. */
int dsgdpp_batch_autotune(const dsgdpp_config* common, uint32_t count,
                          const dsgdpp_problem* problems, uint32_t sample_stride, uint32_t epochs,
                          uint32_t* d_out, uint32_t* ctas_per_sm, double* best_ms);
int dsgdpp_batch_problem_d(dsgdpp_batch* b, uint32_t p, uint32_t* d);
int dsgdpp_batch_get_factors(dsgdpp_batch* b, uint32_t p, double* W, double* H);

/* ---- host utilities (no GPU needed) --------------------------------------- */
/* rg::Random32 as pinned by this library (MT19937, Boost bucket nextInt). */
typedef struct dsgdpp_rng dsgdpp_rng;
dsgdpp_rng* dsgdpp_rng_create(uint32_t seed);
void dsgdpp_rng_destroy(dsgdpp_rng* rng);
uint32_t dsgdpp_rng_next(dsgdpp_rng* rng);
uint32_t dsgdpp_rng_next_int(dsgdpp_rng* rng, uint32_t n);
/* DsgdPpRunner::epoch's master-generator draws (mf/sgd/dsgdpp_impl.h:289-344) */
void dsgdpp_draw_schedule(dsgdpp_rng* master, uint32_t d, int stratum_order,
                          uint32_t* schedule, uint32_t* task_seeds);
/* detail::computeDsgdSchedule (mf/sgd/dsgd_impl.h:246-325): (w t) x (w t) */
void dsgdpp_dsgd_schedule(dsgdpp_rng* rng, uint32_t w, uint32_t t, int stratum_order,
                          uint32_t* out);
/* SgdRunner point orders of one epoch for an explicit schedule: for
 * s = 0..2d-1, task id = 0..d-1, the positions inside block (id, schedule[s][id])
 * given the block sizes block_nnz (d x 2d).  Returns the count written. */
uint64_t dsgdpp_point_orders(uint32_t d, int sgd_order, const uint64_t* block_nnz,
                             const uint32_t* schedule, const uint32_t* task_seeds,
                             uint32_t* out);
/* computeDefaultBlockOffsets (mf/matrix/distributed_matrix_impl.cc:24-40) */
void dsgdpp_block_offsets(uint64_t size, uint32_t blocks, uint64_t* out);
/* ---- file I/O (replaces mf/matrix/io: read_impl.h:45-256, write_impl.h:42-118,
 * descriptor_impl.cc:25-75); failures return DSGDPP_E_IO, message in
 * dsgdpp_io_error().  Arrays returned through pointers are malloc'ed; release
 * them with dsgdpp_free. */
const char* dsgdpp_io_error(void);
void dsgdpp_free(void* p);
/* .mmc, or an .xml descriptor of .mmc blocks: global 0-based coordinates */
int dsgdpp_read_sparse(const char* path, uint64_t* m, uint64_t* n, uint64_t* nnz,
                       uint32_t** rows, uint32_t** cols, double** vals);
int dsgdpp_write_mm_coord(const char* path, uint64_t m, uint64_t n, uint64_t nnz,
                          const uint32_t* rows, const uint32_t* cols, const double* vals);
/* .mma (entries column by column), or an .xml descriptor of .mma blocks (each
 * block placed at its offsets): the whole matrix, column by column */
int dsgdpp_read_mm_array(const char* path, uint64_t* m, uint64_t* n, double** colmajor);
int dsgdpp_write_mm_array(const char* path, uint64_t m, uint64_t n, const double* colmajor);
/* the blocked form written by tools/mfdblock.cc: per-block .mmc files with
 * block-local coordinates named <base>-<b1>-<b2>.mmc in dir, plus the .xml */
int dsgdpp_write_blocked(const char* xml_path, const char* dir, const char* base, uint64_t m,
                         uint64_t n, uint32_t blocks1, uint32_t blocks2, uint64_t nnz,
                         const uint32_t* rows, const uint32_t* cols, const double* vals);
/* Philox4x32-10 of the BF16 stochastic rounding, for known-answer checks */
void dsgdpp_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---- random-matrix descriptors (.rm), generated on the device ----------------
 * replaces: RandomMatrixDescriptor (mf/matrix/io/randomMatrixDescriptor.h:27-77,
 * randomMatrixDescriptor_impl.cc:21-176), the .rm branches of getDataMatrices /
 * getFactors (mf/matrix/io/generateDistributedMatrix_impl.h:655-744) and
 * tools/mfcreateRandomMatrixFile.cc.  The file format, chunk grid, counts per
 * chunk and value model (Worig * Horig + noise) are the reference's; the draws
 * are this library's own counter-based ones (rm.h states them), so a
 * descriptor gives the same matrices here on every run and device, not the
 * reference's.  Failures return DSGDPP_E_IO (file, format) or
 * DSGDPP_E_INVALID, message in dsgdpp_rm_error(). */
typedef struct dsgdpp_rm dsgdpp_rm;
const char* dsgdpp_rm_error(void);
int dsgdpp_rm_load(const char* path, dsgdpp_rm** out);
/* RandomMatrixDescriptor::create; values / noise: "Normal(mean,stddev)" (the
 * mean is ignored, as tools/parse.h:80-88 ignores it) or "Uniform(min,max)" */
int dsgdpp_rm_create(uint64_t size1, uint64_t size2, uint32_t blocks1, uint32_t blocks2,
                     uint64_t nnz, uint64_t nnz_test, uint32_t rank, const char* values,
                     const char* noise, dsgdpp_rm** out);
int dsgdpp_rm_save(const dsgdpp_rm* rm, const char* path);
void dsgdpp_rm_destroy(dsgdpp_rm* rm);
/* out[9]: size1, size2, rank, blocks1, blocks2, nnz, nnzTest (as written), and
 * the data and test nonzeros the chunk counts add up to (0 without a data part) */
int dsgdpp_rm_info(const dsgdpp_rm* rm, uint64_t* out);
/* the data (DSGDPP_TRAIN) or test (DSGDPP_TEST) matrix into host arrays of
 * out[7] / out[8] entries, 0-based; chunk by chunk in row-major chunk order */
int dsgdpp_rm_generate(const dsgdpp_rm* rm, int which, int device, uint32_t* rows,
                       uint32_t* cols, double* vals);
/* Worig (size1 x rank, row-major) and Horig (size2 x rank: column j of the
 * rank x size2 factor contiguous) */
int dsgdpp_rm_generate_factors(const dsgdpp_rm* rm, int device, double* W, double* H);
/* generated straight into the context (no host copy): the data or test
 * matrix of rm, which must be m x n */
int dsgdpp_set_matrix_rm(dsgdpp_ctx* ctx, int which, const dsgdpp_rm* rm);
/* the factors of getFactors(.rm): Worig and Horig of rm (m x n, rank r) */
int dsgdpp_set_factors_rm(dsgdpp_ctx* ctx, const dsgdpp_rm* rm);

#ifdef __cplusplus
}
#endif
#endif
