/*
 * dsgdpp_oracle.h -- C interface of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain C++ restatement of the
 * reference DSGD++ epoch (uma-pi1/DSGDpp, mf/sgd/dsgdpp_impl.h and the code it
 * calls).  It exists to check the CUDA product path; the product never links,
 * loads or calls it.  Only tests/, the smoke check and the CPU-baseline leg of
 * bench.py use it.
 *
 * PARITY UNPINNED: the reference cannot be compiled here (Boost, MPICH2,
 * log4cxx and the unvendored mpi2/rg libraries are missing) and ships no
 * golden vectors or tests, so this restatement is checked only against the
 * one known answer the reference prints (README.md:84-96, BoldDriver step
 * sizes) and against hand-derived cases.  The random-number primitives of the
 * unvendored rg library are pinned by assumption (see dsgdpp_oracle.cc).
 */
#ifndef DSGDPP_ORACLE_H
#define DSGDPP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_problem orc_problem;

/* ---- Random32 (pinned) ------------------------------------------------- */
typedef struct orc_random orc_random;
orc_random* orc_random_create(uint32_t seed);
void orc_random_destroy(orc_random* r);
uint32_t orc_random_next(orc_random* r);              /* raw 32-bit draw   */
uint32_t orc_random_next_int(orc_random* r, uint32_t n); /* uniform [0, n) */
void orc_random_shuffle_u32(orc_random* r, uint32_t* a, uint64_t n);
void orc_random_sample(orc_random* r, uint32_t k, uint32_t n, uint32_t* out);

/* ---- blocking / schedules ---------------------------------------------- */
void orc_block_offsets(uint64_t size, uint32_t blocks, uint64_t* out);
/* computeDsgdSchedule(w, t, order, R): out is (w*t) x (w*t), row-major. */
void orc_compute_dsgd_schedule(orc_random* r, uint32_t w, uint32_t t, int order,
                               uint32_t* out);
/* DsgdPpRunner::epoch master-RNG draws: schedule 2d x d (row = sub-epoch,
 * column = task id) and the d task seeds. */
void orc_dsgdpp_schedule(orc_random* r, uint32_t d, int order,
                         uint32_t* schedule, uint32_t* seeds);

/* ---- problem ------------------------------------------------------------ */
/* Global 0-based COO of the training matrix (and optionally the test matrix,
 * nnz_test may be 0).  W is m x r row-major, H is r x n column-major (i.e.
 * column j's r entries are contiguous). */
orc_problem* orc_create(uint64_t m, uint64_t n, uint32_t r, uint32_t d,
                        uint64_t nnz, const uint32_t* rows, const uint32_t* cols,
                        const double* vals,
                        uint64_t nnz_test, const uint32_t* trows,
                        const uint32_t* tcols, const double* tvals,
                        int method);
void orc_destroy(orc_problem* p);

/* update: 0 Nzsl, 1 Nzsl_L2, 2 Nzsl_Nzl2; regularize: 0 None, 1 L2;
 * loss: 0 Nzsl, 1 Nzsl_L2, 2 Nzsl_Nzl2; sgd_order: 0 SEQ, 1 WR, 2 WOR;
 * stratum_order: 0 SEQ, 1 RSEQ, 2 WR, 3 WOR, 4 COWOR. */
int orc_configure(orc_problem* p, int update, double update_lambda,
                  int regularize, double regularize_lambda,
                  int loss, double loss_lambda,
                  int truncate, double tmin, double tmax,
                  int sgd_order, int stratum_order);
void orc_set_factors(orc_problem* p, const double* W, const double* H);
void orc_get_factors(const orc_problem* p, double* W, double* H);
void orc_seed(orc_problem* p, uint32_t seed);

/* per-row / per-column nonzero counts of the training matrix */
void orc_nnz12(const orc_problem* p, uint64_t* nnz1, uint64_t* nnz2, uint64_t* nnz12max);
/* block nnz, d x 2d row-major; which: 0 train, 1 test */
void orc_block_nnz(const orc_problem* p, int which, uint64_t* out);
/* the sorted block-local records of block (b1,b2) */
uint64_t orc_block_records(const orc_problem* p, int which, uint32_t b1, uint32_t b2,
                           uint32_t* i, uint32_t* j, double* x);

/* One DsgdPpRunner::epoch with an explicit schedule and task seeds.
 * threads <= 1 runs the tasks in order on the calling thread; threads == d
 * runs one thread per task with a barrier per sub-epoch (the CPU baseline).
 * Returns the wall time of the epoch in nanoseconds. */
double orc_epoch_explicit(orc_problem* p, double eps, const uint32_t* schedule,
                          const uint32_t* seeds, int threads);
/* Same, drawing the schedule and seeds from the master RNG first. */
double orc_epoch(orc_problem* p, double eps, int threads);
/* The sequence of in-block positions each task visits, as the SGD order and
 * task RNGs produce it, for an explicit schedule and seeds: out holds, for
 * s = 0..2d-1 and task id = 0..d-1 in that order, the positions of block
 * (id, schedule[s*d+id]) (WOR: nnz_blk positions; SEQ: 0..nnz-1; WR: nnz
 * draws).  Factors are not touched. */
uint64_t orc_positions(const orc_problem* p, const uint32_t* schedule,
                       const uint32_t* seeds, uint32_t* out);

/* Losses on the current factors. which: 0 train, 1 test. */
double orc_nzsl(const orc_problem* p, int which);
double orc_l2w(const orc_problem* p);   /* sum over W blocks of sum(w^2) */
double orc_l2h(const orc_problem* p);
double orc_nzl2w(const orc_problem* p);
double orc_nzl2h(const orc_problem* p);
double orc_loss(const orc_problem* p);  /* the configured training loss */

/* defaultRunner: loss0, test0, then per epoch decay -> epoch -> loss -> test.
 * decay: 0 Const(eps0), 1 BoldDriver(eps0, dec, inc).  trace receives
 * (epochs+1) rows of {loss, test_loss, eps} (eps of row 0 is NaN). */
int orc_run(orc_problem* p, uint32_t epochs, int decay, double eps0, double dec,
            double inc, int threads, double* trace);

/* BoldDriver step: returns the new eps given the previous eps state. */
double orc_bold_driver(double eps, const double* prev_loss, double cur_loss,
                       double dec, double inc);

#ifdef __cplusplus
}
#endif
#endif
