// dsgdpp_oracle.cc -- CPU restatement of the reference DSGD++ epoch.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the CPU
// baseline of bench.py as the checker.  The CUDA product never links it.
//
// PARITY UNPINNED.  The reference (uma-pi1/DSGDpp) cannot be built here and
// holds no tests or golden vectors; its random-number primitives live in the
// unvendored rg/mpi2 library (github.com/uma-pi1/mpi2, no commit pinned).
// This file pins them by assumption:
//   * rg::Random32 = 32-bit MT19937 (Matsumoto & Nishimura 1998) seeded with
//     the standard init_genrand(seed) recurrence; the reference hands
//     Random32::Prng to boost::variate_generator (mf/matrix/op/generate.h:95),
//     which is consistent with a Boost mt19937 engine.
//   * nextInt(n) = uniform integer on [0, n) by Boost's bucket method for an
//     engine of range 2^32-1: bucket = 0xFFFFFFFF / n, plus one when n divides
//     2^32; draw raw >> until raw / bucket < n.  nextInt(1) returns 0 and
//     consumes no draw; nextInt(0) returns one raw draw.
//   * rg::shuffle(first, last, R) = forward Fisher-Yates: for i = 1..n-1,
//     j = nextInt(i+1), swap(a[i], a[j]) (the form of std::random_shuffle
//     with a generator).
//   * rg::sample(R, k, n) = Knuth's selection sampling (Algorithm S, TAOCP
//     vol. 2, 3.4.2): visit t = 0..n-1 and select t when
//     nextInt(n - t) < k - selected; the result is sorted.
//   * mpi2::seed(channels, R) gives task id = 0..d-1, in that order, one raw
//     32-bit draw each; mpi2::getSeed returns it and the task builds
//     Random32(seed).
// Floating-point arithmetic follows the reference expressions operation by
// operation in source order, compiled with -ffp-contract=off (no FMA
// contraction), so the CUDA replay can reproduce it bit for bit.

#include "dsgdpp_oracle.h"

#include <algorithm>
#include <atomic>
#include <barrier>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

namespace {

// ---- Random32 ---------------------------------------------------------------
class Random32 {
 public:
  explicit Random32(uint32_t seed) { reseed(seed); }
  void reseed(uint32_t seed) {
    mt_[0] = seed;
    for (int i = 1; i < 624; ++i)
      mt_[i] = 1812433253u * (mt_[i - 1] ^ (mt_[i - 1] >> 30)) + (uint32_t)i;
    idx_ = 624;
  }
  uint32_t next() {
    if (idx_ >= 624) twist();
    uint32_t y = mt_[idx_++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
  }
  uint32_t nextInt(uint32_t n) {
    if (n == 1) return 0;
    if (n == 0) return next();
    const uint32_t range = n - 1;
    uint32_t bucket = 0xFFFFFFFFu / n;
    if (0xFFFFFFFFu % n == range) ++bucket;
    for (;;) {
      uint32_t v = next() / bucket;
      if (v <= range) return v;
    }
  }

 private:
  void twist() {
    for (int i = 0; i < 624; ++i) {
      uint32_t y = (mt_[i] & 0x80000000u) | (mt_[(i + 1) % 624] & 0x7fffffffu);
      uint32_t v = mt_[(i + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      mt_[i] = v;
    }
    idx_ = 0;
  }
  uint32_t mt_[624];
  int idx_;
};

template <typename T>
void shuffle(std::vector<T>& a, Random32& r) {  // rg::shuffle (pinned)
  for (size_t i = 1; i < a.size(); ++i) {
    size_t j = r.nextInt((uint32_t)(i + 1));
    if (i != j) std::swap(a[i], a[j]);
  }
}

std::vector<uint32_t> sample(Random32& r, uint32_t k, uint32_t n) {  // rg::sample
  std::vector<uint32_t> out;
  out.reserve(k);
  uint32_t selected = 0;
  for (uint32_t t = 0; t < n && selected < k; ++t) {
    if (r.nextInt(n - t) < k - selected) {
      out.push_back(t);
      ++selected;
    }
  }
  return out;
}

// computeDefaultBlockOffsets (mf/matrix/distributed_matrix_impl.cc:24-40)
std::vector<uint64_t> blockOffsets(uint64_t size, uint32_t blocks) {
  std::vector<uint64_t> off(blocks);
  uint64_t minSize = size / blocks, rem = size % blocks;
  for (uint32_t i = 0; i < blocks; ++i) {
    if (i == 0) {
      off[i] = 0;
    } else {
      off[i] = minSize + off[i - 1];
      if (rem > 0) { ++off[i]; --rem; }
    }
  }
  return off;
}

// computeDsgdSchedule (mf/sgd/dsgd_impl.h:246-325), row-major d x d.
enum { SO_SEQ = 0, SO_RSEQ = 1, SO_WR = 2, SO_WOR = 3, SO_COWOR = 4 };

// mf::shuffle (mf/matrix/op/shuffle.h:38-49): rows gathered by v, columns
// scattered by u; v is drawn before u.
void shuffleMatrix(std::vector<uint32_t>& S, uint32_t D, Random32& R) {
  std::vector<uint32_t> v(D), u(D);
  std::iota(v.begin(), v.end(), 0u);
  shuffle(v, R);
  std::iota(u.begin(), u.end(), 0u);
  shuffle(u, R);
  std::vector<uint32_t> rows(S.size());
  for (uint32_t i = 0; i < D; ++i)
    for (uint32_t k = 0; k < D; ++k) rows[i * D + k] = S[v[i] * D + k];
  for (uint32_t i = 0; i < D; ++i)
    for (uint32_t k = 0; k < D; ++k) S[i * D + u[k]] = rows[i * D + k];
}

std::vector<uint32_t> computeDsgdSchedule(uint32_t w, uint32_t t, int order, Random32& R) {
  const uint32_t D = w * t;
  std::vector<uint32_t> S((size_t)D * D);
  for (uint32_t s = 0; s < D; ++s)
    for (uint32_t id = 0; id < D; ++id) S[(size_t)s * D + id] = (s + id) % D;
  switch (order) {
    case SO_SEQ:
      break;
    case SO_RSEQ: {
      std::vector<uint32_t> b(D);
      std::iota(b.begin(), b.end(), 0u);
      shuffle(b, R);
      for (auto& e : S) e = b[e];
    } break;
    case SO_WR:
      for (uint32_t s = 0; s < D; ++s) {
        std::vector<uint32_t> row(S.begin() + (size_t)s * D, S.begin() + (size_t)(s + 1) * D);
        shuffle(row, R);
        std::copy(row.begin(), row.end(), S.begin() + (size_t)s * D);
      }
      break;
    case SO_WOR:
      shuffleMatrix(S, D, R);
      break;
    case SO_COWOR: {
      std::vector<uint32_t> blocks(D);
      std::iota(blocks.begin(), blocks.end(), 0u);
      shuffle(blocks, R);
      std::vector<uint32_t> G = computeDsgdSchedule(w, 1, SO_WOR, R);
      for (uint32_t bi = 0; bi < w; ++bi)
        for (uint32_t bj = 0; bj < w; ++bj) {
          uint32_t go = G[bi * w + bj] * t;
          std::vector<uint32_t> L = computeDsgdSchedule(t, 1, SO_WOR, R);
          for (uint32_t ti = 0; ti < t; ++ti)
            for (uint32_t tj = 0; tj < t; ++tj)
              S[(size_t)(bi * t + ti) * D + bj * t + tj] = blocks[go + L[ti * t + tj]];
        }
    } break;
  }
  return S;
}

// DsgdPpRunner::epoch master-RNG part (mf/sgd/dsgdpp_impl.h:289-344)
void dsgdppSchedule(Random32& R, uint32_t d, int order, uint32_t* sched, uint32_t* seeds) {
  std::vector<uint32_t> b0(d), b1(d);
  if (order == SO_SEQ) {
    for (uint32_t k = 0; k < d; ++k) { b0[k] = 2 * k; b1[k] = 2 * k + 1; }
  } else {
    b0 = sample(R, d, 2 * d);
    uint32_t i0 = 0, i1 = 0;
    for (uint32_t b = 0; i1 < d && b < 2 * d; ++b) {
      if (i0 < d && b0[i0] == b) { ++i0; continue; }
      b1[i1++] = b;
    }
  }
  std::vector<uint32_t> s0 = computeDsgdSchedule(1, d, order, R);
  std::vector<uint32_t> s1 = computeDsgdSchedule(1, d, order, R);
  for (uint32_t i = 0; i < d; ++i)
    for (uint32_t id = 0; id < d; ++id) {
      sched[(size_t)(2 * i) * d + id] = b0[s0[(size_t)i * d + id]];
      sched[(size_t)(2 * i + 1) * d + id] = b1[s1[(size_t)i * d + id]];
    }
  for (uint32_t id = 0; id < d; ++id) seeds[id] = R.next();
}

}  // namespace

// ---- problem ------------------------------------------------------------------
struct Block {
  std::vector<uint32_t> i, j;  // block-local, sorted (i, j)
  std::vector<double> x;
};

struct orc_problem {
  uint64_t m = 0, n = 0;
  uint32_t r = 0, d = 0;
  uint32_t nb2 = 0;  // column blocks = sub-epochs: 2d (DSGD++) or d (DSGD)
  int method = 0;    // 0 DSGD++, 1 DSGD
  std::vector<uint64_t> off1, off2;
  std::vector<Block> train, test;  // d x 2d row-major
  std::vector<double> W, H;        // W m x r row-major; H col-major (col j contiguous)
  std::vector<uint64_t> nnz1, nnz2;
  uint64_t nnz12max = 0;
  int update = 1, regularize = 0, loss = 1, truncate = 0, sgdOrder = 2, stratumOrder = 4;
  double updateLambda = 1, regularizeLambda = 0, lossLambda = 1, tmin = NAN, tmax = NAN;
  Random32 master{0};
};

struct orc_random {
  Random32 r;
  explicit orc_random(uint32_t s) : r(s) {}
};

namespace {

uint32_t blockOf(uint64_t i, const std::vector<uint64_t>& off) {
  return (uint32_t)(std::upper_bound(off.begin(), off.end(), i) - off.begin() - 1);
}

// ReadMatrixBlocksMm::process + coordinate_matrix::sort (mf/matrix/io/read_impl.h:416-422,
// 162-164): block-local coordinates, (i, j) order, duplicates summed in file order.
std::vector<Block> blockMatrix(const orc_problem& p, uint64_t nnz, const uint32_t* rows,
                               const uint32_t* cols, const double* vals) {
  const uint32_t d = p.d, d2 = p.nb2;
  const size_t nblk = (size_t)d * d2;
  // route entries to blocks on all host threads; thread t takes a contiguous
  // range of entries, so each block lists its entries in input order
  const unsigned T = nnz > (1u << 20) ? std::max(1u, std::thread::hardware_concurrency()) : 1u;
  std::vector<uint32_t> bid(nnz);
  std::vector<std::vector<uint64_t>> cnt(T, std::vector<uint64_t>(nblk + 1, 0));
  auto range = [&](unsigned t) { return std::make_pair(nnz * t / T, nnz * (t + 1) / T); };
  auto par = [&](auto&& fn) {
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < T; ++t) pool.emplace_back(fn, t);
    fn(0u);
    for (auto& th : pool) th.join();
  };
  par([&](unsigned t) {
    auto [a, b] = range(t);
    for (uint64_t k = a; k < b; ++k) {
      const uint32_t blk = blockOf(rows[k], p.off1) * d2 + blockOf(cols[k], p.off2);
      bid[k] = blk;
      cnt[t][blk]++;
    }
  });
  std::vector<uint64_t> start(nblk + 1, 0);
  for (size_t blk = 0; blk < nblk; ++blk) {
    uint64_t acc = start[blk];
    for (unsigned t = 0; t < T; ++t) {
      const uint64_t c = cnt[t][blk];
      cnt[t][blk] = acc;
      acc += c;
    }
    start[blk + 1] = acc;
  }
  std::vector<uint64_t> idx(nnz);
  par([&](unsigned t) {
    auto [a, b] = range(t);
    for (uint64_t k = a; k < b; ++k) idx[cnt[t][bid[k]]++] = k;
  });
  std::vector<uint32_t>().swap(bid);
  std::vector<Block> out(nblk);
  // blocks are independent: sort (row-major (i, j), mf/matrix/io/read_impl.h:
  // 162-164) and merge duplicates on all host threads
  std::atomic<size_t> next{0};
  par([&](unsigned) {
    for (size_t blk = next++; blk < nblk; blk = next++) {
      const uint32_t b1 = (uint32_t)(blk / d2), b2 = (uint32_t)(blk % d2);
      uint64_t* ib = idx.data() + start[blk];
      uint64_t* ie = idx.data() + start[blk + 1];
      std::stable_sort(ib, ie, [&](uint64_t a, uint64_t c) {
        return rows[a] != rows[c] ? rows[a] < rows[c] : cols[a] < cols[c];
      });
      Block& B = out[blk];
      B.i.reserve(ie - ib);
      B.j.reserve(ie - ib);
      B.x.reserve(ie - ib);
      for (const uint64_t* q = ib; q != ie; ++q) {
        const uint64_t k = *q;
        uint32_t li = (uint32_t)(rows[k] - p.off1[b1]), lj = (uint32_t)(cols[k] - p.off2[b2]);
        if (!B.i.empty() && B.i.back() == li && B.j.back() == lj) {
          B.x.back() += vals[k];
        } else {
          B.i.push_back(li);
          B.j.push_back(lj);
          B.x.push_back(vals[k]);
        }
      }
    }
  });
  return out;
}

// The factor view one task gets for block (b1, b2) (FactorizationData,
// mf/factorization.h; built at mf/sgd/dsgdpp_impl.h:238-239).
struct BlockJob {
  const Block* v;
  double* w;  // W block base (row-major, r)
  double* h;  // H block base (column-major, r)
  uint32_t r;
  uint64_t mBlk, nBlk;
  const uint64_t* nnz1;  // already offset by blockOffset1(b1)
  const uint64_t* nnz2;  // already offset by blockOffset2(b2)
};

// UpdateNzsl (mf/sgd/functions/update-nzsl.h:33-50), UpdateNzslL2
// (update-nzsl-l2.h:34-57), UpdateNzslNzl2 (update-nzsl-nzl2.h:34-53),
// optionally wrapped by UpdateTruncate (update-truncate.h:50-72).
inline void updateOne(const orc_problem& p, BlockJob& J, uint32_t i, uint32_t j, double x,
                      double eps) {
  const uint32_t r = J.r;
  double* w = J.w + (uint64_t)i * r;
  double* h = J.h + (uint64_t)j * r;
  double wh = 0;
  for (uint32_t z = 0; z < r; ++z) wh += w[z] * h[z];
  if (p.update == 0) {
    double f = eps * -2. * (x - wh);
    for (uint32_t z = 0; z < r; ++z) {
      double temp = w[z];
      w[z] -= f * h[z];
      h[z] -= f * temp;
    }
  } else if (p.update == 1) {
    double f1 = eps * -2. * (x - wh);
    double f2 = eps * 2. * p.updateLambda;
    double f3 = 1. / (double)J.nnz1[i];
    double f4 = 1. / (double)J.nnz2[j];
    for (uint32_t z = 0; z < r; ++z) {
      double temp = w[z];
      w[z] -= f1 * h[z] + f2 * w[z] * f3;
      h[z] -= f1 * temp + f2 * h[z] * f4;
    }
  } else {
    double f1 = eps * -2. * (x - wh);
    double f2 = eps * 2. * p.updateLambda;
    for (uint32_t z = 0; z < r; ++z) {
      double temp = w[z];
      w[z] -= f1 * h[z] + f2 * w[z];
      h[z] -= f1 * temp + f2 * h[z];
    }
  }
  if (p.truncate) {
    for (uint32_t z = 0; z < r; ++z) {
      double& a = w[z];
      if (a <= p.tmin) a = p.tmin + eps;
      else if (a >= p.tmax) a = p.tmax - eps;
      double& b = h[z];
      if (b <= p.tmin) b = p.tmin + eps;
      else if (b >= p.tmax) b = p.tmax - eps;
    }
  }
}

// RegularizeNone / RegularizeL2 (mf/sgd/functions/regularize-l2.h:26-45);
// RegularizeTruncate<RegularizeNone> is a no-op (regularize-truncate.h:89-131).
void regularizeBlock(const orc_problem& p, BlockJob& J, double eps) {
  if (p.regularize != 1) return;
  if (p.regularizeLambda == 0) return;
  double factor = 1 - eps * 2 * p.regularizeLambda;
  if (factor < 0.5) factor = 0.25 / (1 - factor);
  for (uint64_t q = 0; q < J.mBlk * J.r; ++q) J.w[q] *= factor;
  for (uint64_t q = 0; q < J.r * J.nBlk; ++q) J.h[q] *= factor;
  if (p.truncate) {
    for (uint64_t q = 0; q < J.mBlk * J.r; ++q) {
      double& a = J.w[q];
      if (a <= p.tmin) a = p.tmin + eps;
      else if (a >= p.tmax) a = p.tmax - eps;
    }
    for (uint64_t q = 0; q < J.r * J.nBlk; ++q) {
      double& b = J.h[q];
      if (b <= p.tmin) b = p.tmin + eps;
      else if (b >= p.tmax) b = p.tmax - eps;
    }
  }
}

// SgdRunner (mf/sgd/sgd_impl.h): one per task per epoch; permutation_ survives
// across the task's sub-epochs and is reset only when the block size changes.
struct TaskRunner {
  Random32 rng;
  std::vector<uint64_t> perm;
  explicit TaskRunner(uint32_t seed) : rng(seed) {}

  // SgdRunner::permute (sgd_impl.h:255-279)
  void permute(uint64_t n, uint64_t k) {
    if (perm.size() != n) {
      perm.resize(n);
      for (uint64_t q = 0; q < n; ++q) perm[q] = q;
    }
    uint64_t cur = 0, next = rng.nextInt((uint32_t)n);
    for (uint64_t step = 1; step < k; ++step) {
      cur = next;
      next = step + rng.nextInt((uint32_t)(n - step));
      std::swap(perm[step - 1], perm[cur]);
    }
  }

  // Emits the visiting order for a block of n records into out (length n).
  void positions(int order, uint64_t n, uint32_t* out) {
    if (order == 0) {  // SEQ (sgd_impl.h:197-217)
      for (uint64_t q = 0; q < n; ++q) out[q] = (uint32_t)q;
    } else if (order == 1) {  // WR (sgd_impl.h:224-252)
      uint64_t nextPos = rng.nextInt((uint32_t)n);
      uint64_t next2Pos = rng.nextInt((uint32_t)n);
      for (uint64_t step = 0; step < n; ++step) {
        uint64_t curPos = nextPos;
        nextPos = next2Pos;
        next2Pos = rng.nextInt((uint32_t)n);
        out[step] = (uint32_t)curPos;
      }
    } else {  // WOR (sgd_impl.h:282-351)
      if (n == 0) return;
      permute(n, n);
      for (uint64_t q = 0; q < n; ++q) out[q] = (uint32_t)perm[q];
    }
  }
};

BlockJob makeJob(orc_problem& p, uint32_t b1, uint32_t b2) {
  BlockJob J;
  J.v = &p.train[(size_t)b1 * p.nb2 + b2];
  J.r = p.r;
  J.mBlk = (b1 + 1 < p.d ? p.off1[b1 + 1] : p.m) - p.off1[b1];
  J.nBlk = (b2 + 1 < p.nb2 ? p.off2[b2 + 1] : p.n) - p.off2[b2];
  J.w = p.W.data() + p.off1[b1] * p.r;
  J.h = p.H.data() + p.off2[b2] * p.r;
  J.nnz1 = p.nnz1.data() + p.off1[b1];
  J.nnz2 = p.nnz2.data() + p.off2[b2];
  return J;
}

// DsgdPpTask::run body for one sub-epoch (mf/sgd/dsgdpp_impl.h:117-263) and
// SgdRunner::epoch (sgd_impl.h:192-195).
void runTaskSubepoch(orc_problem& p, TaskRunner& tr, uint32_t id, uint32_t b2, double eps,
                     std::vector<uint32_t>& scratch) {
  BlockJob J = makeJob(p, id, b2);
  const uint64_t n = J.v->x.size();
  scratch.resize(n);
  tr.positions(p.sgdOrder, n, scratch.data());
  for (uint64_t q = 0; q < n; ++q) {
    uint32_t pos = scratch[q];
    updateOne(p, J, J.v->i[pos], J.v->j[pos], J.v->x[pos], eps);
  }
  regularizeBlock(p, J, eps / p.d);  // RegularizeNone/L2: rescaleStratumStepsize() == true
}

double epochExplicit(orc_problem& p, double eps, const uint32_t* sched, const uint32_t* seeds,
                     int threads) {
  auto t0 = std::chrono::steady_clock::now();
  const uint32_t d = p.d;
  std::vector<TaskRunner> tasks;
  tasks.reserve(d);
  for (uint32_t id = 0; id < d; ++id) tasks.emplace_back(seeds[id]);
  if (threads <= 1) {
    std::vector<uint32_t> scratch;
    for (uint32_t s = 0; s < p.nb2; ++s)
      for (uint32_t id = 0; id < d; ++id)
        runTaskSubepoch(p, tasks[id], id, sched[(size_t)s * d + id], eps, scratch);
  } else {
    // T threads run the d tasks of each sub-epoch, a task to whichever thread
    // claims it next (the tasks of a sub-epoch are row- and column-disjoint, and
    // each keeps its own generator and permutation, so the result does not
    // depend on which thread runs it); a barrier ends every sub-epoch.
    const int T = std::min<int>(threads, (int)d);
    std::barrier<> bar(T);
    std::vector<std::atomic<uint32_t>> claim(p.nb2);
    for (auto& c : claim) c.store(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) {
      pool.emplace_back([&]() {
        std::vector<uint32_t> scratch;
        for (uint32_t s = 0; s < p.nb2; ++s) {
          for (uint32_t id = claim[s]++; id < d; id = claim[s]++)
            runTaskSubepoch(p, tasks[id], id, sched[(size_t)s * d + id], eps, scratch);
          bar.arrive_and_wait();  // barrier(channels), dsgdpp_impl.h:259-263
        }
      });
    }
    for (auto& th : pool) th.join();
  }
  auto t1 = std::chrono::steady_clock::now();
  return (double)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
}

// nzsl over one block (mf/loss/nzsl.h:29-52)
double nzslBlock(const orc_problem& p, const Block& B, uint32_t b1, uint32_t b2) {
  const double* w = p.W.data() + p.off1[b1] * p.r;
  const double* h = p.H.data() + p.off2[b2] * p.r;
  double result = 0;
  for (size_t q = 0; q < B.x.size(); ++q) {
    double ip = 0;
    const double* wr = w + (uint64_t)B.i[q] * p.r;
    const double* hc = h + (uint64_t)B.j[q] * p.r;
    for (uint32_t z = 0; z < p.r; ++z) ip += wr[z] * hc[z];
    double diff = B.x[q] - ip;
    result += diff * diff;
  }
  return result;
}

}  // namespace

extern "C" {

orc_random* orc_random_create(uint32_t seed) { return new orc_random(seed); }
void orc_random_destroy(orc_random* r) { delete r; }
uint32_t orc_random_next(orc_random* r) { return r->r.next(); }
uint32_t orc_random_next_int(orc_random* r, uint32_t n) { return r->r.nextInt(n); }
void orc_random_shuffle_u32(orc_random* r, uint32_t* a, uint64_t n) {
  std::vector<uint32_t> v(a, a + n);
  shuffle(v, r->r);
  std::copy(v.begin(), v.end(), a);
}
void orc_random_sample(orc_random* r, uint32_t k, uint32_t n, uint32_t* out) {
  std::vector<uint32_t> v = sample(r->r, k, n);
  std::copy(v.begin(), v.end(), out);
}

void orc_block_offsets(uint64_t size, uint32_t blocks, uint64_t* out) {
  std::vector<uint64_t> o = blockOffsets(size, blocks);
  std::copy(o.begin(), o.end(), out);
}

void orc_compute_dsgd_schedule(orc_random* r, uint32_t w, uint32_t t, int order, uint32_t* out) {
  std::vector<uint32_t> S = computeDsgdSchedule(w, t, order, r->r);
  std::copy(S.begin(), S.end(), out);
}

void orc_dsgdpp_schedule(orc_random* r, uint32_t d, int order, uint32_t* schedule,
                         uint32_t* seeds) {
  dsgdppSchedule(r->r, d, order, schedule, seeds);
}

orc_problem* orc_create(uint64_t m, uint64_t n, uint32_t r, uint32_t d, uint64_t nnz,
                        const uint32_t* rows, const uint32_t* cols, const double* vals,
                        uint64_t nnz_test, const uint32_t* trows, const uint32_t* tcols,
                        const double* tvals, int method) {
  if (d == 0 || r == 0 || method < 0 || method > 1) return nullptr;
  auto* p = new orc_problem();
  p->m = m; p->n = n; p->r = r; p->d = d;
  p->method = method;
  p->nb2 = method == 1 ? d : 2 * d;  // DSGD: d x d blocks (mf/sgd/dsgd_impl.h:328-350)
  p->off1 = blockOffsets(m, d);
  p->off2 = blockOffsets(n, p->nb2);
  p->train = blockMatrix(*p, nnz, rows, cols, vals);
  p->test = blockMatrix(*p, nnz_test, trows, tcols, tvals);
  p->W.assign(m * r, 0.0);
  p->H.assign(n * r, 0.0);
  // nnz12 over the blocks (mf/matrix/op/nnz.h:124-163)
  p->nnz1.assign(m, 0);
  p->nnz2.assign(n, 0);
  for (uint32_t b1 = 0; b1 < d; ++b1)
    for (uint32_t b2 = 0; b2 < p->nb2; ++b2) {
      const Block& B = p->train[(size_t)b1 * p->nb2 + b2];
      for (size_t q = 0; q < B.x.size(); ++q) {
        p->nnz1[B.i[q] + p->off1[b1]]++;
        p->nnz2[B.j[q] + p->off2[b2]]++;
      }
    }
  p->nnz12max = 0;
  for (auto c : p->nnz1) p->nnz12max = std::max(p->nnz12max, c);
  for (auto c : p->nnz2) p->nnz12max = std::max(p->nnz12max, c);
  return p;
}

void orc_destroy(orc_problem* p) { delete p; }

int orc_configure(orc_problem* p, int update, double update_lambda, int regularize,
                  double regularize_lambda, int loss, double loss_lambda, int truncate,
                  double tmin, double tmax, int sgd_order, int stratum_order) {
  if (update < 0 || update > 2 || regularize < 0 || regularize > 1 || loss < 0 || loss > 2 ||
      sgd_order < 0 || sgd_order > 2 || stratum_order < 0 || stratum_order > 4)
    return -1;
  p->update = update; p->updateLambda = update_lambda;
  p->regularize = regularize; p->regularizeLambda = regularize_lambda;
  p->loss = loss; p->lossLambda = loss_lambda;
  p->truncate = truncate; p->tmin = tmin; p->tmax = tmax;
  p->sgdOrder = sgd_order; p->stratumOrder = stratum_order;
  return 0;
}

void orc_set_factors(orc_problem* p, const double* W, const double* H) {
  std::copy(W, W + p->m * p->r, p->W.begin());
  std::copy(H, H + p->n * p->r, p->H.begin());
}
void orc_get_factors(const orc_problem* p, double* W, double* H) {
  std::copy(p->W.begin(), p->W.end(), W);
  std::copy(p->H.begin(), p->H.end(), H);
}
void orc_seed(orc_problem* p, uint32_t seed) { p->master.reseed(seed); }

void orc_nnz12(const orc_problem* p, uint64_t* nnz1, uint64_t* nnz2, uint64_t* nnz12max) {
  std::copy(p->nnz1.begin(), p->nnz1.end(), nnz1);
  std::copy(p->nnz2.begin(), p->nnz2.end(), nnz2);
  *nnz12max = p->nnz12max;
}

void orc_block_nnz(const orc_problem* p, int which, uint64_t* out) {
  const auto& Bs = which ? p->test : p->train;
  for (size_t b = 0; b < Bs.size(); ++b) out[b] = Bs[b].x.size();
}

uint64_t orc_block_records(const orc_problem* p, int which, uint32_t b1, uint32_t b2,
                           uint32_t* i, uint32_t* j, double* x) {
  const Block& B = (which ? p->test : p->train)[(size_t)b1 * p->nb2 + b2];
  if (i) std::copy(B.i.begin(), B.i.end(), i);
  if (j) std::copy(B.j.begin(), B.j.end(), j);
  if (x) std::copy(B.x.begin(), B.x.end(), x);
  return B.x.size();
}

double orc_epoch_explicit(orc_problem* p, double eps, const uint32_t* schedule,
                          const uint32_t* seeds, int threads) {
  return epochExplicit(*p, eps, schedule, seeds, threads);
}

double orc_epoch(orc_problem* p, double eps, int threads) {
  std::vector<uint32_t> sched((size_t)p->nb2 * p->d), seeds(p->d);
  auto t0 = std::chrono::steady_clock::now();
  if (p->method == 1) {  // DsgdRunner::epoch (mf/sgd/dsgd_impl.h:328-350): schedule, then task seeds
    const std::vector<uint32_t> S = computeDsgdSchedule(1, p->d, p->stratumOrder, p->master);
    std::copy(S.begin(), S.end(), sched.begin());
    for (uint32_t id = 0; id < p->d; ++id) seeds[id] = p->master.next();
  } else {
    dsgdppSchedule(p->master, p->d, p->stratumOrder, sched.data(), seeds.data());
  }
  auto t1 = std::chrono::steady_clock::now();
  return epochExplicit(*p, eps, sched.data(), seeds.data(), threads) +
         (double)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
}

uint64_t orc_positions(const orc_problem* p, const uint32_t* schedule, const uint32_t* seeds,
                       uint32_t* out) {
  const uint32_t d = p->d;
  std::vector<TaskRunner> tasks;
  for (uint32_t id = 0; id < d; ++id) tasks.emplace_back(seeds[id]);
  uint64_t at = 0;
  for (uint32_t s = 0; s < p->nb2; ++s)
    for (uint32_t id = 0; id < d; ++id) {
      const Block& B = p->train[(size_t)id * p->nb2 + schedule[(size_t)s * d + id]];
      uint64_t n = B.x.size();
      if (out) tasks[id].positions(p->sgdOrder, n, out + at);
      else {
        std::vector<uint32_t> tmp(n);
        tasks[id].positions(p->sgdOrder, n, tmp.data());
      }
      at += n;
    }
  return at;
}

double orc_nzsl(const orc_problem* p, int which) {
  // per-block sums, then sum over the d x 2d result matrix in row-major order
  // (runTaskOnBlocks3 + sum, mf/matrix/op/sum.h:27-30)
  const auto& Bs = which ? p->test : p->train;
  double total = 0;
  for (uint32_t b1 = 0; b1 < p->d; ++b1)
    for (uint32_t b2 = 0; b2 < p->nb2; ++b2)
      total += nzslBlock(*p, Bs[(size_t)b1 * p->nb2 + b2], b1, b2);
  return total;
}

// l2 over the W blocks (mf/loss/l2.h:39-48, 150-181): std::accumulate per
// block, block sums accumulated in block order.
double orc_l2w(const orc_problem* p) {
  double total = 0;
  for (uint32_t b1 = 0; b1 < p->d; ++b1) {
    uint64_t lo = p->off1[b1] * p->r, hi = (b1 + 1 < p->d ? p->off1[b1 + 1] : p->m) * p->r;
    double s = 0;
    for (uint64_t q = lo; q < hi; ++q) s = s + p->W[q] * p->W[q];
    total += s;
  }
  return total;
}
double orc_l2h(const orc_problem* p) {
  double total = 0;
  for (uint32_t b2 = 0; b2 < p->nb2; ++b2) {
    uint64_t lo = p->off2[b2] * p->r, hi = (b2 + 1 < p->nb2 ? p->off2[b2 + 1] : p->n) * p->r;
    double s = 0;
    for (uint64_t q = lo; q < hi; ++q) s = s + p->H[q] * p->H[q];
    total += s;
  }
  return total;
}
// nzl2 (mf/loss/nzl2.h:29-87).  The reference leaves `double result`
// uninitialised; it is taken as 0 here.
double orc_nzl2w(const orc_problem* p) {
  double total = 0;
  for (uint32_t b1 = 0; b1 < p->d; ++b1) {
    uint64_t lo = p->off1[b1], hi = (b1 + 1 < p->d ? p->off1[b1 + 1] : p->m);
    double result = 0;
    for (uint64_t i = lo; i < hi; ++i) {
      double v = 0;
      for (uint32_t z = 0; z < p->r; ++z) { double vv = p->W[i * p->r + z]; v += vv * vv; }
      result += (double)p->nnz1[i] * v;
    }
    total += result;
  }
  return total;
}
double orc_nzl2h(const orc_problem* p) {
  double total = 0;
  for (uint32_t b2 = 0; b2 < p->nb2; ++b2) {
    uint64_t lo = p->off2[b2], hi = (b2 + 1 < p->nb2 ? p->off2[b2 + 1] : p->n);
    double result = 0;
    for (uint64_t j = lo; j < hi; ++j) {
      double v = 0;
      for (uint32_t z = 0; z < p->r; ++z) { double vv = p->H[j * p->r + z]; v += vv * vv; }
      result += (double)p->nnz2[j] * v;
    }
    total += result;
  }
  return total;
}

// SumLoss<NzslLoss, L2Loss|Nzl2Loss> or NzslLoss (mf/loss/loss.h:88-112)
double orc_loss(const orc_problem* p) {
  double l = orc_nzsl(p, 0);
  if (p->loss == 1) l = l + p->lossLambda * (orc_l2w(p) + orc_l2h(p));
  else if (p->loss == 2) l = l + p->lossLambda * (orc_nzl2w(p) + orc_nzl2h(p));
  return l;
}

// BoldDriver (mf/sgd/decay/decay_bolddriver.h:59-67)
double orc_bold_driver(double eps, const double* prev_loss, double cur_loss, double dec,
                       double inc) {
  if (prev_loss == nullptr) return eps;
  if (*prev_loss <= cur_loss) return eps * dec;
  return eps * inc;
}

// detail::defaultRunner (mf/sgd/sgd_impl.h:34-145)
int orc_run(orc_problem* p, uint32_t epochs, int decay, double eps0, double dec, double inc,
            int threads, double* trace) {
  double prev = 0, cur = orc_loss(p);
  double test = orc_nzsl(p, 1);
  trace[0] = cur; trace[1] = test; trace[2] = NAN;
  double epsState = eps0;
  for (uint32_t e = 0; e < epochs; ++e) {
    double eps;
    if (decay == 0) eps = eps0;
    else {
      epsState = orc_bold_driver(epsState, e == 0 ? nullptr : &prev, cur, dec, inc);
      eps = epsState;
    }
    orc_epoch(p, eps, threads);
    prev = cur;
    cur = orc_loss(p);
    test = orc_nzsl(p, 1);
    trace[3 * (e + 1) + 0] = cur;
    trace[3 * (e + 1) + 1] = test;
    trace[3 * (e + 1) + 2] = eps;
  }
  return 0;
}

}  // extern "C"
