// schedule.h -- host-side stratum schedules and point orders of the DSGD++ epoch.
//
// The reference draws every random choice of an epoch from one master
// generator on the driver thread (mf/sgd/dsgdpp_impl.h:282-349) and one
// generator per task (mf/sgd/dsgdpp_impl.h:79).  These draws are O(d^2) per
// epoch for the schedule and O(nnz) for the point orders of the replay mode;
// they stay on the host, while the GPU does the updates.
//
// Random32 pins the unvendored rg::Random32 (uma-pi1/mpi2 util library, no
// commit pinned): 32-bit MT19937 with the standard init_genrand seeding;
// nextInt(n) is Boost's bucket method (see next_int below); shuffle is the
// forward Fisher-Yates of std::random_shuffle; sample is Knuth's selection
// sampling; task seeds are one raw draw per task in task order.
#pragma once

#include <cstdint>
#include <vector>

namespace dsgdpp {

class Random32 {
 public:
  explicit Random32(uint32_t seed = 0) { seed_with(seed); }
  void seed_with(uint32_t seed);
  uint32_t next();               // raw 32-bit draw
  uint32_t next_int(uint32_t n); // uniform on [0, n)

 private:
  void refill();
  uint32_t state_[624];
  uint32_t pos_;
};

enum StratumOrder : int { kStratumSeq = 0, kStratumRseq, kStratumWr, kStratumWor, kStratumCowor };
enum SgdOrder : int { kSgdSeq = 0, kSgdWr, kSgdWor };

// rg::shuffle semantics (pinned)
void shuffle_inplace(uint32_t* a, uint64_t n, Random32& rng);
// rg::sample semantics (pinned): k sorted picks from [0, n)
std::vector<uint32_t> sorted_sample(Random32& rng, uint32_t k, uint32_t n);

// detail::computeDsgdSchedule(w, t, order, R) (mf/sgd/dsgd_impl.h:246-325):
// (w t) x (w t), row = sub-epoch, column = task.
std::vector<uint32_t> dsgd_schedule(uint32_t w, uint32_t t, int order, Random32& rng);

// DsgdPpRunner::epoch (mf/sgd/dsgdpp_impl.h:289-344): 2d x d schedule of
// column blocks (row = sub-epoch, column = task id = row block) and d task
// seeds, drawn from the master generator in the reference order.
void dsgdpp_schedule(Random32& master, uint32_t d, int order, uint32_t* schedule,
                     uint32_t* task_seeds);

// Point order of one task over its 2d sub-epochs, as SgdRunner produces it
// (mf/sgd/sgd_impl.h:197-351): the permutation buffer survives between
// sub-epochs and is reset to the identity only when the block size changes.
class TaskOrder {
 public:
  explicit TaskOrder(uint32_t seed) : rng_(seed) {}
  // Writes the visiting order of a block with n records into out[0..n).
  void next_block(int sgd_order, uint64_t n, uint32_t* out);

 private:
  Random32 rng_;
  std::vector<uint32_t> perm_;
};

// computeDefaultBlockOffsets (mf/matrix/distributed_matrix_impl.cc:24-40)
std::vector<uint64_t> block_offsets(uint64_t size, uint32_t blocks);

}  // namespace dsgdpp
