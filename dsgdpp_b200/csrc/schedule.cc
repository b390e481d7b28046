// schedule.cc -- see schedule.h.
#include "schedule.h"

#include <algorithm>
#include <numeric>

namespace dsgdpp {

// ---- MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998) ------------------
void Random32::seed_with(uint32_t seed) {
  state_[0] = seed;
  for (uint32_t k = 1; k < 624; ++k) {
    uint32_t prev = state_[k - 1];
    state_[k] = 1812433253u * (prev ^ (prev >> 30)) + k;
  }
  pos_ = 624;
}

void Random32::refill() {
  constexpr uint32_t kUpper = 0x80000000u, kLower = 0x7fffffffu, kMatrix = 0x9908b0dfu;
  uint32_t k = 0;
  for (; k < 624 - 397; ++k) {
    uint32_t y = (state_[k] & kUpper) | (state_[k + 1] & kLower);
    state_[k] = state_[k + 397] ^ (y >> 1) ^ ((y & 1u) ? kMatrix : 0u);
  }
  for (; k < 623; ++k) {
    uint32_t y = (state_[k] & kUpper) | (state_[k + 1] & kLower);
    state_[k] = state_[k + 397 - 624] ^ (y >> 1) ^ ((y & 1u) ? kMatrix : 0u);
  }
  uint32_t y = (state_[623] & kUpper) | (state_[0] & kLower);
  state_[623] = state_[396] ^ (y >> 1) ^ ((y & 1u) ? kMatrix : 0u);
  pos_ = 0;
}

uint32_t Random32::next() {
  if (pos_ >= 624) refill();
  uint32_t y = state_[pos_++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

// Boost generate_uniform_int for an engine of range [0, 2^32-1]: raw draws are
// cut into n buckets of equal width and draws past the last full bucket are
// rejected.  n == 1 needs no draw; n == 0 stands for the full 32-bit range.
uint32_t Random32::next_int(uint32_t n) {
  if (n == 1u) return 0u;
  if (n == 0u) return next();
  uint32_t width = 0xFFFFFFFFu / n + ((0xFFFFFFFFu % n == n - 1u) ? 1u : 0u);
  uint32_t v;
  do {
    v = next() / width;
  } while (v >= n);
  return v;
}

void shuffle_inplace(uint32_t* a, uint64_t n, Random32& rng) {
  for (uint64_t i = 1; i < n; ++i) {
    uint64_t j = rng.next_int((uint32_t)(i + 1));
    if (j != i) std::swap(a[i], a[j]);
  }
}

std::vector<uint32_t> sorted_sample(Random32& rng, uint32_t k, uint32_t n) {
  std::vector<uint32_t> picks;
  picks.reserve(k);
  for (uint32_t t = 0; t < n && picks.size() < k; ++t) {
    uint32_t need = k - (uint32_t)picks.size();
    if (rng.next_int(n - t) < need) picks.push_back(t);
  }
  return picks;
}

namespace {

std::vector<uint32_t> identity(uint32_t n) {
  std::vector<uint32_t> v(n);
  std::iota(v.begin(), v.end(), 0u);
  return v;
}

// mf::shuffle on a square matrix: a random row permutation matrix is applied
// from the left and a random column permutation matrix from the right
// (mf/matrix/op/shuffle.h:38-49).  Left product: new row i = old row rp[i];
// right product: old column k moves to column cp[k].
void permute_rows_cols(std::vector<uint32_t>& S, uint32_t D, Random32& rng) {
  std::vector<uint32_t> rp = identity(D);
  shuffle_inplace(rp.data(), D, rng);
  std::vector<uint32_t> cp = identity(D);
  shuffle_inplace(cp.data(), D, rng);
  std::vector<uint32_t> out(S.size());
  for (uint32_t i = 0; i < D; ++i) {
    const uint32_t* src = &S[(size_t)rp[i] * D];
    uint32_t* dst = &out[(size_t)i * D];
    for (uint32_t k = 0; k < D; ++k) dst[cp[k]] = src[k];
  }
  S.swap(out);
}

}  // namespace

std::vector<uint32_t> dsgd_schedule(uint32_t w, uint32_t t, int order, Random32& rng) {
  const uint32_t D = w * t;
  std::vector<uint32_t> S((size_t)D * D);
  for (uint32_t s = 0; s < D; ++s)
    for (uint32_t id = 0; id < D; ++id) S[(size_t)s * D + id] = (s + id) % D;

  if (order == kStratumRseq) {
    std::vector<uint32_t> relabel = identity(D);
    shuffle_inplace(relabel.data(), D, rng);
    for (auto& v : S) v = relabel[v];
  } else if (order == kStratumWr) {
    for (uint32_t s = 0; s < D; ++s) shuffle_inplace(&S[(size_t)s * D], D, rng);
  } else if (order == kStratumWor) {
    permute_rows_cols(S, D, rng);
  } else if (order == kStratumCowor) {
    // groups of t blocks; a WOR schedule over the w groups, and one WOR
    // schedule of size t inside every (group row, group column) cell
    std::vector<uint32_t> relabel = identity(D);
    shuffle_inplace(relabel.data(), D, rng);
    std::vector<uint32_t> groups = dsgd_schedule(w, 1, kStratumWor, rng);
    for (uint32_t gi = 0; gi < w; ++gi)
      for (uint32_t gj = 0; gj < w; ++gj) {
        const uint32_t base = groups[(size_t)gi * w + gj] * t;
        std::vector<uint32_t> local = dsgd_schedule(t, 1, kStratumWor, rng);
        for (uint32_t ti = 0; ti < t; ++ti)
          for (uint32_t tj = 0; tj < t; ++tj)
            S[(size_t)(gi * t + ti) * D + gj * t + tj] = relabel[base + local[(size_t)ti * t + tj]];
      }
  }
  return S;
}

void dsgdpp_schedule(Random32& master, uint32_t d, int order, uint32_t* schedule,
                     uint32_t* task_seeds) {
  // even sub-epochs use the column blocks in `even`, odd sub-epochs the rest
  std::vector<uint32_t> even(d), odd(d);
  if (order == kStratumSeq) {
    for (uint32_t k = 0; k < d; ++k) {
      even[k] = 2 * k;
      odd[k] = 2 * k + 1;
    }
  } else {
    even = sorted_sample(master, d, 2 * d);
    std::vector<char> taken(2 * d, 0);
    for (uint32_t b : even) taken[b] = 1;
    uint32_t k = 0;
    for (uint32_t b = 0; b < 2 * d && k < d; ++b)
      if (!taken[b]) odd[k++] = b;
  }
  std::vector<uint32_t> se = dsgd_schedule(1, d, order, master);
  std::vector<uint32_t> so = dsgd_schedule(1, d, order, master);
  for (uint32_t i = 0; i < d; ++i)
    for (uint32_t id = 0; id < d; ++id) {
      schedule[(size_t)(2 * i) * d + id] = even[se[(size_t)i * d + id]];
      schedule[(size_t)(2 * i + 1) * d + id] = odd[so[(size_t)i * d + id]];
    }
  for (uint32_t id = 0; id < d; ++id) task_seeds[id] = master.next();
}

void TaskOrder::next_block(int sgd_order, uint64_t n, uint32_t* out) {
  if (sgd_order == kSgdSeq) {
    for (uint64_t q = 0; q < n; ++q) out[q] = (uint32_t)q;
    return;
  }
  if (sgd_order == kSgdWr) {
    // two look-ahead draws, then one per step (the last two are unused)
    uint32_t a = rng_.next_int((uint32_t)n);
    uint32_t b = rng_.next_int((uint32_t)n);
    for (uint64_t q = 0; q < n; ++q) {
      out[q] = a;
      a = b;
      b = rng_.next_int((uint32_t)n);
    }
    return;
  }
  // WOR: Knuth shuffle of the persistent buffer, one draw ahead
  if (n == 0) return;
  if (perm_.size() != n) {
    perm_.resize(n);
    std::iota(perm_.begin(), perm_.end(), 0u);
  }
  uint64_t ahead = rng_.next_int((uint32_t)n);
  for (uint64_t step = 1; step < n; ++step) {
    uint64_t cur = ahead;
    ahead = step + rng_.next_int((uint32_t)(n - step));
    std::swap(perm_[step - 1], perm_[cur]);
  }
  std::copy(perm_.begin(), perm_.end(), out);
}

std::vector<uint64_t> block_offsets(uint64_t size, uint32_t blocks) {
  std::vector<uint64_t> off(blocks, 0);
  const uint64_t base = size / blocks, extra = size % blocks;
  // the first `extra` blocks after block 0's start get one more element
  for (uint32_t b = 1; b < blocks; ++b) off[b] = off[b - 1] + base + (b <= extra ? 1 : 0);
  return off;
}

}  // namespace dsgdpp
