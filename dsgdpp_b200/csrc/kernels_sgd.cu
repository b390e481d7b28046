// kernels_sgd.cu -- the per-nonzero SGD step of DSGD++ on sm_100a.
//
// Reference hot loop: SgdRunner::updateWor (mf/sgd/sgd_impl.h:293-351) calling
// UpdateNzslL2 / UpdateNzsl / UpdateNzslNzl2 (mf/sgd/functions/update-*.h),
// one thread per block, d blocks per sub-epoch (mf/sgd/dsgdpp_impl.h:117-263).
//
// Two kernels:
//  * hogwild_subepoch: the throughput path.  The sub-epoch's d blocks share no
//    row of W and no column of H, so their records form one work list that
//    every SM draws 32-record chunks from.  Inside a warp, groups of LPN lanes
//    each own one record; a lane moves VPL 16-byte vectors of the W row and of
//    the H column.  Within a block updates run concurrently (Hogwild).
//  * replay_subepoch: the deterministic FP64 mode.  One warp per task walks its
//    block in the exact point order of the reference and repeats every
//    floating-point operation of the reference in the same order, without FMA
//    contraction, so the result matches the CPU restatement bit for bit.
#include "kernels.cuh"

namespace dsgdpp {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Eight primes just below 2^31; a prime above the chunk count is coprime to
// it, so c -> (A c + B) mod C is a permutation of the chunks.
__constant__ uint32_t kPrimes[8] = {2147483647u, 2147483629u, 2147483587u, 2147483579u,
                                    2147483563u, 2147483549u, 2147483543u, 2147483497u};

template <typename C>
__device__ __forceinline__ C clampw(C v, C lo, C hi, C eps) {
  // UpdateTruncate (mf/sgd/functions/update-truncate.h:50-72)
  if (v <= lo) return lo + eps;
  if (v >= hi) return hi - eps;
  return v;
}

template <typename T>
__device__ __forceinline__ void store_vec(T* p, const typename Elem<T>::C (&f)[Elem<T>::VW],
                                          const Philox4*) {
  *reinterpret_cast<uint4*>(p) = Elem<T>::pack(f);
}
template <>
__device__ __forceinline__ void store_vec<__nv_bfloat16>(__nv_bfloat16* p, const float (&f)[8],
                                                         const Philox4* rnd) {
  uint32_t w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) w[k] = bf16x2_sr(f[2 * k], f[2 * k + 1], rnd->v[k]);
  *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
}

// BF16 atomic write: the new value is rounded stochastically against the
// value read (exactly as a store would write it), and the difference between
// that rounded value and the value read -- exact in BF16 for updates of a few
// ulps -- is added with one 16-byte vector atomic.  Without a concurrent update
// the row ends exactly as a store would leave it; with one, neither is lost.
__device__ __forceinline__ void red_bf16_increment(__nv_bfloat16* q, const uint4& old,
                                                   const float (&nv)[8], const Philox4& rnd) {
  const uint32_t ow[4] = {old.x, old.y, old.z, old.w};
  uint32_t inc[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) inc[k] = bf16x2_sub(bf16x2_sr(nv[2 * k], nv[2 * k + 1], rnd.v[k]), ow[k]);
  asm volatile("red.relaxed.gpu.global.add.noftz.v4.bf16x2 [%0], {%1, %2, %3, %4};"
               ::"l"(q), "r"(inc[0]), "r"(inc[1]), "r"(inc[2]), "r"(inc[3]) : "memory");
}

// Writes one updated W or H vector: an atomic add of its change (FP32 /
// FP64), an atomic add of the change of its stochastically rounded value
// (BF16), or a store (rounded stochastically for BF16).
template <typename T, bool ATOMIC>
__device__ __forceinline__ void write_vec(T* p, const uint4& old,
                                          const typename Elem<T>::C (&was)[Elem<T>::VW],
                                          const typename Elem<T>::C (&now)[Elem<T>::VW],
                                          const Philox4& base, uint32_t tag) {
  constexpr int VW = Elem<T>::VW;
  constexpr bool kSR = sizeof(T) == 2;
  if constexpr (ATOMIC && !kSR) {
    if constexpr (sizeof(T) == 4) {
      atomicAdd(reinterpret_cast<float4*>(p),
                make_float4(now[0] - was[0], now[1] - was[1], now[2] - was[2], now[3] - was[3]));
    } else {
#pragma unroll
      for (int e = 0; e < VW; ++e) atomicAdd(reinterpret_cast<double*>(p) + e, (double)(now[e] - was[e]));
    }
  } else {
    Philox4 rnd;
    if constexpr (kSR) rnd = sr_expand(base, tag);
    if constexpr (ATOMIC && kSR)
      red_bf16_increment(reinterpret_cast<__nv_bfloat16*>(p), old, now, rnd);
    else
      store_vec<T>(p, now, &rnd);
  }
}

// Records of a chunk in runs of one H row (the layout sorts each block by
// column): group g walks records g*LPN .. g*LPN + LPN - 1 in order, keeps the
// H row of the current run in registers -- the run's updates of it are
// sequential SGD -- and writes it back once when the run ends.  Every
// record's W row is read and written as in the shuffled path.  With the sides
// swapped by the host (runs of one W row) the same code caches the W row.
// 16-byte factor load; CG reads through L2 only (the persistent epoch, whose
// chunks of different sub-epochs share an SM's L1 within one launch)
template <bool CG>
__device__ __forceinline__ uint4 ld_vec(const void* p) {
  if constexpr (CG) return __ldcg(reinterpret_cast<const uint4*>(p));
  else return *reinterpret_cast<const uint4*>(p);
}

template <typename T, int LPN, int VPL, bool ATOMIC, bool CG = false>
__device__ __forceinline__ void run_chunk(const HogwildArgs& a, T* W, T* H, uint64_t rb,
                                          uint32_t nrec, uint32_t my_row, uint32_t my_col,
                                          typename Elem<T>::C my_x, typename Elem<T>::C my_a,
                                          typename Elem<T>::C my_b, typename Elem<T>::C eps,
                                          typename Elem<T>::C cwh, typename Elem<T>::C rw,
                                          typename Elem<T>::C rh, typename Elem<T>::C tmin,
                                          typename Elem<T>::C tmax, const Philox4& base,
                                          uint32_t grp, uint32_t gl) {
  using E = Elem<T>;
  using C = typename E::C;
  constexpr int VW = E::VW;
  constexpr uint32_t kNone = 0xffffffffu;
  constexpr int kRunCap = 2;
  uint32_t cur = kNone;  // H row of the open run
  uint4 hv0[VPL];        // ... as loaded
  C h0[VPL][VW];         // ... unpacked as loaded
  C hf[VPL][VW];         // ... as updated so far
  uint32_t last_t = 0;  // the run's last record in the group (its H write tag)
  constexpr int NG = 32 / LPN;
  // A full chunk of one column: a hot column's records fill whole chunks.
  // Then every group runs on the same H row and writes it back at the same
  // steps (every kRunCap records), and with atomic writes the groups add
  // their changes up with a butterfly and the first writes the sum: one
  // atomic per warp and write-back instead of one per group eases the queue
  // at that row's L2 slice.
  // BF16 sums too where a group spans at most 4 lanes (rank 32 and below):
  // there it measured slightly faster and kept a hot column's row stable at
  // large steps, where one rounded increment per group drifts; the wider BF16
  // mappings (ranks 64 and 128) measured slower with it.
  bool one_col = false;
  if constexpr (ATOMIC && NG > 1 && (sizeof(T) != 2 || LPN <= 4))
    one_col = nrec == (uint32_t)kChunk &&
              __all_sync(kFullMask, my_col == __shfl_sync(kFullMask, my_col, 0));
  // Writes back the open run of the groups with wb set; called by every lane.
  auto write_back = [&](bool wb) {
    if (one_col && __all_sync(kFullMask, wb)) {
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const uint32_t e0 = (uint32_t)(v * LPN + gl) * VW;
        C hb[VW];  // the run's base (BF16: unpacked again rather than kept live)
        if constexpr (sizeof(T) == 2) {
          E::unpack(hv0[v], hb);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e) hb[e] = h0[v][e];
        }
#pragma unroll
        for (int e = 0; e < VW; ++e) {
          C dsum = hf[v][e] - hb[e];
#pragma unroll
          for (int off = LPN; off < 32; off <<= 1) dsum += __shfl_xor_sync(kFullMask, dsum, off);
          hf[v][e] = hb[e] + dsum;  // the run's end state with every group's changes
        }
        if (grp == 0 && e0 < a.rp)
          write_vec<T, ATOMIC>(H + (size_t)cur * a.rp + e0, hv0[v], hb, hf[v], base,
                               2u * (last_t * VPL + v) + 1u);
      }
    } else if (wb) {
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const uint32_t e0 = (uint32_t)(v * LPN + gl) * VW;
        if (e0 < a.rp)
          write_vec<T, ATOMIC>(H + (size_t)cur * a.rp + e0, hv0[v], h0[v], hf[v], base,
                               2u * (last_t * VPL + v) + 1u);
      }
    }
    if (wb) cur = kNone;
  };
  // write tags: record t of the group, vector v: 2 (t VPL + v) for W, + 1 for H
#pragma unroll 1
  for (int t = 0; t < LPN; ++t) {
    const uint32_t ri = grp * LPN + t;
    const uint32_t row = __shfl_sync(kFullMask, my_row, ri);
    const uint32_t col = __shfl_sync(kFullMask, my_col, ri);
    const C x = __shfl_sync(kFullMask, my_x, ri);
    const C ca = __shfl_sync(kFullMask, my_a, ri);
    const C cb = __shfl_sync(kFullMask, my_b, ri);
    const bool valid = ri < nrec;
    // a run ends at a new column, or after kRunCap records: the row is then
    // written back and re-read, so other warps' updates of a hot row reach
    // this group at least every kRunCap records (longer runs measured less
    // stable: on the 100M-entry Zipf matrix, runs of 4 or 8 diverged within
    // 60 BoldDriver epochs where runs of 2 and the shuffled order did not)
    write_back(cur != kNone && (!valid || col != cur || (t % kRunCap) == 0));
    if (valid && cur == kNone) {  // a run starts: load its H row
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const uint32_t e0 = (uint32_t)(v * LPN + gl) * VW;
        hv0[v] = e0 < a.rp ? ld_vec<CG>(H + (size_t)col * a.rp + e0) : make_uint4(0, 0, 0, 0);
        E::unpack(hv0[v], h0[v]);
#pragma unroll
        for (int e = 0; e < VW; ++e) hf[v][e] = h0[v][e];
      }
      cur = col;
    }
    T* wp = W + (size_t)row * a.rp;
    uint4 wv[VPL];
    C wf[VPL][VW];
    C dot = 0;
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      const uint32_t e0 = (uint32_t)(v * LPN + gl) * VW;
      wv[v] = (valid && e0 < a.rp) ? ld_vec<CG>(wp + e0) : make_uint4(0, 0, 0, 0);
      E::unpack(wv[v], wf[v]);
      if (valid) {
#pragma unroll
        for (int e = 0; e < VW; ++e) dot += wf[v][e] * hf[v][e];
      }
    }
#pragma unroll
    for (int off = LPN / 2; off > 0; off >>= 1) dot += __shfl_xor_sync(kFullMask, dot, off);
    if (!valid) continue;
    const C f1 = (C)-2 * eps * (x - dot * cwh);
    const C fw = f1 * rw, fh = f1 * rh;
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      const uint32_t e0 = (uint32_t)(v * LPN + gl) * VW;
      if (e0 >= a.rp) continue;
      C nw[VW], nh[VW];
#pragma unroll
      for (int e = 0; e < VW; ++e) {
        nw[e] = wf[v][e] - (fw * hf[v][e] + ca * wf[v][e]);
        nh[e] = hf[v][e] - (fh * wf[v][e] + cb * hf[v][e]);
      }
      if (!ATOMIC && a.truncate) {
#pragma unroll
        for (int e = 0; e < VW; ++e)
          if (e0 + e < a.r) {
            nw[e] = clampw(nw[e], tmin, tmax, eps);
            nh[e] = clampw(nh[e], tmin, tmax, eps);
          }
      }
      write_vec<T, ATOMIC>(wp + e0, wv[v], wf[v], nw, base, 2u * ((uint32_t)t * VPL + v));
#pragma unroll
      for (int e = 0; e < VW; ++e) hf[v][e] = nh[e];
    }
    last_t = (uint32_t)t;
  }
  write_back(cur != kNone);
}

// Records of a chunk in the shuffled order: 32/LPN records at a time, one per
// group of LPN lanes, each W/H vector loaded right before it is used.
template <typename T, int LPN, int VPL, bool ATOMIC>
__device__ __forceinline__ void shuffled_chunk(const HogwildArgs& a, T* W, T* H, uint32_t nrec,
                                               uint32_t my_row, uint32_t my_col,
                                               typename Elem<T>::C my_x, typename Elem<T>::C my_a,
                                               typename Elem<T>::C my_b, typename Elem<T>::C eps,
                                               typename Elem<T>::C cwh, typename Elem<T>::C rw,
                                               typename Elem<T>::C rh, typename Elem<T>::C tmin,
                                               typename Elem<T>::C tmax, const Philox4& base,
                                               uint32_t grp, uint32_t gl) {
  using E = Elem<T>;
  using C = typename E::C;
  constexpr int VW = E::VW;
  constexpr int NG = 32 / LPN;
  for (uint32_t t0 = 0; t0 < nrec; t0 += NG) {
    const uint32_t ri = t0 + grp;
    const uint32_t row = __shfl_sync(kFullMask, my_row, ri);
    const uint32_t col = __shfl_sync(kFullMask, my_col, ri);
    const C x = __shfl_sync(kFullMask, my_x, ri);
    const C ca = __shfl_sync(kFullMask, my_a, ri);
    const C cb = __shfl_sync(kFullMask, my_b, ri);
    const bool valid = ri < nrec;
    T* wp = W + (size_t)row * a.rp;
    T* hp = H + (size_t)col * a.rp;
    uint4 wv[VPL], hv[VPL];
    bool live[VPL];
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      const uint32_t e0 = (uint32_t)(v * LPN + gl) * VW;
      live[v] = valid && e0 < a.rp;
      if (live[v]) {
        wv[v] = *reinterpret_cast<const uint4*>(wp + e0);
        hv[v] = *reinterpret_cast<const uint4*>(hp + e0);
      } else {
        wv[v] = make_uint4(0, 0, 0, 0);
        hv[v] = make_uint4(0, 0, 0, 0);
      }
    }
    C dot = 0;
    C wf[VPL][VW], hf[VPL][VW];
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      E::unpack(wv[v], wf[v]);
      E::unpack(hv[v], hf[v]);
#pragma unroll
      for (int e = 0; e < VW; ++e) dot += wf[v][e] * hf[v][e];
    }
#pragma unroll
    for (int off = LPN / 2; off > 0; off >>= 1) dot += __shfl_xor_sync(kFullMask, dot, off);
    const C f1 = (C)-2 * eps * (x - dot * cwh);
    const C fw = f1 * rw, fh = f1 * rh;
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      if (!live[v]) continue;
      C nw[VW], nh[VW];
#pragma unroll
      for (int e = 0; e < VW; ++e) {
        nw[e] = wf[v][e] - (fw * hf[v][e] + ca * wf[v][e]);
        nh[e] = hf[v][e] - (fh * wf[v][e] + cb * hf[v][e]);
      }
      const uint32_t e0 = (uint32_t)(v * LPN + gl) * VW;
      if (!ATOMIC && a.truncate) {
#pragma unroll
        for (int e = 0; e < VW; ++e)
          if (e0 + e < a.r) {
            nw[e] = clampw(nw[e], tmin, tmax, eps);
            nh[e] = clampw(nh[e], tmin, tmax, eps);
          }
      }
      // tags: iteration t0 / NG of this group, vector v, side
      const uint32_t tg = 2u * ((t0 / NG) * VPL + v);
      write_vec<T, ATOMIC>(wp + e0, wv[v], wf[v], nw, base, tg);
      write_vec<T, ATOMIC>(hp + e0, hv[v], hf[v], nh, base, tg + 1u);
    }
  }
}

// One launch = one work list of segments (a segment = one conflict-free block
// of a sub-epoch; several problems' segments in the batched form), cut into
// 32-entry chunks.  Warp w of the grid takes chunks w, w + (warps in the
// grid), ... of the list (in the epoch's chunk permutation), so no chunk
// counter is needed and the next chunk is known in advance: its entries (one
// per lane) are loaded while the current chunk is updated, and its inverse
// counts at the end, so a chunk costs about one memory round trip per record
// of a group.  32/LPN entries are updated at once, each W/H vector loaded
// right before it is used.  (Prefetching the next chunk's factor rows into
// registers or shared memory measured slower on B200: the registers or shared
// memory cost more resident warps than the prefetch gains; its entries take
// five registers.)
// Register bounds: see HogwildLaunch (FP32 one vector per lane at 48
// registers took the rank-128 FP32 epoch 23.4 -> 21.6 ms; two vectors per
// lane stay unconstrained: capping them measured slower).
// CTA size and register bound of an instance (hogwild_threads has the why):
// FP32 one vector per lane held to 48 registers (10 CTAs of 128), BF16 with
// up to 4 lanes to 73 (7 CTAs of 128), wider BF16 to 64 (4 CTAs of 256);
// two vectors per lane unconstrained.
template <typename T, int LPN, int VPL>
struct HogwildLaunch {
  static constexpr bool kBig = sizeof(T) == 2 && LPN > 4;
  static constexpr int threads = kBig ? 256 : 128;
  static constexpr int min_blocks = VPL != 1         ? (kBig ? 1 : 2)
                                    : sizeof(T) == 4 ? 10
                                    : sizeof(T) == 8 ? 2
                                    : kBig           ? 4
                                                     : 7;
};

template <typename T, int LPN, int VPL, bool ATOMIC, bool SMEM, bool RUNS>
__global__ void __launch_bounds__(HogwildLaunch<T, LPN, VPL>::threads,
                                  HogwildLaunch<T, LPN, VPL>::min_blocks)
    hogwild_subepoch_kernel(HogwildArgs a, uint32_t li) {
  using E = Elem<T>;
  using C = typename E::C;
  constexpr bool kSR = sizeof(T) == 2;

  // Launched after another sub-epoch of the same epoch (programmatic
  // dependent launch), this grid's CTAs take the SM slots the previous
  // grid's CTAs free as they finish, stage the segment table and their first
  // chunk's entries -- none of which that grid writes -- and wait for it to
  // complete (griddepcontrol.wait) before they touch a factor.  Otherwise the
  // wait returns at once.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const LaunchDesc ld = a.launches[li];
  const Segment* gseg = a.segs + ld.seg_begin;
  const uint32_t nseg = ld.nseg;
  // SMEM: the segment table is staged in shared memory; otherwise (large
  // batched tables) it is searched in global memory
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Segment* seg = gseg;
  if constexpr (SMEM) {
    Segment* ss = reinterpret_cast<Segment*>(smem_raw);
    for (uint32_t k = threadIdx.x; k <= nseg; k += blockDim.x) ss[k] = gseg[k];
    __syncthreads();
    seg = ss;
  }
  const uint32_t total = seg[nseg].chunk_begin;
  if (total == 0 || nseg == 0) return;
  const uint32_t warps = blockDim.x >> 5;
  const uint32_t stride = gridDim.x * warps;  // warps in the grid
  uint32_t lc = blockIdx.x * warps + (threadIdx.x >> 5);
  if (lc >= total) return;

  const EpochParams ep = *a.params;
  const C lambda2 = (C)(2.0 * a.lambda);
  const C tmin = (C)a.tmin, tmax = (C)a.tmax;
  const uint64_t h = mix64(((uint64_t)ep.key0 << 32 | ep.key1) ^ ((uint64_t)li << 17) ^ ep.epoch);
  uint64_t mulA = 1, addB = 0;
  if (a.sgd_order == 2) {  // WOR: affine permutation of the chunks
    mulA = kPrimes[h & 7u] % total;
    addB = (h >> 8) % total;
  }
  // position of chunk c of the list in the epoch's order: WR draws it, the
  // affine order (WOR; SEQ with A = 1, B = 0) steps from c to c + stride by
  // adding A * stride mod total, which saves a 64-bit remainder per chunk
  // (C2 BF16 epoch 5.50 -> 5.25 ms).  The wide BF16 mappings (CTAs of 256
  // threads at 64 registers) keep the remainder: their register allocation
  // with the step measured 12% slower at rank 64.
  const bool wr = a.sgd_order == 1 || HogwildLaunch<T, LPN, VPL>::kBig;
  auto position = [&](uint32_t c) -> uint32_t {
    return a.sgd_order == 1 ? (uint32_t)(mix64(h ^ ((uint64_t)c << 20)) % total)
                            : (uint32_t)((mulA * c + addB) % total);
  };
  const uint32_t step = (uint32_t)((mulA * stride) % total);
  const C* inv1 = reinterpret_cast<const C*>(a.inv1);
  const C* inv2 = reinterpret_cast<const C*>(a.inv2);
  const C* vals = reinterpret_cast<const C*>(a.val);
  T* W = reinterpret_cast<T*>(a.W);
  T* H = reinterpret_cast<T*>(a.H);
  const bool weighted = a.update == kUpdNzslL2;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t grp = lane / LPN, gl = lane % LPN;

  // chunk at position pc -> its segment, first record and record count
  auto locate = [&](uint32_t pc, uint32_t& lo, uint64_t& rb, uint32_t& nrec) {
    uint32_t l = 0, hi = nseg - 1;  // the last segment with chunk_begin <= pc
    while (l < hi) {
      const uint32_t mid = (l + hi + 1) >> 1;
      if (seg[mid].chunk_begin <= pc) l = mid; else hi = mid - 1;
    }
    lo = l;
    const uint32_t cin = pc - seg[l].chunk_begin;
    rb = seg[l].rec_begin + (uint64_t)cin * kChunk;
    nrec = min((uint32_t)kChunk, seg[l].count - cin * kChunk);
  };

  // the chunk in hand: its entries, one per lane, and their inverse counts
  uint32_t lo, nrec;
  uint64_t rb;
  uint32_t pc = position(lc);
  locate(pc, lo, rb, nrec);
  uint32_t my_row = 0, my_col = 0;
  C my_x = 0, my_ia = 0, my_ib = 0;
  if (lane < nrec) {
    my_row = a.row[rb + lane];
    my_col = a.col[rb + lane];
    my_x = vals[rb + lane];
    if (weighted) {
      my_ia = inv1[my_row];
      my_ib = inv2[my_col];
    }
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");  // the previous sub-epoch is complete
  for (;;) {
    // the next chunk's entries travel while this chunk is updated
    const uint32_t nlc = lc + stride;
    uint32_t nlo = 0, nnrec = 0, npc = 0;
    uint64_t nrb = 0;
    uint32_t n_row = 0, n_col = 0;
    C n_x = 0;
    if (nlc < total) {
      npc = wr ? position(nlc) : (pc + step >= total ? pc + step - total : pc + step);
      locate(npc, nlo, nrb, nnrec);
      if (lane < nnrec) {
        n_row = a.row[nrb + lane];
        n_col = a.col[nrb + lane];
        n_x = vals[nrb + lane];
      }
    }

    const C eps = (C)seg[lo].eps, f2 = eps * lambda2;
    const C cwh = (C)seg[lo].cwh;
    const C rw = (C)(a.swap_sides ? seg[lo].rho_h : seg[lo].rho_w);
    const C rh = (C)(a.swap_sides ? seg[lo].rho_w : seg[lo].rho_h);
    C my_a = 0, my_b = 0;
    if (weighted) {
      my_a = f2 * my_ia;
      my_b = f2 * my_ib;
    } else if (a.update == kUpdNzslNzl2) {
      my_a = f2;
      my_b = f2;
    }
    // stochastic rounding: one Philox block per chunk and lane (counter:
    // first record of the chunk, epoch, lane; key: the epoch's key)
    Philox4 base{};
    if constexpr (kSR)
      base = philox4x32_10((uint32_t)rb, (uint32_t)(rb >> 32), ep.epoch, lane, ep.key0, ep.key1);
    if constexpr (RUNS)
      run_chunk<T, LPN, VPL, ATOMIC>(a, W, H, rb, nrec, my_row, my_col, my_x, my_a, my_b, eps,
                                     cwh, rw, rh, tmin, tmax, base, grp, gl);
    else
      shuffled_chunk<T, LPN, VPL, ATOMIC>(a, W, H, nrec, my_row, my_col, my_x, my_a, my_b, eps,
                                          cwh, rw, rh, tmin, tmax, base, grp, gl);
    if (nlc >= total) break;
    // the next chunk's inverse counts: their round trip overlaps the first
    // factor loads of that chunk
    C n_ia = 0, n_ib = 0;
    if (weighted && lane < nnrec) {
      n_ia = inv1[n_row];
      n_ib = inv2[n_col];
    }
    lc = nlc;
    pc = npc;
    lo = nlo;
    rb = nrb;
    nrec = nnrec;
    my_row = n_row;
    my_col = n_col;
    my_x = n_x;
    my_ia = n_ia;
    my_ib = n_ib;
  }
}

__device__ __forceinline__ uint32_t load_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Polls until *done >= need; false if it gave up (or another warp did).  A
// wait gives up after limit_ns of the global timer (the epoch then reports an
// error instead of waiting for ever); a poll count of limit_ns / 16 + 1024 --
// more than the timer allows, since every poll is an L2 round trip plus a
// sleep -- bounds it should the timer not advance.
__device__ __forceinline__ bool wait_done(const uint32_t* done, uint32_t need, uint32_t* error,
                                          uint64_t limit_ns) {
  if (load_acquire(done) >= need) return true;
  const uint64_t t0 = global_ns(), max_polls = limit_ns / 16 + 1024;
  for (uint64_t it = 0; load_acquire(done) < need; ++it) {
    if (global_ns() - t0 > limit_ns || it >= max_polls ||
        *reinterpret_cast<volatile uint32_t*>(error)) {
      atomicExch(error, 1u);
      return false;
    }
    __nanosleep(1000);
  }
  return true;
}

// One launch per epoch.  Warps take chunk tickets in sub-epoch order (the
// chunks of sub-epoch s in the same order as the launch-per-sub-epoch form); a
// chunk of segment (s, i) first waits for segment (s-1, i) and for
// dep_col[s][i].  Every chunk waited for holds a smaller ticket, and tickets
// go to running warps only, so the waits end; each is bounded anyway (a wait
// that runs out sets the error flag, and every warp then stops taking
// tickets and returns).  A
// finished chunk publishes its writes (fence) before it counts itself done.
template <typename T, int LPN, int VPL>
__global__ void __launch_bounds__(256) hogwild_epoch_kernel(HogwildArgs a, EpochDeps dp) {
  using E = Elem<T>;
  using C = typename E::C;
  extern __shared__ __align__(16) uint32_t prefix[];  // [2d + 1] chunk offsets per sub-epoch
  const uint32_t d = dp.d, nsub = dp.nsub;
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t s = 0; s < nsub; ++s) {
      prefix[s] = acc;
      const LaunchDesc L = a.launches[s];
      acc += a.segs[L.seg_begin + L.nseg].chunk_begin;
    }
    prefix[nsub] = acc;
  }
  __syncthreads();
  const uint32_t total = prefix[nsub];
  const EpochParams ep = *a.params;
  const C lambda2 = (C)(2.0 * a.lambda);
  const C tmin = (C)a.tmin, tmax = (C)a.tmax;
  const C* inv1 = reinterpret_cast<const C*>(a.inv1);
  const C* inv2 = reinterpret_cast<const C*>(a.inv2);
  const C* vals = reinterpret_cast<const C*>(a.val);
  T* W = reinterpret_cast<T*>(a.W);
  T* H = reinterpret_cast<T*>(a.H);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t grp = lane / LPN, gl = lane % LPN;
  uint32_t ready_seg = 0xffffffffu;  // segment whose dependencies this warp saw met

  for (;;) {
    uint32_t tk = total;
    if (lane == 0 && !*reinterpret_cast<volatile uint32_t*>(dp.error)) tk = atomicAdd(dp.ticket, 1u);
    tk = __shfl_sync(kFullMask, tk, 0);
    if (tk >= total) break;
    uint32_t s = 0, hs = nsub - 1;  // the sub-epoch: the last s with prefix[s] <= tk
    while (s < hs) {
      const uint32_t mid = (s + hs + 1) >> 1;
      if (prefix[mid] <= tk) s = mid; else hs = mid - 1;
    }
    const uint32_t cnt_s = prefix[s + 1] - prefix[s], lc = tk - prefix[s];
    const LaunchDesc L = a.launches[s];
    const Segment* seg = a.segs + L.seg_begin;
    uint32_t pc = lc;
    if (a.sgd_order == 2) {  // WOR: the affine chunk permutation of sub-epoch s
      const uint64_t h =
          mix64(((uint64_t)ep.key0 << 32 | ep.key1) ^ ((uint64_t)s << 17) ^ ep.epoch);
      const uint64_t mulA = kPrimes[h & 7u] % cnt_s, addB = (h >> 8) % cnt_s;
      pc = (uint32_t)((mulA * lc + addB) % cnt_s);
    }
    uint32_t lo = 0, hi = L.nseg - 1;  // the last segment with chunk_begin <= pc
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (__ldg(&seg[mid].chunk_begin) <= pc) lo = mid; else hi = mid - 1;
    }
    const uint32_t me = s * d + lo;
    if (me != ready_seg) {
      uint32_t ok = 1;
      if (lane == 0 && s > 0) {
        const Segment* ps = a.segs + a.launches[s - 1].seg_begin;
        ok = wait_done(dp.done + (me - d), ps[lo + 1].chunk_begin - ps[lo].chunk_begin, dp.error,
                       dp.wait_ns);
        const int32_t dc = dp.dep_col[me];
        if (ok && dc >= 0) {
          const uint32_t ds = (uint32_t)dc / d, dj = (uint32_t)dc % d;
          const Segment* qs = a.segs + a.launches[ds].seg_begin;
          ok = wait_done(dp.done + dc, qs[dj + 1].chunk_begin - qs[dj].chunk_begin, dp.error,
                         dp.wait_ns);
        }
      }
      if (!__shfl_sync(kFullMask, ok, 0)) break;
      __threadfence();
      ready_seg = me;
    }
    const Segment sg = seg[lo];
    const uint32_t cin = pc - sg.chunk_begin;
    const uint64_t rb = sg.rec_begin + (uint64_t)cin * kChunk;
    const uint32_t nrec = min((uint32_t)kChunk, sg.count - cin * kChunk);
    const C eps = (C)sg.eps, f2 = eps * lambda2;
    const C cwh = (C)sg.cwh;
    const C rw = (C)(a.swap_sides ? sg.rho_h : sg.rho_w);
    const C rh = (C)(a.swap_sides ? sg.rho_w : sg.rho_h);
    uint32_t my_row = 0, my_col = 0;
    C my_x = 0, my_a = 0, my_b = 0;
    if (lane < nrec) {
      my_row = a.row[rb + lane];
      my_col = a.col[rb + lane];
      my_x = vals[rb + lane];
      if (a.update == kUpdNzslL2) {
        my_a = f2 * inv1[my_row];
        my_b = f2 * inv2[my_col];
      } else if (a.update == kUpdNzslNzl2) {
        my_a = f2;
        my_b = f2;
      }
    }
    Philox4 base{};
    if constexpr (sizeof(T) == 2)
      base = philox4x32_10((uint32_t)rb, (uint32_t)(rb >> 32), ep.epoch, lane, ep.key0, ep.key1);
    run_chunk<T, LPN, VPL, true, true>(a, W, H, rb, nrec, my_row, my_col, my_x, my_a, my_b, eps,
                                       cwh, rw, rh, tmin, tmax, base, grp, gl);
    __threadfence();  // this lane's writes, before the chunk counts as done
    __syncwarp();
    if (lane == 0) atomicAdd(dp.done + me, 1u);
  }
}

__global__ void build_segments_kernel(SegBuildArgs a) {
  // one CTA per sub-epoch; thread id = task id (d <= 1024)
  __shared__ uint32_t scan[1024];
  const uint32_t s = blockIdx.x, d = a.d, id = threadIdx.x;
  uint32_t chunks = 0;
  uint64_t rb = 0;
  uint32_t cnt = 0, b2 = 0;
  if (id < d) {
    b2 = a.schedule[(size_t)s * d + id];
    const uint64_t blk = (uint64_t)id * a.nb2 + b2;
    rb = a.block_ptr[blk];
    cnt = (uint32_t)(a.block_ptr[blk + 1] - rb);
    chunks = (cnt + kChunk - 1) / kChunk;
  }
  scan[id] = chunks;
  __syncthreads();
  // Hillis-Steele inclusive scan over blockDim.x entries
  for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
    uint32_t v = id >= off ? scan[id - off] : 0;
    __syncthreads();
    scan[id] += v;
    __syncthreads();
  }
  Segment* out = a.segs + (size_t)s * (d + 1);
  if (id < d) {
    Segment g;
    g.rec_begin = rb;
    g.count = cnt;
    g.chunk_begin = scan[id] - chunks;
    if (a.sigma) {
      const float* sg = a.sigma + ((size_t)s * d + id) * 3;
      g.cwh = sg[0]; g.rho_w = sg[1]; g.rho_h = sg[2];
    } else {
      g.cwh = 1.f; g.rho_w = 1.f; g.rho_h = 1.f;
    }
    g.col_block = b2;
    g.eps = a.params->eps;
    out[id] = g;
  }
  if (id == 0) {
    Segment e;
    e.rec_begin = 0; e.count = 0; e.chunk_begin = scan[d - 1];
    e.cwh = e.rho_w = e.rho_h = 1.f; e.col_block = 0xffffffffu;
    e.eps = 0;
    out[d] = e;
    a.counters[s] = 0;
  }
}

// ---- deterministic FP64 replay ---------------------------------------------
constexpr int kReplayMaxK = 8;  // r <= 256

__global__ void __launch_bounds__(128) replay_subepoch_kernel(ReplayArgs a, uint32_t s) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t id = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (id >= a.d) return;
  const uint32_t d = a.d, r = a.r;
  const uint32_t b2 = a.schedule[(size_t)s * d + id];
  const uint64_t blk = (uint64_t)id * a.nb2 + b2;
  const uint64_t rb = a.block_ptr[blk];
  const uint64_t n = a.block_ptr[blk + 1] - rb;
  const uint32_t* pos = a.positions + a.pos_offset[(size_t)s * d + id];
  const double eps = a.params->eps;
  const int kmax = (int)((r + 31) / 32);
  // f1 = eps * -2. * (x - wh); f2 = eps * 2. * lambda
  const double em2 = __dmul_rn(eps, -2.0);
  const double f2 = __dmul_rn(__dmul_rn(eps, 2.0), a.lambda);

  if (n == 0) return;
  // The reads run ahead of the updates: the coordinates, value and counts of
  // record q + 2 and the factor rows of record q + 1 are loaded while record q
  // is updated.  Record q + 1 takes a row or column that record q writes from
  // q's new values in registers (each lane reads back only the elements it
  // writes itself, so rows written earlier are seen in program order); every
  // update therefore reads the values the sequential order gives it, and the
  // arithmetic below is the reference's, operation for operation.
  struct Coord {
    uint32_t i, j, c1, c2;
    double x;
  };
  const bool counts = a.update == kUpdNzslL2;
  auto load_coord = [&](uint64_t q) {
    Coord e;
    const uint64_t rec = rb + pos[q];
    e.i = a.row[rec];
    e.j = a.col[rec];
    e.x = a.val[rec];
    e.c1 = counts ? a.cnt1[e.i] : 1u;
    e.c2 = counts ? a.cnt2[e.j] : 1u;
    return e;
  };
  auto load_rows = [&](const Coord& e, double (&wz)[kReplayMaxK], double (&hz)[kReplayMaxK]) {
    const double* w = a.W + (size_t)e.i * a.rp;
    const double* h = a.H + (size_t)e.j * a.rp;
#pragma unroll
    for (int k = 0; k < kReplayMaxK; ++k) {
      const uint32_t z = (uint32_t)k * 32 + lane;
      wz[k] = 0;
      hz[k] = 0;
      if (k < kmax && z < r) {
        wz[k] = w[z];
        hz[k] = h[z];
      }
    }
  };
  Coord cur = load_coord(0);
  Coord nxt = n > 1 ? load_coord(1) : cur;
  double wz[kReplayMaxK], hz[kReplayMaxK];
  load_rows(cur, wz, hz);

#pragma unroll 1
  for (uint64_t q = 0; q < n; ++q) {
    const Coord after = q + 2 < n ? load_coord(q + 2) : nxt;
    double nwz[kReplayMaxK], nhz[kReplayMaxK];
    if (q + 1 < n) load_rows(nxt, nwz, nhz);
    double pz[kReplayMaxK];
#pragma unroll
    for (int k = 0; k < kReplayMaxK; ++k) {
      const uint32_t z = (uint32_t)k * 32 + lane;
      pz[k] = (k < kmax && z < r) ? __dmul_rn(wz[k], hz[k]) : 0.0;
    }
    // wh = sum_z w[z] h[z] in z order (every lane computes the same sum)
    double wh = 0;
#pragma unroll
    for (int k = 0; k < kReplayMaxK; ++k) {
      if (k >= kmax) break;
      for (uint32_t l = 0; l < 32; ++l) {
        if ((uint32_t)k * 32 + l >= r) break;
        wh = __dadd_rn(wh, __shfl_sync(kFullMask, pz[k], l));
      }
    }
    const double f1 = __dmul_rn(em2, __dsub_rn(cur.x, wh));
    double f3 = 0, f4 = 0;
    if (counts) {
      f3 = __ddiv_rn(1.0, (double)cur.c1);
      f4 = __ddiv_rn(1.0, (double)cur.c2);
    }
    double* w = a.W + (size_t)cur.i * a.rp;
    double* h = a.H + (size_t)cur.j * a.rp;
#pragma unroll
    for (int k = 0; k < kReplayMaxK; ++k) {
      const uint32_t z = (uint32_t)k * 32 + lane;
      if (k >= kmax || z >= r) continue;
      const double t = wz[k];
      double nw, nh;
      if (a.update == kUpdNzsl) {
        nw = __dsub_rn(wz[k], __dmul_rn(f1, hz[k]));
        nh = __dsub_rn(hz[k], __dmul_rn(f1, t));
      } else if (a.update == kUpdNzslL2) {
        nw = __dsub_rn(wz[k], __dadd_rn(__dmul_rn(f1, hz[k]), __dmul_rn(__dmul_rn(f2, wz[k]), f3)));
        nh = __dsub_rn(hz[k], __dadd_rn(__dmul_rn(f1, t), __dmul_rn(__dmul_rn(f2, hz[k]), f4)));
      } else {
        nw = __dsub_rn(wz[k], __dadd_rn(__dmul_rn(f1, hz[k]), __dmul_rn(f2, wz[k])));
        nh = __dsub_rn(hz[k], __dadd_rn(__dmul_rn(f1, t), __dmul_rn(f2, hz[k])));
      }
      if (a.truncate) {
        if (nw <= a.tmin) nw = __dadd_rn(a.tmin, eps);
        else if (nw >= a.tmax) nw = __dsub_rn(a.tmax, eps);
        if (nh <= a.tmin) nh = __dadd_rn(a.tmin, eps);
        else if (nh >= a.tmax) nh = __dsub_rn(a.tmax, eps);
      }
      w[z] = nw;
      h[z] = nh;
      // record q + 1 on the same row or column reads these values
      if (nxt.i == cur.i) nwz[k] = nw;
      if (nxt.j == cur.j) nhz[k] = nh;
    }
    __syncwarp();
    if (q + 1 == n) break;
    cur = nxt;
    nxt = after;
#pragma unroll
    for (int k = 0; k < kReplayMaxK; ++k) {
      wz[k] = nwz[k];
      hz[k] = nhz[k];
    }
  }
}

// RegularizeL2 (mf/sgd/functions/regularize-l2.h:26-45) applied by every task
// after sub-epoch s: each W block and the sub-epoch's H blocks are scaled.
__global__ void regularize_exact_kernel(double* W, double* H, uint64_t m, uint64_t n,
                                        uint32_t rp, uint32_t r, const uint64_t* off2,
                                        const uint8_t* mask, uint32_t d, uint32_t nb2,
                                        const EpochParams* params, double lambda, int truncate,
                                        double tmin, double tmax) {
  const double eps = __ddiv_rn(params->eps, (double)d);  // eps/d: rescaleStratumStepsize()
  double factor = __dsub_rn(1.0, __dmul_rn(__dmul_rn(eps, 2.0), lambda));
  if (factor < 0.5) factor = __ddiv_rn(0.25, __dsub_rn(1.0, factor));
  const uint64_t wtot = m * rp, htot = n * rp;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < wtot + htot; q += stride) {
    double* p;
    uint64_t z;
    if (q < wtot) {
      p = W + q;
      z = q % rp;
    } else {
      const uint64_t hq = q - wtot, j = hq / rp;
      // column block of j
      uint32_t lo = 0, hi = nb2 - 1;
      while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (off2[mid] <= j) lo = mid; else hi = mid - 1;
      }
      if (!mask[lo]) continue;
      p = H + hq;
      z = hq % rp;
    }
    if (z >= r) continue;
    double v = __dmul_rn(*p, factor);
    if (truncate) {
      if (v <= tmin) v = __dadd_rn(tmin, eps);
      else if (v >= tmax) v = __dsub_rn(tmax, eps);
    }
    *p = v;
  }
}

// One 16-byte vector of factor values times s, rounded back to the storage
// type as a store of the scaled value would be (BF16: to nearest).
template <typename T>
__device__ __forceinline__ uint4 scale_vec(const uint4& v, float s) {
  float f[4];
  Elem<float>::unpack(v, f);
#pragma unroll
  for (int e = 0; e < 4; ++e) f[e] *= s;
  return Elem<float>::pack(f);
}
template <>
__device__ __forceinline__ uint4 scale_vec<double>(const uint4& v, float s) {
  double f[2];
  Elem<double>::unpack(v, f);
  f[0] *= (double)s;
  f[1] *= (double)s;
  return Elem<double>::pack(f);
}
template <>
__device__ __forceinline__ uint4 scale_vec<__nv_bfloat16>(const uint4& v, float s) {
  float f[8];
  Elem<__nv_bfloat16>::unpack(v, f);
  uint32_t w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const __nv_bfloat162 b = __floats2bfloat162_rn(f[2 * k] * s, f[2 * k + 1] * s);
    w[k] = *reinterpret_cast<const uint32_t*>(&b);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// The epoch's lazy L2 scales, applied once: scales[b2] to H column block b2,
// scales[nb2] to all of W.  16-byte vectors (rows are padded to whole
// vectors), the column-block offsets staged in shared memory for the block
// search of each H row.
template <typename T>
__global__ void __launch_bounds__(256) normalize_kernel(T* W, T* H, uint64_t m, uint64_t n,
                                                        uint32_t rp, const float* scales,
                                                        const uint64_t* off2, uint32_t nb2) {
  extern __shared__ __align__(16) uint64_t s_off[];  // nb2 + 1 offsets
  for (uint32_t k = threadIdx.x; k <= nb2; k += blockDim.x) s_off[k] = off2[k];
  __syncthreads();
  const float sw = scales[nb2];
  const uint32_t vpr = rp / (16 / sizeof(T));  // vectors per row
  const uint64_t wv = m * vpr, tot = wv + n * vpr;
  uint4* Wv = reinterpret_cast<uint4*>(W);
  uint4* Hv = reinterpret_cast<uint4*>(H);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < tot; q += stride) {
    if (q < wv) {
      Wv[q] = scale_vec<T>(Wv[q], sw);
    } else {
      const uint64_t hq = q - wv, j = hq / vpr;
      uint32_t lo = 0, hi = nb2 - 1;  // the last block with off2[b] <= j
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (s_off[mid] <= j) lo = mid; else hi = mid - 1;
      }
      Hv[hq] = scale_vec<T>(Hv[hq], scales[lo]);
    }
  }
}

template <typename T>
__global__ void scale_rows_kernel(T* W, uint64_t wrows, T* H, uint64_t hrows, uint32_t rp,
                                  const uint32_t* w_slot, const uint32_t* h_slot,
                                  const float* scales) {
  const uint64_t wtot = wrows * rp, tot = wtot + hrows * rp;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < tot; q += stride) {
    if (q < wtot) {
      const float s = scales[w_slot[q / rp]];
      if constexpr (sizeof(T) == 8) W[q] *= (double)s;
      else W[q] = (T)((float)W[q] * s);
    } else {
      const uint64_t hq = q - wtot;
      const float s = scales[h_slot[hq / rp]];
      if constexpr (sizeof(T) == 8) H[hq] *= (double)s;
      else H[hq] = (T)((float)H[hq] * s);
    }
  }
}

template <typename T, int LPN, int VPL, bool RUNS>
void* hogwild_fn3(bool atomic, bool smem) {
  if (smem)
    return atomic
               ? reinterpret_cast<void*>(&hogwild_subepoch_kernel<T, LPN, VPL, true, true, RUNS>)
               : reinterpret_cast<void*>(&hogwild_subepoch_kernel<T, LPN, VPL, false, true, RUNS>);
  return atomic
             ? reinterpret_cast<void*>(&hogwild_subepoch_kernel<T, LPN, VPL, true, false, RUNS>)
             : reinterpret_cast<void*>(&hogwild_subepoch_kernel<T, LPN, VPL, false, false, RUNS>);
}

template <typename T, int LPN, int VPL>
void* hogwild_fn(bool atomic, bool smem, bool runs) {
  return runs ? hogwild_fn3<T, LPN, VPL, true>(atomic, smem)
              : hogwild_fn3<T, LPN, VPL, false>(atomic, smem);
}

template <typename T>
void* pick_hogwild(uint32_t lanes, uint32_t vecs, bool atomic, bool smem, bool runs) {
#define DSGDPP_CASE(L, V) \
  if (lanes == L && vecs == V) return hogwild_fn<T, L, V>(atomic, smem, runs);
  DSGDPP_CASE(2, 1) DSGDPP_CASE(4, 1) DSGDPP_CASE(8, 1) DSGDPP_CASE(16, 1) DSGDPP_CASE(32, 1)
  DSGDPP_CASE(2, 2) DSGDPP_CASE(4, 2) DSGDPP_CASE(8, 2) DSGDPP_CASE(16, 2) DSGDPP_CASE(32, 2)
  DSGDPP_CASE(32, 4)
#undef DSGDPP_CASE
  return nullptr;
}

void* hogwild_kernel_ptr(int precision, uint32_t lanes, uint32_t vecs, bool atomic, bool smem,
                         bool runs) {
  if (precision == kFp64) return pick_hogwild<double>(lanes, vecs, atomic, smem, runs);
  if (precision == kFp32) return pick_hogwild<float>(lanes, vecs, atomic, smem, runs);
  return pick_hogwild<__nv_bfloat16>(lanes, vecs, atomic, smem, runs);
}

}  // namespace

cudaError_t launch_build_segments(const SegBuildArgs& a, cudaStream_t st) {
  uint32_t threads = 32;
  while (threads < a.d) threads <<= 1;
  if (threads > 1024) return cudaErrorInvalidValue;
  build_segments_kernel<<<a.nb2, threads, 0, st>>>(a);
  return cudaGetLastError();
}

int hogwild_ctas_per_sm(int precision, uint32_t lanes, uint32_t vecs, bool atomic,
                        uint32_t smem_segs, bool runs) {
  void* fn = hogwild_kernel_ptr(precision, lanes, vecs, atomic, smem_segs > 0, runs);
  if (!fn) return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, hogwild_threads(precision, lanes),
                                                    sizeof(Segment) * smem_segs) !=
      cudaSuccess)
    return 0;
  return n;
}

cudaError_t launch_hogwild(int precision, uint32_t lanes, uint32_t vecs, const HogwildArgs& a,
                           uint32_t launch_index, uint32_t grid, cudaStream_t st,
                           bool after_subepoch) {
  void* fn = hogwild_kernel_ptr(precision, lanes, vecs, a.atomic != 0, a.smem_segs > 0,
                                a.runs != 0);
  if (!fn) return cudaErrorInvalidValue;
  HogwildArgs args = a;
  uint32_t li = launch_index;
  void* params[] = {&args, &li};
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(hogwild_threads(precision, lanes));
  cfg.dynamicSmemBytes = sizeof(Segment) * a.smem_segs;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  if (after_subepoch) {  // overlap this launch's start with the previous one's end
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelExC(&cfg, fn, params);
}

cudaError_t launch_replay_subepoch(const ReplayArgs& a, uint32_t s, cudaStream_t st) {
  if (a.r > 32u * kReplayMaxK) return cudaErrorInvalidValue;
  const uint32_t warps_per_cta = 4;
  replay_subepoch_kernel<<<(a.d + warps_per_cta - 1) / warps_per_cta, 32 * warps_per_cta, 0, st>>>(
      a, s);
  return cudaGetLastError();
}

cudaError_t launch_regularize_exact(double* W, double* H, uint64_t m, uint64_t n, uint32_t rp,
                                    uint32_t r, const uint64_t* off2, const uint8_t* mask,
                                    uint32_t d, uint32_t nb2, const EpochParams* params,
                                    double lambda, int truncate, double tmin, double tmax,
                                    cudaStream_t st) {
  regularize_exact_kernel<<<1184, 256, 0, st>>>(W, H, m, n, rp, r, off2, mask, d, nb2, params,
                                                lambda, truncate, tmin, tmax);
  return cudaGetLastError();
}

cudaError_t launch_normalize(int precision, void* W, void* H, uint64_t m, uint64_t n,
                             uint32_t rp, const float* scales, const uint64_t* off2,
                             uint32_t nb2, cudaStream_t st) {
  const size_t smem = sizeof(uint64_t) * (nb2 + 1);
  if (precision == kFp64)
    normalize_kernel<double><<<1184, 256, smem, st>>>((double*)W, (double*)H, m, n, rp, scales,
                                                       off2, nb2);
  else if (precision == kFp32)
    normalize_kernel<float><<<1184, 256, smem, st>>>((float*)W, (float*)H, m, n, rp, scales, off2,
                                                      nb2);
  else
    normalize_kernel<__nv_bfloat16><<<1184, 256, smem, st>>>(
        (__nv_bfloat16*)W, (__nv_bfloat16*)H, m, n, rp, scales, off2, nb2);
  return cudaGetLastError();
}

cudaError_t launch_scale_rows(int precision, void* W, uint64_t wrows, void* H, uint64_t hrows,
                              uint32_t rp, const uint32_t* w_slot, const uint32_t* h_slot,
                              const float* scales, cudaStream_t st) {
  if (precision == kFp64)
    scale_rows_kernel<double><<<1184, 256, 0, st>>>((double*)W, wrows, (double*)H, hrows, rp,
                                                    w_slot, h_slot, scales);
  else if (precision == kFp32)
    scale_rows_kernel<float><<<1184, 256, 0, st>>>((float*)W, wrows, (float*)H, hrows, rp,
                                                   w_slot, h_slot, scales);
  else
    scale_rows_kernel<__nv_bfloat16><<<1184, 256, 0, st>>>(
        (__nv_bfloat16*)W, wrows, (__nv_bfloat16*)H, hrows, rp, w_slot, h_slot, scales);
  return cudaGetLastError();
}

}  // namespace dsgdpp

namespace dsgdpp {
namespace {

template <typename T>
void* pick_epoch(uint32_t lanes, uint32_t vecs) {
#define DSGDPP_CASE(L, V) \
  if (lanes == L && vecs == V) return reinterpret_cast<void*>(&hogwild_epoch_kernel<T, L, V>);
  DSGDPP_CASE(2, 1) DSGDPP_CASE(4, 1) DSGDPP_CASE(8, 1) DSGDPP_CASE(16, 1) DSGDPP_CASE(32, 1)
  DSGDPP_CASE(2, 2) DSGDPP_CASE(4, 2) DSGDPP_CASE(8, 2) DSGDPP_CASE(16, 2) DSGDPP_CASE(32, 2)
  DSGDPP_CASE(32, 4)
#undef DSGDPP_CASE
  return nullptr;
}

void* epoch_kernel_ptr(int precision, uint32_t lanes, uint32_t vecs) {
  if (precision == kFp64) return pick_epoch<double>(lanes, vecs);
  if (precision == kFp32) return pick_epoch<float>(lanes, vecs);
  return pick_epoch<__nv_bfloat16>(lanes, vecs);
}

}  // namespace

int hogwild_epoch_ctas_per_sm(int precision, uint32_t lanes, uint32_t vecs, uint32_t nsub) {
  void* fn = epoch_kernel_ptr(precision, lanes, vecs);
  if (!fn) return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 256, sizeof(uint32_t) * (nsub + 1)) !=
      cudaSuccess)
    return 0;
  return n;
}

cudaError_t launch_hogwild_epoch(int precision, uint32_t lanes, uint32_t vecs, const HogwildArgs& a,
                                 const EpochDeps& dp, uint32_t grid, cudaStream_t st) {
  void* fn = epoch_kernel_ptr(precision, lanes, vecs);
  if (!fn || a.atomic == 0 || a.runs == 0) return cudaErrorInvalidValue;
  HogwildArgs args = a;
  EpochDeps deps = dp;
  void* params[] = {&args, &deps};
  return cudaLaunchKernel(fn, dim3(grid), dim3(256), params, sizeof(uint32_t) * (dp.nsub + 1), st);
}

}  // namespace dsgdpp
