// shard.cu -- one DSGD++ job over several ranks: H column blocks handed from
// rank to rank between sub-epochs, each transfer overlapped with the
// sub-epoch that runs while it travels.
//
// Reference: DsgdPpTask::run (mf/sgd/dsgdpp_impl.h:141-263).  A task owns one
// row block of V and W for the whole run; an H column block goes to the task
// that needs it next.  Every epoch splits the 2d column blocks into a red and
// a blue half (dsgdpp_impl.h:289-336) and sub-epochs alternate colours, so a
// block used at sub-epoch s is needed again at s + 2 at the earliest, and its
// transfer (igetCopy / irecv / isend, dsgdpp_impl.h:153-234) runs while
// sub-epoch s + 1 computes.
//
// Here rank r drives one context holding the entries of its tasks' row blocks
// (tasks r d/G .. (r+1) d/G - 1, set with dsgdpp_set_tasks).  Every rank
// derives the same plan from the epoch's schedule: each use of a block on
// another rank than its previous use is a move, posted right after that
// previous use and waited for right before the new use.  The moves posted
// after sub-epoch s form one group on the rank's transfer stream, which starts
// once the rank's sub-epoch s is done; the compute stream goes on with s + 1
// and only the sub-epoch that uses an arriving block waits for its group (a
// stream wait on the group's event).  Blocks move in place, from the sender's
// H to the receiver's H: no staging buffer, no host synchronisation inside an
// epoch.  Before the last sub-epoch (which applies the epoch's lazy L2 scales
// to all of H) every rank waits for its transfers, so no block is scaled
// while it travels.
//
// After an epoch dsgdpp_shard_share gives every rank every block's latest
// version (a broadcast from its holder), which the losses need: a rank's
// entries touch every column block.  The job's training loss is the sum of
// the ranks' losses over their own entries and W rows, plus the H term once.
//
// Transports: NCCL point-to-point and broadcasts (one rank per GPU and
// process; NCCL is loaded at run time, so the library loads without it), or
// device copies between contexts of one process (several emulated ranks on
// one GPU: their streams wait only on events, no kernel waits for another).
// Waits for NCCL work are bounded on the host: a transfer that does not finish
// within the limit (a rank that left, a dead link) aborts the communicator and
// the call returns DSGDPP_E_CUDA.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dsgdpp.h"
#include "context.h"
#include "trace_ranges.h"

using namespace dsgdpp;

namespace {

// ---- NCCL, resolved at run time ----------------------------------------------------
struct NcclApi {
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*CommAbort)(ncclComm_t) = nullptr;
  ncclResult_t (*CommGetAsyncError)(ncclComm_t, ncclResult_t*) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Broadcast)(const void*, void*, size_t, ncclDataType_t, int, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  const char* (*GetErrorString)(ncclResult_t) = nullptr;
  std::string error;  // why loading failed
};

const NcclApi& nccl_api() {
  static NcclApi api = []() {
    NcclApi a;
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      a.error = std::string("NCCL is not available: ") + dlerror();
      return a;
    }
    auto sym = [&](const char* name) {
      void* p = dlsym(h, name);
      if (!p && a.error.empty()) a.error = std::string("NCCL lacks ") + name;
      return p;
    };
    a.GetUniqueId = reinterpret_cast<decltype(a.GetUniqueId)>(sym("ncclGetUniqueId"));
    a.CommInitRank = reinterpret_cast<decltype(a.CommInitRank)>(sym("ncclCommInitRank"));
    a.CommDestroy = reinterpret_cast<decltype(a.CommDestroy)>(sym("ncclCommDestroy"));
    a.CommAbort = reinterpret_cast<decltype(a.CommAbort)>(sym("ncclCommAbort"));
    a.CommGetAsyncError =
        reinterpret_cast<decltype(a.CommGetAsyncError)>(sym("ncclCommGetAsyncError"));
    a.GroupStart = reinterpret_cast<decltype(a.GroupStart)>(sym("ncclGroupStart"));
    a.GroupEnd = reinterpret_cast<decltype(a.GroupEnd)>(sym("ncclGroupEnd"));
    a.Send = reinterpret_cast<decltype(a.Send)>(sym("ncclSend"));
    a.Recv = reinterpret_cast<decltype(a.Recv)>(sym("ncclRecv"));
    a.Broadcast = reinterpret_cast<decltype(a.Broadcast)>(sym("ncclBroadcast"));
    a.AllReduce = reinterpret_cast<decltype(a.AllReduce)>(sym("ncclAllReduce"));
    a.GetErrorString = reinterpret_cast<decltype(a.GetErrorString)>(sym("ncclGetErrorString"));
    return a;
  }();
  if (!api.error.empty()) throw Error(DSGDPP_E_UNSUPPORTED, api.error);
  return api;
}

void check_nccl(ncclResult_t r, const char* what) {
  if (r != ncclSuccess)
    throw Error(DSGDPP_E_CUDA, std::string(what) + ": " + nccl_api().GetErrorString(r));
}

// ---- the plan ------------------------------------------------------------------------
struct Move {
  uint32_t b2;
  int src, dst;
};
constexpr int kEveryone = -1;  // every rank holds the block's latest version

// Group g holds the moves posted before the epoch (g = 0) or after sub-epoch
// s (g = s + 1); waits[s * world + r] lists the groups that bring rank r a
// block it uses at sub-epoch s.
struct Plan {
  std::vector<std::vector<Move>> groups;
  std::vector<std::vector<uint32_t>> waits;
};

Plan make_plan(const uint32_t* sched, uint32_t d, uint32_t nb2, int world,
               std::vector<int>& holder) {
  Plan p;
  p.groups.resize(nb2 + 1);
  p.waits.resize((size_t)nb2 * world);
  const uint32_t per = d / world;
  std::vector<int64_t> last(nb2, -1);  // last use in this epoch (-1: none yet)
  for (uint32_t s = 0; s < nb2; ++s) {
    for (uint32_t t = 0; t < d; ++t) {
      const uint32_t b = sched[(size_t)s * d + t];
      const int r = (int)(t / per);
      if (holder[b] != kEveryone && holder[b] != r) {
        const uint32_t g = (uint32_t)(last[b] + 1);
        p.groups[g].push_back(Move{b, holder[b], r});
        auto& w = p.waits[(size_t)s * world + r];
        if (std::find(w.begin(), w.end(), g) == w.end()) w.push_back(g);
      }
      holder[b] = r;
      last[b] = s;
    }
  }
  return p;
}

}  // namespace

// ---- the shard ---------------------------------------------------------------------
struct ShardRank {
  dsgdpp_ctx* ctx = nullptr;
  int rank = 0;
  cudaStream_t xfer = nullptr;
  cudaEvent_t start = nullptr;           // the epoch's start on the compute stream
  std::vector<cudaEvent_t> sub_end;      // [nb2] sub-epoch s done on the compute stream
  std::vector<cudaEvent_t> group_done;   // [nb2 + 1] group g done on the transfer stream
  // timeline (timed events): [nb2] compute, [nb2 + 1] transfer groups
  std::vector<cudaEvent_t> tc0, tc1, tx0, tx1;
  cudaEvent_t t_origin = nullptr;
  std::vector<uint8_t> group_used;       // this rank's transfer stream carries group g
};

struct dsgdpp_shard {
  bool use_nccl = false;
  int world = 1;
  uint32_t d = 0, nb2 = 0;
  int device = 0;
  std::vector<ShardRank> ranks;  // the ranks this object drives (one with NCCL)
  std::vector<int> holder;
  ncclComm_t comm = nullptr;
  double wait_s = 300.0;
  bool timeline = false, timeline_valid = false;
  uint64_t moved_bytes = 0, moves = 0;  // this object's ranks' received bytes, last epoch
  double* d_sum = nullptr;              // NCCL sums of the losses
  double* h_sum = nullptr;
  std::string err;
};

namespace {

template <typename F>
int shard_guarded(dsgdpp_shard* sh, F&& f) {
  if (!sh) return DSGDPP_E_INVALID;
  try {
    return f();
  } catch (const Error& e) {
    sh->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    sh->err = "host allocation failed";
    return DSGDPP_E_NOMEM;
  }
}

void check_ctx(dsgdpp_ctx* c, int rc, const char* what) {
  if (rc != DSGDPP_OK) throw Error(rc, std::string(what) + ": " + dsgdpp_last_error(c));
}

char* h_block(dsgdpp_ctx* c, uint32_t b2, size_t* bytes) {
  const size_t es = elem_size(c->cfg.precision);
  *bytes = (c->off2[b2 + 1] - c->off2[b2]) * c->rp * es;
  return static_cast<char*>(c->H) + c->off2[b2] * c->rp * es;
}

// Waits for an event on the host, bounded; under NCCL an asynchronous NCCL
// error or the limit aborts the communicator.
void bounded_wait(dsgdpp_shard* sh, cudaEvent_t ev, const char* what) {
  TraceRange range("barrier");
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return;
    if (e != cudaErrorNotReady) check_cuda(e, what);
    if (sh->use_nccl && sh->comm) {
      ncclResult_t ae = ncclSuccess;
      nccl_api().CommGetAsyncError(sh->comm, &ae);
      if (ae != ncclSuccess && ae != ncclInProgress) {
        nccl_api().CommAbort(sh->comm);
        sh->comm = nullptr;
        throw Error(DSGDPP_E_CUDA, std::string(what) + ": NCCL reported " +
                                       nccl_api().GetErrorString(ae) +
                                       "; the communicator was aborted");
      }
    }
    const double s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (s > sh->wait_s) {
      if (sh->use_nccl && sh->comm) {
        nccl_api().CommAbort(sh->comm);
        sh->comm = nullptr;
      }
      throw Error(DSGDPP_E_CUDA, std::string(what) + ": not finished within " +
                                     std::to_string(sh->wait_s) +
                                     " s (a rank may have left); the communicator was aborted");
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

void require_comm(dsgdpp_shard* sh) {
  if (sh->use_nccl && !sh->comm)
    throw Error(DSGDPP_E_STATE, "the communicator was aborted after an earlier failure");
}

void make_events(dsgdpp_shard* sh, ShardRank& R) {
  auto mk = [](cudaEvent_t* e, bool timed) {
    check_cuda(cudaEventCreateWithFlags(e, timed ? cudaEventDefault : cudaEventDisableTiming),
               "event");
  };
  // the transfer stream outranks the compute stream, so a transfer's kernel
  // (NCCL's) takes the SMs that the running sub-epoch frees before the next
  // sub-epoch's CTAs do
  int least = 0, greatest = 0;
  check_cuda(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
  check_cuda(cudaStreamCreateWithPriority(&R.xfer, cudaStreamNonBlocking, greatest),
             "transfer stream");
  mk(&R.start, false);
  R.sub_end.resize(sh->nb2);
  R.group_done.resize(sh->nb2 + 1);
  for (auto& e : R.sub_end) mk(&e, false);
  for (auto& e : R.group_done) mk(&e, false);
  R.tc0.resize(sh->nb2);
  R.tc1.resize(sh->nb2);
  R.tx0.resize(sh->nb2 + 1);
  R.tx1.resize(sh->nb2 + 1);
  for (auto* v : {&R.tc0, &R.tc1, &R.tx0, &R.tx1})
    for (auto& e : *v) mk(&e, true);
  mk(&R.t_origin, true);
  R.group_used.assign(sh->nb2 + 1, 0);
}

void free_rank(ShardRank& R) {
  auto rel = [](cudaEvent_t& e) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  };
  rel(R.start);
  rel(R.t_origin);
  for (auto* v : {&R.sub_end, &R.group_done, &R.tc0, &R.tc1, &R.tx0, &R.tx1})
    for (auto& e : *v) rel(e);
  if (R.xfer) cudaStreamDestroy(R.xfer);
  R.xfer = nullptr;
}

void check_context(const dsgdpp_shard* sh, dsgdpp_ctx* c, int rank) {
  if (!c) throw Error(DSGDPP_E_INVALID, "null context");
  if (c->d != sh->d || c->nb2 != sh->nb2 || c->cfg.device != sh->device)
    throw Error(DSGDPP_E_INVALID, "the contexts of a shard must share d, the method and the device");
  if (c->cfg.exec == DSGDPP_EXEC_HOGWILD && c->cfg.launch == DSGDPP_LAUNCH_PERSISTENT)
    throw Error(DSGDPP_E_UNSUPPORTED, "a shard runs epochs one sub-epoch at a time; "
                                      "the persistent launch runs whole epochs only");
  const uint32_t per = sh->d / sh->world;
  if (c->task_lo != rank * per || c->task_hi != (rank + 1) * per)
    throw Error(DSGDPP_E_STATE, "rank " + std::to_string(rank) + "'s context must run tasks " +
                                    std::to_string(rank * per) + ".." +
                                    std::to_string((rank + 1) * per - 1) + " (dsgdpp_set_tasks)");
}

dsgdpp_shard* new_shard(uint32_t d, uint32_t nb2, int world, int device) {
  auto* sh = new dsgdpp_shard();
  sh->d = d;
  sh->nb2 = nb2;
  sh->world = world;
  sh->device = device;
  sh->holder.assign(nb2, kEveryone);
  return sh;
}

// The transfers of group g for every driven rank.
void post_group(dsgdpp_shard* sh, const Plan& plan, uint32_t g) {
  TraceRange range("communication");
  const auto& moves = plan.groups[g];
  for (auto& R : sh->ranks) {
    cudaEvent_t after = g == 0 ? R.start : R.sub_end[g - 1];
    check_cuda(cudaStreamWaitEvent(R.xfer, after, 0), "transfer wait");
  }
  if (sh->use_nccl) {
    ShardRank& R = sh->ranks[0];
    bool any = false;
    for (const Move& m : moves) any |= m.src == R.rank || m.dst == R.rank;
    R.group_used[g] = any;
    if (sh->timeline) check_cuda(cudaEventRecord(R.tx0[g], R.xfer), "event");
    if (any) {
      const NcclApi& api = nccl_api();
      check_nccl(api.GroupStart(), "ncclGroupStart");
      for (const Move& m : moves) {
        if (m.src != R.rank && m.dst != R.rank) continue;
        size_t bytes = 0;
        char* blk = h_block(R.ctx, m.b2, &bytes);
        if (m.src == R.rank) {
          check_nccl(api.Send(blk, bytes, ncclUint8, m.dst, sh->comm, R.xfer), "ncclSend");
        } else {
          check_nccl(api.Recv(blk, bytes, ncclUint8, m.src, sh->comm, R.xfer), "ncclRecv");
          sh->moved_bytes += bytes;
          sh->moves += 1;
        }
      }
      check_nccl(api.GroupEnd(), "ncclGroupEnd");
    }
    if (sh->timeline) check_cuda(cudaEventRecord(R.tx1[g], R.xfer), "event");
    check_cuda(cudaEventRecord(R.group_done[g], R.xfer), "event");
    return;
  }
  // emulated ranks: the receiver's transfer stream copies once both ranks are
  // past the sub-epoch that last used the block (the timeline's start is
  // taken after those waits, when the copies can begin)
  for (auto& D : sh->ranks) {
    D.group_used[g] = 0;  // the copies run on the receivers' transfer streams
    for (const Move& m : moves) {
      if (m.dst != D.rank) continue;
      const ShardRank& S = sh->ranks[m.src];
      check_cuda(cudaStreamWaitEvent(D.xfer, g == 0 ? S.start : S.sub_end[g - 1], 0),
                 "transfer wait");
      D.group_used[g] = 1;
    }
    if (sh->timeline) check_cuda(cudaEventRecord(D.tx0[g], D.xfer), "event");
    for (const Move& m : moves) {
      if (m.dst != D.rank) continue;
      size_t bytes = 0;
      const char* from = h_block(sh->ranks[m.src].ctx, m.b2, &bytes);
      char* to = h_block(D.ctx, m.b2, &bytes);
      check_cuda(cudaMemcpyAsync(to, from, bytes, cudaMemcpyDeviceToDevice, D.xfer), "block copy");
      sh->moved_bytes += bytes;
      sh->moves += 1;
    }
    if (sh->timeline) check_cuda(cudaEventRecord(D.tx1[g], D.xfer), "event");
    check_cuda(cudaEventRecord(D.group_done[g], D.xfer), "event");
  }
}

void shard_epoch_impl(dsgdpp_shard* sh, double eps, const uint32_t* schedule,
                      const uint32_t* seeds) {
  TraceRange range("epoch");
  require_comm(sh);
  check_cuda(cudaSetDevice(sh->device), "cudaSetDevice");
  const uint32_t d = sh->d, nb2 = sh->nb2;
  std::vector<uint32_t> sched, sd;
  if (!schedule || !seeds) {  // the master generator's draws (the same on every rank)
    sched.resize((size_t)nb2 * d);
    sd.resize(d);
    draw_epoch(sh->ranks[0].ctx, sched.data(), sd.data());
    for (size_t k = 1; k < sh->ranks.size(); ++k) {  // emulated ranks keep their generators in step
      std::vector<uint32_t> a(sched.size()), b(d);
      draw_epoch(sh->ranks[k].ctx, a.data(), b.data());
    }
    schedule = sched.data();
    seeds = sd.data();
  } else {
    for (size_t k = 0; k < (size_t)nb2 * d; ++k)
      if (schedule[k] >= nb2) throw Error(DSGDPP_E_INVALID, "schedule entry out of range");
  }
  std::vector<int> holder = sh->holder;
  const Plan plan = make_plan(schedule, d, nb2, sh->world, holder);
  sh->moved_bytes = 0;
  sh->moves = 0;
  sh->timeline_valid = false;
  for (auto& R : sh->ranks) {
    check_cuda(cudaEventRecord(R.start, R.ctx->stream), "event");
    if (sh->timeline) check_cuda(cudaEventRecord(R.t_origin, R.ctx->stream), "event");
  }
  post_group(sh, plan, 0);
  for (uint32_t s = 0; s < nb2; ++s) {
    for (auto& R : sh->ranks) {
      for (uint32_t g : plan.waits[(size_t)s * sh->world + R.rank])
        check_cuda(cudaStreamWaitEvent(R.ctx->stream, R.group_done[g], 0), "arrival wait");
      if (s + 1 == nb2) {
        // the last part scales all of H (lazy L2): no block may still travel
        for (auto& Q : sh->ranks)
          check_cuda(cudaStreamWaitEvent(R.ctx->stream, Q.group_done[s], 0), "transfer drain");
      }
      if (sh->timeline) check_cuda(cudaEventRecord(R.tc0[s], R.ctx->stream), "event");
      {
        TraceRange range("computation");
        check_ctx(R.ctx, dsgdpp_epoch_part(R.ctx, eps, schedule, seeds, s, s + 1), "sub-epoch");
      }
      if (sh->timeline) check_cuda(cudaEventRecord(R.tc1[s], R.ctx->stream), "event");
      check_cuda(cudaEventRecord(R.sub_end[s], R.ctx->stream), "event");
    }
    if (s + 1 < nb2) post_group(sh, plan, s + 1);
  }
  sh->holder = holder;
  sh->timeline_valid = sh->timeline;
  if (sh->use_nccl) bounded_wait(sh, sh->ranks[0].sub_end[nb2 - 1], "shard epoch");
}

// Every block's latest version to every rank, on the compute streams after
// the epoch.
void share_impl(dsgdpp_shard* sh) {
  TraceRange range("communication");
  require_comm(sh);
  check_cuda(cudaSetDevice(sh->device), "cudaSetDevice");
  if (sh->use_nccl) {
    ShardRank& R = sh->ranks[0];
    bool any = false;
    for (int h : sh->holder) any |= h != kEveryone;
    if (any) {
      const NcclApi& api = nccl_api();
      check_nccl(api.GroupStart(), "ncclGroupStart");
      for (uint32_t b = 0; b < sh->nb2; ++b) {
        if (sh->holder[b] == kEveryone) continue;
        size_t bytes = 0;
        char* blk = h_block(R.ctx, b, &bytes);
        check_nccl(api.Broadcast(blk, blk, bytes, ncclUint8, sh->holder[b], sh->comm,
                                 R.ctx->stream), "ncclBroadcast");
      }
      check_nccl(api.GroupEnd(), "ncclGroupEnd");
      check_cuda(cudaEventRecord(R.start, R.ctx->stream), "event");
      bounded_wait(sh, R.start, "share");
    }
  } else {
    for (auto& R : sh->ranks) check_cuda(cudaStreamSynchronize(R.ctx->stream), "sync");
    for (uint32_t b = 0; b < sh->nb2; ++b) {
      const int src = sh->holder[b];
      if (src == kEveryone) continue;
      size_t bytes = 0;
      const char* from = h_block(sh->ranks[src].ctx, b, &bytes);
      for (auto& R : sh->ranks) {
        if (R.rank == src) continue;
        check_cuda(cudaMemcpyAsync(h_block(R.ctx, b, &bytes), from, bytes,
                                   cudaMemcpyDeviceToDevice, R.ctx->stream), "block copy");
      }
    }
    for (auto& R : sh->ranks) check_cuda(cudaStreamSynchronize(R.ctx->stream), "sync");
  }
  sh->holder.assign(sh->nb2, kEveryone);
}

// The job's losses: per rank its entries' squared errors and its W rows' L2
// term, summed over the ranks, plus the H term once (every rank holds all of H
// after share_impl).
void losses_impl(dsgdpp_shard* sh, double* loss, double* test_loss) {
  for (int h : sh->holder)
    if (h != kEveryone)
      throw Error(DSGDPP_E_STATE, "share the H blocks (dsgdpp_shard_share) before the losses");
  double acc[3] = {0, 0, 0};  // training squared errors + W term, test squared errors, has test
  double hterm = 0;
  const dsgdpp_config& cfg = sh->ranks[0].ctx->cfg;
  for (auto& R : sh->ranks) {
    dsgdpp_ctx* c = R.ctx;
    double v = 0;
    check_ctx(c, dsgdpp_nzsl(c, DSGDPP_TRAIN, &v), "training loss");
    double w = 0, h = 0;
    if (cfg.loss == DSGDPP_LOSS_NZSL_L2) check_ctx(c, dsgdpp_l2(c, &w, &h), "l2");
    if (cfg.loss == DSGDPP_LOSS_NZSL_NZL2) check_ctx(c, dsgdpp_nzl2(c, &w, &h), "nzl2");
    acc[0] += v + (cfg.loss == DSGDPP_LOSS_NZSL ? 0.0 : cfg.loss_lambda * w);
    if (&R == &sh->ranks[0]) hterm = cfg.loss == DSGDPP_LOSS_NZSL ? 0.0 : cfg.loss_lambda * h;
    if (c->mat[DSGDPP_TEST].present) {
      check_ctx(c, dsgdpp_nzsl(c, DSGDPP_TEST, &v), "test loss");
      acc[1] += v;
      acc[2] = 1;
    }
  }
  if (sh->use_nccl && sh->world > 1) {
    ShardRank& R = sh->ranks[0];
    std::memcpy(sh->h_sum, acc, sizeof(acc));
    check_cuda(cudaMemcpyAsync(sh->d_sum, sh->h_sum, sizeof(acc), cudaMemcpyHostToDevice,
                               R.ctx->stream), "H2D sums");
    check_nccl(nccl_api().AllReduce(sh->d_sum, sh->d_sum, 3, ncclFloat64, ncclSum, sh->comm,
                                    R.ctx->stream), "ncclAllReduce");
    check_cuda(cudaMemcpyAsync(sh->h_sum, sh->d_sum, sizeof(acc), cudaMemcpyDeviceToHost,
                               R.ctx->stream), "D2H sums");
    check_cuda(cudaEventRecord(R.start, R.ctx->stream), "event");
    bounded_wait(sh, R.start, "loss sums");
    std::memcpy(acc, sh->h_sum, sizeof(acc));
  }
  if (loss) *loss = acc[0] + hterm;
  if (test_loss) *test_loss = acc[2] > 0 ? acc[1] : NAN;
}

}  // namespace

extern "C" {

int dsgdpp_shard_unique_id(void* id) {
  if (!id) return DSGDPP_E_INVALID;
  try {
    ncclUniqueId u;
    check_nccl(nccl_api().GetUniqueId(&u), "ncclGetUniqueId");
    static_assert(sizeof(ncclUniqueId) == DSGDPP_SHARD_ID_BYTES, "NCCL unique id size");
    std::memcpy(id, &u, sizeof(u));
    return DSGDPP_OK;
  } catch (const Error& e) {
    return e.code;
  }
}

int dsgdpp_shard_create_nccl(dsgdpp_ctx* ctx, int rank, int world, const void* id,
                             dsgdpp_shard** out) {
  if (!ctx || !id || !out || world < 1 || rank < 0 || rank >= world) return DSGDPP_E_INVALID;
  *out = nullptr;
  if (ctx->d % (uint32_t)world) {
    ctx->err = "d must be a multiple of the number of ranks";
    return DSGDPP_E_INVALID;
  }
  dsgdpp_shard* sh = new_shard(ctx->d, ctx->nb2, world, ctx->cfg.device);
  const int rc = shard_guarded(sh, [&]() {
    check_context(sh, ctx, rank);
    const NcclApi& api = nccl_api();
    sh->use_nccl = true;
    check_cuda(cudaSetDevice(sh->device), "cudaSetDevice");
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    check_nccl(api.CommInitRank(&sh->comm, world, u, rank), "ncclCommInitRank");
    sh->ranks.resize(1);
    sh->ranks[0].ctx = ctx;
    sh->ranks[0].rank = rank;
    make_events(sh, sh->ranks[0]);
    sh->d_sum = dalloc<double>(4, "loss sums");
    sh->h_sum = halloc<double>(4, "loss sums");
    return DSGDPP_OK;
  });
  if (rc != DSGDPP_OK) {
    ctx->err = sh->err;
    dsgdpp_shard_destroy(sh);
    return rc;
  }
  *out = sh;
  return DSGDPP_OK;
}

int dsgdpp_shard_create_local(dsgdpp_ctx* const* ctxs, int world, dsgdpp_shard** out) {
  if (!ctxs || !out || world < 1 || !ctxs[0]) return DSGDPP_E_INVALID;
  *out = nullptr;
  if (ctxs[0]->d % (uint32_t)world) {
    ctxs[0]->err = "d must be a multiple of the number of ranks";
    return DSGDPP_E_INVALID;
  }
  dsgdpp_shard* sh = new_shard(ctxs[0]->d, ctxs[0]->nb2, world, ctxs[0]->cfg.device);
  const int rc = shard_guarded(sh, [&]() {
    check_cuda(cudaSetDevice(sh->device), "cudaSetDevice");
    sh->ranks.resize(world);
    for (int r = 0; r < world; ++r) {
      check_context(sh, ctxs[r], r);
      sh->ranks[r].ctx = ctxs[r];
      sh->ranks[r].rank = r;
      make_events(sh, sh->ranks[r]);
    }
    return DSGDPP_OK;
  });
  if (rc != DSGDPP_OK) {
    ctxs[0]->err = sh->err;
    dsgdpp_shard_destroy(sh);
    return rc;
  }
  *out = sh;
  return DSGDPP_OK;
}

void dsgdpp_shard_destroy(dsgdpp_shard* sh) {
  if (!sh) return;
  cudaSetDevice(sh->device);
  for (auto& R : sh->ranks) {
    if (R.xfer) cudaStreamSynchronize(R.xfer);
    free_rank(R);
  }
  if (sh->comm) nccl_api().CommDestroy(sh->comm);
  dfree(sh->d_sum);
  hfree(sh->h_sum);
  delete sh;
}

const char* dsgdpp_shard_last_error(const dsgdpp_shard* sh) {
  return sh ? sh->err.c_str() : "null shard";
}

int dsgdpp_shard_set_wait_limit(dsgdpp_shard* sh, double seconds) {
  return shard_guarded(sh, [&]() {
    if (!(seconds > 0)) throw Error(DSGDPP_E_INVALID, "the wait limit must be positive");
    sh->wait_s = seconds;
    return DSGDPP_OK;
  });
}

int dsgdpp_shard_epoch(dsgdpp_shard* sh, double eps, const uint32_t* schedule,
                       const uint32_t* task_seeds) {
  return shard_guarded(sh, [&]() {
    if (!std::isfinite(eps)) throw Error(DSGDPP_E_INVALID, "step size is not finite");
    shard_epoch_impl(sh, eps, schedule, task_seeds);
    return DSGDPP_OK;
  });
}

int dsgdpp_shard_share(dsgdpp_shard* sh) {
  return shard_guarded(sh, [&]() {
    share_impl(sh);
    return DSGDPP_OK;
  });
}

int dsgdpp_shard_losses(dsgdpp_shard* sh, double* loss, double* test_loss) {
  return shard_guarded(sh, [&]() {
    require_comm(sh);
    check_cuda(cudaSetDevice(sh->device), "cudaSetDevice");
    losses_impl(sh, loss, test_loss);
    return DSGDPP_OK;
  });
}

int dsgdpp_shard_moved(dsgdpp_shard* sh, uint64_t* moves, uint64_t* bytes) {
  return shard_guarded(sh, [&]() {
    if (moves) *moves = sh->moves;
    if (bytes) *bytes = sh->moved_bytes;
    return DSGDPP_OK;
  });
}

int dsgdpp_shard_set_timeline(dsgdpp_shard* sh, int on) {
  return shard_guarded(sh, [&]() {
    sh->timeline = on != 0;
    sh->timeline_valid = false;
    return DSGDPP_OK;
  });
}

int dsgdpp_shard_timeline(dsgdpp_shard* sh, uint32_t index, double* compute, double* transfer) {
  return shard_guarded(sh, [&]() {
    if (!sh->timeline_valid) throw Error(DSGDPP_E_STATE, "no timed epoch (dsgdpp_shard_set_timeline)");
    if (index >= sh->ranks.size()) throw Error(DSGDPP_E_INVALID, "rank index out of range");
    ShardRank& R = sh->ranks[index];
    check_cuda(cudaSetDevice(sh->device), "cudaSetDevice");
    check_cuda(cudaStreamSynchronize(R.ctx->stream), "sync");
    check_cuda(cudaStreamSynchronize(R.xfer), "sync");
    auto ms = [&](cudaEvent_t e) {
      float f = 0;
      check_cuda(cudaEventElapsedTime(&f, R.t_origin, e), "elapsed");
      return (double)f;
    };
    for (uint32_t s = 0; s < sh->nb2; ++s) {
      if (compute) {
        compute[2 * s] = ms(R.tc0[s]);
        compute[2 * s + 1] = ms(R.tc1[s]);
      }
    }
    for (uint32_t g = 0; g < sh->nb2; ++g) {  // groups posted before the epoch and after s < nb2 - 1
      if (!transfer) break;
      if (R.group_used[g]) {
        transfer[2 * g] = ms(R.tx0[g]);
        transfer[2 * g + 1] = ms(R.tx1[g]);
      } else {
        transfer[2 * g] = transfer[2 * g + 1] = NAN;
      }
    }
    return DSGDPP_OK;
  });
}

int dsgdpp_shard_gather_w(dsgdpp_shard* sh) {
  return shard_guarded(sh, [&]() {
    require_comm(sh);
    check_cuda(cudaSetDevice(sh->device), "cudaSetDevice");
    dsgdpp_ctx* c0 = sh->ranks[0].ctx;
    const size_t es = elem_size(c0->cfg.precision);
    if (sh->use_nccl) {
      // every rank's W is zero outside its own rows: the sum over the ranks is W
      if (sh->world > 1) {
        const ncclDataType_t t = c0->cfg.precision == DSGDPP_FP64   ? ncclFloat64
                                 : c0->cfg.precision == DSGDPP_FP32 ? ncclFloat32
                                                                    : ncclBfloat16;
        check_nccl(nccl_api().AllReduce(c0->W, c0->W, c0->cfg.m * c0->rp, t, ncclSum, sh->comm,
                                        c0->stream), "ncclAllReduce");
        check_cuda(cudaEventRecord(sh->ranks[0].start, c0->stream), "event");
        bounded_wait(sh, sh->ranks[0].start, "gather W");
      }
    } else {
      for (auto& R : sh->ranks) check_cuda(cudaStreamSynchronize(R.ctx->stream), "sync");
      for (auto& S : sh->ranks) {
        const uint64_t lo = S.ctx->off1[S.ctx->task_lo], hi = S.ctx->off1[S.ctx->task_hi];
        const char* from = static_cast<const char*>(S.ctx->W) + lo * S.ctx->rp * es;
        for (auto& R : sh->ranks)
          if (&R != &S)
            check_cuda(cudaMemcpyAsync(static_cast<char*>(R.ctx->W) + lo * R.ctx->rp * es, from,
                                       (hi - lo) * R.ctx->rp * es, cudaMemcpyDeviceToDevice,
                                       R.ctx->stream), "row copy");
      }
      for (auto& R : sh->ranks) check_cuda(cudaStreamSynchronize(R.ctx->stream), "sync");
    }
    return DSGDPP_OK;
  });
}

// The hand-off plan of one epoch (host only): for each move, the group it is
// posted in (0 = before the epoch, s + 1 = after sub-epoch s), the block, the
// sending and the receiving rank.  holder (nb2 entries, -1 = every rank) is
// the state before the epoch and is updated.  Returns the number of moves
// (written only when out is not null).
uint64_t dsgdpp_shard_plan(uint32_t d, uint32_t nb2, int world, const uint32_t* schedule,
                           int32_t* holder, uint32_t* out) {
  if (!schedule || !holder || world < 1 || d % (uint32_t)world) return 0;
  std::vector<int> h(holder, holder + nb2);
  const Plan p = make_plan(schedule, d, nb2, world, h);
  uint64_t k = 0;
  for (uint32_t g = 0; g <= nb2; ++g)
    for (const Move& m : p.groups[g]) {
      if (out) {
        out[4 * k] = g;
        out[4 * k + 1] = m.b2;
        out[4 * k + 2] = (uint32_t)m.src;
        out[4 * k + 3] = (uint32_t)m.dst;
      }
      ++k;
    }
  if (out) std::copy(h.begin(), h.end(), holder);
  return k;
}

}  // extern "C"
