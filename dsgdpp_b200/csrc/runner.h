// runner.h -- C++ host driver of the B200 DSGD++ epoch over the C ABI.
//
// Mirrors the reference's runner layer:
//  * Trace / SgdTraceEntry and the R-file writer (mf/trace.h:46-261);
//  * BoldDriver / DecayConstant (mf/sgd/decay/decay_bolddriver.h:59-67,
//    decay_constant.h:31-63);
//  * detail::defaultRunner (mf/sgd/sgd_impl.h:34-145) with its log lines
//    "Loss: ...", "Test loss: ...", "Step size: ...", "Starting epoch k",
//    "Finished epoch k (t)";
//  * DsgdPpRunner::run (mf/sgd/dsgdpp_impl.h:29-61).
// The epochs and losses themselves run on the GPU through include/dsgdpp.h.
#pragma once

#include <chrono>
#include <cmath>
#include <cstdio>
#include <functional>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dsgdpp.h"

namespace dsgdpp {

// log4cxx-like lines: "<ms since start> <logger> | <message>"
class Log {
 public:
  static bool& quiet() {  // ranks other than 0 of a job over several ranks stay quiet
    static bool q = false;
    return q;
  }
  static void info(const char* logger, const std::string& msg) {
    static const auto t0 = std::chrono::steady_clock::now();
    if (quiet()) return;
    long long ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                       std::chrono::steady_clock::now() - t0).count();
    std::printf("%8lld %-4s | %s\n", ms, logger, msg.c_str());
    std::fflush(stdout);
  }
};

inline std::string fmt_g(double v) {  // default ostream formatting (precision 6)
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%g", v);
  return buf;
}

// rg::Timer printing: "<seconds>s"
inline std::string fmt_secs(double ns) { return fmt_g(ns / 1e9) + "s"; }

struct TraceRow {
  uint64_t epoch = 0, iteration = 0;
  double loss = NAN, test_loss = NAN, eps = NAN;
  double time_eps = 0, time_epoch = 0, time_loss = 0, time_test_loss = 0;
};

class Trace {
 public:
  void add(const TraceRow& r) { rows_.push_back(r); }
  void clear() { rows_.clear(); }
  void add_field(const std::string& k, double v) { dbl_[k] = v; }
  void add_field(const std::string& k, const std::string& v) { str_[k] = v; }
  const std::vector<TraceRow>& rows() const { return rows_; }

  // Trace::toRstream (mf/trace.h:224-244) with SgdTraceEntry rows
  std::string to_r(const std::string& var = "trace") const {
    std::ostringstream o;
    o << var << " <- list(trace=list(";
    std::string sep;
    double elapsed = 0;
    for (const auto& r : rows_) {
      o << sep << "\n";
      o << "list(it=" << r.iteration << ", epoch=" << r.epoch << ", loss=" << fmt_g(r.loss)
        << ", loss.test=" << (std::isnan(r.test_loss) ? "NA" : fmt_g(r.test_loss)) << ", ";
      elapsed += (r.time_eps + r.time_epoch + r.time_loss + r.time_test_loss) / 1e9;
      o << "time=list(elapsed=" << fmt_g(elapsed) << ", eps=" << fmt_g(r.time_eps / 1e9)
        << ", epoch=" << fmt_g(r.time_epoch / 1e9) << ", loss=" << fmt_g(r.time_loss / 1e9)
        << ", loss.test=" << fmt_g(r.time_test_loss / 1e9) << "), ";
      o << " eps=" << (std::isnan(r.eps) ? "NA" : fmt_g(r.eps));
      o << ")";
      sep = ", ";
    }
    o << "\n)";
    if (!dbl_.empty() || !str_.empty()) {
      o << ", info=list(";
      std::string s;
      for (auto& kv : dbl_) {
        o << s << kv.first << " = " << fmt_g(kv.second);
        s = ", ";
      }
      s = dbl_.empty() ? "" : ", ";
      for (auto& kv : str_) {
        o << s << kv.first << " = \"" << kv.second << "\"";
        s = ", ";
      }
      o << ")";
    }
    o << ");";
    return o.str();
  }

 private:
  std::vector<TraceRow> rows_;
  std::map<std::string, double> dbl_;
  std::map<std::string, std::string> str_;
};

struct Decay {
  int kind = DSGDPP_DECAY_BOLDDRIVER;
  double eps = 0.001, decrease = 0.5, increase = 1.05;
  // AdaptiveDecayConcept::operator()(data, prevLoss, curLoss, random)
  double operator()(const double* prev, double cur) {
    if (kind == DSGDPP_DECAY_CONST || prev == nullptr) return eps;
    eps *= (*prev <= cur) ? decrease : increase;
    return eps;
  }
};

struct CallError : std::runtime_error {
  int status;
  CallError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(dsgdpp_ctx* ctx, int rc, const char* what) {
  if (rc != DSGDPP_OK)
    throw CallError(rc, std::string(what) + ": " + (ctx ? dsgdpp_last_error(ctx) : "") + " (" +
                            dsgdpp_status_string(rc) + ")");
}

// What the runner drives: one context, or one job over several ranks.
struct RunOps {
  std::function<void(double)> epoch;  // one epoch at this step size, finished on return
  std::function<double()> loss;       // the training loss
  std::function<double()> test_loss;  // the test loss (after loss())
};

// detail::defaultRunner over the C ABI.
inline void run_epochs(const RunOps& ops, uint64_t epochs, Decay decay, Trace& trace,
                       bool has_test) {
  using clock = std::chrono::steady_clock;
  auto ns = [](clock::time_point a, clock::time_point b) {
    return (double)std::chrono::duration_cast<std::chrono::nanoseconds>(b - a).count();
  };
  double previous = 0, current = 0, test = NAN;
  auto t0 = clock::now();
  current = ops.loss();
  auto t1 = clock::now();
  trace.clear();
  Log::info("mf", "Loss: " + fmt_g(current) + " (" + fmt_secs(ns(t0, t1)) + ")");
  TraceRow first;
  first.loss = current;
  first.time_loss = ns(t0, t1);
  if (has_test) {
    auto a = clock::now();
    test = ops.test_loss();
    auto b = clock::now();
    Log::info("mf", "Test loss: " + fmt_g(test) + " (" + fmt_secs(ns(a, b)) + ")");
    first.test_loss = test;
    first.time_test_loss = ns(a, b);
  }
  trace.add(first);
  for (uint64_t e = 0; e < epochs; ++e) {
    auto a = clock::now();
    double eps = e == 0 ? decay(nullptr, current) : decay(&previous, current);
    auto b = clock::now();
    Log::info("mf", "Step size: " + fmt_g(eps) + " (" + fmt_secs(ns(a, b)) + ")");
    Log::info("mf", "Starting epoch " + std::to_string(e + 1));
    auto c = clock::now();
    ops.epoch(eps);
    auto dd = clock::now();
    Log::info("mf", "Finished epoch " + std::to_string(e + 1) + " (" + fmt_secs(ns(c, dd)) + ")");
    previous = current;
    auto f = clock::now();
    current = ops.loss();
    auto g = clock::now();
    Log::info("mf", "Loss: " + fmt_g(current) + " (" + fmt_secs(ns(f, g)) + ")");
    TraceRow row;
    row.epoch = row.iteration = e + 1;
    row.loss = current;
    row.eps = eps;
    row.time_eps = ns(a, b);
    row.time_epoch = ns(c, dd);
    row.time_loss = ns(f, g);
    if (has_test) {
      auto h = clock::now();
      test = ops.test_loss();
      auto k = clock::now();
      Log::info("mf", "Test loss: " + fmt_g(test) + " (" + fmt_secs(ns(h, k)) + ")");
      row.test_loss = test;
      row.time_test_loss = ns(h, k);
    }
    trace.add(row);
  }
}

inline void default_runner(dsgdpp_ctx* ctx, uint64_t epochs, Decay decay, Trace& trace,
                           bool has_test) {
  RunOps ops;
  ops.epoch = [ctx](double eps) {
    check(ctx, dsgdpp_epoch(ctx, eps), "epoch");
    check(ctx, dsgdpp_sync(ctx), "sync");
  };
  ops.loss = [ctx]() {
    double v = 0;
    check(ctx, dsgdpp_loss(ctx, &v), "loss");
    return v;
  };
  ops.test_loss = [ctx]() {
    double v = 0;
    check(ctx, dsgdpp_nzsl(ctx, DSGDPP_TEST, &v), "test loss");
    return v;
  };
  run_epochs(ops, epochs, decay, trace, has_test);
}

inline void check_shard(dsgdpp_shard* sh, int rc, const char* what) {
  if (rc != DSGDPP_OK)
    throw CallError(rc, std::string(what) + ": " + dsgdpp_shard_last_error(sh) + " (" +
                            dsgdpp_status_string(rc) + ")");
}

// The same loop over a job on several ranks: an epoch is the shard's epoch
// (schedule drawn by every rank's master generator, seeded alike) followed by
// the broadcast of every H block from its holder; the losses are the job's.
inline void shard_runner(dsgdpp_shard* sh, uint64_t epochs, Decay decay, Trace& trace,
                         bool has_test) {
  double test = NAN;
  RunOps ops;
  ops.epoch = [sh](double eps) {
    check_shard(sh, dsgdpp_shard_epoch(sh, eps, nullptr, nullptr), "shard epoch");
    check_shard(sh, dsgdpp_shard_share(sh), "shard share");
  };
  ops.loss = [sh, &test]() {
    double v = 0;
    check_shard(sh, dsgdpp_shard_losses(sh, &v, &test), "shard losses");
    return v;
  };
  ops.test_loss = [&test]() { return test; };
  run_epochs(ops, epochs, decay, trace, has_test);
}

}  // namespace dsgdpp
