// controller.cc -- the learned step-size controller's epoch loop over the C ABI.
//
// defaultRunner (mf/sgd/sgd_impl.h:34-145) with the step chosen by the
// controller network instead of BoldDriver's multiplier.  Each epoch:
//   1. the network maps the 16 history features to a log multiplier m in
//      [-1, 1]; the proposed step is eps * exp(m);
//   2. the factors are saved on the device and the epoch runs with the
//      proposed step;
//   3. if the training loss rose, BoldDriver takes over for this decision --
//      a fallback event (decay_bolddriver.h:59-67: halve the step that raised
//      the loss).  A rise of at most kKeepRise is kept, as BoldDriver keeps
//      it, and the next step is the proposal halved.  A larger rise (or a
//      non-finite loss) is rolled back: the factors are restored and the
//      epoch re-runs with the proposal halved, again and again until the loss
//      rises by at most kKeepRise (at most kMaxHalvings times; the last
//      attempt is kept).
//      An epoch in which one factor row moved more than kBombRatio times the
//      mean row movement, and more than kBombGrow times the median largest
//      movement of the last three kept epochs (after the first decision),
//      counts as a large rise even when the loss fell: such a row makes the
//      next epochs diverge at any step near the current one, so it is rolled
//      back at once.  The second condition keeps small steps from a state
//      that still pulls one row back (movement linear in the step, so the
//      ratio alone does not fall) from being rejected without end.
//      The smallest step that raised the loss (fail_eps) is a feature of later
//      decisions and caps them: a proposal is at most kCapFrac * fail_eps,
//      and fail_eps grows by kCapRelax (BoldDriver's increase) after every
//      decision without a rise, so the edge is probed again slowly;
//   4. the run stops early once the test loss reaches the target.
// No reference counterpart (the reference's BoldDriver never rolls back).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "../../include/dsgdpp.h"

namespace {

constexpr double kKeepRise = 0.01;  // relative training-loss rise kept without rollback
constexpr int kMaxHalvings = 8;
constexpr double kCapFrac = 0.9;    // proposals stay below this fraction of fail_eps
constexpr double kCapRelax = 1.05;  // fail_eps growth per decision without a rise
constexpr double kBombRatio = 40.0; // largest / mean row movement of an epoch that is kept ...
constexpr double kBombGrow = 4.0;   // ... unless the largest also grew this much over recent epochs

double since(std::chrono::steady_clock::time_point a) {
  return (double)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now() - a).count();
}

}  // namespace

extern "C" int dsgdpp_run_controlled(dsgdpp_ctx* ctx, dsgdpp_mlp* mlp, uint32_t epochs,
                                     double eps0, double decrease, double increase,
                                     double target_test_loss, dsgdpp_trace_row* trace,
                                     uint32_t* epochs_done, uint32_t* fallbacks) {
  if (!ctx || !mlp || epochs == 0) return DSGDPP_E_INVALID;
  int rc;
  std::vector<double> tr(5, NAN), te(5, NAN);  // index 0 = newest
  auto push = [](std::vector<double>& h, double v) {
    for (int k = 4; k > 0; --k) h[k] = h[k - 1];
    h[0] = v;
  };
  auto t0 = std::chrono::steady_clock::now();
  double loss = 0, test = NAN;
  if ((rc = dsgdpp_loss(ctx, &loss)) != DSGDPP_OK) return rc;
  const double tl = since(t0);
  auto t1 = std::chrono::steady_clock::now();
  const bool has_test = dsgdpp_nzsl(ctx, DSGDPP_TEST, &test) == DSGDPP_OK;
  if (!has_test) test = NAN;
  if (trace) trace[0] = dsgdpp_trace_row{0, loss, test, NAN, 0, 0, tl, has_test ? since(t1) : 0.0};
  push(tr, loss);
  push(te, test);
  // the factor snapshot is allocated by its first save: do that before the timed epochs
  if ((rc = dsgdpp_save_factors(ctx)) != DSGDPP_OK) return rc;
  double eps = eps0, upd_mean = 0, upd_max = 0, last_m = 0, fail_eps = 0;
  std::vector<double> kept_max;  // largest row movement of each kept epoch
  auto recent_max = [&]() {       // median of the last three
    std::vector<double> v(kept_max.end() - std::min<size_t>(3, kept_max.size()), kept_max.end());
    std::sort(v.begin(), v.end());
    return v.empty() ? 0.0 : v[v.size() / 2];
  };
  auto failed = [&](double step) { fail_eps = fail_eps > 0 ? std::fmin(fail_eps, step) : step; };
  uint32_t fb = 0, e = 0;
  for (; e < epochs; ++e) {
    auto a = std::chrono::steady_clock::now();
    float f[16], m = 0;
    dsgdpp_controller_features(tr.data(), te.data(), eps, upd_mean, upd_max,
                               (double)e / (double)epochs, last_m, fail_eps, f);
    if ((rc = dsgdpp_mlp_forward(mlp, f, 1, &m)) != DSGDPP_OK) return rc;
    double proposed = eps * std::exp((double)m);
    if (fail_eps > 0) proposed = std::fmin(proposed, kCapFrac * fail_eps);
    const double t_eps = since(a);
    auto b = std::chrono::steady_clock::now();
    if ((rc = dsgdpp_save_factors(ctx)) != DSGDPP_OK) return rc;
    if ((rc = dsgdpp_epoch(ctx, proposed)) != DSGDPP_OK) return rc;
    double cur = 0;
    if ((rc = dsgdpp_loss(ctx, &cur)) != DSGDPP_OK) return rc;
    if ((rc = dsgdpp_update_norms(ctx, &upd_mean, &upd_max)) != DSGDPP_OK) return rc;
    auto bomb = [&]() {
      return e > 0 && upd_max > kBombRatio * upd_mean && upd_max > kBombGrow * recent_max();
    };
    double used = proposed, next = proposed;
    if (!(cur <= tr[0]) || bomb()) {  // the proposed step raised the training loss: fallback
      ++fb;
      failed(proposed);
      if (!bomb() && cur <= tr[0] * (1.0 + kKeepRise)) {
        next = proposed * decrease;  // kept, as BoldDriver keeps it
      } else {
        double step = proposed;
        for (int k = 0; k < kMaxHalvings; ++k) {
          step *= decrease;
          if ((rc = dsgdpp_restore_factors(ctx)) != DSGDPP_OK) return rc;
          if ((rc = dsgdpp_epoch(ctx, step)) != DSGDPP_OK) return rc;
          if ((rc = dsgdpp_loss(ctx, &cur)) != DSGDPP_OK) return rc;
          if ((rc = dsgdpp_update_norms(ctx, &upd_mean, &upd_max)) != DSGDPP_OK) return rc;
          if (!bomb() && cur <= tr[0] * (1.0 + kKeepRise)) break;  // kept, as the first attempt
          failed(step);
        }
        used = step;
        next = cur <= tr[0] ? step : step * decrease;
      }
    } else if (fail_eps > 0) {
      fail_eps *= kCapRelax;
    }
    (void)increase;
    last_m = std::log(next / eps);
    kept_max.push_back(upd_max);
    const double t_epoch = since(b);
    eps = next;
    auto c = std::chrono::steady_clock::now();
    if (has_test && (rc = dsgdpp_nzsl(ctx, DSGDPP_TEST, &test)) != DSGDPP_OK) return rc;
    const double t_test = has_test ? since(c) : 0.0;
    push(tr, cur);
    push(te, test);
    if (trace) trace[e + 1] = dsgdpp_trace_row{e + 1u, cur, test, used, t_eps, t_epoch, 0.0, t_test};
    if (target_test_loss > 0 && has_test && test <= target_test_loss) {
      ++e;
      break;
    }
  }
  if (epochs_done) *epochs_done = e;
  if (fallbacks) *fallbacks = fb;
  return DSGDPP_OK;
}
