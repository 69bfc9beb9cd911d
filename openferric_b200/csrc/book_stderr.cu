// book_stderr.cu - of_book_price_to_stderr(_greeks): a book priced until
// every option meets a standard-error target.  Host-only: each round is one
// batched-book launch (of_mc_price_book, or of_mc_price_book_greeks with the
// pathwise Greeks) over the options still above their target, and each
// option's estimate pools the samples of all its rounds.
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "of_internal.h"

namespace {

// Total paths that bring a standard error measured over `paths` down to
// `target` (stderr ~ paths^-1/2), times `margin`; the next round runs the
// difference, rounded up to a multiple of 256 (at least 256).
int64_t more_paths_for_stderr(int64_t paths, double se, double target, double margin) {
  const double need = (double)paths * (se / target) * (se / target) * margin;
  const int64_t more = (int64_t)std::ceil((need - (double)paths) / 256.0) * 256;
  return more > 256 ? more : 256;
}

// One option's pooled running sums over its rounds: the five sums of
// MonteCarloEngine::run and, per Greek, the sum and sum of squares of the
// discounted per-sample derivatives.
struct Pool {
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  double g1[4] = {0.0, 0.0, 0.0, 0.0}, g2[4] = {0.0, 0.0, 0.0, 0.0};
  int64_t samples = 0, paths = 0;
};

}  // namespace

// The rounds of of_book_price_to_stderr(_greeks): `greeks` non-null prices
// every launch in mode OF_BOOK_GREEKS.  The rounds draw from independent
// streams (seed + round), so an option's samples from all its rounds form one
// sample of their total size: the pooled running sums give its estimate (the
// control-variate coefficient included) and its standard error, and the next
// round adds only the paths still missing.
static of_status price_to_stderr(of_ctx* ctx, const of_book_entry* entries, int64_t n, const of_book_config* cfg,
                                 const of_stderr_target* target, of_mc_result* results, of_book_greeks* greeks,
                                 int64_t* paths_out, of_stderr_round* rounds, int32_t* n_rounds) {
  if (!ctx) return OF_ERR_INVALID_INPUT;
  if (!entries || !cfg || !target || !results || !n_rounds || n <= 0)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "book, config, target, results and n_rounds are required");
  if (!(target->se_rel > 0.0) || !std::isfinite(target->se_rel))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "se_rel must be finite and > 0");
  if (target->pilot_paths <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "pilot_paths must be > 0");
  if (target->max_rounds <= 0 || target->max_rounds > 64)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "max_rounds must be in 1..64");
  if (!(target->margin >= 0.0) || !std::isfinite(target->margin) || (target->margin > 0.0 && target->margin < 1.0))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "margin must be 0 (default) or finite and >= 1");
  const double margin = target->margin > 0.0 ? target->margin : 1.05;
  std::vector<of_book_entry> cur(entries, entries + n);
  for (of_book_entry& e : cur) e.num_paths = target->pilot_paths;
  std::vector<Pool> pool((size_t)n);
  std::vector<int64_t> pending((size_t)n);
  for (int64_t i = 0; i < n; ++i) pending[(size_t)i] = i;
  std::vector<of_book_entry> sub;
  std::vector<of_mc_result> res;
  std::vector<of_book_greeks> gr;
  int32_t r = 0;
  for (; r < target->max_rounds && !pending.empty(); ++r) {
    sub.clear();
    int64_t total = 0;
    double steps = 0.0;
    for (int64_t i : pending) {
      sub.push_back(cur[(size_t)i]);
      total += cur[(size_t)i].num_paths;
      steps += (double)cur[(size_t)i].num_paths * (double)cur[(size_t)i].model.steps;
    }
    of_book_config c = *cfg;
    c.seed = cfg->seed + (uint64_t)r;  // independent draws per round
    c.use_graph = 0;
    if (c.block <= 0) c.block = 256;
    if (c.paths_per_thread <= 0) {  // at most ~2^18 tiles per launch
      int32_t ppt = 4;
      while (ppt < 256 && total > ((int64_t)c.block * ppt) << 18) ppt *= 2;
      c.paths_per_thread = ppt;
    }
    const auto t0 = std::chrono::steady_clock::now();
    res.assign(sub.size(), of_mc_result{});
    if (greeks) {
      gr.assign(sub.size(), of_book_greeks{});
      OF_TRY(of_mc_price_book_greeks(ctx, sub.data(), (int64_t)sub.size(), &c, res.data(), gr.data()));
    } else {
      OF_TRY(of_mc_price_book(ctx, sub.data(), (int64_t)sub.size(), &c, res.data()));
    }
    std::vector<int64_t> still;
    for (size_t k = 0; k < pending.size(); ++k) {
      const int64_t i = pending[k];
      const of_book_entry& e = entries[i];
      Pool& p = pool[(size_t)i];
      const of_mc_result& o = res[k];
      p.s[0] += o.sum_x;
      p.s[1] += o.sum_x2;
      p.s[2] += o.sum_y;
      p.s[3] += o.sum_xy;
      p.s[4] += o.sum_y2;
      const int64_t m = o.samples;
      p.samples += m;
      p.paths += cur[(size_t)i].num_paths;
      of_mc_finish(p.s, p.samples, e.control_variate, e.cv_expected, e.discount_factor, &results[i]);
      results[i].kernel_ms = o.kernel_ms;
      if (greeks) {
        // the round's sums back from its means and standard errors:
        // S1 = n mean, S2 = n (n - 1) se^2 + S1^2 / n
        const of_book_greeks& q = gr[k];
        const double mean[4] = {q.delta, q.vega, q.rho, q.theta};
        const double se[4] = {q.delta_se, q.vega_se, q.rho_se, q.theta_se};
        const double nm = (double)m, nt = (double)p.samples;
        double pm[4], ps[4];
        for (int t = 0; t < 4; ++t) {
          const double s1 = nm * mean[t];
          p.g1[t] += s1;
          p.g2[t] += nm * (nm - 1.0) * se[t] * se[t] + (nm > 0.0 ? s1 * s1 / nm : 0.0);
          pm[t] = p.g1[t] / nt;
          const double var = nt > 1.0 ? std::fmax(p.g2[t] - p.g1[t] * p.g1[t] / nt, 0.0) / (nt - 1.0) : 0.0;
          ps[t] = std::sqrt(var / nt);
        }
        of_book_greeks& out = greeks[i];
        out = of_book_greeks{};
        out.delta = pm[0];
        out.vega = pm[1];
        out.rho = pm[2];
        out.theta = pm[3];
        out.delta_se = ps[0];
        out.vega_se = ps[1];
        out.rho_se = ps[2];
        out.theta_se = ps[3];
      }
      const double tgt = target->se_rel * e.model.s0;
      if (results[i].stderr_ > tgt) {
        cur[(size_t)i].num_paths = more_paths_for_stderr(p.paths, results[i].stderr_, tgt, margin);
        still.push_back(i);
      }
    }
    if (rounds) {
      of_stderr_round& o = rounds[r];
      o.options = (int64_t)pending.size();
      o.paths = total;
      o.path_steps = steps;
      o.converged = (int64_t)(pending.size() - still.size());
      o.kernel_ms = res.empty() ? 0.0 : res[0].kernel_ms;
      o.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    pending.swap(still);
  }
  if (paths_out)
    for (int64_t i = 0; i < n; ++i) paths_out[i] = pool[(size_t)i].paths;
  *n_rounds = r;
  return OF_OK;
}

extern "C" of_status of_book_price_to_stderr(of_ctx* ctx, const of_book_entry* entries, int64_t n,
                                             const of_book_config* cfg, const of_stderr_target* target,
                                             of_mc_result* results, int64_t* paths_out, of_stderr_round* rounds,
                                             int32_t* n_rounds) {
  return price_to_stderr(ctx, entries, n, cfg, target, results, nullptr, paths_out, rounds, n_rounds);
}

extern "C" of_status of_book_price_to_stderr_greeks(of_ctx* ctx, const of_book_entry* entries, int64_t n,
                                                    const of_book_config* cfg, const of_stderr_target* target,
                                                    of_mc_result* results, of_book_greeks* greeks, int64_t* paths_out,
                                                    of_stderr_round* rounds, int32_t* n_rounds) {
  if (ctx && !greeks) return of_fail(ctx, OF_ERR_INVALID_INPUT, "greeks is required");
  return price_to_stderr(ctx, entries, n, cfg, target, results, greeks, paths_out, rounds, n_rounds);
}
