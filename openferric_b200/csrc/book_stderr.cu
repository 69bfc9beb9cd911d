// book_stderr.cu - of_book_price_to_stderr(_greeks): a book priced until
// every option meets a standard-error target.  Host-only: each round is one
// batched-book launch (of_mc_price_book, or of_mc_price_book_greeks with the
// pathwise Greeks) over the options still above their target.
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "of_internal.h"

namespace {

// Paths that bring a standard error measured with `paths` down to `target`
// (stderr ~ paths^-1/2), with a 10 % margin, rounded up to a multiple of 256;
// never fewer than `paths`.
int64_t paths_for_stderr(int64_t paths, double se, double target) {
  if (!(se > target)) return paths;
  const double need = (double)paths * (se / target) * (se / target) * 1.1;
  const int64_t rounded = (int64_t)std::ceil(need / 256.0) * 256;
  return rounded > paths ? rounded : paths;
}

}  // namespace

// The rounds of of_book_price_to_stderr(_greeks): `greeks` non-null prices
// every launch in mode OF_BOOK_GREEKS and keeps each option's Greeks from its
// last launch.
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
  std::vector<of_book_entry> cur(entries, entries + n);
  for (of_book_entry& e : cur) e.num_paths = target->pilot_paths;
  std::vector<int64_t> used((size_t)n, 0);  // paths of the launch that gave results[i]
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
      results[i] = res[k];
      if (greeks) greeks[i] = gr[k];
      used[(size_t)i] = cur[(size_t)i].num_paths;
      const double tgt = target->se_rel * entries[i].model.s0;
      if (res[k].stderr_ > tgt) {
        cur[(size_t)i].num_paths = paths_for_stderr(cur[(size_t)i].num_paths, res[k].stderr_, tgt);
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
    for (int64_t i = 0; i < n; ++i) paths_out[i] = used[(size_t)i];
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
