// autotune.cu - native tile-shape autotuner of the C ABI.
//
// Each candidate tile shape is built into its own plan (a captured CUDA
// graph), replayed once untimed, then `reps` times between CUDA events on the
// context stream; a candidate's figure is the median of its replays.  The
// plans are the same objects a caller prices with, so the timed work is the
// pricing work.  Host-only code: no kernels of its own.

#include <algorithm>
#include <vector>

#include "of_internal.h"

namespace {

// Median device milliseconds of `reps` replays of `launch` on ctx->stream.
template <class Launch>
of_status time_replays(of_ctx* ctx, Launch launch, int reps, double* ms_out) {
  OF_TRY(launch());  // warm-up: first replay uploads the graph and raises clocks
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  std::vector<float> ms((size_t)reps, 0.0f);
  for (int r = 0; r < reps; ++r) {
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
    OF_TRY(launch());
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
    OF_CUDA_TRY(ctx, cudaEventSynchronize(ctx->ev_stop));
    OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms[(size_t)r], ctx->ev_start, ctx->ev_stop));
  }
  std::sort(ms.begin(), ms.end());
  const size_t h = ms.size() / 2;
  *ms_out = ms.size() % 2 ? ms[h] : 0.5 * ((double)ms[h - 1] + (double)ms[h]);
  return OF_OK;
}

of_status check_args(of_ctx* ctx, const of_tune_candidate* c, int32_t n_cands, int32_t reps, int32_t* best) {
  if (!ctx) return OF_ERR_INVALID_INPUT;
  if (!c || !best || n_cands <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "autotune needs at least one candidate");
  if (reps <= 0 || reps > 1000) return of_fail(ctx, OF_ERR_INVALID_INPUT, "autotune reps must be in 1..1000");
  return OF_OK;
}

int32_t fastest(const of_tune_candidate* c, int32_t n) {
  int32_t b = 0;
  for (int32_t i = 1; i < n; ++i)
    if (c[i].ms < c[b].ms) b = i;
  return b;
}

}  // namespace

extern "C" of_status of_autotune_strip(of_ctx* ctx, const of_model* model, int32_t option_type,
                                       const double* strikes, int64_t n_strikes, const of_mc_config* cfg,
                                       of_tune_candidate* cands, int32_t n_cands, int32_t reps, int32_t* best) {
  OF_TRY(check_args(ctx, cands, n_cands, reps, best));
  if (!cfg) return of_fail(ctx, OF_ERR_INVALID_INPUT, "null config");
  for (int32_t i = 0; i < n_cands; ++i) {
    if (cands[i].paths_per_thread < 1 || cands[i].paths_per_thread > 3)
      return of_fail(ctx, OF_ERR_INVALID_INPUT,
                     "strip candidate %d: tile shape must be 1 or 2 samples in flight per thread, or 3 "
                     "(warp-specialised)", i);
  }
  for (int32_t i = 0; i < n_cands; ++i) {
    of_mc_config c = *cfg;
    c.tile_ilp = cands[i].paths_per_thread;
    of_strip_plan* pl = nullptr;
    OF_TRY(of_strip_plan_create(ctx, model, option_type, strikes, n_strikes, &c, &pl));
    double ms = 0.0;
    const of_status st = time_replays(ctx, [&] { return of_strip_plan_launch(pl); }, reps, &ms);
    of_strip_plan_destroy(pl);
    OF_TRY(st);
    cands[i].block = 0;
    cands[i].ms = ms;
  }
  *best = fastest(cands, n_cands);
  return OF_OK;
}

extern "C" of_status of_autotune_book(of_ctx* ctx, const of_book_entry* entries, int64_t n,
                                      const of_book_config* cfg, of_tune_candidate* cands, int32_t n_cands,
                                      int32_t reps, int32_t* best) {
  OF_TRY(check_args(ctx, cands, n_cands, reps, best));
  if (!cfg) return of_fail(ctx, OF_ERR_INVALID_INPUT, "null config");
  for (int32_t i = 0; i < n_cands; ++i) {
    const int b = cands[i].block, p = cands[i].paths_per_thread;
    // the book kernel is compiled for at most 256 threads per block
    if (b < 32 || b > 256 || b % 32 != 0 || p < 1 || p > 256)
      return of_fail(ctx, OF_ERR_INVALID_INPUT,
                     "book candidate %d: block must be a multiple of 32 in 32..256 and paths_per_thread in 1..256", i);
  }
  for (int32_t i = 0; i < n_cands; ++i) {
    of_book_config c = *cfg;
    c.block = cands[i].block;
    c.paths_per_thread = cands[i].paths_per_thread;
    c.use_graph = 1;
    of_book_plan* pl = nullptr;
    OF_TRY(of_book_plan_create(ctx, entries, n, &c, &pl));
    double ms = 0.0;
    const of_status st = time_replays(ctx, [&] { return of_book_plan_launch(pl); }, reps, &ms);
    of_book_plan_destroy(pl);
    OF_TRY(st);
    cands[i].ms = ms;
  }
  *best = fastest(cands, n_cands);
  return OF_OK;
}
