// of_internal.h - host-side internals shared by the libofgpu translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/of_gpu.h"

// Device scratch slots owned by a context.  Each slot is grown on demand and
// reused across calls (the reference re-allocates every call,
// src/engines/gpu/gpu_mc.rs:211-229).
enum OfSlot {
  SLOT_PARTIALS = 0,   // per-block FP64 partial sums
  SLOT_SUMS = 1,       // final FP64 sums
  SLOT_OBS = 2,        // per-step observation weights
  SLOT_INJECT = 3,     // injected normals (test hook)
  SLOT_STRIKES = 4,    // strike strip
  SLOT_BOOK = 5,       // batched-book option table
  SLOT_TILES = 6,      // batched-book tile table
  SLOT_DIVIDENDS = 7,  // discrete dividend triggers
  SLOT_LSM_PATHS = 8,  // LSM path store (time-major)
  SLOT_LSM_VALUES = 9, // LSM cash flows
  SLOT_LSM_AUX = 10,   // LSM betas / counters
  SLOT_ADJ_CKPT = 11,  // adjoint checkpoints
  SLOT_ADJ_AUX = 12,
  SLOT_STATUS = 13,    // device error word + counters
  SLOT_MISC = 14,
  SLOT_JUMP = 15,      // xoshiro256++ GF(2) jump tables
  SLOT_LSM_PATHS_B = 16,   // second LSM buffer set: the next batch generates into it
  SLOT_LSM_VALUES_B = 17,  // while the current one runs its passes
  SLOT_LSM_AUX_B = 18,
  SLOT_BOOK_DIVS = 19,     // book plans run inside one call (of_mc_price_book, the SE driver):
  SLOT_BOOK_GC = 20,       // their device tables and sums come from these slots
  SLOT_BOOK_COUNTER = 21,
  SLOT_BOOK_PARTIALS = 22,
  SLOT_BOOK_BEGIN = 23,
  SLOT_BOOK_SUMS = 24,
  SLOT_BOOK_OBS = 25,
  SLOT_COUNT = 26
};

struct of_ctx {
  int device = 0;
  int sm_count = 0;
  int max_threads_per_sm = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t side_stream = nullptr;  // lowest priority; created on first use (LSM path generation)
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  void* slot_ptr[SLOT_COUNT] = {};
  size_t slot_bytes[SLOT_COUNT] = {};
  void* pinned = nullptr;  // pinned host staging for results
  size_t pinned_bytes = 0;
  std::string last_error;
  // Set when a kernel gave up on asynchronous copies that were still in
  // flight into shared memory it no longer owns: from then on the context
  // refuses work, and the caller destroys it and creates a new one.
  bool unusable = false;
};

// Records a formatted message as the context's last error and returns `st`.
of_status of_fail(of_ctx* ctx, of_status st, const char* fmt, ...);

// OF_OK, or OF_ERR_CUDA with a message once the context is marked unusable.
of_status of_ctx_check(of_ctx* ctx);

// Returns a device buffer of at least `bytes` for `slot`, growing it if needed.
of_status of_scratch(of_ctx* ctx, int slot, size_t bytes, void** out);
// Returns pinned host memory of at least `bytes`.
of_status of_pinned(of_ctx* ctx, size_t bytes, void** out);

#define OF_CUDA_TRY(ctx, call)                                                                  \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return of_fail((ctx), OF_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                                       \
  } while (0)

#define OF_TRY(expr)                    \
  do {                                  \
    of_status s_ = (expr);              \
    if (s_ != OF_OK) return s_;         \
  } while (0)

// Deterministic reduction of a rows x cols FP64 matrix over its rows
// (fixed order, independent of timing); out[c] = sum_r in[r*cols + c].
of_status of_reduce_rows(of_ctx* ctx, const double* in, int64_t rows, int64_t cols, double* out);
// The same reduction enqueued on an explicit stream (used inside graph capture).
void of_launch_reduce_rows(const double* in, int64_t rows, int64_t cols, double* out, cudaStream_t s);

// Final Monte Carlo statistics of MonteCarloEngine::run (src/mc/simulation.rs:305-347)
// from the five running sums.
void of_mc_finish(const double sums[5], int64_t count, int32_t cv_kind, double cv_expected, double discount,
                  of_mc_result* out);

// Blocks per SM the occupancy calculator allows for `kernel` at `block` threads.
int of_blocks_per_sm(const void* kernel, int block, size_t smem);

// A discrete dividend of a GBM model resolved to the simulation step after
// which it applies (0-based step j: the jump follows the move to t = (j+1) dt).
struct of_div_trigger {
  int32_t step;
  int32_t kind;   // OF_DIV_CASH / OF_DIV_PROPORTIONAL
  double amount;  // cash amount or ratio
};

// Validates m->dividends (DividendSchedule::validate, src/market/dividends.rs:
// 131-144) and resolves them with the loop of DiscreteDividendGbmPathGenerator
// (src/engines/monte_carlo/mc_engine.rs:157-167): events that never trigger
// before maturity are dropped.  Non-GBM models with dividends are rejected.
of_status of_dividend_triggers(of_ctx* ctx, const of_model* m, std::vector<of_div_trigger>& out);
