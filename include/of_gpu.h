/*
 * of_gpu.h - C ABI of the B200 Monte Carlo pricing engine (libofgpu.so).
 *
 * Plain C, no CUDA or torch types: every argument is a POD struct, a plain
 * pointer to caller-owned host memory, or a size.  Device memory is owned by
 * the library inside an of_ctx (pooled, grown on demand, released by
 * of_ctx_destroy).  All calls are synchronous to the caller unless stated.
 *
 * Each entry point names the openferric interface it replaces (path:line in
 * the rosssaunders/openferric source tree).
 *
 * Error behaviour follows openferric's `PricingError` (src/core/engine.rs:293-302):
 * OF_ERR_INVALID_INPUT  -> PricingError::InvalidInput
 * OF_ERR_NUMERICAL      -> PricingError::NumericalError
 * OF_ERR_CONVERGENCE    -> PricingError::ConvergenceFailure
 * the remaining codes are device-side failures with no reference counterpart.
 * The message of the last failure on a context is returned by of_ctx_last_error.
 */
#ifndef OF_GPU_H
#define OF_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OF_GPU_ABI_VERSION 1

typedef enum of_status {
  OF_OK = 0,
  OF_ERR_INVALID_INPUT = 1,
  OF_ERR_NUMERICAL = 2,
  OF_ERR_CUDA = 3,
  OF_ERR_TIMEOUT = 4,
  OF_ERR_UNSUPPORTED = 5,
  OF_ERR_ALLOC = 6,
  OF_ERR_CONVERGENCE = 7
} of_status;

/* openferric core::OptionType (src/core/types.rs:13-19) */
enum { OF_CALL = 0, OF_PUT = 1 };

/* Path dynamics.  GBM = mc::GbmPathGenerator (src/mc/simulation.rs:40-77);
 * HESTON_EULER = mc::HestonPathGenerator full-truncation Euler
 * (src/mc/simulation.rs:80-117, src/models/stochastic.rs:56-71);
 * HESTON_QE = Andersen (2008) quadratic-exponential scheme (no reference
 * counterpart; FP32 Philox mode only). */
enum { OF_MODEL_GBM = 0, OF_MODEL_HESTON_EULER = 1, OF_MODEL_HESTON_QE = 2 };

/* MonteCarloInstrument payoffs (src/engines/monte_carlo/mc_engine.rs:441-584). */
enum { OF_PAYOFF_VANILLA = 0, OF_PAYOFF_BARRIER = 1, OF_PAYOFF_ASIAN = 2 };
enum { OF_BARRIER_UP = 0, OF_BARRIER_DOWN = 1 };
enum { OF_BARRIER_IN = 0, OF_BARRIER_OUT = 1 };
enum { OF_AVG_ARITHMETIC = 0, OF_AVG_GEOMETRIC = 1 };
enum { OF_STRIKE_FIXED = 0, OF_STRIKE_FLOATING = 1 };

/* Control-variate evaluators (ControlVariate, src/mc/simulation.rs:120-124):
 * VANILLA_TERMINAL = vanilla payoff of the terminal spot (mc_engine.rs:458-485),
 * GEOMETRIC_ASIAN  = geometric-average fixed-strike payoff (mc_engine.rs:546-583),
 * TERMINAL_SPOT    = the terminal spot itself (simulation.rs:441-444). */
enum {
  OF_CV_NONE = 0,
  OF_CV_VANILLA_TERMINAL = 1,
  OF_CV_GEOMETRIC_ASIAN = 2,
  OF_CV_TERMINAL_SPOT = 3
};

/* Arithmetic mode of a Monte Carlo run.
 * FP64_REFERENCE: openferric's own draws - one xoshiro256++ stream per sample
 *   seeded with seed + i*7919 (src/math/fast_rng.rs:30-81,181-214), Acklam
 *   inverse CDF (src/math/fast_norm.rs:54-139), FP64 path arithmetic.
 * FP32_PHILOX: counter-based Philox4x32-10 normals, FP32 path state,
 *   compensated FP32 per-thread sums, FP64 cross-thread reduction. */
enum { OF_PREC_FP64_REFERENCE = 0, OF_PREC_FP32_PHILOX = 1 };

/* DividendKind / DividendEvent (src/market/dividends.rs:16-92) */
enum { OF_DIV_CASH = 0, OF_DIV_PROPORTIONAL = 1 };

typedef struct of_dividend_event {
  double time;    /* ex-dividend time in years, > 0 */
  int32_t kind;   /* OF_DIV_CASH: S+ = max(S- - amount, 0); OF_DIV_PROPORTIONAL: S+ = S- (1 - amount) */
  int32_t reserved0;
  double amount;  /* cash amount >= 0, or ratio in [0, 1) */
} of_dividend_event;

typedef struct of_model {
  int32_t kind; /* OF_MODEL_* */
  int32_t reserved0;
  double s0;
  double mu; /* risk-neutral drift r - q */
  double sigma; /* GBM volatility */
  double maturity; /* simulation horizon in years */
  int64_t steps;
  double kappa, theta, xi, rho, v0; /* Heston parameters */
  /* GBM only: a discrete dividend schedule with strictly increasing times
   * (DiscreteDividendGbmPathGenerator, src/engines/monte_carlo/mc_engine.rs:
   * 123-175): after step j every event with time <= maturity + 1e-12 and
   * time <= (j+1) dt + 1e-12 not yet applied jumps the spot.  NULL / 0 = none. */
  const of_dividend_event* dividends;
  int64_t n_dividends;
} of_model;

typedef struct of_payoff {
  int32_t kind; /* OF_PAYOFF_* */
  int32_t option_type; /* OF_CALL / OF_PUT */
  double strike;
  int32_t barrier_direction; /* OF_BARRIER_UP / DOWN */
  int32_t barrier_style; /* OF_BARRIER_IN / OUT */
  double barrier_level;
  double rebate;
  int32_t averaging; /* OF_AVG_* */
  int32_t strike_type; /* OF_STRIKE_* */
  const double* observation_times; /* host array, n_observations entries */
  int64_t n_observations;
  double expiry; /* instrument expiry used to map observation times to steps */
} of_payoff;

typedef struct of_mc_config {
  int64_t num_paths;
  uint64_t seed;
  int32_t antithetic; /* 0/1 */
  int32_t precision; /* OF_PREC_* */
  int32_t control_variate; /* OF_CV_* */
  int32_t tile_ilp; /* FP32 strip tile shape: 0 = default (1), 1 or 2 samples in flight per thread,
                       3 = warp-specialised (half the warps generate the Philox draws into a
                       shared-memory ring, half simulate and price) */
  double cv_expected; /* E[Y] of the control variate, undiscounted */
  double discount_factor;
  /* Test hook (the injection point PathGenerator::generate_from_normals,
   * src/mc/simulation.rs:22): host array of normals laid out
   * [sample][step][stream], streams = 1 for GBM and 2 for Heston.  NULL draws
   * the normals on the device.  FP64_REFERENCE mode only. */
  const double* injected_normals;
  int64_t n_injected;
  /* The reproducible stream kind of FP64_REFERENCE mode (FastRngKind,
   * src/math/fast_rng.rs:20-27): OF_RNG_XOSHIRO256PP (the default) or
   * OF_RNG_PCG64 (PCG XSL-RR 128/64, fast_rng.rs:86-128).  Each sample's
   * stream is seeded with stream_seed(seed, i) either way.  FP32 Philox mode
   * takes OF_RNG_XOSHIRO256PP only (its draws are Philox's). */
  int32_t rng_kind;
  int32_t reserved0;
} of_mc_config;

enum { OF_RNG_XOSHIRO256PP = 0, OF_RNG_PCG64 = 1 };

typedef struct of_mc_result {
  double price;
  double stderr_;
  int64_t samples; /* antithetic pairs count as one sample, as in the reference */
  double sum_x, sum_x2, sum_y, sum_xy, sum_y2; /* the five running sums */
  double kernel_ms; /* device time of the simulation kernels (CUDA events) */
} of_mc_result;

typedef struct of_ctx of_ctx;

/* ---- context ------------------------------------------------------------ */
of_status of_ctx_create(int device, of_ctx** out);
void of_ctx_destroy(of_ctx* ctx);
const char* of_status_str(of_status status);
const char* of_ctx_last_error(const of_ctx* ctx);
/* Runs subsequent work on a caller-owned cudaStream_t (NULL restores the
 * context's own stream).  Lets torch or another runtime order its work with
 * the engine's. */
of_status of_ctx_set_stream(of_ctx* ctx, void* cuda_stream);
of_status of_ctx_get_stream(of_ctx* ctx, void** cuda_stream);
int of_abi_version(void);
int of_device_sm_count(of_ctx* ctx);

/* Throughput of this GPU's FP32 and FP64 pipes and special-function unit
 * (MUFU), measured by three short probe kernels on the context's stream: the
 * denominators of a compute-bound roofline at the clocks of the moment.  No
 * counterpart in the reference.
 *   sfu_ops_per_s: MUFU results per second for the mix that the FP32 Philox
 *     kernels issue (lg2, sqrt, sin, cos), 8 independent chains per thread;
 *   fp32_flops_per_s: FP32 FMA throughput, 2 flops per FMA, 8 independent
 *     chains per thread;
 *   probe_ms: device time of the three probes together;
 *   fp64_flops_per_s: FP64 FMA throughput, 2 flops per FMA, 8 independent
 *     chains per thread. */
typedef struct {
  double sfu_ops_per_s;
  double fp32_flops_per_s;
  double probe_ms;
  double fp64_flops_per_s;
} of_device_peaks;
of_status of_measure_device_peaks(of_ctx* ctx, of_device_peaks* out);

/* ---- generic Monte Carlo run -------------------------------------------- */
/* Replaces mc::MonteCarloEngine::run (src/mc/simulation.rs:182-348) with a
 * built-in payoff in place of the Rust closure; the caller (the Rust
 * PricingEngine impl) has already validated the instrument, resolved the vol
 * and computed cv_expected, as MonteCarloPricingEngine::price does
 * (src/engines/monte_carlo/mc_engine.rs:875-975). */
of_status of_mc_run(of_ctx* ctx, const of_model* model, const of_payoff* payoff,
                    const of_mc_config* cfg, of_mc_result* out);

/* European payoffs on many strikes from ONE shared path set: result[k] is the
 * (price, stderr) of strike k.  The multi-strike form of MonteCarloEngine::run
 * (src/mc/simulation.rs:182-348) for the Heston strike strip; FP32_PHILOX mode
 * (precision field ignored), antithetic supported, no control variate. */
of_status of_mc_strip(of_ctx* ctx, const of_model* model, int32_t option_type,
                      const double* strikes, int64_t n_strikes, const of_mc_config* cfg,
                      of_mc_result* results);

/* Plan form of of_mc_strip: device buffers and a captured CUDA graph are
 * built once; launch enqueues one replay on the context stream without a host
 * sync; results waits for the last replay and reads it back. */
typedef struct of_strip_plan of_strip_plan;
of_status of_strip_plan_create(of_ctx* ctx, const of_model* model, int32_t option_type,
                               const double* strikes, int64_t n_strikes, const of_mc_config* cfg,
                               of_strip_plan** out);
of_status of_strip_plan_launch(of_strip_plan* plan);
of_status of_strip_plan_results(of_strip_plan* plan, of_mc_result* results);
void of_strip_plan_destroy(of_strip_plan* plan);

/* ---- batched book (one persistent launch) ------------------------------- */
/* One option of a book: the model, payoff and variance-reduction settings
 * MonteCarloPricingEngine::price derives per instrument
 * (src/engines/monte_carlo/mc_engine.rs:875-975).  FP32_PHILOX mode. */
typedef struct of_book_entry {
  of_model model;
  of_payoff payoff;
  int64_t num_paths;
  int32_t antithetic;
  int32_t control_variate; /* OF_CV_* */
  double cv_expected;
  double discount_factor;
} of_book_entry;

/* What a book launch computes (of_book_config.mode).
 * OF_BOOK_PRICE:      FP32 prices (the estimator of MonteCarloPricingEngine::price).
 * OF_BOOK_GREEKS:     FP32 prices and pathwise Greeks (delta, vega, rho, theta)
 *                     of GBM options without discrete dividends, the Greeks of
 *                     MonteCarloPricingEngine::price_with_greeks_aad
 *                     (src/engines/monte_carlo/mc_engine.rs:977-987,
 *                     mc_aad.rs:15-219) for every payoff of the book.  Barrier
 *                     options are priced by one-step survival (each step drawn
 *                     on the alive side of the barrier, the path weighted by
 *                     its survival probability), which is unbiased for the
 *                     same discretely monitored price and differentiable; a
 *                     barrier option takes no control variate in this mode.
 * OF_BOOK_PRICE_FP64: the prices of OF_BOOK_GREEKS in FP64 path arithmetic on
 *                     the same draws, for bump-and-revalue checks of the Greeks
 *                     with common random numbers. */
/* OF_BOOK_GREEKS_FP64: the prices and pathwise Greeks of OF_BOOK_GREEKS in
 *                     FP64 path arithmetic on the same draws: the FP32 mode's
 *                     rounding apart, the same estimator. */
enum { OF_BOOK_PRICE = 0, OF_BOOK_GREEKS = 1, OF_BOOK_PRICE_FP64 = 2, OF_BOOK_GREEKS_FP64 = 3 };

typedef struct of_book_config {
  uint64_t seed;
  int32_t block;            /* threads per block, 0 = autotuned */
  int32_t paths_per_thread; /* samples per thread per tile, 0 = autotuned */
  int32_t use_graph;        /* capture the launch in a CUDA graph */
  int32_t mode;             /* OF_BOOK_* */
} of_book_config;

/* Greeks of one book option (openferric core::Greeks, src/core/engine.rs:17-28):
 * d PV / d spot, d PV / d sigma, d PV / d r (with the drift r - q and the
 * discount exp(-r T), r = -ln(discount_factor) / T), theta = -d PV / d T
 * (steps fixed, dt = T / steps).  gamma is 0, as the reference's pathwise AAD
 * returns it.  Each comes with its Monte Carlo standard error. */
typedef struct of_book_greeks {
  double delta, gamma, vega, theta, rho;
  double delta_se, gamma_se, vega_se, theta_se, rho_se;
} of_book_greeks;

/* Prices every entry of a book in one persistent kernel launch: the work is
 * cut into (option, path-block) tiles, longest first, and CTAs pull tiles
 * from a device counter.  Replaces a loop of MonteCarloPricingEngine::price
 * calls (src/engines/monte_carlo/mc_engine.rs:875-975), one per instrument. */
of_status of_mc_price_book(of_ctx* ctx, const of_book_entry* entries, int64_t n,
                           const of_book_config* cfg, of_mc_result* results);

typedef struct of_book_plan of_book_plan;
of_status of_book_plan_create(of_ctx* ctx, const of_book_entry* entries, int64_t n,
                              const of_book_config* cfg, of_book_plan** out);
of_status of_book_plan_launch(of_book_plan* plan);
of_status of_book_plan_results(of_book_plan* plan, of_mc_result* results);
/* Tile shape the plan uses (after autotuning) and its total path-steps. */
of_status of_book_plan_info(of_book_plan* plan, int32_t* block, int32_t* paths_per_thread,
                            int64_t* n_tiles, double* path_steps);
/* Greeks of the plan's last launch (plan created with mode OF_BOOK_GREEKS);
 * waits for the launch like of_book_plan_results. */
of_status of_book_plan_greeks(of_book_plan* plan, of_book_greeks* greeks);
void of_book_plan_destroy(of_book_plan* plan);

/* MonteCarloPricingEngine::price_with_greeks_aad
 * (src/engines/monte_carlo/mc_engine.rs:977-987) for a whole book in one
 * persistent launch: of_mc_price_book in mode OF_BOOK_GREEKS (cfg->mode is
 * ignored).  results[i] and greeks[i] belong to entries[i]. */
of_status of_mc_price_book_greeks(of_ctx* ctx, const of_book_entry* entries, int64_t n, const of_book_config* cfg,
                                  of_mc_result* results, of_book_greeks* greeks);

/* ---- book priced to a standard-error target ----------------------------- */
/* No single reference counterpart: the target is the one the batched-book
 * metric is quoted at (every option at SE <= 1e-4 x spot), reached with
 * MonteCarloPricingEngine::price's estimator (src/engines/monte_carlo/mc_engine.rs:875-975). */
typedef struct of_stderr_target {
  double se_rel;        /* each option's target: stderr <= se_rel x its model.s0 */
  int64_t pilot_paths;  /* paths per option in the first launch */
  int32_t max_rounds;   /* launches at most (1..64) */
  int32_t reserved0;
  double margin;        /* a follow-up launch aims at (stderr / target)^2 x margin x the paths so far;
                           0 = 1.05 */
} of_stderr_target;

/* One launch of of_book_price_to_stderr. */
typedef struct of_stderr_round {
  int64_t options;    /* options priced in this launch */
  int64_t paths;      /* their total paths */
  double path_steps;  /* their total path-steps */
  int64_t converged;  /* of them, how many met their target */
  double kernel_ms;   /* device time of the launch (CUDA events) */
  double wall_ms;     /* host wall clock of the round: planning, uploads, launch and readback */
} of_stderr_round;

/* A pilot launch prices every entry with target->pilot_paths paths
 * (entries[i].num_paths is ignored).  Every option above its target then gets
 * more paths, all in one launch: its total is scaled by (stderr / target)^2 x
 * target->margin (1.05 by default) and the launch runs the difference, rounded
 * up to 256.  This repeats
 * until all meet the target or max_rounds launches have run.
 * Round r draws with seed cfg->seed + r (independent streams), and an option's
 * estimate pools the samples of all its rounds: its running sums are added
 * over the rounds, so the result is that of one run over all those samples
 * (the control-variate coefficient estimated on all of them).  cfg->block and
 * cfg->paths_per_thread of 0 choose a tile shape with at most ~2^18 tiles per
 * launch; cfg->use_graph is ignored.
 * Outputs:
 *   results[i]   = option i's pooled result (sums and samples over its rounds;
 *                  kernel_ms of its last launch);
 *   paths_out[i] = its total paths over its rounds (optional);
 *   rounds[r]    = round r's statistics (optional, capacity max_rounds);
 *   *n_rounds    = the launches run. */
of_status of_book_price_to_stderr(of_ctx* ctx, const of_book_entry* entries, int64_t n, const of_book_config* cfg,
                                  const of_stderr_target* target, of_mc_result* results, int64_t* paths_out,
                                  of_stderr_round* rounds, int32_t* n_rounds);
/* The same in mode OF_BOOK_GREEKS (cfg->mode is ignored): every option priced
 * to its standard-error target with its pathwise Greeks from the same
 * launches (greeks[i] pooled over option i's rounds like its price). */
of_status of_book_price_to_stderr_greeks(of_ctx* ctx, const of_book_entry* entries, int64_t n,
                                         const of_book_config* cfg, const of_stderr_target* target,
                                         of_mc_result* results, of_book_greeks* greeks, int64_t* paths_out,
                                         of_stderr_round* rounds, int32_t* n_rounds);

/* ---- tile-shape autotuner ----------------------------------------------- */
/* The reference has no counterpart (its GPU engine uses one fixed launch
 * shape: WORKGROUP_SIZE 256 and one path per invocation,
 * src/engines/gpu/gpu_mc.rs:19,207).  One candidate tile shape and
 * its measured time. */
typedef struct of_tune_candidate {
  int32_t block;            /* book: threads per block; strip: written as 0 */
  int32_t paths_per_thread; /* book: samples per thread per tile; strip: the tile_ilp shape (1, 2 or 3) */
  double ms;                /* out: median device milliseconds of the timed replays */
} of_tune_candidate;

/* Builds a strip plan for each candidate (cfg->tile_ilp replaced by the
 * candidate's paths_per_thread), replays it once untimed and `reps` times
 * between CUDA events on the context stream, fills each candidate's ms and
 * writes the index of the fastest to *best. */
of_status of_autotune_strip(of_ctx* ctx, const of_model* model, int32_t option_type,
                            const double* strikes, int64_t n_strikes, const of_mc_config* cfg,
                            of_tune_candidate* candidates, int32_t n_candidates, int32_t reps, int32_t* best);
/* The same for the persistent book kernel over (block, paths_per_thread);
 * each candidate's plan is a CUDA graph whatever cfg->use_graph says. */
of_status of_autotune_book(of_ctx* ctx, const of_book_entry* entries, int64_t n, const of_book_config* cfg,
                           of_tune_candidate* candidates, int32_t n_candidates, int32_t reps, int32_t* best);

/* ---- Monte Carlo Greeks on the reference streams (FP64) ----------------- */
typedef struct of_greeks_params {
  int32_t option_type; /* OF_CALL / OF_PUT */
  int32_t antithetic;
  double spot, strike, rate, dividend_yield, vol, expiry;
  int64_t num_paths, num_steps;
  uint64_t seed;
  double spot_bump_rel; /* MonteCarloGreeksEngine gamma bump (>= 1e-6) */
  /* Heston dynamics for of_heston_price_delta_aad (mu = spot drift) */
  double mu, kappa, theta, xi, rho, v0;
} of_greeks_params;

typedef struct of_greeks_result {
  double price, stderr_;
  double delta, gamma, vega, theta, rho;
  double lr_delta, lr_gamma, lr_vega; /* likelihood-ratio estimators */
  int64_t samples;
  double kernel_ms;
} of_greeks_result;

/* Pathwise reverse-mode Greeks of a European vanilla under GBM:
 * mc_european_pathwise_aad (src/engines/monte_carlo/mc_aad.rs:75-219).
 * Fills price, stderr_, delta, vega, theta, rho (gamma = 0). */
of_status of_mc_european_pathwise_aad(of_ctx* ctx, const of_greeks_params* p, of_greeks_result* out);
/* Forward-mode Heston Euler delta: heston_price_delta_aad
 * (src/engines/monte_carlo/mc_aad.rs:280-342).  Fills price (plain mean) and delta. */
of_status of_heston_price_delta_aad(of_ctx* ctx, const of_greeks_params* p, of_greeks_result* out);
/* Terminal-value estimators of MonteCarloGreeksEngine (src/engines/monte_carlo/mc_greeks.rs:95-342):
 * delta/gamma = pathwise, lr_delta/lr_gamma/lr_vega = likelihood ratio. */
of_status of_mc_greek_estimators(of_ctx* ctx, const of_greeks_params* p, of_greeks_result* out);

/* ---- Longstaff-Schwartz (HBM-resident path store) ----------------------- */
enum { OF_EXERCISE_EUROPEAN = 0, OF_EXERCISE_AMERICAN = 1, OF_EXERCISE_BERMUDAN = 2 };

typedef struct of_lsm_contract {
  int32_t option_type; /* OF_CALL / OF_PUT */
  int32_t exercise;    /* OF_EXERCISE_* (ExerciseStyle, src/core/types.rs:41-49) */
  double spot, strike, rate, dividend_yield, vol, expiry;
  int64_t num_steps;
  const double* exercise_dates; /* Bermudan dates in years (host), else NULL */
  int64_t n_exercise_dates;
} of_lsm_contract;

typedef struct of_lsm_config {
  int64_t num_paths;
  uint64_t seed;
  int32_t precision;    /* FP64_REFERENCE: the reference's single xoshiro256++ stream, FP64
                           paths; FP32_PHILOX: Philox normals, FP32 path store */
  int32_t basis_degree; /* 2: {1,S,S^2} + LU (the reference); 3: {1,x,x^2,x^3}, x=S/K, Cholesky */
  int32_t want_delta;   /* also return the pathwise delta under the fitted exercise policy */
  int32_t batch_contracts; /* of_lsm_price: at most this many contracts per date loop (0 = as many
                              as the path-store budget allows) */
  /* Test hook: [contract][path][step] normals replacing the device stream
   * (FP64_REFERENCE only), NULL to draw on the device. */
  const double* injected_normals;
  int64_t n_injected;
} of_lsm_config;

typedef struct of_lsm_result {
  double price, stderr_, delta;
  int64_t regressions; /* exercise dates with >= 3 in-the-money paths */
  double kernel_ms;
} of_lsm_result;

/* LongstaffSchwartzEngine::price(VanillaOption) for a batch of contracts
 * (src/engines/lsm/longstaff_schwartz.rs:421-618): paths in HBM time-major
 * [step][path], per exercise date one fused pass (apply the previous date's
 * exercise, discount, in-the-money basis moments in FP64) whose last block
 * solves the normal equations on the device. */
of_status of_lsm_price(of_ctx* ctx, const of_lsm_contract* contracts, int64_t n,
                       const of_lsm_config* cfg, of_lsm_result* results);

/* ---- Sobol quasi-Monte Carlo --------------------------------------------- */
typedef struct of_qmc_params {
  int32_t option_type; /* OF_CALL / OF_PUT */
  int32_t precision;   /* FP64_REFERENCE: the reference's arithmetic on its point set;
                          FP32_PHILOX: FP32 paths on the same Sobol points */
  double spot, strike, rate;
  double dividend_yield; /* market.effective_dividend_yield(expiry) */
  double vol;            /* market.vol_for(strike, expiry) */
  double expiry;
  int64_t num_paths;     /* Sobol points 1..num_paths, at most 2^40 */
  int64_t num_steps;     /* one Sobol dimension per step, at most 21201 */
  uint64_t seed;
} of_qmc_params;

/* mc_european_qmc_with_seed (src/engines/monte_carlo/mc_qmc.rs:39-150) for a
 * European vanilla under GBM on the reference's SobolSequence
 * (src/math/sobol.rs: canonical dimension 0, hashed direction numbers and an
 * XOR scrambler per further dimension).  The reference's NaN results
 * (no paths, no steps, vol <= 0) are OF_ERR_INVALID_INPUT here; expiry <= 0
 * is the caller's intrinsic shortcut.  `out` gets price, stderr_, samples,
 * sum_x, sum_x2 and kernel_ms. */
of_status of_mc_european_qmc(of_ctx* ctx, const of_qmc_params* params, of_mc_result* out);

/* ---- Bermudan LSM with the exercise boundary ----------------------------- */
/* LsmDynamics (src/engines/lsm/longstaff_schwartz.rs:24-39) */
enum { OF_LSM_GBM = 0, OF_LSM_LOCAL_VOL = 1, OF_LSM_HESTON_EULER = 2 };

typedef struct of_bermudan_contract {
  int32_t option_type; /* OF_CALL / OF_PUT */
  int32_t dynamics;    /* OF_LSM_* */
  double spot, rate, dividend_yield;
  double vol;          /* GBM: market.vol_for(terminal strike, expiry) */
  double expiry;
  int64_t num_steps;
  /* BermudanOption::effective_schedule (src/instruments/bermudan.rs:82-101):
   * strictly increasing times in (0, expiry] and their strikes */
  const double* schedule_times;
  const double* schedule_strikes;
  int64_t n_schedule;
  /* OF_LSM_LOCAL_VOL: the market's sampled surface (SampledVolSurface,
   * src/market/market.rs:52-175), strictly increasing grids, vols row-major
   * [expiry][strike]; a flat vol is a 1 x 1 grid */
  const double* lv_strikes;
  int64_t lv_n_strikes;
  const double* lv_expiries;
  int64_t lv_n_expiries;
  const double* lv_vols;
  /* OF_LSM_HESTON_EULER (with_heston_dynamics, :95-112; drift r - q) */
  double kappa, theta, xi, rho, v0;
} of_bermudan_contract;

/* ExerciseBoundaryPoint (longstaff_schwartz.rs:42-55) */
typedef struct of_boundary_point {
  double time, strike;
  double boundary_spot;  /* NaN when no path exercised (has_boundary = 0) */
  int32_t has_boundary;
  int32_t reserved0;
  int64_t itm_paths, exercised_paths;
} of_boundary_point;

/* LongstaffSchwartzEngine::price_bermudan_with_boundary
 * (src/engines/lsm/longstaff_schwartz.rs:294-417): price, stderr and the
 * exercise boundary (largest exercised spot of a put, smallest of a call)
 * at every scheduled step before expiry plus the terminal point, in
 * chronological order.  FP64 reference mode draws the reference's single
 * xoshiro256++ stream (1 normal per step, 2 for Heston: z1 then z2).
 * `boundary` receives min(capacity, *n_boundary) points; *n_boundary is the
 * full count (at most n_schedule + 1).  want_delta is rejected for local vol. */
of_status of_lsm_bermudan(of_ctx* ctx, const of_bermudan_contract* contract, const of_lsm_config* cfg,
                          of_lsm_result* result, of_boundary_point* boundary, int64_t capacity,
                          int64_t* n_boundary);

/* A European barrier option priced by the LSM engine
 * (LongstaffSchwartzEngine::price(BarrierOption),
 * src/engines/lsm/longstaff_schwartz.rs:632-736). */
typedef struct of_lsm_barrier_contract {
  int32_t option_type;        /* OF_CALL / OF_PUT */
  int32_t barrier_direction;  /* OF_BARRIER_UP / OF_BARRIER_DOWN */
  int32_t barrier_style;      /* OF_BARRIER_IN / OF_BARRIER_OUT */
  int32_t reserved0;
  double spot, strike, rate;
  double dividend_yield;      /* market.effective_dividend_yield(expiry) */
  double vol;                 /* market.vol_for(strike, expiry) */
  double expiry, barrier_level, rebate;
  int64_t num_steps;
} of_lsm_barrier_contract;

/* The LSM engine's European barrier Monte Carlo on its single xoshiro256++
 * stream (FP64_REFERENCE only): path-major draws, log-Euler steps, the barrier
 * monitored on path[0..=steps] (>= up, <= down), the vanilla payoff of the
 * terminal spot when active and the rebate otherwise, discounted by
 * exp(-r T); `result` gets price, stderr_ (mean_and_stderr, :125-140) and
 * kernel_ms.  cfg->injected_normals ([path][step]) replaces the stream. */
of_status of_lsm_barrier(of_ctx* ctx, const of_lsm_barrier_contract* contract, const of_lsm_config* cfg,
                         of_lsm_result* result);

/* xoshiro256++ jump-ahead: the state of the stream seeded with `seed`
 * (Xoshiro256PlusPlus::seed_from_u64, src/math/fast_rng.rs:36-48) after
 * `draws` calls of next_u64, computed on the device by GF(2) matrix powers.
 * Exposed for tests of the LSM reference stream. */
of_status of_xoshiro_jump(of_ctx* ctx, uint64_t seed, const uint64_t* draws, int64_t n, uint64_t* states_out);

/* Test of the bounded mbarrier wait the bulk-copy pipelines use (no
 * reference counterpart).  One block initialises an mbarrier and waits up to
 * `limit_us` microseconds for a phase:
 *   arrive != 0: thread 0 arrives first, so the phase completes and the wait
 *                succeeds;
 *   arrive == 0: nothing arrives, so the wait runs out and gives up.
 * *waited_ok receives 1 if the phase completed and 0 if the wait gave up;
 * *elapsed_us receives the device time the wait took.  The kernel returns
 * either way and the context stays usable. */
of_status of_test_bounded_wait(of_ctx* ctx, int32_t arrive, uint32_t limit_us, int32_t* waited_ok,
                               double* elapsed_us);

/* ---- Heston pathwise adjoint (FP32, checkpointed) ------------------------ */
typedef struct of_heston_adjoint_params {
  double spot, strike, rate, dividend_yield, expiry;
  double kappa, theta, xi, rho, v0;
  int64_t num_paths, num_steps;
  uint64_t seed;
  int32_t option_type;      /* OF_CALL / OF_PUT */
  int32_t payoff;           /* OF_PAYOFF_VANILLA, or OF_PAYOFF_ASIAN: arithmetic average of
                               the spot at every step 1..num_steps */
  int32_t scheme;           /* OF_MODEL_HESTON_QE or OF_MODEL_HESTON_EULER */
  int32_t checkpoint_every; /* path-state checkpoint interval (32) */
  int32_t forward_only;     /* 0: price + adjoint Greeks; 1: price only (FP32); 2: price only
                               in FP64 arithmetic on the same draws (bump-and-revalue with
                               common random numbers: a 1e-4 relative bump is below the FP32
                               resolution of the path state) */
  int32_t reserved0;
  /* Half-width of the band around psi_c = 1.5 in which the QE step blends its
   * quadratic and exponential branches (smoothstep).  0 = Andersen's hard
   * switch, whose jump in v' a pathwise derivative cannot see; > 0 makes the
   * step continuous, so the adjoint Greeks are unbiased for the scheme they
   * differentiate.  At most 0.25. */
  double qe_switch_band;
} of_heston_adjoint_params;

enum {
  OF_ADJ_SPOT = 0, OF_ADJ_RATE = 1, OF_ADJ_V0 = 2, OF_ADJ_KAPPA = 3,
  OF_ADJ_THETA = 4, OF_ADJ_XI = 5, OF_ADJ_RHO = 6, OF_ADJ_COUNT = 7
};

typedef struct of_adjoint_result {
  double price, stderr_;
  double greeks[OF_ADJ_COUNT];        /* d price / d(S0, r, v0, kappa, theta, xi, rho) */
  double greeks_stderr[OF_ADJ_COUNT]; /* Monte Carlo standard error of each */
  int64_t samples;
  double kernel_ms;
} of_adjoint_result;

/* Price and all seven Heston sensitivities from one forward pass (path state
 * checkpointed every `checkpoint_every` steps) and one backward sweep that
 * recomputes each segment and regenerates its counter-based draws.  The
 * reference has forward-mode Heston delta only (heston_price_delta_aad,
 * src/engines/monte_carlo/mc_aad.rs:280-342); the other six have no
 * reference counterpart. */
of_status of_heston_price_adjoint(of_ctx* ctx, const of_heston_adjoint_params* p, of_adjoint_result* out);

/* ---- strike strip without any allocation --------------------------------- */
/* No counterpart in the reference: an addition for callers that cannot
 * allocate device memory at call time.  Examples: a process whose HBM is
 * already reserved in full by another allocator (a framework's caching pool),
 * where a cudaMalloc would fail or fragment that pool; and latency-bound
 * callers that cannot take cudaFree's implicit device-wide synchronisation.
 * It creates no context, stream or event either.
 *
 * Same computation as of_mc_strip (FP32 Philox, one shared path set), with
 * its scratch (strikes, per-block partial sums, final sums) in one static
 * device array of OF_STRIP_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library holds until the process exits.  Limits: at most
 * OF_STRIP_NOALLOC_MAX_STRIKES strikes and OF_STRIP_NOALLOC_MAX_BLOCKS blocks
 * (larger requests are rejected with OF_ERR_INVALID_INPUT and a message).
 *
 * Runs on the calling thread's current device and CUDA context, on
 * `cuda_stream` (NULL = the legacy default stream), and returns when the
 * results are on the host.  The first call in a context (per device, and
 * again after cudaDeviceReset) looks up the array's device address
 * (cudaGetSymbolAddress) with that device current.  Every call synchronises
 * `cuda_stream` and copies through host stack buffers, so it cannot run on a
 * capturing stream: it returns OF_ERR_UNSUPPORTED there, before issuing any
 * work.  The request is validated exactly as of_mc_strip
 * validates it (same statuses and messages), then against the limits below.
 * All calls share the array: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller.  Every call
 * overwrites all of the scratch it reads, so nothing needs clearing between
 * calls.  `err`/`err_len` (may be NULL/0) receive the message of a failure;
 * kernel_ms is not measured (0). */
#define OF_STRIP_NOALLOC_MAX_STRIKES 64
#define OF_STRIP_NOALLOC_MAX_BLOCKS 1024
#define OF_STRIP_NOALLOC_SCRATCH_BYTES                                  \
  (OF_STRIP_NOALLOC_MAX_STRIKES * 4 + (OF_STRIP_NOALLOC_MAX_STRIKES * 2 + 1) * 8 + \
   OF_STRIP_NOALLOC_MAX_BLOCKS * OF_STRIP_NOALLOC_MAX_STRIKES * 2 * 8)
of_status of_mc_strip_noalloc(void* cuda_stream, const of_model* model, int32_t option_type,
                              const double* strikes, int64_t n_strikes, const of_mc_config* cfg,
                              of_mc_result* results, char* err, size_t err_len);

/* ---- the reference's GPU European kernel ---------------------------------- */
/* mc_european_gpu (src/engines/gpu/gpu_mc.rs:322-349, shader
 * src/engines/gpu/mc_shader.wgsl:28-142) on CUDA: f32 GBM paths, xoshiro128++,
 * Box-Muller, 256-wide block reduction, FP64 host sum. */
of_status of_mc_european_gpu(of_ctx* ctx, double spot, double strike, double rate, double vol, double expiry,
                             int64_t num_paths, int64_t num_steps, uint32_t seed, int32_t is_call,
                             double* price, double* stderr_);

#ifdef __cplusplus
}
#endif

#endif /* OF_GPU_H */
