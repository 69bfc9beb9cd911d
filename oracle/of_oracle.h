/*
 * of_oracle.h - CPU restatement of openferric's Monte Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for libofgpu: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 * The product path never links or calls it.
 *
 * Every function restates a reference function (rosssaunders/openferric, Rust,
 * default features, i.e. the scalar non-SIMD paths) and cites the file:line it
 * follows.  Floating-point operations keep the reference's order; `fma` is used
 * exactly where the reference calls `mul_add`, and the file is compiled with
 * -ffp-contract=off so that no other contraction happens.  The reference
 * cannot be built here (no Rust toolchain), so bit-level parity of this
 * restatement is pinned by the reference's own known-answer tests (see
 * tests/test_oracle.py), not by reference outputs.
 */
#ifndef OF_ORACLE_H
#define OF_ORACLE_H

#include <stdint.h>
#include "../include/of_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- math::fast_rng / math::fast_norm ---------------------------------- */
typedef struct orc_xoshiro { uint64_t s[4]; } orc_xoshiro;
void orc_xoshiro_seed(orc_xoshiro* rng, uint64_t seed);
uint64_t orc_xoshiro_next_u64(orc_xoshiro* rng);
double orc_xoshiro_next_f64(orc_xoshiro* rng);
/* Pcg64 (PCG XSL-RR 128/64) of fast_rng.rs:86-128 */
typedef struct orc_pcg64 { unsigned __int128 state, inc; } orc_pcg64;
void orc_pcg64_seed(orc_pcg64* rng, uint64_t seed);
uint64_t orc_pcg64_next_u64(orc_pcg64* rng);
uint64_t orc_stream_seed(uint64_t base_seed, uint64_t stream_index);
double orc_uniform_open01(double u);
double orc_acklam_inv_cdf(double p);
double orc_hart_norm_cdf(double x);
double orc_fast_norm_pdf(double x);

/* Normals exactly as MonteCarloEngine::run draws them: [sample][step][stream]. */
void orc_fill_run_normals(uint64_t seed, int64_t samples, int64_t steps, int streams, double* out);
/* Normals of one sequential stream seeded with `seed` (the LSM draw order). */
void orc_fill_sequential_normals(uint64_t seed, int64_t count, double* out);

/* ---- analytic oracles --------------------------------------------------- */
double orc_bs_price(int option_type, double spot, double strike, double rate, double q, double vol, double expiry);
void orc_bs_greeks(int option_type, double spot, double strike, double rate, double q, double vol, double expiry,
                   double* delta, double* gamma, double* vega, double* theta, double* rho);
double orc_geometric_asian_discrete_fixed(int option_type, double s0, double k, double r, double q, double sigma,
                                          const double* obs, int64_t n_obs);
double orc_heston_call(double s0, double k, double r, double q, double T, double v0, double kappa, double theta,
                       double xi, double rho);
double orc_heston_put(double s0, double k, double r, double q, double T, double v0, double kappa, double theta,
                      double xi, double rho);
double orc_crr_american(int option_type, double s0, double k, double r, double q, double vol, double T, int64_t steps);

/* ---- Monte Carlo ------------------------------------------------------- */
/* MonteCarloEngine::run restated.  threads <= 1 runs the sequential fold in
 * sample order (bit-level reference order); threads > 1 runs an OpenMP fold
 * over contiguous sample chunks combined in chunk order (the Rayon analogue). */
int orc_mc_run(const of_model* model, const of_payoff* payoff, const of_mc_config* cfg, int threads,
               of_mc_result* out);
/* One GBM/Heston path from given normals (PathGenerator::generate_into). */
void orc_generate_path(const of_model* model, const double* z1, const double* z2, double* path);
double orc_payoff_from_path(const of_payoff* payoff, const double* path, int64_t len);

/* Multi-strike European on one shared path set (oracle for of_mc_strip, using the
 * reference draws): returns price/stderr per strike. */
int orc_mc_strip(const of_model* model, int option_type, const double* strikes, int64_t n_strikes,
                 const of_mc_config* cfg, int threads, of_mc_result* out);

/* mc_european_pathwise_aad restated (src/engines/monte_carlo/mc_aad.rs:75-219).
 * out[0]=price out[1]=stderr out[2]=delta out[3]=vega out[4]=theta out[5]=rho */
int orc_gbm_pathwise_aad(int option_type, double strike, double spot, double rate, double q, double vol,
                         double expiry, int64_t num_paths, int64_t num_steps, uint64_t seed, int antithetic,
                         double* out6);
/* heston_price_delta_aad restated (mc_aad.rs:280-342): out[0]=mean price out[1]=mean delta */
int orc_heston_price_delta(int option_type, double strike, double maturity, double spot, double rate, double mu,
                           double kappa, double theta, double xi, double rho, double v0, int64_t num_paths,
                           int64_t num_steps, uint64_t seed, double* out2);
/* MonteCarloGreeksEngine::run_estimators restated (mc_greeks.rs:95-342).
 * out = {pathwise_delta, pathwise_gamma, lr_delta, lr_gamma, lr_vega} */
int orc_mc_greek_estimators(int option_type, double strike, double spot, double rate, double q, double vol,
                            double expiry, int64_t num_paths, uint64_t seed, int antithetic, double spot_bump_rel,
                            double* out5);

/* LongstaffSchwartzEngine::price(VanillaOption) restated
 * (src/engines/lsm/longstaff_schwartz.rs:421-618).
 * exercise: 0 European, 1 American, 2 Bermudan (dates/n_dates).
 * degree 2 = reference basis {1,S,S^2} with partially pivoted LU (nalgebra);
 * degree 3 = basis {1,x,x^2,x^3}, x = S/K, Cholesky (the build's extension).
 * normals: NULL draws one sequential xoshiro stream (the reference order),
 * else [path][step] normals are used.  out[0]=price out[1]=stderr. */
/* LongstaffSchwartzEngine::price(BarrierOption) (longstaff_schwartz.rs:632-736):
 * out2 = {price, stderr}; normals [path][step] replaces the stream if non-null. */
int orc_lsm_barrier(int option_type, double strike, double expiry, int up, int knock_in, double level, double rebate,
                    double spot, double rate, double q, double vol, int64_t num_paths, int64_t num_steps,
                    uint64_t seed, const double* normals, double* out2);

int orc_lsm_price(int option_type, double strike, double expiry, int exercise, const double* dates, int64_t n_dates,
                  double spot, double rate, double q, double vol, int64_t num_paths, int64_t num_steps,
                  uint64_t seed, int degree, const double* normals, double* out2);

/* SobolSequence (src/math/sobol.rs:16-126): direction numbers and scrambler
 * of one dimension; points 1..count in next_into order, row-major [point][dim]. */
void orc_sobol_dimension(uint64_t dim, uint64_t seed, uint64_t* v64, uint64_t* scrambler);
int orc_sobol_points(int64_t dims, uint64_t seed, int64_t count, double* out);

/* mc_european_qmc_with_seed (src/engines/monte_carlo/mc_qmc.rs:39-150) for a
 * European vanilla; q is market.effective_dividend_yield(expiry).
 * out2 = {price, stderr}; NaN, NaN where the reference returns NaN without a stderr. */
int orc_mc_european_qmc(int option_type, double spot, double strike, double rate, double q, double vol,
                        double expiry, int64_t n_paths, int64_t n_steps, uint64_t seed, double* out2);

/* SampledVolSurface::vol (src/market/market.rs:104-174): bilinear lookup on a
 * strictly increasing strike x expiry grid, vols row-major [expiry][strike]. */
double orc_sampled_vol(const double* strikes, int64_t nk, const double* expiries, int64_t nt, const double* vols,
                       double strike, double expiry);

/* LongstaffSchwartzEngine::price_bermudan_with_boundary restated
 * (src/engines/lsm/longstaff_schwartz.rs:294-417; path simulation :190-283).
 * Schedule: n_sched (time, strike) pairs, BermudanOption::effective_schedule.
 * dynamics: 0 GBM (vol), 1 local-vol Euler on the sampled grid lv_*,
 * 2 Heston Euler (kappa..v0, drift r - q).  normals: NULL draws the single
 * sequential xoshiro stream (1 draw per step, 2 for Heston: z1 then z2),
 * else [path][step][draw].  out2 = {price, stderr}; boundary receives
 * n_sched + 1 records at most of {time, strike, boundary_spot (NaN = none),
 * itm_paths, exercised_paths}, chronological; *n_boundary = records. */
int orc_lsm_bermudan(int option_type, double expiry, const double* sched_t, const double* sched_k, int64_t n_sched,
                     int dynamics, double spot, double rate, double q, double vol, const double* lv_strikes,
                     int64_t lv_nk, const double* lv_expiries, int64_t lv_nt, const double* lv_vols, double kappa,
                     double theta, double xi, double rho, double v0, int64_t num_paths, int64_t num_steps,
                     uint64_t seed, int degree, const double* normals, double* out2, double* boundary,
                     int64_t* n_boundary);

/* Reference WGSL kernel math (src/engines/gpu/mc_shader.wgsl:28-142) in C
 * float arithmetic.  Returns the per-workgroup sums the shader writes. */
int orc_wgsl_european(double spot, double strike, double rate, double vol, double expiry, uint32_t num_paths,
                      uint32_t num_steps, uint32_t seed, int is_call, double* price, double* stderr_);

/* Philox4x32-10 (Salmon et al. 2011), the counter-based generator of the
 * FP32 mode; used to check the device generator's streams. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif
