/*
 * of_oracle.c - CPU restatement of openferric's Monte Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for libofgpu, never part of the
 * product path.  Compile with -std=c11 -ffp-contract=off (see oracle/Makefile)
 * so that fma() appears only where the reference calls mul_add.
 * All citations are paths inside rosssaunders/openferric.
 */
#include "of_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPS 2.220446049250313080847263336181640625e-16 /* f64::EPSILON */
#define ORC_PI 3.14159265358979323846264338327950288

/* ------------------------------------------------------------------------ */
/* math::fast_rng (src/math/fast_rng.rs)                                     */
/* ------------------------------------------------------------------------ */

static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* SplitMix64::next_u64, fast_rng.rs:187-199 */
static inline uint64_t splitmix64_next(uint64_t* state) {
  *state += 0x9E3779B97F4A7C15ULL;
  uint64_t z = *state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* Xoshiro256PlusPlus::seed_from_u64, fast_rng.rs:36-48 */
void orc_xoshiro_seed(orc_xoshiro* rng, uint64_t seed) {
  uint64_t sm = seed;
  for (int i = 0; i < 4; ++i) rng->s[i] = splitmix64_next(&sm);
  if ((rng->s[0] | rng->s[1] | rng->s[2] | rng->s[3]) == 0) rng->s[0] = 1;
}

/* Xoshiro256PlusPlus::next_u64, fast_rng.rs:51-67 */
uint64_t orc_xoshiro_next_u64(orc_xoshiro* rng) {
  uint64_t* s = rng->s;
  const uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return result;
}

/* Xoshiro256PlusPlus::next_f64, fast_rng.rs:70-73 */
double orc_xoshiro_next_f64(orc_xoshiro* rng) {
  const uint64_t x = orc_xoshiro_next_u64(rng) >> 11;
  return (double)x * (1.0 / 9007199254740992.0);
}

/* Pcg64::seed_from_u64, fast_rng.rs:92-108: SplitMix64 gives the state's
 * high and low words and the stream; the increment is (stream << 1) | 1; one
 * draw is discarded. */
void orc_pcg64_seed(orc_pcg64* rng, uint64_t seed) {
  uint64_t sm = seed;
  const uint64_t hi = splitmix64_next(&sm), lo = splitmix64_next(&sm), stream = splitmix64_next(&sm);
  rng->inc = ((unsigned __int128)stream << 1) | 1u;
  rng->state = ((unsigned __int128)hi << 64) | lo;
  (void)orc_pcg64_next_u64(rng);
}

/* Pcg64::next_u64, fast_rng.rs:111-121: the 128-bit LCG step with PCG's
 * default multiplier, then the XSL-RR output of the old state. */
uint64_t orc_pcg64_next_u64(orc_pcg64* rng) {
  const unsigned __int128 mul = ((unsigned __int128)0x2360ED051FC65DA4ULL << 64) | 0x4385DF649FCCF645ULL;
  const unsigned __int128 old = rng->state;
  rng->state = old * mul + rng->inc;
  const uint64_t x = (uint64_t)(old >> 64) ^ (uint64_t)old;
  const unsigned rot = (unsigned)(old >> 122);
  return (x >> rot) | (x << ((64u - rot) & 63u));
}

static inline double draw_normal_pcg(orc_pcg64* rng) {
  const double u = (double)(orc_pcg64_next_u64(rng) >> 11) * (1.0 / 9007199254740992.0);
  return orc_acklam_inv_cdf(orc_uniform_open01(u));
}

/* stream_seed, fast_rng.rs:203-205 (wrapping u64 arithmetic) */
uint64_t orc_stream_seed(uint64_t base_seed, uint64_t stream_index) { return base_seed + stream_index * 7919ULL; }

/* uniform_open01, fast_rng.rs:219-221 (f64::clamp) */
double orc_uniform_open01(double u) {
  if (u < ORC_EPS) return ORC_EPS;
  if (u > 1.0 - ORC_EPS) return 1.0 - ORC_EPS;
  return u;
}

/* ------------------------------------------------------------------------ */
/* math::fast_norm (src/math/fast_norm.rs)                                   */
/* ------------------------------------------------------------------------ */

/* fast_norm_pdf, fast_norm.rs:14-19 */
double orc_fast_norm_pdf(double x) { return 0.3989422804014327 * exp((-0.5 * x) * x); }

/* hart_norm_cdf, fast_norm.rs:28-50 */
double orc_hart_norm_cdf(double x) {
  const double P = 0.2316419, A1 = 0.319381530, A2 = -0.356563782, A3 = 1.781477937, A4 = -1.821255978,
               A5 = 1.330274429;
  const double z = fabs(x);
  const double t = 1.0 / fma(P, z, 1.0);
  const double poly = fma(fma(fma(fma(A5, t, A4), t, A3), t, A2), t, A1) * t;
  const double cdf_pos = fma(orc_fast_norm_pdf(z), -poly, 1.0);
  const double sign = signbit(x) ? 1.0 : 0.0;
  return fma(sign, 1.0 - 2.0 * cdf_pos, cdf_pos);
}

/* beasley_springer_moro_inv_cdf (Acklam), fast_norm.rs:54-139 */
double orc_acklam_inv_cdf(double p) {
  static const double A[6] = {-3.969683028665376e1, 2.209460984245205e2, -2.759285104469687e2,
                              1.38357751867269e2,   -3.066479806614716e1, 2.506628277459239};
  static const double B[5] = {-5.447609879822406e1, 1.615858368580409e2, -1.556989798598866e2,
                              6.680131188771972e1,  -1.328068155288572e1};
  static const double C[6] = {-7.784894002430293e-3, -3.223964580411365e-1, -2.400758277161838,
                              -2.549732539343734,    4.374664141464968,     2.938163982698783};
  static const double D[4] = {7.784695709041462e-3, 3.224671290700398e-1, 2.445134137142996, 3.754408661907416};
  const double P_LOW = 0.02425, P_HIGH = 1.0 - 0.02425;
  if (isnan(p) || !(p >= 0.0 && p <= 1.0)) return NAN;
  if (p <= 0.0) return -INFINITY;
  if (p >= 1.0) return INFINITY;
  if (p < P_LOW) {
    const double q = sqrt(-2.0 * log(p));
    return fma(fma(fma(fma(fma(C[0], q, C[1]), q, C[2]), q, C[3]), q, C[4]), q, C[5]) /
           fma(fma(fma(fma(D[0], q, D[1]), q, D[2]), q, D[3]), q, 1.0);
  } else if (p <= P_HIGH) {
    const double q = p - 0.5;
    const double r = q * q;
    return fma(fma(fma(fma(fma(A[0], r, A[1]), r, A[2]), r, A[3]), r, A[4]), r, A[5]) * q /
           fma(fma(fma(fma(fma(B[0], r, B[1]), r, B[2]), r, B[3]), r, B[4]), r, 1.0);
  } else {
    const double q = sqrt(-2.0 * log(1.0 - p));
    return -fma(fma(fma(fma(fma(C[0], q, C[1]), q, C[2]), q, C[3]), q, C[4]), q, C[5]) /
           fma(fma(fma(fma(D[0], q, D[1]), q, D[2]), q, D[3]), q, 1.0);
  }
}

/* sample_standard_normal on a xoshiro stream, fast_rng.rs:224-226 */
static inline double draw_normal(orc_xoshiro* rng) {
  return orc_acklam_inv_cdf(orc_uniform_open01(orc_xoshiro_next_f64(rng)));
}

static inline int model_streams(const of_model* m) { return m->kind == OF_MODEL_GBM ? 1 : 2; }

/* Draw order of MonteCarloEngine::run, simulation.rs:214-225 */
void orc_fill_run_normals(uint64_t seed, int64_t samples, int64_t steps, int streams, double* out) {
  for (int64_t i = 0; i < samples; ++i) {
    orc_xoshiro rng;
    orc_xoshiro_seed(&rng, orc_stream_seed(seed, (uint64_t)i));
    double* o = out + i * steps * streams;
    for (int64_t j = 0; j < steps; ++j) {
      o[j * streams] = draw_normal(&rng);
      if (streams >= 2) o[j * streams + 1] = draw_normal(&rng);
    }
  }
}

void orc_fill_sequential_normals(uint64_t seed, int64_t count, double* out) {
  orc_xoshiro rng;
  orc_xoshiro_seed(&rng, seed);
  for (int64_t i = 0; i < count; ++i) out[i] = draw_normal(&rng);
}

/* ------------------------------------------------------------------------ */
/* Analytic oracles                                                          */
/* ------------------------------------------------------------------------ */

static inline double vanilla_payoff(int option_type, double spot, double strike) {
  /* mc_engine.rs:59-64 (f64::max) */
  const double v = option_type == OF_CALL ? spot - strike : strike - spot;
  return v > 0.0 ? v : 0.0;
}

/* bs_price, src/engines/analytic/black_scholes.rs:62-108 (portable branch) */
double orc_bs_price(int option_type, double spot, double strike, double rate, double q, double vol, double expiry) {
  if (expiry <= 0.0) return vanilla_payoff(option_type, spot, strike);
  const double df_r = exp(-rate * expiry);
  const double df_q = exp(-q * expiry);
  if (vol <= 0.0) {
    const double v = option_type == OF_CALL ? spot * df_q - strike * df_r : strike * df_r - spot * df_q;
    return v > 0.0 ? v : 0.0;
  }
  const double sig_sqrt_t = vol * sqrt(expiry);
  const double d1 = (log(spot / strike) + fma(0.5 * vol, vol, rate - q) * expiry) / sig_sqrt_t;
  const double d2 = d1 - sig_sqrt_t;
  const double nd1 = orc_hart_norm_cdf(d1), nd2 = orc_hart_norm_cdf(d2);
  const double s_df_q = spot * df_q, k_df_r = strike * df_r;
  const double call = fma(s_df_q, nd1, -(k_df_r * nd2));
  return option_type == OF_CALL ? call : call - s_df_q + k_df_r;
}

/* bs_delta/bs_gamma/bs_vega/bs_theta/bs_rho, black_scholes.rs:110-230 */
void orc_bs_greeks(int option_type, double spot, double strike, double rate, double q, double vol, double expiry,
                   double* delta, double* gamma, double* vega, double* theta, double* rho) {
  *delta = *gamma = *vega = *theta = *rho = 0.0;
  if (expiry <= 0.0 || vol <= 0.0 || spot <= 0.0) return;
  const double sqrt_t = sqrt(expiry);
  const double sig_sqrt_t = vol * sqrt_t;
  const double d1 = (log(spot / strike) + fma(0.5 * vol, vol, rate - q) * expiry) / sig_sqrt_t;
  const double d2 = d1 - sig_sqrt_t;
  const double df_q = exp(-q * expiry), df_r = exp(-rate * expiry);
  const double nd1 = orc_hart_norm_cdf(d1), nd2 = orc_hart_norm_cdf(d2);
  const double pdf = orc_fast_norm_pdf(d1);
  *delta = option_type == OF_CALL ? df_q * nd1 : df_q * (nd1 - 1.0);
  *gamma = df_q * pdf / (spot * vol * sqrt_t);
  *vega = spot * df_q * pdf * sqrt_t;
  const double theta_common = -spot * df_q * pdf * vol / (2.0 * sqrt_t);
  if (option_type == OF_CALL) {
    *theta = theta_common + q * spot * df_q * nd1 - rate * strike * df_r * nd2;
    *rho = strike * expiry * df_r * nd2;
  } else {
    *theta = theta_common - q * spot * df_q * (1.0 - nd1) + rate * strike * df_r * (1.0 - nd2);
    *rho = -strike * expiry * df_r * (1.0 - nd2);
  }
}

/* geometric_asian_discrete_fixed_closed_form, src/pricing/asian.rs:86-136 */
double orc_geometric_asian_discrete_fixed(int option_type, double s0, double k, double r, double q, double sigma,
                                          const double* obs, int64_t n_obs) {
  if (n_obs <= 0) return vanilla_payoff(option_type, s0, k);
  double maturity = -INFINITY;
  for (int64_t i = 0; i < n_obs; ++i) maturity = fmax(maturity, obs[i]);
  maturity = fmax(maturity, 0.0);
  if (maturity <= 0.0 || sigma <= 0.0) return exp(-r * maturity) * vanilla_payoff(option_type, s0, k);
  const double n = (double)n_obs;
  double sum_t = 0.0;
  for (int64_t i = 0; i < n_obs; ++i) sum_t += obs[i];
  const double mean_t = sum_t / n;
  double cov_sum = 0.0;
  for (int64_t i = 0; i < n_obs; ++i)
    for (int64_t j = 0; j < n_obs; ++j) cov_sum += fmin(obs[i], obs[j]);
  const double sigma_sq = sigma * sigma;
  const double var = sigma_sq * cov_sum / (n * n);
  const double m = log(s0) + fma(-0.5 * sigma, sigma, r - q) * mean_t;
  const double df = exp(-r * maturity);
  if (var <= 0.0) return df * vanilla_payoff(option_type, exp(m), k);
  const double sqrt_v = sqrt(var);
  const double d1 = (m - log(k) + var) / sqrt_v;
  const double d2 = d1 - sqrt_v;
  const double eg = exp(m + 0.5 * var);
  if (option_type == OF_CALL) return df * (eg * orc_hart_norm_cdf(d1) - k * orc_hart_norm_cdf(d2));
  return df * (k * orc_hart_norm_cdf(-d2) - eg * orc_hart_norm_cdf(-d1));
}

/* Heston semi-analytic price by the Lewis (2000) single-integral formula with
 * the Albrecher et al. ("little trap") characteristic function; the oracle
 * the reference checks with heston_price_fft (src/engines/fft/char_fn.rs:125-154,
 * carr_madan.rs:530-588).  Quadrature: adaptive Simpson on [0, 200] and a
 * mapped tail, FP64. */
typedef struct heston_cf_args {
  double k_log, T, v0, kappa, theta, xi, rho;
} heston_cf_args;

static double lewis_integrand(double u, const heston_cf_args* a) {
  /* phi(w) of X_T = ln(S_T/S0) - (r-q)T at w = u - i/2 */
  const double complex w = u - 0.5 * I;
  const double complex iw = I * w;
  const double complex b = a->kappa - a->rho * a->xi * iw;
  const double complex d = csqrt(b * b + a->xi * a->xi * (iw + w * w));
  const double complex g = (b - d) / (b + d);
  const double complex e = cexp(-d * a->T);
  const double complex Cc =
      a->kappa * a->theta / (a->xi * a->xi) * ((b - d) * a->T - 2.0 * clog((1.0 - g * e) / (1.0 - g)));
  const double complex Dd = (b - d) / (a->xi * a->xi) * (1.0 - e) / (1.0 - g * e);
  const double complex phi = cexp(Cc + Dd * a->v0);
  const double complex val = cexp(I * u * a->k_log) * phi;
  return creal(val) / (u * u + 0.25);
}

static double simpson_rec(const heston_cf_args* a, double lo, double hi, double flo, double fmid, double fhi,
                          double whole, double tol, int depth) {
  const double mid = 0.5 * (lo + hi);
  const double lm = 0.5 * (lo + mid), rm = 0.5 * (mid + hi);
  const double flm = lewis_integrand(lm, a), frm = lewis_integrand(rm, a);
  const double left = (mid - lo) / 6.0 * (flo + 4.0 * flm + fmid);
  const double right = (hi - mid) / 6.0 * (fmid + 4.0 * frm + fhi);
  if (depth <= 0 || fabs(left + right - whole) <= 15.0 * tol)
    return left + right + (left + right - whole) / 15.0;
  return simpson_rec(a, lo, mid, flo, flm, fmid, left, 0.5 * tol, depth - 1) +
         simpson_rec(a, mid, hi, fmid, frm, fhi, right, 0.5 * tol, depth - 1);
}

static double lewis_integral(const heston_cf_args* a) {
  double total = 0.0;
  const double edges[] = {0.0, 1.0, 5.0, 20.0, 60.0, 200.0, 1000.0};
  for (int i = 0; i + 1 < (int)(sizeof(edges) / sizeof(edges[0])); ++i) {
    const double lo = edges[i], hi = edges[i + 1];
    const double flo = lewis_integrand(lo, a), fhi = lewis_integrand(hi, a);
    const double fmid = lewis_integrand(0.5 * (lo + hi), a);
    const double whole = (hi - lo) / 6.0 * (flo + 4.0 * fmid + fhi);
    total += simpson_rec(a, lo, hi, flo, fmid, fhi, whole, 1e-12, 18);
  }
  return total;
}

double orc_heston_call(double s0, double k, double r, double q, double T, double v0, double kappa, double theta,
                       double xi, double rho) {
  heston_cf_args a = {log(s0 / k) + (r - q) * T, T, v0, kappa, theta, xi, rho};
  const double integral = lewis_integral(&a);
  return s0 * exp(-q * T) - sqrt(s0 * k) * exp(-0.5 * (r + q) * T) / ORC_PI * integral;
}

double orc_heston_put(double s0, double k, double r, double q, double T, double v0, double kappa, double theta,
                      double xi, double rho) {
  const double c = orc_heston_call(s0, k, r, q, T, v0, kappa, theta, xi, rho);
  return c - s0 * exp(-q * T) + k * exp(-r * T);
}

/* Cox-Ross-Rubinstein American rollback
 * (src/engines/numerical/american_binomial.rs:58-98 as the reference's tree oracle). */
double orc_crr_american(int option_type, double s0, double k, double r, double q, double vol, double T, int64_t steps) {
  const double dt = T / (double)steps;
  const double u = exp(vol * sqrt(dt)), d = 1.0 / u;
  const double p = (exp((r - q) * dt) - d) / (u - d);
  const double disc = exp(-r * dt);
  double* v = (double*)malloc(sizeof(double) * (size_t)(steps + 1));
  if (!v) return NAN;
  for (int64_t i = 0; i <= steps; ++i) {
    const double s = s0 * pow(u, (double)(steps - i)) * pow(d, (double)i);
    v[i] = vanilla_payoff(option_type, s, k);
  }
  for (int64_t n = steps - 1; n >= 0; --n) {
    for (int64_t i = 0; i <= n; ++i) {
      const double cont = disc * (p * v[i] + (1.0 - p) * v[i + 1]);
      const double s = s0 * pow(u, (double)(n - i)) * pow(d, (double)i);
      const double ex = vanilla_payoff(option_type, s, k);
      v[i] = cont > ex ? cont : ex;
    }
  }
  const double out = v[0];
  free(v);
  return out;
}

/* ------------------------------------------------------------------------ */
/* mc::PathGenerator (src/mc/simulation.rs)                                  */
/* ------------------------------------------------------------------------ */

/* GbmPathGenerator::generate_into, simulation.rs:58-72;
 * HestonPathGenerator::generate_into, simulation.rs:98-117 with
 * Heston::step_euler, src/models/stochastic.rs:56-71 */
void orc_generate_path(const of_model* m, const double* z1, const double* z2, double* path) {
  const double dt = m->maturity / (double)m->steps;
  double s = m->s0;
  path[0] = s;
  if (m->kind == OF_MODEL_GBM) {
    const double sqrt_dt = sqrt(dt);
    const double drift = (m->mu - 0.5 * m->sigma * m->sigma) * dt;
    const double diffusion = m->sigma * sqrt_dt;
    int64_t ev = 0;
    for (int64_t j = 0; j < m->steps; ++j) {
      s *= exp(fma(diffusion, z1[j], drift));
      if (m->n_dividends > 0) {
        /* DiscreteDividendGbmPathGenerator::generate_into, mc_engine.rs:146-170;
         * DividendEvent::apply_jump, market/dividends.rs:76-83 */
        const double t = (double)(j + 1) * dt;
        while (ev < m->n_dividends && m->dividends[ev].time <= m->maturity + 1.0e-12 &&
               m->dividends[ev].time <= t + 1.0e-12) {
          const of_dividend_event* e = &m->dividends[ev];
          if (e->kind == OF_DIV_CASH) {
            const double x = s - e->amount;
            s = x > 0.0 ? x : 0.0;
          } else {
            s = s * (1.0 - e->amount);
          }
          ++ev;
        }
      }
      path[j + 1] = s;
    }
  } else {
    double v = m->v0;
    const double sqrt_dt = sqrt(dt);
    const double rho_c = sqrt(1.0 - m->rho * m->rho);
    for (int64_t j = 0; j < m->steps; ++j) {
      const double v_pos = v > 0.0 ? v : 0.0;
      const double zv = z1[j];
      const double zs = m->rho * z1[j] + rho_c * z2[j];
      double v_next = v + m->kappa * (m->theta - v_pos) * dt + m->xi * sqrt(v_pos) * sqrt_dt * zv;
      v_next = v_next > 0.0 ? v_next : 0.0;
      const double s_next = s * exp((m->mu - 0.5 * v_pos) * dt + sqrt(v_pos) * sqrt_dt * zs);
      s = s_next > 1e-12 ? s_next : 1e-12;
      v = v_next > 0.0 ? v_next : 0.0;
      path[j + 1] = s;
    }
  }
}

/* f64::round then `as usize` (saturating) then min(len-1), mc_engine.rs:100-104 */
static inline int64_t obs_index(double t, double maturity, int64_t len) {
  const double idx = round((t / maturity) * (double)(len - 1));
  int64_t i = (isnan(idx) || idx <= 0.0) ? 0 : (int64_t)idx;
  return i < len - 1 ? i : len - 1;
}

/* average_for_observations, mc_engine.rs:86-121 */
static double average_for_observations(const double* path, int64_t len, double maturity, const double* obs,
                                       int64_t n_obs, int averaging) {
  if (n_obs <= 0 || maturity <= 0.0) return path[len - 1];
  if (averaging == OF_AVG_ARITHMETIC) {
    double sum = -0.0;
    for (int64_t i = 0; i < n_obs; ++i) sum += path[obs_index(obs[i], maturity, len)];
    return sum / (double)n_obs;
  }
  double sum = -0.0;
  for (int64_t i = 0; i < n_obs; ++i) {
    const double s = path[obs_index(obs[i], maturity, len)];
    sum += log(s > 1e-12 ? s : 1e-12);
  }
  return exp(sum / (double)n_obs);
}

/* MonteCarloInstrument::payoff_from_path for Vanilla/Barrier/Asian, mc_engine.rs:453-545 */
double orc_payoff_from_path(const of_payoff* p, const double* path, int64_t len) {
  const double st = path[len - 1];
  switch (p->kind) {
    case OF_PAYOFF_VANILLA:
      return vanilla_payoff(p->option_type, st, p->strike);
    case OF_PAYOFF_BARRIER: {
      int hit = 0; /* path_hits_barrier, mc_engine.rs:79-84 (includes path[0]) */
      for (int64_t i = 0; i < len && !hit; ++i)
        hit = p->barrier_direction == OF_BARRIER_UP ? path[i] >= p->barrier_level : path[i] <= p->barrier_level;
      const int active = p->barrier_style == OF_BARRIER_IN ? hit : !hit;
      return active ? vanilla_payoff(p->option_type, st, p->strike) : p->rebate;
    }
    case OF_PAYOFF_ASIAN: {
      const double avg =
          average_for_observations(path, len, p->expiry, p->observation_times, p->n_observations, p->averaging);
      return p->strike_type == OF_STRIKE_FIXED ? vanilla_payoff(p->option_type, avg, p->strike)
                                               : vanilla_payoff(p->option_type, st, avg);
    }
    default:
      return NAN;
  }
}

/* Control-variate evaluators: mc_engine.rs:481-483 (vanilla), :570-581
 * (geometric Asian), simulation.rs:441-444 (terminal spot). */
static double cv_from_path(const of_payoff* p, int cv_kind, const double* path, int64_t len) {
  switch (cv_kind) {
    case OF_CV_VANILLA_TERMINAL:
      return vanilla_payoff(p->option_type, path[len - 1], p->strike);
    case OF_CV_GEOMETRIC_ASIAN: {
      const double g =
          average_for_observations(path, len, p->expiry, p->observation_times, p->n_observations, OF_AVG_GEOMETRIC);
      return vanilla_payoff(p->option_type, g, p->strike);
    }
    case OF_CV_TERMINAL_SPOT:
      return path[len - 1];
    default:
      return 0.0;
  }
}

typedef struct mc_acc {
  double sx, sx2, sy, sxy, sy2;
  int64_t count;
} mc_acc;

/* One sample of the fold in MonteCarloEngine::run, simulation.rs:212-262.
 * z1/z2/path are per-thread buffers. */
static void mc_sample(const of_model* m, const of_payoff* p, const of_mc_config* c, int64_t i, double* z1,
                      double* z2, double* path, mc_acc* acc) {
  const int64_t steps = m->steps, len = steps + 1;
  const int streams = model_streams(m);
  if (c->injected_normals) {
    const double* inj = c->injected_normals + i * steps * streams;
    for (int64_t j = 0; j < steps; ++j) {
      z1[j] = inj[j * streams];
      if (streams >= 2) z2[j] = inj[j * streams + 1];
    }
  } else if (c->rng_kind == OF_RNG_PCG64) {  /* FastRng::from_seed(Pcg64, stream_seed), simulation.rs:215-216 */
    orc_pcg64 rng;
    orc_pcg64_seed(&rng, orc_stream_seed(c->seed, (uint64_t)i));
    for (int64_t j = 0; j < steps; ++j) {
      z1[j] = draw_normal_pcg(&rng);
      if (streams >= 2) z2[j] = draw_normal_pcg(&rng);
    }
  } else {
    orc_xoshiro rng;
    orc_xoshiro_seed(&rng, orc_stream_seed(c->seed, (uint64_t)i));
    for (int64_t j = 0; j < steps; ++j) {
      z1[j] = draw_normal(&rng);
      if (streams >= 2) z2[j] = draw_normal(&rng);
    }
  }
  orc_generate_path(m, z1, z2, path);
  double x = orc_payoff_from_path(p, path, len);
  double y = c->control_variate != OF_CV_NONE ? cv_from_path(p, c->control_variate, path, len) : 0.0;
  if (c->antithetic) {
    for (int64_t j = 0; j < steps; ++j) {
      z1[j] = -z1[j];
      z2[j] = -z2[j];
    }
    orc_generate_path(m, z1, z2, path);
    const double xa = orc_payoff_from_path(p, path, len);
    const double ya = c->control_variate != OF_CV_NONE ? cv_from_path(p, c->control_variate, path, len) : 0.0;
    x = 0.5 * (x + xa);
    y = 0.5 * (y + ya);
  }
  acc->sx += x;
  acc->sx2 += x * x;
  acc->sy += y;
  acc->sxy += x * y;
  acc->sy2 += y * y;
  acc->count += 1;
}

/* Final statistics, simulation.rs:305-347 */
static void mc_finish(const mc_acc* a, const of_mc_config* c, of_mc_result* out) {
  const double n = (double)a->count;
  const double df = c->discount_factor;
  out->samples = a->count;
  out->sum_x = a->sx;
  out->sum_x2 = a->sx2;
  out->sum_y = a->sy;
  out->sum_xy = a->sxy;
  out->sum_y2 = a->sy2;
  out->kernel_ms = 0.0;
  if (c->control_variate != OF_CV_NONE) {
    const double denom = fmax(n - 1.0, 1.0);
    const double cov_xy = (a->sxy - a->sx * a->sy / n) / denom;
    const double var_y = (a->sy2 - a->sy * a->sy / n) / denom;
    const double beta = var_y > 1e-16 ? cov_xy / var_y : 0.0;
    const double e = c->cv_expected;
    const double sum_adj = a->sx + beta * (n * e - a->sy);
    const double sum_adj_sq = a->sx2 + 2.0 * beta * e * a->sx - 2.0 * beta * a->sxy +
                              beta * beta * (n * e * e - 2.0 * e * a->sy + a->sy2);
    const double mean = sum_adj / n;
    const double var = n > 1.0 ? (sum_adj_sq - sum_adj * sum_adj / n) / (n - 1.0) : 0.0;
    out->price = df * mean;
    out->stderr_ = df * sqrt(var / n);
  } else {
    const double mean = a->sx / n;
    const double var = n > 1.0 ? (a->sx2 - a->sx * a->sx / n) / (n - 1.0) : 0.0;
    out->price = df * mean;
    out->stderr_ = df * sqrt(var / n);
  }
}

int orc_mc_run(const of_model* m, const of_payoff* p, const of_mc_config* c, int threads, of_mc_result* out) {
  if (c->num_paths <= 0 || m->steps <= 0) return OF_ERR_INVALID_INPUT;
  if (c->rng_kind != OF_RNG_XOSHIRO256PP && c->rng_kind != OF_RNG_PCG64) return OF_ERR_INVALID_INPUT;
  const int64_t samples = c->antithetic ? (c->num_paths + 1) / 2 : c->num_paths;
  const int64_t steps = m->steps;
  if (c->injected_normals && c->n_injected < samples * steps * model_streams(m)) return OF_ERR_INVALID_INPUT;
  mc_acc total = {0, 0, 0, 0, 0, 0};
  if (threads <= 1) {
    double* buf = (double*)malloc(sizeof(double) * (size_t)(3 * steps + 1));
    if (!buf) return OF_ERR_ALLOC;
    for (int64_t i = 0; i < samples; ++i) mc_sample(m, p, c, i, buf, buf + steps, buf + 2 * steps, &total);
    free(buf);
  } else {
#ifdef _OPENMP
    mc_acc* parts = (mc_acc*)calloc((size_t)threads, sizeof(mc_acc));
    if (!parts) return OF_ERR_ALLOC;
#pragma omp parallel num_threads(threads)
    {
      const int tid = omp_get_thread_num();
      const int nt = omp_get_num_threads();
      const int64_t lo = samples * tid / nt, hi = samples * (tid + 1) / nt;
      double* buf = (double*)malloc(sizeof(double) * (size_t)(3 * steps + 1));
      mc_acc a = {0, 0, 0, 0, 0, 0};
      if (buf)
        for (int64_t i = lo; i < hi; ++i) mc_sample(m, p, c, i, buf, buf + steps, buf + 2 * steps, &a);
      free(buf);
      parts[tid] = a;
    }
    for (int t = 0; t < threads; ++t) {
      total.sx += parts[t].sx;
      total.sx2 += parts[t].sx2;
      total.sy += parts[t].sy;
      total.sxy += parts[t].sxy;
      total.sy2 += parts[t].sy2;
      total.count += parts[t].count;
    }
    free(parts);
    if (total.count != samples) return OF_ERR_ALLOC;
#else
    return orc_mc_run(m, p, c, 1, out);
#endif
  }
  mc_finish(&total, c, out);
  return OF_OK;
}

/* Shared path set, many European strikes: the reference draws per sample,
 * one payoff per strike (antithetic pair-averaged as in run). */
int orc_mc_strip(const of_model* m, int option_type, const double* strikes, int64_t n_strikes,
                 const of_mc_config* c, int threads, of_mc_result* out) {
  if (c->num_paths <= 0 || m->steps <= 0 || n_strikes <= 0) return OF_ERR_INVALID_INPUT;
  const int64_t samples = c->antithetic ? (c->num_paths + 1) / 2 : c->num_paths;
  const int64_t steps = m->steps;
  const int streams = model_streams(m);
  if (threads < 1) threads = 1;
  double* parts = (double*)calloc((size_t)(threads * n_strikes * 2), sizeof(double));
  if (!parts) return OF_ERR_ALLOC;
#ifdef _OPENMP
#pragma omp parallel num_threads(threads)
#endif
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num(), nt = omp_get_num_threads();
#else
    const int tid = 0, nt = 1;
#endif
    const int64_t lo = samples * tid / nt, hi = samples * (tid + 1) / nt;
    double* z1 = (double*)malloc(sizeof(double) * (size_t)(3 * steps + 1));
    double* acc = parts + (size_t)tid * n_strikes * 2;
    if (z1) {
      double* z2 = z1 + steps;
      double* path = z1 + 2 * steps;
      for (int64_t i = lo; i < hi; ++i) {
        orc_xoshiro rng;
        orc_xoshiro_seed(&rng, orc_stream_seed(c->seed, (uint64_t)i));
        for (int64_t j = 0; j < steps; ++j) {
          z1[j] = draw_normal(&rng);
          if (streams >= 2) z2[j] = draw_normal(&rng);
        }
        orc_generate_path(m, z1, z2, path);
        const double st = path[steps];
        double sta = 0.0;
        if (c->antithetic) {
          for (int64_t j = 0; j < steps; ++j) {
            z1[j] = -z1[j];
            z2[j] = -z2[j];
          }
          orc_generate_path(m, z1, z2, path);
          sta = path[steps];
        }
        for (int64_t k = 0; k < n_strikes; ++k) {
          double x = vanilla_payoff(option_type, st, strikes[k]);
          if (c->antithetic) x = 0.5 * (x + vanilla_payoff(option_type, sta, strikes[k]));
          acc[2 * k] += x;
          acc[2 * k + 1] += x * x;
        }
      }
      free(z1);
    }
  }
  for (int64_t k = 0; k < n_strikes; ++k) {
    mc_acc a = {0, 0, 0, 0, 0, samples};
    for (int t = 0; t < threads; ++t) {
      a.sx += parts[(size_t)t * n_strikes * 2 + 2 * k];
      a.sx2 += parts[(size_t)t * n_strikes * 2 + 2 * k + 1];
    }
    of_mc_config cc = *c;
    cc.control_variate = OF_CV_NONE;
    mc_finish(&a, &cc, &out[k]);
  }
  free(parts);
  return OF_OK;
}

/* ------------------------------------------------------------------------ */
/* mc_aad (src/engines/monte_carlo/mc_aad.rs)                               */
/* ------------------------------------------------------------------------ */

/* gbm_single_path_reverse, mc_aad.rs:15-72: the tape records
 * dt=t/steps, sqrt_dt, sigma^2, drift=(r-q-0.5 sigma^2) dt, diffusion=sigma sqrt_dt,
 * then per step expo = drift + diffusion*z (mul then add), s = s*exp(expo),
 * pv = exp(-r t) max(+-(s-k),0).  The reverse sweep below visits the same
 * nodes in reverse creation order. grads = d pv / d(s0, r, sigma, t). */
static double gbm_path_reverse(int option_type, double strike, double spot, double rate, double q, double vol,
                               double expiry, const double* z, int64_t steps, double* growth, double grads[4]) {
  const double dt = expiry / (double)steps;
  const double sqrt_dt = sqrt(dt);
  const double sigma_sq = vol * vol;
  const double half_sigma_sq = 0.5 * sigma_sq;
  const double r_minus_q = rate - q;
  const double drift_inner = r_minus_q - half_sigma_sq;
  const double drift = drift_inner * dt;
  const double diffusion = vol * sqrt_dt;
  double s = spot;
  for (int64_t j = 0; j < steps; ++j) {
    const double expo = drift + diffusion * z[j];
    growth[j] = exp(expo);
    s = s * growth[j];
  }
  const double intrinsic = option_type == OF_CALL ? s - strike : strike - s;
  const double payoff = intrinsic > 0.0 ? intrinsic : 0.0;
  const double rt = rate * expiry;
  const double discount = exp(-rt);
  const double pv = discount * payoff;
  /* reverse sweep */
  double r_bar = 0.0, t_bar = 0.0, sigma_bar = 0.0, dt_bar = 0.0;
  const double discount_bar = payoff, payoff_bar = discount;
  const double rt_bar = -(discount_bar * discount);
  r_bar += rt_bar * expiry;
  t_bar += rt_bar * rate;
  const double intrinsic_bar = intrinsic > 0.0 ? payoff_bar : 0.0;
  double s_bar = option_type == OF_CALL ? intrinsic_bar : -intrinsic_bar;
  double drift_bar = 0.0, diffusion_bar = 0.0;
  /* the tape stores every intermediate s_j; recompute them forward */
  double* sv = growth + steps; /* caller provides 2*steps+1 */
  sv[0] = spot;
  for (int64_t j = 0; j < steps; ++j) sv[j + 1] = sv[j] * growth[j];
  for (int64_t j = steps - 1; j >= 0; --j) {
    const double growth_bar = s_bar * sv[j];
    s_bar = s_bar * growth[j];
    const double expo_bar = growth_bar * growth[j];
    drift_bar += expo_bar;
    diffusion_bar += expo_bar * z[j];
  }
  sigma_bar += diffusion_bar * sqrt_dt;
  const double sqrt_dt_bar = diffusion_bar * vol;
  const double drift_inner_bar = drift_bar * dt;
  dt_bar += drift_bar * drift_inner;
  r_bar += drift_inner_bar;
  const double half_bar = -drift_inner_bar;
  const double sigma_sq_bar = 0.5 * half_bar;
  sigma_bar += sigma_sq_bar * vol;
  sigma_bar += sigma_sq_bar * vol;
  dt_bar += sqrt_dt_bar * (0.5 / sqrt_dt);
  t_bar += dt_bar / (double)steps;
  grads[0] = s_bar;
  grads[1] = r_bar;
  grads[2] = sigma_bar;
  grads[3] = t_bar;
  return pv;
}

/* mc_european_pathwise_aad, mc_aad.rs:75-219 */
int orc_gbm_pathwise_aad(int option_type, double strike, double spot, double rate, double q, double vol,
                         double expiry, int64_t num_paths, int64_t num_steps, uint64_t seed, int antithetic,
                         double* out) {
  if (num_paths <= 0 || num_steps <= 0) return OF_ERR_INVALID_INPUT;
  const int64_t samples = antithetic ? (num_paths + 1) / 2 : num_paths;
  double* z = (double*)malloc(sizeof(double) * (size_t)(num_steps * 3 + 2));
  if (!z) return OF_ERR_ALLOC;
  double* work = z + num_steps;
  double sum = 0.0, sum_sq = 0.0, g_sum[4] = {0, 0, 0, 0};
  for (int64_t i = 0; i < samples; ++i) {
    orc_xoshiro rng;
    orc_xoshiro_seed(&rng, orc_stream_seed(seed, (uint64_t)i));
    for (int64_t j = 0; j < num_steps; ++j) z[j] = draw_normal(&rng);
    double g0[4], g1[4], pv;
    const double pv0 = gbm_path_reverse(option_type, strike, spot, rate, q, vol, expiry, z, num_steps, work, g0);
    if (antithetic) {
      for (int64_t j = 0; j < num_steps; ++j) z[j] = -z[j];
      const double pv1 = gbm_path_reverse(option_type, strike, spot, rate, q, vol, expiry, z, num_steps, work, g1);
      for (int k = 0; k < 4; ++k) g0[k] = 0.5 * (g0[k] + g1[k]);
      pv = 0.5 * (pv0 + pv1);
    } else {
      pv = pv0;
    }
    sum += pv;
    sum_sq += pv * pv;
    for (int k = 0; k < 4; ++k) g_sum[k] += g0[k];
  }
  free(z);
  const double n = (double)samples;
  const double mean = sum / n;
  const double var = samples > 1 ? (sum_sq - sum * sum / n) / (n - 1.0) : 0.0;
  out[0] = mean;
  out[1] = sqrt(var / n);
  out[2] = g_sum[0] / n;
  out[3] = g_sum[2] / n;
  out[4] = -(g_sum[3] / n);
  out[5] = g_sum[1] / n;
  return OF_OK;
}

/* heston_single_path_price_delta + heston_price_delta_aad, mc_aad.rs:239-342 */
int orc_heston_price_delta(int option_type, double strike, double maturity, double spot, double rate, double mu,
                           double kappa, double theta, double xi, double rho, double v0, int64_t num_paths,
                           int64_t num_steps, uint64_t seed, double* out) {
  if (num_paths <= 0 || num_steps <= 0) return OF_ERR_INVALID_INPUT;
  double* z1 = (double*)malloc(sizeof(double) * (size_t)(2 * num_steps));
  if (!z1) return OF_ERR_ALLOC;
  double* z2 = z1 + num_steps;
  double sum_price = 0.0, sum_delta = 0.0;
  const double dt = maturity / (double)num_steps;
  const double sqrt_dt = sqrt(dt);
  const double rho2 = sqrt(1.0 - rho * rho);
  const double discount = exp(-rate * maturity);
  for (int64_t i = 0; i < num_paths; ++i) {
    orc_xoshiro rng;
    orc_xoshiro_seed(&rng, orc_stream_seed(seed, (uint64_t)i));
    for (int64_t j = 0; j < num_steps; ++j) {
      z1[j] = draw_normal(&rng);
      z2[j] = draw_normal(&rng);
    }
    double s = spot, ds = 1.0, v = v0;
    for (int64_t j = 0; j < num_steps; ++j) {
      const double v_pos = v > 0.0 ? v : 0.0;
      const double sqrt_v = sqrt(v_pos);
      const double zs = rho * z1[j] + rho2 * z2[j];
      double v_next = v + kappa * (theta - v_pos) * dt + xi * sqrt_v * sqrt_dt * z1[j];
      v_next = v_next > 0.0 ? v_next : 0.0;
      const double growth = exp((mu - 0.5 * v_pos) * dt + sqrt_v * sqrt_dt * zs);
      s = s * growth;
      ds = ds * growth;
      v = v_next;
    }
    double pv, dpv;
    if (option_type == OF_CALL) {
      const double val = s - strike;
      pv = val > 0.0 ? val : 0.0;
      dpv = val > 0.0 ? ds : 0.0;
    } else {
      const double val = strike - s;
      pv = val > 0.0 ? val : 0.0;
      dpv = val > 0.0 ? -ds : 0.0;
    }
    sum_price += pv * discount;
    sum_delta += dpv * discount;
  }
  free(z1);
  out[0] = sum_price / (double)num_paths;
  out[1] = sum_delta / (double)num_paths;
  return OF_OK;
}

/* single_path_contribution, mc_greeks.rs:266-314 */
static void greek_contrib(int option_type, double z, double spot, double strike, double spot_up, double spot_dn,
                          double spot_span, double vol, double maturity, double drift, double sig_sqrt_t,
                          double o[5]) {
  const double growth = exp(fma(sig_sqrt_t, z, drift));
  const double st = spot * growth;
  const double payoff = vanilla_payoff(option_type, st, strike);
#define PW_DELTA(ST) \
  (option_type == OF_CALL ? ((ST) > strike ? growth : 0.0) : ((ST) < strike ? -growth : 0.0))
  const double delta_pw = PW_DELTA(st);
  const double delta_up = PW_DELTA(spot_up * growth);
  const double delta_dn = PW_DELTA(spot_dn * growth);
#undef PW_DELTA
  const double gamma_pw = (delta_up - delta_dn) / spot_span;
  const double sqrt_t = sqrt(maturity);
  const double inv_svt = 1.0 / (spot * vol * sqrt_t);
  const double z2m1 = z * z - 1.0;
  const double w_delta = z * inv_svt;
  const double inv2 = inv_svt * inv_svt;
  const double w_gamma = z2m1 * inv2 - z * inv_svt / spot;
  const double w_vega = (z2m1 - vol * sqrt_t * z) / vol;
  o[0] = delta_pw;
  o[1] = gamma_pw;
  o[2] = payoff * w_delta;
  o[3] = payoff * w_gamma;
  o[4] = payoff * w_vega;
}

/* MonteCarloGreeksEngine::run_estimators, mc_greeks.rs:113-241 */
int orc_mc_greek_estimators(int option_type, double strike, double spot, double rate, double q, double vol,
                            double expiry, int64_t num_paths, uint64_t seed, int antithetic, double spot_bump_rel,
                            double* out) {
  for (int k = 0; k < 5; ++k) out[k] = 0.0;
  if (num_paths <= 0) return OF_ERR_INVALID_INPUT;
  if (expiry <= 0.0) return OF_OK;
  const double drift = (rate - q - 0.5 * vol * vol) * expiry;
  const double sig_sqrt_t = vol * sqrt(expiry);
  const double discount = exp(-rate * expiry);
  const double h = fmax(spot * spot_bump_rel, 1.0e-6);
  const double spot_up = spot + h;
  const double spot_dn = fmax(spot - h, 1.0e-8);
  const double spot_span = spot_up - spot_dn;
  const int64_t samples = antithetic ? (num_paths + 1) / 2 : num_paths;
  double sums[5] = {0, 0, 0, 0, 0};
  for (int64_t i = 0; i < samples; ++i) {
    orc_xoshiro rng;
    orc_xoshiro_seed(&rng, orc_stream_seed(seed, (uint64_t)i));
    const double z = draw_normal(&rng);
    double b[5], a[5];
    greek_contrib(option_type, z, spot, strike, spot_up, spot_dn, spot_span, vol, expiry, drift, sig_sqrt_t, b);
    if (antithetic) {
      greek_contrib(option_type, -z, spot, strike, spot_up, spot_dn, spot_span, vol, expiry, drift, sig_sqrt_t, a);
      for (int k = 0; k < 5; ++k) b[k] = 0.5 * (b[k] + a[k]);
    }
    for (int k = 0; k < 5; ++k) sums[k] += b[k];
  }
  const double n = (double)samples;
  for (int k = 0; k < 5; ++k) out[k] = discount * sums[k] / n;
  return OF_OK;
}

/* ------------------------------------------------------------------------ */
/* Longstaff-Schwartz (src/engines/lsm/longstaff_schwartz.rs)                */
/* ------------------------------------------------------------------------ */

/* nalgebra Matrix3::lu().solve(): Gaussian elimination with partial (row)
 * pivoting; None (-> zero beta, longstaff_schwartz.rs:592) when U has a zero
 * diagonal entry. */
static int lu_solve3(double a[3][3], double b[3], double x[3]) {
  int perm[3] = {0, 1, 2};
  for (int i = 0; i < 3; ++i) {
    int piv = i;
    double best = fabs(a[i][i]);
    for (int k = i + 1; k < 3; ++k)
      if (fabs(a[k][i]) > best) {
        best = fabs(a[k][i]);
        piv = k;
      }
    if (best == 0.0) continue;
    if (piv != i) {
      for (int j = 0; j < 3; ++j) {
        const double t = a[i][j];
        a[i][j] = a[piv][j];
        a[piv][j] = t;
      }
      const int tp = perm[i];
      perm[i] = perm[piv];
      perm[piv] = tp;
      const double tb = b[i];
      b[i] = b[piv];
      b[piv] = tb;
    }
    for (int k = i + 1; k < 3; ++k) {
      const double f = a[k][i] / a[i][i];
      a[k][i] = f;
      for (int j = i + 1; j < 3; ++j) a[k][j] -= f * a[i][j];
      b[k] -= f * b[i];
    }
  }
  for (int i = 0; i < 3; ++i)
    if (a[i][i] == 0.0) return 0;
  for (int i = 2; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < 3; ++j) s -= a[i][j] * x[j];
    x[i] = s / a[i][i];
  }
  (void)perm;
  return 1;
}

/* Cholesky solve of the 4x4 normal equations (degree-3 basis in x = S/K). */
static int chol_solve4(double a[4][4], const double b[4], double x[4]) {
  double l[4][4] = {{0}};
  for (int i = 0; i < 4; ++i) {
    for (int j = 0; j <= i; ++j) {
      double s = a[i][j];
      for (int k = 0; k < j; ++k) s -= l[i][k] * l[j][k];
      if (i == j) {
        if (!(s > 0.0)) return 0;
        l[i][i] = sqrt(s);
      } else {
        l[i][j] = s / l[j][j];
      }
    }
  }
  double y[4];
  for (int i = 0; i < 4; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= l[i][k] * y[k];
    y[i] = s / l[i][i];
  }
  for (int i = 3; i >= 0; --i) {
    double s = y[i];
    for (int k = i + 1; k < 4; ++k) s -= l[k][i] * x[k];
    x[i] = s / l[i][i];
  }
  return 1;
}

/* LongstaffSchwartzEngine::price(BarrierOption), src/engines/lsm/longstaff_schwartz.rs:632-736
 * (the portable branch, :691-697): ONE xoshiro256++ stream seeded with `seed`
 * feeds all paths in path-major order; path[0] = spot and
 * path[t+1] = path[t] * exp(mul_add(step_vol, z, drift)) with the Acklam normal
 * of uniform_open01(next_f64); the barrier is monitored on path[0..=steps]
 * (path_hits_barrier, :115-123: >= for up, <= for down); an active path pays
 * the vanilla intrinsic of path[steps], an inactive one the rebate; each
 * value is discounted by exp(-r T) and mean_and_stderr (:125-140) gives the
 * result.  `normals` ([path][step], optional) replaces the stream.
 * out2 = {price, stderr}. */
int orc_lsm_barrier(int option_type, double strike, double expiry, int up, int knock_in, double level, double rebate,
                    double spot, double rate, double q, double vol, int64_t num_paths, int64_t num_steps,
                    uint64_t seed, const double* normals, double* out2) {
  if (num_steps <= 0 || num_paths <= 0) return OF_ERR_INVALID_INPUT;
  const double dt = expiry / (double)num_steps;
  const double drift = (rate - q - 0.5 * vol * vol) * dt;
  const double step_vol = vol * sqrt(dt);
  const double discount = exp(-rate * expiry);
  orc_xoshiro rng;
  orc_xoshiro_seed(&rng, seed);
  double sum = 0.0, sum_sq = 0.0;
  for (int64_t pi = 0; pi < num_paths; ++pi) {
    double s = spot;
    int hit = up ? s >= level : s <= level;
    for (int64_t ti = 0; ti < num_steps; ++ti) {
      const double z = normals ? normals[pi * num_steps + ti] : draw_normal(&rng);
      s = s * exp(fma(step_vol, z, drift));
      hit |= up ? s >= level : s <= level;
    }
    const int active = knock_in ? hit : !hit;
    const double v = discount * (active ? vanilla_payoff(option_type, s, strike) : rebate);
    sum += v;
    sum_sq += v * v;
  }
  const double n = (double)num_paths;
  const double mean = sum / n;
  const double var = num_paths > 1 ? (sum_sq - sum * sum / n) / (n - 1.0) : 0.0;
  out2[0] = mean;
  out2[1] = sqrt(var / n);
  return OF_OK;
}

int orc_lsm_price(int option_type, double strike, double expiry, int exercise, const double* dates, int64_t n_dates,
                  double spot, double rate, double q, double vol, int64_t num_paths, int64_t num_steps,
                  uint64_t seed, int degree, const double* normals, double* out) {
  if (num_steps < 2 || num_paths < 3) return OF_ERR_INVALID_INPUT;
  if (degree != 2 && degree != 3) return OF_ERR_INVALID_INPUT;
  if (expiry == 0.0) {
    out[0] = vanilla_payoff(option_type, spot, strike);
    out[1] = 0.0;
    return OF_OK;
  }
  const double dt = expiry / (double)num_steps;
  const double drift = (rate - q - 0.5 * vol * vol) * dt;
  const double step_vol = vol * sqrt(dt);
  const double disc = exp(-rate * dt);
  const int64_t stride = (num_steps + 1 + 7) & ~(int64_t)7;
  double* paths = (double*)malloc(sizeof(double) * (size_t)(num_paths * stride));
  double* values = (double*)malloc(sizeof(double) * (size_t)num_paths);
  int64_t* itm = (int64_t*)malloc(sizeof(int64_t) * (size_t)num_paths);
  unsigned char* can_ex = (unsigned char*)calloc((size_t)(num_steps + 1), 1);
  if (!paths || !values || !itm || !can_ex) {
    free(paths);
    free(values);
    free(itm);
    free(can_ex);
    return OF_ERR_ALLOC;
  }
  orc_xoshiro rng;
  orc_xoshiro_seed(&rng, seed);
  for (int64_t pi = 0; pi < num_paths; ++pi) {
    double* row = paths + pi * stride;
    row[0] = spot;
    for (int64_t ti = 1; ti <= num_steps; ++ti) {
      const double z = normals ? normals[pi * num_steps + (ti - 1)] : draw_normal(&rng);
      row[ti] = row[ti - 1] * exp(fma(step_vol, z, drift));
    }
  }
  for (int64_t pi = 0; pi < num_paths; ++pi)
    values[pi] = vanilla_payoff(option_type, paths[pi * stride + num_steps], strike);
  /* ExerciseStyle -> can_exercise, longstaff_schwartz.rs:522-540 */
  if (exercise == 0) {
    can_ex[num_steps] = 1;
  } else if (exercise == 1) {
    for (int64_t t = 1; t <= num_steps; ++t) can_ex[t] = 1;
  } else {
    for (int64_t d = 0; d < n_dates; ++d) {
      const double idx = round((dates[d] / expiry) * (double)num_steps);
      int64_t i = (isnan(idx) || idx <= 0.0) ? 0 : (int64_t)idx;
      can_ex[i < num_steps ? i : num_steps] = 1;
    }
    can_ex[num_steps] = 1;
  }
  for (int64_t ti = num_steps - 1; ti >= 1; --ti) {
    for (int64_t pi = 0; pi < num_paths; ++pi) values[pi] *= disc;
    if (!can_ex[ti]) continue;
    int64_t n_itm = 0;
    for (int64_t pi = 0; pi < num_paths; ++pi)
      if (vanilla_payoff(option_type, paths[pi * stride + ti], strike) > 0.0) itm[n_itm++] = pi;
    if (n_itm < 3) continue;
    double beta[4] = {0, 0, 0, 0};
    if (degree == 2) {
      double s1 = 0, s_s = 0, s_s2 = 0, s_s3 = 0, s_s4 = 0, s_y = 0, s_sy = 0, s_s2y = 0;
      for (int64_t k = 0; k < n_itm; ++k) {
        const double s = paths[itm[k] * stride + ti];
        const double s2 = s * s;
        const double y = values[itm[k]];
        s1 += 1.0;
        s_s += s;
        s_s2 += s2;
        s_s3 += s2 * s;
        s_s4 += s2 * s2;
        s_y += y;
        s_sy += s * y;
        s_s2y += s2 * y;
      }
      double a[3][3] = {{s1, s_s, s_s2}, {s_s, s_s2, s_s3}, {s_s2, s_s3, s_s4}};
      double b[3] = {s_y, s_sy, s_s2y};
      double x[3];
      if (lu_solve3(a, b, x)) {
        beta[0] = x[0];
        beta[1] = x[1];
        beta[2] = x[2];
      }
      for (int64_t k = 0; k < n_itm; ++k) {
        const double s = paths[itm[k] * stride + ti];
        const double cont = beta[0] + beta[1] * s + beta[2] * s * s;
        const double ex = vanilla_payoff(option_type, s, strike);
        if (ex > cont) values[itm[k]] = ex;
      }
    } else {
      double m[7] = {0, 0, 0, 0, 0, 0, 0}, r[4] = {0, 0, 0, 0};
      const double inv_k = 1.0 / strike;
      for (int64_t k = 0; k < n_itm; ++k) {
        const double x = paths[itm[k] * stride + ti] * inv_k;
        const double y = values[itm[k]];
        double p = 1.0;
        for (int e = 0; e < 7; ++e) {
          m[e] += p;
          if (e < 4) r[e] += p * y;
          p *= x;
        }
      }
      double a[4][4];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) a[i][j] = m[i + j];
      double x4[4];
      if (chol_solve4(a, r, x4))
        for (int i = 0; i < 4; ++i) beta[i] = x4[i];
      for (int64_t k = 0; k < n_itm; ++k) {
        const double s = paths[itm[k] * stride + ti];
        const double x = s * inv_k;
        const double cont = beta[0] + x * (beta[1] + x * (beta[2] + x * beta[3]));
        const double ex = vanilla_payoff(option_type, s, strike);
        if (ex > cont) values[itm[k]] = ex;
      }
    }
  }
  double sum = 0.0, sum_sq = 0.0;
  for (int64_t pi = 0; pi < num_paths; ++pi) {
    const double v = values[pi] * disc;
    sum += v;
    sum_sq += v * v;
  }
  const double n = (double)num_paths;
  const double mean = sum / n;
  const double var = num_paths > 1 ? (sum_sq - sum * sum / n) / (n - 1.0) : 0.0;
  out[0] = mean;
  out[1] = sqrt(var / n);
  free(paths);
  free(values);
  free(itm);
  free(can_ex);
  return OF_OK;
}

/* ------------------------------------------------------------------------ */
/* Sobol QMC (src/math/sobol.rs, src/engines/monte_carlo/mc_qmc.rs)          */
/* ------------------------------------------------------------------------ */

/* splitmix64 of sobol.rs:121-126 (a pure function of x) */
static inline uint64_t sobol_mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

/* build_direction_numbers (sobol.rs:99-119) and the scrambler of
 * SobolSequence::new (:27-45) for dimension `dim`: v[64], *scr. */
void orc_sobol_dimension(uint64_t dim, uint64_t seed, uint64_t* v, uint64_t* scr) {
  for (int j = 0; j < 64; ++j) {
    if (dim == 0) {
      v[j] = 1ULL << (63 - j);
    } else {
      const uint64_t hash = sobol_mix(seed ^ ((dim + 1) << 40) ^ (uint64_t)j);
      const uint64_t mask = j == 63 ? ~0ULL : (1ULL << (j + 1)) - 1;
      v[j] = ((hash | 1ULL) & mask) << (63 - j);
    }
  }
  *scr = sobol_mix(seed ^ ((dim + 1) << 32));
}

/* Points first..first+count-1 (1-based index, as next_into produces them:
 * x ^= v[ctz(index)], u = fma((double)(x ^ scr), 2^-64, 2^-65)), row-major
 * [point][dim]. */
int orc_sobol_points(int64_t dims, uint64_t seed, int64_t count, double* out) {
  if (dims < 1 || dims > 21201 || count < 0) return OF_ERR_INVALID_INPUT;
  uint64_t* v = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(64 * dims));
  uint64_t* scr = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)dims);
  uint64_t* x = (uint64_t*)calloc((size_t)dims, sizeof(uint64_t));
  if (!v || !scr || !x) {
    free(v);
    free(scr);
    free(x);
    return OF_ERR_ALLOC;
  }
  for (int64_t d = 0; d < dims; ++d) orc_sobol_dimension((uint64_t)d, seed, v + 64 * d, scr + d);
  const double inv = 1.0 / 18446744073709551616.0, half = 0.5 * inv;
  for (int64_t n = 1; n <= count; ++n) {
    const int c = __builtin_ctzll((uint64_t)n);
    for (int64_t d = 0; d < dims; ++d) {
      x[d] ^= v[64 * d + c];
      out[(n - 1) * dims + d] = fma((double)(x[d] ^ scr[d]), inv, half);
    }
  }
  free(v);
  free(scr);
  free(x);
  return OF_OK;
}

/* mc_european_qmc_with_seed (mc_qmc.rs:39-150); q = effective dividend
 * yield.  out[0] = price, out[1] = stderr (NaN/NaN for the reference's
 * invalid-input results, which carry no stderr). */
int orc_mc_european_qmc(int option_type, double spot, double strike, double rate, double q, double vol,
                        double expiry, int64_t n_paths, int64_t n_steps, uint64_t seed, double* out2) {
  if (n_paths <= 0 || n_steps <= 0 || !(vol > 0.0) || !isfinite(vol)) {
    if (n_paths > 0 && n_steps > 0 && expiry <= 0.0) {
      out2[0] = vanilla_payoff(option_type, spot, strike);
      out2[1] = 0.0;
      return OF_OK;
    }
    out2[0] = NAN;
    out2[1] = NAN;
    return OF_OK;
  }
  if (expiry <= 0.0) {
    out2[0] = vanilla_payoff(option_type, spot, strike);
    out2[1] = 0.0;
    return OF_OK;
  }
  if (n_steps > 21201) return OF_ERR_INVALID_INPUT;
  const double dt = expiry / (double)n_steps;
  const double dt_drift = (rate - q - 0.5 * vol * vol) * dt;
  const double dt_vol = vol * sqrt(dt);
  const double discount = exp(-rate * expiry);
  uint64_t* v = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(64 * n_steps));
  uint64_t* scr = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n_steps);
  uint64_t* x = (uint64_t*)calloc((size_t)n_steps, sizeof(uint64_t));
  if (!v || !scr || !x) {
    free(v);
    free(scr);
    free(x);
    return OF_ERR_ALLOC;
  }
  for (int64_t d = 0; d < n_steps; ++d) orc_sobol_dimension((uint64_t)d, seed, v + 64 * d, scr + d);
  const double inv = 1.0 / 18446744073709551616.0, half = 0.5 * inv;
  double sum = 0.0, sum_sq = 0.0;
  for (int64_t n = 1; n <= n_paths; ++n) {
    const int c = __builtin_ctzll((uint64_t)n);
    double s = spot;
    for (int64_t d = 0; d < n_steps; ++d) {
      x[d] ^= v[64 * d + c];
      const double u = fma((double)(x[d] ^ scr[d]), inv, half);
      const double z = orc_acklam_inv_cdf(orc_uniform_open01(u));
      s *= exp(fma(dt_vol, z, dt_drift));
    }
    const double px = vanilla_payoff(option_type, s, strike);
    sum += px;
    sum_sq += px * px;
  }
  const double nn = (double)n_paths;
  const double mean = sum / nn;
  double var = n_paths > 1 ? (sum_sq - sum * sum / nn) / (nn - 1.0) : 0.0;
  var = var > 0.0 ? var : 0.0;
  out2[0] = discount * mean;
  out2[1] = discount * sqrt(var / nn);
  free(v);
  free(scr);
  free(x);
  return OF_OK;
}

/* ------------------------------------------------------------------------ */
/* Bermudan LSM with the exercise boundary                                  */
/* ------------------------------------------------------------------------ */

/* SampledVolSurface::locate_bounds, src/market/market.rs:104-125 */
static void sampled_locate(const double* g, int64_t n, double x, int64_t* lo, int64_t* hi, double* w) {
  if (x <= g[0]) {
    *lo = *hi = 0;
    *w = 0.0;
    return;
  }
  if (x >= g[n - 1]) {
    *lo = *hi = n - 1;
    *w = 0.0;
    return;
  }
  int64_t l = 0;
  for (int64_t i = 0; i < n - 1; ++i)
    if (x >= g[i] && x <= g[i + 1]) {
      l = i;
      break;
    }
  *lo = l;
  *hi = l + 1;
  *w = (x - g[l]) / (g[l + 1] - g[l]);
}

/* SampledVolSurface::vol (bilinear), src/market/market.rs:149-174; vols is
 * row-major [expiry][strike]. */
double orc_sampled_vol(const double* strikes, int64_t nk, const double* expiries, int64_t nt, const double* vols,
                       double strike, double expiry) {
  int64_t e0, e1, s0, s1;
  double ew, sw;
  sampled_locate(expiries, nt, expiry > expiries[0] ? expiry : expiries[0], &e0, &e1, &ew);
  sampled_locate(strikes, nk, strike > strikes[0] ? strike : strikes[0], &s0, &s1, &sw);
  if (e0 == e1 && s0 == s1) return vols[e0 * nk + s0];
  if (e0 == e1) {
    const double v0 = vols[e0 * nk + s0], v1 = vols[e0 * nk + s1];
    return v0 + (v1 - v0) * sw;
  }
  if (s0 == s1) {
    const double v0 = vols[e0 * nk + s0], v1 = vols[e1 * nk + s0];
    return v0 + (v1 - v0) * ew;
  }
  const double v00 = vols[e0 * nk + s0], v01 = vols[e0 * nk + s1];
  const double v10 = vols[e1 * nk + s0], v11 = vols[e1 * nk + s1];
  const double v0 = v00 + (v01 - v00) * sw;
  const double v1 = v10 + (v11 - v10) * sw;
  return v0 + (v1 - v0) * ew;
}

/* LongstaffSchwartzEngine::price_bermudan_with_boundary restated
 * (src/engines/lsm/longstaff_schwartz.rs:294-417, paths :190-283). */
int orc_lsm_bermudan(int option_type, double expiry, const double* sched_t, const double* sched_k, int64_t n_sched,
                     int dynamics, double spot, double rate, double q, double vol, const double* lv_strikes,
                     int64_t lv_nk, const double* lv_expiries, int64_t lv_nt, const double* lv_vols, double kappa,
                     double theta, double xi, double rho, double v0, int64_t num_paths, int64_t num_steps,
                     uint64_t seed, int degree, const double* normals, double* out2, double* boundary,
                     int64_t* n_boundary) {
  if (num_steps < 2 || num_paths < 3 || n_sched < 1) return OF_ERR_INVALID_INPUT;
  if (degree != 2 && degree != 3) return OF_ERR_INVALID_INPUT;
  const int64_t M = num_steps;
  const double dt = expiry / (double)M;
  const double sqrt_dt = sqrt(dt);
  const double drift_rn = rate - q;
  const double terminal_strike = sched_k[n_sched - 1];
  const int64_t stride = (M + 1 + 7) & ~(int64_t)7;
  const int draws = dynamics == 2 ? 2 : 1;
  double* paths = (double*)malloc(sizeof(double) * (size_t)(num_paths * stride));
  double* values = (double*)malloc(sizeof(double) * (size_t)num_paths);
  int64_t* itm = (int64_t*)malloc(sizeof(int64_t) * (size_t)num_paths);
  int64_t* sched_of_step = (int64_t*)malloc(sizeof(int64_t) * (size_t)(M + 1));
  if (!paths || !values || !itm || !sched_of_step) {
    free(paths);
    free(values);
    free(itm);
    free(sched_of_step);
    return OF_ERR_ALLOC;
  }
  orc_xoshiro rng;
  orc_xoshiro_seed(&rng, seed);
  for (int64_t pi = 0; pi < num_paths; ++pi) {
    double* row = paths + pi * stride;
    const double* z = normals ? normals + pi * M * draws : NULL;
    row[0] = spot;
    double s = spot, v = v0;
    for (int64_t ti = 1; ti <= M; ++ti) {
      const double z1 = z ? z[(ti - 1) * draws] : draw_normal(&rng);
      if (dynamics == 0) {
        const double drift = (drift_rn - 0.5 * vol * vol) * dt;
        const double step_vol = vol * sqrt_dt;
        row[ti] = row[ti - 1] * exp(fma(step_vol, z1, drift));
      } else if (dynamics == 1) {
        const double t = (double)ti * dt > 1.0e-8 ? (double)ti * dt : 1.0e-8;
        const double sigma =
            orc_sampled_vol(lv_strikes, lv_nk, lv_expiries, lv_nt, lv_vols, s > 1.0e-8 ? s : 1.0e-8, t);
        const double drift = (drift_rn - 0.5 * sigma * sigma) * dt;
        s *= exp(drift + sigma * sqrt_dt * z1);
        row[ti] = s > 1.0e-12 ? s : 1.0e-12;
        s = row[ti];
      } else {
        const double z2 = z ? z[(ti - 1) * draws + 1] : draw_normal(&rng);
        /* Heston::step_euler, src/models/stochastic.rs:56-71 (mu = r - q) */
        const double v_pos = v > 0.0 ? v : 0.0;
        const double zs = rho * z1 + sqrt(1.0 - rho * rho) * z2;
        double v_next = v + kappa * (theta - v_pos) * dt + xi * sqrt(v_pos) * sqrt_dt * z1;
        v_next = v_next > 0.0 ? v_next : 0.0;
        const double s_next = s * exp((drift_rn - 0.5 * v_pos) * dt + sqrt(v_pos) * sqrt_dt * zs);
        s = s_next > 1.0e-12 ? s_next : 1.0e-12;
        v = v_next > 0.0 ? v_next : 0.0;
        row[ti] = s;
      }
    }
  }
  const double disc = exp(-rate * dt);
  for (int64_t i = 0; i <= M; ++i) sched_of_step[i] = -1;
  for (int64_t d = 0; d < n_sched; ++d) {
    double idx = round((sched_t[d] / expiry) * (double)M);
    int64_t i = isnan(idx) || idx < 1.0 ? 1 : (idx > (double)M ? M : (int64_t)idx);
    sched_of_step[i] = d;
  }
  int64_t terminal_itm = 0;
  for (int64_t pi = 0; pi < num_paths; ++pi) {
    values[pi] = vanilla_payoff(option_type, paths[pi * stride + M], terminal_strike);
    if (values[pi] > 0.0) ++terminal_itm;
  }
  /* boundary records, filled last date first then reversed */
  int64_t nb = 0;
  double* rec = boundary + 5 * nb++;
  rec[0] = expiry;
  rec[1] = terminal_strike;
  rec[2] = terminal_strike;
  rec[3] = (double)terminal_itm;
  rec[4] = (double)terminal_itm;
  for (int64_t ti = M - 1; ti >= 1; --ti) {
    for (int64_t pi = 0; pi < num_paths; ++pi) values[pi] *= disc;
    const int64_t d = sched_of_step[ti];
    if (d < 0) continue;
    const double strike = sched_k[d];
    int64_t n_itm = 0;
    for (int64_t pi = 0; pi < num_paths; ++pi)
      if (vanilla_payoff(option_type, paths[pi * stride + ti], strike) > 0.0) itm[n_itm++] = pi;
    rec = boundary + 5 * nb++;
    rec[0] = sched_t[d];
    rec[1] = strike;
    rec[2] = NAN;
    rec[3] = (double)n_itm;
    rec[4] = 0.0;
    if (n_itm < 3) continue;
    double beta[4] = {0, 0, 0, 0};
    const double inv_k = 1.0 / strike;
    if (degree == 2) {
      double s1 = 0, s_s = 0, s_s2 = 0, s_s3 = 0, s_s4 = 0, s_y = 0, s_sy = 0, s_s2y = 0;
      for (int64_t k = 0; k < n_itm; ++k) {
        const double s = paths[itm[k] * stride + ti];
        const double s2 = s * s;
        const double y = values[itm[k]];
        s1 += 1.0;
        s_s += s;
        s_s2 += s2;
        s_s3 += s2 * s;
        s_s4 += s2 * s2;
        s_y += y;
        s_sy += s * y;
        s_s2y += s2 * y;
      }
      double a[3][3] = {{s1, s_s, s_s2}, {s_s, s_s2, s_s3}, {s_s2, s_s3, s_s4}};
      double b[3] = {s_y, s_sy, s_s2y};
      double x[3];
      if (lu_solve3(a, b, x)) {
        beta[0] = x[0];
        beta[1] = x[1];
        beta[2] = x[2];
      }
    } else {
      double m[7] = {0, 0, 0, 0, 0, 0, 0}, r[4] = {0, 0, 0, 0};
      for (int64_t k = 0; k < n_itm; ++k) {
        const double x = paths[itm[k] * stride + ti] * inv_k;
        const double y = values[itm[k]];
        double p = 1.0;
        for (int e = 0; e < 7; ++e) {
          m[e] += p;
          if (e < 4) r[e] += p * y;
          p *= x;
        }
      }
      double a[4][4];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) a[i][j] = m[i + j];
      double x4[4];
      if (chol_solve4(a, r, x4))
        for (int i = 0; i < 4; ++i) beta[i] = x4[i];
    }
    int64_t n_ex = 0;
    double bnd = NAN;
    for (int64_t k = 0; k < n_itm; ++k) {
      const double s = paths[itm[k] * stride + ti];
      const double cont = degree == 2 ? beta[0] + beta[1] * s + beta[2] * s * s
                                      : beta[0] + (s * inv_k) * (beta[1] + (s * inv_k) * (beta[2] + (s * inv_k) * beta[3]));
      const double ex = vanilla_payoff(option_type, s, strike);
      if (ex > cont) {
        values[itm[k]] = ex;
        /* boundary_from_exercised, :178-188: put max, call min */
        if (n_ex == 0 || (option_type == OF_PUT ? s > bnd : s < bnd)) bnd = s;
        ++n_ex;
      }
    }
    rec[2] = bnd;
    rec[4] = (double)n_ex;
  }
  double sum = 0.0, sum_sq = 0.0;
  for (int64_t pi = 0; pi < num_paths; ++pi) {
    const double v = values[pi] * disc;
    sum += v;
    sum_sq += v * v;
  }
  const double n = (double)num_paths;
  const double mean = sum / n;
  const double var = num_paths > 1 ? (sum_sq - sum * sum / n) / (n - 1.0) : 0.0;
  out2[0] = mean;
  out2[1] = sqrt(var / n);
  /* chronological order */
  for (int64_t i = 0, j = nb - 1; i < j; ++i, --j)
    for (int f = 0; f < 5; ++f) {
      const double t = boundary[5 * i + f];
      boundary[5 * i + f] = boundary[5 * j + f];
      boundary[5 * j + f] = t;
    }
  *n_boundary = nb;
  free(paths);
  free(values);
  free(itm);
  free(sched_of_step);
  return OF_OK;
}

/* ------------------------------------------------------------------------ */
/* Reference WGSL shader math (src/engines/gpu/mc_shader.wgsl, gpu_mc.rs)    */
/* ------------------------------------------------------------------------ */

static inline uint32_t rotl32(uint32_t x, uint32_t k) { return (x << k) | (x >> (32u - k)); }

typedef struct wg_rng { uint32_t s0, s1, s2, s3; } wg_rng;

static inline uint32_t mix32(uint32_t z) {
  z ^= z >> 16;
  z *= 0x45d9f3bu;
  z ^= z >> 16;
  z *= 0x45d9f3bu;
  z ^= z >> 16;
  return z;
}

/* seed_rng, mc_shader.wgsl:57-71 */
static void wg_seed(wg_rng* r, uint32_t global_id, uint32_t seed) {
  uint32_t z = global_id + seed;
  z = mix32(z);
  r->s0 = z;
  z += 0x9e3779b9u;
  z = mix32(z);
  r->s1 = z;
  z += 0x9e3779b9u;
  z = mix32(z);
  r->s2 = z;
  z += 0x9e3779b9u;
  z = mix32(z);
  r->s3 = z;
}

/* xoshiro128pp_next, mc_shader.wgsl:38-48 */
static inline uint32_t wg_next(wg_rng* r) {
  const uint32_t result = rotl32(r->s0 + r->s3, 7u) + r->s0;
  const uint32_t t = r->s1 << 9u;
  r->s2 ^= r->s0;
  r->s3 ^= r->s1;
  r->s1 ^= r->s2;
  r->s0 ^= r->s3;
  r->s2 ^= t;
  r->s3 = rotl32(r->s3, 11u);
  return result;
}

static inline float wg_f32(wg_rng* r) { return (float)(wg_next(r) >> 8u) * 5.9604644775390625e-8f; }

int orc_wgsl_european(double spot, double strike, double rate, double vol, double expiry, uint32_t num_paths,
                      uint32_t num_steps, uint32_t seed, int is_call, double* price, double* stderr_) {
  if (num_paths == 0 || num_steps == 0) return OF_ERR_INVALID_INPUT;
  /* build_params, gpu_mc.rs:59-89 */
  const double dt = expiry / (double)num_steps;
  const float dt_drift = (float)((rate - 0.5 * vol * vol) * dt);
  const float dt_vol = (float)(vol * sqrt(dt));
  const double discount = exp(-rate * expiry);
  const float fspot = (float)spot, fstrike = (float)strike;
  const uint32_t n_groups = (num_paths + 255u) / 256u;
  double sum = 0.0, sum_sq = 0.0;
  float pay[256];
  for (uint32_t g = 0; g < n_groups; ++g) {
    for (uint32_t lid = 0; lid < 256u; ++lid) {
      const uint32_t path_id = g * 256u + lid;
      float payoff = 0.0f;
      if (path_id < num_paths) {
        wg_rng r;
        wg_seed(&r, path_id, seed);
        float s = fspot;
        const uint32_t pairs = num_steps / 2u;
        for (uint32_t p = 0; p <= pairs; ++p) {
          if (p == pairs && (num_steps & 1u) == 0u) break;
          float u1 = wg_f32(&r);
          u1 = u1 > 1.0e-10f ? u1 : 1.0e-10f;
          const float u2 = wg_f32(&r);
          const float rr = sqrtf(-2.0f * logf(u1));
          const float th = 6.283185307179586f * u2;
          s *= expf(fmaf(dt_vol, rr * cosf(th), dt_drift));
          if (p < pairs) s *= expf(fmaf(dt_vol, rr * sinf(th), dt_drift));
        }
        const float v = is_call ? s - fstrike : fstrike - s;
        payoff = v > 0.0f ? v : 0.0f;
      }
      pay[lid] = payoff;
    }
    float ps[256], pq[256];
    for (int i = 0; i < 256; ++i) {
      ps[i] = pay[i];
      pq[i] = pay[i] * pay[i];
    }
    for (int stride = 128; stride > 0; stride >>= 1)
      for (int i = 0; i < stride; ++i) {
        ps[i] += ps[i + stride];
        pq[i] += pq[i + stride];
      }
    sum += (double)ps[0];
    sum_sq += (double)pq[0];
  }
  /* reduce_partial_sums, gpu_mc.rs:96-118 */
  const double n = (double)num_paths;
  const double mean = sum / n;
  const double var = num_paths > 1 ? (sum_sq - sum * sum / n) / (n - 1.0) : 0.0;
  *price = discount * mean;
  *stderr_ = discount * sqrt(var / n);
  return OF_OK;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw 2011)                           */
/* ------------------------------------------------------------------------ */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}
