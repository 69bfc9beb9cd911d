// mc_reference.cu - FP64 reference-stream Monte Carlo (of_mc_run, FP64 mode).
//
// Reproduces openferric's MonteCarloEngine::run (src/mc/simulation.rs:182-348)
// draw for draw: sample i owns a xoshiro256++ stream seeded with
// seed + i*7919, draws z1[j] (and z2[j] for Heston) per step in the reference's
// interleaved order, builds the path with the reference generators and
// evaluates the payoff and control variate.  One thread owns one sample and
// keeps the path in registers: the running barrier flag and the per-step
// observation sums replace the reference's Vec<f64> path buffer.  An
// antithetic sample advances its negated twin in the same loop.
//
// This file is compiled with --fmad=false: the only fused multiply-adds are
// the explicit fma() calls standing for the reference's mul_add.
#include <cmath>
#include <cstring>
#include <vector>

#include "of_device.cuh"
#include "of_internal.h"

namespace {

struct RefParams {
  int32_t model, payoff, option_type, antithetic;
  int32_t cv_kind, barrier_up, barrier_in, averaging;
  int32_t floating, terminal_only, need_arith, need_geo;
  int64_t samples, steps;
  uint64_t seed;
  double s0, strike, barrier, rebate, n_obs;
  double drift, diffusion;  // GBM (simulation.rs:63-66)
  double mu, dt, sqrt_dt, kappa, theta, xi, rho, rho_c, v0;  // Heston (stochastic.rs:56-71)
  const double* obs_w;  // [steps+1] observation counts
  const double* inj;    // injected normals or nullptr
  const of_div_trigger* div;  // GBM discrete dividends by trigger step, or nullptr
  int32_t n_div;
};

struct Leg {
  double s, v, arith, geo;
  bool hit;
};

__device__ __forceinline__ double vanilla(int option_type, double spot, double strike) {
  const double v = option_type == OF_CALL ? spot - strike : strike - spot;
  return v > 0.0 ? v : 0.0;
}

__device__ __forceinline__ void observe(Leg& L, const RefParams& P, int64_t idx) {
  if (P.payoff == OF_PAYOFF_BARRIER) L.hit |= P.barrier_up ? (L.s >= P.barrier) : (L.s <= P.barrier);
  if (P.need_arith | P.need_geo) {
    const double w = __ldg(P.obs_w + idx);
    if (w != 0.0) {
      if (P.need_arith) L.arith += w * L.s;
      if (P.need_geo) L.geo += w * log(L.s > 1e-12 ? L.s : 1e-12);
    }
  }
}

__device__ __forceinline__ void leg_init(Leg& L, const RefParams& P) {
  L.s = P.s0;
  L.v = P.v0;
  L.arith = -0.0;
  L.geo = -0.0;
  L.hit = false;
  observe(L, P, 0);
}

// HestonPathGenerator::generate_into + Heston::step_euler
// (simulation.rs:104-115, stochastic.rs:56-71), operation order preserved.
__device__ __forceinline__ void heston_step(Leg& L, const RefParams& P, double z1, double z2) {
  const double v_pos = L.v > 0.0 ? L.v : 0.0;
  const double zs = P.rho * z1 + P.rho_c * z2;
  double v_next = L.v + P.kappa * (P.theta - v_pos) * P.dt + P.xi * sqrt(v_pos) * P.sqrt_dt * z1;
  v_next = v_next > 0.0 ? v_next : 0.0;
  const double s_next = L.s * exp((P.mu - 0.5 * v_pos) * P.dt + sqrt(v_pos) * P.sqrt_dt * zs);
  L.s = s_next > 1e-12 ? s_next : 1e-12;
  L.v = v_next;
}

// payoff_from_path (mc_engine.rs:453-545) on the register-resident path summary.
__device__ __forceinline__ double leg_payoff(const Leg& L, const RefParams& P) {
  switch (P.payoff) {
    case OF_PAYOFF_VANILLA:
      return vanilla(P.option_type, L.s, P.strike);
    case OF_PAYOFF_BARRIER: {
      const bool active = P.barrier_in ? L.hit : !L.hit;
      return active ? vanilla(P.option_type, L.s, P.strike) : P.rebate;
    }
    default: {
      double avg;
      if (P.terminal_only) avg = L.s;
      else if (P.averaging == OF_AVG_ARITHMETIC) avg = L.arith / P.n_obs;
      else avg = exp(L.geo / P.n_obs);
      return P.floating ? vanilla(P.option_type, L.s, avg) : vanilla(P.option_type, avg, P.strike);
    }
  }
}

// Control-variate evaluators (mc_engine.rs:481-483, :570-581; simulation.rs:441-444).
__device__ __forceinline__ double leg_cv(const Leg& L, const RefParams& P) {
  switch (P.cv_kind) {
    case OF_CV_VANILLA_TERMINAL:
      return vanilla(P.option_type, L.s, P.strike);
    case OF_CV_GEOMETRIC_ASIAN:
      return vanilla(P.option_type, P.terminal_only ? L.s : exp(L.geo / P.n_obs), P.strike);
    case OF_CV_TERMINAL_SPOT:
      return L.s;
    default:
      return 0.0;
  }
}

// DividendEvent::apply_jump (src/market/dividends.rs:76-83).
__device__ __forceinline__ double dividend_jump(const of_div_trigger& e, double s) {
  if (e.kind == OF_DIV_CASH) {
    const double x = s - e.amount;
    return x > 0.0 ? x : 0.0;
  }
  return s * (1.0 - e.amount);
}

// RNG: of::Xoshiro256pp or of::Pcg64, the FastRngKind of the engine.
template <typename RNG>
__global__ void __launch_bounds__(128) mc_ref_kernel(RefParams P, double* __restrict__ partials) {
  __shared__ double sh[5 * 4];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const bool heston = P.model != OF_MODEL_GBM;
  const int streams = heston ? 2 : 1;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.samples; i += stride) {
    RNG rng;
    const double* inj = P.inj ? P.inj + i * P.steps * streams : nullptr;
    if (!inj) rng.seed(P.seed + (uint64_t)i * 7919ULL);  // stream_seed, fast_rng.rs:203-205
    Leg a, b;
    leg_init(a, P);
    if (P.antithetic) leg_init(b, P);
    int32_t ev = 0;  // next dividend trigger
    for (int64_t j = 0; j < P.steps; ++j) {
      double z1, z2 = 0.0;
      if (inj) {
        z1 = inj[j * streams];
        if (heston) z2 = inj[j * streams + 1];
      } else {
        z1 = of::acklam_inv_cdf(rng.next_f64());
        if (heston) z2 = of::acklam_inv_cdf(rng.next_f64());
      }
      if (!heston) {
        a.s *= exp(fma(P.diffusion, z1, P.drift));  // simulation.rs:67-71
        if (P.antithetic) b.s *= exp(fma(P.diffusion, -z1, P.drift));
        for (; ev < P.n_div && P.div[ev].step == j; ++ev) {  // mc_engine.rs:157-167
          a.s = dividend_jump(P.div[ev], a.s);
          if (P.antithetic) b.s = dividend_jump(P.div[ev], b.s);
        }
      } else {
        heston_step(a, P, z1, z2);
        if (P.antithetic) heston_step(b, P, -z1, -z2);
      }
      observe(a, P, j + 1);
      if (P.antithetic) observe(b, P, j + 1);
    }
    double x = leg_payoff(a, P);
    double y = leg_cv(a, P);
    if (P.antithetic) {  // simulation.rs:235-252
      x = 0.5 * (x + leg_payoff(b, P));
      y = 0.5 * (y + leg_cv(b, P));
    }
    acc[0] += x;
    acc[1] += x * x;
    acc[2] += y;
    acc[3] += x * y;
    acc[4] += y * y;
  }
  of::block_sum<5>(acc, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 5; ++k) partials[(int64_t)blockIdx.x * 5 + k] = acc[k];
}

// GBM European without dividends: the path matters only through S_T, a
// product of per-step factors, so two adjacent lanes share a sample.  Both
// step the sample's stream; lane p computes the normal and the factor
// exp(fma(sigma sqrt(dt), z, drift)) of the steps j = p (mod 2), and the pair
// multiplies its two partial products.  The draws and each step's factor are
// mc_ref_kernel's; only the order of the product's roundings differs (S_T to
// about 1e-15 relative).  Half the FP64 work per lane and twice the lanes
// for the same samples: this workload has too few samples per SM to hide the
// FP64 exp and divide latencies with one lane per sample.
template <typename RNG>
__global__ void __launch_bounds__(128) mc_ref_gbm_terminal(RefParams P, double* __restrict__ partials) {
  __shared__ double sh[5 * 4];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int lane = (int)(threadIdx.x & 31u), par = lane & 1;
  const int64_t pair0 = ((int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u)) >> 1;  // the warp's first sample
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 1;
  for (int64_t base = pair0; base < P.samples; base += stride) {  // warp-uniform trip count
    const int64_t i = base + (lane >> 1);
    const bool valid = i < P.samples;
    RNG rng;
    rng.seed(P.seed + (uint64_t)i * 7919ULL);  // stream_seed, fast_rng.rs:203-205
    double fa = 1.0, fb = 1.0;
    // both lanes draw steps j and j+1 of the stream; each takes its own (no
    // divergence: every lane runs the inverse normal and exp each iteration)
    for (int64_t j = 0; j < P.steps; j += 2) {
      const double u0 = rng.next_f64();
      const double u1 = j + 1 < P.steps ? rng.next_f64() : 0.5;
      if (j + par < P.steps) {
        const double z = of::acklam_inv_cdf(par ? u1 : u0);
        fa *= exp(fma(P.diffusion, z, P.drift));  // simulation.rs:67-71
        if (P.antithetic) fb *= exp(fma(P.diffusion, -z, P.drift));
      }
    }
    const double oa = __shfl_xor_sync(of::kFullMask, fa, 1);
    const double ob = __shfl_xor_sync(of::kFullMask, fb, 1);
    if (par == 0 && valid) {
      Leg a{P.s0 * fa * oa, 0.0, 0.0, 0.0, false}, b{P.s0 * fb * ob, 0.0, 0.0, 0.0, false};
      double x = vanilla(P.option_type, a.s, P.strike);
      double y = leg_cv(a, P);
      if (P.antithetic) {  // simulation.rs:235-252
        x = 0.5 * (x + vanilla(P.option_type, b.s, P.strike));
        y = 0.5 * (y + leg_cv(b, P));
      }
      acc[0] += x;
      acc[1] += x * x;
      acc[2] += y;
      acc[3] += x * y;
      acc[4] += y * y;
    }
  }
  of::block_sum<5>(acc, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 5; ++k) partials[(int64_t)blockIdx.x * 5 + k] = acc[k];
}

}  // namespace

// Observation index of average_for_observations (mc_engine.rs:100-104):
// round(t / maturity * (len-1)) saturated into [0, len-1].
static int64_t obs_index(double t, double maturity, int64_t len) {
  const double idx = std::round((t / maturity) * (double)(len - 1));
  int64_t i = (std::isnan(idx) || idx <= 0.0) ? 0 : (int64_t)idx;
  return i < len - 1 ? i : len - 1;
}

of_status of_dividend_triggers(of_ctx* ctx, const of_model* m, std::vector<of_div_trigger>& out) {
  out.clear();
  if (m->n_dividends <= 0) return OF_OK;
  if (!m->dividends) return of_fail(ctx, OF_ERR_INVALID_INPUT, "dividends is null");
  if (m->kind != OF_MODEL_GBM)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "discrete dividends apply to GBM paths only");
  double prev = 0.0;
  for (int64_t e = 0; e < m->n_dividends; ++e) {
    const of_dividend_event& d = m->dividends[e];
    if (!std::isfinite(d.time) || d.time <= 0.0)
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "dividend event time must be finite and > 0");
    if (d.kind == OF_DIV_CASH) {
      if (!std::isfinite(d.amount) || d.amount < 0.0)
        return of_fail(ctx, OF_ERR_INVALID_INPUT, "cash dividend amount must be finite and >= 0");
    } else if (d.kind == OF_DIV_PROPORTIONAL) {
      if (!std::isfinite(d.amount) || d.amount < 0.0 || d.amount >= 1.0)
        return of_fail(ctx, OF_ERR_INVALID_INPUT, "proportional dividend ratio must be finite and in [0, 1)");
    } else {
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown dividend kind %d", d.kind);
    }
    if (d.time <= prev) return of_fail(ctx, OF_ERR_INVALID_INPUT, "dividend event times must be strictly increasing");
    prev = d.time;
  }
  const double dt = m->maturity / (double)m->steps;
  int64_t ev = 0;
  for (int64_t j = 0; j < m->steps && ev < m->n_dividends; ++j) {
    const double t = (double)(j + 1) * dt;
    while (ev < m->n_dividends && m->dividends[ev].time <= m->maturity + 1.0e-12 &&
           m->dividends[ev].time <= t + 1.0e-12) {
      out.push_back(of_div_trigger{(int32_t)j, m->dividends[ev].kind, m->dividends[ev].amount});
      ++ev;
    }
  }
  return OF_OK;
}

of_status of_validate_mc(of_ctx* ctx, const of_model* m, const of_payoff* p, const of_mc_config* c) {
  if (!m || !p || !c) return of_fail(ctx, OF_ERR_INVALID_INPUT, "null argument");
  if (c->num_paths <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths must be > 0");
  if (m->steps <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps must be > 0");
  if (m->steps > (int64_t)1 << 30) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps too large");
  if (!(m->maturity > 0.0) || !std::isfinite(m->maturity))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "maturity must be finite and > 0");
  if (!(m->s0 > 0.0) || !std::isfinite(m->s0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "spot must be > 0");
  if (!std::isfinite(m->mu)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "drift must be finite");
  if (m->kind == OF_MODEL_GBM) {
    if (!(m->sigma > 0.0) || !std::isfinite(m->sigma))
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "market volatility must be > 0");
  } else if (m->kind == OF_MODEL_HESTON_EULER || m->kind == OF_MODEL_HESTON_QE) {
    // Heston::validate, src/models/stochastic.rs:47-54
    if (!(m->kappa > 0.0 && m->theta >= 0.0 && m->xi >= 0.0 && m->v0 >= 0.0 && m->rho > -1.0 && m->rho < 1.0))
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "invalid Heston parameters");
  } else {
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown model kind %d", m->kind);
  }
  if (m->n_dividends > 0) {
    std::vector<of_div_trigger> trig;
    OF_TRY(of_dividend_triggers(ctx, m, trig));
  }
  if (p->option_type != OF_CALL && p->option_type != OF_PUT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown option type %d", p->option_type);
  if (p->kind < OF_PAYOFF_VANILLA || p->kind > OF_PAYOFF_ASIAN)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown payoff kind %d", p->kind);
  if (!std::isfinite(p->strike)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "strike must be finite");
  if (p->kind == OF_PAYOFF_ASIAN && p->n_observations > 0 && !p->observation_times)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "observation_times is null");
  if (c->rng_kind != OF_RNG_XOSHIRO256PP && c->rng_kind != OF_RNG_PCG64)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown rng kind %d", c->rng_kind);
  if (c->rng_kind != OF_RNG_XOSHIRO256PP && c->precision != OF_PREC_FP64_REFERENCE)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "the FP32 Philox mode draws from Philox streams only");
  if (c->control_variate < OF_CV_NONE || c->control_variate > OF_CV_TERMINAL_SPOT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown control variate %d", c->control_variate);
  if (!std::isfinite(c->discount_factor)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "discount factor must be finite");
  return OF_OK;
}

// Observation counts per step index for the Asian payoff / geometric CV.
// Returns terminal_only = true where average_for_observations falls back to
// the terminal spot (no observations or maturity <= 0, mc_engine.rs:92-94).
void of_observation_weights(const of_payoff* p, int64_t steps, std::vector<double>& w, bool& terminal_only) {
  w.assign((size_t)steps + 1, 0.0);
  terminal_only = !(p->n_observations > 0 && p->expiry > 0.0);
  if (terminal_only) return;
  for (int64_t k = 0; k < p->n_observations; ++k) w[(size_t)obs_index(p->observation_times[k], p->expiry, steps + 1)] += 1.0;
}

of_status of_mc_run_fp32(of_ctx* ctx, const of_model* model, const of_payoff* payoff, const of_mc_config* cfg,
                         of_mc_result* out);

extern "C" of_status of_mc_run(of_ctx* ctx, const of_model* m, const of_payoff* p, const of_mc_config* c,
                               of_mc_result* out) {
  if (!ctx || !out) return OF_ERR_INVALID_INPUT;
  OF_TRY(of_validate_mc(ctx, m, p, c));
  if (c->precision == OF_PREC_FP32_PHILOX) return of_mc_run_fp32(ctx, m, p, c, out);
  if (c->precision != OF_PREC_FP64_REFERENCE)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown precision %d", c->precision);
  if (m->kind == OF_MODEL_HESTON_QE)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "the QE scheme has no FP64 reference-stream mode");
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));

  RefParams P{};
  P.model = m->kind;
  P.payoff = p->kind;
  P.option_type = p->option_type;
  P.antithetic = c->antithetic ? 1 : 0;
  P.cv_kind = c->control_variate;
  P.barrier_up = p->barrier_direction == OF_BARRIER_UP;
  P.barrier_in = p->barrier_style == OF_BARRIER_IN;
  P.averaging = p->averaging;
  P.floating = p->strike_type == OF_STRIKE_FLOATING;
  P.samples = c->antithetic ? (c->num_paths + 1) / 2 : c->num_paths;
  P.steps = m->steps;
  P.seed = c->seed;
  P.s0 = m->s0;
  P.strike = p->strike;
  P.barrier = p->barrier_level;
  P.rebate = p->rebate;
  P.v0 = m->v0;
  const double dt = m->maturity / (double)m->steps;
  const double sqrt_dt = std::sqrt(dt);
  P.drift = (m->mu - 0.5 * m->sigma * m->sigma) * dt;
  P.diffusion = m->sigma * sqrt_dt;
  P.mu = m->mu;
  P.dt = dt;
  P.sqrt_dt = sqrt_dt;
  P.kappa = m->kappa;
  P.theta = m->theta;
  P.xi = m->xi;
  P.rho = m->rho;
  P.rho_c = std::sqrt(1.0 - m->rho * m->rho);

  const bool asian = p->kind == OF_PAYOFF_ASIAN;
  P.need_arith = asian && p->averaging == OF_AVG_ARITHMETIC;
  P.need_geo = (asian && p->averaging == OF_AVG_GEOMETRIC) || c->control_variate == OF_CV_GEOMETRIC_ASIAN;
  std::vector<double> w;
  bool terminal_only = true;
  if (P.need_arith || P.need_geo) {
    of_observation_weights(p, m->steps, w, terminal_only);
    if (terminal_only) P.need_arith = P.need_geo = 0;
  }
  P.terminal_only = terminal_only;
  P.n_obs = (double)p->n_observations;

  void* d_obs = nullptr;
  if (P.need_arith || P.need_geo) {
    OF_TRY(of_scratch(ctx, SLOT_OBS, w.size() * sizeof(double), &d_obs));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(d_obs, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  }
  P.obs_w = (const double*)d_obs;

  std::vector<of_div_trigger> trig;
  OF_TRY(of_dividend_triggers(ctx, m, trig));
  if (!trig.empty()) {
    void* d_div = nullptr;
    OF_TRY(of_scratch(ctx, SLOT_DIVIDENDS, trig.size() * sizeof(of_div_trigger), &d_div));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(d_div, trig.data(), trig.size() * sizeof(of_div_trigger),
                                     cudaMemcpyHostToDevice, ctx->stream));
    P.div = (const of_div_trigger*)d_div;
    P.n_div = (int32_t)trig.size();
  }

  const int streams = m->kind == OF_MODEL_GBM ? 1 : 2;
  if (c->injected_normals) {
    const int64_t need = P.samples * P.steps * streams;
    if (c->n_injected < need)
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "injected normals: need %lld values, got %lld", (long long)need,
                     (long long)c->n_injected);
    void* d_inj = nullptr;
    OF_TRY(of_scratch(ctx, SLOT_INJECT, (size_t)need * sizeof(double), &d_inj));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(d_inj, c->injected_normals, (size_t)need * sizeof(double),
                                     cudaMemcpyHostToDevice, ctx->stream));
    P.inj = (const double*)d_inj;
  }

  const int block = 128;
  // a GBM European without dividends (its control variate, if any, reads S_T
  // only): two lanes per sample
  const bool terminal = P.model == OF_MODEL_GBM && P.payoff == OF_PAYOFF_VANILLA && P.n_div == 0 && !P.inj &&
                        P.cv_kind != OF_CV_GEOMETRIC_ASIAN;
  const bool pcg = c->rng_kind == OF_RNG_PCG64;
  const void* kern = terminal ? (pcg ? (const void*)mc_ref_gbm_terminal<of::Pcg64>
                                     : (const void*)mc_ref_gbm_terminal<of::Xoshiro256pp>)
                              : (pcg ? (const void*)mc_ref_kernel<of::Pcg64> : (const void*)mc_ref_kernel<of::Xoshiro256pp>);
  const int64_t lanes = terminal ? 2 * P.samples : P.samples;
  const int64_t want = (lanes + block - 1) / block;
  const int64_t cap = (int64_t)ctx->sm_count * of_blocks_per_sm(kern, block, 0);
  const int grid = (int)(want < cap ? want : cap);
  void *d_part = nullptr, *d_sums = nullptr, *h = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)grid * 5 * sizeof(double), &d_part));
  OF_TRY(of_scratch(ctx, SLOT_SUMS, 5 * sizeof(double), &d_sums));
  OF_TRY(of_pinned(ctx, 5 * sizeof(double), &h));

  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  if (terminal && pcg) mc_ref_gbm_terminal<of::Pcg64><<<grid, block, 0, ctx->stream>>>(P, (double*)d_part);
  else if (terminal) mc_ref_gbm_terminal<of::Xoshiro256pp><<<grid, block, 0, ctx->stream>>>(P, (double*)d_part);
  else if (pcg) mc_ref_kernel<of::Pcg64><<<grid, block, 0, ctx->stream>>>(P, (double*)d_part);
  else mc_ref_kernel<of::Xoshiro256pp><<<grid, block, 0, ctx->stream>>>(P, (double*)d_part);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_TRY(of_reduce_rows(ctx, (const double*)d_part, grid, 5, (double*)d_sums));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(h, d_sums, 5 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
  double sums[5];
  std::memcpy(sums, h, sizeof(sums));
  of_mc_finish(sums, P.samples, c->control_variate, c->cv_expected, c->discount_factor, out);
  out->kernel_ms = ms;
  return OF_OK;
}
