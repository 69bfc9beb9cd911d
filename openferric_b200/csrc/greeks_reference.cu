// greeks_reference.cu - Monte Carlo Greeks on openferric's own streams (FP64).
//
//  of_mc_european_pathwise_aad  <- mc_european_pathwise_aad (src/engines/monte_carlo/mc_aad.rs:75-219)
//  of_heston_price_delta_aad    <- heston_price_delta_aad   (mc_aad.rs:239-342)
//  of_mc_greek_estimators       <- MonteCarloGreeksEngine   (src/engines/monte_carlo/mc_greeks.rs:95-342)
//
// The reference records a reverse-mode tape per path (about 5 nodes a step)
// and sweeps it backwards.  For the GBM log-Euler path the adjoint of every
// step's exponent is the same number, dpv/dS_T * S_T, so the reverse sweep
// collapses to closed forms of the forward quantities S_T, prod(growth) and
// sum(z): the device keeps three registers per leg instead of a tape.
// Compiled with --fmad=false (only explicit fma() contract, as in the
// reference's mul_add).
#include <cmath>
#include <cstring>

#include "of_device.cuh"
#include "of_internal.h"

namespace {

struct GreekP {
  int32_t call, antithetic;
  int64_t samples, steps;
  uint64_t seed;
  double spot, strike, rate, q, vol, expiry;
  // GBM tape constants (mc_aad.rs:34-47)
  double dt, sqrt_dt, drift_inner, drift, diffusion, disc;
  // Heston (mc_aad.rs:249-275)
  double mu, kappa, theta, xi, rho, rho2, v0;
  // MonteCarloGreeksEngine (mc_greeks.rs:157-170)
  double g_drift, sig_sqrt_t, spot_up, spot_dn, spot_span, sqrt_t;
};

// One GBM leg through the tape semantics of gbm_single_path_reverse
// (mc_aad.rs:15-72): expo = drift + diffusion*z (mul then add), s = s*exp(expo).
struct AadLeg {
  double s, prod, sumz;
};

__device__ __forceinline__ void aad_leg_finish(const AadLeg& L, const GreekP& P, double& pv, double g[4]) {
  const double intrinsic = P.call ? L.s - P.strike : P.strike - L.s;
  const double payoff = intrinsic > 0.0 ? intrinsic : 0.0;
  const double rt = P.rate * P.expiry;
  const double discount = exp(-rt);
  pv = discount * payoff;
  // reverse sweep (same node order as the tape)
  double r_bar = 0.0, t_bar = 0.0, sigma_bar = 0.0, dt_bar = 0.0;
  const double rt_bar = -(payoff * discount);
  r_bar += rt_bar * P.expiry;
  t_bar += rt_bar * P.rate;
  const double intrinsic_bar = intrinsic > 0.0 ? discount : 0.0;
  const double sT_bar = P.call ? intrinsic_bar : -intrinsic_bar;
  const double expo_bar = sT_bar * L.s;  // identical for every step
  const double drift_bar = (double)P.steps * expo_bar;
  const double diffusion_bar = expo_bar * L.sumz;
  sigma_bar += diffusion_bar * P.sqrt_dt;
  const double sqrt_dt_bar = diffusion_bar * P.vol;
  const double drift_inner_bar = drift_bar * P.dt;
  dt_bar += drift_bar * P.drift_inner;
  r_bar += drift_inner_bar;
  const double sigma_sq_bar = 0.5 * (-drift_inner_bar);
  sigma_bar += sigma_sq_bar * P.vol;
  sigma_bar += sigma_sq_bar * P.vol;
  dt_bar += sqrt_dt_bar * (0.5 / P.sqrt_dt);
  t_bar += dt_bar / (double)P.steps;
  g[0] = sT_bar * L.prod;
  g[1] = r_bar;
  g[2] = sigma_bar;
  g[3] = t_bar;
}

__global__ void __launch_bounds__(128) aad_kernel(GreekP P, double* __restrict__ partials) {
  __shared__ double sh[6 * 4];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.samples; i += stride) {
    of::Xoshiro256pp rng;
    rng.seed(P.seed + (uint64_t)i * 7919ULL);
    AadLeg a{P.spot, 1.0, 0.0}, b{P.spot, 1.0, 0.0};
    for (int64_t j = 0; j < P.steps; ++j) {
      const double z = of::acklam_inv_cdf(rng.next_f64());
      const double ga = exp(P.drift + P.diffusion * z);
      a.s = a.s * ga;
      a.prod = a.prod * ga;
      a.sumz += z;
      if (P.antithetic) {
        const double gb = exp(P.drift + P.diffusion * -z);
        b.s = b.s * gb;
        b.prod = b.prod * gb;
        b.sumz += -z;
      }
    }
    double pv, g[4];
    aad_leg_finish(a, P, pv, g);
    if (P.antithetic) {  // mc_aad.rs:169-194
      double pv1, g1[4];
      aad_leg_finish(b, P, pv1, g1);
      for (int k = 0; k < 4; ++k) g[k] = 0.5 * (g[k] + g1[k]);
      pv = 0.5 * (pv + pv1);
    }
    acc[0] += pv;
    acc[1] += pv * pv;
    for (int k = 0; k < 4; ++k) acc[2 + k] += g[k];
  }
  of::block_sum<6>(acc, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) partials[(int64_t)blockIdx.x * 6 + k] = acc[k];
}

// heston_single_path_price_delta (mc_aad.rs:239-276): Dual forward mode in s.
__global__ void __launch_bounds__(128) heston_delta_kernel(GreekP P, double* __restrict__ partials) {
  __shared__ double sh[2 * 4];
  double acc[2] = {0, 0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.samples; i += stride) {
    of::Xoshiro256pp rng;
    rng.seed(P.seed + (uint64_t)i * 7919ULL);
    double s = P.spot, ds = 1.0, v = P.v0;
    for (int64_t j = 0; j < P.steps; ++j) {
      const double z1 = of::acklam_inv_cdf(rng.next_f64());
      const double z2 = of::acklam_inv_cdf(rng.next_f64());
      const double v_pos = v > 0.0 ? v : 0.0;
      const double sqrt_v = sqrt(v_pos);
      const double zs = P.rho * z1 + P.rho2 * z2;
      double v_next = v + P.kappa * (P.theta - v_pos) * P.dt + P.xi * sqrt_v * P.sqrt_dt * z1;
      v_next = v_next > 0.0 ? v_next : 0.0;
      const double growth = exp((P.mu - 0.5 * v_pos) * P.dt + sqrt_v * P.sqrt_dt * zs);
      s = s * growth;
      ds = ds * growth;
      v = v_next;
    }
    double pv, dpv;
    const double val = P.call ? s - P.strike : P.strike - s;
    pv = val > 0.0 ? val : 0.0;
    dpv = val > 0.0 ? (P.call ? ds : -ds) : 0.0;
    acc[0] += pv * P.disc;
    acc[1] += dpv * P.disc;
  }
  of::block_sum<2>(acc, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 2; ++k) partials[(int64_t)blockIdx.x * 2 + k] = acc[k];
}

// single_path_contribution (mc_greeks.rs:266-314).
__device__ __forceinline__ void greek_contrib(const GreekP& P, double z, double o[5]) {
  const double growth = exp(fma(P.sig_sqrt_t, z, P.g_drift));
  const double st = P.spot * growth;
  const double pay_v = P.call ? st - P.strike : P.strike - st;
  const double payoff = pay_v > 0.0 ? pay_v : 0.0;
  auto pw = [&](double s) { return P.call ? (s > P.strike ? growth : 0.0) : (s < P.strike ? -growth : 0.0); };
  const double delta_pw = pw(st);
  const double delta_up = pw(P.spot_up * growth);
  const double delta_dn = pw(P.spot_dn * growth);
  const double gamma_pw = (delta_up - delta_dn) / P.spot_span;
  const double inv_svt = 1.0 / (P.spot * P.vol * P.sqrt_t);
  const double z2m1 = z * z - 1.0;
  const double w_delta = z * inv_svt;
  const double inv2 = inv_svt * inv_svt;
  const double w_gamma = z2m1 * inv2 - z * inv_svt / P.spot;
  const double w_vega = (z2m1 - P.vol * P.sqrt_t * z) / P.vol;
  o[0] = delta_pw;
  o[1] = gamma_pw;
  o[2] = payoff * w_delta;
  o[3] = payoff * w_gamma;
  o[4] = payoff * w_vega;
}

__global__ void __launch_bounds__(128) estimators_kernel(GreekP P, double* __restrict__ partials) {
  __shared__ double sh[5 * 4];
  double acc[5] = {0, 0, 0, 0, 0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.samples; i += stride) {
    of::Xoshiro256pp rng;
    rng.seed(P.seed + (uint64_t)i * 7919ULL);
    const double z = of::acklam_inv_cdf(rng.next_f64());
    double b[5];
    greek_contrib(P, z, b);
    if (P.antithetic) {
      double a[5];
      greek_contrib(P, -z, a);
      for (int k = 0; k < 5; ++k) b[k] = 0.5 * (b[k] + a[k]);
    }
    for (int k = 0; k < 5; ++k) acc[k] += b[k];
  }
  of::block_sum<5>(acc, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 5; ++k) partials[(int64_t)blockIdx.x * 5 + k] = acc[k];
}

template <int NS>
of_status launch_and_sum(of_ctx* ctx, void (*kern)(GreekP, double*), const GreekP& P, double sums[NS],
                         double* ms) {
  const int block = 128;
  const int64_t want = (P.samples + block - 1) / block;
  const int64_t cap = (int64_t)ctx->sm_count * of_blocks_per_sm((const void*)kern, block, 0);
  const int grid = (int)(want < cap ? want : cap);
  void *d_part = nullptr, *d_sums = nullptr, *h = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)grid * NS * sizeof(double), &d_part));
  OF_TRY(of_scratch(ctx, SLOT_SUMS, NS * sizeof(double), &d_sums));
  OF_TRY(of_pinned(ctx, NS * sizeof(double), &h));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  kern<<<grid, block, 0, ctx->stream>>>(P, (double*)d_part);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_TRY(of_reduce_rows(ctx, (const double*)d_part, grid, NS, (double*)d_sums));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(h, d_sums, NS * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  float t = 0.0f;
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(&t, ctx->ev_start, ctx->ev_stop));
  std::memcpy(sums, h, NS * sizeof(double));
  *ms = t;
  return OF_OK;
}

of_status check_common(of_ctx* ctx, const of_greeks_params* p, of_greeks_result* out) {
  if (!ctx || !p || !out) return OF_ERR_INVALID_INPUT;
  std::memset(out, 0, sizeof(*out));
  if (p->option_type != OF_CALL && p->option_type != OF_PUT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown option type %d", p->option_type);
  if (!(p->strike > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "vanilla strike must be > 0");
  if (p->num_paths <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths must be > 0");
  if (!(p->spot > 0.0) || !std::isfinite(p->spot)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "market spot must be > 0");
  return OF_OK;
}

}  // namespace

extern "C" of_status of_mc_european_pathwise_aad(of_ctx* ctx, const of_greeks_params* p, of_greeks_result* out) {
  OF_TRY(check_common(ctx, p, out));
  if (p->num_steps <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps must be > 0");
  if (!(p->vol > 0.0) || !std::isfinite(p->vol))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "market volatility must be finite and > 0");
  if (!(p->expiry > 0.0)) {  // mc_aad.rs:98-115
    const double v = p->option_type == OF_CALL ? p->spot - p->strike : p->strike - p->spot;
    out->price = v > 0.0 ? v : 0.0;
    return OF_OK;
  }
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  GreekP P{};
  P.call = p->option_type == OF_CALL;
  P.antithetic = p->antithetic ? 1 : 0;
  P.samples = p->antithetic ? (p->num_paths + 1) / 2 : p->num_paths;
  P.steps = p->num_steps;
  P.seed = p->seed;
  P.spot = p->spot;
  P.strike = p->strike;
  P.rate = p->rate;
  P.q = p->dividend_yield;
  P.vol = p->vol;
  P.expiry = p->expiry;
  P.dt = p->expiry / (double)p->num_steps;
  P.sqrt_dt = std::sqrt(P.dt);
  const double sigma_sq = p->vol * p->vol;
  const double half_sigma_sq = 0.5 * sigma_sq;
  P.drift_inner = (p->rate - p->dividend_yield) - half_sigma_sq;
  P.drift = P.drift_inner * P.dt;
  P.diffusion = p->vol * P.sqrt_dt;
  double s[6], ms = 0.0;
  OF_TRY(launch_and_sum<6>(ctx, aad_kernel, P, s, &ms));
  const double n = (double)P.samples;
  const double mean = s[0] / n;
  const double var = P.samples > 1 ? (s[1] - s[0] * s[0] / n) / (n - 1.0) : 0.0;
  out->price = mean;
  out->stderr_ = std::sqrt(var / n);
  out->delta = s[2] / n;
  out->gamma = 0.0;
  out->vega = s[4] / n;
  out->theta = -(s[5] / n);
  out->rho = s[3] / n;
  out->samples = P.samples;
  out->kernel_ms = ms;
  return OF_OK;
}

extern "C" of_status of_heston_price_delta_aad(of_ctx* ctx, const of_greeks_params* p, of_greeks_result* out) {
  OF_TRY(check_common(ctx, p, out));
  if (p->num_steps <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps must be > 0");
  if (!(p->expiry > 0.0)) {  // mc_aad.rs:303-309
    const double v = p->option_type == OF_CALL ? p->spot - p->strike : p->strike - p->spot;
    out->price = v > 0.0 ? v : 0.0;
    return OF_OK;
  }
  if (!(p->kappa > 0.0 && p->theta >= 0.0 && p->xi >= 0.0 && p->v0 >= 0.0 && p->rho > -1.0 && p->rho < 1.0))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "invalid Heston parameters");
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  GreekP P{};
  P.call = p->option_type == OF_CALL;
  P.samples = p->num_paths;
  P.steps = p->num_steps;
  P.seed = p->seed;
  P.spot = p->spot;
  P.strike = p->strike;
  P.dt = p->expiry / (double)p->num_steps;
  P.sqrt_dt = std::sqrt(P.dt);
  P.rho2 = std::sqrt(1.0 - p->rho * p->rho);
  P.disc = std::exp(-p->rate * p->expiry);
  P.mu = p->mu;
  P.kappa = p->kappa;
  P.theta = p->theta;
  P.xi = p->xi;
  P.rho = p->rho;
  P.v0 = p->v0;
  double s[2], ms = 0.0;
  OF_TRY(launch_and_sum<2>(ctx, heston_delta_kernel, P, s, &ms));
  const double n = (double)p->num_paths;
  out->price = s[0] / n;
  out->delta = s[1] / n;
  out->samples = p->num_paths;
  out->kernel_ms = ms;
  return OF_OK;
}

extern "C" of_status of_mc_greek_estimators(of_ctx* ctx, const of_greeks_params* p, of_greeks_result* out) {
  OF_TRY(check_common(ctx, p, out));
  if (!(p->spot_bump_rel > 0.0) || !std::isfinite(p->spot_bump_rel))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "spot_bump_rel must be finite and > 0");
  if (!(p->expiry > 0.0)) return OF_OK;  // mc_greeks.rs:135-137
  if (!(p->vol > 0.0) || !std::isfinite(p->vol))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "market volatility must be finite and > 0");
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  GreekP P{};
  P.call = p->option_type == OF_CALL;
  P.antithetic = p->antithetic ? 1 : 0;
  P.samples = p->antithetic ? (p->num_paths + 1) / 2 : p->num_paths;
  P.seed = p->seed;
  P.spot = p->spot;
  P.strike = p->strike;
  P.vol = p->vol;
  P.g_drift = (p->rate - p->dividend_yield - 0.5 * p->vol * p->vol) * p->expiry;
  P.sig_sqrt_t = p->vol * std::sqrt(p->expiry);
  P.sqrt_t = std::sqrt(p->expiry);
  const double h = std::fmax(p->spot * p->spot_bump_rel, 1.0e-6);
  P.spot_up = p->spot + h;
  P.spot_dn = std::fmax(p->spot - h, 1.0e-8);
  P.spot_span = P.spot_up - P.spot_dn;
  double s[5], ms = 0.0;
  OF_TRY(launch_and_sum<5>(ctx, estimators_kernel, P, s, &ms));
  const double n = (double)P.samples;
  const double disc = std::exp(-p->rate * p->expiry);
  out->delta = disc * s[0] / n;
  out->gamma = disc * s[1] / n;
  out->lr_delta = disc * s[2] / n;
  out->lr_gamma = disc * s[3] / n;
  out->lr_vega = disc * s[4] / n;
  out->samples = P.samples;
  out->kernel_ms = ms;
  return OF_OK;
}
