// book_greeks.cuh - per-sample kernels of the batched book's Greeks modes.
//
// Two modes share this code and the same draws:
//   R = float,  G = true : price and the pathwise Greeks of a GBM option
//                          (delta, vega, rho, theta), FP32 path arithmetic;
//   R = double, G = false: price only, FP64 path arithmetic on the same
//                          Philox draws (the revaluations of a bump-and-
//                          revalue check with common random numbers).
//
// The Greeks are the ones of MonteCarloPricingEngine::price_with_greeks_aad
// (src/engines/monte_carlo/mc_engine.rs:977-987 -> mc_european_pathwise_aad,
// src/engines/monte_carlo/mc_aad.rs:15-219): d PV / d(S0, sigma, r) and
// theta = -d PV / dT with the step count fixed (dt = T / steps), the rate
// entering the drift r - q and the discount exp(-r T).  The reference's tape
// differentiates exp(drift + diffusion z) step by step; for GBM every step's
// adjoint collapses to closed forms in the path's log-returns y_i:
//   dy_i/dsigma = (y_i - a t_i) / sigma - sigma t_i,  dy_i/dr = t_i,
//   dy_i/dT = (y_i + a t_i) / (2T),                   a = r - q - sigma^2/2,
// so a vanilla needs y_T only and an arithmetic average needs three running
// sums (sum w S, sum w S y, sum w S i), a geometric one sum w y.
//
// A discretely monitored barrier has a payoff that jumps where a path
// touches the barrier; its pathwise derivative misses the jump.  The barrier
// options are priced here by one-step survival (Glasserman & Staum, "Conditioning
// on one-step survival for barrier option simulations", Oper. Res. 49, 2001):
// at every step the next log-return is drawn conditioned to stay on the alive
// side of the barrier, z = Phi^-1(u p) with p = Phi(h) the probability of
// staying alive over the step, and the path carries the weight L = prod p.
// A knock-out pays L f(S_T) + (1 - L) R, a knock-in f(S_T') - L (f(S_T) - R)
// with S_T' the unconditioned path of the same uniforms.  Both estimators
// are unbiased for the discretely monitored price, and smooth in the
// parameters, so their pathwise derivatives (forward tangents of y and ln L
// through every step) are unbiased too.
#pragma once

#include <type_traits>

#include "mills_coeffs.h"
#include "of_device.cuh"

namespace of {

// The book's Greeks-mode kinds (which step loop an option takes).
enum : int32_t { GK_TERMINAL = 0, GK_ASIAN_DAILY = 1, GK_ASIAN_WEIGHTS = 2, GK_BARRIER_OUT = 3, GK_BARRIER_IN = 4 };
enum : int32_t {
  GF_CALL = 1,
  GF_ANTI = 2,
  GF_FLOATING = 4,       // Asian floating strike: max(+-(S_T - avg), 0)
  GF_GEOMETRIC = 8,      // Asian geometric average
  GF_TERMINAL_ONLY = 16  // Asian with no observations: the terminal spot is the average
};
// Control variates of the Greeks modes (the price only; the Greeks carry none).
enum : int32_t { GCV_NONE = 0, GCV_VANILLA_TERMINAL = 1, GCV_GEOMETRIC_ASIAN = 2, GCV_TERMINAL_SPOT = 3 };

// Per-option constants in the path's arithmetic type R, built on the host
// in FP64 and rounded once.
template <typename R>
struct GreekConsts {
  R alpha, beta;        // per step: log drift (r - q - sigma^2/2) dt and sigma sqrt(dt)
  R a, dt, T, sigma, r, df;
  R s0, strike, rebate;
  R inv_n;              // Asian: 1 / number of observations
  R w1;                 // Asian: sum_i w_i i over the observed step indices
  R bar, sgn, sib;      // barrier: log(B/S0); +1 up, -1 down; sgn / beta
  // tangent coefficients (parameters in the order ln S0, sigma, r, T)
  R sig_dt, inv_sig, beta_over_sig, alpha_over_T, inv_2T, beta_over_2T;
  int32_t kind, flags, steps, obs_offset, cv_kind;
  uint32_t stream;
};

// One sample (antithetic pairs averaged): the undiscounted payoff x, the
// control variate y, and the discounted pathwise derivatives
// g = (delta, vega, rho, theta) of df x.
template <typename R>
struct GreekSample {
  R x, y;
  R g[4];
};

template <typename R>
struct GMath;

template <>
struct GMath<float> {
  static constexpr float kTiny = 1e-30f;  // floor of the survival-draw uniform (above FLT_MIN)
  static constexpr float kHMin = -12.0f;  // Phi(-12) = 1.8e-33 is still a normal float
  static __device__ __forceinline__ float exp(float x) { return __expf(x); }
  // Phi(h) and phi(h) / Phi(h): the normal tail Phi(-|h|) = phi(|h|) M(|h|)
  // with the fitted Mills ratio M of mills_coeffs.h (Hastings' form) and
  // phi from an exact split of h^2, so that the tail keeps its relative
  // precision; for h < 0 the ratio is 1 / M.
  static __device__ __forceinline__ void cdf_ratio(float h, float& p, float& g) {
    const float a = fabsf(h);
    const float t = 1.0f / fmaf(OF_MILLS_C, a, 1.0f);
    float m = kMills[OF_MILLS_DEG];
#pragma unroll
    for (int i = OF_MILLS_DEG - 1; i >= 0; --i) m = fmaf(m, t, kMills[i]);
    m *= t;
    const float a2 = a * a, a2lo = fmaf(a, a, -a2);  // a^2 = a2 + a2lo exactly
    const float phi = 0.398942280401432677939946f * __expf(-0.5f * a2) * fmaf(-0.5f, a2lo, 1.0f);
    const float tail = phi * m;
    p = h < 0.0f ? tail : 1.0f - tail;
    g = h < 0.0f ? 1.0f / m : phi / p;
  }
  // Phi^-1(v) with q = 1 - v: the fitted single-log inverse of the Philox kernels
  static __device__ __forceinline__ float icdf2(float v, float q) { return inv_normal_vq(v, q); }
  static __device__ __forceinline__ float unif(uint32_t r) { return uniform_from_u32(r); }
  static __device__ __forceinline__ void pair(uint32_t a, uint32_t b, float& z1, float& z2) {
    const float2 p = normal_pair_from_u32(a, b);
    z1 = p.x;
    z2 = p.y;
  }
};

template <>
struct GMath<double> {
  static constexpr double kTiny = 1e-300;
  static constexpr double kHMin = -37.0;
  static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
  static __device__ __forceinline__ void cdf_ratio(double h, double& p, double& g) {
    p = ::normcdf(h);
    g = 0.398942280401432677939946 * ::exp(-0.5 * h * h) / p;
  }
  static __device__ __forceinline__ double icdf2(double v, double q) {
    return v <= 0.5 ? ::normcdfinv(v) : -::normcdfinv(q);
  }
  // the grid of uniform_from_u32: (k + 0.5) 2^-23, k = the top 23 bits (exact in either type)
  static __device__ __forceinline__ double unif(uint32_t r) { return ((double)(r >> 9) + 0.5) * 0x1p-23; }
  // normal_pair_from_u32's transform in FP64: radius sqrt(-2 ln u1), angle pi (2 f - 3)
  static __device__ __forceinline__ void pair(uint32_t a, uint32_t b, double& z1, double& z2) {
    const double rad = ::sqrt(-2.0 * ::log(unif(a)));
    const double f = 1.0 + (double)(b >> 9) * 0x1p-23;
    double s, c;
    ::sincospi(2.0 * f - 3.0, &s, &c);
    z1 = rad * c;
    z2 = rad * s;
  }
};

// The four draws of Philox block q of sample i: Box-Muller normals (the
// book's draws for GBM steps) or uniforms (survival draws).
template <typename R>
__device__ __forceinline__ void gk_normals(const GreekConsts<R>& c, uint32_t q, uint32_t lo, uint32_t hi,
                                           const PhiloxKeys& K, R (&z)[4]) {
  const uint4 r = philox4x32_10(make_uint4(q, lo, hi, c.stream), K);
  GMath<R>::pair(r.x, r.y, z[0], z[1]);
  GMath<R>::pair(r.z, r.w, z[2], z[3]);
}

template <typename R>
__device__ __forceinline__ void gk_uniforms(const GreekConsts<R>& c, uint32_t q, uint32_t lo, uint32_t hi,
                                            const PhiloxKeys& K, R (&u)[4]) {
  const uint4 r = philox4x32_10(make_uint4(q, lo, hi, c.stream), K);
  u[0] = GMath<R>::unif(r.x);
  u[1] = GMath<R>::unif(r.y);
  u[2] = GMath<R>::unif(r.z);
  u[3] = GMath<R>::unif(r.w);
}

// The terminal spot S_T = s0 e^y and its derivatives along (ln S0, sigma, r, T)
// for an unconditioned GBM path.
template <typename R>
__device__ __forceinline__ R gk_spot(const GreekConsts<R>& c, R y, R (&d)[4]) {
  const R s = c.s0 * GMath<R>::exp(y);
  d[0] = s;
  d[1] = s * ((y - c.a * c.T) * c.inv_sig - c.sigma * c.T);
  d[2] = s * c.T;
  d[3] = s * (y + c.a * c.T) * c.inv_2T;
  return s;
}

// f = max(phi (u - v), 0) and, where G, its derivative df = phi (du - dv) on
// the exercised side (0 elsewhere).
template <typename R, bool G>
__device__ __forceinline__ R gk_vanilla(bool call, R u, R v, const R (&du)[4], const R (&dv)[4], R (&df)[4]) {
  const R diff = call ? u - v : v - u;
  const R f = diff > (R)0 ? diff : (R)0;
  if (G) {
    const R m = diff > (R)0 ? (call ? (R)1 : (R)-1) : (R)0;
#pragma unroll
    for (int t = 0; t < 4; ++t) df[t] = m * (du[t] - dv[t]);
  }
  return f;
}

// Discounted Greeks of one leg from its undiscounted payoff x and dx along
// (ln S0, sigma, r, T): delta = df dx0 / s0, vega = df dx1,
// rho = df dx2 - T df x, theta = -(df dx3 - r df x).
template <typename R>
__device__ __forceinline__ void gk_discount(const GreekConsts<R>& c, R x, const R (&dx)[4], R (&g)[4]) {
  const R pv = c.df * x;
  g[0] = c.df * dx[0] / c.s0;
  g[1] = c.df * dx[1];
  g[2] = c.df * dx[2] - c.T * pv;
  g[3] = c.r * pv - c.df * dx[3];
}

// ---- vanilla / terminal-only Asian: the path needs y_T only --------------
template <typename R, bool G, bool ANTI>
__device__ __forceinline__ void gk_terminal_finish(const GreekConsts<R>& c, R w, GreekSample<R>& out);

template <typename R, bool G, bool ANTI>
__device__ __forceinline__ void gk_terminal(const GreekConsts<R>& c, uint64_t i, const PhiloxKeys& K,
                                            GreekSample<R>& out) {
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  R w = (R)0;  // sum of the path's normals
  const int32_t full = c.steps & ~3;
  if constexpr (std::is_same<R, float>::value) {
    // each Box-Muller pair as its sum, sqrt(2) r sin(t + pi/4); a partial
    // block of one or three steps adds its odd normal from the plain
    // transform.  The FP64 modes add the pair's two normals: the same draws.
    for (int32_t j = 0; j < full; j += 4) {
      const uint4 r = philox4x32_10(make_uint4((uint32_t)(j >> 2), lo, hi, c.stream), K);
      w += normal_pair_sum_from_u32(r.x, r.y) + normal_pair_sum_from_u32(r.z, r.w);
    }
    const int32_t rem = c.steps - full;
    if (rem > 0) {
      const uint4 r = philox4x32_10(make_uint4((uint32_t)(full >> 2), lo, hi, c.stream), K);
      if (rem == 1) {
        w += normal_pair_from_u32(r.x, r.y).x;
      } else {
        w += normal_pair_sum_from_u32(r.x, r.y);
        if (rem == 3) w += normal_pair_from_u32(r.z, r.w).x;
      }
    }
  } else {
    for (int32_t j = 0; j < full; j += 4) {
      R z[4];
      gk_normals(c, (uint32_t)(j >> 2), lo, hi, K, z);
      w += (z[0] + z[1]) + (z[2] + z[3]);
    }
    if (full < c.steps) {
      R z[4];
      gk_normals(c, (uint32_t)(full >> 2), lo, hi, K, z);
      w += z[0];
      if (full + 1 < c.steps) w += z[1];
      if (full + 2 < c.steps) w += z[2];
    }
  }
  gk_terminal_finish<R, G, ANTI>(c, w, out);
}

// The payoff, control variate and discounted Greeks of a terminal-only
// sample from the sum w of its normals (and -w for the antithetic twin).
template <typename R, bool G, bool ANTI>
__device__ __forceinline__ void gk_terminal_finish(const GreekConsts<R>& c, R w, GreekSample<R>& out) {
  const R base = (R)c.steps * c.alpha;
  const bool call = c.flags & GF_CALL;
  const bool floating = (c.flags & GF_TERMINAL_ONLY) && (c.flags & GF_FLOATING);
  R xs = (R)0, ys = (R)0, gs[4] = {(R)0, (R)0, (R)0, (R)0};
#pragma unroll
  for (int leg = 0; leg < (ANTI ? 2 : 1); ++leg) {
    const R y = leg == 0 ? base + c.beta * w : base - c.beta * w;
    R ds[4], dk[4] = {(R)0, (R)0, (R)0, (R)0}, dx[4];
    const R s = gk_spot(c, y, ds);
    // a floating-strike Asian on the terminal spot alone pays max(+-(S_T - S_T), 0) = 0
    const R x = floating ? (R)0 : gk_vanilla<R, G>(call, s, c.strike, ds, dk, dx);
    if (floating)
      for (int t = 0; t < 4; ++t) dx[t] = (R)0;
    R y_cv = (R)0;
    if (c.cv_kind == GCV_VANILLA_TERMINAL || c.cv_kind == GCV_GEOMETRIC_ASIAN)
      y_cv = call ? (s > c.strike ? s - c.strike : (R)0) : (c.strike > s ? c.strike - s : (R)0);
    else if (c.cv_kind == GCV_TERMINAL_SPOT)
      y_cv = s;
    xs += x;
    ys += y_cv;
    if (G) {
      R g[4];
      gk_discount(c, x, dx, g);
#pragma unroll
      for (int t = 0; t < 4; ++t) gs[t] += g[t];
    }
  }
  const R h = ANTI ? (R)0.5 : (R)1;
  out.x = h * xs;
  out.y = h * ys;
#pragma unroll
  for (int t = 0; t < 4; ++t) out.g[t] = h * gs[t];
}

// ---- Asian: running sums of the observed spots ----------------------------
template <typename R>
struct AsianLeg {
  R y;
  R p0, p0c;  // sum w e^y (compensated in FP32)
  R p1, p2;   // sum w e^y y, sum w e^y i
  R q;        // sum w y
};

template <typename R, bool G, bool NEED_ARITH, bool NEED_GEO>
__device__ __forceinline__ void gk_observe(AsianLeg<R>& L, R w, R idx) {
  if (NEED_ARITH) {
    const R e = w * GMath<R>::exp(L.y);
    const R yk = e - L.p0c;
    const R t = L.p0 + yk;
    L.p0c = (t - L.p0) - yk;
    L.p0 = t;
    if (G) {
      L.p1 = fma(e, L.y, L.p1);
      L.p2 = fma(e, idx, L.p2);
    }
  }
  if (NEED_GEO) L.q = fma(w, L.y, L.q);
}

// The payoff, control variate and discounted Greeks of an Asian sample from
// its leg(s) (B is the antithetic twin when ANTI).
template <typename R, bool G, bool ANTI, bool NEED_GEO>
__device__ __forceinline__ void gk_asian_finish(const GreekConsts<R>& c, const AsianLeg<R>& A, const AsianLeg<R>& B,
                                                GreekSample<R>& out) {
  const bool call = c.flags & GF_CALL;
  const bool floating = c.flags & GF_FLOATING;
  R xs = (R)0, ys = (R)0, gs[4] = {(R)0, (R)0, (R)0, (R)0};
#pragma unroll
  for (int leg = 0; leg < (ANTI ? 2 : 1); ++leg) {
    const AsianLeg<R>& L = leg == 0 ? A : B;
    R ds[4], da[4], dg[4], dk[4] = {(R)0, (R)0, (R)0, (R)0}, dx[4];
    const R s = gk_spot(c, L.y, ds);
    R geo = (R)0;
    if (NEED_GEO) {  // G = s0 exp(q / n); d/dtheta = G sum_i w_i dy_i/dtheta / n
      geo = c.s0 * GMath<R>::exp(L.q * c.inv_n);
      dg[0] = geo;
      dg[1] = geo * c.inv_n * (L.q * c.inv_sig - (c.a * c.inv_sig + c.sigma) * c.dt * c.w1);
      dg[2] = geo * c.inv_n * c.dt * c.w1;
      dg[3] = geo * c.inv_n * (L.q + c.a * c.dt * c.w1) * c.inv_2T;
    }
    R avg;
    if (c.flags & GF_GEOMETRIC) {
      avg = geo;
#pragma unroll
      for (int t = 0; t < 4; ++t) da[t] = dg[t];
    } else {
      const R sn = c.s0 * c.inv_n;
      avg = sn * (L.p0 - L.p0c);
      if (G) {
        da[0] = avg;
        da[1] = sn * (L.p1 * c.inv_sig - (c.a * c.inv_sig + c.sigma) * c.dt * L.p2);
        da[2] = sn * c.dt * L.p2;
        da[3] = sn * (L.p1 + c.a * c.dt * L.p2) * c.inv_2T;
      }
    }
    const R x = floating ? gk_vanilla<R, G>(call, s, avg, ds, da, dx) : gk_vanilla<R, G>(call, avg, c.strike, da, dk, dx);
    R y_cv = (R)0;
    if (c.cv_kind == GCV_VANILLA_TERMINAL)
      y_cv = call ? (s > c.strike ? s - c.strike : (R)0) : (c.strike > s ? c.strike - s : (R)0);
    else if (c.cv_kind == GCV_GEOMETRIC_ASIAN)
      y_cv = call ? (geo > c.strike ? geo - c.strike : (R)0) : (c.strike > geo ? c.strike - geo : (R)0);
    else if (c.cv_kind == GCV_TERMINAL_SPOT)
      y_cv = s;
    xs += x;
    ys += y_cv;
    if (G) {
      R g[4];
      gk_discount(c, x, dx, g);
#pragma unroll
      for (int t = 0; t < 4; ++t) gs[t] += g[t];
    }
  }
  const R h = ANTI ? (R)0.5 : (R)1;
  out.x = h * xs;
  out.y = h * ys;
#pragma unroll
  for (int t = 0; t < 4; ++t) out.g[t] = h * gs[t];
}

template <typename R, bool G, bool ANTI, bool DAILY, bool NEED_ARITH, bool NEED_GEO>
__device__ __forceinline__ void gk_asian(const GreekConsts<R>& c, uint64_t i, const PhiloxKeys& K,
                                         const float* __restrict__ obs_w, GreekSample<R>& out) {
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  AsianLeg<R> A{}, B{};
  if (!DAILY) {  // an observation at t = 0: e^0 = 1, y = 0, i = 0
    const R w0 = (R)__ldg(obs_w + c.obs_offset);
    if (NEED_ARITH) A.p0 = B.p0 = w0;
  }
  R idx = (R)0;
  auto step = [&](R z, int32_t j) {
    idx += (R)1;
    A.y = fma(c.beta, z, A.y + c.alpha);
    if (ANTI) B.y = fma(-c.beta, z, B.y + c.alpha);
    const R w = DAILY ? (R)1 : (R)__ldg(obs_w + c.obs_offset + j + 1);
    if (DAILY || w != (R)0) {
      gk_observe<R, G, NEED_ARITH, NEED_GEO>(A, w, idx);
      if (ANTI) gk_observe<R, G, NEED_ARITH, NEED_GEO>(B, w, idx);
    }
  };
  const int32_t full = c.steps & ~3;
  for (int32_t j = 0; j < full; j += 4) {
    R z[4];
    gk_normals(c, (uint32_t)(j >> 2), lo, hi, K, z);
    step(z[0], j);
    step(z[1], j + 1);
    step(z[2], j + 2);
    step(z[3], j + 3);
  }
  if (full < c.steps) {
    R z[4];
    gk_normals(c, (uint32_t)(full >> 2), lo, hi, K, z);
    step(z[0], full);
    if (full + 1 < c.steps) step(z[1], full + 1);
    if (full + 2 < c.steps) step(z[2], full + 2);
  }
  gk_asian_finish<R, G, ANTI, NEED_GEO>(c, A, B, out);
}

// gk_terminal<float, G, ANTI> of samples i0 and i1: the normals' sums in
// packed pairs, in the scalar loop's order (each half bit for bit the scalar
// sum).
template <bool G, bool ANTI>
__device__ __forceinline__ void gk_terminal_pair(const GreekConsts<float>& c, uint64_t i0, uint64_t i1,
                                                 const PhiloxKeys& K, GreekSample<float>& o0, GreekSample<float>& o1) {
  const uint32_t lo0 = (uint32_t)i0, hi0 = (uint32_t)(i0 >> 32), lo1 = (uint32_t)i1, hi1 = (uint32_t)(i1 >> 32);
  float2 w = make_float2(0.0f, 0.0f);
  const int32_t full = c.steps & ~3;
  for (int32_t j = 0; j < full; j += 4) {
    const uint4 r0 = philox4x32_10(make_uint4((uint32_t)(j >> 2), lo0, hi0, c.stream), K);
    const uint4 r1 = philox4x32_10(make_uint4((uint32_t)(j >> 2), lo1, hi1, c.stream), K);
    w = add2(w, add2(normal_pair_sums2_from_u32(r0.x, r0.y, r1.x, r1.y),
                     normal_pair_sums2_from_u32(r0.z, r0.w, r1.z, r1.w)));
  }
  const int32_t rem = c.steps - full;
  if (rem > 0) {
    const uint4 r0 = philox4x32_10(make_uint4((uint32_t)(full >> 2), lo0, hi0, c.stream), K);
    const uint4 r1 = philox4x32_10(make_uint4((uint32_t)(full >> 2), lo1, hi1, c.stream), K);
    float2 a1, a2;
    if (rem == 1) {
      normal_pairs_scaled2_from_u32(r0.x, r0.y, r1.x, r1.y, kBoxMullerK2, a1, a2);
      w = add2(w, a1);
    } else {
      w = add2(w, normal_pair_sums2_from_u32(r0.x, r0.y, r1.x, r1.y));
      if (rem == 3) {
        normal_pairs_scaled2_from_u32(r0.z, r0.w, r1.z, r1.w, kBoxMullerK2, a1, a2);
        w = add2(w, a1);
      }
    }
  }
  gk_terminal_finish<float, G, ANTI>(c, w.x, o0);
  gk_terminal_finish<float, G, ANTI>(c, w.y, o1);
}

// ---- Asian legs in packed pairs (FP32) -------------------------------------
// Two Asian legs per FP32 instruction: two samples, or a sample and its
// antithetic twin.  Each half is gk_asian's arithmetic bit for bit.
struct AsianLeg2 {
  float2 y, p0, p0c, p1, p2, q;
};

template <bool G, bool NEED_ARITH, bool NEED_GEO>
__device__ __forceinline__ void gk_observe2(AsianLeg2& L, float w, float idx) {
  if (NEED_ARITH) {
    const float2 e = mul2(splat2(w), make_float2(__expf(L.y.x), __expf(L.y.y)));
    const float2 yk = sub2(e, L.p0c);
    const float2 t = add2(L.p0, yk);
    L.p0c = sub2(sub2(t, L.p0), yk);
    L.p0 = t;
    if (G) {
      L.p1 = fma2(e, L.y, L.p1);
      L.p2 = fma2(e, splat2(idx), L.p2);
    }
  }
  if (NEED_GEO) L.q = fma2(splat2(w), L.y, L.q);
}

__device__ __forceinline__ AsianLeg<float> asian_half(const AsianLeg2& L, int e) {
  AsianLeg<float> o;
  o.y = e ? L.y.y : L.y.x;
  o.p0 = e ? L.p0.y : L.p0.x;
  o.p0c = e ? L.p0c.y : L.p0c.x;
  o.p1 = e ? L.p1.y : L.p1.x;
  o.p2 = e ? L.p2.y : L.p2.x;
  o.q = e ? L.q.y : L.q.x;
  return o;
}

// The step loop of gk_asian<float, G, ...> for two legs.  TWIN: sample i0 and
// its antithetic twin (one stream, normals z and -z); otherwise samples i0
// and i1.
template <bool G, bool TWIN, bool DAILY, bool NEED_ARITH, bool NEED_GEO>
__device__ __forceinline__ void gk_asian_legs2(const GreekConsts<float>& c, uint64_t i0, uint64_t i1,
                                               const PhiloxKeys& K, const float* __restrict__ obs_w, AsianLeg2& L) {
  const uint32_t lo0 = (uint32_t)i0, hi0 = (uint32_t)(i0 >> 32), lo1 = (uint32_t)i1, hi1 = (uint32_t)(i1 >> 32);
  L = AsianLeg2{};
  if (!DAILY) {
    const float w0 = __ldg(obs_w + c.obs_offset);
    if (NEED_ARITH) L.p0 = splat2(w0);
  }
  const float2 beta = TWIN ? make_float2(c.beta, -c.beta) : splat2(c.beta);
  float idx = 0.0f;
  auto step = [&](float2 z, int32_t j) {
    idx += 1.0f;
    L.y = fma2(beta, z, add2(L.y, splat2(c.alpha)));
    const float w = DAILY ? 1.0f : __ldg(obs_w + c.obs_offset + j + 1);
    if (DAILY || w != 0.0f) gk_observe2<G, NEED_ARITH, NEED_GEO>(L, w, idx);
  };
  for (int32_t j = 0; j < c.steps; j += 4) {
    const uint4 r0 = philox4x32_10(make_uint4((uint32_t)(j >> 2), lo0, hi0, c.stream), K);
    float2 w1, w2, w3, w4;
    if (TWIN) {  // w1 = (z_j, z_j+2), w2 = (z_j+1, z_j+3)
      normal_pairs_scaled2_from_u32(r0.x, r0.y, r0.z, r0.w, kBoxMullerK2, w1, w2);
      w3 = splat2(w1.y);
      w4 = splat2(w2.y);
      w1 = splat2(w1.x);
      w2 = splat2(w2.x);
    } else {
      const uint4 r1 = philox4x32_10(make_uint4((uint32_t)(j >> 2), lo1, hi1, c.stream), K);
      normal_pairs_scaled2_from_u32(r0.x, r0.y, r1.x, r1.y, kBoxMullerK2, w1, w2);
      normal_pairs_scaled2_from_u32(r0.z, r0.w, r1.z, r1.w, kBoxMullerK2, w3, w4);
    }
    step(w1, j);
    if (j + 1 < c.steps) step(w2, j + 1);
    if (j + 2 < c.steps) step(w3, j + 2);
    if (j + 3 < c.steps) step(w4, j + 3);
  }
}

template <bool G, bool DAILY, bool NEED_ARITH, bool NEED_GEO>
__device__ __forceinline__ void gk_asian_twin(const GreekConsts<float>& c, uint64_t i, const PhiloxKeys& K,
                                              const float* __restrict__ obs_w, GreekSample<float>& out) {
  AsianLeg2 L;
  gk_asian_legs2<G, true, DAILY, NEED_ARITH, NEED_GEO>(c, i, i, K, obs_w, L);
  gk_asian_finish<float, G, true, NEED_GEO>(c, asian_half(L, 0), asian_half(L, 1), out);
}

template <bool G, bool DAILY, bool NEED_ARITH, bool NEED_GEO>
__device__ __forceinline__ void gk_asian_pair(const GreekConsts<float>& c, uint64_t i0, uint64_t i1,
                                              const PhiloxKeys& K, const float* __restrict__ obs_w,
                                              GreekSample<float>& o0, GreekSample<float>& o1) {
  AsianLeg2 L;
  gk_asian_legs2<G, false, DAILY, NEED_ARITH, NEED_GEO>(c, i0, i1, K, obs_w, L);
  const AsianLeg<float> a = asian_half(L, 0), b = asian_half(L, 1);
  gk_asian_finish<float, G, false, NEED_GEO>(c, a, a, o0);
  gk_asian_finish<float, G, false, NEED_GEO>(c, b, b, o1);
}

// ---- barrier: one-step survival -------------------------------------------
template <typename R, bool G>
struct SurvLeg {
  R y, L;    // log-return of the conditioned path and its survival weight
  R ypl;     // knock-in: the unconditioned path of the same uniforms
  R e[3];    // tangent basis (u, y, z of surv_step, each times sib)
  R le[3];   // the matching sums for ln L
};

template <typename R, bool G>
__device__ __forceinline__ void surv_init(SurvLeg<R, G>& s, const GreekConsts<R>& c) {
  s.y = (R)0;
  s.ypl = (R)0;
  s.L = c.sgn * c.bar > (R)0 ? (R)1 : (R)0;  // the scan includes path[0]: a spot already beyond the barrier is out
  s.e[0] = s.e[1] = c.sib;
  s.e[2] = (R)0;
#pragma unroll
  for (int t = 0; t < 3; ++t) s.le[t] = (R)0;
}

// One step: h = sgn (bar - y - alpha) / beta is the standardised distance to
// the barrier, p = Phi(h) the probability of staying alive, and the step's
// normal is drawn from the alive side, z = sgn Phi^-1(u p).  Tangents (for
// each parameter with b' = d bar, alpha', beta'):
//   h' = sgn (b' - y' - alpha') / beta - h beta' / beta,
//   (ln p)' = g h' with g = phi(h) / p,
//   z' = sgn u p' / phi(Phi^-1(u p)) = sgn w h',   w = u phi(h) / phi(zeta),
//   y_next' = y' + alpha' + beta' z + beta z'.
// w = u exp((zeta - h)(zeta + h) / 2) in [0, 1] (the Mills ratio Phi / phi
// increases and zeta <= h).  Written this way its exponent is small where a
// draw lands at the barrier (u -> 1, zeta -> h), the steps whose w ~ 1 carries
// the barrier's sensitivity into y', so that w keeps its relative precision
// there; the relative error of w adds up over the steps near the barrier.
//
// The four parameters share one linear recursion.  With sib = sgn / beta,
// A = b' - alpha' and B = -beta' / beta, the parameter's e = A - y' obeys
//   h' = sib e + B h,   e_next = (1 - w) e + B beta sgn (zeta - w h) - alpha',
// and here alpha' = -A for sigma, r and T (the barrier does not move with
// them), while ln S0 has A = -1 and alpha' = B = 0.  So every e is a fixed
// combination of three sequences, kept scaled by sib:
//   u_next = (1 - w) u,                 u_0 = sib   (ln S0: e = -u / sib)
//   y_next = (1 - w) y + sib,           y_0 = sib   (e = A y / sib + B z / sib)
//   z_next = (1 - w) z + zeta - w h,    z_0 = 0
// with (ln L)' = -sum g u (ln S0) or A sum g y + B sum g (z + h): six running
// values in place of eight, and no per-parameter arithmetic in the step.
// surv_tangents turns them into y' and (ln L)' for the payoff.
template <typename R, bool G, bool IN>
__device__ __forceinline__ void surv_step(SurvLeg<R, G>& s, const GreekConsts<R>& c, R u) {
  R h = fma(-c.sib, s.y, c.sib * (c.bar - c.alpha));
  h = h > GMath<R>::kHMin ? h : GMath<R>::kHMin;
  R p, g;  // Phi(h) and phi(h) / Phi(h)
  GMath<R>::cdf_ratio(h, p, g);
  R v = u * p;
  R q = fma(-u, p, (R)1);  // 1 - u p with one rounding
  v = v > GMath<R>::kTiny ? v : GMath<R>::kTiny;
  q = q > GMath<R>::kTiny ? q : GMath<R>::kTiny;
  const R zeta = GMath<R>::icdf2(v, q);
  if (G) {
    const R zmh = zeta - h;
    const R w = u * GMath<R>::exp((R)0.5 * zmh * (zeta + h));
    const R kap = (R)1 - w;
    s.le[0] = fma(g, s.e[0], s.le[0]);
    s.le[1] = fma(g, s.e[1], s.le[1]);
    s.le[2] = fma(g, s.e[2] + h, s.le[2]);
    s.e[0] = kap * s.e[0];
    s.e[1] = fma(kap, s.e[1], c.sib);
    s.e[2] = fma(kap, s.e[2], fma(kap, h, zmh));  // zeta - w h = (zeta - h) + (1 - w) h
  }
  s.y = fma(c.beta * c.sgn, zeta, s.y + c.alpha);
  s.L *= p;
  if (IN) s.ypl = fma(c.beta, GMath<R>::icdf2(u, (R)1 - u), s.ypl + c.alpha);
}

// y' and (ln L)' along (ln S0, sigma, r, T) from the tangent basis: with
// A = (-1, sigma dt, -dt, -alpha / T), B = (0, -1 / sigma, 0, -1 / (2T)) and
// the basis unscaled by beta sgn = 1 / sib,
//   ln S0: y' = u - 1, (ln L)' = -lu;   others: y' = A (1 - y) - B z,
//   (ln L)' = A ly + B lz.
template <typename R, bool G>
__device__ __forceinline__ void surv_tangents(const SurvLeg<R, G>& s, const GreekConsts<R>& c, R (&yd)[4],
                                              R (&ld)[4]) {
  const R bs = c.beta * c.sgn;
  const R uu = bs * s.e[0], yy = (R)1 - bs * s.e[1], zz = bs * s.e[2];
  yd[0] = uu - (R)1;
  ld[0] = -s.le[0];
  yd[1] = fma(c.sig_dt, yy, c.inv_sig * zz);
  ld[1] = fma(c.sig_dt, s.le[1], -c.inv_sig * s.le[2]);
  yd[2] = -c.dt * yy;
  ld[2] = -c.dt * s.le[1];
  yd[3] = fma(-c.alpha_over_T, yy, c.inv_2T * zz);
  ld[3] = fma(-c.alpha_over_T, s.le[1], -c.inv_2T * s.le[2]);
}

template <typename R, bool G, bool IN>
__device__ __forceinline__ void surv_payoff(const SurvLeg<R, G>& s, const GreekConsts<R>& c, R& x, R (&g)[4]) {
  const bool call = c.flags & GF_CALL;
  R ds[4], dk[4] = {(R)0, (R)0, (R)0, (R)0}, dfo[4], dx[4];
  const R so = c.s0 * GMath<R>::exp(s.y);
  R yd[4], ld[4];
  if (G) {  // S = s0 e^y with y depending on ln S0 through the barrier: dS/dlnS0 = S (1 + y')
    surv_tangents(s, c, yd, ld);
    ds[0] = so * ((R)1 + yd[0]);
#pragma unroll
    for (int t = 1; t < 4; ++t) ds[t] = so * yd[t];
  }
  const R fo = gk_vanilla<R, G>(call, so, c.strike, ds, dk, dfo);
  if (!IN) {
    x = s.L * fo + ((R)1 - s.L) * c.rebate;  // L f + (1 - L) R
    if (G) {
#pragma unroll
      for (int t = 0; t < 4; ++t) dx[t] = s.L * fma(ld[t], fo - c.rebate, dfo[t]);
    }
  } else {
    R dp[4], dfp[4];
    const R sp = gk_spot(c, s.ypl, dp);
    const R fp = gk_vanilla<R, G>(call, sp, c.strike, dp, dk, dfp);
    x = fp - s.L * (fo - c.rebate);  // f(S') - L (f(S) - R)
    if (G) {
#pragma unroll
      for (int t = 0; t < 4; ++t) dx[t] = dfp[t] - s.L * fma(ld[t], fo - c.rebate, dfo[t]);
    }
  }
  if (G) gk_discount(c, x, dx, g);
}

template <typename R, bool G, bool ANTI, bool IN>
__device__ __forceinline__ void gk_barrier(const GreekConsts<R>& c, uint64_t i, const PhiloxKeys& K,
                                           GreekSample<R>& out) {
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  SurvLeg<R, G> A, B;
  surv_init(A, c);
  if (ANTI) surv_init(B, c);
  for (int32_t j = 0; j < c.steps; j += 4) {
    R u[4];
    gk_uniforms(c, (uint32_t)(j >> 2), lo, hi, K, u);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (j + q >= c.steps) break;
      surv_step<R, G, IN>(A, c, u[q]);
      if (ANTI) surv_step<R, G, IN>(B, c, (R)1 - u[q]);  // antithetic in the uniform
    }
  }
  R x, g[4];
  surv_payoff<R, G, IN>(A, c, x, g);
  out.x = x;
  out.y = (R)0;
#pragma unroll
  for (int t = 0; t < 4; ++t) out.g[t] = g[t];
  if (ANTI) {
    surv_payoff<R, G, IN>(B, c, x, g);
    out.x = (R)0.5 * (out.x + x);
#pragma unroll
    for (int t = 0; t < 4; ++t) out.g[t] = (R)0.5 * (out.g[t] + g[t]);
  }
}

// ---- dispatch ---------------------------------------------------------------
// Kind groups: each is priced by a persistent launch of its own, so that the
// registers of the survival step (the largest) do not set the occupancy of
// the vanilla and Asian loops.
enum : int { KG_TERMINAL = 0, KG_ASIAN = 1, KG_BARRIER = 2, KG_COUNT = 3 };

__host__ __device__ __forceinline__ int gk_group(int kind) {
  return kind == GK_TERMINAL ? KG_TERMINAL : (kind == GK_ASIAN_DAILY || kind == GK_ASIAN_WEIGHTS) ? KG_ASIAN
                                                                                                  : KG_BARRIER;
}

// ---- barrier legs in packed pairs (FP32) ----------------------------------
// Two survival legs share each FP32 instruction (sm_100 f32x2): two
// independent samples, or a sample and its antithetic twin (uniforms u and
// 1 - u).  Every packed operation is the scalar step's operation in its order,
// so each half is surv_step's arithmetic bit for bit; the table lookups of the
// inverse normal (two fitted branches), the exponentials and the divisions
// stay scalar per half.
struct SurvLeg2 {
  float2 y, L, ypl;
  float2 e[3], le[3];
};

__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// GMath<float>::cdf_ratio of both halves
__device__ __forceinline__ void cdf_ratio2(float2 h, float2& p, float2& g) {
  const float2 a = make_float2(fabsf(h.x), fabsf(h.y));
  const float2 den = fma2(splat2(OF_MILLS_C), a, splat2(1.0f));
  const float2 t = make_float2(1.0f / den.x, 1.0f / den.y);
  float2 m = splat2(kMills[OF_MILLS_DEG]);
#pragma unroll
  for (int i = OF_MILLS_DEG - 1; i >= 0; --i) m = fma2(m, t, splat2(kMills[i]));
  m = mul2(m, t);
  const float2 a2 = mul2(a, a), a2lo = fma2(a, a, neg2(a2));
  const float2 ex = mul2(splat2(-0.5f), a2);
  const float2 phi = mul2(mul2(splat2(0.398942280401432677939946f), make_float2(__expf(ex.x), __expf(ex.y))),
                          fma2(splat2(-0.5f), a2lo, splat2(1.0f)));
  const float2 tail = mul2(phi, m);
  p.x = h.x < 0.0f ? tail.x : 1.0f - tail.x;
  p.y = h.y < 0.0f ? tail.y : 1.0f - tail.y;
  g.x = h.x < 0.0f ? 1.0f / m.x : phi.x / p.x;
  g.y = h.y < 0.0f ? 1.0f / m.y : phi.y / p.y;
}

__device__ __forceinline__ void surv_init2(SurvLeg2& s, const GreekConsts<float>& c) {
  s.y = s.ypl = make_float2(0.0f, 0.0f);
  s.L = splat2(c.sgn * c.bar > 0.0f ? 1.0f : 0.0f);
#pragma unroll
  for (int t = 0; t < 3; ++t) s.le[t] = make_float2(0.0f, 0.0f);
  s.e[0] = s.e[1] = splat2(c.sib);
  s.e[2] = make_float2(0.0f, 0.0f);
}

// surv_step<float, G, IN> of both halves
template <bool G, bool IN>
__device__ __forceinline__ void surv_step2(SurvLeg2& s, const GreekConsts<float>& c, float2 u) {
  using M = GMath<float>;
  float2 h = fma2(splat2(-c.sib), s.y, splat2(c.sib * (c.bar - c.alpha)));
  h.x = h.x > M::kHMin ? h.x : M::kHMin;
  h.y = h.y > M::kHMin ? h.y : M::kHMin;
  float2 p, g;
  cdf_ratio2(h, p, g);
  float2 v = mul2(u, p);
  float2 q = fma2(neg2(u), p, splat2(1.0f));
  v.x = v.x > M::kTiny ? v.x : M::kTiny;
  v.y = v.y > M::kTiny ? v.y : M::kTiny;
  q.x = q.x > M::kTiny ? q.x : M::kTiny;
  q.y = q.y > M::kTiny ? q.y : M::kTiny;
  const float2 zeta = make_float2(M::icdf2(v.x, q.x), M::icdf2(v.y, q.y));
  if (G) {
    const float2 zmh = sub2(zeta, h);
    const float2 d = mul2(mul2(splat2(0.5f), zmh), add2(zeta, h));
    const float2 w = mul2(u, make_float2(__expf(d.x), __expf(d.y)));
    const float2 kap = sub2(splat2(1.0f), w);
    s.le[0] = fma2(g, s.e[0], s.le[0]);
    s.le[1] = fma2(g, s.e[1], s.le[1]);
    s.le[2] = fma2(g, add2(s.e[2], h), s.le[2]);
    s.e[0] = mul2(kap, s.e[0]);
    s.e[1] = fma2(kap, s.e[1], splat2(c.sib));
    s.e[2] = fma2(kap, s.e[2], fma2(kap, h, zmh));
  }
  s.y = fma2(splat2(c.beta * c.sgn), zeta, add2(s.y, splat2(c.alpha)));
  s.L = mul2(s.L, p);
  if (IN) {
    const float2 zp = make_float2(M::icdf2(u.x, 1.0f - u.x), M::icdf2(u.y, 1.0f - u.y));
    s.ypl = fma2(splat2(c.beta), zp, add2(s.ypl, splat2(c.alpha)));
  }
}

// half e (0: .x, 1: .y) of a packed leg as a scalar leg
template <bool G>
__device__ __forceinline__ SurvLeg<float, G> surv_half(const SurvLeg2& s, int e) {
  SurvLeg<float, G> o;
  o.y = e ? s.y.y : s.y.x;
  o.L = e ? s.L.y : s.L.x;
  o.ypl = e ? s.ypl.y : s.ypl.x;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    o.e[t] = e ? s.e[t].y : s.e[t].x;
    o.le[t] = e ? s.le[t].y : s.le[t].x;
  }
  return o;
}

// gk_barrier<float, G, true, IN>: the sample and its antithetic twin as the
// two halves
template <bool G, bool IN>
__device__ __forceinline__ void gk_barrier_twin(const GreekConsts<float>& c, uint64_t i, const PhiloxKeys& K,
                                                GreekSample<float>& out) {
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  SurvLeg2 s;
  surv_init2(s, c);
  for (int32_t j = 0; j < c.steps; j += 4) {
    float u[4];
    gk_uniforms(c, (uint32_t)(j >> 2), lo, hi, K, u);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (j + q >= c.steps) break;
      surv_step2<G, IN>(s, c, make_float2(u[q], 1.0f - u[q]));
    }
  }
  float xa, xb, ga[4], gb[4];
  surv_payoff<float, G, IN>(surv_half<G>(s, 0), c, xa, ga);
  surv_payoff<float, G, IN>(surv_half<G>(s, 1), c, xb, gb);
  out.x = 0.5f * (xa + xb);
  out.y = 0.0f;
#pragma unroll
  for (int t = 0; t < 4; ++t) out.g[t] = 0.5f * (ga[t] + gb[t]);
}

// gk_barrier<float, G, false, IN> of samples i0 and i1 in one packed loop
template <bool G, bool IN>
__device__ __forceinline__ void gk_barrier_pair(const GreekConsts<float>& c, uint64_t i0, uint64_t i1,
                                                const PhiloxKeys& K, GreekSample<float>& o0, GreekSample<float>& o1) {
  const uint32_t lo0 = (uint32_t)i0, hi0 = (uint32_t)(i0 >> 32), lo1 = (uint32_t)i1, hi1 = (uint32_t)(i1 >> 32);
  SurvLeg2 s;
  surv_init2(s, c);
  for (int32_t j = 0; j < c.steps; j += 4) {
    float u0[4], u1[4];
    gk_uniforms(c, (uint32_t)(j >> 2), lo0, hi0, K, u0);
    gk_uniforms(c, (uint32_t)(j >> 2), lo1, hi1, K, u1);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (j + q >= c.steps) break;
      surv_step2<G, IN>(s, c, make_float2(u0[q], u1[q]));
    }
  }
  float x, g[4];
  surv_payoff<float, G, IN>(surv_half<G>(s, 0), c, x, g);
  o0.x = x;
  o0.y = 0.0f;
#pragma unroll
  for (int t = 0; t < 4; ++t) o0.g[t] = g[t];
  surv_payoff<float, G, IN>(surv_half<G>(s, 1), c, x, g);
  o1.x = x;
  o1.y = 0.0f;
#pragma unroll
  for (int t = 0; t < 4; ++t) o1.g[t] = g[t];
}

template <typename R, bool G, int KG, bool ANTI>
__device__ __forceinline__ void gk_sample_group_anti(const GreekConsts<R>& c, uint64_t i, const PhiloxKeys& K,
                                                     const float* obs_w, GreekSample<R>& out) {
  if (KG == KG_TERMINAL) {
    gk_terminal<R, G, ANTI>(c, i, K, out);
  } else if (KG == KG_ASIAN) {
    if constexpr (std::is_same<R, float>::value && ANTI) {  // the twin legs in packed pairs
      if (c.kind == GK_ASIAN_DAILY) {
        if (c.flags & GF_GEOMETRIC) gk_asian_twin<G, true, false, true>(c, i, K, obs_w, out);
        else if (c.cv_kind == GCV_GEOMETRIC_ASIAN) gk_asian_twin<G, true, true, true>(c, i, K, obs_w, out);
        else gk_asian_twin<G, true, true, false>(c, i, K, obs_w, out);
      } else {
        if (c.flags & GF_GEOMETRIC) gk_asian_twin<G, false, false, true>(c, i, K, obs_w, out);
        else if (c.cv_kind == GCV_GEOMETRIC_ASIAN) gk_asian_twin<G, false, true, true>(c, i, K, obs_w, out);
        else gk_asian_twin<G, false, true, false>(c, i, K, obs_w, out);
      }
      return;
    }
    if (c.kind == GK_ASIAN_DAILY) {
      if (c.flags & GF_GEOMETRIC) gk_asian<R, G, ANTI, true, false, true>(c, i, K, obs_w, out);
      else if (c.cv_kind == GCV_GEOMETRIC_ASIAN) gk_asian<R, G, ANTI, true, true, true>(c, i, K, obs_w, out);
      else gk_asian<R, G, ANTI, true, true, false>(c, i, K, obs_w, out);
    } else {
      if (c.flags & GF_GEOMETRIC) gk_asian<R, G, ANTI, false, false, true>(c, i, K, obs_w, out);
      else if (c.cv_kind == GCV_GEOMETRIC_ASIAN) gk_asian<R, G, ANTI, false, true, true>(c, i, K, obs_w, out);
      else gk_asian<R, G, ANTI, false, true, false>(c, i, K, obs_w, out);
    }
  } else {
    if constexpr (std::is_same<R, float>::value && ANTI) {  // the twin legs in packed pairs
      if (c.kind == GK_BARRIER_OUT) gk_barrier_twin<G, false>(c, i, K, out);
      else gk_barrier_twin<G, true>(c, i, K, out);
    } else {
      if (c.kind == GK_BARRIER_OUT) gk_barrier<R, G, ANTI, false>(c, i, K, out);
      else gk_barrier<R, G, ANTI, true>(c, i, K, out);
    }
  }
}

// Two samples of a terminal-only option (FP32 modes; antithetic twins are
// the negated sum of the same normals).
template <bool G>
__device__ __forceinline__ void gk_terminal_pair_group(const GreekConsts<float>& c, uint64_t i0, uint64_t i1,
                                                       const PhiloxKeys& K, GreekSample<float>& o0,
                                                       GreekSample<float>& o1) {
  if (c.flags & GF_ANTI) gk_terminal_pair<G, true>(c, i0, i1, K, o0, o1);
  else gk_terminal_pair<G, false>(c, i0, i1, K, o0, o1);
}

// Two samples of an Asian option without antithetic twins (FP32 modes).
template <bool G>
__device__ __forceinline__ void gk_asian_pair_group(const GreekConsts<float>& c, uint64_t i0, uint64_t i1,
                                                    const PhiloxKeys& K, const float* __restrict__ obs_w,
                                                    GreekSample<float>& o0, GreekSample<float>& o1) {
  if (c.kind == GK_ASIAN_DAILY) {
    if (c.flags & GF_GEOMETRIC) gk_asian_pair<G, true, false, true>(c, i0, i1, K, obs_w, o0, o1);
    else if (c.cv_kind == GCV_GEOMETRIC_ASIAN) gk_asian_pair<G, true, true, true>(c, i0, i1, K, obs_w, o0, o1);
    else gk_asian_pair<G, true, true, false>(c, i0, i1, K, obs_w, o0, o1);
  } else {
    if (c.flags & GF_GEOMETRIC) gk_asian_pair<G, false, false, true>(c, i0, i1, K, obs_w, o0, o1);
    else if (c.cv_kind == GCV_GEOMETRIC_ASIAN) gk_asian_pair<G, false, true, true>(c, i0, i1, K, obs_w, o0, o1);
    else gk_asian_pair<G, false, true, false>(c, i0, i1, K, obs_w, o0, o1);
  }
}

// Two samples of a barrier option without antithetic twins (FP32 modes).
template <bool G>
__device__ __forceinline__ void gk_barrier_pair_group(const GreekConsts<float>& c, uint64_t i0, uint64_t i1,
                                                      const PhiloxKeys& K, GreekSample<float>& o0,
                                                      GreekSample<float>& o1) {
  if (c.kind == GK_BARRIER_OUT) gk_barrier_pair<G, false>(c, i0, i1, K, o0, o1);
  else gk_barrier_pair<G, true>(c, i0, i1, K, o0, o1);
}

template <typename R, bool G, int KG>
__device__ __forceinline__ void gk_sample_group(const GreekConsts<R>& c, uint64_t i, const PhiloxKeys& K,
                                                const float* obs_w, GreekSample<R>& out) {
  if (c.flags & GF_ANTI) gk_sample_group_anti<R, G, KG, true>(c, i, K, obs_w, out);
  else gk_sample_group_anti<R, G, KG, false>(c, i, K, obs_w, out);
}

}  // namespace of
