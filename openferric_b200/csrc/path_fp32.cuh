// path_fp32.cuh - FP32 path steppers shared by the Philox kernels.
//
// State is kept relative to the spot: y = ln(S/S0), so that the FP32 rounding
// of each step is relative to |y| (~0.1-1) instead of |ln S| (~4.6).
#pragma once

#include "f32x2.cuh"
#include "of_device.cuh"

namespace of {

// Per-option constants of the FP32 steppers (built on the host in FP64 and
// rounded once).
struct StepConsts {
  // GBM log-Euler (src/mc/simulation.rs:63-71): y += drift + diff z
  float drift, diff;
  // Heston Euler of the reference (src/models/stochastic.rs:56-71, with the
  // variance floored after every step as src/mc/simulation.rs:111-113 does):
  // y += mudt - half_dt v + sqrt(v) sqdt zs ; v = max(v + kdt_theta - kdt v + xi sqrt(v) sqdt z1, 0)
  // The normals arrive as sqdt (z1, z2): bm_k2 = -2 ln(2) dt is the radius
  // constant of normal_pair_scaled_from_u32.
  float mudt, half_dt, sqdt, kdt, kdt_theta, xi, rho, rho_c, v0, y_floor, one_m_kdt, bm_k2;
  // Heston QE (Andersen 2008, gamma1 = gamma2 = 1/2, psi_c = 1.5)
  float qe_e, qe_c1, qe_c2, qe_theta, qe_k0, qe_k1, qe_k2, qe_k3, qe_k4;
};

struct LegState {
  float y, v;
};

// Reference Heston Euler step in FP32 (variance kept >= 0 after each step).
// w1, w2 = sqdt (z1, z2), the pair of normal_pair_scaled_from_u32(.., c.bm_k2).
__device__ __forceinline__ void heston_euler_step(LegState& L, const StepConsts& c, float w1, float w2) {
  const float sq = sqrtf(L.v);
  const float ws = fmaf(c.rho, w1, c.rho_c * w2);  // sqdt zs
  const float y = fmaf(sq, ws, fmaf(-c.half_dt, L.v, L.y + c.mudt));
  // v + kappa (theta - v) dt = (1 - kappa dt) v + kappa theta dt
  const float vn = fmaf(c.xi * sq, w1, fmaf(c.one_m_kdt, L.v, c.kdt_theta));
  L.v = fmaxf(vn, 0.0f);
  L.y = fmaxf(y, c.y_floor);
}

// Two samples' Heston Euler legs in one packed pair each (.x = the first
// sample, .y = the second): heston_euler_step's operations in its order, two
// samples per instruction, so each half is bit-identical to the scalar step.
struct LegState2 {
  float2 y, v;
};

__device__ __forceinline__ void heston_euler_step2(LegState2& L, const StepConsts& c, float2 w1, float2 w2) {
  const float2 sq = make_float2(sqrtf(L.v.x), sqrtf(L.v.y));
  const float2 ws = fma2(splat2(c.rho), w1, mul2(splat2(c.rho_c), w2));
  const float2 y = fma2(sq, ws, fma2(splat2(-c.half_dt), L.v, add2(L.y, splat2(c.mudt))));
  const float2 vn = fma2(mul2(splat2(c.xi), sq), w1, fma2(splat2(c.one_m_kdt), L.v, splat2(c.kdt_theta)));
  L.v = make_float2(fmaxf(vn.x, 0.0f), fmaxf(vn.y, 0.0f));
  L.y = make_float2(fmaxf(y.x, c.y_floor), fmaxf(y.y, c.y_floor));
}

// Andersen QE step.  uv: uniform for the variance, zv = Phi^-1(uv) is
// computed only on the quadratic branch; zx: normal for the log-spot.
__device__ __forceinline__ void heston_qe_step(LegState& L, const StepConsts& c, float uv, float zv_sign,
                                               float zx, uint32_t uv_bits) {
  const float v = L.v;
  const float m = fmaf(v - c.qe_theta, c.qe_e, c.qe_theta);
  const float s2 = fmaf(v, c.qe_c1, c.qe_c2);
  const float inv_m = (1.0f / (m));
  const float psi = s2 * inv_m * inv_m;
  float vn;
  if (psi <= 1.5f) {
    const float t = 2.0f * (1.0f / (psi));
    const float b2 = (t - 1.0f) + sqrtf(t * (t - 1.0f));
    const float a = m * (1.0f / (1.0f + b2));
    const float zv = zv_sign * normal_from_u32(uv_bits);
    const float bz = sqrtf(b2) + zv;
    vn = a * bz * bz;
  } else {
    const float p = (psi - 1.0f) * (1.0f / (psi + 1.0f));
    // beta = (1-p)/m ; v' = ln((1-p)/(1-u)) / beta
    vn = (uv <= p) ? 0.0f : (__log2f(1.0f - p) - __log2f(1.0f - uv)) * 0.69314718055994531f * m * (1.0f / (1.0f - p));
  }
  const float var = fmaxf(fmaf(c.qe_k3, v, c.qe_k4 * vn), 0.0f);
  L.y = fmaf(sqrtf(var), zx, L.y + c.mudt + c.qe_k0 + c.qe_k1 * v + c.qe_k2 * vn);
  L.v = vn;
}

}  // namespace of
