// adjoint.cu - pathwise reverse-mode Heston Greeks with checkpointing (FP32).
//
// Price and d/d(S0, r, v0, kappa, theta, xi, rho) of a European or arithmetic
// Asian option under Andersen's QE scheme (gamma1 = gamma2 = 1/2, psi_c = 1.5):
//   m = theta + (v - theta) e,  s2 = v c1 + c2,  psi = s2 / m^2
//   psi <= 1.5: v' = a (b + Zv)^2,  b^2 = 2/psi - 1 + sqrt(2/psi (2/psi - 1)),  a = m / (1 + b^2)
//   psi >  1.5: v' = 0 if U <= p else m ln((1-p)/(1-U)) / (1-p),  p = (psi-1)/(psi+1)
//   y' = y + (r-q) dt + K0 + K1 v + K2 v' + sqrt(K34 (v + v')) Zx,   S = S0 e^y
// Forward pass: one thread per path, (v, y) checkpointed every C steps.
// Backward sweep: per segment (last first) the C steps are recomputed from
// their checkpoint into registers (v, e^y), the Philox draws of each step are
// regenerated from their counters, and the adjoints (y_bar, v_bar) and the
// parameter adjoints are propagated through the analytic step Jacobian.
// Paths that finish out of the money have zero pathwise derivatives and skip
// the sweep.
//
// Compiled with --fmad=false: every fused multiply-add is an explicit fmaf so
// the forward pass and the recompute produce bit-identical states.
#include <cmath>
#include <cstring>

#include "of_device.cuh"
#include "of_internal.h"

namespace {

constexpr uint32_t kAdjStreamTag = 0x41444A31u;  // "ADJ1"
constexpr int kMaxSegments = 64;
constexpr float kLn2 = 0.69314718055994531f;

__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

struct AdjC {
  // step
  float e, c1, c2, theta, c0 /* (r-q) dt + K0 */, K1, K2, k34, dt;
  // parameter partials of the step constants
  float de_dk, c1_k, c2_k, c1_x, c2_x, c2_t;
  float K0_k, K0_t, K0_x, K0_r, K1_k, K1_x, K1_r, K2_k, K2_x, K2_r, k34_r;
  // payoff
  float s0, strike, v0, inv_steps;
  double disc, T;
  int32_t steps, seg_len, n_seg, call, asian, forward_only;
  int64_t paths;
  of::PhiloxKeys keys;
};

struct QeDraw {
  float u, zx;
  uint32_t ubits;
};

__device__ __forceinline__ QeDraw draw_of(const uint4& r, int odd) {
  QeDraw d;
  d.ubits = odd ? r.z : r.x;
  d.u = of::uniform_from_u32(d.ubits);
  d.zx = of::normal_from_u32(odd ? r.w : r.y);
  return d;
}

// Forward QE variance step.
__device__ __forceinline__ float qe_vnext(const AdjC& c, float v, const QeDraw& d) {
  const float m = fmaf(v - c.theta, c.e, c.theta);
  const float s2 = fmaf(v, c.c1, c.c2);
  const float inv_m = __fdividef(1.0f, m);
  const float psi = s2 * inv_m * inv_m;
  if (psi <= 1.5f) {
    const float t = __fdividef(2.0f, psi);
    const float b2 = (t - 1.0f) + sqrt_approx(t * (t - 1.0f));
    const float a = __fdividef(m, 1.0f + b2);
    const float bz = sqrt_approx(b2) + of::normal_from_u32(d.ubits);
    return a * bz * bz;
  }
  const float p = __fdividef(psi - 1.0f, psi + 1.0f);
  if (d.u <= p) return 0.0f;
  const float L = (__log2f(1.0f - p) - __log2f(1.0f - d.u)) * kLn2;
  return __fdividef(m * L, 1.0f - p);
}

__device__ __forceinline__ float qe_ynext(const AdjC& c, float y, float v, float vn, float zx) {
  const float var = c.k34 * (v + vn);
  return fmaf(sqrt_approx(var), zx, fmaf(c.K2, vn, fmaf(c.K1, v, y + c.c0)));
}

// Jacobian of one step at (v, vn): dvn/d{v,kappa,theta,xi} and dy'/d{v,vn,kappa,theta,xi,rho}.
struct StepJac {
  float dvn_v, dvn_k, dvn_t, dvn_x;
  float dy_v, dy_vn, dy_k, dy_t, dy_x, dy_r;
};

__device__ __forceinline__ StepJac qe_jacobian(const AdjC& c, float v, float vn, const QeDraw& d) {
  StepJac J;
  const float m = fmaf(v - c.theta, c.e, c.theta);
  const float s2 = fmaf(v, c.c1, c.c2);
  const float inv_m = __fdividef(1.0f, m);
  const float psi = s2 * inv_m * inv_m;
  float A1 = 0.0f, A2 = 0.0f;  // dvn = A1 dm + A2 dpsi
  if (psi <= 1.5f) {
    const float t = __fdividef(2.0f, psi);
    const float root = sqrt_approx(t * (t - 1.0f));
    const float b2 = (t - 1.0f) + root;
    const float b = sqrt_approx(b2);
    const float inv_1b2 = __fdividef(1.0f, 1.0f + b2);
    const float a = m * inv_1b2;
    const float bz = b + of::normal_from_u32(d.ubits);
    const float dv_da = bz * bz;
    const float dv_db = 2.0f * a * bz;
    const float da_db2 = -a * inv_1b2;
    const float db_db2 = __fdividef(0.5f, b);
    const float db2_dt = 1.0f + __fdividef(fmaf(2.0f, t, -1.0f), 2.0f * root);
    const float dt_dpsi = -0.5f * t * t;
    A1 = dv_da * inv_1b2;
    A2 = fmaf(dv_da, da_db2, dv_db * db_db2) * db2_dt * dt_dpsi;
  } else {
    const float inv_p1 = __fdividef(1.0f, psi + 1.0f);
    const float p = (psi - 1.0f) * inv_p1;
    if (d.u > p) {
      const float inv_1p = __fdividef(1.0f, 1.0f - p);
      const float L = (__log2f(1.0f - p) - __log2f(1.0f - d.u)) * kLn2;
      A1 = L * inv_1p;
      A2 = m * (L - 1.0f) * inv_1p * inv_1p * (2.0f * inv_p1 * inv_p1);
    }
  }
  // m_q and psi_q = inv_m^2 s2_q - 2 psi inv_m m_q
  const float im2 = inv_m * inv_m, tpm = 2.0f * psi * inv_m;
  const float m_v = c.e, m_t = 1.0f - c.e, m_k = (v - c.theta) * c.de_dk;
  const float s2_v = c.c1, s2_t = c.c2_t, s2_k = fmaf(v, c.c1_k, c.c2_k), s2_x = fmaf(v, c.c1_x, c.c2_x);
  J.dvn_v = fmaf(A1, m_v, A2 * fmaf(im2, s2_v, -tpm * m_v));
  J.dvn_t = fmaf(A1, m_t, A2 * fmaf(im2, s2_t, -tpm * m_t));
  J.dvn_k = fmaf(A1, m_k, A2 * fmaf(im2, s2_k, -tpm * m_k));
  J.dvn_x = A2 * im2 * s2_x;
  const float var = c.k34 * (v + vn);
  const float h = var > 0.0f ? __fdividef(0.5f * d.zx, sqrt_approx(var)) : 0.0f;
  J.dy_v = fmaf(c.k34, h, c.K1);
  J.dy_vn = fmaf(c.k34, h, c.K2);
  J.dy_k = fmaf(c.K2_k, vn, fmaf(c.K1_k, v, c.K0_k));
  J.dy_t = c.K0_t;
  J.dy_x = fmaf(c.K2_x, vn, fmaf(c.K1_x, v, c.K0_x));
  J.dy_r = fmaf(c.k34_r * (v + vn), h, fmaf(c.K2_r, vn, fmaf(c.K1_r, v, c.K0_r)));
  return J;
}

template <int C>
__global__ void __launch_bounds__(128) adjoint_kernel(const __grid_constant__ AdjC c,
                                                      double* __restrict__ partials) {
  __shared__ double sh[16 * 4];
  double acc[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.paths; i += stride) {
    const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
    float ck_v[kMaxSegments], ck_y[kMaxSegments];
    float v = c.v0, y = 0.0f;
    of::Kahan32 sum_s;
    // ---- forward pass with checkpoints ----
    for (int seg = 0; seg < c.n_seg; ++seg) {
      ck_v[seg] = v;
      ck_y[seg] = y;
      const int j0 = seg * C;
#pragma unroll 2
      for (int k = 0; k < C; k += 2) {
        const int j = j0 + k;
        if (j >= c.steps) break;
        const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 1), lo, hi, kAdjStreamTag), c.keys);
#pragma unroll
        for (int o = 0; o < 2; ++o) {
          if (j + o < c.steps) {
            const QeDraw d = draw_of(r, o);
            const float vn = qe_vnext(c, v, d);
            y = qe_ynext(c, y, v, vn, d.zx);
            v = vn;
            if (c.asian) sum_s.add(__expf(y));
          }
        }
      }
    }
    // payoff and its derivative w.r.t. the average (or the terminal spot)
    const float und = c.asian ? c.s0 * (float)(sum_s.value() * (double)c.inv_steps) : c.s0 * __expf(y);
    const float intr = c.call ? und - c.strike : c.strike - und;
    const double pv = intr > 0.0f ? c.disc * (double)intr : 0.0;
    acc[0] += pv;
    acc[1] += pv * pv;
    if (c.forward_only || !(intr > 0.0f)) continue;
    const float g = (float)c.disc * (c.call ? 1.0f : -1.0f);  // d pv / d underlying
    const float dS0 = g * und / c.s0;
    // ---- backward sweep ----
    const float direct = c.asian ? g * c.s0 * c.inv_steps : 0.0f;  // d pv / d y_j = direct * e^{y_j}
    float ybar = c.asian ? 0.0f : g * und;  // European: seed at y_M
    float wbar = 0.0f, kbar = 0.0f, tbar = 0.0f, xbar = 0.0f, rbar = 0.0f, mubar = 0.0f;
    for (int seg = c.n_seg - 1; seg >= 0; --seg) {
      const int j0 = seg * C;
      const int len = (c.steps - j0) < C ? (c.steps - j0) : C;
      float sv[C + 1], ss[C + 1];
      float vv = ck_v[seg], yy = ck_y[seg];
      sv[0] = vv;
      ss[0] = 0.0f;
#pragma unroll
      for (int k = 0; k < C; k += 2) {
        if (k < len) {
          const int j = j0 + k;
          const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 1), lo, hi, kAdjStreamTag), c.keys);
#pragma unroll
          for (int o = 0; o < 2; ++o) {
            if (k + o < len) {
              const QeDraw d = draw_of(r, o);
              const float vn = qe_vnext(c, vv, d);
              yy = qe_ynext(c, yy, vv, vn, d.zx);
              vv = vn;
              sv[k + o + 1] = vv;
              ss[k + o + 1] = __expf(yy);
            }
          }
        }
      }
#pragma unroll
      for (int k = C - 2; k >= 0; k -= 2) {
        if (k < len) {
          const int j = j0 + k;
          const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 1), lo, hi, kAdjStreamTag), c.keys);
#pragma unroll
          for (int o = 1; o >= 0; --o) {
            if (k + o < len) {
              ybar = fmaf(direct, ss[k + o + 1], ybar);  // y_{j+o+1} enters the average
              const QeDraw d = draw_of(r, o);
              const StepJac J = qe_jacobian(c, sv[k + o], sv[k + o + 1], d);
              const float Vbar = fmaf(ybar, J.dy_vn, wbar);
              kbar = fmaf(Vbar, J.dvn_k, fmaf(ybar, J.dy_k, kbar));
              tbar = fmaf(Vbar, J.dvn_t, fmaf(ybar, J.dy_t, tbar));
              xbar = fmaf(Vbar, J.dvn_x, fmaf(ybar, J.dy_x, xbar));
              rbar = fmaf(ybar, J.dy_r, rbar);
              mubar = fmaf(ybar, c.dt, mubar);
              wbar = fmaf(Vbar, J.dvn_v, ybar * J.dy_v);
            }
          }
        }
      }
    }
    const double gk[7] = {dS0, (double)mubar - c.T * pv, wbar, kbar, tbar, xbar, rbar};
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      acc[2 + k] += gk[k];
      acc[9 + k] += gk[k] * gk[k];
    }
  }
  of::block_sum<16>(acc, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 16; ++k) partials[(int64_t)blockIdx.x * 16 + k] = acc[k];
}

// Price-only FP64 pass over the same draws (the bits of each Philox counter
// give the same U, Zv, Zx), for bump-and-revalue with common random numbers:
// a relative bump of 1e-4 moves a step's log-increment by ~1e-8, below the
// FP32 resolution of the path state, so the revaluation runs in FP64.
struct AdjC64 {
  double e, c1, c2, theta, c0, K1, K2, k34, s0, strike, inv_steps, disc, v0;
  int32_t steps, call, asian;
  int64_t paths;
  of::PhiloxKeys keys;
};

__global__ void __launch_bounds__(128) forward64_kernel(const __grid_constant__ AdjC64 c,
                                                        double* __restrict__ partials) {
  __shared__ double sh[16 * 4];
  double acc[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.paths; i += stride) {
    const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
    double v = c.v0, y = 0.0, sum_s = 0.0;
    for (int j = 0; j < c.steps; j += 2) {
      const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 1), lo, hi, kAdjStreamTag), c.keys);
      for (int o = 0; o < 2 && j + o < c.steps; ++o) {
        const uint32_t ub = o ? r.z : r.x;
        const double u = (double)of::uniform_from_u32(ub);
        const double zx = (double)of::normal_from_u32(o ? r.w : r.y);
        const double m = c.theta + (v - c.theta) * c.e;
        const double s2 = v * c.c1 + c.c2;
        const double psi = s2 / (m * m);
        double vn;
        if (psi <= 1.5) {
          const double t = 2.0 / psi;
          const double b2 = (t - 1.0) + sqrt(t * (t - 1.0));
          const double a = m / (1.0 + b2);
          const double bz = sqrt(b2) + (double)of::normal_from_u32(ub);
          vn = a * bz * bz;
        } else {
          const double p = (psi - 1.0) / (psi + 1.0);
          vn = (u <= p) ? 0.0 : m * log((1.0 - p) / (1.0 - u)) / (1.0 - p);
        }
        y = y + c.c0 + c.K1 * v + c.K2 * vn + sqrt(c.k34 * (v + vn)) * zx;
        v = vn;
        if (c.asian) sum_s += exp(y);
      }
    }
    const double und = c.asian ? c.s0 * sum_s * c.inv_steps : c.s0 * exp(y);
    const double intr = c.call ? und - c.strike : c.strike - und;
    const double pv = intr > 0.0 ? c.disc * intr : 0.0;
    acc[0] += pv;
    acc[1] += pv * pv;
  }
  of::block_sum<16>(acc, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 16; ++k) partials[(int64_t)blockIdx.x * 16 + k] = acc[k];
}

}  // namespace

extern "C" of_status of_heston_price_adjoint(of_ctx* ctx, const of_heston_adjoint_params* p, of_adjoint_result* out) {
  if (!ctx || !p || !out) return OF_ERR_INVALID_INPUT;
  std::memset(out, 0, sizeof(*out));
  if (p->option_type != OF_CALL && p->option_type != OF_PUT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown option type %d", p->option_type);
  if (p->payoff != OF_PAYOFF_VANILLA && p->payoff != OF_PAYOFF_ASIAN)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "adjoint payoff must be vanilla or arithmetic Asian");
  if (p->scheme != OF_MODEL_HESTON_QE)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "the adjoint kernel implements the QE scheme");
  if (p->num_paths <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths must be > 0");
  if (p->num_steps <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps must be > 0");
  if (p->checkpoint_every != 32) return of_fail(ctx, OF_ERR_UNSUPPORTED, "checkpoint interval must be 32");
  if (p->forward_only < 0 || p->forward_only > 2)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "forward_only must be 0, 1 or 2");
  if (p->num_steps > (int64_t)kMaxSegments * 32)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "at most %d steps", kMaxSegments * 32);
  if (!(p->spot > 0.0) || !(p->strike > 0.0) || !(p->expiry > 0.0))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "spot, strike and expiry must be > 0");
  if (!(p->kappa > 0.0 && p->theta > 0.0 && p->xi > 0.0 && p->v0 >= 0.0 && p->rho > -1.0 && p->rho < 1.0))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "invalid Heston parameters (QE needs kappa, theta, xi > 0)");
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const double dt = p->expiry / (double)p->num_steps;
  const double k = p->kappa, th = p->theta, x = p->xi, r = p->rho;
  const double e = std::exp(-k * dt);
  const double c1 = x * x * e * (1.0 - e) / k;
  const double c2 = th * x * x * (1.0 - e) * (1.0 - e) / (2.0 * k);
  const double de_dk = -dt * e;
  AdjC c{};
  c.e = (float)e;
  c.c1 = (float)c1;
  c.c2 = (float)c2;
  c.theta = (float)th;
  const double K0 = -r * k * th * dt / x;
  const double K1 = 0.5 * dt * (k * r / x - 0.5) - r / x;
  const double K2 = 0.5 * dt * (k * r / x - 0.5) + r / x;
  const double k34 = 0.5 * dt * (1.0 - r * r);
  c.c0 = (float)((p->rate - p->dividend_yield) * dt + K0);
  c.K1 = (float)K1;
  c.K2 = (float)K2;
  c.k34 = (float)k34;
  c.dt = (float)dt;
  c.de_dk = (float)de_dk;
  c.c1_k = (float)(x * x * de_dk * (1.0 - 2.0 * e) / k - c1 / k);
  c.c2_k = (float)(-th * x * x * (1.0 - e) * de_dk / k - c2 / k);
  c.c1_x = (float)(2.0 * c1 / x);
  c.c2_x = (float)(2.0 * c2 / x);
  c.c2_t = (float)(x * x * (1.0 - e) * (1.0 - e) / (2.0 * k));
  c.K0_k = (float)(-r * th * dt / x);
  c.K0_t = (float)(-r * k * dt / x);
  c.K0_x = (float)(r * k * th * dt / (x * x));
  c.K0_r = (float)(-k * th * dt / x);
  c.K1_k = (float)(0.5 * dt * r / x);
  c.K1_x = (float)(-0.5 * dt * k * r / (x * x) + r / (x * x));
  c.K1_r = (float)(0.5 * dt * k / x - 1.0 / x);
  c.K2_k = (float)(0.5 * dt * r / x);
  c.K2_x = (float)(-0.5 * dt * k * r / (x * x) - r / (x * x));
  c.K2_r = (float)(0.5 * dt * k / x + 1.0 / x);
  c.k34_r = (float)(-dt * r);
  c.s0 = (float)p->spot;
  c.strike = (float)p->strike;
  c.v0 = (float)p->v0;
  c.inv_steps = (float)(1.0 / (double)p->num_steps);
  c.disc = std::exp(-p->rate * p->expiry);
  c.T = p->expiry;
  c.steps = (int32_t)p->num_steps;
  c.seg_len = 32;
  c.n_seg = (int32_t)((p->num_steps + 31) / 32);
  c.call = p->option_type == OF_CALL;
  c.asian = p->payoff == OF_PAYOFF_ASIAN;
  c.forward_only = p->forward_only ? 1 : 0;
  c.paths = p->num_paths;
  c.keys = of::philox_keys(p->seed);

  const int block = 128;
  const int64_t want = (p->num_paths + block - 1) / block;
  const int64_t cap = (int64_t)ctx->sm_count * of_blocks_per_sm((const void*)adjoint_kernel<32>, block, 0);
  const int grid = (int)(want < cap ? want : cap);
  void *d_part = nullptr, *d_sums = nullptr, *h = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)grid * 16 * sizeof(double), &d_part));
  OF_TRY(of_scratch(ctx, SLOT_SUMS, 16 * sizeof(double), &d_sums));
  OF_TRY(of_pinned(ctx, 16 * sizeof(double), &h));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  if (p->forward_only == 2) {
    AdjC64 d{};
    d.e = e;
    d.c1 = c1;
    d.c2 = c2;
    d.theta = th;
    d.c0 = (p->rate - p->dividend_yield) * dt + K0;
    d.K1 = K1;
    d.K2 = K2;
    d.k34 = k34;
    d.s0 = p->spot;
    d.strike = p->strike;
    d.inv_steps = 1.0 / (double)p->num_steps;
    d.disc = std::exp(-p->rate * p->expiry);
    d.v0 = p->v0;
    d.steps = (int32_t)p->num_steps;
    d.call = c.call;
    d.asian = c.asian;
    d.paths = p->num_paths;
    d.keys = c.keys;
    forward64_kernel<<<grid, block, 0, ctx->stream>>>(d, (double*)d_part);
  } else {
    adjoint_kernel<32><<<grid, block, 0, ctx->stream>>>(c, (double*)d_part);
  }
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_TRY(of_reduce_rows(ctx, (const double*)d_part, grid, 16, (double*)d_sums));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(h, d_sums, 16 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
  double s[16];
  std::memcpy(s, h, sizeof(s));
  const double n = (double)p->num_paths;
  auto se = [&](double sum, double sum2) {
    const double var = n > 1.0 ? (sum2 - sum * sum / n) / (n - 1.0) : 0.0;
    return std::sqrt((var > 0.0 ? var : 0.0) / n);
  };
  out->price = s[0] / n;
  out->stderr_ = se(s[0], s[1]);
  for (int k2 = 0; k2 < OF_ADJ_COUNT; ++k2) {
    out->greeks[k2] = s[2 + k2] / n;
    out->greeks_stderr[k2] = se(s[2 + k2], s[9 + k2]);
  }
  out->samples = p->num_paths;
  out->kernel_ms = ms;
  return OF_OK;
}
