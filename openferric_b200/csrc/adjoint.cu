// adjoint.cu - pathwise reverse-mode Heston Greeks with checkpointing (FP32).
//
// Price and d/d(S0, r, v0, kappa, theta, xi, rho) of a European or arithmetic
// Asian option under Andersen's QE scheme (gamma1 = gamma2 = 1/2, psi_c = 1.5):
//   m = theta + (v - theta) e,  s2 = v c1 + c2,  psi = s2 / m^2
//   quadratic: v' = a (b + Zv)^2,  b^2 = 2/psi - 1 + sqrt(2/psi (2/psi - 1)),  a = m / (1 + b^2)
//   exponential: v' = 0 if U <= p else m ln((1-p)/(1-U)) / (1-p),  p = (psi-1)/(psi+1)
//   y' = y + (r-q) dt + K0 + K1 v + K2 v' + sqrt(K34 (v + v')) Zx,   S = S0 e^y
// The branch is the quadratic one for psi <= psi_c - band, the exponential
// one for psi > psi_c + band, and a smoothstep blend of the two in between.
// band = 0 is Andersen's hard switch; its v' jumps at psi_c, and a pathwise
// derivative cannot see that jump, so the Greeks of kappa/theta/xi then miss
// the jump's contribution.  A band > 0 makes the step continuous and the
// pathwise estimator unbiased for the scheme it differentiates.
//
// Kernel 1 (forward): one thread per path; (v, y) checkpointed every 32 steps
// to HBM, time-major ckpt[segment][path]; the payoff gradient of each path.
// Kernel 2 (backward): each warp scans 128-path ranges (grid stride), queues
// the in-the-money paths in shared memory (ballot; the queue carries over
// between ranges), and sweeps them 32 at a time:
// per segment (last first) the 32 steps are recomputed from the checkpoint
// into shared memory (v, e^y), each step's Philox draws are regenerated from
// its counter, and the adjoints (y_bar, v_bar) and parameter adjoints are
// propagated through the analytic step Jacobian.  Out-of-the-money paths
// have zero pathwise derivatives and are never swept.
//
// Compiled with --fmad=false: every fused multiply-add is an explicit fmaf, so
// the forward pass and the recompute produce bit-identical states.
#include <cmath>
#include <cstring>

#include "of_device.cuh"
#include "of_internal.h"

namespace {

constexpr uint32_t kAdjStreamTag = 0x41444A31u;  // "ADJ1"
constexpr int kSeg = 32;                          // checkpoint interval
constexpr int kMaxSegments = 64;
constexpr int kBwdThreads = 128;
constexpr int kBwdWarps = kBwdThreads / 32;
constexpr int kRangePerWarp = 32 * 4;  // paths one warp scans for in-the-money paths per grid-stride turn
constexpr float kLn2 = 0.69314718055994531f;

__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

struct AdjC {
  // step
  float e, c1, c2, theta, c0 /* (r-q) dt + K0 */, K1, K2, k34, dt;
  float sw_lo, sw_hi, sw_inv_width;  // smoothed switch band [lo, hi]
  // parameter partials of the step constants
  float de_dk, c1_k, c2_k, c1_x, c2_x, c2_t;
  float K0_k, K0_t, K0_x, K0_r, K1_k, K1_x, K1_r, K2_k, K2_x, K2_r, k34_r;
  // payoff
  float s0, strike, v0, inv_steps;
  double disc, T;
  int32_t steps, n_seg, call, asian;
  int64_t paths;
  of::PhiloxKeys keys;
  // device buffers
  float* ck_v;   // [n_seg][paths]
  float* ck_y;   // [n_seg][paths]
  float* grad;   // [paths] d pv / d underlying (0 out of the money)
  float* und;    // [paths] average (or terminal spot)
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

__device__ __forceinline__ float quad_branch(float m, float psi, uint32_t ubits) {
  const float t = __fdividef(2.0f, psi);
  const float b2 = (t - 1.0f) + sqrt_approx(t * (t - 1.0f));
  const float a = __fdividef(m, 1.0f + b2);
  const float bz = sqrt_approx(b2) + of::normal_from_u32(ubits);
  return a * bz * bz;
}

__device__ __forceinline__ float exp_branch(float m, float psi, float u) {
  const float p = __fdividef(psi - 1.0f, psi + 1.0f);
  if (u <= p) return 0.0f;
  const float L = (__log2f(1.0f - p) - __log2f(1.0f - u)) * kLn2;
  return __fdividef(m * L, 1.0f - p);
}

// Forward QE variance step with the (optional) smoothed switch.
__device__ __forceinline__ float qe_vnext(const AdjC& c, float v, const QeDraw& d) {
  const float m = fmaf(v - c.theta, c.e, c.theta);
  const float s2 = fmaf(v, c.c1, c.c2);
  const float inv_m = __fdividef(1.0f, m);
  const float psi = s2 * inv_m * inv_m;
  // each branch inlined once: quadratic below the band's top, exponential
  // above its bottom, blended inside the band
  const bool need_q = psi <= c.sw_hi, need_e = psi > c.sw_lo;
  float vq = 0.0f, ve = 0.0f;
  if (need_q) vq = quad_branch(m, psi, d.ubits);
  if (need_e) ve = exp_branch(m, psi, d.u);
  if (!need_e) return vq;
  if (!need_q) return ve;
  const float s = (psi - c.sw_lo) * c.sw_inv_width;
  const float w = s * s * fmaf(-2.0f, s, 3.0f);
  return fmaf(w, ve - vq, vq);
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

// dvn = A1 dm + A2 dpsi on the quadratic branch
__device__ __forceinline__ void quad_jac(float m, float psi, uint32_t ubits, float& vq, float& A1, float& A2) {
  const float t = __fdividef(2.0f, psi);
  const float root = sqrt_approx(t * (t - 1.0f));
  const float b2 = (t - 1.0f) + root;
  const float b = sqrt_approx(b2);
  const float inv_1b2 = __fdividef(1.0f, 1.0f + b2);
  const float a = m * inv_1b2;
  const float bz = b + of::normal_from_u32(ubits);
  const float dv_da = bz * bz;
  const float dv_db = 2.0f * a * bz;
  const float da_db2 = -a * inv_1b2;
  const float db_db2 = __fdividef(0.5f, b);
  const float db2_dt = 1.0f + __fdividef(fmaf(2.0f, t, -1.0f), 2.0f * root);
  const float dt_dpsi = -0.5f * t * t;
  vq = a * dv_da;
  A1 = dv_da * inv_1b2;
  A2 = fmaf(dv_da, da_db2, dv_db * db_db2) * db2_dt * dt_dpsi;
}

// the same on the exponential branch
__device__ __forceinline__ void exp_jac(float m, float psi, float u, float& ve, float& A1, float& A2) {
  const float inv_p1 = __fdividef(1.0f, psi + 1.0f);
  const float p = (psi - 1.0f) * inv_p1;
  ve = A1 = A2 = 0.0f;
  if (u > p) {
    const float inv_1p = __fdividef(1.0f, 1.0f - p);
    const float L = (__log2f(1.0f - p) - __log2f(1.0f - u)) * kLn2;
    ve = m * L * inv_1p;
    A1 = L * inv_1p;
    A2 = m * (L - 1.0f) * inv_1p * inv_1p * (2.0f * inv_p1 * inv_p1);
  }
}

__device__ __forceinline__ StepJac qe_jacobian(const AdjC& c, float v, float vn, const QeDraw& d) {
  StepJac J;
  const float m = fmaf(v - c.theta, c.e, c.theta);
  const float s2 = fmaf(v, c.c1, c.c2);
  const float inv_m = __fdividef(1.0f, m);
  const float psi = s2 * inv_m * inv_m;
  float A1, A2;
  {
    // each branch inlined once, as in qe_vnext
    const bool need_q = psi <= c.sw_hi, need_e = psi > c.sw_lo;
    float vq = 0.0f, q1 = 0.0f, q2 = 0.0f, ve = 0.0f, e1 = 0.0f, e2 = 0.0f;
    if (need_q) quad_jac(m, psi, d.ubits, vq, q1, q2);
    if (need_e) exp_jac(m, psi, d.u, ve, e1, e2);
    if (!need_e) {
      A1 = q1;
      A2 = q2;
    } else if (!need_q) {
      A1 = e1;
      A2 = e2;
    } else {
      const float s = (psi - c.sw_lo) * c.sw_inv_width;
      const float w = s * s * fmaf(-2.0f, s, 3.0f);
      const float dw = 6.0f * s * (1.0f - s) * c.sw_inv_width;
      A1 = fmaf(w, e1 - q1, q1);
      A2 = fmaf(w, e2 - q2, q2) + (ve - vq) * dw;
    }
  }
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

// ---- kernel 1: forward pass, checkpoints, payoff ------------------------------
__global__ void __launch_bounds__(128) adjoint_forward(const __grid_constant__ AdjC c, double* __restrict__ partials,
                                                       int write_ckpt) {
  __shared__ double sh[2 * 4];
  double acc[2] = {0.0, 0.0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.paths; i += stride) {
    const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
    float v = c.v0, y = 0.0f;
    of::Kahan32 sum_s;
    for (int seg = 0; seg < c.n_seg; ++seg) {
      if (write_ckpt) {
        c.ck_v[(size_t)seg * c.paths + i] = v;
        c.ck_y[(size_t)seg * c.paths + i] = y;
      }
      const int j0 = seg * kSeg;
#pragma unroll 2
      for (int k = 0; k < kSeg; k += 2) {
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
    const float und = c.asian ? c.s0 * (float)(sum_s.value() * (double)c.inv_steps) : c.s0 * __expf(y);
    const float intr = c.call ? und - c.strike : c.strike - und;
    const double pv = intr > 0.0f ? c.disc * (double)intr : 0.0;
    acc[0] += pv;
    acc[1] += pv * pv;
    if (write_ckpt) {
      c.und[i] = und;
      c.grad[i] = intr > 0.0f ? (float)c.disc * (c.call ? 1.0f : -1.0f) : 0.0f;
    }
  }
  of::block_sum<2>(acc, sh);
  if (threadIdx.x == 0) {
    partials[(int64_t)blockIdx.x * 2] = acc[0];
    partials[(int64_t)blockIdx.x * 2 + 1] = acc[1];
  }
}

// One path's backward sweep; sv/ss are this lane's columns of the block's
// shared segment buffers (stride kBwdThreads).
__device__ void sweep_path(const AdjC& c, int64_t i, float* sv, float* ss, double* acc) {
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  const float g = c.grad[i];
  const float und = c.und[i];
  const float direct = c.asian ? g * c.s0 * c.inv_steps : 0.0f;  // d pv / d y_j = direct * e^{y_j}
  float ybar = c.asian ? 0.0f : g * und;                         // European: seed at y_M
  float wbar = 0.0f, kbar = 0.0f, tbar = 0.0f, xbar = 0.0f, rbar = 0.0f, mubar = 0.0f;
  for (int seg = c.n_seg - 1; seg >= 0; --seg) {
    const int j0 = seg * kSeg;
    const int len = (c.steps - j0) < kSeg ? (c.steps - j0) : kSeg;
    float vv = c.ck_v[(size_t)seg * c.paths + i], yy = c.ck_y[(size_t)seg * c.paths + i];
    sv[0] = vv;
    for (int k = 0; k < len; k += 2) {
      const int j = j0 + k;
      const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 1), lo, hi, kAdjStreamTag), c.keys);
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        if (k + o < len) {
          const QeDraw d = draw_of(r, o);
          const float vn = qe_vnext(c, vv, d);
          yy = qe_ynext(c, yy, vv, vn, d.zx);
          vv = vn;
          sv[(k + o + 1) * kBwdThreads] = vv;
          ss[(k + o + 1) * kBwdThreads] = __expf(yy);
        }
      }
    }
    for (int k = (len - 1) & ~1; k >= 0; k -= 2) {
      const int j = j0 + k;
      const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 1), lo, hi, kAdjStreamTag), c.keys);
      // not unrolled: one copy of the step Jacobian keeps the kernel's code
      // within the instruction cache (instruction-fetch stalls were the
      // largest stall with two copies)
#pragma unroll 1
      for (int o = 1; o >= 0; --o) {
        if (k + o < len) {
          ybar = fmaf(direct, ss[(k + o + 1) * kBwdThreads], ybar);  // y_{j+o+1} enters the average
          const QeDraw d = draw_of(r, o);
          const StepJac J = qe_jacobian(c, sv[(k + o) * kBwdThreads], sv[(k + o + 1) * kBwdThreads], d);
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
  const double pv = c.disc * (double)(c.call ? und - c.strike : c.strike - und);
  const double gk[7] = {(double)(g * und / c.s0), (double)mubar - c.T * pv, wbar, kbar, tbar, xbar, rbar};
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    acc[k] += gk[k];
    acc[7 + k] += gk[k] * gk[k];
  }
}

// ---- kernel 2: backward sweeps over the in-the-money paths ------------------
// Six 128-thread blocks per SM (the 36 KB of segment buffers allow six): at
// most 80 registers, 1.6 % faster than 93 registers and five blocks.
__global__ void __launch_bounds__(kBwdThreads, 6) adjoint_backward(const __grid_constant__ AdjC c,
                                                               double* __restrict__ partials) {
  __shared__ float seg_v[(kSeg + 1) * kBwdThreads];
  __shared__ float seg_s[(kSeg + 1) * kBwdThreads];
  __shared__ int64_t queue[kBwdWarps][64];
  __shared__ double sh[14 * kBwdWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double acc[14];
#pragma unroll
  for (int k = 0; k < 14; ++k) acc[k] = 0.0;
  const int64_t nranges = (c.paths + kRangePerWarp - 1) / kRangePerWarp;
  const int64_t gwarps = (int64_t)gridDim.x * kBwdWarps;
  int qn = 0;  // queued in-the-money paths; the queue carries over from one range to the next
  for (int64_t rg = (int64_t)blockIdx.x * kBwdWarps + warp; rg < nranges; rg += gwarps) {
    const int64_t r0 = rg * kRangePerWarp;
    for (int chunk = 0; chunk < kRangePerWarp; chunk += 32) {
      const int64_t i = r0 + chunk + lane;
      const bool itm = i < c.paths && c.grad[i] != 0.0f;
      const unsigned mask = __ballot_sync(of::kFullMask, itm);
      if (itm) queue[warp][qn + __popc(mask & ((1u << lane) - 1u))] = i;
      qn += __popc(mask);
      __syncwarp();
      if (qn >= 32) {
        sweep_path(c, queue[warp][lane], seg_v + threadIdx.x, seg_s + threadIdx.x, acc);
        __syncwarp();
        if (lane < qn - 32) queue[warp][lane] = queue[warp][32 + lane];
        qn -= 32;
        __syncwarp();
      }
    }
  }
  if (lane < qn) sweep_path(c, queue[warp][lane], seg_v + threadIdx.x, seg_s + threadIdx.x, acc);
  __syncwarp();
  // block reduction of the 14 sums (fixed order)
#pragma unroll
  for (int k = 0; k < 14; ++k) {
    const double w = of::warp_sum(acc[k]);
    if (lane == 0) sh[warp * 14 + k] = w;
  }
  __syncthreads();
  if (threadIdx.x < 14) {
    double a = 0.0;
    for (int w = 0; w < kBwdWarps; ++w) a += sh[w * 14 + threadIdx.x];
    partials[(int64_t)blockIdx.x * 14 + threadIdx.x] = a;
  }
}

// Price-only FP64 pass over the same draws (the bits of each Philox counter
// give the same U, Zv, Zx), for bump-and-revalue with common random numbers:
// a relative bump of 1e-4 moves a step's log-increment by ~1e-8, below the
// FP32 resolution of the path state, so the revaluation runs in FP64.
struct AdjC64 {
  double e, c1, c2, theta, c0, K1, K2, k34, s0, strike, inv_steps, disc, v0;
  double sw_lo, sw_hi, sw_inv_width;
  int32_t steps, call, asian;
  int64_t paths;
  of::PhiloxKeys keys;
};

__device__ __forceinline__ double quad64(double m, double psi, double zv) {
  const double t = 2.0 / psi;
  const double b2 = (t - 1.0) + sqrt(t * (t - 1.0));
  const double a = m / (1.0 + b2);
  const double bz = sqrt(b2) + zv;
  return a * bz * bz;
}

__device__ __forceinline__ double exp64(double m, double psi, double u) {
  const double p = (psi - 1.0) / (psi + 1.0);
  return (u <= p) ? 0.0 : m * log((1.0 - p) / (1.0 - u)) / (1.0 - p);
}

__global__ void __launch_bounds__(128) forward64_kernel(const __grid_constant__ AdjC64 c,
                                                        double* __restrict__ partials) {
  __shared__ double sh[2 * 4];
  double acc[2] = {0.0, 0.0};
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
        const double zv = (double)of::normal_from_u32(ub);
        const double m = c.theta + (v - c.theta) * c.e;
        const double s2 = v * c.c1 + c.c2;
        const double psi = s2 / (m * m);
        double vn;
        if (psi <= c.sw_lo) {
          vn = quad64(m, psi, zv);
        } else if (psi > c.sw_hi) {
          vn = exp64(m, psi, u);
        } else {
          const double vq = quad64(m, psi, zv), ve = exp64(m, psi, u);
          const double s = (psi - c.sw_lo) * c.sw_inv_width;
          vn = vq + s * s * (3.0 - 2.0 * s) * (ve - vq);
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
  of::block_sum<2>(acc, sh);
  if (threadIdx.x == 0) {
    partials[(int64_t)blockIdx.x * 2] = acc[0];
    partials[(int64_t)blockIdx.x * 2 + 1] = acc[1];
  }
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
  if (p->checkpoint_every != kSeg) return of_fail(ctx, OF_ERR_UNSUPPORTED, "checkpoint interval must be 32");
  if (p->forward_only < 0 || p->forward_only > 2)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "forward_only must be 0, 1 or 2");
  if (!(p->qe_switch_band >= 0.0 && p->qe_switch_band <= 0.25))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "qe_switch_band must lie in [0, 0.25]");
  if (p->num_steps > (int64_t)kMaxSegments * kSeg)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "at most %d steps", kMaxSegments * kSeg);
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
  const double K0 = -r * k * th * dt / x;
  const double K1 = 0.5 * dt * (k * r / x - 0.5) - r / x;
  const double K2 = 0.5 * dt * (k * r / x - 0.5) + r / x;
  const double k34 = 0.5 * dt * (1.0 - r * r);
  const double band = p->qe_switch_band;
  const double sw_lo = 1.5 - band, sw_hi = 1.5 + band;
  const double sw_inv_width = band > 0.0 ? 1.0 / (2.0 * band) : 0.0;
  const int32_t n_seg = (int32_t)((p->num_steps + kSeg - 1) / kSeg);
  const bool call = p->option_type == OF_CALL, asian = p->payoff == OF_PAYOFF_ASIAN;

  void *d_part = nullptr, *d_sums = nullptr, *h = nullptr;
  const int blk = 128;
  const int64_t want = (p->num_paths + blk - 1) / blk;
  float ms = 0.0f;
  double s[16] = {0};
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
    d.sw_lo = sw_lo;
    d.sw_hi = sw_hi;
    d.sw_inv_width = sw_inv_width;
    d.steps = (int32_t)p->num_steps;
    d.call = call;
    d.asian = asian;
    d.paths = p->num_paths;
    d.keys = of::philox_keys(p->seed);
    const int64_t cap = (int64_t)ctx->sm_count * of_blocks_per_sm((const void*)forward64_kernel, blk, 0);
    const int grid = (int)(want < cap ? want : cap);
    OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)grid * 2 * sizeof(double), &d_part));
    OF_TRY(of_scratch(ctx, SLOT_SUMS, 16 * sizeof(double), &d_sums));
    OF_TRY(of_pinned(ctx, 16 * sizeof(double), &h));
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
    forward64_kernel<<<grid, blk, 0, ctx->stream>>>(d, (double*)d_part);
    OF_CUDA_TRY(ctx, cudaGetLastError());
    OF_TRY(of_reduce_rows(ctx, (const double*)d_part, grid, 2, (double*)d_sums));
  } else {
    AdjC c{};
    c.e = (float)e;
    c.c1 = (float)c1;
    c.c2 = (float)c2;
    c.theta = (float)th;
    c.c0 = (float)((p->rate - p->dividend_yield) * dt + K0);
    c.K1 = (float)K1;
    c.K2 = (float)K2;
    c.k34 = (float)k34;
    c.dt = (float)dt;
    c.sw_lo = (float)sw_lo;
    c.sw_hi = (float)sw_hi;
    c.sw_inv_width = (float)sw_inv_width;
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
    c.n_seg = n_seg;
    c.call = call;
    c.asian = asian;
    c.paths = p->num_paths;
    c.keys = of::philox_keys(p->seed);
    const bool greeks = p->forward_only == 0;
    void* d_ck = nullptr;
    if (greeks) {
      // checkpoints (v, y) + per-path gradient and underlying
      const size_t ck_bytes = (size_t)n_seg * p->num_paths * 2 * sizeof(float) + (size_t)p->num_paths * 2 * sizeof(float);
      OF_TRY(of_scratch(ctx, SLOT_ADJ_CKPT, ck_bytes, &d_ck));
      c.ck_v = (float*)d_ck;
      c.ck_y = c.ck_v + (size_t)n_seg * p->num_paths;
      c.grad = c.ck_y + (size_t)n_seg * p->num_paths;
      c.und = c.grad + p->num_paths;
    }
    const int64_t capf = (int64_t)ctx->sm_count * of_blocks_per_sm((const void*)adjoint_forward, blk, 0);
    const int gridf = (int)(want < capf ? want : capf);
    const int64_t nranges = (p->num_paths + kRangePerWarp - 1) / kRangePerWarp;
    const int64_t wantb = (nranges + kBwdWarps - 1) / kBwdWarps;
    const int64_t capb = (int64_t)ctx->sm_count * of_blocks_per_sm((const void*)adjoint_backward, kBwdThreads, 0);
    const int gridb = (int)(wantb < capb ? wantb : capb);
    void* d_bpart = nullptr;
    OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)gridf * 2 * sizeof(double), &d_part));
    OF_TRY(of_scratch(ctx, SLOT_ADJ_AUX, (size_t)(gridb > 0 ? gridb : 1) * 14 * sizeof(double), &d_bpart));
    OF_TRY(of_scratch(ctx, SLOT_SUMS, 16 * sizeof(double), &d_sums));
    OF_TRY(of_pinned(ctx, 16 * sizeof(double), &h));
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
    adjoint_forward<<<gridf, blk, 0, ctx->stream>>>(c, (double*)d_part, greeks ? 1 : 0);
    OF_CUDA_TRY(ctx, cudaGetLastError());
    OF_TRY(of_reduce_rows(ctx, (const double*)d_part, gridf, 2, (double*)d_sums));
    if (greeks) {
      adjoint_backward<<<gridb, kBwdThreads, 0, ctx->stream>>>(c, (double*)d_bpart);
      OF_CUDA_TRY(ctx, cudaGetLastError());
      OF_TRY(of_reduce_rows(ctx, (const double*)d_bpart, gridb, 14, (double*)d_sums + 2));
    }
  }
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(h, d_sums, 16 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
  std::memcpy(s, h, sizeof(s));
  const double n = (double)p->num_paths;
  auto se = [&](double sum, double sum2) {
    const double var = n > 1.0 ? (sum2 - sum * sum / n) / (n - 1.0) : 0.0;
    return std::sqrt((var > 0.0 ? var : 0.0) / n);
  };
  out->price = s[0] / n;
  out->stderr_ = se(s[0], s[1]);
  if (p->forward_only == 0) {
    for (int k2 = 0; k2 < OF_ADJ_COUNT; ++k2) {
      out->greeks[k2] = s[2 + k2] / n;
      out->greeks_stderr[k2] = se(s[2 + k2], s[9 + k2]);
    }
  }
  out->samples = p->num_paths;
  out->kernel_ms = ms;
  return OF_OK;
}
