// mc_philox.cu - FP32 Philox Monte Carlo: the strike strip and the batched book.
//
// Generator: Philox4x32-10, counter {draw block, sample lo, sample hi, stream},
// key = the 64-bit seed; one call yields 4 draws (4 GBM steps or 2 Heston
// steps).  GBM and Heston Euler turn each draw pair into two normals by
// Box-Muller; Heston QE keeps the inverse CDF, which its variance step
// needs (the same uniform drives the exponential branch and, through
// Phi^-1, the quadratic one).  Paths live in registers (one path per thread at a time), payoff
// sums are compensated FP32 per thread and FP64 from the warp level up.
// Compiled with -use_fast_math: sqrt/exp/log/div map to single MUFU
// operations; the few places that need more accuracy say so.
#include <cuda.h>  // CUcontext / CUresult types only; the driver functions are resolved at run time

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "book_greeks.cuh"
#include "bulk_copy.cuh"
#include "of_internal.h"
#include "path_fp32.cuh"

using of::LegState;
using of::StepConsts;

namespace {

constexpr uint32_t kStripStreamTag = 0x53545250u;  // "STRP"

// FP32 constants of a model (computed in FP64, rounded once).
StepConsts make_consts(const of_model* m) {
  StepConsts c{};
  const double dt = m->maturity / (double)m->steps;
  const double sqdt = std::sqrt(dt);
  c.drift = (float)((m->mu - 0.5 * m->sigma * m->sigma) * dt);
  c.diff = (float)(m->sigma * sqdt);
  c.mudt = (float)(m->mu * dt);
  c.half_dt = (float)(0.5 * dt);
  c.sqdt = (float)sqdt;
  c.kdt = (float)(m->kappa * dt);
  c.kdt_theta = (float)(m->kappa * m->theta * dt);
  c.one_m_kdt = (float)(1.0 - m->kappa * dt);
  c.xi = (float)m->xi;
  c.bm_k2 = (float)(-2.0 * 0.69314718055994531 * dt);
  c.rho = (float)m->rho;
  c.rho_c = (float)std::sqrt(1.0 - m->rho * m->rho);
  c.v0 = (float)m->v0;
  c.y_floor = (float)std::log(1e-12 / m->s0);  // s.max(1e-12), simulation.rs:112
  if (m->kind == OF_MODEL_HESTON_QE) {
    const double e = std::exp(-m->kappa * dt);
    c.qe_e = (float)e;
    c.qe_c1 = (float)(m->xi * m->xi * e * (1.0 - e) / m->kappa);
    c.qe_c2 = (float)(m->theta * m->xi * m->xi * (1.0 - e) * (1.0 - e) / (2.0 * m->kappa));
    c.qe_theta = (float)m->theta;
    const double g1 = 0.5, g2 = 0.5, kr = m->kappa * m->rho / m->xi - 0.5;
    c.qe_k0 = (float)(-m->rho * m->kappa * m->theta * dt / m->xi);
    c.qe_k1 = (float)(g1 * dt * kr - m->rho / m->xi);
    c.qe_k2 = (float)(g2 * dt * kr + m->rho / m->xi);
    c.qe_k3 = (float)(g1 * dt * (1.0 - m->rho * m->rho));
    c.qe_k4 = (float)(g2 * dt * (1.0 - m->rho * m->rho));
  }
  return c;
}

// Simulates the terminal log-return of sample i (and of its antithetic twin).
template <int MODEL, bool ANTI>
__device__ __forceinline__ void simulate_terminal(const StepConsts& c, int32_t steps, uint64_t i, uint32_t stream,
                                                  const of::PhiloxKeys& K, float& ya, float& yb) {
  LegState a{0.0f, c.v0}, b{0.0f, c.v0};
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  if (MODEL == OF_MODEL_GBM) {
    float wa = 0.0f;  // sum of normals; y_T = steps*drift + diff*sum
    for (int32_t j = 0; j < steps; j += 4) {
      const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 2), lo, hi, stream), K);
      const float2 p = of::normal_pair_from_u32(r.x, r.y), q = of::normal_pair_from_u32(r.z, r.w);
      wa += p.x;
      if (j + 1 < steps) wa += p.y;
      if (j + 2 < steps) wa += q.x;
      if (j + 3 < steps) wa += q.y;
    }
    const float base = (float)steps * c.drift;
    ya = fmaf(c.diff, wa, base);
    yb = fmaf(-c.diff, wa, base);
  } else if (MODEL == OF_MODEL_HESTON_EULER) {
    const int32_t pairs = steps >> 1;  // full Philox calls; an odd last step below
    for (int32_t q = 0; q < pairs; ++q) {
      const uint4 r = of::philox4x32_10(make_uint4((uint32_t)q, lo, hi, stream), K);
      float2 z = of::normal_pair_scaled_from_u32(r.x, r.y, c.bm_k2);
      of::heston_euler_step(a, c, z.x, z.y);
      if (ANTI) of::heston_euler_step(b, c, -z.x, -z.y);
      z = of::normal_pair_scaled_from_u32(r.z, r.w, c.bm_k2);
      of::heston_euler_step(a, c, z.x, z.y);
      if (ANTI) of::heston_euler_step(b, c, -z.x, -z.y);
    }
    if (steps & 1) {
      const uint4 r = of::philox4x32_10(make_uint4((uint32_t)pairs, lo, hi, stream), K);
      const float2 z = of::normal_pair_scaled_from_u32(r.x, r.y, c.bm_k2);
      of::heston_euler_step(a, c, z.x, z.y);
      if (ANTI) of::heston_euler_step(b, c, -z.x, -z.y);
    }
    ya = a.y;
    yb = b.y;
  } else {
    for (int32_t j = 0; j < steps; j += 2) {
      const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 1), lo, hi, stream), K);
      float u = of::uniform_from_u32(r.x), zx = of::normal_from_u32(r.y);
      of::heston_qe_step(a, c, u, 1.0f, zx, r.x);
      if (ANTI) of::heston_qe_step(b, c, 1.0f - u, -1.0f, -zx, r.x);
      if (j + 1 < steps) {
        u = of::uniform_from_u32(r.z);
        zx = of::normal_from_u32(r.w);
        of::heston_qe_step(a, c, u, 1.0f, zx, r.z);
        if (ANTI) of::heston_qe_step(b, c, 1.0f - u, -1.0f, -zx, r.z);
      }
    }
    ya = a.y;
    yb = b.y;
  }
}

// ILP independent samples advanced in the same loop by one thread: the
// Philox rounds of the samples are separate dependency chains, so their
// instructions interleave and fill the fixed-latency gaps of one chain.
template <int MODEL, bool ANTI, int ILP>
__device__ __forceinline__ void simulate_terminal_n(const StepConsts& c, int32_t steps, const uint64_t (&idx)[ILP],
                                                    uint32_t stream, const of::PhiloxKeys& K, float (&ya)[ILP],
                                                    float (&yb)[ILP]) {
  if (ILP == 1) {
    simulate_terminal<MODEL, ANTI>(c, steps, idx[0], stream, K, ya[0], yb[0]);
    return;
  }
  uint32_t lo[ILP], hi[ILP];
#pragma unroll
  for (int l = 0; l < ILP; ++l) {
    lo[l] = (uint32_t)idx[l];
    hi[l] = (uint32_t)(idx[l] >> 32);
  }
  if (MODEL == OF_MODEL_GBM) {
    float w[ILP];
#pragma unroll
    for (int l = 0; l < ILP; ++l) w[l] = 0.0f;
    for (int32_t j = 0; j < steps; j += 4) {
#pragma unroll
      for (int l = 0; l < ILP; ++l) {
        const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 2), lo[l], hi[l], stream), K);
        const float2 p = of::normal_pair_from_u32(r.x, r.y), q = of::normal_pair_from_u32(r.z, r.w);
        w[l] += p.x;
        if (j + 1 < steps) w[l] += p.y;
        if (j + 2 < steps) w[l] += q.x;
        if (j + 3 < steps) w[l] += q.y;
      }
    }
    const float base = (float)steps * c.drift;
#pragma unroll
    for (int l = 0; l < ILP; ++l) {
      ya[l] = fmaf(c.diff, w[l], base);
      yb[l] = fmaf(-c.diff, w[l], base);
    }
  } else if (MODEL == OF_MODEL_HESTON_EULER && ILP == 2 && !ANTI) {
    // the two samples' legs in packed pairs: each half is the one-sample
    // loop's arithmetic, bit for bit (antithetic pairs keep the scalar loop,
    // whose four legs fit the register budget without the pair alignment)
    of::LegState2 a{make_float2(0.0f, 0.0f), make_float2(c.v0, c.v0)};
    const int32_t pairs = steps >> 1;
    float2 w1, w2;
    for (int32_t q = 0; q < pairs; ++q) {
      const uint4 r0 = of::philox4x32_10(make_uint4((uint32_t)q, lo[0], hi[0], stream), K);
      const uint4 r1 = of::philox4x32_10(make_uint4((uint32_t)q, lo[1], hi[1], stream), K);
      of::normal_pairs_scaled2_from_u32(r0.x, r0.y, r1.x, r1.y, c.bm_k2, w1, w2);
      of::heston_euler_step2(a, c, w1, w2);
      of::normal_pairs_scaled2_from_u32(r0.z, r0.w, r1.z, r1.w, c.bm_k2, w1, w2);
      of::heston_euler_step2(a, c, w1, w2);
    }
    if (steps & 1) {
      const uint4 r0 = of::philox4x32_10(make_uint4((uint32_t)pairs, lo[0], hi[0], stream), K);
      const uint4 r1 = of::philox4x32_10(make_uint4((uint32_t)pairs, lo[1], hi[1], stream), K);
      of::normal_pairs_scaled2_from_u32(r0.x, r0.y, r1.x, r1.y, c.bm_k2, w1, w2);
      of::heston_euler_step2(a, c, w1, w2);
    }
    ya[0] = a.y.x;  // yb stays 0: there is no antithetic leg
    ya[1] = a.y.y;
  } else if (MODEL == OF_MODEL_HESTON_EULER) {
    LegState a[ILP], b[ILP];
#pragma unroll
    for (int l = 0; l < ILP; ++l) a[l] = b[l] = LegState{0.0f, c.v0};
    const int32_t pairs = steps >> 1;
    for (int32_t q = 0; q < pairs; ++q) {
#pragma unroll
      for (int l = 0; l < ILP; ++l) {
        const uint4 r = of::philox4x32_10(make_uint4((uint32_t)q, lo[l], hi[l], stream), K);
        float2 z = of::normal_pair_scaled_from_u32(r.x, r.y, c.bm_k2);
        of::heston_euler_step(a[l], c, z.x, z.y);
        if (ANTI) of::heston_euler_step(b[l], c, -z.x, -z.y);
        z = of::normal_pair_scaled_from_u32(r.z, r.w, c.bm_k2);
        of::heston_euler_step(a[l], c, z.x, z.y);
        if (ANTI) of::heston_euler_step(b[l], c, -z.x, -z.y);
      }
    }
    if (steps & 1) {
#pragma unroll
      for (int l = 0; l < ILP; ++l) {
        const uint4 r = of::philox4x32_10(make_uint4((uint32_t)pairs, lo[l], hi[l], stream), K);
        const float2 z = of::normal_pair_scaled_from_u32(r.x, r.y, c.bm_k2);
        of::heston_euler_step(a[l], c, z.x, z.y);
        if (ANTI) of::heston_euler_step(b[l], c, -z.x, -z.y);
      }
    }
#pragma unroll
    for (int l = 0; l < ILP; ++l) {
      ya[l] = a[l].y;
      yb[l] = b[l].y;
    }
  } else {
#pragma unroll
    for (int l = 0; l < ILP; ++l) simulate_terminal<MODEL, ANTI>(c, steps, idx[l], stream, K, ya[l], yb[l]);
  }
}

// ---------------------------------------------------------------------------
// Strike strip: one shared path set, KPL strikes per lane.
// ---------------------------------------------------------------------------
struct StripParams {
  StepConsts c;
  int64_t samples;
  int32_t steps, n_strikes, option_type, antithetic;
  float s0;
  of::PhiloxKeys keys;
  const float* strikes;
  uint32_t* status;  // warp-specialised kernel: nonzero when a ring wait gave up
};

template <int KPL, int MODEL, bool ANTI, int ILP = 1>
__global__ void __launch_bounds__(256, 5) strip_kernel(const __grid_constant__ StripParams P,
                                                    double* __restrict__ partials) {
  extern __shared__ double sh_strip[];  // [warps][n_strikes][2]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  float K[KPL];
  of::Kahan32 s1[KPL], s2[KPL];
#pragma unroll
  for (int q = 0; q < KPL; ++q) {
    const int k = lane + 32 * q;
    K[q] = k < P.n_strikes ? P.strikes[k] : 0.0f;
  }
  const bool call = P.option_type == OF_CALL;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  // a warp round covers 32*ILP consecutive samples: lane + 32*l for l < ILP
  for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + warp * 32) * ILP; base < P.samples;
       base += nthreads * ILP) {
    uint64_t idx[ILP];
    float ya[ILP], yb[ILP], sa[ILP], sb[ILP];
#pragma unroll
    for (int l = 0; l < ILP; ++l) {
      idx[l] = (uint64_t)(base + lane + 32 * l);
      ya[l] = yb[l] = 0.0f;
    }
    if (base + lane < P.samples)  // lanes past the end skip the paths; their shuffled values are unused
      simulate_terminal_n<MODEL, ANTI, ILP>(P.c, P.steps, idx, kStripStreamTag, P.keys, ya, yb);
#pragma unroll
    for (int l = 0; l < ILP; ++l) {
      sa[l] = P.s0 * __expf(ya[l]);
      sb[l] = P.s0 * __expf(yb[l]);
    }
#pragma unroll
    for (int l = 0; l < ILP; ++l) {
      const int64_t rem = P.samples - (base + 32 * l);
      const int nvalid = rem < 0 ? 0 : (rem < 32 ? (int)rem : 32);
      for (int j = 0; j < nvalid; ++j) {
        const float st = __shfl_sync(of::kFullMask, sa[l], j);
        const float sta = ANTI ? __shfl_sync(of::kFullMask, sb[l], j) : 0.0f;
#pragma unroll
        for (int q = 0; q < KPL; ++q) {
          float x = fmaxf(call ? st - K[q] : K[q] - st, 0.0f);
          if (ANTI) x = 0.5f * (x + fmaxf(call ? sta - K[q] : K[q] - sta, 0.0f));
          s1[q].add(x);
          s2[q].add(x * x);
        }
      }
    }
  }
  const int n = P.n_strikes;
#pragma unroll
  for (int q = 0; q < KPL; ++q) {
    const int k = lane + 32 * q;
    if (k < n) {
      sh_strip[(warp * n + k) * 2] = s1[q].value();
      sh_strip[(warp * n + k) * 2 + 1] = s2[q].value();
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 2 * n; t += blockDim.x) {
    double acc = 0.0;
    for (int w = 0; w < nw; ++w) acc += sh_strip[w * 2 * n + t];
    partials[(int64_t)blockIdx.x * 2 * n + t] = acc;
  }
}

// ---------------------------------------------------------------------------
// Warp-specialised strike strip (tile_ilp = 3).
//
// The step loop of strip_kernel alternates two instruction mixes: the Philox
// rounds (32x32->64 integer multiplies on the FMA-heavy pipe, three-input
// XORs on the ALU) and the Box-Muller pair plus the Heston step (lg2, sqrt,
// sin, cos and sqrt on the MUFU pipe, FP32 FMAs).  All warps of an SM run the
// same phase at about the same time, so one pipe waits while the other is
// saturated.  Here half of the warps only generate: producer warp c + 4
// computes the Philox blocks of the 32 samples its consumer warp c simulates
// and writes them to a ring in shared memory; the consumer warps only turn
// draws into normals, steps and payoffs.  The scheduler then always has
// warps of both mixes to issue.  Same draws, same steps and same payoffs per
// sample as strip_kernel<..., ILP = 1>; the per-warp sums group samples
// differently, so results agree to the rounding of the FP32 partial sums.
//
// Ring: per consumer kWsSlots chunks of kWsChunk Philox blocks x 32 lanes
// (uint4), with a full and an empty mbarrier per chunk (32 arrivals each).
// Every wait is bounded (kWsWaitNs of the global timer), suspends the warp in
// the barrier between polls so a waiting warp leaves the issue slots to
// working ones, and its outcome is made warp-uniform; a warp whose wait gives up sets P.status and leaves its
// loops, so its partner's next wait gives up too and the block still reaches
// its final reduction.
// ---------------------------------------------------------------------------
constexpr int kWsPairs = 4;   // consumer warps 0..3, producer warps 4..7
constexpr int kWsChunk = 4;   // Philox blocks per ring chunk
constexpr int kWsSlots = 3;   // chunks in flight per pair
constexpr uint64_t kWsWaitNs = 1000000000ull;
constexpr uint32_t kWsSleepNs = 20000;  // suspend-time hint of a ring barrier poll
constexpr size_t kWsRingBytes = (size_t)kWsPairs * kWsSlots * kWsChunk * 32 * sizeof(uint4);

// The steps of Philox block q of one sample (and its antithetic twin), as
// simulate_terminal consumes them.
template <int MODEL, bool ANTI>
__device__ __forceinline__ void ws_consume(const StepConsts& c, const uint4 r, int32_t q, int32_t steps,
                                           LegState& a, LegState& b, float& w) {
  if (MODEL == OF_MODEL_GBM) {
    const int32_t j = q * 4;
    const float2 p = of::normal_pair_from_u32(r.x, r.y), pq = of::normal_pair_from_u32(r.z, r.w);
    w += p.x;
    if (j + 1 < steps) w += p.y;
    if (j + 2 < steps) w += pq.x;
    if (j + 3 < steps) w += pq.y;
  } else if (MODEL == OF_MODEL_HESTON_EULER) {
    float2 z = of::normal_pair_scaled_from_u32(r.x, r.y, c.bm_k2);
    of::heston_euler_step(a, c, z.x, z.y);
    if (ANTI) of::heston_euler_step(b, c, -z.x, -z.y);
    if (2 * q + 1 < steps) {
      z = of::normal_pair_scaled_from_u32(r.z, r.w, c.bm_k2);
      of::heston_euler_step(a, c, z.x, z.y);
      if (ANTI) of::heston_euler_step(b, c, -z.x, -z.y);
    }
  } else {
    float u = of::uniform_from_u32(r.x), zx = of::normal_from_u32(r.y);
    of::heston_qe_step(a, c, u, 1.0f, zx, r.x);
    if (ANTI) of::heston_qe_step(b, c, 1.0f - u, -1.0f, -zx, r.x);
    if (2 * q + 1 < steps) {
      u = of::uniform_from_u32(r.z);
      zx = of::normal_from_u32(r.w);
      of::heston_qe_step(a, c, u, 1.0f, zx, r.z);
      if (ANTI) of::heston_qe_step(b, c, 1.0f - u, -1.0f, -zx, r.z);
    }
  }
}

template <int KPL, int MODEL, bool ANTI>
__global__ void __launch_bounds__(256, 5) strip_kernel_ws(const __grid_constant__ StripParams P,
                                                       double* __restrict__ partials) {
  extern __shared__ __align__(16) unsigned char ws_smem[];
  uint4* ring = reinterpret_cast<uint4*>(ws_smem);                       // [pair][slot][block][lane]
  double* sh_strip = reinterpret_cast<double*>(ws_smem + kWsRingBytes);  // [warps][n_strikes][2]
  __shared__ __align__(8) uint64_t full[kWsPairs * kWsSlots], empty[kWsPairs * kWsSlots];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool producer = warp >= kWsPairs;
  const int pair = producer ? warp - kWsPairs : warp;
  if (threadIdx.x == 0) {
    for (int k = 0; k < kWsPairs * kWsSlots; ++k) {
      of::mbar_init(of::smem_u32(full + k), 32);
      of::mbar_init(of::smem_u32(empty + k), 32);
    }
    of::mbar_fence_init();
  }
  __syncthreads();
  float K[KPL];
  of::Kahan32 s1[KPL], s2[KPL];
#pragma unroll
  for (int q = 0; q < KPL; ++q) {
    const int k = lane + 32 * q;
    K[q] = k < P.n_strikes ? P.strikes[k] : 0.0f;
  }
  const bool call = P.option_type == OF_CALL;
  const int32_t spb = MODEL == OF_MODEL_GBM ? 4 : 2;  // steps per Philox block
  const int32_t nq = (P.steps + spb - 1) / spb;       // Philox blocks per sample
  const int64_t stride = (int64_t)gridDim.x * kWsPairs * 32;
  uint4* my_ring = ring + (size_t)pair * kWsSlots * kWsChunk * 32;
  uint32_t g = 0;  // chunks this pair has passed through its ring
  bool ok = true;
  for (int64_t base = ((int64_t)blockIdx.x * kWsPairs + pair) * 32; base < P.samples && ok; base += stride) {
    const uint64_t i = (uint64_t)(base + lane);
    const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
    LegState a{0.0f, P.c.v0}, b{0.0f, P.c.v0};
    float w = 0.0f;
    for (int32_t q0 = 0; q0 < nq; q0 += kWsChunk, ++g) {
      const int slot = (int)(g % kWsSlots);
      const uint32_t use = g / kWsSlots;
      uint4* chunk = my_ring + (size_t)slot * kWsChunk * 32;
      if (producer) {
        const bool free_ok =
            use == 0 || of::mbar_wait_backoff(of::smem_u32(empty + pair * kWsSlots + slot), (use - 1) & 1u,
                                              kWsWaitNs, kWsSleepNs);
        if (!__all_sync(of::kFullMask, free_ok)) {  // the warp leaves together
          ok = false;
          break;
        }
#pragma unroll
        for (int k = 0; k < kWsChunk; ++k)
          if (q0 + k < nq)
            chunk[k * 32 + lane] = of::philox4x32_10(make_uint4((uint32_t)(q0 + k), lo, hi, kStripStreamTag), P.keys);
        of::mbar_arrive(of::smem_u32(full + pair * kWsSlots + slot));
      } else {
        const bool full_ok =
            of::mbar_wait_backoff(of::smem_u32(full + pair * kWsSlots + slot), use & 1u, kWsWaitNs, kWsSleepNs);
        if (!__all_sync(of::kFullMask, full_ok)) {
          ok = false;
          break;
        }
#pragma unroll
        for (int k = 0; k < kWsChunk; ++k)
          if (q0 + k < nq) ws_consume<MODEL, ANTI>(P.c, chunk[k * 32 + lane], q0 + k, P.steps, a, b, w);
        of::mbar_arrive(of::smem_u32(empty + pair * kWsSlots + slot));
      }
    }
    if (producer || !ok) continue;
    float ya, yb;
    if (MODEL == OF_MODEL_GBM) {
      const float basev = (float)P.steps * P.c.drift;
      ya = fmaf(P.c.diff, w, basev);
      yb = fmaf(-P.c.diff, w, basev);
    } else {
      ya = a.y;
      yb = b.y;
    }
    const float sa = P.s0 * __expf(ya), sb = P.s0 * __expf(yb);
    const int64_t rem = P.samples - base;
    const int nvalid = rem < 32 ? (int)rem : 32;
    for (int j = 0; j < nvalid; ++j) {
      const float st = __shfl_sync(of::kFullMask, sa, j);
      const float sta = ANTI ? __shfl_sync(of::kFullMask, sb, j) : 0.0f;
#pragma unroll
      for (int q = 0; q < KPL; ++q) {
        float x = fmaxf(call ? st - K[q] : K[q] - st, 0.0f);
        if (ANTI) x = 0.5f * (x + fmaxf(call ? sta - K[q] : K[q] - sta, 0.0f));
        s1[q].add(x);
        s2[q].add(x * x);
      }
    }
  }
  if (!ok && lane == 0) atomicOr(P.status, 1u);
  const int n = P.n_strikes;
#pragma unroll
  for (int q = 0; q < KPL; ++q) {
    const int k = lane + 32 * q;
    if (k < n) {
      sh_strip[(warp * n + k) * 2] = s1[q].value();
      sh_strip[(warp * n + k) * 2 + 1] = s2[q].value();
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 2 * n; t += blockDim.x) {
    double acc = 0.0;
    for (int w2 = 0; w2 < nw; ++w2) acc += sh_strip[w2 * 2 * n + t];
    partials[(int64_t)blockIdx.x * 2 * n + t] = acc;
  }
}

typedef void (*StripKernelFn)(StripParams, double*);

template <int KPL, int ILP = 1>
StripKernelFn pick_strip(int model, bool anti) {
  if (model == OF_MODEL_GBM)
    return anti ? strip_kernel<KPL, OF_MODEL_GBM, true, ILP> : strip_kernel<KPL, OF_MODEL_GBM, false, ILP>;
  if (model == OF_MODEL_HESTON_EULER)
    return anti ? strip_kernel<KPL, OF_MODEL_HESTON_EULER, true, ILP>
                : strip_kernel<KPL, OF_MODEL_HESTON_EULER, false, ILP>;
  return anti ? strip_kernel<KPL, OF_MODEL_HESTON_QE, true, ILP> : strip_kernel<KPL, OF_MODEL_HESTON_QE, false, ILP>;
}

template <int KPL>
StripKernelFn pick_strip_ws_kpl(int model, bool anti) {
  if (model == OF_MODEL_GBM) return anti ? strip_kernel_ws<KPL, OF_MODEL_GBM, true> : strip_kernel_ws<KPL, OF_MODEL_GBM, false>;
  if (model == OF_MODEL_HESTON_EULER)
    return anti ? strip_kernel_ws<KPL, OF_MODEL_HESTON_EULER, true> : strip_kernel_ws<KPL, OF_MODEL_HESTON_EULER, false>;
  return anti ? strip_kernel_ws<KPL, OF_MODEL_HESTON_QE, true> : strip_kernel_ws<KPL, OF_MODEL_HESTON_QE, false>;
}

StripKernelFn pick_strip_ilp(int kpl, int ilp, int model, bool anti);

// The kernel, its dynamic shared memory and the samples one block covers per
// round, for a strip tile shape: tile 1 or 2 = strip_kernel with that many
// samples in flight per thread (0 = 1), tile 3 = the warp-specialised
// strip_kernel_ws.
struct StripShape {
  StripKernelFn fn;
  size_t smem;
  int64_t samples_per_block;
  bool ws;
};

StripShape strip_shape(int tile, int64_t n_strikes, int model, bool anti, int block) {
  const int kpl = (int)((n_strikes + 31) / 32);
  const size_t sums = (size_t)(block / 32) * (size_t)n_strikes * 2 * sizeof(double);
  if (tile == 3) {
    const StripKernelFn fn = kpl <= 1 ? pick_strip_ws_kpl<1>(model, anti)
                             : kpl <= 2 ? pick_strip_ws_kpl<2>(model, anti) : pick_strip_ws_kpl<4>(model, anti);
    return {fn, kWsRingBytes + sums, (int64_t)kWsPairs * 32, true};
  }
  const int ilp = tile == 2 ? 2 : 1;
  return {pick_strip_ilp(kpl, ilp, model, anti), sums, (int64_t)block * ilp, false};
}

// Kernel for KPL strikes per lane and ILP samples in flight per thread.
StripKernelFn pick_strip_ilp(int kpl, int ilp, int model, bool anti) {
  if (ilp == 2) {
    if (kpl <= 1) return pick_strip<1, 2>(model, anti);
    if (kpl <= 2) return pick_strip<2, 2>(model, anti);
    return pick_strip<4, 2>(model, anti);
  }
  if (kpl <= 1) return pick_strip<1>(model, anti);
  if (kpl <= 2) return pick_strip<2>(model, anti);
  return pick_strip<4>(model, anti);
}

}  // namespace

of_status of_validate_mc(of_ctx* ctx, const of_model* m, const of_payoff* p, const of_mc_config* c);
void of_observation_weights(const of_payoff* p, int64_t steps, std::vector<double>& w, bool& terminal_only);

static of_status validate_fp32_model(of_ctx* ctx, const of_model* m) {
  if (m->steps > 2147483647LL) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps too large for FP32 mode");
  if (m->kind == OF_MODEL_HESTON_QE && !(m->xi > 0.0 && m->theta > 0.0))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "the QE scheme needs xi > 0 and theta > 0");
  return OF_OK;
}

struct of_strip_plan {
  of_ctx* ctx = nullptr;
  StripParams P{};
  int n_strikes = 0, grid = 0, block = 256;
  size_t smem = 0;
  StripKernelFn fn = nullptr;
  bool ws = false;  // warp-specialised kernel: clears and reads back the status word after the sums
  double discount = 1.0;
  int64_t samples = 0;
  float* d_strikes = nullptr;
  double* d_partials = nullptr;
  double* d_sums = nullptr;
  double* h_sums = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

// d_sums holds the 2n sums and one more double whose first word is the
// status of the warp-specialised kernel.
static of_status strip_enqueue(of_strip_plan* pl, cudaStream_t s) {
  const int64_t cols = 2 * (int64_t)pl->n_strikes;
  if (pl->ws) cudaMemsetAsync(pl->d_sums + cols, 0, sizeof(double), s);
  pl->fn<<<pl->grid, pl->block, pl->smem, s>>>(pl->P, pl->d_partials);
  of_launch_reduce_rows(pl->d_partials, pl->grid, cols, pl->d_sums, s);
  cudaMemcpyAsync(pl->h_sums, pl->d_sums, (cols + (pl->ws ? 1 : 0)) * sizeof(double), cudaMemcpyDeviceToHost, s);
  return OF_OK;
}

// OF_ERR_TIMEOUT when the warp-specialised kernel's ring gave up.
static of_status strip_status(of_ctx* ctx, const of_strip_plan* pl) {
  if (pl->ws && *(const uint32_t*)(pl->h_sums + 2 * pl->n_strikes))
    return of_fail(ctx, OF_ERR_TIMEOUT, "strike strip: a producer/consumer ring wait did not complete in time");
  return OF_OK;
}

extern "C" void of_strip_plan_destroy(of_strip_plan* pl) {
  if (!pl) return;
  if (pl->ctx) cudaStreamSynchronize(pl->ctx->stream);
  if (pl->exec) cudaGraphExecDestroy(pl->exec);
  if (pl->graph) cudaGraphDestroy(pl->graph);
  cudaFree(pl->d_strikes);
  cudaFree(pl->d_partials);
  cudaFree(pl->d_sums);
  if (pl->h_sums) cudaFreeHost(pl->h_sums);
  delete pl;
}

// Checks of a strip request that need no device: every strip entry point
// (of_mc_strip, the plans, of_mc_strip_noalloc) runs exactly these.  `ctx`
// only receives the message; it may be a stack context that owns nothing.
static of_status strip_validate(of_ctx* ctx, const of_model* m, int32_t option_type, const double* strikes,
                                int64_t n_strikes, const of_mc_config* cfg) {
  if (!m || !cfg) return of_fail(ctx, OF_ERR_INVALID_INPUT, "null argument");
  of_payoff dummy{};
  dummy.kind = OF_PAYOFF_VANILLA;
  dummy.option_type = option_type;
  dummy.strike = 1.0;
  OF_TRY(of_validate_mc(ctx, m, &dummy, cfg));
  OF_TRY(validate_fp32_model(ctx, m));
  if (m->n_dividends > 0)  // the strip keeps only the sum of the normals of a GBM path
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "the strike strip takes no discrete dividends (price them as a book)");
  if (n_strikes <= 0 || !strikes) return of_fail(ctx, OF_ERR_INVALID_INPUT, "strip needs at least one strike");
  if (n_strikes > 128) return of_fail(ctx, OF_ERR_UNSUPPORTED, "strip supports at most 128 strikes per call");
  for (int64_t k = 0; k < n_strikes; ++k)
    if (!(strikes[k] > 0.0) || !std::isfinite(strikes[k]))
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "strike %lld must be finite and > 0", (long long)k);
  if (cfg->control_variate != OF_CV_NONE)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "the strike strip has no control variate");
  if (cfg->injected_normals)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "injected normals are a FP64 reference-mode test hook");
  if (cfg->tile_ilp < 0 || cfg->tile_ilp > 3)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "tile_ilp must be 0 (default), 1, 2 or 3");
  return OF_OK;
}

// Validates a strip request and fills the plan's parameters, kernel and
// launch shape (no allocation).
static of_status strip_setup(of_ctx* ctx, const of_model* m, int32_t option_type, const double* strikes,
                             int64_t n_strikes, const of_mc_config* cfg, of_strip_plan* pl) {
  OF_TRY(strip_validate(ctx, m, option_type, strikes, n_strikes, cfg));
  OF_TRY(of_ctx_check(ctx));
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  pl->ctx = ctx;
  pl->n_strikes = (int)n_strikes;
  pl->discount = cfg->discount_factor;
  pl->samples = cfg->antithetic ? (cfg->num_paths + 1) / 2 : cfg->num_paths;
  StripParams& P = pl->P;
  P.c = make_consts(m);
  P.samples = pl->samples;
  P.steps = (int32_t)m->steps;
  P.n_strikes = (int32_t)n_strikes;
  P.option_type = option_type;
  P.antithetic = cfg->antithetic ? 1 : 0;
  P.s0 = (float)m->s0;
  P.keys = of::philox_keys(cfg->seed);
  const StripShape sh = strip_shape(cfg->tile_ilp, n_strikes, m->kind, P.antithetic, pl->block);
  pl->fn = sh.fn;
  pl->smem = sh.smem;
  pl->ws = sh.ws;
  const int per_sm = of_blocks_per_sm((const void*)pl->fn, pl->block, pl->smem);
  const int64_t want = (pl->samples + sh.samples_per_block - 1) / sh.samples_per_block;
  const int64_t cap = (int64_t)ctx->sm_count * per_sm;
  pl->grid = (int)std::max<int64_t>(1, std::min(want, cap));
  return OF_OK;
}

extern "C" of_status of_strip_plan_create(of_ctx* ctx, const of_model* m, int32_t option_type, const double* strikes,
                                          int64_t n_strikes, const of_mc_config* cfg, of_strip_plan** out) {
  if (!ctx || !out) return OF_ERR_INVALID_INPUT;
  *out = nullptr;
  of_strip_plan* pl = new of_strip_plan();
  {
    const of_status st = strip_setup(ctx, m, option_type, strikes, n_strikes, cfg, pl);
    if (st != OF_OK) {
      delete pl;
      return st;
    }
  }
  auto fail = [&](of_status st) {
    of_strip_plan_destroy(pl);
    return st;
  };
  std::vector<float> ks((size_t)n_strikes);
  for (int64_t k = 0; k < n_strikes; ++k) ks[(size_t)k] = (float)strikes[k];
  if (cudaMalloc(&pl->d_strikes, ks.size() * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&pl->d_partials, (size_t)pl->grid * 2 * n_strikes * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&pl->d_sums, (2 * n_strikes + 1) * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&pl->h_sums, (2 * n_strikes + 1) * sizeof(double)) != cudaSuccess)
    return fail(of_fail(ctx, OF_ERR_ALLOC, "strip plan allocation failed"));
  if (cudaMemcpy(pl->d_strikes, ks.data(), ks.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(of_fail(ctx, OF_ERR_CUDA, "strike upload failed"));
  pl->P.strikes = pl->d_strikes;
  pl->P.status = (uint32_t*)(pl->d_sums + 2 * n_strikes);
  // Capture kernel + reduction + readback once; launches replay the graph.
  cudaStream_t cap_stream = nullptr;
  if (cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(of_fail(ctx, OF_ERR_CUDA, "capture stream creation failed"));
  cudaError_t e = cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    strip_enqueue(pl, cap_stream);
    e = cudaStreamEndCapture(cap_stream, &pl->graph);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&pl->exec, pl->graph, 0);
  cudaStreamDestroy(cap_stream);
  if (e != cudaSuccess) return fail(of_fail(ctx, OF_ERR_CUDA, "strip graph capture failed: %s", cudaGetErrorString(e)));
  *out = pl;
  return OF_OK;
}

extern "C" of_status of_strip_plan_launch(of_strip_plan* pl) {
  if (!pl) return OF_ERR_INVALID_INPUT;
  OF_TRY(of_ctx_check(pl->ctx));
  OF_CUDA_TRY(pl->ctx, cudaGraphLaunch(pl->exec, pl->ctx->stream));
  return OF_OK;
}

extern "C" of_status of_strip_plan_results(of_strip_plan* pl, of_mc_result* res) {
  if (!pl || !res) return OF_ERR_INVALID_INPUT;
  OF_CUDA_TRY(pl->ctx, cudaStreamSynchronize(pl->ctx->stream));
  OF_TRY(strip_status(pl->ctx, pl));
  for (int k = 0; k < pl->n_strikes; ++k) {
    const double s[5] = {pl->h_sums[2 * k], pl->h_sums[2 * k + 1], 0.0, 0.0, 0.0};
    of_mc_finish(s, pl->samples, OF_CV_NONE, 0.0, pl->discount, &res[k]);
    res[k].kernel_ms = 0.0;
  }
  return OF_OK;
}

// One-shot strip: the context's pooled buffers instead of a plan's own, no
// graph (a single replay would not amortise the capture).
extern "C" of_status of_mc_strip(of_ctx* ctx, const of_model* m, int32_t option_type, const double* strikes,
                                 int64_t n_strikes, const of_mc_config* cfg, of_mc_result* results) {
  if (!ctx || !results) return OF_ERR_INVALID_INPUT;
  of_strip_plan pl;  // setup only; buffers come from the context
  OF_TRY(strip_setup(ctx, m, option_type, strikes, n_strikes, cfg, &pl));
  const int64_t cols = 2 * n_strikes;
  void *d_k = nullptr, *d_part = nullptr, *d_sums = nullptr, *h = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_STRIKES, (size_t)n_strikes * sizeof(float), &d_k));
  OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)pl.grid * cols * sizeof(double), &d_part));
  OF_TRY(of_scratch(ctx, SLOT_SUMS, (size_t)(cols + 1) * sizeof(double), &d_sums));
  OF_TRY(of_pinned(ctx, (size_t)(cols + 1) * sizeof(double) + (size_t)n_strikes * sizeof(float), &h));
  float* hk = (float*)((double*)h + cols + 1);
  for (int64_t k = 0; k < n_strikes; ++k) hk[k] = (float)strikes[k];
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(d_k, hk, (size_t)n_strikes * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  pl.P.strikes = (const float*)d_k;
  pl.P.status = (uint32_t*)((double*)d_sums + cols);
  pl.d_partials = (double*)d_part;
  pl.d_sums = (double*)d_sums;
  pl.h_sums = (double*)h;
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  strip_enqueue(&pl, ctx->stream);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
  const of_status st = strip_status(ctx, &pl);
  for (int64_t k = 0; k < n_strikes && st == OF_OK; ++k) {
    const double s[5] = {pl.h_sums[2 * k], pl.h_sums[2 * k + 1], 0.0, 0.0, 0.0};
    of_mc_finish(s, pl.samples, OF_CV_NONE, 0.0, pl.discount, &results[k]);
    results[k].kernel_ms = ms;
  }
  // The buffers belong to the context: detach them before `pl` goes out of scope.
  pl.d_partials = nullptr;
  pl.d_sums = nullptr;
  pl.h_sums = nullptr;
  return st;
}

// ---------------------------------------------------------------------------
// Batched book: persistent kernel over (option, path-block) tiles.
// ---------------------------------------------------------------------------
namespace {

enum : int32_t {
  BF_ANTI = 1,
  BF_UP = 2,
  BF_IN = 4,
  BF_GEOMETRIC = 8,
  BF_FLOATING = 16,
  BF_TERMINAL_ONLY = 32,
  BF_DAILY = 64,        // every step 1..M observed once (daily fixings)
  BF_NEED_ARITH = 128,
  BF_NEED_GEO = 256,
  BF_CALL = 512
};

struct BookOpt {
  StepConsts c;
  int32_t model, payoff, flags, cv_kind;
  int32_t steps;
  int32_t obs_offset;  // into the shared weight array, -1 when unused
  float s0, strike, barrier_y, rebate, inv_nobs;
  uint32_t stream;
  int32_t div_offset, n_div;  // discrete dividend triggers (GBM), in the shared table
  int32_t kind;               // BK_*: which step loop the option needs
};

// Step loops of the book.  GBM options without dividends and without a
// geometric-average control variate get a loop that carries only what their
// payoff reads: nothing per step (vanilla, terminal-only Asian), the barrier
// test, or the daily-fixing arithmetic sum.  Everything else takes the
// general loop.
// BK_ASIAN_DAILY_GEO: a daily-fixing arithmetic Asian that also carries the
// geometric sum of its control variate.
enum : int32_t { BK_GENERIC = 0, BK_TERMINAL = 1, BK_BARRIER = 2, BK_ASIAN_DAILY = 3, BK_ASIAN_DAILY_GEO = 4 };

// A dividend trigger in log-spot form: after step `step`, a cash dividend
// sets y = log(max(e^y - a, 0)) with a = D/S0; a proportional one adds
// a = log(1 - p).
struct BookDiv {
  int32_t step, kind;
  float a, pad;
};

struct BookTile {
  int32_t opt;
  int32_t count;
  int64_t first;
  int32_t slot;  // position of the tile's partials (option-major order)
  int32_t reserved;
};

struct BookParams {
  const BookOpt* opts;
  const BookTile* tiles;
  const float* obs_w;
  const BookDiv* divs;
  int32_t n_tiles;
  int32_t ppt;  // samples per thread per tile (tile = block * ppt samples)
  of::PhiloxKeys keys;
  int* counter;
  double* partials;  // [slot][5]
};

struct PathObs {
  float arith_sum, arith_comp, geo_sum;
  bool hit;
};

__device__ __forceinline__ void book_observe(const BookOpt& o, PathObs& ob, float y, int32_t idx, const float* obs_w) {
  const int f = o.flags;
  if (o.payoff == OF_PAYOFF_BARRIER) ob.hit |= (f & BF_UP) ? (y >= o.barrier_y) : (y <= o.barrier_y);
  if (f & (BF_NEED_ARITH | BF_NEED_GEO)) {
    const float w = (f & BF_DAILY) ? (idx > 0 ? 1.0f : 0.0f) : __ldg(obs_w + o.obs_offset + idx);
    if (w != 0.0f) {
      if (f & BF_NEED_ARITH) {
        const float add = w * __expf(y);
        const float yk = add - ob.arith_comp;
        const float t = ob.arith_sum + yk;
        ob.arith_comp = (t - ob.arith_sum) - yk;
        ob.arith_sum = t;
      }
      if (f & BF_NEED_GEO) ob.geo_sum = fmaf(w, y, ob.geo_sum);
    }
  }
}

__device__ __forceinline__ float vanilla32(bool call, float s, float k) { return fmaxf(call ? s - k : k - s, 0.0f); }

__device__ __forceinline__ void book_payoff(const BookOpt& o, const PathObs& ob, float y, float& x, float& cv) {
  const int f = o.flags;
  const bool call = f & BF_CALL;
  const float st = o.s0 * __expf(y);
  switch (o.payoff) {
    case OF_PAYOFF_VANILLA:
      x = vanilla32(call, st, o.strike);
      break;
    case OF_PAYOFF_BARRIER: {
      const bool active = (f & BF_IN) ? ob.hit : !ob.hit;
      x = active ? vanilla32(call, st, o.strike) : o.rebate;
      break;
    }
    default: {
      float avg;
      if (f & BF_TERMINAL_ONLY) avg = st;
      else if (f & BF_GEOMETRIC) avg = o.s0 * __expf(ob.geo_sum * o.inv_nobs);
      else avg = o.s0 * ((ob.arith_sum - ob.arith_comp) * o.inv_nobs);
      x = (f & BF_FLOATING) ? vanilla32(call, st, avg) : vanilla32(call, avg, o.strike);
    }
  }
  switch (o.cv_kind) {
    case OF_CV_VANILLA_TERMINAL: cv = vanilla32(call, st, o.strike); break;
    case OF_CV_GEOMETRIC_ASIAN:
      cv = vanilla32(call, (f & BF_TERMINAL_ONLY) ? st : o.s0 * __expf(ob.geo_sum * o.inv_nobs), o.strike);
      break;
    case OF_CV_TERMINAL_SPOT: cv = st; break;
    default: cv = 0.0f;
  }
}

// One sample (and its antithetic twin) of option o; returns (x, y).
// DividendEvent::apply_jump (src/market/dividends.rs:76-83) on the log-spot.
__device__ __forceinline__ float book_dividend(const BookDiv& d, float y) {
  return d.kind == OF_DIV_CASH ? __logf(fmaxf(__expf(y) - d.a, 0.0f)) : y + d.a;
}

// DIVS: the option has discrete dividends (GBM only); without them the step
// loop carries no trigger check.
template <int MODEL, bool DIVS = false>
__device__ __forceinline__ void book_sample(const BookOpt& o, uint64_t i, const of::PhiloxKeys& K, const float* obs_w,
                                            const BookDiv* divs, float& x, float& cvy) {
  const bool anti = o.flags & BF_ANTI;
  const StepConsts& c = o.c;
  LegState a{0.0f, c.v0}, b{0.0f, c.v0};
  PathObs oa{0.0f, 0.0f, 0.0f, false}, obb{0.0f, 0.0f, 0.0f, false};
  book_observe(o, oa, 0.0f, 0, obs_w);
  if (anti) book_observe(o, obb, 0.0f, 0, obs_w);
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  int32_t ev = 0;  // next dividend trigger (GBM)
  const bool observe_each = (o.payoff != OF_PAYOFF_VANILLA) || (o.flags & (BF_NEED_ARITH | BF_NEED_GEO));
  constexpr int SPC = MODEL == OF_MODEL_GBM ? 4 : 2;  // steps per Philox call
  for (int32_t j = 0; j < o.steps; j += SPC) {
    const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j / SPC), lo, hi, o.stream), K);
    const uint32_t rr[4] = {r.x, r.y, r.z, r.w};
    // Box-Muller normals of the two draw pairs (GBM and Heston Euler)
    float2 p01 = make_float2(0.0f, 0.0f), p23 = make_float2(0.0f, 0.0f);
    if (MODEL != OF_MODEL_HESTON_QE) {
      // Heston Euler takes its normals scaled by sqrt(dt) (heston_euler_step)
      const float k2 = MODEL == OF_MODEL_HESTON_EULER ? c.bm_k2 : of::kBoxMullerK2;
      p01 = of::normal_pair_scaled_from_u32(r.x, r.y, k2);
      p23 = of::normal_pair_scaled_from_u32(r.z, r.w, k2);
    }
#pragma unroll
    for (int q = 0; q < SPC; ++q) {
      if (j + q >= o.steps) break;
      if (MODEL == OF_MODEL_GBM) {
        const float z = q == 0 ? p01.x : q == 1 ? p01.y : q == 2 ? p23.x : p23.y;
        a.y = fmaf(c.diff, z, a.y + c.drift);
        if (anti) b.y = fmaf(-c.diff, z, b.y + c.drift);
        for (; DIVS && ev < o.n_div && divs[o.div_offset + ev].step == j + q; ++ev) {  // mc_engine.rs:157-167
          const BookDiv d = divs[o.div_offset + ev];
          a.y = book_dividend(d, a.y);
          if (anti) b.y = book_dividend(d, b.y);
        }
      } else if (MODEL == OF_MODEL_HESTON_EULER) {
        const float2 z = q == 0 ? p01 : p23;
        const float z1 = z.x, z2 = z.y;
        of::heston_euler_step(a, c, z1, z2);
        if (anti) of::heston_euler_step(b, c, -z1, -z2);
      } else {
        const float u = of::uniform_from_u32(rr[2 * q]), zx = of::normal_from_u32(rr[2 * q + 1]);
        of::heston_qe_step(a, c, u, 1.0f, zx, rr[2 * q]);
        if (anti) of::heston_qe_step(b, c, 1.0f - u, -1.0f, -zx, rr[2 * q]);
      }
      if (observe_each) {
        book_observe(o, oa, a.y, j + q + 1, obs_w);
        if (anti) book_observe(o, obb, b.y, j + q + 1, obs_w);
      }
    }
  }
  book_payoff(o, oa, a.y, x, cvy);
  if (anti) {
    float xb, yb;
    book_payoff(o, obb, b.y, xb, yb);
    x = 0.5f * (x + xb);
    cvy = 0.5f * (cvy + yb);
  }
}

// The GBM step loop of one sample (and its antithetic twin) for the option
// kinds BK_BARRIER, BK_ASIAN_DAILY and BK_ASIAN_DAILY_GEO: the same draws,
// steps and observations as book_sample<OF_MODEL_GBM, false>, bit for bit,
// with the option's payoff and flags resolved at compile time instead of
// tested every step.  Whole Philox counter blocks (four steps) run without a
// bounds test; the last, partial block follows.  BK_TERMINAL options take the
// sum of their normals instead (book_terminal_sum).
template <int KIND, bool TWIN>
__device__ __forceinline__ void book_gbm_legs2(const BookOpt& o, uint64_t i0, uint64_t i1, const of::PhiloxKeys& K,
                                               float2& y, PathObs& oa, PathObs& ob);

// Terminal-only options (BK_TERMINAL) need y_T alone: y_T = steps drift +
// diff sum z.  The sum of the path's normals takes each Box-Muller pair as
// its sum (normal_pair_sum_from_u32), four steps at a time ((z0 + z1) +
// (z2 + z3)); a last partial block of one or three steps adds its odd normal
// from the plain transform.  The antithetic twin has y_T = steps drift -
// diff sum z.  The drift is added once instead of every step, so y_T differs
// from the stepwise sum of the general loop by FP32 rounding only.  The
// packed-pair form below sums in the same order, so each of its halves is
// this scalar sum bit for bit.
__device__ __forceinline__ float book_terminal_sum(const BookOpt& o, uint64_t i, const of::PhiloxKeys& K) {
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  float w = 0.0f;
  const int32_t full = o.steps & ~3;
  for (int32_t j = 0; j < full; j += 4) {
    const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 2), lo, hi, o.stream), K);
    w += of::normal_pair_sum_from_u32(r.x, r.y) + of::normal_pair_sum_from_u32(r.z, r.w);
  }
  const int32_t rem = o.steps - full;
  if (rem > 0) {
    const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(full >> 2), lo, hi, o.stream), K);
    if (rem == 1) {
      w += of::normal_pair_from_u32(r.x, r.y).x;
    } else {
      w += of::normal_pair_sum_from_u32(r.x, r.y);
      if (rem == 3) w += of::normal_pair_from_u32(r.z, r.w).x;
    }
  }
  return w;
}

// book_terminal_sum of samples i0 and i1 in packed pairs
__device__ __forceinline__ float2 book_terminal_sums2(const BookOpt& o, uint64_t i0, uint64_t i1,
                                                      const of::PhiloxKeys& K) {
  using of::add2;
  const uint32_t lo0 = (uint32_t)i0, hi0 = (uint32_t)(i0 >> 32), lo1 = (uint32_t)i1, hi1 = (uint32_t)(i1 >> 32);
  float2 w = make_float2(0.0f, 0.0f);
  const int32_t full = o.steps & ~3;
  for (int32_t j = 0; j < full; j += 4) {
    const uint4 r0 = of::philox4x32_10(make_uint4((uint32_t)(j >> 2), lo0, hi0, o.stream), K);
    const uint4 r1 = of::philox4x32_10(make_uint4((uint32_t)(j >> 2), lo1, hi1, o.stream), K);
    w = add2(w, add2(of::normal_pair_sums2_from_u32(r0.x, r0.y, r1.x, r1.y),
                     of::normal_pair_sums2_from_u32(r0.z, r0.w, r1.z, r1.w)));
  }
  const int32_t rem = o.steps - full;
  if (rem > 0) {
    const uint4 r0 = of::philox4x32_10(make_uint4((uint32_t)(full >> 2), lo0, hi0, o.stream), K);
    const uint4 r1 = of::philox4x32_10(make_uint4((uint32_t)(full >> 2), lo1, hi1, o.stream), K);
    float2 a1, a2;
    if (rem == 1) {
      of::normal_pairs_scaled2_from_u32(r0.x, r0.y, r1.x, r1.y, of::kBoxMullerK2, a1, a2);
      w = add2(w, a1);
    } else {
      w = add2(w, of::normal_pair_sums2_from_u32(r0.x, r0.y, r1.x, r1.y));
      if (rem == 3) {
        of::normal_pairs_scaled2_from_u32(r0.z, r0.w, r1.z, r1.w, of::kBoxMullerK2, a1, a2);
        w = add2(w, a1);
      }
    }
  }
  return w;
}

// The payoff of a terminal-only sample from its sum of normals w, averaged
// with its antithetic twin's (-w) when ANTI.
template <bool ANTI>
__device__ __forceinline__ void book_terminal_payoff(const BookOpt& o, float w, float& x, float& cvy) {
  const PathObs none{0.0f, 0.0f, 0.0f, false};
  const float base = (float)o.steps * o.c.drift;
  book_payoff(o, none, fmaf(o.c.diff, w, base), x, cvy);
  if (ANTI) {
    float xb, yb;
    book_payoff(o, none, fmaf(-o.c.diff, w, base), xb, yb);
    x = 0.5f * (x + xb);
    cvy = 0.5f * (cvy + yb);
  }
}

template <int KIND, bool ANTI>
__device__ __forceinline__ void book_sample_gbm(const BookOpt& o, uint64_t i, const of::PhiloxKeys& K, float& x,
                                                float& cvy) {
  if (KIND == BK_TERMINAL) {
    book_terminal_payoff<ANTI>(o, book_terminal_sum(o, i, K), x, cvy);
    return;
  }
  if (ANTI) {  // the sample and its antithetic twin as the two halves of packed pairs
    float2 y;
    PathObs oa, ob;
    book_gbm_legs2<KIND, true>(o, i, i, K, y, oa, ob);
    float xb, yb2;
    book_payoff(o, oa, y.x, x, cvy);
    book_payoff(o, ob, y.y, xb, yb2);
    x = 0.5f * (x + xb);
    cvy = 0.5f * (cvy + yb2);
    return;
  }
  const float drift = o.c.drift, diff = o.c.diff;
  // barrier test as sg*y >= sg*b: sg = +1 for an up barrier, -1 for a down one
  const float sg = (o.flags & BF_UP) ? 1.0f : -1.0f, sgb = sg * o.barrier_y;
  float ya = 0.0f, yb = 0.0f;
  PathObs oa{0.0f, 0.0f, 0.0f, false}, ob{0.0f, 0.0f, 0.0f, false};
  if (KIND == BK_BARRIER) oa.hit = ob.hit = 0.0f >= sgb;  // the scan includes path[0]
  auto add_fixing = [](PathObs& p, float y) {  // Kahan sum of the daily fixings S/S0
    const float yk = __expf(y) - p.arith_comp;
    const float t = p.arith_sum + yk;
    p.arith_comp = (t - p.arith_sum) - yk;
    p.arith_sum = t;
  };
  auto step = [&](float z) {
    ya = fmaf(diff, z, ya + drift);
    if (ANTI) yb = fmaf(-diff, z, yb + drift);
    if (KIND == BK_BARRIER) {
      oa.hit |= sg * ya >= sgb;
      if (ANTI) ob.hit |= sg * yb >= sgb;
    } else if (KIND == BK_ASIAN_DAILY || KIND == BK_ASIAN_DAILY_GEO) {
      add_fixing(oa, ya);
      if (ANTI) add_fixing(ob, yb);
      if (KIND == BK_ASIAN_DAILY_GEO) {  // the general loop's fmaf(1, y, sum): one rounding
        oa.geo_sum += ya;
        if (ANTI) ob.geo_sum += yb;
      }
    }
  };
  const uint32_t lo = (uint32_t)i, hi = (uint32_t)(i >> 32);
  const int32_t full = o.steps & ~3;
  for (int32_t j = 0; j < full; j += 4) {
    const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(j >> 2), lo, hi, o.stream), K);
    const float2 p01 = of::normal_pair_from_u32(r.x, r.y), p23 = of::normal_pair_from_u32(r.z, r.w);
    step(p01.x);
    step(p01.y);
    step(p23.x);
    step(p23.y);
  }
  if (full < o.steps) {
    const uint4 r = of::philox4x32_10(make_uint4((uint32_t)(full >> 2), lo, hi, o.stream), K);
    const float2 p01 = of::normal_pair_from_u32(r.x, r.y), p23 = of::normal_pair_from_u32(r.z, r.w);
    step(p01.x);
    if (full + 1 < o.steps) step(p01.y);
    if (full + 2 < o.steps) step(p23.x);
  }
  book_payoff(o, oa, ya, x, cvy);
  if (ANTI) {
    float xb, yb2;
    book_payoff(o, ob, yb, xb, yb2);
    x = 0.5f * (x + xb);
    cvy = 0.5f * (cvy + yb2);
  }
}

// Two legs of the specialised GBM loop in packed pairs (.x and .y), each half
// the arithmetic of book_sample_gbm bit for bit.  TWIN: the legs are sample
// i0 and its antithetic twin (one Philox stream, normals z and -z); otherwise
// the independent samples i0 and i1 (two streams, Box-Muller of both in packed
// pairs).
template <int KIND, bool TWIN>
__device__ __forceinline__ void book_gbm_legs2(const BookOpt& o, uint64_t i0, uint64_t i1, const of::PhiloxKeys& K,
                                               float2& y, PathObs& oa, PathObs& ob) {
  using of::add2;
  using of::fma2;
  using of::mul2;
  using of::splat2;
  using of::sub2;
  const float2 drift = splat2(o.c.drift);
  const float2 diff = TWIN ? make_float2(o.c.diff, -o.c.diff) : splat2(o.c.diff);
  const float sg = (o.flags & BF_UP) ? 1.0f : -1.0f, sgb = sg * o.barrier_y;
  y = make_float2(0.0f, 0.0f);
  float2 as = make_float2(0.0f, 0.0f), ac = make_float2(0.0f, 0.0f);  // Kahan sums of the daily fixings
  float2 ag = make_float2(0.0f, 0.0f);                                 // geometric sums
  bool ha = false, hb = false;
  if (KIND == BK_BARRIER) ha = hb = 0.0f >= sgb;  // the scan includes path[0]
  auto step = [&](float2 z) {
    y = fma2(diff, z, add2(y, drift));
    if (KIND == BK_BARRIER) {
      const float2 t = mul2(splat2(sg), y);
      ha |= t.x >= sgb;
      hb |= t.y >= sgb;
    } else if (KIND == BK_ASIAN_DAILY || KIND == BK_ASIAN_DAILY_GEO) {
      const float2 yk = sub2(make_float2(__expf(y.x), __expf(y.y)), ac);
      const float2 t = add2(as, yk);
      ac = sub2(sub2(t, as), yk);
      as = t;
      if (KIND == BK_ASIAN_DAILY_GEO) ag = add2(ag, y);
    }
  };
  const uint32_t lo0 = (uint32_t)i0, hi0 = (uint32_t)(i0 >> 32), lo1 = (uint32_t)i1, hi1 = (uint32_t)(i1 >> 32);
  for (int32_t j = 0; j < o.steps; j += 4) {
    const uint4 r0 = of::philox4x32_10(make_uint4((uint32_t)(j >> 2), lo0, hi0, o.stream), K);
    float2 w1, w2, w3, w4;
    if (TWIN) {  // w1 = (z_j, z_j+2), w2 = (z_j+1, z_j+3)
      of::normal_pairs_scaled2_from_u32(r0.x, r0.y, r0.z, r0.w, of::kBoxMullerK2, w1, w2);
      w3 = splat2(w1.y);
      w4 = splat2(w2.y);
      w1 = splat2(w1.x);
      w2 = splat2(w2.x);
    } else {  // wk = step j+k-1 of (i0, i1)
      const uint4 r1 = of::philox4x32_10(make_uint4((uint32_t)(j >> 2), lo1, hi1, o.stream), K);
      of::normal_pairs_scaled2_from_u32(r0.x, r0.y, r1.x, r1.y, of::kBoxMullerK2, w1, w2);
      of::normal_pairs_scaled2_from_u32(r0.z, r0.w, r1.z, r1.w, of::kBoxMullerK2, w3, w4);
    }
    if (j + 4 <= o.steps) {
      step(w1);
      step(w2);
      step(w3);
      step(w4);
    } else {
      step(w1);
      if (j + 1 < o.steps) step(w2);
      if (j + 2 < o.steps) step(w3);
    }
  }
  oa = PathObs{as.x, ac.x, ag.x, ha};
  ob = PathObs{as.y, ac.y, ag.y, hb};
}

// book_sample_gbm<KIND, false> of two samples in one packed loop.
template <int KIND>
__device__ __forceinline__ void book_sample_gbm_pair(const BookOpt& o, uint64_t i0, uint64_t i1,
                                                     const of::PhiloxKeys& K, float& x0, float& cv0, float& x1,
                                                     float& cv1) {
  float2 y;
  PathObs oa, ob;
  book_gbm_legs2<KIND, false>(o, i0, i1, K, y, oa, ob);
  book_payoff(o, oa, y.x, x0, cv0);
  book_payoff(o, ob, y.y, x1, cv1);
}

// book_sample_gbm<BK_TERMINAL, ANTI> of samples i0 and i1: their sums of
// normals in packed pairs (two Philox streams per thread), then each sample's
// payoff (and its twin's) as the scalar form takes it.
template <bool ANTI>
__device__ __forceinline__ void book_terminal_pair(const BookOpt& o, uint64_t i0, uint64_t i1, const of::PhiloxKeys& K,
                                                   float& x0, float& cv0, float& x1, float& cv1) {
  const float2 w = book_terminal_sums2(o, i0, i1, K);
  book_terminal_payoff<ANTI>(o, w.x, x0, cv0);
  book_terminal_payoff<ANTI>(o, w.y, x1, cv1);
}

// One sample of option o: the specialised GBM loop when the option has one,
// the general loop otherwise.
__device__ __forceinline__ void book_dispatch(const BookOpt& o, uint64_t i, const BookParams& P, float& x, float& y) {
  const bool anti = o.flags & BF_ANTI;
  switch (o.kind) {
    case BK_TERMINAL:
      if (anti) book_sample_gbm<BK_TERMINAL, true>(o, i, P.keys, x, y);
      else book_sample_gbm<BK_TERMINAL, false>(o, i, P.keys, x, y);
      return;
    case BK_BARRIER:
      if (anti) book_sample_gbm<BK_BARRIER, true>(o, i, P.keys, x, y);
      else book_sample_gbm<BK_BARRIER, false>(o, i, P.keys, x, y);
      return;
    case BK_ASIAN_DAILY:
      if (anti) book_sample_gbm<BK_ASIAN_DAILY, true>(o, i, P.keys, x, y);
      else book_sample_gbm<BK_ASIAN_DAILY, false>(o, i, P.keys, x, y);
      return;
    case BK_ASIAN_DAILY_GEO:
      if (anti) book_sample_gbm<BK_ASIAN_DAILY_GEO, true>(o, i, P.keys, x, y);
      else book_sample_gbm<BK_ASIAN_DAILY_GEO, false>(o, i, P.keys, x, y);
      return;
    default:
      break;
  }
  if (o.model == OF_MODEL_GBM) {
    if (o.n_div) book_sample<OF_MODEL_GBM, true>(o, i, P.keys, P.obs_w, P.divs, x, y);
    else book_sample<OF_MODEL_GBM, false>(o, i, P.keys, P.obs_w, P.divs, x, y);
  } else if (o.model == OF_MODEL_HESTON_EULER) {
    book_sample<OF_MODEL_HESTON_EULER>(o, i, P.keys, P.obs_w, P.divs, x, y);
  } else {
    book_sample<OF_MODEL_HESTON_QE>(o, i, P.keys, P.obs_w, P.divs, x, y);
  }
}

// Three 256-thread blocks per SM: ptxas's own choice without the hint is 64
// registers with spills in the step loop.
__global__ void __launch_bounds__(256, 3) book_kernel(const __grid_constant__ BookParams P) {
  __shared__ int tile_sh;
  __shared__ double red_sh[5 * 8];
  for (;;) {
    if (threadIdx.x == 0) tile_sh = atomicAdd(P.counter, 1);
    __syncthreads();
    const int t = tile_sh;
    if (t >= P.n_tiles) break;
    const BookTile tile = P.tiles[t];
    const BookOpt o = P.opts[tile.opt];
    of::Kahan32 acc[5];
    auto add = [&](float x, float y) {
      acc[0].add(x);
      acc[1].add(x * x);
      acc[2].add(y);
      acc[3].add(x * y);
      acc[4].add(y * y);
    };
    // specialised GBM kinds without antithetic twins, and terminal-only
    // options with them, run two samples at a time in packed pairs; the sums
    // take them in the same order
    const bool pairs = o.kind != BK_GENERIC && (!(o.flags & BF_ANTI) || o.kind == BK_TERMINAL);
    for (int k = 0; k < P.ppt; ++k) {
      const int local = k * blockDim.x + threadIdx.x;
      if (local >= tile.count) break;
      const uint64_t i = (uint64_t)(tile.first + local);
      float x, y;
      if (pairs && k + 1 < P.ppt && local + (int)blockDim.x < tile.count) {
        const uint64_t i1 = i + blockDim.x;
        float x1, y1;
        if (o.kind == BK_TERMINAL) {
          if (o.flags & BF_ANTI) book_terminal_pair<true>(o, i, i1, P.keys, x, y, x1, y1);
          else book_terminal_pair<false>(o, i, i1, P.keys, x, y, x1, y1);
        }
        else if (o.kind == BK_BARRIER) book_sample_gbm_pair<BK_BARRIER>(o, i, i1, P.keys, x, y, x1, y1);
        else if (o.kind == BK_ASIAN_DAILY_GEO) book_sample_gbm_pair<BK_ASIAN_DAILY_GEO>(o, i, i1, P.keys, x, y, x1, y1);
        else book_sample_gbm_pair<BK_ASIAN_DAILY>(o, i, i1, P.keys, x, y, x1, y1);
        add(x, y);
        add(x1, y1);
        ++k;
        continue;
      }
      book_dispatch(o, i, P, x, y);
      add(x, y);
    }
    double v[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] = acc[k].value();
    of::block_sum<5>(v, red_sh);
    if (threadIdx.x == 0)
      for (int k = 0; k < 5; ++k) P.partials[(int64_t)tile.slot * 5 + k] = v[k];
    __syncthreads();
  }
}

// Running sums of the Greeks modes.  FP32 (with Greeks): the five sums of
// MonteCarloEngine::run compensated, then per Greek its compensated sum and
// plain sum of squares (a few samples per thread per tile; only the standard
// error reads them).  FP64: the five sums.
template <typename R, bool G>
struct GreekAcc;

template <>
struct GreekAcc<float, true> {
  of::Kahan32 s[5], g[4];
  float g2[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  __device__ __forceinline__ void add(const of::GreekSample<float>& v) {
    s[0].add(v.x);
    s[1].add(v.x * v.x);
    s[2].add(v.y);
    s[3].add(v.x * v.y);
    s[4].add(v.y * v.y);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      g[t].add(v.g[t]);
      g2[t] = fmaf(v.g[t], v.g[t], g2[t]);
    }
  }
  __device__ __forceinline__ void values(double (&out)[13]) const {
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = s[k].value();
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      out[5 + t] = g[t].value();
      out[9 + t] = (double)g2[t];
    }
  }
};

template <>
struct GreekAcc<double, true> {
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, g[4] = {0.0, 0.0, 0.0, 0.0}, g2[4] = {0.0, 0.0, 0.0, 0.0};
  __device__ __forceinline__ void add(const of::GreekSample<double>& v) {
    s[0] += v.x;
    s[1] += v.x * v.x;
    s[2] += v.y;
    s[3] += v.x * v.y;
    s[4] += v.y * v.y;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      g[t] += v.g[t];
      g2[t] = fma(v.g[t], v.g[t], g2[t]);
    }
  }
  __device__ __forceinline__ void values(double (&out)[13]) const {
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = s[k];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      out[5 + t] = g[t];
      out[9 + t] = g2[t];
    }
  }
};

template <>
struct GreekAcc<double, false> {
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  __device__ __forceinline__ void add(const of::GreekSample<double>& v) {
    s[0] += v.x;
    s[1] += v.x * v.x;
    s[2] += v.y;
    s[3] += v.x * v.y;
    s[4] += v.y * v.y;
  }
  __device__ __forceinline__ void values(double (&out)[5]) const {
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = s[k];
  }
};

// The book's Greeks modes: the persistent tile loop of book_kernel over the
// per-sample kernels of book_greeks.cuh, one launch per kind group (the
// group's tiles only).  <float, true>: prices and pathwise Greeks (13 sums
// per tile); <double, false>: FP64 prices on the same draws.  FP32 Greeks:
// the terminal group at four blocks per SM (64 registers), the Asian and
// survival-barrier groups at three (the survival step's 91 registers capped
// at 80, with a 4-byte spill: 351 ms for the 4096-option book against
// 368 ms at two blocks); the FP64 modes at two.
template <typename R, bool G, int KG>
__global__ void __launch_bounds__(256, (!G || sizeof(R) == 8) ? 2 : (KG == of::KG_TERMINAL ? 4 : 3))
    book_greeks_kernel(const __grid_constant__ BookParams P, const of::GreekConsts<R>* __restrict__ gc) {
  constexpr int NC = G ? 13 : 5;
  __shared__ int tile_sh;
  __shared__ double red_sh[NC * 8];
  for (;;) {
    if (threadIdx.x == 0) tile_sh = atomicAdd(P.counter, 1);
    __syncthreads();
    const int t = tile_sh;
    if (t >= P.n_tiles) break;
    const BookTile tile = P.tiles[t];
    const of::GreekConsts<R>& c = gc[tile.opt];
    GreekAcc<R, G> acc;
    // FP32: two samples at a time in packed pairs (terminal-only options, and
    // Asian and barrier options without antithetic twins, whose twins pair
    // inside one sample); the sums take them in the same order
    constexpr bool kPairs = std::is_same<R, float>::value;
    const bool pairs = kPairs && (KG == of::KG_TERMINAL || !(c.flags & of::GF_ANTI));
    for (int k = 0; k < P.ppt; ++k) {
      const int local = k * blockDim.x + threadIdx.x;
      if (local >= tile.count) break;
      if constexpr (kPairs) {
        if (pairs && k + 1 < P.ppt && local + (int)blockDim.x < tile.count) {
          of::GreekSample<float> v0, v1;
          const uint64_t i0 = (uint64_t)(tile.first + local), i1 = i0 + blockDim.x;
          if constexpr (KG == of::KG_BARRIER) of::gk_barrier_pair_group<G>(c, i0, i1, P.keys, v0, v1);
          else if constexpr (KG == of::KG_ASIAN) of::gk_asian_pair_group<G>(c, i0, i1, P.keys, P.obs_w, v0, v1);
          else of::gk_terminal_pair_group<G>(c, i0, i1, P.keys, v0, v1);
          acc.add(v0);
          acc.add(v1);
          ++k;
          continue;
        }
      }
      of::GreekSample<R> v;
      of::gk_sample_group<R, G, KG>(c, (uint64_t)(tile.first + local), P.keys, P.obs_w, v);
      acc.add(v);
    }
    double v[NC];
    acc.values(v);
    of::block_sum<NC>(v, red_sh);
    if (threadIdx.x == 0)
      for (int k = 0; k < NC; ++k) P.partials[(int64_t)tile.slot * NC + k] = v[k];
    __syncthreads();
  }
}

// Per-option sums over its tile slots [begin[o], begin[o+1]) in fixed order;
// NC sums per slot.
template <int NC>
__global__ void book_reduce_kernel(const double* __restrict__ partials, const int32_t* __restrict__ begin, int n_opts,
                                   double* __restrict__ sums) {
  const int o = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (o >= n_opts) return;
  double acc[NC];
#pragma unroll
  for (int k = 0; k < NC; ++k) acc[k] = 0.0;
  for (int s = begin[o] + lane; s < begin[o + 1]; s += 32)
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k] += partials[(int64_t)s * NC + k];
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    const double v = of::warp_sum(acc[k]);
    if (lane == 0) sums[(int64_t)o * NC + k] = v;
  }
}

}  // namespace

static_assert(OF_CV_NONE == of::GCV_NONE && OF_CV_VANILLA_TERMINAL == of::GCV_VANILLA_TERMINAL &&
                  OF_CV_GEOMETRIC_ASIAN == of::GCV_GEOMETRIC_ASIAN && OF_CV_TERMINAL_SPOT == of::GCV_TERMINAL_SPOT,
              "the Greeks modes read the control-variate kinds of the ABI");

// Constants of one entry in the Greeks modes (FP64; the FP32 mode rounds
// them once).  `d` is the entry's price-mode record (flags, observation
// weights' offset), `w` its observation weights by step index (empty when it
// has none) and `daily` whether they are the daily fixings 1..steps.
static of_status book_greek_consts(of_ctx* ctx, const of_book_entry& b, int64_t o, const BookOpt& d,
                                   const std::vector<double>& w, bool daily, of::GreekConsts<double>& g) {
  const of_model& m = b.model;
  const of_payoff& p = b.payoff;
  if (m.kind != OF_MODEL_GBM)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "the Greeks modes price GBM options (Heston: of_heston_price_adjoint)");
  if (m.n_dividends > 0) return of_fail(ctx, OF_ERR_UNSUPPORTED, "the Greeks modes take no discrete dividends");
  if (!(b.discount_factor > 0.0) || !std::isfinite(b.discount_factor))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "the Greeks modes need a discount factor exp(-r T) > 0");
  g = of::GreekConsts<double>{};
  const double T = m.maturity, M = (double)m.steps, dt = T / M, sig = m.sigma;
  g.dt = dt;
  g.T = T;
  g.sigma = sig;
  g.a = m.mu - 0.5 * sig * sig;
  g.alpha = g.a * dt;
  g.beta = sig * std::sqrt(dt);
  g.df = b.discount_factor;
  g.r = -std::log(b.discount_factor) / T;
  g.s0 = m.s0;
  g.strike = p.strike;
  g.sig_dt = sig * dt;
  g.inv_sig = 1.0 / sig;
  g.beta_over_sig = std::sqrt(dt);
  g.alpha_over_T = g.alpha / T;
  g.inv_2T = 0.5 / T;
  g.beta_over_2T = g.beta / (2.0 * T);
  g.steps = (int32_t)m.steps;
  g.obs_offset = d.obs_offset;
  g.cv_kind = b.control_variate;
  g.stream = d.stream;
  int32_t f = 0;
  if (p.option_type == OF_CALL) f |= of::GF_CALL;
  if (b.antithetic) f |= of::GF_ANTI;
  switch (p.kind) {
    case OF_PAYOFF_VANILLA:
      g.kind = of::GK_TERMINAL;
      break;
    case OF_PAYOFF_ASIAN:
      if (p.strike_type == OF_STRIKE_FLOATING) f |= of::GF_FLOATING;
      if (p.averaging == OF_AVG_GEOMETRIC) f |= of::GF_GEOMETRIC;
      if (d.flags & BF_TERMINAL_ONLY) {
        f |= of::GF_TERMINAL_ONLY;
        g.kind = of::GK_TERMINAL;
      } else {
        g.kind = daily ? of::GK_ASIAN_DAILY : of::GK_ASIAN_WEIGHTS;
        g.inv_n = 1.0 / (double)p.n_observations;
        double w1 = 0.0;
        for (size_t i = 1; i < w.size(); ++i) w1 += w[i] * (double)i;
        g.w1 = w1;
      }
      break;
    default:  // barrier
      if (!(p.barrier_level > 0.0) || !std::isfinite(p.barrier_level))
        return of_fail(ctx, OF_ERR_INVALID_INPUT, "barrier level must be > 0");
      if (b.control_variate != OF_CV_NONE)
        return of_fail(ctx, OF_ERR_UNSUPPORTED, "a barrier option takes no control variate in the Greeks modes");
      g.kind = p.barrier_style == OF_BARRIER_IN ? of::GK_BARRIER_IN : of::GK_BARRIER_OUT;
      g.rebate = p.rebate;
      g.bar = std::log(p.barrier_level / m.s0);
      g.sgn = p.barrier_direction == OF_BARRIER_UP ? 1.0 : -1.0;
      g.sib = g.sgn / g.beta;
  }
  g.flags = f;
  (void)o;
  return OF_OK;
}

static of::GreekConsts<float> round_greek_consts(const of::GreekConsts<double>& d) {
  of::GreekConsts<float> f{};
  f.alpha = (float)d.alpha;
  f.beta = (float)d.beta;
  f.a = (float)d.a;
  f.dt = (float)d.dt;
  f.T = (float)d.T;
  f.sigma = (float)d.sigma;
  f.r = (float)d.r;
  f.df = (float)d.df;
  f.s0 = (float)d.s0;
  f.strike = (float)d.strike;
  f.rebate = (float)d.rebate;
  f.inv_n = (float)d.inv_n;
  f.w1 = (float)d.w1;
  f.bar = (float)d.bar;
  f.sgn = (float)d.sgn;
  f.sib = (float)d.sib;
  f.sig_dt = (float)d.sig_dt;
  f.inv_sig = (float)d.inv_sig;
  f.beta_over_sig = (float)d.beta_over_sig;
  f.alpha_over_T = (float)d.alpha_over_T;
  f.inv_2T = (float)d.inv_2T;
  f.beta_over_2T = (float)d.beta_over_2T;
  f.kind = d.kind;
  f.flags = d.flags;
  f.steps = d.steps;
  f.obs_offset = d.obs_offset;
  f.cv_kind = d.cv_kind;
  f.stream = d.stream;
  return f;
}

struct of_book_plan {
  of_ctx* ctx = nullptr;
  bool scratch = false;  // buffers borrowed from the context (a plan that lives inside one call)
  int64_t n = 0;
  int mode = OF_BOOK_PRICE;
  int nc = 5;  // sums per option: 5, or 13 with the Greeks
  int block = 256, ppt = 4, grid = 0;
  int64_t n_tiles = 0;
  double path_steps = 0.0;
  std::vector<int64_t> samples;
  std::vector<int32_t> cv_kind;
  std::vector<double> cv_expected, discount;
  BookParams P{};
  BookParams Pg[of::KG_COUNT]{};  // Greeks modes: one launch per kind group
  int grid_g[of::KG_COUNT] = {0, 0, 0};
  BookOpt* d_opts = nullptr;
  BookTile* d_tiles = nullptr;
  float* d_obs = nullptr;
  BookDiv* d_divs = nullptr;
  void* d_gc = nullptr;  // GreekConsts<float> (Greeks mode) or <double> (FP64 mode)
  int* d_counter = nullptr;
  double* d_partials = nullptr;
  int32_t* d_begin = nullptr;
  double* d_sums = nullptr;
  double* h_sums = nullptr;
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

template <typename R, bool G>
static const void* book_greeks_kernel_for(int kg) {
  return kg == of::KG_TERMINAL ? (const void*)book_greeks_kernel<R, G, of::KG_TERMINAL>
         : kg == of::KG_ASIAN  ? (const void*)book_greeks_kernel<R, G, of::KG_ASIAN>
                               : (const void*)book_greeks_kernel<R, G, of::KG_BARRIER>;
}

static const void* book_kernel_for(int mode, int kg) {
  if (mode == OF_BOOK_GREEKS) return book_greeks_kernel_for<float, true>(kg);
  if (mode == OF_BOOK_PRICE_FP64) return book_greeks_kernel_for<double, false>(kg);
  if (mode == OF_BOOK_GREEKS_FP64) return book_greeks_kernel_for<double, true>(kg);
  return (const void*)book_kernel;
}

template <typename R, bool G>
static void book_greeks_enqueue(of_book_plan* pl, cudaStream_t s) {
  const of::GreekConsts<R>* gc = (const of::GreekConsts<R>*)pl->d_gc;
  for (int kg = 0; kg < of::KG_COUNT; ++kg) {
    if (pl->Pg[kg].n_tiles == 0) continue;
    const dim3 grid((unsigned)pl->grid_g[kg]);
    if (kg == of::KG_TERMINAL) book_greeks_kernel<R, G, of::KG_TERMINAL><<<grid, pl->block, 0, s>>>(pl->Pg[kg], gc);
    else if (kg == of::KG_ASIAN) book_greeks_kernel<R, G, of::KG_ASIAN><<<grid, pl->block, 0, s>>>(pl->Pg[kg], gc);
    else book_greeks_kernel<R, G, of::KG_BARRIER><<<grid, pl->block, 0, s>>>(pl->Pg[kg], gc);
  }
}

static void book_enqueue(of_book_plan* pl, cudaStream_t s) {
  cudaMemsetAsync(pl->d_counter, 0, of::KG_COUNT * sizeof(int), s);
  const unsigned rgrid = (unsigned)((pl->n + 7) / 8);
  if (pl->mode == OF_BOOK_GREEKS) {
    book_greeks_enqueue<float, true>(pl, s);
    book_reduce_kernel<13><<<rgrid, 256, 0, s>>>(pl->d_partials, pl->d_begin, (int)pl->n, pl->d_sums);
  } else if (pl->mode == OF_BOOK_PRICE_FP64) {
    book_greeks_enqueue<double, false>(pl, s);
    book_reduce_kernel<5><<<rgrid, 256, 0, s>>>(pl->d_partials, pl->d_begin, (int)pl->n, pl->d_sums);
  } else if (pl->mode == OF_BOOK_GREEKS_FP64) {
    book_greeks_enqueue<double, true>(pl, s);
    book_reduce_kernel<13><<<rgrid, 256, 0, s>>>(pl->d_partials, pl->d_begin, (int)pl->n, pl->d_sums);
  } else {
    book_kernel<<<pl->grid, pl->block, 0, s>>>(pl->P);
    book_reduce_kernel<5><<<rgrid, 256, 0, s>>>(pl->d_partials, pl->d_begin, (int)pl->n, pl->d_sums);
  }
  cudaMemcpyAsync(pl->h_sums, pl->d_sums, (size_t)pl->n * pl->nc * sizeof(double), cudaMemcpyDeviceToHost, s);
}

extern "C" void of_book_plan_destroy(of_book_plan* pl) {
  if (!pl) return;
  if (pl->ctx) cudaStreamSynchronize(pl->ctx->stream);
  if (pl->exec) cudaGraphExecDestroy(pl->exec);
  if (pl->graph) cudaGraphDestroy(pl->graph);
  if (pl->scratch) {  // the context owns the buffers
    delete pl;
    return;
  }
  cudaFree(pl->d_opts);
  cudaFree(pl->d_tiles);
  cudaFree(pl->d_obs);
  cudaFree(pl->d_divs);
  cudaFree(pl->d_gc);
  cudaFree(pl->d_counter);
  cudaFree(pl->d_partials);
  cudaFree(pl->d_begin);
  cudaFree(pl->d_sums);
  if (pl->h_sums) cudaFreeHost(pl->h_sums);
  delete pl;
}

// scratch: the plan lives inside one library call and borrows the context's
// cached buffers (of_scratch / of_pinned) instead of allocating its own.
static of_status book_plan_create(of_ctx* ctx, const of_book_entry* e, int64_t n, const of_book_config* cfg,
                                  bool scratch, of_book_plan** out) {
  if (!ctx || !out || !cfg) return OF_ERR_INVALID_INPUT;
  *out = nullptr;
  if (n <= 0 || !e) return of_fail(ctx, OF_ERR_INVALID_INPUT, "book must hold at least one option");
  if (n > (1 << 24)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "book too large");
  OF_TRY(of_ctx_check(ctx));
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  of_book_plan* pl = new of_book_plan();
  pl->ctx = ctx;
  pl->scratch = scratch;
  pl->n = n;
  pl->block = cfg->block > 0 ? cfg->block : 256;
  pl->ppt = cfg->paths_per_thread > 0 ? cfg->paths_per_thread : 4;
  pl->use_graph = cfg->use_graph != 0;
  pl->mode = cfg->mode;
  if (pl->mode != OF_BOOK_PRICE && pl->mode != OF_BOOK_GREEKS && pl->mode != OF_BOOK_PRICE_FP64 &&
      pl->mode != OF_BOOK_GREEKS_FP64) {
    const int m = pl->mode;
    of_book_plan_destroy(pl);
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown book mode %d", m);
  }
  pl->nc = (pl->mode == OF_BOOK_GREEKS || pl->mode == OF_BOOK_GREEKS_FP64) ? 13 : 5;
  if (pl->block % 32 != 0 || pl->block > 256) {
    of_book_plan_destroy(pl);
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "block must be a multiple of 32 and <= 256");
  }
  auto fail = [&](of_status st) {
    of_book_plan_destroy(pl);
    return st;
  };
  std::vector<BookOpt> opts((size_t)n);
  std::vector<of::GreekConsts<double>> gcs;  // Greeks modes only
  if (pl->mode != OF_BOOK_PRICE) gcs.resize((size_t)n);
  std::vector<float> obs;
  std::vector<BookDiv> divs;
  std::vector<of_div_trigger> trig;
  pl->samples.resize((size_t)n);
  pl->cv_kind.resize((size_t)n);
  pl->cv_expected.resize((size_t)n);
  pl->discount.resize((size_t)n);
  struct Pending {
    int32_t opt;
    int64_t first;
    int32_t count;
    double cost;
  };
  std::vector<Pending> pend;
  const int64_t tile_samples = (int64_t)pl->block * pl->ppt;
  for (int64_t o = 0; o < n; ++o) {
    const of_book_entry& b = e[o];
    of_mc_config c{};
    c.num_paths = b.num_paths;
    c.antithetic = b.antithetic;
    c.control_variate = b.control_variate;
    c.discount_factor = b.discount_factor;
    c.precision = OF_PREC_FP32_PHILOX;
    of_status st = of_validate_mc(ctx, &b.model, &b.payoff, &c);
    if (st == OF_OK) st = validate_fp32_model(ctx, &b.model);
    if (st != OF_OK) {
      ctx->last_error = "book entry " + std::to_string(o) + ": " + ctx->last_error;
      return fail(st);
    }
    BookOpt& d = opts[(size_t)o];
    d.c = make_consts(&b.model);
    d.model = b.model.kind;
    d.payoff = b.payoff.kind;
    d.cv_kind = b.control_variate;
    d.steps = (int32_t)b.model.steps;
    d.s0 = (float)b.model.s0;
    d.strike = (float)b.payoff.strike;
    d.rebate = (float)b.payoff.rebate;
    d.barrier_y = (float)std::log(b.payoff.barrier_level / b.model.s0);
    if (!(b.payoff.barrier_level > 0.0)) d.barrier_y = b.payoff.barrier_direction == OF_BARRIER_UP ? INFINITY : -INFINITY;
    d.stream = (uint32_t)o;
    d.obs_offset = -1;
    st = of_dividend_triggers(ctx, &b.model, trig);
    if (st != OF_OK) {
      ctx->last_error = "book entry " + std::to_string(o) + ": " + ctx->last_error;
      return fail(st);
    }
    d.div_offset = (int32_t)divs.size();
    d.n_div = (int32_t)trig.size();
    for (const of_div_trigger& t : trig)
      divs.push_back(BookDiv{t.step, t.kind,
                             (float)(t.kind == OF_DIV_CASH ? t.amount / b.model.s0 : std::log1p(-t.amount)), 0.0f});
    int32_t f = 0;
    if (b.antithetic) f |= BF_ANTI;
    if (b.payoff.barrier_direction == OF_BARRIER_UP) f |= BF_UP;
    if (b.payoff.barrier_style == OF_BARRIER_IN) f |= BF_IN;
    if (b.payoff.averaging == OF_AVG_GEOMETRIC) f |= BF_GEOMETRIC;
    if (b.payoff.strike_type == OF_STRIKE_FLOATING) f |= BF_FLOATING;
    if (b.payoff.option_type == OF_CALL) f |= BF_CALL;
    const bool asian = b.payoff.kind == OF_PAYOFF_ASIAN;
    bool need_arith = asian && b.payoff.averaging == OF_AVG_ARITHMETIC;
    bool need_geo = (asian && b.payoff.averaging == OF_AVG_GEOMETRIC) || b.control_variate == OF_CV_GEOMETRIC_ASIAN;
    std::vector<double> w;
    bool daily_obs = false;
    if (need_arith || need_geo) {
      bool terminal_only = true;
      of_observation_weights(&b.payoff, b.model.steps, w, terminal_only);
      if (terminal_only) {
        f |= BF_TERMINAL_ONLY;
        need_arith = need_geo = false;
      } else {
        bool daily = w[0] == 0.0;
        for (size_t k = 1; k < w.size() && daily; ++k) daily = w[k] == 1.0;
        daily_obs = daily;
        if (daily) {
          f |= BF_DAILY;
        } else {
          d.obs_offset = (int32_t)obs.size();
          for (double x : w) obs.push_back((float)x);
        }
        d.inv_nobs = (float)(1.0 / (double)b.payoff.n_observations);
      }
    }
    if (need_arith) f |= BF_NEED_ARITH;
    if (need_geo) f |= BF_NEED_GEO;
    if (asian && !need_arith && !need_geo) f |= BF_TERMINAL_ONLY;
    d.flags = f;
    d.kind = BK_GENERIC;
    if (d.model == OF_MODEL_GBM && d.n_div == 0) {
      if (!need_geo) {
        if (b.payoff.kind == OF_PAYOFF_VANILLA || (f & BF_TERMINAL_ONLY)) d.kind = BK_TERMINAL;
        else if (b.payoff.kind == OF_PAYOFF_BARRIER) d.kind = BK_BARRIER;
        else if (need_arith && (f & BF_DAILY)) d.kind = BK_ASIAN_DAILY;
      } else if (need_arith && (f & BF_DAILY)) {  // with the geometric control variate
        d.kind = BK_ASIAN_DAILY_GEO;
      }
    }
    if (pl->mode != OF_BOOK_PRICE) {
      st = book_greek_consts(ctx, b, o, d, w, daily_obs, gcs[(size_t)o]);
      if (st != OF_OK) {
        ctx->last_error = "book entry " + std::to_string(o) + ": " + ctx->last_error;
        return fail(st);
      }
    }
    const int64_t samples = b.antithetic ? (b.num_paths + 1) / 2 : b.num_paths;
    pl->samples[(size_t)o] = samples;
    pl->cv_kind[(size_t)o] = b.control_variate;
    pl->cv_expected[(size_t)o] = b.cv_expected;
    pl->discount[(size_t)o] = b.discount_factor;
    pl->path_steps += (double)b.num_paths * (double)b.model.steps;
    for (int64_t first = 0; first < samples; first += tile_samples) {
      const int32_t cnt = (int32_t)std::min<int64_t>(tile_samples, samples - first);
      const double legs = b.antithetic ? 2.0 : 1.0;
      pend.push_back({(int32_t)o, first, cnt, (double)cnt * legs * (double)b.model.steps});
    }
  }
  if (pend.size() > (size_t)2147483647) return fail(of_fail(ctx, OF_ERR_INVALID_INPUT, "too many tiles"));
  // Slots in option-major order, schedule longest tile first.
  std::vector<int32_t> begin((size_t)n + 1, 0);
  for (size_t k = 0; k < pend.size(); ++k) begin[(size_t)pend[k].opt + 1]++;
  for (int64_t o = 0; o < n; ++o) begin[(size_t)o + 1] += begin[(size_t)o];
  // The schedule: the Greeks modes' kind groups in turn, longest tile first
  // within a group, ties in slot order (a stable sort of the tiles by group,
  // then cost descending).  An option's tiles are consecutive slots; all but
  // its last share one cost, and the last may be shorter.  So the schedule is
  // built from runs of equal-cost tiles, at most two per option, sorted
  // stably: the same order as sorting the tiles, at O(n log n + tiles)
  // instead of O(tiles log tiles) (a million tiles for a book of long-dated
  // options at 2^25 paths each).
  struct Run {
    size_t begin, end;
    int group;
    double cost;
  };
  std::vector<Run> runs;
  runs.reserve((size_t)n * 2);
  for (size_t k = 0; k < pend.size();) {
    const int32_t o = pend[k].opt;
    const int group = pl->mode != OF_BOOK_PRICE ? of::gk_group(gcs[(size_t)o].kind) : 0;
    size_t e = k;
    while (e < pend.size() && pend[e].opt == o && pend[e].cost == pend[k].cost) ++e;
    runs.push_back({k, e, group, pend[k].cost});
    k = e;
  }
  std::stable_sort(runs.begin(), runs.end(), [](const Run& a, const Run& b) {
    return a.group != b.group ? a.group < b.group : a.cost > b.cost;
  });
  std::vector<BookTile> sorted;
  sorted.reserve(pend.size());
  for (const Run& r : runs)
    for (size_t k = r.begin; k < r.end; ++k)
      sorted.push_back({pend[k].opt, pend[k].count, pend[k].first, (int32_t)k, 0});
  pl->n_tiles = (int64_t)sorted.size();

  const size_t nt = sorted.size();
  // A plan that lives inside one call borrows the context's cached buffers:
  // no cudaMalloc / cudaFree / cudaMallocHost per call.
  auto dalloc = [&](void** p, size_t bytes, int slot) {
    if (pl->scratch) return of_scratch(ctx, slot, bytes, p) == OF_OK;
    return cudaMalloc(p, bytes) == cudaSuccess;
  };
  const size_t sum_bytes = (size_t)n * pl->nc * sizeof(double);
  bool ok = dalloc((void**)&pl->d_opts, opts.size() * sizeof(BookOpt), SLOT_BOOK) &&
            dalloc((void**)&pl->d_tiles, nt * sizeof(BookTile), SLOT_TILES) &&
            dalloc((void**)&pl->d_obs, std::max<size_t>(1, obs.size()) * sizeof(float), SLOT_BOOK_OBS) &&
            dalloc((void**)&pl->d_divs, std::max<size_t>(1, divs.size()) * sizeof(BookDiv), SLOT_BOOK_DIVS) &&
            dalloc((void**)&pl->d_counter, of::KG_COUNT * sizeof(int), SLOT_BOOK_COUNTER) &&
            dalloc((void**)&pl->d_partials, nt * pl->nc * sizeof(double), SLOT_BOOK_PARTIALS) &&
            dalloc((void**)&pl->d_begin, begin.size() * sizeof(int32_t), SLOT_BOOK_BEGIN) &&
            dalloc((void**)&pl->d_sums, sum_bytes, SLOT_BOOK_SUMS);
  if (ok) ok = pl->scratch ? of_pinned(ctx, sum_bytes, (void**)&pl->h_sums) == OF_OK
                           : cudaMallocHost(&pl->h_sums, sum_bytes) == cudaSuccess;
  if (!ok) return fail(of_fail(ctx, OF_ERR_ALLOC, "book plan allocation failed"));
  if (pl->mode == OF_BOOK_GREEKS) {  // the constants rounded once to FP32
    std::vector<of::GreekConsts<float>> gf(gcs.size());
    for (size_t k = 0; k < gcs.size(); ++k) gf[k] = round_greek_consts(gcs[k]);
    if (!dalloc(&pl->d_gc, gf.size() * sizeof(gf[0]), SLOT_BOOK_GC))
      return fail(of_fail(ctx, OF_ERR_ALLOC, "book plan allocation failed"));
    if (cudaMemcpy(pl->d_gc, gf.data(), gf.size() * sizeof(gf[0]), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(of_fail(ctx, OF_ERR_CUDA, "book upload failed"));
  } else if (pl->mode == OF_BOOK_PRICE_FP64 || pl->mode == OF_BOOK_GREEKS_FP64) {
    if (!dalloc(&pl->d_gc, gcs.size() * sizeof(gcs[0]), SLOT_BOOK_GC))
      return fail(of_fail(ctx, OF_ERR_ALLOC, "book plan allocation failed"));
    if (cudaMemcpy(pl->d_gc, gcs.data(), gcs.size() * sizeof(gcs[0]), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(of_fail(ctx, OF_ERR_CUDA, "book upload failed"));
  }
  if (cudaMemcpy(pl->d_opts, opts.data(), opts.size() * sizeof(BookOpt), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(pl->d_tiles, sorted.data(), nt * sizeof(BookTile), cudaMemcpyHostToDevice) != cudaSuccess ||
      (!obs.empty() && cudaMemcpy(pl->d_obs, obs.data(), obs.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) ||
      (!divs.empty() &&
       cudaMemcpy(pl->d_divs, divs.data(), divs.size() * sizeof(BookDiv), cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(pl->d_begin, begin.data(), begin.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(of_fail(ctx, OF_ERR_CUDA, "book upload failed"));
  BookParams& P = pl->P;
  P.opts = pl->d_opts;
  P.tiles = pl->d_tiles;
  P.obs_w = pl->d_obs;
  P.divs = pl->d_divs;
  P.n_tiles = (int32_t)nt;
  P.ppt = pl->ppt;
  P.keys = of::philox_keys(cfg->seed);
  P.counter = pl->d_counter;
  P.partials = pl->d_partials;
  const int per_sm = of_blocks_per_sm(book_kernel_for(pl->mode, of::KG_TERMINAL), pl->block, 0);
  const int64_t cap = (int64_t)ctx->sm_count * per_sm;
  pl->grid = (int)std::max<int64_t>(1, std::min<int64_t>(cap, (int64_t)nt));
  if (pl->mode != OF_BOOK_PRICE) {
    size_t start = 0;
    for (int kg = 0; kg < of::KG_COUNT; ++kg) {
      size_t end = start;
      while (end < nt && of::gk_group(gcs[(size_t)sorted[end].opt].kind) == kg) ++end;
      BookParams& Q = pl->Pg[kg];
      Q = P;
      Q.tiles = pl->d_tiles + start;
      Q.n_tiles = (int32_t)(end - start);
      Q.counter = pl->d_counter + kg;
      const int per = of_blocks_per_sm(book_kernel_for(pl->mode, kg), pl->block, 0);
      pl->grid_g[kg] = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->sm_count * per, (int64_t)(end - start)));
      start = end;
    }
  }
  if (pl->use_graph) {
    cudaStream_t cs = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess)
      return fail(of_fail(ctx, OF_ERR_CUDA, "capture stream creation failed"));
    cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      book_enqueue(pl, cs);
      err = cudaStreamEndCapture(cs, &pl->graph);
    }
    if (err == cudaSuccess) err = cudaGraphInstantiate(&pl->exec, pl->graph, 0);
    cudaStreamDestroy(cs);
    if (err != cudaSuccess) return fail(of_fail(ctx, OF_ERR_CUDA, "book graph capture failed: %s", cudaGetErrorString(err)));
  }
  *out = pl;
  return OF_OK;
}

extern "C" of_status of_book_plan_launch(of_book_plan* pl) {
  if (!pl) return OF_ERR_INVALID_INPUT;
  OF_TRY(of_ctx_check(pl->ctx));
  if (pl->use_graph) {
    OF_CUDA_TRY(pl->ctx, cudaGraphLaunch(pl->exec, pl->ctx->stream));
  } else {
    book_enqueue(pl, pl->ctx->stream);
    OF_CUDA_TRY(pl->ctx, cudaGetLastError());
  }
  return OF_OK;
}

extern "C" of_status of_book_plan_results(of_book_plan* pl, of_mc_result* res) {
  if (!pl || !res) return OF_ERR_INVALID_INPUT;
  OF_CUDA_TRY(pl->ctx, cudaStreamSynchronize(pl->ctx->stream));
  for (int64_t o = 0; o < pl->n; ++o) {
    of_mc_finish(pl->h_sums + o * pl->nc, pl->samples[(size_t)o], pl->cv_kind[(size_t)o], pl->cv_expected[(size_t)o],
                 pl->discount[(size_t)o], &res[o]);
    res[o].kernel_ms = 0.0;
  }
  return OF_OK;
}

extern "C" of_status of_book_plan_greeks(of_book_plan* pl, of_book_greeks* out) {
  if (!pl || !out) return OF_ERR_INVALID_INPUT;
  if (pl->mode != OF_BOOK_GREEKS && pl->mode != OF_BOOK_GREEKS_FP64)
    return of_fail(pl->ctx, OF_ERR_INVALID_INPUT, "the plan was not created in mode OF_BOOK_GREEKS(_FP64)");
  OF_CUDA_TRY(pl->ctx, cudaStreamSynchronize(pl->ctx->stream));
  for (int64_t o = 0; o < pl->n; ++o) {
    const double* s = pl->h_sums + o * pl->nc;
    const double n = (double)pl->samples[(size_t)o];
    double mean[4], se[4];
    for (int t = 0; t < 4; ++t) {  // the sums are of discounted per-sample derivatives
      mean[t] = s[5 + t] / n;
      const double var = n > 1.0 ? std::fmax(s[9 + t] - s[5 + t] * s[5 + t] / n, 0.0) / (n - 1.0) : 0.0;
      se[t] = std::sqrt(var / n);
    }
    of_book_greeks& g = out[o];
    g.delta = mean[0];
    g.vega = mean[1];
    g.rho = mean[2];
    g.theta = mean[3];
    g.gamma = 0.0;
    g.delta_se = se[0];
    g.vega_se = se[1];
    g.rho_se = se[2];
    g.theta_se = se[3];
    g.gamma_se = 0.0;
  }
  return OF_OK;
}

extern "C" of_status of_book_plan_info(of_book_plan* pl, int32_t* block, int32_t* ppt, int64_t* n_tiles,
                                       double* path_steps) {
  if (!pl) return OF_ERR_INVALID_INPUT;
  if (block) *block = pl->block;
  if (ppt) *ppt = pl->ppt;
  if (n_tiles) *n_tiles = pl->n_tiles;
  if (path_steps) *path_steps = pl->path_steps;
  return OF_OK;
}

// One launch of a book: plan, launch, results (and Greeks when `greeks`).
extern "C" of_status of_book_plan_create(of_ctx* ctx, const of_book_entry* e, int64_t n, const of_book_config* cfg,
                                         of_book_plan** out) {
  return book_plan_create(ctx, e, n, cfg, false, out);
}

static of_status book_run(of_ctx* ctx, const of_book_entry* e, int64_t n, const of_book_config* cfg,
                          of_mc_result* res, of_book_greeks* greeks) {
  of_book_plan* pl = nullptr;
  OF_TRY(book_plan_create(ctx, e, n, cfg, true, &pl));
  cudaEventRecord(ctx->ev_start, ctx->stream);
  of_status st = of_book_plan_launch(pl);
  cudaEventRecord(ctx->ev_stop, ctx->stream);
  if (st == OF_OK) st = of_book_plan_results(pl, res);
  if (st == OF_OK && greeks) st = of_book_plan_greeks(pl, greeks);
  float ms = 0.0f;
  if (st == OF_OK && cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess)
    for (int64_t o = 0; o < n; ++o) res[o].kernel_ms = ms;
  of_book_plan_destroy(pl);
  return st;
}

extern "C" of_status of_mc_price_book(of_ctx* ctx, const of_book_entry* e, int64_t n, const of_book_config* cfg,
                                      of_mc_result* res) {
  if (!ctx || !res || !cfg) return OF_ERR_INVALID_INPUT;
  return book_run(ctx, e, n, cfg, res, nullptr);
}

extern "C" of_status of_mc_price_book_greeks(of_ctx* ctx, const of_book_entry* e, int64_t n, const of_book_config* cfg,
                                             of_mc_result* res, of_book_greeks* greeks) {
  if (!ctx || !res || !cfg || !greeks) return OF_ERR_INVALID_INPUT;
  of_book_config c = *cfg;
  c.mode = OF_BOOK_GREEKS;
  return book_run(ctx, e, n, &c, res, greeks);
}

// FP32 branch of of_mc_run: a one-option book.
of_status of_mc_run_fp32(of_ctx* ctx, const of_model* m, const of_payoff* p, const of_mc_config* c,
                         of_mc_result* out) {
  if (c->injected_normals)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "injected normals are a FP64 reference-mode test hook");
  of_book_entry b{};
  b.model = *m;
  b.payoff = *p;
  b.num_paths = c->num_paths;
  b.antithetic = c->antithetic;
  b.control_variate = c->control_variate;
  b.cv_expected = c->cv_expected;
  b.discount_factor = c->discount_factor;
  of_book_config bc{};
  bc.seed = c->seed;
  bc.use_graph = 0;
  return of_mc_price_book(ctx, &b, 1, &bc, out);
}

// ---------------------------------------------------------------------------
// Strike strip without any allocation (of_mc_strip_noalloc).
//
// For callers that cannot allocate device memory when they price: every
// byte of scratch the strip kernel needs lives in the static array below,
// which each GPU that loads this library holds until the process exits.
// Layout: [strikes: MAX_STRIKES floats][sums: 2*MAX_STRIKES doubles]
//         [per-block partials: MAX_BLOCKS * 2*MAX_STRIKES doubles].
// In host code `g_strip_noalloc_scratch` names a host-side stand-in, not the
// device array: its device address is looked up with cudaGetSymbolAddress
// with the caller's device current, once per CUDA context (a device's
// primary context, or a context the caller made current), and that address
// is what the kernels get.  The lookups are cached by the context's
// process-unique ID, so a context created after cudaDeviceReset, whose copy
// of the array may sit elsewhere, gets a lookup of its own.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_strip_noalloc_scratch[OF_STRIP_NOALLOC_SCRATCH_BYTES];

namespace {

typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);

struct NoallocAddr {
  unsigned long long ctx_id;
  void* addr;
};
constexpr int kNoallocCache = 64;
NoallocAddr g_noalloc_cache[kNoallocCache] = {};
int g_noalloc_used = 0;
std::mutex g_noalloc_mutex;

void noalloc_msg(char* err, size_t len, const char* fmt, ...) {
  if (!err || len == 0) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(err, len, fmt, ap);
  va_end(ap);
}

// The process-unique ID of the calling thread's current CUDA context (0 when
// none is current).  The two driver functions are resolved once through the
// runtime, so the library keeps no link-time dependency on libcuda.
cudaError_t noalloc_ctx_id(unsigned long long* id) {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  static cudaError_t resolved = [] {
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void**)&get_current, 12000,
                                                     cudaEnableDefault, &q1);
    if (e == cudaSuccess)
      e = cudaGetDriverEntryPointByVersion("cuCtxGetId", (void**)&get_id, 12000, cudaEnableDefault, &q2);
    if (e == cudaSuccess && (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !get_current ||
                             !get_id))
      e = cudaErrorSymbolNotFound;
    return e;
  }();
  *id = 0;
  if (resolved != cudaSuccess) return resolved;
  CUcontext c = nullptr;
  if (get_current(&c) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  if (!c) return cudaSuccess;
  return get_id(c, id) == CUDA_SUCCESS ? cudaSuccess : cudaErrorDeviceUninitialized;
}

// Device address of the scratch array in the current context.  The first
// call in a context makes the runtime's context current (cudaGetSymbolAddress
// initialises the primary context of the current device if needed).
cudaError_t noalloc_scratch_addr(void** out) {
  unsigned long long id = 0;
  cudaError_t e = noalloc_ctx_id(&id);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> guard(g_noalloc_mutex);
  if (id != 0)
    for (int k = 0; k < g_noalloc_used; ++k)
      if (g_noalloc_cache[k].ctx_id == id) {
        *out = g_noalloc_cache[k].addr;
        return cudaSuccess;
      }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_strip_noalloc_scratch);
  if (e != cudaSuccess) return e;
  if (!p) return cudaErrorInvalidSymbol;
  if (id == 0 && (e = noalloc_ctx_id(&id)) != cudaSuccess) return e;  // the lookup made a context current
  if (id != 0 && g_noalloc_used < kNoallocCache) g_noalloc_cache[g_noalloc_used++] = {id, p};
  *out = p;
  return cudaSuccess;
}

}  // namespace

extern "C" of_status of_mc_strip_noalloc(void* cuda_stream, const of_model* m, int32_t option_type,
                                         const double* strikes, int64_t n_strikes, const of_mc_config* cfg,
                                         of_mc_result* results, char* err, size_t err_len) {
  if (err && err_len) err[0] = '\0';
  if (!results) {
    noalloc_msg(err, err_len, "null argument");
    return OF_ERR_INVALID_INPUT;
  }
  {
    // The checks of of_mc_strip; the stack context only carries the message.
    of_ctx sink;
    const of_status st = strip_validate(&sink, m, option_type, strikes, n_strikes, cfg);
    if (st != OF_OK) {
      noalloc_msg(err, err_len, "%s", sink.last_error.c_str());
      return st;
    }
  }
  if (n_strikes > OF_STRIP_NOALLOC_MAX_STRIKES) {
    noalloc_msg(err, err_len, "n_strikes must be in [1, %d] (static scratch limit), got %lld",
                OF_STRIP_NOALLOC_MAX_STRIKES, (long long)n_strikes);
    return OF_ERR_INVALID_INPUT;
  }
  float hk[OF_STRIP_NOALLOC_MAX_STRIKES];
  for (int64_t k = 0; k < n_strikes; ++k) hk[k] = (float)strikes[k];

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    noalloc_msg(err, err_len, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    return OF_ERR_CUDA;
  }
  // The call synchronises its stream and copies through host stack buffers,
  // neither of which a stream capture allows: refuse before touching it.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if ((e = cudaStreamIsCapturing((cudaStream_t)cuda_stream, &capture)) != cudaSuccess) {
    noalloc_msg(err, err_len, "cudaStreamIsCapturing failed: %s", cudaGetErrorString(e));
    return OF_ERR_CUDA;
  }
  if (capture != cudaStreamCaptureStatusNone) {
    noalloc_msg(err, err_len, "of_mc_strip_noalloc cannot run on a capturing stream");
    return OF_ERR_UNSUPPORTED;
  }
  void* base = nullptr;
  if ((e = noalloc_scratch_addr(&base)) != cudaSuccess) {
    noalloc_msg(err, err_len, "device address of the static scratch: %s", cudaGetErrorString(e));
    return OF_ERR_CUDA;
  }
  float* d_strikes = (float*)base;
  double* d_sums = (double*)((char*)base + OF_STRIP_NOALLOC_MAX_STRIKES * 4);
  double* d_status = d_sums + OF_STRIP_NOALLOC_MAX_STRIKES * 2;  // the warp-specialised kernel's status word
  double* d_partials = d_status + 1;

  StripParams P{};
  P.c = make_consts(m);
  P.samples = cfg->antithetic ? (cfg->num_paths + 1) / 2 : cfg->num_paths;
  P.steps = (int32_t)m->steps;
  P.n_strikes = (int32_t)n_strikes;
  P.option_type = option_type;
  P.antithetic = cfg->antithetic ? 1 : 0;
  P.s0 = (float)m->s0;
  P.keys = of::philox_keys(cfg->seed);
  P.strikes = d_strikes;
  P.status = (uint32_t*)d_status;
  // the kernel of_mc_strip picks for the same request (strikes per lane, tile shape)
  const int block = 256;
  const StripShape sh = strip_shape(cfg->tile_ilp, n_strikes, m->kind, P.antithetic, block);
  const StripKernelFn fn = sh.fn;
  const size_t smem = sh.smem;
  int sms = 0, per_sm = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, block, smem)) != cudaSuccess) {
    noalloc_msg(err, err_len, "device query failed: %s", cudaGetErrorString(e));
    return OF_ERR_CUDA;
  }
  const int64_t want = (P.samples + sh.samples_per_block - 1) / sh.samples_per_block;
  int64_t grid = std::min<int64_t>(want, (int64_t)sms * std::max(per_sm, 1));
  grid = std::max<int64_t>(1, std::min<int64_t>(grid, OF_STRIP_NOALLOC_MAX_BLOCKS));

  cudaStream_t s = (cudaStream_t)cuda_stream;
  const int64_t cols = 2 * n_strikes;
  double hs[2 * OF_STRIP_NOALLOC_MAX_STRIKES];
  uint32_t h_status = 0;
  if ((e = cudaMemcpyAsync(d_strikes, hk, (size_t)n_strikes * sizeof(float), cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      (sh.ws && (e = cudaMemsetAsync(d_status, 0, sizeof(double), s)) != cudaSuccess)) {
    noalloc_msg(err, err_len, "strike upload failed: %s", cudaGetErrorString(e));
    return OF_ERR_CUDA;
  }
  fn<<<(unsigned)grid, block, smem, s>>>(P, d_partials);
  of_launch_reduce_rows(d_partials, grid, cols, d_sums, s);
  if ((e = cudaGetLastError()) != cudaSuccess ||
      (e = cudaMemcpyAsync(hs, d_sums, (size_t)cols * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (sh.ws &&
       (e = cudaMemcpyAsync(&h_status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess) ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    noalloc_msg(err, err_len, "strip launch failed: %s", cudaGetErrorString(e));
    return OF_ERR_CUDA;
  }
  if (h_status) {
    noalloc_msg(err, err_len, "strike strip: a producer/consumer ring wait did not complete in time");
    return OF_ERR_TIMEOUT;
  }
  for (int64_t k = 0; k < n_strikes; ++k) {
    const double sums[5] = {hs[2 * k], hs[2 * k + 1], 0.0, 0.0, 0.0};
    of_mc_finish(sums, P.samples, OF_CV_NONE, 0.0, cfg->discount_factor, &results[k]);
    results[k].kernel_ms = 0.0;
  }
  return OF_OK;
}

// ---------------------------------------------------------------------------
// Device peak probes (of_measure_device_peaks)
// ---------------------------------------------------------------------------
namespace {

constexpr int kProbeChains = 8;
constexpr int kProbeBlock = 256;

// kProbeChains independent chains per thread.  One link is five MUFU
// operations (lg2, sqrt, sin, cos, sqrt) and a few FP32 adds that keep the
// value bounded: lg2(x + 1.5) in (0.58, 1.81), sqrt(. + 0.5) in (1.04, 1.52),
// sin in (0.86, 1), cos in (0.54, 0.65), sqrt(. + 0.25) in (0.89, 0.95).
__global__ void __launch_bounds__(kProbeBlock) sfu_probe_kernel(int iters, float* sink) {
  float a[kProbeChains];
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) a[k] = 0.5f + 0.01f * k + 1e-7f * threadIdx.x;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) {
      float x = __log2f(a[k] + 1.5f);
      x = sqrtf(x + 0.5f);
      x = __sinf(x);
      x = __cosf(x);
      a[k] = sqrtf(x + 0.25f);
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) s += a[k];
  if (s < 0.0f) sink[blockIdx.x] = s;  // never taken (s > 7); keeps the chains live
}

// kProbeChains independent FMA chains per thread converging to 1.
__global__ void __launch_bounds__(kProbeBlock) fma_probe_kernel(int iters, float* sink) {
  float a[kProbeChains];
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) a[k] = 0.5f + 0.01f * k + 1e-7f * threadIdx.x;
#pragma unroll 16
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) a[k] = fmaf(a[k], 0.99993896484375f, 6.103515625e-5f);
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) s += a[k];
  if (s < 0.0f) sink[blockIdx.x] = s;  // never taken; keeps the chains live
}

// kProbeChains independent FP64 FMA chains per thread converging to 1.
__global__ void __launch_bounds__(kProbeBlock) dfma_probe_kernel(int iters, double* sink) {
  double a[kProbeChains];
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) a[k] = 0.5 + 0.01 * k + 1e-7 * threadIdx.x;
#pragma unroll 16
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) a[k] = fma(a[k], 0.99993896484375, 6.103515625e-5);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) s += a[k];
  if (s < 0.0) sink[blockIdx.x] = s;  // never taken; keeps the chains live
}

}  // namespace

extern "C" of_status of_measure_device_peaks(of_ctx* ctx, of_device_peaks* out) {
  if (!ctx || !out) return OF_ERR_INVALID_INPUT;
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int per_sm_s = of_blocks_per_sm((const void*)sfu_probe_kernel, kProbeBlock, 0);
  const int per_sm_f = of_blocks_per_sm((const void*)fma_probe_kernel, kProbeBlock, 0);
  const int per_sm_d = of_blocks_per_sm((const void*)dfma_probe_kernel, kProbeBlock, 0);
  const int grid_s = ctx->sm_count * std::max(per_sm_s, 1), grid_f = ctx->sm_count * std::max(per_sm_f, 1);
  const int grid_d = ctx->sm_count * std::max(per_sm_d, 1);
  void* sink = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_MISC, (size_t)std::max(std::max(grid_s, grid_f), grid_d) * sizeof(double), &sink));
  const int it_s = 2048, it_f = 65536;
  // warm-up (clocks up), then the best of three timed launches of each probe
  sfu_probe_kernel<<<grid_s, kProbeBlock, 0, ctx->stream>>>(it_s / 8, (float*)sink);
  fma_probe_kernel<<<grid_f, kProbeBlock, 0, ctx->stream>>>(it_f / 8, (float*)sink);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  float best_s = 1e30f, best_f = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    float ms = 0.0f;
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
    sfu_probe_kernel<<<grid_s, kProbeBlock, 0, ctx->stream>>>(it_s, (float*)sink);
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
    OF_CUDA_TRY(ctx, cudaEventSynchronize(ctx->ev_stop));
    OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
    best_s = std::min(best_s, ms);
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
    fma_probe_kernel<<<grid_f, kProbeBlock, 0, ctx->stream>>>(it_f, (float*)sink);
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
    OF_CUDA_TRY(ctx, cudaEventSynchronize(ctx->ev_stop));
    OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
    best_f = std::min(best_f, ms);
  }
  // FP64: warm-up, then the best of three
  const int it_d = 4096;
  float best_d = 1e30f;
  dfma_probe_kernel<<<grid_d, kProbeBlock, 0, ctx->stream>>>(it_d / 8, (double*)sink);
  for (int rep = 0; rep < 3; ++rep) {
    float ms = 0.0f;
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
    dfma_probe_kernel<<<grid_d, kProbeBlock, 0, ctx->stream>>>(it_d, (double*)sink);
    OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
    OF_CUDA_TRY(ctx, cudaEventSynchronize(ctx->ev_stop));
    OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
    best_d = std::min(best_d, ms);
  }
  OF_CUDA_TRY(ctx, cudaGetLastError());
  const double threads_s = (double)grid_s * kProbeBlock, threads_f = (double)grid_f * kProbeBlock;
  const double threads_d = (double)grid_d * kProbeBlock;
  out->sfu_ops_per_s = threads_s * it_s * kProbeChains * 5.0 / (best_s * 1e-3);
  out->fp32_flops_per_s = threads_f * (double)it_f * kProbeChains * 2.0 / (best_f * 1e-3);
  out->fp64_flops_per_s = threads_d * (double)it_d * kProbeChains * 2.0 / (best_d * 1e-3);
  out->probe_ms = (double)best_s + (double)best_f + (double)best_d;
  return OF_OK;
}
