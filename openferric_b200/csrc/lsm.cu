// lsm.cu - Longstaff-Schwartz with an HBM-resident, time-major path store.
//
// Replaces LongstaffSchwartzEngine::price(VanillaOption)
// (src/engines/lsm/longstaff_schwartz.rs:421-618) for a batch of contracts.
//
// Layout: S[contract][step-1][path] (time-major: a date's column is one
// contiguous, coalesced read), cash flows V[contract][path] and, for the
// pathwise delta, the step tau at which each path's cash flow is paid: in FP64
// mode an array tau[contract][path] written when a path exercises, in FP32
// mode one dense row of exercise flags per date (a bit per path) from which
// the final kernel takes the first flagged date.  The final kernel derives
// dV = +-S_tau disc^tau / S0 from V and tau.  One kernel per exercise date does
//   exercise(t+1) with the betas of the previous pass -> discount ->
//   in-the-money basis moments at t -> block partials,
// and the last block of each contract (last-block-done counter, no spin)
// reduces the partials in a fixed order and solves the normal equations:
// degree 2 = the reference's {1,S,S^2} with partially pivoted LU (nalgebra),
// degree 3 = {1,x,x^2,x^3} with Cholesky, x = S/K in the FP64 mode and
// x = S/K - 1 (centred at the strike) in the FP32 mode, whose cubic moments
// are FP32 sums carried into FP64 per warp.
//
// FP64 reference mode reproduces the reference's draws: ONE xoshiro256++
// stream seeded with `seed` feeds all paths in path-major order
// (longstaff_schwartz.rs:467-509).  A thread owns a chunk of consecutive paths
// and jumps its copy of the stream to the chunk's first draw with GF(2)
// matrix powers of the (linear) xoshiro state transition.
// FP32 Philox mode: counter-based normals, FP32 path store.
//
// Compiled with --fmad=false (FP32 code uses explicit fmaf) and with the
// single-precision-only flags -ftz=true -prec-sqrt=false -prec-div=false,
// which leave the FP64 reference mode untouched.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "of_device.cuh"
#include "of_internal.h"
#include "bulk_copy.cuh"
#include "path_fp32.cuh"
#include "f32x2.cuh"

namespace {

constexpr uint32_t kLsmStreamTag = 0x4C534D31u;  // "LSM1"
constexpr int kPassThreads = 256;
constexpr int kPathsPerThread = 4;
constexpr int kPathsPerBlock = kPassThreads * kPathsPerThread;
constexpr int kMaxMoments = 12;  // degree 3: x^0..x^6 (7) + y x^0..x^3 (4) ; degree 2: 8

// ---------------------------------------------------------------------------
// xoshiro256++ jump-ahead over GF(2)
// ---------------------------------------------------------------------------
void xoshiro_linear_step(uint64_t s[4]) {  // the state update of next_u64 (fast_rng.rs:58-66)
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = (s[3] << 45) | (s[3] >> 19);
}

void gf2_apply_host(const uint64_t* M, const uint64_t v[4], uint64_t out[4]) {
  uint64_t r[4] = {0, 0, 0, 0};
  for (int w = 0; w < 4; ++w)
    for (int b = 0; b < 64; ++b)
      if ((v[w] >> b) & 1ULL) {
        const uint64_t* c = M + (size_t)(w * 64 + b) * 4;
        for (int k = 0; k < 4; ++k) r[k] ^= c[k];
      }
  for (int k = 0; k < 4; ++k) out[k] = r[k];
}

// tables[k] = columns of T^(2^k), k = 0..63; column j = T^(2^k) e_j.
const std::vector<uint64_t>& jump_tables() {
  static std::vector<uint64_t> tab;
  static std::once_flag once;
  std::call_once(once, [] {
    tab.assign((size_t)64 * 256 * 4, 0);
    for (int j = 0; j < 256; ++j) {
      uint64_t s[4] = {0, 0, 0, 0};
      s[j / 64] = 1ULL << (j % 64);
      xoshiro_linear_step(s);
      for (int k = 0; k < 4; ++k) tab[(size_t)j * 4 + k] = s[k];
    }
    for (int p = 1; p < 64; ++p) {
      const uint64_t* prev = tab.data() + (size_t)(p - 1) * 1024;
      uint64_t* cur = tab.data() + (size_t)p * 1024;
      for (int j = 0; j < 256; ++j) gf2_apply_host(prev, prev + (size_t)j * 4, cur + (size_t)j * 4);
    }
  });
  return tab;
}

__device__ void gf2_apply(const uint64_t* __restrict__ M, uint64_t s[4]) {
  uint64_t r0 = 0, r1 = 0, r2 = 0, r3 = 0;
#pragma unroll 1
  for (int w = 0; w < 4; ++w) {
    const uint64_t word = s[w];
#pragma unroll 8
    for (int b = 0; b < 64; ++b) {
      const uint64_t m = 0ULL - ((word >> b) & 1ULL);
      const ulonglong2* c = reinterpret_cast<const ulonglong2*>(M + (size_t)(w * 64 + b) * 4);
      const ulonglong2 c01 = __ldg(c), c23 = __ldg(c + 1);
      r0 ^= c01.x & m;
      r1 ^= c01.y & m;
      r2 ^= c23.x & m;
      r3 ^= c23.y & m;
    }
  }
  s[0] = r0;
  s[1] = r1;
  s[2] = r2;
  s[3] = r3;
}

__device__ void xoshiro_jump(of::Xoshiro256pp& x, uint64_t n, const uint64_t* __restrict__ tables) {
  uint64_t s[4] = {x.s0, x.s1, x.s2, x.s3};
  for (int k = 0; k < 64 && n; ++k, n >>= 1)
    if (n & 1ULL) gf2_apply(tables + (size_t)k * 1024, s);
  x.s0 = s[0];
  x.s1 = s[1];
  x.s2 = s[2];
  x.s3 = s[3];
}

__global__ void jump_test_kernel(uint64_t seed, const uint64_t* draws, int64_t n, const uint64_t* tables,
                                 uint64_t* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  of::Xoshiro256pp x;
  x.seed(seed);
  xoshiro_jump(x, draws[i], tables);
  out[i * 4 + 0] = x.s0;
  out[i * 4 + 1] = x.s1;
  out[i * 4 + 2] = x.s2;
  out[i * 4 + 3] = x.s3;
}

// ---------------------------------------------------------------------------
// Contract constants
// ---------------------------------------------------------------------------
enum : int32_t { DYN_GBM = 0, DYN_LOCAL_VOL = 1, DYN_HESTON = 2 };

struct LsmC {
  int32_t put;
  int32_t steps;
  int32_t dynamics;
  int32_t lv_nk;             // local vol: strikes in the sampled grid
  double spot, strike, inv_strike, drift, step_vol, disc, inv_spot;  // strike = terminal strike
  // local-vol and Heston Euler (longstaff_schwartz.rs:218-281), FP64
  double mu, dt, sqrt_dt, kappa, theta, xi, rho, v0;
  const double* lv_k;        // [lv_nk] strikes of the sampled surface
  const double* lv_v;        // [n_expiries][lv_nk] vols
  const float* lv_kf;        // FP32 copies for the Philox mode
  const float* lv_vf;
  float fdrift, fstep_vol, fspot, fmudt, fsqrt_dt, fdt, fy_floor;
  of::StepConsts hc;         // FP32 Heston Euler constants
  uint32_t cid;              // FP32 mode: the contract's Philox stream, its index in the caller's list
};

// Per simulation step: the strike of an exercise date there (the terminal
// strike elsewhere) and the local-vol expiry bracket of the step's end time
// t = max(ti dt, 1e-8) (path-independent, so computed once on the host).
struct LsmStep {
  double strike, inv_strike;
  int32_t e0, e1;
  double ew;
  float fstrike, finv_strike, few, pad;
};

struct LsmBatch {
  const LsmC* c;             // [nc]
  const uint8_t* can_ex;     // [nc][steps+1]
  const LsmStep* st;         // [nc][steps+1]
  int32_t nc, steps;
  int64_t n, npad;           // paths, padded path stride
  void* S;                   // [nc][steps][npad] (T)
  void* V;                   // [nc][npad]
  int32_t* tau;             // [nc][npad] step of each path's cash flow (FP64 mode, delta only)
  uint32_t* exflags;        // [nc][steps+1][npad/32] FP32 mode, delta only: per date, word 4g+e
                            // bit L = path 4(32g+L)+e exercised at that date
  double* partials;          // [nc][blocks][kMaxMoments]
  double* betas;             // [2][nc][4] + valid flag in [2][nc] (separate)
  int32_t* beta_ok;          // [2][nc]
  int32_t* regress_count;    // [nc]
  uint32_t* counters;        // [nc]
  double* results;           // [nc][3]: price, stderr, delta
  int32_t blocks;            // blocks per contract
  int32_t degree;
  int32_t want_delta;
  int32_t track;             // exercise-boundary statistics wanted
  unsigned long long* ex_count;  // [nc][steps+1] paths exercised at each date
  unsigned long long* ex_bits;   // [nc][steps+1] bits of the max (put) / min (call) exercised spot
  double* itm_count;             // [nc][steps+1] in-the-money paths at each regression date
  const double* disc_pow;        // [nc][steps+1] disc^k by repeated multiplication, as V is discounted
  uint32_t* status;              // bit 0: a pass gave up waiting for its bulk copies; bit 1: its drain gave up too
  unsigned long long* term_itm;  // [nc] paths in the money at expiry
  uint64_t seed;
  of::PhiloxKeys keys;
  uint32_t contract_base;
  const double* inj;         // [nc][n][steps][draws] or null
  const uint64_t* jump;      // jump tables
  int32_t chunk;             // paths per thread in the reference generator
};

template <typename T>
__device__ __forceinline__ T intrinsic_v(bool put, T s, T k) {
  const T v = put ? k - s : s - k;
  return v > T(0) ? v : T(0);
}

// SampledVolSurface::vol (src/market/market.rs:104-174) with the expiry
// bracket of the step precomputed: locate the strike by the same first-match
// linear scan (a grid point takes the lower interval with weight 1), then
// interpolate in strike, then in expiry.
template <typename T>
__device__ __forceinline__ T lsm_local_vol(const T* __restrict__ g, const T* __restrict__ v, int nk, int e0, int e1,
                                           T ew, T strike) {
  const T x = strike > __ldg(g) ? strike : __ldg(g);
  int s0 = 0, s1 = 0;
  T sw = T(0);
  if (x >= __ldg(g + nk - 1)) {
    s0 = s1 = nk - 1;
  } else if (x > __ldg(g)) {
    int lo = 0;
    for (int i = 0; i < nk - 1; ++i)
      if (x >= __ldg(g + i) && x <= __ldg(g + i + 1)) {
        lo = i;
        break;
      }
    s0 = lo;
    s1 = lo + 1;
    sw = (x - __ldg(g + lo)) / (__ldg(g + lo + 1) - __ldg(g + lo));
  }
  const T* r0 = v + (size_t)e0 * nk;
  const T* r1 = v + (size_t)e1 * nk;
  if (e0 == e1 && s0 == s1) return __ldg(r0 + s0);
  if (e0 == e1) return __ldg(r0 + s0) + (__ldg(r0 + s1) - __ldg(r0 + s0)) * sw;
  if (s0 == s1) return __ldg(r0 + s0) + (__ldg(r1 + s0) - __ldg(r0 + s0)) * ew;
  const T a = __ldg(r0 + s0) + (__ldg(r0 + s1) - __ldg(r0 + s0)) * sw;
  const T b = __ldg(r1 + s0) + (__ldg(r1 + s1) - __ldg(r1 + s0)) * sw;
  return a + (b - a) * ew;
}

// Terminal cash flow of a path and, when boundary statistics are wanted,
// the count of in-the-money paths at expiry (one atomic per thread that has any).
__device__ __forceinline__ int terminal_value(const LsmC& C, double k_T, double s, double& v, double& dv) {
  v = intrinsic_v<double>(C.put, s, k_T);
  dv = v > 0.0 ? (C.put ? -s * C.inv_spot : s * C.inv_spot) : 0.0;
  return v > 0.0 ? 1 : 0;
}

// FP64 reference generator: chunk of consecutive paths per thread.  The
// single xoshiro256++ stream feeds path after path; 1 draw per step (GBM,
// local vol) or 2 (Heston: z1 then z2), longstaff_schwartz.rs:190-283.
__global__ void __launch_bounds__(128) lsm_gen_ref(LsmBatch B) {
  const int c = blockIdx.y;
  const LsmC C = B.c[c];
  const int64_t chunk0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * B.chunk;
  if (chunk0 >= B.n) return;
  const int draws = C.dynamics == DYN_HESTON ? 2 : 1;
  const LsmStep* st = B.st + (size_t)c * (B.steps + 1);
  double* S = (double*)B.S + (size_t)c * B.steps * B.npad;
  double* V = (double*)B.V + (size_t)c * B.npad;
  int32_t* tau = B.tau + (size_t)c * B.npad;
  of::Xoshiro256pp rng;
  if (!B.inj) {
    rng.seed(B.seed);
    xoshiro_jump(rng, (uint64_t)chunk0 * (uint64_t)B.steps * (uint64_t)draws, B.jump);
  }
  const double k_T = st[B.steps].strike;
  const double rho_c = sqrt(1.0 - C.rho * C.rho);
  int itm = 0;
  const int64_t end = chunk0 + B.chunk < B.n ? chunk0 + B.chunk : B.n;
  for (int64_t p = chunk0; p < end; ++p) {
    double s = C.spot, var = C.v0;
    const double* z = B.inj ? B.inj + ((size_t)c * B.n + p) * B.steps * draws : nullptr;
    for (int t = 1; t <= B.steps; ++t) {
      const double z1 = z ? z[(size_t)(t - 1) * draws] : of::acklam_inv_cdf(rng.next_f64());
      if (C.dynamics == DYN_GBM) {
        s = s * exp(fma(C.step_vol, z1, C.drift));  // longstaff_schwartz.rs:213-214
      } else if (C.dynamics == DYN_LOCAL_VOL) {
        // :223-235: sigma at the step's end time and the previous spot
        const double sigma = lsm_local_vol<double>(C.lv_k, C.lv_v, C.lv_nk, st[t].e0, st[t].e1, st[t].ew,
                                                   s > 1.0e-8 ? s : 1.0e-8);
        const double drift = (C.mu - 0.5 * sigma * sigma) * C.dt;
        s *= exp(drift + sigma * C.sqrt_dt * z1);
        s = s > 1.0e-12 ? s : 1.0e-12;
      } else {
        // Heston::step_euler (src/models/stochastic.rs:56-71), :259-275
        const double z2 = z ? z[(size_t)(t - 1) * draws + 1] : of::acklam_inv_cdf(rng.next_f64());
        const double v_pos = var > 0.0 ? var : 0.0;
        const double zs = C.rho * z1 + rho_c * z2;
        double v_next = var + C.kappa * (C.theta - v_pos) * C.dt + C.xi * sqrt(v_pos) * C.sqrt_dt * z1;
        v_next = v_next > 0.0 ? v_next : 0.0;
        const double s_next = s * exp((C.mu - 0.5 * v_pos) * C.dt + sqrt(v_pos) * C.sqrt_dt * zs);
        s = s_next > 1.0e-12 ? s_next : 1.0e-12;
        var = v_next;
      }
      S[(size_t)(t - 1) * B.npad + p] = s;
    }
    double v, dv;
    itm += terminal_value(C, k_T, s, v, dv);
    V[p] = v;
    if (B.want_delta) tau[p] = B.steps;
  }
  if (B.track && itm) atomicAdd(B.term_itm + c, (unsigned long long)itm);
}

// FP32 Philox generator: 4 consecutive paths per thread, float4 stores.  The
// dynamics are a template parameter and the time loop walks whole counter
// blocks, so each step reads its Philox words without a select.  Normals come
// in Box-Muller pairs: GBM and local vol take steps t, t+1 (t even) from words
// (0,1) or (2,3) of counter block t/4; Heston's (z1, z2) of step t are the pair
// of words 2(t%2), 2(t%2)+1 of counter block t/2.  A batch holds one dynamics
// kind.
template <int DYN>
__global__ void __launch_bounds__(256, DYN == DYN_GBM ? 4 : 2) lsm_gen_philox(const __grid_constant__ LsmBatch B) {
  constexpr int kStepsPerBlock = DYN == DYN_HESTON ? 2 : 4;
  const int c = blockIdx.y;
  const LsmC& C = B.c[c];
  const int64_t p0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  const bool live = p0 < B.npad;  // the grid's last block may reach past the padded path count
  const LsmStep* st = B.st + (size_t)c * (B.steps + 1);
  const uint32_t cid = C.cid;
  const bool put = C.put != 0;
  const float fspot = C.fspot;
  int itm = 0;
  if (live) {
    // padding paths (p >= n) store a spot that is out of the money at every date
    const float pad = put ? __int_as_float(0x7F800000) : 0.0f;
    bool in[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) in[q] = p0 + q < B.n;
    float* S = (float*)B.S + (size_t)c * B.steps * B.npad + p0;
    of::LegState L[4];
    float s[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      L[q] = of::LegState{0.0f, DYN == DYN_HESTON ? C.hc.v0 : 0.0f};
      s[q] = fspot;
    }
    for (int tb = 0; tb < B.steps; tb += kStepsPerBlock) {
      const uint32_t blk = (uint32_t)(tb / kStepsPerBlock);
      uint4 r[4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        r[q] = of::philox4x32_10(make_uint4(blk, (uint32_t)(p0 + q), cid, kLsmStreamTag), B.keys);
      if (DYN == DYN_GBM) {
        // paths (0,1) and (2,3) in packed pairs: each half is the scalar
        // loop's arithmetic below, bit for bit
#pragma unroll
        for (int k = 0; k < kStepsPerBlock; k += 2) {
          float2 za[2], zb[2];  // the normals of steps tb+k and tb+k+1
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const uint32_t* w0 = &r[2 * h].x;
            const uint32_t* w1 = &r[2 * h + 1].x;
            of::normal_pairs_scaled2_from_u32(w0[k], w0[k + 1], w1[k], w1[k + 1], of::kBoxMullerK2, za[h], zb[h]);
          }
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int t = tb + k + e;
            if (t >= B.steps) break;
            float4 out;
            float* o = &out.x;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              float2 y = make_float2(L[2 * h].y, L[2 * h + 1].y);
              y = of::fma2(of::splat2(C.fstep_vol), e ? zb[h] : za[h], of::add2(y, of::splat2(C.fdrift)));
              L[2 * h].y = y.x;
              L[2 * h + 1].y = y.y;
              const float2 sp = of::mul2(of::splat2(fspot), make_float2(__expf(y.x), __expf(y.y)));
              s[2 * h] = sp.x;
              s[2 * h + 1] = sp.y;
              o[2 * h] = in[2 * h] ? sp.x : pad;
              o[2 * h + 1] = in[2 * h + 1] ? sp.y : pad;
            }
            __stcs(reinterpret_cast<float4*>(S + (size_t)t * B.npad), out);
          }
        }
        continue;
      }
      float2 zp[4];  // Box-Muller pair of words (0,1) or (2,3) of the counter block
#pragma unroll
      for (int k = 0; k < kStepsPerBlock; ++k) {
        const int t = tb + k;
        if (t >= B.steps) break;
        float4 out;
        float* o = &out.x;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t* w = &r[q].x;
          if (DYN == DYN_HESTON) {
            const float2 z = of::normal_pair_scaled_from_u32(w[2 * k], w[2 * k + 1], C.hc.bm_k2);
            of::heston_euler_step(L[q], C.hc, z.x, z.y);
          } else {
            if ((k & 1) == 0) zp[q] = of::normal_pair_from_u32(w[k], w[k + 1]);
            const float z = (k & 1) ? zp[q].y : zp[q].x;
            if (DYN == DYN_GBM) {
              L[q].y = fmaf(C.fstep_vol, z, L[q].y + C.fdrift);
            } else {
              const LsmStep& e = st[t + 1];
              const float sig = lsm_local_vol<float>(C.lv_kf, C.lv_vf, C.lv_nk, e.e0, e.e1, e.few,
                                                     s[q] > 1.0e-8f ? s[q] : 1.0e-8f);
              const float y = fmaf(sig * C.fsqrt_dt, z, fmaf(-0.5f * sig * sig, C.fdt, L[q].y + C.fmudt));
              L[q].y = y > C.fy_floor ? y : C.fy_floor;
            }
          }
          s[q] = fspot * __expf(L[q].y);
          o[q] = in[q] ? s[q] : pad;
        }
        // streaming (evict-first) stores: the generator of the next batch runs
        // beside this batch's passes, whose cash flows and path columns
        // should keep their place in L2
        __stcs(reinterpret_cast<float4*>(S + (size_t)t * B.npad), out);
      }
    }
    const float fk = st[B.steps].fstrike;
    float4 v4;
    float* vv = &v4.x;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float v = intrinsic_v<float>(put, s[q], fk);
      vv[q] = in[q] ? v : 0.0f;
      itm += (in[q] && v > 0.0f) ? 1 : 0;
    }
    __stcs(reinterpret_cast<float4*>((float*)B.V + (size_t)c * B.npad + p0), v4);
  }
  if (B.track) {
    itm = __reduce_add_sync(of::kFullMask, itm);
    if ((threadIdx.x & 31) == 0 && itm) atomicAdd(B.term_itm + c, (unsigned long long)itm);
  }
}

// Continuation value of the fitted basis, FP64 (longstaff_schwartz.rs:597).
// Degree 3: the cubic in x = S/K_t - shift (shift 0 in the FP64 mode, 1 in
// the FP32 mode's centred basis).
__device__ __forceinline__ double continuation(int degree, const double* b, double s, double inv_k,
                                               double shift = 0.0) {
  if (degree == 2) return b[0] + b[1] * s + b[2] * s * s;
  const double x = s * inv_k - shift;
  return b[0] + x * (b[1] + x * (b[2] + x * b[3]));
}

// Solves the normal equations from the reduced moments (thread 0 of the last block).
__device__ void solve_beta(int degree, const double* m, double* beta, int32_t* ok) {
  if (m[0] < 3.0) {  // fewer than 3 in-the-money paths: no regression (:561-563)
    *ok = 0;
    return;
  }
  *ok = 1;
  beta[0] = beta[1] = beta[2] = beta[3] = 0.0;
  if (degree == 2) {
    // m = {s1, S, S^2, S^3, S^4, y, Sy, S^2y}; nalgebra LU with partial pivoting
    double a[3][3] = {{m[0], m[1], m[2]}, {m[1], m[2], m[3]}, {m[2], m[3], m[4]}};
    double b[3] = {m[5], m[6], m[7]};
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
      if (a[i][i] == 0.0) return;  // singular: beta = 0 (:592)
    double x[3];
    for (int i = 2; i >= 0; --i) {
      double s = b[i];
      for (int j = i + 1; j < 3; ++j) s -= a[i][j] * x[j];
      x[i] = s / a[i][i];
    }
    beta[0] = x[0];
    beta[1] = x[1];
    beta[2] = x[2];
  } else {
    // m = {x^0..x^6, y x^0..x^3}; Cholesky of the 4x4 Gram matrix
    double a[4][4], l[4][4] = {{0}};
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) a[i][j] = m[i + j];
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = a[i][j];
        for (int k = 0; k < j; ++k) s -= l[i][k] * l[j][k];
        if (i == j) {
          if (!(s > 0.0)) return;
          l[i][i] = sqrt(s);
        } else {
          l[i][j] = s / l[j][j];
        }
      }
    double y[4], x[4];
    for (int i = 0; i < 4; ++i) {
      double s = m[7 + i];
      for (int k = 0; k < i; ++k) s -= l[i][k] * y[k];
      y[i] = s / l[i][i];
    }
    for (int i = 3; i >= 0; --i) {
      double s = y[i];
      for (int k = i + 1; k < 4; ++k) s -= l[k][i] * x[k];
      x[i] = s / l[i][i];
    }
    for (int i = 0; i < 4; ++i) beta[i] = x[i];
  }
}

// Fixed-order reduction of the per-block partials of one contract by the
// block that finished last: warp w sums moments w, w + 8, ... with its lanes
// striding over the blocks' rows and a shuffle tree (one barrier in all);
// thread 0 then solves for the betas.
__device__ void last_block_reduce(const LsmBatch& B, int c, int nm, int nblk, double* moments_sh, double* red_sh,
                                  int t_pass) {
  const double* part = B.partials + (size_t)c * B.blocks * kMaxMoments;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = warp; k < nm; k += nw) {
    double acc = 0.0;
    for (int b = lane; b < nblk; b += 32) acc += __ldcg(part + (size_t)b * kMaxMoments + k);
    acc = of::warp_sum(acc);
    if (lane == 0) moments_sh[k] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int buf = t_pass & 1;
    double* beta = B.betas + ((size_t)buf * B.nc + c) * 4;
    int32_t* ok = B.beta_ok + (size_t)buf * B.nc + c;
    solve_beta(B.degree, moments_sh, beta, ok);
    if (*ok) B.regress_count[c] += 1;
    if (B.track) B.itm_count[(size_t)c * (B.steps + 1) + t_pass] = moments_sh[0];
  }
}

// Exercise statistics of one date, reduced over the warp and added with one
// atomic per warp: the count, and the largest (put) or smallest (call)
// exercised spot.  Positive doubles order like their bit patterns; a lane
// that exercised nothing passes 0 (put) or +inf (call).  Called by all 32
// lanes of the warp.
__device__ __forceinline__ void record_exercise(const LsmBatch& B, int c, int date, bool put, unsigned cnt,
                                                double ext) {
  cnt = __reduce_add_sync(of::kFullMask, cnt);
  unsigned long long bits = (unsigned long long)__double_as_longlong(ext);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(of::kFullMask, bits, o);
    bits = put ? (other > bits ? other : bits) : (other < bits ? other : bits);
  }
  if ((threadIdx.x & 31) == 0 && cnt) {
    const size_t k = (size_t)c * (B.steps + 1) + date;
    atomicAdd(B.ex_count + k, (unsigned long long)cnt);
    if (put) atomicMax(B.ex_bits + k, bits);
    else atomicMin(B.ex_bits + k, bits);
  }
}

// The end of a pass: the block's moments are reduced with one barrier (warp
// shuffles, then one thread per moment sums the warps in a fixed order) into
// its partials; the block that finishes last reduces every block's partials
// and solves for the betas of date t.
template <int NM>
__device__ __forceinline__ void block_moments(const LsmBatch& B, int c, int t, const double* mom, double* red_sh,
                                              double* mom_sh) {
  __shared__ bool is_last;
  double* part = B.partials + ((size_t)c * B.blocks + blockIdx.x) * kMaxMoments;
#pragma unroll
  for (int k = 0; k < NM; ++k) {
    const double w = of::warp_sum(mom[k]);
    if ((threadIdx.x & 31) == 0) red_sh[(threadIdx.x >> 5) * kMaxMoments + k] = w;
  }
  __syncthreads();
  if ((int)threadIdx.x < NM) {
    double acc = 0.0;
    for (int i = 0; i < kPassThreads / 32; ++i) acc += red_sh[i * kMaxMoments + threadIdx.x];
    part[threadIdx.x] = acc;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t done = atomicAdd(B.counters + c, 1u);
    is_last = done == gridDim.x - 1;
  }
  __syncthreads();
  if (is_last) {
    __threadfence();
    last_block_reduce(B, c, NM, (int)gridDim.x, mom_sh, red_sh, t);
    if (threadIdx.x == 0) B.counters[c] = 0;
  }
}

// One path of a pass: exercise at date t+1 (spot s1) with the betas of that
// date, discount one step, and the in-the-money basis moments at date t
// (spot s0, longstaff_schwartz.rs:543-601).
// k1/ik1: strike and its inverse at date t+1, k0/ik0 at date t.  Returns
// whether the path exercised at t+1.
template <int DEG>
__device__ __forceinline__ bool lsm_path_update(const LsmC& C, const double* beta, bool have_beta, bool ex_now,
                                                double k1, double ik1, double k0, double ik0, double s1, double s0,
                                                double& v, double* mom) {
  bool exercised = false;
  if (have_beta) {
    const double ex = intrinsic_v<double>(C.put, s1, k1);
    if (ex > 0.0 && ex > continuation(DEG, beta, s1, ik1)) {
      v = ex;
      exercised = true;
    }
  }
  v *= C.disc;
  if (ex_now && intrinsic_v<double>(C.put, s0, k0) > 0.0) {
    if (DEG == 2) {
      const double s2 = s0 * s0;
      mom[0] += 1.0;
      mom[1] += s0;
      mom[2] += s2;
      mom[3] += s2 * s0;
      mom[4] += s2 * s2;
      mom[5] += v;
      mom[6] += s0 * v;
      mom[7] += s2 * v;
    } else {
      const double x = s0 * ik0;
      double pw = 1.0;
#pragma unroll
      for (int e = 0; e < 7; ++e) {
        mom[e] += pw;
        if (e < 4) mom[7 + e] += pw * v;
        pw *= x;
      }
    }
  }
  return exercised;
}

// One exercise date t (1 <= t <= steps-1) of the FP64 reference mode:
// exercise(t+1), discount, moments(t), all in FP64 with the reference's
// operation order (no contraction).  A block walks the contract's chunks of
// kPathsPerBlock paths with a grid stride and reduces its moments once at the
// end; DEG (the basis degree) is a template parameter so that the moment count
// is known at compile time.
template <typename T, int DEG>
__global__ void __launch_bounds__(kPassThreads, 3) lsm_pass(LsmBatch B, int t) {
  __shared__ double red_sh[kPassThreads];
  __shared__ double mom_sh[kMaxMoments];
  const int c = blockIdx.y;
  const LsmC C = B.c[c];
  const T* S = (const T*)B.S + (size_t)c * B.steps * B.npad;
  T* V = (T*)B.V + (size_t)c * B.npad;
  int32_t* tau = B.tau + (size_t)c * B.npad;
  const bool ex_next = (t + 1 < B.steps) && B.can_ex[(size_t)c * (B.steps + 1) + t + 1];
  const bool ex_now = B.can_ex[(size_t)c * (B.steps + 1) + t];
  const int nb = (t + 1) & 1;  // betas of date t+1 were written by the previous pass
  const bool have_beta = ex_next && B.beta_ok[(size_t)nb * B.nc + c];
  double beta[4] = {0, 0, 0, 0};
  if (have_beta)
    for (int k = 0; k < 4; ++k) beta[k] = B.betas[((size_t)nb * B.nc + c) * 4 + k];
  const LsmStep* st = B.st + (size_t)c * (B.steps + 1);
  const double k1 = st[t + 1].strike, ik1 = st[t + 1].inv_strike, k0 = st[t].strike, ik0 = st[t].inv_strike;
  unsigned n_ex = 0;
  double ext = C.put ? 0.0 : __longlong_as_double(0x7FF0000000000000LL);
  constexpr int nm = DEG == 2 ? 8 : 11;
  double mom[nm];
#pragma unroll
  for (int k = 0; k < nm; ++k) mom[k] = 0.0;
  for (int64_t chunk = blockIdx.x; chunk < B.blocks; chunk += gridDim.x) {
    const int64_t base = chunk * kPathsPerBlock;
#pragma unroll
    for (int q = 0; q < kPathsPerThread; ++q) {
      const int64_t p = base + q * kPassThreads + threadIdx.x;
      if (p >= B.n) break;
      double v = (double)V[p];
      const double s1 = have_beta ? (double)S[(size_t)t * B.npad + p] : 0.0;      // spot at date t+1
      const double s0 = ex_now ? (double)S[(size_t)(t - 1) * B.npad + p] : 0.0;  // spot at date t
      if (lsm_path_update<DEG>(C, beta, have_beta, ex_now, k1, ik1, k0, ik0, s1, s0, v, mom)) {
        ++n_ex;
        ext = C.put ? fmax(ext, s1) : fmin(ext, s1);
        if (B.want_delta) tau[p] = t + 1;  // the cash flow now comes at date t+1
      }
      V[p] = (T)v;
    }
  }
  if (B.track && have_beta) record_exercise(B, c, t + 1, C.put, n_ex, ext);  // block-uniform condition
  if (!ex_now) return;
  block_moments<nm>(B, c, t, mom, red_sh, mom_sh);
}

// FP32 path store, FP32 arithmetic for everything but the regression moments:
// the exercise decision (continuation with FP32 betas, explicit fmaf), the
// one-step discount (v*d with d split into two floats, so the rounding of d
// does not compound over the dates) and the in-the-money test.  The moments
// stay FP64 (one fma per cross moment, the count as an integer).  No per-path
// bounds test: the generator stores an out-of-the-money spot (+inf for a put,
// 0 for a call) and V = 0 for the padding paths p >= n, so they never exercise
// and never enter the moments.  For the pathwise delta each pass writes one
// dense row of exercise flags (a bit per path, warp ballots) for its date
// instead of scattered per-path payment steps: a scattered 4-byte store
// leaves a partly written sector that the L2 fills from DRAM, which cost a
// quarter of the pass's traffic.  The final kernel takes each path's payment
// step as the first date whose flag is set.
struct F32Pass {
  bool have_beta, ex_now, want_delta;
  float b0, b1, b2, b3, k1, ik1, k0, ik0, dh, dl;
};

// One quad (four consecutive paths) of an FP32 pass; returns the paths that
// exercised at date t+1 as a 4-bit mask.
template <int DEG, bool PUT>
__device__ __forceinline__ unsigned f32_quad(const F32Pass& P, float4& v4, const float4& a4, const float4& p4,
                                             double* mom, unsigned& n_ex, unsigned& n_itm, float& ext) {
  float* vv = &v4.x;
  const float* s1 = &a4.x;
  const float* s0 = &p4.x;
  unsigned exm = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    float v = vv[e];
    if (P.have_beta) {
      const float ex = PUT ? P.k1 - s1[e] : s1[e] - P.k1;
      const float x1 = DEG == 3 ? s1[e] * P.ik1 : s1[e];
      const float cont = DEG == 3 ? fmaf(x1, fmaf(x1, fmaf(x1, P.b3, P.b2), P.b1), P.b0)
                                  : fmaf(x1, fmaf(x1, P.b2, P.b1), P.b0);
      if (ex > 0.0f && ex > cont) {
        v = ex;
        ++n_ex;
        ext = PUT ? fmaxf(ext, s1[e]) : fminf(ext, s1[e]);
        exm |= 1u << e;
      }
    }
    v = fmaf(v, P.dh, v * P.dl);
    vv[e] = v;
    if (P.ex_now && (PUT ? P.k0 - s0[e] : s0[e] - P.k0) > 0.0f) {
      ++n_itm;
      const double x = DEG == 3 ? (double)(s0[e] * P.ik0) : (double)s0[e];
      const double y = (double)v;
      const double x2 = x * x, x3 = x2 * x;
      if (DEG == 2) {
        mom[1] += x;
        mom[2] += x2;
        mom[3] += x3;
        mom[4] += x2 * x2;
        mom[5] += y;
        mom[6] = fma(x, y, mom[6]);
        mom[7] = fma(x2, y, mom[7]);
      } else {
        const double x4 = x2 * x2;
        mom[1] += x;
        mom[2] += x2;
        mom[3] += x3;
        mom[4] += x4;
        mom[5] += x4 * x;
        mom[6] += x3 * x3;
        mom[7] += y;
        mom[8] = fma(x, y, mom[8]);
        mom[9] = fma(x2, y, mom[9]);
        mom[10] = fma(x3, y, mom[10]);
      }
    }
  }
  return exm;
}

// The cubic-basis quad with packed pair arithmetic (paths 0,1 and 2,3 of the
// quad share each instruction).  The FP32 mode's cubic basis is 1, x, x^2, x^3
// in x = S/K_t - 1 (one fma, exact near the money): the same span as the
// monomials of S/K_t, but centred at the strike, where the in-the-money paths
// lie, so that the normal equations are some 10-100x better conditioned and
// moments with FP32 rounding fit the same continuation to about 1e-6 (with
// monomials of S/K_t, FP32 moments moved fitted values by up to 0.2 on
// near-expiry dates, whose in-the-money spots span a narrow range).
// The basis moments of the in-the-money paths (x as above, y = discounted cash
// flow; out-of-the-money paths enter as x = y = 0 and add nothing) go into FP32
// pair accumulators instead of FP64 registers: acc[0..5] = sum x^1..x^6,
// acc[6] = sum y, acc[7..9] = sum y x^1..x^3; the count is n_itm.  Every kFlushChunks chunks the pass
// adds each accumulator's two halves, sums them over the warp in FP32 and adds
// the warp's total to the warp's FP64 moments in shared memory; so an FP32 sum
// covers at most 2 kFlushChunks paths of one lane half and 32 lanes, whatever
// the path count, and the FP64 sums carry the rest.  (The rounding of these
// short FP32 sums, about 1e-6 relative at worst, moves the fitted betas far
// less than the FP32 rounding of the betas themselves does.)
template <bool PUT, bool TRACK>
__device__ __forceinline__ unsigned f32_quad3_packed(const F32Pass& P, float4& v4, const float4& a4, const float4& p4,
                                                     float2* acc, unsigned& n_ex, unsigned& n_itm, float& ext) {
  using of::add2;
  using of::fma2;
  using of::mul2;
  using of::splat2;
  using of::sub2;
  float2 v[2] = {make_float2(v4.x, v4.y), make_float2(v4.z, v4.w)};
  const float2 s1[2] = {make_float2(a4.x, a4.y), make_float2(a4.z, a4.w)};
  const float2 s0[2] = {make_float2(p4.x, p4.y), make_float2(p4.z, p4.w)};
  unsigned exm = 0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (P.have_beta) {
      const float2 ex = PUT ? sub2(splat2(P.k1), s1[h]) : sub2(s1[h], splat2(P.k1));
      const float2 x1 = fma2(s1[h], splat2(P.ik1), splat2(-1.0f));
      const float2 cont = fma2(x1, fma2(x1, fma2(x1, splat2(P.b3), splat2(P.b2)), splat2(P.b1)), splat2(P.b0));
      if (ex.x > 0.0f && ex.x > cont.x) {
        v[h].x = ex.x;
        if (TRACK) {  // the Bermudan boundary statistics
          ++n_ex;
          ext = PUT ? fmaxf(ext, s1[h].x) : fminf(ext, s1[h].x);
        }
        exm |= 1u << (2 * h);
      }
      if (ex.y > 0.0f && ex.y > cont.y) {
        v[h].y = ex.y;
        if (TRACK) {
          ++n_ex;
          ext = PUT ? fmaxf(ext, s1[h].y) : fminf(ext, s1[h].y);
        }
        exm |= 2u << (2 * h);
      }
    }
    v[h] = fma2(v[h], splat2(P.dh), mul2(v[h], splat2(P.dl)));
    if (P.ex_now) {
      const bool ia = (PUT ? P.k0 - s0[h].x : s0[h].x - P.k0) > 0.0f;
      const bool ib = (PUT ? P.k0 - s0[h].y : s0[h].y - P.k0) > 0.0f;
      n_itm += (unsigned)ia + (unsigned)ib;
      const float2 x0 = fma2(s0[h], splat2(P.ik0), splat2(-1.0f));
      const float2 x = make_float2(ia ? x0.x : 0.0f, ib ? x0.y : 0.0f);
      const float2 y = make_float2(ia ? v[h].x : 0.0f, ib ? v[h].y : 0.0f);
      const float2 x2 = mul2(x, x), x3 = mul2(x2, x);
      acc[0] = add2(acc[0], x);
      acc[1] = add2(acc[1], x2);
      acc[2] = add2(acc[2], x3);
      acc[3] = fma2(x2, x2, acc[3]);
      acc[4] = fma2(x2, x3, acc[4]);
      acc[5] = fma2(x3, x3, acc[5]);
      acc[6] = add2(acc[6], y);
      acc[7] = fma2(y, x, acc[7]);
      acc[8] = fma2(y, x2, acc[8]);
      acc[9] = fma2(y, x3, acc[9]);
    }
  }
  v4 = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
  return exm;
}

constexpr int kFlushChunks = 32;  // FP32 moment accumulators flushed into FP64 this often

constexpr int kStages = 3;                                     // ring depth of the FP32 pass
constexpr uint32_t kChunkBytes = kPathsPerBlock * sizeof(float);  // one array's share of a chunk
constexpr uint64_t kWaitLimitNs = 1000000000ull;               // a bulk copy lands in microseconds

// The FP32 pass streams its three inputs through shared memory: chunk j of
// the block (1024 paths, grid-stride over the contract) has its V, S(t+1) and
// S(t) segments (4 KB each, only the ones the date needs) copied by
// cp.async.bulk into ring stage j % kStages, completed on that stage's
// mbarrier.  Thread 0 keeps kStages chunks in flight; one barrier per chunk
// both publishes the landed stage and frees the one consumed before it.  The
// new cash flows go straight to global memory.  A copy that has not landed
// after kWaitLimitNs sets B.status, and the block drains its outstanding
// copies (bounded the same way) and returns without its moments.  A drain
// that gives up as well sets a second status bit: the host then marks the
// context unusable, since copies may still land in shared memory that the
// returned block no longer owns.
template <int DEG, bool PUT, bool TRACK>
__device__ __forceinline__ void lsm_pass_f32_body(const LsmBatch& B, int t, float* ring, uint64_t* full,
                                                  double* red_sh, double* mom_sh, double* warp_mom) {
  constexpr int nm = DEG == 2 ? 8 : 11;
  const int c = blockIdx.y;
  const float* S = (const float*)B.S + (size_t)c * B.steps * B.npad;
  const float* gS1 = S + (size_t)t * B.npad;        // spot at date t+1
  const float* gS0 = S + (size_t)(t - 1) * B.npad;  // spot at date t
  float* gV = (float*)B.V + (size_t)c * B.npad;
  uint32_t* flags = B.exflags + ((size_t)c * (B.steps + 1) + (t + 1)) * (B.npad / 32);  // date t+1
  const uint8_t* can = B.can_ex + (size_t)c * (B.steps + 1);
  F32Pass P;
  P.ex_now = can[t];
  // S(t+1) is loaded whenever date t+1 may exercise; whether it does (betas
  // fitted there) is known only once the previous pass has completed
  const bool load1 = (t + 1 < B.steps) && can[t + 1];
  P.have_beta = false;
  P.b0 = P.b1 = P.b2 = P.b3 = 0.0f;
  const LsmStep* st = B.st + (size_t)c * (B.steps + 1);
  P.k1 = st[t + 1].fstrike;
  P.ik1 = st[t + 1].finv_strike;
  P.k0 = st[t].fstrike;
  P.ik0 = st[t].finv_strike;
  const double disc = B.c[c].disc;
  P.dh = (float)disc;
  P.dl = (float)(disc - (double)P.dh);
  P.want_delta = B.want_delta != 0;
  const int n_chunks = (B.blocks - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const uint32_t bytes = kChunkBytes * (1u + (load1 ? 1u : 0u) + (P.ex_now ? 1u : 0u));
  // stage layout: [S(t+1) | S(t) | V], kPathsPerBlock floats each.  The path
  // columns (written by the generator, long complete) and the cash flows
  // (written by the previous pass) are issued separately: see below.
  auto issue_s = [&](int j) {
    const int s = j % kStages;
    const int64_t off = ((int64_t)blockIdx.x + (int64_t)j * gridDim.x) * kPathsPerBlock;
    float* dst = ring + (size_t)s * 3 * kPathsPerBlock;
    const uint32_t bar = of::smem_u32(full + s);
    of::mbar_arrive_expect_tx(bar, bytes);
    if (load1) of::bulk_load(of::smem_u32(dst), gS1 + off, kChunkBytes, bar);
    if (P.ex_now) of::bulk_load(of::smem_u32(dst + kPathsPerBlock), gS0 + off, kChunkBytes, bar);
  };
  auto issue_v = [&](int j) {
    const int s = j % kStages;
    const int64_t off = ((int64_t)blockIdx.x + (int64_t)j * gridDim.x) * kPathsPerBlock;
    float* dst = ring + (size_t)s * 3 * kPathsPerBlock;
    of::bulk_load(of::smem_u32(dst + 2 * kPathsPerBlock), gV + off, kChunkBytes, of::smem_u32(full + s));
  };
  auto issue = [&](int j) {
    issue_s(j);
    issue_v(j);
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) of::mbar_init(of::smem_u32(full + s), 1);
    of::mbar_fence_init();
  }
  __syncthreads();
  // The first chunks' path columns stream in while the previous date's pass
  // finishes (it was launched with programmatic stream serialisation); its
  // outputs (cash flows, betas) are read only after griddepcontrol.wait.
  if (threadIdx.x == 0)
    for (int j = 0; j < kStages && j < n_chunks; ++j) issue_s(j);
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int nb = (t + 1) & 1;  // betas of date t+1 were written by the previous pass
  P.have_beta = load1 && B.beta_ok[(size_t)nb * B.nc + c];
  if (P.have_beta) {
    const double* bp = B.betas + ((size_t)nb * B.nc + c) * 4;
    P.b0 = (float)bp[0];
    P.b1 = (float)bp[1];
    P.b2 = (float)bp[2];
    P.b3 = (float)bp[3];
  }
  if (threadIdx.x == 0)
    for (int j = 0; j < kStages && j < n_chunks; ++j) issue_v(j);
  unsigned n_ex = 0, n_itm = 0;
  float ext = PUT ? 0.0f : __int_as_float(0x7F800000);
  double mom[nm];
#pragma unroll
  for (int k = 0; k < nm; ++k) mom[k] = 0.0;
  float2 acc[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) acc[k] = make_float2(0.f, 0.f);
  // lane 0 of each warp owns the warp's 10 FP64 moments in shared memory
  double* wm = warp_mom + (threadIdx.x >> 5) * 10;
  if (DEG == 3 && (threadIdx.x & 31u) == 0)
    for (int k = 0; k < 10; ++k) wm[k] = 0.0;
  auto flush = [&]() {  // called by all lanes of the warp
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      float a = acc[k].x + acc[k].y;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(of::kFullMask, a, o);
      if ((threadIdx.x & 31u) == 0) wm[k] += (double)a;
      acc[k] = make_float2(0.f, 0.f);
    }
  };
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  int i = 0;
  for (; i < n_chunks; ++i) {
    const int s = i % kStages;
    const bool landed = of::mbar_wait(of::smem_u32(full + s), (uint32_t)(i / kStages) & 1u, kWaitLimitNs);
    // every thread has finished chunk i-1, so its stage can be refilled
    if (!__syncthreads_and(landed)) break;
    if (threadIdx.x == 0 && i >= 1 && i - 1 + kStages < n_chunks) issue(i - 1 + kStages);
    const float* src = ring + (size_t)s * 3 * kPathsPerBlock;
    const float4 a4 = P.have_beta ? reinterpret_cast<const float4*>(src)[threadIdx.x] : zero;
    const float4 p4 = P.ex_now ? reinterpret_cast<const float4*>(src + kPathsPerBlock)[threadIdx.x] : zero;
    float4 v4 = reinterpret_cast<const float4*>(src + 2 * kPathsPerBlock)[threadIdx.x];
    const int64_t q = ((int64_t)blockIdx.x + (int64_t)i * gridDim.x) * kPassThreads + threadIdx.x;
    unsigned exm;
    if (DEG == 3) {
      exm = f32_quad3_packed<PUT, TRACK>(P, v4, a4, p4, acc, n_ex, n_itm, ext);
      if (P.ex_now && (i % kFlushChunks) == kFlushChunks - 1) flush();
    } else {
      exm = f32_quad<DEG, PUT>(P, v4, a4, p4, mom, n_ex, n_itm, ext);
    }
    reinterpret_cast<float4*>(gV)[q] = v4;
    if (P.want_delta) {
      // word 4g+e of the date's flag row: bit L = path 4(32g+L)+e exercised,
      // for the warp's 32 quads 32g .. 32g+31
      const unsigned lane = threadIdx.x & 31u;
      uint32_t word = 0;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t m = __ballot_sync(of::kFullMask, (exm >> e) & 1u);
        if (lane == (unsigned)e) word = m;
      }
      if (lane < 4) flags[(q >> 5) * 4 + lane] = word;
    }
  }
  if (i < n_chunks) {  // a copy did not land: record it, drain what is in flight, give up
    if (threadIdx.x == 0) {
      // issued so far: chunks 0 .. kStages-1, then chunk k-1+kStages at each completed iteration k >= 1
      const int issued = i >= 1 ? i - 2 + kStages : kStages - 1;
      const int last = issued < n_chunks - 1 ? issued : n_chunks - 1;
      bool drained = true;
      for (int j = i; j <= last; ++j)
        drained &= of::mbar_wait(of::smem_u32(full + j % kStages), (uint32_t)(j / kStages) & 1u, kWaitLimitNs);
      // bit 0: a copy timed out; bit 1: the drain timed out too, so copies
      // may still land in shared memory the block no longer owns
      atomicOr(B.status, drained ? 1u : 3u);
    }
    __syncthreads();
    return;
  }
  if (TRACK && P.have_beta) record_exercise(B, c, t + 1, PUT, n_ex, (double)ext);  // block-uniform condition
  if (!P.ex_now) return;
  if (DEG == 3) {
    flush();
#pragma unroll
    for (int k = 0; k < 10; ++k) mom[k + 1] = (threadIdx.x & 31u) == 0 ? wm[k] : 0.0;
  }
  mom[0] = (double)n_itm;
  block_moments<nm>(B, c, t, mom, red_sh, mom_sh);
}

template <int DEG>
// Launched with programmatic stream serialisation: the next date's pass may
// be scheduled while this one finishes (its last blocks reduce the moments
// and solve for the betas).  It issues its first path-column copies at once
// and waits (griddepcontrol.wait, in the body) for this grid to complete and
// its writes (betas, cash flows, flag rows) to be visible before it reads any.
__global__ void __launch_bounds__(kPassThreads, 4) lsm_pass_f32(const __grid_constant__ LsmBatch B, int t) {
  __shared__ __align__(128) float ring[kStages * 3 * kPathsPerBlock];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ double red_sh[kPassThreads];
  __shared__ double mom_sh[kMaxMoments];
  __shared__ double warp_mom[kPassThreads / 32 * 10];
  // griddepcontrol.wait is in the body, after the loads that do not depend on
  // the previous pass
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const bool put = B.c[blockIdx.y].put;
  if (B.track) {
    if (put) lsm_pass_f32_body<DEG, true, true>(B, t, ring, full, red_sh, mom_sh, warp_mom);
    else lsm_pass_f32_body<DEG, false, true>(B, t, ring, full, red_sh, mom_sh, warp_mom);
  } else {
    if (put) lsm_pass_f32_body<DEG, true, false>(B, t, ring, full, red_sh, mom_sh, warp_mom);
    else lsm_pass_f32_body<DEG, false, false>(B, t, ring, full, red_sh, mom_sh, warp_mom);
  }
}

// 32 x 32 bit transpose across a warp: lane i holds row i on entry and column
// i on exit (bit j of the result = bit i of lane j's row).  Recursive block
// swap with one shuffle per level (the transpose32 recurrence of Hacker's
// Delight, 2nd ed., section 7-3, with the rows spread over the lanes).
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, unsigned lane) {
  uint32_t m = 0x0000FFFFu;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1, m ^= m << s) {
    const uint32_t y = __shfl_xor_sync(of::kFullMask, x, s);
    x = (lane & (unsigned)s) ? ((x & ~m) | ((y & ~m) >> s)) : ((x & m) | ((y & m) << s));
  }
  return x;
}

// Payment steps of the calling lane's quad q (FP32 mode): the first date in
// [2, steps-1] whose exercise flag is set, else `steps` (paid at expiry).  The
// lanes of a warp hold quads 32g .. 32g+31, i.e. the 16 bytes 4g .. 4g+3 of
// each flag row.  Lane j loads those 16 bytes of row d0+j, so one load covers
// 32 dates; a bit transpose per word then gives lane L, for each of its four
// paths, the dates of the 32 at which it was flagged, and the first is a
// find-first-set.  Stops when every path of the warp has its date.  All 32
// lanes call it.
__device__ __forceinline__ void first_exercise_dates(const LsmBatch& B, int c, int64_t q, int tp[4]) {
  const size_t row4 = (size_t)(B.npad / 128);  // uint4 per flag row
  const uint4* col = reinterpret_cast<const uint4*>(B.exflags) + (size_t)c * (B.steps + 1) * row4 + (size_t)(q >> 5);
  const unsigned lane = threadIdx.x & 31u;  // == q & 31
  unsigned todo = 0xFu;
#pragma unroll
  for (int e = 0; e < 4; ++e) tp[e] = B.steps;
  for (int d0 = 2; d0 < B.steps; d0 += 32) {
    if (!__any_sync(of::kFullMask, todo != 0u)) break;
    const int d = d0 + (int)lane;
    const uint4 w = d < B.steps ? __ldg(col + (size_t)d * row4) : make_uint4(0u, 0u, 0u, 0u);
    const uint32_t words[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const uint32_t dates = warp_transpose32(words[e], lane);  // bit j: path e flagged at date d0+j
      if (((todo >> e) & 1u) && dates) {
        tp[e] = d0 + __ffs((int)dates) - 1;
        todo &= ~(1u << e);
      }
    }
  }
}

// Exercise at date 1, final discount, price/stderr/delta sums
// (longstaff_schwartz.rs:604-605, mean_and_stderr :125-140).
template <typename T>
__global__ void __launch_bounds__(kPassThreads) lsm_final(LsmBatch B) {
  __shared__ double red_sh[kPassThreads];
  __shared__ double mom_sh[kMaxMoments];
  __shared__ bool is_last;
  const int c = blockIdx.y;
  const LsmC C = B.c[c];
  const T* S = (const T*)B.S + (size_t)c * B.steps * B.npad;
  const T* V = (const T*)B.V + (size_t)c * B.npad;
  const LsmStep* st = B.st + (size_t)c * (B.steps + 1);
  const bool ex1 = (1 < B.steps) && B.can_ex[(size_t)c * (B.steps + 1) + 1];
  const int nb = 1 & 1;
  const bool have_beta = ex1 && B.beta_ok[(size_t)nb * B.nc + c];
  double beta[4] = {0, 0, 0, 0};
  if (have_beta)
    for (int k = 0; k < 4; ++k) beta[k] = B.betas[((size_t)nb * B.nc + c) * 4 + k];
  double acc[3] = {0, 0, 0};
  const LsmStep& st1 = B.st[(size_t)c * (B.steps + 1) + 1];
  unsigned n_ex = 0;
  double ext = C.put ? 0.0 : __longlong_as_double(0x7FF0000000000000LL);
  // v: the path's cash flow discounted to date 1; s1: its spot at date 1;
  // tp: the step its cash flow is paid at
  auto path_final = [&](double v, double s1, int tp) {
    if (have_beta) {
      const double ex = intrinsic_v<double>(C.put, s1, st1.strike);
      if (ex > 0.0 && ex > continuation(B.degree, beta, s1, st1.inv_strike, sizeof(T) == 4 ? 1.0 : 0.0)) {
        v = ex;
        tp = 1;
        ++n_ex;
        ext = C.put ? fmax(ext, s1) : fmin(ext, s1);
      }
    }
    v *= C.disc;
    // Pathwise delta under the fitted policy: the cash flow E paid at step tp
    // is now v = E disc^tp with S_tp = K_tp -/+ E, so dv = +-S_tp disc^tp / S0
    // = +-(K_tp disc^tp -/+ v) / S0 (put / call); no cash flow, no delta.
    double dv = 0.0;
    if (B.want_delta && v > 0.0) {
      const double D = B.disc_pow[(size_t)c * (B.steps + 1) + tp];
      const double K = st[tp].strike;
      dv = C.put ? -(K * D - v) * C.inv_spot : (K * D + v) * C.inv_spot;
    }
    acc[0] += v;
    acc[1] += v * v;
    acc[2] += dv;
  };
  if constexpr (sizeof(T) == 4) {
    // FP32 store: four consecutive paths per thread (padding paths carry
    // V = 0 and an out-of-the-money spot); payment steps from the flag rows
    const int64_t q = (int64_t)blockIdx.x * kPassThreads + threadIdx.x;
    const float4 v4 = reinterpret_cast<const float4*>(V)[q];
    const float4 s4 = have_beta ? reinterpret_cast<const float4*>(S)[q] : make_float4(0.f, 0.f, 0.f, 0.f);
    int tp[4] = {0, 0, 0, 0};
    if (B.want_delta) first_exercise_dates(B, c, q, tp);
    path_final(v4.x, s4.x, tp[0]);
    path_final(v4.y, s4.y, tp[1]);
    path_final(v4.z, s4.z, tp[2]);
    path_final(v4.w, s4.w, tp[3]);
  } else {
    const int32_t* tau = B.tau + (size_t)c * B.npad;
    const int64_t base = (int64_t)blockIdx.x * kPathsPerBlock;
    for (int q = 0; q < kPathsPerThread; ++q) {
      const int64_t p = base + q * kPassThreads + threadIdx.x;
      if (p >= B.n) break;
      path_final((double)V[p], have_beta ? (double)S[p] : 0.0, B.want_delta ? tau[p] : 0);
    }
  }
  if (B.track && have_beta) record_exercise(B, c, 1, C.put, n_ex, ext);  // block-uniform condition
  double* part = B.partials + ((size_t)c * B.blocks + blockIdx.x) * kMaxMoments;
  for (int k = 0; k < 3; ++k) {
    double w = of::warp_sum(acc[k]);
    if ((threadIdx.x & 31) == 0) red_sh[threadIdx.x >> 5] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0;
      for (int i = 0; i < kPassThreads / 32; ++i) a += red_sh[i];
      part[k] = a;
    }
    __syncthreads();
  }
  __threadfence();
  if (threadIdx.x == 0) {
    const uint32_t done = atomicAdd(B.counters + c, 1u);
    is_last = done == (uint32_t)B.blocks - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  const double* pp = B.partials + (size_t)c * B.blocks * kMaxMoments;
  for (int k = 0; k < 3; ++k) {
    double a = 0.0;
    for (int b = threadIdx.x; b < B.blocks; b += blockDim.x) a += pp[(size_t)b * kMaxMoments + k];
    red_sh[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s) red_sh[threadIdx.x] += red_sh[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) mom_sh[k] = red_sh[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double n = (double)B.n;
    const double mean = mom_sh[0] / n;
    const double var = B.n > 1 ? (mom_sh[1] - mom_sh[0] * mom_sh[0] / n) / (n - 1.0) : 0.0;
    B.results[c * 3 + 0] = mean;
    B.results[c * 3 + 1] = sqrt(var / n);
    B.results[c * 3 + 2] = mom_sh[2] / n;
    B.counters[c] = 0;
  }
}

}  // namespace

static of_status lsm_validate(of_ctx* ctx, const of_lsm_contract* k, int64_t paths) {
  if (k->option_type != OF_CALL && k->option_type != OF_PUT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown option type %d", k->option_type);
  if (!(k->strike > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "vanilla strike must be > 0");
  if (!(k->expiry >= 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "vanilla expiry must be >= 0");
  if (k->exercise == OF_EXERCISE_BERMUDAN) {
    if (k->n_exercise_dates <= 0 || !k->exercise_dates)
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "bermudan exercise dates cannot be empty");
    for (int64_t d = 0; d < k->n_exercise_dates; ++d)
      if (k->exercise_dates[d] <= 0.0 || k->exercise_dates[d] > k->expiry)
        return of_fail(ctx, OF_ERR_INVALID_INPUT, "bermudan exercise dates must lie in (0, expiry]");
  } else if (k->exercise != OF_EXERCISE_EUROPEAN && k->exercise != OF_EXERCISE_AMERICAN) {
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown exercise style %d", k->exercise);
  }
  if (k->num_steps < 2) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps must be >= 2 for Longstaff-Schwartz");
  if (k->num_steps > (1 << 20)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps too large");
  if (paths < 3) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths must be >= 3 for Longstaff-Schwartz");
  if (k->expiry > 0.0 && !(k->vol > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "market volatility must be > 0");
  if (!(k->spot > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "market spot must be > 0");
  return OF_OK;
}

static of_status upload_jump_tables(of_ctx* ctx, const uint64_t** out) {
  const std::vector<uint64_t>& t = jump_tables();
  const size_t bytes = t.size() * sizeof(uint64_t);
  const bool fresh = ctx->slot_bytes[SLOT_JUMP] < bytes;
  void* d = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_JUMP, bytes, &d));
  if (fresh) OF_CUDA_TRY(ctx, cudaMemcpy(d, t.data(), bytes, cudaMemcpyHostToDevice));
  *out = (const uint64_t*)d;
  return OF_OK;
}

extern "C" of_status of_xoshiro_jump(of_ctx* ctx, uint64_t seed, const uint64_t* draws, int64_t n,
                                     uint64_t* states_out) {
  if (!ctx || !draws || !states_out || n <= 0) return OF_ERR_INVALID_INPUT;
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const uint64_t* tab = nullptr;
  OF_TRY(upload_jump_tables(ctx, &tab));
  void *d_in = nullptr, *d_out = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_MISC, (size_t)n * 5 * sizeof(uint64_t), &d_in));
  d_out = (uint64_t*)d_in + n;
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(d_in, draws, (size_t)n * sizeof(uint64_t), cudaMemcpyHostToDevice, ctx->stream));
  jump_test_kernel<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(seed, (const uint64_t*)d_in, n, tab,
                                                                       (uint64_t*)d_out);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(states_out, d_out, (size_t)n * 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                   ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return OF_OK;
}

namespace {

// Host description of one contract of a batch.
struct LsmHost {
  LsmC C{};                              // device grid pointers are set by lsm_run_batch
  std::vector<uint8_t> can;              // [steps+1] exercise allowed at step t
  std::vector<LsmStep> st;               // [steps+1]
  std::vector<double> lv_k, lv_t, lv_v;  // sampled local-vol grid (local-vol dynamics only)
};

// Exercise-boundary statistics of one contract, [steps+1] entries each.
struct LsmTrack {
  std::vector<unsigned long long> ex_count, ex_bits;
  std::vector<double> itm;
  unsigned long long term_itm = 0;
};

// SampledVolSurface::locate_bounds (src/market/market.rs:104-125).
void locate_bounds(const std::vector<double>& g, double x, int32_t* lo, int32_t* hi, double* w) {
  const int n = (int)g.size();
  if (x <= g[0]) {
    *lo = *hi = 0;
    *w = 0.0;
    return;
  }
  if (x >= g[(size_t)n - 1]) {
    *lo = *hi = n - 1;
    *w = 0.0;
    return;
  }
  int l = 0;
  for (int i = 0; i < n - 1; ++i)
    if (x >= g[(size_t)i] && x <= g[(size_t)i + 1]) {
      l = i;
      break;
    }
  *lo = l;
  *hi = l + 1;
  *w = (x - g[(size_t)l]) / (g[(size_t)l + 1] - g[(size_t)l]);
}

// Per-step strikes and local-vol expiry brackets of a contract.
void fill_steps(LsmHost& h, int64_t steps, double expiry, const double* strike_of_step) {
  h.st.assign((size_t)steps + 1, LsmStep{});
  const double dt = expiry / (double)steps;
  for (int64_t t = 0; t <= steps; ++t) {
    LsmStep& s = h.st[(size_t)t];
    s.strike = strike_of_step[t];
    s.inv_strike = 1.0 / s.strike;
    s.fstrike = (float)s.strike;
    s.finv_strike = (float)s.inv_strike;
    if (!h.lv_t.empty()) {
      const double te = (double)t * dt > 1.0e-8 ? (double)t * dt : 1.0e-8;  // longstaff_schwartz.rs:224
      locate_bounds(h.lv_t, te > h.lv_t[0] ? te : h.lv_t[0], &s.e0, &s.e1, &s.ew);
      s.few = (float)s.ew;
    }
  }
}

// Offsets of a run's tables in its auxiliary device block.
struct DevOffsets {
  size_t part = 0, beta = 0, res = 0, c = 0, ok = 0, reg = 0, cnt = 0, can = 0, st = 0, exc = 0, exb = 0, itm = 0,
         term = 0, dpow = 0, status = 0;
};

// One batch of contracts sharing a step count, staged for an asynchronous
// run on one of two device buffer sets: pinned host images of its tables
// (uploaded when enqueued) and of its results (read back when enqueued, used
// once the streams have drained).
struct LsmRun {
  std::vector<LsmHost> hs;
  int64_t steps = 0;
  uint32_t contract_base = 0;
  const double* inj_host = nullptr;  // injected normals (FP64 test hook), or null
  int draws = 1;
  bool track = false;
  std::vector<int64_t> index;  // the caller's contract of each batch slot (of_lsm_price)
  LsmBatch B{};
  DevOffsets dev;
  void* d_inj = nullptr;
  char* pin = nullptr;  // pinned staging, laid out by the o_* offsets
  size_t o_hc = 0, o_can = 0, o_st = 0, o_dpow = 0, o_bits0 = 0, o_res = 0, o_reg = 0, o_status = 0, o_cnt = 0,
         o_bits = 0, o_itm = 0, o_term = 0;
  std::vector<size_t> o_lvh;  // [nc][4] staging offsets of the local-vol arrays
  std::vector<size_t> o_lvd;  // [nc][4] their offsets in the auxiliary device block
  size_t aux_bytes = 0, path_bytes = 0, value_bytes = 0;
  cudaEvent_t gen_done = nullptr, done = nullptr;
  LsmRun() = default;
  LsmRun(const LsmRun&) = delete;
  LsmRun& operator=(const LsmRun&) = delete;
  ~LsmRun() {
    if (pin) cudaFreeHost(pin);
    if (gen_done) cudaEventDestroy(gen_done);
    if (done) cudaEventDestroy(done);
  }
  int nc() const { return (int)hs.size(); }
  size_t ns() const { return (size_t)nc() * (size_t)(steps + 1); }
};

// Sizes of a run's device buffers, the layout of its auxiliary block and the
// scalar fields of its LsmBatch.
void lsm_layout(LsmRun& r, const of_lsm_config* cfg) {
  const bool fp64 = cfg->precision == OF_PREC_FP64_REFERENCE;
  const int64_t N = cfg->num_paths;
  const size_t esz = fp64 ? sizeof(double) : sizeof(float);
  const int64_t npad = (N + kPathsPerBlock - 1) / kPathsPerBlock * kPathsPerBlock;
  const int blocks = (int)(npad / kPathsPerBlock);
  const int nc = r.nc();
  const size_t ns = r.ns();
  r.path_bytes = (size_t)nc * (size_t)r.steps * npad * esz;
  // after the cash flows: payment steps (FP64 mode) or the per-date exercise
  // flag rows (FP32 mode), for the delta
  const size_t aux_values = fp64 ? (size_t)nc * npad * sizeof(int32_t)
                                 : (size_t)nc * (size_t)(r.steps + 1) * (size_t)(npad / 32) * sizeof(uint32_t);
  r.value_bytes = (size_t)nc * npad * esz + aux_values;
  size_t off = 0;
  auto take = [&off](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) & ~(size_t)255;
    return o;
  };
  DevOffsets& d = r.dev;
  d.part = take((size_t)nc * blocks * kMaxMoments * sizeof(double));
  d.beta = take((size_t)nc * 8 * sizeof(double));
  d.res = take((size_t)nc * 3 * sizeof(double));
  d.c = take((size_t)nc * sizeof(LsmC));
  d.ok = take((size_t)nc * 2 * sizeof(int32_t));
  d.reg = take((size_t)nc * sizeof(int32_t));
  d.cnt = take((size_t)nc * sizeof(uint32_t));
  d.can = take(ns);
  d.st = take(ns * sizeof(LsmStep));
  d.exc = take(ns * sizeof(unsigned long long));
  d.exb = take(ns * sizeof(unsigned long long));
  d.itm = take(ns * sizeof(double));
  d.term = take((size_t)nc * sizeof(unsigned long long));
  d.dpow = take(ns * sizeof(double));
  d.status = take(sizeof(uint32_t));
  r.o_lvd.assign((size_t)nc * 4, 0);
  for (int c = 0; c < nc; ++c) {
    const size_t nk = r.hs[(size_t)c].lv_k.size(), nv = r.hs[(size_t)c].lv_v.size();
    if (!nk) continue;
    r.o_lvd[(size_t)c * 4 + 0] = take(nk * sizeof(double));
    r.o_lvd[(size_t)c * 4 + 1] = take(nv * sizeof(double));
    r.o_lvd[(size_t)c * 4 + 2] = take(nk * sizeof(float));
    r.o_lvd[(size_t)c * 4 + 3] = take(nv * sizeof(float));
  }
  r.aux_bytes = off;
  LsmBatch& B = r.B;
  B.nc = nc;
  B.steps = (int32_t)r.steps;
  B.n = N;
  B.npad = npad;
  B.blocks = blocks;
  B.degree = cfg->basis_degree;
  B.want_delta = cfg->want_delta;
  B.track = r.track ? 1 : 0;
  B.seed = cfg->seed;
  B.keys = of::philox_keys(cfg->seed);
  B.contract_base = r.contract_base;
  B.chunk = 8;
}

// Points a laid-out run at its device buffers, fills its pinned staging and
// creates its events.
of_status lsm_bind(of_ctx* ctx, LsmRun& r, const of_lsm_config* cfg, void* dS, void* dVal, void* dAux,
                   const uint64_t* jump) {
  const bool fp64 = cfg->precision == OF_PREC_FP64_REFERENCE;
  const size_t esz = fp64 ? sizeof(double) : sizeof(float);
  const int nc = r.nc();
  const size_t ns = r.ns();
  const int dyn = r.hs[0].C.dynamics;
  for (const LsmHost& h : r.hs)
    if (h.C.dynamics != dyn) return of_fail(ctx, OF_ERR_INVALID_INPUT, "an LSM batch mixes path dynamics");
  LsmBatch& B = r.B;
  char* a = (char*)dAux;
  const DevOffsets& d = r.dev;
  B.partials = (double*)(a + d.part);
  B.betas = (double*)(a + d.beta);
  B.results = (double*)(a + d.res);
  B.c = (const LsmC*)(a + d.c);
  B.beta_ok = (int32_t*)(a + d.ok);
  B.regress_count = (int32_t*)(a + d.reg);
  B.counters = (uint32_t*)(a + d.cnt);
  B.can_ex = (const uint8_t*)(a + d.can);
  B.st = (const LsmStep*)(a + d.st);
  B.ex_count = (unsigned long long*)(a + d.exc);
  B.ex_bits = (unsigned long long*)(a + d.exb);
  B.itm_count = (double*)(a + d.itm);
  B.term_itm = (unsigned long long*)(a + d.term);
  B.disc_pow = (const double*)(a + d.dpow);
  B.status = (uint32_t*)(a + d.status);
  B.S = dS;
  B.V = dVal;
  B.tau = fp64 ? (int32_t*)((char*)dVal + (size_t)nc * B.npad * esz) : nullptr;
  B.exflags = fp64 ? nullptr : (uint32_t*)((char*)dVal + (size_t)nc * B.npad * esz);
  B.jump = jump;
  size_t off = 0;
  auto take = [&off](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 15) & ~(size_t)15;
    return o;
  };
  r.o_hc = take((size_t)nc * sizeof(LsmC));
  r.o_can = take(ns);
  r.o_st = take(ns * sizeof(LsmStep));
  r.o_dpow = take(ns * sizeof(double));
  r.o_bits0 = take(r.track ? ns * sizeof(unsigned long long) : 0);
  r.o_lvh.assign((size_t)nc * 4, 0);
  for (int c = 0; c < nc; ++c) {
    const size_t nk = r.hs[(size_t)c].lv_k.size(), nv = r.hs[(size_t)c].lv_v.size();
    if (!nk) continue;
    r.o_lvh[(size_t)c * 4 + 0] = take(nk * sizeof(double));
    r.o_lvh[(size_t)c * 4 + 1] = take(nv * sizeof(double));
    r.o_lvh[(size_t)c * 4 + 2] = take(nk * sizeof(float));
    r.o_lvh[(size_t)c * 4 + 3] = take(nv * sizeof(float));
  }
  r.o_res = take((size_t)nc * 3 * sizeof(double));
  r.o_reg = take((size_t)nc * sizeof(int32_t));
  r.o_status = take(sizeof(uint32_t));
  r.o_cnt = take(r.track ? ns * sizeof(unsigned long long) : 0);
  r.o_bits = take(r.track ? ns * sizeof(unsigned long long) : 0);
  r.o_itm = take(r.track ? ns * sizeof(double) : 0);
  r.o_term = take(r.track ? (size_t)nc * sizeof(unsigned long long) : 0);
  if (cudaMallocHost(&r.pin, off) != cudaSuccess) {
    r.pin = nullptr;
    return of_fail(ctx, OF_ERR_ALLOC, "LSM staging allocation failed");
  }
  LsmC* hc = (LsmC*)(r.pin + r.o_hc);
  uint8_t* can = (uint8_t*)(r.pin + r.o_can);
  LsmStep* st = (LsmStep*)(r.pin + r.o_st);
  double* dpow = (double*)(r.pin + r.o_dpow);
  for (int c = 0; c < nc; ++c) {
    const LsmHost& h = r.hs[(size_t)c];
    LsmC C = h.C;
    // the stream follows the contract, not its batch slot, so that the draws
    // do not depend on how the contracts were batched
    C.cid = r.index.empty() ? r.contract_base + (uint32_t)c : (uint32_t)r.index[(size_t)c];
    std::copy(h.can.begin(), h.can.end(), can + (size_t)c * (r.steps + 1));
    std::copy(h.st.begin(), h.st.end(), st + (size_t)c * (r.steps + 1));
    double* dp = dpow + (size_t)c * (r.steps + 1);
    dp[0] = 1.0;
    for (int64_t k = 1; k <= r.steps; ++k) dp[k] = dp[k - 1] * h.C.disc;
    if (!h.lv_k.empty()) {
      C.lv_k = (const double*)(a + r.o_lvd[(size_t)c * 4 + 0]);
      C.lv_v = (const double*)(a + r.o_lvd[(size_t)c * 4 + 1]);
      C.lv_kf = (const float*)(a + r.o_lvd[(size_t)c * 4 + 2]);
      C.lv_vf = (const float*)(a + r.o_lvd[(size_t)c * 4 + 3]);
      C.lv_nk = (int32_t)h.lv_k.size();
      std::copy(h.lv_k.begin(), h.lv_k.end(), (double*)(r.pin + r.o_lvh[(size_t)c * 4 + 0]));
      std::copy(h.lv_v.begin(), h.lv_v.end(), (double*)(r.pin + r.o_lvh[(size_t)c * 4 + 1]));
      std::copy(h.lv_k.begin(), h.lv_k.end(), (float*)(r.pin + r.o_lvh[(size_t)c * 4 + 2]));
      std::copy(h.lv_v.begin(), h.lv_v.end(), (float*)(r.pin + r.o_lvh[(size_t)c * 4 + 3]));
    }
    hc[c] = C;
  }
  if (r.track) {
    unsigned long long* bits0 = (unsigned long long*)(r.pin + r.o_bits0);
    for (int c = 0; c < nc; ++c)  // identity of max (put) / min (call) over positive doubles
      std::fill(bits0 + (size_t)c * (r.steps + 1), bits0 + (size_t)(c + 1) * (r.steps + 1),
                r.hs[(size_t)c].C.put ? 0ULL : 0x7FF0000000000000ULL);
  }
  if (cudaEventCreateWithFlags(&r.gen_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming) != cudaSuccess)
    return of_fail(ctx, OF_ERR_CUDA, "LSM event creation failed");
  return OF_OK;
}

// Enqueues a bound run: its tables, the path generation and the `gen_done`
// event on `gs`; on `ms`, after `gen_done`, the passes, the final kernel, the
// readback of the results into the pinned staging and the `done` event.
of_status lsm_enqueue(of_ctx* ctx, LsmRun& r, const of_lsm_config* cfg, cudaStream_t gs, cudaStream_t ms) {
  const bool fp64 = cfg->precision == OF_PREC_FP64_REFERENCE;
  const int nc = r.nc();
  const size_t ns = r.ns();
  LsmBatch& B = r.B;
  OF_CUDA_TRY(ctx, cudaMemcpyAsync((void*)B.c, r.pin + r.o_hc, (size_t)nc * sizeof(LsmC), cudaMemcpyHostToDevice, gs));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync((void*)B.can_ex, r.pin + r.o_can, ns, cudaMemcpyHostToDevice, gs));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync((void*)B.st, r.pin + r.o_st, ns * sizeof(LsmStep), cudaMemcpyHostToDevice, gs));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync((void*)B.disc_pow, r.pin + r.o_dpow, ns * sizeof(double), cudaMemcpyHostToDevice,
                                   gs));
  const LsmC* hc = (const LsmC*)(r.pin + r.o_hc);
  for (int c = 0; c < nc; ++c) {
    const LsmHost& h = r.hs[(size_t)c];
    if (h.lv_k.empty()) continue;
    const size_t nk = h.lv_k.size(), nv = h.lv_v.size();
    OF_CUDA_TRY(ctx, cudaMemcpyAsync((void*)hc[c].lv_k, r.pin + r.o_lvh[(size_t)c * 4 + 0], nk * sizeof(double),
                                     cudaMemcpyHostToDevice, gs));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync((void*)hc[c].lv_v, r.pin + r.o_lvh[(size_t)c * 4 + 1], nv * sizeof(double),
                                     cudaMemcpyHostToDevice, gs));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync((void*)hc[c].lv_kf, r.pin + r.o_lvh[(size_t)c * 4 + 2], nk * sizeof(float),
                                     cudaMemcpyHostToDevice, gs));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync((void*)hc[c].lv_vf, r.pin + r.o_lvh[(size_t)c * 4 + 3], nv * sizeof(float),
                                     cudaMemcpyHostToDevice, gs));
  }
  OF_CUDA_TRY(ctx, cudaMemsetAsync(B.beta_ok, 0, (size_t)nc * 2 * sizeof(int32_t), gs));
  OF_CUDA_TRY(ctx, cudaMemsetAsync(B.regress_count, 0, (size_t)nc * sizeof(int32_t), gs));
  OF_CUDA_TRY(ctx, cudaMemsetAsync(B.counters, 0, (size_t)nc * sizeof(uint32_t), gs));
  OF_CUDA_TRY(ctx, cudaMemsetAsync(B.status, 0, sizeof(uint32_t), gs));
  if (r.track) {
    OF_CUDA_TRY(ctx, cudaMemsetAsync(B.ex_count, 0, ns * sizeof(unsigned long long), gs));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(B.ex_bits, r.pin + r.o_bits0, ns * sizeof(unsigned long long),
                                     cudaMemcpyHostToDevice, gs));
    OF_CUDA_TRY(ctx, cudaMemsetAsync(B.itm_count, 0, ns * sizeof(double), gs));
    OF_CUDA_TRY(ctx, cudaMemsetAsync(B.term_itm, 0, (size_t)nc * sizeof(unsigned long long), gs));
  }
  if (r.inj_host) {
    const size_t cnt = (size_t)B.n * r.steps * r.draws;
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(r.d_inj, r.inj_host, cnt * sizeof(double), cudaMemcpyHostToDevice, gs));
    B.inj = (const double*)r.d_inj;
  }
  if (fp64) {
    const int64_t chunks = (B.n + B.chunk - 1) / B.chunk;
    lsm_gen_ref<<<dim3((unsigned)((chunks + 127) / 128), nc), 128, 0, gs>>>(B);
  } else {
    const int64_t quads = B.npad / 4;
    const int dyn = r.hs[0].C.dynamics;
    void (*gen)(LsmBatch) = dyn == DYN_HESTON ? lsm_gen_philox<DYN_HESTON>
                            : dyn == DYN_LOCAL_VOL ? lsm_gen_philox<DYN_LOCAL_VOL> : lsm_gen_philox<DYN_GBM>;
    gen<<<dim3((unsigned)((quads + 255) / 256), nc), 256, 0, gs>>>(B);
  }
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_CUDA_TRY(ctx, cudaEventRecord(r.gen_done, gs));
  OF_CUDA_TRY(ctx, cudaStreamWaitEvent(ms, r.gen_done, 0));
  // The passes: one wave of resident blocks over the whole batch, each block
  // striding over its contract's chunks.
  void (*pass)(LsmBatch, int) = fp64 ? (B.degree == 2 ? lsm_pass<double, 2> : lsm_pass<double, 3>)
                                     : (B.degree == 2 ? lsm_pass_f32<2> : lsm_pass_f32<3>);
  const int bps = std::max(1, of_blocks_per_sm((const void*)pass, kPassThreads, 0));
  const int64_t wave = (int64_t)ctx->sm_count * bps;
  // Blocks per contract: floor(k wave / nc) fills exactly k waves up to the
  // rounding; take the smallest k whose waves are at least 95% occupied (a
  // grid a few blocks over a wave would run those blocks as a second wave).
  int64_t pass_blocks = 1;
  double best = 0.0;
  for (int k = 1; k <= 8; ++k) {
    const int64_t bpc = std::max<int64_t>(1, std::min<int64_t>(B.blocks, k * wave / nc));
    const int64_t total = bpc * nc, waves = (total + wave - 1) / wave;
    const double fill = (double)total / (double)(waves * wave);
    if (fill > best + 1e-9) {
      best = fill;
      pass_blocks = bpc;
    }
    if (fill >= 0.95 || bpc == B.blocks) break;
  }
  const dim3 pgrid((unsigned)pass_blocks, nc);
  if (fp64) {
    for (int t = (int)r.steps - 1; t >= 1; --t) pass<<<pgrid, kPassThreads, 0, ms>>>(B, t);
  } else {
    // FP32 passes: programmatic dependent launches (lsm_pass_f32 waits on its
    // predecessor grid before reading anything it wrote)
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = pgrid;
    lc.blockDim = dim3(kPassThreads);
    lc.dynamicSmemBytes = 0;
    lc.stream = ms;
    lc.attrs = at;
    lc.numAttrs = 1;
    for (int t = (int)r.steps - 1; t >= 1; --t) OF_CUDA_TRY(ctx, cudaLaunchKernelEx(&lc, pass, B, t));
  }
  const dim3 grid((unsigned)B.blocks, nc);
  if (fp64) lsm_final<double><<<grid, kPassThreads, 0, ms>>>(B);
  else lsm_final<float><<<grid, kPassThreads, 0, ms>>>(B);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(r.pin + r.o_res, B.results, (size_t)nc * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                   ms));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(r.pin + r.o_reg, B.regress_count, (size_t)nc * sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, ms));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(r.pin + r.o_status, B.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ms));
  if (r.track) {
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(r.pin + r.o_cnt, B.ex_count, ns * 8, cudaMemcpyDeviceToHost, ms));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(r.pin + r.o_bits, B.ex_bits, ns * 8, cudaMemcpyDeviceToHost, ms));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(r.pin + r.o_itm, B.itm_count, ns * 8, cudaMemcpyDeviceToHost, ms));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(r.pin + r.o_term, B.term_itm, (size_t)nc * 8, cudaMemcpyDeviceToHost, ms));
  }
  OF_CUDA_TRY(ctx, cudaEventRecord(r.done, ms));
  return OF_OK;
}

// Results of a run whose streams have drained: {price, stderr, delta} per
// contract, the regression counts and, when tracked, the boundary statistics.
of_status lsm_collect(of_ctx* ctx, const LsmRun& r, std::vector<double>& results, std::vector<int32_t>& regs,
                      std::vector<LsmTrack>* track) {
  const int nc = r.nc();
  const uint32_t status = *(const uint32_t*)(r.pin + r.o_status);
  if (status & 2u) {
    ctx->unusable = true;
    return of_fail(ctx, OF_ERR_TIMEOUT,
                   "LSM pass: a bulk copy into shared memory did not complete in time and could not be drained; "
                   "the context is unusable: destroy it and create a new one");
  }
  if (status)
    return of_fail(ctx, OF_ERR_TIMEOUT, "LSM pass: a bulk copy into shared memory did not complete in time");
  const double* hres = (const double*)(r.pin + r.o_res);
  const int32_t* hreg = (const int32_t*)(r.pin + r.o_reg);
  results.assign(hres, hres + (size_t)nc * 3);
  regs.assign(hreg, hreg + nc);
  if (track && r.track) {
    const unsigned long long* hcnt = (const unsigned long long*)(r.pin + r.o_cnt);
    const unsigned long long* hbits = (const unsigned long long*)(r.pin + r.o_bits);
    const double* hitm = (const double*)(r.pin + r.o_itm);
    const unsigned long long* hterm = (const unsigned long long*)(r.pin + r.o_term);
    track->assign((size_t)nc, LsmTrack{});
    for (int c = 0; c < nc; ++c) {
      LsmTrack& tr = (*track)[(size_t)c];
      const size_t b = (size_t)c * (r.steps + 1), e = b + (size_t)r.steps + 1;
      tr.ex_count.assign(hcnt + b, hcnt + e);
      tr.ex_bits.assign(hbits + b, hbits + e);
      tr.itm.assign(hitm + b, hitm + e);
      tr.term_itm = hterm[c];
    }
  }
  return OF_OK;
}

// The context's lowest-priority stream, created on first use.
of_status lsm_side_stream(of_ctx* ctx, cudaStream_t* out) {
  if (!ctx->side_stream) {
    int least = 0, greatest = 0;
    OF_CUDA_TRY(ctx, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    OF_CUDA_TRY(ctx, cudaStreamCreateWithPriority(&ctx->side_stream, cudaStreamNonBlocking, least));
  }
  *out = ctx->side_stream;
  return OF_OK;
}

// Generation, the backward passes and the final reduction for contracts that
// share a step count, run synchronously on the context stream and buffer set
// 0; results[c] = {price, stderr, delta}.
of_status lsm_run_batch(of_ctx* ctx, std::vector<LsmHost>& hs, int64_t steps, const of_lsm_config* cfg,
                        const uint64_t* jump, uint32_t contract_base, const double* inj_host, int draws,
                        std::vector<LsmTrack>* track, std::vector<double>& results, std::vector<int32_t>& regs,
                        float* ms_out) {
  LsmRun r;
  r.hs = hs;
  r.steps = steps;
  r.contract_base = contract_base;
  r.inj_host = inj_host;
  r.draws = draws;
  r.track = track != nullptr;
  lsm_layout(r, cfg);
  void *dS = nullptr, *dVal = nullptr, *dAux = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_LSM_PATHS, r.path_bytes, &dS));
  OF_TRY(of_scratch(ctx, SLOT_LSM_VALUES, r.value_bytes, &dVal));
  OF_TRY(of_scratch(ctx, SLOT_LSM_AUX, r.aux_bytes, &dAux));
  if (inj_host)
    OF_TRY(of_scratch(ctx, SLOT_INJECT, (size_t)cfg->num_paths * steps * draws * sizeof(double), &r.d_inj));
  OF_TRY(lsm_bind(ctx, r, cfg, dS, dVal, dAux, jump));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  const of_status st = lsm_enqueue(ctx, r, cfg, ctx->stream, ctx->stream);
  if (st == OF_OK) OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  // drain before the staging goes away, error or not
  const cudaError_t e = cudaStreamSynchronize(ctx->stream);
  OF_TRY(st);
  if (e != cudaSuccess) return of_fail(ctx, OF_ERR_CUDA, "LSM run failed: %s", cudaGetErrorString(e));
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(ms_out, ctx->ev_start, ctx->ev_stop));
  return lsm_collect(ctx, r, results, regs, track);
}

}  // namespace

extern "C" of_status of_lsm_price(of_ctx* ctx, const of_lsm_contract* ks, int64_t n, const of_lsm_config* cfg,
                                  of_lsm_result* res) {
  if (!ctx || !ks || !cfg || !res || n <= 0) return OF_ERR_INVALID_INPUT;
  if (cfg->basis_degree != 2 && cfg->basis_degree != 3)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "basis_degree must be 2 or 3");
  const bool fp64 = cfg->precision == OF_PREC_FP64_REFERENCE;
  if (!fp64 && cfg->precision != OF_PREC_FP32_PHILOX)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown precision %d", cfg->precision);
  if (cfg->injected_normals && !fp64)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "injected normals are a FP64 reference-mode test hook");
  const int64_t N = cfg->num_paths;
  for (int64_t i = 0; i < n; ++i) OF_TRY(lsm_validate(ctx, &ks[i], N));
  if (cfg->injected_normals) {
    int64_t need = 0;
    for (int64_t i = 0; i < n; ++i) need += N * ks[i].num_steps;
    if (cfg->n_injected < need)
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "injected normals: need %lld values, got %lld", (long long)need,
                     (long long)cfg->n_injected);
  }
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::memset(res, 0, sizeof(of_lsm_result) * (size_t)n);
  const uint64_t* jump = nullptr;
  if (fp64 && !cfg->injected_normals) OF_TRY(upload_jump_tables(ctx, &jump));

  const size_t esz = fp64 ? sizeof(double) : sizeof(float);
  const int64_t npad = (N + kPathsPerBlock - 1) / kPathsPerBlock * kPathsPerBlock;
  if (cfg->batch_contracts < 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "batch_contracts must be >= 0");
  // Contracts sharing a step count go through the date loop together, in
  // batches bounded by a path-store budget.
  const size_t budget = (size_t)24 << 30;
  std::vector<int64_t> order((size_t)n);
  for (int64_t i = 0; i < n; ++i) order[(size_t)i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return ks[a].num_steps < ks[b].num_steps; });
  // injected-normal offsets in the caller's contract order
  std::vector<int64_t> inj_off((size_t)n, 0);
  for (int64_t i = 1; i < n; ++i) inj_off[(size_t)i] = inj_off[(size_t)i - 1] + N * ks[i - 1].num_steps;

  std::vector<std::unique_ptr<LsmRun>> runs;
  size_t pos = 0;
  while (pos < order.size()) {
    // trivial contracts (expiry == 0): intrinsic, stderr 0 (longstaff_schwartz.rs:440-447)
    const of_lsm_contract& k0 = ks[order[pos]];
    if (k0.expiry == 0.0) {
      const double v = k0.option_type == OF_CALL ? k0.spot - k0.strike : k0.strike - k0.spot;
      res[order[pos]].price = v > 0.0 ? v : 0.0;
      ++pos;
      continue;
    }
    const int64_t steps = k0.num_steps;
    const size_t per = (size_t)steps * npad * esz;
    size_t cap = std::max<size_t>(1, budget / per);
    if (cfg->batch_contracts > 0) {
      cap = std::min<size_t>(cap, (size_t)cfg->batch_contracts);
    } else {
      // Automatic sizes: the group's contracts in equal batches under the
      // budget, rather than full batches and a small remainder whose passes
      // cost the same launches for little work.  (A small first batch, so
      // that less generation runs before the first passes, measured slower:
      // the passes fill every SM, so the next batch's generation runs in
      // their gaps rather than beside them, and more batches mean more passes.)
      size_t g = 0;
      for (size_t q = pos; q < order.size() && ks[order[q]].num_steps == steps && ks[order[q]].expiry != 0.0; ++q)
        ++g;
      const size_t nb = (g + cap - 1) / cap;
      cap = (g + nb - 1) / nb;
    }
    if (cfg->injected_normals) cap = 1;  // one contract per batch keeps the injected layout simple
    std::vector<int64_t> batch;
    while (pos < order.size() && batch.size() < cap && ks[order[pos]].num_steps == steps &&
           ks[order[pos]].expiry != 0.0)
      batch.push_back(order[pos++]);
    const int nc = (int)batch.size();
    std::vector<LsmHost> hs((size_t)nc);
    for (int c = 0; c < nc; ++c) {
      const of_lsm_contract& k = ks[batch[(size_t)c]];
      LsmHost& h = hs[(size_t)c];
      h.can.assign((size_t)steps + 1, 0);
      const std::vector<double> kk((size_t)steps + 1, k.strike);
      fill_steps(h, steps, k.expiry, kk.data());
      LsmC& C = h.C;
      C.dynamics = DYN_GBM;
      const double dt = k.expiry / (double)steps;
      C.put = k.option_type == OF_PUT;
      C.steps = (int32_t)steps;
      C.spot = k.spot;
      C.strike = k.strike;
      C.inv_strike = 1.0 / k.strike;
      C.inv_spot = 1.0 / k.spot;
      C.drift = (k.rate - k.dividend_yield - 0.5 * k.vol * k.vol) * dt;  // :452
      C.step_vol = k.vol * std::sqrt(dt);
      C.disc = std::exp(-k.rate * dt);
      C.fdrift = (float)C.drift;
      C.fstep_vol = (float)C.step_vol;
      C.fspot = (float)k.spot;
      uint8_t* ce = h.can.data();
      if (k.exercise == OF_EXERCISE_EUROPEAN) {
        ce[steps] = 1;
      } else if (k.exercise == OF_EXERCISE_AMERICAN) {
        for (int64_t t = 1; t <= steps; ++t) ce[t] = 1;
      } else {
        for (int64_t d = 0; d < k.n_exercise_dates; ++d) {
          const double idx = std::round((k.exercise_dates[d] / k.expiry) * (double)steps);
          int64_t i = (std::isnan(idx) || idx <= 0.0) ? 0 : (int64_t)idx;
          ce[i < steps ? i : steps] = 1;
        }
        ce[steps] = 1;
      }
    }
    std::unique_ptr<LsmRun> run(new LsmRun());
    run->hs.swap(hs);
    run->steps = steps;
    run->contract_base = (uint32_t)batch[0];
    run->inj_host = cfg->injected_normals ? cfg->injected_normals + inj_off[(size_t)batch[0]] : nullptr;
    run->index = batch;
    runs.push_back(std::move(run));
  }
  if (runs.empty()) return OF_OK;
  // Two device buffer sets alternate: batch i generates into set i % 2 on the
  // lowest-priority side stream (compute-bound, little HBM traffic) while
  // batch i-1 runs its passes (HBM-bound) on the context stream.  Each set is
  // sized for the largest of its batches before anything is enqueued.
  const int sets = runs.size() > 1 ? 2 : 1;
  const int slots[2][3] = {{SLOT_LSM_PATHS, SLOT_LSM_VALUES, SLOT_LSM_AUX},
                           {SLOT_LSM_PATHS_B, SLOT_LSM_VALUES_B, SLOT_LSM_AUX_B}};
  size_t need[2][3] = {{0, 0, 0}, {0, 0, 0}};
  size_t inj_need = 0;
  for (size_t i = 0; i < runs.size(); ++i) {
    LsmRun& r = *runs[i];
    lsm_layout(r, cfg);
    size_t* nd = need[i % 2];
    nd[0] = std::max(nd[0], r.path_bytes);
    nd[1] = std::max(nd[1], r.value_bytes);
    nd[2] = std::max(nd[2], r.aux_bytes);
    if (r.inj_host) inj_need = std::max(inj_need, (size_t)N * r.steps * sizeof(double));
  }
  void* dbuf[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  for (int s = 0; s < sets; ++s)
    for (int k = 0; k < 3; ++k) OF_TRY(of_scratch(ctx, slots[s][k], need[s][k], &dbuf[s][k]));
  void* d_inj = nullptr;
  if (inj_need) OF_TRY(of_scratch(ctx, SLOT_INJECT, inj_need, &d_inj));  // fed by the side stream, in order
  for (size_t i = 0; i < runs.size(); ++i) {
    runs[i]->d_inj = d_inj;
    const int s = (int)(i % 2);
    OF_TRY(lsm_bind(ctx, *runs[i], cfg, dbuf[s][0], dbuf[s][1], dbuf[s][2], jump));
  }
  const cudaStream_t ms = ctx->stream;
  cudaStream_t gs = ms;
  if (sets == 2) OF_TRY(lsm_side_stream(ctx, &gs));
  of_status st = OF_OK;
  if (cudaEventRecord(ctx->ev_start, ms) != cudaSuccess ||
      (gs != ms && cudaStreamWaitEvent(gs, ctx->ev_start, 0) != cudaSuccess))
    st = of_fail(ctx, OF_ERR_CUDA, "LSM stream set-up failed");
  for (size_t i = 0; i < runs.size() && st == OF_OK; ++i) {
    // set i % 2 was last used by batch i-2: its passes, final kernel and readback
    if (i >= 2 && cudaStreamWaitEvent(gs, runs[i - 2]->done, 0) != cudaSuccess)
      st = of_fail(ctx, OF_ERR_CUDA, "LSM stream wait failed");
    if (st == OF_OK) st = lsm_enqueue(ctx, *runs[i], cfg, gs, ms);
  }
  if (st == OF_OK && cudaEventRecord(ctx->ev_stop, ms) != cudaSuccess)
    st = of_fail(ctx, OF_ERR_CUDA, "LSM stream set-up failed");
  // drain both streams before the staging buffers go away, error or not
  const cudaError_t e1 = cudaStreamSynchronize(ms);
  const cudaError_t e2 = gs != ms ? cudaStreamSynchronize(gs) : cudaSuccess;
  OF_TRY(st);
  if (e1 != cudaSuccess || e2 != cudaSuccess)
    return of_fail(ctx, OF_ERR_CUDA, "LSM run failed: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
  float total_ms = 0.0f;
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(&total_ms, ctx->ev_start, ctx->ev_stop));
  std::vector<double> hres;
  std::vector<int32_t> hreg;
  for (const std::unique_ptr<LsmRun>& run : runs) {
    OF_TRY(lsm_collect(ctx, *run, hres, hreg, nullptr));
    for (int c = 0; c < run->nc(); ++c) {
      of_lsm_result& r = res[run->index[(size_t)c]];
      r.price = hres[(size_t)c * 3];
      r.stderr_ = hres[(size_t)c * 3 + 1];
      r.delta = cfg->want_delta ? hres[(size_t)c * 3 + 2] : 0.0;
      r.regressions = hreg[(size_t)c];
    }
  }
  for (int64_t i = 0; i < n; ++i) res[i].kernel_ms = total_ms;
  return OF_OK;
}

static bool strictly_increasing(const double* g, int64_t n) {
  for (int64_t i = 1; i < n; ++i)
    if (!(g[i] > g[i - 1])) return false;
  return true;
}

extern "C" of_status of_lsm_bermudan(of_ctx* ctx, const of_bermudan_contract* k, const of_lsm_config* cfg,
                                     of_lsm_result* result, of_boundary_point* boundary, int64_t capacity,
                                     int64_t* n_boundary) {
  if (!ctx || !k || !cfg || !result || !n_boundary || (capacity > 0 && !boundary)) return OF_ERR_INVALID_INPUT;
  if (cfg->basis_degree != 2 && cfg->basis_degree != 3)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "basis_degree must be 2 or 3");
  const bool fp64 = cfg->precision == OF_PREC_FP64_REFERENCE;
  if (!fp64 && cfg->precision != OF_PREC_FP32_PHILOX)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown precision %d", cfg->precision);
  if (cfg->injected_normals && !fp64)
    return of_fail(ctx, OF_ERR_UNSUPPORTED, "injected normals are a FP64 reference-mode test hook");
  // BermudanOption::validate (src/instruments/bermudan.rs:104-150) and the
  // engine's own checks (longstaff_schwartz.rs:302-313, 198-204, 226-231, 256-260)
  if (k->option_type != OF_CALL && k->option_type != OF_PUT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown option type %d", k->option_type);
  if (!(k->expiry > 0.0) || !std::isfinite(k->expiry))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "bermudan expiry must be finite and > 0");
  if (k->n_schedule <= 0 || !k->schedule_times || !k->schedule_strikes)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "bermudan exercise_dates cannot be empty");
  for (int64_t d = 0; d < k->n_schedule; ++d) {
    const double t = k->schedule_times[d], K = k->schedule_strikes[d];
    if (!std::isfinite(t) || t <= 0.0 || t > k->expiry)
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "bermudan exercise_dates must be finite and in (0, expiry]");
    if (!std::isfinite(K) || K <= 0.0)
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "bermudan strike_schedule entries must be finite and > 0");
  }
  if (!strictly_increasing(k->schedule_times, k->n_schedule))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "bermudan exercise_dates must be strictly increasing");
  if (k->num_steps < 2) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps must be >= 2 for Longstaff-Schwartz");
  if (k->num_steps > (1 << 20)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps too large");
  if (cfg->num_paths < 3) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths must be >= 3 for Longstaff-Schwartz");
  if (!(k->spot > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "market spot must be > 0");
  if (k->dynamics == OF_LSM_GBM) {
    if (!std::isfinite(k->vol) || k->vol <= 0.0)
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "market volatility must be finite and > 0");
  } else if (k->dynamics == OF_LSM_LOCAL_VOL) {
    if (k->lv_n_strikes < 1 || k->lv_n_expiries < 1 || !k->lv_strikes || !k->lv_expiries || !k->lv_vols ||
        !strictly_increasing(k->lv_strikes, k->lv_n_strikes) || !strictly_increasing(k->lv_expiries, k->lv_n_expiries))
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "local volatility grid must be non-empty and strictly increasing");
    for (int64_t i = 0; i < k->lv_n_strikes * k->lv_n_expiries; ++i)
      if (!std::isfinite(k->lv_vols[i]) || k->lv_vols[i] <= 0.0)
        return of_fail(ctx, OF_ERR_INVALID_INPUT, "local volatility surface returned non-positive value");
    if (cfg->want_delta)
      return of_fail(ctx, OF_ERR_UNSUPPORTED, "pathwise delta is not defined for local-vol dynamics");
  } else if (k->dynamics == OF_LSM_HESTON_EULER) {
    if (!(k->kappa > 0.0 && k->theta >= 0.0 && k->xi >= 0.0 && k->v0 >= 0.0 && k->rho > -1.0 && k->rho < 1.0))
      return of_fail(ctx, OF_ERR_INVALID_INPUT, "invalid Heston parameters for Bermudan LSM dynamics");
  } else {
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown LSM dynamics %d", k->dynamics);
  }
  const int64_t steps = k->num_steps, N = cfg->num_paths;
  const int draws = k->dynamics == OF_LSM_HESTON_EULER ? 2 : 1;
  if (cfg->injected_normals && cfg->n_injected < N * steps * draws)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "injected normals: need %lld values, got %lld",
                   (long long)(N * steps * draws), (long long)cfg->n_injected);
  if ((double)N * (double)steps * (fp64 ? 8.0 : 4.0) > (double)((size_t)48 << 30))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "path store of %lld x %lld exceeds 48 GB", (long long)N,
                   (long long)steps);
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::memset(result, 0, sizeof(*result));
  *n_boundary = 0;
  const uint64_t* jump = nullptr;
  if (fp64 && !cfg->injected_normals) OF_TRY(upload_jump_tables(ctx, &jump));

  // schedule -> steps (longstaff_schwartz.rs:329-335): the later date wins a shared step
  std::vector<int64_t> date_of_step((size_t)steps + 1, -1);
  for (int64_t d = 0; d < k->n_schedule; ++d) {
    const double idx = std::round((k->schedule_times[d] / k->expiry) * (double)steps);
    const int64_t i = (std::isnan(idx) || idx < 1.0) ? 1 : (idx > (double)steps ? steps : (int64_t)idx);
    date_of_step[(size_t)i] = d;
  }
  const double k_T = k->schedule_strikes[k->n_schedule - 1];
  std::vector<LsmHost> hs(1);
  LsmHost& h = hs[0];
  h.can.assign((size_t)steps + 1, 0);
  std::vector<double> kk((size_t)steps + 1, k_T);
  for (int64_t t = 1; t < steps; ++t)
    if (date_of_step[(size_t)t] >= 0) {
      h.can[(size_t)t] = 1;
      kk[(size_t)t] = k->schedule_strikes[date_of_step[(size_t)t]];
    }
  h.can[(size_t)steps] = 1;
  if (k->dynamics == OF_LSM_LOCAL_VOL) {
    h.lv_k.assign(k->lv_strikes, k->lv_strikes + k->lv_n_strikes);
    h.lv_t.assign(k->lv_expiries, k->lv_expiries + k->lv_n_expiries);
    h.lv_v.assign(k->lv_vols, k->lv_vols + k->lv_n_strikes * k->lv_n_expiries);
  }
  fill_steps(h, steps, k->expiry, kk.data());
  LsmC& C = h.C;
  const double dt = k->expiry / (double)steps, sqdt = std::sqrt(dt);
  const double mu = k->rate - k->dividend_yield;
  C.put = k->option_type == OF_PUT;
  C.steps = (int32_t)steps;
  C.dynamics = k->dynamics == OF_LSM_GBM ? DYN_GBM : (k->dynamics == OF_LSM_LOCAL_VOL ? DYN_LOCAL_VOL : DYN_HESTON);
  C.spot = k->spot;
  C.strike = k_T;
  C.inv_strike = 1.0 / k_T;
  C.inv_spot = 1.0 / k->spot;
  C.drift = (mu - 0.5 * k->vol * k->vol) * dt;  // longstaff_schwartz.rs:205
  C.step_vol = k->vol * sqdt;
  C.disc = std::exp(-k->rate * dt);
  C.mu = mu;
  C.dt = dt;
  C.sqrt_dt = sqdt;
  C.kappa = k->kappa;
  C.theta = k->theta;
  C.xi = k->xi;
  C.rho = k->rho;
  C.v0 = k->v0;
  C.fdrift = (float)C.drift;
  C.fstep_vol = (float)C.step_vol;
  C.fspot = (float)k->spot;
  C.fmudt = (float)(mu * dt);
  C.fsqrt_dt = (float)sqdt;
  C.fdt = (float)dt;
  C.fy_floor = (float)std::log(1e-12 / k->spot);
  C.hc.mudt = (float)(mu * dt);
  C.hc.half_dt = (float)(0.5 * dt);
  C.hc.sqdt = (float)sqdt;
  C.hc.kdt = (float)(k->kappa * dt);
  C.hc.kdt_theta = (float)(k->kappa * k->theta * dt);
  C.hc.one_m_kdt = (float)(1.0 - k->kappa * dt);
  C.hc.xi = (float)k->xi;
  C.hc.bm_k2 = (float)(-2.0 * 0.69314718055994531 * dt);
  C.hc.rho = (float)k->rho;
  C.hc.rho_c = (float)std::sqrt(1.0 - k->rho * k->rho);
  C.hc.v0 = (float)k->v0;
  C.hc.y_floor = C.fy_floor;

  std::vector<double> hres;
  std::vector<int32_t> hreg;
  std::vector<LsmTrack> tr;
  float ms = 0.0f;
  OF_TRY(lsm_run_batch(ctx, hs, steps, cfg, jump, 0u, cfg->injected_normals, draws, &tr, hres, hreg, &ms));
  result->price = hres[0];
  result->stderr_ = hres[1];
  result->delta = cfg->want_delta ? hres[2] : 0.0;
  result->regressions = hreg[0];
  result->kernel_ms = ms;

  // boundary points, chronological (longstaff_schwartz.rs:337-412): every
  // scheduled step before expiry, then the terminal point
  std::vector<of_boundary_point> pts;
  for (int64_t t = 1; t < steps; ++t) {
    const int64_t d = date_of_step[(size_t)t];
    if (d < 0) continue;
    of_boundary_point p{};
    p.time = k->schedule_times[d];
    p.strike = k->schedule_strikes[d];
    p.itm_paths = (int64_t)tr[0].itm[(size_t)t];
    p.exercised_paths = p.itm_paths >= 3 ? (int64_t)tr[0].ex_count[(size_t)t] : 0;
    p.has_boundary = p.exercised_paths > 0 ? 1 : 0;
    double b;
    const unsigned long long bits = tr[0].ex_bits[(size_t)t];
    std::memcpy(&b, &bits, sizeof(b));
    p.boundary_spot = p.has_boundary ? b : std::nan("");
    pts.push_back(p);
  }
  of_boundary_point term{};
  term.time = k->expiry;
  term.strike = k_T;
  term.boundary_spot = k_T;
  term.has_boundary = 1;
  term.itm_paths = term.exercised_paths = (int64_t)tr[0].term_itm;
  pts.push_back(term);
  *n_boundary = (int64_t)pts.size();
  for (int64_t i = 0; i < (int64_t)pts.size() && i < capacity; ++i) boundary[i] = pts[(size_t)i];
  return OF_OK;
}

// ---------------------------------------------------------------------------
// LongstaffSchwartzEngine::price(BarrierOption)
// (src/engines/lsm/longstaff_schwartz.rs:632-736): European barrier Monte
// Carlo on the engine's single xoshiro256++ stream.  A thread owns kBarChunk
// consecutive paths and jumps its copy of the stream to the chunk's first
// draw; each path runs log-Euler with the barrier tested at every point of
// path[0..=steps] and adds its discounted payoff (or rebate) to FP64 sums.
// ---------------------------------------------------------------------------
namespace {

constexpr int kBarThreads = 128;
constexpr int kBarChunk = 8;

struct LsmBarrierParams {
  double spot, strike, level, rebate, drift, step_vol, discount;
  int64_t n, steps;
  uint64_t seed;
  int32_t call, up, knock_in;
  const uint64_t* jump;
  const double* inj;  // [path][step] test hook, or null
  double* partials;   // [block][2]: sum and sum of squares of the discounted values
};

__global__ void __launch_bounds__(kBarThreads) lsm_barrier_ref(const __grid_constant__ LsmBarrierParams P) {
  __shared__ double red_sh[2 * (kBarThreads / 32)];
  const int64_t chunk0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * kBarChunk;
  double acc[2] = {0.0, 0.0};
  if (chunk0 < P.n) {
    of::Xoshiro256pp rng;
    if (!P.inj) {
      rng.seed(P.seed);
      xoshiro_jump(rng, (uint64_t)chunk0 * (uint64_t)P.steps, P.jump);
    }
    const int64_t end = chunk0 + kBarChunk < P.n ? chunk0 + kBarChunk : P.n;
    for (int64_t p = chunk0; p < end; ++p) {
      const double* z = P.inj ? P.inj + (size_t)p * P.steps : nullptr;
      double s = P.spot;
      bool hit = P.up ? s >= P.level : s <= P.level;  // the scan includes path[0]
      for (int64_t t = 0; t < P.steps; ++t) {
        const double zt = z ? z[t] : of::acklam_inv_cdf(rng.next_f64());
        s = s * exp(fma(P.step_vol, zt, P.drift));
        hit |= P.up ? s >= P.level : s <= P.level;
      }
      const bool active = P.knock_in ? hit : !hit;
      const double intrinsic = P.call ? s - P.strike : P.strike - s;
      const double v = P.discount * (active ? (intrinsic > 0.0 ? intrinsic : 0.0) : P.rebate);
      acc[0] += v;
      acc[1] += v * v;
    }
  }
  of::block_sum<2>(acc, red_sh);
  if (threadIdx.x == 0) {
    P.partials[(int64_t)blockIdx.x * 2] = acc[0];
    P.partials[(int64_t)blockIdx.x * 2 + 1] = acc[1];
  }
}

}  // namespace

extern "C" of_status of_lsm_barrier(of_ctx* ctx, const of_lsm_barrier_contract* k, const of_lsm_config* cfg,
                                    of_lsm_result* out) {
  if (!ctx || !k || !cfg || !out) return OF_ERR_INVALID_INPUT;
  // BarrierOption::validate (src/instruments/barrier.rs:36-60), then :640-657
  if (k->option_type != OF_CALL && k->option_type != OF_PUT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown option type %d", k->option_type);
  if (!(k->strike > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "barrier strike must be > 0");
  if (!(k->expiry >= 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "barrier expiry must be >= 0");
  if (!(k->barrier_level > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "barrier level must be > 0");
  if (!(k->rebate >= 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "barrier rebate must be >= 0");
  if (k->barrier_direction != OF_BARRIER_UP && k->barrier_direction != OF_BARRIER_DOWN)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown barrier direction %d", k->barrier_direction);
  if (k->barrier_style != OF_BARRIER_IN && k->barrier_style != OF_BARRIER_OUT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown barrier style %d", k->barrier_style);
  if (k->num_steps <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps must be > 0");
  if (k->num_steps > (int64_t)1 << 30) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps too large");
  if (cfg->num_paths <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths must be > 0");
  if (!(k->vol > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "market volatility must be > 0");
  if (cfg->precision != OF_PREC_FP64_REFERENCE)
    return of_fail(ctx, OF_ERR_UNSUPPORTED,
                   "the LSM engine's barrier pricing runs on the reference stream (FP32 barriers: the batched book)");
  if (cfg->injected_normals && cfg->n_injected < cfg->num_paths * k->num_steps)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "injected normals: need num_paths x num_steps values");
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  LsmBarrierParams P{};
  const double dt = k->expiry / (double)k->num_steps;
  P.spot = k->spot;
  P.strike = k->strike;
  P.level = k->barrier_level;
  P.rebate = k->rebate;
  P.drift = (k->rate - k->dividend_yield - 0.5 * k->vol * k->vol) * dt;
  P.step_vol = k->vol * std::sqrt(dt);
  P.discount = std::exp(-k->rate * k->expiry);
  P.n = cfg->num_paths;
  P.steps = k->num_steps;
  P.seed = cfg->seed;
  P.call = k->option_type == OF_CALL;
  P.up = k->barrier_direction == OF_BARRIER_UP;
  P.knock_in = k->barrier_style == OF_BARRIER_IN;
  const int64_t per_block = (int64_t)kBarThreads * kBarChunk;
  const int64_t blocks = (P.n + per_block - 1) / per_block;
  if (blocks > 2147483647LL) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths too large");
  if (cfg->injected_normals) {
    void* d = nullptr;
    const size_t bytes = (size_t)(P.n * P.steps) * sizeof(double);
    OF_TRY(of_scratch(ctx, SLOT_INJECT, bytes, &d));
    OF_CUDA_TRY(ctx, cudaMemcpyAsync(d, cfg->injected_normals, bytes, cudaMemcpyHostToDevice, ctx->stream));
    P.inj = (const double*)d;
  } else {
    OF_TRY(upload_jump_tables(ctx, &P.jump));
  }
  void *d_part = nullptr, *d_sums = nullptr, *h = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)blocks * 2 * sizeof(double), &d_part));
  OF_TRY(of_scratch(ctx, SLOT_SUMS, 2 * sizeof(double), &d_sums));
  OF_TRY(of_pinned(ctx, 2 * sizeof(double), &h));
  P.partials = (double*)d_part;
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  lsm_barrier_ref<<<(unsigned)blocks, kBarThreads, 0, ctx->stream>>>(P);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_TRY(of_reduce_rows(ctx, (const double*)d_part, blocks, 2, (double*)d_sums));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(h, d_sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
  // mean_and_stderr, longstaff_schwartz.rs:125-140
  const double sum = ((const double*)h)[0], sum_sq = ((const double*)h)[1], n = (double)P.n;
  const double var = P.n > 1 ? (sum_sq - sum * sum / n) / (n - 1.0) : 0.0;
  out->price = sum / n;
  out->stderr_ = std::sqrt(var / n);
  out->delta = 0.0;
  out->regressions = 0;
  out->kernel_ms = ms;
  return OF_OK;
}
