// of_device.cuh - device-side generators and reductions shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "f32x2.cuh"
#include "invnorm_coeffs.h"

namespace of {

constexpr unsigned kFullMask = 0xffffffffu;

// ---------------------------------------------------------------------------
// openferric's reference stream (FP64 reference mode).
// xoshiro256++ seeded by SplitMix64: src/math/fast_rng.rs:30-81,181-200.
// ---------------------------------------------------------------------------
struct Xoshiro256pp {
  uint64_t s0, s1, s2, s3;

  __device__ __forceinline__ static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

  __device__ __forceinline__ void seed(uint64_t seed) {
    uint64_t sm = seed;
    uint64_t st[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      sm += 0x9E3779B97F4A7C15ULL;
      uint64_t z = sm;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
      st[i] = z ^ (z >> 31);
    }
    if ((st[0] | st[1] | st[2] | st[3]) == 0) st[0] = 1;
    s0 = st[0];
    s1 = st[1];
    s2 = st[2];
    s3 = st[3];
  }

  __device__ __forceinline__ uint64_t next_u64() {
    const uint64_t result = rotl(s0 + s3, 23) + s0;
    const uint64_t t = s1 << 17;
    s2 ^= s0;
    s3 ^= s1;
    s1 ^= s2;
    s0 ^= s3;
    s2 ^= t;
    s3 = rotl(s3, 45);
    return result;
  }

  // next_f64, fast_rng.rs:70-73
  __device__ __forceinline__ double next_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
};

// PCG XSL-RR 128/64 (O'Neill 2014), the reference's Pcg64
// (src/math/fast_rng.rs:86-128): a 128-bit LCG with PCG's default multiplier
// 0x2360ED051FC65DA4_4385DF649FCCF645, odd increment (stream << 1) | 1; the
// output is (hi ^ lo) rotated right by the top 6 bits of the old state.
// Seeded by SplitMix64 (state hi, state lo, stream) and advanced once.  The
// 128-bit state is two 64-bit words; the product keeps its low 128 bits.
struct Pcg64 {
  uint64_t hi, lo, inc_hi, inc_lo;

  static constexpr uint64_t kMulHi = 0x2360ED051FC65DA4ULL, kMulLo = 0x4385DF649FCCF645ULL;

  __device__ __forceinline__ static uint64_t splitmix(uint64_t& sm) {
    sm += 0x9E3779B97F4A7C15ULL;
    uint64_t z = sm;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }

  __device__ __forceinline__ void seed(uint64_t seed) {
    uint64_t sm = seed;
    hi = splitmix(sm);
    lo = splitmix(sm);
    const uint64_t stream = splitmix(sm);
    inc_hi = stream >> 63;
    inc_lo = (stream << 1) | 1ULL;
    (void)next_u64();
  }

  __device__ __forceinline__ uint64_t next_u64() {
    const uint64_t ohi = hi, olo = lo;
    // state = old * M + inc (mod 2^128)
    const uint64_t plo = olo * kMulLo;
    const uint64_t phi = __umul64hi(olo, kMulLo) + olo * kMulHi + ohi * kMulLo;
    lo = plo + inc_lo;
    hi = phi + inc_hi + (lo < plo ? 1ULL : 0ULL);
    const uint64_t x = ohi ^ olo;
    const unsigned rot = (unsigned)(ohi >> 58);
    return (x >> rot) | (x << ((64u - rot) & 63u));
  }

  __device__ __forceinline__ double next_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
};

// uniform_open01 (fast_rng.rs:219-221) then the Acklam inverse
// (beasley_springer_moro_inv_cdf, src/math/fast_norm.rs:54-139), FP64.
// Translation units using this must be compiled with --fmad=false so that
// only the explicit fma() calls (the reference's mul_add) contract.
__device__ __forceinline__ double acklam_inv_cdf(double p) {
  const double eps = 2.220446049250313080847263336181640625e-16;
  p = p < eps ? eps : (p > 1.0 - eps ? 1.0 - eps : p);
  const double a0 = -3.969683028665376e1, a1 = 2.209460984245205e2, a2 = -2.759285104469687e2,
               a3 = 1.38357751867269e2, a4 = -3.066479806614716e1, a5 = 2.506628277459239;
  const double b0 = -5.447609879822406e1, b1 = 1.615858368580409e2, b2 = -1.556989798598866e2,
               b3 = 6.680131188771972e1, b4 = -1.328068155288572e1;
  const double c0 = -7.784894002430293e-3, c1 = -3.223964580411365e-1, c2 = -2.400758277161838,
               c3 = -2.549732539343734, c4 = 4.374664141464968, c5 = 2.938163982698783;
  const double d0 = 7.784695709041462e-3, d1 = 3.224671290700398e-1, d2 = 2.445134137142996,
               d3 = 3.754408661907416;
  const double p_low = 0.02425, p_high = 1.0 - 0.02425;
  if (p < p_low) {
    const double q = sqrt(-2.0 * log(p));
    return fma(fma(fma(fma(fma(c0, q, c1), q, c2), q, c3), q, c4), q, c5) /
           fma(fma(fma(fma(d0, q, d1), q, d2), q, d3), q, 1.0);
  } else if (p <= p_high) {
    const double q = p - 0.5;
    const double r = q * q;
    return fma(fma(fma(fma(fma(a0, r, a1), r, a2), r, a3), r, a4), r, a5) * q /
           fma(fma(fma(fma(fma(b0, r, b1), r, b2), r, b3), r, b4), r, 1.0);
  } else {
    const double q = sqrt(-2.0 * log(1.0 - p));
    return -fma(fma(fma(fma(fma(c0, q, c1), q, c2), q, c3), q, c4), q, c5) /
           fma(fma(fma(fma(d0, q, d1), q, d2), q, d3), q, 1.0);
  }
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) - FP32 mode generator.
// Counter layout used by every kernel: {draw block, path lo, path hi, stream tag}.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// The ten round keys of a 64-bit seed, computed once on the host.  Kernels
// carry them in their (constant-bank) parameters, so a round is two wide
// multiplies and two three-input XORs with no key arithmetic.
struct PhiloxKeys {
  uint32_t k0[10], k1[10];
};

__host__ __device__ inline PhiloxKeys philox_keys(uint64_t seed) {
  PhiloxKeys K;
  uint32_t a = (uint32_t)seed, b = (uint32_t)(seed >> 32);
  for (int r = 0; r < 10; ++r) {
    K.k0[r] = a;
    K.k1[r] = b;
    a += 0x9E3779B9u;
    b += 0xBB67AE85u;
  }
  return K;
}

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, const PhiloxKeys& K) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ K.k0[r], (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ K.k1[r],
                   (uint32_t)p0);
  }
  return c;
}

// u32 -> standard normal in FP32: u = (k + 0.5) 2^-23 with k the top 23 bits,
// then Phi^-1(u) = x P(w), x = 2u-1, w = -log2((1+x)(1-x)) with the fitted
// polynomials of invnorm_coeffs.h (one MUFU lg2 per draw; the tail branch,
// w >= OF_INVN_W_SPLIT, is taken with probability 0.34 %).
__device__ __forceinline__ float normal_from_u32(uint32_t r) {
  const float f = __uint_as_float(0x3F800000u | (r >> 9));  // 1 + k 2^-23, exact
  const float x = fmaf(2.0f, f, -3.0f) + 1.1920928955078125e-7f;  // (2k + 1 - 2^23) 2^-23, exact
  const float t = fmaf(-x, x, 1.0f);  // 1 - x^2 = 4u(1-u), one rounding of the exact value
  const float w = -__log2f(t);
  float p;
  if (w < OF_INVN_W_SPLIT) {
    const float s = w - OF_INVN_C_CENTER;
    p = kInvnCentral[OF_INVN_DEG_C];
#pragma unroll
    for (int i = OF_INVN_DEG_C - 1; i >= 0; --i) p = fmaf(p, s, kInvnCentral[i]);
  } else {
    const float s = sqrtf(w) - OF_INVN_T_CENTER;
    p = kInvnTail[OF_INVN_DEG_T];
#pragma unroll
    for (int i = OF_INVN_DEG_T - 1; i >= 0; --i) p = fmaf(p, s, kInvnTail[i]);
  }
  return x * p;
}

// Phi^-1(v) for v in (0,1) given q = 1 - v (each exact or rounded once, so
// that either tail keeps its relative precision): the polynomials of
// normal_from_u32 on x = v - q = 2v - 1 and w = -log2(4 v q), whose fit
// covers w <= 26 (v or q down to ~3.7e-9); CUDA's normcdfinvf beyond that.
__device__ __forceinline__ float inv_normal_vq(float v, float q) {
  const float t = 4.0f * v * q;  // 1 - x^2
  if (t < 1.4901161193847656e-8f)  // 2^-26: past the tail fit (probability ~1e-8 per draw)
    return v <= 0.5f ? normcdfinvf(v) : -normcdfinvf(q);
  const float x = v - q;
  const float w = -__log2f(t);
  float p;
  if (w < OF_INVN_W_SPLIT) {
    const float s = w - OF_INVN_C_CENTER;
    p = kInvnCentral[OF_INVN_DEG_C];
#pragma unroll
    for (int i = OF_INVN_DEG_C - 1; i >= 0; --i) p = fmaf(p, s, kInvnCentral[i]);
  } else {
    const float s = sqrtf(w) - OF_INVN_T_CENTER;
    p = kInvnTail[OF_INVN_DEG_T];
#pragma unroll
    for (int i = OF_INVN_DEG_T - 1; i >= 0; --i) p = fmaf(p, s, kInvnTail[i]);
  }
  return x * p;
}

// u32 -> uniform in (0,1), the same grid as normal_from_u32: (k + 0.5) 2^-23.
__device__ __forceinline__ float uniform_from_u32(uint32_t r) {
  const float f = __uint_as_float(0x3F800000u | (r >> 9));
  // f - (1 - 2^-24) = (2k + 1) 2^-24: one exact subtraction (Sterbenz), the
  // same value as (f - 1) + 2^-24
  return f - 0.999999940395355224609375f;
}

// Two independent standard normals from two u32 draws, Box-Muller transform
// (Box & Muller, Ann. Math. Stat. 29, 1958): radius sqrt(-2 ln u1) with
// u1 = (k + 0.5) 2^-23 from the top 23 bits of a (never 0 or 1, so the
// radius is finite and at most sqrt(48 ln 2) = 5.77), angle pi (2 f - 3) in
// [-pi, pi) with f = 1 + k 2^-23 from the top 23 bits of b, which covers one
// turn exactly once.  The angle is one fma, 2 pi f - 3 pi (the two rounded
// constants move it by at most 3e-7 rad).  MUFU lg2, sqrt, sin and cos plus
// ~9 FP32/integer ops per pair, against ~2 x 16 for two normal_from_u32 draws.
//
// normal_pair_scaled_from_u32 returns s (z1, z2) for a scale s > 0 folded
// into the radius: k2 = -2 ln(2) s^2, r = sqrt(k2 log2(u1)) = s sqrt(-2 ln u1),
// at the cost of the unscaled pair (the constant of the multiply changes).
constexpr float kBoxMullerK2 = -1.3862943611198906f;  // -2 ln 2: unit scale

__device__ __forceinline__ float2 normal_pair_scaled_from_u32(uint32_t a, uint32_t b, float k2) {
  const float u1 = uniform_from_u32(a);
  const float r = sqrtf(k2 * __log2f(u1));  // k2 log2(u1) = -2 s^2 ln(u1)
  const float ang = fmaf(6.28318530717959f, __uint_as_float(0x3F800000u | (b >> 9)), -9.42477796076938f);
  float s, c;
  __sincosf(ang, &s, &c);
  return make_float2(r * c, r * s);
}

__device__ __forceinline__ float2 normal_pair_from_u32(uint32_t a, uint32_t b) {
  return normal_pair_scaled_from_u32(a, b, kBoxMullerK2);
}

// normal_pair_scaled_from_u32 of two samples' draw pairs (a0, b0) and (a1, b1)
// with the FP32 arithmetic in packed pairs: w1 = (z1 of sample 0, z1 of
// sample 1), w2 likewise for z2; each half is bit-identical to the scalar
// transform (the same operations in the same order).
__device__ __forceinline__ void normal_pairs_scaled2_from_u32(uint32_t a0, uint32_t b0, uint32_t a1, uint32_t b1,
                                                              float k2, float2& w1, float2& w2) {
  const float2 u1 = sub2(make_float2(__uint_as_float(0x3F800000u | (a0 >> 9)), __uint_as_float(0x3F800000u | (a1 >> 9))),
                         splat2(0.999999940395355224609375f));
  const float2 rr = mul2(splat2(k2), make_float2(__log2f(u1.x), __log2f(u1.y)));
  const float2 r = make_float2(sqrtf(rr.x), sqrtf(rr.y));
  const float2 ang = fma2(splat2(6.28318530717959f),
                          make_float2(__uint_as_float(0x3F800000u | (b0 >> 9)), __uint_as_float(0x3F800000u | (b1 >> 9))),
                          splat2(-9.42477796076938f));
  float s0, c0, s1, c1;
  __sincosf(ang.x, &s0, &c0);
  __sincosf(ang.y, &s1, &c1);
  w1 = mul2(r, make_float2(c0, c1));
  w2 = mul2(r, make_float2(s0, s1));
}

// The sum z1 + z2 of normal_pair_from_u32(a, b), r (cos t + sin t), as
// sqrt(2) r sin(t + pi/4): one sine instead of a sine and a cosine, and one
// multiply instead of two, for loops that read only the sum of a path's
// normals.  The same draws as the pair, to FP32 rounding: sqrt(2) goes inside
// the square root (k2 doubled, exactly) and pi/4 into the angle's constant
// (-3 pi + pi/4 = -11 pi/4; the angle then spans [-3 pi/4, 5 pi/4)).
constexpr float kBoxMullerAngSum = -8.63937979737193f;

__device__ __forceinline__ float normal_pair_sum_from_u32(uint32_t a, uint32_t b) {
  const float u1 = uniform_from_u32(a);
  const float r = sqrtf((2.0f * kBoxMullerK2) * __log2f(u1));
  const float ang = fmaf(6.28318530717959f, __uint_as_float(0x3F800000u | (b >> 9)), kBoxMullerAngSum);
  return r * __sinf(ang);
}

// normal_pair_sum_from_u32 of two samples' draw pairs (a0, b0) and (a1, b1)
// in packed pairs; each half is the scalar form bit for bit.
__device__ __forceinline__ float2 normal_pair_sums2_from_u32(uint32_t a0, uint32_t b0, uint32_t a1, uint32_t b1) {
  const float2 u1 = sub2(make_float2(__uint_as_float(0x3F800000u | (a0 >> 9)), __uint_as_float(0x3F800000u | (a1 >> 9))),
                         splat2(0.999999940395355224609375f));
  const float2 rr = mul2(splat2(2.0f * kBoxMullerK2), make_float2(__log2f(u1.x), __log2f(u1.y)));
  const float2 r = make_float2(sqrtf(rr.x), sqrtf(rr.y));
  const float2 ang = fma2(splat2(6.28318530717959f),
                          make_float2(__uint_as_float(0x3F800000u | (b0 >> 9)), __uint_as_float(0x3F800000u | (b1 >> 9))),
                          splat2(kBoxMullerAngSum));
  return mul2(r, make_float2(__sinf(ang.x), __sinf(ang.y)));
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFullMask, v, o);
  return v;
}

// Block-wide sum of N doubles per thread; result valid in thread 0 (out[]).
// `sh` must hold N * (blockDim.x / 32) doubles.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) sh[warp * N + k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double acc = 0.0;
      for (int w = 0; w < nw; ++w) acc += sh[w * N + k];
      v[k] = acc;
    }
  }
}

// Compensated FP32 accumulator (Kahan); flushed to FP64 as sum - comp.
struct Kahan32 {
  float sum = 0.0f, comp = 0.0f;
  __device__ __forceinline__ void add(float v) {
    const float y = v - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
  }
  __device__ __forceinline__ double value() const { return (double)sum - (double)comp; }
};

}  // namespace of
