// qmc.cu - Sobol quasi-Monte Carlo European pricer (of_mc_european_qmc).
//
// Replaces mc_european_qmc_with_seed (src/engines/monte_carlo/mc_qmc.rs:39-150)
// with the reference's own point set: SobolSequence (src/math/sobol.rs) with
// one dimension per time step, canonical direction numbers in dimension 0,
// hashed ones elsewhere, and a per-dimension XOR scrambler.
//
// The sequence walks Gray-code order: point n (1-based) has
// x_d(n) = XOR of v_d[j] over the set bits j of gray(n) = n ^ (n >> 1), and
// x_d(n) = x_d(n-1) ^ v_d[ctz(n)].  A thread prices kQmcPaths consecutive
// points: per dimension it forms the first one from the Gray-code bits and
// the rest by the recurrence, with the direction numbers in shared memory.
//
// FP64 reference mode keeps the reference's arithmetic (u = fma(x, 2^-64,
// 2^-65), Acklam inverse, s *= exp(fma(dt_vol, z, dt_drift))); FP32 mode
// walks the same points with FP32 paths (the top bits of each coordinate
// through the inverse-CDF transform, which keeps the points' stratification).
//
// Compiled with --fmad=false: every fused multiply-add is an explicit fma.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "of_device.cuh"
#include "of_internal.h"

namespace {

constexpr int kQmcThreads = 128;
constexpr int kQmcPaths = 8;        // consecutive Sobol points per thread
constexpr int kQmcMaxDims = 21201;  // SOBOL_MAX_DIMENSIONS, sobol.rs:14
constexpr size_t kQmcSmemMax = 96 * 1024;

struct QmcParams {
  int32_t dims, bits, put, fp32;
  int32_t smem;  // direction numbers staged in shared memory
  int64_t n_paths;
  double spot, strike, dt_drift, dt_vol;
  float fdrift, fvol, fspot, fstrike;
  const uint64_t* v;    // [dims][bits] direction numbers
  const uint64_t* scr;  // [dims] scramblers
};

// splitmix64 of sobol.rs:121-126 (a pure function of x).
uint64_t sobol_mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

__device__ __forceinline__ double vanilla64(bool put, double s, double k) {
  const double v = put ? k - s : s - k;
  return v > 0.0 ? v : 0.0;
}

__global__ void __launch_bounds__(kQmcThreads) qmc_kernel(const __grid_constant__ QmcParams P,
                                                          double* __restrict__ partials) {
  extern __shared__ uint64_t v_sh[];
  __shared__ double red[2 * (kQmcThreads / 32)];
  const uint64_t* V = P.v;
  if (P.smem) {
    const int total = P.dims * P.bits;
    for (int i = threadIdx.x; i < total; i += blockDim.x) v_sh[i] = P.v[i];
    __syncthreads();
    V = v_sh;
  }
  const int64_t first = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * kQmcPaths + 1;  // 1-based index
  const int64_t last = first + kQmcPaths - 1 <= P.n_paths ? first + kQmcPaths - 1 : P.n_paths;
  const int count = first <= P.n_paths ? (int)(last - first + 1) : 0;
  double s[kQmcPaths];
  float y[kQmcPaths];
#pragma unroll
  for (int k = 0; k < kQmcPaths; ++k) {
    s[k] = P.spot;
    y[k] = 0.0f;
  }
  const uint64_t g0 = (uint64_t)first ^ ((uint64_t)first >> 1);
  const double inv = 5.42101086242752217e-20, half = 2.71050543121376109e-20;  // 2^-64, 2^-65
  if (count > 0) {
    for (int d = 0; d < P.dims; ++d) {
      const uint64_t* vd = V + (size_t)d * P.bits;
      const uint64_t sc = __ldg(P.scr + d);
      uint64_t x = 0;
      for (uint64_t g = g0; g; g &= g - 1) x ^= vd[__ffsll((long long)g) - 1];
#pragma unroll
      for (int k = 0; k < kQmcPaths; ++k) {
        if (k >= count) break;  // first + k <= n_paths < 2^bits, so ctz(first + k) < bits
        if (k > 0) x ^= vd[__ffsll((long long)(first + k)) - 1];  // ctz(n) of the next point
        const uint64_t w = x ^ sc;
        if (P.fp32) {
          const float z = of::normal_from_u32((uint32_t)(w >> 32));
          y[k] = fmaf(P.fvol, z, y[k] + P.fdrift);
        } else {
          const double u = fma((double)w, inv, half);  // sobol.rs:70
          s[k] *= exp(fma(P.dt_vol, of::acklam_inv_cdf(u), P.dt_drift));  // mc_qmc.rs:106-117
        }
      }
    }
  }
  double a0 = 0.0, a1 = 0.0;
#pragma unroll
  for (int k = 0; k < kQmcPaths; ++k) {
    if (k < count) {
      const double st = P.fp32 ? (double)(P.fspot * __expf(y[k])) : s[k];
      const double px = vanilla64(P.put, st, P.strike);
      a0 += px;
      a1 += px * px;
    }
  }
  a0 = of::warp_sum(a0);
  a1 = of::warp_sum(a1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[2 * warp] = a0;
    red[2 * warp + 1] = a1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double b0 = 0.0, b1 = 0.0;
    for (int w = 0; w < kQmcThreads / 32; ++w) {
      b0 += red[2 * w];
      b1 += red[2 * w + 1];
    }
    partials[(int64_t)blockIdx.x * 2] = b0;
    partials[(int64_t)blockIdx.x * 2 + 1] = b1;
  }
}

}  // namespace

extern "C" of_status of_mc_european_qmc(of_ctx* ctx, const of_qmc_params* q, of_mc_result* out) {
  if (!ctx || !q || !out) return OF_ERR_INVALID_INPUT;
  if (q->option_type != OF_CALL && q->option_type != OF_PUT)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown option type %d", q->option_type);
  if (q->num_paths <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths must be > 0");
  if (q->num_paths > ((int64_t)1 << 40)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths must be <= 2^40");
  if (q->num_steps <= 0) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps must be > 0");
  if (q->num_steps > kQmcMaxDims)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "Sobol dimensions must be in [1, %d]", kQmcMaxDims);
  if (!(q->expiry > 0.0) || !std::isfinite(q->expiry))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "expiry must be finite and > 0");
  if (!(q->vol > 0.0) || !std::isfinite(q->vol))
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "market volatility must be finite and > 0");
  if (!(q->spot > 0.0)) return of_fail(ctx, OF_ERR_INVALID_INPUT, "market spot must be > 0");
  const bool fp64 = q->precision == OF_PREC_FP64_REFERENCE;
  if (!fp64 && q->precision != OF_PREC_FP32_PHILOX)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "unknown precision %d", q->precision);
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));

  // direction numbers (build_direction_numbers, sobol.rs:99-119) for the bits
  // an index up to num_paths uses, and the scramblers (:36-37)
  const int64_t dims = q->num_steps;
  int bits = 0;
  while (bits < 64 && (((uint64_t)q->num_paths) >> bits) != 0) ++bits;
  std::vector<uint64_t> v((size_t)dims * bits), scr((size_t)dims);
  for (int64_t d = 0; d < dims; ++d) {
    for (int j = 0; j < bits; ++j) {
      uint64_t vj;
      if (d == 0) {
        vj = 1ULL << (63 - j);
      } else {
        const uint64_t hash = sobol_mix(q->seed ^ (((uint64_t)d + 1) << 40) ^ (uint64_t)j);
        const uint64_t mask = j == 63 ? ~0ULL : (1ULL << (j + 1)) - 1;
        vj = ((hash | 1ULL) & mask) << (63 - j);
      }
      v[(size_t)d * bits + j] = vj;
    }
    scr[(size_t)d] = sobol_mix(q->seed ^ (((uint64_t)d + 1) << 32));
  }
  void *d_tab = nullptr, *d_part = nullptr, *d_sums = nullptr, *h = nullptr;
  const size_t vbytes = v.size() * sizeof(uint64_t);
  OF_TRY(of_scratch(ctx, SLOT_MISC, vbytes + scr.size() * sizeof(uint64_t), &d_tab));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(d_tab, v.data(), vbytes, cudaMemcpyHostToDevice, ctx->stream));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync((char*)d_tab + vbytes, scr.data(), scr.size() * sizeof(uint64_t),
                                   cudaMemcpyHostToDevice, ctx->stream));
  QmcParams P{};
  P.dims = (int32_t)dims;
  P.bits = bits;
  P.put = q->option_type == OF_PUT;
  P.fp32 = fp64 ? 0 : 1;
  P.n_paths = q->num_paths;
  P.spot = q->spot;
  P.strike = q->strike;
  const double dt = q->expiry / (double)dims;
  P.dt_drift = (q->rate - q->dividend_yield - 0.5 * q->vol * q->vol) * dt;  // mc_qmc.rs:90
  P.dt_vol = q->vol * std::sqrt(dt);
  P.fdrift = (float)P.dt_drift;
  P.fvol = (float)P.dt_vol;
  P.fspot = (float)q->spot;
  P.fstrike = (float)q->strike;
  P.v = (const uint64_t*)d_tab;
  P.scr = (const uint64_t*)((char*)d_tab + vbytes);
  size_t smem = 0;
  if (vbytes <= kQmcSmemMax) {
    P.smem = 1;
    smem = vbytes;
    if (smem > 48 * 1024)
      OF_CUDA_TRY(ctx, cudaFuncSetAttribute(qmc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  const int64_t threads = (q->num_paths + kQmcPaths - 1) / kQmcPaths;
  const int64_t grid = (threads + kQmcThreads - 1) / kQmcThreads;
  if (grid > 2147483647LL) return of_fail(ctx, OF_ERR_INVALID_INPUT, "too many paths");
  OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)grid * 2 * sizeof(double), &d_part));
  OF_TRY(of_scratch(ctx, SLOT_SUMS, 2 * sizeof(double), &d_sums));
  OF_TRY(of_pinned(ctx, 2 * sizeof(double), &h));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  qmc_kernel<<<(unsigned)grid, kQmcThreads, smem, ctx->stream>>>(P, (double*)d_part);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_TRY(of_reduce_rows(ctx, (const double*)d_part, grid, 2, (double*)d_sums));
  OF_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(h, d_sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  OF_CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
  double sums[2];
  std::memcpy(sums, h, sizeof(sums));
  // mean / variance of mc_qmc.rs:125-144
  const double n = (double)q->num_paths;
  const double mean = sums[0] / n;
  double var = q->num_paths > 1 ? (sums[1] - sums[0] * sums[0] / n) / (n - 1.0) : 0.0;
  var = var > 0.0 ? var : 0.0;
  const double disc = std::exp(-q->rate * q->expiry);
  std::memset(out, 0, sizeof(*out));
  out->price = disc * mean;
  out->stderr_ = disc * std::sqrt(var / n);
  out->samples = q->num_paths;
  out->sum_x = sums[0];
  out->sum_x2 = sums[1];
  out->kernel_ms = ms;
  return OF_OK;
}
