// wgsl_port.cu - the reference's GPU European kernel on CUDA.
//
// openferric's only GPU code is a WGSL compute shader behind wgpu
// (src/engines/gpu/mc_shader.wgsl:28-142, host src/engines/gpu/gpu_mc.rs:59-349).
// This is the same computation as a CUDA kernel so that `mc_european_gpu`
// callers get identical semantics without a graphics API: one thread per GBM
// path in f32, xoshiro128++ seeded by a 32-bit mix of (path id + seed),
// Box-Muller normals consumed in pairs, 256-thread shared-memory tree
// reduction of (sum, sum^2) per block, FP64 final sum on the host.
#include <cmath>
#include <vector>

#include "of_internal.h"

namespace {

struct WgslParams {
  float spot, strike, dt_drift, dt_vol;
  uint32_t num_steps, num_paths, seed, is_call;
};

__device__ __forceinline__ uint32_t rotl32(uint32_t x, uint32_t k) { return (x << k) | (x >> (32u - k)); }

__device__ __forceinline__ uint32_t mix32(uint32_t z) {
  z ^= z >> 16;
  z *= 0x45d9f3bu;
  z ^= z >> 16;
  z *= 0x45d9f3bu;
  z ^= z >> 16;
  return z;
}

struct X128 {
  uint32_t s0, s1, s2, s3;
  __device__ __forceinline__ uint32_t next() {  // mc_shader.wgsl:38-48
    const uint32_t result = rotl32(s0 + s3, 7u) + s0;
    const uint32_t t = s1 << 9u;
    s2 ^= s0;
    s3 ^= s1;
    s1 ^= s2;
    s0 ^= s3;
    s2 ^= t;
    s3 = rotl32(s3, 11u);
    return result;
  }
  __device__ __forceinline__ float f32() { return (float)(next() >> 8u) * 5.9604644775390625e-8f; }
};

__global__ void __launch_bounds__(256) wgsl_european_kernel(WgslParams P, float* __restrict__ partials) {
  __shared__ float sh_sum[256], sh_sq[256];
  const uint32_t path_id = blockIdx.x * 256u + threadIdx.x;
  float payoff = 0.0f;
  if (path_id < P.num_paths) {
    X128 r;
    uint32_t z = path_id + P.seed;  // seed_rng, mc_shader.wgsl:57-71
    z = mix32(z);
    r.s0 = z;
    z += 0x9e3779b9u;
    z = mix32(z);
    r.s1 = z;
    z += 0x9e3779b9u;
    z = mix32(z);
    r.s2 = z;
    z += 0x9e3779b9u;
    z = mix32(z);
    r.s3 = z;
    float spot = P.spot;
    const uint32_t pairs = P.num_steps / 2u;
    for (uint32_t p = 0; p < pairs; ++p) {
      const float u1 = fmaxf(r.f32(), 1.0e-10f);
      const float u2 = r.f32();
      const float rr = sqrtf(-2.0f * logf(u1));
      const float th = 6.283185307179586f * u2;
      spot *= expf(fmaf(P.dt_vol, rr * cosf(th), P.dt_drift));
      spot *= expf(fmaf(P.dt_vol, rr * sinf(th), P.dt_drift));
    }
    if (P.num_steps & 1u) {
      const float u1 = fmaxf(r.f32(), 1.0e-10f);
      const float u2 = r.f32();
      const float rr = sqrtf(-2.0f * logf(u1));
      spot *= expf(fmaf(P.dt_vol, rr * cosf(6.283185307179586f * u2), P.dt_drift));
    }
    payoff = P.is_call ? fmaxf(spot - P.strike, 0.0f) : fmaxf(P.strike - spot, 0.0f);
  }
  sh_sum[threadIdx.x] = payoff;
  sh_sq[threadIdx.x] = payoff * payoff;
  __syncthreads();
  for (uint32_t stride = 128u; stride > 0u; stride >>= 1u) {  // mc_shader.wgsl:122-133
    if (threadIdx.x < stride) {
      sh_sum[threadIdx.x] += sh_sum[threadIdx.x + stride];
      sh_sq[threadIdx.x] += sh_sq[threadIdx.x + stride];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 2u] = sh_sum[0];
    partials[blockIdx.x * 2u + 1u] = sh_sq[0];
  }
}

}  // namespace

extern "C" of_status of_mc_european_gpu(of_ctx* ctx, double spot, double strike, double rate, double vol,
                                        double expiry, int64_t num_paths, int64_t num_steps, uint32_t seed,
                                        int32_t is_call, double* price, double* stderr_) {
  if (!ctx || !price || !stderr_) return OF_ERR_INVALID_INPUT;
  if (num_paths <= 0 || num_paths > 0xFFFFFFFFLL) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_paths out of range");
  if (num_steps <= 0 || num_steps > 0xFFFFFFFFLL) return of_fail(ctx, OF_ERR_INVALID_INPUT, "num_steps out of range");
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  // build_params (gpu_mc.rs:59-89): FP64 then rounded to f32
  const double dt = expiry / (double)num_steps;
  WgslParams P;
  P.spot = (float)spot;
  P.strike = (float)strike;
  P.dt_drift = (float)((rate - 0.5 * vol * vol) * dt);
  P.dt_vol = (float)(vol * std::sqrt(dt));
  P.num_steps = (uint32_t)num_steps;
  P.num_paths = (uint32_t)num_paths;
  P.seed = seed;
  P.is_call = is_call ? 1u : 0u;
  const double discount = std::exp(-rate * expiry);
  const uint32_t groups = (uint32_t)((num_paths + 255) / 256);
  void *d = nullptr, *h = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_PARTIALS, (size_t)groups * 2 * sizeof(float), &d));
  OF_TRY(of_pinned(ctx, (size_t)groups * 2 * sizeof(float), &h));
  wgsl_european_kernel<<<groups, 256, 0, ctx->stream>>>(P, (float*)d);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(h, d, (size_t)groups * 2 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  // reduce_partial_sums (gpu_mc.rs:96-118)
  const float* ps = (const float*)h;
  double sum = 0.0, sum_sq = 0.0;
  for (uint32_t g = 0; g < groups; ++g) {
    sum += (double)ps[2 * g];
    sum_sq += (double)ps[2 * g + 1];
  }
  const double n = (double)num_paths;
  const double mean = sum / n;
  const double var = num_paths > 1 ? (sum_sq - sum * sum / n) / (n - 1.0) : 0.0;
  *price = discount * mean;
  *stderr_ = discount * std::sqrt(var / n);
  return OF_OK;
}
