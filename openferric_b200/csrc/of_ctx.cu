// of_ctx.cu - context lifecycle, scratch pool, errors and shared host helpers.
#include <cmath>
#include <cstring>

#include "of_device.cuh"
#include "of_internal.h"

of_status of_fail(of_ctx* ctx, of_status st, const char* fmt, ...) {
  if (ctx) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return st;
}

of_status of_ctx_check(of_ctx* ctx) {
  if (ctx && ctx->unusable)
    return of_fail(ctx, OF_ERR_CUDA,
                   "context unusable: an earlier kernel gave up with copies in flight; destroy it and create a new one");
  return OF_OK;
}

of_status of_scratch(of_ctx* ctx, int slot, size_t bytes, void** out) {
  OF_TRY(of_ctx_check(ctx));
  if (slot < 0 || slot >= SLOT_COUNT) return of_fail(ctx, OF_ERR_INVALID_INPUT, "bad scratch slot %d", slot);
  if (bytes == 0) bytes = 16;
  if (ctx->slot_bytes[slot] < bytes) {
    if (ctx->slot_ptr[slot]) {
      // The streams may still use the old buffer.
      OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
      if (ctx->side_stream) OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->side_stream));
      OF_CUDA_TRY(ctx, cudaFree(ctx->slot_ptr[slot]));
      ctx->slot_ptr[slot] = nullptr;
      ctx->slot_bytes[slot] = 0;
    }
    // Round up to 2 MiB to limit regrowth.
    const size_t rounded = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    cudaError_t e = cudaMalloc(&ctx->slot_ptr[slot], rounded);
    if (e != cudaSuccess) {
      ctx->slot_ptr[slot] = nullptr;
      return of_fail(ctx, OF_ERR_ALLOC, "cudaMalloc(%zu) failed: %s", rounded, cudaGetErrorString(e));
    }
    ctx->slot_bytes[slot] = rounded;
  }
  *out = ctx->slot_ptr[slot];
  return OF_OK;
}

of_status of_pinned(of_ctx* ctx, size_t bytes, void** out) {
  OF_TRY(of_ctx_check(ctx));
  if (ctx->pinned_bytes < bytes) {
    if (ctx->pinned) {
      OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
      OF_CUDA_TRY(ctx, cudaFreeHost(ctx->pinned));
      ctx->pinned = nullptr;
      ctx->pinned_bytes = 0;
    }
    const size_t rounded = (bytes + 65535) & ~size_t(65535);
    cudaError_t e = cudaMallocHost(&ctx->pinned, rounded);
    if (e != cudaSuccess) {
      ctx->pinned = nullptr;
      return of_fail(ctx, OF_ERR_ALLOC, "cudaMallocHost(%zu) failed: %s", rounded, cudaGetErrorString(e));
    }
    ctx->pinned_bytes = rounded;
  }
  *out = ctx->pinned;
  return OF_OK;
}

int of_blocks_per_sm(const void* kernel, int block, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, smem) != cudaSuccess || n < 1) n = 1;
  return n;
}

// Column sums of a rows x cols matrix: one block per column, fixed-order tree.
__global__ void reduce_rows_kernel(const double* __restrict__ in, int64_t rows, int64_t cols,
                                   double* __restrict__ out) {
  __shared__ double sh[256];
  const int64_t c = blockIdx.x;
  double acc = 0.0;
  for (int64_t r = threadIdx.x; r < rows; r += blockDim.x) acc += in[r * cols + c];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = sh[0];
}

void of_launch_reduce_rows(const double* in, int64_t rows, int64_t cols, double* out, cudaStream_t s) {
  reduce_rows_kernel<<<(unsigned)cols, 256, 0, s>>>(in, rows, cols, out);
}

of_status of_reduce_rows(of_ctx* ctx, const double* in, int64_t rows, int64_t cols, double* out) {
  if (cols <= 0) return OF_OK;
  if (cols > 2147483647LL) return of_fail(ctx, OF_ERR_INVALID_INPUT, "too many columns");
  reduce_rows_kernel<<<(unsigned)cols, 256, 0, ctx->stream>>>(in, rows, cols, out);
  OF_CUDA_TRY(ctx, cudaGetLastError());
  return OF_OK;
}

void of_mc_finish(const double s[5], int64_t count, int32_t cv_kind, double e, double df, of_mc_result* out) {
  const double n = (double)count;
  out->samples = count;
  out->sum_x = s[0];
  out->sum_x2 = s[1];
  out->sum_y = s[2];
  out->sum_xy = s[3];
  out->sum_y2 = s[4];
  if (cv_kind != OF_CV_NONE) {
    const double denom = std::fmax(n - 1.0, 1.0);
    const double cov_xy = (s[3] - s[0] * s[2] / n) / denom;
    const double var_y = (s[4] - s[2] * s[2] / n) / denom;
    const double beta = var_y > 1e-16 ? cov_xy / var_y : 0.0;
    const double sum_adj = s[0] + beta * (n * e - s[2]);
    const double sum_adj_sq =
        s[1] + 2.0 * beta * e * s[0] - 2.0 * beta * s[3] + beta * beta * (n * e * e - 2.0 * e * s[2] + s[4]);
    const double mean = sum_adj / n;
    const double var = n > 1.0 ? (sum_adj_sq - sum_adj * sum_adj / n) / (n - 1.0) : 0.0;
    out->price = df * mean;
    out->stderr_ = df * std::sqrt(var / n);
  } else {
    const double mean = s[0] / n;
    const double var = n > 1.0 ? (s[1] - s[0] * s[0] / n) / (n - 1.0) : 0.0;
    out->price = df * mean;
    out->stderr_ = df * std::sqrt(var / n);
  }
}

extern "C" {

int of_abi_version(void) { return OF_GPU_ABI_VERSION; }

const char* of_status_str(of_status st) {
  switch (st) {
    case OF_OK: return "ok";
    case OF_ERR_INVALID_INPUT: return "invalid input";
    case OF_ERR_NUMERICAL: return "numerical error";
    case OF_ERR_CUDA: return "cuda error";
    case OF_ERR_TIMEOUT: return "timeout";
    case OF_ERR_UNSUPPORTED: return "unsupported";
    case OF_ERR_ALLOC: return "allocation failure";
    case OF_ERR_CONVERGENCE: return "convergence failure";
  }
  return "unknown status";
}

of_status of_ctx_create(int device, of_ctx** out) {
  if (!out) return OF_ERR_INVALID_INPUT;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return OF_ERR_CUDA;
  if (device < 0 || device >= n) return OF_ERR_INVALID_INPUT;
  of_ctx* ctx = new of_ctx();
  ctx->device = device;
  // the context stream at the highest priority: work that overlaps it on the
  // side stream (LSM path generation) yields to it
  int least = 0, greatest = 0;
  if (cudaSetDevice(device) != cudaSuccess || cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
      cudaStreamCreateWithPriority(&ctx->own_stream, cudaStreamNonBlocking, greatest) != cudaSuccess ||
      cudaEventCreate(&ctx->ev_start) != cudaSuccess || cudaEventCreate(&ctx->ev_stop) != cudaSuccess) {
    of_ctx_destroy(ctx);
    return OF_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&ctx->max_threads_per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device);
  *out = ctx;
  return OF_OK;
}

void of_ctx_destroy(of_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->side_stream) {
    cudaStreamSynchronize(ctx->side_stream);
    cudaStreamDestroy(ctx->side_stream);
  }
  for (int i = 0; i < SLOT_COUNT; ++i)
    if (ctx->slot_ptr[i]) cudaFree(ctx->slot_ptr[i]);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

const char* of_ctx_last_error(const of_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

of_status of_ctx_set_stream(of_ctx* ctx, void* stream) {
  if (!ctx) return OF_ERR_INVALID_INPUT;
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return OF_OK;
}

of_status of_ctx_get_stream(of_ctx* ctx, void** stream) {
  if (!ctx || !stream) return OF_ERR_INVALID_INPUT;
  *stream = (void*)ctx->stream;
  return OF_OK;
}

int of_device_sm_count(of_ctx* ctx) { return ctx ? ctx->sm_count : 0; }

}  // extern "C"
