// wait_test.cu - of_test_bounded_wait: the bounded mbarrier wait of the
// bulk-copy pipelines, exercised on its own.  With no arrival the phase never
// completes, so the wait must give up after its limit and the kernel return.
#include "bulk_copy.cuh"
#include "of_internal.h"

namespace {

__global__ void bounded_wait_kernel(int32_t arrive, uint64_t limit_ns, int32_t* out_ok, uint64_t* out_ns) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = of::smem_u32(&bar);
  if (threadIdx.x == 0) {
    of::mbar_init(b, 1);
    of::mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && arrive) of::mbar_arrive_expect_tx(b, 0);  // one arrival, no transactions
  const uint64_t t0 = of::global_ns();
  const bool ok = of::mbar_wait(b, 0u, limit_ns);
  const uint64_t t1 = of::global_ns();
  const bool all = __syncthreads_and(ok);
  if (threadIdx.x == 0) {
    *out_ok = all ? 1 : 0;
    *out_ns = t1 - t0;
  }
}

}  // namespace

extern "C" of_status of_test_bounded_wait(of_ctx* ctx, int32_t arrive, uint32_t limit_us, int32_t* waited_ok,
                                          double* elapsed_us) {
  if (!ctx || !waited_ok || !elapsed_us) return OF_ERR_INVALID_INPUT;
  if (limit_us == 0 || limit_us > 1000000u)
    return of_fail(ctx, OF_ERR_INVALID_INPUT, "limit_us must be in 1..1000000");
  OF_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  void* d = nullptr;
  OF_TRY(of_scratch(ctx, SLOT_MISC, 16, &d));
  bounded_wait_kernel<<<1, 64, 0, ctx->stream>>>(arrive, (uint64_t)limit_us * 1000u, (int32_t*)d,
                                                 (uint64_t*)((char*)d + 8));
  OF_CUDA_TRY(ctx, cudaGetLastError());
  int32_t ok = 0;
  uint64_t ns = 0;
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(&ok, d, sizeof(ok), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaMemcpyAsync(&ns, (char*)d + 8, sizeof(ns), cudaMemcpyDeviceToHost, ctx->stream));
  OF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *waited_ok = ok;
  *elapsed_us = (double)ns * 1e-3;
  return OF_OK;
}
