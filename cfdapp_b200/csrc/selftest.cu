// Self-test of the bounded device-side wait that every persistent kernel of
// this library uses for its grid and team barriers (grid_sync.cuh): a
// barrier that can never complete must give up after its time limit, raise
// the error flag, and let the kernel return, leaving the context usable.
// No GPU fault is involved: the waiting blocks poll %globaltimer and return.
#include <cuda_runtime.h>

#include <cstdint>

#include "cfdb.h"
#include "cfdb_internal.cuh"
#include "grid_sync.cuh"

namespace cfdb {
namespace {

// nblocks of the barrier is one more than the grid, so the last arrival
// never comes; every block records whether its barrier call succeeded.
__global__ void k_unreachable_barrier(GridSync s, int* passed) {
  const bool ok = grid_sync(s);
  if (threadIdx.x == 0) passed[blockIdx.x] = ok ? 1 : 0;
}

}  // namespace
}  // namespace cfdb

using namespace cfdb;

extern "C" cfdb_status cfdb_selftest_wait_timeout(cfdb_context* ctx, double timeout_s,
                                                  int* blocks_released) {
  if (!ctx || !(timeout_s > 0.0) || timeout_s > 10.0) return CFDB_ERR_INVALID_ARGUMENT;
  constexpr int kBlocks = 2;
  unsigned* words = nullptr;
  int* passed = nullptr;
  CFDB_CUDA(ctx, cudaMalloc((void**)&words, 3 * sizeof(unsigned)));
  cudaError_t e = cudaMalloc((void**)&passed, kBlocks * sizeof(int));
  if (e != cudaSuccess) {
    cudaFree(words);
    return cuda_error(ctx, e, "selftest allocation", __FILE__, __LINE__);
  }
  cudaMemsetAsync(words, 0, 3 * sizeof(unsigned), ctx->stream);
  cudaMemsetAsync(passed, 0xff, kBlocks * sizeof(int), ctx->stream);
  GridSync s;
  s.count = words;
  s.gen = words + 1;
  s.error = words + 2;
  s.nblocks = kBlocks + 1;
  s.timeout_ns = (unsigned long long)(timeout_s * 1e9);
  k_unreachable_barrier<<<kBlocks, 64, 0, ctx->stream>>>(s, passed);
  e = cudaGetLastError();
  unsigned err = 0;
  int got[kBlocks] = {-1, -1};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&err, words + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(got, passed, sizeof(got), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(words);
  cudaFree(passed);
  if (e != cudaSuccess) return cuda_error(ctx, e, "selftest", __FILE__, __LINE__);
  int released = 0;
  for (int b = 0; b < kBlocks; ++b) released += got[b] == 0 ? 1 : 0;
  if (blocks_released) *blocks_released = released;
  if (err) return set_error(ctx, CFDB_ERR_DEVICE_TIMEOUT, "the test barrier timed out as intended");
  return CFDB_OK;
}
