// Bounded grid-wide barrier and deterministic reductions for the persistent
// (cooperatively launched) kernels.
//
// The barrier is a generation counter: every block's leader fences its
// writes, arrives on an atomic counter, and the last arrival resets the
// counter and bumps the generation.  Waiters poll the generation with a
// wall-clock limit read from %globaltimer; when the limit passes, or another
// block already gave up, the waiter raises the shared error flag and returns
// false so that the kernel can exit cleanly -- a wait never spins forever.
//
// Data written by other blocks before a barrier is read after it with
// ld.global.cg (L2, bypassing the non-coherent L1): see ldcg() uses.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace cfdb {

struct GridSync {
  unsigned* count;
  unsigned* gen;
  unsigned* error;
  unsigned nblocks;
  unsigned long long timeout_ns;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Returns false when the barrier timed out (here or in another block).
__device__ __forceinline__ bool grid_sync(const GridSync& s) {
  __shared__ int ok_shared;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    volatile unsigned* vgen = s.gen;
    volatile unsigned* verr = s.error;
    const unsigned g = *vgen;
    // Global data this block wrote with ordinary stores may be read after the
    // barrier by TMA (the async proxy) in other blocks: proxy fence first.
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __threadfence();
    const unsigned prev = atomicAdd(s.count, 1u);
    int good = (*verr == 0u);
    if (prev == s.nblocks - 1) {
      atomicExch(s.count, 0u);
      __threadfence();
      atomicAdd(s.gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      while (*vgen == g) {
        if (*verr != 0u) {
          good = 0;
          break;
        }
        if (global_ns() - t0 > s.timeout_ns) {
          atomicExch(s.error, 1u);
          good = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    asm volatile("fence.proxy.async.global;" ::: "memory");
    ok_shared = good;
  }
  __syncthreads();
  return ok_shared != 0;
}

// Block-wide sum of NV doubles per thread, fixed order (deterministic).
// Result valid in every thread.  `scratch` holds >= 32*NV doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthreads = blockDim.x * blockDim.y;
  const int lane = tid & 31, warp = tid >> 5, nwarps = (nthreads + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) scratch[warp * NV + q] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = 0.0;
    for (int w = 0; w < nwarps; ++w) s += scratch[w * NV + q];
    v[q] = s;
  }
  __syncthreads();
}

// Sum of partials[b*stride + q] over b in [0, nblocks) for q < NV, in a fixed
// order identical in every block (so every block derives bitwise-identical
// scalars).  Uses warp 0; the result is broadcast through shared memory.
template <int NV>
__device__ __forceinline__ void grid_total(const double* partials, int stride, int nblocks,
                                           double (&out)[NV], double* scratch) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  if (tid < 32) {
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = 0.0;
    for (int b = tid; b < nblocks; b += 32)
#pragma unroll
      for (int q = 0; q < NV; ++q) acc[q] += __ldcg(partials + (size_t)b * stride + q);
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    if (tid == 0)
#pragma unroll
      for (int q = 0; q < NV; ++q) scratch[q] = acc[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) out[q] = scratch[q];
  __syncthreads();
}

}  // namespace cfdb
