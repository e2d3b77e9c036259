// TMA (cp.async.bulk.tensor) helpers for the p' kernels: tensor-map creation
// on the host through the driver entry point, and device-side mbarrier
// waits with a wall-clock bound (a wait never spins forever: on timeout the
// shared error flag is raised and the caller returns).
//
// Only plain (non-multicast) tiled loads from this GPU's own memory are used.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "grid_sync.cuh"

namespace cfdb {

// -------------------------------------------------------------------- host
// Encodes a tiled tensor map of `rank` (2 or 3) over a dense array whose
// innermost dimension is dims[0].  Returns false if the driver rejects it.
bool encode_tensor_map(CUtensorMap* map, CUtensorMapDataType dtype, int elem_bytes, int rank,
                       const void* base, const uint64_t* dims, const uint32_t* box);

// ------------------------------------------------------------------ device
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait on phase `parity` of `bar`; false (and the error flag raised)
// when the bound passes or another block already failed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned* error,
                                          unsigned long long timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (*(volatile unsigned*)error != 0u) return false;
    if (global_ns() - t0 > timeout_ns) {
      atomicExch(error, 1u);
      return false;
    }
  }
  return true;
}

// Bounded wait on phase `parity` of `bar` that ignores the error flag: a
// block that gives up on an error first lets the bulk copies it issued into
// its shared memory land, so that none is still writing when the block
// exits.  Returns at the latest after timeout_ns.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity,
                                           unsigned long long timeout_ns) {
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > timeout_ns) return;
}

// Orders this thread's earlier generic-proxy accesses of shared memory before
// subsequent async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace cfdb
