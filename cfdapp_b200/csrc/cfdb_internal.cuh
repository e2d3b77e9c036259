// Internal definitions shared by the cfdb CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "cfdb.h"

struct cfdb_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 0;
  std::string last_error;
  int64_t launches = 0;
  // Scratch of the persistent kernels: per-block partial sums, the grid
  // barrier words and device-side status, allocated once per context.
  double* partials = nullptr;
  size_t partials_cap = 0;  // doubles
  unsigned* sync_words = nullptr;  // [0] arrival count [1] generation [2] error flag
  double* scalars = nullptr;       // device scalars written by kernels (64 doubles)
  double* scalars_host = nullptr;  // pinned mirror
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  cudaEvent_t ev_k0 = nullptr, ev_k1 = nullptr;  // around persistent kernel launches
  // Learned-preconditioner weights of this context (owned; see mg.cu).
  void* mg_weights = nullptr;
  void (*mg_weights_free)(void*) = nullptr;
};

namespace cfdb {

cfdb_status set_error(cfdb_context* ctx, cfdb_status code, const std::string& msg);
cfdb_status cuda_error(cfdb_context* ctx, cudaError_t err, const char* what, const char* file,
                       int line);
// Grows the per-block partials scratch to at least `doubles` entries.
cfdb_status ensure_partials(cfdb_context* ctx, size_t doubles);

inline void count_launch(cfdb_context* ctx, int n = 1) { ctx->launches += n; }

}  // namespace cfdb

#define CFDB_CUDA(ctx, call)                                                   \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) return cfdb::cuda_error((ctx), e_, #call, __FILE__, __LINE__); \
  } while (0)

#define CFDB_CHECK_LAUNCH(ctx)                                                 \
  do {                                                                         \
    cudaError_t e_ = cudaGetLastError();                                       \
    if (e_ != cudaSuccess) return cfdb::cuda_error((ctx), e_, "kernel launch", __FILE__, __LINE__); \
  } while (0)
