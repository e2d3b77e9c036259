// Context management, error reporting, device memory helpers and the
// synthetic-workload generator of the cfdb C ABI.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cfdb.h"
#include "cfdb_internal.cuh"

namespace cfdb {

cfdb_status set_error(cfdb_context* ctx, cfdb_status code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return code;
}

cfdb_status cuda_error(cfdb_context* ctx, cudaError_t err, const char* what, const char* file,
                       int line) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(err), file, line);
  cfdb_status code = (err == cudaErrorMemoryAllocation) ? CFDB_ERR_OUT_OF_MEMORY : CFDB_ERR_CUDA;
  return set_error(ctx, code, buf);
}

cfdb_status ensure_partials(cfdb_context* ctx, size_t doubles) {
  if (ctx->partials_cap >= doubles) return CFDB_OK;
  if (ctx->partials) cudaFree(ctx->partials);
  ctx->partials = nullptr;
  ctx->partials_cap = 0;
  const size_t cap = doubles < 4096 ? 4096 : doubles;
  CFDB_CUDA(ctx, cudaMalloc((void**)&ctx->partials, cap * sizeof(double)));
  ctx->partials_cap = cap;
  return CFDB_OK;
}

}  // namespace cfdb

using namespace cfdb;

extern "C" {

int cfdb_cuda_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
    cudaGetLastError();
    return 0;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return prop.major == 10 ? 1 : 0;
}

cfdb_status cfdb_create(int device, void* stream, cfdb_context** out) {
  if (!out) return CFDB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return CFDB_ERR_NO_DEVICE;
  }
  auto* ctx = new cfdb_context();
  ctx->device = device;
  auto fail = [&](cudaError_t e, const char* what) {
    std::fprintf(stderr, "cfdb_create: %s: %s\n", what, cudaGetErrorString(e));
    cfdb_destroy(ctx);
    return e == cudaErrorMemoryAllocation ? CFDB_ERR_OUT_OF_MEMORY : CFDB_ERR_CUDA;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return fail(e, "cudaGetDeviceProperties");
  if (prop.major != 10) {
    cfdb_destroy(ctx);
    return CFDB_ERR_NO_DEVICE;  // built for sm_100a only
  }
  ctx->num_sms = prop.multiProcessorCount;
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
  } else {
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e, "cudaStreamCreate");
    ctx->own_stream = true;
  }
  if ((e = cudaMalloc((void**)&ctx->sync_words, 16 * sizeof(unsigned))) != cudaSuccess)
    return fail(e, "cudaMalloc");
  // on the context's (non-blocking) stream, then waited for, so that no later
  // work of the context can run ahead of the clear
  if ((e = cudaMemsetAsync(ctx->sync_words, 0, 16 * sizeof(unsigned), ctx->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return fail(e, "cudaMemsetAsync");
  if ((e = cudaMalloc((void**)&ctx->scalars, 64 * sizeof(double))) != cudaSuccess)
    return fail(e, "cudaMalloc");
  if ((e = cudaMallocHost((void**)&ctx->scalars_host, 64 * sizeof(double))) != cudaSuccess)
    return fail(e, "cudaMallocHost");
  if ((e = cudaEventCreate(&ctx->ev_start)) != cudaSuccess) return fail(e, "cudaEventCreate");
  if ((e = cudaEventCreate(&ctx->ev_stop)) != cudaSuccess) return fail(e, "cudaEventCreate");
  if ((e = cudaEventCreate(&ctx->ev_k0)) != cudaSuccess) return fail(e, "cudaEventCreate");
  if ((e = cudaEventCreate(&ctx->ev_k1)) != cudaSuccess) return fail(e, "cudaEventCreate");
  if (ensure_partials(ctx, 4096) != CFDB_OK) {
    cfdb_destroy(ctx);
    return CFDB_ERR_OUT_OF_MEMORY;
  }
  *out = ctx;
  return CFDB_OK;
}

void cfdb_destroy(cfdb_context* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->partials);
  cudaFree(ctx->sync_words);
  cudaFree(ctx->scalars);
  if (ctx->scalars_host) cudaFreeHost(ctx->scalars_host);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  if (ctx->ev_k0) cudaEventDestroy(ctx->ev_k0);
  if (ctx->ev_k1) cudaEventDestroy(ctx->ev_k1);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->mg_weights_free) ctx->mg_weights_free(ctx->mg_weights);
  delete ctx;
}

const char* cfdb_last_error(const cfdb_context* ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

void* cfdb_stream(cfdb_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t cfdb_kernel_launches(const cfdb_context* ctx) { return ctx ? ctx->launches : 0; }

// SplitMix64 (Steele, Lea & Flood 2014) and the generator described in
// cfdb.h; the same definition as the oracle's, written out here so the
// product does not depend on test infrastructure.
static uint64_t splitmix64(uint64_t* s) {
  uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

cfdb_status cfdb_synth_rhs(int64_t nx, int64_t ny, int64_t nz, uint64_t seed, double* b) {
  if (nx < 1 || ny < 1 || nz < 0 || !b) return CFDB_ERR_INVALID_ARGUMENT;
  const double pi = 3.14159265358979323846;
  const bool dim3 = nz > 0;
  const int64_t nzz = dim3 ? nz : 1;
  const int64_t n = nx * ny * nzz;
  std::vector<double> cx(nx), cy(ny), cz(nzz);
  for (int64_t i = 0; i < n; ++i) b[i] = 0.0;
  uint64_t s = seed;
  for (int m = 0; m < 32; ++m) {
    const double kx = (double)(1 + (splitmix64(&s) >> 58));
    const double ky = (double)(1 + (splitmix64(&s) >> 58));
    const double kz = dim3 ? (double)(1 + (splitmix64(&s) >> 58)) : 0.0;
    const double phx = (double)(splitmix64(&s) >> 11) * 0x1.0p-53 * (2.0 * pi);
    const double phy = (double)(splitmix64(&s) >> 11) * 0x1.0p-53 * (2.0 * pi);
    const double phz = dim3 ? (double)(splitmix64(&s) >> 11) * 0x1.0p-53 * (2.0 * pi) : 0.0;
    const double a = 1.0 / (kx * kx + ky * ky + kz * kz);
    for (int64_t i = 0; i < nx; ++i) cx[i] = std::cos(pi * kx * (((double)i + 0.5) / (double)nx) + phx);
    for (int64_t j = 0; j < ny; ++j) cy[j] = std::cos(pi * ky * (((double)j + 0.5) / (double)ny) + phy);
    if (dim3)
      for (int64_t k = 0; k < nz; ++k)
        cz[k] = std::cos(pi * kz * (((double)k + 0.5) / (double)nz) + phz);
    for (int64_t k = 0; k < nzz; ++k)
      for (int64_t j = 0; j < ny; ++j) {
        double* row = b + (k * ny + j) * nx;
        for (int64_t i = 0; i < nx; ++i) {
          double t = (a * cx[i]) * cy[j];
          if (dim3) t = t * cz[k];
          row[i] += t;
        }
      }
  }
  double sum = 0.0;
  for (int64_t i = 0; i < n; ++i) sum += b[i];
  const double mean = sum / (double)n;
  const double vol = dim3 ? 1.0 / ((double)nx * (double)ny * (double)nz) : 1.0 / ((double)nx * (double)ny);
  for (int64_t i = 0; i < n; ++i) b[i] = vol * b[i] - vol * mean;
  b[0] = 0.0;
  return CFDB_OK;
}

cfdb_status cfdb_device_alloc(cfdb_context* ctx, size_t bytes, void** out) {
  if (!ctx || !out) return CFDB_ERR_INVALID_ARGUMENT;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  CFDB_CUDA(ctx, cudaMalloc(out, bytes));
  return CFDB_OK;
}

cfdb_status cfdb_device_free(cfdb_context* ctx, void* ptr) {
  if (!ctx) return CFDB_ERR_INVALID_ARGUMENT;
  CFDB_CUDA(ctx, cudaFree(ptr));
  return CFDB_OK;
}

cfdb_status cfdb_copy_to_device(cfdb_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx) return CFDB_ERR_INVALID_ARGUMENT;
  CFDB_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

cfdb_status cfdb_copy_to_host(cfdb_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!ctx) return CFDB_ERR_INVALID_ARGUMENT;
  CFDB_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

cfdb_status cfdb_memset_device(cfdb_context* ctx, void* dst, int value, size_t bytes) {
  if (!ctx) return CFDB_ERR_INVALID_ARGUMENT;
  CFDB_CUDA(ctx, cudaMemsetAsync(dst, value, bytes, ctx->stream));
  return CFDB_OK;
}

cfdb_status cfdb_synchronize(cfdb_context* ctx) {
  if (!ctx) return CFDB_ERR_INVALID_ARGUMENT;
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

}  // extern "C"
