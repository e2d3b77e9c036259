// Krylov solves on a structured stencil matrix (diagonal + up to six
// neighbour couplings per row): BiCGSTAB with the reference's breakdown and
// restart semantics (src/algebra/BiCGSTAB.cpp:48-275) and CG
// (src/algebra/CG.cpp:14-148), optional Jacobi, as one persistent cooperative
// kernel per solve whose whole grid runs the routine of stencil_krylov.cuh.  These serve the momentum systems (non-symmetric, a few
// iterations per outer step from a warm start) and the p' system when a case
// asks for BiCGSTAB; the bandwidth-critical p' CG runs in pcg.cu.
//
// Layout: cell c = i + nx*(j + ny*k); off[2a] couples to the low neighbour
// along axis a, off[2a+1] to the high one (0 at the domain edge).  Row sums
// follow the reference's CSR column order (SparseMatrix.cpp:93-100).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "cfdb.h"
#include "cfdb_internal.cuh"
#include "grid_sync.cuh"
#include "stencil_krylov.cuh"
#include "stencil_solve.cuh"

namespace cfdb {
namespace {

using krylov::kThreads;
using krylov::SParams;
using krylov::O_STATUS;
using krylov::O_ITER;
using krylov::O_B0;
using krylov::O_FINAL;
using krylov::O_RESTARTS;
constexpr unsigned long long kTimeoutNs = 2000000000ull;

// The whole grid is one team.
struct GridTeam {
  GridSync s;
  __device__ int rank() const { return blockIdx.x; }
  __device__ int size() const { return gridDim.x; }
  __device__ bool sync() const { return grid_sync(s); }
};

// Four resident blocks per SM (64 registers): the 256^3 cavity's outer
// iteration takes 111 ms with two, 97 ms with three and 92 ms with four.
__global__ void __launch_bounds__(kThreads, 4) stencil_krylov(SParams P, GridSync sync) {
  const GridTeam T{sync};
  krylov::krylov_run(P, T);
}

__global__ void k_inverse_diag(int64_t n, const double* diag, double* inv, unsigned* bad) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const double d = diag[c];
    if (!isfinite(d) || d == 0.0 || fabs(d) < 1.0e-12) atomicExch(bad, 1u);
    inv[c] = 1.0 / d;
  }
}

__global__ void k_matrix_finite(StencilMatrix M, const double* b, const double* x, unsigned* bad) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < M.n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % M.nx), j = (int)((c / M.nx) % M.ny), k = (int)(c / M.sz);
    bool ok = isfinite(M.diag[c]) && isfinite(b[c]) && isfinite(x[c]);
    if (i > 0) ok = ok && isfinite(M.off[0][c]);
    if (i < M.nx - 1) ok = ok && isfinite(M.off[1][c]);
    if (j > 0) ok = ok && isfinite(M.off[2][c]);
    if (j < M.ny - 1) ok = ok && isfinite(M.off[3][c]);
    if (M.dim == 3 && k > 0) ok = ok && isfinite(M.off[4][c]);
    if (M.dim == 3 && k < M.nz - 1) ok = ok && isfinite(M.off[5][c]);
    if (!ok) atomicExch(bad, 1u);
  }
}

}  // namespace

cfdb_status stencil_solve(cfdb_context* ctx, const StencilMatrix& Min, StencilWork& W,
                          const double* b, double* x, int krylov, int jacobi, double abs_tol,
                          double rel_tol, int64_t max_it, double* hist_dev, int64_t hist_cap,
                          cfdb_linear_result* res) {
  std::memset(res, 0, sizeof(*res));
  const int64_t n = Min.n;
  if (W.n < n) {
    W.release();
    for (double** q : {&W.r, &W.rh, &W.v, &W.p, &W.s, &W.t, &W.inv}) {
      cudaError_t e = cudaMalloc((void**)q, sizeof(double) * (size_t)n);
      if (e != cudaSuccess) return cuda_error(ctx, e, "stencil work", __FILE__, __LINE__);
    }
    W.n = n;
  }
  StencilMatrix M = Min;
  const int g = (int)std::min<int64_t>((n + 255) / 256, 4096);
  // NonFiniteInput (BiCGSTAB.cpp:57-60) and the Jacobi build (InvalidSystem)
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->sync_words + 4, 0, 2 * sizeof(unsigned), ctx->stream));
  k_matrix_finite<<<std::max(g, 1), 256, 0, ctx->stream>>>(M, b, x, ctx->sync_words + 4);
  if (jacobi) k_inverse_diag<<<std::max(g, 1), 256, 0, ctx->stream>>>(n, M.diag, W.inv, ctx->sync_words + 5);
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx, jacobi ? 2 : 1);
  unsigned flags[2] = {0, 0};
  CFDB_CUDA(ctx, cudaMemcpyAsync(flags, ctx->sync_words + 4, 2 * sizeof(unsigned),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (flags[0]) {
    res->status = CFDB_SOLVER_NONFINITE_INPUT;
    return CFDB_OK;
  }
  if (jacobi && flags[1]) {
    res->status = CFDB_SOLVER_INVALID_SYSTEM;
    return CFDB_OK;
  }
  M.inv = jacobi ? W.inv : nullptr;
  SParams P{};
  P.M = M;
  P.b = b;
  P.x = x;
  P.r = W.r;
  P.rh = W.rh;
  P.v = W.v;
  P.p = W.p;
  P.s = W.s;
  P.t = W.t;
  P.krylov = krylov;
  P.jacobi = jacobi;
  P.abs_tol = abs_tol;
  P.rel_tol = rel_tol;
  P.max_it = max_it;
  P.hist = hist_dev;
  P.hist_cap = hist_dev ? hist_cap : 0;
  int per_sm = 0;
  CFDB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stencil_krylov, kThreads, 0));
  int64_t grid = std::min<int64_t>((int64_t)std::max(per_sm, 1) * ctx->num_sms, (n + kThreads - 1) / kThreads);
  grid = std::max<int64_t>(grid, 1);
  cfdb_status st = ensure_partials(ctx, 6 * (size_t)grid);
  if (st != CFDB_OK) return st;
  P.partials = ctx->partials;
  GridSync sync;
  sync.count = ctx->sync_words;
  sync.gen = ctx->sync_words + 1;
  sync.error = ctx->sync_words + 2;
  sync.nblocks = (unsigned)grid;
  sync.timeout_ns = kTimeoutNs;
  P.out = ctx->scalars;
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->sync_words, 0, 4 * sizeof(unsigned), ctx->stream));
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->scalars, 0, 8 * sizeof(double), ctx->stream));
  void* args[] = {&P, &sync};
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_k0, ctx->stream));
  CFDB_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)stencil_krylov, dim3((unsigned)grid),
                                             dim3(kThreads), args, 0, ctx->stream));
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_k1, ctx->stream));
  count_launch(ctx);
  CFDB_CUDA(ctx, cudaMemcpyAsync(ctx->scalars_host, ctx->scalars, 8 * sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  unsigned err = 0;
  CFDB_CUDA(ctx, cudaMemcpyAsync(&err, ctx->sync_words + 2, sizeof(unsigned),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (err)
    return set_error(ctx, CFDB_ERR_DEVICE_TIMEOUT,
                     "a grid barrier of the stencil Krylov solver timed out (no fault)");
  const double* o = ctx->scalars_host;
  res->status = (int)o[O_STATUS];
  res->iterations = (int64_t)o[O_ITER];
  res->initial_residual = o[O_B0];
  res->final_residual = o[O_FINAL];
  res->restarts = (int64_t)o[O_RESTARTS];
  float ms = 0.f;
  CFDB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev_k0, ctx->ev_k1));
  res->krylov_ms = ms;
  res->krylov_launches = 1;
  res->kernel_launches = jacobi ? 3 : 2;
  return CFDB_OK;
}

void StencilWork::release() {
  for (double** q : {&r, &rh, &v, &p, &s, &t, &inv}) {
    cudaFree(*q);
    *q = nullptr;
  }
  n = 0;
}

}  // namespace cfdb
