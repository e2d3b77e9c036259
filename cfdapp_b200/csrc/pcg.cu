// p' operator objects and their Krylov solves.
//
// The plain method is the reference's Jacobi-preconditioned CG
// (src/algebra/CG.cpp:14-148, JacobiPreconditioner src/algebra/Preconditioner.cpp:11-49)
// with its exact status and convergence semantics, run as ONE persistent
// cooperative kernel per solve: two fused sweeps per iteration
//   sweep A: p = D^-1 r + beta p_old (computed on the fly, halo included),
//            Ap = A p, partial p.Ap, store p
//   sweep B: x += alpha p, r -= alpha A p (A p recomputed from p),
//            partial r.r and r.z (z = D^-1 r)
// separated by bounded grid barriers; every block derives alpha/beta from the
// same fixed-order sum of the per-block partials, so the whole solve runs on
// the device with no host round trip (the reference synchronises and sums on
// the host once per reduction, DeviceVectorOpsKernel.cu:226-260).
//
// The FP32-refined method runs the same kernel in FP32 (FP64 reductions)
// inside FP64 iterative refinement: r = b - A x in FP64 (fused with the update
// x += e), inner PCG on A e = r in FP32 to a moderate reduction, repeat until
// the FP64 true residual meets the tolerance.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "cfdb.h"
#include "cfdb_internal.cuh"
#include "grid_sync.cuh"
#include "mg.cuh"
#include "pcg_internal.cuh"
#include "poperator.cuh"
#include "tile.cuh"
#include "tma.cuh"

struct cfdb_poperator {
  cfdb_context* ctx = nullptr;
  cfdb_grid grid{};
  int knx = 0, kny = 0, knz = 0;  // kernel-space extents
  int64_t cells = 0;
  int pinned = 0;
  int64_t ref = 0;
  // FP64 and FP32 copies of the coefficients (tables always; faces optional)
  double* t64[3] = {nullptr, nullptr, nullptr};
  float* t32[3] = {nullptr, nullptr, nullptr};
  double* f64[3] = {nullptr, nullptr, nullptr};
  float* f32[3] = {nullptr, nullptr, nullptr};
  // work vectors, allocated on first solve
  double* w64[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // r p0 p1 xalt b x (host staging) z
  float* w32[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};   // r p0 p1 e b32 z
  double* hist_dev = nullptr;
  int64_t hist_cap = 0;
  double* invd64 = nullptr;  // 1/diag, face-coefficient operators only
  float* invd32 = nullptr;
  bool faces_borrowed = false;  // f64[] point into a caller's device array
  uint64_t version = 1;         // bumped whenever the coefficients change
  cfdb::LearnedSolver* learned = nullptr;
};

namespace cfdb {
namespace {

constexpr int kThreads = 256;
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s per barrier wait

enum { OUT_STATUS = 0, OUT_ITER = 1, OUT_B0 = 2, OUT_FINAL = 3, OUT_PCUR = 4, OUT_TIMEOUT = 5,
       OUT_REPLACEMENTS = 6 };

template <typename T>
OpView<T> view(const cfdb_poperator* op) {
  OpView<T> v;
  v.nx = op->knx;
  v.ny = op->kny;
  v.nz = op->knz;
  if constexpr (sizeof(T) == 8) {
    v.tx = op->t64[0]; v.ty = op->t64[1]; v.tz = op->t64[2];
    v.fx = op->f64[0]; v.fy = op->f64[1]; v.fz = op->f64[2];
  } else {
    v.tx = op->t32[0]; v.ty = op->t32[1]; v.tz = op->t32[2];
    v.fx = op->f32[0]; v.fy = op->f32[1]; v.fz = op->f32[2];
  }
  v.ref = op->ref;
  v.pinned = op->pinned;
  return v;
}

template <typename T>
struct PcgParams {
  OpView<T> A;
  ColumnSplit cs;
  const T* invd;  // precomputed 1/diag (face-coefficient operators) or null
  const T* b;
  T* x;
  T* r;
  T* p0;
  T* p1;
  T* z;  // D^-1 r, written by the TMA kernel's residual sweeps for its next direction sweep
  int x0_zero;
  double abs_tol, rel_tol;
  int64_t max_it;
  double* hist;
  int64_t hist_cap;
  double* partials;
  GridSync sync;
  double* out;
  // mixed precision (T = float): the iterate, residual and right-hand side
  // live in FP64 (x64, r64, b64) and the stencil arithmetic uses the FP64
  // coefficients (A64); p and z are stored in FP32.  The residual is
  // replaced by the FP64 b - A x whenever it has fallen by `delta` since
  // the last replacement, when it reaches the tolerance, and at the
  // iteration cap.
  OpView<double> A64;
  const double* b64;
  double* x64;
  double* r64;
  double delta;
};

__device__ __forceinline__ bool finite(double v) { return isfinite(v); }

template <typename T>
__device__ __forceinline__ T inv_at(const OpView<T>& A, const T* invd, int i, int j, int k) {
  if (invd) return __ldg(invd + (i + (int64_t)A.nx * (j + (int64_t)A.ny * k)));
  return load_coef(A, i, j, k).inv;
}

template <typename T, class S>
__global__ void __launch_bounds__(kThreads, 2) pcg_persistent(PcgParams<T> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* box = reinterpret_cast<T*>(smem_raw);
  __shared__ double red[64];
  const OpView<T>& A = P.A;
  const int B = gridDim.x, blk = blockIdx.x;
  const bool leader = (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0);
  const ColumnSplit cs = P.cs;
  // Partials are double-buffered by reduction round: a block that already
  // summed round k and raced ahead writes round k+1 into the other half while
  // slower blocks may still be reading round k.
  int round = 0;
  auto part = [&]() { return P.partials + (size_t)(round & 1) * 2 * B; };

  // ---- r0 = b - A x0, ||r0||^2, r0.z0
  double acc[2] = {0.0, 0.0};
  for_chunks<S>(cs, A.nz, blk, B, [&](const Chunk& c) {
    if (!P.x0_zero) {
      stage_box<S, 8>(A, c, box, [&](int, int, int, int64_t idx) { return P.x[idx]; },
                      [&](T v, int, int, int) { return v; });
      __syncthreads();
    }
    for_interior<S, 8>(A, c, [&](int64_t idx) { return __ldg(P.b + idx); },
                       [&](int i, int j, int k, int64_t idx, int e, T bv) {
      const Coef<T> cf = load_coef(A, i, j, k);
      T rn = bv;
      if (!P.x0_zero) rn = rn - apply_box<S>(cf, box, e);
      P.r[idx] = rn;
      const double rd = (double)rn;
      acc[0] += rd * rd;
      acc[1] += rd * (double)(cf.inv * rn);
    });
    __syncthreads();
  });
  block_sum<2>(acc, red);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    part()[2 * blk] = acc[0];
    part()[2 * blk + 1] = acc[1];
  }
  if (!grid_sync(P.sync)) return;
  double tot[2];
  grid_total<2>(part(), 2, B, tot, red);
  ++round;
  const double b0 = sqrt(tot[0]);
  double rz = tot[1];
  auto converged = [&](double res) {
    return (res <= P.abs_tol) || ((b0 > 0.0) && (res / b0 <= P.rel_tol));
  };
  if (leader) {
    P.out[OUT_B0] = b0;
    if (P.hist_cap > 0) P.hist[0] = b0;
  }
  if (b0 == 0.0 || converged(b0)) {
    if (leader) {
      P.out[OUT_STATUS] = CFDB_SOLVER_CONVERGED;
      P.out[OUT_ITER] = 0;
      P.out[OUT_FINAL] = b0;
    }
    return;
  }
  if (!finite(rz)) {
    if (leader) {
      P.out[OUT_STATUS] = CFDB_SOLVER_BREAKDOWN;
      P.out[OUT_ITER] = 0;
      P.out[OUT_FINAL] = b0;
    }
    return;
  }

  double res_cur = b0;
  double beta = 0.0;
  T* pold = P.p0;
  T* pnew = P.p1;
  for (int64_t it = 1; it <= P.max_it; ++it) {
    const bool first = (it == 1);
    const T tbeta = (T)beta;
    // ---- sweep A: stage p = D^-1 r + beta p_old over chunk + halo; Ap; p.Ap
    double pap = 0.0;
    for_chunks<S>(cs, A.nz, blk, B, [&](const Chunk& c) {
      stage_box<S, 6>(
          A, c, box,
          [&](int, int, int, int64_t idx) {
            Pair<T> v;
            v.a = __ldcg(P.r + idx);
            v.b = first ? T(0) : __ldcg(pold + idx);
            return v;
          },
          [&](Pair<T> v, int i, int j, int k) {
            const T z = inv_at(A, P.invd, i, j, k) * v.a;
            return first ? z : fma(tbeta, v.b, z);
          });
      __syncthreads();
      for_interior<S, 1>(A, c, [&](int64_t) { return 0; },
                         [&](int i, int j, int k, int64_t idx, int e, int) {
        const Coef<T> cf = load_coef(A, i, j, k);
        const T v = box[e];
        const T ap = apply_box<S>(cf, box, e);
        pnew[idx] = v;
        pap += (double)v * (double)ap;
      });
      __syncthreads();
    });
    {
      double a1[1] = {pap};
      block_sum<1>(a1, red);
      if (threadIdx.x == 0 && threadIdx.y == 0) part()[2 * blk] = a1[0];
    }
    if (!grid_sync(P.sync)) return;
    double t1[1];
    grid_total<1>(part(), 2, B, t1, red);
    ++round;
    const double pAp = t1[0];
    const double alpha = rz / pAp;
    if (!finite(pAp) || fabs(pAp) < 1.0e-30 || !finite(alpha)) {
      if (leader) {
        P.out[OUT_STATUS] = CFDB_SOLVER_BREAKDOWN;
        P.out[OUT_ITER] = (double)(it - 1);
        P.out[OUT_FINAL] = res_cur;
      }
      return;
    }
    const T talpha = (T)alpha;
    // ---- sweep B: x += alpha p; r -= alpha A p; r.r, r.z
    double ab[2] = {0.0, 0.0};
    for_chunks<S>(cs, A.nz, blk, B, [&](const Chunk& c) {
      stage_box<S, 8>(A, c, box, [&](int, int, int, int64_t idx) { return __ldcg(pnew + idx); },
                      [&](T v, int, int, int) { return v; });
      __syncthreads();
      for_interior<S, 6>(
          A, c,
          [&](int64_t idx) {
            Pair<T> v;
            v.a = P.x[idx];
            v.b = P.r[idx];
            return v;
          },
          [&](int i, int j, int k, int64_t idx, int e, Pair<T> xr) {
        const Coef<T> cf = load_coef(A, i, j, k);
        const T ap = apply_box<S>(cf, box, e);
        P.x[idx] = fma(talpha, box[e], xr.a);
        const T rn = fma(-talpha, ap, xr.b);
        P.r[idx] = rn;
        const double rd = (double)rn;
        ab[0] += rd * rd;
        ab[1] += rd * (double)(cf.inv * rn);
      });
      __syncthreads();
    });
    block_sum<2>(ab, red);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      part()[2 * blk] = ab[0];
      part()[2 * blk + 1] = ab[1];
    }
    if (!grid_sync(P.sync)) return;
    grid_total<2>(part(), 2, B, tot, red);
    ++round;
    const double res = sqrt(tot[0]);
    if (leader && it < P.hist_cap) P.hist[it] = res;
    if (!finite(res)) {
      if (leader) {
        P.out[OUT_STATUS] = CFDB_SOLVER_NONFINITE_RESIDUAL;
        P.out[OUT_ITER] = (double)it;
        P.out[OUT_FINAL] = res;
      }
      return;
    }
    res_cur = res;
    if (converged(res)) {
      if (leader) {
        P.out[OUT_STATUS] = CFDB_SOLVER_CONVERGED;
        P.out[OUT_ITER] = (double)it;
        P.out[OUT_FINAL] = res;
      }
      return;
    }
    const double rzNew = tot[1];
    beta = rzNew / rz;
    if (!finite(rzNew) || !finite(beta)) {
      if (leader) {
        P.out[OUT_STATUS] = CFDB_SOLVER_BREAKDOWN;
        P.out[OUT_ITER] = (double)it;
        P.out[OUT_FINAL] = res;
      }
      return;
    }
    rz = rzNew;
    T* tmp = pold;
    pold = pnew;
    pnew = tmp;
  }
  if (leader) {
    P.out[OUT_STATUS] = CFDB_SOLVER_MAX_ITERATIONS;
    P.out[OUT_ITER] = (double)P.max_it;
    P.out[OUT_FINAL] = res_cur;
  }
}

// Inverse diagonal of a face-coefficient operator (computed once per operator).
template <typename T>
__global__ void inverse_diagonal(OpView<T> A, T* invd) {
  const int64_t n = (int64_t)A.nx * A.ny * A.nz;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % A.nx);
    const int j = (int)((q / A.nx) % A.ny);
    const int k = (int)(q / ((int64_t)A.nx * A.ny));
    invd[q] = load_coef(A, i, j, k).inv;
  }
}

#include "pcg_tma.cuh"

// FP64 residual pass of the refinement: x_out = x_in + scale * e (e may be
// null), r = b - A x_out; optionally r32 = (float) r; per-block ||r||^2.
template <int PY>
__global__ void __launch_bounds__(kThreads) refine_residual(OpView<double> A, Tiling tl,
                                                            const double* b, const double* x_in,
                                                            double* x_out, const float* e,
                                                            double scale, float* r32,
                                                            double* r64, double* partials) {
  constexpr int PX = kThreads / PY;
  __shared__ double buf[2][PY + 2][PX + 2];
  __shared__ double red[64];
  double acc[1] = {0.0};
  auto value = [&](int i, int j, int k) {
    const int64_t idx = i + (int64_t)A.nx * (j + (int64_t)A.ny * k);
    double v = __ldg(x_in + idx);
    if (e) v = fma(scale, (double)__ldg(e + idx), v);
    return v;
  };
  for_segments(tl, A.nz, blockIdx.x, gridDim.x, [&](int64_t tile, int k0, int k1) {
    march<double, PX, PY>(
        A, tl, tile, k0, k1, buf,
        value, value,
        [&](int i, int j, int k, int64_t idx, double v, double w, double ee, double s, double n,
            double bb, double t) {
          const Coef<double> c = load_coef(A, i, j, k);
          if (x_out) x_out[idx] = v;
          const double rn = __ldg(b + idx) - apply_coef(c, v, w, ee, s, n, bb, t);
          if (r32) r32[idx] = (float)rn;
          if (r64) r64[idx] = rn;
          acc[0] += rn * rn;
        });
  });
  block_sum<1>(acc, red);
  if (threadIdx.x == 0 && threadIdx.y == 0) partials[blockIdx.x] = acc[0];
}

// One block: out[slot] = sum of partials[0..n) in fixed order.
__global__ void sum_partials(const double* partials, int n, double* out, int slot) {
  __shared__ double red[64];
  double a[1] = {0.0};
  for (int q = threadIdx.x; q < n; q += blockDim.x) a[0] += partials[q];
  block_sum<1>(a, red);
  if (threadIdx.x == 0) out[slot] = a[0];
}

// y = A x (FP64).
template <int PY>
__global__ void __launch_bounds__(kThreads) apply_kernel(OpView<double> A, Tiling tl,
                                                         const double* x, double* y) {
  constexpr int PX = kThreads / PY;
  __shared__ double buf[2][PY + 2][PX + 2];
  auto value = [&](int i, int j, int k) {
    return __ldg(x + (i + (int64_t)A.nx * (j + (int64_t)A.ny * k)));
  };
  for_segments(tl, A.nz, blockIdx.x, gridDim.x, [&](int64_t tile, int k0, int k1) {
    march<double, PX, PY>(
        A, tl, tile, k0, k1, buf,
        value, value,
        [&](int i, int j, int k, int64_t idx, double v, double w, double e, double s, double n,
            double bb, double t) {
          const Coef<double> c = load_coef(A, i, j, k);
          y[idx] = apply_coef(c, v, w, e, s, n, bb, t);
        });
  });
}

__global__ void all_finite(const double* v, int64_t n, unsigned* flag) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(v[q])) atomicExch(flag, 1u);
}

// ------------------------------------------------------------------ host side

bool is3d(const cfdb_poperator* op) { return op->grid.dim == 3; }

template <typename T, class S>
cfdb_status launch_pcg(cfdb_context* ctx, PcgParams<T>& P) {
  auto kernel = pcg_persistent<T, S>;
  const size_t smem = sizeof(T) * (size_t)S::BOX;
  CFDB_CUDA(ctx, cudaFuncSetAttribute((const void*)kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  CFDB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem));
  if (per_sm < 1) return set_error(ctx, CFDB_ERR_CUDA, "pcg kernel cannot be resident");
  int64_t grid = (int64_t)per_sm * ctx->num_sms;
  grid = std::min<int64_t>(grid, P.cs.items);
  grid = std::max<int64_t>(grid, 1);
  cfdb_status st = ensure_partials(ctx, 4 * (size_t)grid);
  if (st != CFDB_OK) return st;
  P.partials = ctx->partials;
  P.sync.count = ctx->sync_words;
  P.sync.gen = ctx->sync_words + 1;
  P.sync.error = ctx->sync_words + 2;
  P.sync.nblocks = (unsigned)grid;
  P.sync.timeout_ns = kBarrierTimeoutNs;
  P.out = ctx->scalars;
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->sync_words, 0, 4 * sizeof(unsigned), ctx->stream));
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->scalars, 0, 8 * sizeof(double), ctx->stream));
  dim3 block(kThreads);
  void* args[] = {&P};
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_k0, ctx->stream));
  CFDB_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)kernel, dim3((unsigned)grid), block, args,
                                             smem, ctx->stream));
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_k1, ctx->stream));
  count_launch(ctx);
  return CFDB_OK;
}

bool getenv_flag(const char* name) {
  const char* v = std::getenv(name);
  return v && v[0] && v[0] != '0';
}

template <typename T, class S, bool MIXED = false>
cfdb_status launch_pcg_tma(cfdb_context* ctx, PcgParams<T>& P) {
  TmaParams<T> TP{};
  const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                                : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const int rank = S::D3 ? 3 : 2;
  const uint64_t dims3[3] = {(uint64_t)P.A.nx, (uint64_t)P.A.ny, (uint64_t)P.A.nz};
  const uint64_t dims2[2] = {(uint64_t)P.A.nx, (uint64_t)P.A.nz};
  const uint64_t* dims = S::D3 ? dims3 : dims2;
  const uint32_t halo3[3] = {(uint32_t)S::HX, (uint32_t)S::HY, (uint32_t)S::HZ};
  const uint32_t halo2[2] = {(uint32_t)S::HX, (uint32_t)S::HZ};
  const uint32_t intr3[3] = {(uint32_t)S::TX, (uint32_t)S::TY, (uint32_t)S::TZ};
  const uint32_t intr2[2] = {(uint32_t)S::TX, (uint32_t)S::TZ};
  const uint32_t* halo = S::D3 ? halo3 : halo2;
  const uint32_t* intr = S::D3 ? intr3 : intr2;
  const int es = (int)sizeof(T);
  // MIXED: x and r are the FP64 x64, r64 (interior boxes of doubles)
  const CUtensorMapDataType dti = MIXED ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : dt;
  const int esi = MIXED ? 8 : es;
  void* xint = MIXED ? (void*)P.x64 : (void*)P.x;
  void* rint = MIXED ? (void*)P.r64 : (void*)P.r;
  if (!encode_tensor_map(&TP.maps.z_halo, dt, es, rank, P.z, dims, halo) ||
      !encode_tensor_map(&TP.maps.p0_halo, dt, es, rank, P.p0, dims, halo) ||
      !encode_tensor_map(&TP.maps.p1_halo, dt, es, rank, P.p1, dims, halo) ||
      !encode_tensor_map(&TP.maps.x_int, dti, esi, rank, xint, dims, intr) ||
      !encode_tensor_map(&TP.maps.r_int, dti, esi, rank, rint, dims, intr))
    return set_error(ctx, CFDB_ERR_CUDA, "cuTensorMapEncodeTiled rejected a p' tensor map");
  auto kernel = P.A.fx ? pcg_tma<T, S, true, MIXED> : pcg_tma<T, S, false, MIXED>;
  // stage: MIXED carries FP64 x and r boxes (2 x INTR_P doubles after the halo)
  const size_t stage_words = MIXED ? (size_t)std::max(2 * S::HALO_P, S::HALO_P + 4 * S::INTR_P)
                                   : (size_t)S::STAGE;
  const size_t smem = sizeof(T) * stage_words * 2;
  CFDB_CUDA(ctx, cudaFuncSetAttribute((const void*)kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  CFDB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTmaThreads, smem));
  if (per_sm < 1) return set_error(ctx, CFDB_ERR_CUDA, "TMA pcg kernel cannot be resident");
  int64_t grid = (int64_t)per_sm * ctx->num_sms;
  grid = std::min<int64_t>(grid, P.cs.items);
  grid = std::max<int64_t>(grid, 1);
  cfdb_status st = ensure_partials(ctx, 4 * (size_t)grid);
  if (st != CFDB_OK) return st;
  P.partials = ctx->partials;
  P.sync.count = ctx->sync_words;
  P.sync.gen = ctx->sync_words + 1;
  P.sync.error = ctx->sync_words + 2;
  P.sync.nblocks = (unsigned)grid;
  P.sync.timeout_ns = kBarrierTimeoutNs;
  P.out = ctx->scalars;
  TP.P = P;
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->sync_words, 0, 4 * sizeof(unsigned), ctx->stream));
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->scalars, 0, 8 * sizeof(double), ctx->stream));
  void* args[] = {&TP};
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_k0, ctx->stream));
  CFDB_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)kernel, dim3((unsigned)grid),
                                             dim3(kTmaThreads), args, smem, ctx->stream));
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_k1, ctx->stream));
  count_launch(ctx);
  return CFDB_OK;
}

// The TMA kernel needs rows that start on 16-byte boundaries.
bool pcg_uses_tma(const cfdb_poperator* op, size_t word) {
  return ((int64_t)op->knx * (int64_t)word) % 16 == 0 && !getenv_flag("CFDB_NO_TMA");
}

template <typename T>
cfdb_status run_pcg(cfdb_context* ctx, const cfdb_poperator* op, const T* b, T* x, T* r, T* p0,
                    T* p1, T* z, int x0_zero, double abs_tol, double rel_tol, int64_t max_it,
                    double* hist_dev, int64_t hist_cap) {
  PcgParams<T> P{};
  P.A = view<T>(op);
  if constexpr (sizeof(T) == 8) P.invd = op->invd64; else P.invd = op->invd32;
  P.b = b;
  P.x = x;
  P.r = r;
  P.p0 = p0;
  P.p1 = p1;
  P.z = z;
  P.x0_zero = x0_zero;
  P.abs_tol = abs_tol;
  P.rel_tol = rel_tol;
  P.max_it = max_it;
  P.hist = hist_dev;
  P.hist_cap = hist_cap;
  if (pcg_uses_tma(op, sizeof(T))) {
    if (is3d(op)) {
      P.cs = make_split<TmaTile3D<T>>(op->knx, op->kny, op->knz);
      return launch_pcg_tma<T, TmaTile3D<T>>(ctx, P);
    }
    P.cs = make_split<TmaTile2D<T>>(op->knx, op->kny, op->knz);
    return launch_pcg_tma<T, TmaTile2D<T>>(ctx, P);
  }
  if (is3d(op)) {
    P.cs = make_split<Tile3D>(op->knx, op->kny, op->knz);
    return launch_pcg<T, Tile3D>(ctx, P);
  }
  P.cs = make_split<Tile2D>(op->knx, op->kny, op->knz);
  return launch_pcg<T, Tile2D>(ctx, P);
}

// The mixed-precision PCG (FP32 r, p, z; FP64 x with FP64 residual
// replacement) on the TMA kernel; needs rows of a multiple of 16 bytes in
// FP32 (nx % 4 == 0).
cfdb_status run_pcg_mixed(cfdb_context* ctx, const cfdb_poperator* op, const double* b64,
                          double* x64, double* r64, float* p0, float* p1, float* z, int x0_zero,
                          double abs_tol, double rel_tol, int64_t max_it, double delta,
                          double* hist_dev, int64_t hist_cap) {
  PcgParams<float> P{};
  P.A = view<float>(op);
  P.A64 = view<double>(op);
  P.invd = op->invd32;
  P.b = nullptr;
  P.x = nullptr;
  P.b64 = b64;
  P.x64 = x64;
  P.r64 = r64;
  P.r = z;  // FP32 residual unused: the TMA map that would carry it points at z
  P.p0 = p0;
  P.p1 = p1;
  P.z = z;
  P.x0_zero = x0_zero;
  P.abs_tol = abs_tol;
  P.rel_tol = rel_tol;
  P.max_it = max_it;
  P.delta = delta;
  P.hist = hist_dev;
  P.hist_cap = hist_cap;
  if (is3d(op)) {
    P.cs = make_split<TmaTile3D<float>>(op->knx, op->kny, op->knz);
    return launch_pcg_tma<float, TmaTile3D<float>, true>(ctx, P);
  }
  P.cs = make_split<TmaTile2D<float>>(op->knx, op->kny, op->knz);
  return launch_pcg_tma<float, TmaTile2D<float>, true>(ctx, P);
}

// Algorithmic bytes of one mixed-precision PCG launch: per iteration the
// FP32 words (sweep A: z, p_old in, p out; sweep B: p in, z out) and the FP64
// x and r read and written in sweep B; per residual replacement (and the
// initial residual) x (unless zero) and b in, r out in FP64 and z out in
// FP32; FP64 face coefficients read by every sweep.
double pcg_mixed_bytes(const cfdb_poperator* op, int64_t iterations, int64_t replacements,
                       bool x0_zero) {
  const double cells = (double)op->cells;
  int fw = 0;
  for (int q = 0; q < 3; ++q) fw += op->f64[q] ? 1 : 0;
  const double per_it = cells * (5.0 * 4.0 + 4.0 * 8.0 + 2.0 * fw * 8.0);
  const double per_repl = cells * (3.0 * 8.0 + 4.0 + fw * 8.0);
  const double init = cells * ((x0_zero ? 2.0 : 3.0) * 8.0 + 4.0 + fw * 8.0);
  return init + per_it * (double)iterations + per_repl * (double)replacements;
}

// Algorithmic bytes of one persistent PCG launch: the initial pass reads b
// (and x0) and writes r; each iteration moves 8 vector words per cell (sweep
// A: r, p_old in, p out; sweep B: x, r, p in, x, r out) plus, with per-face
// coefficients, the face words each sweep reads.  The TMA kernel also writes
// z = D^-1 r in the initial pass and in sweep B, and sweep A reads z in
// place of r: one more word per cell in each.
double pcg_bytes(const cfdb_poperator* op, size_t word, int64_t iterations, bool x0_zero) {
  const double cells = (double)op->cells;
  int face_words = 0;
  for (int q = 0; q < 3; ++q) face_words += op->f64[q] ? 1 : 0;
  const double zw = pcg_uses_tma(op, word) ? 1.0 : 0.0;
  const double init = cells * ((x0_zero ? 2.0 : 3.0) + zw) * (double)word;
  const double per_it = cells * (8.0 + zw + 2.0 * face_words) * (double)word;
  return init + per_it * (double)iterations;
}

cfdb_status add_krylov_time(cfdb_context* ctx, cfdb_linear_result* res) {
  float ms = 0.f;
  CFDB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev_k0, ctx->ev_k1));
  res->krylov_ms += ms;
  res->krylov_launches += 1;
  return CFDB_OK;
}

// Reads the solver scalars back (one small synchronous copy).
cfdb_status read_scalars(cfdb_context* ctx, int n) {
  CFDB_CUDA(ctx, cudaMemcpyAsync(ctx->scalars_host, ctx->scalars, n * sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  unsigned err = 0;
  CFDB_CUDA(ctx, cudaMemcpyAsync(&err, ctx->sync_words + 2, sizeof(unsigned),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (err != 0)
    return set_error(ctx, CFDB_ERR_DEVICE_TIMEOUT,
                     "a grid barrier of the persistent solver timed out (no fault; solve abandoned)");
  return CFDB_OK;
}

// FP64 ||b - A x_in - scale e|| with optional outputs; returns the norm.
cfdb_status refine_pass(cfdb_context* ctx, const cfdb_poperator* op, const double* b,
                        const double* x_in, double* x_out, const float* e, double scale,
                        float* r32, double* r64, double* norm_out) {
  const OpView<double> A = view<double>(op);
  Tiling tl;
  int grid;
  const int chunk = 16;
  if (is3d(op)) {
    tl = make_tiling<32, 8>(op->knx, op->kny, op->knz);
  } else {
    tl = make_tiling<256, 1>(op->knx, op->kny, op->knz);
  }
  grid = (int)std::max<int64_t>(1, std::min<int64_t>((tl.items + chunk - 1) / chunk, 1 << 20));
  cfdb_status st = ensure_partials(ctx, grid);
  if (st != CFDB_OK) return st;
  if (is3d(op))
    refine_residual<8><<<grid, dim3(32, 8), 0, ctx->stream>>>(A, tl, b, x_in, x_out, e, scale, r32,
                                                              r64, ctx->partials);
  else
    refine_residual<1><<<grid, dim3(256, 1), 0, ctx->stream>>>(A, tl, b, x_in, x_out, e, scale,
                                                               r32, r64, ctx->partials);
  CFDB_CHECK_LAUNCH(ctx);
  sum_partials<<<1, 256, 0, ctx->stream>>>(ctx->partials, grid, ctx->scalars, 8);
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx, 2);
  CFDB_CUDA(ctx, cudaMemcpyAsync(ctx->scalars_host + 8, ctx->scalars + 8, sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *norm_out = std::sqrt(ctx->scalars_host[8]);
  return CFDB_OK;
}

template <typename T>
cfdb_status alloc_vec(cfdb_context* ctx, T** p, int64_t n) {
  if (*p) return CFDB_OK;
  CFDB_CUDA(ctx, cudaMalloc((void**)p, sizeof(T) * (size_t)n));
  return CFDB_OK;
}

cfdb_status ensure_hist(cfdb_context* ctx, cfdb_poperator* op, int64_t cap) {
  if (op->hist_cap >= cap && op->hist_dev) return CFDB_OK;
  if (op->hist_dev) cudaFree(op->hist_dev);
  op->hist_dev = nullptr;
  op->hist_cap = 0;
  CFDB_CUDA(ctx, cudaMalloc((void**)&op->hist_dev, sizeof(double) * (size_t)cap));
  op->hist_cap = cap;
  return CFDB_OK;
}

cfdb_status check_finite(cfdb_context* ctx, const double* v, int64_t n, bool* ok) {
  CFDB_CUDA(ctx, cudaMemsetAsync(ctx->sync_words + 3, 0, sizeof(unsigned), ctx->stream));
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 4 * 148 * 8);
  all_finite<<<std::max(grid, 1), 256, 0, ctx->stream>>>(v, n, ctx->sync_words + 3);
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx);
  unsigned flag = 0;
  CFDB_CUDA(ctx, cudaMemcpyAsync(&flag, ctx->sync_words + 3, sizeof(unsigned),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *ok = (flag == 0);
  return CFDB_OK;
}

// Plain FP64 PCG on device vectors.
cfdb_status solve_fp64(cfdb_context* ctx, cfdb_poperator* op, const cfdb_linear_settings* s,
                       const double* b, double* x, bool x0_zero, int64_t hist_cap,
                       cfdb_linear_result* res) {
  const int64_t n = op->cells;
  for (int q : {0, 1, 2, 6}) {
    cfdb_status st = alloc_vec(ctx, &op->w64[q], n);
    if (st != CFDB_OK) return st;
  }
  cfdb_status st = ensure_hist(ctx, op, std::max<int64_t>(hist_cap, 1));
  if (st != CFDB_OK) return st;
  st = run_pcg<double>(ctx, op, b, x, op->w64[0], op->w64[1], op->w64[2], op->w64[6], x0_zero ? 1 : 0,
                       s->abs_tol, s->rel_tol, s->max_iterations, op->hist_dev, hist_cap);
  if (st != CFDB_OK) return st;
  st = read_scalars(ctx, 8);
  if (st != CFDB_OK) return st;
  const double* o = ctx->scalars_host;
  res->status = (int)o[OUT_STATUS];
  res->iterations = (int64_t)o[OUT_ITER];
  res->initial_residual = o[OUT_B0];
  res->final_residual = o[OUT_FINAL];
  res->krylov_bytes += pcg_bytes(op, sizeof(double), res->iterations, x0_zero);
  return add_krylov_time(ctx, res);
}

// FP32 Jacobi-PCG with FP64 residual replacement (one Krylov space).
cfdb_status solve_mixed(cfdb_context* ctx, cfdb_poperator* op, const cfdb_linear_settings* s,
                        const double* b, double* x, int64_t hist_cap,
                        cfdb_linear_result* res) {
  const int64_t n = op->cells;
  for (int q : {1, 2, 5}) {
    cfdb_status st = alloc_vec(ctx, &op->w32[q], n);
    if (st != CFDB_OK) return st;
  }
  cfdb_status st = alloc_vec(ctx, &op->w64[0], n);
  if (st != CFDB_OK) return st;
  st = ensure_hist(ctx, op, std::max<int64_t>(hist_cap, 1));
  if (st != CFDB_OK) return st;
  const double delta = s->inner_rel_tol > 0.0 ? s->inner_rel_tol : 0.1;
  st = run_pcg_mixed(ctx, op, b, x, op->w64[0], op->w32[1], op->w32[2], op->w32[5], 0, s->abs_tol,
                     s->rel_tol, s->max_iterations, delta, op->hist_dev, hist_cap);
  if (st != CFDB_OK) return st;
  st = read_scalars(ctx, 8);
  if (st != CFDB_OK) return st;
  const double* o = ctx->scalars_host;
  res->status = (int)o[OUT_STATUS];
  res->iterations = (int64_t)o[OUT_ITER];
  res->initial_residual = o[OUT_B0];
  res->final_residual = o[OUT_FINAL];
  res->refinements = (int64_t)o[OUT_REPLACEMENTS];
  res->krylov_bytes += pcg_mixed_bytes(op, res->iterations, res->refinements, false);
  return add_krylov_time(ctx, res);
}

// FP32 inner sweeps inside FP64 iterative refinement (each refinement a new
// FP32 Krylov solve of the correction): for grids whose rows the TMA kernel
// cannot take in FP32 (nx % 4 != 0).
cfdb_status solve_refined(cfdb_context* ctx, cfdb_poperator* op, const cfdb_linear_settings* s,
                          const double* b, double* x, int64_t hist_cap, double* hist_host,
                          cfdb_linear_result* res) {
  const int64_t n = op->cells;
  for (int q = 0; q < 6; ++q) {
    cfdb_status st = alloc_vec(ctx, &op->w32[q], n);
    if (st != CFDB_OK) return st;
  }
  cfdb_status st = alloc_vec(ctx, &op->w64[3], n);
  if (st != CFDB_OK) return st;
  st = ensure_hist(ctx, op, 2);
  if (st != CFDB_OK) return st;
  const double inner_tol = s->inner_rel_tol > 0.0 ? s->inner_rel_tol : 1.0e-4;
  const int64_t max_ref = s->max_refinements > 0 ? s->max_refinements : 50;
  float* r32 = op->w32[0];
  float* e32 = op->w32[3];
  float* b32 = op->w32[4];
  double* xa = x;
  double* xb = op->w64[3];
  // r = b - A x0 (FP64), r32 = float(r)
  double rnorm = 0.0;
  st = refine_pass(ctx, op, b, xa, nullptr, nullptr, 0.0, b32, nullptr, &rnorm);
  if (st != CFDB_OK) return st;
  const double b0 = rnorm;
  res->initial_residual = b0;
  int64_t hc = 0;
  if (hist_host && hc < hist_cap) hist_host[hc] = b0;
  ++hc;
  auto conv = [&](double r) { return r <= s->abs_tol || (b0 > 0.0 && r / b0 <= s->rel_tol); };
  int64_t inner_total = 0, steps = 0;
  res->status = CFDB_SOLVER_MAX_ITERATIONS;
  if (!std::isfinite(b0)) {
    res->status = CFDB_SOLVER_NONFINITE_RESIDUAL;
    res->final_residual = b0;
    return CFDB_OK;
  }
  if (b0 == 0.0 || conv(b0)) {
    res->status = CFDB_SOLVER_CONVERGED;
    res->final_residual = b0;
    return CFDB_OK;
  }
  while (steps < max_ref && inner_total < s->max_iterations) {
    // inner: A e = r32 from e = 0 in FP32, reduction inner_tol
    const int64_t budget = s->max_iterations - inner_total;
    CFDB_CUDA(ctx, cudaMemsetAsync(e32, 0, sizeof(float) * (size_t)n, ctx->stream));
    st = run_pcg<float>(ctx, op, b32, e32, r32, op->w32[1], op->w32[2], op->w32[5], 1, 0.0, inner_tol,
                        budget, op->hist_dev, 0);
    if (st != CFDB_OK) return st;
    st = read_scalars(ctx, 8);
    if (st != CFDB_OK) return st;
    const double* o = ctx->scalars_host;
    const int inner_status = (int)o[OUT_STATUS];
    inner_total += (int64_t)o[OUT_ITER];
    res->krylov_bytes += pcg_bytes(op, sizeof(float), (int64_t)o[OUT_ITER], true);
    st = add_krylov_time(ctx, res);
    if (st != CFDB_OK) return st;
    ++steps;
    // x += e; r = b - A x (FP64); r32 = float(r)
    st = refine_pass(ctx, op, b, xa, xb, e32, 1.0, b32, nullptr, &rnorm);
    if (st != CFDB_OK) return st;
    std::swap(xa, xb);
    if (hist_host && hc < hist_cap) hist_host[hc] = rnorm;
    ++hc;
    if (!std::isfinite(rnorm)) {
      res->status = CFDB_SOLVER_NONFINITE_RESIDUAL;
      break;
    }
    if (conv(rnorm)) {
      res->status = CFDB_SOLVER_CONVERGED;
      break;
    }
    if (inner_status == CFDB_SOLVER_BREAKDOWN && (int64_t)o[OUT_ITER] == 0) {
      res->status = CFDB_SOLVER_BREAKDOWN;
      break;
    }
  }
  if (xa != x) CFDB_CUDA(ctx, cudaMemcpyAsync(x, xa, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                              ctx->stream));
  res->final_residual = rnorm;
  res->iterations = inner_total;
  res->refinements = steps;
  return CFDB_OK;
}

// Learned V-cycle inside FP64 flexible CG; when it stagnates (or breaks
// down) the FP64 Jacobi-PCG continues from its iterate with the remaining
// iteration budget and the original tolerance.
// *verified: the FP64 true residual of the returned x when the solve ended
// on a checked, converged FCG run (-1 otherwise).
cfdb_status solve_learned(cfdb_context* ctx, cfdb_poperator* op, const cfdb_linear_settings* s,
                          const double* b, double* x, double* history, int64_t history_cap,
                          cfdb_linear_result* res, double* verified) {
  *verified = -1.0;
  const cfdb_grid& g = op->grid;
  FineOperator fo;
  LearnedSolver* solver = nullptr;
  uint64_t version = 0;
  poperator_learned(op, &fo, &solver, &version);
  const int64_t cap = std::min<int64_t>(s->max_iterations, 100000);
  LearnedOutcome o;
  cfdb_status st = learned_solve(ctx, solver, fo, version, mg_context_weights(ctx, g.dim),
                                 b, x, s->abs_tol, s->rel_tol, cap,
                                 std::max<int64_t>(history_cap, 1), &o);
  if (st != CFDB_OK) return st;
  res->initial_residual = o.initial_residual;
  res->final_residual = o.final_residual;
  res->iterations = o.iterations;
  res->status = o.status;
  res->krylov_ms += o.kernel_ms;
  res->krylov_bytes += o.bytes;
  res->krylov_launches += 1;
  if (history && history_cap > 0) {
    st = learned_history(ctx, solver, history, std::min<int64_t>(history_cap, o.iterations + 1));
    if (st != CFDB_OK) return st;
  }
  // FCG stops on its recurrence residual, which drifts from b - A x at about
  // the 1e-10 level: a converged solve is checked against the FP64 true
  // residual and, while that misses the caller's target, continued from its
  // iterate by a fresh FCG start on b - A x (at most three times; the history
  // covers the first run)
  for (int again = 0; again < 3 && o.status == CFDB_SOLVER_CONVERGED; ++again) {
    double tr = 0.0;
    st = refine_pass(ctx, op, b, x, nullptr, nullptr, 0.0, nullptr, nullptr, &tr);
    if (st != CFDB_OK) return st;
    *verified = tr;
    const double target = std::max(s->abs_tol, s->rel_tol * res->initial_residual);
    const int64_t left = cap - res->iterations;
    if (!(tr > target) || !(tr > 0.0) || !std::isfinite(tr) || left < 1) break;
    *verified = -1.0;  // x changes again below
    st = learned_solve(ctx, solver, fo, version, mg_context_weights(ctx, g.dim), b, x, s->abs_tol,
                       target / tr, left, 1, &o);
    if (st != CFDB_OK) return st;
    res->iterations += o.iterations;
    res->final_residual = o.final_residual;
    res->status = o.status;
    res->krylov_ms += o.kernel_ms;
    res->krylov_bytes += o.bytes;
    res->krylov_launches += 1;
  }
  const bool stalled = o.status == kLearnedStagnated ||
                       (o.status == CFDB_SOLVER_MAX_ITERATIONS && cap < s->max_iterations);
  if (!stalled) return CFDB_OK;
  *verified = -1.0;
  const int64_t left = s->max_iterations - res->iterations;
  if (left < 1) {
    res->status = CFDB_SOLVER_MAX_ITERATIONS;
    return CFDB_OK;
  }
  cfdb_linear_settings s2 = *s;
  s2.max_iterations = left;
  // keep the caller's relative target, measured against the original start
  if (o.final_residual > 0.0 && std::isfinite(o.final_residual))
    s2.rel_tol = s->rel_tol * res->initial_residual / o.final_residual;
  cfdb_linear_result sub;
  std::memset(&sub, 0, sizeof(sub));
  st = solve_fp64(ctx, op, &s2, b, x, false, 0, &sub);
  if (st != CFDB_OK) return st;
  res->status = sub.status;
  res->iterations += sub.iterations;
  res->fallback_iterations = sub.iterations;
  res->final_residual = sub.final_residual;
  res->krylov_ms += sub.krylov_ms;
  res->krylov_bytes += sub.krylov_bytes;
  res->krylov_launches += sub.krylov_launches;
  return CFDB_OK;
}

cfdb_status build_tables(cfdb_context* ctx, cfdb_poperator* op, double rho, unsigned dmask) {
  // Geometry exactly as the reference evaluates it (MeshGrading.cpp
  // AxisSpacing::uniform/center/node; MeshGeometry.cpp:513-552,1047-1140):
  // D = ((rho * |S|) * d_face) / |x_N - x_P| with d_face = 1 (the scalar
  // interpolation of a unit field is exactly 1), Dirichlet boundary faces
  // ((rho * |S|) * 1) / |x_f - x_P|.
  const cfdb_grid& g = op->grid;
  const int dim = g.dim;
  double delta[3] = {0, 0, 0};
  for (int a = 0; a < dim; ++a) delta[a] = g.len[a] / (double)g.n[a];
  double area[3] = {0, 0, 0};
  if (dim == 2) {
    area[0] = delta[1];
    area[1] = delta[0];
  } else {
    area[0] = delta[1] * delta[2];
    area[1] = delta[0] * delta[2];
    area[2] = delta[0] * delta[1];
  }
  // real axis a -> kernel axis: 2D (x, y) -> (x, z); 3D identity
  const int kaxis[3] = {0, dim == 2 ? 2 : 1, 2};
  std::vector<double> tab[3];
  tab[0].assign(op->knx + 1, 0.0);
  tab[1].assign(op->kny + 1, 0.0);
  tab[2].assign(op->knz + 1, 0.0);
  for (int a = 0; a < dim; ++a) {
    const int64_t n = g.n[a];
    auto center = [&](int64_t i) { return ((double)i + 0.5) * delta[a]; };
    auto node = [&](int64_t i) { return (double)i * delta[a]; };
    std::vector<double>& t = tab[kaxis[a]];
    for (int64_t f = 1; f < n; ++f) {
      const double dPf = std::fabs(node(f) - center(f - 1));
      const double dNf = std::fabs(node(f) - center(f));
      const double dFace = ((dNf * 1.0) + (dPf * 1.0)) / (dPf + dNf);
      const double dist = std::fabs(center(f) - center(f - 1));
      t[f] = rho * area[a] * dFace / dist;
    }
    if (dmask & (1u << (2 * a))) t[0] = rho * area[a] * 1.0 / std::fabs(node(0) - center(0));
    if (dmask & (1u << (2 * a + 1)))
      t[n] = rho * area[a] * 1.0 / std::fabs(node(n) - center(n - 1));
  }
  for (int q = 0; q < 3; ++q) {
    const size_t m = tab[q].size();
    std::vector<float> t32(m);
    for (size_t i = 0; i < m; ++i) t32[i] = (float)tab[q][i];
    CFDB_CUDA(ctx, cudaMalloc((void**)&op->t64[q], m * sizeof(double)));
    CFDB_CUDA(ctx, cudaMalloc((void**)&op->t32[q], m * sizeof(float)));
    // stream-ordered (the context stream is non-blocking): the solves that
    // read the tables run on the same stream
    CFDB_CUDA(ctx, cudaMemcpyAsync(op->t64[q], tab[q].data(), m * sizeof(double),
                                   cudaMemcpyHostToDevice, ctx->stream));
    CFDB_CUDA(ctx, cudaMemcpyAsync(op->t32[q], t32.data(), m * sizeof(float), cudaMemcpyHostToDevice,
                                   ctx->stream));
    CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return CFDB_OK;
}

cfdb_status validate_grid(cfdb_context* ctx, const cfdb_grid* g) {
  if (!g || (g->dim != 2 && g->dim != 3))
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "grid: dim must be 2 or 3");
  for (int a = 0; a < g->dim; ++a) {
    if (g->n[a] < 2 || g->n[a] > (1 << 20))
      return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "grid: each axis needs 2..2^20 cells");
    if (!(g->len[a] > 0.0) || !std::isfinite(g->len[a]))
      return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "grid: lengths must be finite and > 0");
  }
  const int64_t cells = g->n[0] * g->n[1] * (g->dim == 3 ? g->n[2] : 1);
  if (cells > ((int64_t)1 << 31))
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "grid: more than 2^31 cells");
  return CFDB_OK;
}

cfdb_status new_operator(cfdb_context* ctx, const cfdb_grid* grid, int pinned, int64_t ref,
                         cfdb_poperator** out) {
  cfdb_status st = validate_grid(ctx, grid);
  if (st != CFDB_OK) return st;
  auto* op = new cfdb_poperator();
  op->ctx = ctx;
  op->grid = *grid;
  op->knx = (int)grid->n[0];
  if (grid->dim == 2) {
    op->kny = 1;
    op->knz = (int)grid->n[1];
  } else {
    op->kny = (int)grid->n[1];
    op->knz = (int)grid->n[2];
  }
  op->cells = (int64_t)op->knx * op->kny * op->knz;
  op->pinned = pinned ? 1 : 0;
  op->ref = ref;
  if (pinned && (ref < 0 || ref >= op->cells)) {
    delete op;
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "reference cell out of range");
  }
  *out = op;
  return CFDB_OK;
}

__global__ void k_to_f32(const double* in, float* out, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    out[q] = (float)in[q];
}

}  // namespace

// Points the operator's face coefficients at a device array in global face
// order (x-, y-, z-faces) and refreshes the inverse diagonal (and FP32
// copies when `fp32`).  The array must outlive the operator's next solves.
cfdb_status poperator_bind_faces(cfdb_context* ctx, cfdb_poperator* op, const double* D, bool fp32) {
  const cfdb_grid& g = op->grid;
  const int64_t nx = g.n[0], ny = g.n[1], nz = g.dim == 3 ? g.n[2] : 1;
  const int64_t nfx = (nx + 1) * ny * nz, nfy = nx * (ny + 1) * nz;
  const int64_t counts[3] = {nfx, nfy, g.dim == 3 ? nx * ny * (nz + 1) : 0};
  const int64_t offs[3] = {0, nfx, nfx + nfy};
  const int kaxis[3] = {0, g.dim == 2 ? 2 : 1, 2};
  op->faces_borrowed = true;
  ++op->version;
  for (int a = 0; a < g.dim; ++a) {
    const int ka = kaxis[a];
    op->f64[ka] = const_cast<double*>(D + offs[a]);
    if (fp32) {
      if (!op->f32[ka]) CFDB_CUDA(ctx, cudaMalloc((void**)&op->f32[ka], sizeof(float) * counts[a]));
      k_to_f32<<<1024, 256, 0, ctx->stream>>>(D + offs[a], op->f32[ka], counts[a]);
    }
  }
  if (!op->invd64) CFDB_CUDA(ctx, cudaMalloc((void**)&op->invd64, sizeof(double) * (size_t)op->cells));
  inverse_diagonal<double><<<1024, 256, 0, ctx->stream>>>(view<double>(op), op->invd64);
  if (fp32) {
    if (!op->invd32) CFDB_CUDA(ctx, cudaMalloc((void**)&op->invd32, sizeof(float) * (size_t)op->cells));
    inverse_diagonal<float><<<1024, 256, 0, ctx->stream>>>(view<float>(op), op->invd32);
  }
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx, fp32 ? 2 + g.dim : 1);
  return CFDB_OK;
}

void poperator_learned(cfdb_poperator* op, FineOperator* fo, LearnedSolver** solver,
                       uint64_t* version) {
  std::memset(fo, 0, sizeof(*fo));
  fo->dim = op->grid.dim;
  fo->n[0] = op->knx;
  fo->n[1] = op->kny;
  fo->n[2] = op->knz;
  fo->A = view<double>(op);
  for (int q = 0; q < 3; ++q) {
    const bool active = op->grid.dim == 3 || q != 1;  // 2D kernel space has no y-faces
    fo->full[q] = active ? op->f64[q] : nullptr;
    fo->table[q] = active ? op->t64[q] : nullptr;
  }
  fo->pinned = op->pinned;
  fo->ref = op->ref;
  if (!op->learned) op->learned = learned_create();
  *solver = op->learned;
  *version = op->version;
}

// Copies host face coefficients (global face order) into the operator's own
// FP64/FP32 face arrays (allocated when `alloc`), refreshes the inverse
// diagonals and bumps the coefficient version, so that a learned solve
// refreshes its hierarchy's values instead of rebuilding it.
cfdb_status upload_faces(cfdb_context* ctx, cfdb_poperator* op, const double* face_coeff_host,
                         bool alloc) {
  const cfdb_grid& g = op->grid;
  const int64_t nx = g.n[0], ny = g.n[1], nz = g.dim == 3 ? g.n[2] : 1;
  const int64_t nfx = (nx + 1) * ny * nz, nfy = nx * (ny + 1) * nz, nfz = g.dim == 3 ? nx * ny * (nz + 1) : 0;
  const int64_t counts[3] = {nfx, nfy, nfz};
  const int64_t offs[3] = {0, nfx, nfx + nfy};
  // real axis -> kernel axis: 2D y-faces become kernel z-faces
  const int kaxis[3] = {0, g.dim == 2 ? 2 : 1, 2};
  for (int64_t q = 0; q < nfx + nfy + nfz; ++q)
    if (!std::isfinite(face_coeff_host[q]))
      return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "non-finite face coefficient");
  for (int a = 0; a < g.dim; ++a) {
    const int ka = kaxis[a];
    const int64_t m = counts[a];
    std::vector<float> f32(m);
    for (int64_t q = 0; q < m; ++q) f32[q] = (float)face_coeff_host[offs[a] + q];
    if (alloc) {
      cudaError_t e1 = cudaMalloc((void**)&op->f64[ka], m * sizeof(double));
      cudaError_t e2 = cudaMalloc((void**)&op->f32[ka], m * sizeof(float));
      if (e1 != cudaSuccess || e2 != cudaSuccess)
        return set_error(ctx, CFDB_ERR_OUT_OF_MEMORY, "face coefficient allocation failed");
    }
    // stream-ordered behind the context's earlier solves and ahead of its next
    CFDB_CUDA(ctx, cudaMemcpyAsync(op->f64[ka], face_coeff_host + offs[a], m * sizeof(double),
                                   cudaMemcpyHostToDevice, ctx->stream));
    CFDB_CUDA(ctx, cudaMemcpyAsync(op->f32[ka], f32.data(), m * sizeof(float), cudaMemcpyHostToDevice,
                                   ctx->stream));
    CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (alloc) {
    CFDB_CUDA(ctx, cudaMalloc((void**)&op->invd64, sizeof(double) * (size_t)op->cells));
    CFDB_CUDA(ctx, cudaMalloc((void**)&op->invd32, sizeof(float) * (size_t)op->cells));
  }
  inverse_diagonal<double><<<1024, 256, 0, ctx->stream>>>(view<double>(op), op->invd64);
  inverse_diagonal<float><<<1024, 256, 0, ctx->stream>>>(view<float>(op), op->invd32);
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx, 2);
  ++op->version;
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

}  // namespace cfdb

using namespace cfdb;

extern "C" {

cfdb_status cfdb_poperator_create_uniform(cfdb_context* ctx, const cfdb_grid* grid, double rho,
                                          unsigned dirichlet_patch_mask, int pinned,
                                          int64_t reference_cell, cfdb_poperator** out) {
  if (!ctx || !out) return CFDB_ERR_INVALID_ARGUMENT;
  if (!(rho > 0.0) || !std::isfinite(rho))
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "density must be finite and > 0");
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  cfdb_poperator* op = nullptr;
  cfdb_status st = new_operator(ctx, grid, pinned, reference_cell, &op);
  if (st != CFDB_OK) return st;
  st = build_tables(ctx, op, rho, dirichlet_patch_mask);
  if (st != CFDB_OK) {
    cfdb_poperator_destroy(op);
    return st;
  }
  *out = op;
  return CFDB_OK;
}

cfdb_status cfdb_poperator_create_faces(cfdb_context* ctx, const cfdb_grid* grid,
                                        const double* face_coeff_host, int pinned,
                                        int64_t reference_cell, cfdb_poperator** out) {
  if (!ctx || !out || !face_coeff_host) return CFDB_ERR_INVALID_ARGUMENT;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  cfdb_poperator* op = nullptr;
  cfdb_status st = new_operator(ctx, grid, pinned, reference_cell, &op);
  if (st != CFDB_OK) return st;
  st = build_tables(ctx, op, 1.0, 0u);  // zero-filled fallbacks for absent axes
  if (st == CFDB_OK) st = upload_faces(ctx, op, face_coeff_host, true);
  if (st != CFDB_OK) {
    cfdb_poperator_destroy(op);
    return st;
  }
  *out = op;
  return CFDB_OK;
}

cfdb_status cfdb_poperator_update_faces(cfdb_context* ctx, cfdb_poperator* op,
                                        const double* face_coeff_host) {
  if (!ctx || !op || !face_coeff_host) return CFDB_ERR_INVALID_ARGUMENT;
  if (op->faces_borrowed || !op->f64[0])
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT,
                     "the operator holds no face arrays of its own (cfdb_poperator_create_faces "
                     "makes one that does)");
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  return upload_faces(ctx, op, face_coeff_host, false);
}

void cfdb_poperator_destroy(cfdb_poperator* op) {
  if (!op) return;
  for (int q = 0; q < 3; ++q) {
    cudaFree(op->t64[q]);
    cudaFree(op->t32[q]);
    if (!op->faces_borrowed) cudaFree(op->f64[q]);
    cudaFree(op->f32[q]);
  }
  for (int q = 0; q < 7; ++q) cudaFree(op->w64[q]);
  for (int q = 0; q < 6; ++q) cudaFree(op->w32[q]);
  cudaFree(op->hist_dev);
  cudaFree(op->invd64);
  cudaFree(op->invd32);
  cfdb::learned_destroy(op->learned);
  delete op;
}

int64_t cfdb_poperator_cells(const cfdb_poperator* op) { return op ? op->cells : 0; }

cfdb_status cfdb_poperator_apply(cfdb_context* ctx, const cfdb_poperator* op, const double* x_dev,
                                 double* y_dev) {
  if (!ctx || !op || !x_dev || !y_dev) return CFDB_ERR_INVALID_ARGUMENT;
  const OpView<double> A = view<double>(op);
  if (op->grid.dim == 3) {
    Tiling tl = make_tiling<32, 8>(op->knx, op->kny, op->knz);
    const int grid = (int)std::max<int64_t>(1, (tl.items + 15) / 16);
    apply_kernel<8><<<grid, dim3(32, 8), 0, ctx->stream>>>(A, tl, x_dev, y_dev);
  } else {
    Tiling tl = make_tiling<256, 1>(op->knx, op->kny, op->knz);
    const int grid = (int)std::max<int64_t>(1, (tl.items + 15) / 16);
    apply_kernel<1><<<grid, dim3(256, 1), 0, ctx->stream>>>(A, tl, x_dev, y_dev);
  }
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx);
  return CFDB_OK;
}

cfdb_status cfdb_poperator_solve_device(cfdb_context* ctx, const cfdb_poperator* opc,
                                        const cfdb_linear_settings* s, const double* b_dev,
                                        double* x_dev, double* history, int64_t history_cap,
                                        cfdb_linear_result* result) {
  if (!ctx || !opc || !s || !b_dev || !x_dev || !result) return CFDB_ERR_INVALID_ARGUMENT;
  auto* op = const_cast<cfdb_poperator*>(opc);
  std::memset(result, 0, sizeof(*result));
  if (s->krylov != CFDB_KRYLOV_CG)
    return set_error(ctx, CFDB_ERR_UNSUPPORTED, "the structured p' solve runs CG");
  if (s->preconditioner != CFDB_PRECOND_JACOBI && s->preconditioner != CFDB_PRECOND_LEARNED_MG)
    return set_error(ctx, CFDB_ERR_UNSUPPORTED,
                     "the structured p' solve takes the Jacobi or the learned preconditioner");
  if (s->max_iterations < 1)
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "max_iterations must be >= 1");
  if (history_cap < 0) history_cap = 0;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  const int64_t launches0 = ctx->launches;
  // NonFiniteInput (CG.cpp:23-26): the operator was validated at creation.
  bool ok_b = true, ok_x = true;
  cfdb_status st = check_finite(ctx, b_dev, op->cells, &ok_b);
  if (st != CFDB_OK) return st;
  st = check_finite(ctx, x_dev, op->cells, &ok_x);
  if (st != CFDB_OK) return st;
  if (!ok_b || !ok_x) {
    result->status = CFDB_SOLVER_NONFINITE_INPUT;
    return CFDB_OK;
  }
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  double verified = -1.0;
  if (s->preconditioner == CFDB_PRECOND_LEARNED_MG) {
    st = solve_learned(ctx, op, s, b_dev, x_dev, history, history_cap, result, &verified);
  } else if (s->precision == CFDB_PRECISION_FP32_REFINED && pcg_uses_tma(op, sizeof(float))) {
    st = solve_mixed(ctx, op, s, b_dev, x_dev, history_cap, result);
    if (st == CFDB_OK && history && history_cap > 0) {
      const int64_t m = std::min<int64_t>(history_cap, result->iterations + 1);
      CFDB_CUDA(ctx, cudaMemcpyAsync(history, op->hist_dev, sizeof(double) * m,
                                     cudaMemcpyDeviceToHost, ctx->stream));
    }
  } else if (s->precision == CFDB_PRECISION_FP32_REFINED) {
    st = solve_refined(ctx, op, s, b_dev, x_dev, history_cap, history, result);
  } else {
    st = solve_fp64(ctx, op, s, b_dev, x_dev, false, history_cap, result);
    if (st == CFDB_OK && history && history_cap > 0) {
      const int64_t m = std::min<int64_t>(history_cap, result->iterations + 1);
      CFDB_CUDA(ctx, cudaMemcpyAsync(history, op->hist_dev, sizeof(double) * m,
                                     cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  if (st != CFDB_OK) return st;
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  CFDB_CUDA(ctx, cudaEventSynchronize(ctx->ev_stop));
  float ms = 0.f;
  CFDB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
  result->device_ms = ms;
  // FP64 true residual of the returned x (outside the timed region; the
  // learned solve's own check already holds it when x has not changed since)
  double tr = verified;
  if (!(tr >= 0.0)) {
    st = refine_pass(ctx, op, b_dev, x_dev, nullptr, nullptr, 0.0, nullptr, nullptr, &tr);
    if (st != CFDB_OK) return st;
  }
  result->true_residual = tr;
  result->kernel_launches = ctx->launches - launches0;
  return CFDB_OK;
}

cfdb_status cfdb_poperator_solve_host(cfdb_context* ctx, const cfdb_poperator* opc,
                                      const cfdb_linear_settings* s, const double* b_host,
                                      double* x_host, double* history, int64_t history_cap,
                                      cfdb_linear_result* result) {
  if (!ctx || !opc || !b_host || !x_host) return CFDB_ERR_INVALID_ARGUMENT;
  auto* op = const_cast<cfdb_poperator*>(opc);
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t bytes = sizeof(double) * (size_t)op->cells;
  for (int q = 4; q < 6; ++q) {
    cfdb_status st = alloc_vec(ctx, &op->w64[q], op->cells);
    if (st != CFDB_OK) return st;
  }
  CFDB_CUDA(ctx, cudaMemcpyAsync(op->w64[4], b_host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(op->w64[5], x_host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  cfdb_status st = cfdb_poperator_solve_device(ctx, op, s, op->w64[4], op->w64[5], history,
                                               history_cap, result);
  if (st != CFDB_OK) return st;
  CFDB_CUDA(ctx, cudaMemcpyAsync(x_host, op->w64[5], bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

}  // extern "C"
