// Batched SIMPLE: host orchestration, the per-case Krylov team kernel, the
// work-list planners, the autotuner and the C ABI (layout: batch.cuh).
//
// One outer iteration of the batch, in the single-case stage order
// (simple.cu, after SIMPLE.cpp:148-1124):
//   clear flags; face values and Green-Gauss gradient of p; per component:
//   [velocity gradient], momentum assembly (+ Us = U, input checks), team
//   Krylov solve; response coefficients (+ Us finite check); predictor flux
//   [+ Rhie-Chow]; p' faces (+ Fs finite check); p' rows and rhs; team p'
//   solve; p' finite gate; face values and gradient of p'; pressure and
//   velocity corrections; flux correction; residuals, per-case gate and
//   convergence test.
// It is captured once as a CUDA graph and launched once per outer iteration;
// per-case state lives on the device, so the host reads only the active set
// (and, with adaptive team sizing, each case's last p' iteration count)
// between launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "batch.cuh"
#include "pcg_internal.cuh"
#include "cfdb.h"
#include "cfdb_internal.cuh"
#include "grid_sync.cuh"
#include "simple_kernels.cuh"
#include "stencil_krylov.cuh"

namespace cfdb {
namespace {

constexpr unsigned long long kTeamTimeoutNs = 2000000000ull;
constexpr int kKoutStride = 8;
// Host threads (each with its own context and stream) that run the learned
// p' solves of a batch's cases concurrently.
constexpr int kLearnedWorkers = 8;
constexpr int64_t kMinCellsPerBlock = 2048;
constexpr int kAlign = 32;  // elements: every case starts on a 256-byte boundary

// Barrier over the blocks of one case's team (a one-block team only needs
// the block barrier).
struct TeamSync {
  GridSync s;
  int r, n;
  __device__ int rank() const { return r; }
  __device__ int size() const { return n; }
  __device__ bool sync() const {
    if (n == 1) {
      __syncthreads();
      return true;
    }
    return grid_sync(s);
  }
};

struct KArgs {
  BatchDev B;
  const int* block_case;
  const int* team_first;
  int mode;  // 0: momentum component `comp`; 1: p'
  int comp;
  int krylov, jacobi;
  int mixed;  // 1: p' by the mixed-precision CG (CFDB_PRECISION_FP32_REFINED)
  double abs_tol, rel_tol;
  int64_t max_it;
  unsigned* bar;    // 2 words per case
  unsigned* error;  // shared barrier error flag
  double* kpart;    // 6 doubles per block
  double* kout;     // kKoutStride doubles per (mode, case)
  int record;       // 1: update the case records (0 while tuning)
};

// Every case's linear solve of one stage; the leader of each team then
// applies the single-case session's outcome rules (simple.cu
// outer_iteration): a momentum solve that does not converge stops the case
// with MOMENTUM_FAILURE, a p' solve with PRESSURE_FAILURE; a case whose
// fields went non-finite earlier in the iteration stops at the p' stage with
// NONFINITE_STATE.
// Five resident blocks per SM (48 registers, some spilled to L1): the team
// solves are latency-bound; measured on the 64-case batch, an outer iteration
// takes 297 ms with two blocks per SM, 222 ms with three, 197 ms with four
// and 187 ms with five.
__global__ void __launch_bounds__(krylov::kThreads, 5) k_batch_krylov(KArgs A) {
  const int k = A.block_case[blockIdx.x];
  if (k < 0) return;
  const BatchDev& B = A.B;
  if (!B.active[k]) return;
  const BCase& K = B.cases[k];
  const int first = A.team_first[k];
  const int n = A.team_first[k + 1] - first;
  const int rank = (int)blockIdx.x - first;
  const bool leader = rank == 0 && threadIdx.x == 0;
  double* out = A.kout + (size_t)(A.mode * B.ncases + k) * kKoutStride;
  int* status = B.status + k;
  if (A.mode == 1 && B.flags[(size_t)BF_NONFINITE * B.ncases + k] != 0u) {
    if (leader && A.record) {
      *status = CFDB_SIMPLE_NONFINITE_STATE;
      B.active[k] = 0;
    }
    return;
  }
  const unsigned fl = B.flags[(size_t)(A.mode == 0 ? BF_MOM0 + A.comp : BF_PP) * B.ncases + k];
  const int64_t o = K.c0;
  krylov::SParams P{};
  P.M.dim = K.G.dim;
  P.M.nx = K.G.n[0];
  P.M.ny = K.G.n[1];
  P.M.nz = K.G.n[2];
  P.M.n = K.G.nc;
  P.M.sy = K.G.stride[1];
  P.M.sz = K.G.stride[2];
  P.M.diag = (A.mode == 0 ? B.mdiag[A.comp] : B.pdiag) + o;
  for (int q = 0; q < 6; ++q) P.M.off[q] = (A.mode == 0 ? B.moff[q] : B.poff[q]) + o;
  P.M.inv = A.jacobi ? B.kinv + o : nullptr;
  P.b = (A.mode == 0 ? B.mrhs : B.prhs) + o;
  P.x = (A.mode == 0 ? B.Us[A.comp] : B.pp) + o;
  P.r = B.kr + o;
  P.rh = B.krh + o;
  P.v = B.kv + o;
  P.p = B.kp + o;
  P.s = B.ks + o;
  P.t = B.kt + o;
  P.krylov = A.krylov;
  P.jacobi = A.jacobi;
  P.abs_tol = A.abs_tol;
  P.rel_tol = A.rel_tol;
  P.max_it = A.max_it;
  P.hist = nullptr;
  P.hist_cap = 0;
  P.partials = A.kpart + (size_t)6 * first;
  P.out = out;
  if (fl & BFLAG_NONFINITE_INPUT) {
    if (leader) out[krylov::O_STATUS] = CFDB_SOLVER_NONFINITE_INPUT;
  } else if (A.jacobi && (fl & BFLAG_INVALID_SYSTEM)) {
    if (leader) out[krylov::O_STATUS] = CFDB_SOLVER_INVALID_SYSTEM;
  } else {
    if (leader) out[krylov::O_STATUS] = -1.0;
    TeamSync T;
    T.s.count = A.bar + 2 * (size_t)k;
    T.s.gen = A.bar + 2 * (size_t)k + 1;
    T.s.error = A.error;
    T.s.nblocks = (unsigned)n;
    T.s.timeout_ns = kTeamTimeoutNs;
    T.r = rank;
    T.n = n;
    if (A.mixed) {
      // FP32 storage inside the case's own BiCGSTAB-only vectors (unused by
      // CG) and the upper halves of p and v: 2 floats per double slot
      float* w[5] = {reinterpret_cast<float*>(B.krh + o), reinterpret_cast<float*>(B.ks + o),
                     reinterpret_cast<float*>(B.kt + o), reinterpret_cast<float*>(B.kp + o),
                     reinterpret_cast<float*>(B.kv + o)};
      const int64_t nc = K.G.nc;
      P.m32[0] = w[0];
      P.m32[1] = w[0] + nc;
      P.m32[2] = w[1];
      P.m32[3] = w[1] + nc;
      P.m32[4] = w[2];
      P.m32[5] = w[2] + nc;
      P.m32[6] = w[3] + nc;
      P.p32 = w[3];
      P.v32 = w[4];
      krylov::cg_mixed_run(P, T);
    } else {
      krylov::krylov_run(P, T);
    }
  }
  if (!leader || !A.record) return;
  const int st = (int)out[krylov::O_STATUS];
  double* R = B.res + (size_t)k * BR_COUNT;
  if (st != CFDB_SOLVER_CONVERGED) {
    *status = A.mode == 0 ? CFDB_SIMPLE_MOMENTUM_FAILURE : CFDB_SIMPLE_PRESSURE_FAILURE;
    B.active[k] = 0;
    return;
  }
  if (A.mode == 0) {
    R[BR_IU + A.comp] = out[krylov::O_B0];
    B.mom_it[k] += (int64_t)out[krylov::O_ITER];
  } else {
    R[BR_IP] = out[krylov::O_B0];
    B.p_it[k] += (int64_t)out[krylov::O_ITER];
  }
}

// The learned p' solves' outcomes (lout: status, iterations, initial
// residual per case, written by the host) applied with k_batch_krylov's
// record rules: a case whose fields went non-finite stops with
// NONFINITE_STATE, a p' solve that did not converge stops it with
// PRESSURE_FAILURE.
__global__ void k_batch_pp_record(BatchDev B, const double* __restrict__ lout) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.ncases; k += gridDim.x * blockDim.x) {
    if (!B.active[k]) continue;
    if (B.flags[(size_t)BF_NONFINITE * B.ncases + k] != 0u) {
      B.status[k] = CFDB_SIMPLE_NONFINITE_STATE;
      B.active[k] = 0;
      continue;
    }
    if ((int)lout[3 * k] != CFDB_SOLVER_CONVERGED) {
      B.status[k] = CFDB_SIMPLE_PRESSURE_FAILURE;
      B.active[k] = 0;
      continue;
    }
    B.res[(size_t)k * BR_COUNT + BR_IP] = lout[3 * k + 2];
    B.p_it[k] += (int64_t)lout[3 * k + 1];
  }
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Events around every launch of an eager profiling iteration; ids: stage
// number, or -1 / -2 for the momentum / p' Krylov kernels.
struct Timeline {
  std::vector<cudaEvent_t> ev;
  std::vector<int> id;
};

}  // namespace
}  // namespace cfdb

using namespace cfdb;

struct cfdb_batch {
  cfdb_context* ctx = nullptr;
  int n = 0, dim = 0;
  cfdb_simple_settings st{};
  std::vector<BCase> hc;
  std::vector<cfdb_simple_case> cases;  // as given (for the result files)
  std::vector<int64_t> cells, faces;
  int64_t cpool = 0, fpool = 0;
  BatchDev D{};
  std::vector<void*> owned;
  // work lists (device), allocated for the smallest tile the tuner may pick
  int *d_ctile_case = nullptr, *d_ftile_case = nullptr, *d_ctile_first = nullptr,
      *d_ftile_first = nullptr;
  int64_t *d_ctile_start = nullptr, *d_ftile_start = nullptr;
  int64_t tile_cap_cells = 0, tile_cap_faces = 0;
  // teams
  int kgrid = 0;
  int *d_bcase_m = nullptr, *d_tfirst_m = nullptr, *d_bcase_p = nullptr, *d_tfirst_p = nullptr;
  unsigned *d_bar = nullptr, *d_err = nullptr;
  double *d_kpart = nullptr, *d_kout = nullptr;
  std::vector<int> h_active;  // host view of the active set the teams were planned for
  std::vector<double> h_pweight;
  // tuning and launch shapes
  cfdb_batch_tuning tune{};
  std::map<std::pair<int, int>, int> occ;  // (stage, threads) -> resident blocks per SM
  bool any_transfer = false, any_ugrad = false;
  int face_flux = 0;
  // graph of one outer iteration
  cudaGraphExec_t exec = nullptr;
  bool dirty = true;
  int64_t launches_per_iteration = 0;
  // pinned mirrors
  int* h_nactive = nullptr;
  unsigned* h_err = nullptr;
  double* h_kout = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int64_t history_cap = 0;
  Timeline* timeline = nullptr;  // set during a profiling iteration
  // learned p' preconditioner: one p' operator per case, bound to the case's
  // pooled face coefficients every outer iteration; the outer iteration is
  // then two graphs around a host loop of the cases' learned solves
  bool learned = false;
  std::vector<cfdb_context*> wctx;  // worker contexts (own streams); case k on wctx[k % size]
  std::vector<cfdb_poperator*> pops;
  cudaGraphExec_t exec_post = nullptr;
  double* d_lout = nullptr;     // per case: status, iterations, initial residual
  double* h_lout = nullptr;     // pinned mirror
  unsigned* h_flags = nullptr;  // pinned mirror of the flags (BF_COUNT x n)
  int* h_act = nullptr;         // pinned mirror of the active set

  ~cfdb_batch() {
    if (ctx) cudaStreamSynchronize(ctx->stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (exec_post) cudaGraphExecDestroy(exec_post);
    for (cfdb_poperator* op : pops) cfdb_poperator_destroy(op);
    for (cfdb_context* w : wctx) cfdb_destroy(w);
    if (h_lout) cudaFreeHost(h_lout);
    if (h_flags) cudaFreeHost(h_flags);
    if (h_act) cudaFreeHost(h_act);
    for (void* p : owned) cudaFree(p);
    if (h_nactive) cudaFreeHost(h_nactive);
    if (h_err) cudaFreeHost(h_err);
    if (h_kout) cudaFreeHost(h_kout);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

namespace {

template <class T>
cfdb_status dalloc(cfdb_batch* b, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
  if (e != cudaSuccess) return cuda_error(b->ctx, e, "batch allocation", __FILE__, __LINE__);
  b->owned.push_back((void*)*p);
  e = cudaMemsetAsync((void*)*p, 0, sizeof(T) * std::max<size_t>(count, 1), b->ctx->stream);
  if (e != cudaSuccess) return cuda_error(b->ctx, e, "batch memset", __FILE__, __LINE__);
  return CFDB_OK;
}

// Stream-ordered copies (the context stream does not synchronise with the
// legacy default stream).
cfdb_status d2h(cfdb_batch* b, void* dst, const void* src, size_t bytes) {
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, b->ctx->stream));
  CFDB_CUDA(b->ctx, cudaStreamSynchronize(b->ctx->stream));
  return CFDB_OK;
}
cfdb_status h2d(cfdb_batch* b, void* dst, const void* src, size_t bytes) {
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, b->ctx->stream));
  CFDB_CUDA(b->ctx, cudaStreamSynchronize(b->ctx->stream));
  return CFDB_OK;
}

int occupancy(cfdb_batch* b, int stage, int threads) {
  const auto key = std::make_pair(stage, threads);
  auto it = b->occ.find(key);
  if (it != b->occ.end()) return it->second;
  int per_sm = 0;
  const void* fn = stage < 0 ? (const void*)k_batch_krylov : batch_stage_kernel(stage);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  per_sm = std::max(per_sm, 1);
  b->occ[key] = per_sm;
  return per_sm;
}

void mark(cfdb_batch* b, int id, cudaStream_t s) {
  Timeline* tl = b->timeline;
  if (!tl) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, s);
  tl->ev.push_back(e);
  tl->id.push_back(id);
}

bool face_stage(int stage) {
  return stage == BS_FACE_VALUES_P || stage == BS_FACE_VALUES_PP || stage == BS_MASS_FLUX ||
         stage == BS_RHIE_CHOW || stage == BS_PFACES || stage == BS_FLUX_CORRECT;
}

void launch_stage(cfdb_batch* b, int stage, int comp, cudaStream_t s) {
  const bool faces = face_stage(stage);
  const int threads = faces ? b->tune.face_threads : b->tune.cell_threads;
  int64_t tiles = faces ? b->D.nface_tiles : b->D.ncell_tiles;
  if (stage == BS_RESIDUAL) tiles = b->D.ncell_tiles + b->D.nface_tiles;
  const int64_t cap = (int64_t)occupancy(b, stage, threads) * b->ctx->num_sms;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, cap));
  batch_stage_launch(b->D, stage, comp, grid, threads, s);
  b->launches_per_iteration += 1;
  mark(b, stage, s);
}

void launch_krylov(cfdb_batch* b, int mode, int comp, int record, cudaStream_t s) {
  const cfdb_linear_settings& L = mode == 0 ? b->st.momentum : b->st.pressure;
  KArgs A{};
  A.B = b->D;
  A.block_case = mode == 0 ? b->d_bcase_m : b->d_bcase_p;
  A.team_first = mode == 0 ? b->d_tfirst_m : b->d_tfirst_p;
  A.mode = mode;
  A.comp = comp;
  A.krylov = L.krylov;
  A.jacobi = L.preconditioner == CFDB_PRECOND_JACOBI;
  A.mixed = mode == 1 && L.precision == CFDB_PRECISION_FP32_REFINED;
  A.abs_tol = L.abs_tol;
  A.rel_tol = L.rel_tol;
  A.max_it = L.max_iterations;
  A.bar = b->d_bar;
  A.error = b->d_err;
  A.kpart = b->d_kpart;
  A.kout = b->d_kout;
  A.record = record;
  k_batch_krylov<<<b->kgrid, krylov::kThreads, 0, s>>>(A);
  b->launches_per_iteration += 1;
  mark(b, mode == 0 ? -1 : -2, s);
}

// Stages of an outer iteration up to the p' solve (record = 0: the linear
// solves leave the case records alone, for the tuner).
void enqueue_prefix(cfdb_batch* b, int record, cudaStream_t s) {
  cudaMemsetAsync(b->D.flags, 0, sizeof(unsigned) * BF_COUNT * (size_t)b->n, s);
  launch_stage(b, BS_FACE_VALUES_P, 0, s);
  launch_stage(b, BS_GG_P, 0, s);
  if (b->any_transfer)
    for (int q = 0; q < 4; ++q) {
      launch_stage(b, BS_GG_P_SWEEP, 0, s);
      launch_stage(b, BS_GG_P_COPY, 0, s);
    }
  for (int comp = 0; comp < b->dim; ++comp) {
    if (b->any_ugrad) launch_stage(b, BS_UGRAD, comp, s);
    launch_stage(b, BS_ASSEMBLE, comp, s);
    launch_krylov(b, 0, comp, record, s);
  }
  launch_stage(b, BS_RESPONSE, 0, s);
  launch_stage(b, BS_MASS_FLUX, 0, s);
  if (b->face_flux == CFDB_FLUX_RHIE_CHOW) launch_stage(b, BS_RHIE_CHOW, 0, s);
  launch_stage(b, BS_PFACES, 0, s);
  launch_stage(b, BS_PROWS, 0, s);
}

// The stages after the p' solve.
void enqueue_suffix(cfdb_batch* b, cudaStream_t s) {
  launch_stage(b, BS_CHECK_PP, 0, s);
  launch_stage(b, BS_FACE_VALUES_PP, 0, s);
  launch_stage(b, BS_GG_PP, 0, s);
  if (b->any_transfer)
    for (int q = 0; q < 4; ++q) {
      launch_stage(b, BS_GG_PP_SWEEP, 0, s);
      launch_stage(b, BS_GG_PP_COPY, 0, s);
    }
  launch_stage(b, BS_CORRECT, 0, s);
  launch_stage(b, BS_FLUX_CORRECT, 0, s);
  launch_stage(b, BS_RESIDUAL, 0, s);
}

void enqueue_iteration(cfdb_batch* b, cudaStream_t s) {
  b->launches_per_iteration = 0;
  enqueue_prefix(b, 1, s);
  launch_krylov(b, 1, 0, 1, s);
  enqueue_suffix(b, s);
}

// With the learned p' preconditioner: the record of the host's p' outcomes,
// then the stages after the p' solve.
void enqueue_learned_post(cfdb_batch* b, cudaStream_t s) {
  k_batch_pp_record<<<std::max(1, (b->n + 255) / 256), 256, 0, s>>>(b->D, b->d_lout);
  b->launches_per_iteration += 1;
  mark(b, -2, s);
  enqueue_suffix(b, s);
}

// Every active case's p' system by the single-case learned solve, on its
// pooled face coefficients, right-hand side and p' (zero) in place; the
// outcomes go to d_lout.  The stages before (enqueue_prefix) must have run.
// The cases are shared among the worker contexts, each on its own host
// thread and stream, so several solves run on the GPU at once; every solve
// synchronises its own stream, and the host has synchronised the batch's
// stream before, so the work is ordered against both graphs.
cfdb_status run_learned_pprime(cfdb_batch* b) {
  cfdb_context* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  const int n = b->n;
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->h_flags, b->D.flags, sizeof(unsigned) * BF_COUNT * (size_t)n,
                                 cudaMemcpyDeviceToHost, s));
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->h_act, b->D.active, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost,
                                 s));
  CFDB_CUDA(ctx, cudaStreamSynchronize(s));
  const int nw = (int)b->wctx.size();
  std::vector<cfdb_status> wrc(nw, CFDB_OK);
  std::vector<int64_t> l0(nw);
  for (int w = 0; w < nw; ++w) l0[w] = b->wctx[w]->launches;
  auto work = [&](int w) {
    cfdb_context* wc = b->wctx[w];
    if (cudaSetDevice(wc->device) != cudaSuccess) {
      wrc[w] = set_error(wc, CFDB_ERR_CUDA, "cudaSetDevice on a batch worker thread");
      return;
    }
    for (int k = w; k < n; k += nw) {
      double* o = b->h_lout + 3 * (size_t)k;
      o[0] = -1.0;
      o[1] = 0.0;
      o[2] = 0.0;
      if (!b->h_act[k] || b->h_flags[(size_t)BF_NONFINITE * n + k] != 0u) continue;
      if (b->h_flags[(size_t)BF_PP * n + k] & BFLAG_NONFINITE_INPUT) {
        o[0] = CFDB_SOLVER_NONFINITE_INPUT;
        continue;
      }
      cfdb_status rc = poperator_bind_faces(wc, b->pops[k], b->D.D + b->hc[k].f0, false);
      cfdb_linear_result r{};
      if (rc == CFDB_OK)
        rc = cfdb_poperator_solve_device(wc, b->pops[k], &b->st.pressure, b->D.prhs + b->hc[k].c0,
                                         b->D.pp + b->hc[k].c0, nullptr, 0, &r);
      if (rc != CFDB_OK) {
        wrc[w] = rc;
        return;
      }
      o[0] = r.status;
      o[1] = (double)r.iterations;
      o[2] = r.initial_residual;
    }
  };
  {
    // a worker whose thread cannot be started runs on this thread afterwards
    std::vector<std::thread> threads;
    std::vector<int> here = {0};
    for (int w = 1; w < nw; ++w) {
      try {
        threads.emplace_back(work, w);
      } catch (...) {
        here.push_back(w);
      }
    }
    for (int w : here) work(w);
    for (std::thread& t : threads) t.join();
  }
  for (int w = 0; w < nw; ++w) {
    ctx->launches += b->wctx[w]->launches - l0[w];
    if (wrc[w] != CFDB_OK)
      return set_error(ctx, wrc[w], std::string("learned p' solve of a batched case: ") +
                                        b->wctx[w]->last_error);
  }
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->d_lout, b->h_lout, sizeof(double) * 3 * (size_t)n,
                                 cudaMemcpyHostToDevice, s));
  return CFDB_OK;
}

cfdb_status upload_tiles(cfdb_batch* b) {
  const int n = b->n;
  std::vector<int> cf(n + 1), ff(n + 1);
  cfdb_batch_plan_tiles(n, b->cells.data(), b->tune.cell_tile, cf.data(), nullptr, nullptr);
  cfdb_batch_plan_tiles(n, b->faces.data(), b->tune.face_tile, ff.data(), nullptr, nullptr);
  if (cf[n] > b->tile_cap_cells || ff[n] > b->tile_cap_faces)
    return set_error(b->ctx, CFDB_ERR_INVALID_ARGUMENT, "tile list larger than its allocation");
  std::vector<int> cc(cf[n]), fc(ff[n]);
  std::vector<int64_t> cs(cf[n]), fs(ff[n]);
  cfdb_batch_plan_tiles(n, b->cells.data(), b->tune.cell_tile, cf.data(), cc.data(), cs.data());
  cfdb_batch_plan_tiles(n, b->faces.data(), b->tune.face_tile, ff.data(), fc.data(), fs.data());
  cudaStream_t s = b->ctx->stream;
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(b->d_ctile_case, cc.data(), sizeof(int) * cc.size(), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(b->d_ctile_start, cs.data(), sizeof(int64_t) * cs.size(), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(b->d_ftile_case, fc.data(), sizeof(int) * fc.size(), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(b->d_ftile_start, fs.data(), sizeof(int64_t) * fs.size(), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(b->d_ctile_first, cf.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(b->d_ftile_first, ff.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(b->ctx, cudaStreamSynchronize(s));
  b->D.ncell_tiles = cf[n];
  b->D.nface_tiles = ff[n];
  b->D.cell_tile = b->tune.cell_tile;
  b->D.face_tile = b->tune.face_tile;
  b->dirty = true;
  return CFDB_OK;
}

// Plans and uploads one team table (mode 0 momentum, 1 p').
cfdb_status upload_teams(cfdb_batch* b, int mode, const std::vector<double>& w) {
  const int n = b->n;
  std::vector<int> tf(n + 1), bc(b->kgrid);
  cfdb_status rc = cfdb_batch_plan_teams(n, w.data(), b->cells.data(), b->h_active.data(), b->kgrid,
                                         kMinCellsPerBlock, tf.data(), bc.data());
  if (rc != CFDB_OK) return set_error(b->ctx, rc, "more active cases than Krylov blocks");
  cudaStream_t s = b->ctx->stream;
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(mode == 0 ? b->d_tfirst_m : b->d_tfirst_p, tf.data(),
                                    sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(b->ctx, cudaMemcpyAsync(mode == 0 ? b->d_bcase_m : b->d_bcase_p, bc.data(),
                                    sizeof(int) * b->kgrid, cudaMemcpyHostToDevice, s));
  // the host vectors die here: finish the copies
  CFDB_CUDA(b->ctx, cudaStreamSynchronize(s));
  return CFDB_OK;
}

std::vector<double> power_weights(const cfdb_batch* b, double e) {
  std::vector<double> w(b->n);
  for (int k = 0; k < b->n; ++k) w[k] = std::pow((double)b->cells[k], e);
  return w;
}

cfdb_status plan_all_teams(cfdb_batch* b) {
  cfdb_status rc = upload_teams(b, 0, power_weights(b, 1.0));
  if (rc != CFDB_OK) return rc;
  return upload_teams(b, 1, b->h_pweight);
}

cfdb_status refresh_active(cfdb_batch* b, bool* changed) {
  std::vector<int> act(b->n);
  cfdb_status rc = d2h(b, act.data(), b->D.active, sizeof(int) * b->n);
  if (rc != CFDB_OK) return rc;
  *changed = act != b->h_active;
  b->h_active = act;
  return CFDB_OK;
}

cfdb_status build_graph(cfdb_batch* b) {
  cfdb_context* ctx = b->ctx;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  // occupancy queries are answered before the capture starts
  occupancy(b, -1, krylov::kThreads);
  for (int st = 0; st < BS_COUNT; ++st) {
    occupancy(b, st, b->tune.cell_threads);
    occupancy(b, st, b->tune.face_threads);
  }
  if (b->exec_post) {
    cudaGraphExecDestroy(b->exec_post);
    b->exec_post = nullptr;
  }
  auto capture = [&](cudaGraphExec_t* out, auto body) -> cfdb_status {
    cudaGraph_t g = nullptr;
    CFDB_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    body();
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (e != cudaSuccess) return cuda_error(ctx, e, "batch graph capture", __FILE__, __LINE__);
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_error(ctx, e, "batch graph instantiation", __FILE__, __LINE__);
    return CFDB_OK;
  };
  cfdb_status rc;
  if (b->learned) {
    b->launches_per_iteration = 0;
    if ((rc = capture(&b->exec, [&] { enqueue_prefix(b, 1, ctx->stream); }))) return rc;
    if ((rc = capture(&b->exec_post, [&] { enqueue_learned_post(b, ctx->stream); }))) return rc;
  } else if ((rc = capture(&b->exec, [&] { enqueue_iteration(b, ctx->stream); }))) {
    return rc;
  }
  b->dirty = false;
  return CFDB_OK;
}

cfdb_status check_error(cfdb_batch* b) {
  unsigned err = 0;
  cfdb_status rc = d2h(b, &err, b->d_err, sizeof(unsigned));
  if (rc != CFDB_OK) return rc;
  if (err)
    return set_error(b->ctx, CFDB_ERR_DEVICE_TIMEOUT,
                     "a team barrier of the batched Krylov solves timed out (no fault)");
  return CFDB_OK;
}

bool tuning_valid(const cfdb_batch_tuning& t) {
  auto ok_threads = [](int v) { return v >= 32 && v <= 1024 && v % 32 == 0; };
  return ok_threads(t.cell_threads) && ok_threads(t.face_threads) && t.cell_tile >= t.cell_threads &&
         t.face_tile >= t.face_threads && t.cell_tile <= (1 << 20) && t.face_tile <= (1 << 20) &&
         std::isfinite(t.team_exponent) && t.team_exponent >= 0.0 && t.team_exponent <= 3.0;
}

cfdb_status apply_tuning(cfdb_batch* b, const cfdb_batch_tuning& t) {
  if (!tuning_valid(t)) return set_error(b->ctx, CFDB_ERR_INVALID_ARGUMENT, "invalid batch tuning");
  b->tune = t;
  cfdb_status rc = upload_tiles(b);
  if (rc != CFDB_OK) return rc;
  b->h_pweight = power_weights(b, t.team_exponent);
  rc = plan_all_teams(b);
  b->dirty = true;
  return rc;
}

}  // namespace

extern "C" {

cfdb_status cfdb_batch_plan_tiles(int ncases, const int64_t* count, int tile, int* first,
                                  int* tile_case, int64_t* tile_start) {
  if (ncases < 0 || !count || tile < 1 || !first) return CFDB_ERR_INVALID_ARGUMENT;
  int64_t t = 0;
  for (int k = 0; k < ncases; ++k) {
    if (count[k] < 0) return CFDB_ERR_INVALID_ARGUMENT;
    first[k] = (int)t;
    const int64_t nt = (count[k] + tile - 1) / tile;
    if (tile_case && tile_start)
      for (int64_t q = 0; q < nt; ++q) {
        tile_case[t + q] = k;
        tile_start[t + q] = q * tile;
      }
    t += nt;
    if (t > (int64_t)1 << 30) return CFDB_ERR_UNSUPPORTED;
  }
  first[ncases] = (int)t;
  return CFDB_OK;
}

cfdb_status cfdb_batch_plan_teams(int ncases, const double* weight, const int64_t* cells,
                                  const int* active, int nblocks, int64_t min_cells_per_block,
                                  int* team_first, int* block_case) {
  if (ncases < 0 || !weight || !cells || !active || nblocks < 1 || min_cells_per_block < 1 ||
      !team_first || !block_case)
    return CFDB_ERR_INVALID_ARGUMENT;
  std::vector<int64_t> blocks(ncases, 0), cap(ncases, 0);
  int nact = 0;
  for (int k = 0; k < ncases; ++k) {
    if (!active[k] || cells[k] <= 0) continue;
    if (!(weight[k] >= 0.0) || !std::isfinite(weight[k])) return CFDB_ERR_INVALID_ARGUMENT;
    blocks[k] = 1;
    cap[k] = std::max<int64_t>(1, cells[k] / min_cells_per_block);
    ++nact;
  }
  if (nact > nblocks) return CFDB_ERR_UNSUPPORTED;
  int64_t left = nblocks - nact;
  while (left > 0) {
    int best = -1;
    double bw = -1.0;
    for (int k = 0; k < ncases; ++k) {
      if (blocks[k] == 0 || blocks[k] >= cap[k]) continue;
      const double per = weight[k] / (double)blocks[k];
      if (per > bw) {
        bw = per;
        best = k;
      }
    }
    if (best < 0) break;
    ++blocks[best];
    --left;
  }
  int64_t pos = 0;
  for (int k = 0; k < ncases; ++k) {
    team_first[k] = (int)pos;
    for (int64_t q = 0; q < blocks[k]; ++q) block_case[pos + q] = k;
    pos += blocks[k];
  }
  team_first[ncases] = (int)pos;
  for (int64_t q = pos; q < nblocks; ++q) block_case[q] = -1;
  return CFDB_OK;
}

cfdb_status cfdb_batch_create(cfdb_context* ctx, int ncases, const cfdb_simple_case* cases,
                              const cfdb_simple_settings* st, int64_t history_cap, cfdb_batch** out) {
  if (!ctx || !out || !cases || !st || ncases < 1 || history_cap < 0) return CFDB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const int dim = cases[0].grid.dim;
  for (int k = 0; k < ncases; ++k) {
    cfdb_status rc = simple_validate(ctx, &cases[k], st);
    if (rc != CFDB_OK) return rc;
    if (cases[k].grid.dim != dim) return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "a batch holds one dimension");
    for (int a = 0; a < 3; ++a)
      if (cases[k].nodes[a])
        return set_error(ctx, CFDB_ERR_UNSUPPORTED, "a batch holds uniform grids only");
  }
  if (st->max_outer < 1 || !(st->alpha_u > 0.0) || st->alpha_u > 1.0 || !(st->alpha_p > 0.0) ||
      st->alpha_p > 1.0 ||
      st->momentum.max_iterations < 1 || st->pressure.max_iterations < 1)
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "invalid relaxation or iteration limits");
  for (const cfdb_linear_settings* L : {&st->momentum, &st->pressure}) {
    const bool learned_pp = L == &st->pressure && L->preconditioner == CFDB_PRECOND_LEARNED_MG &&
                            L->krylov == CFDB_KRYLOV_CG && L->precision == CFDB_PRECISION_FP64;
    if ((L->preconditioner != CFDB_PRECOND_NONE && L->preconditioner != CFDB_PRECOND_JACOBI &&
         !learned_pp) ||
        (L->krylov != CFDB_KRYLOV_CG && L->krylov != CFDB_KRYLOV_BICGSTAB))
      return set_error(ctx, CFDB_ERR_UNSUPPORTED,
                       "batched solves support CG/BiCGSTAB with no or Jacobi preconditioning, "
                       "or an FP64 CG p' solve with the learned preconditioner");
    const bool mixed_pp = L == &st->pressure && L->krylov == CFDB_KRYLOV_CG &&
                          L->precision == CFDB_PRECISION_FP32_REFINED;
    if (L->precision != CFDB_PRECISION_FP64 && !mixed_pp)
      return set_error(ctx, CFDB_ERR_UNSUPPORTED,
                       "batched solves take FP64, or FP32_REFINED for a CG p' solve");
  }
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  std::unique_ptr<cfdb_batch> b(new cfdb_batch());
  b->ctx = ctx;
  b->n = ncases;
  b->dim = dim;
  b->st = *st;
  b->history_cap = history_cap;
  b->face_flux = st->face_flux == CFDB_FLUX_AUTOMATIC ? (dim == 2 ? CFDB_FLUX_LINEAR : CFDB_FLUX_RHIE_CHOW)
                                                      : st->face_flux;
  b->hc.resize(ncases);
  b->cases.assign(cases, cases + ncases);
  b->cells.resize(ncases);
  b->faces.resize(ncases);
  int64_t cp = 0, fp = 0;
  for (int k = 0; k < ncases; ++k) {
    BCase& K = b->hc[k];
    std::memset(&K, 0, sizeof(K));
    K.G = simple_geometry(cases[k]);
    K.rho = cases[k].rho;
    K.mu = cases[k].mu;
    bool fixed_value = false;
    for (int q = 0; q < 2 * dim; ++q) fixed_value |= cases[k].pbc_type[q] == CFDB_PBC_FIXED_VALUE;
    K.pin = fixed_value ? 0 : 1;
    K.ref = st->reference_cell;
    if (K.ref < 0 || K.ref >= K.G.nc)
      return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "reference cell out of range for a case");
    K.need_ugrad = (st->scheme == CFDB_SCHEME_LINEAR_UPWIND || simple_wall_offsets(K.G)) ? 1 : 0;
    for (int q = 0; q < 6; ++q) {
      K.pctype[q] = cases[k].pbc_type[q] == CFDB_PBC_FIXED_VALUE ? CFDB_PBC_FIXED_VALUE : CFDB_PBC_FIXED_GRADIENT;
      K.pcvalue[q] = 0.0;
    }
    K.c0 = cp;
    K.f0 = fp;
    b->cells[k] = K.G.nc;
    b->faces[k] = K.G.nf;
    cp += round_up(K.G.nc, kAlign);
    fp += round_up(K.G.nf, kAlign);
    b->any_transfer |= K.G.transfer != 0;
    b->any_ugrad |= K.need_ugrad != 0;
  }
  b->cpool = cp;
  b->fpool = fp;
  BatchDev& D = b->D;
  D.ncases = ncases;
  D.dim = dim;
  cfdb_status rc;
  auto cell = [&](double** p) { return dalloc(b.get(), p, (size_t)cp); };
  auto face = [&](double** p) { return dalloc(b.get(), p, (size_t)fp); };
  for (int a = 0; a < 3; ++a)
    if ((rc = cell(&D.U[a])) || (rc = cell(&D.Us[a])) || (rc = cell(&D.mdiag[a])) ||
        (rc = cell(&D.gradP[a])) || (rc = cell(&D.gradU[a])) || (rc = cell(&D.gtmp[a])) ||
        (rc = cell(&D.dres[a])))
      return rc;
  for (int q = 0; q < 6; ++q)
    if ((rc = cell(&D.moff[q])) || (rc = cell(&D.poff[q]))) return rc;
  if ((rc = cell(&D.mrhs)) || (rc = cell(&D.p)) || (rc = cell(&D.pdiag)) || (rc = cell(&D.prhs)) ||
      (rc = cell(&D.pp)) || (rc = cell(&D.kinv)) || (rc = cell(&D.kr)) || (rc = cell(&D.krh)) ||
      (rc = cell(&D.kv)) || (rc = cell(&D.kp)) || (rc = cell(&D.ks)) || (rc = cell(&D.kt)) ||
      (rc = face(&D.Fbuf[0])) || (rc = face(&D.Fbuf[1])) || (rc = face(&D.Fs)) || (rc = face(&D.fv)) ||
      (rc = face(&D.D)))
    return rc;
  BCase* dc = nullptr;
  if ((rc = dalloc(b.get(), &dc, ncases))) return rc;
  if ((rc = h2d(b.get(), dc, b->hc.data(), sizeof(BCase) * ncases))) return rc;
  D.cases = dc;
  if ((rc = dalloc(b.get(), &D.active, ncases)) || (rc = dalloc(b.get(), &D.status, ncases)) ||
      (rc = dalloc(b.get(), &D.fsel, ncases)) || (rc = dalloc(b.get(), &D.outer, ncases)) ||
      (rc = dalloc(b.get(), &D.mom_it, ncases)) || (rc = dalloc(b.get(), &D.p_it, ncases)) ||
      (rc = dalloc(b.get(), &D.res, (size_t)ncases * BR_COUNT)) ||
      (rc = dalloc(b.get(), &D.flags, (size_t)ncases * BF_COUNT)) ||
      (rc = dalloc(b.get(), &D.ticket, 2)) || (rc = dalloc(b.get(), &D.nactive, 1)))
    return rc;
  if (history_cap > 0 && (rc = dalloc(b.get(), &D.history, (size_t)ncases * history_cap * 5))) return rc;
  D.history_cap = history_cap;
  D.max_outer = st->max_outer;
  D.alpha_u = st->alpha_u;
  D.alpha_p = st->alpha_p;
  D.tol_u = st->tol_u;
  D.tol_p = st->tol_p;
  D.tol_c = st->tol_c;
  D.scheme = st->scheme;
  D.face_flux = b->face_flux;
  D.mom_jacobi = st->momentum.preconditioner == CFDB_PRECOND_JACOBI;
  D.p_jacobi = st->pressure.preconditioner == CFDB_PRECOND_JACOBI;
  // every case starts active with status "running"
  std::vector<int> ones(ncases, 1), running(ncases, -1);
  if ((rc = h2d(b.get(), D.active, ones.data(), sizeof(int) * ncases)) ||
      (rc = h2d(b.get(), D.status, running.data(), sizeof(int) * ncases)))
    return rc;
  b->h_active = ones;
  // work lists sized for the smallest tile the tuner tries (32 items)
  int64_t ct = 0, ft = 0;
  for (int k = 0; k < ncases; ++k) {
    ct += (b->cells[k] + 31) / 32;
    ft += (b->faces[k] + 31) / 32;
  }
  b->tile_cap_cells = ct;
  b->tile_cap_faces = ft;
  if ((rc = dalloc(b.get(), &b->d_ctile_case, ct)) || (rc = dalloc(b.get(), &b->d_ctile_start, ct)) ||
      (rc = dalloc(b.get(), &b->d_ftile_case, ft)) || (rc = dalloc(b.get(), &b->d_ftile_start, ft)) ||
      (rc = dalloc(b.get(), &b->d_ctile_first, ncases + 1)) ||
      (rc = dalloc(b.get(), &b->d_ftile_first, ncases + 1)))
    return rc;
  D.ctile_case = b->d_ctile_case;
  D.ctile_start = b->d_ctile_start;
  D.ftile_case = b->d_ftile_case;
  D.ftile_start = b->d_ftile_start;
  D.ctile_first = b->d_ctile_first;
  D.ftile_first = b->d_ftile_first;
  // partials: one double per tile
  if ((rc = dalloc(b.get(), &D.partials, (size_t)(ct + ft)))) return rc;
  // Krylov teams: the grid is what fits on the GPU at once
  b->kgrid = occupancy(b.get(), -1, krylov::kThreads) * ctx->num_sms;
  if (ncases > b->kgrid)
    return set_error(ctx, CFDB_ERR_UNSUPPORTED, "more cases than resident Krylov blocks");
  if ((rc = dalloc(b.get(), &b->d_bcase_m, b->kgrid)) || (rc = dalloc(b.get(), &b->d_bcase_p, b->kgrid)) ||
      (rc = dalloc(b.get(), &b->d_tfirst_m, ncases + 1)) ||
      (rc = dalloc(b.get(), &b->d_tfirst_p, ncases + 1)) ||
      (rc = dalloc(b.get(), &b->d_bar, 2 * (size_t)ncases)) || (rc = dalloc(b.get(), &b->d_err, 1)) ||
      (rc = dalloc(b.get(), &b->d_kpart, 6 * (size_t)b->kgrid)) ||
      (rc = dalloc(b.get(), &b->d_kout, 2 * (size_t)ncases * kKoutStride)))
    return rc;
  CFDB_CUDA(ctx, cudaMallocHost((void**)&b->h_nactive, sizeof(int)));
  CFDB_CUDA(ctx, cudaMallocHost((void**)&b->h_err, sizeof(unsigned)));
  CFDB_CUDA(ctx, cudaMallocHost((void**)&b->h_kout, sizeof(double) * 2 * ncases * kKoutStride));
  *b->h_nactive = ncases;
  CFDB_CUDA(ctx, cudaEventCreate(&b->e0));
  CFDB_CUDA(ctx, cudaEventCreate(&b->e1));
  if (st->pressure.preconditioner == CFDB_PRECOND_LEARNED_MG) {
    b->learned = true;
    if ((rc = dalloc(b.get(), &b->d_lout, 3 * (size_t)ncases))) return rc;
    CFDB_CUDA(ctx, cudaMallocHost((void**)&b->h_lout, sizeof(double) * 3 * ncases));
    CFDB_CUDA(ctx, cudaMallocHost((void**)&b->h_flags, sizeof(unsigned) * BF_COUNT * ncases));
    CFDB_CUDA(ctx, cudaMallocHost((void**)&b->h_act, sizeof(int) * ncases));
    // worker contexts for concurrent per-case solves (their own streams)
    const int nw = std::min(kLearnedWorkers, ncases);
    for (int w = 0; w < nw; ++w) {
      cfdb_context* wc = nullptr;
      if ((rc = cfdb_create(ctx->device, nullptr, &wc)) != CFDB_OK)
        return set_error(ctx, rc, "batch worker context");
      b->wctx.push_back(wc);
    }
    b->pops.assign(ncases, nullptr);
    for (int k = 0; k < ncases; ++k)
      if ((rc = cfdb_poperator_create_uniform(b->wctx[k % nw], &cases[k].grid, 1.0, 0u,
                                              b->hc[k].pin, b->hc[k].ref, &b->pops[k])))
        return set_error(ctx, rc, b->wctx[k % nw]->last_error);
  }
  cfdb_batch_tuning t{};
  t.cell_threads = 256;
  t.cell_tile = 1024;
  t.face_threads = 256;
  t.face_tile = 1024;
  t.team_exponent = 1.5;
  t.adaptive_teams = 1;
  if ((rc = apply_tuning(b.get(), t))) return rc;
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *out = b.release();
  return CFDB_OK;
}

void cfdb_batch_destroy(cfdb_batch* b) { delete b; }

int cfdb_batch_cases(const cfdb_batch* b) { return b ? b->n : 0; }

cfdb_status cfdb_batch_set_state(cfdb_batch* b, int k, const double* u, const double* v,
                                 const double* w, const double* p) {
  if (!b || k < 0 || k >= b->n || !u || !v || !p || (b->dim == 3 && !w)) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  const BCase& K = b->hc[k];
  const size_t bytes = sizeof(double) * (size_t)K.G.nc;
  const int64_t o = K.c0;
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.U[0] + o, u, bytes, cudaMemcpyHostToDevice, s));
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.U[1] + o, v, bytes, cudaMemcpyHostToDevice, s));
  if (b->dim == 3) CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.U[2] + o, w, bytes, cudaMemcpyHostToDevice, s));
  else CFDB_CUDA(ctx, cudaMemsetAsync(b->D.U[2] + o, 0, bytes, s));
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.p + o, p, bytes, cudaMemcpyHostToDevice, s));
  const double* Uc[3] = {b->D.U[0] + o, b->D.U[1] + o, b->D.U[2] + o};
  launch_mass_flux(K.G, K.rho, Uc, b->D.Fbuf[0] + K.f0, s);
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx);
  // a non-finite initial state stops the case before its first iteration,
  // as cfdb_simple_solve's initial check does
  auto finite = [&](const double* a) {
    for (int64_t i = 0; i < K.G.nc; ++i)
      if (!std::isfinite(a[i])) return false;
    return true;
  };
  const bool ok = finite(u) && finite(v) && (b->dim == 2 || finite(w)) && finite(p);
  const int act = ok ? 1 : 0, status = ok ? -1 : CFDB_SIMPLE_NONFINITE_STATE, zero = 0;
  const int64_t z64 = 0;
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.active + k, &act, sizeof(int), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.status + k, &status, sizeof(int), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.fsel + k, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.outer + k, &z64, sizeof(int64_t), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.mom_it + k, &z64, sizeof(int64_t), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(ctx, cudaMemcpyAsync(b->D.p_it + k, &z64, sizeof(int64_t), cudaMemcpyHostToDevice, s));
  CFDB_CUDA(ctx, cudaMemsetAsync(b->D.res + (size_t)k * BR_COUNT, 0, sizeof(double) * BR_COUNT, s));
  CFDB_CUDA(ctx, cudaStreamSynchronize(s));
  bool changed = false;
  cfdb_status rc = refresh_active(b, &changed);
  if (rc != CFDB_OK) return rc;
  if (changed) rc = plan_all_teams(b);
  return rc;
}

cfdb_status cfdb_batch_get_state(cfdb_batch* b, int k, double* u, double* v, double* w, double* p,
                                 double* flux) {
  if (!b || k < 0 || k >= b->n) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  const BCase& K = b->hc[k];
  const size_t bytes = sizeof(double) * (size_t)K.G.nc;
  const int64_t o = K.c0;
  int fsel = 0;
  CFDB_CUDA(ctx, cudaMemcpyAsync(&fsel, b->D.fsel + k, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (u) CFDB_CUDA(ctx, cudaMemcpyAsync(u, b->D.U[0] + o, bytes, cudaMemcpyDeviceToHost, s));
  if (v) CFDB_CUDA(ctx, cudaMemcpyAsync(v, b->D.U[1] + o, bytes, cudaMemcpyDeviceToHost, s));
  if (w && b->dim == 3) CFDB_CUDA(ctx, cudaMemcpyAsync(w, b->D.U[2] + o, bytes, cudaMemcpyDeviceToHost, s));
  if (p) CFDB_CUDA(ctx, cudaMemcpyAsync(p, b->D.p + o, bytes, cudaMemcpyDeviceToHost, s));
  CFDB_CUDA(ctx, cudaStreamSynchronize(s));
  if (flux) return d2h(b, flux, b->D.Fbuf[fsel & 1] + K.f0, sizeof(double) * (size_t)K.G.nf);
  return CFDB_OK;
}

cfdb_status cfdb_batch_get_tuning(cfdb_batch* b, cfdb_batch_tuning* t) {
  if (!b || !t) return CFDB_ERR_INVALID_ARGUMENT;
  *t = b->tune;
  return CFDB_OK;
}

cfdb_status cfdb_batch_set_tuning(cfdb_batch* b, const cfdb_batch_tuning* t) {
  if (!b || !t) return CFDB_ERR_INVALID_ARGUMENT;
  return apply_tuning(b, *t);
}

cfdb_status cfdb_batch_iterate(cfdb_batch* b, int64_t nmax, cfdb_batch_stats* stats) {
  if (!b || nmax < 0) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  cfdb_batch_stats S{};
  cfdb_status rc;
  bool changed = false;
  if ((rc = refresh_active(b, &changed))) return rc;
  if (changed && (rc = plan_all_teams(b))) return rc;
  if (b->dirty && (rc = build_graph(b))) return rc;
  int nact = 0;
  for (int a : b->h_active) nact += a;
  for (int64_t it = 0; it < nmax && nact > 0; ++it) {
    CFDB_CUDA(ctx, cudaEventRecord(b->e0, s));
    CFDB_CUDA(ctx, cudaGraphLaunch(b->exec, s));
    if (b->learned) {
      const int64_t l0 = ctx->launches;
      if ((rc = run_learned_pprime(b))) return rc;
      S.kernel_launches += ctx->launches - l0;
      CFDB_CUDA(ctx, cudaGraphLaunch(b->exec_post, s));
    }
    CFDB_CUDA(ctx, cudaEventRecord(b->e1, s));
    CFDB_CUDA(ctx, cudaMemcpyAsync(b->h_nactive, b->D.nactive, sizeof(int), cudaMemcpyDeviceToHost, s));
    CFDB_CUDA(ctx, cudaMemcpyAsync(b->h_err, b->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    if (b->tune.adaptive_teams)
      CFDB_CUDA(ctx, cudaMemcpyAsync(b->h_kout, b->d_kout, sizeof(double) * 2 * b->n * kKoutStride,
                                     cudaMemcpyDeviceToHost, s));
    CFDB_CUDA(ctx, cudaStreamSynchronize(s));
    float ms = 0.f;
    CFDB_CUDA(ctx, cudaEventElapsedTime(&ms, b->e0, b->e1));
    S.device_ms += ms;
    S.graph_launches += 1;
    S.kernel_launches += b->launches_per_iteration;
    ctx->launches += b->launches_per_iteration;
    if (*b->h_err)
      return set_error(ctx, CFDB_ERR_DEVICE_TIMEOUT,
                       "a team barrier of the batched Krylov solves timed out (no fault)");
    const int now = *b->h_nactive;
    if (now == 0) {
      nact = 0;
      break;
    }
    if ((rc = refresh_active(b, &changed))) return rc;
    if (b->tune.adaptive_teams) {
      for (int k = 0; k < b->n; ++k) {
        const double pit = b->h_kout[((size_t)b->n + k) * kKoutStride + krylov::O_ITER];
        b->h_pweight[k] = (double)b->cells[k] * std::max(1.0, pit);
      }
      if ((rc = upload_teams(b, 1, b->h_pweight))) return rc;
      if (changed && (rc = upload_teams(b, 0, power_weights(b, 1.0)))) return rc;
    } else if (changed && (rc = plan_all_teams(b))) {
      return rc;
    }
    nact = now;
  }
  S.active = nact;
  if (stats) *stats = S;
  return CFDB_OK;
}

cfdb_status cfdb_batch_profile_iteration(cfdb_batch* b, int* ids, double* ms, int cap, int* count) {
  if (!b || cap < 0 || (cap > 0 && (!ids || !ms))) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  cfdb_status rc;
  bool changed = false;
  if ((rc = refresh_active(b, &changed))) return rc;
  if (changed && (rc = plan_all_teams(b))) return rc;
  Timeline tl;
  b->timeline = &tl;
  mark(b, -100, s);
  if (b->learned) {
    b->launches_per_iteration = 0;
    enqueue_prefix(b, 1, s);
    if ((rc = run_learned_pprime(b))) {
      b->timeline = nullptr;
      return rc;
    }
    enqueue_learned_post(b, s);
  } else {
    enqueue_iteration(b, s);
  }
  b->timeline = nullptr;
  b->dirty = true;  // the graph's launch count is re-counted at its next capture
  cudaError_t e = cudaStreamSynchronize(s);
  int n = 0;
  for (size_t q = 1; q < tl.ev.size() && e == cudaSuccess; ++q) {
    float t = 0.f;
    cudaEventElapsedTime(&t, tl.ev[q - 1], tl.ev[q]);
    if (n < cap) {
      ids[n] = tl.id[q];
      ms[n] = t;
    }
    ++n;
  }
  for (cudaEvent_t ev : tl.ev) cudaEventDestroy(ev);
  if (e != cudaSuccess) return cuda_error(ctx, e, "batch profiling iteration", __FILE__, __LINE__);
  ctx->launches += b->launches_per_iteration;
  if (count) *count = n;
  return check_error(b);
}

cfdb_status cfdb_batch_results(cfdb_batch* b, cfdb_simple_result* results) {
  if (!b || !results) return CFDB_ERR_INVALID_ARGUMENT;
  const int n = b->n;
  std::vector<int> st(n);
  std::vector<int64_t> outer(n), mit(n), pit(n);
  std::vector<double> res((size_t)n * BR_COUNT);
  cfdb_status rc;
  if ((rc = d2h(b, st.data(), b->D.status, sizeof(int) * n)) ||
      (rc = d2h(b, outer.data(), b->D.outer, sizeof(int64_t) * n)) ||
      (rc = d2h(b, mit.data(), b->D.mom_it, sizeof(int64_t) * n)) ||
      (rc = d2h(b, pit.data(), b->D.p_it, sizeof(int64_t) * n)) ||
      (rc = d2h(b, res.data(), b->D.res, sizeof(double) * res.size())))
    return rc;
  for (int k = 0; k < n; ++k) {
    cfdb_simple_result& r = results[k];
    std::memset(&r, 0, sizeof(r));
    r.status = st[k] < 0 ? CFDB_SIMPLE_MAX_ITERATIONS : st[k];
    r.iterations = outer[k];
    const double* R = res.data() + (size_t)k * BR_COUNT;
    r.final_u = R[BR_U];
    r.final_v = R[BR_V];
    r.final_w = R[BR_W];
    r.final_p = R[BR_P];
    r.final_continuity = R[BR_CONT];
    r.global_imbalance = R[BR_GLOB];
    r.momentum_linear_iterations = mit[k];
    r.pressure_linear_iterations = pit[k];
  }
  return CFDB_OK;
}

cfdb_status cfdb_batch_history(cfdb_batch* b, int k, double* history, int64_t cap, int64_t* rows) {
  if (!b || k < 0 || k >= b->n || cap < 0 || (cap > 0 && !history)) return CFDB_ERR_INVALID_ARGUMENT;
  int64_t outer = 0;
  cfdb_status rc = d2h(b, &outer, b->D.outer + k, sizeof(int64_t));
  if (rc != CFDB_OK) return rc;
  const int64_t kept = std::min(std::min(outer, b->history_cap), cap);
  if (kept > 0 && (rc = d2h(b, history, b->D.history + (size_t)k * b->history_cap * 5,
                            sizeof(double) * 5 * kept)))
    return rc;
  if (rows) *rows = kept;
  return CFDB_OK;
}

cfdb_status cfdb_batch_write_results(cfdb_batch* b, int k, const char* dir, int* fields_written) {
  if (!b || k < 0 || k >= b->n || !dir) return CFDB_ERR_INVALID_ARGUMENT;
  const BCase& K = b->hc[k];
  const size_t n = (size_t)K.G.nc;
  std::vector<double> u(n), v(n), w(n), p(n);
  cfdb_status rc = cfdb_batch_get_state(b, k, u.data(), v.data(), w.data(), p.data(), nullptr);
  if (rc != CFDB_OK) return rc;
  int64_t outer = 0;
  std::vector<double> res(BR_COUNT);
  if ((rc = d2h(b, &outer, b->D.outer + k, sizeof(int64_t))) ||
      (rc = d2h(b, res.data(), b->D.res + (size_t)k * BR_COUNT, sizeof(double) * BR_COUNT)))
    return rc;
  const int64_t rows = std::min(outer, b->history_cap);
  std::vector<double> hist(5 * (size_t)std::max<int64_t>(rows, 1));
  if (rows > 0 && (rc = d2h(b, hist.data(), b->D.history + (size_t)k * b->history_cap * 5,
                            sizeof(double) * 5 * rows)))
    return rc;
  rc = cfdb_write_results(&b->cases[k], u.data(), v.data(), w.data(), p.data(), hist.data(), rows,
                          res[BR_GLOB], dir, fields_written);
  if (rc != CFDB_OK) return set_error(b->ctx, rc, "cannot write the result files");
  return CFDB_OK;
}

cfdb_status cfdb_batch_autotune(cfdb_batch* b, cfdb_batch_tuning* chosen) {
  if (!b) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  cfdb_status rc;
  bool changed = false;
  if ((rc = refresh_active(b, &changed))) return rc;
  if (changed && (rc = plan_all_teams(b))) return rc;
  cfdb_batch_tuning best = b->tune;
  int candidates = 0;
  auto time_it = [&](auto&& body, int reps, float* out_ms) -> cfdb_status {
    body();  // warm-up
    float bestms = 1e30f;
    for (int r = 0; r < reps; ++r) {
      CFDB_CUDA(ctx, cudaEventRecord(b->e0, s));
      body();
      CFDB_CUDA(ctx, cudaEventRecord(b->e1, s));
      CFDB_CUDA(ctx, cudaEventSynchronize(b->e1));
      float ms = 0.f;
      CFDB_CUDA(ctx, cudaEventElapsedTime(&ms, b->e0, b->e1));
      bestms = std::min(bestms, ms);
    }
    CFDB_CHECK_LAUNCH(ctx);
    *out_ms = bestms;
    return CFDB_OK;
  };
  // 1. stage shapes: cell stages timed on the momentum assembly, face stages
  //    on the predictor flux (both write scratch fields only)
  const int threads_c[3] = {128, 256, 512};
  const int per_thread[4] = {1, 2, 4, 8};
  float best_cell = 1e30f, best_face = 1e30f;
  for (int ti : threads_c)
    for (int pt : per_thread) {
      b->tune.cell_threads = b->tune.face_threads = ti;
      b->tune.cell_tile = b->tune.face_tile = ti * pt;
      if ((rc = upload_tiles(b))) return rc;
      float mc = 0.f, mf = 0.f;
      if ((rc = time_it([&] { launch_stage(b, BS_ASSEMBLE, 0, s); }, 3, &mc))) return rc;
      if ((rc = time_it([&] { launch_stage(b, BS_MASS_FLUX, 0, s); }, 3, &mf))) return rc;
      candidates += 2;
      if (mc < best_cell) {
        best_cell = mc;
        best.cell_threads = ti;
        best.cell_tile = ti * pt;
      }
      if (mf < best_face) {
        best_face = mf;
        best.face_threads = ti;
        best.face_tile = ti * pt;
      }
    }
  b->tune.cell_threads = best.cell_threads;
  b->tune.cell_tile = best.cell_tile;
  b->tune.face_threads = best.face_threads;
  b->tune.face_tile = best.face_tile;
  if ((rc = upload_tiles(b))) return rc;
  // 2. p' team sizing, timed on the p' systems of the current state: the
  //    stages before the p' solve write scratch fields only, and the linear
  //    solves run with the case records left alone
  enqueue_prefix(b, 0, s);
  CFDB_CHECK_LAUNCH(ctx);
  CFDB_CUDA(ctx, cudaStreamSynchronize(s));
  if ((rc = check_error(b))) return rc;
  float best_p = 1e30f;
  std::vector<double> wbest = b->h_pweight;
  const double exps[3] = {1.0, 1.25, 1.5};
  auto time_pprime = [&](float* ms) {
    return time_it([&] {
      launch_stage(b, BS_PROWS, 0, s);
      launch_krylov(b, 1, 0, 0, s);
    }, 2, ms);
  };
  for (double e : exps) {
    std::vector<double> w = power_weights(b, e);
    if ((rc = upload_teams(b, 1, w))) return rc;
    float ms = 0.f;
    if ((rc = time_pprime(&ms))) return rc;
    if ((rc = check_error(b))) return rc;
    ++candidates;
    if (ms < best_p) {
      best_p = ms;
      best.team_exponent = e;
      best.adaptive_teams = 0;
      wbest = w;
    }
  }
  // the adaptive rule: weights from the iteration counts just measured
  if ((rc = d2h(b, b->h_kout, b->d_kout, sizeof(double) * 2 * b->n * kKoutStride))) return rc;
  std::vector<double> wa(b->n);
  for (int k = 0; k < b->n; ++k)
    wa[k] = (double)b->cells[k] *
            std::max(1.0, b->h_kout[((size_t)b->n + k) * kKoutStride + krylov::O_ITER]);
  if ((rc = upload_teams(b, 1, wa))) return rc;
  float ma = 0.f;
  if ((rc = time_pprime(&ma))) return rc;
  if ((rc = check_error(b))) return rc;
  ++candidates;
  if (ma < best_p) {
    best_p = ma;
    best.adaptive_teams = 1;
    wbest = wa;
  }
  best.cell_stage_ms = best_cell;
  best.face_stage_ms = best_face;
  best.pprime_solve_ms = best_p;
  best.candidates = candidates;
  b->tune = best;
  b->h_pweight = wbest;
  if ((rc = plan_all_teams(b))) return rc;
  b->dirty = true;
  if (chosen) *chosen = best;
  return CFDB_OK;
}

}  // extern "C"
