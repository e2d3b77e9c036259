// Allocation-free p' solve.
//
// Some callers cannot allocate device memory at the point where they need a
// solve: hosts whose device memory is owned by another runtime (an embedding
// application or FFI host that hands us pre-registered buffers and reserves
// the rest of the device for its own pool), or real-time loops that forbid
// cudaMalloc/cudaFree after start-up (both synchronise the device and can
// stall).  For them, cfdb_pcg_solve_noalloc runs the FP64 Jacobi-PCG of the
// uniform p' operator using only the caller's b and x plus the fixed scratch
// array below; it creates no context, stream, event or allocation.  It does
// wait for its own result (a stream synchronisation), so it cannot be
// recorded into a CUDA graph: on a capturing stream it returns
// CFDB_ERR_UNSUPPORTED before it issues any work, and the capture stays
// valid.
//
// The scratch is one file-scope device array of kScratchBytes (about 1.6 MB)
// that every GPU which loads this library holds until the process exits.  It
// bounds the problem to kMaxCells cells.  All calls on a device share it and
// it keeps the last call's contents, so every call clears what must start at
// zero; two calls whose work overlaps on the GPU (different streams, or a
// second call before the first finished) race on it and give wrong results.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "cfdb.h"
#include "grid_sync.cuh"

namespace cfdb {
namespace {

constexpr int64_t kMaxCells = 65536;
constexpr int kMaxBlocks = 1024;
constexpr int kNaThreads = 256;
constexpr unsigned long long kNaTimeoutNs = 2000000000ull;

// Byte layout of the scratch array.
constexpr size_t kOffVec = 0;                                      // r, p0, p1: 3 * kMaxCells doubles
constexpr size_t kOffPart = kOffVec + 3 * kMaxCells * sizeof(double);  // 4 * kMaxBlocks doubles
constexpr size_t kOffOut = kOffPart + 4 * kMaxBlocks * sizeof(double);  // 8 doubles
constexpr size_t kOffSync = kOffOut + 8 * sizeof(double);               // 4 unsigned
constexpr size_t kScratchBytes = kOffSync + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct NaGrid {
  int nx, ny, nz;  // kernel space: 2D maps (nx, ny) to (nx, 1, ny)
  double dx[3], area[3];  // per kernel axis: spacing and face area
  double rho;
  int pinned;
  int64_t ref;
};

// Face coefficient of the face at coordinate f along kernel axis a, computed
// with the reference's expressions: ((rho |S|) d_face) / |x_N - x_P| with the
// unit response interpolated (exactly 1), Neumann (0) on the boundary.
__device__ __forceinline__ double face_d(const NaGrid& G, int a, int f, int n) {
  if (f <= 0 || f >= n) return 0.0;
  const double cp = ((double)(f - 1) + 0.5) * G.dx[a], cn = ((double)f + 0.5) * G.dx[a];
  const double node = (double)f * G.dx[a];
  const double dPf = fabs(node - cp), dNf = fabs(node - cn);
  const double dFace = ((dNf * 1.0) + (dPf * 1.0)) / (dPf + dNf);
  return G.rho * G.area[a] * dFace / fabs(cn - cp);
}

struct NaParams {
  NaGrid G;
  const double* b;
  double* x;
  double abs_tol, rel_tol;
  int64_t max_it;
  GridSync sync;
  unsigned char* scratch;  // device address of g_noalloc_scratch
};

__device__ __forceinline__ void cell_coef(const NaGrid& G, int64_t c, double cf[6], double& diag,
                                          int& i, int& j, int& k) {
  i = (int)(c % G.nx);
  j = (int)((c / G.nx) % G.ny);
  k = (int)(c / ((int64_t)G.nx * G.ny));
  const double xl = face_d(G, 0, i, G.nx), xh = face_d(G, 0, i + 1, G.nx);
  const double yl = face_d(G, 1, j, G.ny), yh = face_d(G, 1, j + 1, G.ny);
  const double zl = face_d(G, 2, k, G.nz), zh = face_d(G, 2, k + 1, G.nz);
  diag = ((((xl + xh) + yl) + yh) + zl) + zh;
  cf[0] = xl;
  cf[1] = xh;
  cf[2] = yl;
  cf[3] = yh;
  cf[4] = zl;
  cf[5] = zh;
  if (G.pinned && c == G.ref) {
    diag = 1.0;
    for (int q = 0; q < 6; ++q) cf[q] = 0.0;
  }
}

__device__ __forceinline__ double apply(const NaGrid& G, const double* v, int64_t c) {
  double cf[6], diag;
  int i, j, k;
  cell_coef(G, c, cf, diag, i, j, k);
  const int64_t sy = G.nx, sz = (int64_t)G.nx * G.ny;
  double off = 0.0;
  if (i > 0) off += cf[0] * __ldcg(v + c - 1);
  if (i < G.nx - 1) off += cf[1] * __ldcg(v + c + 1);
  if (j > 0) off += cf[2] * __ldcg(v + c - sy);
  if (j < G.ny - 1) off += cf[3] * __ldcg(v + c + sy);
  if (k > 0) off += cf[4] * __ldcg(v + c - sz);
  if (k < G.nz - 1) off += cf[5] * __ldcg(v + c + sz);
  return diag * __ldcg(v + c) - off;
}

__device__ __forceinline__ double inv_diag(const NaGrid& G, int64_t c) {
  double cf[6], diag;
  int i, j, k;
  cell_coef(G, c, cf, diag, i, j, k);
  return 1.0 / diag;
}

// The persistent Jacobi-PCG (same algorithm, statuses and convergence test as
// the library's main p' solve), every vector and reduction slot in scratch.
__global__ void __launch_bounds__(kNaThreads) na_pcg(NaParams P) {
  __shared__ double red[64];
  const NaGrid& G = P.G;
  double* r = reinterpret_cast<double*>(P.scratch + kOffVec);
  double* p = r + kMaxCells;
  double* ap = p + kMaxCells;
  double* partials = reinterpret_cast<double*>(P.scratch + kOffPart);
  double* out = reinterpret_cast<double*>(P.scratch + kOffOut);
  const int B = gridDim.x, blk = blockIdx.x, tid = threadIdx.x;
  const int64_t n = (int64_t)G.nx * G.ny * G.nz;
  const int64_t c0 = n * blk / B, c1 = n * (blk + 1) / B;
  const bool leader = blk == 0 && tid == 0;
  int round = 0;
  auto reduce2 = [&](double a0, double a1, double (&o)[2]) -> bool {
    double a[2] = {a0, a1};
    block_sum<2>(a, red);
    double* part = partials + (size_t)(round & 1) * 2 * B;
    if (tid == 0) {
      part[2 * blk] = a[0];
      part[2 * blk + 1] = a[1];
    }
    if (!grid_sync(P.sync)) return false;
    grid_total<2>(part, 2, B, o, red);
    ++round;
    return true;
  };
  auto finish = [&](int status, int64_t it, double fin) {
    if (leader) {
      out[0] = status;
      out[1] = (double)it;
      out[3] = fin;
    }
  };
  double s0 = 0.0, s1 = 0.0;
  for (int64_t c = c0 + tid; c < c1; c += kNaThreads) {
    const double rn = __ldg(P.b + c) - apply(G, P.x, c);
    r[c] = rn;
    s0 += rn * rn;
    s1 += rn * (inv_diag(G, c) * rn);
  }
  double tot[2];
  if (!reduce2(s0, s1, tot)) return;
  const double b0 = sqrt(tot[0]);
  if (leader) out[2] = b0;
  auto conv = [&](double res) { return res <= P.abs_tol || (b0 > 0.0 && res / b0 <= P.rel_tol); };
  if (b0 == 0.0 || conv(b0)) return finish(CFDB_SOLVER_CONVERGED, 0, b0);
  double rz = tot[1];
  if (!isfinite(rz)) return finish(CFDB_SOLVER_BREAKDOWN, 0, b0);
  double res_cur = b0, beta = 0.0;
  for (int64_t it = 1; it <= P.max_it; ++it) {
    for (int64_t c = c0 + tid; c < c1; c += kNaThreads) {
      const double z = inv_diag(G, c) * r[c];
      p[c] = (it == 1) ? z : z + beta * p[c];
    }
    if (!grid_sync(P.sync)) return;
    double pap = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kNaThreads) {
      const double a = apply(G, p, c);
      ap[c] = a;
      pap += p[c] * a;
    }
    if (!reduce2(pap, 0.0, tot)) return;
    const double alpha = rz / tot[0];
    if (!isfinite(tot[0]) || fabs(tot[0]) < 1.0e-30 || !isfinite(alpha))
      return finish(CFDB_SOLVER_BREAKDOWN, it - 1, res_cur);
    double rr = 0.0, rzn = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kNaThreads) {
      P.x[c] = P.x[c] + alpha * p[c];
      const double rn = r[c] - alpha * ap[c];
      r[c] = rn;
      rr += rn * rn;
      rzn += rn * (inv_diag(G, c) * rn);
    }
    if (!reduce2(rr, rzn, tot)) return;
    const double res = sqrt(tot[0]);
    if (!isfinite(res)) return finish(CFDB_SOLVER_NONFINITE_RESIDUAL, it, res);
    res_cur = res;
    if (conv(res)) return finish(CFDB_SOLVER_CONVERGED, it, res);
    beta = tot[1] / rz;
    if (!isfinite(tot[1]) || !isfinite(beta)) return finish(CFDB_SOLVER_BREAKDOWN, it, res);
    rz = tot[1];
  }
  finish(CFDB_SOLVER_MAX_ITERATIONS, P.max_it, res_cur);
}

// Device address of the scratch array.  In host code g_noalloc_scratch names
// a host-side stand-in, not device memory, so the kernel gets the address
// cudaGetSymbolAddress returns, looked up once per device and CUDA context
// with that device current.  The cache is keyed on the context as well as the
// device: after cudaDeviceReset the primary context (and the library's module
// with its array) is created anew, and an address of the old one would
// dangle.  cuCtxGetCurrent is reached through the runtime's driver entry
// point, so the library does not link the driver library itself.
using CtxGetCurrentFn = int (*)(void**);

std::mutex g_lookup_mutex;
struct ScratchSlot {
  void* context = nullptr;
  void* addr = nullptr;
};
ScratchSlot g_scratch_slot[128];
CtxGetCurrentFn g_ctx_get_current = nullptr;
bool g_ctx_lookup_done = false;

cudaError_t scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_lookup_mutex);
  if (device < 0 || device >= 128) return cudaErrorInvalidDevice;
  if (!g_ctx_lookup_done) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    g_ctx_lookup_done = true;
  }
  void* context = nullptr;
  if (!g_ctx_get_current || g_ctx_get_current(&context) != 0 || !context)
    return cudaErrorDeviceUninitialized;
  ScratchSlot& slot = g_scratch_slot[device];
  if (!slot.addr || slot.context != context) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    slot.addr = p;
    slot.context = context;
  }
  *out = static_cast<unsigned char*>(slot.addr);
  return cudaSuccess;
}

}  // namespace
}  // namespace cfdb

using namespace cfdb;

extern "C" cfdb_status cfdb_pcg_solve_noalloc(void* stream, const cfdb_grid* grid, double rho,
                                              int pinned, int64_t reference_cell,
                                              const cfdb_linear_settings* s, const double* b_dev,
                                              double* x_dev, cfdb_linear_result* result) {
  if (!grid || !s || !b_dev || !x_dev || !result) return CFDB_ERR_INVALID_ARGUMENT;
  std::memset(result, 0, sizeof(*result));
  if (grid->dim != 2 && grid->dim != 3) return CFDB_ERR_INVALID_ARGUMENT;
  int64_t cells = 1;
  for (int a = 0; a < grid->dim; ++a) {
    if (grid->n[a] < 2 || !(grid->len[a] > 0.0)) return CFDB_ERR_INVALID_ARGUMENT;
    cells *= grid->n[a];
  }
  if (cells > kMaxCells) return CFDB_ERR_UNSUPPORTED;  // beyond the fixed scratch
  if (s->krylov != CFDB_KRYLOV_CG || s->preconditioner != CFDB_PRECOND_JACOBI ||
      s->precision != CFDB_PRECISION_FP64 || s->max_iterations < 1 || !(rho > 0.0))
    return CFDB_ERR_UNSUPPORTED;
  if (pinned && (reference_cell < 0 || reference_cell >= cells)) return CFDB_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  // the call waits for its own result, which a capturing stream forbids:
  // refuse before any other CUDA call so that the caller's capture survives
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &capture) != cudaSuccess ||
      capture != cudaStreamCaptureStatusNone)
    return CFDB_ERR_UNSUPPORTED;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return CFDB_ERR_NO_DEVICE;
  unsigned char* scratch = nullptr;
  if (scratch_address(device, &scratch) != cudaSuccess) return CFDB_ERR_CUDA;

  NaParams P{};
  NaGrid& G = P.G;
  const int dim = grid->dim;
  double delta[3] = {0, 0, 0}, area[3] = {0, 0, 0};
  for (int a = 0; a < dim; ++a) delta[a] = grid->len[a] / (double)grid->n[a];
  if (dim == 2) {
    area[0] = delta[1];
    area[1] = delta[0];
    G.nx = (int)grid->n[0];
    G.ny = 1;
    G.nz = (int)grid->n[1];
    G.dx[0] = delta[0];
    G.area[0] = area[0];
    G.dx[1] = 1.0;
    G.area[1] = 0.0;
    G.dx[2] = delta[1];
    G.area[2] = area[1];
  } else {
    area[0] = delta[1] * delta[2];
    area[1] = delta[0] * delta[2];
    area[2] = delta[0] * delta[1];
    G.nx = (int)grid->n[0];
    G.ny = (int)grid->n[1];
    G.nz = (int)grid->n[2];
    for (int a = 0; a < 3; ++a) {
      G.dx[a] = delta[a];
      G.area[a] = area[a];
    }
  }
  G.rho = rho;
  G.pinned = pinned ? 1 : 0;
  G.ref = reference_cell;
  P.b = b_dev;
  P.x = x_dev;
  P.abs_tol = s->abs_tol;
  P.rel_tol = s->rel_tol;
  P.max_it = s->max_iterations;
  P.scratch = scratch;
  int sms = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, na_pcg, kNaThreads, 0) != cudaSuccess)
    return CFDB_ERR_CUDA;
  int64_t blocks = std::min<int64_t>((int64_t)std::max(per_sm, 1) * sms, (cells + kNaThreads - 1) / kNaThreads);
  blocks = std::max<int64_t>(1, std::min<int64_t>(blocks, kMaxBlocks));
  P.sync.count = reinterpret_cast<unsigned*>(scratch + kOffSync);
  P.sync.gen = P.sync.count + 1;
  P.sync.error = P.sync.count + 2;
  P.sync.nblocks = (unsigned)blocks;
  P.sync.timeout_ns = kNaTimeoutNs;
  // the previous call's barrier words and outputs must not leak into this one
  if (cudaMemsetAsync(scratch + kOffOut, 0, kScratchBytes - kOffOut, st) != cudaSuccess)
    return CFDB_ERR_CUDA;
  void* args[] = {&P};
  if (cudaLaunchCooperativeKernel((const void*)na_pcg, dim3((unsigned)blocks), dim3(kNaThreads),
                                  args, 0, st) != cudaSuccess)
    return CFDB_ERR_CUDA;
  double out[8];
  unsigned sync_words[4];
  if (cudaMemcpyAsync(out, scratch + kOffOut, sizeof(out), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(sync_words, scratch + kOffSync, sizeof(sync_words), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return CFDB_ERR_CUDA;
  if (sync_words[2] != 0) {
    // x_dev holds a partial iterate: undefined as a solution or a start
    result->iterations = (int64_t)out[1];
    return CFDB_ERR_DEVICE_TIMEOUT;
  }
  result->status = (int)out[0];
  result->iterations = (int64_t)out[1];
  result->initial_residual = out[2];
  result->final_residual = out[3];
  result->kernel_launches = 1;
  result->krylov_launches = 1;
  return CFDB_OK;
}
