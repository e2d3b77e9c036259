// Solves of the reference's own LinearSystem (host CSR) on the device.
//
// The reference's linear-solver contract (LinearSolver::solve,
// include/cfd/algebra/LinearSolver.hpp:176-180) hands a solver a CSR matrix
// (SparseMatrix.hpp:19-56) built by SparseMatrixBuilder from the triplets of
// an assembly.  On the reference's Cartesian meshes every such system -- the
// relaxed momentum rows (RelaxedMomentum.cpp:30-104), the p' rows
// (PressureCorrectionEquation.cpp:181-339) -- is a 5-point (2D) or 7-point
// (3D) stencil in cell order i + nx*(j + ny*k).  This file recognises that
// shape on the host (the grid comes from the neighbour strides that occur),
// moves the bands to the device and runs one of the library's solvers:
//   * the face-coefficient p' operator (persistent Jacobi-PCG, or the learned
//     preconditioner in flexible CG) when the matrix is exactly that
//     operator: symmetric couplings apart from one pinned identity row, no
//     boundary coefficients, and a stored diagonal equal bit for bit to the
//     face-order sum of its couplings (so the matrix-free operator, which
//     re-sums the diagonal, is the same matrix);
//   * the stencil Krylov solver (CG or BiCGSTAB, optional Jacobi) on the
//     stored bands otherwise.
// A matrix of any other shape is refused (CFDB_ERR_UNSUPPORTED): no CSR
// kernel and no CPU solver stands behind these entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cfdb.h"
#include "cfdb_internal.cuh"
#include "stencil_solve.cuh"

struct cfdb_csr_solver {
  cfdb_context* ctx = nullptr;
  int64_t n = 0;  // cells the stencil-path buffers hold
  double* b = nullptr;
  double* x = nullptr;
  double* diag = nullptr;
  double* off[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double* hist = nullptr;
  int64_t hist_cap = 0;
  cfdb::StencilWork work;
  cfdb_poperator* op = nullptr;  // faces path, kept while the shape stays
  int op_dim = 0;
  int64_t op_n[3] = {0, 0, 0};
  int op_pinned = 0;
  int64_t op_ref = -1;

  void release_vectors() {
    cudaFree(b);
    cudaFree(x);
    cudaFree(diag);
    for (double*& q : off) {
      cudaFree(q);
      q = nullptr;
    }
    b = x = diag = nullptr;
    n = 0;
  }
  ~cfdb_csr_solver() {
    release_vectors();
    cudaFree(hist);
    if (op) cfdb_poperator_destroy(op);
  }
};

namespace cfdb {
namespace {

// Jacobi's rejection threshold, constants::small of the reference
// (include/cfd/core/Constants.hpp), used by computeInverseDiagonal
// (src/algebra/Preconditioner.cpp:11-32).
constexpr double kSmallDiagonal = 1.0e-12;

struct Csr {
  int64_t rows;
  const uint64_t* ro;
  const uint64_t* ci;
  const double* v;
};

struct Structure {
  int dim = 0;
  int64_t n[3] = {1, 1, 1};
  int64_t sy = 0, sz = 0;
  std::vector<double> diag;    // stored diagonal, 0 where the row stores none
  std::vector<double> off[6];  // 2a: low neighbour along axis a, 2a+1: high
  std::vector<char> has_diag;
  int pinned = 0;
  int64_t ref = -1;
  bool faces_ok = false;
  std::vector<double> faces;  // global face order (x-, y-, z-faces), when faces_ok
};

// Grid and bands of a CSR matrix, or false with the reason.
bool recognise(const Csr& A, Structure& S, std::string* why) {
  if (A.rows < 4) {
    *why = "fewer than four rows";
    return false;
  }
  if (A.ro[0] != 0) {
    *why = "row offsets do not start at 0";
    return false;
  }
  uint64_t strides[3] = {0, 0, 0};
  int ns = 0;
  for (int64_t r = 0; r < A.rows; ++r) {
    if (A.ro[r + 1] < A.ro[r]) {
      *why = "row offsets decrease";
      return false;
    }
    for (uint64_t q = A.ro[r]; q < A.ro[r + 1]; ++q) {
      const uint64_t c = A.ci[q];
      if (c >= (uint64_t)A.rows) {
        *why = "column index out of range";
        return false;
      }
      if (c == (uint64_t)r) continue;
      const uint64_t d = c > (uint64_t)r ? c - (uint64_t)r : (uint64_t)r - c;
      bool seen = false;
      for (int t = 0; t < ns; ++t) seen = seen || strides[t] == d;
      if (seen) continue;
      if (ns == 3) {
        *why = "more than three distinct neighbour strides: not a 5-/7-point Cartesian operator";
        return false;
      }
      strides[ns++] = d;
    }
  }
  std::sort(strides, strides + ns);
  if (ns < 1 || strides[0] != 1) {
    *why = "the strides 1 and nx (and nx*ny) do not all occur: not a 5-/7-point Cartesian operator";
    return false;
  }
  const int64_t nx = ns == 1 ? A.rows : (int64_t)strides[1];
  if (ns == 1) {
    // a 3-point band: one row of cells (stencil path only)
    S.dim = 2;
    S.n[0] = A.rows;
    S.n[1] = 1;
    S.n[2] = 1;
  } else if (ns == 2) {
    if (A.rows % nx != 0) {
      *why = "row count is not a multiple of the x extent";
      return false;
    }
    S.dim = 2;
    S.n[0] = nx;
    S.n[1] = A.rows / nx;
    S.n[2] = 1;
  } else {
    const int64_t sxy = (int64_t)strides[2];
    if (sxy % nx != 0 || A.rows % sxy != 0) {
      *why = "strides and row count do not form an nx x ny x nz grid";
      return false;
    }
    S.dim = 3;
    S.n[0] = nx;
    S.n[1] = sxy / nx;
    S.n[2] = A.rows / sxy;
  }
  if (S.n[0] < 2 || (ns > 1 && S.n[1] < 2) || (S.dim == 3 && S.n[2] < 2) || S.n[0] > INT32_MAX ||
      S.n[1] > INT32_MAX || S.n[2] > INT32_MAX) {
    *why = "grid extents out of range";
    return false;
  }
  S.sy = S.n[0];
  S.sz = S.n[0] * S.n[1];
  S.diag.assign(A.rows, 0.0);
  S.has_diag.assign(A.rows, 0);
  for (int q = 0; q < 6; ++q) S.off[q].assign(A.rows, 0.0);
  std::vector<unsigned char> filled(A.rows, 0);  // bit q: off[q] set
  const int64_t st[3] = {1, S.sy, S.sz};
  for (int64_t r = 0; r < A.rows; ++r) {
    const int64_t ijk[3] = {r % S.n[0], (r / S.n[0]) % S.n[1], r / S.sz};
    for (uint64_t q = A.ro[r]; q < A.ro[r + 1]; ++q) {
      const int64_t d = (int64_t)A.ci[q] - r;
      if (d == 0) {
        if (S.has_diag[r]) {
          *why = "a row stores its diagonal twice";
          return false;
        }
        S.has_diag[r] = 1;
        S.diag[r] = A.v[q];
        continue;
      }
      int slot = -1;
      for (int a = 0; a < S.dim && slot < 0; ++a) {
        if (d == -st[a] && ijk[a] > 0) slot = 2 * a;
        else if (d == st[a] && ijk[a] < S.n[a] - 1) slot = 2 * a + 1;
      }
      if (slot < 0) {
        *why = "row " + std::to_string(r) + " couples to column " + std::to_string(A.ci[q]) +
               ", which is not a grid neighbour";
        return false;
      }
      if (filled[r] & (1u << slot)) {
        *why = "a row stores one neighbour twice";
        return false;
      }
      filled[r] |= (unsigned char)(1u << slot);
      S.off[slot][r] = A.v[q];
    }
  }
  return true;
}

// Whether the matrix is exactly the face-coefficient p' operator, and its
// face coefficients (global face order) if so.
void face_form(const Csr& A, Structure& S) {
  S.faces_ok = false;
  S.pinned = 0;
  S.ref = -1;
  if (S.n[1] < 2) return;  // the face operator needs two cells per axis
  // identity rows: a stored diagonal of exactly 1 and no stored coupling
  int64_t identity_rows = 0;
  for (int64_t r = 0; r < A.rows; ++r) {
    if (!S.has_diag[r] || S.diag[r] != 1.0) continue;
    bool lone = true;
    for (int q = 0; q < 6; ++q) lone = lone && S.off[q][r] == 0.0;
    if (lone && A.ro[r + 1] - A.ro[r] == 1) {
      ++identity_rows;
      S.ref = r;
    }
  }
  if (identity_rows > 1) return;
  S.pinned = identity_rows == 1 ? 1 : 0;
  if (!S.pinned) S.ref = -1;
  const int64_t nx = S.n[0], ny = S.n[1], nz = S.n[2];
  const int64_t nfx = (nx + 1) * ny * nz, nfy = nx * (ny + 1) * nz;
  const int64_t nfz = S.dim == 3 ? nx * ny * (nz + 1) : 0;
  S.faces.assign(nfx + nfy + nfz, 0.0);
  const int64_t st[3] = {1, S.sy, S.sz};
  auto face_index = [&](int a, int64_t i, int64_t j, int64_t k) -> int64_t {
    if (a == 0) return i + (nx + 1) * (j + ny * k);
    if (a == 1) return nfx + i + nx * (j + (ny + 1) * k);
    return nfx + nfy + i + nx * (j + ny * k);
  };
  // couplings: the face between lo and hi = lo + stride carries D with
  // A(lo,hi) = A(hi,lo) = -D, except that the pinned row stores none
  for (int64_t lo = 0; lo < A.rows; ++lo) {
    const int64_t ijk[3] = {lo % nx, (lo / nx) % ny, lo / S.sz};
    for (int a = 0; a < S.dim; ++a) {
      if (ijk[a] == S.n[a] - 1) continue;
      const int64_t hi = lo + st[a];
      const double up = S.off[2 * a + 1][lo], down = S.off[2 * a][hi];
      double D;
      if (S.pinned && lo == S.ref) D = -down;
      else if (S.pinned && hi == S.ref) D = -up;
      else if (up == down) D = -up;
      else return;  // not symmetric
      S.faces[face_index(a, ijk[0] + (a == 0), ijk[1] + (a == 1), ijk[2] + (a == 2))] = D;
    }
  }
  // the diagonal the matrix-free operator forms: the face-order sum x-low,
  // x-high, y-low, y-high, z-low, z-high, boundary faces contributing 0
  for (int64_t r = 0; r < A.rows; ++r) {
    if (S.pinned && r == S.ref) continue;
    const int64_t i = r % nx, j = (r / nx) % ny, k = r / S.sz;
    double d = S.faces[face_index(0, i, j, k)] + S.faces[face_index(0, i + 1, j, k)];
    d = d + S.faces[face_index(1, i, j, k)];
    d = d + S.faces[face_index(1, i, j + 1, k)];
    if (S.dim == 3) {
      d = d + S.faces[face_index(2, i, j, k)];
      d = d + S.faces[face_index(2, i, j, k + 1)];
    }
    if (!S.has_diag[r] || d != S.diag[r]) return;
  }
  S.faces_ok = true;
}

cfdb_status ensure(cfdb_context* ctx, double** p, int64_t n) {
  if (*p) return CFDB_OK;
  CFDB_CUDA(ctx, cudaMalloc((void**)p, sizeof(double) * (size_t)std::max<int64_t>(n, 1)));
  return CFDB_OK;
}

void fill_info(const Structure& S, int path, int learned_declined, cfdb_csr_info* info) {
  if (!info) return;
  info->dim = S.dim;
  for (int a = 0; a < 3; ++a) info->n[a] = S.n[a];
  info->path = path;
  info->faces_eligible = S.faces_ok ? 1 : 0;
  info->pinned = S.pinned;
  info->reference_cell = S.ref;
  info->learned_declined = learned_declined;
}

}  // namespace
}  // namespace cfdb

using namespace cfdb;

extern "C" {

cfdb_status cfdb_csr_analyze(int64_t rows, const uint64_t* row_offsets, const uint64_t* columns,
                             const double* values, cfdb_csr_info* info) {
  if (rows <= 0 || !row_offsets || !columns || !values || !info) return CFDB_ERR_INVALID_ARGUMENT;
  std::memset(info, 0, sizeof(*info));
  const Csr A{rows, row_offsets, columns, values};
  Structure S;
  std::string why;
  if (!recognise(A, S, &why)) return CFDB_ERR_UNSUPPORTED;
  face_form(A, S);
  fill_info(S, S.faces_ok ? CFDB_CSR_PATH_FACES : CFDB_CSR_PATH_STENCIL, 0, info);
  return CFDB_OK;
}

cfdb_status cfdb_csr_solver_create(cfdb_context* ctx, cfdb_csr_solver** out) {
  if (!ctx || !out) return CFDB_ERR_INVALID_ARGUMENT;
  auto* s = new cfdb_csr_solver();
  s->ctx = ctx;
  *out = s;
  return CFDB_OK;
}

void cfdb_csr_solver_destroy(cfdb_csr_solver* s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  delete s;
}

cfdb_status cfdb_csr_solve_host(cfdb_csr_solver* s, const cfdb_linear_settings* settings,
                                int64_t rows, const uint64_t* row_offsets, const uint64_t* columns,
                                const double* values, const double* b_host, double* x_host,
                                double* history, int64_t history_cap, cfdb_linear_result* result,
                                cfdb_csr_info* info) {
  if (!s || !settings || rows <= 0 || !row_offsets || !columns || !values || !b_host || !x_host ||
      !result)
    return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = s->ctx;
  std::memset(result, 0, sizeof(*result));
  if (info) std::memset(info, 0, sizeof(*info));
  if (settings->max_iterations < 1)
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "max_iterations must be >= 1");
  if (settings->krylov != CFDB_KRYLOV_CG && settings->krylov != CFDB_KRYLOV_BICGSTAB)
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "unknown Krylov method");
  const Csr A{rows, row_offsets, columns, values};
  // NonFiniteInput first, as CG.cpp:23-26 / BiCGSTAB.cpp:57-60
  const uint64_t nnz = row_offsets[rows];
  bool finite = true;
  for (uint64_t q = 0; q < nnz && finite; ++q) finite = std::isfinite(values[q]);
  for (int64_t r = 0; r < rows && finite; ++r)
    finite = std::isfinite(b_host[r]) && std::isfinite(x_host[r]);
  if (!finite) {
    result->status = CFDB_SOLVER_NONFINITE_INPUT;
    return CFDB_OK;
  }
  Structure S;
  std::string why;
  if (!recognise(A, S, &why))
    return set_error(ctx, CFDB_ERR_UNSUPPORTED, "CSR system not supported: " + why);
  const int pre = settings->preconditioner;
  const bool jacobi = pre == CFDB_PRECOND_JACOBI || pre == CFDB_PRECOND_LEARNED_MG;
  // InvalidSystem: the Jacobi build's rejections (Preconditioner.cpp:11-32)
  if (jacobi) {
    for (int64_t r = 0; r < rows; ++r) {
      const double d = S.diag[r];
      if (!S.has_diag[r] || d == 0.0 || std::fabs(d) < kSmallDiagonal) {
        fill_info(S, CFDB_CSR_PATH_STENCIL, 0, info);
        result->status = CFDB_SOLVER_INVALID_SYSTEM;
        return CFDB_OK;
      }
    }
  }
  if (settings->krylov == CFDB_KRYLOV_CG && jacobi) face_form(A, S);
  const bool faces = S.faces_ok;
  const int declined = (pre == CFDB_PRECOND_LEARNED_MG && !faces) ? 1 : 0;
  fill_info(S, faces ? CFDB_CSR_PATH_FACES : CFDB_CSR_PATH_STENCIL, declined, info);
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t bytes = sizeof(double) * (size_t)rows;
  if (s->n != rows) {
    s->release_vectors();
    s->n = rows;
  }
  cfdb_status st = ensure(ctx, &s->b, rows);
  if (st == CFDB_OK) st = ensure(ctx, &s->x, rows);
  if (st != CFDB_OK) return st;
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->b, b_host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->x, x_host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  if (faces) {
    cfdb_grid g{};
    g.dim = S.dim;
    for (int a = 0; a < 3; ++a) {
      g.n[a] = S.n[a];
      g.len[a] = 1.0;  // unused: the operator takes its coefficients from the faces
    }
    const bool same = s->op && s->op_dim == S.dim && s->op_n[0] == S.n[0] &&
                      s->op_n[1] == S.n[1] && s->op_n[2] == S.n[2] &&
                      s->op_pinned == S.pinned && s->op_ref == S.ref;
    if (same) {
      st = cfdb_poperator_update_faces(ctx, s->op, S.faces.data());
    } else {
      if (s->op) cfdb_poperator_destroy(s->op);
      s->op = nullptr;
      st = cfdb_poperator_create_faces(ctx, &g, S.faces.data(), S.pinned, S.pinned ? S.ref : 0,
                                       &s->op);
      if (st == CFDB_OK) {
        s->op_dim = S.dim;
        for (int a = 0; a < 3; ++a) s->op_n[a] = S.n[a];
        s->op_pinned = S.pinned;
        s->op_ref = S.ref;
      }
    }
    if (st != CFDB_OK) return st;
    st = cfdb_poperator_solve_device(ctx, s->op, settings, s->b, s->x, history, history_cap,
                                     result);
    if (st != CFDB_OK) return st;
  } else {
    for (int q = 0; q < 6 && st == CFDB_OK; ++q) st = ensure(ctx, &s->off[q], rows);
    if (st == CFDB_OK) st = ensure(ctx, &s->diag, rows);
    if (st != CFDB_OK) return st;
    CFDB_CUDA(ctx, cudaMemcpyAsync(s->diag, S.diag.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
    for (int q = 0; q < 6; ++q)
      CFDB_CUDA(ctx, cudaMemcpyAsync(s->off[q], S.off[q].data(), bytes, cudaMemcpyHostToDevice,
                                     ctx->stream));
    const int64_t cap = history ? std::max<int64_t>(history_cap, 0) : 0;
    if (cap > s->hist_cap) {
      cudaFree(s->hist);
      s->hist = nullptr;
      s->hist_cap = 0;
      CFDB_CUDA(ctx, cudaMalloc((void**)&s->hist, sizeof(double) * (size_t)cap));
      s->hist_cap = cap;
    }
    StencilMatrix M{};
    M.dim = S.dim;
    M.nx = (int)S.n[0];
    M.ny = (int)S.n[1];
    M.nz = (int)S.n[2];
    M.n = rows;
    M.sy = S.sy;
    M.sz = S.sz;
    M.diag = s->diag;
    for (int q = 0; q < 6; ++q) M.off[q] = s->off[q];
    M.inv = nullptr;
    st = stencil_solve(ctx, M, s->work, s->b, s->x, settings->krylov == CFDB_KRYLOV_CG ? 0 : 1,
                       jacobi ? 1 : 0, settings->abs_tol, settings->rel_tol,
                       settings->max_iterations, cap > 0 ? s->hist : nullptr, cap, result);
    if (st != CFDB_OK) return st;
    result->device_ms = result->krylov_ms;
    if (cap > 0) {
      const int64_t m = std::min<int64_t>(cap, result->iterations + 1);
      if (result->status == CFDB_SOLVER_CONVERGED || result->status == CFDB_SOLVER_MAX_ITERATIONS ||
          result->status == CFDB_SOLVER_BREAKDOWN || result->status == CFDB_SOLVER_NONFINITE_RESIDUAL)
        CFDB_CUDA(ctx, cudaMemcpyAsync(history, s->hist, sizeof(double) * (size_t)m,
                                       cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  if (result->status != CFDB_SOLVER_NONFINITE_INPUT && result->status != CFDB_SOLVER_INVALID_SYSTEM)
    CFDB_CUDA(ctx, cudaMemcpyAsync(x_host, s->x, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

}  // extern "C"
