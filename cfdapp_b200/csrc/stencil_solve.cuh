// Structured stencil matrices and their persistent Krylov solves.
#pragma once

#include <cstdint>

#include "cfdb.h"

namespace cfdb {

struct StencilMatrix {
  int dim;
  int nx, ny, nz;
  int64_t n, sy, sz;         // cells, y stride (nx), z stride (nx*ny)
  const double* diag;
  const double* off[6];      // 2a: low neighbour along axis a, 2a+1: high
  const double* inv;         // Jacobi inverse diagonal (set by the solver)
};

struct StencilWork {
  int64_t n = 0;
  double *r = nullptr, *rh = nullptr, *v = nullptr, *p = nullptr, *s = nullptr, *t = nullptr,
         *inv = nullptr;
  void release();
  ~StencilWork() { release(); }
};

// krylov: 0 CG, 1 BiCGSTAB.  x holds x0 on entry.  hist_dev (device, may be
// null) receives the residual history.  Fills status, iterations, initial
// and final residual, restarts, krylov_ms.
cfdb_status stencil_solve(cfdb_context* ctx, const StencilMatrix& M, StencilWork& W,
                          const double* b, double* x, int krylov, int jacobi, double abs_tol,
                          double rel_tol, int64_t max_it, double* hist_dev, int64_t hist_cap,
                          cfdb_linear_result* res);

}  // namespace cfdb
