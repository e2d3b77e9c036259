/* CPU restatement of the reference's SIMPLE pressure-velocity path on uniform
 * Cartesian 2D/3D grids.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA product is checked
 * against; only tests, the smoke check and the bench's CPU-baseline leg may
 * load it.  Every function restates the reference's arithmetic in the same
 * operation order (file:line citations beside each), so that on the grids it
 * supports it reproduces the reference bit for bit; that pin is checked by
 * tests/test_oracle_pin.py against oracle/_ref (the reference compiled from
 * its own sources) and against the fixtures under tests/golden/.
 *
 * Layout (shared with the product):
 *   cell (i,j,k) -> i + nx*(j + ny*k)                  (MeshGeometry.cpp:419,1070)
 *   faces: all x-faces, then y-faces, then z-faces      (MeshGeometry.cpp:417-476,1090-1137)
 *     x-face (i,j,k), i in [0,nx]: i + (nx+1)*(j + ny*k)
 *     y-face (i,j,k), j in [0,ny]: i + nx*(j + (ny+1)*k)
 *     z-face (i,j,k), k in [0,nz]: i + nx*(j + ny*k)
 *   patches: 0 xmin(left) 1 xmax(right) 2 ymin(bottom) 3 ymax(top) 4 zmin 5 zmax
 *   stencil matrix rows: diag + off[6] (off[2a] = low neighbour along axis a,
 *   off[2a+1] = high neighbour), entries absent at the domain edge are 0.
 */
#ifndef CFDB_ORACLE_H
#define CFDB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OG_VBC_WALL = 0, OG_VBC_MOVING_WALL = 1, OG_VBC_INLET = 2, OG_VBC_OUTLET = 3 };
enum { OG_PBC_FIXED_GRADIENT = 0, OG_PBC_FIXED_VALUE = 1 };
enum { OG_SCHEME_UPWIND = 0, OG_SCHEME_CENTRAL = 1, OG_SCHEME_LUD = 2, OG_SCHEME_QUICK = 3 };
enum { OG_FLUX_LINEAR = 0, OG_FLUX_RHIECHOW = 1 };
enum { OG_SOLVER_CG = 0, OG_SOLVER_BICGSTAB = 1 };
/* SolverStatus (LinearSolver.hpp:16-23) */
enum {
  OG_CONVERGED = 0, OG_MAX_ITERATIONS = 1, OG_BREAKDOWN = 2, OG_NONFINITE_INPUT = 3,
  OG_NONFINITE_RESIDUAL = 4, OG_INVALID_SYSTEM = 5
};
/* SIMPLEStatus (SIMPLEResult.hpp:21-31) */
enum {
  OG_S_CONVERGED = 0, OG_S_MAX_ITERATIONS = 1, OG_S_MOMENTUM_FAILURE = 2,
  OG_S_PRESSURE_FAILURE = 3, OG_S_NONFINITE = 4, OG_S_INVALID_CONFIGURATION = 5
};

typedef struct {
  int dim;          /* 2 or 3 */
  int64_t n[3];     /* cells per axis (n[2] = 1 in 2D) */
  double len[3];    /* domain lengths */
} og_grid;

typedef struct {
  int vtype[6];
  double vvalue[6][3];
  int ptype[6];
  double pvalue[6];
} og_bcs;

typedef struct {
  int type;          /* OG_SOLVER_* */
  int jacobi;        /* 1: Jacobi preconditioner */
  double abs_tol;
  double rel_tol;
  int64_t max_iterations;
} og_linear_settings;

typedef struct {
  int status;
  int64_t iterations;
  double initial_residual;
  double final_residual;
  int64_t restarts;
} og_linear_result;

typedef struct {
  int64_t max_outer;
  double alpha_u, alpha_p;
  double tol_u, tol_p, tol_c;
  double rho, mu;
  int scheme;       /* OG_SCHEME_* */
  int face_flux;    /* OG_FLUX_* (resolved: the reference's Automatic is Linear in 2D, RhieChow in 3D) */
  int64_t reference_cell;
  og_linear_settings momentum;
  og_linear_settings pressure;
} og_simple_settings;

typedef struct {
  int status;
  int64_t iterations;
  double final_u, final_v, final_w, final_p, final_continuity, global_imbalance;
  int64_t momentum_linear_iterations;
  int64_t pressure_linear_iterations;
} og_simple_result;

int64_t og_cells(const og_grid* g);
int64_t og_faces(const og_grid* g);

/* Seeded synthetic p' right-hand side (synth_rhs.h). */
int og_synth_rhs(int64_t nx, int64_t ny, int64_t nz, uint64_t seed, double* b);

/* y = A x for a stencil matrix, summed in CSR ascending-column order
 * (SparseMatrix.cpp:93-100). */
void og_stencil_apply(const og_grid* g, const double* diag, const double* const off[6],
                      const double* x, double* y);

/* CG (CG.cpp:14-148) or BiCGSTAB (BiCGSTAB.cpp:48-275), optional Jacobi
 * (Preconditioner.cpp:11-49), on a stencil matrix.  x holds x0 on entry and the
 * solution on return; hist (may be NULL) receives residualHistory, at most
 * hist_cap entries; the count written is min(iterations+1, hist_cap). */
int og_stencil_solve(const og_grid* g, const og_linear_settings* s, const double* diag,
                     const double* const off[6], const double* b, double* x, double* hist,
                     int64_t hist_cap, og_linear_result* out);

/* p' assembly (PressureCorrectionEquation.cpp:181-339, via :341) from the
 * predictor flux and response coefficients (dw ignored in 2D).  Writes the
 * face coefficients D_f (global face order), the stencil matrix and the RHS. */
int og_assemble_pprime(const og_grid* g, const og_bcs* bc, double rho, const double* flux,
                       const double* du, const double* dv, const double* dw,
                       int64_t reference_cell, double* face_coeff, double* diag,
                       double* const off[6], double* rhs);

/* SIMPLE::solve (SIMPLE.cpp:148-1124) from the given initial state; u,v,w,p
 * (w ignored in 2D) and flux (global face order) are overwritten with the
 * result; hist (may be NULL) receives per outer iteration {u,v,w,p,continuity}. */
int og_simple(const og_grid* g, const og_bcs* bc, const og_simple_settings* s, double* u,
              double* v, double* w, double* p, double* flux, double* hist,
              og_simple_result* out);

/* The relaxed momentum system of component comp at the start of a SIMPLE
 * solve from (u, v, w, p): flux from calculateMassFlux(U), then
 * assembleRelaxedMomentumComponent (RelaxedMomentum.cpp:30-104). */
int og_momentum_system(const og_grid* g, const og_bcs* bc, const og_simple_settings* s, int comp,
                       const double* u, const double* v, const double* w, const double* p,
                       double* diag, double* const off[6], double* rhs);

/* Green-Gauss gradient of a scalar with pressure-type BCs (Gradient.cpp:534-607),
 * gx/gy/gz per cell. */
int og_scalar_gradient(const og_grid* g, const og_bcs* bc, const double* phi, double* gx,
                       double* gy, double* gz);

#ifdef __cplusplus
}
#endif
#endif
