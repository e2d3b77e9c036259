/* cfdb -- C ABI of the B200-native SIMPLE pressure-velocity path.
 *
 * Plain C types only (pointers, sizes, PODs): no C++, no torch.  Every entry
 * point returns a cfdb_status; on error the context keeps a message readable
 * with cfdb_last_error().  Calls on one context must be serialised by the
 * caller (the reference's GPU solvers carry the same one-host-thread rule,
 * GpuLinearSolverCuda.cpp:327-334); distinct contexts are independent.
 *
 * Layout of every field (shared with the reference's Cartesian meshes,
 * MeshGeometry.cpp:417-476 and :1047-1140):
 *   cell (i,j,k)     -> i + nx*(j + ny*k)                (2D: k = 0)
 *   faces, global order: x-faces, then y-faces, then z-faces
 *     x-face (i,j,k), i in [0,nx]: i + (nx+1)*(j + ny*k)
 *     y-face (i,j,k), j in [0,ny]: i + nx*(j + (ny+1)*k)
 *     z-face (i,j,k), k in [0,nz]: i + nx*(j + ny*k)
 *   patches: 0 xmin (left) 1 xmax (right) 2 ymin (bottom) 3 ymax (top) 4 zmin 5 zmax
 */
#ifndef CFDB_H
#define CFDB_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CFDB_API __attribute__((visibility("default")))
#else
#define CFDB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int cfdb_status;
enum {
  CFDB_OK = 0,
  CFDB_ERR_INVALID_ARGUMENT = -1,
  CFDB_ERR_CUDA = -2,
  CFDB_ERR_NO_DEVICE = -3,
  CFDB_ERR_OUT_OF_MEMORY = -4,
  CFDB_ERR_DEVICE_TIMEOUT = -5, /* a bounded device-side wait gave up (no fault) */
  CFDB_ERR_UNSUPPORTED = -6
};

/* Linear-solve outcome, SolverStatus (include/cfd/algebra/LinearSolver.hpp:16-23). */
enum {
  CFDB_SOLVER_CONVERGED = 0,
  CFDB_SOLVER_MAX_ITERATIONS = 1,
  CFDB_SOLVER_BREAKDOWN = 2,
  CFDB_SOLVER_NONFINITE_INPUT = 3,
  CFDB_SOLVER_NONFINITE_RESIDUAL = 4,
  CFDB_SOLVER_INVALID_SYSTEM = 5
};

/* SIMPLE outcome, SIMPLEStatus (include/cfd/pressure_velocity/SIMPLEResult.hpp:21-31). */
enum {
  CFDB_SIMPLE_CONVERGED = 0,
  CFDB_SIMPLE_MAX_ITERATIONS = 1,
  CFDB_SIMPLE_MOMENTUM_FAILURE = 2,
  CFDB_SIMPLE_PRESSURE_FAILURE = 3,
  CFDB_SIMPLE_NONFINITE_STATE = 4,
  CFDB_SIMPLE_INVALID_CONFIGURATION = 5
};

typedef struct cfdb_context cfdb_context;
typedef struct cfdb_poperator cfdb_poperator;

typedef struct {
  int dim;        /* 2 or 3 */
  int64_t n[3];   /* cells per axis; n[2] ignored in 2D */
  double len[3];  /* domain lengths; len[2] ignored in 2D */
} cfdb_grid;

/* Krylov method / precision / preconditioner selection. */
enum { CFDB_KRYLOV_CG = 0, CFDB_KRYLOV_BICGSTAB = 1 };
enum {
  CFDB_PRECISION_FP64 = 0,          /* every sweep in FP64 (the reference's arithmetic) */
  CFDB_PRECISION_FP32_REFINED = 1   /* mixed precision: FP32 directions, FP64 iterate and
                                       residual with residual replacement (one Krylov space;
                                       rows a multiple of 16 bytes in FP32), else FP32 inner
                                       solves inside FP64 iterative refinement */
};
enum {
  CFDB_PRECOND_NONE = 0,
  CFDB_PRECOND_JACOBI = 1,     /* JacobiPreconditioner (src/algebra/Preconditioner.cpp:11-49) */
  CFDB_PRECOND_LEARNED_MG = 2  /* no counterpart in the reference: learned V-cycle inside FP64
                                  flexible CG; Jacobi-PCG takes over if it stagnates */
};

/* LinearSolverSettings (LinearSolver.hpp:136-166) plus the precision knobs. */
typedef struct {
  int krylov;             /* CFDB_KRYLOV_* */
  int preconditioner;     /* CFDB_PRECOND_* */
  int precision;          /* CFDB_PRECISION_* */
  double abs_tol;         /* ||r||_2 <= abs_tol, or */
  double rel_tol;         /* ||r||_2 / ||r0||_2 <= rel_tol (unpreconditioned residual) */
  int64_t max_iterations; /* FP64: Krylov iterations; FP32_REFINED: total inner iterations */
  double inner_rel_tol;   /* FP32_REFINED: residual drop between FP64 residual replacements
                             (default 0.1), or the reduction asked of each inner solve of the
                             refinement form (default 1e-4); 0 = default */
  int64_t max_refinements;/* FP32_REFINED, refinement form: outer FP64 steps (0 = default) */
} cfdb_linear_settings;

/* SolverResult (LinearSolver.hpp:110-134) plus refinement counters. */
typedef struct {
  int status;                 /* CFDB_SOLVER_* */
  int64_t iterations;         /* Krylov iterations (FP32_REFINED: inner iterations, summed) */
  double initial_residual;    /* ||b - A x0||_2 */
  double final_residual;      /* ||b - A x||_2 as the method tracks it */
  double true_residual;       /* FP64-recomputed ||b - A x||_2 of the returned x */
  int64_t refinements;        /* FP32_REFINED: FP64 residual replacements (refinement form:
                                 outer FP64 steps) taken */
  int64_t restarts;           /* BiCGSTAB restarts */
  double device_ms;           /* device time of the solve (CUDA events, launching stream) */
  int64_t kernel_launches;    /* kernels this library launched for the solve */
  double krylov_ms;           /* device time inside the persistent Krylov kernels */
  double krylov_bytes;        /* algorithmic bytes those kernels move (words read + written) */
  int64_t krylov_launches;    /* number of persistent Krylov kernel launches */
  int64_t fallback_iterations;/* LEARNED_MG: Jacobi-PCG iterations after a stagnated learned solve */
} cfdb_linear_result;

/* ------------------------------------------------------------------ context */

/* cudaAvailable() (include/cfd/gpu/GPUBackend.hpp:15): 1 if a CUDA device of
 * compute capability 10.x is usable, else 0.  Never fails loudly. */
CFDB_API int cfdb_cuda_available(void);

/* One context per device and host thread.  stream may be NULL (the context
 * creates its own non-blocking stream) or a caller cudaStream_t. */
CFDB_API cfdb_status cfdb_create(int device, void* stream, cfdb_context** out);
CFDB_API void cfdb_destroy(cfdb_context* ctx);
CFDB_API const char* cfdb_last_error(const cfdb_context* ctx);
/* The cudaStream_t every call of this context launches on. */
CFDB_API void* cfdb_stream(cfdb_context* ctx);
/* Number of kernels this context launched so far (instrumentation). */
CFDB_API int64_t cfdb_kernel_launches(const cfdb_context* ctx);

/* Seeded synthetic p' RHS of the isolated solve (32 random-phase
 * sinusoids, wavenumbers 1..64, amplitude |k|^-2, zero mean, cell 0 pinned):
 * host output of nx*ny[*nz] doubles.  nz = 0 selects 2D. */
CFDB_API cfdb_status cfdb_synth_rhs(int64_t nx, int64_t ny, int64_t nz, uint64_t seed, double* b_host);

/* ------------------------------------------------- structured p' operator */

/* The p' operator of assembleGeometricPressureCorrection
 * (src/pressure_velocity/PressureCorrectionEquation.cpp:181-339) on a uniform
 * Cartesian grid, held on the device matrix-free:
 *   (A x)_P = (sum_f D_f) x_P - sum_{internal f} D_f x_N,
 * the diagonal summed in face order; when `pinned`, row `reference_cell` is
 * the identity (the reference pins it when no FixedValue pressure patch
 * exists, :221-228 and :326-329) while the neighbouring rows keep their
 * coupling to it.
 *
 * _uniform: unit response coefficients and density rho on all faces,
 *   D_f = rho |S_f| / |d_f| computed from the grid exactly as the reference
 *   does; boundary faces Neumann (0) unless dirichlet_patch_mask has the
 *   patch's bit set (then D_b = rho |S_f| / |x_f - x_P|).  This is the
 *   isolated p' system of the benchmark.
 * _faces: arbitrary face coefficients (host, global face order, boundary
 *   faces included: 0 for Neumann), e.g. the faceCoefficient field of a
 *   SIMPLE iteration. */
CFDB_API cfdb_status cfdb_poperator_create_uniform(cfdb_context* ctx, const cfdb_grid* grid, double rho,
                                          unsigned dirichlet_patch_mask, int pinned,
                                          int64_t reference_cell, cfdb_poperator** out);
CFDB_API cfdb_status cfdb_poperator_create_faces(cfdb_context* ctx, const cfdb_grid* grid,
                                        const double* face_coeff_host, int pinned,
                                        int64_t reference_cell, cfdb_poperator** out);
/* New face coefficients for an operator made by _create_faces (same grid,
 * pinning and layout): the values a SIMPLE host assembles again every outer
 * iteration (assembleGeometricPressureCorrection, :181-339).  Keeps the
 * operator's device arrays and, for the learned solve, its hierarchy and
 * solve graph (only their values are refreshed). */
CFDB_API cfdb_status cfdb_poperator_update_faces(cfdb_context* ctx, cfdb_poperator* op,
                                                 const double* face_coeff_host);
CFDB_API void cfdb_poperator_destroy(cfdb_poperator* op);
CFDB_API int64_t cfdb_poperator_cells(const cfdb_poperator* op);

/* y = A x on device pointers (FP64). */
CFDB_API cfdb_status cfdb_poperator_apply(cfdb_context* ctx, const cfdb_poperator* op, const double* x_dev,
                                 double* y_dev);

/* Solve A x = b.  Replaces the reference's CG::solve / BiCGSTAB::solve
 * (src/algebra/CG.cpp:14-148) for this operator, same status semantics and
 * convergence test.
 *   _device: b_dev, x_dev (x0 on entry, solution on exit) are device pointers;
 *   _host:   host pointers, copied in and out inside the call.
 * history (host, may be NULL) receives residualHistory: entry 0 = ||r0||,
 * entry k = ||r|| after iteration k, at most history_cap entries. */
CFDB_API cfdb_status cfdb_poperator_solve_device(cfdb_context* ctx, const cfdb_poperator* op,
                                        const cfdb_linear_settings* settings, const double* b_dev,
                                        double* x_dev, double* history, int64_t history_cap,
                                        cfdb_linear_result* result);
CFDB_API cfdb_status cfdb_poperator_solve_host(cfdb_context* ctx, const cfdb_poperator* op,
                                      const cfdb_linear_settings* settings, const double* b_host,
                                      double* x_host, double* history, int64_t history_cap,
                                      cfdb_linear_result* result);

/* ------------------------------------------- CSR systems (LinearSystem) */

/* The reference's solver contract takes a host CSR LinearSystem
 * (include/cfd/algebra/LinearSystem.hpp:12-24, SparseMatrix.hpp:19-56:
 * row offsets and ascending 64-bit column indices, exact zeros dropped) and
 * an initial guess, LinearSolver::solve (LinearSolver.hpp:176-180); the GPU
 * plugin that serves it is cfd::gpu::makeGpuCG / makeGpuBiCGSTAB
 * (include/cfd/gpu/GpuLinearSolver.hpp:48-54).  These entry points take the
 * same arrays.
 *
 * Recognition: the matrix must be the structured 5-point (2D) or 7-point
 * (3D) operator of a Cartesian grid in the reference's cell order
 * (i + nx*(j + ny*k)): every stored off-diagonal couples a cell to a grid
 * neighbour, and the strides 1, nx (, nx*ny) all occur (a band with stride 1
 * only is taken as one row of cells, nx x 1).  That is the shape of
 * every momentum and p' system the reference assembles on createCartesian2D
 * / createCartesian3D meshes (the wall three-point term couples a wall cell
 * to its first neighbour, so it stays in the band).  Anything else is
 * CFDB_ERR_UNSUPPORTED: the library runs no CSR kernel and no CPU solver.
 *
 * Paths: a CG system whose couplings are symmetric apart from at most one
 * identity row (the pinned reference cell, PressureCorrectionEquation.cpp:
 * 326-329), whose boundary faces carry no coefficient, and whose stored
 * diagonal equals the face-order sum of its couplings bit for bit is solved
 * by the face-coefficient p' operator (CFDB_CSR_PATH_FACES: the persistent
 * Jacobi-PCG, or the learned preconditioner); every other recognised system
 * (BiCGSTAB, non-symmetric momentum rows, Dirichlet faces, no
 * preconditioner) by the stencil Krylov solver with the stored diagonal
 * (CFDB_CSR_PATH_STENCIL).  A learned-preconditioner request on a system that
 * only the stencil path takes runs Jacobi-PCG and says so in
 * info->learned_declined. */
enum { CFDB_CSR_PATH_STENCIL = 0, CFDB_CSR_PATH_FACES = 1 };
typedef struct {
  int dim;                 /* 2 or 3 */
  int64_t n[3];            /* cells per axis (n[2] = 1 in 2D) */
  int path;                /* CFDB_CSR_PATH_* the solve took (faces_eligible for _analyze) */
  int faces_eligible;      /* the face-coefficient operator reproduces the matrix exactly */
  int pinned;              /* one identity row found */
  int64_t reference_cell;  /* its index (-1 if none) */
  int learned_declined;    /* LEARNED_MG asked for but the system needs the stencil path */
} cfdb_csr_info;

/* Host-only recognition (no device needed): fills info or returns
 * CFDB_ERR_UNSUPPORTED. */
CFDB_API cfdb_status cfdb_csr_analyze(int64_t rows, const uint64_t* row_offsets,
                                      const uint64_t* columns, const double* values,
                                      cfdb_csr_info* info);

typedef struct cfdb_csr_solver cfdb_csr_solver;
/* A solver keeps its device buffers (and, on the faces path, the operator
 * with its learned hierarchy) between solves of systems of one shape, as the
 * reference's GPU solvers keep theirs (GpuLinearSolverCuda.cpp:327-334). */
CFDB_API cfdb_status cfdb_csr_solver_create(cfdb_context* ctx, cfdb_csr_solver** out);
CFDB_API void cfdb_csr_solver_destroy(cfdb_csr_solver* s);
/* Solves A x = b from x0 (x_host in, solution out) with the settings'
 * Krylov method and preconditioner; statuses, convergence test and
 * residual history as CG::solve / BiCGSTAB::solve (src/algebra/CG.cpp:14-148,
 * BiCGSTAB.cpp:48-275): NonFiniteInput for a non-finite value of A, b or x0
 * (checked first), InvalidSystem when the Jacobi build fails
 * (Preconditioner.cpp:11-32), then the solve.  history (may be NULL) gets up
 * to history_cap entries of residualHistory.  info (may be NULL) reports the
 * recognised grid and the path taken. */
CFDB_API cfdb_status cfdb_csr_solve_host(cfdb_csr_solver* s, const cfdb_linear_settings* settings,
                                         int64_t rows, const uint64_t* row_offsets,
                                         const uint64_t* columns, const double* values,
                                         const double* b_host, double* x_host, double* history,
                                         int64_t history_cap, cfdb_linear_result* result,
                                         cfdb_csr_info* info);

/* Device buffers owned by the context's allocator (for callers without a
 * CUDA runtime of their own: tests, FFI hosts). */
CFDB_API cfdb_status cfdb_device_alloc(cfdb_context* ctx, size_t bytes, void** out);
CFDB_API cfdb_status cfdb_device_free(cfdb_context* ctx, void* ptr);
CFDB_API cfdb_status cfdb_copy_to_device(cfdb_context* ctx, void* dst_dev, const void* src_host, size_t bytes);
CFDB_API cfdb_status cfdb_copy_to_host(cfdb_context* ctx, void* dst_host, const void* src_dev, size_t bytes);
CFDB_API cfdb_status cfdb_memset_device(cfdb_context* ctx, void* dst_dev, int value, size_t bytes);
CFDB_API cfdb_status cfdb_synchronize(cfdb_context* ctx);

/* ------------------------------------------------------------------ SIMPLE */

/* Velocity and pressure boundary conditions per patch (reference classes
 * src/boundary/{Wall,MovingWall,Inlet,Outlet,FixedGradient,FixedValue}.cpp). */
enum { CFDB_VBC_WALL = 0, CFDB_VBC_MOVING_WALL = 1, CFDB_VBC_INLET = 2, CFDB_VBC_OUTLET = 3 };
enum { CFDB_PBC_FIXED_GRADIENT = 0, CFDB_PBC_FIXED_VALUE = 1 };
/* ConvectionScheme (include/cfd/discretization/Convection.hpp:22-27). */
enum { CFDB_SCHEME_UPWIND = 0, CFDB_SCHEME_CENTRAL = 1, CFDB_SCHEME_LINEAR_UPWIND = 2,
       CFDB_SCHEME_QUICK = 3 };
/* FaceFluxScheme (SIMPLESettings.hpp), resolved: Automatic is Linear in 2D,
 * RhieChow in 3D (resolveFaceFluxScheme). */
enum { CFDB_FLUX_LINEAR = 0, CFDB_FLUX_RHIE_CHOW = 1, CFDB_FLUX_AUTOMATIC = 2 };

/* A laminar incompressible case on a Cartesian grid, one BC per patch,
 * constant rho, mu.  Uniform axes are those of
 * MeshGeometry::createCartesian2D/3D (spacing len/n); an axis with node
 * coordinates is that of MeshGeometry::createRectilinear2D / createGraded2D
 * (MeshGeometry.hpp:228-240, AxisSpacing::fromNodes): nodes[a] holds its
 * n[a] + 1 strictly increasing node coordinates (host memory, copied at
 * session creation; len[a] is then not used), NULL for a uniform axis.
 * Cell centres, widths, face areas and volumes follow from the nodes as the
 * reference's AxisSpacing computes them. */
typedef struct {
  cfdb_grid grid;
  int vbc_type[6];
  double vbc_value[6][3];
  int pbc_type[6];
  double pbc_value[6];
  double rho, mu;
  const double* nodes[3];
} cfdb_simple_case;

/* SIMPLESettings (include/cfd/pressure_velocity/SIMPLESettings.hpp:42-145),
 * the subset this path supports (absolute convergence criterion, no
 * non-orthogonal corrections, Green-Gauss gradients). */
typedef struct {
  int64_t max_outer;
  double alpha_u, alpha_p;
  double tol_u, tol_p, tol_c;
  int scheme;             /* CFDB_SCHEME_* */
  int face_flux;          /* CFDB_FLUX_* */
  int64_t reference_cell;
  cfdb_linear_settings momentum;
  cfdb_linear_settings pressure;
} cfdb_simple_settings;

/* SIMPLEResult (SIMPLEResult.hpp:80-200), scalar part. */
typedef struct {
  int status;             /* CFDB_SIMPLE_* */
  int64_t iterations;
  double final_u, final_v, final_w, final_p, final_continuity, global_imbalance;
  int64_t momentum_linear_iterations;
  int64_t pressure_linear_iterations;
  double device_ms;       /* whole solve, CUDA events on the context stream */
  double pressure_solve_ms, momentum_solve_ms;
  int64_t kernel_launches;
} cfdb_simple_result;

typedef struct cfdb_simple cfdb_simple;

/* SIMPLE::solve (src/pressure_velocity/SIMPLE.cpp:148-1124), GPU-resident:
 * every stage runs on the device and only scalars cross per outer iteration.
 * u, v, w (ignored in 2D), p: host initial fields in, solution out; flux:
 * host output (global face order); history (may be NULL): 5 doubles per
 * outer iteration {u, v, w, p, continuity} residuals, up to max_outer rows. */
CFDB_API cfdb_status cfdb_simple_solve(cfdb_context* ctx, const cfdb_simple_case* cs,
                                       const cfdb_simple_settings* settings, double* u, double* v,
                                       double* w, double* p, double* flux, double* history,
                                       cfdb_simple_result* result);

/* No counterpart in the reference.  The face coefficients D_f (global face
 * order) of the p' system the session assembled last, with its pinning (1
 * and the reference cell when no FixedValue pressure patch exists): the
 * systems the learned preconditioner is trained and evaluated on. */
CFDB_API cfdb_status cfdb_simple_pprime_faces(cfdb_simple* s, double* faces, int* pinned,
                                             int64_t* reference_cell);

/* Stage-level session (the reference's GpuSimpleDiscretization,
 * include/cfd/gpu/GpuSimpleDiscretization.hpp:56-262): upload a state, run
 * single stages or outer iterations, read results back. */
CFDB_API cfdb_status cfdb_simple_create(cfdb_context* ctx, const cfdb_simple_case* cs,
                                        const cfdb_simple_settings* settings, cfdb_simple** out);
CFDB_API void cfdb_simple_destroy(cfdb_simple* s);
/* Uploads u, v, w, p and computes the face flux from u (calculateMassFlux). */
CFDB_API cfdb_status cfdb_simple_set_state(cfdb_simple* s, const double* u, const double* v,
                                           const double* w, const double* p);
CFDB_API cfdb_status cfdb_simple_get_state(cfdb_simple* s, double* u, double* v, double* w,
                                           double* p, double* flux);
/* Green-Gauss gradient of p with the pressure BCs (Gradient.cpp:534-607). */
CFDB_API cfdb_status cfdb_simple_pressure_gradient(cfdb_simple* s, double* gx, double* gy,
                                                   double* gz);
/* Relaxed momentum system of component comp from the current state
 * (RelaxedMomentum.cpp:30-104): diag, off[6] (low/high neighbour per axis), rhs. */
CFDB_API cfdb_status cfdb_simple_assemble_momentum(cfdb_simple* s, int comp, double* diag,
                                                   double* const off[6], double* rhs);
/* Runs up to n outer iterations from the current state (stops early on
 * convergence or failure); history as in cfdb_simple_solve. */
CFDB_API cfdb_status cfdb_simple_iterate(cfdb_simple* s, int64_t n, double* history,
                                         cfdb_simple_result* result);

/* Result files of a SIMPLE run in the reference's export formats
 * (ResultExporter::write, src/io/ResultExporter.cpp:36-110, without its
 * metadata.json): dir/residuals.csv (CSVWriter::writeResiduals) always, and,
 * when every u, v, (w,) p value is finite, dir/fields.csv
 * (CSVWriter::writeFields / writeFields3D) and dir/solution.vtk
 * (VTKWriter::writeSolution in 2D, writeCellFields in 3D); dir and its
 * parents are created.  Byte for byte what the reference writes for the same
 * values.  _results: host fields (u, v, w (3D), p in cell order), history
 * rows of 5 doubles {u, v, w, p, continuity} as cfdb_simple_solve writes
 * them, the run's final global mass imbalance; *fields_written (may be NULL)
 * = 1 when the field files were written.  Host only, no device needed. */
CFDB_API cfdb_status cfdb_write_results(const cfdb_simple_case* cs, const double* u, const double* v,
                                        const double* w, const double* p, const double* history,
                                        int64_t rows, double global_imbalance, const char* dir,
                                        int* fields_written);
/* The same files from a session's device fields (downloaded first). */
CFDB_API cfdb_status cfdb_simple_write_results(cfdb_simple* s, const double* history, int64_t rows,
                                               double global_imbalance, const char* dir,
                                               int* fields_written);

/* ---------------------------------------------------------- batched SIMPLE */

/* No counterpart in the reference, which solves one case per process
 * (ProjectRunner.cpp:278-282).  A batch advances many independent cases of
 * one dimension and uneven size together on one GPU, all under one settings
 * record: each SIMPLE stage is one persistent kernel over a tile list of all
 * cases, each momentum and p' solve one kernel in which every case's
 * Krylov solve runs on its own team of blocks, and one outer iteration of
 * the whole batch is one CUDA graph launch.  Each case stops on its own
 * (converged or failed) and keeps its state; the others go on.  Per case the
 * stages, statuses and convergence test are those of cfdb_simple_iterate.
 * Supported: CG or BiCGSTAB, no or Jacobi preconditioning, FP64 solves or,
 * for a CG p' solve, CFDB_PRECISION_FP32_REFINED (a mixed-precision CG that
 * keeps one Krylov space: FP32 matrix copy, direction and A p; FP64 x, r and
 * reductions; the FP64 true residual replaces the recurrence after every
 * ten-fold drop, at the tolerance and at the cap; inner_rel_tol and
 * max_refinements are not used), or, for an FP64 CG p' solve,
 * CFDB_PRECOND_LEARNED_MG (every active case's p' system by the single-case
 * learned FCG, case by case, between two graph launches of the stages),
 * uniform grids (others return CFDB_ERR_UNSUPPORTED). */
typedef struct cfdb_batch cfdb_batch;

/* Launch shapes of the batch: cells (faces) per tile and threads per block
 * of the cell (face) stage kernels; the p' team sizes of the first outer
 * iteration are proportional to cells^team_exponent, and with adaptive_teams
 * every later iteration sizes them by cells x the case's last p' iteration
 * count.  The autotuner fills the *_ms fields with the best times it
 * measured (device time of one launch; 0 when not tuned). */
typedef struct {
  int cell_threads, cell_tile;
  int face_threads, face_tile;
  double team_exponent;
  int adaptive_teams;
  double cell_stage_ms, face_stage_ms, pprime_solve_ms;
  int candidates;
} cfdb_batch_tuning;

typedef struct {
  int64_t graph_launches;   /* outer iterations of the batch run by this call */
  int active;               /* cases still iterating */
  double device_ms;         /* summed device time of the launches (CUDA events) */
  int64_t kernel_launches;  /* kernels those launches ran */
} cfdb_batch_stats;

/* cases[ncases], one dimension; history_cap > 0 keeps the first history_cap
 * rows of every case's residual history ({u, v, w, p, continuity} per outer
 * iteration, as cfdb_simple_solve writes it).  Initial state: zero fields. */
CFDB_API cfdb_status cfdb_batch_create(cfdb_context* ctx, int ncases, const cfdb_simple_case* cases,
                                       const cfdb_simple_settings* settings, int64_t history_cap,
                                       cfdb_batch** out);
CFDB_API void cfdb_batch_destroy(cfdb_batch* b);
CFDB_API int cfdb_batch_cases(const cfdb_batch* b);
/* Uploads case k's u, v, w (3D), p, computes its face flux from u and
 * restarts its outer-iteration count (as cfdb_simple_set_state); a
 * non-finite field stops the case at once with CFDB_SIMPLE_NONFINITE_STATE
 * (the initial check of cfdb_simple_solve). */
CFDB_API cfdb_status cfdb_batch_set_state(cfdb_batch* b, int k, const double* u, const double* v,
                                          const double* w, const double* p);
CFDB_API cfdb_status cfdb_batch_get_state(cfdb_batch* b, int k, double* u, double* v, double* w,
                                          double* p, double* flux);
/* Times candidate launch shapes on the batch's current state and keeps the
 * fastest: stage tile and block sizes on the momentum-assembly and mass-flux
 * stages, p' team sizing on the p' solves of the current state.  The state,
 * statuses and counters are left as they were. */
CFDB_API cfdb_status cfdb_batch_autotune(cfdb_batch* b, cfdb_batch_tuning* chosen);
CFDB_API cfdb_status cfdb_batch_set_tuning(cfdb_batch* b, const cfdb_batch_tuning* t);
CFDB_API cfdb_status cfdb_batch_get_tuning(cfdb_batch* b, cfdb_batch_tuning* t);
/* Up to n outer iterations of every case still iterating (fewer if all stop);
 * a case stops at convergence, on failure, or after settings->max_outer
 * outer iterations in all (status CFDB_SIMPLE_MAX_ITERATIONS). */
CFDB_API cfdb_status cfdb_batch_iterate(cfdb_batch* b, int64_t n, cfdb_batch_stats* stats);
/* One outer iteration run eagerly (not as a graph) with CUDA events around
 * every launch, for profiling: ids[i] is the launch's stage (an internal
 * stage number, -1 for a momentum solve kernel, -2 for the p' solve kernel)
 * and ms[i] its device time; *count = launches (at most cap are written).
 * The iteration is a real one: it advances the state like cfdb_batch_iterate. */
CFDB_API cfdb_status cfdb_batch_profile_iteration(cfdb_batch* b, int* ids, double* ms, int cap,
                                                  int* count);
/* Per-case outcome (results[ncases]): status (CFDB_SIMPLE_MAX_ITERATIONS
 * while a case still iterates), outer iterations, residuals of its last
 * completed iteration, linear-iteration totals (timings are left 0). */
CFDB_API cfdb_status cfdb_batch_results(cfdb_batch* b, cfdb_simple_result* results);
/* Case k's residual history: up to cap rows of 5 doubles; *rows = rows kept. */
CFDB_API cfdb_status cfdb_batch_history(cfdb_batch* b, int k, double* history, int64_t cap,
                                        int64_t* rows);

/* Case k's result files (see cfdb_write_results) from the batch's device
 * fields and the history it kept (history_cap rows at most). */
CFDB_API cfdb_status cfdb_batch_write_results(cfdb_batch* b, int k, const char* dir,
                                              int* fields_written);

/* Host-only planning of the batch's work lists (no device needed).
 * Tiles: case k's count[k] items split into ceil(count[k]/tile) tiles;
 * first[ncases+1] is the prefix sum; tile_case/tile_start (may be NULL)
 * receive each tile's case and first item. */
CFDB_API cfdb_status cfdb_batch_plan_tiles(int ncases, const int64_t* count, int tile, int* first,
                                           int* tile_case, int64_t* tile_start);
/* Teams: nblocks blocks split among the active cases, each active case at
 * least one block and at most max(1, cells[k] / min_cells_per_block);
 * blocks go one at a time to the case with the most weight per block
 * (highest weight[k] / blocks[k], lowest k on ties), which minimises the
 * largest weight per block.  team_first[ncases+1] is the prefix sum (0
 * blocks for inactive cases); block_case[nblocks] the case of each block
 * (-1: idle).  CFDB_ERR_UNSUPPORTED if more cases are active than blocks. */
CFDB_API cfdb_status cfdb_batch_plan_teams(int ncases, const double* weight, const int64_t* cells,
                                           const int* active, int nblocks,
                                           int64_t min_cells_per_block, int* team_first,
                                           int* block_case);

/* ------------------------------------------- learned preconditioner weights */

/* No counterpart in the reference.  Weights of the CFDB_PRECOND_LEARNED_MG
 * V-cycle used by this context's solves of dimension `dim` (2 or 3):
 * `levels` kernels of 27 taps each (3x3x3, x fastest; 2D kernels use taps
 * 9..17 only and must leave the others 0), point-symmetric (tap t equals tap
 * 26-t), one coarse-correction weight per level; levels deeper than `levels`
 * reuse the last kernel.  nu = smoothing sweeps per side (1..8),
 * coarse_sweeps = damped-Jacobi sweeps on the coarsest level (0..1000).
 * Invalid sets return CFDB_ERR_INVALID_ARGUMENT and change nothing. */
CFDB_API cfdb_status cfdb_mg_set_weights(cfdb_context* ctx, int dim, int levels, int nu,
                                         int coarse_sweeps, const float* kernels,
                                         const float* coarse_weights);
/* Reads the current set: kernels[16*27], coarse_weights[16] (any may be NULL). */
CFDB_API cfdb_status cfdb_mg_get_weights(cfdb_context* ctx, int dim, int* levels, int* nu,
                                         int* coarse_sweeps, float* kernels,
                                         float* coarse_weights);
/* trained = 1: the weights shipped with the library; 0: untrained damped Jacobi. */
CFDB_API cfdb_status cfdb_mg_reset_weights(cfdb_context* ctx, int dim, int trained);
/* No counterpart in the reference.  z = M r: one application of the learned
 * V-cycle of `op` (the context's weights) through the solve's own kernels;
 * host FP32 vectors in op's cell order (r[reference cell] reads as 0 and
 * z[reference cell] = r[reference cell] when the operator is pinned). */
CFDB_API cfdb_status cfdb_mg_apply(cfdb_context* ctx, cfdb_poperator* op, const float* r_host,
                                   float* z_host);
/* No counterpart in the reference.  Training signal of the learned V-cycle on
 * the GPU: for `nsamples` error fields e (host, nsamples x cells FP32, cell
 * order of `op`; e[reference cell] is taken as 0 when the operator is pinned)
 * the loss  mean ||e - M A e||_A^2 / ||e||_A^2  of the context's current
 * weights for op's dimension, and its exact gradient by reverse-mode
 * differentiation: grad_kernels[16*27] (tied taps t and 26-t receive the same
 * summed value; 2D sets use taps 9..17) and grad_coarse[16], per level that
 * owns weights (levels deeper than the weight set's count add into the last).
 * Either gradient pointer may be NULL. */
CFDB_API cfdb_status cfdb_mg_loss_grad(cfdb_context* ctx, cfdb_poperator* op, int nsamples,
                                       const float* e_host, double* loss, double* grad_kernels,
                                       double* grad_coarse);

/* ------------------------------------------------------------------ self-test */

/* No counterpart in the reference.  Exercises the bounded device-side wait
 * that the persistent kernels' grid and team barriers use: a two-block kernel
 * waits on a barrier sized for three blocks, which can never complete; after
 * timeout_s (0 < timeout_s <= 10) the blocks give up, raise the barrier's
 * error flag and return.  Returns CFDB_ERR_DEVICE_TIMEOUT (the expected
 * outcome) with *blocks_released = the number of blocks whose barrier call
 * reported the failure (2); the context stays usable.  No GPU fault. */
CFDB_API cfdb_status cfdb_selftest_wait_timeout(cfdb_context* ctx, double timeout_s,
                                                int* blocks_released);

/* ------------------------------------------------------ allocation-free solve */

/* No counterpart in the reference.  The FP64 Jacobi-PCG of the uniform p'
 * operator (the system cfdb_poperator_create_uniform builds with no
 * Dirichlet patch) for callers that cannot allocate device memory when they
 * solve -- a host whose device memory belongs to another runtime's
 * allocator, or a loop that forbids cudaMalloc/cudaFree after start-up
 * (both synchronise the device).  It needs no context: it launches on
 * `stream` (NULL: the legacy default stream) of the current device, reads
 * b_dev, updates x_dev (x0 on entry), and keeps every other vector and
 * reduction slot in one fixed device array of about 1.6 MB that each GPU
 * loading this library holds until exit.  Grids above 65536 cells return
 * CFDB_ERR_UNSUPPORTED, as do settings other than CG + Jacobi in FP64.
 * The call waits for its result (it synchronises `stream`), so it cannot be
 * recorded into a CUDA graph: on a capturing stream it returns
 * CFDB_ERR_UNSUPPORTED before issuing any work and the capture stays valid.
 * The first call on each device (and again after the device's context is
 * re-created, e.g. by cudaDeviceReset) looks the array's address up with
 * cudaGetSymbolAddress.  Every call clears what must start at zero, but all
 * calls share the array: calls whose work overlaps on the GPU race on it.
 * Fills status, iterations, initial and final residual of `result`; no
 * timing.  After CFDB_ERR_DEVICE_TIMEOUT (a bounded device-side wait gave
 * up) x_dev holds a partial iterate, undefined as a solution or as a start;
 * result->iterations then tells how far the solve got. */
CFDB_API cfdb_status cfdb_pcg_solve_noalloc(void* stream, const cfdb_grid* grid, double rho,
                                            int pinned, int64_t reference_cell,
                                            const cfdb_linear_settings* settings,
                                            const double* b_dev, double* x_dev,
                                            cfdb_linear_result* result);

#ifdef __cplusplus
}
#endif
#endif
