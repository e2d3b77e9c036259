// Learned multigrid-shaped preconditioner for the p' operator and the
// flexible CG that uses it (no counterpart in the reference, whose p' solve
// is Jacobi-PCG, src/algebra/CG.cpp:14-148).
//
// The network is a V-cycle whose layers are convolutions over the grid:
// level l holds the p' operator agglomerated 2x2(x2) from level l-1 (coarse
// face coefficient = sum of the fine face coefficients it covers, i.e. the
// Galerkin operator of piecewise-constant prolongation), and its smoothing
// layer is a learned symmetric 3x3 (3x3x3) kernel W_l applied to the
// diagonally scaled residual:
//     x <- x + D^-1/2 (W_l * (D^-1/2 (r - A_l x)))          (nu times)
// The coarse correction is restricted by summation, prolongated by
// injection and scaled by a learned weight c_l; the coarsest level takes a
// fixed number of damped-Jacobi sweeps.  Pre- and post-smoothing use the same
// kernel, so the cycle is a symmetric linear operator.  Untrained, W_l is
// damped Jacobi (0.8 at the centre).
//
// The Krylov method around it is FCG(1) in FP64: the V-cycle runs in FP32 on
// an FP32 copy of the residual, and the search directions are
// A-orthogonalised against the previous one, so rounding in the
// preconditioner costs iterations, never accuracy.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "cfdb.h"
#include "cfdb_internal.cuh"
#include "poperator.cuh"

namespace cfdb {

constexpr int kMgMaxLevels = 16;
constexpr int kMgTaps = 27;  // 3x3x3 kernel, x fastest; 2D uses the middle 3x3 plane

struct MgWeights {
  int dim = 2;
  int levels = 1;                  // levels with their own kernel (deeper ones reuse the last)
  int nu = 2;                      // smoothing sweeps per side
  int coarse_sweeps = 50;          // damped-Jacobi sweeps on the coarsest level
  float w[kMgMaxLevels][kMgTaps];  // smoothing kernels
  float c[kMgMaxLevels];           // coarse-correction weights
};

// Damped Jacobi, unit coarse correction.
MgWeights mg_default_weights(int dim);
// Checks the symmetry and finiteness a usable weight set needs.
bool mg_weights_valid(const MgWeights& W, std::string* why);

// Levels live in kernel space: a 2D grid (nx, ny) is (nx, 1, ny) with no
// y-faces, so one set of kernels serves the 5- and 7-point operators.
struct MgLevel {
  int n[3];  // kernel-space cells per axis
  int64_t cells;
  float* f[3];  // face coefficients per kernel axis (f[1] null in 2D)
  float* isq;   // D^-1/2 (0 where the diagonal is 0)
  float* x;     // correction of this level
  float* r;     // right-hand side of this level
  float* res;   // residual scratch
};

struct MgHierarchy {
  int dim = 2;
  int levels = 0;
  int coarse_from = 0;        // levels >= coarse_from run inside one thread block
  size_t coarse_smem = 0;     // dynamic shared memory of that block
  MgLevel L[kMgMaxLevels];
  std::vector<void*> owned;
  MgHierarchy() = default;
  MgHierarchy(const MgHierarchy&) = delete;
  MgHierarchy& operator=(const MgHierarchy&) = delete;
  ~MgHierarchy();
};

// The fine operator as the learned solve sees it, in kernel space: the FP64
// view (the exact reference operator, pinned row included) and, per kernel
// axis, either a full face array or a per-axis table of face coefficients
// (both null for the 2D y axis).
struct FineOperator {
  int dim;
  int n[3];                // kernel-space cells per axis
  OpView<double> A;
  const double* full[3];
  const double* table[3];
  int pinned;
  int64_t ref;
};

cfdb_status mg_build(cfdb_context* ctx, MgHierarchy& H, const FineOperator& op);

// z = M r on FP32 fine-level vectors (r[skip] read as 0, z[skip] = r[skip]).
cfdb_status mg_apply(cfdb_context* ctx, const MgHierarchy& H, const MgWeights& W, const float* r,
                     float* z, int64_t skip);

// One learned-FCG solver bound to an operator; owns its hierarchy, vectors
// and the captured CUDA graph of the solve loop.
struct LearnedSolver;

LearnedSolver* learned_create();
void learned_destroy(LearnedSolver* s);

struct LearnedOutcome {
  int status;          // CFDB_SOLVER_*, or kLearnedStagnated
  int64_t iterations;
  double initial_residual, final_residual;
  double kernel_ms;    // device time of the solve graph
  double bytes;        // algorithmic bytes moved
  int64_t launches;    // kernels in the executed graph
};
constexpr int kLearnedStagnated = 100;

// Solves A x = b (FP64 device vectors; x holds the initial guess).  The
// operator must stay the same between calls with the same `version`.
// hist_cap: residual-history entries kept on the device (iteration 0..).
cfdb_status learned_solve(cfdb_context* ctx, LearnedSolver* s, const FineOperator& op,
                          uint64_t version, const MgWeights& W, const double* b, double* x,
                          double abs_tol, double rel_tol, int64_t max_it, int64_t hist_cap,
                          LearnedOutcome* out);
// The solver's hierarchy for `op`, built or refreshed as a solve would.
cfdb_status learned_hierarchy(cfdb_context* ctx, LearnedSolver* s, const FineOperator& op,
                              uint64_t version, const MgHierarchy** out);
// Copies the first m residual-history entries of the last solve to the host.
cfdb_status learned_history(cfdb_context* ctx, LearnedSolver* s, double* host, int64_t m);

// Kernel-space taps of level l (2D weight sets keep their 3x3 taps in the
// middle plane of the 27; kernel space maps real y to z).
void mg_kernel_taps(const MgWeights& W, int l, float out[kMgTaps]);

// The weights shipped with the library (trained), or the defaults when none.
MgWeights mg_builtin_weights(int dim);
// The per-context weight set used by CFDB_PRECOND_LEARNED_MG solves.
const MgWeights& mg_context_weights(cfdb_context* ctx, int dim);

}  // namespace cfdb
