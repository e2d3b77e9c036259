// Batched SIMPLE: many independent cases of uneven size, all of one
// dimension and one settings record, advanced together on one GPU.
//
// Device layout.  Every field is one pool holding the cases back to back:
// case k's cells start at cell offset c0 and its faces at f0, both multiples
// of 32 elements (256 B) so every case starts on its own cache lines.  The
// case table (BCase) holds each case's geometry and constants.
//
// Work lists.  The stage kernels walk a tile list: tile t covers cells
// [start, start + tile) of case tile_case[t] (the prefix sum of each case's
// tile count orders the list case by case), and likewise for faces.  A kernel
// is persistent -- a grid of at most (SMs x resident blocks) blocks strides
// over the list -- and skips the tiles of cases that stopped.  Tile size and
// block size come from the autotuner.
//
// Krylov solves.  One kernel per solve stage runs every case's solve at
// once: a team of blocks per case (block_case maps blocks to cases) runs the
// routine of stencil_krylov.cuh with a barrier over the team only, so each
// case iterates to its own tolerance and its team leaves when done.
//
// Per-case state: active (1 while the case iterates), status, outer
// iteration count, residuals, linear-iteration counters; flags written by the
// stage kernels (non-finite fields, Krylov input checks) and read by later
// kernels of the same outer iteration; fsel, which of the two flux buffers
// holds the case's current face flux (the corrected flux is written to the
// other one and becomes current when the case passes its end-of-iteration
// checks, as the reference swaps it in, SIMPLE.cpp:983).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "simple_geo.cuh"

namespace cfdb {

struct BCase {
  SGeo G;
  double rho, mu;
  int pin;
  int need_ugrad;
  int64_t ref;
  int64_t c0, f0;  // pool offsets of the case's cells and faces
  int pctype[6];   // BCs of p' in its gradient: FixedValue(0) where p is FixedValue
  double pcvalue[6];
};

// Per-case result record (doubles): the residuals of the last completed outer
// iteration and the initial residuals of the linear solves in progress.
enum {
  BR_U = 0, BR_V, BR_W, BR_P, BR_CONT, BR_GLOB,
  BR_IU, BR_IV, BR_IW, BR_IP,
  BR_COUNT = 10
};
// Per-case flag words, one array of ncases each, cleared at the start of
// every outer iteration: non-finite state; momentum-solve input checks per
// component; p'-solve input checks.
enum { BF_NONFINITE = 0, BF_MOM0 = 1, BF_MOM1 = 2, BF_MOM2 = 3, BF_PP = 4, BF_COUNT = 5 };
enum { BFLAG_NONFINITE_INPUT = 1u, BFLAG_INVALID_SYSTEM = 2u };

struct BatchDev {
  int ncases;
  int dim;
  const BCase* cases;
  // tile lists
  int ncell_tiles, nface_tiles;
  int cell_tile, face_tile;  // cells / faces per tile
  const int* ctile_case;
  const int64_t* ctile_start;
  const int* ftile_case;
  const int64_t* ftile_start;
  const int* ctile_first;  // ncases + 1: first cell tile of each case
  const int* ftile_first;  // ncases + 1: first face tile of each case
  // cell pools
  double *U[3], *Us[3], *mdiag[3], *moff[6], *mrhs;
  double *gradP[3], *gradU[3], *gtmp[3], *dres[3];
  double *p, *pdiag, *poff[6], *prhs, *pp;
  double *kinv;  // Jacobi inverse diagonal of the system being solved
  double *kr, *krh, *kv, *kp, *ks, *kt;  // Krylov work vectors
  // face pools
  double *Fbuf[2], *Fs, *fv, *D;
  // per-case state
  int* active;
  int* status;
  int* fsel;
  int64_t* outer;
  int64_t* mom_it;
  int64_t* p_it;
  double* res;        // BR_COUNT per case
  unsigned* flags;    // BF_COUNT x ncases
  double* partials;   // one double per tile (cell tiles, then face tiles)
  unsigned* ticket;   // last-block ticket of the gate kernels
  int* nactive;       // active cases after the last outer iteration
  double* history;    // optional: 5 doubles per case per outer iteration
  int64_t history_cap;
  int64_t max_outer;  // outer iterations after which a case stops (MAX_ITERATIONS)
  // settings shared by the batch
  double alpha_u, alpha_p, tol_u, tol_p, tol_c;
  int scheme, face_flux;
  int mom_jacobi, p_jacobi;
};

// Stage kernels (batch_stages.cu).  `threads` is the block size of the
// launch, `grid` its block count.
enum BatchStage {
  BS_FACE_VALUES_P,   // fv = face values of p (pressure BCs)
  BS_FACE_VALUES_PP,  // fv = face values of p' (p' BCs)
  BS_GG_P,            // gradP = Green-Gauss of p, first sweep
  BS_GG_PP,           // gradU = Green-Gauss of p', first sweep
  BS_GG_P_SWEEP,      // gtmp = sweep(p, prev = gradP)   (cases with tangential transfer)
  BS_GG_PP_SWEEP,     // gtmp = sweep(p', prev = gradU)
  BS_GG_P_COPY,       // gradP = gtmp                     (same cases)
  BS_GG_PP_COPY,      // gradU = gtmp
  BS_UGRAD,           // gradU = velocity gradient of component comp
  BS_ASSEMBLE,        // momentum row of component comp, Us = U, input checks, Jacobi inverse
  BS_RESPONSE,        // d = V / aP for every component; Us finite check
  BS_MASS_FLUX,       // Fs = mass flux of Us
  BS_RHIE_CHOW,       // Fs += Rhie-Chow correction
  BS_PFACES,          // D = p' face coefficients; Fs finite check
  BS_PROWS,           // p' rows, rhs, p' = 0, input checks, Jacobi inverse
  BS_CHECK_PP,        // p' finite check; cases that fail stop (last-block gate)
  BS_CORRECT,         // p += alpha_p p'; U = Us - d grad p'
  BS_FLUX_CORRECT,    // F(next) = Fs + D (p'_P - p'_N)
  BS_RESIDUAL,        // continuity, net flux, finite checks; per-case gate and convergence
  BS_COUNT
};

void batch_stage_launch(const BatchDev& B, int stage, int comp, int grid, int threads,
                        cudaStream_t s);
// Kernel address of a stage (for occupancy queries).
const void* batch_stage_kernel(int stage);

}  // namespace cfdb
