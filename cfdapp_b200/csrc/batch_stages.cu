// Stage kernels of the batched SIMPLE (layout and work lists: batch.cuh).
//
// Every kernel is persistent: its blocks stride over the tile list of all
// cases, skip the tiles of cases that stopped, and apply to each cell (or
// face) of a tile the same per-item operation as the single-case kernel of
// the stage (simple_ops.cuh).  This translation unit is compiled without FMA
// contraction (-fmad=false), like simple_kernels.cu, so a batched stage
// computes bit for bit what the single-case stage computes for that case.
//
// Two kernels end with a per-case gate run by the last block to finish (an
// atomic ticket): BS_CHECK_PP stops the cases whose p' is not finite, and
// BS_RESIDUAL sums each case's continuity and net-flux partials in tile
// order (deterministic), stops cases with non-finite fields, makes the
// corrected flux current, counts the outer iteration, applies the
// convergence test (SolverRobustness.cpp:361-372 through SIMPLE.cpp:1025-1103)
// and stops a case at the settings' outer-iteration limit.
#include <cuda_runtime.h>

#include <cmath>

#include "batch.cuh"
#include "cfdb.h"
#include "grid_sync.cuh"
#include "simple_geo.cuh"
#include "simple_ops.cuh"

namespace cfdb {
namespace {

// Pointers of one case into a 3- or 6-array cell pool.
struct C3 {
  double* a[3];
  __device__ C3(double* const pool[3], int64_t off) {
    for (int q = 0; q < 3; ++q) a[q] = pool[q] ? pool[q] + off : nullptr;
  }
};
struct C6 {
  double* a[6];
  __device__ C6(double* const pool[6], int64_t off) {
    for (int q = 0; q < 6; ++q) a[q] = pool[q] + off;
  }
};

__device__ __forceinline__ unsigned* flag_of(const BatchDev& B, int word, int k) {
  return B.flags + (size_t)word * B.ncases + k;
}

// Walk the cell tiles of active cases: op(K, k, c) for each local cell c.
template <class Op>
__device__ __forceinline__ void for_cells(const BatchDev& B, Op&& op) {
  for (int t = blockIdx.x; t < B.ncell_tiles; t += gridDim.x) {
    const int k = B.ctile_case[t];
    if (!B.active[k]) continue;
    const BCase& K = B.cases[k];
    const int64_t s0 = B.ctile_start[t];
    const int64_t s1 = min(s0 + (int64_t)B.cell_tile, K.G.nc);
    for (int64_t c = s0 + threadIdx.x; c < s1; c += blockDim.x) op(K, k, c);
  }
}

template <class Op>
__device__ __forceinline__ void for_faces(const BatchDev& B, Op&& op) {
  for (int t = blockIdx.x; t < B.nface_tiles; t += gridDim.x) {
    const int k = B.ftile_case[t];
    if (!B.active[k]) continue;
    const BCase& K = B.cases[k];
    const int64_t s0 = B.ftile_start[t];
    const int64_t s1 = min(s0 + (int64_t)B.face_tile, K.G.nf);
    for (int64_t f = s0 + threadIdx.x; f < s1; f += blockDim.x) op(K, k, f);
  }
}

// Input checks of a stencil system row and its Jacobi inverse, as the
// single-case solver makes them before it starts (stencil_solve.cu:
// NonFiniteInput, BiCGSTAB.cpp:57-60; InvalidSystem from the Jacobi build,
// Preconditioner.cpp:11-32).
__device__ __forceinline__ unsigned row_checks(const SGeo& G, const double* diag,
                                               double* const off[6], const double* b,
                                               const double* x, int jacobi, double* inv,
                                               int64_t c) {
  int ijk[3];
  g_coords(G, c, ijk);
  bool ok = isfinite(diag[c]) && isfinite(b[c]) && isfinite(x[c]);
  for (int a = 0; a < G.dim; ++a) {
    if (ijk[a] > 0) ok = ok && isfinite(off[2 * a][c]);
    if (ijk[a] < G.n[a] - 1) ok = ok && isfinite(off[2 * a + 1][c]);
  }
  unsigned bad = ok ? 0u : BFLAG_NONFINITE_INPUT;
  if (jacobi) {
    const double d = diag[c];
    if (!isfinite(d) || d == 0.0 || fabs(d) < 1.0e-12) bad |= BFLAG_INVALID_SYSTEM;
    inv[c] = 1.0 / d;
  }
  return bad;
}

// ------------------------------------------------------------------ kernels

__global__ void k_face_values(BatchDev B, int prime) {
  for_faces(B, [&](const BCase& K, int k, int64_t id) {
    const double* phi = (prime ? B.pp : B.p) + K.c0;
    const int* ty = prime ? K.pctype : K.G.ptype;
    const double* va = prime ? K.pcvalue : K.G.pvalue;
    B.fv[K.f0 + id] = ops::scalar_face_value(K.G, ty, va, phi, id);
  });
}

// mode 0: first sweep into g; 1: sweep with prev = g into gtmp; 2: g = gtmp.
__global__ void k_gg(BatchDev B, int prime, int mode) {
  for_cells(B, [&](const BCase& K, int k, int64_t c) {
    if (mode != 0 && !K.G.transfer) return;
    double* const* gpool = prime ? B.gradU : B.gradP;
    const C3 g(gpool, K.c0), tmp(B.gtmp, K.c0);
    if (mode == 2) {
      for (int a = 0; a < K.G.dim; ++a) g.a[a][c] = tmp.a[a][c];
      return;
    }
    const double* phi = (prime ? B.pp : B.p) + K.c0;
    const double* fv = B.fv + K.f0;
    const double* none[3] = {nullptr, nullptr, nullptr};
    const double* prev[3] = {g.a[0], g.a[1], g.a[2]};
    ops::gg_sweep(K.G, phi, fv, mode == 0 ? none : prev, mode == 0 ? g.a : tmp.a, c);
  });
}

__global__ void k_ugrad(BatchDev B, int comp) {
  for_cells(B, [&](const BCase& K, int k, int64_t c) {
    if (!K.need_ugrad) return;
    const C3 g(B.gradU, K.c0);
    ops::velocity_gradient(K.G, B.U[comp] + K.c0, comp, g.a, c);
  });
}

__global__ void k_assemble(BatchDev B, int comp) {
  for_cells(B, [&](const BCase& K, int k, int64_t c) {
    const int64_t o = K.c0;
    const C3 gu(B.gradU, o);
    const double* none[3] = {nullptr, nullptr, nullptr};
    const double* gus[3] = {gu.a[0], gu.a[1], gu.a[2]};
    const C6 off(B.moff, o);
    const double* F = B.Fbuf[B.fsel[k]] + K.f0;
    double* diag = B.mdiag[comp] + o;
    double* rhs = B.mrhs + o;
    const double* uc = B.U[comp] + o;
    ops::assemble_momentum(K.G, K.mu, B.scheme, comp, uc, F, B.gradP[comp] + o,
                           K.need_ugrad ? gus : none, B.alpha_u, diag, off.a, rhs, c);
    double* us = B.Us[comp] + o;
    us[c] = uc[c];
    const unsigned bad = row_checks(K.G, diag, off.a, rhs, us, B.mom_jacobi, B.kinv + o, c);
    if (bad) atomicOr(flag_of(B, BF_MOM0 + comp, k), bad);
  });
}

__global__ void k_response(BatchDev B) {
  for_cells(B, [&](const BCase& K, int k, int64_t c) {
    const int64_t o = K.c0;
    for (int a = 0; a < K.G.dim; ++a) B.dres[a][o + c] = ops::response(K.G, B.mdiag[a][o + c], c);
    // the single-case path checks Us[0], Us[1] and Us[dim-1]
    const bool ok = isfinite(B.Us[0][o + c]) && isfinite(B.Us[1][o + c]) &&
                    isfinite(B.Us[K.G.dim - 1][o + c]);
    if (!ok) atomicOr(flag_of(B, BF_NONFINITE, k), 1u);
  });
}

__global__ void k_mass_flux(BatchDev B) {
  for_faces(B, [&](const BCase& K, int k, int64_t id) {
    const double* U[3] = {B.Us[0] + K.c0, B.Us[1] + K.c0, B.Us[2] + K.c0};
    B.Fs[K.f0 + id] = ops::mass_flux(K.G, K.rho, U, id);
  });
}

__global__ void k_rhie_chow(BatchDev B) {
  for_faces(B, [&](const BCase& K, int k, int64_t id) {
    const int64_t o = K.c0;
    const double* gp[3] = {B.gradP[0] + o, B.gradP[1] + o, B.gradP[2] + o};
    const double* d[3] = {B.dres[0] + o, B.dres[1] + o, B.dres[2] + o};
    ops::rhie_chow(K.G, K.rho, B.alpha_u, B.p + o, gp, d, B.Fs + K.f0, id);
  });
}

__global__ void k_pfaces(BatchDev B) {
  for_faces(B, [&](const BCase& K, int k, int64_t id) {
    const int64_t o = K.c0;
    const double* d[3] = {B.dres[0] + o, B.dres[1] + o, B.dres[2] + o};
    B.D[K.f0 + id] = ops::pprime_face(K.G, K.rho, d, id);
    if (!isfinite(B.Fs[K.f0 + id])) atomicOr(flag_of(B, BF_NONFINITE, k), 1u);
  });
}

__global__ void k_prows(BatchDev B) {
  for_cells(B, [&](const BCase& K, int k, int64_t c) {
    const int64_t o = K.c0;
    const C6 off(B.poff, o);
    double* diag = B.pdiag + o;
    double* rhs = B.prhs + o;
    double* x = B.pp + o;
    rhs[c] = ops::pprime_rhs(K.G, B.Fs + K.f0, K.pin, K.ref, c);
    x[c] = 0.0;
    ops::pprime_row(K.G, B.D + K.f0, K.pin, K.ref, diag, off.a, c);
    const unsigned bad = row_checks(K.G, diag, off.a, rhs, x, B.p_jacobi, B.kinv + o, c);
    if (bad) atomicOr(flag_of(B, BF_PP, k), bad);
  });
}

// The last block to arrive (atomic ticket) runs `gate`; the ticket is reset
// for the next launch.  Every block calls this exactly once, after its tiles.
template <class Gate>
__device__ __forceinline__ void last_block(const BatchDev& B, Gate&& gate) {
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(B.ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  gate();
  __syncthreads();
  if (threadIdx.x == 0) *B.ticket = 0u;
}

__global__ void k_check_pp(BatchDev B) {
  for_cells(B, [&](const BCase& K, int k, int64_t c) {
    if (!isfinite(B.pp[K.c0 + c])) atomicOr(flag_of(B, BF_NONFINITE, k), 1u);
  });
  last_block(B, [&]() {
    for (int k = threadIdx.x; k < B.ncases; k += blockDim.x) {
      if (B.active[k] && __ldcg(flag_of(B, BF_NONFINITE, k)) != 0u) {
        B.status[k] = CFDB_SIMPLE_NONFINITE_STATE;
        B.active[k] = 0;
      }
    }
  });
}

__global__ void k_correct(BatchDev B) {
  for_cells(B, [&](const BCase& K, int k, int64_t c) {
    const int64_t o = K.c0 + c;
    B.p[o] = B.p[o] + (B.alpha_p * B.pp[o]);
    for (int a = 0; a < K.G.dim; ++a) B.U[a][o] = B.Us[a][o] - (B.dres[a][o] * B.gradU[a][o]);
  });
}

__global__ void k_flux_correct(BatchDev B) {
  for_faces(B, [&](const BCase& K, int k, int64_t id) {
    double* Fn = B.Fbuf[1 - B.fsel[k]] + K.f0;
    Fn[id] = ops::flux_correct(K.G, B.Fs + K.f0, B.D + K.f0, B.pp + K.c0, id);
  });
}

__global__ void k_residual(BatchDev B) {
  __shared__ double red[32];
  const int nt = B.ncell_tiles + B.nface_tiles;
  for (int t = blockIdx.x; t < nt; t += gridDim.x) {
    const bool cells = t < B.ncell_tiles;
    const int k = cells ? B.ctile_case[t] : B.ftile_case[t - B.ncell_tiles];
    if (!B.active[k]) continue;  // uniform over the block
    const BCase& K = B.cases[k];
    const double* Fn = B.Fbuf[1 - B.fsel[k]] + K.f0;
    double acc = 0.0;
    bool ok = true;
    if (cells) {
      const int64_t s0 = B.ctile_start[t];
      const int64_t s1 = min(s0 + (int64_t)B.cell_tile, K.G.nc);
      for (int64_t c = s0 + threadIdx.x; c < s1; c += blockDim.x) {
        const double imb = ops::cell_imbalance(K.G, Fn, c);
        acc += imb * imb;
        const int64_t o = K.c0 + c;
        ok = ok && isfinite(B.U[0][o]) && isfinite(B.U[1][o]) && isfinite(B.U[K.G.dim - 1][o]) &&
             isfinite(B.p[o]);
      }
    } else {
      const int64_t s0 = B.ftile_start[t - B.ncell_tiles];
      const int64_t s1 = min(s0 + (int64_t)B.face_tile, K.G.nf);
      for (int64_t f = s0 + threadIdx.x; f < s1; f += blockDim.x) {
        if (ops::boundary_face(K.G, f)) acc += Fn[f];
        ok = ok && isfinite(Fn[f]);
      }
    }
    if (!ok) atomicOr(flag_of(B, BF_NONFINITE, k), 1u);
    double v[1] = {acc};
    block_sum<1>(v, red);
    if (threadIdx.x == 0) B.partials[t] = v[0];
  }
  last_block(B, [&]() {
    // one warp per case; lanes sum tiles lane, lane+32, ... then a fixed tree
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = warp; k < B.ncases; k += nw) {
      if (!B.active[k]) continue;
      double ss = 0.0, sb = 0.0;
      for (int t = B.ctile_first[k] + lane; t < B.ctile_first[k + 1]; t += 32)
        ss += __ldcg(B.partials + t);
      for (int t = B.ftile_first[k] + lane; t < B.ftile_first[k + 1]; t += 32)
        sb += __ldcg(B.partials + B.ncell_tiles + t);
      for (int o = 16; o > 0; o >>= 1) {
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
        sb += __shfl_xor_sync(0xffffffffu, sb, o);
      }
      if (lane != 0) continue;
      const BCase& K = B.cases[k];
      double* R = B.res + (size_t)k * BR_COUNT;
      if (__ldcg(flag_of(B, BF_NONFINITE, k)) != 0u) {
        B.status[k] = CFDB_SIMPLE_NONFINITE_STATE;
        B.active[k] = 0;
        continue;
      }
      B.fsel[k] = 1 - B.fsel[k];
      const int64_t it = B.outer[k];
      const double cont = sqrt(ss / (double)K.G.nc);
      const double glob = fabs(sb);
      R[BR_U] = R[BR_IU];
      R[BR_V] = R[BR_IV];
      R[BR_W] = K.G.dim == 3 ? R[BR_IW] : 0.0;
      R[BR_P] = R[BR_IP];
      R[BR_CONT] = cont;
      R[BR_GLOB] = glob;
      B.outer[k] = it + 1;
      if (B.history && it < B.history_cap) {
        double* h = B.history + ((size_t)k * B.history_cap + it) * 5;
        h[0] = R[BR_U];
        h[1] = R[BR_V];
        h[2] = R[BR_W];
        h[3] = R[BR_P];
        h[4] = cont;
      }
      const bool conv = (R[BR_U] <= B.tol_u) && (R[BR_V] <= B.tol_u) && (R[BR_P] <= B.tol_p) &&
                        (cont <= B.tol_c) && (glob <= B.tol_c) &&
                        (K.G.dim == 2 || R[BR_W] <= B.tol_u);
      if (conv) {
        B.status[k] = CFDB_SIMPLE_CONVERGED;
        B.active[k] = 0;
      } else if (it + 1 >= B.max_outer) {
        B.status[k] = CFDB_SIMPLE_MAX_ITERATIONS;
        B.active[k] = 0;
      }
    }
    __syncthreads();
    // active count after this iteration (fixed order)
    if (threadIdx.x == 0) {
      int nact = 0;
      for (int k = 0; k < B.ncases; ++k) nact += B.active[k] ? 1 : 0;
      *B.nactive = nact;
    }
  });
}

}  // namespace

void batch_stage_launch(const BatchDev& B, int stage, int comp, int grid, int threads,
                        cudaStream_t s) {
  switch (stage) {
    case BS_FACE_VALUES_P: k_face_values<<<grid, threads, 0, s>>>(B, 0); break;
    case BS_FACE_VALUES_PP: k_face_values<<<grid, threads, 0, s>>>(B, 1); break;
    case BS_GG_P: k_gg<<<grid, threads, 0, s>>>(B, 0, 0); break;
    case BS_GG_PP: k_gg<<<grid, threads, 0, s>>>(B, 1, 0); break;
    case BS_GG_P_SWEEP: k_gg<<<grid, threads, 0, s>>>(B, 0, 1); break;
    case BS_GG_PP_SWEEP: k_gg<<<grid, threads, 0, s>>>(B, 1, 1); break;
    case BS_GG_P_COPY: k_gg<<<grid, threads, 0, s>>>(B, 0, 2); break;
    case BS_GG_PP_COPY: k_gg<<<grid, threads, 0, s>>>(B, 1, 2); break;
    case BS_UGRAD: k_ugrad<<<grid, threads, 0, s>>>(B, comp); break;
    case BS_ASSEMBLE: k_assemble<<<grid, threads, 0, s>>>(B, comp); break;
    case BS_RESPONSE: k_response<<<grid, threads, 0, s>>>(B); break;
    case BS_MASS_FLUX: k_mass_flux<<<grid, threads, 0, s>>>(B); break;
    case BS_RHIE_CHOW: k_rhie_chow<<<grid, threads, 0, s>>>(B); break;
    case BS_PFACES: k_pfaces<<<grid, threads, 0, s>>>(B); break;
    case BS_PROWS: k_prows<<<grid, threads, 0, s>>>(B); break;
    case BS_CHECK_PP: k_check_pp<<<grid, threads, 0, s>>>(B); break;
    case BS_CORRECT: k_correct<<<grid, threads, 0, s>>>(B); break;
    case BS_FLUX_CORRECT: k_flux_correct<<<grid, threads, 0, s>>>(B); break;
    case BS_RESIDUAL: k_residual<<<grid, threads, 0, s>>>(B); break;
    default: break;
  }
}

const void* batch_stage_kernel(int stage) {
  switch (stage) {
    case BS_FACE_VALUES_P:
    case BS_FACE_VALUES_PP: return (const void*)k_face_values;
    case BS_GG_P:
    case BS_GG_PP:
    case BS_GG_P_SWEEP:
    case BS_GG_PP_SWEEP:
    case BS_GG_P_COPY:
    case BS_GG_PP_COPY: return (const void*)k_gg;
    case BS_UGRAD: return (const void*)k_ugrad;
    case BS_ASSEMBLE: return (const void*)k_assemble;
    case BS_RESPONSE: return (const void*)k_response;
    case BS_MASS_FLUX: return (const void*)k_mass_flux;
    case BS_RHIE_CHOW: return (const void*)k_rhie_chow;
    case BS_PFACES: return (const void*)k_pfaces;
    case BS_PROWS: return (const void*)k_prows;
    case BS_CHECK_PP: return (const void*)k_check_pp;
    case BS_CORRECT: return (const void*)k_correct;
    case BS_FLUX_CORRECT: return (const void*)k_flux_correct;
    case BS_RESIDUAL: return (const void*)k_residual;
    default: return nullptr;
  }
}

}  // namespace cfdb
