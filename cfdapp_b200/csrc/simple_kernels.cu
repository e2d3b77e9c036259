// Stage kernels of the resident SIMPLE loop on uniform Cartesian grids.
//
// One thread per cell (or face) applies the per-item operation of
// simple_ops.cuh that restates the reference function named beside each
// kernel; this translation unit is compiled without FMA contraction
// (-fmad=false), so a stage reproduces the reference bit for bit given
// bit-identical inputs.
#include <cuda_runtime.h>

#include "simple_geo.cuh"
#include "simple_kernels.cuh"
#include "simple_ops.cuh"

namespace cfdb {
namespace {

constexpr int kBlock = 256;

inline int grid_for(int64_t n) {
  int64_t g = (n + kBlock - 1) / kBlock;
  if (g < 1) g = 1;
  if (g > 65535LL * 32) g = 65535LL * 32;
  return (int)g;
}

#define GRID_STRIDE(q, n) \
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < (n); q += (int64_t)gridDim.x * blockDim.x)

// calculateMassFlux (physics/MassFlux.cpp:15-35).
__global__ void k_mass_flux(SGeo G, double rho, const double* u0, const double* u1,
                            const double* u2, double* F) {
  const double* U[3] = {u0, u1, u2};
  GRID_STRIDE(id, G.nf) F[id] = ops::mass_flux(G, rho, U, id);
}

// Scalar face values with pressure-type BCs (Interpolation.cpp interpolateFace).
__global__ void k_scalar_face_values(SGeo G, const int* ptype, const double* pvalue,
                                     const double* phi, double* fv) {
  GRID_STRIDE(id, G.nf) fv[id] = ops::scalar_face_value(G, ptype, pvalue, phi, id);
}

// One boundary-consistent Green-Gauss sweep (Gradient.cpp:104-162, :431-482).
__global__ void k_gg_sweep(SGeo G, const double* phi, const double* fv, const double* prev0,
                           const double* prev1, const double* prev2, double* g0, double* g1,
                           double* g2) {
  const double* prev[3] = {prev0, prev1, prev2};
  double* out[3] = {g0, g1, g2};
  GRID_STRIDE(c, G.nc) ops::gg_sweep(G, phi, fv, prev, out, c);
}

// Plain Green-Gauss gradient of a velocity component (VectorGradient.cpp:19-52).
__global__ void k_velocity_gradient(SGeo G, const double* uc, int comp, double* g0, double* g1,
                                    double* g2) {
  double* grad[3] = {g0, g1, g2};
  GRID_STRIDE(c, G.nc) ops::velocity_gradient(G, uc, comp, grad, c);
}

// assembleRelaxedMomentumComponent (pressure_velocity/RelaxedMomentum.cpp:30-104).
__global__ void k_assemble_momentum(SGeo G, double mu, int scheme, int comp, const double* uc,
                                    const double* F, const double* gradPc, const double* gu0,
                                    const double* gu1, const double* gu2, double alpha,
                                    double* diag, double* o0, double* o1, double* o2, double* o3,
                                    double* o4, double* o5, double* rhs) {
  const double* gradU[3] = {gu0, gu1, gu2};
  double* off[6] = {o0, o1, o2, o3, o4, o5};
  GRID_STRIDE(c, G.nc)
  ops::assemble_momentum(G, mu, scheme, comp, uc, F, gradPc, gradU, alpha, diag, off, rhs, c);
}

// d = V / aP (PressureCorrectionEquation.cpp:103-114).
__global__ void k_response(SGeo G, const double* diag, double* d) {
  GRID_STRIDE(c, G.nc) d[c] = ops::response(G, diag[c], c);
}

// Rhie-Chow correction of the internal faces (RhieChow.cpp:17-51).
__global__ void k_rhie_chow(SGeo G, double rho, double alpha, const double* p, const double* gp0,
                            const double* gp1, const double* gp2, const double* d0,
                            const double* d1, const double* d2, double* F) {
  const double* gp[3] = {gp0, gp1, gp2};
  const double* d[3] = {d0, d1, d2};
  GRID_STRIDE(id, G.nf) ops::rhie_chow(G, rho, alpha, p, gp, d, F, id);
}

// p' face coefficients (pressureCorrectionFaceCoupling, PressureCorrectionEquation.cpp:146-179).
__global__ void k_pprime_faces(SGeo G, double rho, const double* d0, const double* d1,
                               const double* d2, double* D) {
  const double* d[3] = {d0, d1, d2};
  GRID_STRIDE(id, G.nf) D[id] = ops::pprime_face(G, rho, d, id);
}

// p' RHS = -imbalance(F*), pinned reference row 0 (PressureCorrectionEquation.cpp:300-329).
__global__ void k_pprime_rhs(SGeo G, const double* F, int pin, int64_t ref, double* rhs) {
  GRID_STRIDE(c, G.nc) rhs[c] = ops::pprime_rhs(G, F, pin, ref, c);
}

// p += alpha_p p' (SIMPLE.cpp:937-943).
__global__ void k_pressure_update(int64_t n, double alpha, const double* pp, double* p) {
  GRID_STRIDE(c, n) p[c] = p[c] + (alpha * pp[c]);
}

// U = U* - d grad(p') (PressureCorrectionEquation.cpp:404-438).
__global__ void k_velocity_correct(int64_t n, const double* us, const double* d, const double* g,
                                   double* u) {
  GRID_STRIDE(c, n) u[c] = us[c] - (d[c] * g[c]);
}

// F = F* + D_f (p'_P - p'_N) (PressureCorrectionEquation.cpp:369-402).
__global__ void k_flux_correct(SGeo G, const double* Fs, const double* D, const double* pp,
                               double* F) {
  GRID_STRIDE(id, G.nf) F[id] = ops::flux_correct(G, Fs, D, pp, id);
}

// Per-block sums of imbalance^2 (continuity residual) and of the boundary
// fluxes (global net flux), plus a non-finite flag over cells.
__global__ void k_residual_sums(SGeo G, const double* F, double* partials) {
  __shared__ double sh[2][kBlock];
  double s2 = 0.0, sb = 0.0;
  GRID_STRIDE(c, G.nc) {
    const double imb = ops::cell_imbalance(G, F, c);
    s2 += imb * imb;
  }
  GRID_STRIDE(id, G.nf) {
    if (ops::boundary_face(G, id)) sb += F[id];
  }
  sh[0][threadIdx.x] = s2;
  sh[1][threadIdx.x] = sb;
  __syncthreads();
  for (int w = kBlock / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = sh[0][0];
    partials[2 * blockIdx.x + 1] = sh[1][0];
  }
}

__global__ void k_nonfinite(int64_t n, const double* v, unsigned* flag) {
  GRID_STRIDE(c, n) if (!isfinite(v[c])) atomicExch(flag, 1u);
}

}  // namespace

// ------------------------------------------------------------ launch wrappers
void launch_mass_flux(const SGeo& G, double rho, const double* const U[3], double* F, cudaStream_t s) {
  k_mass_flux<<<grid_for(G.nf), kBlock, 0, s>>>(G, rho, U[0], U[1], U[2], F);
}
void launch_scalar_face_values(const SGeo& G, const int* ptype, const double* pvalue,
                               const double* phi, double* fv, cudaStream_t s) {
  k_scalar_face_values<<<grid_for(G.nf), kBlock, 0, s>>>(G, ptype, pvalue, phi, fv);
}
void launch_gg_sweep(const SGeo& G, const double* phi, const double* fv, const double* const prev[3],
                     double* const out[3], cudaStream_t s) {
  k_gg_sweep<<<grid_for(G.nc), kBlock, 0, s>>>(G, phi, fv, prev ? prev[0] : nullptr,
                                               prev ? prev[1] : nullptr, prev ? prev[2] : nullptr,
                                               out[0], out[1], out[2]);
}
void launch_velocity_gradient(const SGeo& G, const double* uc, int comp, double* const g[3],
                              cudaStream_t s) {
  k_velocity_gradient<<<grid_for(G.nc), kBlock, 0, s>>>(G, uc, comp, g[0], g[1], g[2]);
}
void launch_assemble_momentum(const SGeo& G, double mu, int scheme, int comp, const double* uc,
                              const double* F, const double* gradPc, const double* const gu[3],
                              double alpha, double* diag, double* const off[6], double* rhs,
                              cudaStream_t s) {
  k_assemble_momentum<<<grid_for(G.nc), kBlock, 0, s>>>(
      G, mu, scheme, comp, uc, F, gradPc, gu ? gu[0] : nullptr, gu ? gu[1] : nullptr,
      gu ? gu[2] : nullptr, alpha, diag, off[0], off[1], off[2], off[3], off[4], off[5], rhs);
}
void launch_response(const SGeo& G, const double* diag, double* d, cudaStream_t s) {
  k_response<<<grid_for(G.nc), kBlock, 0, s>>>(G, diag, d);
}
void launch_rhie_chow(const SGeo& G, double rho, double alpha, const double* p,
                      const double* const gp[3], const double* const d[3], double* F,
                      cudaStream_t s) {
  k_rhie_chow<<<grid_for(G.nf), kBlock, 0, s>>>(G, rho, alpha, p, gp[0], gp[1], gp[2], d[0], d[1],
                                                d[2], F);
}
void launch_pprime_faces(const SGeo& G, double rho, const double* const d[3], double* D,
                         cudaStream_t s) {
  k_pprime_faces<<<grid_for(G.nf), kBlock, 0, s>>>(G, rho, d[0], d[1], d[2], D);
}
void launch_pprime_rhs(const SGeo& G, const double* F, int pin, int64_t ref, double* rhs,
                       cudaStream_t s) {
  k_pprime_rhs<<<grid_for(G.nc), kBlock, 0, s>>>(G, F, pin, ref, rhs);
}
void launch_pressure_update(int64_t n, double alpha, const double* pp, double* p, cudaStream_t s) {
  k_pressure_update<<<grid_for(n), kBlock, 0, s>>>(n, alpha, pp, p);
}
void launch_velocity_correct(int64_t n, const double* us, const double* d, const double* g,
                             double* u, cudaStream_t s) {
  k_velocity_correct<<<grid_for(n), kBlock, 0, s>>>(n, us, d, g, u);
}
void launch_flux_correct(const SGeo& G, const double* Fs, const double* D, const double* pp,
                         double* F, cudaStream_t s) {
  k_flux_correct<<<grid_for(G.nf), kBlock, 0, s>>>(G, Fs, D, pp, F);
}
int residual_sums_blocks(const SGeo& G) {
  int64_t g = (G.nc + kBlock - 1) / kBlock;
  if (g > 1024) g = 1024;
  return (int)(g < 1 ? 1 : g);
}
void launch_residual_sums(const SGeo& G, const double* F, double* partials, cudaStream_t s) {
  k_residual_sums<<<residual_sums_blocks(G), kBlock, 0, s>>>(G, F, partials);
}
void launch_nonfinite(int64_t n, const double* v, unsigned* flag, cudaStream_t s) {
  k_nonfinite<<<grid_for(n), kBlock, 0, s>>>(n, v, flag);
}

}  // namespace cfdb
