// Stage kernels of the resident SIMPLE loop on uniform Cartesian grids.
//
// Each kernel restates one reference function on the device, one thread per
// cell (or face), in the reference's operation order; this translation unit
// is compiled without FMA contraction (-fmad=false, as the reference's own
// device port was, cuda/CMakeLists.txt:61-77), so a stage reproduces the
// reference bit for bit given bit-identical inputs.  Citations name the
// reference function each kernel restates.
#include <cuda_runtime.h>

#include "simple_geo.cuh"
#include "simple_kernels.cuh"

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

// calculateMassFlux (physics/MassFlux.cpp:15-35): F = rho * (u_f . S_f).
__global__ void k_mass_flux(SGeo G, double rho, const double* u0, const double* u1,
                            const double* u2, double* F) {
  const double* U[3] = {u0, u1, u2};
  GRID_STRIDE(id, G.nf) {
    const FaceInfo fi = g_face_decode(G, id);
    const int a = fi.a;
    double ua, sa = G.area[a];
    if (fi.low >= 0 && fi.high >= 0) {
      ua = g_interp_v(G, a, fi.f, U[a][fi.low], U[a][fi.high]);
    } else if (fi.low < 0) {
      ua = g_vbc_value(G, 2 * a, a, U[a][fi.high]);
      sa = -sa;
    } else {
      ua = g_vbc_value(G, 2 * a + 1, a, U[a][fi.low]);
    }
    F[id] = rho * (ua * sa);
  }
}

// Scalar face values with pressure-type BCs (Interpolation.cpp interpolateFace).
__global__ void k_scalar_face_values(SGeo G, const int* ptype, const double* pvalue,
                                     const double* phi, double* fv) {
  GRID_STRIDE(id, G.nf) {
    const FaceInfo fi = g_face_decode(G, id);
    if (fi.low >= 0 && fi.high >= 0) {
      fv[id] = g_interp_s(G, fi.a, fi.f, phi[fi.low], phi[fi.high]);
    } else {
      const int side = fi.low < 0 ? 0 : 1;
      const int patch = 2 * fi.a + side;
      const int64_t owner = side == 0 ? fi.high : fi.low;
      fv[id] = (ptype[patch] == PBC_FIXED_VALUE) ? pvalue[patch]
                                                 : phi[owner] + (pvalue[patch] * g_dbnd(G, fi.a, side));
    }
  }
}

// One Green-Gauss sweep with boundary-consistent opposite-face values
// (Gradient.cpp:104-162 boundaryConsistentFaceValue, :431-482 greenGaussSweep).
__global__ void k_gg_sweep(SGeo G, const double* phi, const double* fv, const double* prev0,
                           const double* prev1, const double* prev2, double* g0, double* g1,
                           double* g2) {
  const double* prev[3] = {prev0, prev1, prev2};
  double* out[3] = {g0, g1, g2};
  GRID_STRIDE(c, G.nc) {
    int ijk[3];
    g_coords(G, c, ijk);
    double corr[3][2];
    int has[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    for (int a = 0; a < G.dim; ++a)
      for (int s = 0; s < 2; ++s) {
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G.n[a] - 1);
        const SideGeo& q = G.side[a][s];
        if (!boundary || !q.valid) continue;
        const int64_t bf = g_face_of(G, ijk, a, s);
        const int64_t of = g_face_of(G, ijk, a, 1 - s);
        const int64_t far = c + (s == 0 ? G.stride[a] : -G.stride[a]);
        const double gown = prev0 ? prev[a][c] : 0.0;
        const double phiB = fv[bf] + (gown * q.offset);
        const double phiP = phi[c], phiF = phi[far];
        const double sd = 2.0 * (((phiB - phiP) / q.tb) + ((phiF - phiP) / q.L)) / (q.tb + q.L);
        const double correction = -0.5 * q.w * (1.0 - q.w) * q.L * q.L * sd;
        corr[a][1 - s] = fv[of] + correction;
        has[a][1 - s] = 1;
      }
    const double inv = 1.0 / G.vol;
    for (int a = 0; a < G.dim; ++a) {
      double sum = 0.0;
      for (int s = 0; s < 2; ++s) {
        const int64_t f = g_face_of(G, ijk, a, s);
        const double val = has[a][s] ? corr[a][s] : fv[f];
        const double sf = (s == 0) ? -G.area[a] : G.area[a];
        sum += sf * val;
      }
      out[a][c] = sum * inv;
    }
  }
}

// Plain Green-Gauss gradient of a velocity component (VectorGradient.cpp:19-52).
__global__ void k_velocity_gradient(SGeo G, const double* uc, int comp, double* g0, double* g1,
                                    double* g2) {
  double* grad[3] = {g0, g1, g2};
  GRID_STRIDE(c, G.nc) {
    int ijk[3];
    g_coords(G, c, ijk);
    const double inv = 1.0 / G.vol;
    for (int a = 0; a < G.dim; ++a) {
      double sum = 0.0;
      for (int s = 0; s < 2; ++s) {
        double val;
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G.n[a] - 1);
        if (boundary) {
          val = g_vbc_value(G, 2 * a + s, comp, uc[c]);
        } else {
          const int64_t f = ijk[a] + s;
          const int64_t lo = s == 0 ? c - G.stride[a] : c;
          const int64_t hi = s == 0 ? c : c + G.stride[a];
          val = g_interp_v(G, a, f, uc[lo], uc[hi]);
        }
        const double sf = (s == 0) ? -G.area[a] : G.area[a];
        sum += sf * val;
      }
      grad[a][c] = sum * inv;
    }
  }
}

// quickFaceValue (discretization/Convection.cpp:104-119).
__device__ inline double quick_face(double phiC, double hCU, double phiU, double hUf, double phiD,
                                    double hfD) {
  const double wC = (-hUf * hfD) / (hCU * (hUf + hCU + hfD));
  const double wU = ((hUf + hCU) * hfD) / (hCU * (hUf + hfD));
  const double wD = (hUf * (hUf + hCU)) / ((hUf + hCU + hfD) * (hUf + hfD));
  return (wC * phiC) + (wU * phiU) + (wD * phiD);
}

// Deferred-correction increment phiFace - phiUpwind of an internal face
// (MomentumEquation.cpp:329-411: scheme value, van Leer TVD blend, clamp).
__device__ inline double deferred(const SGeo& G, int scheme, const double* uc, const double* gA,
                                  int a, int64_t f, int64_t lo, int64_t hi, double F) {
  const int ownerUpwind = F >= 0.0;
  const int64_t up = ownerUpwind ? lo : hi;
  const int64_t dn = ownerUpwind ? hi : lo;
  const double phiU = uc[up], phiD = uc[dn];
  const int64_t upCoord = ownerUpwind ? f - 1 : f;
  int64_t farC = -1;
  double hCU = 0.0;
  if (ownerUpwind && upCoord > 0) {
    farC = up - G.stride[a];
    hCU = g_dpn(G, a, upCoord);
  } else if (!ownerUpwind && upCoord < G.n[a] - 1) {
    farC = up + G.stride[a];
    hCU = g_dpn(G, a, upCoord + 1);
  }
  double phiHO = phiU;
  if (scheme == SCHEME_CENTRAL) {
    phiHO = g_interp_v(G, a, f, uc[lo], uc[hi]);
  } else if (scheme == SCHEME_LUD) {
    const double dx = g_node(G, a, f) - g_center(G, a, upCoord);
    phiHO = phiU + (gA[up] * dx);
  } else if (scheme == SCHEME_QUICK && farC >= 0) {
    const double hUf = fabs(g_node(G, a, f) - g_center(G, a, upCoord));
    const int64_t dnCoord = ownerUpwind ? f : f - 1;
    const double hfD = fabs(g_center(G, a, dnCoord) - g_node(G, a, f));
    phiHO = quick_face(uc[farC], hCU, phiU, hUf, phiD, hfD);
  }
  double psi = 0.0;
  if (farC >= 0) {
    const double lg = phiD - phiU;
    if (lg != 0.0) {
      const double r = (phiU - uc[farC]) / lg;
      if (r > 0.0) psi = (r + fabs(r)) / (1.0 + fabs(r));
    }
  }
  const double blended = phiU + (psi * (phiHO - phiU));
  const double lo_ = phiU < phiD ? phiU : phiD;
  const double hi_ = phiU < phiD ? phiD : phiU;
  const double phiFace = blended < lo_ ? lo_ : (hi_ < blended ? hi_ : blended);
  return phiFace - phiU;
}

// assembleRelaxedMomentumComponent (pressure_velocity/RelaxedMomentum.cpp:30-104):
// diffusion (MomentumEquation.cpp:167-262), convection (:264-413), pressure
// source (:415-430) and implicit under-relaxation (UnderRelaxation.cpp:13-36),
// gathered per row in the reference's triplet insertion order.
__global__ void k_assemble_momentum(SGeo G, double mu, int scheme, int comp, const double* uc,
                                    const double* F, const double* gradPc, const double* gu0,
                                    const double* gu1, const double* gu2, double alpha,
                                    double* diag, double* o0, double* o1, double* o2, double* o3,
                                    double* o4, double* o5, double* rhs) {
  const double* gradU[3] = {gu0, gu1, gu2};
  double* off[6] = {o0, o1, o2, o3, o4, o5};
  const double factor = (1.0 / alpha) - 1.0;
  GRID_STRIDE(c, G.nc) {
    int ijk[3];
    g_coords(G, c, ijk);
    double dg = 0.0, rh = 0.0;
    double o[6] = {0, 0, 0, 0, 0, 0};
    for (int a = 0; a < G.dim; ++a)
      for (int s = 0; s < 2; ++s) {
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G.n[a] - 1);
        if (boundary) {
          const int patch = 2 * a + s;
          const double phiB = g_vbc_value(G, patch, comp, uc[c]);
          const SideGeo& q = G.side[a][s];
          if (g_vbc_prescribed(G.vtype[patch]) && q.valid && q.stencil_ok) {
            const double ga = mu * G.area[a];
            const double cP = q.h2 / (q.h1 * (q.h2 - q.h1));
            const double cF = q.h1 / (q.h2 * (q.h2 - q.h1));
            const double cB = (1.0 / q.h1) + (1.0 / q.h2);
            const int64_t far = c + (s == 0 ? G.stride[a] : -G.stride[a]);
            const double gP = gradU[a] ? gradU[a][c] : 0.0;
            const double gF = gradU[a] ? gradU[a][far] : 0.0;
            rh += ga * ((cP * (gP * q.deltaP)) - (cF * (gF * q.deltaF)));
            dg += ga * cP;
            rh += (ga * cB) * phiB;
            o[2 * a + (1 - s)] += -(ga * cF);
          } else {
            const double coef = mu * G.area[a] / g_dbnd(G, a, s);
            dg += coef;
            rh += coef * phiB;
          }
        } else {
          const int64_t f = ijk[a] + s;
          const double muf = g_interp_s(G, a, f, mu, mu);
          const double D = muf * G.area[a] / g_dpn(G, a, f);
          dg += D;
          o[2 * a + s] += -D;
        }
      }
    for (int a = 0; a < G.dim; ++a)
      for (int s = 0; s < 2; ++s) {
        const double Ff = F[g_face_of(G, ijk, a, s)];
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G.n[a] - 1);
        if (boundary) {
          if (Ff >= 0.0) dg += Ff;
          else rh -= Ff * g_vbc_value(G, 2 * a + s, comp, uc[c]);
          continue;
        }
        const int owner = (s == 1);
        if (owner) {
          if (Ff >= 0.0) dg += Ff;
          else o[2 * a + 1] += Ff;
        } else {
          if (Ff >= 0.0) o[2 * a] += -Ff;
          else dg += -Ff;
        }
        if (scheme != SCHEME_UPWIND) {
          const int64_t f = ijk[a] + s;
          const int64_t lo = s == 0 ? c - G.stride[a] : c;
          const int64_t hi = s == 0 ? c : c + G.stride[a];
          const double corr = Ff * deferred(G, scheme, uc, gradU[a], a, f, lo, hi, Ff);
          if (owner) rh -= corr;
          else rh += corr;
        }
      }
    rh += -G.vol * gradPc[c];
    if (alpha != 1.0) {
      const double extra = dg * factor;
      dg += extra;
      rh += extra * uc[c];
    }
    diag[c] = dg;
    rhs[c] = rh;
    for (int q = 0; q < 6; ++q) off[q][c] = o[q];
  }
}

// d = V / aP (PressureCorrectionEquation.cpp:103-114).
__global__ void k_response(SGeo G, const double* diag, double* d) {
  GRID_STRIDE(c, G.nc) d[c] = G.vol / diag[c];
}

__device__ inline double pface_internal(const SGeo& G, double rho, int a, int64_t f, double dP,
                                        double dN) {
  const double dFace = g_interp_s(G, a, f, dP, dN);
  return rho * G.area[a] * dFace / g_dpn(G, a, f);
}

// Rhie-Chow correction of the internal faces (RhieChow.cpp:17-51).
__global__ void k_rhie_chow(SGeo G, double rho, double alpha, const double* p, const double* gp0,
                            const double* gp1, const double* gp2, const double* d0,
                            const double* d1, const double* d2, double* F) {
  const double* gp[3] = {gp0, gp1, gp2};
  const double* d[3] = {d0, d1, d2};
  GRID_STRIDE(id, G.nf) {
    const FaceInfo fi = g_face_decode(G, id);
    if (fi.low < 0 || fi.high < 0) continue;
    const int a = fi.a;
    const double coupling = pface_internal(G, rho, a, fi.f, d[a][fi.low], d[a][fi.high]);
    const double dvec = g_center(G, a, fi.f) - g_center(G, a, fi.f - 1);
    const double gf = g_interp_v(G, a, fi.f, gp[a][fi.low], gp[a][fi.high]);
    const double cmi = (p[fi.high] - p[fi.low]) - (gf * dvec);
    F[id] += -(coupling / alpha) * cmi;
  }
}

// p' face coefficients (pressureCorrectionFaceCoupling, PressureCorrectionEquation.cpp:146-179).
__global__ void k_pprime_faces(SGeo G, double rho, const double* d0, const double* d1,
                               const double* d2, double* D) {
  const double* d[3] = {d0, d1, d2};
  GRID_STRIDE(id, G.nf) {
    const FaceInfo fi = g_face_decode(G, id);
    if (fi.low >= 0 && fi.high >= 0) {
      D[id] = pface_internal(G, rho, fi.a, fi.f, d[fi.a][fi.low], d[fi.a][fi.high]);
    } else {
      const int side = fi.low < 0 ? 0 : 1;
      const int64_t owner = side == 0 ? fi.high : fi.low;
      D[id] = (G.ptype[2 * fi.a + side] == PBC_FIXED_VALUE)
                  ? rho * G.area[fi.a] * d[fi.a][owner] / g_dbnd(G, fi.a, side)
                  : 0.0;
    }
  }
}

// Cell imbalance sum_f s_f F_f in cell face order (ContinuityEquation.cpp:14-28).
__device__ inline double cell_imbalance(const SGeo& G, const double* F, int64_t c) {
  int ijk[3];
  g_coords(G, c, ijk);
  double sum = 0.0;
  for (int a = 0; a < G.dim; ++a) {
    const int64_t lo = g_face_of(G, ijk, a, 0), hi = g_face_of(G, ijk, a, 1);
    sum += (ijk[a] == 0) ? F[lo] : -F[lo];
    sum += F[hi];
  }
  return sum;
}

// p' RHS = -imbalance(F*), pinned reference row 0 (PressureCorrectionEquation.cpp:300-329).
__global__ void k_pprime_rhs(SGeo G, const double* F, int pin, int64_t ref, double* rhs) {
  GRID_STRIDE(c, G.nc) rhs[c] = (pin && c == ref) ? 0.0 : -cell_imbalance(G, F, c);
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
  GRID_STRIDE(id, G.nf) {
    const FaceInfo fi = g_face_decode(G, id);
    const double pO = (fi.low >= 0) ? pp[fi.low] : pp[fi.high];
    const double pN = (fi.low >= 0 && fi.high >= 0) ? pp[fi.high] : 0.0;
    F[id] = Fs[id] + D[id] * (pO - pN);
  }
}

// Per-block sums of imbalance^2 (continuity residual) and of the boundary
// fluxes (global net flux), plus a non-finite flag over cells.
__global__ void k_residual_sums(SGeo G, const double* F, double* partials) {
  __shared__ double sh[2][kBlock];
  double s2 = 0.0, sb = 0.0;
  GRID_STRIDE(c, G.nc) {
    const double imb = cell_imbalance(G, F, c);
    s2 += imb * imb;
  }
  GRID_STRIDE(id, G.nf) {
    const FaceInfo fi = g_face_decode(G, id);
    if (fi.low < 0 || fi.high < 0) sb += F[id];
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
