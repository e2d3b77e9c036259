// Per-cell and per-face operations of the SIMPLE stages on Cartesian grids
// (uniform or rectilinear), shared by the single-case kernels (simple_kernels.cu) and the batched
// persistent kernels (batch_stages.cu), so that a stage computes the same
// value for a cell whichever of them runs it.
//
// Each function restates one reference function for one cell (or face), in
// the reference's operation order.  Every translation unit that includes this
// header must be compiled without FMA contraction (-fmad=false, as the
// reference's own device port was, cuda/CMakeLists.txt:61-77): the stages
// then reproduce the reference bit for bit given bit-identical inputs.
#pragma once

#include <cuda_runtime.h>

#include "simple_geo.cuh"

namespace cfdb {
namespace ops {

// calculateMassFlux (physics/MassFlux.cpp:15-35): F = rho * (u_f . S_f).
__device__ inline double mass_flux(const SGeo& G, double rho, const double* const U[3], int64_t id) {
  const FaceInfo fi = g_face_decode(G, id);
  const int a = fi.a;
  double ua, sa = g_face_area(G, fi);
  if (fi.low >= 0 && fi.high >= 0) {
    ua = g_interp_v(G, a, fi.f, U[a][fi.low], U[a][fi.high]);
  } else if (fi.low < 0) {
    ua = g_vbc_value(G, 2 * a, a, U[a][fi.high]);
    sa = -sa;
  } else {
    ua = g_vbc_value(G, 2 * a + 1, a, U[a][fi.low]);
  }
  return rho * (ua * sa);
}

// Scalar face value with pressure-type BCs (Interpolation.cpp interpolateFace).
__device__ inline double scalar_face_value(const SGeo& G, const int* ptype, const double* pvalue,
                                           const double* phi, int64_t id) {
  const FaceInfo fi = g_face_decode(G, id);
  if (fi.low >= 0 && fi.high >= 0) return g_interp_s(G, fi.a, fi.f, phi[fi.low], phi[fi.high]);
  const int side = fi.low < 0 ? 0 : 1;
  const int patch = 2 * fi.a + side;
  const int64_t owner = side == 0 ? fi.high : fi.low;
  return (ptype[patch] == PBC_FIXED_VALUE) ? pvalue[patch]
                                           : phi[owner] + (pvalue[patch] * g_dbnd(G, fi.a, side));
}

// One Green-Gauss sweep with boundary-consistent opposite-face values
// (Gradient.cpp:104-162 boundaryConsistentFaceValue, :431-482 greenGaussSweep).
// prev[0] == nullptr: the first sweep (no owner gradient yet).
__device__ inline void gg_sweep(const SGeo& G, const double* phi, const double* fv,
                                const double* const prev[3], double* const out[3], int64_t c) {
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
      const double gown = prev[0] ? prev[a][c] : 0.0;
      const double phiB = fv[bf] + (gown * q.offset);
      const double phiP = phi[c], phiF = phi[far];
      const double sd = 2.0 * (((phiB - phiP) / q.tb) + ((phiF - phiP) / q.L)) / (q.tb + q.L);
      const double correction = -0.5 * q.w * (1.0 - q.w) * q.L * q.L * sd;
      corr[a][1 - s] = fv[of] + correction;
      has[a][1 - s] = 1;
    }
  const double inv = 1.0 / g_vol(G, ijk);
  for (int a = 0; a < G.dim; ++a) {
    double sum = 0.0;
    for (int s = 0; s < 2; ++s) {
      const int64_t f = g_face_of(G, ijk, a, s);
      const double val = has[a][s] ? corr[a][s] : fv[f];
      const double sf = (s == 0) ? -g_area(G, a, ijk) : g_area(G, a, ijk);
      sum += sf * val;
    }
    out[a][c] = sum * inv;
  }
}

// Plain Green-Gauss gradient of a velocity component (VectorGradient.cpp:19-52).
__device__ inline void velocity_gradient(const SGeo& G, const double* uc, int comp,
                                         double* const grad[3], int64_t c) {
  int ijk[3];
  g_coords(G, c, ijk);
  const double inv = 1.0 / g_vol(G, ijk);
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
      const double sf = (s == 0) ? -g_area(G, a, ijk) : g_area(G, a, ijk);
      sum += sf * val;
    }
    grad[a][c] = sum * inv;
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

// One row of assembleRelaxedMomentumComponent (pressure_velocity/RelaxedMomentum.cpp:30-104):
// diffusion (MomentumEquation.cpp:167-262), convection (:264-413), pressure
// source (:415-430) and implicit under-relaxation (UnderRelaxation.cpp:13-36),
// gathered in the reference's triplet insertion order.  gradU[a] may be null.
__device__ inline void assemble_momentum(const SGeo& G, double mu, int scheme, int comp,
                                         const double* uc, const double* F, const double* gradPc,
                                         const double* const gradU[3], double alpha, double* diag,
                                         double* const off[6], double* rhs, int64_t c) {
  const double factor = (1.0 / alpha) - 1.0;
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
          const double ga = mu * g_area(G, a, ijk);
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
          const double coef = mu * g_area(G, a, ijk) / g_dbnd(G, a, s);
          dg += coef;
          rh += coef * phiB;
        }
      } else {
        const int64_t f = ijk[a] + s;
        const double muf = g_interp_s(G, a, f, mu, mu);
        const double D = muf * g_area(G, a, ijk) / g_dpn(G, a, f);
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
  rh += -g_vol(G, ijk) * gradPc[c];
  if (alpha != 1.0) {
    const double extra = dg * factor;
    dg += extra;
    rh += extra * uc[c];
  }
  diag[c] = dg;
  rhs[c] = rh;
  for (int q = 0; q < 6; ++q) off[q][c] = o[q];
}

// d = V / aP (PressureCorrectionEquation.cpp:103-114).
__device__ inline double response(const SGeo& G, double aP, int64_t c) {
  return g_vol_c(G, c) / aP;
}

__device__ inline double pface_internal(const SGeo& G, double rho, const FaceInfo& fi, double dP,
                                        double dN) {
  const double dFace = g_interp_s(G, fi.a, fi.f, dP, dN);
  return rho * g_face_area(G, fi) * dFace / g_dpn(G, fi.a, fi.f);
}

// Rhie-Chow correction of one internal face (RhieChow.cpp:17-51); boundary
// faces are left alone.
__device__ inline void rhie_chow(const SGeo& G, double rho, double alpha, const double* p,
                                 const double* const gp[3], const double* const d[3], double* F,
                                 int64_t id) {
  const FaceInfo fi = g_face_decode(G, id);
  if (fi.low < 0 || fi.high < 0) return;
  const int a = fi.a;
  const double coupling = pface_internal(G, rho, fi, d[a][fi.low], d[a][fi.high]);
  const double dvec = g_center(G, a, fi.f) - g_center(G, a, fi.f - 1);
  const double gf = g_interp_v(G, a, fi.f, gp[a][fi.low], gp[a][fi.high]);
  const double cmi = (p[fi.high] - p[fi.low]) - (gf * dvec);
  F[id] += -(coupling / alpha) * cmi;
}

// p' face coefficient (pressureCorrectionFaceCoupling, PressureCorrectionEquation.cpp:146-179).
__device__ inline double pprime_face(const SGeo& G, double rho, const double* const d[3], int64_t id) {
  const FaceInfo fi = g_face_decode(G, id);
  if (fi.low >= 0 && fi.high >= 0) return pface_internal(G, rho, fi, d[fi.a][fi.low], d[fi.a][fi.high]);
  const int side = fi.low < 0 ? 0 : 1;
  const int64_t owner = side == 0 ? fi.high : fi.low;
  return (G.ptype[2 * fi.a + side] == PBC_FIXED_VALUE)
             ? rho * g_face_area(G, fi) * d[fi.a][owner] / g_dbnd(G, fi.a, side)
             : 0.0;
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
__device__ inline double pprime_rhs(const SGeo& G, const double* F, int pin, int64_t ref, int64_t c) {
  return (pin && c == ref) ? 0.0 : -cell_imbalance(G, F, c);
}

// F = F* + D_f (p'_P - p'_N) (PressureCorrectionEquation.cpp:369-402).
__device__ inline double flux_correct(const SGeo& G, const double* Fs, const double* D,
                                      const double* pp, int64_t id) {
  const FaceInfo fi = g_face_decode(G, id);
  const double pO = (fi.low >= 0) ? pp[fi.low] : pp[fi.high];
  const double pN = (fi.low >= 0 && fi.high >= 0) ? pp[fi.high] : 0.0;
  return Fs[id] + D[id] * (pO - pN);
}

// One row of the p' matrix in stencil form from its face coefficients
// (assembleGeometricPressureCorrection, PressureCorrectionEquation.cpp:181-339):
// diagonal = sum of the row's face coefficients, off-diagonal = -D_f on
// interior faces, and the identity row at the pinned reference cell.
__device__ inline void pprime_row(const SGeo& G, const double* D, int pin, int64_t ref, double* diag,
                                  double* const off[6], int64_t c) {
  int ijk[3];
  g_coords(G, c, ijk);
  for (int q = 0; q < 6; ++q) off[q][c] = 0.0;
  if (pin && c == ref) {
    diag[c] = 1.0;
    return;
  }
  double dg = 0.0;
  for (int a = 0; a < G.dim; ++a)
    for (int s = 0; s < 2; ++s) {
      const double Df = D[g_face_of(G, ijk, a, s)];
      const bool boundary = s == 0 ? ijk[a] == 0 : ijk[a] == G.n[a] - 1;
      dg += Df;
      if (!boundary) off[2 * a + s][c] = -Df;
    }
  diag[c] = dg;
}

// Boundary face (owner on one side only): its flux enters the global net flux.
__device__ inline bool boundary_face(const SGeo& G, int64_t id) {
  const FaceInfo fi = g_face_decode(G, id);
  return fi.low < 0 || fi.high < 0;
}

}  // namespace ops
}  // namespace cfdb
