/* CPU restatement of the reference's SIMPLE pressure-velocity path on uniform
 * Cartesian grids.  TEST INFRASTRUCTURE ONLY (the checker, never the product):
 * see cfdb_oracle.h for the layout and the pinning tests.
 *
 * Parity is pinned: tests/test_oracle_pin.py runs the reference compiled from
 * its own sources (oracle/_ref) beside this file and requires bit-identical
 * p' solves and SIMPLE fields; tests/golden/ holds fixtures generated the same
 * way (tests/golden/make_golden.py) for hosts without the reference build.
 *
 * Geometry is evaluated with the reference's own expressions (MeshGrading.cpp
 * AxisSpacing::uniform/center/node/width, MeshGeometry.cpp:513-552,1047-1140),
 * including the few places where rounding makes a "unit" normal or a
 * boundary offset differ from the ideal value by an ulp.
 */
#include "cfdb_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "synth_rhs.h"

/* ------------------------------------------------------------------ geometry */

typedef struct {
  int dim;
  int64_t n[3];
  int64_t stride[3];
  double delta[3];
  double area[3]; /* area of a face normal to axis a */
  double vol;
  int64_t nc, nf;
  int64_t foff[3];
} geo;

static void geo_init(geo* G, const og_grid* g) {
  memset(G, 0, sizeof(*G));
  G->dim = g->dim;
  for (int a = 0; a < 3; ++a) G->n[a] = (a < g->dim) ? g->n[a] : 1;
  G->stride[0] = 1;
  G->stride[1] = G->n[0];
  G->stride[2] = G->n[0] * G->n[1];
  for (int a = 0; a < g->dim; ++a) G->delta[a] = g->len[a] / (double)g->n[a];
  if (g->dim == 2) {
    G->area[0] = G->delta[1];
    G->area[1] = G->delta[0];
    G->vol = G->delta[0] * G->delta[1];
  } else {
    G->area[0] = G->delta[1] * G->delta[2];
    G->area[1] = G->delta[0] * G->delta[2];
    G->area[2] = G->delta[0] * G->delta[1];
    G->vol = (G->delta[0] * G->delta[1]) * G->delta[2];
  }
  G->nc = G->n[0] * G->n[1] * G->n[2];
  const int64_t nfx = (G->n[0] + 1) * G->n[1] * G->n[2];
  const int64_t nfy = G->n[0] * (G->n[1] + 1) * G->n[2];
  const int64_t nfz = (g->dim == 3) ? G->n[0] * G->n[1] * (G->n[2] + 1) : 0;
  G->foff[0] = 0;
  G->foff[1] = nfx;
  G->foff[2] = nfx + nfy;
  G->nf = nfx + nfy + nfz;
}

static inline double center(const geo* G, int a, int64_t i) { return ((double)i + 0.5) * G->delta[a]; }
static inline double node(const geo* G, int a, int64_t i) { return (double)i * G->delta[a]; }

static inline void cell_coords(const geo* G, int64_t c, int64_t ijk[3]) {
  ijk[0] = c % G->n[0];
  ijk[1] = (c / G->n[0]) % G->n[1];
  ijk[2] = c / (G->n[0] * G->n[1]);
}

/* Global id of the face of cell ijk on axis a, side s (0 low, 1 high). */
static inline int64_t face_of(const geo* G, const int64_t ijk[3], int a, int s) {
  const int64_t i = ijk[0] + (a == 0 ? s : 0);
  const int64_t j = ijk[1] + (a == 1 ? s : 0);
  const int64_t k = ijk[2] + (a == 2 ? s : 0);
  if (a == 0) return i + (G->n[0] + 1) * (j + G->n[1] * k);
  if (a == 1) return G->foff[1] + i + G->n[0] * (j + (G->n[1] + 1) * k);
  return G->foff[2] + i + G->n[0] * (j + G->n[1] * k);
}

/* Decode a global face id into axis, face coordinate along that axis, and the
 * low/high cells (-1 when outside the domain). */
typedef struct {
  int a;
  int64_t f;       /* face coordinate along axis a, 0..n_a */
  int64_t low;     /* cell on the low side (owner of an internal face) */
  int64_t high;    /* cell on the high side (neighbour of an internal face) */
} face_info;

static face_info face_decode(const geo* G, int64_t id) {
  face_info fi;
  int64_t i, j, k;
  if (id < G->foff[1]) {
    fi.a = 0;
    i = id % (G->n[0] + 1);
    j = (id / (G->n[0] + 1)) % G->n[1];
    k = id / ((G->n[0] + 1) * G->n[1]);
    fi.f = i;
  } else if (G->dim == 2 || id < G->foff[2]) {
    const int64_t r = id - G->foff[1];
    fi.a = 1;
    i = r % G->n[0];
    j = (r / G->n[0]) % (G->n[1] + 1);
    k = r / (G->n[0] * (G->n[1] + 1));
    fi.f = j;
  } else {
    const int64_t r = id - G->foff[2];
    fi.a = 2;
    i = r % G->n[0];
    j = (r / G->n[0]) % G->n[1];
    k = r / (G->n[0] * G->n[1]);
    fi.f = k;
  }
  int64_t c[3] = {i, j, k};
  c[fi.a] = fi.f;
  const int64_t base = c[0] + G->n[0] * (c[1] + G->n[1] * c[2]);
  fi.high = (fi.f < G->n[fi.a]) ? base : -1;
  fi.low = (fi.f > 0) ? base - G->stride[fi.a] : -1;
  return fi;
}

/* Distances of an internal face at coordinate f along axis a (owner f-1,
 * neighbour f): MeshGeometry::distance = magnitude, exact |x| for a vector
 * with a single non-zero component. */
static inline double d_pf(const geo* G, int a, int64_t f) { return fabs(node(G, a, f) - center(G, a, f - 1)); }
static inline double d_nf(const geo* G, int a, int64_t f) { return fabs(node(G, a, f) - center(G, a, f)); }
static inline double d_pn(const geo* G, int a, int64_t f) { return fabs(center(G, a, f) - center(G, a, f - 1)); }
/* Owner-to-face distance of a boundary face (side s of axis a). */
static inline double d_bnd(const geo* G, int a, int s) {
  return s == 0 ? fabs(node(G, a, 0) - center(G, a, 0))
                : fabs(node(G, a, G->n[a]) - center(G, a, G->n[a] - 1));
}

/* interpolateInternalFace, scalar form (Interpolation.cpp:21-30). */
static inline double interp_s(const geo* G, int a, int64_t f, double phiP, double phiN) {
  const double dPf = d_pf(G, a, f), dNf = d_nf(G, a, f);
  return ((dNf * phiP) + (dPf * phiN)) / (dPf + dNf);
}
/* interpolateInternalFace, vector form, one component (Interpolation.cpp:32-41). */
static inline double interp_v(const geo* G, int a, int64_t f, double uP, double uN) {
  const double dPf = d_pf(G, a, f), dNf = d_nf(G, a, f);
  return ((uP * dNf) + (uN * dPf)) * (1.0 / (dPf + dNf));
}

/* ---------------------------------------------------- boundary-side geometry */

/* Per (axis, side) quantities of the boundary-consistent gradient
 * (Gradient.cpp:104-162) and the wall three-point stencil
 * (MeshGeometry.cpp:253-284, NonOrthogonalDiffusion.cpp:64-103). */
typedef struct {
  int valid;        /* an opposite interior face exists (n_a >= 2) */
  double L;         /* |x_F - x_P| */
  double w;         /* crossing weight of the opposite face */
  double tb;        /* back distance from P to the boundary along the fit line */
  double offset;    /* (B' - face centroid) along the axis: 0 unless rounding */
  double h1, h2;    /* normal distances face->P, face->F */
  double deltaP, deltaF; /* tangential transfers of the wall stencil (0 unless rounding) */
  int stencil_ok;
} side_geo;

static side_geo side_geometry(const geo* G, int a, int s) {
  side_geo sg;
  memset(&sg, 0, sizeof(sg));
  const int64_t n = G->n[a];
  if (n < 2) return sg;
  sg.valid = 1;
  const int64_t ip = (s == 0) ? 0 : n - 1;
  const int64_t iF = (s == 0) ? 1 : n - 2;
  const double xb = (s == 0) ? node(G, a, 0) : node(G, a, n);
  const double sfa = (s == 0) ? -G->area[a] : G->area[a];
  const double cP = center(G, a, ip), cF = center(G, a, iF);
  /* d = x_F - x_P, L = |d|, inward = d * (1/L) */
  const double d = cF - cP;
  sg.L = fabs(d);
  const double inward = d * (1.0 / sg.L);
  /* crossing of the opposite face: owner = low cell fo-1, neighbour = fo */
  const int64_t fo = (s == 0) ? 1 : n - 1;
  const double toFace = node(G, a, fo) - center(G, a, fo - 1);
  const double dd = center(G, a, fo) - center(G, a, fo - 1);
  sg.w = (toFace * dd) / (dd * dd);
  /* boundaryLineIntersection (MeshGeometry.cpp:229-251) */
  sg.tb = ((cP - xb) * sfa) / (inward * sfa);
  const double point = cP - (inward * sg.tb);
  sg.offset = point - xb;
  /* boundaryInwardStencil: unit normal = S * (1/area) */
  const double normal = sfa * (1.0 / G->area[a]);
  sg.h1 = (xb - cP) * normal;
  sg.h2 = (xb - cF) * normal;
  sg.stencil_ok = (sg.h1 > 0.0) && (sg.h2 > sg.h1);
  sg.deltaP = cP - (xb - (normal * sg.h1));
  sg.deltaF = cF - (xb - (normal * sg.h2));
  return sg;
}

int64_t og_cells(const og_grid* g) {
  geo G;
  geo_init(&G, g);
  return G.nc;
}
int64_t og_faces(const og_grid* g) {
  geo G;
  geo_init(&G, g);
  return G.nf;
}

int og_synth_rhs(int64_t nx, int64_t ny, int64_t nz, uint64_t seed, double* b) {
  return oracle_synth_rhs(nx, ny, nz, seed, b);
}

/* ----------------------------------------------------------- linear algebra */

void og_stencil_apply(const og_grid* g, const double* diag, const double* const off[6],
                      const double* x, double* y) {
  geo G;
  geo_init(&G, g);
  for (int64_t c = 0; c < G.nc; ++c) {
    int64_t ijk[3];
    cell_coords(&G, c, ijk);
    double sum = 0.0;
    /* ascending column order: z-low, y-low, x-low, P, x-high, y-high, z-high */
    for (int a = G.dim - 1; a >= 0; --a)
      if (ijk[a] > 0) sum += off[2 * a][c] * x[c - G.stride[a]];
    sum += diag[c] * x[c];
    for (int a = 0; a < G.dim; ++a)
      if (ijk[a] < G.n[a] - 1) sum += off[2 * a + 1][c] * x[c + G.stride[a]];
    y[c] = sum;
  }
}

static double vdot(const double* a, const double* b, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
static double vnorm(const double* a, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * a[i];
  return sqrt(s);
}
static int vfinite(const double* a, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    if (!isfinite(a[i])) return 0;
  return 1;
}

/* BiCGSTAB.cpp:34-41 */
static int cancelled(double ip, const double* x, const double* y, int64_t n, double nx, double ny) {
  const double eps = DBL_EPSILON;
  if (fabs(ip) > eps * nx * ny) return 0;
  double t = 0.0;
  for (int64_t i = 0; i < n; ++i) t += fabs(x[i] * y[i]);
  return fabs(ip) <= eps * t;
}

static void hist_push(double* hist, int64_t cap, int64_t* count, double v) {
  if (hist && *count < cap) hist[*count] = v;
  ++*count;
}

/* Matrix-level finiteness of a stencil matrix (SparseMatrix::allFinite): only
 * entries that exist inside the domain count. */
static int stencil_finite(const geo* G, const double* diag, const double* const off[6]) {
  for (int64_t c = 0; c < G->nc; ++c) {
    if (!isfinite(diag[c])) return 0;
    int64_t ijk[3];
    cell_coords(G, c, ijk);
    for (int a = 0; a < G->dim; ++a) {
      if (ijk[a] > 0 && !isfinite(off[2 * a][c])) return 0;
      if (ijk[a] < G->n[a] - 1 && !isfinite(off[2 * a + 1][c])) return 0;
    }
  }
  return 1;
}

static int solve_cg(const og_grid* g, const geo* G, const og_linear_settings* s,
                    const double* inv, const double* diag, const double* const off[6],
                    const double* b, double* x, double* hist, int64_t cap, og_linear_result* out,
                    double* work) {
  const int64_t n = G->nc;
  double *r = work, *z = work + n, *p = work + 2 * n, *Ap = work + 3 * n;
  int64_t hc = 0;
  og_stencil_apply(g, diag, off, x, Ap);
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - Ap[i];
  const double b0 = vnorm(r, n);
  out->initial_residual = b0;
  hist_push(hist, cap, &hc, b0);
#define CONV(res) (((res) <= s->abs_tol) || ((b0 > 0.0) && ((res) / b0 <= s->rel_tol)))
  if (b0 == 0.0 || CONV(b0)) {
    out->status = OG_CONVERGED;
    out->iterations = 0;
    out->final_residual = b0;
    return 0;
  }
  for (int64_t i = 0; i < n; ++i) z[i] = inv ? inv[i] * r[i] : r[i];
  memcpy(p, z, sizeof(double) * n);
  double rz = vdot(r, z, n);
  if (!isfinite(rz)) {
    out->status = OG_BREAKDOWN;
    out->final_residual = b0;
    return 0;
  }
  double last = b0;
  for (int64_t iter = 1; iter <= s->max_iterations; ++iter) {
    og_stencil_apply(g, diag, off, p, Ap);
    const double pAp = vdot(p, Ap, n);
    if (!isfinite(pAp) || fabs(pAp) < 1.0e-30) {
      out->status = OG_BREAKDOWN;
      out->final_residual = vnorm(r, n);
      out->iterations = iter - 1;
      return 0;
    }
    const double alpha = rz / pAp;
    if (!isfinite(alpha)) {
      out->status = OG_BREAKDOWN;
      out->final_residual = vnorm(r, n);
      out->iterations = iter - 1;
      return 0;
    }
    for (int64_t i = 0; i < n; ++i) x[i] = x[i] + p[i] * alpha;
    for (int64_t i = 0; i < n; ++i) r[i] = r[i] - Ap[i] * alpha;
    const double res = vnorm(r, n);
    if (!isfinite(res)) {
      out->status = OG_NONFINITE_RESIDUAL;
      out->final_residual = res;
      out->iterations = iter;
      hist_push(hist, cap, &hc, res);
      return 0;
    }
    hist_push(hist, cap, &hc, res);
    out->iterations = iter;
    last = res;
    if (CONV(res)) {
      out->status = OG_CONVERGED;
      out->final_residual = res;
      return 0;
    }
    for (int64_t i = 0; i < n; ++i) z[i] = inv ? inv[i] * r[i] : r[i];
    const double rzNew = vdot(r, z, n);
    if (!isfinite(rzNew)) {
      out->status = OG_BREAKDOWN;
      out->final_residual = res;
      return 0;
    }
    const double beta = rzNew / rz;
    if (!isfinite(beta)) {
      out->status = OG_BREAKDOWN;
      out->final_residual = res;
      return 0;
    }
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + p[i] * beta;
    rz = rzNew;
  }
  out->status = OG_MAX_ITERATIONS;
  out->final_residual = last;
  return 0;
#undef CONV
}

static int solve_bicgstab(const og_grid* g, const geo* G, const og_linear_settings* s,
                          const double* inv, const double* diag, const double* const off[6],
                          const double* b, double* x, double* hist, int64_t cap,
                          og_linear_result* out, double* work) {
  const int64_t n = G->nc;
  double *r = work, *rHat = work + n, *v = work + 2 * n, *p = work + 3 * n;
  double *pHat = work + 4 * n, *sv = work + 5 * n, *sHat = work + 6 * n, *t = work + 7 * n;
  int64_t hc = 0;
  og_stencil_apply(g, diag, off, x, t);
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - t[i];
  memcpy(rHat, r, sizeof(double) * n);
  const double b0 = vnorm(r, n);
  out->initial_residual = b0;
  out->restarts = 0;
  hist_push(hist, cap, &hc, b0);
#define CONV(res) (((res) <= s->abs_tol) || ((b0 > 0.0) && ((res) / b0 <= s->rel_tol)))
  if (b0 == 0.0 || CONV(b0)) {
    out->status = OG_CONVERGED;
    out->iterations = 0;
    out->final_residual = b0;
    return 0;
  }
  double rhoOld = 1.0, alpha = 1.0, omega = 1.0;
  for (int64_t i = 0; i < n; ++i) v[i] = 0.0, p[i] = 0.0;
  int64_t completed = 0;
  double rHatNorm = b0, rNorm = b0, restartResidual = b0;
  double lastHist = b0;

#define BREAKDOWN()                         \
  do {                                      \
    out->status = OG_BREAKDOWN;             \
    out->final_residual = vnorm(r, n);      \
    out->iterations = completed;            \
    return 0;                               \
  } while (0)
  /* restart(): 0 restarted, 1 converged, 2 stop (BiCGSTAB.cpp:127-151) */
#define RESTART(outcome)                                              \
  do {                                                                \
    if (!(rNorm < restartResidual)) {                                 \
      outcome = 2;                                                    \
      break;                                                          \
    }                                                                 \
    og_stencil_apply(g, diag, off, x, t);                             \
    for (int64_t i_ = 0; i_ < n; ++i_) r[i_] = b[i_] - t[i_];         \
    rNorm = vnorm(r, n);                                              \
    if (!isfinite(rNorm)) {                                           \
      outcome = 2;                                                    \
      break;                                                          \
    }                                                                 \
    if (CONV(rNorm)) {                                                \
      outcome = 1;                                                    \
      break;                                                          \
    }                                                                 \
    memcpy(rHat, r, sizeof(double) * n);                              \
    rHatNorm = rNorm;                                                 \
    restartResidual = rNorm;                                          \
    rhoOld = 1.0;                                                     \
    alpha = 1.0;                                                      \
    omega = 1.0;                                                      \
    for (int64_t i_ = 0; i_ < n; ++i_) v[i_] = 0.0, p[i_] = 0.0;      \
    ++out->restarts;                                                  \
    outcome = 0;                                                      \
  } while (0)
#define HANDLE_RESTART()                       \
  {                                            \
    int oc_ = 2;                               \
    RESTART(oc_);                              \
    if (oc_ == 0) continue;                    \
    if (oc_ == 1) {                            \
      out->status = OG_CONVERGED;              \
      out->final_residual = rNorm;             \
      out->iterations = completed;             \
      return 0;                                \
    }                                          \
    BREAKDOWN();                               \
  }

  while (completed < s->max_iterations) {
    const int64_t iter = completed + 1;
    const double rho = vdot(rHat, r, n);
    if (!isfinite(rho)) BREAKDOWN();
    if (cancelled(rho, rHat, r, n, rHatNorm, rNorm)) HANDLE_RESTART();
    const double beta = (rho / rhoOld) * (alpha / omega);
    if (!isfinite(beta)) BREAKDOWN();
    for (int64_t i = 0; i < n; ++i) p[i] = r[i] + (p[i] - v[i] * omega) * beta;
    for (int64_t i = 0; i < n; ++i) pHat[i] = inv ? inv[i] * p[i] : p[i];
    og_stencil_apply(g, diag, off, pHat, v);
    const double rHatDotV = vdot(rHat, v, n);
    if (!isfinite(rHatDotV)) BREAKDOWN();
    if (cancelled(rHatDotV, rHat, v, n, rHatNorm, vnorm(v, n))) HANDLE_RESTART();
    alpha = rho / rHatDotV;
    if (!isfinite(alpha)) BREAKDOWN();
    for (int64_t i = 0; i < n; ++i) sv[i] = r[i] - v[i] * alpha;
    const double sNorm = vnorm(sv, n);
    if (!isfinite(sNorm)) {
      out->status = OG_NONFINITE_RESIDUAL;
      out->final_residual = sNorm;
      out->iterations = iter;
      hist_push(hist, cap, &hc, sNorm);
      return 0;
    }
    if (CONV(sNorm)) {
      for (int64_t i = 0; i < n; ++i) x[i] = x[i] + pHat[i] * alpha;
      out->status = OG_CONVERGED;
      out->final_residual = sNorm;
      out->iterations = iter;
      hist_push(hist, cap, &hc, sNorm);
      return 0;
    }
    for (int64_t i = 0; i < n; ++i) sHat[i] = inv ? inv[i] * sv[i] : sv[i];
    og_stencil_apply(g, diag, off, sHat, t);
    const double tDotT = vdot(t, t, n);
    if (!isfinite(tDotT) || tDotT < DBL_MIN) BREAKDOWN();
    const double tDotS = vdot(t, sv, n);
    if (!isfinite(tDotS)) BREAKDOWN();
    if (cancelled(tDotS, t, sv, n, sqrt(tDotT), sNorm)) HANDLE_RESTART();
    omega = tDotS / tDotT;
    if (!isfinite(omega)) BREAKDOWN();
    for (int64_t i = 0; i < n; ++i) x[i] = x[i] + pHat[i] * alpha;
    for (int64_t i = 0; i < n; ++i) x[i] = x[i] + sHat[i] * omega;
    for (int64_t i = 0; i < n; ++i) r[i] = sv[i] - t[i] * omega;
    const double res = vnorm(r, n);
    rNorm = res;
    if (!isfinite(res)) {
      out->status = OG_NONFINITE_RESIDUAL;
      out->final_residual = res;
      out->iterations = iter;
      hist_push(hist, cap, &hc, res);
      return 0;
    }
    completed = iter;
    hist_push(hist, cap, &hc, res);
    lastHist = res;
    out->iterations = iter;
    if (CONV(res)) {
      out->status = OG_CONVERGED;
      out->final_residual = res;
      return 0;
    }
    rhoOld = rho;
  }
  out->status = OG_MAX_ITERATIONS;
  out->final_residual = lastHist;
  return 0;
#undef CONV
#undef BREAKDOWN
#undef RESTART
#undef HANDLE_RESTART
}

int og_stencil_solve(const og_grid* g, const og_linear_settings* s, const double* diag,
                     const double* const off[6], const double* b, double* x, double* hist,
                     int64_t hist_cap, og_linear_result* out) {
  geo G;
  geo_init(&G, g);
  const int64_t n = G.nc;
  memset(out, 0, sizeof(*out));
  out->status = OG_MAX_ITERATIONS;
  if (!stencil_finite(&G, diag, off) || !vfinite(b, n) || !vfinite(x, n)) {
    out->status = OG_NONFINITE_INPUT;
    return 0;
  }
  double* inv = NULL;
  if (s->jacobi) {
    inv = (double*)malloc(sizeof(double) * n);
    if (!inv) return -1;
    for (int64_t i = 0; i < n; ++i) {
      const double d = diag[i];
      if (!isfinite(d) || d == 0.0 || fabs(d) < 1.0e-12) {
        free(inv);
        out->status = OG_INVALID_SYSTEM;
        return 0;
      }
      inv[i] = 1.0 / d;
    }
  }
  double* work = (double*)malloc(sizeof(double) * n * 8);
  if (!work) {
    free(inv);
    return -1;
  }
  int rc;
  if (s->type == OG_SOLVER_CG)
    rc = solve_cg(g, &G, s, inv, diag, off, b, x, hist, hist_cap, out, work);
  else
    rc = solve_bicgstab(g, &G, s, inv, diag, off, b, x, hist, hist_cap, out, work);
  free(work);
  free(inv);
  return rc;
}

/* ------------------------------------------------------------------ fields */

static inline int vbc_prescribed(int t) {
  return t == OG_VBC_WALL || t == OG_VBC_MOVING_WALL || t == OG_VBC_INLET;
}

/* Boundary velocity component (Wall.cpp:8, MovingWall.cpp:22, Inlet.cpp:19,
 * Outlet.cpp:8). */
static inline double vbc_value(const og_bcs* bc, int patch, int comp, double owner) {
  switch (bc->vtype[patch]) {
    case OG_VBC_WALL: return 0.0;
    case OG_VBC_MOVING_WALL:
    case OG_VBC_INLET: return bc->vvalue[patch][comp];
    default: return owner;
  }
}

/* calculateMassFlux (MassFlux.cpp:15-35) with the velocity components u[3]. */
static void mass_flux(const geo* G, const og_bcs* bc, double rho, double* const U[3], double* F) {
  for (int64_t id = 0; id < G->nf; ++id) {
    const face_info fi = face_decode(G, id);
    const int a = fi.a;
    double ua;
    double sa = G->area[a];
    if (fi.low >= 0 && fi.high >= 0) {
      ua = interp_v(G, a, fi.f, U[a][fi.low], U[a][fi.high]);
    } else if (fi.low < 0) {
      ua = vbc_value(bc, 2 * a, a, U[a][fi.high]);
      sa = -sa;
    } else {
      ua = vbc_value(bc, 2 * a + 1, a, U[a][fi.low]);
    }
    F[id] = rho * (ua * sa);
  }
}

/* Per-cell imbalance sum_f s_f F_f in cell face order (ContinuityEquation.cpp:14-28). */
static void imbalance(const geo* G, const double* F, double* imb) {
  for (int64_t c = 0; c < G->nc; ++c) {
    int64_t ijk[3];
    cell_coords(G, c, ijk);
    double sum = 0.0;
    for (int a = 0; a < G->dim; ++a) {
      const int64_t lo = face_of(G, ijk, a, 0), hi = face_of(G, ijk, a, 1);
      /* low face: this cell is the neighbour (or owner if boundary) */
      sum += (ijk[a] == 0) ? F[lo] : -F[lo];
      sum += F[hi];
    }
    imb[c] = sum;
  }
}

/* Sum of boundary fluxes over patches in order, each patch's faces in
 * creation (= increasing id) order (ContinuityEquation.cpp:30-36). */
static double global_net_flux(const geo* G, const double* F) {
  double s = 0.0;
  for (int patch = 0; patch < 2 * G->dim; ++patch) {
    const int a = patch / 2, side = patch % 2;
    const int64_t first = G->foff[a];
    const int64_t last = (a + 1 < G->dim) ? G->foff[a + 1] : G->nf;
    for (int64_t id = first; id < last; ++id) {
      const face_info fi = face_decode(G, id);
      if ((side == 0 && fi.low < 0) || (side == 1 && fi.high < 0)) s += F[id];
    }
  }
  return s;
}

/* Scalar face values with pressure-type BCs (Gradient.cpp:537, interpolate). */
static void scalar_face_values(const geo* G, const og_bcs* bc, const double* phi, double* fv) {
  for (int64_t id = 0; id < G->nf; ++id) {
    const face_info fi = face_decode(G, id);
    if (fi.low >= 0 && fi.high >= 0) {
      fv[id] = interp_s(G, fi.a, fi.f, phi[fi.low], phi[fi.high]);
    } else {
      const int side = fi.low < 0 ? 0 : 1;
      const int patch = 2 * fi.a + side;
      const int64_t owner = side == 0 ? fi.high : fi.low;
      fv[id] = (bc->ptype[patch] == OG_PBC_FIXED_VALUE)
                   ? bc->pvalue[patch]
                   : phi[owner] + (bc->pvalue[patch] * d_bnd(G, fi.a, side));
    }
  }
}

/* One Green-Gauss sweep with boundary-consistent opposite-face values
 * (Gradient.cpp:104-162, 431-482).  prev may be NULL (first sweep). */
static void gg_sweep(const geo* G, const side_geo sg[3][2], const double* phi, const double* fv,
                     double* const prev[3], double* const out[3]) {
  for (int64_t c = 0; c < G->nc; ++c) {
    int64_t ijk[3];
    cell_coords(G, c, ijk);
    double corr[3][2];
    int has[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    for (int a = 0; a < G->dim; ++a)
      for (int s = 0; s < 2; ++s) {
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G->n[a] - 1);
        if (!boundary || !sg[a][s].valid) continue;
        const side_geo* q = &sg[a][s];
        const int64_t bf = face_of(G, ijk, a, s);
        const int64_t of = face_of(G, ijk, a, 1 - s);
        const int64_t far = c + (s == 0 ? G->stride[a] : -G->stride[a]);
        const double gown = prev ? prev[a][c] : 0.0;
        const double phiB = fv[bf] + (gown * q->offset);
        const double phiP = phi[c], phiF = phi[far];
        const double sd =
            2.0 * (((phiB - phiP) / q->tb) + ((phiF - phiP) / q->L)) / (q->tb + q->L);
        const double correction = -0.5 * q->w * (1.0 - q->w) * q->L * q->L * sd;
        corr[a][1 - s] = fv[of] + correction;
        has[a][1 - s] = 1;
      }
    const double inv = 1.0 / G->vol;
    for (int a = 0; a < G->dim; ++a) {
      double sum = 0.0;
      for (int s = 0; s < 2; ++s) {
        const int64_t f = face_of(G, ijk, a, s);
        const double val = has[a][s] ? corr[a][s] : fv[f];
        const double sf = (s == 0) ? -G->area[a] : G->area[a];
        sum += sf * val;
      }
      out[a][c] = sum * inv;
    }
    for (int a = G->dim; a < 3; ++a)
      if (out[a]) out[a][c] = 0.0;
  }
}

static int transfer_needed(const geo* G, const side_geo sg[3][2]) {
  for (int a = 0; a < G->dim; ++a)
    for (int s = 0; s < 2; ++s)
      if (sg[a][s].valid && sg[a][s].offset != 0.0) return 1;
  return 0;
}

/* greenGaussGradient with kGreenGaussSkewCorrectionSweeps = 4 (Gradient.cpp:534-596). */
static void gg_gradient(const geo* G, const side_geo sg[3][2], const og_bcs* bc,
                        const double* phi, double* fv, double* const g[3], double* const tmp[3]) {
  scalar_face_values(G, bc, phi, fv);
  gg_sweep(G, sg, phi, fv, NULL, g);
  if (!transfer_needed(G, sg)) return;
  for (int sweep = 0; sweep < 4; ++sweep) {
    gg_sweep(G, sg, phi, fv, g, tmp);
    for (int a = 0; a < G->dim; ++a) memcpy(g[a], tmp[a], sizeof(double) * G->nc);
  }
}

int og_scalar_gradient(const og_grid* g, const og_bcs* bc, const double* phi, double* gx,
                       double* gy, double* gz) {
  geo G;
  geo_init(&G, g);
  side_geo sg[3][2];
  for (int a = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s)
      sg[a][s] = (a < G.dim) ? side_geometry(&G, a, s) : (side_geo){0};
  double* fv = (double*)malloc(sizeof(double) * (G.nf + 3 * G.nc));
  if (!fv) return -1;
  double* tmp[3] = {fv + G.nf, fv + G.nf + G.nc, fv + G.nf + 2 * G.nc};
  double* out[3] = {gx, gy, G.dim == 3 ? gz : NULL};
  gg_gradient(&G, sg, bc, phi, fv, out, tmp);
  free(fv);
  return 0;
}

/* Plain Green-Gauss gradient of velocity component `comp` with velocity BCs
 * (VectorGradient.cpp:19-52): grad[a][c] = d(u_comp)/dx_a. */
static void velocity_gradient(const geo* G, const og_bcs* bc, double* const U[3], int comp,
                              double* const grad[3]) {
  for (int64_t c = 0; c < G->nc; ++c) {
    int64_t ijk[3];
    cell_coords(G, c, ijk);
    const double inv = 1.0 / G->vol;
    for (int a = 0; a < G->dim; ++a) {
      double sum = 0.0;
      for (int s = 0; s < 2; ++s) {
        double val;
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G->n[a] - 1);
        if (boundary) {
          val = vbc_value(bc, 2 * a + s, comp, U[comp][c]);
        } else {
          const int64_t f = ijk[a] + s;
          const int64_t lo = s == 0 ? c - G->stride[a] : c;
          const int64_t hi = s == 0 ? c : c + G->stride[a];
          val = interp_v(G, a, f, U[comp][lo], U[comp][hi]);
        }
        const double sf = (s == 0) ? -G->area[a] : G->area[a];
        sum += sf * val;
      }
      grad[a][c] = sum * inv;
    }
  }
}

/* ------------------------------------------------------------- momentum row */

/* quickFaceValue (Convection.cpp:104-119) */
static double quick_face(double phiC, double hCU, double phiU, double hUf, double phiD, double hfD) {
  const double wC = (-hUf * hfD) / (hCU * (hUf + hCU + hfD));
  const double wU = ((hUf + hCU) * hfD) / (hCU * (hUf + hfD));
  const double wD = (hUf * (hUf + hCU)) / ((hUf + hCU + hfD) * (hUf + hfD));
  return (wC * phiC) + (wU * phiU) + (wD * phiD);
}

/* Deferred-correction face value for an internal face (MomentumEquation.cpp:
 * 329-411): returns phiFace - phiUpwind. */
static double deferred(const geo* G, int scheme, double* const U[3], int comp,
                       double* const gradU[3], int a, int64_t f, int64_t lo, int64_t hi,
                       double F) {
  const int ownerUpwind = F >= 0.0;
  const int64_t up = ownerUpwind ? lo : hi;
  const int64_t dn = ownerUpwind ? hi : lo;
  const double phiU = U[comp][up], phiD = U[comp][dn];
  /* far-upstream cell across the upwind cell's opposite face */
  const int64_t upCoord = ownerUpwind ? f - 1 : f;
  int64_t farC = -1;
  double hCU = 0.0;
  if (ownerUpwind && upCoord > 0) {
    farC = up - G->stride[a];
    hCU = d_pn(G, a, upCoord);
  } else if (!ownerUpwind && upCoord < G->n[a] - 1) {
    farC = up + G->stride[a];
    hCU = d_pn(G, a, upCoord + 1);
  }
  double phiHO = phiU;
  switch (scheme) {
    case OG_SCHEME_CENTRAL:
      phiHO = interp_v(G, a, f, U[comp][lo], U[comp][hi]);
      break;
    case OG_SCHEME_LUD: {
      /* faceCentroid - upwindCentroid along a */
      const double dx = node(G, a, f) - center(G, a, upCoord);
      phiHO = phiU + (gradU[a][up] * dx);
      break;
    }
    case OG_SCHEME_QUICK:
      if (farC >= 0) {
        const double hUf = fabs(node(G, a, f) - center(G, a, upCoord));
        const int64_t dnCoord = ownerUpwind ? f : f - 1;
        const double hfD = fabs(center(G, a, dnCoord) - node(G, a, f));
        phiHO = quick_face(U[comp][farC], hCU, phiU, hUf, phiD, hfD);
      }
      break;
    default:
      break;
  }
  double psi = 0.0;
  if (farC >= 0) {
    const double lg = phiD - phiU;
    if (lg != 0.0) {
      const double r = (phiU - U[comp][farC]) / lg;
      if (r > 0.0) psi = (r + fabs(r)) / (1.0 + fabs(r));
    }
  }
  const double blended = phiU + (psi * (phiHO - phiU));
  const double lo_ = phiU < phiD ? phiU : phiD;
  const double hi_ = phiU < phiD ? phiD : phiU;
  const double phiFace = blended < lo_ ? lo_ : (hi_ < blended ? hi_ : blended);
  return phiFace - phiU;
}

typedef struct {
  const geo* G;
  const side_geo (*sg)[2];
  const og_bcs* bc;
  double rho, mu;
  int scheme;
} mctx;

/* assembleRelaxedMomentumComponent (RelaxedMomentum.cpp:30-104) for one
 * component: diffusion (MomentumEquation.cpp:167-262) + convection (:264-413)
 * + pressure source (:415-430) + implicit under-relaxation
 * (UnderRelaxation.cpp:13-36), gathered row by row in the reference's
 * triplet insertion order. */
static void assemble_momentum(const mctx* M, double* const U[3], int comp, const double* F,
                              double* const gradP[3], double* const gradU[3], double alpha,
                              double* diag, double* const off[6], double* rhs) {
  const geo* G = M->G;
  const double factor = (1.0 / alpha) - 1.0;
  for (int64_t c = 0; c < G->nc; ++c) {
    int64_t ijk[3];
    cell_coords(G, c, ijk);
    double dg = 0.0, rh = 0.0;
    double o[6] = {0, 0, 0, 0, 0, 0};
    /* diffusion pass */
    for (int a = 0; a < G->dim; ++a)
      for (int s = 0; s < 2; ++s) {
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G->n[a] - 1);
        if (boundary) {
          const int patch = 2 * a + s;
          const double phiB = vbc_value(M->bc, patch, comp, U[comp][c]);
          const side_geo* q = &M->sg[a][s];
          if (vbc_prescribed(M->bc->vtype[patch]) && q->valid && q->stencil_ok) {
            const double ga = M->mu * G->area[a];
            const double cP = q->h2 / (q->h1 * (q->h2 - q->h1));
            const double cF = q->h1 / (q->h2 * (q->h2 - q->h1));
            const double cB = (1.0 / q->h1) + (1.0 / q->h2);
            const int64_t far = c + (s == 0 ? G->stride[a] : -G->stride[a]);
            const double ex =
                ga * ((cP * (gradU[a][c] * q->deltaP)) - (cF * (gradU[a][far] * q->deltaF)));
            rh += ex;
            dg += ga * cP;
            rh += (ga * cB) * phiB;
            o[2 * a + (1 - s)] += -(ga * cF);
          } else {
            const double coef = M->mu * G->area[a] / d_bnd(G, a, s);
            dg += coef;
            rh += coef * phiB;
          }
        } else {
          const int64_t f = ijk[a] + s;
          const double muf = interp_s(G, a, f, M->mu, M->mu);
          const double D = muf * G->area[a] / d_pn(G, a, f);
          dg += D;
          o[2 * a + s] += -D;
        }
      }
    /* convection pass */
    for (int a = 0; a < G->dim; ++a)
      for (int s = 0; s < 2; ++s) {
        const int64_t fid = face_of(G, ijk, a, s);
        const double Ff = F[fid];
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G->n[a] - 1);
        if (boundary) {
          if (Ff >= 0.0) {
            dg += Ff;
          } else {
            rh -= Ff * vbc_value(M->bc, 2 * a + s, comp, U[comp][c]);
          }
          continue;
        }
        const int owner = (s == 1); /* this cell owns its high face */
        if (owner) {
          if (Ff >= 0.0) dg += Ff;
          else o[2 * a + 1] += Ff;
        } else {
          if (Ff >= 0.0) o[2 * a] += -Ff;
          else dg += -Ff;
        }
        if (M->scheme != OG_SCHEME_UPWIND) {
          const int64_t f = ijk[a] + s;
          const int64_t lo = s == 0 ? c - G->stride[a] : c;
          const int64_t hi = s == 0 ? c : c + G->stride[a];
          const double corr = Ff * deferred(G, M->scheme, U, comp, gradU, a, f, lo, hi, Ff);
          if (owner) rh -= corr;
          else rh += corr;
        }
      }
    /* pressure source */
    rh += -G->vol * gradP[comp][c];
    /* implicit under-relaxation */
    if (alpha != 1.0) {
      const double extra = dg * factor;
      dg += extra;
      rh += extra * U[comp][c];
    }
    diag[c] = dg;
    rhs[c] = rh;
    for (int q = 0; q < 6; ++q) off[q][c] = o[q];
  }
}

int og_momentum_system(const og_grid* g, const og_bcs* bc, const og_simple_settings* S, int comp,
                       const double* u, const double* v, const double* w, const double* p,
                       double* diag, double* const off[6], double* rhs) {
  geo G;
  geo_init(&G, g);
  side_geo sg[3][2];
  for (int a = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s) sg[a][s] = (a < G.dim) ? side_geometry(&G, a, s) : (side_geo){0};
  const int64_t n = G.nc;
  double* mem = (double*)calloc((size_t)(13 * n + 2 * G.nf), sizeof(double));
  if (!mem) return -1;
  double* U[3] = {(double*)u, (double*)v, G.dim == 3 ? (double*)w : mem};
  double* gradP[3] = {mem + n, mem + 2 * n, mem + 3 * n};
  double* gradU[3] = {mem + 4 * n, mem + 5 * n, mem + 6 * n};
  double* tmp[3] = {mem + 7 * n, mem + 8 * n, mem + 9 * n};
  double* F = mem + 13 * n;
  double* fv = F + G.nf;
  mctx M = {&G, (const side_geo(*)[2])sg, bc, S->rho, S->mu, S->scheme};
  mass_flux(&G, bc, S->rho, U, F);
  gg_gradient(&G, sg, bc, p, fv, gradP, tmp);
  velocity_gradient(&G, bc, U, comp, gradU);
  assemble_momentum(&M, U, comp, F, gradP, gradU, S->alpha_u, diag, off, rhs);
  free(mem);
  return 0;
}

/* ------------------------------------------------------------ p' assembly */

static int has_fixed_value(const geo* G, const og_bcs* bc) {
  for (int p = 0; p < 2 * G->dim; ++p)
    if (bc->ptype[p] == OG_PBC_FIXED_VALUE) return 1;
  return 0;
}

/* p' face coefficient of an internal face (pressureCorrectionFaceCoupling,
 * PressureCorrectionEquation.cpp:146-179 -> coupling :74-99). */
static inline double pface_internal(const geo* G, double rho, int a, int64_t f, double dP,
                                    double dN) {
  const double dFace = interp_s(G, a, f, dP, dN);
  return rho * G->area[a] * dFace / d_pn(G, a, f);
}

int og_assemble_pprime(const og_grid* g, const og_bcs* bc, double rho, const double* flux,
                       const double* du, const double* dv, const double* dw,
                       int64_t reference_cell, double* face_coeff, double* diag,
                       double* const off[6], double* rhs) {
  geo G;
  geo_init(&G, g);
  const double* dcomp[3] = {du, dv, dw};
  const int pin = !has_fixed_value(&G, bc);
  for (int64_t id = 0; id < G.nf; ++id) {
    const face_info fi = face_decode(&G, id);
    if (fi.low >= 0 && fi.high >= 0) {
      face_coeff[id] = pface_internal(&G, rho, fi.a, fi.f, dcomp[fi.a][fi.low], dcomp[fi.a][fi.high]);
    } else {
      const int side = fi.low < 0 ? 0 : 1;
      const int64_t owner = side == 0 ? fi.high : fi.low;
      face_coeff[id] = (bc->ptype[2 * fi.a + side] == OG_PBC_FIXED_VALUE)
                           ? rho * G.area[fi.a] * dcomp[fi.a][owner] / d_bnd(&G, fi.a, side)
                           : 0.0;
    }
  }
  double* imb = (double*)malloc(sizeof(double) * G.nc);
  if (!imb) return -1;
  imbalance(&G, flux, imb);
  for (int64_t c = 0; c < G.nc; ++c) {
    int64_t ijk[3];
    cell_coords(&G, c, ijk);
    for (int q = 0; q < 6; ++q) off[q][c] = 0.0;
    rhs[c] = -imb[c];
    if (pin && c == reference_cell) {
      diag[c] = 1.0;
      rhs[c] = 0.0;
      continue;
    }
    double dg = 0.0;
    for (int a = 0; a < G.dim; ++a)
      for (int s = 0; s < 2; ++s) {
        const int64_t f = face_of(&G, ijk, a, s);
        const int boundary = (s == 0) ? (ijk[a] == 0) : (ijk[a] == G.n[a] - 1);
        if (boundary) {
          if (bc->ptype[2 * a + s] != OG_PBC_FIXED_VALUE) continue;
          dg += face_coeff[f];
        } else {
          dg += face_coeff[f];
          off[2 * a + s][c] = -face_coeff[f];
        }
      }
    diag[c] = dg;
  }
  free(imb);
  return 0;
}

/* ------------------------------------------------------------------ SIMPLE */

int og_simple(const og_grid* g, const og_bcs* bc, const og_simple_settings* S, double* u,
              double* v, double* w, double* p, double* flux, double* hist,
              og_simple_result* out) {
  geo G;
  geo_init(&G, g);
  const int64_t n = G.nc, nf = G.nf, dim = G.dim;
  memset(out, 0, sizeof(*out));
  if (S->reference_cell < 0 || S->reference_cell >= n || !(S->alpha_u > 0.0) ||
      S->alpha_u > 1.0 || !(S->alpha_p > 0.0) || S->alpha_p > 1.0 ||
      S->momentum.max_iterations < 1 || S->pressure.max_iterations < 1) {
    out->status = OG_S_INVALID_CONFIGURATION;
    return 0;
  }
  side_geo sg[3][2];
  for (int a = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s) sg[a][s] = (a < dim) ? side_geometry(&G, a, s) : (side_geo){0};
  /* p' gradient BCs (PressureCorrectionEquation.cpp:43-54) */
  og_bcs pcbc = *bc;
  for (int q = 0; q < 6; ++q) {
    pcbc.ptype[q] = (bc->ptype[q] == OG_PBC_FIXED_VALUE) ? OG_PBC_FIXED_VALUE : OG_PBC_FIXED_GRADIENT;
    pcbc.pvalue[q] = 0.0;
  }
  const size_t nvec = 48;
  double* mem = (double*)calloc((size_t)(nvec * n + 4 * nf), sizeof(double));
  if (!mem) return -1;
  double* slot = mem;
#define TAKE(k) (slot += (k), slot - (k))
  double* U[3] = {u, v, dim == 3 ? w : TAKE(n)};
  double* Us[3] = {TAKE(n), TAKE(n), TAKE(n)};
  double* mdiag[3] = {TAKE(n), TAKE(n), TAKE(n)};
  double* moff[6] = {TAKE(n), TAKE(n), TAKE(n), TAKE(n), TAKE(n), TAKE(n)};
  double* mrhs = TAKE(n);
  double* gradP[3] = {TAKE(n), TAKE(n), TAKE(n)};
  double* gradU[3] = {TAKE(n), TAKE(n), TAKE(n)};
  double* gtmp[3] = {TAKE(n), TAKE(n), TAKE(n)};
  double* dres[3] = {TAKE(n), TAKE(n), TAKE(n)};
  double* pdiag = TAKE(n);
  double* poff[6] = {TAKE(n), TAKE(n), TAKE(n), TAKE(n), TAKE(n), TAKE(n)};
  double* prhs = TAKE(n);
  double* pp = TAKE(n);
  double* imb = TAKE(n);
  double* fv = TAKE(nf);
  double* Fs = TAKE(nf);
  double* Dface = TAKE(nf);
  double* Fnew = TAKE(nf);
  if (dim == 2) memset(U[2], 0, sizeof(double) * n);

  mctx M = {&G, (const side_geo(*)[2])sg, bc, S->rho, S->mu, S->scheme};
  mass_flux(&G, bc, S->rho, U, flux);
  int status = OG_S_MAX_ITERATIONS;
  for (int64_t c = 0; c < n; ++c)
    if (!isfinite(U[0][c]) || !isfinite(U[1][c]) || !isfinite(U[2][c]) || !isfinite(p[c])) {
      out->status = OG_S_NONFINITE;
      free(mem);
      return 0;
    }

  for (int64_t it = 0; it < S->max_outer; ++it) {
    /* pressure gradient for the momentum source (Gradient.cpp:598) */
    gg_gradient(&G, sg, bc, p, fv, gradP, gtmp);
    double initRes[3] = {0, 0, 0};
    int fail = 0;
    for (int comp = 0; comp < dim && !fail; ++comp) {
      velocity_gradient(&G, bc, U, comp, gradU);
      assemble_momentum(&M, U, comp, flux, gradP, gradU, S->alpha_u, mdiag[comp], moff, mrhs);
      /* momentum solve warm-started from the current component (SIMPLE.cpp:589-623) */
      memcpy(Us[comp], U[comp], sizeof(double) * n);
      og_linear_result lr;
      if (og_stencil_solve(g, &S->momentum, mdiag[comp], (const double* const*)moff, mrhs,
                           Us[comp], NULL, 0, &lr) != 0) {
        free(mem);
        return -1;
      }
      if (lr.status != OG_CONVERGED) {
        status = OG_S_MOMENTUM_FAILURE;
        fail = 1;
        break;
      }
      initRes[comp] = lr.initial_residual;
      out->momentum_linear_iterations += lr.iterations;
    }
    if (fail) break;
    for (int comp = 0; comp < dim; ++comp)
      for (int64_t c = 0; c < n; ++c)
        if (!isfinite(Us[comp][c])) fail = 1;
    if (dim == 2) memset(Us[2], 0, sizeof(double) * n);
    if (fail) {
      status = OG_S_NONFINITE;
      break;
    }
    /* response coefficients d = V / aP (PressureCorrectionEquation.cpp:103-114) */
    for (int comp = 0; comp < dim; ++comp)
      for (int64_t c = 0; c < n; ++c) dres[comp][c] = G.vol / mdiag[comp][c];
    /* predictor flux: linear interpolation, or Rhie-Chow (RhieChow.cpp:17-65) */
    mass_flux(&G, bc, S->rho, Us, Fs);
    if (S->face_flux == OG_FLUX_RHIECHOW) {
      gg_gradient(&G, sg, bc, p, fv, gradP, gtmp);
      for (int64_t id = 0; id < nf; ++id) {
        const face_info fi = face_decode(&G, id);
        if (fi.low < 0 || fi.high < 0) continue;
        const int a = fi.a;
        const double coupling =
            pface_internal(&G, S->rho, a, fi.f, dres[a][fi.low], dres[a][fi.high]);
        const double dvec = center(&G, a, fi.f) - center(&G, a, fi.f - 1);
        const double gf = interp_v(&G, a, fi.f, gradP[a][fi.low], gradP[a][fi.high]);
        const double cmi = (p[fi.high] - p[fi.low]) - (gf * dvec);
        Fs[id] += -(coupling / S->alpha_u) * cmi;
      }
    }
    for (int64_t id = 0; id < nf; ++id)
      if (!isfinite(Fs[id])) fail = 1;
    if (fail) {
      status = OG_S_NONFINITE;
      break;
    }
    /* p' assembly and solve from x0 = 0 */
    if (og_assemble_pprime(g, bc, S->rho, Fs, dres[0], dres[1], dres[2], S->reference_cell, Dface,
                           pdiag, poff, prhs) != 0) {
      free(mem);
      return -1;
    }
    memset(pp, 0, sizeof(double) * n);
    og_linear_result pr;
    if (og_stencil_solve(g, &S->pressure, pdiag, (const double* const*)poff, prhs, pp, NULL, 0,
                         &pr) != 0) {
      free(mem);
      return -1;
    }
    if (pr.status != OG_CONVERGED) {
      status = OG_S_PRESSURE_FAILURE;
      break;
    }
    out->pressure_linear_iterations += pr.iterations;
    for (int64_t c = 0; c < n; ++c)
      if (!isfinite(pp[c])) fail = 1;
    if (fail) {
      status = OG_S_NONFINITE;
      break;
    }
    /* pressure update, velocity and flux corrections (SIMPLE.cpp:937-991) */
    for (int64_t c = 0; c < n; ++c) p[c] = p[c] + (S->alpha_p * pp[c]);
    gg_gradient(&G, sg, &pcbc, pp, fv, gradU, gtmp);
    for (int comp = 0; comp < dim; ++comp)
      for (int64_t c = 0; c < n; ++c) U[comp][c] = Us[comp][c] - (dres[comp][c] * gradU[comp][c]);
    for (int64_t id = 0; id < nf; ++id) {
      const face_info fi = face_decode(&G, id);
      const double pO = (fi.low >= 0) ? pp[fi.low] : pp[fi.high];
      const double pN = (fi.low >= 0 && fi.high >= 0) ? pp[fi.high] : 0.0;
      Fnew[id] = Fs[id] + Dface[id] * (pO - pN);
    }
    for (int comp = 0; comp < dim; ++comp)
      for (int64_t c = 0; c < n; ++c)
        if (!isfinite(U[comp][c]) || !isfinite(p[c])) fail = 1;
    for (int64_t id = 0; id < nf; ++id)
      if (!isfinite(Fnew[id])) fail = 1;
    if (fail) {
      status = OG_S_NONFINITE;
      break;
    }
    /* residuals (SIMPLE.cpp:1019-1030) */
    imbalance(&G, Fnew, imb);
    double ss = 0.0;
    for (int64_t c = 0; c < n; ++c) ss += imb[c] * imb[c];
    const double cont = sqrt(ss / (double)n);
    const double glob = fabs(global_net_flux(&G, Fnew));
    memcpy(flux, Fnew, sizeof(double) * nf);
    out->iterations = it + 1;
    out->final_u = initRes[0];
    out->final_v = initRes[1];
    out->final_w = dim == 3 ? initRes[2] : 0.0;
    out->final_p = pr.initial_residual;
    out->final_continuity = cont;
    out->global_imbalance = glob;
    if (hist) {
      hist[5 * it + 0] = initRes[0];
      hist[5 * it + 1] = initRes[1];
      hist[5 * it + 2] = out->final_w;
      hist[5 * it + 3] = pr.initial_residual;
      hist[5 * it + 4] = cont;
    }
    /* OuterIterationMonitor::isConverged, absolute criterion (SolverRobustness.cpp:361-372) */
    const int conv = (initRes[0] <= S->tol_u) && (initRes[1] <= S->tol_u) &&
                     (pr.initial_residual <= S->tol_p) && (cont <= S->tol_c) &&
                     (glob <= S->tol_c) && (dim == 2 || initRes[2] <= S->tol_u);
    if (conv) {
      status = OG_S_CONVERGED;
      break;
    }
  }
#undef TAKE
  out->status = status;
  free(mem);
  return 0;
}
