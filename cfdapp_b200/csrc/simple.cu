// GPU-resident SIMPLE outer loop (replaces SIMPLE::solve,
// src/pressure_velocity/SIMPLE.cpp:148-1124, on uniform Cartesian grids).
//
// Host C++ orchestrates the stage kernels of simple_kernels.cu, the stencil
// Krylov solves of stencil_solve.cu (momentum; p' when BiCGSTAB is asked) and
// the p' PCG of pcg.cu; all fields stay on the device and only a handful of
// scalars (solver statuses, residual norms) cross per outer iteration.  The
// stage order, the failure statuses and the convergence test follow the
// reference: momentum assembly for every component, momentum solves warm
// started from the current velocity, response coefficients, predictor flux
// (linear or Rhie-Chow), p' assembly and solve from zero, pressure update,
// velocity and flux corrections, residuals, absolute convergence gate
// (SolverRobustness.cpp:361-372).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <utility>
#include <vector>

#include "cfdb.h"
#include "cfdb_internal.cuh"
#include "pcg_internal.cuh"
#include "simple_geo.cuh"
#include "simple_kernels.cuh"
#include "stencil_solve.cuh"

namespace cfdb {
namespace {

SideGeo side_geometry(const SGeo& G, int a, int s) {
  SideGeo sg;
  std::memset(&sg, 0, sizeof(sg));
  const int n = G.n[a];
  if (n < 2) return sg;
  sg.valid = 1;
  const int ip = (s == 0) ? 0 : n - 1;
  const int iF = (s == 0) ? 1 : n - 2;
  const double xb = (s == 0) ? g_node(G, a, 0) : g_node(G, a, n);
  // the boundary face's area vector (only its sign and scale enter); on a
  // rectilinear mesh the first face of the side stands for all of them,
  // whose quantities below differ from it at most in their last bits
  const int ijk0[3] = {ip * (a == 0), ip * (a == 1), ip * (a == 2)};
  const double area = g_area(G, a, ijk0);
  const double sfa = (s == 0) ? -area : area;
  const double cP = g_center(G, a, ip), cF = g_center(G, a, iF);
  const double d = cF - cP;
  sg.L = std::fabs(d);
  const double inward = d * (1.0 / sg.L);
  const int fo = (s == 0) ? 1 : n - 1;
  const double toFace = g_node(G, a, fo) - g_center(G, a, fo - 1);
  const double dd = g_center(G, a, fo) - g_center(G, a, fo - 1);
  sg.w = (toFace * dd) / (dd * dd);
  sg.tb = ((cP - xb) * sfa) / (inward * sfa);
  const double point = cP - (inward * sg.tb);
  sg.offset = point - xb;
  const double normal = sfa * (1.0 / area);
  sg.h1 = (xb - cP) * normal;
  sg.h2 = (xb - cF) * normal;
  sg.stencil_ok = (sg.h1 > 0.0) && (sg.h2 > sg.h1);
  sg.deltaP = cP - (xb - (normal * sg.h1));
  sg.deltaF = cF - (xb - (normal * sg.h2));
  return sg;
}

// node[a]: node coordinates of axis a in the memory the SGeo will be used
// from (host during construction), or null for a uniform axis.
SGeo make_geo(const cfdb_simple_case& cs) {
  SGeo G;
  std::memset(&G, 0, sizeof(G));
  const cfdb_grid& g = cs.grid;
  G.dim = g.dim;
  for (int a = 0; a < 3; ++a) G.n[a] = (a < g.dim) ? (int)g.n[a] : 1;
  G.stride[0] = 1;
  G.stride[1] = G.n[0];
  G.stride[2] = (int64_t)G.n[0] * G.n[1];
  for (int a = 0; a < g.dim; ++a) {
    G.node[a] = cs.nodes[a];
    G.delta[a] = cs.nodes[a] ? 0.0 : g.len[a] / (double)g.n[a];
  }
  if (g.dim == 2) {
    G.area[0] = G.delta[1];
    G.area[1] = G.delta[0];
    G.vol = G.delta[0] * G.delta[1];
  } else {
    G.area[0] = G.delta[1] * G.delta[2];
    G.area[1] = G.delta[0] * G.delta[2];
    G.area[2] = G.delta[0] * G.delta[1];
    G.vol = (G.delta[0] * G.delta[1]) * G.delta[2];
  }
  G.nc = (int64_t)G.n[0] * G.n[1] * G.n[2];
  const int64_t nfx = (int64_t)(G.n[0] + 1) * G.n[1] * G.n[2];
  const int64_t nfy = (int64_t)G.n[0] * (G.n[1] + 1) * G.n[2];
  const int64_t nfz = g.dim == 3 ? (int64_t)G.n[0] * G.n[1] * (G.n[2] + 1) : 0;
  G.foff[0] = 0;
  G.foff[1] = nfx;
  G.foff[2] = nfx + nfy;
  G.nf = nfx + nfy + nfz;
  for (int a = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s) {
      if (a < g.dim) G.side[a][s] = side_geometry(G, a, s);
      else std::memset(&G.side[a][s], 0, sizeof(SideGeo));
      if (a < g.dim && G.side[a][s].valid && G.side[a][s].offset != 0.0) G.transfer = 1;
    }
  for (int q = 0; q < 6; ++q) {
    G.vtype[q] = cs.vbc_type[q];
    for (int c = 0; c < 3; ++c) G.vvalue[q][c] = cs.vbc_value[q][c];
    G.ptype[q] = cs.pbc_type[q];
    G.pvalue[q] = cs.pbc_value[q];
  }
  return G;
}

bool wall_offsets_nonzero(const SGeo& G) {
  for (int a = 0; a < G.dim; ++a)
    for (int s = 0; s < 2; ++s)
      if (G.side[a][s].deltaP != 0.0 || G.side[a][s].deltaF != 0.0) return true;
  return false;
}

__global__ void k_pprime_stencil(int64_t n, int nx, int ny, int nz, int dim, const double* D,
                                 int64_t foff1, int64_t foff2, int pin, int64_t ref,
                                 double* diag, double* o0, double* o1, double* o2, double* o3,
                                 double* o4, double* o5) {
  double* off[6] = {o0, o1, o2, o3, o4, o5};
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((int64_t)nx * ny));
    const int ijk[3] = {i, j, k};
    const int nn[3] = {nx, ny, nz};
    for (int q = 0; q < 6; ++q) off[q][c] = 0.0;
    if (pin && c == ref) {
      diag[c] = 1.0;
      continue;
    }
    double dg = 0.0;
    for (int a = 0; a < dim; ++a)
      for (int s = 0; s < 2; ++s) {
        int64_t f;
        const int64_t ii = i + (a == 0 ? s : 0), jj = j + (a == 1 ? s : 0), kk = k + (a == 2 ? s : 0);
        if (a == 0) f = ii + (int64_t)(nx + 1) * (jj + (int64_t)ny * kk);
        else if (a == 1) f = foff1 + ii + (int64_t)nx * (jj + (int64_t)(ny + 1) * kk);
        else f = foff2 + ii + (int64_t)nx * (jj + (int64_t)ny * kk);
        const bool boundary = s == 0 ? ijk[a] == 0 : ijk[a] == nn[a] - 1;
        dg += D[f];
        if (!boundary) off[2 * a + s][c] = -D[f];
      }
    diag[c] = dg;
  }
}

}  // namespace
}  // namespace cfdb

using namespace cfdb;

struct cfdb_simple {
  cfdb_context* ctx = nullptr;
  cfdb_simple_case cs{};
  cfdb_simple_settings st{};
  SGeo G{};
  int face_flux = 0;
  int pin = 0;
  bool need_ugrad = false;
  int64_t n = 0, nf = 0;
  std::vector<double*> owned;
  double *U[3] = {}, *Us[3] = {}, *p = nullptr, *F = nullptr, *Fs = nullptr, *Fn = nullptr;
  double *mdiag[3] = {}, *moff[6] = {}, *mrhs = nullptr;
  double *gradP[3] = {}, *gradU[3] = {}, *gtmp[3] = {}, *dres[3] = {};
  double *pdiag = nullptr, *poff[6] = {}, *prhs = nullptr, *pp = nullptr, *fv = nullptr, *D = nullptr;
  double* partials = nullptr;
  int* d_ptype = nullptr;       // pressure BCs
  double* d_pvalue = nullptr;
  int* d_pctype = nullptr;      // p' BCs for its gradient
  double* d_pcvalue = nullptr;
  unsigned* flag = nullptr;
  cfdb_poperator* pop = nullptr;
  StencilWork work;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<double> hnodes[3];  // node coordinates of non-uniform axes (host copy)
  double* dnodes[3] = {nullptr, nullptr, nullptr};

  ~cfdb_simple() {
    for (double* q : owned) cudaFree(q);
    cudaFree(d_ptype);
    cudaFree(d_pvalue);
    cudaFree(d_pctype);
    cudaFree(d_pcvalue);
    cudaFree(flag);
    for (double* q : dnodes) cudaFree(q);
    if (pop) cfdb_poperator_destroy(pop);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

namespace {

cfdb_status alloc_d(cfdb_simple* s, double** p, int64_t n) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(double) * (size_t)std::max<int64_t>(n, 1));
  if (e != cudaSuccess) return cuda_error(s->ctx, e, "SIMPLE field allocation", __FILE__, __LINE__);
  s->owned.push_back(*p);
  return cudaMemsetAsync(*p, 0, sizeof(double) * (size_t)std::max<int64_t>(n, 1), s->ctx->stream) ==
                 cudaSuccess
             ? CFDB_OK
             : CFDB_ERR_CUDA;
}

StencilMatrix stencil_of(const cfdb_simple* s, const double* diag, double* const off[6]) {
  StencilMatrix M{};
  M.dim = s->G.dim;
  M.nx = s->G.n[0];
  M.ny = s->G.n[1];
  M.nz = s->G.n[2];
  M.n = s->n;
  M.sy = s->G.stride[1];
  M.sz = s->G.stride[2];
  M.diag = diag;
  for (int q = 0; q < 6; ++q) M.off[q] = off[q];
  M.inv = nullptr;
  return M;
}

cfdb_status validate(cfdb_context* ctx, const cfdb_simple_case* cs, const cfdb_simple_settings* st) {
  if (!cs || !st) return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "null case or settings");
  const cfdb_grid& g = cs->grid;
  if (g.dim != 2 && g.dim != 3) return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
  for (int a = 0; a < g.dim; ++a) {
    if (g.n[a] < 2 || g.n[a] > (1 << 20) || (!cs->nodes[a] && !(g.len[a] > 0.0)))
      return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "each axis needs >= 2 cells and a positive length");
    if (cs->nodes[a])
      for (int64_t i = 0; i <= g.n[a]; ++i)
        if (!std::isfinite(cs->nodes[a][i]) || (i > 0 && !(cs->nodes[a][i] > cs->nodes[a][i - 1])))
          return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT,
                           "node coordinates must be finite and strictly increasing");
  }
  if (!(cs->rho > 0.0) || !(cs->mu > 0.0) || !std::isfinite(cs->rho) || !std::isfinite(cs->mu))
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "rho and mu must be finite and > 0");
  for (int q = 0; q < 2 * g.dim; ++q) {
    if (cs->vbc_type[q] < 0 || cs->vbc_type[q] > 3 || cs->pbc_type[q] < 0 || cs->pbc_type[q] > 1)
      return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "unknown boundary condition type");
  }
  return CFDB_OK;
}

// Green-Gauss gradient (greenGaussGradient with its tangential sweeps).
void gradient(cfdb_simple* s, const int* ptype, const double* pvalue, const double* phi,
              double* const g[3]) {
  cudaStream_t st = s->ctx->stream;
  launch_scalar_face_values(s->G, ptype, pvalue, phi, s->fv, st);
  launch_gg_sweep(s->G, phi, s->fv, nullptr, g, st);
  s->ctx->launches += 2;
  if (!s->G.transfer) return;
  for (int sweep = 0; sweep < 4; ++sweep) {
    const double* prev[3] = {g[0], g[1], g[2]};
    launch_gg_sweep(s->G, phi, s->fv, prev, s->gtmp, st);
    for (int a = 0; a < s->G.dim; ++a)
      cudaMemcpyAsync(g[a], s->gtmp[a], sizeof(double) * s->n, cudaMemcpyDeviceToDevice, st);
    s->ctx->launches += 1;
  }
}

cfdb_status check_nonfinite(cfdb_simple* s, std::initializer_list<std::pair<const double*, int64_t>> vs,
                            bool* bad) {
  cudaStream_t st = s->ctx->stream;
  CFDB_CUDA(s->ctx, cudaMemsetAsync(s->flag, 0, sizeof(unsigned), st));
  for (auto& v : vs) {
    launch_nonfinite(v.second, v.first, s->flag, st);
    s->ctx->launches += 1;
  }
  unsigned f = 0;
  CFDB_CUDA(s->ctx, cudaMemcpyAsync(&f, s->flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  CFDB_CUDA(s->ctx, cudaStreamSynchronize(st));
  *bad = f != 0;
  return CFDB_OK;
}

// One SIMPLE outer iteration.  status_out: -1 to continue, else a CFDB_SIMPLE_*.
cfdb_status outer_iteration(cfdb_simple* s, int64_t it, double* hist, cfdb_simple_result* out,
                            int* status_out) {
  cfdb_context* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  const SGeo& G = s->G;
  const int dim = G.dim;
  const cfdb_simple_settings& S = s->st;
  *status_out = -1;
  gradient(s, s->d_ptype, s->d_pvalue, s->p, s->gradP);
  double initRes[3] = {0, 0, 0};
  // assemble all components from the lagged state, then solve each
  for (int comp = 0; comp < dim; ++comp) {
    const double* const* gu = nullptr;
    if (s->need_ugrad) {
      launch_velocity_gradient(G, s->U[comp], comp, s->gradU + 0, st);
      ctx->launches += 1;
      gu = s->gradU;
    }
    launch_assemble_momentum(G, s->cs.mu, S.scheme, comp, s->U[comp], s->F, s->gradP[comp], gu,
                             S.alpha_u, s->mdiag[comp], s->moff, s->mrhs, st);
    ctx->launches += 1;
    CFDB_CUDA(ctx, cudaMemcpyAsync(s->Us[comp], s->U[comp], sizeof(double) * s->n,
                                   cudaMemcpyDeviceToDevice, st));
    cfdb_linear_result lr;
    const StencilMatrix M = stencil_of(s, s->mdiag[comp], s->moff);
    cfdb_status rc = stencil_solve(ctx, M, s->work, s->mrhs, s->Us[comp], S.momentum.krylov,
                                   S.momentum.preconditioner == CFDB_PRECOND_JACOBI,
                                   S.momentum.abs_tol, S.momentum.rel_tol,
                                   S.momentum.max_iterations, nullptr, 0, &lr);
    if (rc != CFDB_OK) return rc;
    ctx->launches += lr.kernel_launches;
    out->momentum_solve_ms += lr.krylov_ms;
    if (lr.status != CFDB_SOLVER_CONVERGED) {
      *status_out = CFDB_SIMPLE_MOMENTUM_FAILURE;
      return CFDB_OK;
    }
    initRes[comp] = lr.initial_residual;
    out->momentum_linear_iterations += lr.iterations;
  }
  bool bad = false;
  cfdb_status rc = check_nonfinite(s, {{s->Us[0], s->n}, {s->Us[1], s->n}, {s->Us[dim - 1], s->n}}, &bad);
  if (rc != CFDB_OK) return rc;
  if (bad) {
    *status_out = CFDB_SIMPLE_NONFINITE_STATE;
    return CFDB_OK;
  }
  for (int comp = 0; comp < dim; ++comp) launch_response(G, s->mdiag[comp], s->dres[comp], st);
  const double* Usc[3] = {s->Us[0], s->Us[1], s->Us[2]};
  launch_mass_flux(G, s->cs.rho, Usc, s->Fs, st);
  ctx->launches += dim + 1;
  if (s->face_flux == CFDB_FLUX_RHIE_CHOW) {
    const double* gp[3] = {s->gradP[0], s->gradP[1], s->gradP[2]};
    const double* dr[3] = {s->dres[0], s->dres[1], s->dres[2]};
    launch_rhie_chow(G, s->cs.rho, S.alpha_u, s->p, gp, dr, s->Fs, st);
    ctx->launches += 1;
  }
  rc = check_nonfinite(s, {{s->Fs, s->nf}}, &bad);
  if (rc != CFDB_OK) return rc;
  if (bad) {
    *status_out = CFDB_SIMPLE_NONFINITE_STATE;
    return CFDB_OK;
  }
  // p' assembly and solve from zero
  const double* dr[3] = {s->dres[0], s->dres[1], s->dres[2]};
  launch_pprime_faces(G, s->cs.rho, dr, s->D, st);
  launch_pprime_rhs(G, s->Fs, s->pin, S.reference_cell, s->prhs, st);
  ctx->launches += 2;
  CFDB_CUDA(ctx, cudaMemsetAsync(s->pp, 0, sizeof(double) * s->n, st));
  cfdb_linear_result pr;
  const bool use_pcg = S.pressure.krylov == CFDB_KRYLOV_CG &&
                       (S.pressure.preconditioner == CFDB_PRECOND_JACOBI ||
                        S.pressure.preconditioner == CFDB_PRECOND_LEARNED_MG);
  if (use_pcg) {
    rc = poperator_bind_faces(ctx, s->pop, s->D, S.pressure.precision == CFDB_PRECISION_FP32_REFINED);
    if (rc != CFDB_OK) return rc;
    const int64_t l0 = ctx->launches;
    rc = cfdb_poperator_solve_device(ctx, s->pop, &S.pressure, s->prhs, s->pp, nullptr, 0, &pr);
    if (rc != CFDB_OK) return rc;
    (void)l0;
  } else {
    k_pprime_stencil<<<1024, 256, 0, st>>>(s->n, G.n[0], G.n[1], G.n[2], dim, s->D, G.foff[1],
                                          G.foff[2], s->pin, S.reference_cell, s->pdiag, s->poff[0],
                                          s->poff[1], s->poff[2], s->poff[3], s->poff[4], s->poff[5]);
    ctx->launches += 1;
    const StencilMatrix M = stencil_of(s, s->pdiag, s->poff);
    rc = stencil_solve(ctx, M, s->work, s->prhs, s->pp, S.pressure.krylov,
                       S.pressure.preconditioner == CFDB_PRECOND_JACOBI, S.pressure.abs_tol,
                       S.pressure.rel_tol, S.pressure.max_iterations, nullptr, 0, &pr);
    if (rc != CFDB_OK) return rc;
    ctx->launches += pr.kernel_launches;
  }
  out->pressure_solve_ms += pr.krylov_ms;
  if (pr.status != CFDB_SOLVER_CONVERGED) {
    *status_out = CFDB_SIMPLE_PRESSURE_FAILURE;
    return CFDB_OK;
  }
  out->pressure_linear_iterations += pr.iterations;
  rc = check_nonfinite(s, {{s->pp, s->n}}, &bad);
  if (rc != CFDB_OK) return rc;
  if (bad) {
    *status_out = CFDB_SIMPLE_NONFINITE_STATE;
    return CFDB_OK;
  }
  // corrections
  launch_pressure_update(s->n, S.alpha_p, s->pp, s->p, st);
  gradient(s, s->d_pctype, s->d_pcvalue, s->pp, s->gradU);
  for (int comp = 0; comp < dim; ++comp)
    launch_velocity_correct(s->n, s->Us[comp], s->dres[comp], s->gradU[comp], s->U[comp], st);
  launch_flux_correct(G, s->Fs, s->D, s->pp, s->Fn, st);
  ctx->launches += 2 + dim;
  rc = check_nonfinite(s, {{s->U[0], s->n}, {s->U[1], s->n}, {s->U[dim - 1], s->n}, {s->p, s->n},
                          {s->Fn, s->nf}},
                       &bad);
  if (rc != CFDB_OK) return rc;
  if (bad) {
    *status_out = CFDB_SIMPLE_NONFINITE_STATE;
    return CFDB_OK;
  }
  // residuals
  const int nb = residual_sums_blocks(G);
  launch_residual_sums(G, s->Fn, s->partials, st);
  ctx->launches += 1;
  std::vector<double> h(2 * nb);
  CFDB_CUDA(ctx, cudaMemcpyAsync(h.data(), s->partials, sizeof(double) * 2 * nb,
                                 cudaMemcpyDeviceToHost, st));
  std::swap(s->F, s->Fn);
  CFDB_CUDA(ctx, cudaStreamSynchronize(st));
  double ss = 0.0, gb = 0.0;
  for (int b = 0; b < nb; ++b) {
    ss += h[2 * b];
    gb += h[2 * b + 1];
  }
  const double cont = std::sqrt(ss / (double)s->n);
  const double glob = std::fabs(gb);
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
  const bool conv = (initRes[0] <= S.tol_u) && (initRes[1] <= S.tol_u) &&
                    (pr.initial_residual <= S.tol_p) && (cont <= S.tol_c) && (glob <= S.tol_c) &&
                    (dim == 2 || initRes[2] <= S.tol_u);
  if (conv) *status_out = CFDB_SIMPLE_CONVERGED;
  return CFDB_OK;
}

}  // namespace

namespace cfdb {
SGeo simple_geometry(const cfdb_simple_case& cs) { return make_geo(cs); }
bool simple_wall_offsets(const SGeo& G) { return wall_offsets_nonzero(G); }
cfdb_status simple_validate(cfdb_context* ctx, const cfdb_simple_case* cs,
                            const cfdb_simple_settings* st) {
  return validate(ctx, cs, st);
}
}  // namespace cfdb

extern "C" {

cfdb_status cfdb_simple_create(cfdb_context* ctx, const cfdb_simple_case* cs,
                               const cfdb_simple_settings* st, cfdb_simple** out) {
  if (!ctx || !out) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_status rc = validate(ctx, cs, st);
  if (rc != CFDB_OK) return rc;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  std::unique_ptr<cfdb_simple> s(new cfdb_simple());
  s->ctx = ctx;
  s->cs = *cs;
  s->st = *st;
  for (int a = 0; a < 3; ++a) {  // the session keeps its own copy of the nodes
    if (a < cs->grid.dim && cs->nodes[a]) {
      s->hnodes[a].assign(cs->nodes[a], cs->nodes[a] + cs->grid.n[a] + 1);
      s->cs.nodes[a] = s->hnodes[a].data();
    } else {
      s->cs.nodes[a] = nullptr;
    }
  }
  s->G = make_geo(s->cs);  // host node pointers: the side geometry is computed here
  for (int a = 0; a < 3; ++a)
    if (s->cs.nodes[a]) {
      const size_t bytes = sizeof(double) * s->hnodes[a].size();
      CFDB_CUDA(ctx, cudaMalloc((void**)&s->dnodes[a], bytes));
      CFDB_CUDA(ctx, cudaMemcpyAsync(s->dnodes[a], s->hnodes[a].data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
      s->G.node[a] = s->dnodes[a];  // the kernels read the device copy
    }
  s->n = s->G.nc;
  s->nf = s->G.nf;
  s->face_flux = st->face_flux == CFDB_FLUX_AUTOMATIC ? (cs->grid.dim == 2 ? CFDB_FLUX_LINEAR
                                                                           : CFDB_FLUX_RHIE_CHOW)
                                                      : st->face_flux;
  bool fixed_value = false;
  for (int q = 0; q < 2 * cs->grid.dim; ++q) fixed_value |= cs->pbc_type[q] == CFDB_PBC_FIXED_VALUE;
  s->pin = fixed_value ? 0 : 1;
  s->need_ugrad = st->scheme == CFDB_SCHEME_LINEAR_UPWIND || wall_offsets_nonzero(s->G);
  if (st->reference_cell < 0 || st->reference_cell >= s->n)
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "reference cell out of range");
  const int64_t n = s->n, nf = s->nf;
  for (int c = 0; c < 3; ++c) {
    if ((rc = alloc_d(s.get(), &s->U[c], n)) || (rc = alloc_d(s.get(), &s->Us[c], n)) ||
        (rc = alloc_d(s.get(), &s->mdiag[c], n)) || (rc = alloc_d(s.get(), &s->gradP[c], n)) ||
        (rc = alloc_d(s.get(), &s->gradU[c], n)) || (rc = alloc_d(s.get(), &s->gtmp[c], n)) ||
        (rc = alloc_d(s.get(), &s->dres[c], n)))
      return rc;
  }
  for (int q = 0; q < 6; ++q)
    if ((rc = alloc_d(s.get(), &s->moff[q], n)) || (rc = alloc_d(s.get(), &s->poff[q], n))) return rc;
  if ((rc = alloc_d(s.get(), &s->mrhs, n)) || (rc = alloc_d(s.get(), &s->p, n)) ||
      (rc = alloc_d(s.get(), &s->pdiag, n)) || (rc = alloc_d(s.get(), &s->prhs, n)) ||
      (rc = alloc_d(s.get(), &s->pp, n)) || (rc = alloc_d(s.get(), &s->F, nf)) ||
      (rc = alloc_d(s.get(), &s->Fs, nf)) || (rc = alloc_d(s.get(), &s->Fn, nf)) ||
      (rc = alloc_d(s.get(), &s->fv, nf)) || (rc = alloc_d(s.get(), &s->D, nf)) ||
      (rc = alloc_d(s.get(), &s->partials, 2 * 1024)))
    return rc;
  int pct[6];
  double pcv[6] = {0, 0, 0, 0, 0, 0};
  for (int q = 0; q < 6; ++q)
    pct[q] = cs->pbc_type[q] == CFDB_PBC_FIXED_VALUE ? CFDB_PBC_FIXED_VALUE : CFDB_PBC_FIXED_GRADIENT;
  CFDB_CUDA(ctx, cudaMalloc((void**)&s->d_ptype, 6 * sizeof(int)));
  CFDB_CUDA(ctx, cudaMalloc((void**)&s->d_pvalue, 6 * sizeof(double)));
  CFDB_CUDA(ctx, cudaMalloc((void**)&s->d_pctype, 6 * sizeof(int)));
  CFDB_CUDA(ctx, cudaMalloc((void**)&s->d_pcvalue, 6 * sizeof(double)));
  CFDB_CUDA(ctx, cudaMalloc((void**)&s->flag, sizeof(unsigned)));
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->d_ptype, cs->pbc_type, 6 * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->d_pvalue, cs->pbc_value, 6 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->d_pctype, pct, 6 * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->d_pcvalue, pcv, 6 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaEventCreate(&s->e0));
  CFDB_CUDA(ctx, cudaEventCreate(&s->e1));
  rc = cfdb_poperator_create_uniform(ctx, &cs->grid, 1.0, 0u, s->pin, st->reference_cell, &s->pop);
  if (rc != CFDB_OK) return rc;
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *out = s.release();
  return CFDB_OK;
}

void cfdb_simple_destroy(cfdb_simple* s) {
  if (!s) return;
  cudaStreamSynchronize(s->ctx->stream);
  delete s;
}

cfdb_status cfdb_simple_set_state(cfdb_simple* s, const double* u, const double* v, const double* w,
                                  const double* p) {
  if (!s || !u || !v || !p || (s->G.dim == 3 && !w)) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = s->ctx;
  const size_t b = sizeof(double) * (size_t)s->n;
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->U[0], u, b, cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->U[1], v, b, cudaMemcpyHostToDevice, ctx->stream));
  if (s->G.dim == 3) CFDB_CUDA(ctx, cudaMemcpyAsync(s->U[2], w, b, cudaMemcpyHostToDevice, ctx->stream));
  else CFDB_CUDA(ctx, cudaMemsetAsync(s->U[2], 0, b, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->p, p, b, cudaMemcpyHostToDevice, ctx->stream));
  const double* Uc[3] = {s->U[0], s->U[1], s->U[2]};
  launch_mass_flux(s->G, s->cs.rho, Uc, s->F, ctx->stream);
  ctx->launches += 1;
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

cfdb_status cfdb_simple_get_state(cfdb_simple* s, double* u, double* v, double* w, double* p,
                                  double* flux) {
  if (!s) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = s->ctx;
  const size_t b = sizeof(double) * (size_t)s->n;
  if (u) CFDB_CUDA(ctx, cudaMemcpyAsync(u, s->U[0], b, cudaMemcpyDeviceToHost, ctx->stream));
  if (v) CFDB_CUDA(ctx, cudaMemcpyAsync(v, s->U[1], b, cudaMemcpyDeviceToHost, ctx->stream));
  if (w && s->G.dim == 3) CFDB_CUDA(ctx, cudaMemcpyAsync(w, s->U[2], b, cudaMemcpyDeviceToHost, ctx->stream));
  if (p) CFDB_CUDA(ctx, cudaMemcpyAsync(p, s->p, b, cudaMemcpyDeviceToHost, ctx->stream));
  if (flux)
    CFDB_CUDA(ctx, cudaMemcpyAsync(flux, s->F, sizeof(double) * (size_t)s->nf, cudaMemcpyDeviceToHost,
                                   ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

cfdb_status cfdb_simple_pprime_faces(cfdb_simple* s, double* faces, int* pinned,
                                     int64_t* reference_cell) {
  if (!s || !faces) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = s->ctx;
  CFDB_CUDA(ctx, cudaMemcpyAsync(faces, s->D, sizeof(double) * (size_t)s->nf,
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (pinned) *pinned = s->pin ? 1 : 0;
  if (reference_cell) *reference_cell = s->st.reference_cell;
  return CFDB_OK;
}

cfdb_status cfdb_simple_write_results(cfdb_simple* s, const double* history, int64_t rows,
                                      double global_imbalance, const char* dir,
                                      int* fields_written) {
  if (!s || !dir) return CFDB_ERR_INVALID_ARGUMENT;
  const size_t n = (size_t)s->n;
  std::vector<double> u(n), v(n), w(n), p(n);
  cfdb_status rc = cfdb_simple_get_state(s, u.data(), v.data(), w.data(), p.data(), nullptr);
  if (rc != CFDB_OK) return rc;
  rc = cfdb_write_results(&s->cs, u.data(), v.data(), w.data(), p.data(), history, rows,
                          global_imbalance, dir, fields_written);
  if (rc != CFDB_OK) return set_error(s->ctx, rc, "cannot write the result files");
  return CFDB_OK;
}

cfdb_status cfdb_simple_pressure_gradient(cfdb_simple* s, double* gx, double* gy, double* gz) {
  if (!s || !gx || !gy) return CFDB_ERR_INVALID_ARGUMENT;
  gradient(s, s->d_ptype, s->d_pvalue, s->p, s->gradP);
  const size_t b = sizeof(double) * (size_t)s->n;
  cfdb_context* ctx = s->ctx;
  CFDB_CUDA(ctx, cudaMemcpyAsync(gx, s->gradP[0], b, cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(gy, s->gradP[1], b, cudaMemcpyDeviceToHost, ctx->stream));
  if (gz && s->G.dim == 3) CFDB_CUDA(ctx, cudaMemcpyAsync(gz, s->gradP[2], b, cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

cfdb_status cfdb_simple_assemble_momentum(cfdb_simple* s, int comp, double* diag, double* const off[6],
                                          double* rhs) {
  if (!s || comp < 0 || comp >= s->G.dim || !diag || !off || !rhs) return CFDB_ERR_INVALID_ARGUMENT;
  cfdb_context* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  gradient(s, s->d_ptype, s->d_pvalue, s->p, s->gradP);
  const double* const* gu = nullptr;
  if (s->need_ugrad) {
    launch_velocity_gradient(s->G, s->U[comp], comp, s->gradU, st);
    gu = s->gradU;
  }
  launch_assemble_momentum(s->G, s->cs.mu, s->st.scheme, comp, s->U[comp], s->F, s->gradP[comp], gu,
                           s->st.alpha_u, s->mdiag[comp], s->moff, s->mrhs, st);
  ctx->launches += 2;
  const size_t b = sizeof(double) * (size_t)s->n;
  CFDB_CUDA(ctx, cudaMemcpyAsync(diag, s->mdiag[comp], b, cudaMemcpyDeviceToHost, st));
  CFDB_CUDA(ctx, cudaMemcpyAsync(rhs, s->mrhs, b, cudaMemcpyDeviceToHost, st));
  for (int q = 0; q < 6; ++q)
    if (off[q]) CFDB_CUDA(ctx, cudaMemcpyAsync(off[q], s->moff[q], b, cudaMemcpyDeviceToHost, st));
  CFDB_CUDA(ctx, cudaStreamSynchronize(st));
  return CFDB_OK;
}

cfdb_status cfdb_simple_iterate(cfdb_simple* s, int64_t nmax, double* hist, cfdb_simple_result* out) {
  if (!s || !out) return CFDB_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  cfdb_context* ctx = s->ctx;
  const int64_t launches0 = ctx->launches;
  CFDB_CUDA(ctx, cudaEventRecord(s->e0, ctx->stream));
  int status = CFDB_SIMPLE_MAX_ITERATIONS;
  for (int64_t it = 0; it < nmax; ++it) {
    int st = -1;
    cfdb_status rc = outer_iteration(s, it, hist, out, &st);
    if (rc != CFDB_OK) return rc;
    if (st >= 0) {
      status = st;
      break;
    }
  }
  CFDB_CUDA(ctx, cudaEventRecord(s->e1, ctx->stream));
  CFDB_CUDA(ctx, cudaEventSynchronize(s->e1));
  float ms = 0.f;
  CFDB_CUDA(ctx, cudaEventElapsedTime(&ms, s->e0, s->e1));
  out->device_ms = ms;
  out->status = status;
  out->kernel_launches = ctx->launches - launches0;
  return CFDB_OK;
}

cfdb_status cfdb_simple_solve(cfdb_context* ctx, const cfdb_simple_case* cs,
                              const cfdb_simple_settings* st, double* u, double* v, double* w,
                              double* p, double* flux, double* hist, cfdb_simple_result* out) {
  if (!ctx || !out || !u || !v || !p) return CFDB_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  if (validate(ctx, cs, st) != CFDB_OK || st->max_outer < 0 || !(st->alpha_u > 0.0) ||
      st->alpha_u > 1.0 || !(st->alpha_p > 0.0) || st->alpha_p > 1.0 ||
      st->momentum.max_iterations < 1 || st->pressure.max_iterations < 1) {
    // SIMPLE::solve reports configuration errors as a status (SIMPLE.cpp:164-234)
    out->status = CFDB_SIMPLE_INVALID_CONFIGURATION;
    return CFDB_OK;
  }
  cfdb_simple* s = nullptr;
  cfdb_status rc = cfdb_simple_create(ctx, cs, st, &s);
  if (rc != CFDB_OK) return rc;
  rc = cfdb_simple_set_state(s, u, v, w, p);
  if (rc == CFDB_OK) {
    bool bad = false;
    rc = check_nonfinite(s, {{s->U[0], s->n}, {s->U[1], s->n}, {s->U[2], s->n}, {s->p, s->n}}, &bad);
    if (rc == CFDB_OK && bad) {
      out->status = CFDB_SIMPLE_NONFINITE_STATE;
      cfdb_simple_destroy(s);
      return CFDB_OK;
    }
  }
  if (rc == CFDB_OK) rc = cfdb_simple_iterate(s, st->max_outer, hist, out);
  if (rc == CFDB_OK) rc = cfdb_simple_get_state(s, u, v, w, p, flux);
  cfdb_simple_destroy(s);
  return rc;
}

}  // extern "C"
