// The stencil Krylov solves (BiCGSTAB with the reference's breakdown and
// restart semantics, src/algebra/BiCGSTAB.cpp:48-275, and CG,
// src/algebra/CG.cpp:14-148, optional Jacobi) as one device routine run by a
// team of thread blocks: the whole grid of a persistent kernel for one
// system (stencil_solve.cu), or the blocks a batched kernel gives one case
// of many (batch.cu).  A Team supplies rank(), size() and a bounded
// barrier sync() over its blocks; reductions run over the team's blocks in
// a fixed order, so a team's results do not depend on timing.
//
// Layout: cell c = i + nx*(j + ny*k); off[2a] couples to the low neighbour
// along axis a, off[2a+1] to the high one (0 at the domain edge).  Row sums
// follow the reference's CSR column order (SparseMatrix.cpp:93-100).
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>

#include "cfdb.h"
#include "grid_sync.cuh"
#include "stencil_solve.cuh"

namespace cfdb {
namespace krylov {

constexpr int kThreads = 256;  // threads per block of every team

enum { O_STATUS = 0, O_ITER = 1, O_B0 = 2, O_FINAL = 3, O_RESTARTS = 4, O_REPLACEMENTS = 5 };

struct SParams {
  StencilMatrix M;
  const double* b;
  double* x;
  double *r, *rh, *v, *p, *s, *t;
  int krylov;  // 0 CG, 1 BiCGSTAB
  int jacobi;
  double abs_tol, rel_tol;
  int64_t max_it;
  double* hist;
  int64_t hist_cap;
  double* partials;
  double* out;
  // mixed-precision CG (cg_mixed_run): the FP32 copies of the diagonal and
  // the six couplings, the FP32 direction and its product (the caller's
  // storage, filled by the solve)
  float* m32[7];
  float *p32, *v32;
};

__device__ __forceinline__ double spmv_row(const StencilMatrix& M, const double* v, int64_t c,
                                           int i, int j, int k) {
  // ascending column order: z-low, y-low, x-low, diag, x-high, y-high, z-high
  double sum = 0.0;
  if (M.dim == 3 && k > 0) sum += __ldg(M.off[4] + c) * __ldcg(v + c - M.sz);
  if (j > 0) sum += __ldg(M.off[2] + c) * __ldcg(v + c - M.sy);
  if (i > 0) sum += __ldg(M.off[0] + c) * __ldcg(v + c - 1);
  sum += __ldg(M.diag + c) * __ldcg(v + c);
  if (i < M.nx - 1) sum += __ldg(M.off[1] + c) * __ldcg(v + c + 1);
  if (j < M.ny - 1) sum += __ldg(M.off[3] + c) * __ldcg(v + c + M.sy);
  if (M.dim == 3 && k < M.nz - 1) sum += __ldg(M.off[5] + c) * __ldcg(v + c + M.sz);
  return sum;
}

// Same product with the Jacobi-preconditioned input v_c * inv_c.
__device__ __forceinline__ double spmv_row_prec(const StencilMatrix& M, const double* v,
                                                const double* inv, int64_t c, int i, int j,
                                                int k) {
  auto w = [&](int64_t q) { return __ldcg(v + q) * __ldg(inv + q); };
  double sum = 0.0;
  if (M.dim == 3 && k > 0) sum += __ldg(M.off[4] + c) * w(c - M.sz);
  if (j > 0) sum += __ldg(M.off[2] + c) * w(c - M.sy);
  if (i > 0) sum += __ldg(M.off[0] + c) * w(c - 1);
  sum += __ldg(M.diag + c) * w(c);
  if (i < M.nx - 1) sum += __ldg(M.off[1] + c) * w(c + 1);
  if (j < M.ny - 1) sum += __ldg(M.off[3] + c) * w(c + M.sy);
  if (M.dim == 3 && k < M.nz - 1) sum += __ldg(M.off[5] + c) * w(c + M.sz);
  return sum;
}

template <class Team>
__device__ void krylov_run(const SParams& P, const Team& T) {
  __shared__ double red[3 * 32];
  const StencilMatrix& M = P.M;
  const int B = T.size(), blk = T.rank(), tid = threadIdx.x;
  const bool leader = (blk == 0 && tid == 0);
  const int64_t n = M.n;
  const int64_t c0 = n * blk / B, c1 = n * (blk + 1) / B;
  int round = 0;
  auto part = [&]() { return P.partials + (size_t)(round & 1) * 3 * B; };
  auto coords = [&](int64_t c, int& i, int& j, int& k) {
    i = (int)(c % M.nx);
    j = (int)((c / M.nx) % M.ny);
    k = (int)(c / M.sz);
  };
  const double* inv = M.inv;
  // reduce 3 values over the grid; false on a failed barrier
  auto reduce3 = [&](double a0, double a1, double a2, double (&o)[3]) -> bool {
    double a[3] = {a0, a1, a2};
    block_sum<3>(a, red);
    if (tid == 0) {
      part()[3 * blk] = a[0];
      part()[3 * blk + 1] = a[1];
      part()[3 * blk + 2] = a[2];
    }
    if (!T.sync()) return false;
    grid_total<3>(part(), 3, B, o, red);
    ++round;
    return true;
  };
  auto finish = [&](int status, int64_t it, double fin) {
    if (leader) {
      P.out[O_STATUS] = status;
      P.out[O_ITER] = (double)it;
      P.out[O_FINAL] = fin;
    }
  };
  const double eps = DBL_EPSILON;
  auto cancelled = [&](double ip, double nx_, double ny_, double terms) {
    if (fabs(ip) > eps * nx_ * ny_) return false;
    return fabs(ip) <= eps * terms;
  };

  // ---- r = b - A x; rHat = r (BiCGSTAB); v = p = 0
  double a0 = 0.0, a1 = 0.0;
  for (int64_t c = c0 + tid; c < c1; c += kThreads) {
    int i, j, k;
    coords(c, i, j, k);
    const double rn = __ldg(P.b + c) - spmv_row(M, P.x, c, i, j, k);
    P.r[c] = rn;
    if (P.krylov == 1) {
      P.rh[c] = rn;
      P.v[c] = 0.0;
      P.p[c] = 0.0;
    }
    a0 += rn * rn;
    a1 += rn * (inv ? __ldg(inv + c) * rn : rn);
  }
  double tot[3];
  if (!reduce3(a0, a1, 0.0, tot)) return;
  const double b0 = sqrt(tot[0]);
  if (leader) {
    P.out[O_B0] = b0;
    P.out[O_RESTARTS] = 0;
    if (P.hist_cap > 0) P.hist[0] = b0;
  }
  auto conv = [&](double res) {
    return (res <= P.abs_tol) || ((b0 > 0.0) && (res / b0 <= P.rel_tol));
  };
  if (b0 == 0.0 || conv(b0)) return finish(CFDB_SOLVER_CONVERGED, 0, b0);

  if (P.krylov == 0) {
    // ------------------------------------------------------------------ CG
    double rz = tot[1];
    if (!isfinite(rz)) return finish(CFDB_SOLVER_BREAKDOWN, 0, b0);
    double res_cur = b0, beta = 0.0;
    for (int64_t it = 1; it <= P.max_it; ++it) {
      // p = z + beta p
      for (int64_t c = c0 + tid; c < c1; c += kThreads) {
        const double z = inv ? __ldg(inv + c) * __ldcg(P.r + c) : __ldcg(P.r + c);
        P.p[c] = (it == 1) ? z : z + __ldcg(P.p + c) * beta;
      }
      if (!T.sync()) return;
      double pap = 0.0;
      for (int64_t c = c0 + tid; c < c1; c += kThreads) {
        int i, j, k;
        coords(c, i, j, k);
        const double ap = spmv_row(M, P.p, c, i, j, k);
        P.v[c] = ap;
        pap += __ldcg(P.p + c) * ap;
      }
      if (!reduce3(pap, 0.0, 0.0, tot)) return;
      const double pAp = tot[0];
      const double alpha = rz / pAp;
      if (!isfinite(pAp) || fabs(pAp) < 1.0e-30 || !isfinite(alpha))
        return finish(CFDB_SOLVER_BREAKDOWN, it - 1, res_cur);
      double rr = 0.0, rzn = 0.0;
      for (int64_t c = c0 + tid; c < c1; c += kThreads) {
        P.x[c] = P.x[c] + __ldcg(P.p + c) * alpha;
        const double rn = __ldcg(P.r + c) - P.v[c] * alpha;
        P.r[c] = rn;
        rr += rn * rn;
        rzn += rn * (inv ? __ldg(inv + c) * rn : rn);
      }
      if (!reduce3(rr, rzn, 0.0, tot)) return;
      const double res = sqrt(tot[0]);
      if (leader && it < P.hist_cap) P.hist[it] = res;
      if (!isfinite(res)) return finish(CFDB_SOLVER_NONFINITE_RESIDUAL, it, res);
      res_cur = res;
      if (conv(res)) return finish(CFDB_SOLVER_CONVERGED, it, res);
      beta = tot[1] / rz;
      if (!isfinite(tot[1]) || !isfinite(beta)) return finish(CFDB_SOLVER_BREAKDOWN, it, res);
      rz = tot[1];
    }
    return finish(CFDB_SOLVER_MAX_ITERATIONS, P.max_it, res_cur);
  }

  // -------------------------------------------------------------- BiCGSTAB
  double rhoOld = 1.0, alpha = 1.0, omega = 1.0;
  int64_t completed = 0, restarts = 0;
  double rHatNorm = b0, rNorm = b0, restartResidual = b0, lastHist = b0;
  double rho = tot[0], rhoTerms = tot[0];  // (rHat, r) and sum |rHat_i r_i| of r0
  int64_t hc = 1;
  auto push = [&](double v) {
    if (leader && hc < P.hist_cap) P.hist[hc] = v;
    ++hc;
  };
  // restart (BiCGSTAB.cpp:127-151): 0 restarted, 1 converged, 2 stop
  auto restart = [&](int& outcome) -> bool {
    if (!(rNorm < restartResidual)) {
      outcome = 2;
      return true;
    }
    double q = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      int i, j, k;
      coords(c, i, j, k);
      const double rn = __ldg(P.b + c) - spmv_row(M, P.x, c, i, j, k);
      P.r[c] = rn;
      P.rh[c] = rn;
      P.v[c] = 0.0;
      P.p[c] = 0.0;
      q += rn * rn;
    }
    double o[3];
    if (!reduce3(q, 0.0, 0.0, o)) return false;
    rNorm = sqrt(o[0]);
    if (!isfinite(rNorm)) {
      outcome = 2;
      return true;
    }
    if (conv(rNorm)) {
      outcome = 1;
      return true;
    }
    rHatNorm = rNorm;
    restartResidual = rNorm;
    rhoOld = 1.0;
    alpha = 1.0;
    omega = 1.0;
    rho = o[0];
    rhoTerms = o[0];
    ++restarts;
    if (leader) P.out[O_RESTARTS] = (double)restarts;
    outcome = 0;
    return true;
  };
  while (completed < P.max_it) {
    const int64_t iter = completed + 1;
    if (!isfinite(rho)) return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    if (cancelled(rho, rHatNorm, rNorm, rhoTerms)) {
      int oc;
      if (!restart(oc)) return;
      if (oc == 0) continue;
      if (oc == 1) return finish(CFDB_SOLVER_CONVERGED, completed, rNorm);
      return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    }
    const double beta = (rho / rhoOld) * (alpha / omega);
    if (!isfinite(beta)) return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    // p = r + (p - v*omega)*beta
    for (int64_t c = c0 + tid; c < c1; c += kThreads)
      P.p[c] = __ldcg(P.r + c) + (__ldcg(P.p + c) - __ldcg(P.v + c) * omega) * beta;
    if (!T.sync()) return;
    // v = A pHat; (rHat, v), |v|^2, sum |rHat_i v_i|
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      int i, j, k;
      coords(c, i, j, k);
      const double vv = inv ? spmv_row_prec(M, P.p, inv, c, i, j, k) : spmv_row(M, P.p, c, i, j, k);
      P.v[c] = vv;
      const double rh = __ldcg(P.rh + c);
      d0 += rh * vv;
      d1 += vv * vv;
      d2 += fabs(rh * vv);
    }
    if (!reduce3(d0, d1, d2, tot)) return;
    const double rHatDotV = tot[0];
    if (!isfinite(rHatDotV)) return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    if (cancelled(rHatDotV, rHatNorm, sqrt(tot[1]), tot[2])) {
      int oc;
      if (!restart(oc)) return;
      if (oc == 0) continue;
      if (oc == 1) return finish(CFDB_SOLVER_CONVERGED, completed, rNorm);
      return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    }
    alpha = rho / rHatDotV;
    if (!isfinite(alpha)) return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    // s = r - v*alpha; |s|^2
    double ss = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      const double sv = __ldcg(P.r + c) - __ldcg(P.v + c) * alpha;
      P.s[c] = sv;
      ss += sv * sv;
    }
    if (!reduce3(ss, 0.0, 0.0, tot)) return;
    const double sNorm = sqrt(tot[0]);
    if (!isfinite(sNorm)) {
      push(sNorm);
      return finish(CFDB_SOLVER_NONFINITE_RESIDUAL, iter, sNorm);
    }
    if (conv(sNorm)) {
      for (int64_t c = c0 + tid; c < c1; c += kThreads) {
        const double ph = inv ? __ldcg(P.p + c) * __ldg(inv + c) : __ldcg(P.p + c);
        P.x[c] = P.x[c] + ph * alpha;
      }
      push(sNorm);
      return finish(CFDB_SOLVER_CONVERGED, iter, sNorm);
    }
    // t = A sHat; t.t, t.s, sum |t_i s_i|
    double e0 = 0.0, e1 = 0.0, e2 = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      int i, j, k;
      coords(c, i, j, k);
      const double tv = inv ? spmv_row_prec(M, P.s, inv, c, i, j, k) : spmv_row(M, P.s, c, i, j, k);
      P.t[c] = tv;
      const double sv = __ldcg(P.s + c);
      e0 += tv * tv;
      e1 += tv * sv;
      e2 += fabs(tv * sv);
    }
    if (!reduce3(e0, e1, e2, tot)) return;
    const double tDotT = tot[0], tDotS = tot[1];
    if (!isfinite(tDotT) || tDotT < DBL_MIN) return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    if (!isfinite(tDotS)) return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    if (cancelled(tDotS, sqrt(tDotT), sNorm, tot[2])) {
      int oc;
      if (!restart(oc)) return;
      if (oc == 0) continue;
      if (oc == 1) return finish(CFDB_SOLVER_CONVERGED, completed, rNorm);
      return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    }
    omega = tDotS / tDotT;
    if (!isfinite(omega)) return finish(CFDB_SOLVER_BREAKDOWN, completed, rNorm);
    // x += pHat*alpha; x += sHat*omega; r = s - t*omega; |r|^2, (rHat, r), sum |rHat_i r_i|
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      const double ivc = inv ? __ldg(inv + c) : 1.0;
      const double ph = inv ? __ldcg(P.p + c) * ivc : __ldcg(P.p + c);
      const double sv = __ldcg(P.s + c);
      const double sh = inv ? sv * ivc : sv;
      double xv = P.x[c] + ph * alpha;
      xv = xv + sh * omega;
      P.x[c] = xv;
      const double rn = sv - __ldcg(P.t + c) * omega;
      P.r[c] = rn;
      const double rh = __ldcg(P.rh + c);
      f0 += rn * rn;
      f1 += rh * rn;
      f2 += fabs(rh * rn);
    }
    if (!reduce3(f0, f1, f2, tot)) return;
    const double res = sqrt(tot[0]);
    rNorm = res;
    if (!isfinite(res)) {
      push(res);
      return finish(CFDB_SOLVER_NONFINITE_RESIDUAL, iter, res);
    }
    completed = iter;
    push(res);
    lastHist = res;
    if (conv(res)) return finish(CFDB_SOLVER_CONVERGED, iter, res);
    rhoOld = rho;
    rho = tot[1];
    rhoTerms = tot[2];
  }
  finish(CFDB_SOLVER_MAX_ITERATIONS, completed, lastHist);
}

// The FP32 product of the FP32 copy of the matrix with v (same column order
// as spmv_row).
__device__ __forceinline__ float spmv_row32(const StencilMatrix& M, float* const (&m)[7],
                                            const float* v, int64_t c, int i, int j, int k) {
  float sum = 0.f;
  if (M.dim == 3 && k > 0) sum += m[5][c] * __ldcg(v + c - M.sz);
  if (j > 0) sum += m[3][c] * __ldcg(v + c - M.sy);
  if (i > 0) sum += m[1][c] * __ldcg(v + c - 1);
  sum += m[0][c] * __ldcg(v + c);
  if (i < M.nx - 1) sum += m[2][c] * __ldcg(v + c + 1);
  if (j < M.ny - 1) sum += m[4][c] * __ldcg(v + c + M.sy);
  if (M.dim == 3 && k < M.nz - 1) sum += m[6][c] * __ldcg(v + c + M.sz);
  return sum;
}

// Mixed-precision CG (+ Jacobi) that keeps one Krylov space: the matrix is
// copied to FP32 once per solve; the direction p and q = A p live in FP32
// and the inner product A p runs on the FP32 copy, while x, r and every
// reduction stay FP64.  The recurrence residual is replaced by the FP64 true
// residual b - A x (the "reliable updates" of van der Vorst and Ye, 2000)
// after every ten-fold drop since the last replacement, whenever the
// recurrence meets the tolerance, and at the iteration cap, so the solve
// only stops as converged on an FP64 true residual.  Breakdown and
// non-finite tests are those of the FP64 CG above.
template <class Team>
__device__ void cg_mixed_run(const SParams& P, const Team& T) {
  __shared__ double red[3 * 32];
  const StencilMatrix& M = P.M;
  const int B = T.size(), blk = T.rank(), tid = threadIdx.x;
  const bool leader = (blk == 0 && tid == 0);
  const int64_t n = M.n;
  const int64_t c0 = n * blk / B, c1 = n * (blk + 1) / B;
  int round = 0;
  auto part = [&]() { return P.partials + (size_t)(round & 1) * 3 * B; };
  auto coords = [&](int64_t c, int& i, int& j, int& k) {
    i = (int)(c % M.nx);
    j = (int)((c / M.nx) % M.ny);
    k = (int)(c / M.sz);
  };
  const double* inv = M.inv;
  float* const m[7] = {P.m32[0], P.m32[1], P.m32[2], P.m32[3], P.m32[4], P.m32[5], P.m32[6]};
  float* const p32 = P.p32;
  float* const v32 = P.v32;
  auto reduce3 = [&](double a0, double a1, double a2, double (&o)[3]) -> bool {
    double a[3] = {a0, a1, a2};
    block_sum<3>(a, red);
    if (tid == 0) {
      part()[3 * blk] = a[0];
      part()[3 * blk + 1] = a[1];
      part()[3 * blk + 2] = a[2];
    }
    if (!T.sync()) return false;
    grid_total<3>(part(), 3, B, o, red);
    ++round;
    return true;
  };
  auto finish = [&](int status, int64_t it, double fin, int64_t reps) {
    if (leader) {
      P.out[O_STATUS] = status;
      P.out[O_ITER] = (double)it;
      P.out[O_FINAL] = fin;
      P.out[O_REPLACEMENTS] = (double)reps;
    }
  };
  // FP64 true residual r = b - A x; returns (r.r, r.z) through the team
  auto true_residual = [&](double (&o)[3]) -> bool {
    double a0 = 0.0, a1 = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      int i, j, k;
      coords(c, i, j, k);
      const double rn = __ldg(P.b + c) - spmv_row(M, P.x, c, i, j, k);
      P.r[c] = rn;
      a0 += rn * rn;
      a1 += rn * (inv ? __ldg(inv + c) * rn : rn);
    }
    return reduce3(a0, a1, 0.0, o);
  };

  // ---- the FP32 copy of the matrix (published to the team by the first
  // reduction's barrier), then r = b - A x
  for (int64_t c = c0 + tid; c < c1; c += kThreads) {
    m[0][c] = (float)__ldg(M.diag + c);
#pragma unroll
    for (int q = 0; q < 6; ++q)
      if (q < 2 * M.dim) m[1 + q][c] = (float)__ldg(M.off[q] + c);
  }
  double tot[3];
  if (!true_residual(tot)) return;
  const double b0 = sqrt(tot[0]);
  if (leader) {
    P.out[O_B0] = b0;
    P.out[O_RESTARTS] = 0;
    if (P.hist_cap > 0) P.hist[0] = b0;
  }
  auto conv = [&](double res) {
    return (res <= P.abs_tol) || ((b0 > 0.0) && (res / b0 <= P.rel_tol));
  };
  if (b0 == 0.0 || conv(b0)) return finish(CFDB_SOLVER_CONVERGED, 0, b0, 0);
  double rz = tot[1];
  if (!isfinite(rz)) return finish(CFDB_SOLVER_BREAKDOWN, 0, b0, 0);
  double res_cur = b0, res_rep = b0, beta = 0.0;
  int64_t reps = 0;
  for (int64_t it = 1; it <= P.max_it; ++it) {
    // p = z + beta p (FP32), z = M^-1 r rounded to FP32
    const float bf = (float)beta;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      const float z = (float)(inv ? __ldg(inv + c) * __ldcg(P.r + c) : __ldcg(P.r + c));
      p32[c] = (it == 1) ? z : fmaf(bf, __ldcg(p32 + c), z);
    }
    if (!T.sync()) return;
    double pap = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      int i, j, k;
      coords(c, i, j, k);
      const float ap = spmv_row32(M, m, p32, c, i, j, k);
      v32[c] = ap;
      pap += (double)__ldcg(p32 + c) * (double)ap;
    }
    if (!reduce3(pap, 0.0, 0.0, tot)) return;
    const double pAp = tot[0];
    const double alpha = rz / pAp;
    if (!isfinite(pAp) || fabs(pAp) < 1.0e-30 || !isfinite(alpha))
      return finish(CFDB_SOLVER_BREAKDOWN, it - 1, res_cur, reps);
    double rr = 0.0, rzn = 0.0;
    for (int64_t c = c0 + tid; c < c1; c += kThreads) {
      P.x[c] = fma(alpha, (double)__ldcg(p32 + c), P.x[c]);
      const double rn = fma(-alpha, (double)__ldcg(v32 + c), __ldcg(P.r + c));
      P.r[c] = rn;
      rr += rn * rn;
      rzn += rn * (inv ? __ldg(inv + c) * rn : rn);
    }
    if (!reduce3(rr, rzn, 0.0, tot)) return;
    double res = sqrt(tot[0]);
    if (isfinite(res) && (conv(res) || res <= 0.1 * res_rep || it == P.max_it)) {
      if (!true_residual(tot)) return;
      res = sqrt(tot[0]);
      res_rep = res;
      ++reps;
    }
    if (leader && it < P.hist_cap) P.hist[it] = res;
    if (!isfinite(res)) return finish(CFDB_SOLVER_NONFINITE_RESIDUAL, it, res, reps);
    res_cur = res;
    if (conv(res)) return finish(CFDB_SOLVER_CONVERGED, it, res, reps);
    beta = tot[1] / rz;
    if (!isfinite(tot[1]) || !isfinite(beta)) return finish(CFDB_SOLVER_BREAKDOWN, it, res, reps);
    rz = tot[1];
  }
  return finish(CFDB_SOLVER_MAX_ITERATIONS, P.max_it, res_cur, reps);
}

}  // namespace krylov
}  // namespace cfdb
