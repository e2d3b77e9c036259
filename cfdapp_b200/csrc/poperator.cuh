// Matrix-free p' operator on a uniform Cartesian grid and the plane-marching
// tile traversal shared by the p' kernels.
//
// Kernel space is always three-dimensional (nx, ny, nz) with z the marching
// axis: a 2D grid (nx, ny) maps to (nx, 1, ny) with no y-faces, so one code
// path serves the 5- and 7-point operators.  A thread block covers a PX x PY
// patch of an (x,y) plane and marches along z through its assigned planes,
// keeping the z-neighbours of its own cells in registers and staging the
// plane (with a one-cell x/y halo) in shared memory; every global element is
// loaded once per block pass (halo cells once more by the neighbouring
// block), so DRAM traffic stays at one read per word per sweep.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace cfdb {

// Face coefficients D_f of the p' operator.  Either per-axis tables (uniform
// response, `t*` of length n_axis+1, boundary entries 0 for Neumann) or
// per-face arrays (`f*`, global face layout per axis); a null face array
// falls back to the table.
template <typename T>
struct OpView {
  int nx, ny, nz;
  const T* tx;
  const T* ty;
  const T* tz;
  const T* fx;
  const T* fy;
  const T* fz;
  int64_t ref;
  int pinned;
};

template <typename T>
struct Coef {
  T xl, xh, yl, yh, zl, zh;  // couplings to the six neighbours (0 across a boundary)
  T diag, inv;               // diagonal (face-order sum incl. Dirichlet faces) and 1/diag
};

// Correctly rounded reciprocal (== 1/x in IEEE round-to-nearest).
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }

template <typename T>
__device__ __forceinline__ Coef<T> load_coef(const OpView<T>& A, int i, int j, int k) {
  Coef<T> c;
  if (A.fx) {
    const int64_t bx = i + (int64_t)(A.nx + 1) * (j + (int64_t)A.ny * k);
    c.xl = __ldg(A.fx + bx);
    c.xh = __ldg(A.fx + bx + 1);
  } else {
    c.xl = __ldg(A.tx + i);
    c.xh = __ldg(A.tx + i + 1);
  }
  if (A.fy) {
    const int64_t by = i + (int64_t)A.nx * (j + (int64_t)(A.ny + 1) * k);
    c.yl = __ldg(A.fy + by);
    c.yh = __ldg(A.fy + by + A.nx);
  } else {
    c.yl = __ldg(A.ty + j);
    c.yh = __ldg(A.ty + j + 1);
  }
  if (A.fz) {
    const int64_t bz = i + (int64_t)A.nx * (j + (int64_t)A.ny * k);
    c.zl = __ldg(A.fz + bz);
    c.zh = __ldg(A.fz + bz + (int64_t)A.nx * A.ny);
  } else {
    c.zl = __ldg(A.tz + k);
    c.zh = __ldg(A.tz + k + 1);
  }
  const int64_t idx = i + (int64_t)A.nx * (j + (int64_t)A.ny * k);
  if (A.pinned && idx == A.ref) {
    c.xl = c.xh = c.yl = c.yh = c.zl = c.zh = T(0);
    c.diag = T(1);
    c.inv = T(1);
    return c;
  }
  // The reference sums the diagonal in face order: x-low, x-high, y-low,
  // y-high, z-low, z-high (PressureCorrectionEquation.cpp:266-298).
  c.diag = ((((c.xl + c.xh) + c.yl) + c.yh) + c.zl) + c.zh;
  c.inv = rcp_rn(c.diag);
  if (i == 0) c.xl = T(0);
  if (i == A.nx - 1) c.xh = T(0);
  if (j == 0) c.yl = T(0);
  if (j == A.ny - 1) c.yh = T(0);
  if (k == 0) c.zl = T(0);
  if (k == A.nz - 1) c.zh = T(0);
  return c;
}

template <typename T>
__device__ __forceinline__ T apply_coef(const Coef<T>& c, T v, T w, T e, T s, T n, T b, T t) {
  T off = c.xl * w;
  off = fma(c.xh, e, off);
  off = fma(c.yl, s, off);
  off = fma(c.yh, n, off);
  off = fma(c.zl, b, off);
  off = fma(c.zh, t, off);
  return fma(c.diag, v, -off);
}

// Work split of a pass: items = tiles * nz (tile-major, plane-minor), block b
// handles [items*b/B, items*(b+1)/B) as up to a few contiguous plane segments.
struct Tiling {
  int tiles_x, tiles_y;
  int64_t items;
};

template <int PX, int PY>
inline Tiling make_tiling(int nx, int ny, int nz) {
  Tiling t;
  t.tiles_x = (nx + PX - 1) / PX;
  t.tiles_y = (ny + PY - 1) / PY;
  t.items = (int64_t)t.tiles_x * t.tiles_y * nz;
  return t;
}

// Marches the block over planes [k0, k1) of tile `tile`.
//   own(i,j,k)  -> stencil input at an own cell
//   halo(i,j,k) -> stencil input at an in-domain halo cell
//   cell(i,j,k, idx, vC, vW, vE, vS, vN, vB, vT) -> work of an own cell
// Coefficients are not carried between planes (they are re-read where
// needed, from L1) to keep the register footprint low enough for several
// resident blocks per SM.
template <typename T, int PX, int PY, typename Own, typename Halo, typename Cell>
__device__ __forceinline__ void march(const OpView<T>& A, const Tiling& tl, int64_t tile, int k0,
                                      int k1, T (*buf)[PY + 2][PX + 2], Own own, Halo halo,
                                      Cell cell) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tix = (int)(tile % tl.tiles_x), tiy = (int)(tile / tl.tiles_x);
  const int i = tix * PX + tx, j = tiy * PY + ty;
  const bool act = (i < A.nx) && (j < A.ny);
  T vprev = T(0), vcur = T(0);
  if (act) {
    if (k0 > 0) vprev = halo(i, j, k0 - 1);
    vcur = own(i, j, k0);
  }
  for (int k = k0; k < k1; ++k) {
    T vnext = T(0);
    if (act && k + 1 < A.nz) vnext = own(i, j, k + 1);
    T(*s)[PX + 2] = buf[k & 1];
    s[ty + 1][tx + 1] = vcur;
    if (tx == 0) s[ty + 1][0] = (i > 0 && j < A.ny) ? halo(i - 1, j, k) : T(0);
    if (tx == PX - 1) s[ty + 1][PX + 1] = (i + 1 < A.nx && j < A.ny) ? halo(i + 1, j, k) : T(0);
    if (PY > 1) {
      if (ty == 0) s[0][tx + 1] = (j > 0 && i < A.nx) ? halo(i, j - 1, k) : T(0);
      if (ty == PY - 1) s[PY + 1][tx + 1] = (j + 1 < A.ny && i < A.nx) ? halo(i, j + 1, k) : T(0);
    }
    __syncthreads();
    if (act) {
      const int64_t idx = i + (int64_t)A.nx * (j + (int64_t)A.ny * k);
      // With a single row of threads (PY == 1, the 2D layout) the y-halo rows
      // of the plane buffer are never written: pass zeros, not stale memory.
      const T vs = (PY > 1) ? s[ty][tx + 1] : T(0);
      const T vn = (PY > 1) ? s[ty + 2][tx + 1] : T(0);
      cell(i, j, k, idx, vcur, s[ty + 1][tx], s[ty + 1][tx + 2], vs, vn, vprev, vnext);
    }
    vprev = vcur;
    vcur = vnext;
  }
  __syncthreads();
}

// Iterates the segments of block `b` of `B` over a tiling.
template <typename F>
__device__ __forceinline__ void for_segments(const Tiling& tl, int nz, int b, int B, F f) {
  const int64_t w0 = tl.items * b / B, w1 = tl.items * (b + 1) / B;
  int64_t w = w0;
  while (w < w1) {
    const int64_t tile = w / nz;
    const int k0 = (int)(w % nz);
    const int64_t rem = w1 - w;
    const int k1 = (int)((k0 + rem < nz) ? k0 + rem : nz);
    f(tile, k0, k1);
    w += k1 - k0;
  }
}

}  // namespace cfdb
