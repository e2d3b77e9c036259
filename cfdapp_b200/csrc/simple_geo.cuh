// Geometry and boundary data of a Cartesian SIMPLE case, evaluated with the
// reference's own expressions (MeshGrading.cpp AxisSpacing::uniform /
// fromNodes center/node/width; MeshGeometry.cpp:513-552, 1047-1140, 197-284)
// so the stage kernels reproduce the reference's arithmetic.  An axis is
// either uniform (spacing delta, createCartesian2D/3D) or given by its node
// coordinates (a rectilinear mesh: createRectilinear2D / createGraded2D,
// MeshGeometry.hpp:228-240), in which case cell widths, face areas and cell
// volumes vary along it.  Shared by host and device; passed to kernels by
// value.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

namespace cfdb {

enum { VBC_WALL = 0, VBC_MOVING_WALL = 1, VBC_INLET = 2, VBC_OUTLET = 3 };
enum { PBC_FIXED_GRADIENT = 0, PBC_FIXED_VALUE = 1 };
enum { SCHEME_UPWIND = 0, SCHEME_CENTRAL = 1, SCHEME_LUD = 2, SCHEME_QUICK = 3 };

// Boundary-side quantities (per axis, side) of the boundary-consistent
// Green-Gauss face value (Gradient.cpp:104-162) and of the wall three-point
// diffusion stencil (NonOrthogonalDiffusion.cpp:64-103).
struct SideGeo {
  int valid;
  double L, w, tb, offset, h1, h2, deltaP, deltaF;
  int stencil_ok;
};

struct SGeo {
  int dim;
  int n[3];
  int64_t stride[3];
  double delta[3];
  // node coordinates of a non-uniform axis (n[a] + 1 values; host or device
  // memory to match where the SGeo is used), null for a uniform axis
  const double* node[3];
  double area[3];  // face areas and cell volume of an all-uniform grid
  double vol;
  int64_t nc, nf;
  int64_t foff[3];
  SideGeo side[3][2];
  int transfer;  // the boundary-consistent gradient needs its tangential sweeps
  int vtype[6];
  double vvalue[6][3];
  int ptype[6];
  double pvalue[6];
};

__host__ __device__ inline double g_center(const SGeo& G, int a, int64_t i) {
  return G.node[a] ? 0.5 * (G.node[a][i] + G.node[a][i + 1]) : ((double)i + 0.5) * G.delta[a];
}
__host__ __device__ inline double g_node(const SGeo& G, int a, int64_t i) {
  return G.node[a] ? G.node[a][i] : (double)i * G.delta[a];
}
__host__ __device__ inline double g_width(const SGeo& G, int a, int64_t i) {
  return G.node[a] ? G.node[a][i + 1] - G.node[a][i] : G.delta[a];
}
__host__ __device__ inline bool g_uniform(const SGeo& G) {
  return !G.node[0] && !G.node[1] && !G.node[2];
}
// Area of the axis-a faces of cell ijk: the widths of the other axes (a 2D
// x-face's area vector is (+-height, 0), a y-face's (0, +-width)).
__host__ __device__ inline double g_area(const SGeo& G, int a, const int ijk[3]) {
  if (g_uniform(G)) return G.area[a];
  if (G.dim == 2) return g_width(G, 1 - a, ijk[1 - a]);
  if (a == 0) return g_width(G, 1, ijk[1]) * g_width(G, 2, ijk[2]);
  if (a == 1) return g_width(G, 0, ijk[0]) * g_width(G, 2, ijk[2]);
  return g_width(G, 0, ijk[0]) * g_width(G, 1, ijk[1]);
}
// Volume of cell ijk (width x height [x depth]).
__host__ __device__ inline double g_vol(const SGeo& G, const int ijk[3]) {
  if (g_uniform(G)) return G.vol;
  const double v = g_width(G, 0, ijk[0]) * g_width(G, 1, ijk[1]);
  return G.dim == 2 ? v : v * g_width(G, 2, ijk[2]);
}
// Internal face at coordinate f along a (owner f-1, neighbour f).
__host__ __device__ inline double g_dpf(const SGeo& G, int a, int64_t f) {
  return fabs(g_node(G, a, f) - g_center(G, a, f - 1));
}
__host__ __device__ inline double g_dnf(const SGeo& G, int a, int64_t f) {
  return fabs(g_node(G, a, f) - g_center(G, a, f));
}
__host__ __device__ inline double g_dpn(const SGeo& G, int a, int64_t f) {
  return fabs(g_center(G, a, f) - g_center(G, a, f - 1));
}
__host__ __device__ inline double g_dbnd(const SGeo& G, int a, int s) {
  return s == 0 ? fabs(g_node(G, a, 0) - g_center(G, a, 0))
                : fabs(g_node(G, a, G.n[a]) - g_center(G, a, G.n[a] - 1));
}
// interpolateInternalFace, scalar (Interpolation.cpp:21-30) and vector (:32-41).
__host__ __device__ inline double g_interp_s(const SGeo& G, int a, int64_t f, double phiP,
                                             double phiN) {
  const double dPf = g_dpf(G, a, f), dNf = g_dnf(G, a, f);
  return ((dNf * phiP) + (dPf * phiN)) / (dPf + dNf);
}
__host__ __device__ inline double g_interp_v(const SGeo& G, int a, int64_t f, double uP,
                                             double uN) {
  const double dPf = g_dpf(G, a, f), dNf = g_dnf(G, a, f);
  return ((uP * dNf) + (uN * dPf)) * (1.0 / (dPf + dNf));
}

__host__ __device__ inline void g_coords(const SGeo& G, int64_t c, int ijk[3]) {
  ijk[0] = (int)(c % G.n[0]);
  ijk[1] = (int)((c / G.n[0]) % G.n[1]);
  ijk[2] = (int)(c / ((int64_t)G.n[0] * G.n[1]));
}

__host__ __device__ inline double g_vol_c(const SGeo& G, int64_t c) {
  if (g_uniform(G)) return G.vol;
  int ijk[3];
  g_coords(G, c, ijk);
  return g_vol(G, ijk);
}

// Global id of the face of cell ijk on axis a, side s.
__host__ __device__ inline int64_t g_face_of(const SGeo& G, const int ijk[3], int a, int s) {
  const int64_t i = ijk[0] + (a == 0 ? s : 0);
  const int64_t j = ijk[1] + (a == 1 ? s : 0);
  const int64_t k = ijk[2] + (a == 2 ? s : 0);
  if (a == 0) return i + (int64_t)(G.n[0] + 1) * (j + (int64_t)G.n[1] * k);
  if (a == 1) return G.foff[1] + i + (int64_t)G.n[0] * (j + (int64_t)(G.n[1] + 1) * k);
  return G.foff[2] + i + (int64_t)G.n[0] * (j + (int64_t)G.n[1] * k);
}

struct FaceInfo {
  int a;
  int64_t f, low, high;
};

__host__ __device__ inline FaceInfo g_face_decode(const SGeo& G, int64_t id) {
  FaceInfo fi;
  int64_t i, j, k;
  if (id < G.foff[1]) {
    fi.a = 0;
    i = id % (G.n[0] + 1);
    j = (id / (G.n[0] + 1)) % G.n[1];
    k = id / ((int64_t)(G.n[0] + 1) * G.n[1]);
    fi.f = i;
  } else if (G.dim == 2 || id < G.foff[2]) {
    const int64_t r = id - G.foff[1];
    fi.a = 1;
    i = r % G.n[0];
    j = (r / G.n[0]) % (G.n[1] + 1);
    k = r / ((int64_t)G.n[0] * (G.n[1] + 1));
    fi.f = j;
  } else {
    const int64_t r = id - G.foff[2];
    fi.a = 2;
    i = r % G.n[0];
    j = (r / G.n[0]) % G.n[1];
    k = r / ((int64_t)G.n[0] * G.n[1]);
    fi.f = k;
  }
  int64_t c[3] = {i, j, k};
  c[fi.a] = fi.f;
  const int64_t base = c[0] + (int64_t)G.n[0] * (c[1] + (int64_t)G.n[1] * c[2]);
  fi.high = (fi.f < G.n[fi.a]) ? base : -1;
  fi.low = (fi.f > 0) ? base - G.stride[fi.a] : -1;
  return fi;
}

// Area of a face given its decoded info (from the cell on either side).
__host__ __device__ inline double g_face_area(const SGeo& G, const FaceInfo& fi) {
  if (g_uniform(G)) return G.area[fi.a];
  int ijk[3];
  g_coords(G, fi.high >= 0 ? fi.high : fi.low, ijk);
  return g_area(G, fi.a, ijk);
}

__host__ __device__ inline int g_vbc_prescribed(int t) {
  return t == VBC_WALL || t == VBC_MOVING_WALL || t == VBC_INLET;
}

// Boundary velocity component (Wall.cpp:8, MovingWall.cpp:22, Inlet.cpp:19, Outlet.cpp:8).
__host__ __device__ inline double g_vbc_value(const SGeo& G, int patch, int comp, double owner) {
  switch (G.vtype[patch]) {
    case VBC_WALL: return 0.0;
    case VBC_MOVING_WALL:
    case VBC_INLET: return G.vvalue[patch][comp];
    default: return owner;
  }
}

// Host-side construction (simple.cu).
struct SimpleCaseDesc;
}  // namespace cfdb
