// Geometry and boundary data of a uniform Cartesian SIMPLE case, evaluated
// with the reference's own expressions (MeshGrading.cpp AxisSpacing::uniform
// center/node/width; MeshGeometry.cpp:513-552, 1047-1140, 197-284) so the
// stage kernels reproduce the reference's arithmetic.  Shared by host and
// device; passed to kernels by value.
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
  double area[3];
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
  return ((double)i + 0.5) * G.delta[a];
}
__host__ __device__ inline double g_node(const SGeo& G, int a, int64_t i) {
  return (double)i * G.delta[a];
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
