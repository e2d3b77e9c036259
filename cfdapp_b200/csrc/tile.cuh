// Tile passes of the p' kernels: a block stages a TX x TY x TZ chunk of cells
// plus a one-cell halo in shared memory with a burst of independent
// L2-coherent loads (ld.global.cg: data other blocks wrote in the previous
// sweep is never served from a stale L1 line), then computes the interior
// from shared memory.
//
// Work split: the (x,y) plane is cut into columns of TX x TY cells; the pass
// is the list of (column, z-plane) items, cut into B equal contiguous ranges
// (one per block, deterministic), each processed in chunks of <= TZ planes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "poperator.cuh"

namespace cfdb {

template <int TX_, int TY_, int TZ_>
struct TileShape {
  static constexpr int TX = TX_, TY = TY_, TZ = TZ_;
  static constexpr bool D3 = (TY_ > 1);
  static constexpr int OY = D3 ? 1 : 0;          // y halo width
  static constexpr int BX = TX + 2, BY = TY + 2 * OY, BZ = TZ + 2;
  static constexpr int BOX = BX * BY * BZ;       // staged elements per chunk
};

using Tile2D = TileShape<256, 1, 16>;
using Tile3D = TileShape<32, 8, 16>;

struct Chunk {
  int i0, j0, z0, z1;  // interior origin and plane range [z0, z1)
};

struct ColumnSplit {
  int cols_x, cols_y;
  int64_t items;  // columns * nz
};

template <class S>
inline ColumnSplit make_split(int nx, int ny, int nz) {
  ColumnSplit c;
  c.cols_x = (nx + S::TX - 1) / S::TX;
  c.cols_y = (ny + S::TY - 1) / S::TY;
  c.items = (int64_t)c.cols_x * c.cols_y * nz;
  return c;
}

// Calls f(Chunk) for every chunk of block b of B.
template <class S, typename F>
__device__ __forceinline__ void for_chunks(const ColumnSplit& cs, int nz, int b, int B, F f) {
  const int64_t w0 = cs.items * b / B, w1 = cs.items * (b + 1) / B;
  int64_t w = w0;
  while (w < w1) {
    const int64_t col = w / nz;
    const int z = (int)(w % nz);
    int64_t len = w1 - w;
    if (len > nz - z) len = nz - z;
    if (len > S::TZ) len = S::TZ;
    Chunk c;
    c.i0 = (int)(col % cs.cols_x) * S::TX;
    c.j0 = (int)(col / cs.cols_x) * S::TY;
    c.z0 = z;
    c.z1 = z + (int)len;
    f(c);
    w += len;
  }
}

// Stages make(fetch(i,j,k,idx), i, j, k) for every in-domain cell of the
// chunk box into smem (box layout x fastest); out-of-domain entries are 0.
// Loads are issued in batches of K independent fetches per thread before any
// is consumed, so each thread keeps K (times the words per fetch) loads in
// flight instead of one.
template <class S, int K, typename T, typename Fetch, typename Make>
__device__ __forceinline__ void stage_box(const OpView<T>& A, const Chunk& c, T* box, Fetch fetch,
                                          Make make) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nth = blockDim.x * blockDim.y;
  const int bz = c.z1 - c.z0 + 2;
  const int n = S::BX * S::BY * bz;
  using V = decltype(fetch(0, 0, 0, (int64_t)0));
  auto coords = [&](int e, int& i, int& j, int& k) {
    i = c.i0 - 1 + e % S::BX;
    j = c.j0 - S::OY + (e / S::BX) % S::BY;
    k = c.z0 - 1 + e / (S::BX * S::BY);
    return (e < n) && i >= 0 && i < A.nx && j >= 0 && j < A.ny && k >= 0 && k < A.nz;
  };
  for (int e0 = tid; e0 < n; e0 += nth * K) {
    V v[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
      int i, j, k;
      if (coords(e0 + q * nth, i, j, k)) v[q] = fetch(i, j, k, i + (int64_t)A.nx * (j + (int64_t)A.ny * k));
    }
#pragma unroll
    for (int q = 0; q < K; ++q) {
      const int e = e0 + q * nth;
      int i, j, k;
      const bool in = coords(e, i, j, k);
      if (e < n) box[e] = in ? make(v[q], i, j, k) : T(0);
    }
  }
}

// Visits the interior cells of the chunk in batches of K per thread:
// fetch(idx) issues the cell's global loads (all K before any use), then
// f(i, j, k, idx, e, fetched) computes, e being the box offset of the cell
// (neighbours at e +- 1, e +- BX, e +- BX*BY).
template <class S, int K, typename T, typename Fetch, typename F>
__device__ __forceinline__ void for_interior(const OpView<T>& A, const Chunk& c, Fetch fetch, F f) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nth = blockDim.x * blockDim.y;
  const int n = S::TX * S::TY * (c.z1 - c.z0);
  using V = decltype(fetch((int64_t)0));
  auto coords = [&](int q, int& i, int& j, int& k, int& e) {
    const int qx = q % S::TX, qy = (q / S::TX) % S::TY, qz = q / (S::TX * S::TY);
    i = c.i0 + qx;
    j = c.j0 + qy;
    k = c.z0 + qz;
    e = (qx + 1) + S::BX * ((qy + S::OY) + S::BY * (qz + 1));
    return (q < n) && i < A.nx && j < A.ny;
  };
  for (int q0 = tid; q0 < n; q0 += nth * K) {
    V v[K];
#pragma unroll
    for (int u = 0; u < K; ++u) {
      int i, j, k, e;
      if (coords(q0 + u * nth, i, j, k, e)) v[u] = fetch(i + (int64_t)A.nx * (j + (int64_t)A.ny * k));
    }
#pragma unroll
    for (int u = 0; u < K; ++u) {
      int i, j, k, e;
      if (coords(q0 + u * nth, i, j, k, e))
        f(i, j, k, i + (int64_t)A.nx * (j + (int64_t)A.ny * k), e, v[u]);
    }
  }
}

template <typename T>
struct Pair {
  T a, b;
};

template <class S, typename T>
__device__ __forceinline__ T apply_box(const Coef<T>& c, const T* box, int e) {
  const T v = box[e];
  const T w = box[e - 1], ee = box[e + 1];
  const T s = S::D3 ? box[e - S::BX] : T(0);
  const T n = S::D3 ? box[e + S::BX] : T(0);
  const T b = box[e - S::BX * S::BY], t = box[e + S::BX * S::BY];
  return apply_coef(c, v, w, ee, s, n, b, t);
}

}  // namespace cfdb
