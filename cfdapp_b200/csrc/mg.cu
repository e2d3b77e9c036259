// Learned multigrid-shaped preconditioner (see mg.cuh): hierarchy
// construction, the V-cycle kernels, and the FCG(1) solve loop captured as
// one CUDA graph with a device-side WHILE node (the loop runs without a host
// round trip; the last kernel of each iteration decides whether another one
// follows).
//
// Work layout.  Fine levels run one thread per cell, x fastest (coalesced),
// blocks over (x-segment, row) with rows = ny*nz; neighbour reads go through
// L1/L2, so DRAM sees each array about once per kernel.  All levels at or
// below 4096 cells run inside ONE thread block with the level data in shared
// memory (about 130 KB), which removes a dozen launches per cycle.
//
// Reductions are deterministic without a grid barrier: every block stores its
// partial sums, and the last block to finish (atomic ticket) adds all partials
// in block order and publishes the scalars.  Nothing in this file waits on
// another block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "cfdb_internal.cuh"
#include "grid_sync.cuh"
#include "mg.cuh"

namespace cfdb {

MgWeights mg_default_weights(int dim) {
  MgWeights W;
  std::memset(&W, 0, sizeof(W));
  W.dim = dim;
  W.levels = 1;
  W.nu = 2;
  W.coarse_sweeps = 50;
  for (int l = 0; l < kMgMaxLevels; ++l) {
    W.w[l][13] = 0.8f;  // centre tap: damped Jacobi
    W.c[l] = 1.0f;
  }
  return W;
}

#include "mg_trained.inc"

bool mg_weights_valid(const MgWeights& W, std::string* why) {
  auto fail = [&](const char* m) {
    if (why) *why = m;
    return false;
  };
  if (W.dim != 2 && W.dim != 3) return fail("weights: dim must be 2 or 3");
  if (W.levels < 1 || W.levels > kMgMaxLevels) return fail("weights: levels must be 1..16");
  if (W.nu < 1 || W.nu > 8) return fail("weights: nu must be 1..8");
  if (W.coarse_sweeps < 0 || W.coarse_sweeps > 1000) return fail("weights: coarse sweeps 0..1000");
  for (int l = 0; l < W.levels; ++l) {
    if (!std::isfinite(W.c[l])) return fail("weights: non-finite coarse weight");
    for (int t = 0; t < kMgTaps; ++t) {
      if (!std::isfinite(W.w[l][t])) return fail("weights: non-finite kernel tap");
      if (W.w[l][t] != W.w[l][kMgTaps - 1 - t]) return fail("weights: kernels must be point-symmetric");
      if (W.dim == 2 && (t < 9 || t >= 18) && W.w[l][t] != 0.f)
        return fail("weights: 2D kernels use the middle 3x3 plane only");
    }
  }
  return true;
}

MgHierarchy::~MgHierarchy() {
  for (void* p : owned) cudaFree(p);
}

namespace {

constexpr int kMaxBlocks = 148 * 16;
constexpr int64_t kCoarseCells = 4096;
constexpr int kMaxCoarse = 8;
constexpr int kCoarseThreads = 1024;
constexpr size_t kCoarseSmemCap = 200 * 1024;

struct Kern {
  float w[kMgTaps];
};

struct LV {
  int nx, ny, nz;
  const float* fx;
  const float* fy;
  const float* fz;
  const float* isq;
};

__host__ __device__ inline LV lv(const MgLevel& M) {
  return LV{M.n[0], M.n[1], M.n[2], M.f[0], M.f[1], M.f[2], M.isq};
}

Kern kern_of(const MgWeights& W, int l) {
  Kern K;
  std::memcpy(K.w, W.w[std::min(l, W.levels - 1)], sizeof(K.w));
  return K;
}
float cw_of(const MgWeights& W, int l) { return W.c[std::min(l, W.levels - 1)]; }

__device__ __forceinline__ int64_t at(const LV& L, int i, int j, int k) {
  return i + (int64_t)L.nx * (j + (int64_t)L.ny * k);
}

// (A_l x) at (i,j,k); x(q, i, j, k) returns x at linear cell q with
// coordinates (i,j,k).  Boundary face coefficients enter the diagonal only.
template <int DIM, class X>
__device__ __forceinline__ float lap(const LV& L, int i, int j, int k, X x) {
  const int64_t c = at(L, i, j, k);
  const int64_t bx = i + (int64_t)(L.nx + 1) * (j + (int64_t)L.ny * k);
  const int64_t by = i + (int64_t)L.nx * (j + (int64_t)(L.ny + 1) * k);
  const float axl = L.fx[bx], axh = L.fx[bx + 1], ayl = L.fy[by], ayh = L.fy[by + L.nx];
  float d = (axl + axh) + (ayl + ayh);
  float off = 0.f;
  if (i > 0) off += axl * x(c - 1, i - 1, j, k);
  if (i + 1 < L.nx) off += axh * x(c + 1, i + 1, j, k);
  if (j > 0) off += ayl * x(c - L.nx, i, j - 1, k);
  if (j + 1 < L.ny) off += ayh * x(c + L.nx, i, j + 1, k);
  if (DIM == 3) {
    const int64_t plane = (int64_t)L.nx * L.ny;
    const float azl = L.fz[c], azh = L.fz[c + plane];
    d += azl + azh;
    if (k > 0) off += azl * x(c - plane, i, j, k - 1);
    if (k + 1 < L.nz) off += azh * x(c + plane, i, j, k + 1);
  }
  return d * x(c, i, j, k) - off;
}

// isq(c) * sum_o W[o] isq(c+o) v(c+o): the learned smoothing convolution.
template <int DIM, class V>
__device__ __forceinline__ float conv(const LV& L, const Kern& K, int i, int j, int k, V v) {
  float s = 0.f;
#pragma unroll
  for (int dk = -1; dk <= 1; ++dk) {
    if (DIM == 2 && dk != 0) continue;
    const int kk = k + dk;
    if (kk < 0 || kk >= L.nz) continue;
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
      const int jj = j + dj;
      if (jj < 0 || jj >= L.ny) continue;
#pragma unroll
      for (int di = -1; di <= 1; ++di) {
        const int ii = i + di;
        if (ii < 0 || ii >= L.nx) continue;
        const int64_t q = at(L, ii, jj, kk);
        s += K.w[(dk + 1) * 9 + (dj + 1) * 3 + (di + 1)] * (L.isq[q] * v(q));
      }
    }
  }
  return L.isq[at(L, i, j, k)] * s;
}

// Parent (coarse) cell of fine cell (i,j,k).
__device__ __forceinline__ int64_t parent(const LV& C, int i, int j, int k) {
  return (i >> 1) + (int64_t)C.nx * ((j >> 1) + (int64_t)C.ny * (k >> 1));
}

// ------------------------------------------------------------- launch shape

struct Shape {
  dim3 grid, block;
};

Shape cells_shape(int nx, int64_t rows) {
  const int bx = nx >= 96 ? 128 : (nx >= 48 ? 64 : 32);
  const int gx = (nx + bx - 1) / bx;
  const int64_t gy = std::max<int64_t>(1, std::min<int64_t>(rows, std::max(1, kMaxBlocks / gx)));
  return Shape{dim3(gx, (unsigned)gy), dim3(bx)};
}

template <class F>
__device__ __forceinline__ void each_cell(int nx, int ny, int rows, F f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx) return;
  for (int row = blockIdx.y; row < rows; row += gridDim.y) f(i, row % ny, row / ny, (int64_t)row * nx + i);
}

// ----------------------------------------------------------------- FCG state

struct FcgState {
  // set by the host before each solve
  const double* b;
  double* x;
  double abs_tol, rel_tol;
  long long max_it, window;
  // progress
  double b0, res, best;
  double pq, pr, alpha, beta;
  long long it, best_it;
  int status, done;
  unsigned ticket;
};

constexpr int kRunning = -1;

// Block partials -> fixed-order total in the last block; fin(tot) runs in
// thread 0 of that block.  Every thread of the block must call this.
template <int NV, class Fin>
__device__ __forceinline__ void reduce_last(double (&v)[NV], double* partials, unsigned* ticket,
                                            Fin fin) {
  __shared__ double red[32 * NV];
  __shared__ int is_last;
  block_sum<NV>(v, red);
  const int nb = gridDim.x * gridDim.y;
  const int b = blockIdx.x + gridDim.x * blockIdx.y;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[(size_t)b * NV + q] = v[q];
    __threadfence();
    is_last = (atomicAdd(ticket, 1u) == (unsigned)(nb - 1));
  }
  __syncthreads();
  if (is_last) {
    __threadfence();
    double tot[NV];
    grid_total<NV>(partials, NV, nb, tot, red);
    if (threadIdx.x == 0) {
      fin(tot);
      atomicExch(ticket, 0u);
    }
  }
}


// The WHILE node's condition, or nothing when the kernels run outside a
// graph (stream mode: active = 0).
struct Loop {
  cudaGraphConditionalHandle h;
  int active;
};

__device__ __forceinline__ void set_loop(const Loop& lp, unsigned v) {
  if (lp.active) cudaGraphSetConditional(lp.h, v);
}

__device__ __forceinline__ void stop_loop(FcgState* S, const Loop& h, int status) {
  S->status = status;
  S->done = 1;
  set_loop(h, 0);
}

struct Hook {
  const double* q;  // previous A p
  double* partials;
  FcgState* S;
  Loop h;
};

// ------------------------------------------------------------ level kernels

template <int DIM>
__global__ void k_first(LV L, Kern K, const float* __restrict__ r, float* __restrict__ x,
                        int64_t skip) {
  each_cell(L.nx, L.ny, L.ny * L.nz, [&](int i, int j, int k, int64_t c) {
    x[c] = conv<DIM>(L, K, i, j, k, [&](int64_t q) { return q == skip ? 0.f : r[q]; });
  });
}

template <int DIM>
__global__ void k_resid(LV L, const float* __restrict__ x, const float* __restrict__ r,
                        float* __restrict__ res, int64_t skip) {
  each_cell(L.nx, L.ny, L.ny * L.nz, [&](int i, int j, int k, int64_t c) {
    res[c] = (c == skip ? 0.f : r[c]) -
             lap<DIM>(L, i, j, k, [&](int64_t q, int, int, int) { return x[q]; });
  });
}

// res = r - A (x + cw P ec)
template <int DIM>
__global__ void k_prolong_resid(LV L, LV C, const float* __restrict__ ec, float cw,
                                const float* __restrict__ x, const float* __restrict__ r,
                                float* __restrict__ res, int64_t skip) {
  each_cell(L.nx, L.ny, L.ny * L.nz, [&](int i, int j, int k, int64_t c) {
    auto xv = [&](int64_t q, int qi, int qj, int qk) {
      return x[q] + cw * ec[parent(C, qi, qj, qk)];
    };
    res[c] = (c == skip ? 0.f : r[c]) - lap<DIM>(L, i, j, k, xv);
  });
}

// x <- x (+ cw P ec) + S res; at level 0 the last sweep also pins z[skip] =
// r[skip] and, with a hook, accumulates z.q for the FCG coefficient.
template <int DIM, bool HOOK>
__global__ void k_smooth(LV L, LV C, Kern K, const float* __restrict__ ec, float cw,
                         const float* __restrict__ res, float* __restrict__ x, int64_t skip,
                         const float* __restrict__ r, Hook hk) {
  double acc[1] = {0.0};
  each_cell(L.nx, L.ny, L.ny * L.nz, [&](int i, int j, int k, int64_t c) {
    float v = x[c] + conv<DIM>(L, K, i, j, k, [&](int64_t q) { return res[q]; });
    if (ec) v += cw * ec[parent(C, i, j, k)];
    if (c == skip) v = r[c];
    x[c] = v;
    if (HOOK) acc[0] += (double)v * hk.q[c];
  });
  if (HOOK) {
    reduce_last<1>(acc, hk.partials, &hk.S->ticket, [&](const double* tot) {
      FcgState* S = hk.S;
      if (S->it == 0) return;  // the first direction is z itself
      const double beta = tot[0] / S->pq;
      if (!isfinite(beta)) {
        stop_loop(S, hk.h, kLearnedStagnated);
        return;
      }
      S->beta = beta;
    });
  }
}

// rc(C) = sum over the children of C of (r - A x)
template <int DIM>
__global__ void k_resid_restrict(LV L, LV C, const float* __restrict__ x,
                                 const float* __restrict__ r, float* __restrict__ rc, int64_t skip) {
  each_cell(C.nx, C.ny, C.ny * C.nz, [&](int ci, int cj, int ck, int64_t qc) {
    float s = 0.f;
#pragma unroll
    for (int u = 0; u < (DIM == 3 ? 2 : 1); ++u)
#pragma unroll
      for (int v = 0; v < 2; ++v)
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int i = 2 * ci + t, j = 2 * cj + v, k = 2 * ck + u;
          if (i >= L.nx || j >= L.ny || k >= L.nz) continue;
          const int64_t c = at(L, i, j, k);
          s += (c == skip ? 0.f : r[c]) -
               lap<DIM>(L, i, j, k, [&](int64_t q, int, int, int) { return x[q]; });
        }
    rc[qc] = s;
  });
}

// ----------------------------------------------------- coarse-level block

struct CoarseLevel {
  int n[3];
  int cells;
  const float* f[3];  // global sources
  const float* isq;
  float* x_glob;      // global x (written back for the first coarse level)
  const float* r_glob;
  int off[7];         // shared-memory offsets (floats): fx fy fz isq x r res
};

struct CoarsePlan {
  int count;
  int nu, sweeps;
  CoarseLevel lv[kMaxCoarse];
  Kern K[kMaxCoarse];
  float cw[kMaxCoarse];
};

template <int DIM>
__global__ void __launch_bounds__(kCoarseThreads) k_coarse(CoarsePlan P) {
  extern __shared__ float4 smem4[];
  float* sm = reinterpret_cast<float*>(smem4);
  const int tid = threadIdx.x, nt = blockDim.x;
  // stage the levels' coefficients into shared memory
  for (int l = 0; l < P.count; ++l) {
    const CoarseLevel& c = P.lv[l];
    const int nf[3] = {(c.n[0] + 1) * c.n[1] * c.n[2], c.n[0] * (c.n[1] + 1) * c.n[2],
                       DIM == 3 ? c.n[0] * c.n[1] * (c.n[2] + 1) : 0};
    for (int a = 0; a < DIM; ++a)
      for (int q = tid; q < nf[a]; q += nt) sm[c.off[a] + q] = c.f[a][q];
    for (int q = tid; q < c.cells; q += nt) sm[c.off[3] + q] = c.isq[q];
  }
  for (int q = tid; q < P.lv[0].cells; q += nt) sm[P.lv[0].off[5] + q] = P.lv[0].r_glob[q];
  __syncthreads();
  auto level = [&](int l) {
    const CoarseLevel& c = P.lv[l];
    return LV{c.n[0], c.n[1], c.n[2], sm + c.off[0], sm + c.off[1],
              DIM == 3 ? sm + c.off[2] : nullptr, sm + c.off[3]};
  };
  auto X = [&](int l) { return sm + P.lv[l].off[4]; };
  auto R = [&](int l) { return sm + P.lv[l].off[5]; };
  auto RES = [&](int l) { return sm + P.lv[l].off[6]; };
  auto cell_loop = [&](const LV& M, auto f) {
    const int cells = M.nx * M.ny * M.nz;
    for (int c = tid; c < cells; c += nt) {
      const int i = c % M.nx, rest = c / M.nx;
      f(i, rest % M.ny, rest / M.ny, c);
    }
  };
  auto xval = [](const float* x) { return [x](int64_t q, int, int, int) { return x[q]; }; };
  const int last = P.count - 1;
  for (int l = 0; l < last; ++l) {
    const LV M = level(l);
    float* x = X(l);
    const float* r = R(l);
    float* res = RES(l);
    cell_loop(M, [&](int i, int j, int k, int c) {
      x[c] = conv<DIM>(M, P.K[l], i, j, k, [&](int64_t q) { return r[q]; });
    });
    __syncthreads();
    for (int s = 1; s < P.nu; ++s) {
      cell_loop(M, [&](int i, int j, int k, int c) { res[c] = r[c] - lap<DIM>(M, i, j, k, xval(x)); });
      __syncthreads();
      cell_loop(M, [&](int i, int j, int k, int c) {
        x[c] += conv<DIM>(M, P.K[l], i, j, k, [&](int64_t q) { return res[q]; });
      });
      __syncthreads();
    }
    cell_loop(M, [&](int i, int j, int k, int c) { res[c] = r[c] - lap<DIM>(M, i, j, k, xval(x)); });
    __syncthreads();
    const LV Cc = level(l + 1);
    float* rc = R(l + 1);
    cell_loop(Cc, [&](int ci, int cj, int ck, int qc) {
      float s = 0.f;
      for (int u = 0; u < (DIM == 3 ? 2 : 1); ++u)
        for (int v = 0; v < 2; ++v)
          for (int t = 0; t < 2; ++t) {
            const int i = 2 * ci + t, j = 2 * cj + v, k = 2 * ck + u;
            if (i < M.nx && j < M.ny && k < M.nz) s += res[at(M, i, j, k)];
          }
      rc[qc] = s;
    });
    __syncthreads();
  }
  {
    const LV M = level(last);
    float* x = X(last);
    const float* r = R(last);
    float* res = RES(last);
    cell_loop(M, [&](int, int, int, int c) { x[c] = 0.f; });
    __syncthreads();
    for (int s = 0; s < P.sweeps; ++s) {
      cell_loop(M, [&](int i, int j, int k, int c) { res[c] = r[c] - lap<DIM>(M, i, j, k, xval(x)); });
      __syncthreads();
      cell_loop(M, [&](int, int, int, int c) {
        const float is = M.isq[c];
        x[c] += 0.8f * (is * is) * res[c];
      });
      __syncthreads();
    }
  }
  for (int l = last - 1; l >= 0; --l) {
    const LV M = level(l);
    const LV Cc = level(l + 1);
    float* x = X(l);
    const float* r = R(l);
    float* res = RES(l);
    const float* ec = X(l + 1);
    const float cw = P.cw[l];
    cell_loop(M, [&](int i, int j, int k, int c) {
      auto xv = [&](int64_t q, int qi, int qj, int qk) {
        return x[q] + cw * ec[parent(Cc, qi, qj, qk)];
      };
      res[c] = r[c] - lap<DIM>(M, i, j, k, xv);
    });
    __syncthreads();
    cell_loop(M, [&](int i, int j, int k, int c) {
      x[c] += cw * ec[parent(Cc, i, j, k)] +
              conv<DIM>(M, P.K[l], i, j, k, [&](int64_t q) { return res[q]; });
    });
    __syncthreads();
    for (int s = 1; s < P.nu; ++s) {
      cell_loop(M, [&](int i, int j, int k, int c) { res[c] = r[c] - lap<DIM>(M, i, j, k, xval(x)); });
      __syncthreads();
      cell_loop(M, [&](int i, int j, int k, int c) {
        x[c] += conv<DIM>(M, P.K[l], i, j, k, [&](int64_t q) { return res[q]; });
      });
      __syncthreads();
    }
  }
  for (int q = tid; q < P.lv[0].cells; q += nt) P.lv[0].x_glob[q] = X(0)[q];
}

// ------------------------------------------------------ hierarchy build

__global__ void k_faces0(float* out, int e0, int e1, int e2, int axis, const double* full,
                         const double* table) {
  const int64_t m = (int64_t)e0 * e1 * e2;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m;
       q += (int64_t)gridDim.x * blockDim.x) {
    double v;
    if (full) {
      v = full[q];
    } else {
      const int i = (int)(q % e0);
      const int64_t rest = q / e0;
      const int j = (int)(rest % e1), k = (int)(rest / e1);
      v = table[axis == 0 ? i : (axis == 1 ? j : k)];
    }
    out[q] = (float)v;
  }
}

// Coarse faces of axis a: sum of the fine faces they cover.
__global__ void k_agglomerate(MgLevel F, MgLevel C, int a) {
  int ext[3] = {C.n[0], C.n[1], C.n[2]};
  ext[a] += 1;
  int fext[3] = {F.n[0], F.n[1], F.n[2]};
  fext[a] += 1;
  const int64_t m = (int64_t)ext[0] * ext[1] * ext[2];
  const int b1 = (a == 0) ? 1 : 0, b2 = (a == 2) ? 1 : 2;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m;
       q += (int64_t)gridDim.x * blockDim.x) {
    int cc[3];
    cc[0] = (int)(q % ext[0]);
    const int64_t rest = q / ext[0];
    cc[1] = (int)(rest % ext[1]);
    cc[2] = (int)(rest / ext[1]);
    const int fa = (cc[a] == C.n[a]) ? F.n[a] : 2 * cc[a];
    float s = 0.f;
    for (int u = 0; u < 2; ++u)
      for (int v = 0; v < 2; ++v) {
        int fc[3];
        fc[a] = fa;
        fc[b1] = 2 * cc[b1] + u;
        fc[b2] = 2 * cc[b2] + v;
        if (fc[b1] >= F.n[b1] || fc[b2] >= F.n[b2]) continue;
        s += F.f[a][fc[0] + (int64_t)fext[0] * (fc[1] + (int64_t)fext[1] * fc[2])];
      }
    C.f[a][q] = s;
  }
}

template <int DIM>
__global__ void k_isq(MgLevel M) {
  const LV L = lv(M);
  each_cell(L.nx, L.ny, L.ny * L.nz, [&](int i, int j, int k, int64_t c) {
    const float d = lap<DIM>(L, i, j, k, [&](int64_t q, int, int, int) { return q == c ? 1.f : 0.f; });
    M.isq[c] = d > 0.f ? rsqrtf(d) : 0.f;
  });
}

int flat_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, kMaxBlocks));
}

template <int DIM>
void launch_isq(const MgLevel& M, cudaStream_t st) {
  const Shape s = cells_shape(M.n[0], (int64_t)M.n[1] * M.n[2]);
  k_isq<DIM><<<s.grid, s.block, 0, st>>>(M);
}

cfdb_status refresh_values(cfdb_context* ctx, MgHierarchy& H, const FineOperator& op) {
  cudaStream_t st = ctx->stream;
  for (int l = 0; l < H.levels; ++l) {
    MgLevel& M = H.L[l];
    for (int a = 0; a < H.dim; ++a) {
      int e[3] = {M.n[0], M.n[1], M.n[2]};
      e[a] += 1;
      const int64_t m = (int64_t)e[0] * e[1] * e[2];
      if (l == 0)
        k_faces0<<<flat_grid(m), 256, 0, st>>>(M.f[a], e[0], e[1], e[2], a, op.full[a], op.table[a]);
      else
        k_agglomerate<<<flat_grid(m), 256, 0, st>>>(H.L[l - 1], M, a);
    }
    if (H.dim == 2) launch_isq<2>(M, st);
    else launch_isq<3>(M, st);
  }
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx, H.levels * (H.dim + 1));
  return CFDB_OK;
}

// --------------------------------------------------------- cycle enqueue

size_t up4(int64_t n) { return (size_t)((n + 3) & ~(int64_t)3); }

size_t coarse_bytes(const MgHierarchy& H, int from) {
  size_t floats = 0;
  for (int l = from; l < H.levels; ++l) {
    const MgLevel& M = H.L[l];
    floats += up4((int64_t)(M.n[0] + 1) * M.n[1] * M.n[2]) + up4((int64_t)M.n[0] * (M.n[1] + 1) * M.n[2]);
    if (H.dim == 3) floats += up4((int64_t)M.n[0] * M.n[1] * (M.n[2] + 1));
    floats += 4 * up4(M.cells);
  }
  return floats * sizeof(float);
}

CoarsePlan coarse_plan(const MgHierarchy& H, const MgWeights& W) {
  CoarsePlan P;
  std::memset(&P, 0, sizeof(P));
  P.count = H.levels - H.coarse_from;
  P.nu = W.nu;
  P.sweeps = W.coarse_sweeps;
  int off = 0;
  auto take = [&](int64_t n) {
    const int o = off;
    off += (int)up4(n);  // 16-byte aligned sub-arrays
    return o;
  };
  for (int q = 0; q < P.count; ++q) {
    const MgLevel& M = H.L[H.coarse_from + q];
    CoarseLevel& c = P.lv[q];
    for (int a = 0; a < 3; ++a) c.n[a] = M.n[a];
    c.cells = (int)M.cells;
    for (int a = 0; a < 3; ++a) c.f[a] = M.f[a];
    c.isq = M.isq;
    c.x_glob = M.x;
    c.r_glob = M.r;
    c.off[0] = take((int64_t)(c.n[0] + 1) * c.n[1] * c.n[2]);
    c.off[1] = take((int64_t)c.n[0] * (c.n[1] + 1) * c.n[2]);
    c.off[2] = H.dim == 3 ? take((int64_t)c.n[0] * c.n[1] * (c.n[2] + 1)) : 0;
    for (int s = 3; s < 7; ++s) c.off[s] = take(c.cells);
    P.K[q] = kern_of(W, H.coarse_from + q);
    P.cw[q] = cw_of(W, H.coarse_from + q);
  }
  return P;
}

// Enqueues z = M r (level-0 FP32 vectors) on `st`; returns the number of
// kernels launched.
template <int DIM>
int enqueue_cycle(const MgHierarchy& H, const MgWeights& W, const float* r0, float* z0,
                  int64_t skip, const Hook* hook, cudaStream_t st) {
  int launches = 0;
  const int cf = H.coarse_from;
  auto rp = [&](int l) -> const float* { return l == 0 ? r0 : H.L[l].r; };
  auto xp = [&](int l) -> float* { return l == 0 ? z0 : H.L[l].x; };
  for (int l = 0; l < cf; ++l) {
    const MgLevel& M = H.L[l];
    const LV L = lv(M);
    const Kern K = kern_of(W, l);
    const int64_t sk = l == 0 ? skip : -1;
    const Shape s = cells_shape(M.n[0], (int64_t)M.n[1] * M.n[2]);
    k_first<DIM><<<s.grid, s.block, 0, st>>>(L, K, rp(l), xp(l), sk);
    ++launches;
    for (int q = 1; q < W.nu; ++q) {
      k_resid<DIM><<<s.grid, s.block, 0, st>>>(L, xp(l), rp(l), M.res, sk);
      k_smooth<DIM, false><<<s.grid, s.block, 0, st>>>(L, L, K, nullptr, 0.f, M.res, xp(l), -1,
                                                       nullptr, Hook{});
      launches += 2;
    }
    const MgLevel& C = H.L[l + 1];
    const Shape sc = cells_shape(C.n[0], (int64_t)C.n[1] * C.n[2]);
    k_resid_restrict<DIM><<<sc.grid, sc.block, 0, st>>>(L, lv(C), xp(l), rp(l), C.r, sk);
    ++launches;
  }
  if (cf < H.levels) {
    const CoarsePlan P = coarse_plan(H, W);
    k_coarse<DIM><<<1, kCoarseThreads, H.coarse_smem, st>>>(P);
    ++launches;
  }
  for (int l = cf - 1; l >= 0; --l) {
    const MgLevel& M = H.L[l];
    const MgLevel& C = H.L[l + 1];
    const LV L = lv(M), LC = lv(C);
    const Kern K = kern_of(W, l);
    const float cw = cw_of(W, l);
    const int64_t sk = l == 0 ? skip : -1;
    const Shape s = cells_shape(M.n[0], (int64_t)M.n[1] * M.n[2]);
    for (int q = 0; q < W.nu; ++q) {
      if (q == 0)
        k_prolong_resid<DIM><<<s.grid, s.block, 0, st>>>(L, LC, C.x, cw, xp(l), rp(l), M.res, sk);
      else
        k_resid<DIM><<<s.grid, s.block, 0, st>>>(L, xp(l), rp(l), M.res, sk);
      const bool last = (l == 0 && q == W.nu - 1);
      const float* ec = q == 0 ? C.x : nullptr;
      if (last && hook)
        k_smooth<DIM, true><<<s.grid, s.block, 0, st>>>(L, LC, K, ec, cw, M.res, xp(l), sk,
                                                        rp(l), *hook);
      else
        k_smooth<DIM, false><<<s.grid, s.block, 0, st>>>(L, LC, K, ec, cw, M.res, xp(l),
                                                         last ? sk : -1, rp(l), Hook{});
      launches += 2;
    }
  }
  return launches;
}

// Algorithmic bytes of one V-cycle: FP32 words read and written per level,
// each array counted once per kernel.
double cycle_bytes(const MgHierarchy& H, const MgWeights& W) {
  const double d = H.dim, fr = 1.0 / (H.dim == 3 ? 8.0 : 4.0);
  double words = 0.0;
  for (int l = 0; l < H.coarse_from; ++l) {
    const double n = (double)H.L[l].cells;
    const double resid = 3.0 + d, smooth = 4.0;
    const double down = 3.0 + (W.nu - 1) * (resid + smooth) + (2.0 + d + fr);
    const double up = (3.0 + d + fr) + (smooth + fr) + (W.nu - 1) * (resid + smooth);
    words += n * (down + up);
  }
  if (H.coarse_from < H.levels) words += 2.0 * (double)H.L[H.coarse_from].cells;
  return words * 4.0;
}

// ------------------------------------------------------------ FCG kernels

// r = b - A x, r32 = float(r); ||r|| decides whether the loop runs at all.
__global__ void k_fcg_init(OpView<double> A, FcgState* S, double* __restrict__ r,
                           float* __restrict__ r32, double* partials, double* hist, int64_t hcap,
                           Loop h) {
  const double* __restrict__ b = S->b;
  const double* __restrict__ x = S->x;
  double acc[1] = {0.0};
  const int64_t plane = (int64_t)A.nx * A.ny;
  each_cell(A.nx, A.ny, A.ny * A.nz, [&](int i, int j, int k, int64_t c) {
    const Coef<double> cf = load_coef(A, i, j, k);
    const double w = i > 0 ? x[c - 1] : 0.0, e = i + 1 < A.nx ? x[c + 1] : 0.0;
    const double s = j > 0 ? x[c - A.nx] : 0.0, n = j + 1 < A.ny ? x[c + A.nx] : 0.0;
    const double bo = k > 0 ? x[c - plane] : 0.0, t = k + 1 < A.nz ? x[c + plane] : 0.0;
    const double rn = b[c] - apply_coef(cf, x[c], w, e, s, n, bo, t);
    r[c] = rn;
    r32[c] = (float)rn;
    acc[0] += rn * rn;
  });
  reduce_last<1>(acc, partials, &S->ticket, [&](const double* tot) {
    const double b0 = sqrt(tot[0]);
    S->b0 = b0;
    S->res = b0;
    S->best = b0;
    S->it = 0;
    S->best_it = 0;
    S->beta = 0.0;
    if (hcap > 0) hist[0] = b0;
    // CG.cpp:49-63: a zero or already converged start returns at once
    if (!isfinite(b0)) {
      stop_loop(S, h, CFDB_SOLVER_NONFINITE_RESIDUAL);
    } else if (b0 == 0.0 || b0 <= S->abs_tol || 1.0 <= S->rel_tol) {
      stop_loop(S, h, CFDB_SOLVER_CONVERGED);
    } else {
      S->status = kRunning;
      S->done = 0;
      set_loop(h, 1);
    }
  });
}

// p = z - beta p_old (p = z on the first iteration), q = A p; p.q and p.r
// give alpha.  p alternates between two buffers by iteration parity.
__global__ void k_fcg_dir(OpView<double> A, FcgState* S, const float* __restrict__ z,
                          double* P0, double* P1, double* __restrict__ q,
                          const double* __restrict__ r, double* partials,
                          Loop h) {
  if (S->done) return;
  const long long it = S->it;
  const bool first = (it == 0);
  const double beta = first ? 0.0 : S->beta;
  double* __restrict__ pn = (it & 1) ? P1 : P0;
  const double* __restrict__ po = (it & 1) ? P0 : P1;
  auto pv = [&](int64_t c) { return first ? (double)z[c] : fma(-beta, po[c], (double)z[c]); };
  double acc[2] = {0.0, 0.0};
  const int64_t plane = (int64_t)A.nx * A.ny;
  each_cell(A.nx, A.ny, A.ny * A.nz, [&](int i, int j, int k, int64_t c) {
    const Coef<double> cf = load_coef(A, i, j, k);
    const double v = pv(c);
    const double w = i > 0 ? pv(c - 1) : 0.0, e = i + 1 < A.nx ? pv(c + 1) : 0.0;
    const double s = j > 0 ? pv(c - A.nx) : 0.0, n = j + 1 < A.ny ? pv(c + A.nx) : 0.0;
    const double bo = k > 0 ? pv(c - plane) : 0.0, t = k + 1 < A.nz ? pv(c + plane) : 0.0;
    const double aq = apply_coef(cf, v, w, e, s, n, bo, t);
    pn[c] = v;
    q[c] = aq;
    acc[0] += v * aq;
    acc[1] += v * r[c];
  });
  reduce_last<2>(acc, partials, &S->ticket, [&](const double* tot) {
    const double pq = tot[0], pr = tot[1];
    const double alpha = pr / pq;
    // A is positive definite on the space the directions live in: a
    // non-positive p.Ap means rounding has taken over (a scale-free test; the
    // reference's absolute 1e-30 trips on small well-converged systems)
    if (!isfinite(pq) || !(pq > 0.0) || !isfinite(alpha)) {
      stop_loop(S, h, kLearnedStagnated);
      return;
    }
    S->pq = pq;
    S->pr = pr;
    S->alpha = alpha;
  });
}

// x += alpha p; r -= alpha q; r32 = float(r); convergence, stagnation and
// the iteration cap decide whether the loop continues.
__global__ void k_fcg_update(int64_t n, FcgState* S, double* __restrict__ r,
                             float* __restrict__ r32, const double* P0, const double* P1,
                             const double* __restrict__ q, double* partials, double* hist,
                             int64_t hcap, Loop h) {
  if (S->done) return;
  const long long it = S->it;
  const double alpha = S->alpha;
  const double* __restrict__ p = (it & 1) ? P1 : P0;
  double* __restrict__ x = S->x;
  double acc[1] = {0.0};
  const int64_t stride = (int64_t)gridDim.x * gridDim.y * blockDim.x;
  for (int64_t c = (blockIdx.x + (int64_t)gridDim.x * blockIdx.y) * blockDim.x + threadIdx.x; c < n;
       c += stride) {
    x[c] = fma(alpha, p[c], x[c]);
    const double rn = fma(-alpha, q[c], r[c]);
    r[c] = rn;
    r32[c] = (float)rn;
    acc[0] += rn * rn;
  }
  reduce_last<1>(acc, partials, &S->ticket, [&](const double* tot) {
    const double res = sqrt(tot[0]);
    const long long k = it + 1;
    S->it = k;
    S->res = res;
    if (k < hcap) hist[k] = res;
    if (!isfinite(res)) {
      stop_loop(S, h, CFDB_SOLVER_NONFINITE_RESIDUAL);
      return;
    }
    if (res <= S->abs_tol || (S->b0 > 0.0 && res / S->b0 <= S->rel_tol)) {
      stop_loop(S, h, CFDB_SOLVER_CONVERGED);
      return;
    }
    if (res < S->best) {
      S->best = res;
      S->best_it = k;
    } else if (k - S->best_it >= S->window) {
      stop_loop(S, h, kLearnedStagnated);
      return;
    }
    if (k >= S->max_it) stop_loop(S, h, CFDB_SOLVER_MAX_ITERATIONS);
  });
}

}  // namespace

// ------------------------------------------------------------------ host API

cfdb_status mg_build(cfdb_context* ctx, MgHierarchy& H, const FineOperator& op) {
  H.dim = op.dim;
  int n[3] = {op.n[0], op.n[1], op.dim == 3 ? op.n[2] : 1};
  int l = 0;
  auto alloc = [&](float** p, int64_t count) -> cfdb_status {
    CFDB_CUDA(ctx, cudaMalloc((void**)p, sizeof(float) * (size_t)std::max<int64_t>(count, 4)));
    H.owned.push_back(*p);
    return CFDB_OK;
  };
  while (true) {
    MgLevel& M = H.L[l];
    std::memset(&M, 0, sizeof(M));
    for (int a = 0; a < 3; ++a) M.n[a] = n[a];
    M.cells = (int64_t)n[0] * n[1] * n[2];
    for (int a = 0; a < op.dim; ++a) {
      int e[3] = {n[0], n[1], n[2]};
      e[a] += 1;
      cfdb_status rc = alloc(&M.f[a], (int64_t)e[0] * e[1] * e[2]);
      if (rc != CFDB_OK) return rc;
    }
    cfdb_status rc;
    if ((rc = alloc(&M.isq, M.cells)) != CFDB_OK || (rc = alloc(&M.res, M.cells)) != CFDB_OK)
      return rc;
    if (l > 0 && ((rc = alloc(&M.x, M.cells)) != CFDB_OK || (rc = alloc(&M.r, M.cells)) != CFDB_OK))
      return rc;
    ++l;
    int mn = n[0];
    for (int a = 1; a < op.dim; ++a) mn = std::min(mn, n[a]);
    const bool stop = (l > 1 && (mn <= 4 || M.cells <= 64)) || mn == 1 || l == kMgMaxLevels;
    if (stop) break;
    for (int a = 0; a < op.dim; ++a) n[a] = (n[a] + 1) / 2;
  }
  H.levels = l;
  if (H.levels < 2)
    return set_error(ctx, CFDB_ERR_UNSUPPORTED, "learned preconditioner: grid too small to coarsen");
  // the block-resident tail: the longest run of levels >= 1 ending at the
  // coarsest whose levels hold at most kCoarseCells cells and whose data fit
  // in shared memory together
  int cf = H.levels - 1;
  if (coarse_bytes(H, cf) > kCoarseSmemCap)
    return set_error(ctx, CFDB_ERR_UNSUPPORTED,
                     "learned preconditioner: the coarsest level does not fit a thread block "
                     "(grid too anisotropic)");
  while (cf - 1 >= 1 && H.L[cf - 1].cells <= kCoarseCells && H.levels - (cf - 1) <= kMaxCoarse &&
         coarse_bytes(H, cf - 1) <= kCoarseSmemCap)
    --cf;
  H.coarse_from = cf;
  H.coarse_smem = coarse_bytes(H, cf);
  if (op.dim == 2)
    CFDB_CUDA(ctx, cudaFuncSetAttribute(k_coarse<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)H.coarse_smem));
  else
    CFDB_CUDA(ctx, cudaFuncSetAttribute(k_coarse<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)H.coarse_smem));
  return refresh_values(ctx, H, op);
}

cfdb_status mg_apply(cfdb_context* ctx, const MgHierarchy& H, const MgWeights& W, const float* r,
                     float* z, int64_t skip) {
  const int n = H.dim == 2 ? enqueue_cycle<2>(H, W, r, z, skip, nullptr, ctx->stream)
                           : enqueue_cycle<3>(H, W, r, z, skip, nullptr, ctx->stream);
  CFDB_CHECK_LAUNCH(ctx);
  count_launch(ctx, n);
  return CFDB_OK;
}

struct LearnedSolver {
  MgHierarchy* H = nullptr;
  int dim = 0;
  int n[3] = {0, 0, 0};
  int64_t cells = 0;
  uint64_t version = 0;
  MgWeights W{};
  bool have_w = false;
  double *r = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr, *partials = nullptr;
  float *r32 = nullptr, *z32 = nullptr;
  FcgState* S = nullptr;
  FcgState* S_host = nullptr;
  double* hist = nullptr;
  int64_t hist_cap = 0;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t launches_init = 0, launches_body = 0;
  double bytes_init = 0, bytes_iter = 0;

  void free_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  void free_all() {
    free_graph();
    delete H;
    H = nullptr;
    for (void* p : {(void*)r, (void*)p0, (void*)p1, (void*)q, (void*)partials, (void*)r32,
                    (void*)z32, (void*)S, (void*)hist})
      cudaFree(p);
    r = p0 = p1 = q = partials = nullptr;
    r32 = z32 = nullptr;
    S = nullptr;
    hist = nullptr;
    hist_cap = 0;
    if (S_host) cudaFreeHost(S_host);
    S_host = nullptr;
    if (cap) cudaStreamDestroy(cap);
    cap = nullptr;
  }
};

LearnedSolver* learned_create() { return new LearnedSolver(); }

void learned_destroy(LearnedSolver* s) {
  if (!s) return;
  s->free_all();
  delete s;
}

namespace {

// Blocks of the widest reduction launch (one partial per block and value).
int64_t partial_slots(const FineOperator& op) {
  const Shape sh = cells_shape(op.A.nx, (int64_t)op.A.ny * op.A.nz);
  return std::max<int64_t>((int64_t)sh.grid.x * sh.grid.y, kMaxBlocks);
}

// One FCG iteration: V-cycle z = M r (its last kernel also forms z.q and
// beta), direction + A p, update.  Returns the number of kernels.
int enqueue_body(LearnedSolver* s, const FineOperator& op, Loop h, cudaStream_t st) {
  const int64_t skip = op.pinned ? op.ref : -1;
  const Shape sh = cells_shape(op.A.nx, (int64_t)op.A.ny * op.A.nz);
  const Hook hk{s->q, s->partials, s->S, h};
  const int nv = op.dim == 2 ? enqueue_cycle<2>(*s->H, s->W, s->r32, s->z32, skip, &hk, st)
                             : enqueue_cycle<3>(*s->H, s->W, s->r32, s->z32, skip, &hk, st);
  k_fcg_dir<<<sh.grid, sh.block, 0, st>>>(op.A, s->S, s->z32, s->p0, s->p1, s->q, s->r,
                                           s->partials, h);
  k_fcg_update<<<flat_grid(s->cells), 256, 0, st>>>(s->cells, s->S, s->r, s->r32, s->p0, s->p1,
                                                    s->q, s->partials, s->hist, s->hist_cap, h);
  return nv + 2;
}

// Solve loop without a graph, for profilers that cannot look inside graphs
// with conditional nodes (CFDB_LEARNED_LAUNCH=stream): the same kernels,
// launched per iteration, the host reading the state after each iteration.
cfdb_status run_stream_mode(cfdb_context* ctx, LearnedSolver* s, const FineOperator& op) {
  const Shape sh = cells_shape(op.A.nx, (int64_t)op.A.ny * op.A.nz);
  k_fcg_init<<<sh.grid, sh.block, 0, ctx->stream>>>(op.A, s->S, s->r, s->r32, s->partials, s->hist,
                                                     s->hist_cap, Loop{0, 0});
  CFDB_CHECK_LAUNCH(ctx);
  while (true) {
    CFDB_CUDA(ctx, cudaMemcpyAsync(s->S_host, s->S, sizeof(FcgState), cudaMemcpyDeviceToHost,
                                   ctx->stream));
    CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (s->S_host->done) break;
    enqueue_body(s, op, Loop{0, 0}, ctx->stream);
    CFDB_CHECK_LAUNCH(ctx);
  }
  return CFDB_OK;
}

cfdb_status capture_graph(cfdb_context* ctx, LearnedSolver* s, const FineOperator& op) {
  s->free_graph();
  CFDB_CUDA(ctx, cudaGraphCreate(&s->graph, 0));
  cudaGraphConditionalHandle h;
  CFDB_CUDA(ctx, cudaGraphConditionalHandleCreate(&h, s->graph, 1, cudaGraphCondAssignDefault));
  const Shape sh = cells_shape(op.A.nx, (int64_t)op.A.ny * op.A.nz);
  // parent graph: the initial residual, then the WHILE node
  CFDB_CUDA(ctx, cudaStreamBeginCaptureToGraph(s->cap, s->graph, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
  const Loop lp{h, 1};
  k_fcg_init<<<sh.grid, sh.block, 0, s->cap>>>(op.A, s->S, s->r, s->r32, s->partials, s->hist,
                                                s->hist_cap, lp);
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(s->cap, &g);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "capture of the FCG start", __FILE__, __LINE__);
  size_t nn = 0;
  CFDB_CUDA(ctx, cudaGraphGetNodes(s->graph, nullptr, &nn));
  if (nn != 1) return set_error(ctx, CFDB_ERR_CUDA, "unexpected FCG start graph");
  cudaGraphNode_t init_node;
  CFDB_CUDA(ctx, cudaGraphGetNodes(s->graph, &init_node, &nn));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t loop_node;
  CFDB_CUDA(ctx, cudaGraphAddNode(&loop_node, s->graph, &init_node, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // body: one FCG iteration
  CFDB_CUDA(ctx, cudaStreamBeginCaptureToGraph(s->cap, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
  const int nv = enqueue_body(s, op, lp, s->cap);
  cudaGraph_t b2 = nullptr;
  ce = cudaStreamEndCapture(s->cap, &b2);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "capture of the FCG loop", __FILE__, __LINE__);
  CFDB_CHECK_LAUNCH(ctx);
  CFDB_CUDA(ctx, cudaGraphInstantiate(&s->exec, s->graph, 0));
  s->launches_init = 1;
  s->launches_body = nv;
  // algorithmic bytes: the start (b, x in; r, r32 out) and per iteration the
  // V-cycle, the direction pass (z, p_old, r in; p, q out), the update (x, p,
  // r, q in; x, r, r32 out) and the z.q read of q; face arrays when present
  int face_words = 0;
  for (int a = 0; a < op.dim; ++a) face_words += op.full[a] ? 1 : 0;
  const double n = (double)s->cells;
  s->bytes_init = n * (8.0 * (3 + face_words) + 4.0);
  s->bytes_iter = cycle_bytes(*s->H, s->W) + n * (4.0 + 8.0 * (4 + face_words)) +
                  n * (8.0 * 6 + 4.0) + n * 8.0;
  return CFDB_OK;
}

}  // namespace

cfdb_status learned_solve(cfdb_context* ctx, LearnedSolver* s, const FineOperator& op,
                          uint64_t version, const MgWeights& W, const double* b, double* x,
                          double abs_tol, double rel_tol, int64_t max_it, int64_t hist_cap,
                          LearnedOutcome* out) {
  std::memset(out, 0, sizeof(*out));
  const int64_t cells = (int64_t)op.n[0] * op.n[1] * (op.dim == 3 ? op.n[2] : 1);
  const bool same_shape = s->H && s->dim == op.dim && s->n[0] == op.n[0] && s->n[1] == op.n[1] &&
                          s->n[2] == op.n[2];
  bool recapture = false;
  if (!same_shape) {
    s->free_all();
    s->H = new MgHierarchy();
    s->dim = op.dim;
    for (int a = 0; a < 3; ++a) s->n[a] = op.n[a];
    s->cells = cells;
    cfdb_status st = mg_build(ctx, *s->H, op);
    auto a64 = [&](double** p, int64_t m) -> cfdb_status {
      CFDB_CUDA(ctx, cudaMalloc((void**)p, sizeof(double) * (size_t)m));
      return CFDB_OK;
    };
    auto a32 = [&](float** p, int64_t m) -> cfdb_status {
      CFDB_CUDA(ctx, cudaMalloc((void**)p, sizeof(float) * (size_t)m));
      return CFDB_OK;
    };
    if (st != CFDB_OK || (st = a64(&s->r, cells)) != CFDB_OK || (st = a64(&s->p0, cells)) != CFDB_OK ||
        (st = a64(&s->p1, cells)) != CFDB_OK || (st = a64(&s->q, cells)) != CFDB_OK ||
        (st = a64(&s->partials, 2 * partial_slots(op))) != CFDB_OK ||
        (st = a32(&s->r32, cells)) != CFDB_OK || (st = a32(&s->z32, cells)) != CFDB_OK) {
      s->free_all();
      return st;
    }
    cudaError_t e1 = cudaMalloc((void**)&s->S, sizeof(FcgState));
    cudaError_t e2 = e1 == cudaSuccess ? cudaMemset(s->S, 0, sizeof(FcgState)) : e1;
    cudaError_t e3 = e2 == cudaSuccess ? cudaMemset(s->q, 0, sizeof(double) * cells) : e2;
    cudaError_t e4 = e3 == cudaSuccess ? cudaMallocHost((void**)&s->S_host, sizeof(FcgState)) : e3;
    cudaError_t e5 = e4 == cudaSuccess ? cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking) : e4;
    if (e5 != cudaSuccess) {
      s->free_all();
      return cuda_error(ctx, e5, "learned solver state", __FILE__, __LINE__);
    }
    s->version = version;
    recapture = true;
  } else if (s->version != version) {
    cfdb_status st = refresh_values(ctx, *s->H, op);
    if (st != CFDB_OK) return st;
    s->version = version;
  }
  const int64_t want_hist = std::max<int64_t>(hist_cap, 1);
  if (s->hist_cap < want_hist) {
    cudaFree(s->hist);
    s->hist = nullptr;
    s->hist_cap = 0;
    CFDB_CUDA(ctx, cudaMalloc((void**)&s->hist, sizeof(double) * (size_t)want_hist));
    s->hist_cap = want_hist;
    recapture = true;
  }
  if (!s->have_w || std::memcmp(&s->W, &W, sizeof(W)) != 0) {
    s->W = W;
    s->have_w = true;
    recapture = true;
  }
  if (recapture || !s->exec) {
    cfdb_status st = capture_graph(ctx, s, op);
    if (st != CFDB_OK) {
      s->free_graph();
      return st;
    }
  }
  FcgState& hs = *s->S_host;
  std::memset(&hs, 0, sizeof(hs));
  hs.b = b;
  hs.x = x;
  hs.abs_tol = abs_tol;
  hs.rel_tol = rel_tol;
  hs.max_it = max_it;
  hs.window = 50;
  hs.status = kRunning;
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->S, &hs, sizeof(FcgState), cudaMemcpyHostToDevice, ctx->stream));
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_k0, ctx->stream));
  const char* mode = std::getenv("CFDB_LEARNED_LAUNCH");
  if (mode && std::strcmp(mode, "stream") == 0) {
    cfdb_status st = run_stream_mode(ctx, s, op);
    if (st != CFDB_OK) return st;
  } else {
    CFDB_CUDA(ctx, cudaGraphLaunch(s->exec, ctx->stream));
  }
  CFDB_CUDA(ctx, cudaEventRecord(ctx->ev_k1, ctx->stream));
  CFDB_CUDA(ctx, cudaMemcpyAsync(s->S_host, s->S, sizeof(FcgState), cudaMemcpyDeviceToHost, ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  CFDB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev_k0, ctx->ev_k1));
  out->status = hs.status;
  out->iterations = hs.it;
  out->initial_residual = hs.b0;
  out->final_residual = hs.res;
  out->kernel_ms = ms;
  out->bytes = s->bytes_init + s->bytes_iter * (double)hs.it;
  out->launches = s->launches_init + s->launches_body * hs.it;
  count_launch(ctx, (int)std::min<int64_t>(out->launches, 1 << 30));
  return CFDB_OK;
}

cfdb_status learned_history(cfdb_context* ctx, LearnedSolver* s, double* host, int64_t m) {
  if (!s->hist || m <= 0) return CFDB_OK;
  m = std::min(m, s->hist_cap);
  CFDB_CUDA(ctx, cudaMemcpyAsync(host, s->hist, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost,
                                 ctx->stream));
  CFDB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CFDB_OK;
}

namespace {
struct CtxWeights {
  MgWeights w[2];
};
void free_ctx_weights(void* p) { delete static_cast<CtxWeights*>(p); }

CtxWeights& ctx_weights(cfdb_context* ctx) {
  if (!ctx->mg_weights) {
    auto* cw = new CtxWeights();
    cw->w[0] = mg_builtin_weights(2);
    cw->w[1] = mg_builtin_weights(3);
    ctx->mg_weights = cw;
    ctx->mg_weights_free = free_ctx_weights;
  }
  return *static_cast<CtxWeights*>(ctx->mg_weights);
}
}  // namespace

const MgWeights& mg_context_weights(cfdb_context* ctx, int dim) {
  return ctx_weights(ctx).w[dim == 3 ? 1 : 0];
}

}  // namespace cfdb

using namespace cfdb;

extern "C" {

cfdb_status cfdb_mg_set_weights(cfdb_context* ctx, int dim, int levels, int nu, int coarse_sweeps,
                                const float* kernels, const float* coarse_weights) {
  if (!ctx || !kernels || !coarse_weights) return CFDB_ERR_INVALID_ARGUMENT;
  if (levels < 1 || levels > kMgMaxLevels)
    return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, "weights: levels must be 1..16");
  MgWeights W = mg_default_weights(dim);
  W.levels = levels;
  W.nu = nu;
  W.coarse_sweeps = coarse_sweeps;
  for (int l = 0; l < kMgMaxLevels; ++l) {
    const int src = std::min(l, levels - 1);
    for (int t = 0; t < kMgTaps; ++t) W.w[l][t] = kernels[src * kMgTaps + t];
    W.c[l] = coarse_weights[src];
  }
  std::string why;
  if (!mg_weights_valid(W, &why)) return set_error(ctx, CFDB_ERR_INVALID_ARGUMENT, why);
  ctx_weights(ctx).w[dim == 3 ? 1 : 0] = W;
  return CFDB_OK;
}

cfdb_status cfdb_mg_get_weights(cfdb_context* ctx, int dim, int* levels, int* nu,
                                int* coarse_sweeps, float* kernels, float* coarse_weights) {
  if (!ctx || (dim != 2 && dim != 3)) return CFDB_ERR_INVALID_ARGUMENT;
  const MgWeights& W = mg_context_weights(ctx, dim);
  if (levels) *levels = W.levels;
  if (nu) *nu = W.nu;
  if (coarse_sweeps) *coarse_sweeps = W.coarse_sweeps;
  if (kernels) std::memcpy(kernels, W.w, sizeof(W.w));
  if (coarse_weights) std::memcpy(coarse_weights, W.c, sizeof(W.c));
  return CFDB_OK;
}

cfdb_status cfdb_mg_reset_weights(cfdb_context* ctx, int dim, int trained) {
  if (!ctx || (dim != 2 && dim != 3)) return CFDB_ERR_INVALID_ARGUMENT;
  ctx_weights(ctx).w[dim == 3 ? 1 : 0] = trained ? mg_builtin_weights(dim) : mg_default_weights(dim);
  return CFDB_OK;
}

}  // extern "C"
