// Training of the learned preconditioner on the GPU: the V-cycle network's
// loss and its exact gradient with respect to the smoothing kernels and the
// coarse-correction weights, by reverse-mode differentiation through every
// layer with hand-written forward and adjoint kernels.
//
// Loss of one error field e (e[pin] = 0):  r = A e (r[pin] = 0),  z = M r,
//     L(e) = (z - e)^T A (z - e) / (e^T A e),
// the A-norm contraction of the preconditioned error propagator I - M A on e
// -- the quantity that sets the convergence rate of (flexible) CG.  A is the
// hierarchy's level-0 operator and M the V-cycle of mg.cu, same layers, same
// FP32 arithmetic.  The forward pass keeps the scaled residual u of every
// smoothing layer (the only activations the parameters multiply); the
// adjoint of a layer x' = x + D^-1/2 (W * u), u = D^-1/2 (r - A x) is, with
// g the adjoint of x' and t = D^-1/2 g,
//     dL/dW[o] += sum_c t_c u_(c+o),   l = D^-1/2 (W * t)  (W symmetric),
//     adjoint of r += l,               adjoint of x = g - A l.
// These kernels are plain one-thread-per-cell passes: training runs on small
// grids, and clarity beats speed here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "cfdb_internal.cuh"
#include "mg.cuh"
#include "pcg_internal.cuh"

namespace cfdb {
namespace {

constexpr int kTB = 256;

struct TL {
  int nx, ny, nz;
  int64_t cells;
  const float* fx;
  const float* fy;
  const float* fz;
  const float* isq;
};

TL tl(const MgLevel& M) {
  return TL{M.n[0], M.n[1], M.n[2], M.cells, M.f[0], M.f[1], M.f[2], M.isq};
}

struct Taps {
  float w[kMgTaps];
};

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kTB - 1) / kTB, 4096)); }

#define FOR_CELLS(c, n) \
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < (n); c += (int64_t)gridDim.x * blockDim.x)

__device__ __forceinline__ void ijk(const TL& L, int64_t c, int& i, int& j, int& k) {
  i = (int)(c % L.nx);
  const int64_t rest = c / L.nx;
  j = (int)(rest % L.ny);
  k = (int)(rest / L.ny);
}

// (A x)_c of the level operator; f(q) returns x at cell q.
template <class F>
__device__ __forceinline__ float apply_at(const TL& L, int64_t c, int i, int j, int k, F f) {
  const int64_t bx = i + (int64_t)(L.nx + 1) * (j + (int64_t)L.ny * k);
  const float xl = L.fx[bx], xh = L.fx[bx + 1];
  float yl = 0.f, yh = 0.f;
  if (L.fy) {
    const int64_t by = i + (int64_t)L.nx * (j + (int64_t)(L.ny + 1) * k);
    yl = L.fy[by];
    yh = L.fy[by + L.nx];
  }
  const int64_t plane = (int64_t)L.nx * L.ny;
  const float zl = L.fz[c], zh = L.fz[c + plane];
  const float d = ((xl + xh) + (yl + yh)) + (zl + zh);
  float off = 0.f;
  if (i > 0) off += xl * f(c - 1);
  if (i + 1 < L.nx) off += xh * f(c + 1);
  if (j > 0) off += yl * f(c - L.nx);
  if (j + 1 < L.ny) off += yh * f(c + L.nx);
  if (k > 0) off += zl * f(c - plane);
  if (k + 1 < L.nz) off += zh * f(c + plane);
  return d * f(c) - off;
}

// sum_o K[o] v(c+o)
template <class F>
__device__ __forceinline__ float conv_at(const TL& L, const Taps& K, int i, int j, int k, F v) {
  float s = 0.f;
  for (int dk = -1; dk <= 1; ++dk) {
    const int kk = k + dk;
    if (kk < 0 || kk >= L.nz) continue;
    for (int dj = -1; dj <= 1; ++dj) {
      const int jj = j + dj;
      if (jj < 0 || jj >= L.ny) continue;
      for (int di = -1; di <= 1; ++di) {
        const int ii = i + di;
        if (ii < 0 || ii >= L.nx) continue;
        s += K.w[(dk + 1) * 9 + (dj + 1) * 3 + (di + 1)] * v(ii + (int64_t)L.nx * (jj + (int64_t)L.ny * kk));
      }
    }
  }
  return s;
}

__device__ __forceinline__ int64_t parent_of(const TL& C, int i, int j, int k) {
  return (i >> 1) + (int64_t)C.nx * ((j >> 1) + (int64_t)C.ny * (k >> 1));
}

// out = [r (r[skip] = 0)] - [A x]
__global__ void t_res(TL L, const float* x, const float* r, int64_t skip, float* out) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    float v = (r && c != skip) ? r[c] : 0.f;
    if (x) v -= apply_at(L, c, i, j, k, [&](int64_t q) { return x[q]; });
    out[c] = v;
  }
}

// out = A x, out[pin] = 0
__global__ void t_apply(TL L, const float* x, int64_t pin, float* out) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    out[c] = (c == pin) ? 0.f : apply_at(L, c, i, j, k, [&](int64_t q) { return x[q]; });
  }
}

__global__ void t_scale(TL L, const float* a, float* out) {
  FOR_CELLS(c, L.cells) out[c] = L.isq[c] * a[c];
}

// x_out = [x_in] + D^-1/2 (K * u)
__global__ void t_conv_add(TL L, Taps K, const float* u, const float* x_in, float* x_out) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    const float s = conv_at(L, K, i, j, k, [&](int64_t q) { return u[q]; });
    x_out[c] = (x_in ? x_in[c] : 0.f) + L.isq[c] * s;
  }
}

// out_c = scale * sum of the children's a
__global__ void t_restrict(TL L, TL C, const float* a, float scale, float* out) {
  FOR_CELLS(qc, C.cells) {
    int ci, cj, ck;
    ijk(C, qc, ci, cj, ck);
    float s = 0.f;
    for (int u = 0; u < 2; ++u)
      for (int v = 0; v < 2; ++v)
        for (int t = 0; t < 2; ++t) {
          const int i = 2 * ci + t, j = 2 * cj + v, k = 2 * ck + u;
          if (i < L.nx && j < L.ny && k < L.nz) s += a[i + (int64_t)L.nx * (j + (int64_t)L.ny * k)];
        }
    out[qc] = scale * s;
  }
}

// x += scale * P ec
__global__ void t_prolong_add(TL L, TL C, const float* ec, float scale, float* x) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    x[c] += scale * ec[parent_of(C, i, j, k)];
  }
}

__global__ void t_jacobi(TL L, const float* r, const float* x_in, float* x_out) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    const float ax = x_in ? apply_at(L, c, i, j, k, [&](int64_t q) { return x_in[q]; }) : 0.f;
    const float is = L.isq[c];
    x_out[c] = (x_in ? x_in[c] : 0.f) + 0.8f * (is * is) * (r[c] - ax);
  }
}

// ----------------------------------------------------------------- adjoints

// acc[o] += sum_c t_c u_(c+o) for the 27 offsets (block sums, then atomics)
__global__ void t_tapgrad(TL L, const float* t, const float* u, double* acc) {
  __shared__ double red[kTB / 32][kMgTaps];
  double a[kMgTaps];
#pragma unroll
  for (int o = 0; o < kMgTaps; ++o) a[o] = 0.0;
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    const float tc = t[c];
    if (tc == 0.f) continue;
#pragma unroll
    for (int dk = -1; dk <= 1; ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const int ii = i + di, jj = j + dj, kk = k + dk;
          if (ii < 0 || ii >= L.nx || jj < 0 || jj >= L.ny || kk < 0 || kk >= L.nz) continue;
          a[(dk + 1) * 9 + (dj + 1) * 3 + (di + 1)] +=
              (double)tc * u[ii + (int64_t)L.nx * (jj + (int64_t)L.ny * kk)];
        }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 0; o < kMgTaps; ++o) {
    double v = a[o];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (lane == 0) red[warp][o] = v;
  }
  __syncthreads();
  if (threadIdx.x < kMgTaps) {
    double s = 0.0;
    for (int w = 0; w < kTB / 32; ++w) s += red[w][threadIdx.x];
    atomicAdd(acc + threadIdx.x, s);
  }
}

// out = D^-1/2 (K * t)   (K symmetric: its own adjoint)
__global__ void t_conv_isq(TL L, Taps K, const float* t, float* out) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    out[c] = L.isq[c] * conv_at(L, K, i, j, k, [&](int64_t q) { return t[q]; });
  }
}

// g_out = g - A l;  lr += l
__global__ void t_sweep_back(TL L, const float* g, const float* l, float* g_out, float* lr) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    g_out[c] = g[c] - apply_at(L, c, i, j, k, [&](int64_t q) { return l[q]; });
    lr[c] += l[c];
  }
}

// out = P lc (injection)
__global__ void t_inject(TL L, TL C, const float* lc, float* out) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    out[c] = lc[parent_of(C, i, j, k)];
  }
}

// Jacobi sweep x' = x + w D^-1 (r - A x): lam_out = lam - A m, lr += m with
// m = w D^-1 lam.
__global__ void t_jacobi_back(TL L, const float* lam, float* lam_out, float* lr) {
  FOR_CELLS(c, L.cells) {
    int i, j, k;
    ijk(L, c, i, j, k);
    auto m = [&](int64_t q) {
      const float is = L.isq[q];
      return 0.8f * (is * is) * lam[q];
    };
    lam_out[c] = lam[c] - apply_at(L, c, i, j, k, m);
    lr[c] += m(c);
  }
}

// out += sum_c a_c b_c (b_c = ec[parent(c)] when C is given)
__global__ void t_dot(TL L, const float* a, const float* b, const TL* Cp, double* out) {
  __shared__ double red[kTB / 32];
  double s = 0.0;
  FOR_CELLS(c, L.cells) {
    float bv;
    if (Cp) {
      int i, j, k;
      ijk(L, c, i, j, k);
      bv = b[parent_of(*Cp, i, j, k)];
    } else {
      bv = b[c];
    }
    s += (double)a[c] * bv;
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kTB / 32; ++w) t += red[w];
    atomicAdd(out, t);
  }
}

__global__ void t_sub(int64_t n, const float* a, const float* b, float* out) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
    out[c] = a[c] - b[c];
}

__global__ void t_grad_top(int64_t n, const float* ad, const double* den, int64_t pin, float* lz) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
    lz[c] = (c == pin) ? 0.f : (float)(2.0 * ad[c] / *den);
}

// ------------------------------------------------------------------ driver

struct Trainer {
  cfdb_context* ctx;
  const MgHierarchy& H;
  const MgWeights& W;
  cudaStream_t st;
  int64_t pin;
  std::vector<float*> bufs;
  struct Lv {
    float *r, *x, *tmp, *res, *g, *g2, *lr, *l;
    std::vector<float*> ud, uu;
  };
  std::vector<Lv> lv;
  TL* d_tl = nullptr;  // device copies of the level views (for t_dot's parent mode)
  double* d_acc = nullptr;  // [16*27 kernel grads][16 coarse grads][num][den]
  cudaError_t err = cudaSuccess;

  Trainer(cfdb_context* c, const MgHierarchy& h, const MgWeights& w, int64_t p)
      : ctx(c), H(h), W(w), st(c->stream), pin(p) {}
  ~Trainer() {
    for (float* b : bufs) cudaFree(b);
    cudaFree(d_tl);
    cudaFree(d_acc);
  }
  float* alloc(int64_t n) {
    float* p = nullptr;
    cudaError_t e = cudaMalloc((void**)&p, sizeof(float) * (size_t)std::max<int64_t>(n, 4));
    if (e != cudaSuccess) err = e;
    bufs.push_back(p);
    return p;
  }
  bool setup() {
    lv.resize(H.levels);
    for (int l = 0; l < H.levels; ++l) {
      const int64_t n = H.L[l].cells;
      Lv& v = lv[l];
      v.r = alloc(n);
      v.x = alloc(n);
      v.tmp = alloc(n);
      v.res = alloc(n);
      v.g = alloc(n);
      v.g2 = alloc(n);
      v.lr = alloc(n);
      v.l = alloc(n);
      for (int s = 0; s < W.nu; ++s) {
        v.ud.push_back(alloc(n));
        v.uu.push_back(alloc(n));
      }
    }
    std::vector<TL> h(H.levels);
    for (int l = 0; l < H.levels; ++l) h[l] = tl(H.L[l]);
    if (cudaMalloc((void**)&d_tl, sizeof(TL) * H.levels) != cudaSuccess) return false;
    // stream-ordered: the context stream is non-blocking
    if (cudaMemcpyAsync(d_tl, h.data(), sizeof(TL) * H.levels, cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return false;
    if (cudaMalloc((void**)&d_acc, sizeof(double) * (16 * 27 + 16 + 2)) != cudaSuccess) return false;
    return err == cudaSuccess;
  }
  Taps taps(int l) const {
    Taps K;
    mg_kernel_taps(W, l, K.w);
    return K;
  }
  int wl(int l) const { return std::min(l, W.levels - 1); }
  float cw(int l) const { return W.c[wl(l)]; }
  int g(int64_t n) const { return grid_for(n); }

  // z_l = V_l(r_l); r_l in lv[l].r, result in lv[l].x
  void forward(int l) {
    const TL L = tl(H.L[l]);
    Lv& v = lv[l];
    const int64_t n = L.cells;
    const int last = H.levels - 1;
    if (l == last) {
      float* a = v.x;
      float* b = v.tmp;
      cudaMemsetAsync(a, 0, sizeof(float) * n, st);
      for (int s = 0; s < W.coarse_sweeps; ++s) {
        t_jacobi<<<g(n), kTB, 0, st>>>(L, v.r, a, b);
        std::swap(a, b);
      }
      if (a != v.x) cudaMemcpyAsync(v.x, a, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
      return;
    }
    const TL C = tl(H.L[l + 1]);
    const Taps K = taps(l);
    const int64_t sk = l == 0 ? pin : -1;
    for (int s = 0; s < W.nu; ++s) {
      t_res<<<g(n), kTB, 0, st>>>(L, s == 0 ? nullptr : v.x, v.r, sk, v.res);
      t_scale<<<g(n), kTB, 0, st>>>(L, v.res, v.ud[s]);
      t_conv_add<<<g(n), kTB, 0, st>>>(L, K, v.ud[s], s == 0 ? nullptr : v.x, v.x);
    }
    t_res<<<g(n), kTB, 0, st>>>(L, v.x, v.r, sk, v.res);
    t_restrict<<<g(C.cells), kTB, 0, st>>>(L, C, v.res, 1.f, lv[l + 1].r);
    forward(l + 1);
    t_prolong_add<<<g(n), kTB, 0, st>>>(L, C, lv[l + 1].x, cw(l), v.x);
    for (int s = 0; s < W.nu; ++s) {
      t_res<<<g(n), kTB, 0, st>>>(L, v.x, v.r, sk, v.res);
      t_scale<<<g(n), kTB, 0, st>>>(L, v.res, v.uu[s]);
      t_conv_add<<<g(n), kTB, 0, st>>>(L, K, v.uu[s], v.x, v.x);
    }
  }

  // one smoothing layer backwards: g (adjoint of x') -> g2 (adjoint of x),
  // lr += adjoint of r, kernel gradient of level l
  void layer_back(int l, const float* u, float*& gcur, float*& gnext) {
    const TL L = tl(H.L[l]);
    Lv& v = lv[l];
    const int64_t n = L.cells;
    const Taps K = taps(l);
    t_scale<<<g(n), kTB, 0, st>>>(L, gcur, v.tmp);  // t = D^-1/2 g
    t_tapgrad<<<g(n), kTB, 0, st>>>(L, v.tmp, u, d_acc + 27 * wl(l));
    t_conv_isq<<<g(n), kTB, 0, st>>>(L, K, v.tmp, v.l);
    t_sweep_back<<<g(n), kTB, 0, st>>>(L, gcur, v.l, gnext, v.lr);
    std::swap(gcur, gnext);
  }

  // lv[l].g holds the adjoint of z_l; accumulates the adjoint of r_l into lv[l].lr
  void backward(int l) {
    const TL L = tl(H.L[l]);
    Lv& v = lv[l];
    const int64_t n = L.cells;
    const int last = H.levels - 1;
    cudaMemsetAsync(v.lr, 0, sizeof(float) * n, st);
    float* gcur = v.g;
    float* gnext = v.g2;
    if (l == last) {
      for (int s = 0; s < W.coarse_sweeps; ++s) {
        t_jacobi_back<<<g(n), kTB, 0, st>>>(L, gcur, gnext, v.lr);
        std::swap(gcur, gnext);
      }
      return;
    }
    const TL C = tl(H.L[l + 1]);
    for (int s = W.nu - 1; s >= 0; --s) layer_back(l, v.uu[s], gcur, gnext);
    // prolongation x' = x + c P ec
    t_dot<<<g(n), kTB, 0, st>>>(L, gcur, lv[l + 1].x, d_tl + (l + 1), d_acc + 16 * 27 + wl(l));
    t_restrict<<<g(C.cells), kTB, 0, st>>>(L, C, gcur, cw(l), lv[l + 1].g);
    backward(l + 1);
    // restriction rc = R (r - A x): adjoint P lambda_rc
    t_inject<<<g(n), kTB, 0, st>>>(L, C, lv[l + 1].lr, v.l);
    t_sweep_back<<<g(n), kTB, 0, st>>>(L, gcur, v.l, gnext, v.lr);
    std::swap(gcur, gnext);
    for (int s = W.nu - 1; s >= 0; --s) layer_back(l, v.ud[s], gcur, gnext);
  }
};

}  // namespace
}  // namespace cfdb

using namespace cfdb;

extern "C" {

cfdb_status cfdb_mg_loss_grad(cfdb_context* ctx, cfdb_poperator* op, int nsamples,
                              const float* e_host, double* loss, double* grad_kernels,
                              double* grad_coarse) {
  if (!ctx || !op || nsamples < 1 || !e_host || !loss) return CFDB_ERR_INVALID_ARGUMENT;
  CFDB_CUDA(ctx, cudaSetDevice(ctx->device));
  FineOperator fo;
  LearnedSolver* solver = nullptr;
  uint64_t version = 0;
  poperator_learned(op, &fo, &solver, &version);
  const MgHierarchy* H = nullptr;
  cfdb_status st = learned_hierarchy(ctx, solver, fo, version, &H);
  if (st != CFDB_OK) return st;
  const MgWeights& W = mg_context_weights(ctx, fo.dim);
  const int64_t pin = fo.pinned ? fo.ref : -1;
  Trainer T(ctx, *H, W, pin);
  if (!T.setup()) return set_error(ctx, CFDB_ERR_OUT_OF_MEMORY, "training buffers");
  const TL L0 = tl(H->L[0]);
  const int64_t n = L0.cells;
  cudaStream_t s = ctx->stream;
  CFDB_CUDA(ctx, cudaMemsetAsync(T.d_acc, 0, sizeof(double) * (16 * 27 + 16), s));
  float* e = T.alloc(n);
  float* ad = T.alloc(n);
  if (T.err != cudaSuccess) return cuda_error(ctx, T.err, "training buffers", __FILE__, __LINE__);
  double* num = T.d_acc + 16 * 27 + 16;
  double* den = num + 1;
  double total = 0.0;
  const int gn = grid_for(n);
  for (int q = 0; q < nsamples; ++q) {
    CFDB_CUDA(ctx, cudaMemcpyAsync(e, e_host + (size_t)q * n, sizeof(float) * n,
                                   cudaMemcpyHostToDevice, s));
    if (pin >= 0) CFDB_CUDA(ctx, cudaMemsetAsync(e + pin, 0, sizeof(float), s));
    // r = A e with the pinned row: r[pin] = e[pin] = 0
    t_apply<<<gn, kTB, 0, s>>>(L0, e, pin, T.lv[0].r);
    CFDB_CHECK_LAUNCH(ctx);
    T.forward(0);
    if (pin >= 0) CFDB_CUDA(ctx, cudaMemsetAsync(T.lv[0].x + pin, 0, sizeof(float), s));
    // d = z - e, Ad, num = d.Ad, den = e.Ae
    CFDB_CUDA(ctx, cudaMemsetAsync(num, 0, 2 * sizeof(double), s));
    t_sub<<<gn, kTB, 0, s>>>(n, T.lv[0].x, e, T.lv[0].res);
    t_res<<<gn, kTB, 0, s>>>(L0, T.lv[0].res, nullptr, -1, ad);  // ad = -A d
    t_dot<<<gn, kTB, 0, s>>>(L0, T.lv[0].res, ad, nullptr, num);  // -d.Ad
    t_res<<<gn, kTB, 0, s>>>(L0, e, nullptr, -1, T.lv[0].tmp);    // -A e
    t_dot<<<gn, kTB, 0, s>>>(L0, e, T.lv[0].tmp, nullptr, den);   // -e.Ae
    // adjoint of z: 2 A d / den = 2 (-Ad) / (-den)
    t_grad_top<<<gn, kTB, 0, s>>>(n, ad, den, pin, T.lv[0].g);
    CFDB_CHECK_LAUNCH(ctx);
    T.backward(0);
    CFDB_CHECK_LAUNCH(ctx);
    double nd[2];
    CFDB_CUDA(ctx, cudaMemcpyAsync(nd, num, sizeof(nd), cudaMemcpyDeviceToHost, s));
    CFDB_CUDA(ctx, cudaStreamSynchronize(s));
    total += nd[0] / nd[1];
  }
  std::vector<double> acc(16 * 27 + 16);
  CFDB_CUDA(ctx, cudaMemcpyAsync(acc.data(), T.d_acc, sizeof(double) * acc.size(),
                                 cudaMemcpyDeviceToHost, s));
  CFDB_CUDA(ctx, cudaStreamSynchronize(s));
  *loss = total / nsamples;
  // kernel-space tap gradients -> the weight layout, tied taps summed
  if (grad_kernels) {
    for (int l = 0; l < 16; ++l) {
      double gk[kMgTaps];
      for (int t = 0; t < kMgTaps; ++t) gk[t] = acc[l * 27 + t] / nsamples;
      double gw[kMgTaps] = {0};
      if (fo.dim == 3) {
        for (int t = 0; t < kMgTaps; ++t) gw[t] = gk[t];
      } else {
        for (int dj = 0; dj < 3; ++dj)
          for (int di = 0; di < 3; ++di) gw[9 + dj * 3 + di] = gk[dj * 9 + 3 + di];
      }
      for (int t = 0; t < kMgTaps; ++t)
        grad_kernels[l * kMgTaps + t] = (t == 13) ? gw[t] : gw[t] + gw[kMgTaps - 1 - t];
    }
  }
  if (grad_coarse)
    for (int l = 0; l < 16; ++l) grad_coarse[l] = acc[16 * 27 + l] / nsamples;
  return CFDB_OK;
}

}  // extern "C"
