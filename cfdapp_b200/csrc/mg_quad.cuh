// Wide-level variants of the V-cycle and FCG passes (included by mg.cu inside
// its anonymous namespace): every thread owns FOUR CONTIGUOUS cells of a row
// (one float4 / two double2 per array), so global traffic moves in 16-byte
// vectors and the stencil reads a thread's own x-neighbours from registers
// and its own shared-memory row.  Used where the row length is a multiple of
// 4 and at least one tile wide; the one-cell-per-thread kernels of mg.cu
// cover every other level.
//
// Tile: TX x TY threads own a (4*TX) x TY patch of an (x,y) plane and march
// along z exactly like the generic kernels (pair-aligned plane runs).  A
// staged plane row holds x in [x0-1, x0+4*TX] at offsets 3 .. 4*TX+4, so the
// thread's quad sits 16-byte aligned at 4+4*tx.
#pragma once

template <int DIM>
struct Quad;
template <>
struct Quad<2> {
  static constexpr int TX = 64, TY = 1;
};
template <>
struct Quad<3> {
  static constexpr int TX = 32, TY = 8;
};

template <int DIM>
constexpr int quad_px() {
  return 4 * Quad<DIM>::TX;
}

template <int DIM>
bool quad_ok(int nx) {
  return nx % 4 == 0 && nx >= quad_px<DIM>();
}

// Blocks of a quad pass: 2D blocks are 64 threads, so up to 32 per SM; a
// pass whose blocks need more registers passes its own cap.
template <int DIM>
int quad_grid(const Seg& s, int64_t cap = DIM == 2 ? 148 * 32 : kGridCap) {
  const int64_t per = std::max<int64_t>(1, (s.items + cap - 1) / cap);
  return (int)std::max<int64_t>(1, (s.items + per - 1) / per);
}

template <int DIM>
Seg make_quad_seg(int nx, int ny, int nz) {
  constexpr int PX = quad_px<DIM>(), PY = Quad<DIM>::TY;
  Seg s;
  s.tiles_x = (nx + PX - 1) / PX;
  const int64_t tiles = (int64_t)s.tiles_x * ((ny + PY - 1) / PY);
  s.pairs = (nz + 1) / 2;
  s.items = tiles * s.pairs;
  return s;
}

template <typename T>
struct V4 {
  T v[4];
};

__device__ __forceinline__ V4<float> ld4(const float* p) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  return V4<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ void st4(float* p, const V4<float>& a) {
  *reinterpret_cast<float4*>(p) = make_float4(a.v[0], a.v[1], a.v[2], a.v[3]);
}
__device__ __forceinline__ V4<double> ld4(const double* p) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  return V4<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(double* p, const V4<double>& a) {
  *reinterpret_cast<double2*>(p) = make_double2(a.v[0], a.v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(a.v[2], a.v[3]);
}
template <typename T>
__device__ __forceinline__ V4<T> zero4() {
  return V4<T>{{T(0), T(0), T(0), T(0)}};
}

// 7-point march over quads.  val4(i0,j,k) -> the quad's stencil inputs,
// val1(i,j,k) -> one input (x-halo).  cell(act, i0, j, k, v, w, e, s, n, b,
// t) gets the quad and its six neighbour quads; after(k) runs in every
// thread once per plane.
template <typename T, int TX, int TY, class Val4, class Val1, class Cell, class After>
__device__ __forceinline__ void march7q(int nx, int ny, int nz, int tix, int tiy, int k0, int k1,
                                        T (*buf)[Rows<TY>::N][4 * TX + 8], Val4 val4, Val1 val1,
                                        Cell cell, After after) {
  constexpr int PX = 4 * TX, R0 = Rows<TY>::R0;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int x0 = tix * PX, i0 = x0 + 4 * tx, j = tiy * TY + ty;
  const bool act = i0 < nx && j < ny;
  V4<T> vp = zero4<T>(), vc = zero4<T>(), vn;
  if (act) {
    if (k0 > 0) vp = val4(i0, j, k0 - 1);
    vc = val4(i0, j, k0);
  }
  for (int k = k0; k < k1; ++k) {
    vn = (act && k + 1 < nz) ? val4(i0, j, k + 1) : zero4<T>();
    T(*s)[PX + 8] = buf[k & 1];
    st4(&s[ty + R0][4 + 4 * tx], vc);
    if (tx == 0) s[ty + R0][3] = (j < ny && x0 > 0) ? val1(x0 - 1, j, k) : T(0);
    if (tx == TX - 1) s[ty + R0][PX + 4] = (j < ny && x0 + PX < nx) ? val1(x0 + PX, j, k) : T(0);
    if (TY > 1) {
      if (ty == 0) st4(&s[0][4 + 4 * tx], (j > 0 && i0 < nx) ? val4(i0, j - 1, k) : zero4<T>());
      if (ty == TY - 1)
        st4(&s[TY + 1][4 + 4 * tx], (j + 1 < ny && i0 < nx) ? val4(i0, j + 1, k) : zero4<T>());
    }
    __syncthreads();
    V4<T> w, e, sv = zero4<T>(), nv = zero4<T>();
    w.v[0] = s[ty + R0][3 + 4 * tx];
    e.v[3] = s[ty + R0][8 + 4 * tx];
#pragma unroll
    for (int q = 1; q < 4; ++q) w.v[q] = vc.v[q - 1];
#pragma unroll
    for (int q = 0; q < 3; ++q) e.v[q] = vc.v[q + 1];
    if (TY > 1) {
      sv = ld4(&s[ty][4 + 4 * tx]);
      nv = ld4(&s[ty + 2][4 + 4 * tx]);
    }
    cell(act, i0, j, k, vc, w, e, sv, nv, vp, vn);
    after(k);
    vp = vc;
    vc = vn;
  }
  __syncthreads();
}

// Face couplings of the quad at (i0, j, k) (level layout, float).
template <int DIM>
__device__ __forceinline__ void coef4(const LV& L, int i0, int j, int k, float (&fxs)[5],
                                      V4<float>& yl, V4<float>& yh, V4<float>& zl, V4<float>& zh) {
  const int64_t bx = i0 + (int64_t)(L.nx + 1) * (j + (int64_t)L.ny * k);
#pragma unroll
  for (int q = 0; q < 5; ++q) fxs[q] = L.fx[bx + q];
  if (DIM == 3) {
    const int64_t by = i0 + (int64_t)L.nx * (j + (int64_t)(L.ny + 1) * k);
    yl = ld4(L.fy + by);
    yh = ld4(L.fy + by + L.nx);
  } else {
    yl = yh = zero4<float>();
  }
  const int64_t c = at(L, i0, j, k);
  zl = ld4(L.fz + c);
  zh = ld4(L.fz + c + (int64_t)L.nx * L.ny);
}

// The quad counterpart of k_res (see there).
// 3D: four resident blocks per SM (64 registers, no spills): 2.6 % faster
// per FCG iteration at 256^3; 2D keeps the compiler's own allocation.
template <int DIM, bool PRO, bool RESTRICT>
__global__ void __launch_bounds__(Quad<DIM>::TX* Quad<DIM>::TY, DIM == 3 ? 4 : 0)
    k_res_q(LV L, LV C, Seg sg, const float* __restrict__ x, const float* __restrict__ ec, float cw,
            const float* __restrict__ r, float* __restrict__ res, float* __restrict__ rc,
            int64_t skip) {
  pdl_enter();
  constexpr int TX = Quad<DIM>::TX, TY = Quad<DIM>::TY, PX = 4 * TX;
  __shared__ __align__(16) float buf[2][Rows<TY>::N][PX + 8];
  __shared__ float2 rows[TY][TX];
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  auto val4 = [&](int i, int j, int k) {
    V4<float> v = ld4(x + at(L, i, j, k));
    if (PRO) {
      const int64_t pc = parent(C, i, j, k);
      const float a = cw * ec[pc], b = cw * ec[pc + 1];
      v.v[0] += a;
      v.v[1] += a;
      v.v[2] += b;
      v.v[3] += b;
    }
    return v;
  };
  auto val1 = [&](int i, int j, int k) {
    float v = x[at(L, i, j, k)];
    if (PRO) v += cw * ec[parent(C, i, j, k)];
    return v;
  };
  for_runs(sg, L.nz, [&](int tix, int tiy, int k0, int k1) {
    float2 racc = make_float2(0.f, 0.f);
    float2 pair = make_float2(0.f, 0.f);
    const int i0 = tix * PX + 4 * tx, j = tiy * TY + ty;
    march7q<float, TX, TY>(
        L.nx, L.ny, L.nz, tix, tiy, k0, k1, buf, val4, val1,
        [&](bool act, int i0_, int jj, int k, const V4<float>& v, const V4<float>& w,
            const V4<float>& e, const V4<float>& s, const V4<float>& n, const V4<float>& b,
            const V4<float>& t) {
          pair = make_float2(0.f, 0.f);
          if (!act) return;
          float fx[5];
          V4<float> yl, yh, zl, zh;
          coef4<DIM>(L, i0_, jj, k, fx, yl, yh, zl, zh);
          const int64_t c = at(L, i0_, jj, k);
          V4<float> rr = ld4(r + c);
          V4<float> out;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float d = ((fx[q] + fx[q + 1]) + (yl.v[q] + yh.v[q])) + (zl.v[q] + zh.v[q]);
            const float ax = d * v.v[q] - (((fx[q] * w.v[q] + fx[q + 1] * e.v[q]) +
                                            (yl.v[q] * s.v[q] + yh.v[q] * n.v[q])) +
                                           (zl.v[q] * b.v[q] + zh.v[q] * t.v[q]));
            out.v[q] = (c + q == skip ? 0.f : rr.v[q]) - ax;
          }
          if (!RESTRICT) st4(res + c, out);
          pair = make_float2(out.v[0] + out.v[1], out.v[2] + out.v[3]);
        },
        [&](int k) {
          if constexpr (!RESTRICT) return;
          float2 quad = pair;
          if (TY > 1) {
            if (ty & 1) rows[ty][tx] = pair;
            __syncthreads();
            if ((ty & 1) == 0) {
              const float2 o = rows[ty + 1][tx];
              quad.x += o.x;
              quad.y += o.y;
            }
          }
          if ((k & 1) == 0) {
            racc = quad;
          } else {
            racc.x += quad.x;
            racc.y += quad.y;
          }
          const bool flush = (k & 1) == 1 || k + 1 == L.nz;
          if (flush && (TY == 1 || (ty & 1) == 0) && i0 < L.nx && j < L.ny) {
            const int64_t qc = (i0 >> 1) + (int64_t)C.nx * ((j >> 1) + (int64_t)C.ny * (k >> 1));
            rc[qc] = racc.x;
            rc[qc + 1] = racc.y;
          }
        });
  });
}

// The quad counterpart of k_sm (see there): 27-point (2D: 9-point)
// convolution over a three-plane ring of staged rows.
template <int DIM, int MODE, bool HOOK>
__global__ void __launch_bounds__(Quad<DIM>::TX* Quad<DIM>::TY)
    k_sm_q(LV L, LV C, Seg sg, Kern K, const float* __restrict__ src, const float* __restrict__ ec,
           float cw, float* __restrict__ x, int64_t skip, int64_t pin, const float* __restrict__ r,
           Hook hk) {
  pdl_enter();
  constexpr int TX = Quad<DIM>::TX, TY = Quad<DIM>::TY, PX = 4 * TX, R0 = Rows<TY>::R0;
  constexpr int NR = Rows<TY>::N;
  __shared__ __align__(16) float ring[3][NR][PX + 8];
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  double acc_dot = 0.0;
  for_runs(sg, L.nz, [&](int tix, int tiy, int k0, int k1) {
    const int x0 = tix * PX, i0 = x0 + 4 * tx, j = tiy * TY + ty;
    auto load = [&](int kp, int slot) {
      const bool zin = kp >= 0 && kp < L.nz;
      for (int row = ty; row < NR; row += TY) {
        const int gj = tiy * TY + row - R0;
        const bool rin = zin && gj >= 0 && gj < L.ny;
        float* sr = ring[slot][row];
        V4<float> u = zero4<float>();
        if (rin && i0 < L.nx) {
          const int64_t c = at(L, i0, gj, kp);
          u = ld4(src + c);
          const V4<float> is = ld4(L.isq + c);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            u.v[q] *= is.v[q];
            if (MODE == SM_FIRST && c + q == skip) u.v[q] = 0.f;
          }
        }
        st4(sr + 4 + 4 * tx, u);
        if (tx == 0) {
          float h = 0.f;
          if (rin && x0 > 0) {
            const int64_t c = at(L, x0 - 1, gj, kp);
            h = (MODE == SM_FIRST && c == skip) ? 0.f : src[c] * L.isq[c];
          }
          sr[3] = h;
        }
        if (tx == TX - 1) {
          float h = 0.f;
          if (rin && x0 + PX < L.nx) {
            const int64_t c = at(L, x0 + PX, gj, kp);
            h = (MODE == SM_FIRST && c == skip) ? 0.f : src[c] * L.isq[c];
          }
          sr[PX + 4] = h;
        }
      }
    };
    int lo = 0, mi = 1, hi = 2;
    load(k0 - 1, lo);
    load(k0, mi);
    for (int k = k0; k < k1; ++k) {
      load(k + 1, hi);
      __syncthreads();
      float a[4] = {0.f, 0.f, 0.f, 0.f};
      const int sl[3] = {lo, mi, hi};
#pragma unroll
      for (int dk = 0; dk < 3; ++dk)
#pragma unroll
        for (int dj = (TY > 1 ? -1 : 0); dj <= (TY > 1 ? 1 : 0); ++dj) {
          const float* row = ring[sl[dk]][ty + R0 + dj];
          const V4<float> m = ld4(row + 4 + 4 * tx);
          const float v[6] = {row[3 + 4 * tx], m.v[0], m.v[1], m.v[2], m.v[3], row[8 + 4 * tx]};
#pragma unroll
          for (int di = 0; di < 3; ++di) {
            const float wt = K.w[dk * 9 + (dj + 1) * 3 + di];
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] += wt * v[q + di];
          }
        }
      if (i0 < L.nx && j < L.ny) {
        const int64_t c = at(L, i0, j, k);
        const V4<float> is = ld4(L.isq + c);
        V4<float> o;
        if (MODE == SM_ADD) o = ld4(x + c);
        else o = zero4<float>();
        float e0 = 0.f, e1 = 0.f;
        if (ec) {
          const int64_t pc = parent(C, i0, j, k);
          e0 = cw * ec[pc];
          e1 = cw * ec[pc + 1];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float vq = o.v[q] + is.v[q] * a[q];
          if (ec) vq += (q < 2 ? e0 : e1);
          if (c + q == pin) vq = r[c + q];
          o.v[q] = vq;
        }
        st4(x + c, o);
        if (HOOK) {
          const V4<double> qq = ld4(hk.q + c);
#pragma unroll
          for (int q = 0; q < 4; ++q) acc_dot += (double)o.v[q] * qq.v[q];
        }
      }
      __syncthreads();
      const int t = lo;
      lo = mi;
      mi = hi;
      hi = t;
    }
  });
  if (HOOK) {
    double acc[1] = {acc_dot};
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

// The quad counterpart of the FCG direction pass (see k_fcg_dir).
// Resident blocks per SM of the direction pass (its register budget); its
// grid is one wave of them, so every block marches a long run of planes.
// TABLES: the operator's couplings are its per-axis tables (a uniform
// operator), which needs fewer registers than the per-face form.
template <int DIM, bool TABLES = false>
constexpr int dir_blocks_per_sm() {
  return DIM == 3 ? 2 : (TABLES ? 12 : 8);
}

template <int DIM, bool TABLES = false>
__global__ void __launch_bounds__(Quad<DIM>::TX* Quad<DIM>::TY, dir_blocks_per_sm<DIM, TABLES>())
    k_fcg_dir_q(OpView<double> A, Seg sg, FcgState* S, const float* __restrict__ z, double* P0,
                double* P1, double* __restrict__ q, const double* __restrict__ r, double* partials,
                Loop h) {
  pdl_enter();
  constexpr int TX = Quad<DIM>::TX, TY = Quad<DIM>::TY, PX = 4 * TX;
  __shared__ __align__(16) double buf[2][Rows<TY>::N][PX + 8];
  if (S->done) return;
  const long long it = S->it;
  const bool first = (it == 0);
  const double beta = first ? 0.0 : S->beta;
  double* __restrict__ pn = (it & 1) ? P1 : P0;
  const double* __restrict__ po = (it & 1) ? P0 : P1;
  auto idx = [&](int i, int j, int k) { return i + (int64_t)A.nx * (j + (int64_t)A.ny * k); };
  auto val4 = [&](int i, int j, int k) {
    const int64_t c = idx(i, j, k);
    const V4<float> zz = ld4(z + c);
    V4<double> v;
    if (first) {
#pragma unroll
      for (int t = 0; t < 4; ++t) v.v[t] = (double)zz.v[t];
    } else {
      const V4<double> p = ld4(po + c);
#pragma unroll
      for (int t = 0; t < 4; ++t) v.v[t] = fma(-beta, p.v[t], (double)zz.v[t]);
    }
    return v;
  };
  auto val1 = [&](int i, int j, int k) {
    const int64_t c = idx(i, j, k);
    return first ? (double)z[c] : fma(-beta, po[c], (double)z[c]);
  };
  double acc[2] = {0.0, 0.0};
  for_runs(sg, A.nz, [&](int tix, int tiy, int k0, int k1) {
    march7q<double, TX, TY>(
        A.nx, A.ny, A.nz, tix, tiy, k0, k1, buf, val4, val1,
        [&](bool act, int i0, int j, int k, const V4<double>& v, const V4<double>& w,
            const V4<double>& e, const V4<double>& s, const V4<double>& n, const V4<double>& b,
            const V4<double>& t) {
          if (!act) return;
          const int64_t c = idx(i0, j, k);
          // couplings of the quad: per-face arrays or per-axis tables
          double fx[5];
          if (!TABLES && A.fx) {
            const int64_t bx = i0 + (int64_t)(A.nx + 1) * (j + (int64_t)A.ny * k);
#pragma unroll
            for (int u = 0; u < 5; ++u) fx[u] = A.fx[bx + u];
          } else {
#pragma unroll
            for (int u = 0; u < 5; ++u) fx[u] = A.tx[i0 + u];
          }
          V4<double> yl, yh, zl, zh;
          if (!TABLES && A.fy) {
            const int64_t by = i0 + (int64_t)A.nx * (j + (int64_t)(A.ny + 1) * k);
            yl = ld4(A.fy + by);
            yh = ld4(A.fy + by + A.nx);
          } else {
            const double a = A.ty[j], bb = A.ty[j + 1];
            yl = V4<double>{{a, a, a, a}};
            yh = V4<double>{{bb, bb, bb, bb}};
          }
          if (!TABLES && A.fz) {
            zl = ld4(A.fz + c);
            zh = ld4(A.fz + c + (int64_t)A.nx * A.ny);
          } else {
            const double a = A.tz[k], bb = A.tz[k + 1];
            zl = V4<double>{{a, a, a, a}};
            zh = V4<double>{{bb, bb, bb, bb}};
          }
          V4<double> aq;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            // diagonal summed in the reference's face order (as load_coef)
            const double d =
                ((((fx[u] + fx[u + 1]) + yl.v[u]) + yh.v[u]) + zl.v[u]) + zh.v[u];
            double off = fx[u] * w.v[u];
            off = fma(fx[u + 1], e.v[u], off);
            off = fma(yl.v[u], s.v[u], off);
            off = fma(yh.v[u], n.v[u], off);
            off = fma(zl.v[u], b.v[u], off);
            off = fma(zh.v[u], t.v[u], off);
            aq.v[u] = (A.pinned && c + u == A.ref) ? v.v[u] : fma(d, v.v[u], -off);
          }
          st4(pn + c, v);
          st4(q + c, aq);
          const V4<double> rr = ld4(r + c);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            acc[0] += v.v[u] * aq.v[u];
            acc[1] += v.v[u] * rr.v[u];
          }
        },
        [](int) {});
  });
  reduce_last<2>(acc, partials, &S->ticket, [&](const double* tot) {
    const double pq = tot[0], pr = tot[1];
    const double alpha = pr / pq;
    if (!isfinite(pq) || !(pq > 0.0) || !isfinite(alpha)) {
      stop_loop(S, h, kLearnedStagnated);
      return;
    }
    S->pq = pq;
    S->pr = pr;
    S->alpha = alpha;
  });
}

// The direction pass without a marching tile: one thread per four-cell quad,
// its six neighbour values read straight from global memory (L1/L2 serve the
// re-reads of the neighbouring quads), so a thread keeps little state and
// many warps stay resident to hide DRAM latency.  Same arithmetic and
// coefficient order as k_fcg_dir_q.
template <int DIM>
__global__ void __launch_bounds__(256) k_fcg_dir_v(OpView<double> A, FcgState* S,
                                                   const float* __restrict__ z, double* P0,
                                                   double* P1, double* __restrict__ q,
                                                   const double* __restrict__ r, double* partials,
                                                   Loop h) {
  pdl_enter();
  if (S->done) return;
  const long long it = S->it;
  const bool first = (it == 0);
  const double beta = first ? 0.0 : S->beta;
  double* __restrict__ pn = (it & 1) ? P1 : P0;
  const double* __restrict__ po = (it & 1) ? P0 : P1;
  const int nx = A.nx, ny = A.ny, nz = A.nz, qxn = nx >> 2;
  const int nq = qxn * ny * nz;
  const int64_t plane = (int64_t)nx * ny;
  auto val4 = [&](int64_t c) {
    const V4<float> zz = ld4(z + c);
    V4<double> v;
    if (first) {
#pragma unroll
      for (int t = 0; t < 4; ++t) v.v[t] = (double)zz.v[t];
    } else {
      const V4<double> p = ld4(po + c);
#pragma unroll
      for (int t = 0; t < 4; ++t) v.v[t] = fma(-beta, p.v[t], (double)zz.v[t]);
    }
    return v;
  };
  auto val1 = [&](int64_t c) { return first ? (double)z[c] : fma(-beta, po[c], (double)z[c]); };
  const V4<double> zero{{0.0, 0.0, 0.0, 0.0}};
  double acc[2] = {0.0, 0.0};
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nq; g += gridDim.x * blockDim.x) {
    const int qx = g % qxn, rest = g / qxn;
    const int j = rest % ny, k = rest / ny;
    const int i0 = 4 * qx;
    const int64_t c = i0 + (int64_t)nx * (j + (int64_t)ny * k);
    const V4<double> v = val4(c);
    const double wl = i0 > 0 ? val1(c - 1) : 0.0;
    const double er = i0 + 4 < nx ? val1(c + 4) : 0.0;
    const V4<double> s = (DIM == 3 && j > 0) ? val4(c - nx) : zero;
    const V4<double> n = (DIM == 3 && j + 1 < ny) ? val4(c + nx) : zero;
    const V4<double> b = k > 0 ? val4(c - plane) : zero;
    const V4<double> t = k + 1 < nz ? val4(c + plane) : zero;
    double fx[5];
    if (A.fx) {
      const int64_t bx = i0 + (int64_t)(nx + 1) * (j + (int64_t)ny * k);
#pragma unroll
      for (int u = 0; u < 5; ++u) fx[u] = A.fx[bx + u];
    } else {
#pragma unroll
      for (int u = 0; u < 5; ++u) fx[u] = A.tx[i0 + u];
    }
    V4<double> yl, yh, zl, zh;
    if (A.fy) {
      const int64_t by = i0 + (int64_t)nx * (j + (int64_t)(ny + 1) * k);
      yl = ld4(A.fy + by);
      yh = ld4(A.fy + by + nx);
    } else {
      const double a = A.ty[j], bb = A.ty[j + 1];
      yl = V4<double>{{a, a, a, a}};
      yh = V4<double>{{bb, bb, bb, bb}};
    }
    if (A.fz) {
      zl = ld4(A.fz + c);
      zh = ld4(A.fz + c + plane);
    } else {
      const double a = A.tz[k], bb = A.tz[k + 1];
      zl = V4<double>{{a, a, a, a}};
      zh = V4<double>{{bb, bb, bb, bb}};
    }
    V4<double> aq;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double w = u == 0 ? wl : v.v[u - 1];
      const double e = u == 3 ? er : v.v[u + 1];
      // diagonal summed in the reference's face order (as load_coef)
      const double d = ((((fx[u] + fx[u + 1]) + yl.v[u]) + yh.v[u]) + zl.v[u]) + zh.v[u];
      double off = fx[u] * w;
      off = fma(fx[u + 1], e, off);
      off = fma(yl.v[u], s.v[u], off);
      off = fma(yh.v[u], n.v[u], off);
      off = fma(zl.v[u], b.v[u], off);
      off = fma(zh.v[u], t.v[u], off);
      aq.v[u] = (A.pinned && c + u == A.ref) ? v.v[u] : fma(d, v.v[u], -off);
    }
    st4(pn + c, v);
    st4(q + c, aq);
    const V4<double> rr = ld4(r + c);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      acc[0] += v.v[u] * aq.v[u];
      acc[1] += v.v[u] * rr.v[u];
    }
  }
  reduce_last<2>(acc, partials, &S->ticket, [&](const double* tot) {
    const double pq = tot[0], pr = tot[1];
    const double alpha = pr / pq;
    if (!isfinite(pq) || !(pq > 0.0) || !isfinite(alpha)) {
      stop_loop(S, h, kLearnedStagnated);
      return;
    }
    S->pq = pq;
    S->pr = pr;
    S->alpha = alpha;
  });
}
