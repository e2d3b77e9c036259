// Persistent Jacobi-PCG with TMA-staged sweeps (included by pcg.cu).
//
// Same algorithm and reductions as the register-staged kernel; the
// differences are the order in which blocks take chunks (SlabIter) and how a
// chunk reaches shared memory: one thread issues
// cp.async.bulk.tensor loads of the chunk's halo box (and interior boxes)
// into one of two stages while the block computes the other stage, and every
// thread waits on the stage's mbarrier (bounded).  Requires the row pitch to
// be a multiple of 16 bytes (nx even in FP64, nx % 4 == 0 in FP32); boxes
// start 16/sizeof(T) cells left of the chunk so that x is 16-byte aligned.
#pragma once

template <typename T, int TX_, int TY_, int TZ_>
struct TmaShape {
  static constexpr int XO = 16 / (int)sizeof(T);
  static constexpr bool D3 = TY_ > 1;
  static constexpr int OY = D3 ? 1 : 0;
  static constexpr int TX = TX_, TY = TY_, TZ = TZ_;
  static constexpr int HX = TX + 2 * XO, HY = D3 ? TY + 2 : 1, HZ = TZ + 2;
  static constexpr int HALO = HX * HY * HZ;
  static constexpr int INTR = TX * TY * TZ;
  static constexpr int pad(int elems) { return ((elems * (int)sizeof(T) + 127) / 128) * 128 / (int)sizeof(T); }
  static constexpr int HALO_P = pad(HALO), INTR_P = pad(INTR);
  static constexpr int STAGE = (2 * HALO_P > HALO_P + 2 * INTR_P) ? 2 * HALO_P : HALO_P + 2 * INTR_P;
  static constexpr uint32_t BYTES_A = 2u * HALO * sizeof(T);
  static constexpr uint32_t BYTES_B = (uint32_t)(HALO + 2 * INTR) * sizeof(T);
};

template <typename T>
using TmaTile2D = TmaShape<T, 128, 1, 32>;
template <typename T>
using TmaTile3D = TmaShape<T, 32, 8, 12>;

struct alignas(64) TmaMaps {
  CUtensorMap z_halo, p0_halo, p1_halo, x_int, r_int;
};

template <typename T>
struct TmaParams {
  TmaMaps maps;
  PcgParams<T> P;
};

// Chunks of a sweep in slab order: chunk g is column g % C (C columns of
// TX x TY cells) of the z-slab g / C (TZ planes), and block b takes chunks b,
// b + B, b + 2B, ...  All blocks then work on neighbouring columns of the
// same slab at the same time, so the halo planes one block loads are still
// in L2 when its neighbours load them; blocks marching their own runs of
// columns along z meet their neighbours' planes long after L2 has evicted
// them, and every halo comes from DRAM again (measured: 1.6x the algorithmic
// bytes at 256^3).
struct SlabIter {
  int64_t g;
  template <int TZ>
  __device__ __forceinline__ bool next(const ColumnSplit& cs, int nz, int tx, int ty, int B,
                                       Chunk& c) {
    const int64_t cols = (int64_t)cs.cols_x * cs.cols_y;
    if (g >= cols * ((nz + TZ - 1) / TZ)) return false;
    const int64_t col = g % cols;
    c.i0 = (int)(col % cs.cols_x) * tx;
    c.j0 = (int)(col / cs.cols_x) * ty;
    c.z0 = (int)(g / cols) * TZ;
    c.z1 = min(c.z0 + TZ, nz);
    g += B;
    return true;
  }
};


// Per-column part of a cell's coefficients: the x/y couplings and their
// partial diagonal sum are constant along z, so a thread walking a column
// loads them once.  raw* keep boundary faces (they enter the diagonal),
// c* are the couplings (zero across a boundary).
template <typename T>
struct ColCoef {
  T sxy;                 // ((xl + xh) + yl) + yh, the reference's summation order
  T cxl, cxh, cyl, cyh;  // couplings
  bool has_ref;          // the pinned reference cell lies in this column
  int ref_k;
};

template <typename T>
__device__ __forceinline__ ColCoef<T> column_coef(const OpView<T>& A, int i, int j) {
  ColCoef<T> c;
  const T xl = __ldg(A.tx + i), xh = __ldg(A.tx + i + 1);
  const T yl = __ldg(A.ty + j), yh = __ldg(A.ty + j + 1);
  c.sxy = ((xl + xh) + yl) + yh;
  c.cxl = i > 0 ? xl : T(0);
  c.cxh = i < A.nx - 1 ? xh : T(0);
  c.cyl = j > 0 ? yl : T(0);
  c.cyh = j < A.ny - 1 ? yh : T(0);
  const int64_t plane = (int64_t)A.nx * A.ny;
  const int64_t col = i + (int64_t)A.nx * j;
  c.has_ref = A.pinned && (A.ref % plane) == col;
  c.ref_k = (int)(A.ref / plane);
  return c;
}

// Coefficients of cell (i,j,k) for operators with per-face arrays.
template <typename T>
__device__ __forceinline__ Coef<T> face_coef(const OpView<T>& A, int i, int j, int k) {
  return load_coef(A, i, j, k);
}

constexpr int kTmaThreads = 512;

// The coefficient view the stencil arithmetic of a sweep uses.
template <bool MIXED, typename T>
__device__ __forceinline__ const auto& coef_view(const PcgParams<T>& P) {
  if constexpr (MIXED) return P.A64;
  else return P.A;
}

// MIXED (T = float only): the search direction p and z = D^-1 r are stored in
// FP32 (the vectors the TMA boxes carry); the iterate x and the residual r
// stay in FP64 (P.x64, P.r64, plain coalesced loads in sweep B) and every
// A p is evaluated in FP64 from the FP32-stored p, so the FP64 recurrence
// r -= alpha A p stays consistent with x += alpha p exactly as in the FP64
// solve: only the directions are rounded to FP32.  The residual is also
// replaced by the FP64 b - A x (one plain sweep) when it has fallen by
// P.delta since the last replacement, when it reaches the tolerance (so
// convergence is decided on the FP64 residual of the iterate) and at the
// iteration cap.  One Krylov space for the whole solve.
template <typename T, class S, bool FACE, bool MIXED>
__global__ void __launch_bounds__(kTmaThreads, 1) pcg_tma(const __grid_constant__ TmaParams<T> TP) {
  static_assert(!MIXED || sizeof(T) == 4, "the mixed-precision solve stores p and z in FP32");
  // coefficients and stencil arithmetic: FP64 in the mixed solve, else T
  using C = typename std::conditional<MIXED, double, T>::type;
  // sweep B stage of the mixed solve: the FP32 p halo box, then FP64 x and r
  // interior boxes (each 128-byte aligned); stage size in T words
  constexpr int XOFF = S::HALO_P, ROFF = S::HALO_P + 2 * S::INTR_P;
  constexpr int STG = MIXED ? (2 * S::HALO_P > ROFF + 2 * S::INTR_P ? 2 * S::HALO_P
                                                                     : ROFF + 2 * S::INTR_P)
                            : S::STAGE;
  extern __shared__ __align__(128) unsigned char smem_tma[];
  T* stage_mem = reinterpret_cast<T*>(smem_tma);
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ double red[64];
  const PcgParams<T>& P = TP.P;
  const OpView<T>& A = P.A;
  const OpView<C>& AC = coef_view<MIXED>(P);
  const int B = gridDim.x, blk = blockIdx.x;
  const int tid = threadIdx.x;
  const bool leader = (blk == 0 && tid == 0);
  const ColumnSplit cs = P.cs;
  int round = 0;
  auto part = [&]() { return P.partials + (size_t)(round & 1) * 2 * B; };
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  uint32_t parity[2] = {0u, 0u};

  auto idx_of = [&](int i, int j, int k) { return i + (int64_t)A.nx * (j + (int64_t)A.ny * k); };

  // Generic pipelined sweep: load(c, base, bar) issues the chunk's TMA copies
  // (thread 0), body(c, base) computes it.  Returns false on a failed wait;
  // before that, thread 0 waits (bounded) for the copies still in flight in
  // either stage, so that the block leaves no bulk copy writing its shared
  // memory behind.
  auto pipeline = [&](auto load, auto body) -> bool {
    SlabIter ld{blk}, cp{blk};
    Chunk cl, cc;
    if (ld.template next<S::TZ>(cs, A.nz, S::TX, S::TY, B, cl) && tid == 0)
      load(cl, stage_mem, &bars[0]);
    int q = 0;
    while (cp.template next<S::TZ>(cs, A.nz, S::TX, S::TY, B, cc)) {
      const int st = q & 1;
      Chunk cn;
      const bool issued = ld.template next<S::TZ>(cs, A.nz, S::TX, S::TY, B, cn);
      if (issued && tid == 0)
        load(cn, stage_mem + (size_t)(st ^ 1) * STG, &bars[st ^ 1]);
      const bool ok = mbar_wait(&bars[st], parity[st], P.sync.error, P.sync.timeout_ns);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          if (!ok) mbar_drain(&bars[st], parity[st], P.sync.timeout_ns);
          if (issued) mbar_drain(&bars[st ^ 1], parity[st ^ 1], P.sync.timeout_ns);
        }
        return false;
      }
      parity[st] ^= 1u;
      body(cc, stage_mem + (size_t)st * STG);
      __syncthreads();
      ++q;
    }
    return true;
  };

  // FP64 residual b64 - A64 x64 of the cells of this block into r64, with
  // z = D^-1 r stored in FP32 (MIXED): the initial residual and every
  // replacement
  auto true_residual = [&](bool x_zero, double (&acc)[2]) {
    SlabIter cp{blk};
    Chunk c;
    while (cp.template next<S::TZ>(cs, A.nz, S::TX, S::TY, B, c)) {
      const int n = S::TX * S::TY * (c.z1 - c.z0);
      for (int q = tid; q < n; q += kTmaThreads) {
        const int i = c.i0 + q % S::TX, j = c.j0 + (q / S::TX) % S::TY, k = c.z0 + q / (S::TX * S::TY);
        if (i >= A.nx || j >= A.ny) continue;
        const int64_t idx = idx_of(i, j, k);
        const Coef<double> c64 = load_coef(P.A64, i, j, k);
        double rd = P.b64[idx];
        if (!x_zero) {
          auto xv = [&](int ii, int jj, int kk) {
            return (ii >= 0 && ii < A.nx && jj >= 0 && jj < A.ny && kk >= 0 && kk < A.nz)
                       ? P.x64[idx_of(ii, jj, kk)] : 0.0;
          };
          rd = rd - apply_coef(c64, P.x64[idx], xv(i - 1, j, k), xv(i + 1, j, k), xv(i, j - 1, k),
                               xv(i, j + 1, k), xv(i, j, k - 1), xv(i, j, k + 1));
        }
        P.r64[idx] = rd;
        const T zn = (T)(c64.inv * rd);
        P.z[idx] = zn;
        acc[0] += rd * rd;
        acc[1] += rd * (double)zn;
      }
    }
  };

  // ---- r0 = b - A x0 (plain loads: once per solve), ||r0||^2, r0.z0
  double acc[2] = {0.0, 0.0};
  if constexpr (MIXED) {
    true_residual(P.x0_zero != 0, acc);
  } else {
    SlabIter cp{blk};
    Chunk c;
    while (cp.template next<S::TZ>(cs, A.nz, S::TX, S::TY, B, c)) {
      const int n = S::TX * S::TY * (c.z1 - c.z0);
      for (int q = tid; q < n; q += kTmaThreads) {
        const int i = c.i0 + q % S::TX, j = c.j0 + (q / S::TX) % S::TY, k = c.z0 + q / (S::TX * S::TY);
        if (i >= A.nx || j >= A.ny) continue;
        const int64_t idx = idx_of(i, j, k);
        const Coef<T> cf = load_coef(A, i, j, k);
        T rn = __ldg(P.b + idx);
        if (!P.x0_zero) {
          auto xv = [&](int ii, int jj, int kk) {
            return (ii >= 0 && ii < A.nx && jj >= 0 && jj < A.ny && kk >= 0 && kk < A.nz)
                       ? P.x[idx_of(ii, jj, kk)] : T(0);
          };
          rn = rn - apply_coef(cf, P.x[idx], xv(i - 1, j, k), xv(i + 1, j, k), xv(i, j - 1, k),
                               xv(i, j + 1, k), xv(i, j, k - 1), xv(i, j, k + 1));
        }
        P.r[idx] = rn;
        const T zn = cf.inv * rn;
        P.z[idx] = zn;
        const double rd = (double)rn;
        acc[0] += rd * rd;
        acc[1] += rd * (double)zn;
      }
    }
  }
  block_sum<2>(acc, red);
  if (tid == 0) {
    part()[2 * blk] = acc[0];
    part()[2 * blk + 1] = acc[1];
  }
  if (!grid_sync(P.sync)) return;
  double tot[2];
  grid_total<2>(part(), 2, B, tot, red);
  ++round;
  const double b0 = sqrt(tot[0]);
  double rz = tot[1];
  auto converged = [&](double res) {
    return (res <= P.abs_tol) || ((b0 > 0.0) && (res / b0 <= P.rel_tol));
  };
  if (leader) {
    P.out[OUT_B0] = b0;
    if (P.hist_cap > 0) P.hist[0] = b0;
  }
  if (b0 == 0.0 || converged(b0) || !finite(rz)) {
    if (leader) {
      P.out[OUT_STATUS] = (b0 == 0.0 || converged(b0)) ? CFDB_SOLVER_CONVERGED : CFDB_SOLVER_BREAKDOWN;
      P.out[OUT_ITER] = 0;
      P.out[OUT_FINAL] = b0;
    }
    return;
  }

  double res_cur = b0;
  double beta = 0.0;
  bool pold_is_p0 = true;
  double res_replaced = b0;  // MIXED: FP64 residual at the last replacement
  int64_t replacements = 0;
  for (int64_t it = 1; it <= P.max_it; ++it) {
    const bool first = (it == 1);
    const T tbeta = (T)beta;
    const CUtensorMap* pold_map = pold_is_p0 ? &TP.maps.p0_halo : &TP.maps.p1_halo;
    const CUtensorMap* pnew_map = pold_is_p0 ? &TP.maps.p1_halo : &TP.maps.p0_halo;
    T* pnew = pold_is_p0 ? P.p1 : P.p0;
    // ---- sweep A: stage z = D^-1 r and p_old halo boxes; p = z + beta p_old; Ap; p.Ap
    double pap = 0.0;
    const bool okA = pipeline(
        [&](const Chunk& c, T* base, uint64_t* bar) {
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(bar, S::BYTES_A);
          const int hx = c.i0 - S::XO, hy = c.j0 - S::OY, hz = c.z0 - 1;
          if constexpr (S::D3) {
            tma_load_3d(base, &TP.maps.z_halo, hx, hy, hz, bar);
            tma_load_3d(base + S::HALO_P, pold_map, hx, hy, hz, bar);
          } else {
            tma_load_2d(base, &TP.maps.z_halo, hx, hz, bar);
            tma_load_2d(base + S::HALO_P, pold_map, hx, hz, bar);
          }
        },
        [&](const Chunk& c, T* base) {
          // p = z + beta p_old is formed where it is read, by the same fma
          // everywhere, so each value equals the one stored; outside the
          // domain both boxes hold the TMA fill 0 and so does p
          const T* zb = base;
          const T* pb = base + S::HALO_P;
          auto pv = [&](int e) { return first ? zb[e] : fma(tbeta, pb[e], zb[e]); };
          const int zl = c.z1 - c.z0;
          constexpr int PL = S::HX * S::HY;  // box plane stride
          // one thread per column (x fastest), z neighbours carried in registers
          constexpr int ICOL = S::TX * S::TY;
          constexpr int SPLIT = kTmaThreads / ICOL > 0 ? kTmaThreads / ICOL : 1;
          for (int t = tid; t < ICOL * SPLIT; t += kTmaThreads) {
            const int col = t % ICOL, part_z = t / ICOL;
            const int qx = col % S::TX, qy = col / S::TX;
            const int i = c.i0 + qx, j = c.j0 + qy;
            if (i >= A.nx || j >= A.ny) continue;
            const int kb = zl * part_z / SPLIT, ke = zl * (part_z + 1) / SPLIT;
            int e = (qx + S::XO) + S::HX * (qy + S::OY) + PL * (kb + 1);
            int64_t idx = i + (int64_t)A.nx * (j + (int64_t)A.ny * (c.z0 + kb));
            const int64_t pstride = (int64_t)A.nx * A.ny;
            T lo = pv(e - PL), v = pv(e);
            if constexpr (FACE) {
              for (int kk = kb; kk < ke; ++kk, e += PL, idx += pstride) {
                const T hi = pv(e + PL);
                const Coef<C> cf = face_coef(AC, i, j, c.z0 + kk);
                const C ap = apply_coef(cf, (C)v, (C)pv(e - 1), (C)pv(e + 1),
                                        S::D3 ? (C)pv(e - S::HX) : C(0),
                                        S::D3 ? (C)pv(e + S::HX) : C(0), (C)lo, (C)hi);
                pnew[idx] = v;
                pap += (double)v * (double)ap;
                lo = v;
                v = hi;
              }
            } else {
              const ColCoef<C> cc = column_coef(AC, i, j);
              for (int kk = kb; kk < ke; ++kk, e += PL, idx += pstride) {
                const int k = c.z0 + kk;
                const T hi = pv(e + PL);
                const C zl_ = __ldg(AC.tz + k), zh_ = __ldg(AC.tz + k + 1);
                C ap;
                if (cc.has_ref && k == cc.ref_k) {
                  ap = (C)v;
                } else {
                  const C dg = (cc.sxy + zl_) + zh_;
                  C off = cc.cxl * (C)pv(e - 1);
                  off = fma(cc.cxh, (C)pv(e + 1), off);
                  if (S::D3) {
                    off = fma(cc.cyl, (C)pv(e - S::HX), off);
                    off = fma(cc.cyh, (C)pv(e + S::HX), off);
                  }
                  off = fma(k > 0 ? zl_ : C(0), (C)lo, off);
                  off = fma(k < A.nz - 1 ? zh_ : C(0), (C)hi, off);
                  ap = fma(dg, (C)v, -off);
                }
                pnew[idx] = v;
                pap += (double)v * (double)ap;
                lo = v;
                v = hi;
              }
            }
          }
        });
    {
      double a1[1] = {pap};
      block_sum<1>(a1, red);
      if (tid == 0) part()[2 * blk] = a1[0];
    }
    if (!okA || !grid_sync(P.sync)) return;
    double t1[1];
    grid_total<1>(part(), 2, B, t1, red);
    ++round;
    const double pAp = t1[0];
    const double alpha = rz / pAp;
    if (!finite(pAp) || fabs(pAp) < 1.0e-30 || !finite(alpha)) {
      if (leader) {
        P.out[OUT_STATUS] = CFDB_SOLVER_BREAKDOWN;
        P.out[OUT_ITER] = (double)(it - 1);
        P.out[OUT_FINAL] = res_cur;
      }
      return;
    }
    const T talpha = (T)alpha;
    // ---- sweep B: stage p halo, x and r interiors; x += alpha p; r -= alpha A p;
    // z = D^-1 r stored for the next sweep A
    double ab[2] = {0.0, 0.0};
    const bool okB = pipeline(
        [&](const Chunk& c, T* base, uint64_t* bar) {
          fence_proxy_async_smem();
          // MIXED: the x and r boxes are FP64 (maps over x64 and r64)
          mbar_arrive_expect_tx(bar, MIXED ? (uint32_t)(S::HALO * sizeof(T) + 2 * S::INTR * sizeof(double))
                                           : S::BYTES_B);
          const int hx = c.i0 - S::XO, hy = c.j0 - S::OY, hz = c.z0 - 1;
          T* xdst = base + (MIXED ? XOFF : S::HALO_P);
          T* rdst = base + (MIXED ? ROFF : S::HALO_P + S::INTR_P);
          if constexpr (S::D3) {
            tma_load_3d(base, pnew_map, hx, hy, hz, bar);
            tma_load_3d(xdst, &TP.maps.x_int, c.i0, c.j0, c.z0, bar);
            tma_load_3d(rdst, &TP.maps.r_int, c.i0, c.j0, c.z0, bar);
          } else {
            tma_load_2d(base, pnew_map, hx, hz, bar);
            tma_load_2d(xdst, &TP.maps.x_int, c.i0, c.z0, bar);
            tma_load_2d(rdst, &TP.maps.r_int, c.i0, c.z0, bar);
          }
        },
        [&](const Chunk& c, T* base) {
          const T* pb = base;
          const T* xb = base + S::HALO_P;
          const T* rb = base + S::HALO_P + S::INTR_P;
          const int zl = c.z1 - c.z0;
          constexpr int PL = S::HX * S::HY;
          constexpr int IPL = S::TX * S::TY;
          constexpr int ICOL = S::TX * S::TY;
          constexpr int SPLIT = kTmaThreads / ICOL > 0 ? kTmaThreads / ICOL : 1;
          for (int t = tid; t < ICOL * SPLIT; t += kTmaThreads) {
            const int col = t % ICOL, part_z = t / ICOL;
            const int qx = col % S::TX, qy = col / S::TX;
            const int i = c.i0 + qx, j = c.j0 + qy;
            if (i >= A.nx || j >= A.ny) continue;
            const int kb = zl * part_z / SPLIT, ke = zl * (part_z + 1) / SPLIT;
            int e = (qx + S::XO) + S::HX * (qy + S::OY) + PL * (kb + 1);
            int q = col + IPL * kb;
            int64_t idx = i + (int64_t)A.nx * (j + (int64_t)A.ny * (c.z0 + kb));
            const int64_t pstride = (int64_t)A.nx * A.ny;
            ColCoef<C> cc;
            if constexpr (!FACE) cc = column_coef(AC, i, j);
            for (int kk = kb; kk < ke; ++kk, e += PL, q += IPL, idx += pstride) {
              const int k = c.z0 + kk;
              const T v = pb[e];
              C ap, inv;
              if constexpr (FACE) {
                const Coef<C> cf = face_coef(AC, i, j, k);
                ap = apply_coef(cf, (C)v, (C)pb[e - 1], (C)pb[e + 1],
                                S::D3 ? (C)pb[e - S::HX] : C(0), S::D3 ? (C)pb[e + S::HX] : C(0),
                                (C)pb[e - PL], (C)pb[e + PL]);
                if constexpr (MIXED) inv = cf.inv;
                else inv = __ldg(P.invd + idx);
              } else if (cc.has_ref && k == cc.ref_k) {
                ap = (C)v;
                inv = C(1);
              } else {
                const C zl_ = __ldg(AC.tz + k), zh_ = __ldg(AC.tz + k + 1);
                const C dg = (cc.sxy + zl_) + zh_;
                C off = cc.cxl * (C)pb[e - 1];
                off = fma(cc.cxh, (C)pb[e + 1], off);
                if (S::D3) {
                  off = fma(cc.cyl, (C)pb[e - S::HX], off);
                  off = fma(cc.cyh, (C)pb[e + S::HX], off);
                }
                off = fma(k > 0 ? zl_ : C(0), (C)pb[e - PL], off);
                off = fma(k < A.nz - 1 ? zh_ : C(0), (C)pb[e + PL], off);
                ap = fma(dg, (C)v, -off);
                inv = rcp_rn(dg);
              }
              if constexpr (MIXED) {
                const double* xb64 = reinterpret_cast<const double*>(base + XOFF);
                const double* rb64 = reinterpret_cast<const double*>(base + ROFF);
                P.x64[idx] = fma(alpha, (double)v, xb64[q]);
                const double rn = fma(-alpha, ap, rb64[q]);
                P.r64[idx] = rn;
                const T zn = (T)(inv * rn);
                P.z[idx] = zn;
                ab[0] += rn * rn;
                ab[1] += rn * (double)zn;
              } else {
                P.x[idx] = fma(talpha, v, xb[q]);
                const T rn = fma(-talpha, ap, rb[q]);
                P.r[idx] = rn;
                const T zn = inv * rn;
                P.z[idx] = zn;
                const double rd = (double)rn;
                ab[0] += rd * rd;
                ab[1] += rd * (double)zn;
              }
            }
          }
        });
    block_sum<2>(ab, red);
    if (tid == 0) {
      part()[2 * blk] = ab[0];
      part()[2 * blk + 1] = ab[1];
    }
    if (!okB || !grid_sync(P.sync)) return;
    grid_total<2>(part(), 2, B, tot, red);
    ++round;
    double res = sqrt(tot[0]);
    if constexpr (MIXED) {
      // replace the FP32 recurrence by the FP64 residual (grid-uniform decision)
      if (finite(res) && (converged(res) || res <= P.delta * res_replaced || it == P.max_it)) {
        if (!grid_sync(P.sync)) return;  // every x64 update of this iteration is visible
        double acc2[2] = {0.0, 0.0};
        true_residual(false, acc2);
        block_sum<2>(acc2, red);
        if (tid == 0) {
          part()[2 * blk] = acc2[0];
          part()[2 * blk + 1] = acc2[1];
        }
        if (!grid_sync(P.sync)) return;
        grid_total<2>(part(), 2, B, tot, red);
        ++round;
        res = sqrt(tot[0]);
        res_replaced = res;
        ++replacements;
        if (leader) P.out[OUT_REPLACEMENTS] = (double)replacements;
      }
    }
    if (leader && it < P.hist_cap) P.hist[it] = res;
    if (!finite(res)) {
      if (leader) {
        P.out[OUT_STATUS] = CFDB_SOLVER_NONFINITE_RESIDUAL;
        P.out[OUT_ITER] = (double)it;
        P.out[OUT_FINAL] = res;
      }
      return;
    }
    res_cur = res;
    if (converged(res)) {
      if (leader) {
        P.out[OUT_STATUS] = CFDB_SOLVER_CONVERGED;
        P.out[OUT_ITER] = (double)it;
        P.out[OUT_FINAL] = res;
      }
      return;
    }
    const double rzNew = tot[1];
    beta = rzNew / rz;
    if (!finite(rzNew) || !finite(beta)) {
      if (leader) {
        P.out[OUT_STATUS] = CFDB_SOLVER_BREAKDOWN;
        P.out[OUT_ITER] = (double)it;
        P.out[OUT_FINAL] = res;
      }
      return;
    }
    rz = rzNew;
    pold_is_p0 = !pold_is_p0;
  }
  if (leader) {
    P.out[OUT_STATUS] = CFDB_SOLVER_MAX_ITERATIONS;
    P.out[OUT_ITER] = (double)P.max_it;
    P.out[OUT_FINAL] = res_cur;
  }
}
