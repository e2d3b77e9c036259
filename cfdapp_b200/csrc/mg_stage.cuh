// Staged variants of the 3D wide-level FCG and V-cycle passes (included by
// mg.cu inside its anonymous namespace, after mg_quad.cuh): the same
// per-cell arithmetic as k_res_q / k_sm_q / k_fcg_dir_v, with every plane
// tile brought into shared memory by cp.async D planes ahead of its use, so
// a block keeps loads in flight while it computes instead of stalling on
// each plane's halo and couplings.  Measured on the B200 at 256^3 (warm, per
// FCG iteration, CUPTI): the two residual passes 229 -> 177 us, the
// smoothing passes 256 -> 186 us, the direction pass 197 -> 165 us; the
// whole 37-iteration solve 34.4 -> 28.6 ms.  2D keeps the plane-march
// kernels, which suit its one-row tiles of 64 threads (the staged 2D passes
// measured slower there).
#pragma once

// The cp.async helpers (cp16 / cp8 / cp4, cp_commit, cp_wait) are defined
// in mg.cu ahead of the coarse-level block, which uses them too.

// Staged plane tile of a quad pass (3D: 32 x 8 threads, a 128 x 8 patch): a
// slot holds rows gj = tiy*TY - 1 .. tiy*TY + TY of x in [x0 - 4, x0 + 132)
// as 16-byte chunks (the x halo is one chunk per side, of which the passes
// read the element next to the tile).  Chunk ch: row ch / CPR, column chunk
// ch % CPR.
struct PlaneTile {
  static constexpr int TX = Quad<3>::TX, TY = Quad<3>::TY, T = TX * TY, PX = 4 * TX;
  static constexpr int R0 = Rows<TY>::R0, NR = Rows<TY>::N, W = PX + 8, CPR = W / 4;
  static constexpr int CH = NR * CPR;
  static constexpr int NC = (CH + T - 1) / T;  // chunks per thread (at most)
};

// The chunks a thread copies for every plane of one tile, set up once per
// plane run: chunk q is ch = threadIdx.x + q*T; off = its float offset in a
// slot, xy = its first cell within a plane (-1: outside the level), pxy =
// its parent's within a coarse plane.  For plane kp the cell is xy + kp*nx*ny.
struct TileChunks {
  int n;
  int off[PlaneTile::NC];
  int64_t xy[PlaneTile::NC];
  int64_t pxy[PlaneTile::NC];
  __device__ TileChunks(const LV& L, const LV& C, int tix, int tiy) {
    using P = PlaneTile;
    n = 0;
#pragma unroll
    for (int q = 0; q < P::NC; ++q) {
      const int ch = threadIdx.x + q * P::T;
      off[q] = 0;
      xy[q] = -1;
      pxy[q] = 0;
      if (ch >= P::CH) continue;
      n = q + 1;
      const int row = ch / P::CPR, cx = ch % P::CPR;
      const int gi = tix * P::PX - 4 + 4 * cx, gj = tiy * P::TY + row - P::R0;
      off[q] = row * P::W + 4 * cx;
      if (gj >= 0 && gj < L.ny && gi >= 0 && gi < L.nx) {
        xy[q] = gi + (int64_t)L.nx * gj;
        pxy[q] = (gi >> 1) + (int64_t)C.nx * (gj >> 1);
      }
    }
  }
  // chunk q of plane kp inside the level?  c: its first cell (0 outside)
  __device__ bool at_plane(const LV& L, int q, int kp, int64_t& c) const {
    const bool in = xy[q] >= 0 && kp >= 0 && kp < L.nz;
    c = in ? xy[q] + (int64_t)L.nx * L.ny * kp : 0;
    return in;
  }
};

// ------------------------------------------------------------ residual

// Planes the residual pass keeps in flight ahead of the one it evaluates.
constexpr int kResAhead = 1;
// Per-thread operands of one plane, staged by the thread for itself: the
// quads yl, yh, zl, zh, r, then the five x-face couplings (padded to 8),
// each array [T] over the block's threads.
constexpr int kResQuads = 5;
constexpr int kResOwn = PlaneTile::T * (4 * kResQuads + 8);

// Dynamic shared memory of k_res_s: the x ring (D + 3 plane slots), the
// coarse correction of every staged chunk (two floats, D + 3 slots) and
// D + 1 slots of per-thread operands.
constexpr size_t res_s_smem() {
  using P = PlaneTile;
  constexpr int RS = kResAhead + 3;
  return sizeof(float) *
         ((size_t)RS * P::NR * P::W + (size_t)RS * P::CH * 2 + (size_t)(kResAhead + 1) * kResOwn);
}

// res = r - A x (PRO: x + cw P ec in place of x; RESTRICT: rc(parent) =
// sum of the children's res instead of res), as k_res_q<3>.  The x tiles
// (with cw P ec added by the copying thread once its copies have landed) and
// every thread's own couplings and r arrive by cp.async.
template <bool PRO, bool RESTRICT>
__global__ void __launch_bounds__(PlaneTile::T)
    k_res_s(LV L, LV C, Seg sg, const float* __restrict__ x, const float* __restrict__ ec, float cw,
            const float* __restrict__ r, float* __restrict__ res, float* __restrict__ rc,
            int64_t skip) {
  pdl_enter();
  using P = PlaneTile;
  constexpr int TX = P::TX, TY = P::TY, T = P::T, R0 = P::R0, NR = P::NR, W = P::W;
  constexpr int CH = P::CH, D = kResAhead, RS = D + 3, OS = D + 1;
  constexpr int NQ = kResQuads, OWN = kResOwn;
  extern __shared__ __align__(16) float smem_f[];
  float(*xs)[NR][W] = reinterpret_cast<float(*)[NR][W]>(smem_f);
  float2(*ecs)[CH] = reinterpret_cast<float2(*)[CH]>(smem_f + RS * NR * W);
  float* own = smem_f + RS * NR * W + RS * CH * 2;
  __shared__ float2 rows[TY][TX];
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  for_runs(sg, L.nz, [&](int tix, int tiy, int k0, int k1) {
    const int i0 = tix * P::PX + 4 * tx, j = tiy * TY + ty;
    const bool act = i0 < L.nx && j < L.ny;
    auto slot = [&](int kp) { return (kp + RS) % RS; };  // kp >= -1
    auto quad_at = [&](int s, int q) { return own + (size_t)s * OWN + 4 * (q * T + threadIdx.x); };
    auto fx_at = [&](int s, int u) {
      return own + (size_t)s * OWN + 4 * NQ * T + u * T + threadIdx.x;
    };
    const TileChunks tc(L, C, tix, tiy);
    const int64_t cplane = (int64_t)C.nx * C.ny;
    // plane kp's x tile, and this thread's own operands of plane kp - 1
    auto issue = [&](int kp) {
      const int s = slot(kp);
#pragma unroll
      for (int q = 0; q < P::NC; ++q) {
        if (q >= tc.n) break;
        int64_t c;
        const bool in = tc.at_plane(L, q, kp, c);
        cp16(&xs[s][0][0] + tc.off[q], x + c, in);
        if (PRO) cp8(&ecs[s][threadIdx.x + q * T], ec + (in ? tc.pxy[q] + cplane * (kp >> 1) : 0), in);
      }
      const int ko = kp - 1;
      if (act && ko >= k0 && ko < k1) {
        const int os = ko % OS;
        const int64_t c = at(L, i0, j, ko);
        const int64_t by = i0 + (int64_t)L.nx * (j + (int64_t)(L.ny + 1) * ko);
        cp16(quad_at(os, 0), L.fy + by, true);
        cp16(quad_at(os, 1), L.fy + by + L.nx, true);
        cp16(quad_at(os, 2), L.fz + c, true);
        cp16(quad_at(os, 3), L.fz + c + (int64_t)L.nx * L.ny, true);
        cp16(quad_at(os, 4), r + c, true);
        const int64_t bx = i0 + (int64_t)(L.nx + 1) * (j + (int64_t)L.ny * ko);
#pragma unroll
        for (int u = 0; u < 5; ++u) cp4(fx_at(os, u), L.fx + bx + u, true);
      }
      cp_commit();
    };
    auto land = [&](int kp) {
      if (!PRO) return;
      const int s = slot(kp);
#pragma unroll
      for (int q = 0; q < P::NC; ++q) {
        if (q >= tc.n) break;
        float* xp = &xs[s][0][0] + tc.off[q];
        V4<float> v = ld4(xp);
        const float2 e = ecs[s][threadIdx.x + q * T];
        v.v[0] += cw * e.x;
        v.v[1] += cw * e.x;
        v.v[2] += cw * e.y;
        v.v[3] += cw * e.y;
        st4(xp, v);
      }
    };
    for (int kp = k0 - 1; kp <= k0 + D; ++kp) issue(kp);
    cp_wait<D>();
    land(k0 - 1);
    land(k0);
    float2 racc = make_float2(0.f, 0.f);
    for (int k = k0; k < k1; ++k) {
      issue(k + 1 + D);
      cp_wait<D>();
      land(k + 1);
      __syncthreads();
      float2 pair = make_float2(0.f, 0.f);
      if (act) {
        const int os = k % OS;
        const float* mid = xs[slot(k)][ty + R0];
        const V4<float> v = ld4(mid + 4 + 4 * tx);
        const V4<float> b = ld4(xs[slot(k - 1)][ty + R0] + 4 + 4 * tx);
        const V4<float> t = ld4(xs[slot(k + 1)][ty + R0] + 4 + 4 * tx);
        const V4<float> sv = ld4(xs[slot(k)][ty + R0 - 1] + 4 + 4 * tx);
        const V4<float> nv = ld4(xs[slot(k)][ty + R0 + 1] + 4 + 4 * tx);
        const V4<float> yl = ld4(quad_at(os, 0));
        const V4<float> yh = ld4(quad_at(os, 1));
        const V4<float> zl = ld4(quad_at(os, 2));
        const V4<float> zh = ld4(quad_at(os, 3));
        const V4<float> rr = ld4(quad_at(os, 4));
        float fx[5];
#pragma unroll
        for (int u = 0; u < 5; ++u) fx[u] = *fx_at(os, u);
        const float wl = mid[3 + 4 * tx], er = mid[8 + 4 * tx];
        const int64_t c = at(L, i0, j, k);
        V4<float> out;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float w = u == 0 ? wl : v.v[u - 1];
          const float e = u == 3 ? er : v.v[u + 1];
          const float d = ((fx[u] + fx[u + 1]) + (yl.v[u] + yh.v[u])) + (zl.v[u] + zh.v[u]);
          const float ax = d * v.v[u] - (((fx[u] * w + fx[u + 1] * e) +
                                          (yl.v[u] * sv.v[u] + yh.v[u] * nv.v[u])) +
                                         (zl.v[u] * b.v[u] + zh.v[u] * t.v[u]));
          out.v[u] = (c + u == skip ? 0.f : rr.v[u]) - ax;
        }
        if (!RESTRICT) st4(res + c, out);
        pair = make_float2(out.v[0] + out.v[1], out.v[2] + out.v[3]);
      }
      if (RESTRICT) {
        // pairs of rows, then pairs of planes, sum into the parent cells
        float2 quad = pair;
        if (ty & 1) rows[ty][tx] = pair;
        __syncthreads();
        if ((ty & 1) == 0) {
          const float2 o = rows[ty + 1][tx];
          quad.x += o.x;
          quad.y += o.y;
        }
        if ((k & 1) == 0) {
          racc = quad;
        } else {
          racc.x += quad.x;
          racc.y += quad.y;
        }
        const bool flush = (k & 1) == 1 || k + 1 == L.nz;
        if (flush && (ty & 1) == 0 && act) {
          const int64_t qc = (i0 >> 1) + (int64_t)C.nx * ((j >> 1) + (int64_t)C.ny * (k >> 1));
          rc[qc] = racc.x;
          rc[qc + 1] = racc.y;
        }
      }
      __syncthreads();
    }
    // the run's trailing copies are drained before the next run reuses the
    // slots, or before the block exits
    cp_wait<0>();
  });
}

// ------------------------------------------------------------ smoothing

// Planes a smoothing block keeps in flight ahead of the one it reads.
constexpr int kSmAhead = 2;

// Dynamic shared memory of k_sm_s: two rings (u = src * isq, and isq) of
// D + 1 plane tiles.
constexpr size_t sm_s_smem() {
  using P = PlaneTile;
  return sizeof(float) * 2 * (kSmAhead + 1) * P::NR * P::W;
}

// x <- [x] (+ cw P ec) + D^-1/2 (W * (D^-1/2 u)) with the 27-point kernel W,
// as k_sm_q<3>.  Each plane tile arrives by cp.async D planes ahead; the
// thread that copied a chunk scales it by isq (and zeroes the pinned cell)
// once its own copies have landed.  Every staged plane is read ONCE: its
// three rows around the thread's quad (x-neighbours by warp shuffle) give
// the partial sums of all three kernel planes, which roll in registers into
// the outputs of planes p + 1, p and p - 1; output plane p - 1 is complete
// after plane p and is written then, its own operands (x, the coarse
// correction, q) loaded one plane earlier.  (Reading nine staged rows per
// output plane instead made the pass shared-memory bound.)
template <int MODE, bool HOOK>
__global__ void __launch_bounds__(PlaneTile::T, 3)
    k_sm_s(LV L, LV C, Seg sg, Kern K, const float* __restrict__ src, const float* __restrict__ ec,
           float cw, float* __restrict__ x, int64_t skip, int64_t pin, const float* __restrict__ r,
           Hook hk) {
  pdl_enter();
  using P = PlaneTile;
  constexpr int TX = P::TX, TY = P::TY, R0 = P::R0, NR = P::NR, W = P::W;
  constexpr int D = kSmAhead, RS = D + 1;
  extern __shared__ __align__(16) float smem_f[];
  float(*u)[NR][W] = reinterpret_cast<float(*)[NR][W]>(smem_f);
  float(*is)[NR][W] = reinterpret_cast<float(*)[NR][W]>(smem_f + RS * NR * W);
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX, lane = threadIdx.x & 31;
  double acc_dot = 0.0;
  for_runs(sg, L.nz, [&](int tix, int tiy, int k0, int k1) {
    const int i0 = tix * P::PX + 4 * tx, j = tiy * TY + ty;
    const bool act = i0 < L.nx && j < L.ny;
    auto slot = [&](int kp) { return (kp + RS) % RS; };  // kp >= -1
    const TileChunks tc(L, C, tix, tiy);
    auto issue = [&](int kp) {
      const int s = slot(kp);
#pragma unroll
      for (int q = 0; q < P::NC; ++q) {
        if (q >= tc.n) break;
        int64_t c;
        const bool in = tc.at_plane(L, q, kp, c);
        cp16(&u[s][0][0] + tc.off[q], src + c, in);
        cp16(&is[s][0][0] + tc.off[q], L.isq + c, in);
      }
      cp_commit();
    };
    auto scale = [&](int kp) {
      const int s = slot(kp);
#pragma unroll
      for (int qq = 0; qq < P::NC; ++qq) {
        if (qq >= tc.n) break;
        int64_t c;
        const bool in = tc.at_plane(L, qq, kp, c);
        float* up = &u[s][0][0] + tc.off[qq];
        V4<float> a = ld4(up);
        const V4<float> b = ld4(&is[s][0][0] + tc.off[qq]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          a.v[q] *= b.v[q];
          if (MODE == SM_FIRST && in && c + q == skip) a.v[q] = 0.f;
        }
        st4(up, a);
      }
    };
    // operands of output plane k, loaded at plane k (written at plane k + 1)
    V4<float> o_n = zero4<float>();
    float e0_n = 0.f, e1_n = 0.f;
    V4<double> q_n = zero4<double>();
    auto operands = [&](int k) {
      o_n = zero4<float>();
      e0_n = e1_n = 0.f;
      q_n = zero4<double>();
      if (!act || k < k0 || k >= k1) return;
      const int64_t c = at(L, i0, j, k);
      if (MODE == SM_ADD) o_n = ld4(x + c);
      if (ec) {
        const int64_t pc = parent(C, i0, j, k);
        e0_n = cw * ec[pc];
        e1_n = cw * ec[pc + 1];
      }
      if (HOOK) q_n = ld4(hk.q + c);
    };
    float am[4] = {0.f, 0.f, 0.f, 0.f}, ac[4] = {0.f, 0.f, 0.f, 0.f}, an[4];
    V4<float> is_c = zero4<float>(), is_m;
    V4<float> o_m = zero4<float>();
    float e0_m = 0.f, e1_m = 0.f;
    V4<double> q_m = zero4<double>();
    for (int kp = k0 - 1; kp < k0 - 1 + D; ++kp) issue(kp);
    for (int p = k0 - 1; p <= k1; ++p) {
      issue(p + D);
      operands(p);
      cp_wait<D>();
      scale(p);
      __syncthreads();
      const int s = slot(p);
      // partial sums of plane p: pz[dk] belongs to output plane p + 1 - dk
      float pz[3][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj) {
        const float* row = u[s][ty + R0 + dj];
        const V4<float> m = ld4(row + 4 + 4 * tx);
        float wl = __shfl_up_sync(0xffffffffu, m.v[3], 1);
        float er = __shfl_down_sync(0xffffffffu, m.v[0], 1);
        if (lane == 0) wl = row[3 + 4 * tx];
        if (lane == 31) er = row[8 + 4 * tx];
        const float v[6] = {wl, m.v[0], m.v[1], m.v[2], m.v[3], er};
#pragma unroll
        for (int dk = 0; dk < 3; ++dk)
#pragma unroll
          for (int di = 0; di < 3; ++di) {
            const float wt = K.w[dk * 9 + (dj + 1) * 3 + di];
#pragma unroll
            for (int q = 0; q < 4; ++q) pz[dk][q] += wt * v[q + di];
          }
      }
      is_m = is_c;
      is_c = ld4(&is[s][ty + R0][4 + 4 * tx]);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        am[q] += pz[2][q];  // output plane p - 1 complete
        an[q] = pz[0][q];
      }
      if (p - 1 >= k0 && act) {
        const int64_t c = at(L, i0, j, p - 1);
        V4<float> out;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float vq = o_m.v[q] + is_m.v[q] * am[q];
          if (ec) vq += (q < 2 ? e0_m : e1_m);
          if (c + q == pin) vq = r[c + q];
          out.v[q] = vq;
        }
        st4(x + c, out);
        if (HOOK) {
#pragma unroll
          for (int q = 0; q < 4; ++q) acc_dot += (double)out.v[q] * q_m.v[q];
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        am[q] = ac[q] + pz[1][q];
        ac[q] = an[q];
      }
      o_m = o_n, e0_m = e0_n, e1_m = e1_n, q_m = q_n;
      __syncthreads();
    }
    cp_wait<0>();
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

// ------------------------------------------------------------ FCG direction

// Planes the direction pass keeps in flight ahead of the one it evaluates.
constexpr int kDirAhead = 1;

// Dynamic shared memory of k_dir_s: D + 3 plane slots of the staged z
// (float) and of p_old, overwritten on landing by the new direction (double).
constexpr size_t dir_s_smem() {
  using P = PlaneTile;
  return (size_t)(kDirAhead + 3) * P::NR * P::W * (sizeof(float) + sizeof(double));
}

// p = z - beta p_old (p = z on the first iteration), q = A p, and the dot
// products p.q and p.r that give alpha: the 3D counterpart of k_fcg_dir_q
// with the same arithmetic and coefficient order.  The z and p_old tiles
// arrive by cp.async; the copying thread forms p in place once its copies
// have landed; the couplings and r of the current plane are loaded before
// the block waits for the plane.  FACES: per-face coupling arrays on all
// axes (a p' system from a SIMPLE run); otherwise the per-axis tables of a
// uniform operator, whose smaller register footprint lets three blocks
// share an SM.
template <bool FACES>
__global__ void __launch_bounds__(PlaneTile::T, FACES ? 2 : 3)
    k_dir_s(OpView<double> A, Seg sg, FcgState* S, const float* __restrict__ z, double* P0,
            double* P1, double* __restrict__ q, const double* __restrict__ r, double* partials,
            Loop h) {
  pdl_enter();
  using P = PlaneTile;
  constexpr int TX = P::TX, TY = P::TY, R0 = P::R0, NR = P::NR, W = P::W;
  constexpr int D = kDirAhead, RS = D + 3;
  extern __shared__ __align__(16) unsigned char smem_b[];
  double(*vs)[NR][W] = reinterpret_cast<double(*)[NR][W]>(smem_b);
  float(*zs)[NR][W] = reinterpret_cast<float(*)[NR][W]>(smem_b + sizeof(double) * RS * NR * W);
  if (S->done) return;
  const long long it = S->it;
  const bool first = (it == 0);
  const double beta = first ? 0.0 : S->beta;
  double* __restrict__ pn = (it & 1) ? P1 : P0;
  const double* __restrict__ po = (it & 1) ? P0 : P1;
  const LV L{A.nx, A.ny, A.nz, nullptr, nullptr, nullptr, nullptr};
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX, lane = threadIdx.x & 31;
  double acc[2] = {0.0, 0.0};
  for_runs(sg, A.nz, [&](int tix, int tiy, int k0, int k1) {
    const int i0 = tix * P::PX + 4 * tx, j = tiy * TY + ty;
    const bool act = i0 < A.nx && j < A.ny;
    auto slot = [&](int kp) { return (kp + RS) % RS; };  // kp >= -1
    const TileChunks tc(L, L, tix, tiy);
    auto issue = [&](int kp) {
      const int s = slot(kp);
#pragma unroll
      for (int q = 0; q < P::NC; ++q) {
        if (q >= tc.n) break;
        int64_t c;
        const bool in = tc.at_plane(L, q, kp, c);
        double* vp = &vs[s][0][0] + tc.off[q];
        cp16(&zs[s][0][0] + tc.off[q], z + c, in);
        if (!first) {
          cp16(vp, po + c, in);
          cp16(vp + 2, po + c + 2, in);
        }
      }
      cp_commit();
    };
    auto land = [&](int kp) {
      const int s = slot(kp);
#pragma unroll
      for (int q = 0; q < P::NC; ++q) {
        if (q >= tc.n) break;
        double* vp = &vs[s][0][0] + tc.off[q];
        const V4<float> zz = ld4(&zs[s][0][0] + tc.off[q]);
        V4<double> v;
        if (first) {
#pragma unroll
          for (int t = 0; t < 4; ++t) v.v[t] = (double)zz.v[t];
        } else {
          const V4<double> pp = ld4(vp);
#pragma unroll
          for (int t = 0; t < 4; ++t) v.v[t] = fma(-beta, pp.v[t], (double)zz.v[t]);
        }
        st4(vp, v);
      }
    };
    for (int kp = k0 - 1; kp <= k0 + D; ++kp) issue(kp);
    cp_wait<D>();
    land(k0 - 1);
    land(k0);
    for (int k = k0; k < k1; ++k) {
      issue(k + 1 + D);
      // the plane's couplings and r, in flight while the block waits
      const int64_t c = act ? i0 + (int64_t)A.nx * (j + (int64_t)A.ny * k) : 0;
      double fx[5];
      V4<double> yl, yh, zl, zh, rr = zero4<double>();
      if (act) {
        if (FACES) {
          const int64_t bx = i0 + (int64_t)(A.nx + 1) * (j + (int64_t)A.ny * k);
#pragma unroll
          for (int u = 0; u < 5; ++u) fx[u] = A.fx[bx + u];
          const int64_t by = i0 + (int64_t)A.nx * (j + (int64_t)(A.ny + 1) * k);
          yl = ld4(A.fy + by);
          yh = ld4(A.fy + by + A.nx);
          zl = ld4(A.fz + c);
          zh = ld4(A.fz + c + (int64_t)A.nx * A.ny);
        } else {
#pragma unroll
          for (int u = 0; u < 5; ++u) fx[u] = A.tx[i0 + u];
          const double ya = A.ty[j], yb = A.ty[j + 1], za = A.tz[k], zb = A.tz[k + 1];
          yl = V4<double>{{ya, ya, ya, ya}};
          yh = V4<double>{{yb, yb, yb, yb}};
          zl = V4<double>{{za, za, za, za}};
          zh = V4<double>{{zb, zb, zb, zb}};
        }
        rr = ld4(r + c);
      }
      cp_wait<D>();
      land(k + 1);
      __syncthreads();
      const double* mid = vs[slot(k)][ty + R0];
      const V4<double> v = ld4(mid + 4 + 4 * tx);
      double wl = __shfl_up_sync(0xffffffffu, v.v[3], 1);
      double er = __shfl_down_sync(0xffffffffu, v.v[0], 1);
      if (lane == 0) wl = mid[3 + 4 * tx];
      if (lane == 31) er = mid[8 + 4 * tx];
      if (act) {
        const V4<double> sv = ld4(vs[slot(k)][ty + R0 - 1] + 4 + 4 * tx);
        const V4<double> nv = ld4(vs[slot(k)][ty + R0 + 1] + 4 + 4 * tx);
        const V4<double> bv = ld4(vs[slot(k - 1)][ty + R0] + 4 + 4 * tx);
        const V4<double> tv = ld4(vs[slot(k + 1)][ty + R0] + 4 + 4 * tx);
        V4<double> aq;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double w = u == 0 ? wl : v.v[u - 1];
          const double e = u == 3 ? er : v.v[u + 1];
          // diagonal summed in the reference's face order (as load_coef)
          const double d = ((((fx[u] + fx[u + 1]) + yl.v[u]) + yh.v[u]) + zl.v[u]) + zh.v[u];
          double off = fx[u] * w;
          off = fma(fx[u + 1], e, off);
          off = fma(yl.v[u], sv.v[u], off);
          off = fma(yh.v[u], nv.v[u], off);
          off = fma(zl.v[u], bv.v[u], off);
          off = fma(zh.v[u], tv.v[u], off);
          aq.v[u] = (A.pinned && c + u == A.ref) ? v.v[u] : fma(d, v.v[u], -off);
        }
        st4(pn + c, v);
        st4(q + c, aq);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          acc[0] += v.v[u] * aq.v[u];
          acc[1] += v.v[u] * rr.v[u];
        }
      }
      __syncthreads();
    }
    cp_wait<0>();
  });
  reduce_last<2>(acc, partials, &S->ticket, [&](const double* tot) {
    const double pq = tot[0], pr = tot[1];
    const double alpha = pr / pq;
    // a non-positive p.Ap means rounding has taken over (scale-free test)
    if (!isfinite(pq) || !(pq > 0.0) || !isfinite(alpha)) {
      stop_loop(S, h, kLearnedStagnated);
      return;
    }
    S->pq = pq;
    S->pr = pr;
    S->alpha = alpha;
  });
}
