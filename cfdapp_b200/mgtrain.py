"""Train the learned V-cycle preconditioner on the GPU.

    python -m cfdapp_b200.mgtrain [--dims 2 3] [--steps 400] [--out DIR]

The loss and its gradient come from the library (cfdb_mg_loss_grad: the
network's own forward kernels and hand-written adjoint kernels); this script
only draws the training problems, runs Adam on the few dozen weights, and
keeps the weight set that needs the fewest flexible-CG iterations on the
validation systems.  Training problems are p' operators of the kind the
SIMPLE loop produces: the isolated (unit-response) operator, operators whose
face coefficients follow smooth random log-normal response fields (the
momentum response d = V / a_P varies smoothly across a flow), and p' systems
harvested from the library's own GPU SIMPLE runs of lid-driven cavities at
Re 100, 400 and 1000 (cfdb_simple_pprime_faces), on grids small enough that
one step takes milliseconds.  Error samples are
multi-scale random fields (white noise at every level of the hierarchy,
prolongated by injection), so smooth and rough error components are both
represented; optionally some samples are replaced by the error fields the
current network reduces slowest (a few power iterations of I - M A), which
sharpens the 3D network but destabilises the 2D one (its validation solves
stop converging), hence the per-dimension default.

Writes DIR/mg_trained.inc (compiled into the library as the shipped
weights) and DIR/mg_weights.json (the weights and the training record).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import time

import numpy as np

from . import cfdb

MG_TAPS = 27
TRAIN_LEVELS = 4


def free_taps(dim):
    if dim == 2:
        return [t for t in range(9, 18) if t <= 26 - t]
    return [t for t in range(MG_TAPS) if t <= 26 - t]


def kernel_shape(dim, n):
    return (n[1], 1, n[0]) if dim == 2 else (n[2], n[1], n[0])


def smooth_field(shape, rng, modes=6, amp=0.6):
    """A smooth random log-normal field on a grid of `shape` (z, y, x)."""
    grids = np.meshgrid(*[np.linspace(0, 1, s) for s in shape], indexing="ij")
    f = np.zeros(shape)
    for _ in range(modes):
        k = rng.integers(1, 5, size=len(shape))
        ph = rng.uniform(0, 2 * np.pi, size=len(shape))
        term = np.ones(shape)
        for g, kk, p in zip(grids, k, ph):
            term = term * np.cos(np.pi * kk * g + p)
        f += term
    return np.exp(amp * f / np.sqrt(modes))


def uniform_faces(dim, n):
    """Unit interior face coefficients, all-Neumann (the isolated p' system up
    to a scale the network is invariant to)."""
    if dim == 2:
        nx, ny = n
        fx = np.ones((ny, nx + 1))
        fy = np.ones((ny + 1, nx))
        fx[:, 0] = fx[:, -1] = 0.0
        fy[0, :] = fy[-1, :] = 0.0
        return np.concatenate([fx.ravel(), fy.ravel()])
    nx, ny, nz = n
    fx = np.ones((nz, ny, nx + 1))
    fy = np.ones((nz, ny + 1, nx))
    fz = np.ones((nz + 1, ny, nx))
    fx[:, :, 0] = fx[:, :, -1] = 0.0
    fy[:, 0, :] = fy[:, -1, :] = 0.0
    fz[0] = fz[-1] = 0.0
    return np.concatenate([fx.ravel(), fy.ravel(), fz.ravel()])


def apply_faces(dim, n, fc, e):
    """A e for global-order face coefficients fc (interior faces couple,
    boundary faces add to the diagonal); e in cell order."""
    if dim == 2:
        nx, ny = n
        fx = fc[: (nx + 1) * ny].reshape(ny, nx + 1)
        fy = fc[(nx + 1) * ny:].reshape(ny + 1, nx)
        x = e.reshape(ny, nx)
        y = (fx[:, :-1] + fx[:, 1:] + fy[:-1, :] + fy[1:, :]) * x
        y[:, 1:] -= fx[:, 1:-1] * x[:, :-1]
        y[:, :-1] -= fx[:, 1:-1] * x[:, 1:]
        y[1:, :] -= fy[1:-1, :] * x[:-1, :]
        y[:-1, :] -= fy[1:-1, :] * x[1:, :]
        return y.ravel()
    nx, ny, nz = n
    a, b = (nx + 1) * ny * nz, nx * (ny + 1) * nz
    fx = fc[:a].reshape(nz, ny, nx + 1)
    fy = fc[a:a + b].reshape(nz, ny + 1, nx)
    fz = fc[a + b:].reshape(nz + 1, ny, nx)
    x = e.reshape(nz, ny, nx)
    y = (fx[:, :, :-1] + fx[:, :, 1:] + fy[:, :-1] + fy[:, 1:] + fz[:-1] + fz[1:]) * x
    y[:, :, 1:] -= fx[:, :, 1:-1] * x[:, :, :-1]
    y[:, :, :-1] -= fx[:, :, 1:-1] * x[:, :, 1:]
    y[:, 1:] -= fy[:, 1:-1] * x[:, :-1]
    y[:, :-1] -= fy[:, 1:-1] * x[:, 1:]
    y[1:] -= fz[1:-1] * x[:-1]
    y[:-1] -= fz[1:-1] * x[1:]
    return y.ravel()


def hard_errors(op, dim, n, fc, e0, sweeps=4):
    """Error fields the current network reduces slowest: a few power
    iterations of I - M A (the network applied on the GPU) from e0."""
    out = []
    for e in e0.astype(np.float64):
        for _ in range(sweeps):
            e[0] = 0.0
            r = apply_faces(dim, n, fc, e)
            r[0] = 0.0
            e = e - op.mg_apply(r).astype(np.float64)
            e /= np.sqrt(np.mean(e * e)) + 1e-300
        e[0] = 0.0
        out.append(e)
    return np.array(out, dtype=np.float32)


def harvest_cavity(ctx, dim, n, reynolds, snapshots, chunk=10):
    """p' systems of the solver's own GPU SIMPLE runs: a lid-driven cavity at
    each Reynolds number, the p' face coefficients taken every `chunk` outer
    iterations until `snapshots` are collected.  Returns [(faces, pinned,
    reference cell)]."""
    out = []
    for re in reynolds:
        case = cfdb.SimpleCase.cavity(dim, n, lid=1.0, mu=1.0 / re)
        ps = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                       max_iterations=20000, type="cg",
                                       preconditioner="learned_mg")
        ms = cfdb.LinearSolverSettings(absolute_tolerance=1e-12, relative_tolerance=1e-8,
                                       max_iterations=2000, type="bicgstab", preconditioner="none")
        st = cfdb.SIMPLESettings(max_iterations=chunk * snapshots, momentum_solver=ms,
                                 pressure_solver=ps)
        sim = cfdb.Simple(ctx, case, st)
        sim.set_state(None, None, None, None)
        for _ in range(snapshots):
            sim.iterate(chunk)
            out.append(sim.pprime_faces())
        sim.close()
    return out


def random_operator_faces(dim, n, rng):
    """Face coefficients (global real order) of a SIMPLE-like p' operator:
    D_f = interpolated smooth response d across each interior face, all-Neumann."""
    if dim == 2:
        nx, ny = n
        d = smooth_field((ny, nx), rng)
        fx = np.zeros((ny, nx + 1))
        fy = np.zeros((ny + 1, nx))
        fx[:, 1:-1] = 0.5 * (d[:, 1:] + d[:, :-1]) * (nx / ny)
        fy[1:-1, :] = 0.5 * (d[1:, :] + d[:-1, :]) * (ny / nx)
        return np.concatenate([fx.ravel(), fy.ravel()])
    nx, ny, nz = n
    d = smooth_field((nz, ny, nx), rng)
    fx = np.zeros((nz, ny, nx + 1))
    fy = np.zeros((nz, ny + 1, nx))
    fz = np.zeros((nz + 1, ny, nx))
    fx[:, :, 1:-1] = 0.5 * (d[:, :, 1:] + d[:, :, :-1])
    fy[:, 1:-1, :] = 0.5 * (d[:, 1:, :] + d[:, :-1, :])
    fz[1:-1] = 0.5 * (d[1:] + d[:-1])
    return np.concatenate([fx.ravel(), fy.ravel(), fz.ravel()])


def multiscale_errors(dim, n, count, rng):
    """Unit-RMS error fields: white noise at every hierarchy scale, prolongated
    by injection, the coarser scales weighted up (x1.5 per level)."""
    shape = kernel_shape(dim, n)
    active = [ax for ax in range(3) if shape[ax] > 1]
    out = np.zeros((count,) + shape)
    for q in range(count):
        e = np.zeros(shape)
        level = 0
        while True:
            f = 2 ** level
            cs = tuple((s + f - 1) // f if s > 1 else 1 for s in shape)
            if min(cs[ax] for ax in active) < 2:
                break
            up = rng.normal(size=cs)
            for ax in active:
                up = np.repeat(up, f, axis=ax)
            e += up[: shape[0], : shape[1], : shape[2]] * (1.5 ** level)
            level += 1
        out[q] = e / np.sqrt(np.mean(e * e))
    return out.reshape(count, -1).astype(np.float32)


class Params:
    """Free weights (tied taps) <-> the library's weight arrays."""

    def __init__(self, dim, kernels, coarse):
        self.dim = dim
        self.idx = free_taps(dim)
        self.k = np.array(kernels, dtype=np.float64)[:TRAIN_LEVELS]
        self.c = np.array(coarse, dtype=np.float64)[:TRAIN_LEVELS]

    def vector(self):
        return np.concatenate([self.k[:, self.idx].ravel(), self.c])

    def set_vector(self, v):
        m = len(self.idx)
        for l in range(TRAIN_LEVELS):
            for q, t in enumerate(self.idx):
                self.k[l, t] = self.k[l, 26 - t] = v[l * m + q]
        self.c = v[TRAIN_LEVELS * m:].copy()

    def grad_vector(self, gk, gc):
        return np.concatenate([gk[:TRAIN_LEVELS][:, self.idx].ravel(), gc[:TRAIN_LEVELS]])

    def push(self, ctx, nu, sweeps):
        ctx.mg_set_weights(self.dim, self.k.astype(np.float32), self.c.astype(np.float32), nu=nu,
                           coarse_sweeps=sweeps)


def fcg_iterations(ctx, ops, b_list):
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                  max_iterations=20000, preconditioner="learned_mg")
    its = []
    for op, b in zip(ops, b_list):
        r = op.solve(b, s, history_cap=0)
        its.append(r.iterations if r.converged() and r.fallback_iterations == 0 else 10 ** 6)
    return its


def train_dim(ctx, dim, steps, seed, log, hard, nu=2, sweeps=50, grids=None, re_samples=0,
              val_n=None):
    """grids=None: the compact recipe (one 128^2 / 32^3 grid, cavities at Re
    100, 400, 1000).  grids=[n, ...]: p' systems harvested from cavity runs on
    every grid n^dim at `re_samples` Reynolds numbers drawn uniformly from
    [100, 1000] each (one snapshot after 20-100 outer iterations), plus the
    isolated and two smooth-response operators on the first grid."""
    rng = np.random.default_rng(seed)
    n_train = (128, 128) if dim == 2 else (32, 32, 32)
    n_val = (384, 384) if dim == 2 else (64, 64, 64)
    if val_n:
        n_val = (val_n,) * dim
    # training operators: isolated, smooth random response, and p' systems
    # harvested from the solver's own SIMPLE runs of cavities at Re 100..1000
    if grids:
        n_train = (grids[0],) * dim
    train_set = [(n_train, uniform_faces(dim, n_train))] + \
        [(n_train, random_operator_faces(dim, n_train, rng)) for _ in range(2)]
    if grids:
        harvested = []
        for g in grids:
            for re in rng.uniform(100.0, 1000.0, size=re_samples):
                h = harvest_cavity(ctx, dim, g, [float(re)], 1, chunk=int(rng.integers(20, 101)))
                harvested += [((g,) * dim, f) for f, _, _ in h]
                log(f"dim {dim}: harvested {g}^{dim} at Re {re:.0f}")
    else:
        harvested = [(n_train, f) for f, _, _ in
                     harvest_cavity(ctx, dim, n_train[0], [100.0, 400.0, 1000.0], 2)]
    train_set += harvested
    train_fc = [fc for _, fc in train_set]
    train_sz = [sz for sz, _ in train_set]
    train_ops = [cfdb.POperator(ctx, dim, sz, face_coeff=fc) for sz, fc in train_set]
    log(f"dim {dim}: {len(train_ops)} training operators ({len(harvested)} harvested)")
    # validation: the isolated system, a smooth-response system and a
    # harvested cavity system (Re 700), synthetic RHS
    hv = harvest_cavity(ctx, dim, n_val[0], [700.0], 1, chunk=20)[0][0]
    val_ops = [cfdb.POperator(ctx, dim, n_val),
               cfdb.POperator(ctx, dim, n_val,
                              face_coeff=random_operator_faces(dim, n_val, np.random.default_rng(seed + 99))),
               cfdb.POperator(ctx, dim, n_val, face_coeff=hv)]
    b_val = [cfdb.synth_rhs(dim, n_val[0])] * 3
    ctx.mg_reset_weights(dim, trained=False)
    base = ctx.mg_get_weights(dim)
    k0 = np.repeat(base["kernels"][:1], TRAIN_LEVELS, axis=0)
    c0 = np.repeat(base["coarse_weights"][:1], TRAIN_LEVELS)
    P = Params(dim, k0, c0)
    P.push(ctx, nu, sweeps)
    untrained = fcg_iterations(ctx, val_ops, b_val)
    log(f"dim {dim}: untrained validation iterations {untrained}")
    theta = P.vector()
    m = np.zeros_like(theta)
    v = np.zeros_like(theta)
    lr0, b1, b2, eps = 3e-3, 0.9, 0.999, 1e-8
    best = (sum(untrained), theta.copy(), untrained)
    history = []
    for step in range(1, steps + 1):
        q = step % len(train_ops)
        op = train_ops[q]
        e = multiscale_errors(dim, train_sz[q], 4, rng)
        if hard:
            e[4 - hard:] = hard_errors(op, dim, train_sz[q], train_fc[q], e[4 - hard:])
        loss, gk, gc = op.mg_loss_grad(e)
        lr = lr0 * 0.5 * (1.0 + np.cos(np.pi * step / steps))
        g = P.grad_vector(gk, gc)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        theta = theta - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
        P.set_vector(theta)
        P.push(ctx, nu, sweeps)
        history.append(float(loss))
        if step % 100 == 0 or step == steps:
            its = fcg_iterations(ctx, val_ops, b_val)
            log(f"dim {dim} step {step}: loss {np.mean(history[-100:]):.4f} validation iterations {its}")
            if sum(its) < best[0]:
                best = (sum(its), theta.copy(), its)
    P.set_vector(best[1])
    for op in train_ops + val_ops:
        op.close()
    return P, {"untrained_validation_iterations": untrained,
               "trained_validation_iterations": best[2],
               "validation_grids": list(n_val), "training_grid": list(n_train),
               "training_grids": sorted({int(sz[0]) for sz in train_sz}),
               "harvested_systems": len(harvested),
               "loss_first50": float(np.mean(history[:50])),
               "loss_last50": float(np.mean(history[-50:])), "steps": steps,
               "nu": nu, "coarse_sweeps": sweeps, "hard_samples_of_4": hard}


def cfloat(x):
    """A C float literal that reads back to the same FP32 value."""
    t = f"{float(x):.9g}"
    if "." not in t and "e" not in t and "n" not in t:
        t += ".0"
    return t + "f"


def write_outputs(out_dir, sets):
    os.makedirs(out_dir, exist_ok=True)
    payload = {str(dim): {"levels": TRAIN_LEVELS, "nu": rec["nu"],
                          "coarse_sweeps": rec["coarse_sweeps"],
                          "kernels": P.k.astype(np.float32).tolist(),
                          "coarse_weights": P.c.astype(np.float32).tolist(), "record": rec}
               for dim, (P, rec) in sets.items()}
    blob = json.dumps({d: {k: v for k, v in p.items() if k != "record"} for d, p in payload.items()},
                      sort_keys=True).encode()
    digest = hashlib.sha256(blob).hexdigest()
    with open(os.path.join(out_dir, "mg_weights.json"), "w") as f:
        json.dump({"format": 1, "sha256": digest, "sets": payload}, f, indent=1)
    lines = ["// Trained weights of the learned preconditioner, generated by",
             "// cfdapp_b200/mgtrain.py (do not edit; mg_weights.json holds the training",
             f"// record).  sha256 of the weights: {digest}",
             "MgWeights mg_builtin_weights(int dim) {",
             "  MgWeights W = mg_default_weights(dim);"]
    for dim, (P, rec) in sorted(sets.items()):
        lines.append(f"  if (dim == {dim}) {{")
        lines.append(f"    static const float k[{TRAIN_LEVELS}][{MG_TAPS}] = {{")
        for row in P.k.astype(np.float32):
            lines.append("        {" + ", ".join(cfloat(x) for x in row) + "},")
        lines.append("    };")
        lines.append(f"    static const float c[{TRAIN_LEVELS}] = {{" +
                     ", ".join(cfloat(x) for x in P.c.astype(np.float32)) + "};")
        lines.append(f"    W.levels = {TRAIN_LEVELS};")
        lines.append(f"    W.nu = {rec['nu']};")
        lines.append(f"    W.coarse_sweeps = {rec['coarse_sweeps']};")
        lines.append("    for (int l = 0; l < kMgMaxLevels; ++l) {")
        lines.append(f"      const int s = l < {TRAIN_LEVELS} ? l : {TRAIN_LEVELS - 1};")
        lines.append("      for (int t = 0; t < kMgTaps; ++t) W.w[l][t] = k[s][t];")
        lines.append("      W.c[l] = c[s];")
        lines.append("    }")
        lines.append("  }")
    lines.append("  return W;")
    lines.append("}")
    with open(os.path.join(out_dir, "mg_trained.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")
    return digest


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs="+", default=[2, 3])
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--nu", type=int, nargs="+", default=[1, 1],
                    help="smoothing layers per side, per dim (2D, 3D)")
    ap.add_argument("--coarse-sweeps", type=int, nargs="+", default=[5, 20],
                    help="damped-Jacobi sweeps on the coarsest level, per dim (2D, 3D)")
    ap.add_argument("--hard", type=int, nargs="+", default=[0, 2],
                    help="per dim (2D, 3D): samples of 4 drawn by power iteration of I - M A")
    ap.add_argument("--grids2d", type=int, nargs="*", default=None,
                    help="2D: harvest p' systems on these grids (e.g. 256 512 1024) at "
                         "--re-samples Reynolds numbers uniform in [100, 1000] each")
    ap.add_argument("--re-samples", type=int, default=2)
    ap.add_argument("--val2d", type=int, default=None, help="2D validation grid (default 384)")
    ap.add_argument("--keep", default=None,
                    help="mg_weights.json whose sets for the dimensions not trained are kept")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "csrc"))
    a = ap.parse_args()
    ctx = cfdb.Context(0)
    t0 = time.time()
    log = lambda s: print(f"[{time.time() - t0:7.1f}s] {s}", flush=True)
    sets = {}
    for dim in a.dims:
        q = 0 if dim == 2 else 1
        pick = lambda v: v[q] if len(v) > q else v[-1]
        sets[dim] = train_dim(ctx, dim, a.steps, a.seed + dim, log, pick(a.hard), pick(a.nu),
                              pick(a.coarse_sweeps), grids=a.grids2d if dim == 2 else None,
                              re_samples=a.re_samples, val_n=a.val2d if dim == 2 else None)
    if a.keep:
        with open(a.keep) as f:
            old_sets = json.load(f)["sets"]
        for d, rec in old_sets.items():
            if int(d) not in sets:
                P = Params(int(d), rec["kernels"], rec["coarse_weights"])
                sets[int(d)] = (P, dict(rec["record"], nu=rec["nu"],
                                        coarse_sweeps=rec["coarse_sweeps"]))
    digest = write_outputs(a.out, sets)
    log(f"wrote {a.out}/mg_trained.inc and mg_weights.json (sha256 {digest[:16]})")
    ctx.close()


if __name__ == "__main__":
    main()
