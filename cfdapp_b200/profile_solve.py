"""One p' solve of the isolated system, for profilers.

    CFDB_LEARNED_LAUNCH=stream ncu ... python -m cfdapp_b200.profile_solve --dim 2 --n 2048

Runs a single solve (default: the learned-FCG solve to rel-res 1e-8 from
x0 = 0 with the seeded synthetic RHS) and prints its outcome.  With
CFDB_LEARNED_LAUNCH=stream the learned solve launches its kernels one by one
instead of as one CUDA graph with a conditional WHILE node, whose kernel
nodes profilers cannot see individually; the kernels and their order are the
same.
"""
from __future__ import annotations

import argparse

from . import cfdb


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dim", type=int, default=2)
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--preconditioner", default="learned_mg", choices=["learned_mg", "jacobi"])
    ap.add_argument("--max-iterations", type=int, default=100000)
    a = ap.parse_args()
    ctx = cfdb.Context(0)
    b = cfdb.synth_rhs(a.dim, a.n)
    op = cfdb.POperator(ctx, a.dim, [a.n] * a.dim)
    bd = ctx.to_device(b)
    xd = ctx.alloc(b.nbytes)
    ctx.memset(xd, 0, b.nbytes)
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                  max_iterations=a.max_iterations, preconditioner=a.preconditioner)
    r = op.solve_device(bd, xd, s)
    print(f"{a.dim}D {a.n}: {r.status} in {r.iterations} iterations, {r.device_ms:.3f} ms, "
          f"true rel-res {r.true_residual / r.initial_residual:.3e}")
    ctx.free(bd)
    ctx.free(xd)
    op.close()
    ctx.close()


if __name__ == "__main__":
    main()
