"""The benchmark's own systems at their own sizes (5-point 2048^2, 7-point
256^3, seeded synthetic RHS, cell 0 pinned) against the reference's full CG
+ Jacobi solves of them (tests/golden/fullsize_*.npz, made by
tests/golden/make_fullsize_golden.py: the reference's status, iteration
count, residual history and x at 16 384 seeded cells).

Bars: the FP64 Jacobi-PCG follows the reference's iterates (the same
algorithm, reductions in another order): same status, iterations within
2 %, the first 200 history entries within 1e-6 relative, x within 1e-9 on
the sampled cells.  The learned FCG solve to rel-res 1e-10 lands on the
reference's solution within 1e-6 on the sampled cells (the reference's own
x carries its 1e-8 stopping error)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = [f for f in ("fullsize_2d2048", "fullsize_3d256")
            if os.path.exists(os.path.join(GOLDEN, f + ".npz"))]


def _load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z, json.loads(str(z["meta"]))


def _sampled_rel(x, z):
    idx = z["idx"]
    return float(np.linalg.norm(x[idx] - z["x_at"]) / np.linalg.norm(z["x_at"]))


@pytest.mark.parametrize("name", FIXTURES)
def test_fp64_pcg_follows_the_reference_full_solve(ctx, name):
    from cfdapp_b200 import cfdb
    z, meta = _load(name)
    dim, n = meta["dim"], meta["n"]
    b = cfdb.synth_rhs(dim, n)
    op = cfdb.POperator(ctx, dim, [n] * dim)
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                  max_iterations=200000)
    r = op.solve(b, s, history_cap=201)
    assert r.status == meta["status"] == "Converged"
    assert abs(r.iterations - meta["iterations"]) <= max(2, 0.02 * meta["iterations"])
    np.testing.assert_allclose(r.residual_history[:200], z["hist"][:200], rtol=1e-6)
    assert _sampled_rel(r.solution, z) <= 1e-9
    assert abs(np.linalg.norm(r.solution) - float(z["x_norm"])) <= 1e-9 * float(z["x_norm"])
    op.close()


@pytest.mark.parametrize("name", FIXTURES)
def test_learned_solve_lands_on_the_reference_full_solve(ctx, name):
    from cfdapp_b200 import cfdb
    z, meta = _load(name)
    dim, n = meta["dim"], meta["n"]
    b = cfdb.synth_rhs(dim, n)
    op = cfdb.POperator(ctx, dim, [n] * dim)
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-10,
                                  max_iterations=5000, preconditioner="learned_mg")
    r = op.solve(b, s, history_cap=0)
    assert r.status == "Converged" and r.fallback_iterations == 0
    assert r.true_residual / r.initial_residual <= 1e-10 * 1.01
    assert _sampled_rel(r.solution, z) <= 1e-6
    op.close()
