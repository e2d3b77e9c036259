"""Device solves of the reference's CSR LinearSystem (cfdb_csr_solve_host)
against the reference's own outcomes and the oracle.

The reference's known answers for its stored BiCGSTAB regression systems
(tests/unit/algebra/test_bicgstab_breakdown.cpp:137-153): default settings
(abs 1e-12, rel 1e-10) converge with no restart and final and true residual
<= 1e-12; its scale-invariance property (:156-178): scaling a system by a
power of two scales the residual history by exactly that factor and leaves
the iterations and the solution bit-identical.  p' systems of the reference's
own assembly take the face-operator path and must meet the p' bars: same
status, iterations within 2 %, solution within 1e-9 relative L2.
"""
import numpy as np
import pytest

from oracle import oracle as O

from test_csr import csr_from_bands, csr_to_bands, load_system

pytestmark = pytest.mark.gpu


def _settings(**kw):
    from cfdapp_b200.cfdb import LinearSolverSettings
    return LinearSolverSettings(**kw)


def _csr_multiply(ro, ci, va, x):
    y = np.zeros(len(ro) - 1)
    for r in range(len(ro) - 1):
        lo, hi = int(ro[r]), int(ro[r + 1])
        y[r] = np.dot(va[lo:hi], x[ci[lo:hi].astype(np.int64)])
    return y


@pytest.mark.parametrize("name", ["csr_mesh004_smooth", "csr_mesh004_rough"])
def test_bicgstab_on_the_stored_breakdown_systems(ctx, name):
    from cfdapp_b200 import cfdb
    s, meta = load_system(name)
    st = meta["settings"]
    solver = cfdb.CsrSolver(ctx)
    r = solver.solve(s["offsets"], s["columns"], s["values"], s["rhs"],
                     _settings(type="bicgstab", preconditioner="none", absolute_tolerance=st["atol"],
                               relative_tolerance=st["rtol"], max_iterations=st["maxit"]),
                     x0=s["x0"])
    assert solver.info["path"] == "stencil" and solver.info["n"] == (32, 32)
    assert r.status == "Converged" and r.restarts == 0
    assert r.final_residual <= st["atol"]
    true_res = np.linalg.norm(s["rhs"] - _csr_multiply(s["offsets"], s["columns"], s["values"],
                                                       r.solution))
    assert true_res <= st["atol"]
    # these systems sit near a BiCGSTAB breakdown, so the iteration count
    # follows the reduction order (the oracle, in the reference's order,
    # repeats the reference's count exactly: tests/test_csr.py)
    assert abs(r.iterations - meta["iterations"]) <= 0.15 * meta["iterations"]
    assert np.linalg.norm(r.solution - s["x"]) <= 1e-6 * np.linalg.norm(s["x"])
    solver.close()


def _convection_diffusion_1d(n, scale):
    """A non-symmetric 3-point band (upwinded convection plus diffusion),
    scaled by `scale` (a power of two)."""
    diag = np.full(n, 3.0) * scale
    lo = np.full(n, -2.0) * scale
    hi = np.full(n, -0.75) * scale
    lo[0] = 0.0
    hi[-1] = 0.0
    off = [lo, hi] + [np.zeros(n) for _ in range(4)]
    b = np.sin(np.arange(n) * 0.37) * scale
    return csr_from_bands(diag, off, (n,)), b


def test_bicgstab_is_invariant_under_power_of_two_scaling(ctx):
    from cfdapp_b200 import cfdb
    s = _settings(type="bicgstab", preconditioner="none", absolute_tolerance=0.0,
                  relative_tolerance=1e-10, max_iterations=500)
    (ro, ci, va), b = _convection_diffusion_1d(60, 1.0)
    solver = cfdb.CsrSolver(ctx)
    ref = solver.solve(ro, ci, va, b, s)
    assert ref.status == "Converged"
    for e in (-100, 100):
        scale = float(np.ldexp(1.0, e))
        (ro, ci, va), b = _convection_diffusion_1d(60, scale)
        r = solver.solve(ro, ci, va, b, s)
        assert r.status == "Converged" and r.iterations == ref.iterations
        np.testing.assert_array_equal(r.residual_history, ref.residual_history * scale)
        np.testing.assert_array_equal(r.solution, ref.solution)
    solver.close()


@pytest.mark.parametrize("name", ["csr_pprime2d_24", "csr_pprime3d_8"])
def test_reference_pprime_csr_takes_the_face_path_and_matches(ctx, name):
    from cfdapp_b200 import cfdb
    s, meta = load_system(name)
    st = meta["settings"]
    solver = cfdb.CsrSolver(ctx)
    r = solver.solve(s["offsets"], s["columns"], s["values"], s["rhs"],
                     _settings(type="cg", preconditioner="jacobi", absolute_tolerance=st["atol"],
                               relative_tolerance=st["rtol"], max_iterations=st["maxit"]))
    assert solver.info["path"] == "faces" and solver.info["pinned"]
    assert r.status == meta["status"] == "Converged"
    assert abs(r.iterations - meta["iterations"]) <= max(2, 0.02 * meta["iterations"])
    m = min(len(r.residual_history), len(s["hist"]))
    np.testing.assert_allclose(r.residual_history[:m], s["hist"][:m], rtol=1e-6)
    assert np.linalg.norm(r.solution - s["x"]) <= 1e-9 * np.linalg.norm(s["x"])
    solver.close()


def test_unpreconditioned_cg_takes_the_stencil_path(ctx):
    from cfdapp_b200 import cfdb
    s, _ = load_system("csr_pprime2d_24")
    case = O.Case(2, (24, 24))
    diag, off = csr_to_bands(s["offsets"], s["columns"], s["values"], (24, 24))
    want = O.stencil_solve(case, diag, off, s["rhs"], jacobi=False, rel_tol=1e-10)
    solver = cfdb.CsrSolver(ctx)
    r = solver.solve(s["offsets"], s["columns"], s["values"], s["rhs"],
                     _settings(type="cg", preconditioner="none", absolute_tolerance=0.0,
                               relative_tolerance=1e-10, max_iterations=5000))
    assert solver.info["path"] == "stencil"
    assert r.status == want.status == "Converged"
    assert abs(r.iterations - want.iterations) <= max(2, 0.02 * want.iterations)
    assert np.linalg.norm(r.solution - want.solution) <= 1e-9 * np.linalg.norm(want.solution)
    solver.close()


def test_learned_preconditioner_through_csr_and_new_values(ctx):
    """The learned solve through the CSR entry on an oracle-assembled 64^2 p'
    system, then the same solver on the same pattern with new values (the
    operator and its hierarchy are kept, the values refreshed)."""
    from cfdapp_b200 import cfdb
    n = 64
    case, fc, diag, off, b = O.isolated_pprime(2, n)
    ro, ci, va = csr_from_bands(diag, off, (n, n))
    solver = cfdb.CsrSolver(ctx)
    s = _settings(type="cg", preconditioner="learned_mg", absolute_tolerance=0.0,
                  relative_tolerance=1e-10, max_iterations=2000)
    want = O.stencil_solve(case, diag, off, b, rel_tol=1e-12, max_iterations=20000)
    r = solver.solve(ro, ci, va, b, s)
    assert solver.info["path"] == "faces" and not solver.info["learned_declined"]
    assert r.status == "Converged" and r.fallback_iterations == 0
    assert np.linalg.norm(r.solution - want.solution) <= 1e-6 * np.linalg.norm(want.solution)
    # doubled coefficients on the same pattern: x halves
    r2 = solver.solve(ro, ci, 2.0 * va, b, s)
    assert r2.status == "Converged"
    np.testing.assert_allclose(r2.solution, 0.5 * r.solution, rtol=1e-6, atol=1e-12)
    solver.close()


def test_statuses_of_bad_systems(ctx):
    from cfdapp_b200 import cfdb
    s, _ = load_system("csr_pprime2d_24")
    ro, ci, va, b = s["offsets"], s["columns"], s["values"], s["rhs"]
    solver = cfdb.CsrSolver(ctx)
    cg = _settings(type="cg", preconditioner="jacobi", absolute_tolerance=0.0,
                   relative_tolerance=1e-8, max_iterations=100)
    # a NaN in A (CG.cpp:23-26), checked before anything else
    bad = va.copy()
    bad[7] = np.nan
    assert solver.solve(ro, ci, bad, b, cg).status == "NonFiniteInput"
    # a NaN in the initial guess
    x0 = np.zeros(len(b))
    x0[3] = np.inf
    assert solver.solve(ro, ci, va, b, cg, x0=x0).status == "NonFiniteInput"
    # a near-zero diagonal: the Jacobi build refuses it (Preconditioner.cpp:11-32)
    tiny = va.copy()
    r = 50
    q = next(q for q in range(int(ro[r]), int(ro[r + 1])) if int(ci[q]) == r)
    tiny[q] = 1e-13
    assert solver.solve(ro, ci, tiny, b, cg).status == "InvalidSystem"
    # an unstructured matrix is refused loudly (no CPU solver behind the entry)
    dense_ro = np.array([0, 4, 8, 12, 16], np.uint64)
    dense_ci = np.tile(np.arange(4, dtype=np.uint64), 4)
    with pytest.raises(cfdb.CfdbError, match="unsupported"):
        solver.solve(dense_ro, dense_ci, np.eye(4).reshape(-1) + 0.1, np.ones(4), cg)
    solver.close()
