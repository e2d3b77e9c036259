"""GPU-resident SIMPLE against the reference.

Stage parity (pressure gradient, relaxed momentum system) is checked against
the oracle, which is bit-identical to the reference; whole solves are checked
against the reference's own outputs (tests/golden/, generated by
tests/golden/make_golden.py from the reference build): same status, outer
iteration count within 2 %, converged fields within 1e-6 relative L2.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _kv(args):
    return dict(a.split("=", 1) for a in args.split())


def gpu_case_from_args(args, golden=None):
    """The case and settings of a reference driver argument string; a graded
    mesh (gradex / gradey) takes the reference's node coordinates from the
    golden fixture."""
    from cfdapp_b200.cfdb import LinearSolverSettings, SIMPLESettings, SimpleCase
    a = _kv(args)
    dim = int(a.get("dim", 2))
    nx = int(a["nx"])
    ny, nz = int(a.get("ny", nx)), int(a.get("nz", nx))
    mu, rho = float(a.get("mu", 0.01)), float(a.get("rho", 1.0))
    if a.get("flow", "cavity") == "channel":
        case = SimpleCase.channel(nx, ny, float(a.get("lx", 1)), float(a.get("ly", 1)),
                                  float(a.get("inlet", 1)), mu=mu, rho=rho)
    else:
        case = SimpleCase.cavity(dim, nx, float(a.get("lid", 1)), mu=mu, rho=rho)
        case.n = (nx, ny, nz)[:dim]
    ms = LinearSolverSettings(absolute_tolerance=float(a.get("mabs", 1e-10)),
                              relative_tolerance=float(a.get("mrel", 1e-8)),
                              max_iterations=int(a.get("mmax", 500)),
                              type=a.get("msolver", "bicgstab"), preconditioner="none")
    ps = LinearSolverSettings(absolute_tolerance=float(a.get("pabs", 0.0)),
                              relative_tolerance=float(a.get("prel", 1e-8)),
                              max_iterations=int(a.get("pmax", 5000)),
                              type=a.get("psolver", "cg"),
                              preconditioner=a.get("ppre", "jacobi"))
    if "gradex" in a or "gradey" in a:
        case.nodes = (golden["x_nodes"], golden["y_nodes"])
    s = SIMPLESettings(max_iterations=int(a.get("outer", 1000)),
                       velocity_relaxation=float(a.get("au", 0.7)),
                       pressure_relaxation=float(a.get("ap", 0.3)),
                       velocity_tolerance=float(a.get("tolu", 1e-6)),
                       pressure_tolerance=float(a.get("tolp", 1e-6)),
                       continuity_tolerance=float(a.get("tolc", 1e-6)),
                       convection_scheme=a.get("scheme", "upwind"),
                       face_flux=a.get("flux", "auto"), momentum_solver=ms, pressure_solver=ps)
    return case, s


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("case_args", [
    "dim=2 nx=20 ny=20",
    "dim=2 nx=24 ny=8 lx=8 ly=1 flow=channel mu=0.1",
    "dim=3 nx=7 ny=6 nz=5",
])
def test_pressure_gradient_matches_oracle(ctx, case_args):
    from cfdapp_b200.cfdb import Simple
    from test_oracle_pin import simple_from_args
    case, s = gpu_case_from_args(case_args)
    ocase, _ = simple_from_args(case_args)
    rng = np.random.default_rng(11)
    n = case.cells()
    u, v, w, p = (rng.normal(size=n) for _ in range(4))
    sim = Simple(ctx, case, s)
    sim.set_state(u, v, w if case.dim == 3 else None, p)
    g = sim.pressure_gradient()
    go = O.scalar_gradient(ocase, p)
    for a in range(case.dim):
        np.testing.assert_allclose(g[a], go[a], rtol=1e-14, atol=1e-14 * np.abs(go[a]).max())


@pytest.mark.parametrize("scheme", ["upwind", "central", "lud", "quick"])
@pytest.mark.parametrize("case_args", [
    "dim=2 nx=16 ny=12",
    "dim=2 nx=20 ny=6 lx=4 ly=1 flow=channel mu=0.05",
    "dim=3 nx=6 ny=5 nz=7",
])
def test_momentum_system_matches_oracle(ctx, case_args, scheme):
    from cfdapp_b200.cfdb import Simple
    from test_oracle_pin import simple_from_args
    case, s = gpu_case_from_args(case_args + f" scheme={scheme}")
    ocase, os_ = simple_from_args(case_args + f" scheme={scheme}")
    rng = np.random.default_rng(5)
    n = case.cells()
    u, v, w, p = (rng.normal(size=n) for _ in range(4))
    sim = Simple(ctx, case, s)
    sim.set_state(u, v, w if case.dim == 3 else None, p)
    for comp in range(case.dim):
        d, off, rhs = sim.assemble_momentum(comp)
        do, offo, rhso = O.momentum_system(ocase, os_, comp, u, v, w if case.dim == 3 else None, p)
        np.testing.assert_allclose(d, do, rtol=1e-14)
        np.testing.assert_allclose(rhs, rhso, rtol=1e-13, atol=1e-14 * np.abs(rhso).max())
        for q in range(2 * case.dim):
            np.testing.assert_allclose(off[q], offo[q], rtol=1e-14, atol=1e-16)


def _golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return g, json.loads(str(g["meta"]))


@pytest.mark.parametrize("name", ["cavity2d_20_bicgstab", "cavity2d_16_jacobicg",
                                  "channel2d_32x8_central_rc", "cavity2d_16_lud",
                                  "cavity3d_8_quick_rc", "cavity2d_129_config1",
                                  "cavity3d_32_lud_rc_re1000", "cavity3d_48_lud_rc_re1000",
                                  "cavity2d_33_jacobicg", "cavity2d_24_graded",
                                  "cavity2d_24_graded_lud_rc", "channel2d_32x12_graded"])
def test_simple_matches_reference_outputs(ctx, name):
    from cfdapp_b200.cfdb import simple_solve
    g, meta = _golden(name)
    case, s = gpu_case_from_args(meta["args"], g)
    r = simple_solve(ctx, case, s)
    assert r.status == meta["status"]
    if meta["status"] == "Converged":
        assert abs(r.iterations - meta["iterations"]) <= max(2, 0.02 * meta["iterations"])
    else:
        assert r.iterations == meta["iterations"]
    for f in ("u", "v", "w", "p"):
        if f in g.files:
            assert _rel(getattr(r, f), g[f]) <= 1e-6, f
    assert _rel(r.flux, g["flux"]) <= 1e-6
    assert r.kernel_launches > 0


def test_simple_failure_statuses(ctx):
    """Configuration errors and starved linear solves map to the reference's statuses."""
    from cfdapp_b200.cfdb import LinearSolverSettings, SIMPLESettings, SimpleCase, simple_solve
    case = SimpleCase.cavity(2, 12)
    bad = SIMPLESettings(max_iterations=5, velocity_relaxation=1.5)
    assert simple_solve(ctx, case, bad).status == "InvalidConfiguration"
    starved_p = SIMPLESettings(max_iterations=5, pressure_solver=LinearSolverSettings(
        type="cg", preconditioner="jacobi", absolute_tolerance=0.0, relative_tolerance=1e-12,
        max_iterations=2))
    assert simple_solve(ctx, case, starved_p).status == "PressureCorrectionFailure"
    starved_m = SIMPLESettings(max_iterations=5, momentum_solver=LinearSolverSettings(
        type="bicgstab", preconditioner="none", absolute_tolerance=0.0, relative_tolerance=1e-14,
        max_iterations=1))
    assert simple_solve(ctx, case, starved_m).status == "MomentumFailure"
    nan = np.zeros(case.cells())
    nan[3] = np.nan
    assert simple_solve(ctx, case, SIMPLESettings(max_iterations=5), u0=nan).status == "NonFiniteState"


@pytest.mark.parametrize("name", ["cavity2d_16_jacobicg", "channel2d_32x8_central_rc",
                                  "cavity2d_16_lud", "cavity3d_8_quick_rc",
                                  "cavity2d_129_config1", "cavity3d_32_lud_rc_re1000",
                                  "cavity3d_48_lud_rc_re1000", "cavity2d_24_graded"])
def test_simple_with_learned_pressure_solver_matches_reference(ctx, name):
    """The same SIMPLE runs with every p' system solved by the learned-
    preconditioned FCG (to the same tolerance) land on the reference's fields."""
    from cfdapp_b200.cfdb import simple_solve
    g, meta = _golden(name)
    args = meta["args"].replace("psolver=bicgstab", "psolver=cg")
    args = " ".join(a for a in args.split() if not a.startswith("ppre="))
    case, s = gpu_case_from_args(args + " psolver=cg ppre=learned_mg", g)
    r = simple_solve(ctx, case, s)
    assert r.status == meta["status"]
    if meta["status"] == "Converged":
        assert abs(r.iterations - meta["iterations"]) <= max(3, 0.03 * meta["iterations"])
    else:
        assert r.iterations == meta["iterations"]
    # a run stopped early carries the p' solve tolerance into its fields
    bar = 1e-6 if float(_kv(args).get("prel", 1e-8)) <= 1e-8 else 1e-3
    for f in ("u", "v", "w", "p"):
        if f in g.files:
            assert _rel(getattr(r, f), g[f]) <= bar, f
    assert _rel(r.flux, g["flux"]) <= bar
