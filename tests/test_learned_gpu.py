"""The learned-preconditioner p' solve (CFDB_PRECOND_LEARNED_MG): a V-cycle
network inside FP64 flexible CG, falling back to Jacobi-PCG on stagnation.

It has no counterpart in the reference, so the bars are the reference's own
acceptance quantities: the same converged status and the same FP64
relative-residual target as CG + Jacobi (src/algebra/CG.cpp:14-148), the
true residual recomputed on the CPU by the oracle from the returned x, and a
solution within 1e-6 relative L2 (the bar for fields) of the oracle's CG
solution when both are driven to 1e-10 (at 1e-11 the reference's absolute
1e-30 test on p.Ap already ends its CG in Breakdown on these systems).  The point of the method -- far fewer iterations than
Jacobi-PCG -- is asserted too.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _settings(**kw):
    from cfdapp_b200.cfdb import LinearSolverSettings
    base = dict(absolute_tolerance=0.0, relative_tolerance=1e-8, max_iterations=100000,
                preconditioner="learned_mg")
    base.update(kw)
    return LinearSolverSettings(**base)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _true_rel_residual(case, diag, off, b, x):
    return float(np.linalg.norm(b - O.stencil_apply(case, diag, off, x)) / np.linalg.norm(b))


@pytest.mark.parametrize("dim,n", [(2, 64), (2, 256), (3, 16), (3, 48)])
def test_learned_reaches_tolerance_in_few_iterations(ctx, dim, n):
    from cfdapp_b200.cfdb import POperator
    case, fc, diag, off, b = O.isolated_pprime(dim, n)
    op = POperator(ctx, dim, [n] * dim)
    res = op.solve(b, _settings())
    jac = op.solve(b, _settings(preconditioner="jacobi"))
    assert res.status == jac.status == "Converged"
    assert res.fallback_iterations == 0
    assert _true_rel_residual(case, diag, off, b, res.solution) <= 1.05e-8
    assert res.true_residual / res.initial_residual <= 1.05e-8
    assert res.residual_history[0] == pytest.approx(res.initial_residual)
    assert res.residual_history[-1] / res.initial_residual <= 1e-8
    assert res.iterations * 4 <= jac.iterations


@pytest.mark.parametrize("dim,n", [(2, 128), (3, 24)])
def test_learned_solution_matches_oracle(ctx, dim, n):
    from cfdapp_b200.cfdb import POperator
    case, fc, diag, off, b = O.isolated_pprime(dim, n)
    ref = O.stencil_solve(case, diag, off, b, rel_tol=1e-10, history=False)
    op = POperator(ctx, dim, [n] * dim)
    res = op.solve(b, _settings(relative_tolerance=1e-10))
    assert res.status == ref.status == "Converged"
    assert _rel(res.solution, ref.solution) <= 1e-6
    # tighter than the reference can go: FCG keeps converging
    tight = op.solve(b, _settings(relative_tolerance=1e-12))
    assert tight.status == "Converged" and tight.fallback_iterations == 0


def test_learned_face_operator_non_square(ctx):
    """Per-face coefficients of a SIMPLE iteration (random response field)."""
    from cfdapp_b200.cfdb import POperator
    case = O.Case(2, (96, 80), (1.2, 1.0), [("wall", (0, 0, 0))] * 4,
                  [("fixed_gradient", 0.0)] * 4)
    rng = np.random.default_rng(11)
    cells = case.cells()
    du = np.exp(rng.normal(size=cells) * 0.5)
    dv = np.exp(rng.normal(size=cells) * 0.5)
    flux = rng.normal(size=case.faces()) * 1e-3
    fc, diag, off, rhs = O.assemble_pprime(case, 1.0, flux, du, dv)
    op = POperator(ctx, 2, (96, 80), (1.2, 1.0), face_coeff=fc)
    res = op.solve(rhs, _settings())
    assert res.status == "Converged"
    assert _true_rel_residual(case, diag, off, rhs, res.solution) <= 1.05e-8
    ref = O.stencil_solve(case, diag, off, rhs, history=False)
    assert res.iterations * 3 <= ref.iterations


def test_learned_dirichlet_unpinned(ctx):
    from cfdapp_b200.cfdb import POperator
    case = O.channel(64, 16, 4.0, 1.0)
    ones = np.ones(case.cells())
    rng = np.random.default_rng(3)
    flux = rng.normal(size=case.faces()) * 1e-2
    fc, diag, off, rhs = O.assemble_pprime(case, 1.0, flux, ones, ones)
    op = POperator(ctx, 2, (64, 16), (4.0, 1.0), face_coeff=fc, pinned=False)
    res = op.solve(rhs, _settings())
    assert res.status == "Converged"
    assert _true_rel_residual(case, diag, off, rhs, res.solution) <= 1.05e-8


def test_learned_status_edge_cases(ctx):
    from cfdapp_b200.cfdb import POperator
    op = POperator(ctx, 2, (32, 32))
    zero = op.solve(np.zeros(1024), _settings())
    assert zero.status == "Converged" and zero.iterations == 0
    b = O.synth_rhs(2, 32)
    capped = op.solve(b, _settings(max_iterations=3))
    assert capped.status == "MaxIterations" and capped.iterations == 3
    bad = b.copy()
    bad[5] = np.inf
    assert op.solve(bad, _settings()).status == "NonFiniteInput"
    loose = op.solve(b, _settings(absolute_tolerance=1.0))
    assert loose.status == "Converged" and loose.iterations == 0
    # repeated solves reuse the captured graph and give identical results
    r1 = op.solve(b, _settings())
    r2 = op.solve(b, _settings())
    assert r1.iterations == r2.iterations
    np.testing.assert_array_equal(r1.solution, r2.solution)


def test_learned_falls_back_to_jacobi_when_the_network_is_useless(ctx):
    """A zero network gives z = 0: FCG stops and Jacobi-PCG finishes the solve."""
    from cfdapp_b200.cfdb import POperator
    case, fc, diag, off, b = O.isolated_pprime(2, 48)
    op = POperator(ctx, 2, (48, 48))
    try:
        ctx.mg_set_weights(2, np.zeros((1, 27), np.float32), np.zeros(1, np.float32),
                           coarse_sweeps=0)
        res = op.solve(b, _settings())
    finally:
        ctx.mg_reset_weights(2, trained=True)
    assert res.status == "Converged"
    assert res.fallback_iterations > 0
    assert _true_rel_residual(case, diag, off, b, res.solution) <= 1.05e-8


def test_weights_api(ctx):
    from cfdapp_b200.cfdb import CfdbError
    w = ctx.mg_get_weights(3)
    assert w["kernels"].shape == (w["levels"], 27)
    bad = np.zeros((1, 27), np.float32)
    bad[0, 12] = 1.0  # not point-symmetric
    with pytest.raises(CfdbError):
        ctx.mg_set_weights(3, bad, np.ones(1, np.float32))
    flat = np.zeros((1, 27), np.float32)
    flat[0, 0] = 1.0  # 2D kernels live in the middle plane only
    flat[0, 26] = 1.0
    with pytest.raises(CfdbError):
        ctx.mg_set_weights(2, flat, np.ones(1, np.float32))
    k = np.zeros((2, 27), np.float32)
    k[:, 13] = 0.7
    k[:, 12] = k[:, 14] = 0.05
    ctx.mg_set_weights(3, k, np.array([1.0, 0.9], np.float32), nu=3, coarse_sweeps=20)
    got = ctx.mg_get_weights(3)
    assert got["levels"] == 2 and got["nu"] == 3 and got["coarse_sweeps"] == 20
    np.testing.assert_array_equal(got["kernels"], k)
    ctx.mg_reset_weights(3, trained=False)
    assert ctx.mg_get_weights(3)["kernels"][0, 13] == np.float32(0.8)
    ctx.mg_reset_weights(3, trained=True)


# ------------------------------------------------ the network against its oracle
from oracle import mg_oracle as MO  # noqa: E402


def _face_op(ctx, dim, n, seed):
    from cfdapp_b200.cfdb import POperator
    fc = MO.random_faces(dim, n, seed)
    op = POperator(ctx, dim, n, face_coeff=fc, pinned=True, reference_cell=0)
    dims, f = MO.kernel_faces(dim, n, fc)
    return op, MO.hierarchy(dims, f, dim)


@pytest.mark.parametrize("dim,n", [(2, (40, 36)), (3, (24, 20, 18))])
def test_vcycle_kernels_match_oracle(ctx, dim, n):
    """One application of the solve's tiled V-cycle (grid levels + the
    block-resident coarse levels) against the FP64 restatement."""
    op, H = _face_op(ctx, dim, n, 21)
    k, c = MO.random_weights(dim, 2, 22)
    k32, c32 = k.astype(np.float32), c.astype(np.float32)
    ctx.mg_set_weights(dim, k32, c32, nu=2, coarse_sweeps=10)
    try:
        r = np.random.default_rng(23).normal(size=int(np.prod(n))).astype(np.float32)
        z = op.mg_apply(r)
        V = MO.VCycle(dim, H, k32.astype(np.float64), c32.astype(np.float64), nu=2,
                      coarse_sweeps=10)
        zr = V.apply(r.astype(np.float64), pin=0)
        assert _rel(z.astype(np.float64), zr) <= 2e-5
    finally:
        ctx.mg_reset_weights(dim, trained=True)


@pytest.mark.parametrize("dim,n", [(2, (20, 18)), (3, (10, 8, 8))])
def test_gradient_matches_finite_differences(ctx, dim, n):
    """The GPU reverse-mode gradient of the training loss against central
    differences of the FP64 oracle loss (h = 1e-4 on every free weight)."""
    op, H = _face_op(ctx, dim, n, 31)
    k, c = MO.random_weights(dim, 2, 32)
    k = k.astype(np.float32).astype(np.float64)
    c = c.astype(np.float32).astype(np.float64)
    nu, sweeps = 2, 6
    ctx.mg_set_weights(dim, k.astype(np.float32), c.astype(np.float32), nu=nu,
                       coarse_sweeps=sweeps)
    e = np.random.default_rng(33).normal(size=(3, int(np.prod(n)))).astype(np.float32)
    try:
        loss, gk, gc = op.mg_loss_grad(e)
    finally:
        ctx.mg_reset_weights(dim, trained=True)

    def oracle_loss(kk, cc):
        V = MO.VCycle(dim, H, kk, cc, nu=nu, coarse_sweeps=sweeps)
        return float(np.mean([V.loss(ei.astype(np.float64), pin=0) for ei in e]))

    assert loss == pytest.approx(oracle_loss(k, c), rel=1e-4)
    h = 1e-4
    g_gpu, g_fd = [], []
    for l in range(2):
        for t in MO.free_params(dim):
            kp, km = k.copy(), k.copy()
            for kk, sgn in ((kp, 1.0), (km, -1.0)):
                kk[l, t] += sgn * h
                if t != 13:
                    kk[l, 26 - t] += sgn * h
            g_fd.append((oracle_loss(kp, c) - oracle_loss(km, c)) / (2 * h))
            g_gpu.append(gk[l, t])
        cp, cm = c.copy(), c.copy()
        cp[l] += h
        cm[l] -= h
        g_fd.append((oracle_loss(k, cp) - oracle_loss(k, cm)) / (2 * h))
        g_gpu.append(gc[l])
    g_gpu, g_fd = np.array(g_gpu), np.array(g_fd)
    assert np.linalg.norm(g_gpu - g_fd) <= 2e-3 * np.linalg.norm(g_fd)
    # tied taps carry the same gradient
    for l in range(2):
        for t in MO.free_params(dim):
            assert gk[l, t] == gk[l, 26 - t]


# ---------------------------------------------------- what training buys
@pytest.mark.parametrize("dim,n,gain", [(2, 512, 0.8), (3, 96, 0.6)])
def test_trained_weights_cut_iterations(ctx, dim, n, gain):
    """The shipped (GPU-trained) weights need clearly fewer FCG iterations
    than the untrained network (damped-Jacobi layers in the same cycle) on
    systems larger than any seen in training (128^2 / 32^3): the isolated p'
    system and a smooth-response one."""
    from cfdapp_b200.cfdb import POperator
    from cfdapp_b200.mgtrain import random_operator_faces
    b = O.synth_rhs(dim, n)
    ops = [POperator(ctx, dim, [n] * dim),
           POperator(ctx, dim, [n] * dim,
                     face_coeff=random_operator_faces(dim, [n] * dim, np.random.default_rng(5)))]
    ctx.mg_reset_weights(dim, trained=True)
    w = ctx.mg_get_weights(dim)
    jacobi = np.zeros((1, 27), np.float32)
    jacobi[0, 13] = 0.8  # the untrained layers: damped Jacobi, same cycle shape
    for op in ops:
        ctx.mg_set_weights(dim, jacobi, np.ones(1, np.float32), nu=w["nu"],
                           coarse_sweeps=w["coarse_sweeps"])
        untrained = op.solve(b, _settings())
        ctx.mg_reset_weights(dim, trained=True)
        trained = op.solve(b, _settings())
        assert untrained.status == trained.status == "Converged"
        assert trained.fallback_iterations == 0
        assert trained.iterations <= gain * untrained.iterations, (trained.iterations,
                                                                   untrained.iterations)


def test_learned_beats_jacobi_on_a_harvested_2048_cavity_system(ctx):
    """Evaluation at 2048^2 on a p' system the solver's own SIMPLE produced
    (lid-driven cavity, Re 400, after 5 outer iterations): the learned FCG
    reaches the FP64-verified 1e-8 relative residual at least 3x faster than
    FP64 Jacobi-PCG on the same GPU."""
    from cfdapp_b200.cfdb import POperator
    from cfdapp_b200.mgtrain import harvest_cavity
    faces, pinned, ref = harvest_cavity(ctx, 2, 2048, [400.0], 1, chunk=5)[0]
    assert pinned and np.all(np.isfinite(faces)) and faces.max() > 0
    op = POperator(ctx, 2, (2048, 2048), face_coeff=faces, pinned=pinned, reference_cell=ref)
    b = O.synth_rhs(2, 2048)
    learned = op.solve(b, _settings(), history_cap=0)
    jac = op.solve(b, _settings(preconditioner="jacobi"), history_cap=0)
    assert learned.status == jac.status == "Converged"
    assert learned.fallback_iterations == 0
    assert learned.true_residual / learned.initial_residual <= 1e-8
    assert jac.device_ms >= 3.0 * learned.device_ms, (jac.device_ms, learned.device_ms)
