"""Batched SIMPLE on the GPU (cfdb_batch_*).

Each golden case of the reference (tests/golden/) runs inside a batch next
to cases of other sizes under the same settings: the golden case must land on
the reference's outputs with the single-case bar (same status, outer
iterations within 2 %, fields within 1e-6 relative L2), and every other case
on what the single-case GPU session computes for it alone.  Per-case failure
statuses, the autotuner (which must leave the state alone) and multi-block
Krylov teams are covered too.
"""
import json
import os

import numpy as np
import pytest

from test_simple_gpu import _kv, _rel, gpu_case_from_args

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return g, json.loads(str(g["meta"]))


def _extras(args):
    """Two more cases of the golden case's family, of other sizes."""
    a = _kv(args)
    dim = int(a.get("dim", 2))
    drop = ("nx", "ny", "nz", "lx", "ly", "mu", "lid")
    base = " ".join(x for x in args.split() if x.split("=")[0] not in drop)
    if a.get("flow") == "channel":
        return [base + " nx=16 ny=6 lx=4 ly=1 mu=0.1", base + " nx=40 ny=10 lx=8 ly=1 mu=0.12"]
    if dim == 3:
        return [base + " nx=6 ny=6 nz=6 mu=0.001", base + " nx=8 ny=6 nz=7 mu=0.002"]
    return [base + " nx=12 ny=12 mu=0.02", base + " nx=24 ny=18 mu=0.01 lid=0.5"]


def _check_against_single(ctx, case, s, got, res, bar=1e-6):
    from cfdapp_b200.cfdb import simple_solve
    ref = simple_solve(ctx, case, s)
    assert res["status"] == ref.status
    assert abs(res["iterations"] - ref.iterations) <= max(2, 0.02 * ref.iterations)
    u, v, w, p, f = got
    for name, a, b in (("u", u, ref.u), ("v", v, ref.v), ("p", p, ref.p), ("flux", f, ref.flux)):
        assert _rel(a, b) <= bar, name
    if case.dim == 3:
        assert _rel(w, ref.w) <= bar


@pytest.mark.parametrize("name", ["cavity2d_16_jacobicg", "cavity2d_20_bicgstab",
                                  "channel2d_32x8_central_rc", "cavity2d_16_lud",
                                  "cavity3d_8_quick_rc"])
def test_batch_matches_reference_and_single_case(ctx, name):
    from cfdapp_b200.cfdb import Batch
    g, meta = _golden(name)
    case, s = gpu_case_from_args(meta["args"])
    others = [gpu_case_from_args(x) for x in _extras(meta["args"])]
    cases = [others[0][0], case, others[1][0]]
    b = Batch(ctx, cases, s)
    for k in range(3):
        b.set_state(k)
    st = b.iterate(s.max_iterations)
    res = b.results()
    assert st["graph_launches"] <= s.max_iterations
    # the golden case
    r = res[1]
    assert r["status"] == meta["status"]
    if meta["status"] == "Converged":
        assert abs(r["iterations"] - meta["iterations"]) <= max(2, 0.02 * meta["iterations"])
    else:
        assert r["iterations"] == meta["iterations"]
    u, v, w, p, f = b.get_state(1)
    for fld, arr in (("u", u), ("v", v), ("w", w), ("p", p)):
        if fld in g.files:
            assert _rel(arr, g[fld]) <= 1e-6, fld
    assert _rel(f, g["flux"]) <= 1e-6
    # the other cases against the single-case session
    for k in (0, 2):
        _check_against_single(ctx, cases[k], s, b.get_state(k), res[k])
    b.close()


def test_batch_failure_statuses_are_per_case(ctx):
    from cfdapp_b200.cfdb import Batch, LinearSolverSettings, SIMPLESettings, SimpleCase, simple_solve
    cases = [SimpleCase.cavity(2, 12), SimpleCase.cavity(2, 14), SimpleCase.cavity(2, 10)]
    s = SIMPLESettings(max_iterations=5)
    b = Batch(ctx, cases, s)
    nan = np.zeros(cases[1].cells())
    nan[3] = np.nan
    b.set_state(0)
    b.set_state(1, u=nan)
    b.set_state(2)
    b.iterate(10)
    res = b.results()
    assert res[1]["status"] == "NonFiniteState" and res[1]["iterations"] == 0
    for k in (0, 2):
        assert res[k]["status"] == "MaxIterations" and res[k]["iterations"] == 5
        _check_against_single(ctx, cases[k], s, b.get_state(k), res[k], bar=1e-7)
    b.close()
    starved_p = SIMPLESettings(max_iterations=5, pressure_solver=LinearSolverSettings(
        type="cg", preconditioner="jacobi", absolute_tolerance=0.0, relative_tolerance=1e-12,
        max_iterations=2))
    starved_m = SIMPLESettings(max_iterations=5, momentum_solver=LinearSolverSettings(
        type="bicgstab", preconditioner="none", absolute_tolerance=0.0, relative_tolerance=1e-14,
        max_iterations=1))
    for s, want in ((starved_p, "PressureCorrectionFailure"), (starved_m, "MomentumFailure")):
        b = Batch(ctx, cases[:2], s)
        b.iterate(5)
        res = b.results()
        for k in range(2):
            single = simple_solve(ctx, cases[k], s)
            assert single.status == want
            assert res[k]["status"] == want and res[k]["iterations"] == single.iterations
        b.close()


def _uneven_batch():
    from cfdapp_b200.cfdb import LinearSolverSettings, SIMPLESettings, SimpleCase
    sides = [16, 40, 24, 128, 64]
    cases = [SimpleCase.cavity(2, n, mu=0.01 * (1 + k % 3)) for k, n in enumerate(sides)]
    s = SIMPLESettings(max_iterations=25, pressure_solver=LinearSolverSettings(
        type="cg", preconditioner="jacobi", absolute_tolerance=0.0, relative_tolerance=1e-8,
        max_iterations=5000))
    return cases, s


def test_autotune_keeps_the_state_and_the_results(ctx):
    """The tuner times candidates on the current state without advancing it;
    a tuned batch (multi-block Krylov teams on the 128^2 case) computes what
    an untuned one does, to rounding."""
    from cfdapp_b200.cfdb import Batch
    cases, s = _uneven_batch()
    tuned, plain = Batch(ctx, cases, s), Batch(ctx, cases, s)
    for k in range(len(cases)):
        tuned.set_state(k)
        plain.set_state(k)
    t = tuned.autotune()
    assert t.candidates >= 12 and t.cell_threads in (128, 256, 512)
    assert t.face_threads in (128, 256, 512)
    assert t.cell_stage_ms > 0 and t.face_stage_ms > 0 and t.pprime_solve_ms > 0
    assert all(r["iterations"] == 0 for r in tuned.results())
    tuned.iterate(s.max_iterations)
    plain.iterate(s.max_iterations)
    rt, rp = tuned.results(), plain.results()
    for k in range(len(cases)):
        assert rt[k]["status"] == rp[k]["status"] and rt[k]["iterations"] == rp[k]["iterations"]
        for a, c in zip(tuned.get_state(k), plain.get_state(k)):
            if a.size:
                assert _rel(a, c) <= 1e-9
    tuned.close()
    plain.close()


def test_uneven_batch_matches_single_cases(ctx):
    from cfdapp_b200.cfdb import Batch
    cases, s = _uneven_batch()
    b = Batch(ctx, cases, s, history_cap=s.max_iterations)
    for k in range(len(cases)):
        b.set_state(k)
    stats = b.iterate(s.max_iterations)
    assert stats["graph_launches"] == s.max_iterations and stats["device_ms"] > 0
    assert stats["kernel_launches"] >= 15 * s.max_iterations
    res = b.results()
    for k, case in enumerate(cases):
        _check_against_single(ctx, case, s, b.get_state(k), res[k], bar=1e-7)
        h = b.history(k)
        assert h.shape == (res[k]["iterations"], 5)
        assert h[-1, 4] == pytest.approx(res[k]["final"]["continuity"], rel=1e-12)
    b.close()


def test_profiled_iteration_times_every_launch(ctx):
    from cfdapp_b200.cfdb import Batch
    cases, s = _uneven_batch()
    b = Batch(ctx, cases, s)
    for k in range(len(cases)):
        b.set_state(k)
    prof = b.profile_iteration()
    ids = [i for i, _ in prof]
    assert ids.count(-1) == 2 and ids.count(-2) == 1 and all(ms >= 0 for _, ms in prof)
    assert all(r["iterations"] == 1 for r in b.results())
    b.close()


def test_batch_edge_cases(ctx):
    """One-case and minimal-grid batches, mixed families in one batch, and the
    configurations a batch refuses."""
    from cfdapp_b200.cfdb import (Batch, CfdbError, LinearSolverSettings, SIMPLESettings,
                                  SimpleCase)
    s = SIMPLESettings(max_iterations=8)
    cases = [SimpleCase.cavity(2, 2), SimpleCase.channel(9, 3, 3.0, 1.0),
             SimpleCase.cavity(2, 33)]
    b = Batch(ctx, cases, s)
    for k in range(len(cases)):
        b.set_state(k)
    b.iterate(20)
    res = b.results()
    for k, case in enumerate(cases):
        _check_against_single(ctx, case, s, b.get_state(k), res[k], bar=1e-7)
    b.close()
    one = Batch(ctx, [SimpleCase.cavity(2, 17)], s)
    one.set_state(0)
    one.iterate(8)
    _check_against_single(ctx, SimpleCase.cavity(2, 17), s, one.get_state(0), one.results()[0],
                          bar=1e-7)
    one.close()
    with pytest.raises(CfdbError):
        Batch(ctx, [SimpleCase.cavity(2, 8), SimpleCase.cavity(3, 6)], s)
    learned_bicgstab = SIMPLESettings(max_iterations=8, pressure_solver=LinearSolverSettings(
        type="bicgstab", preconditioner="learned_mg"))
    with pytest.raises(CfdbError):
        Batch(ctx, [SimpleCase.cavity(2, 8)], learned_bicgstab)


@pytest.mark.parametrize("name", ["cavity2d_16_jacobicg", "cavity3d_32_lud_rc_re1000"])
def test_batch_mixed_precision_pprime_matches_reference(ctx, name):
    """The batch's FP32_REFINED p' solve (a mixed-precision CG that keeps one
    Krylov space, FP64 residual replacement): every p' solve still stops on
    an FP64 true residual at the case's tolerance, so the golden case lands
    on the reference's fields with the single-case bar (outer iterations
    within 2 %, fields within 1e-6 relative L2)."""
    from cfdapp_b200.cfdb import Batch
    import dataclasses
    g, meta = _golden(name)
    case, s = gpu_case_from_args(meta["args"])
    s = dataclasses.replace(s, pressure_solver=dataclasses.replace(s.pressure_solver,
                                                                  precision="fp32_refined"))
    other = gpu_case_from_args(_extras(meta["args"])[0])[0]
    b = Batch(ctx, [other, case], s)
    for k in range(2):
        b.set_state(k)
    b.iterate(s.max_iterations)
    r = b.results()[1]
    assert r["status"] == meta["status"] == "Converged"
    assert abs(r["iterations"] - meta["iterations"]) <= max(2, 0.02 * meta["iterations"])
    u, v, w, p, f = b.get_state(1)
    for fld, arr in (("u", u), ("v", v), ("w", w), ("p", p)):
        if fld in g.files:
            assert _rel(arr, g[fld]) <= 1e-6, fld
    assert _rel(f, g["flux"]) <= 1e-6
    assert b.results()[0]["status"] == "Converged"
    b.close()


@pytest.mark.parametrize("name", ["cavity2d_16_jacobicg", "cavity3d_32_lud_rc_re1000"])
def test_batch_learned_pprime_matches_reference(ctx, name):
    """The batch's learned p' solve (every active case's p' system by the
    single-case learned FCG on the case's pooled face coefficients): the
    golden case lands on the reference's fields with the bar of the
    single-case learned SIMPLE test (outer iterations within 3 %, fields within
    1e-6 relative L2), and the other case converges."""
    from cfdapp_b200.cfdb import Batch
    import dataclasses
    g, meta = _golden(name)
    case, s = gpu_case_from_args(meta["args"])
    s = dataclasses.replace(s, pressure_solver=dataclasses.replace(s.pressure_solver,
                                                                  preconditioner="learned_mg"))
    other = gpu_case_from_args(_extras(meta["args"])[0])[0]
    b = Batch(ctx, [other, case], s)
    for k in range(2):
        b.set_state(k)
    st = b.iterate(s.max_iterations)
    assert st["kernel_launches"] > 0
    r = b.results()[1]
    assert r["status"] == meta["status"] == "Converged"
    assert abs(r["iterations"] - meta["iterations"]) <= max(3, 0.03 * meta["iterations"])
    u, v, w, p, f = b.get_state(1)
    for fld, arr in (("u", u), ("v", v), ("w", w), ("p", p)):
        if fld in g.files:
            assert _rel(arr, g[fld]) <= 1e-6, fld
    assert _rel(f, g["flux"]) <= 1e-6
    assert b.results()[0]["status"] == "Converged"
    b.close()
