"""Case directories in the reference's format (cfdapp_b200.cases): the
reader against the reference's own example cases (copied to
tests/golden/cases/ by tests/golden/make_results_fixtures.py), its
refusals, the GPU opt-in block, and -- on the GPU -- whole runs whose result
files land on the reference's committed results."""
import json
import os
import shutil

import numpy as np
import pytest

from cfdapp_b200 import cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = os.path.join(GOLDEN, "cases")


def test_reads_the_2d_cavity():
    c = cases.read_case(os.path.join(CASES, "lid_driven_cavity"))
    assert c.case.dim == 2 and tuple(c.case.n) == (20, 20) and c.case.length[:2] == (1.0, 1.0)
    assert c.case.rho == 1.0 and c.case.mu == 0.01
    assert [v[0] for v in c.case.vbc] == ["wall", "wall", "wall", "moving_wall"]
    assert c.case.vbc[3][1] == (1.0, 0.0, 0.0)
    assert all(p == ("fixed_gradient", 0.0) for p in c.case.pbc)
    s = c.settings
    assert s.max_iterations == 6000 and s.velocity_tolerance == 1e-6
    assert s.convection_scheme == "upwind" and s.face_flux == "automatic"
    assert s.pressure_solver.type == "bicgstab" and s.pressure_solver.preconditioner == "none"
    assert s.pressure_solver.absolute_tolerance == 1e-10 and s.pressure_solver.max_iterations == 2000


def test_reads_the_3d_cavity_and_the_channel():
    c3 = cases.read_case(os.path.join(CASES, "lid_driven_cavity_3d"))
    assert c3.case.dim == 3 and tuple(c3.case.n) == (16, 16, 16)
    assert c3.case.vbc[3][0] == "moving_wall" and c3.settings.convection_scheme == "quick"
    ch = cases.read_case(os.path.join(CASES, "poiseuille_flow"))
    assert tuple(ch.case.n) == (64, 8) and ch.case.length[:2] == (8.0, 1.0)
    assert ch.case.vbc[0] == ("inlet", (1.0, 0.0, 0.0)) and ch.case.vbc[1][0] == "outlet"
    assert ch.case.pbc[1] == ("fixed_value", 0.0)


def _copy(tmp_path, name):
    d = str(tmp_path / name)
    shutil.copytree(os.path.join(CASES, name), d)
    return d


def _edit(d, fn, f):
    p = os.path.join(d, fn)
    j = json.load(open(p))
    f(j)
    json.dump(j, open(p, "w"))


def test_gpu_opt_in_block(tmp_path):
    d = _copy(tmp_path, "lid_driven_cavity")
    _edit(d, "solver.json", lambda j: j.update(
        gpu={"pressure_preconditioner": "learned_mg"},
        pressure_linear_solver=dict(j["pressure_linear_solver"], type="CG")))
    s = cases.read_case(d).settings
    assert s.pressure_solver.type == "cg" and s.pressure_solver.preconditioner == "learned_mg"


@pytest.mark.parametrize("fn,change", [
    ("mesh.json", lambda j: j.update(grading={"y": {"type": "geometric", "ratio": 1.2}})),
    ("physics.json", lambda j: j.update(model="incompressible_turbulent")),
    ("solver.json", lambda j: j["pressure_linear_solver"].update(type="GMRES")),
    ("boundaries.json", lambda j: j["patches"]["left"]["velocity"].update(type="symmetry")),
    ("mesh.json", lambda j: j.update(type="unstructured")),
])
def test_refuses_what_is_not_on_the_gpu_path(tmp_path, fn, change):
    d = _copy(tmp_path, "lid_driven_cavity")
    _edit(d, fn, change)
    with pytest.raises(cases.CaseError):
        cases.read_case(d)


def _compare(out_dir, fixture, iterations_bar=0.02, p_rel_tol=1e-8):
    """Fields within 1e-6 relative L2 of the reference's committed run.  A case
    whose own p' solves stop at a looser relative tolerance (the reference's
    40x40 and 80x80 examples: 1e-6 and 1e-5) leaves its fields as exact as
    that stopping point, which follows the solver's rounding (measured: p
    6.7e-6 at 40x40, u 1.3e-6 at 80x80): the bar is then 1e-5.  Its pressure
    level is held only by the pinned cell, and BiCGSTAB stopped at 1e-5
    leaves the slowest, near-constant p' mode behind, which accumulates into
    an offset of the whole field against the pinned cell (80x80: 1e-4, 9.2e-4
    relative): such pressures are compared with their means removed, within
    ten times the case's own p' tolerance (80x80 measured: 1.5e-5)."""
    g = np.load(os.path.join(GOLDEN, fixture + ".npz"))
    rows = open(os.path.join(out_dir, "fields.csv")).read().splitlines()
    col = {h: i for i, h in enumerate(rows[0].split(","))}
    f = np.array([[float(x) for x in r.split(",")] for r in rows[1:]])
    rel = lambda a, b: np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
    bar = 1e-6 if p_rel_tol <= 1e-8 else 1e-5
    assert rel(f[:, col["velocity_x"]], g["u"]) <= bar
    assert rel(f[:, col["velocity_y"]], g["v"]) <= bar
    if "velocity_z" in col:
        assert rel(f[:, col["velocity_z"]], g["w"]) <= bar
    p, pref = f[:, col["pressure"]], g["p"]
    if p_rel_tol > 1e-8:
        p, pref = p - p.mean(), pref - pref.mean()
    assert rel(p, pref) <= max(bar, 10.0 * p_rel_tol)
    res = open(os.path.join(out_dir, "residuals.csv")).read().splitlines()
    assert abs((len(res) - 1) - len(g["hist"])) <= max(2, iterations_bar * len(g["hist"]))
    assert os.path.exists(os.path.join(out_dir, "solution.vtk"))


@pytest.mark.gpu
@pytest.mark.parametrize("name,fixture", [("lid_driven_cavity", "results_cavity2d_20"),
                                          ("poiseuille_flow", "results_channel2d_64x8"),
                                          ("lid_driven_cavity_40x40", "results_cavity2d_40"),
                                          ("lid_driven_cavity_80x80", "results_cavity2d_80"),
                                          ("lid_driven_cavity_3d", "results_cavity3d_16"),
                                          ("lid_driven_cavity_3d_re1000",
                                           "results_cavity3d_32_re1000"),
                                          ("duct_3d", "results_duct3d_48x8x8")])
def test_gpu_run_lands_on_the_reference_results(ctx, tmp_path, name, fixture):
    c = cases.read_case(os.path.join(CASES, name))
    row = cases.run_case(ctx, c, str(tmp_path))
    assert row["status"] == "Converged" and row["fields_written"]
    # the 3D examples' p' solves stop at 1e-4 too, yet land within 1e-6
    p_tol = c.settings.pressure_solver.relative_tolerance if c.case.dim == 2 else 1e-8
    _compare(row["directory"], fixture, p_rel_tol=p_tol)


@pytest.mark.gpu
def test_gpu_batch_of_case_directories(ctx, tmp_path):
    small = _copy(tmp_path, "lid_driven_cavity")
    os.rename(small, str(tmp_path / "cavity_16"))
    _edit(str(tmp_path / "cavity_16"), "mesh.json", lambda j: j.update(nx=16, ny=16))
    cs = [cases.read_case(os.path.join(CASES, "lid_driven_cavity")),
          cases.read_case(str(tmp_path / "cavity_16"))]
    rows = cases.run_batch(ctx, cs, str(tmp_path / "out"))
    assert all(r["status"] == "Converged" and r["fields_written"] for r in rows)
    _compare(rows[0]["directory"], "results_cavity2d_20")
