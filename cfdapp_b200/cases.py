"""Case directories in the reference's format, run on the GPU.

    python -m cfdapp_b200.cases CASE_DIR [CASE_DIR ...] [--out DIR] [--batch]

Reads a case directory as the reference's CaseReader/CaseBuilder do
(case.json naming geometry.json, mesh.json, physics.json, boundaries.json and
solver.json; src/io/SolverConfigParser.cpp for solver.json), for the subset
this library runs: a uniform ``structured_cartesian`` mesh on a rectangle or
box, ``incompressible_laminar`` physics, velocity BCs wall / moving_wall /
inlet / outlet, pressure BCs fixed_gradient / fixed_value, a SIMPLE solver
with BiCGSTAB or CG linear solvers (no preconditioner, as the reference's
LinearSolverSettings default).  Anything else raises CaseError naming the
key, rather than running a different model.

GPU opt-in: solver.json may carry one additive block the reference's parser
does not know, ``"gpu": {"pressure_preconditioner": "none" | "jacobi" |
"learned_mg", "pressure_precision": "fp64" | "fp32_refined"}``; without it
the case runs with the reference's own settings.

Results land in ``<out>/<case name>/``: fields.csv, residuals.csv and
solution.vtk in the reference's formats (cfdb_write_results).  With
``--batch`` every case of one dimension and identical solver settings runs as
one cfdb batch.
"""
from __future__ import annotations

import argparse
import json
import os
from dataclasses import dataclass

from . import cfdb

PATCHES_2D = ("left", "right", "bottom", "top")
PATCHES_3D = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")


class CaseError(ValueError):
    pass


@dataclass
class Case:
    name: str
    directory: str
    case: cfdb.SimpleCase
    settings: cfdb.SIMPLESettings


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except OSError as e:
        raise CaseError(f"{path}: cannot read ({e.strerror})") from None
    except json.JSONDecodeError as e:
        raise CaseError(f"{path}: not valid JSON ({e})") from None


def _need(d, key, where):
    if key not in d:
        raise CaseError(f"{where}: missing required key '{key}'")
    return d[key]


def _linear(block, where, precond="none", precision="fp64"):
    kind = _need(block, "type", where)
    if kind not in ("BiCGSTAB", "CG"):
        raise CaseError(f"{where}.type: '{kind}' is not on the GPU path (BiCGSTAB, CG)")
    if block.get("backend", "CPU") not in ("CPU", "GPU"):
        raise CaseError(f"{where}.backend: be one of CPU, GPU")
    return cfdb.LinearSolverSettings(
        absolute_tolerance=float(_need(block, "absolute_tolerance", where)),
        relative_tolerance=float(_need(block, "relative_tolerance", where)),
        max_iterations=int(_need(block, "max_iterations", where)),
        type=kind.lower(), preconditioner=precond, precision=precision)


def read_case(directory: str) -> Case:
    """One case directory as (cfdb.SimpleCase, cfdb.SIMPLESettings)."""
    top = _load(os.path.join(directory, "case.json"))
    part = {k: _load(os.path.join(directory, _need(top, k, "case.json")))
            for k in ("geometry", "mesh", "physics", "boundaries", "solver")}
    mesh, geom, phys = part["mesh"], part["geometry"], part["physics"]
    if mesh.get("type") != "structured_cartesian":
        raise CaseError(f"mesh.json: type '{mesh.get('type')}' is not on the GPU path")
    for ax, g in (mesh.get("grading") or {}).items():
        if (g or {}).get("type", "uniform") != "uniform":
            raise CaseError(f"mesh.json: grading of {ax} is not uniform (not on the GPU path)")
    dim = 3 if "nz" in mesh else 2
    n = (int(mesh["nx"]), int(mesh["ny"])) + ((int(mesh["nz"]),) if dim == 3 else ())
    want = "box" if dim == 3 else "rectangle"
    if geom.get("type") != want:
        raise CaseError(f"geometry.json: type '{geom.get('type')}' (a {dim}D mesh needs '{want}')")
    length = (float(geom["length"]), float(geom["height"]),
              float(geom["depth"]) if dim == 3 else 1.0)
    if phys.get("model") != "incompressible_laminar":
        raise CaseError(f"physics.json: model '{phys.get('model')}' is not on the GPU path")
    rho = float(_need(phys, "density", "physics.json"))
    mu = float(_need(phys, "dynamic_viscosity", "physics.json"))
    patches = _need(part["boundaries"], "patches", "boundaries.json")
    names = PATCHES_3D if dim == 3 else PATCHES_2D
    vbc, pbc = [], []
    for q in names:
        p = _need(patches, q, "boundaries.json.patches")
        v = _need(p, "velocity", f"patches.{q}")
        vt = v.get("type")
        if vt not in ("wall", "moving_wall", "inlet", "outlet"):
            raise CaseError(f"patches.{q}.velocity: type '{vt}' is not on the GPU path")
        val = [float(x) for x in v.get("value", [0.0, 0.0, 0.0])] + [0.0, 0.0, 0.0]
        vbc.append((vt, tuple(val[:3])))
        pr = _need(p, "pressure", f"patches.{q}")
        pt = pr.get("type")
        if pt not in ("fixed_gradient", "fixed_value"):
            raise CaseError(f"patches.{q}.pressure: type '{pt}' is not on the GPU path")
        pbc.append((pt, float(pr.get("value", 0.0))))
    solver = part["solver"]
    if solver.get("type", "SIMPLE") != "SIMPLE":
        raise CaseError(f"solver.json: type '{solver.get('type')}' is not on the GPU path")
    for key in ("gradient_scheme", "non_orthogonal_corrections"):
        if key in solver and solver[key] not in ("green_gauss", 0, False, None):
            raise CaseError(f"solver.json: {key} = {solver[key]!r} is not on the GPU path")
    gpu = solver.get("gpu") or {}
    settings = cfdb.SIMPLESettings(
        max_iterations=int(_need(solver, "max_iterations", "solver.json")),
        velocity_relaxation=float(solver.get("velocity_relaxation", 0.7)),
        pressure_relaxation=float(solver.get("pressure_relaxation", 0.3)),
        velocity_tolerance=float(_need(solver, "velocity_tolerance", "solver.json")),
        pressure_tolerance=float(_need(solver, "pressure_tolerance", "solver.json")),
        continuity_tolerance=float(_need(solver, "continuity_tolerance", "solver.json")),
        convection_scheme=solver.get("convection_scheme", "upwind"),
        face_flux=solver.get("face_flux", "automatic"),
        momentum_solver=_linear(_need(solver, "momentum_linear_solver", "solver.json"),
                                "momentum_linear_solver"),
        pressure_solver=_linear(_need(solver, "pressure_linear_solver", "solver.json"),
                                "pressure_linear_solver",
                                precond=gpu.get("pressure_preconditioner", "none"),
                                precision=gpu.get("pressure_precision", "fp64")))
    if settings.convection_scheme not in cfdb.SCHEME or settings.face_flux not in cfdb.FACE_FLUX:
        raise CaseError("solver.json: unknown convection_scheme or face_flux")
    case = cfdb.SimpleCase(dim, n, length, tuple(vbc), tuple(pbc), rho, mu)
    return Case(top.get("name", os.path.basename(os.path.normpath(directory))), directory, case,
                settings)


def _out_dir(out, c: Case):
    return os.path.join(out, os.path.basename(os.path.normpath(c.directory)))


def run_case(ctx: cfdb.Context, c: Case, out: str) -> dict:
    """SIMPLE on the GPU, results written in the reference's formats."""
    r = cfdb.simple_solve(ctx, c.case, c.settings)
    d = _out_dir(out, c)
    wrote = cfdb.write_results(c.case, r.u, r.v, r.w if c.case.dim == 3 else None, r.p, r.history,
                               r.final["global_imbalance"], d)
    return {"case": c.name, "status": r.status, "iterations": r.iterations, "device_ms": r.device_ms,
            "fields_written": wrote, "directory": d}


def run_batch(ctx: cfdb.Context, cases, out: str) -> list:
    """Cases of one dimension and identical settings as one cfdb batch."""
    s = cases[0].settings
    b = cfdb.Batch(ctx, [c.case for c in cases], s, history_cap=s.max_iterations)
    for k in range(len(cases)):
        b.set_state(k)
    stats = b.iterate(s.max_iterations)
    res = b.results()
    out_rows = []
    for k, c in enumerate(cases):
        d = _out_dir(out, c)
        wrote = b.write_results(k, d)
        out_rows.append({"case": c.name, "status": res[k]["status"],
                         "iterations": res[k]["iterations"], "device_ms": stats["device_ms"],
                         "fields_written": wrote, "directory": d})
    b.close()
    return out_rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("cases", nargs="+")
    ap.add_argument("--out", default="cfdb_results")
    ap.add_argument("--batch", action="store_true")
    a = ap.parse_args(argv)
    cases = [read_case(d) for d in a.cases]
    ctx = cfdb.Context(0)
    if a.batch:
        groups = {}
        for c in cases:
            key = (c.case.dim, repr(c.settings))
            groups.setdefault(key, []).append(c)
        rows = [r for g in groups.values() for r in run_batch(ctx, g, a.out)]
    else:
        rows = [run_case(ctx, c, a.out) for c in cases]
    for r in rows:
        print(json.dumps(r))
    ctx.close()


if __name__ == "__main__":
    main()
