"""The result-file writer (cfdb_write_results) against the reference's own
committed example outputs, byte for byte: the field values and residual
history of cases/lid_driven_cavity (20x20), cases/lid_driven_cavity_3d
(16^3) and cases/poiseuille_flow (64x8), parsed back from the reference's files (tests/golden/
make_results_fixtures.py), written again must hash to the reference's
fields.csv, residuals.csv and solution.vtk.  No device needed."""
import hashlib
import json
import os

import numpy as np
import pytest

from cfdapp_b200 import cfdb

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _fixture(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return g, json.loads(str(g["meta"]))


def _case(meta):
    dim = meta["dim"]
    return cfdb.SimpleCase(dim, tuple(meta["n"]), tuple(meta["length"]) + (1.0,) * (3 - dim))


@pytest.mark.parametrize("name", ["results_cavity2d_20", "results_cavity3d_16",
                                  "results_channel2d_64x8", "results_cavity2d_40",
                                  "results_cavity2d_80", "results_cavity3d_32_re1000",
                                  "results_duct3d_48x8x8"])
def test_writer_reproduces_the_reference_files(tmp_path, name):
    g, meta = _fixture(name)
    d = str(tmp_path / "results")
    wrote = cfdb.write_results(_case(meta), g["u"], g["v"], g["w"], g["p"], g["hist"],
                               meta["global_imbalance"], d)
    assert wrote
    for fn, want in meta["files"].items():
        data = open(os.path.join(d, fn), "rb").read()
        assert len(data) == want["bytes"], fn
        assert hashlib.sha256(data).hexdigest() == want["sha256"], fn


def test_non_finite_fields_write_residuals_only(tmp_path):
    g, meta = _fixture("results_cavity2d_20")
    u = g["u"].copy()
    u[7] = np.nan
    d = str(tmp_path / "nan")
    assert not cfdb.write_results(_case(meta), u, g["v"], None, g["p"], g["hist"][:3], 0.0, d)
    assert sorted(os.listdir(d)) == ["residuals.csv"]
    assert len(open(os.path.join(d, "residuals.csv")).read().splitlines()) == 4


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _check_against_reference(d, ref_dir, g, meta):
    """Files written from a GPU run of the reference's case: same layout as the
    reference's (headers, ids, coordinates, mesh), values within 1e-6."""
    ours = open(os.path.join(d, "fields.csv")).read().splitlines()
    ref = open(os.path.join(ref_dir, "fields.csv")).read().splitlines()
    assert len(ours) == len(ref) and ours[0] == ref[0]
    assert [r.split(",")[:3] for r in ours] == [r.split(",")[:3] for r in ref]
    f = np.array([[float(x) for x in r.split(",")] for r in ours[1:]])
    assert _rel(f[:, 3], g["u"]) <= 1e-6 and _rel(f[:, 4], g["v"]) <= 1e-6
    assert _rel(f[:, 6], g["p"]) <= 1e-6
    ov = open(os.path.join(d, "solution.vtk")).read().splitlines()
    rv = open(os.path.join(ref_dir, "solution.vtk")).read().splitlines()
    cut = rv.index(next(x for x in rv if x.startswith("CELL_DATA")))
    assert len(ov) == len(rv) and ov[:cut + 1] == rv[:cut + 1]
    res = open(os.path.join(d, "residuals.csv")).read().splitlines()
    rows = len(g["hist"])
    assert abs((len(res) - 1) - rows) <= max(2, 0.02 * rows)
    h = np.array([[float(x) for x in r.split(",")] for r in res[1:101]])
    ref_h = g["hist"][:100]
    for ours_col, ref_col in ((1, 0), (2, 1), (3, 3)):
        assert _rel(h[:, ours_col], ref_h[:, ref_col]) <= 1e-6


@pytest.mark.gpu
def test_gpu_session_and_batch_write_the_reference_files(ctx, tmp_path):
    """The reference's committed 20x20 cavity, solved on the GPU by the
    single-case session and inside a batch, exported from device fields."""
    from test_simple_gpu import gpu_case_from_args
    g, meta = _fixture("results_cavity2d_20")
    ref_dir = str(tmp_path / "ref")
    cfdb.write_results(_case(meta), g["u"], g["v"], g["w"], g["p"], g["hist"],
                       meta["global_imbalance"], ref_dir)
    case, s = gpu_case_from_args("dim=2 nx=20 ny=20 psolver=bicgstab ppre=none pabs=1e-10 "
                                 "prel=1e-8 pmax=2000 outer=6000")
    sim = cfdb.Simple(ctx, case, s)
    sim.set_state(None, None, None, None)
    r = sim.iterate(s.max_iterations)
    assert r.status == "Converged"
    d = str(tmp_path / "session")
    assert sim.write_results(r.history, r.final["global_imbalance"], d)
    sim.close()
    _check_against_reference(d, ref_dir, g, meta)
    b = cfdb.Batch(ctx, [cfdb.SimpleCase.cavity(2, 12), case], s, history_cap=s.max_iterations)
    b.set_state(0)
    b.set_state(1)
    b.iterate(s.max_iterations)
    d = str(tmp_path / "batch")
    assert b.write_results(1, d)
    b.close()
    _check_against_reference(d, ref_dir, g, meta)
