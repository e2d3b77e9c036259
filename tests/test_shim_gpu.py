"""The C++ drop-in (cfdapp_b200/shim) under the reference's own, unmodified
code: oracle/_ref/ref_driver_cfdb is the reference driver linked with the
reference's objects minus its GPU seam and SIMPLE.cpp, plus the shim and
libcfdb (oracle/Makefile.ref `shim`).

* Linear-solver plugin: the reference's SIMPLE loop (ReferenceCpuSIMPLE) with
  "backend": GPU on its linear solvers reaches cfd::gpu::makeGpuCG /
  makeGpuBiCGSTAB through the unmodified LinearSolverFactory
  (src/algebra/LinearSolverFactory.cpp:14-33); every solve runs on the
  device (gpuExecutionStats().gpuLinearSolves counts them, no fallback).
* GPU outer loop: with both backends GPU, SIMPLE::solve runs the whole loop
  on the device (SIMPLEResult::residentSimpleLoop), including the learned
  p' preconditioner selected by CFDB_GPU_CG_PRECONDITIONER=learned_mg.

Each run is checked against the reference's own CPU run of the same case
(tests/golden/*.npz): same status, outer iterations within 2 %, and fields
within the bar of each test (relative L2).
"""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver_cfdb")


def _golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z, json.loads(str(z["meta"]))


def _run(args, env_extra=None):
    if not os.path.exists(DRIVER):
        pytest.fail(f"{DRIVER} is missing: build it with __graft_entry__.build()")
    env = dict(os.environ, OMP_NUM_THREADS="1", **(env_extra or {}))
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([DRIVER, "simple"] + args.split() + [f"out={d}"], capture_output=True,
                           text=True, env=env, timeout=3000)
        assert r.returncode == 0, r.stderr[-2000:]
        meta = json.loads(r.stdout.strip().splitlines()[-1])
        dim = 3 if "dim=3" in args else 2
        names = ("u", "v", "w", "p", "flux") if dim == 3 else ("u", "v", "p", "flux")
        fields = {f: np.fromfile(os.path.join(d, f + ".bin")) for f in names}
    return meta, fields


def _compare(meta, fields, z, gmeta, bar):
    assert meta["status"] == gmeta["status"]
    assert abs(meta["iterations"] - gmeta["iterations"]) <= max(2, 0.02 * gmeta["iterations"])
    errs = {}
    for f in fields:
        if f == "flux":
            continue
        ref = z[f]
        errs[f] = float(np.linalg.norm(fields[f] - ref) / max(np.linalg.norm(ref), 1e-300))
    assert max(errs.values()) <= bar, f"relative L2 differences {errs} above {bar}"
    return errs


def test_plugin_pressure_solves_under_the_reference_simple_loop():
    """The reference's SIMPLE loop at 33^2 (Jacobi-CG p' to 1e-8, tolerances
    1e-6) with only the pressure solver on the GPU backend."""
    z, g = _golden("cavity2d_33_jacobicg")
    meta, fields = _run(g["args"] + " pbackend=gpu")
    assert not meta["gpu_simple_loop"]
    assert meta["gpu_backend_fallbacks"] == 0
    assert meta["gpu_linear_solves"] == meta["iterations"]  # every p' solve on the device
    _compare(meta, fields, z, g, 1e-8)


def test_plugin_momentum_and_pressure_solves_under_the_reference_loop():
    """Both linear solvers on the GPU backend, the reference's loop kept
    (CFDB_GPU_SIMPLE=0): the momentum BiCGSTAB rows (with the wall
    three-point band) and the p' rows go through the CSR entry."""
    z, g = _golden("cavity2d_16_jacobicg")
    meta, fields = _run(g["args"] + " mbackend=gpu pbackend=gpu", {"CFDB_GPU_SIMPLE": "0"})
    assert not meta["gpu_simple_loop"]
    assert meta["gpu_backend_fallbacks"] == 0
    assert meta["gpu_linear_solves"] == 3 * meta["iterations"]
    _compare(meta, fields, z, g, 1e-8)


@pytest.mark.parametrize("name", ["cavity2d_129_config1", "cavity2d_16_lud",
                                  "channel2d_32x8_central_rc", "cavity3d_8_quick_rc",
                                  "cavity2d_24_graded_lud_rc", "channel2d_32x12_graded"])
def test_gpu_outer_loop_through_the_reference_simple_api(name):
    """Both backends GPU: SIMPLE::solve runs the GPU loop (configuration 1 at
    129^2 included) and lands on the reference's fields."""
    z, g = _golden(name)
    meta, fields = _run(g["args"] + " mbackend=gpu pbackend=gpu")
    assert meta["gpu_simple_loop"], meta["gpu_fallback_reason"]
    assert meta["gpu_linear_solves"] == 0  # no CSR round trip: the loop is resident
    _compare(meta, fields, z, g, 1e-6)


def test_gpu_outer_loop_with_the_learned_preconditioner():
    z, g = _golden("cavity2d_129_config1")
    meta, fields = _run(g["args"] + " mbackend=gpu pbackend=gpu",
                        {"CFDB_GPU_CG_PRECONDITIONER": "learned_mg"})
    assert meta["gpu_simple_loop"]
    _compare(meta, fields, z, g, 1e-6)
