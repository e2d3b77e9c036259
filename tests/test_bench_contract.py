"""The benchmark's JSON contract on the CPU: the reference arm's line (the
reference's own CG + Jacobi build, timed on the host cores) and the device
arm's refusal to run without a B200."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          capture_output=True, text=True, timeout=600)


def test_workload_names_the_grids():
    import bench
    assert bench.pprime_workload(bench.GRIDS).startswith(
        "isolated p' solve: 5-point 2048^2 + 7-point 256^3, ")
    assert "5-point 64^2 + 7-point 16^3" in bench.pprime_workload(((2, 64), (3, 16)))


def test_reference_arm_prints_one_measured_line():
    from oracle import oracle as O
    if not O.ref_driver_available():
        pytest.skip("the reference build (oracle/_ref) is not present")
    p = run_bench("--impl", "reference", "--grids", "2:64", "--steps", "2", "--warmup", "1")
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "ms" and d["higher_is_better"] is False
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] == d["value"]
    assert "5-point 64^2" in d["config"]["workload"] and d["config"]["grids"] == ["2D 64"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "budgets of 1 and 6" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "ms", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    g = d["grids"]["2D 64"]
    assert g["iterations"] > 0 and g["per_iteration_s"] > 0 and g["setup_s"] >= 0


def test_device_arm_refuses_without_a_b200():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    p = run_bench("--grids", "2:64", "--steps", "1", "--warmup", "1", "--no-cpu-baseline",
                  "--no-config1")
    assert p.returncode != 0
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert "no CPU path" in p.stdout + p.stderr
