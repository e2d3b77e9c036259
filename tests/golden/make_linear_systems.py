"""Generates the CSR linear-system fixtures of tests/golden/ from the
reference: its two stored BiCGSTAB regression systems
(tests/data/linear_systems/p12_mesh004_thermal_{smooth_a005,rough_f03}_n32.txt,
5-point 32x32 thermal rows of a non-uniform mesh) and two p' systems of its
own assembly (assemblePressureCorrection through oracle/_ref/ref_driver
poisson ... dump_matrix=1), each solved by the reference's own solver
(oracle/_ref/ref_driver csr / poisson, built by oracle/Makefile.ref).  Run
from the repository root:

    make -f oracle/Makefile.ref REF=<reference checkout> -j8
    python tests/golden/make_linear_systems.py <reference checkout>

Each fixture holds the CSR arrays (uint64 offsets and columns, float64
values), rhs, x0, the settings used and the reference's status, iteration
and restart counts, residuals, residual history and solution.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
STORED = {"csr_mesh004_smooth": "p12_mesh004_thermal_smooth_a005_n32.txt",
          "csr_mesh004_rough": "p12_mesh004_thermal_rough_f03_n32.txt"}
PPRIME = {"csr_pprime2d_24": "dim=2 n=24", "csr_pprime3d_8": "dim=3 n=8"}


def read_stored(path):
    """The reference's text format: comment lines, 'rows nnz', row offsets,
    column indices, values, rhs, initial guess (reals as %.17g)."""
    toks = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            toks.extend(line.split())
    rows, nnz = int(toks[0]), int(toks[1])
    p = 2
    ro = np.array([int(t) for t in toks[p:p + rows + 1]], dtype=np.uint64)
    p += rows + 1
    ci = np.array([int(t) for t in toks[p:p + nnz]], dtype=np.uint64)
    p += nnz
    va = np.array([float(t) for t in toks[p:p + nnz]])
    p += nnz
    rhs = np.array([float(t) for t in toks[p:p + rows]])
    p += rows
    x0 = np.array([float(t) for t in toks[p:p + rows]])
    assert p + rows == len(toks), "trailing tokens"
    return ro, ci, va, rhs, x0


def run_csr(ro, ci, va, rhs, x0, args):
    with tempfile.TemporaryDirectory() as d:
        ro.astype(np.uint64).tofile(os.path.join(d, "offsets.bin"))
        ci.astype(np.uint64).tofile(os.path.join(d, "columns.bin"))
        va.tofile(os.path.join(d, "values.bin"))
        rhs.tofile(os.path.join(d, "rhs.bin"))
        x0.tofile(os.path.join(d, "x0.bin"))
        r = subprocess.run([DRIVER, "csr", f"in={d}", f"out={d}"] + args, capture_output=True,
                           text=True, check=True, env=dict(os.environ, OMP_NUM_THREADS="1"))
        meta = json.loads(r.stdout)
        return meta, np.fromfile(os.path.join(d, "x.bin")), np.fromfile(os.path.join(d, "hist.bin"))


def main(ref):
    settings = {"solver": "bicgstab", "pre": "none", "atol": 1e-12, "rtol": 1e-10, "maxit": 1000}
    for name, fn in STORED.items():
        ro, ci, va, rhs, x0 = read_stored(os.path.join(ref, "tests", "data", "linear_systems", fn))
        meta, x, hist = run_csr(ro, ci, va, rhs, x0, [f"{k}={v}" for k, v in settings.items()])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), offsets=ro, columns=ci, values=va,
                            rhs=rhs, x0=x0, x=x, hist=hist,
                            meta=json.dumps({**meta, "settings": settings, "source": fn}))
        print(name, meta)
    cg = {"solver": "cg", "pre": "jacobi", "atol": 0.0, "rtol": 1e-10, "maxit": 5000}
    for name, args in PPRIME.items():
        with tempfile.TemporaryDirectory() as d:
            subprocess.run([DRIVER, "poisson"] + args.split() + ["maxit=1", "dump_matrix=1",
                                                                 f"out={d}"],
                           capture_output=True, text=True, check=True)
            ro = np.fromfile(os.path.join(d, "csr_offsets.bin")).astype(np.uint64)
            ci = np.fromfile(os.path.join(d, "csr_columns.bin")).astype(np.uint64)
            va = np.fromfile(os.path.join(d, "csr_values.bin"))
            rhs = np.fromfile(os.path.join(d, "rhs.bin"))
        x0 = np.zeros_like(rhs)
        meta, x, hist = run_csr(ro, ci, va, rhs, x0, [f"{k}={v}" for k, v in cg.items()])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), offsets=ro, columns=ci, values=va,
                            rhs=rhs, x0=x0, x=x, hist=hist,
                            meta=json.dumps({**meta, "settings": cg, "source": args}))
        print(name, meta)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_linear_systems.py <reference checkout>")
    main(sys.argv[1])
