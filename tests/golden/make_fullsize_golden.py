"""Generates the full-size p' solve fixtures of tests/golden/ by running the
reference's own CG + Jacobi (oracle/_ref/ref_driver, built from the
reference sources by oracle/Makefile.ref) on the isolated p' systems of the
benchmark, 5-point 2048^2 and 7-point 256^3, from x0 = 0 to a relative
residual of 1e-8, on every core of this host.  Run from the repository root:

    make -f oracle/Makefile.ref REF=<reference checkout> -j8
    python tests/golden/make_fullsize_golden.py [2d2048] [3d256]

The solutions (32 MB and 134 MB) are too large to commit, so each fixture
keeps what a size-independent comparison needs: the reference's status,
iteration count, residual history and wall time; the FP64 norm and sum of
x; and x at 16384 seeded cells (the indices are stored).  A full solve
takes about an hour per grid on 8 cores.
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
GRIDS = {"2d2048": (2, 2048), "3d256": (3, 256)}
SAMPLES = 16384


def run(args, threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([DRIVER] + args, capture_output=True, text=True, env=env, check=True)
    return json.loads(r.stdout)


def main(names):
    threads = os.cpu_count() or 1
    # the O(n) CSR writer of the driver must equal the reference's own
    # assembly (triplet sort) bit for bit; checked on grids it finishes fast
    for dim, n in ((2, 256), (3, 32)):
        if not run(["poisson", f"dim={dim}", f"n={n}", "check_direct=1"], 1)["direct_matches_reference"]:
            raise SystemExit(f"direct CSR differs from the reference assembly at {dim}D {n}")
    for name in names:
        dim, n = GRIDS[name]
        with tempfile.TemporaryDirectory() as d:
            meta = run(["poisson", f"dim={dim}", f"n={n}", "direct=1", "rtol=1e-8", "atol=0",
                        "maxit=200000", f"out={d}"], threads)
            x = np.fromfile(os.path.join(d, "x.bin"))
            hist = np.fromfile(os.path.join(d, "hist.bin"))
        rng = np.random.default_rng(20261204 + dim)
        idx = np.sort(rng.choice(x.size, size=SAMPLES, replace=False)).astype(np.int64)
        np.savez_compressed(os.path.join(HERE, f"fullsize_{name}.npz"),
                            idx=idx, x_at=x[idx], x_norm=np.linalg.norm(x), x_sum=x.sum(),
                            hist=hist, meta=json.dumps({**meta, "dim": dim, "n": n}))
        print(name, meta["status"], meta["iterations"], f"{meta['seconds']:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(GRIDS))
