"""Fixtures of the reference's result-file formats, taken from its committed
example runs of uniform Cartesian laminar cases (cases/lid_driven_cavity,
20x20, _40x40, _80x80; cases/lid_driven_cavity_3d, 16^3;
cases/lid_driven_cavity_3d_re1000, 32^3; cases/duct_3d, 48x8x8;
cases/poiseuille_flow, 64x8): the field values and residual history
parsed back from their fields.csv / residuals.csv (17 significant digits
round-trip exactly), the final global mass imbalance, the grid, and the
SHA-256 and size of each committed fields.csv, residuals.csv and
solution.vtk.  tests/test_results_io.py writes the same values through
cfdb_write_results and compares the files byte for byte by hash.  The case
input files (case.json and the five files it names) are copied to
tests/golden/cases/<case>/ for tests/test_cases.py.

    python tests/golden/make_results_fixtures.py <reference checkout>
"""
import csv
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = {"results_cavity2d_20": "lid_driven_cavity", "results_cavity3d_16": "lid_driven_cavity_3d",
         "results_channel2d_64x8": "poiseuille_flow",
         # the reference's other uniform Cartesian laminar examples: field values only
         "results_cavity2d_40": "lid_driven_cavity_40x40",
         "results_cavity2d_80": "lid_driven_cavity_80x80",
         "results_cavity3d_32_re1000": "lid_driven_cavity_3d_re1000",
         "results_duct3d_48x8x8": "duct_3d"}
CASE_FILES = ("case.json", "geometry.json", "mesh.json", "physics.json", "boundaries.json",
              "solver.json")


def main(ref):
    for name, case in CASES.items():
        base = os.path.join(ref, "cases", case)
        res = os.path.join(base, "results")
        mesh = json.load(open(os.path.join(base, "mesh.json")))
        geom = json.load(open(os.path.join(base, "geometry.json")))
        dim = 3 if "nz" in mesh else 2
        n = [mesh["nx"], mesh["ny"]] + ([mesh["nz"]] if dim == 3 else [])
        length = [geom["length"], geom["height"]] + ([geom["depth"]] if dim == 3 else [])
        rows = list(csv.reader(open(os.path.join(res, "fields.csv"))))
        hdr = rows[0]
        col = {h: i for i, h in enumerate(hdr)}
        f = np.array([[float(x) for x in r] for r in rows[1:]])
        u, v, p = f[:, col["velocity_x"]], f[:, col["velocity_y"]], f[:, col["pressure"]]
        w = f[:, col["velocity_z"]] if dim == 3 else np.zeros(0)
        rr = list(csv.reader(open(os.path.join(res, "residuals.csv"))))
        rcol = {h: i for i, h in enumerate(rr[0])}
        R = np.array([[float(x) for x in r] for r in rr[1:]])
        hist = np.zeros((R.shape[0], 5))
        hist[:, 0] = R[:, rcol["u_residual"]]
        hist[:, 1] = R[:, rcol["v_residual"]]
        if dim == 3:
            hist[:, 2] = R[:, rcol["w_residual"]]
        hist[:, 3] = R[:, rcol["p_residual"]]
        hist[:, 4] = R[:, rcol["continuity_residual"]]
        glob = float(R[-1, rcol["global_mass_imbalance"]]) if len(R) else 0.0
        files = {}
        for fn in ("fields.csv", "residuals.csv", "solution.vtk"):
            data = open(os.path.join(res, fn), "rb").read()
            files[fn] = {"sha256": hashlib.sha256(data).hexdigest(), "bytes": len(data)}
        meta = {"case": case, "dim": dim, "n": n, "length": length, "global_imbalance": glob,
                "files": files}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), u=u, v=v, w=w, p=p, hist=hist,
                            meta=json.dumps(meta))
        dst = os.path.join(HERE, "cases", case)
        os.makedirs(dst, exist_ok=True)
        for fn in CASE_FILES:
            with open(os.path.join(base, fn), "rb") as fi, open(os.path.join(dst, fn), "wb") as fo:
                fo.write(fi.read())
        print(name, meta["n"], R.shape[0], "rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_results_fixtures.py <reference checkout>")
    main(sys.argv[1])
