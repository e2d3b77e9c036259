"""Generates the golden fixtures of tests/golden/ by running the reference's
own CPU code (oracle/_ref/ref_driver, built from the reference sources by
oracle/Makefile.ref).  Run from the repository root:

    make -f oracle/Makefile.ref REF=<reference checkout> -j8
    python tests/golden/make_golden.py [fixture names]

Each fixture is a compressed .npz of the reference's outputs plus its JSON
summary; the oracle is checked against them in tests/test_oracle_pin.py.
"""
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")

POISSON = {
    "poisson2d_64": "dim=2 n=64",
    "poisson3d_16": "dim=3 n=16",
}
SIMPLE = {
    # the reference's committed 20x20 cavity case (BiCGSTAB p' solve)
    "cavity2d_20_bicgstab": ("dim=2 nx=20 ny=20 psolver=bicgstab ppre=none pabs=1e-10 prel=1e-8 "
                             "pmax=2000 outer=6000", ["u", "v", "p", "flux"]),
    # configuration 1 itself: the 129x129 Re-100 cavity, Jacobi-CG p', to convergence
    "cavity2d_129_config1": ("dim=2 nx=129 ny=129 outer=20000", ["u", "v", "p", "flux"]),
    # config-1 settings on a 33x33 cavity, to convergence (the C++ drop-in's
    # linear-solver plugin runs it with the reference's own SIMPLE loop)
    "cavity2d_33_jacobicg": ("dim=2 nx=33 ny=33 outer=20000", ["u", "v", "p", "flux"]),
    # config-1 settings (Jacobi-CG p') on a small grid, to convergence
    "cavity2d_16_jacobicg": ("dim=2 nx=16 ny=16 outer=6000", ["u", "v", "p", "flux"]),
    "cavity2d_16_lud": ("dim=2 nx=16 ny=16 scheme=lud outer=200", ["u", "v", "p", "flux"]),
    "channel2d_32x8_central_rc": ("dim=2 nx=32 ny=8 lx=8 ly=1 flow=channel mu=0.1 scheme=central "
                                  "flux=rhiechow outer=150", ["u", "v", "p", "flux"]),
    # configuration 5's discretization (linear upwind + Rhie-Chow, Re 1000,
    # Jacobi-CG p' to 1e-8) on a 32^3 cavity, to convergence
    "cavity3d_32_lud_rc_re1000": ("dim=3 nx=32 ny=32 nz=32 mu=0.001 scheme=lud flux=rhiechow "
                                  "outer=5000", ["u", "v", "w", "p", "flux"]),
    # the same at 48^3
    "cavity3d_48_lud_rc_re1000": ("dim=3 nx=48 ny=48 nz=48 mu=0.001 scheme=lud flux=rhiechow "
                                  "outer=5000", ["u", "v", "w", "p", "flux"]),
    # rectilinear (graded) meshes, createGraded2D with geometric ratios: the
    # node coordinates are stored with the fields
    "cavity2d_24_graded": ("dim=2 nx=24 ny=24 gradex=1.12 gradey=1.12 outer=20000",
                           ["u", "v", "p", "flux"]),
    "cavity2d_24_graded_lud_rc": ("dim=2 nx=24 ny=20 gradex=1.1 gradey=1.15 cluster=start "
                                  "scheme=lud flux=rhiechow outer=20000", ["u", "v", "p", "flux"]),
    "channel2d_32x12_graded": ("dim=2 nx=32 ny=12 lx=6 ly=1 flow=channel mu=0.05 gradey=1.2 "
                               "outer=300", ["u", "v", "p", "flux"]),
    "cavity3d_8_quick_rc": ("dim=3 nx=8 ny=8 nz=8 mu=0.001 scheme=quick flux=rhiechow outer=40 "
                            "psolver=bicgstab ppre=none prel=1e-4 pabs=1e-13 mrel=1e-6 mabs=1e-13 "
                            "tolu=1e-7 tolp=1e-7 tolc=1e-7", ["u", "v", "w", "p", "flux"]),
}


def run(cmd, args, out):
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run([DRIVER, cmd] + args.split() + [f"out={out}"], capture_output=True,
                       text=True, env=env, check=True)
    return json.loads(r.stdout)


def main(only=()):
    for name, args in POISSON.items():
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as d:
            meta = run("poisson", args, d)
            np.savez_compressed(os.path.join(HERE, name + ".npz"),
                                x=np.fromfile(os.path.join(d, "x.bin")),
                                hist=np.fromfile(os.path.join(d, "hist.bin")),
                                rhs=np.fromfile(os.path.join(d, "rhs.bin")),
                                meta=json.dumps({**meta, "args": args}))
            print(name, meta["status"], meta["iterations"])
    for name, (args, fields) in SIMPLE.items():
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as d:
            meta = run("simple", args, d)
            arrays = {f: np.fromfile(os.path.join(d, f + ".bin")) for f in fields}
            arrays["hist"] = np.fromfile(os.path.join(d, "hist.bin"))
            for nd in ("x_nodes", "y_nodes"):  # graded meshes
                if os.path.exists(os.path.join(d, nd + ".bin")):
                    arrays[nd] = np.fromfile(os.path.join(d, nd + ".bin"))
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays,
                                meta=json.dumps({**meta, "args": args}))
            print(name, meta["status"], meta["iterations"])


if __name__ == "__main__":
    import sys
    main(tuple(sys.argv[1:]))  # fixture names to (re)generate; all when none
