"""Host-side recognition of the reference's CSR LinearSystem (cfdb_csr_analyze,
no device needed) and the oracle's BiCGSTAB / CG on the reference's own
stored systems.

Fixtures (tests/golden/make_linear_systems.py, from the reference build):
the two 5-point 32x32 thermal systems the reference keeps for its BiCGSTAB
breakdown regression (tests/data/linear_systems/p12_mesh004_*.txt, checked by
tests/unit/algebra/test_bicgstab_breakdown.cpp:137-153) and two p' systems
of its own assemblePressureCorrection, each with the reference solver's
outcome.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_system(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files if k != "meta"}, json.loads(str(z["meta"]))


def csr_to_bands(offsets, columns, values, shape):
    """Diagonal and six neighbour bands of a structured CSR matrix (test helper
    for the oracle's stencil routines; shape = cells per axis)."""
    n = len(offsets) - 1
    nx = shape[0]
    ny = shape[1] if len(shape) > 1 else 1
    strides = [1, nx, nx * ny]
    diag = np.zeros(n)
    off = [np.zeros(n) for _ in range(6)]
    for r in range(n):
        for q in range(int(offsets[r]), int(offsets[r + 1])):
            d = int(columns[q]) - r
            if d == 0:
                diag[r] = values[q]
                continue
            a = strides.index(abs(d))
            off[2 * a + (d > 0)][r] = values[q]
    return diag, off


def csr_from_bands(diag, off, shape):
    """CSR (ascending columns, exact zeros dropped) of a banded matrix."""
    n = len(diag)
    nx = shape[0]
    ny = shape[1] if len(shape) > 1 else 1
    st = [1, nx, nx * ny]
    ro, ci, va = [0], [], []
    for r in range(n):
        ents = [(r, diag[r])]
        for q in range(6):
            v = off[q][r]
            if v != 0.0:
                ents.append((r + (st[q // 2] if q % 2 else -st[q // 2]), v))
        for c, v in sorted(ents):
            if v != 0.0 or c == r:
                ci.append(c)
                va.append(v)
        ro.append(len(ci))
    return np.array(ro, np.uint64), np.array(ci, np.uint64), np.array(va)


def test_stored_thermal_systems_are_recognised_as_5_point_32x32():
    from cfdapp_b200 import cfdb
    for name in ("csr_mesh004_smooth", "csr_mesh004_rough"):
        s, _ = load_system(name)
        info = cfdb.csr_analyze(s["offsets"], s["columns"], s["values"])
        assert info is not None
        assert info["dim"] == 2 and info["n"] == (32, 32)
        # thermal convection rows are not symmetric: stencil path
        assert not info["faces_eligible"] and info["path"] == "stencil"


@pytest.mark.parametrize("name,dim,shape", [("csr_pprime2d_24", 2, (24, 24)),
                                            ("csr_pprime3d_8", 3, (8, 8, 8))])
def test_reference_pprime_matrix_is_the_face_operator(name, dim, shape):
    """The reference's assembled p' CSR is exactly the matrix-free operator:
    pinned identity row 0, symmetric couplings, the diagonal equal bit for bit
    to the face-order sum."""
    from cfdapp_b200 import cfdb
    s, _ = load_system(name)
    info = cfdb.csr_analyze(s["offsets"], s["columns"], s["values"])
    assert info["dim"] == dim and info["n"] == shape
    assert info["faces_eligible"] and info["path"] == "faces"
    assert info["pinned"] and info["reference_cell"] == 0


def test_perturbed_diagonal_leaves_the_face_path():
    """One ulp on one diagonal entry makes the matrix differ from the face
    operator, so it must take the stencil path (which keeps the stored
    diagonal)."""
    from cfdapp_b200 import cfdb
    s, _ = load_system("csr_pprime2d_24")
    v = s["values"].copy()
    r = 100
    q = next(q for q in range(int(s["offsets"][r]), int(s["offsets"][r + 1]))
             if int(s["columns"][q]) == r)
    v[q] = np.nextafter(v[q], np.inf)
    info = cfdb.csr_analyze(s["offsets"], s["columns"], v)
    assert info["dim"] == 2 and not info["faces_eligible"] and info["path"] == "stencil"


def test_unstructured_matrices_are_refused():
    from cfdapp_b200 import cfdb
    # dense 4x4
    ro = np.array([0, 4, 8, 12, 16], np.uint64)
    ci = np.tile(np.arange(4, dtype=np.uint64), 4)
    assert cfdb.csr_analyze(ro, ci, np.ones(16)) is None
    # a 2D grid with one coupling to a non-neighbour (wraps around a row end)
    s, _ = load_system("csr_pprime2d_24")
    ro, ci, va = s["offsets"], s["columns"].copy(), s["values"]
    r = 23  # last cell of the first row: its x+1 column would be the next row's first cell
    lo, hi = int(ro[r]), int(ro[r + 1])
    assert not any(int(c) == r + 1 for c in ci[lo:hi])
    ci2 = np.insert(ci, hi, r + 1)
    va2 = np.insert(va, hi, -1.0)
    ro2 = ro.copy()
    ro2[r + 1:] += 1
    assert cfdb.csr_analyze(ro2, ci2, va2) is None
    # four distinct strides
    n = 64
    ro = np.arange(0, 2 * n + 1, 2, dtype=np.uint64)
    ci = np.array([[i, (i + [1, 3, 5, 7][i % 4]) % n] for i in range(n)], np.uint64).reshape(-1)
    assert cfdb.csr_analyze(ro, ci, np.ones(2 * n)) is None


def test_one_row_band_is_recognised():
    from cfdapp_b200 import cfdb
    n = 60
    diag = np.full(n, 2.0)
    off = [np.full(n, -1.0), np.full(n, -0.5)] + [np.zeros(n) for _ in range(4)]
    off[0][0] = 0.0
    off[1][-1] = 0.0
    ro, ci, va = csr_from_bands(diag, off, (n,))
    info = cfdb.csr_analyze(ro, ci, va)
    assert info["dim"] == 2 and info["n"] == (n, 1) and info["path"] == "stencil"


@pytest.mark.parametrize("name", ["csr_mesh004_smooth", "csr_mesh004_rough"])
def test_oracle_bicgstab_on_the_stored_systems_matches_the_reference(name):
    """The oracle's BiCGSTAB restatement (oracle/cfdb_oracle.c) on the
    reference's stored breakdown-regression systems: the reference's own
    outcome (Converged, no restart, final and true residual <= 1e-12)."""
    s, meta = load_system(name)
    assert meta["status"] == "Converged" and meta["restarts"] == 0
    case = O.Case(2, (32, 32))
    diag, off = csr_to_bands(s["offsets"], s["columns"], s["values"], (32, 32))
    st = meta["settings"]
    r = O.stencil_solve(case, diag, off, s["rhs"], x0=s["x0"], solver="bicgstab", jacobi=False,
                        abs_tol=st["atol"], rel_tol=st["rtol"], max_iterations=st["maxit"])
    assert r.status == "Converged" and r.restarts == 0
    assert r.iterations == meta["iterations"]
    np.testing.assert_allclose(r.history, s["hist"], rtol=1e-6)
    assert np.linalg.norm(r.solution - s["x"]) <= 1e-9 * np.linalg.norm(s["x"])
    ax = O.stencil_apply(case, diag, off, r.solution)
    assert np.linalg.norm(s["rhs"] - ax) <= st["atol"]
