"""ctypes front end of the CPU oracle (oracle/cfdb_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker; the product never imports
it.  The oracle restates the reference's arithmetic (see cfdb_oracle.h); its
pin against the reference is tests/test_oracle_pin.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcfdb_oracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")

VBC = {"wall": 0, "moving_wall": 1, "inlet": 2, "outlet": 3}
PBC = {"fixed_gradient": 0, "fixed_value": 1}
SCHEME = {"upwind": 0, "central": 1, "lud": 2, "linear_upwind": 2, "quick": 3}
FLUX = {"linear": 0, "rhiechow": 1, "rhie_chow": 1}
SOLVER = {"cg": 0, "bicgstab": 1}
LINEAR_STATUS = ["Converged", "MaxIterations", "Breakdown", "NonFiniteInput",
                 "NonFiniteResidual", "InvalidSystem"]
SIMPLE_STATUS = ["Converged", "MaxIterations", "MomentumFailure",
                 "PressureCorrectionFailure", "NonFiniteState", "InvalidConfiguration"]


def build(force: bool = False) -> str:
    """Compile the oracle shared library (gcc, no GPU needed)."""
    src = os.path.join(HERE, "cfdb_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "cfdb_oracle.h")),
            os.path.getmtime(os.path.join(HERE, "synth_rhs.h"))):
        subprocess.check_call(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", src, "-o",
                               LIB_PATH, "-lm"])
    return LIB_PATH


class _Grid(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int64 * 3), ("len", C.c_double * 3)]


class _Bcs(C.Structure):
    _fields_ = [("vtype", C.c_int * 6), ("vvalue", (C.c_double * 3) * 6),
                ("ptype", C.c_int * 6), ("pvalue", C.c_double * 6)]


class _LinSettings(C.Structure):
    _fields_ = [("type", C.c_int), ("jacobi", C.c_int), ("abs_tol", C.c_double),
                ("rel_tol", C.c_double), ("max_iterations", C.c_int64)]


class _LinResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("restarts", C.c_int64)]


class _SimpleSettings(C.Structure):
    _fields_ = [("max_outer", C.c_int64), ("alpha_u", C.c_double), ("alpha_p", C.c_double),
                ("tol_u", C.c_double), ("tol_p", C.c_double), ("tol_c", C.c_double),
                ("rho", C.c_double), ("mu", C.c_double), ("scheme", C.c_int),
                ("face_flux", C.c_int), ("reference_cell", C.c_int64),
                ("momentum", _LinSettings), ("pressure", _LinSettings)]


class _SimpleResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64), ("final_u", C.c_double),
                ("final_v", C.c_double), ("final_w", C.c_double), ("final_p", C.c_double),
                ("final_continuity", C.c_double), ("global_imbalance", C.c_double),
                ("momentum_linear_iterations", C.c_int64),
                ("pressure_linear_iterations", C.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        L.og_faces.restype = C.c_int64
        L.og_cells.restype = C.c_int64
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _grid(dim, n, length=(1.0, 1.0, 1.0)):
    g = _Grid()
    g.dim = dim
    nn = list(n) + [1] * (3 - len(n))
    for a in range(3):
        g.n[a] = int(nn[a]) if a < dim else 1
        g.len[a] = float(length[a]) if a < len(length) else 1.0
    return g


@dataclass
class Case:
    """A uniform Cartesian case: grid, BCs and fluid."""
    dim: int
    n: tuple
    length: tuple = (1.0, 1.0, 1.0)
    vbc: list = field(default_factory=list)      # per patch (type, (vx, vy, vz))
    pbc: list = field(default_factory=list)      # per patch (type, value)

    def cells(self) -> int:
        return int(np.prod(self.n[: self.dim]))

    def faces(self) -> int:
        return int(lib().og_faces(C.byref(_grid(self.dim, self.n, self.length))))

    def c_grid(self):
        return _grid(self.dim, self.n, self.length)

    def c_bcs(self):
        b = _Bcs()
        for p in range(6):
            t, val = self.vbc[p] if p < len(self.vbc) else ("wall", (0.0, 0.0, 0.0))
            b.vtype[p] = VBC[t]
            for c in range(3):
                b.vvalue[p][c] = float(val[c]) if c < len(val) else 0.0
            pt, pv = self.pbc[p] if p < len(self.pbc) else ("fixed_gradient", 0.0)
            b.ptype[p] = PBC[pt]
            b.pvalue[p] = float(pv)
        return b


def cavity(dim: int, n: int, lid: float = 1.0) -> Case:
    """Lid-driven cavity on the unit square/cube: Wall everywhere, the top
    (ymax) patch a MovingWall {lid, 0[, 0]}; pressure FixedGradient(0)."""
    patches = 2 * dim
    vbc = [("wall", (0.0, 0.0, 0.0)) for _ in range(patches)]
    vbc[3] = ("moving_wall", (lid, 0.0, 0.0))
    pbc = [("fixed_gradient", 0.0) for _ in range(patches)]
    return Case(dim, tuple([n] * dim), (1.0, 1.0, 1.0), vbc, pbc)


def channel(nx: int, ny: int, lx: float, ly: float, inlet: float = 1.0) -> Case:
    """2D channel: Inlet {inlet, 0} left, Outlet right (pressure FixedValue 0),
    Walls top and bottom."""
    vbc = [("inlet", (inlet, 0.0, 0.0)), ("outlet", (0.0, 0.0, 0.0)),
           ("wall", (0.0, 0.0, 0.0)), ("wall", (0.0, 0.0, 0.0))]
    pbc = [("fixed_gradient", 0.0), ("fixed_value", 0.0), ("fixed_gradient", 0.0),
           ("fixed_gradient", 0.0)]
    return Case(2, (nx, ny), (lx, ly, 1.0), vbc, pbc)


def synth_rhs(dim: int, n: int, seed: int = 20261203) -> np.ndarray:
    cells = n ** dim
    b = np.empty(cells, dtype=np.float64)
    rc = lib().og_synth_rhs(C.c_int64(n), C.c_int64(n), C.c_int64(n if dim == 3 else 0),
                            C.c_uint64(seed), _dp(b))
    assert rc == 0
    return b


def assemble_pprime(case: Case, rho: float, flux: np.ndarray, du, dv, dw=None,
                    reference_cell: int = 0):
    """p' face coefficients, stencil matrix (diag, off[6]) and RHS."""
    n = case.cells()
    nf = case.faces()
    fc = np.zeros(nf)
    diag = np.zeros(n)
    off = [np.zeros(n) for _ in range(6)]
    rhs = np.zeros(n)
    offp = (C.POINTER(C.c_double) * 6)(*[_dp(o) for o in off])
    dw_arr = np.ascontiguousarray(dw if dw is not None else np.zeros(n), dtype=np.float64)
    rc = lib().og_assemble_pprime(C.byref(case.c_grid()), C.byref(case.c_bcs()),
                                  C.c_double(rho), _dp(np.ascontiguousarray(flux)),
                                  _dp(np.ascontiguousarray(du)), _dp(np.ascontiguousarray(dv)),
                                  _dp(dw_arr), C.c_int64(reference_cell), _dp(fc), _dp(diag),
                                  offp, _dp(rhs))
    assert rc == 0
    return fc, diag, off, rhs


def isolated_pprime(dim: int, n: int, seed: int = 20261203):
    """The isolated p' system: unit response coefficients, rho = 1, all-Neumann
    pressure, cell 0 pinned, synthetic RHS."""
    case = Case(dim, tuple([n] * dim), (1.0, 1.0, 1.0),
                [("wall", (0, 0, 0))] * (2 * dim), [("fixed_gradient", 0.0)] * (2 * dim))
    cells = case.cells()
    ones = np.ones(cells)
    fc, diag, off, _ = assemble_pprime(case, 1.0, np.zeros(case.faces()), ones, ones, ones)
    return case, fc, diag, off, synth_rhs(dim, n, seed)


def stencil_apply(case: Case, diag, off, x) -> np.ndarray:
    y = np.empty_like(x)
    offp = (C.POINTER(C.c_double) * 6)(*[_dp(np.ascontiguousarray(o)) for o in off])
    lib().og_stencil_apply(C.byref(case.c_grid()), _dp(diag), offp, _dp(x), _dp(y))
    return y


@dataclass
class LinearResult:
    status: str
    iterations: int
    initial_residual: float
    final_residual: float
    restarts: int
    solution: np.ndarray
    history: np.ndarray


def stencil_solve(case: Case, diag, off, b, x0=None, solver="cg", jacobi=True, abs_tol=0.0,
                  rel_tol=1e-8, max_iterations=100000, history=True) -> LinearResult:
    s = _LinSettings(SOLVER[solver], 1 if jacobi else 0, abs_tol, rel_tol, max_iterations)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    cap = max_iterations + 1 if history else 0
    hist = np.zeros(max(cap, 1))
    res = _LinResult()
    offp = (C.POINTER(C.c_double) * 6)(*[_dp(np.ascontiguousarray(o)) for o in off])
    rc = lib().og_stencil_solve(C.byref(case.c_grid()), C.byref(s), _dp(diag), offp,
                                _dp(np.ascontiguousarray(b)), _dp(x), _dp(hist),
                                C.c_int64(cap), C.byref(res))
    assert rc == 0
    count = min(res.iterations + 1, cap) if history else 0
    return LinearResult(LINEAR_STATUS[res.status], res.iterations, res.initial_residual,
                        res.final_residual, res.restarts, x, hist[:count].copy())


def scalar_gradient(case: Case, phi):
    n = case.cells()
    g = [np.zeros(n) for _ in range(3)]
    rc = lib().og_scalar_gradient(C.byref(case.c_grid()), C.byref(case.c_bcs()),
                                  _dp(np.ascontiguousarray(phi)), _dp(g[0]), _dp(g[1]), _dp(g[2]))
    assert rc == 0
    return g[: case.dim]


def momentum_system(case: Case, settings, comp: int, u, v, w, p):
    """(diag, off[6], rhs) of the relaxed momentum system of `comp`."""
    n = case.cells()
    diag = np.zeros(n)
    off = [np.zeros(n) for _ in range(6)]
    rhs = np.zeros(n)
    offp = (C.POINTER(C.c_double) * 6)(*[_dp(o) for o in off])
    arr = [np.ascontiguousarray(a if a is not None else np.zeros(n), dtype=np.float64)
           for a in (u, v, w, p)]
    rc = lib().og_momentum_system(C.byref(case.c_grid()), C.byref(case.c_bcs()),
                                  C.byref(settings.c(case.dim)), comp, *[_dp(a) for a in arr],
                                  _dp(diag), offp, _dp(rhs))
    assert rc == 0
    return diag, off, rhs


@dataclass
class SimpleSettings:
    max_outer: int = 1000
    alpha_u: float = 0.7
    alpha_p: float = 0.3
    tol_u: float = 1e-6
    tol_p: float = 1e-6
    tol_c: float = 1e-6
    rho: float = 1.0
    mu: float = 0.01
    scheme: str = "upwind"
    face_flux: str = "auto"
    reference_cell: int = 0
    momentum: tuple = ("bicgstab", False, 1e-10, 1e-8, 500)
    pressure: tuple = ("cg", True, 0.0, 1e-8, 5000)

    def c(self, dim):
        ff = self.face_flux
        if ff == "auto":
            ff = "linear" if dim == 2 else "rhiechow"
        m = _LinSettings(SOLVER[self.momentum[0]], int(self.momentum[1]), *self.momentum[2:])
        p = _LinSettings(SOLVER[self.pressure[0]], int(self.pressure[1]), *self.pressure[2:])
        return _SimpleSettings(self.max_outer, self.alpha_u, self.alpha_p, self.tol_u,
                               self.tol_p, self.tol_c, self.rho, self.mu, SCHEME[self.scheme],
                               FLUX[ff], self.reference_cell, m, p)


@dataclass
class SimpleResult:
    status: str
    iterations: int
    final: dict
    momentum_linear_iterations: int
    pressure_linear_iterations: int
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    p: np.ndarray
    flux: np.ndarray
    history: np.ndarray


def simple(case: Case, settings: SimpleSettings, u0=None, v0=None, w0=None, p0=None):
    n = case.cells()
    u = np.zeros(n) if u0 is None else np.array(u0, dtype=np.float64)
    v = np.zeros(n) if v0 is None else np.array(v0, dtype=np.float64)
    w = np.zeros(n) if w0 is None else np.array(w0, dtype=np.float64)
    p = np.zeros(n) if p0 is None else np.array(p0, dtype=np.float64)
    flux = np.zeros(case.faces())
    hist = np.zeros(5 * max(settings.max_outer, 1))
    res = _SimpleResult()
    rc = lib().og_simple(C.byref(case.c_grid()), C.byref(case.c_bcs()),
                         C.byref(settings.c(case.dim)), _dp(u), _dp(v), _dp(w), _dp(p),
                         _dp(flux), _dp(hist), C.byref(res))
    assert rc == 0
    final = dict(u=res.final_u, v=res.final_v, w=res.final_w, p=res.final_p,
                 continuity=res.final_continuity, global_imbalance=res.global_imbalance)
    return SimpleResult(SIMPLE_STATUS[res.status], res.iterations, final,
                        res.momentum_linear_iterations, res.pressure_linear_iterations,
                        u, v, w if case.dim == 3 else np.zeros(0), p, flux,
                        hist[: 5 * res.iterations].reshape(-1, 5))


def ref_driver_available() -> bool:
    return os.path.exists(REF_DRIVER)
