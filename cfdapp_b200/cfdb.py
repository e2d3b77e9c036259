"""ctypes binding of libcfdb.so (include/cfdb.h).

The names mirror the reference's linear-solver interface
(include/cfd/algebra/LinearSolver.hpp): ``LinearSolverSettings``,
``SolverResult``, ``SolverStatus``.  The library is loaded from the package's
``lib/`` directory; when it is missing, or no sm_100 device is present, every
entry point raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libcfdb.so")

CFDB_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "no usable sm_100 device",
          -4: "out of memory", -5: "device-side wait timed out", -6: "unsupported"}

SOLVER_STATUS = ["Converged", "MaxIterations", "Breakdown", "NonFiniteInput",
                 "NonFiniteResidual", "InvalidSystem"]
SIMPLE_STATUS = ["Converged", "MaxIterations", "MomentumFailure", "PressureCorrectionFailure",
                 "NonFiniteState", "InvalidConfiguration"]

KRYLOV = {"cg": 0, "bicgstab": 1}
PRECISION = {"fp64": 0, "fp32_refined": 1}
PRECOND = {"none": 0, "jacobi": 1}


class CfdbError(RuntimeError):
    pass


class _Grid(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int64 * 3), ("len", C.c_double * 3)]


class _LinSettings(C.Structure):
    _fields_ = [("krylov", C.c_int), ("preconditioner", C.c_int), ("precision", C.c_int),
                ("abs_tol", C.c_double), ("rel_tol", C.c_double), ("max_iterations", C.c_int64),
                ("inner_rel_tol", C.c_double), ("max_refinements", C.c_int64)]


class _LinResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("true_residual", C.c_double), ("refinements", C.c_int64),
                ("restarts", C.c_int64), ("device_ms", C.c_double),
                ("kernel_launches", C.c_int64), ("krylov_ms", C.c_double),
                ("krylov_bytes", C.c_double), ("krylov_launches", C.c_int64)]


_lib = None


def library_path() -> str:
    return LIB_PATH


def load() -> C.CDLL:
    """Loads libcfdb.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CfdbError(f"{LIB_PATH} is missing: build it with `python -m cfdapp_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i64, dbl = C.c_void_p, C.c_int64, C.c_double
    L.cfdb_cuda_available.restype = C.c_int
    L.cfdb_create.argtypes = [C.c_int, vp, C.POINTER(vp)]
    L.cfdb_destroy.argtypes = [vp]
    L.cfdb_destroy.restype = None
    L.cfdb_last_error.argtypes = [vp]
    L.cfdb_last_error.restype = C.c_char_p
    L.cfdb_stream.argtypes = [vp]
    L.cfdb_stream.restype = vp
    L.cfdb_kernel_launches.argtypes = [vp]
    L.cfdb_kernel_launches.restype = i64
    L.cfdb_synth_rhs.argtypes = [i64, i64, i64, C.c_uint64, C.POINTER(dbl)]
    L.cfdb_poperator_create_uniform.argtypes = [vp, C.POINTER(_Grid), dbl, C.c_uint, C.c_int, i64,
                                                C.POINTER(vp)]
    L.cfdb_poperator_create_faces.argtypes = [vp, C.POINTER(_Grid), C.POINTER(dbl), C.c_int, i64,
                                              C.POINTER(vp)]
    L.cfdb_poperator_destroy.argtypes = [vp]
    L.cfdb_poperator_destroy.restype = None
    L.cfdb_poperator_cells.argtypes = [vp]
    L.cfdb_poperator_cells.restype = i64
    L.cfdb_poperator_apply.argtypes = [vp, vp, vp, vp]
    for name in ("cfdb_poperator_solve_device", "cfdb_poperator_solve_host"):
        getattr(L, name).argtypes = [vp, vp, C.POINTER(_LinSettings), vp, vp, C.POINTER(dbl), i64,
                                     C.POINTER(_LinResult)]
    L.cfdb_device_alloc.argtypes = [vp, C.c_size_t, C.POINTER(vp)]
    L.cfdb_device_free.argtypes = [vp, vp]
    L.cfdb_copy_to_device.argtypes = [vp, vp, vp, C.c_size_t]
    L.cfdb_copy_to_host.argtypes = [vp, vp, vp, C.c_size_t]
    L.cfdb_synchronize.argtypes = [vp]
    L.cfdb_memset_device.argtypes = [vp, vp, C.c_int, C.c_size_t]
    _lib = L
    return L


def cuda_available() -> bool:
    """cfd::gpu::cudaAvailable() (include/cfd/gpu/GPUBackend.hpp:15)."""
    return bool(load().cfdb_cuda_available())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """A cfdb context on one device (and one stream)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        L = load()
        h = C.c_void_p()
        st = L.cfdb_create(device, C.c_void_p(stream) if stream else None, C.byref(h))
        if st != CFDB_OK:
            raise CfdbError(f"cfdb_create failed: {ERRORS.get(st, st)}")
        self._h = h
        self.lib = L

    @property
    def handle(self):
        return self._h

    def check(self, st: int, what: str):
        if st != CFDB_OK:
            msg = self.lib.cfdb_last_error(self._h).decode(errors="replace")
            raise CfdbError(f"{what}: {ERRORS.get(st, st)}: {msg}")

    def stream(self) -> int:
        return self.lib.cfdb_stream(self._h) or 0

    def launches(self) -> int:
        return int(self.lib.cfdb_kernel_launches(self._h))

    def alloc(self, nbytes: int) -> int:
        p = C.c_void_p()
        self.check(self.lib.cfdb_device_alloc(self._h, nbytes, C.byref(p)), "cfdb_device_alloc")
        return p.value

    def free(self, ptr: int):
        self.check(self.lib.cfdb_device_free(self._h, C.c_void_p(ptr)), "cfdb_device_free")

    def to_device(self, arr: np.ndarray) -> int:
        arr = np.ascontiguousarray(arr)
        p = self.alloc(arr.nbytes)
        self.check(self.lib.cfdb_copy_to_device(self._h, C.c_void_p(p), arr.ctypes.data_as(C.c_void_p),
                                                arr.nbytes), "cfdb_copy_to_device")
        return p

    def upload(self, dst: int, arr: np.ndarray):
        arr = np.ascontiguousarray(arr)
        self.check(self.lib.cfdb_copy_to_device(self._h, C.c_void_p(dst), arr.ctypes.data_as(C.c_void_p),
                                                arr.nbytes), "cfdb_copy_to_device")

    def download(self, src: int, shape, dtype=np.float64) -> np.ndarray:
        out = np.empty(shape, dtype=dtype)
        self.check(self.lib.cfdb_copy_to_host(self._h, out.ctypes.data_as(C.c_void_p), C.c_void_p(src),
                                              out.nbytes), "cfdb_copy_to_host")
        return out

    def memset(self, dst: int, value: int, nbytes: int):
        self.check(self.lib.cfdb_memset_device(self._h, C.c_void_p(dst), value, nbytes),
                   "cfdb_memset_device")

    def synchronize(self):
        self.check(self.lib.cfdb_synchronize(self._h), "cfdb_synchronize")

    def close(self):
        if getattr(self, "_h", None):
            self.lib.cfdb_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class LinearSolverSettings:
    """LinearSolverSettings (LinearSolver.hpp:136-166) plus precision knobs."""
    absolute_tolerance: float = 1e-12
    relative_tolerance: float = 1e-10
    max_iterations: int = 1000
    type: str = "cg"
    preconditioner: str = "jacobi"
    precision: str = "fp64"
    inner_relative_tolerance: float = 0.0
    max_refinements: int = 0

    def c(self) -> _LinSettings:
        return _LinSettings(KRYLOV[self.type], PRECOND[self.preconditioner],
                            PRECISION[self.precision], self.absolute_tolerance,
                            self.relative_tolerance, self.max_iterations,
                            self.inner_relative_tolerance, self.max_refinements)


@dataclass
class SolverResult:
    """SolverResult (LinearSolver.hpp:110-134)."""
    status: str
    iterations: int
    initial_residual: float
    final_residual: float
    true_residual: float
    refinements: int
    restarts: int
    device_ms: float
    kernel_launches: int
    krylov_ms: float
    krylov_bytes: float
    krylov_launches: int
    residual_history: np.ndarray
    solution: np.ndarray | None = None

    def converged(self) -> bool:
        return self.status == "Converged"


def grid(dim: int, n, length=(1.0, 1.0, 1.0)) -> _Grid:
    g = _Grid()
    g.dim = dim
    n = list(n) + [1, 1, 1]
    for a in range(3):
        g.n[a] = int(n[a]) if a < dim else 1
        g.len[a] = float(length[a]) if a < len(length) else 1.0
    return g


def synth_rhs(dim: int, n: int, seed: int = 20261203) -> np.ndarray:
    """The seeded synthetic p' RHS (see cfdb_synth_rhs)."""
    b = np.empty(n ** dim, dtype=np.float64)
    st = load().cfdb_synth_rhs(n, n, n if dim == 3 else 0, seed, _dp(b))
    if st != CFDB_OK:
        raise CfdbError("cfdb_synth_rhs failed")
    return b


class POperator:
    """The matrix-free p' operator on the device (cfdb_poperator_*)."""

    def __init__(self, ctx: Context, dim: int, n, length=(1.0, 1.0, 1.0), *, rho: float = 1.0,
                 face_coeff: np.ndarray | None = None, dirichlet_patch_mask: int = 0,
                 pinned: bool = True, reference_cell: int = 0):
        self.ctx = ctx
        self.dim = dim
        self.n = tuple(int(v) for v in n)
        g = grid(dim, n, length)
        h = C.c_void_p()
        if face_coeff is None:
            st = ctx.lib.cfdb_poperator_create_uniform(ctx.handle, C.byref(g), rho,
                                                       dirichlet_patch_mask, int(pinned),
                                                       reference_cell, C.byref(h))
        else:
            fc = np.ascontiguousarray(face_coeff, dtype=np.float64)
            st = ctx.lib.cfdb_poperator_create_faces(ctx.handle, C.byref(g), _dp(fc), int(pinned),
                                                     reference_cell, C.byref(h))
        ctx.check(st, "cfdb_poperator_create")
        self._h = h
        self.cells = int(ctx.lib.cfdb_poperator_cells(h))

    def apply_device(self, x_dev: int, y_dev: int):
        self.ctx.check(self.ctx.lib.cfdb_poperator_apply(self.ctx.handle, self._h, C.c_void_p(x_dev),
                                                         C.c_void_p(y_dev)), "cfdb_poperator_apply")

    def apply(self, x: np.ndarray) -> np.ndarray:
        xd = self.ctx.to_device(np.asarray(x, dtype=np.float64))
        yd = self.ctx.alloc(8 * self.cells)
        try:
            self.apply_device(xd, yd)
            return self.ctx.download(yd, (self.cells,))
        finally:
            self.ctx.free(xd)
            self.ctx.free(yd)

    def _result(self, r: _LinResult, hist, cap, sol=None) -> SolverResult:
        m = min(cap, (r.iterations + 1) if self._precision == 0 else (r.refinements + 1))
        return SolverResult(SOLVER_STATUS[r.status], r.iterations, r.initial_residual,
                            r.final_residual, r.true_residual, r.refinements, r.restarts,
                            r.device_ms, r.kernel_launches, r.krylov_ms, r.krylov_bytes,
                            r.krylov_launches, hist[:m].copy(), sol)

    def solve(self, b: np.ndarray, settings: LinearSolverSettings, x0: np.ndarray | None = None,
              history_cap: int | None = None) -> SolverResult:
        """Host buffers in and out (copies inside the call)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.cells) if x0 is None else np.array(x0, dtype=np.float64)
        cap = (settings.max_iterations + 1) if history_cap is None else history_cap
        hist = np.zeros(max(cap, 1))
        res = _LinResult()
        cs = settings.c()
        self._precision = cs.precision
        self.ctx.check(self.ctx.lib.cfdb_poperator_solve_host(self.ctx.handle, self._h, C.byref(cs),
                                                              _dp(b), _dp(x), _dp(hist), cap,
                                                              C.byref(res)), "cfdb_poperator_solve_host")
        return self._result(res, hist, cap, x)

    def solve_device(self, b_dev: int, x_dev: int, settings: LinearSolverSettings,
                     history_cap: int = 0) -> SolverResult:
        """Device-resident b and x (x holds x0 on entry)."""
        hist = np.zeros(max(history_cap, 1))
        res = _LinResult()
        cs = settings.c()
        self._precision = cs.precision
        self.ctx.check(self.ctx.lib.cfdb_poperator_solve_device(
            self.ctx.handle, self._h, C.byref(cs), C.c_void_p(b_dev), C.c_void_p(x_dev),
            _dp(hist) if history_cap > 0 else None, history_cap, C.byref(res)),
            "cfdb_poperator_solve_device")
        return self._result(res, hist, history_cap)

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.cfdb_poperator_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
